"""fivo_rhs_noalloc: the right-hand side for callers that cannot allocate device memory.

Hosts whose device memory belongs to someone else's allocator (a Julia driver
on CUDA.jl's pool), or services that forbid device allocation after start-up,
cannot use the context-based entry points, which cudaMalloc their work arrays. fivo_rhs_noalloc keeps its work
memory in a fixed file-scope device array instead; the caller passes the state
and the output buffer. This test calls it twice in a row through the C ABI and
checks each result against the context-based fivo_rhs on the same state, to the
bit (the tests' tolerance for this stage), the recovery counters it reports
(also on a state whose recoveries fail), plus the size limit's error.

The file name sorts last so a run that stops at the first failure has run every
other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D, set_cells

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    same = a.view(np.int64) == b.view(np.int64)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


def _states():
    """Two different states on one grid: an MC-Glauber event and an ideal
    Gubser-like profile, both on the full viscous layout."""
    g = fivo2d.make_grid2d(48, 40, xmax=15.0, ymax=12.0)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                              enable_diff=True, eta_over_s=0.16, zeta_over_s=0.05, bulk_model="gaussian",
                              bulk_T0=0.18, bulk_width=0.024, kappa_coeff=0.5)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1001)
    U1, _ = set_cells(m, 0.6, T, a, ux, uy)
    Tg, ag, uxg, uyg = ic.gubser_fields(g, 1.0, q=0.5, Tscale=0.4, alpha=-3.0)
    U2, _ = set_cells(m, 1.0, Tg, ag, uxg, uyg)
    return g, m, [(0.6, U1), (1.0, U2)]


def test_rhs_noalloc_matches_context_rhs_twice(gpu_lib):
    import torch
    lib = gpu_lib
    g, m, states = _states()
    stream = torch.cuda.current_stream()
    for tau, U in states:
        # reference result: the context-based entry point (allocates its work arrays)
        w = GPUWork2D(m, g, lib=lib)
        w.set_state(U)
        dU_ref = w.rhs(tau)
        amax_ref = w.counters().amax
        U_ref = w.get_state()
        w.close()
        # the same state as device planes (nv x Ntot), owned by the caller
        planes = torch.tensor(np.ascontiguousarray(U.T), dtype=torch.float64, device="cuda")
        dU = torch.full_like(planes, float("nan"))
        amax = C.c_double(-1.0)
        cnt = A.FivoCounters()
        st = lib.fivo_rhs_noalloc(C.byref(m.params), g.Nx, g.Ny, g.xmax, g.ymax, tau, A.FIVO_BC_OUTFLOW,
                                  C.c_void_p(planes.data_ptr()), C.c_void_p(dU.data_ptr()), C.byref(amax),
                                  C.byref(cnt), C.c_void_p(stream.cuda_stream))
        assert st == A.FIVO_OK, lib.fivo_last_error()
        torch.cuda.synchronize()
        assert _bits_equal(dU.cpu().numpy().T, dU_ref)
        assert amax.value == amax_ref and cnt.amax == amax_ref
        assert _bits_equal(planes.cpu().numpy().T, U_ref)        # ghost frame refilled in place
        assert cnt.nprimfail == 0 and cnt.primfail_index == -1


def test_rhs_noalloc_reports_recovery_failures(gpu_lib):
    """On an evolved state (flow everywhere), with the Newton capped at one iteration
    (primrec_maxit = 1), the recoveries of the matter cells fail and are floored to
    the cold vacuum state; the call still returns FIVO_OK, and its counters say so
    exactly as the context path's do."""
    import torch
    lib = gpu_lib
    g = fivo2d.make_grid2d(40, 36, xmax=15.0, ymax=12.0)
    kw = dict(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True, eta_over_s=0.16,
              zeta_over_s=0.05, bulk_model="gaussian", bulk_T0=0.18, bulk_width=0.024, kappa_coeff=0.5)
    m0 = fivo2d.build_model_2d(**kw)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1002)
    U, _ = set_cells(m0, 0.6, T, a, ux, uy)
    w0 = GPUWork2D(m0, g, lib=lib)
    w0.set_state(U)
    w0.finalize_ic(0.6)
    r = w0.run(0.6, 1.2, 0.2, 0.05, A.FIVO_SSPRK3)
    assert r["ok"]
    U = w0.get_state()
    w0.close()
    m = fivo2d.build_model_2d(**kw, primrec_maxit=1)
    w = GPUWork2D(m, g, lib=lib)
    w.set_state(U)
    dU_ref = w.rhs(1.2)
    c_ref = w.counters()
    w.close()
    assert c_ref.nprimfail > 0
    planes = torch.tensor(np.ascontiguousarray(U.T), dtype=torch.float64, device="cuda")
    dU = torch.empty_like(planes)
    amax = C.c_double(-1.0)
    cnt = A.FivoCounters()
    for _ in range(2):                       # the second call must not see the first one's counts
        st = lib.fivo_rhs_noalloc(C.byref(m.params), g.Nx, g.Ny, g.xmax, g.ymax, 1.2, A.FIVO_BC_OUTFLOW,
                                  C.c_void_p(planes.data_ptr()), C.c_void_p(dU.data_ptr()), C.byref(amax),
                                  C.byref(cnt), None)
        assert st == A.FIVO_OK, lib.fivo_last_error()
        assert cnt.nprimfail == c_ref.nprimfail
        assert cnt.nvacuum == c_ref.nvacuum
        assert cnt.primfail_index == c_ref.primfail_index >= 0
        assert cnt.primfail_reason == c_ref.primfail_reason
        assert _bits_equal(dU.cpu().numpy().T, dU_ref)


def test_rhs_noalloc_rejects_oversize(gpu_lib):
    import torch
    lib = gpu_lib
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS())
    nx = ny = 400                                                  # (406)^2 > FIVO_NOALLOC_MAX_CELLS
    assert (nx + 6) * (ny + 6) > A.FIVO_NOALLOC_MAX_CELLS
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    amax = C.c_double(0.0)
    st = lib.fivo_rhs_noalloc(C.byref(m.params), nx, ny, 15.0, 15.0, 1.0, A.FIVO_BC_OUTFLOW,
                              C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), C.byref(amax), None, None)
    assert st == A.FIVO_ERR_ARG
    assert b"FIVO_NOALLOC_MAX_CELLS" in lib.fivo_last_error()
