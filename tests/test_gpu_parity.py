"""GPU parity: the CUDA stage against the CPU oracle, bit for bit.

Every float result of the device path must carry the oracle's exact bits (NaN
compared as NaN): both evaluate the same restatement of the reference's Julia
with the same operation order, the same transcendental-function algorithms and
no floating-point contraction. Inputs are seeded and small enough for the oracle
to finish in seconds.
"""
import zlib

import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D, cons_to_prim, eos_Pne, set_cells

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    same = a.view(np.int64) == b.view(np.int64)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


def where_differs(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    bad = ~((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b)))
    idx = np.argwhere(bad)
    return f"{bad.sum()} differing entries, first {idx[:5].tolist()}"


EOSES = {
    "conformal_g0": fivo2d.ConformalHQEOS(g_eff=47.5, g_hq=0.0),
    "conformal_hq": fivo2d.ConformalHQEOS(),
    "lattice_hrg": fivo2d.LatticeHRGEOS(),
}


@pytest.mark.parametrize("name", list(EOSES))
def test_eos_bitwise(gpu_lib, name):
    eos = EOSES[name]
    m = fivo2d.build_model_2d(eos=eos)
    rng = np.random.default_rng(11)
    T = np.exp(rng.uniform(np.log(1e-3), np.log(5.0), 5000))
    T[:4] = [1e-20, 1e-12, 0.1565, 10.0]
    mu = eos.m_hq + T * rng.uniform(-40, 3, T.size)
    P, n, e = eos_Pne(m, T, mu)
    Po, no, eo = O.eos_Pne(m.params, T, mu)
    assert bits_equal(P, Po) and bits_equal(n, no) and bits_equal(e, eo)


def _random_cells(eos, n, diss, umax, seed, tau=1.3):
    rng = np.random.default_rng(seed)
    T = 0.12 + 0.43 * rng.random(n)
    phi = 4.0 * (2 * rng.random(n) - 1)
    ux = umax * (2 * rng.random(n) - 1)
    uy = umax * (2 * rng.random(n) - 1)
    mfull = fivo2d.build_model_2d(eos=eos, enable_shear=True, enable_bulk=True)
    P, nq, _ = O.eos_Pne(mfull.params, T, eos.m_hq + T * phi)
    Pi, pxx, pxy, pyy = (diss * P * (2 * rng.random(n) - 1) for _ in range(4))
    nux, nuy = (diss * nq * (2 * rng.random(n) - 1) for _ in range(2))
    alpha = (eos.m_hq + T * phi) / T
    U, ok = O.set_cells(mfull.params, tau, T, alpha, ux, uy, mfull.nv, Pi, pxx, pxy, pyy, nux, nuy)
    cons = np.column_stack([U[:, 0] / tau] + [U[:, k] for k in range(1, 11)])
    return mfull, cons, T, ux, uy


@pytest.mark.parametrize("name", list(EOSES))
@pytest.mark.parametrize("diss,umax", [(0.0, 1.5), (0.1, 1.5), (0.1, 4.0)])
def test_cons_to_prim_bitwise_and_roundtrip(gpu_lib, name, diss, umax):
    """The recovery gate of test/test_primrec2d.jl:35-118 (1500 states per sweep,
    0 failures, 1e-9) on the GPU, bitwise against the oracle."""
    eos = EOSES[name]
    m, cons, T, ux, uy = _random_cells(eos, 1500, diss, umax, seed=zlib.crc32(f"{name}{diss}{umax}".encode()))
    prim, ok, reason = cons_to_prim(m, 1.3, cons)
    po, oko, ro = O.cons_to_prim(m.params, 1.3, cons)
    assert bits_equal(prim, po), where_differs(prim, po)
    assert np.array_equal(ok, oko) and np.array_equal(reason, ro)
    assert ok.all()
    assert np.max(np.abs(prim[:, 0] - T) / T) < 1e-9
    assert np.max(np.maximum(np.abs(prim[:, 2] - ux), np.abs(prim[:, 3] - uy)) /
                  np.maximum(1.0, np.maximum(np.abs(ux), np.abs(uy)))) < 1e-9
    warm = np.column_stack([np.log(T) * 1.01, np.zeros_like(T), ux * 0.9, uy * 1.1])
    prim_w, ok_w, _ = cons_to_prim(m, 1.3, cons, warm)
    po_w, oko_w, _ = O.cons_to_prim(m.params, 1.3, cons, warm)
    assert bits_equal(prim_w, po_w) and np.array_equal(ok_w, oko_w)


def test_recovery_vacuum_and_zero_flow(gpu_lib):
    """test/test_primrec2d.jl:168-191."""
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS())
    cons = np.zeros((2, 11))
    U, ok = O.set_cells(m.params, 1.0, np.array([0.30]), np.array([1.5 / 0.30]), np.zeros(1), np.zeros(1), m.nv)
    cons[1, :4] = [U[0, 0], U[0, 1], U[0, 2], U[0, 3]]
    prim, ok, reason = cons_to_prim(m, 1.0, cons)
    assert not ok[0] and reason[0] == 1                          # PRR_VACUUM
    assert ok[1] and abs(prim[1, 0] - 0.30) / 0.30 < 1e-10 and np.hypot(prim[1, 2], prim[1, 3]) < 1e-12


def _gubser_setup(N, eos, box=10.0, alpha=-20.0, Tc0=0.6, with_charge=True):
    g = fivo2d.make_grid2d(N, N, xmax=box, ymax=box)
    m = fivo2d.build_model_2d(eos=eos, with_charge=with_charge)
    Tsc = ic.gubser_Tscale_from_center_T(1.0, 1.0, Tc0)
    T, a, ux, uy = ic.gubser_fields(g, 1.0, q=1.0, Tscale=Tsc, alpha=alpha)
    U, ok = O.set_cells(m.params, 1.0, T, a, ux, uy, m.nv)
    return g, m, U


def _glauber_setup(N, box=15.0, tau0=0.6, seed=1001, **kw):
    g = fivo2d.make_grid2d(N, N, xmax=box, ymax=box)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                              enable_diff=True, eta_over_s=0.16, tauShear_coeff=0.2, zeta_over_s=0.05,
                              bulk_model="gaussian", bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5, **kw)
    T, a, ux, uy, _ = ic.glauber_fields(g, tau0, seed)
    U, ok = O.set_cells(m.params, tau0, T, a, ux, uy, m.nv)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(tau0)
    return g, m, o.get_state()


def test_set_cells_bitwise(gpu_lib):
    g = fivo2d.make_grid2d(40, 40, xmax=15.0, ymax=15.0)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1001)
    U, ok = set_cells(m, 0.6, T, a, ux, uy)
    Uo, oko = O.set_cells(m.params, 0.6, T, a, ux, uy, m.nv)
    assert bits_equal(U, Uo) and np.array_equal(ok, oko.astype(bool))


def _pair(m, g, U):
    w = GPUWork2D(m, g)
    w.set_state(U)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    return w, o


def _assert_same_work(w, o, what=""):
    pw, po = w.primitives(), o.primitives()
    for k in ("yT", "phi", "mu", "alpha", "ux", "uy", "P", "n", "e"):
        assert bits_equal(pw[k], po[k]), f"{what} primitive {k}: {where_differs(pw[k], po[k])}"
    assert np.array_equal(pw["ok"], po["ok"]), what
    hw, ho = w.get_history(), o.get_history()
    if w.model.layout.hasM2:
        hw.update(w.get_nu_history())
        ho.update(o.get_nu_history())
    for k in hw:
        assert bits_equal(hw[k], ho[k]), f"{what} history {k}: {where_differs(hw[k], ho[k])}"
    Uw, Uo = w.get_state(), o.get_state()
    assert bits_equal(Uw, Uo), f"{what} state: {where_differs(Uw, Uo)}"


@pytest.mark.parametrize("case", ["gubser_ideal", "gubser_hq", "glauber_viscous"])
def test_rhs_bitwise(gpu_lib, case):
    if case == "gubser_ideal":
        g, m, U = _gubser_setup(32, EOSES["conformal_g0"], alpha=0.0, with_charge=False)
        tau = 1.0
    elif case == "gubser_hq":
        g, m, U = _gubser_setup(32, EOSES["conformal_hq"])
        tau = 1.0
    else:
        g, m, U = _glauber_setup(40)
        tau = 0.6
    w, o = _pair(m, g, U)
    dw, do = w.rhs(tau), o.rhs(tau)
    assert bits_equal(dw, do), where_differs(dw, do)
    assert w.counters().amax == o.counters().amax
    _assert_same_work(w, o, case)
    assert w.compute_dt(tau, 0.2, 0.05) == o.compute_dt(tau, 0.2, 0.05)


@pytest.mark.parametrize("integrator", [A.FIVO_SSPRK2, A.FIVO_SSPRK3])
def test_step_bitwise(gpu_lib, integrator):
    g, m, U = _glauber_setup(40)
    w, o = _pair(m, g, U)
    w.rhs(0.6)
    o.rhs(0.6)
    dt = o.compute_dt(0.6, 0.2, 0.05)
    okw, uw = w.step(integrator, 0.6, dt)
    oko, uo = o.step(integrator, 0.6, dt)
    assert okw == oko and uw == uo
    _assert_same_work(w, o, "step")


def test_relax_and_project_bitwise(gpu_lib):
    g, m, U = _glauber_setup(40)
    w, o = _pair(m, g, U)
    for s in (w, o):
        s.rhs(0.6)
        s.update_primitives(0.62)
        s.relax(0.62, 0.02)
    _assert_same_work(w, o, "relax")
    rw, ro = w.project_shear(), o.project_shear()
    assert rw[0] == ro[0]
    _assert_same_work(w, o, "project")


def test_run_gubser_config_bitwise(gpu_lib):
    """Ideal conformal Gubser (e = 3P with 47.5 d.o.f., no charge), SSPRK2,
    CFLtau = 0.25, T0hat = 5.55 fm^-1: the whole run_sim_2d! on both."""
    g = fivo2d.make_grid2d(48, 48, xmax=10.0, ymax=10.0)
    m = fivo2d.build_model_2d(eos=EOSES["conformal_g0"], with_charge=False)
    T, a, ux, uy = ic.gubser_fields(g, 1.0, q=1.0, Tscale=5.55 * fivo2d.model.HBARC, alpha=0.0)
    U, _ = O.set_cells(m.params, 1.0, T, a, ux, uy, m.nv)
    w, o = _pair(m, g, U)
    rw = w.run(1.0, 1.6, 0.2, 0.25, A.FIVO_SSPRK2)
    ro = o.run(1.0, 1.6, 0.2, 0.25, A.FIVO_SSPRK2)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    assert abs(rw["dQ"] - ro["dQ"]) < 1e-12
    _assert_same_work(w, o, "gubser run")


@pytest.mark.parametrize("integrator", [A.FIVO_SSPRK2, A.FIVO_SSPRK3])
def test_run_viscous_glauber_bitwise(gpu_lib, integrator):
    """Shear + bulk + charm diffusion on a seeded MC-Glauber event (LatticeHRG)."""
    g, m, U = _glauber_setup(40)
    w, o = _pair(m, g, U)
    rw = w.run(0.6, 0.9, 0.2, 0.05, integrator)
    ro = o.run(0.6, 0.9, 0.2, 0.05, integrator)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    _assert_same_work(w, o, "viscous run")


def test_advance_chunks_equal_one_run(gpu_lib):
    """run_sim_2d! resumed step by step (fivo_advance, the on_dump join) gives the
    bits of the oracle's continuous loop, and the kernel timers count launches."""
    g, m, U = _glauber_setup(40)
    w, o = _pair(m, g, U)
    w.rhs(0.6)
    o.rhs(0.6)
    lib = w.lib
    import ctypes as C
    lib.fivo_profile(w.h, 1)
    tau_w = tau_o = 0.6
    for _ in range(6):
        rw = w.advance(tau_w, 5.0, 0.2, 0.05, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 1)
        ro = o.advance(tau_o, 5.0, 0.2, 0.05, A.FIVO_SSPRK3, 0, 1)
        assert rw["ok"] and ro["ok"] and rw["tau"] == ro["tau"] and rw["nsteps"] == 1
        tau_w, tau_o = rw["tau"], ro["tau"]
    kt = A.FivoKernelTimes()
    lib.fivo_profile_read(w.h, C.byref(kt), 1)
    # every stage is one recovery pass (fast + slow) + faces + update + deferred
    # admissibility; every step adds one refresh pass + one relaxation
    L = kt.launches
    assert L[A.FIVO_KCLASS_RELAX] == 6 and L[A.FIVO_KCLASS_UPDATE] >= 6 * 3
    assert L[A.FIVO_KCLASS_PRIM_FAST] == L[A.FIVO_KCLASS_UPDATE] + L[A.FIVO_KCLASS_RELAX]
    assert L[A.FIVO_KCLASS_PRIM_SLOW] == L[A.FIVO_KCLASS_PRIM_FAST]
    assert L[A.FIVO_KCLASS_FACES] == L[A.FIVO_KCLASS_UPDATE] == L[A.FIVO_KCLASS_ADM_SLOW]
    for k in (A.FIVO_KCLASS_PRIM_FAST, A.FIVO_KCLASS_FACES, A.FIVO_KCLASS_UPDATE, A.FIVO_KCLASS_RELAX):
        assert kt.ms[k] > 0
    assert kt.units[A.FIVO_KCLASS_PRIM_FAST] == L[A.FIVO_KCLASS_PRIM_FAST] * g.Ntot
    assert 0 <= kt.units[A.FIVO_KCLASS_PRIM_SLOW] <= kt.units[A.FIVO_KCLASS_PRIM_FAST]
    assert kt.total_launches > sum(L)
    _assert_same_work(w, o, "advance")


def test_failure_injection_maxit(gpu_lib):
    """Force the Newton to one iteration on an evolved state: the recovery-failure
    fallback (cold vacuum cells, NaN warm starts, PRR_RESIDUAL_TOO_LARGE) runs
    identically on both and the failure counter rises."""
    g, m, U = _glauber_setup(40, tau0=0.6)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.run(0.6, 1.2, 0.2, 0.05, A.FIVO_SSPRK3)
    U1 = o.get_state()
    m1 = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                               enable_diff=True, eta_over_s=0.16, zeta_over_s=0.05, bulk_model="gaussian",
                               bulk_T0=0.18, bulk_width=0.024, kappa_coeff=0.5, primrec_maxit=1)
    w, o1 = _pair(m1, g, U1)
    nw = w.update_primitives(1.2)
    no = o1.update_primitives(1.2)
    assert nw == no and nw > 100
    assert w.counters().primfail_reason == o1.counters().primfail_reason == 8
    _assert_same_work(w, o1, "maxit=1")


def test_clone_state_replays_the_same_steps(gpu_lib):
    """fivo_ctx_clone_state: a copy taken mid-run advances to the bits of the
    original (the bench replays its timed steps this way with kernel timing)."""
    g, m, U = _glauber_setup(40)
    w, o = _pair(m, g, U)
    w.rhs(0.6)
    r = w.advance(0.6, 5.0, 0.2, 0.05, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 3)
    twin = GPUWork2D(m, g, lib=w.lib)
    twin.clone_state_from(w)
    ra = w.advance(r["tau"], 5.0, 0.2, 0.05, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 4)
    rb = twin.advance(r["tau"], 5.0, 0.2, 0.05, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 4)
    assert ra == rb
    assert bits_equal(w.get_state(), twin.get_state())
    hw, ht = w.get_history(), twin.get_history()
    for k in hw:
        assert bits_equal(hw[k], ht[k]), k
    other = GPUWork2D(fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS()), g, lib=w.lib)
    with pytest.raises(A.FivoError):
        other.clone_state_from(w)
    other.close()
    twin.close()
