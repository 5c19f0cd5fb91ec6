"""The TMA-staged face pass (k_faces_tile) against the oracle, bit for bit.

Every tile shape, pinned with fivo_ctx_set_face_pass, runs rhs_2d! and a few
SSPRK3 steps of the viscous MC-Glauber event and of ideal Gubser flow (no
dissipative planes, no charge) on grids whose extents are not multiples of the
tile (ragged last tiles in both directions) and on a non-square grid; the
global-load kernel and the autotuned choice run the same cases. A grid whose
Ny + 6 is odd cannot use tensor maps: pinning a tile shape there is refused and
the autotuner keeps the global-load kernel.
"""
import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D

from test_gpu_parity import _assert_same_work, _glauber_setup, _gubser_setup, bits_equal, EOSES

pytestmark = pytest.mark.gpu

CFGS = [A.FIVO_FACES_GLOBAL, A.FIVO_FACES_AUTO] + list(range(len(A.FACE_TILE_SHAPES)))


def _glauber_rect(nx, ny):
    g = fivo2d.make_grid2d(nx, ny, xmax=15.0, ymax=15.0 * ny / nx)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True,
                              eta_over_s=0.16, tauShear_coeff=0.2, zeta_over_s=0.05, bulk_model="gaussian",
                              bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1003)
    U, _ = O.set_cells(m.params, 0.6, T, a, ux, uy, m.nv)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(0.6)
    U = o.get_state()
    o.close()
    return g, m, U


@pytest.mark.parametrize("cfg", CFGS)
@pytest.mark.parametrize("case", ["glauber_40", "glauber_rect_34x58", "gubser_ideal_32"])
def test_face_pass_bitwise(gpu_lib, cfg, case):
    if case == "glauber_40":
        g, m, U = _glauber_setup(40)
        tau, integ = 0.6, A.FIVO_SSPRK3
    elif case == "glauber_rect_34x58":
        g, m, U = _glauber_rect(34, 58)
        tau, integ = 0.6, A.FIVO_SSPRK3
    else:
        g, m, U = _gubser_setup(32, EOSES["conformal_g0"], alpha=0.0, with_charge=False)
        tau, integ = 1.0, A.FIVO_SSPRK2
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.set_state(U)
    w.set_face_pass(cfg)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    dw, do = w.rhs(tau), o.rhs(tau)
    assert bits_equal(dw, do)
    assert w.counters().amax == o.counters().amax
    rw = w.run(tau, 1e9, 0.2, 0.05, integ, max_steps=3)
    ro = o.run(tau, 1e9, 0.2, 0.05, integ, max_steps=3)
    assert rw["tau"] == ro["tau"] and rw["nsteps"] == ro["nsteps"] == 3
    _assert_same_work(w, o, f"face pass {cfg}, {case}")
    x, y = w.face_pass()
    if cfg != A.FIVO_FACES_AUTO:
        assert (x, y) == (cfg, cfg)
    else:
        assert -1 <= x < len(A.FACE_TILE_SHAPES) and -1 <= y < len(A.FACE_TILE_SHAPES)
    w.close()
    o.close()


def test_tiles_refused_on_odd_row_pitch(gpu_lib):
    g = fivo2d.make_grid2d(40, 41, xmax=15.0, ymax=15.0)       # Ny + 6 = 47
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS())
    w = GPUWork2D(m, g, lib=gpu_lib)
    with pytest.raises(A.FivoError):
        w.set_face_pass(0)
    T, a, ux, uy = ic.uniform_fields(g, T0=0.3, alpha0=-4.0)
    U, _ = O.set_cells(m.params, 1.0, T, a, ux, uy, m.nv)
    w.set_state(U)
    w.rhs(1.0)
    assert w.face_pass() == (A.FIVO_FACES_GLOBAL, A.FIVO_FACES_GLOBAL)
    w.close()
