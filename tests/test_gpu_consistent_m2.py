"""The consistent charm second moment on the device, against the oracle.

The sector adds five rows (pQxx, pQxy, pQyy, pQeta, PiQ) that pass through every
stage with no flux and no source and are relaxed after each step by backward Euler
with implicit coefficients measured by one perturbed source evaluation per channel
(src2d/dissipation2d.jl:722-888, src2d/hq_consistent_m2_2d.jl:247-404). Every run
here must equal the oracle's to the bit, state, primitives and history (the
current's nux_prev/nuy_prev included).
"""
import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d.solver import GPUWork2D
from fivo2d import ic

from test_gpu_parity import _assert_same_work, _glauber_setup, _pair, bits_equal

pytestmark = pytest.mark.gpu


def _gm5_state(g, m):
    T, a, ux, uy = ic.uniform_fields(g, T0=0.40, alpha0=-4.2)
    U, _ = O.set_cells(m.params, 0.4, T, a, ux, uy, m.nv)
    sx, sy = g.interior()
    X, Y = np.meshgrid(g.xC[sx], g.yC[sy], indexing="ij")
    Um = U.reshape(g.Nxtot, g.Nytot, m.nv)
    Um[sx, sy, m.layout.idx("Dtau")] *= 1 + 0.10 * np.exp(-(X ** 2 + Y ** 2) / 8)
    return U


@pytest.mark.parametrize("terms", [None, {"m2_vorticity": True}, {"m2_projector": False, "m2_bg_Dalpha": False}],
                         ids=["default", "vorticity", "no_projector_Dalpha"])
def test_gm5_solve_matches_oracle(gpu_lib, terms):
    """Gm5's solve (48^2, a 10 % Gaussian bump in the charge, tau 0.4 -> 0.6, both
    closures on) on the device: bitwise the oracle's whole run"""
    g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2, consistent_fm=True,
                              consistent_m2=True, terms=terms)
    w, o = _pair(m, g, _gm5_state(g, m))
    rw = w.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    ro = o.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    _assert_same_work(w, o, "Gm5 solve")
    pq = w.get_state()[:, m.layout.idx("pQxx"):]
    assert np.max(np.abs(pq)) > 0.0
    w.close()
    o.close()


def test_viscous_event_with_both_closures(gpu_lib):
    """An MC-Glauber event with shear, bulk, diffusion and both charm closures at 40^2
    (a transport mass apart from the EOS mass, so both masses are exercised): a
    stepped run bitwise against the oracle, then a relaxation alone on the evolved
    state (the history planes then hold real d_tau differences)"""
    g, m, U = _glauber_setup(40, consistent_fm=True, consistent_m2=True, transport_mass=1.3)
    w, o = _pair(m, g, U)
    for s in (w, o):
        s.finalize_ic(0.6)
    rw = w.run(0.6, 0.9, 0.2, 0.05, A.FIVO_SSPRK3)
    ro = o.run(0.6, 0.9, 0.2, 0.05, A.FIVO_SSPRK3)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    _assert_same_work(w, o, "event with both closures")
    for s in (w, o):
        s.update_primitives(0.9)
        s.relax(0.9, 0.01)
    _assert_same_work(w, o, "relaxation after the run")
    w.close()
    o.close()


def test_passive_sector_leaves_the_medium_alone(gpu_lib):
    """On the device too the second moment feeds back into nothing: the medium's rows
    of a run with it equal a run without it, bit for bit"""
    g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
    out = []
    for cm2 in (False, True):
        m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2,
                                  consistent_fm=True, consistent_m2=cm2)
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.set_state(_gm5_state(g, m))
        assert w.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)["ok"]
        out.append((m.nv, w.get_state()))
        w.close()
    (nv0, U0), (_, U1) = out
    assert bits_equal(U1[:, :nv0], U0)


def test_rhs_rows_of_the_second_moment_are_zero(gpu_lib):
    """rhs_2d! gives the five rows dU = +0 exactly (no flux entries, zero face
    columns, no source), bitwise as the oracle's assembly computes them"""
    g, m, U = _glauber_setup(40, consistent_m2=True)
    rng = np.random.default_rng(3)
    Um = U.reshape(-1, m.nv)
    Um[:, m.layout.idx("pQxx"):] = rng.normal(0.0, 1e-3, (Um.shape[0], 5))
    w, o = _pair(m, g, U)
    dw, do = w.rhs(0.6), o.rhs(0.6)
    assert bits_equal(dw, do)
    assert not np.any(dw[:, m.layout.idx("pQxx"):].view(np.int64))
    w.close()
    o.close()


def test_readout_and_record_of_a_device_run(gpu_lib, tmp_path):
    """fields_2d (main2D.jl:588-600) of a device run carries the second moment's rows by
    their layout names, equals the same readout of the oracle's run, and survives
    save_fields / load_fields bit for bit"""
    from fivo2d.solver import fields_2d
    g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2, consistent_fm=True,
                              consistent_m2=True)
    w, o = _pair(m, g, _gm5_state(g, m))
    w.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    o.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    fw = fields_2d(g, w.get_state(), w, m)
    fo = fields_2d(g, o.get_state(), o, m)
    assert {"pQxx", "pQxy", "pQyy", "pQeta", "PiQ"} <= set(fw)
    for k in fw:
        assert bits_equal(fw[k], fo[k]), k
    d = fivo2d.load_fields(fivo2d.save_fields(tmp_path / "f.npz", fw, model=m, meta={"tau": 0.6}))
    for k in fw:
        assert bits_equal(d["fields"][k], fw[k]), k
    assert d["model_fields"]["consistent_m2"] == "True" and d["meta"]["tau"] == 0.6
    w.close()
    o.close()
