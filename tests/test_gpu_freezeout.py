"""The freeze-out surface and its Cooper-Frye yield on the device (fivo_fo_*,
fivo_cooper_frye) against the oracle: the recorded surface of a short
axisymmetric run must be the oracle's to the bit (the run is, and the recorder's
arithmetic is the same), and the yield must agree to summation order."""
import numpy as np
import pytest

from fivo2d import _abi as A
from fivo2d.freezeout import FreezeOut, cf_params, freeze_surface
from fivo2d.solver import GPUWork2D

import test_freezeout_host as H

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))))


def test_surface_of_a_short_run_matches_oracle(gpu_lib):
    g, m, U = H.small_control()
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.set_state(U)
    w.finalize_ic(0.4)
    fo, chunks = freeze_surface(w, 0.4, H.SHORT["tau_max"], T_fo=H.SHORT["T_fo"])
    s = fo.surface()
    o = H.oracle_freeze_surface(m, g, U, 0.4, H.SHORT["tau_max"], T_fo=H.SHORT["T_fo"])
    assert chunks > 100
    for k in ("nhot", "nfroze", "refroze"):
        assert s[k] == o[k], k
    for k in ("tau_fo", "uxf", "uyf"):
        assert bits_equal(s[k], o[k]), k
    p = dict(H.PRM, T_fo=H.SHORT["T_fo"])
    dev = fo.pion_yield(cf_params(**p))
    ref = H.oracle_pion_yield(o["tau_fo"], o["uxf"], o["uyf"], g.dx, p)
    assert dev[0] > 0
    for a, b in zip(dev, ref):
        assert abs(a - b) <= 1e-10 * max(abs(b), 1e-30), (dev, ref)
    fo.close()
    w.close()


def test_cooper_frye_on_a_given_surface(gpu_lib):
    import fivo2d
    n = 14
    g = fivo2d.make_grid2d(n, n, xmax=n / 2, ymax=n / 2)          # dx = 1
    w = GPUWork2D(H.freeze_model(), g, lib=gpu_lib)
    fo = FreezeOut(w)
    tau, ux, uy = H.synthetic_surface(n)
    fo.set_surface(tau, ux, uy)
    for p in (dict(H.PRM), dict(H.PRM, n_eta=12, n_pt=10, n_phi=8, m=0.494)):
        dev = fo.pion_yield(cf_params(**p))
        ref = H.oracle_pion_yield(tau, ux, uy, 1.0, p)
        for a, b in zip(dev, ref):
            assert abs(a - b) <= 1e-11 * max(abs(b), 1e-30), (dev, ref)
    fo.close()
    w.close()


def test_empty_surface_and_refusals(gpu_lib):
    """no frozen cell: zero yield; a surface refuses a context of another grid"""
    import ctypes as C
    import fivo2d
    g = fivo2d.make_grid2d(12, 12, xmax=6.0, ymax=6.0)
    w = GPUWork2D(H.freeze_model(), g, lib=gpu_lib)
    fo = FreezeOut(w)
    assert fo.pion_yield() == (0.0, 0.0, 0.0)
    s = fo.surface()
    assert s["nfroze"] == 0 and s["nhot"] == 0 and np.isnan(s["tau_fo"]).all()
    g2 = fivo2d.make_grid2d(14, 12, xmax=7.0, ymax=6.0)
    w2 = GPUWork2D(H.freeze_model(), g2, lib=gpu_lib)
    assert gpu_lib.fivo_fo_record(fo.h, w2.h, C.c_double(1.0)) == A.FIVO_ERR_ARG
    bad = cf_params(n_pt=1)
    out = np.zeros(3)
    assert gpu_lib.fivo_cooper_frye(fo.h, C.byref(bad), out.ctypes.data_as(A._D)) == A.FIVO_ERR_ARG
    fo.close()
    w.close()
    w2.close()


@pytest.mark.parametrize("N,published", [(200, 1171.3), (300, 1183.9)])
def test_axisymmetric_control_yield_matches_reference(gpu_lib, N, published):
    """The axisymmetric control of freezeout2d.jl (the calibrated radial profile on
    N^2 cells over [-18, 18] fm, tau 0.4 -> 16 in chunks of 0.02, the T = 0.156
    surface, then Cooper-Frye) against the reference's own post-fix yields: 1171.3
    at N = 200 and 1183.9 at N = 300 (TWOD_PROGRAM.md:1845-1847, the one-sided rim
    differences of freezeout2d.jl:156-163). The runs differ from the reference's in
    the exp/log/Bessel implementations only; the tolerance is 0.5 %."""
    import pathlib

    import fivo2d
    from fivo2d.freezeout import axisym_fields, freeze_model
    from fivo2d.solver import set_cells
    g = fivo2d.make_grid2d(N, N, xmax=18.0, ymax=18.0)
    m = freeze_model()
    prof = pathlib.Path(__file__).resolve().parent / "golden" / "initial_profiles_physical.csv"
    T, a, ux, uy = axisym_fields(g, prof)
    U, _ = set_cells(m, 0.4, T, a, ux, uy, lib=gpu_lib)
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.set_state(U)
    w.finalize_ic(0.4)
    fo, chunks = freeze_surface(w, 0.4, 16.0, dtau=0.02)
    NB, Nb, negf = fo.pion_yield(cf_params())
    assert abs(Nb / published - 1) < 5e-3, (N, NB, Nb)
    fo.close()
    w.close()
