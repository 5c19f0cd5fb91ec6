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
