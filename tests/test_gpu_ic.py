"""The MC-Glauber initial condition built on the device (fivo_glauber_ic) against
the host construction of the same event (fivo2d.ic.glauber_fields, numpy/scipy).

The two use different exp/log and Bessel implementations and sum the interior
charm density in a different order, so they agree to rounding, not to the bit:
T to 1e-12 relative, alpha to 1e-9 absolute, the conserved state to 1e-10.
"""
import numpy as np
import pytest

import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D, set_cells

pytestmark = pytest.mark.gpu


def _model():
    return fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                                 enable_diff=True, eta_over_s=0.16, zeta_over_s=0.05, bulk_model="gaussian",
                                 bulk_T0=0.18, bulk_width=0.024, kappa_coeff=0.5)


@pytest.mark.parametrize("n,seed,T_edge", [(48, 1001, ic.EDGE_T), (64, 1005, ic.EDGE_T), (48, 1001, 0.0)],
                         ids=["edge-48", "edge-64", "vacuum-48"])
def test_device_ic_matches_host_construction(gpu_lib, n, seed, T_edge):
    g = fivo2d.make_grid2d(n, n, xmax=15.0, ymax=15.0)
    m = _model()
    w = GPUWork2D(m, g, lib=gpu_lib)
    Td, ad = w.glauber_ic(0.6, seed, T_edge=T_edge, fields=True)
    Th, ah, ux, uy, _ = ic.glauber_fields(g, 0.6, seed, T_edge=T_edge)
    assert np.allclose(Td, Th, rtol=1e-12, atol=0.0)
    assert np.max(np.abs(ad - ah)) < 1e-9
    # the state: set_cell! + finalize_ic! of the host fields
    Uh, _ = set_cells(m, 0.6, Th, ah, ux, uy, lib=gpu_lib)
    wh = GPUWork2D(m, g, lib=gpu_lib)
    wh.set_state(Uh)
    wh.finalize_ic(0.6)
    Ud, Uhf = w.get_state(), wh.get_state()
    scale = np.max(np.abs(Uhf), axis=0)
    assert np.all(np.abs(Ud - Uhf) <= 1e-10 * np.maximum(scale, 1e-300))
    # and it runs
    w.rhs(0.6)
    r = w.advance(0.6, 5.0, 0.2, 0.05, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 3)
    assert r["ok"] and r["nsteps"] == 3
    w.close()
    wh.close()


def test_device_ic_refuses_conformal_eos(gpu_lib):
    g = fivo2d.make_grid2d(16, 16, xmax=5.0, ymax=5.0)
    m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS())
    w = GPUWork2D(m, g, lib=gpu_lib)
    with pytest.raises(A.FivoError):
        w.glauber_ic(0.6, 1001)
    w.close()
