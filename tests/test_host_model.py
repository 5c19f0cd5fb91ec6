"""Host-side mirror of the reference's model construction (no GPU): grid geometry,
state layout, build_model_2d's keywords, defaults and refusals, the Terms
resolution, and the invariants of the seeded initial conditions.

Reference behaviour followed: make_grid2d (src2d/grid2d.jl:52-71),
make_layout2d (src2d/state_layout2d.jl:61-84), build_model_2d (main2D.jl:85-123),
reject_unwired_knobs_2d (src2d/primitives2d.jl:246-272), Terms/check_terms
(src/terms.jl), allocate_state (main2D.jl:125-126).
"""
import numpy as np
import pytest

import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.model import make_layout2d


def test_grid_geometry_and_flat_index():
    g = fivo2d.make_grid2d(384, 384, xmax=15.0, ymax=15.0)
    assert (g.Nxtot, g.Nytot, g.Ntot) == (390, 390, 390 * 390)
    assert g.dx == 30.0 / 384 and g.dy == 30.0 / 384
    # cell centres: first interior cell at -xmax + dx/2, ghosts beyond
    assert abs(g.xC[g.nghost] - (-15.0 + g.dx / 2)) < 1e-15
    assert abs(g.xC[g.nghost + g.Nx - 1] - (15.0 - g.dx / 2)) < 1e-14
    with pytest.raises(ValueError):
        fivo2d.make_grid2d(8, 64)


@pytest.mark.parametrize("charge,bulk,shear,nv", [
    (True, True, True, 11), (False, False, False, 4), (True, False, False, 6), (False, True, True, 9)])
def test_layout_rows(charge, bulk, shear, nv):
    L = make_layout2d(with_charge=charge, with_bulk=bulk, with_shear=shear)
    assert L.nv == nv
    expect = ["Dtau", "Sx", "Sy", "E"]
    if charge:
        expect += ["nux", "nuy"]
    if bulk:
        expect += ["Pi"]
    if shear:
        expect += ["pixx", "pixy", "piyy", "pieta"]
    assert L.names == expect and [L.idx(n) for n in expect] == list(range(nv))
    assert (L.hasNu, L.hasPi, L.hasShear) == (charge, bulk, shear)


def test_layout_appends_the_charm_second_moment():
    """make_layout2d(with_m2 = true) appends pQxx, pQxy, pQyy, pQeta, PiQ after the
    medium's rows (src2d/state_layout2d.jl:61-84)"""
    L = make_layout2d(with_m2=True)
    assert L.names == ["Dtau", "Sx", "Sy", "E", "nux", "nuy", "Pi", "pixx", "pixy", "piyy", "pieta",
                       "pQxx", "pQxy", "pQyy", "pQeta", "PiQ"]
    assert L.hasM2 and L.nv == 16 and L.idx("PiQ") == 15


def test_model_flattens_to_params():
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True,
                              eta_over_s=0.16, zeta_over_s=0.05, bulk_model="gaussian", bulk_T0=0.18,
                              bulk_width=0.024, kappa_coeff=0.5)
    p = m.params
    assert m.nv == 11
    assert p.eos_kind == A.FIVO_EOS_LATTICE_HRG and p.with_charge == 1
    assert (p.enable_shear, p.enable_bulk, p.enable_diff) == (1, 1, 1)
    assert p.bulk_kind == A.FIVO_BULK_GAUSS and p.bulk_T0 == 0.18 and p.bulk_width == 0.024
    assert p.eta_over_s == 0.16 and p.kappa_coeff == 0.5 and p.primrec_maxit == 80
    assert p.terms == A.FIVO_TERMS_DEFAULT
    # the reference's own Lorentzian bulk viscosity pins its peak and width
    m2 = fivo2d.build_model_2d(enable_bulk=True, bulk_model="lorentzian", bulk_T0=0.3, bulk_width=0.5)
    assert m2.params.bulk_kind == A.FIVO_BULK_LORENTZ
    assert (m2.params.bulk_T0, m2.params.bulk_width) == (0.175, 0.024)


def test_conformal_eos_without_charge_is_three_unknowns():
    m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS(g_eff=47.5, g_hq=0.0), with_charge=False)
    assert m.nv == 4 and m.params.eos_kind == A.FIVO_EOS_CONFORMAL_HQ and m.params.g_hq == 0.0


def test_refusals_follow_the_reference():
    with pytest.raises(TypeError):
        fivo2d.build_model_2d(no_such_knob=1)
    assert fivo2d.build_model_2d(consistent_fm=True).params.consistent_fm == 1
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(consistent_fm=True, tauN_coeff=1.5)
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(terms={"fm_dlnh": False})           # its sector (consistent_fm) is off
    assert fivo2d.build_model_2d(consistent_fm=True, terms={"fm_dlnh": False}).params.terms & \
        A.TERM_BIT["fm_dlnh"] == 0
    m2 = fivo2d.build_model_2d(enable_diff=True, consistent_m2=True)
    assert m2.params.consistent_m2 == 1 and m2.nv == 6 + 5 and m2.layout.names[-5:] == \
        ["pQxx", "pQxy", "pQyy", "pQeta", "PiQ"]
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(terms={"m2_vorticity": True})       # its sector (consistent_m2) is off
    assert fivo2d.build_model_2d(consistent_m2=True, terms={"m2_vorticity": True}).params.terms & \
        A.TERM_BIT["m2_vorticity"]
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(enable_bulk=True, bulk_model="triangular")
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(shear_constraint="ignore")


def test_state_is_julias_column_major_bytes():
    g = fivo2d.make_grid2d(16, 12, xmax=2.0, ymax=1.5)
    m = fivo2d.build_model_2d(enable_shear=True)
    U = fivo2d.allocate_state(g, m)
    assert U.shape == (g.Ntot, m.nv) and U.flags.c_contiguous and not U.any()


def test_glauber_ic_is_seeded_and_normalised():
    g = fivo2d.make_grid2d(48, 48, xmax=15.0, ymax=15.0)
    T1, a1, ux, uy, ev1 = ic.glauber_fields(g, 0.6, 1001)
    T2, a2, _, _, ev2 = ic.glauber_fields(g, 0.6, 1001)
    T3, _, _, _, _ = ic.glauber_fields(g, 0.6, 1002)
    assert np.array_equal(T1, T2) and np.array_equal(a1, a2)
    assert not np.array_equal(T1, T3)
    assert abs(T1.max() - 0.450) < 1e-9                    # peak T through the EOS inverse
    assert not ux.any() and not uy.any()                    # u = 0 at tau0
    assert 0.0 <= ev1["b"] <= 8.0
    assert a1.min() >= -20.0                                # alpha floored where there is no charm


def test_gubser_ic_matches_the_closed_form():
    g = fivo2d.make_grid2d(32, 32, xmax=10.0, ymax=10.0)
    Tsc = ic.gubser_Tscale_from_center_T(1.0, 1.0, 0.6)
    T, a, ux, uy = ic.gubser_fields(g, 1.0, q=1.0, Tscale=Tsc, alpha=-20.0)
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    r = np.hypot(X, Y).ravel()
    # u^r = v/sqrt(1-v^2) with v^r = 2 q^2 tau r / (1 + q^2 tau^2 + q^2 r^2) (src/gubser.jl:27-37)
    v = 2 * r / (1 + 1 + r * r)
    ur = v / np.sqrt(1 - v * v)
    assert np.allclose(np.hypot(ux, uy), ur, rtol=1e-12, atol=1e-14)
    assert abs(T.reshape(g.Nxtot, g.Nytot)[g.Nxtot // 2, g.Nytot // 2] - 0.6) < 0.05
    assert np.all(a == -20.0)


def test_terms_switches_and_refusals():
    """resolve_terms/check_terms (src/terms.jl): a term may be switched only when its
    sector is on; unknown names are refused."""
    on = fivo2d.build_model_2d(enable_diff=True, enable_shear=True,
                               terms={"nu_gradalpha": False, "shear_vorticity": True})
    p = on.params.terms
    assert not (p & A.TERM_BIT["nu_gradalpha"]) and (p & A.TERM_BIT["shear_vorticity"])
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(enable_diff=False, terms={"nu_gradalpha": False})
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(terms={"no_such_term": True})
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(terms=3.5)


def test_save_fields_round_trip(tmp_path):
    """save_fields / load_fields (src/fields_io.jl:70-106): the arrays come back
    bit for bit with the record of the model that made them"""
    g = fivo2d.make_grid2d(16, 12, xmax=2.0, ymax=1.5)
    m = fivo2d.build_model_2d(enable_diff=True, enable_shear=True, consistent_fm=True, consistent_m2=True,
                              terms={"m2_vorticity": True})
    rng = np.random.default_rng(5)
    f = {"x": g.xC[3:-3].copy(), "y": g.yC[3:-3].copy()}
    for name in ["T", "mu", "alpha", "n", "e", "P", "ux", "uy"] + m.layout.names[4:]:
        f[name] = rng.normal(size=(g.Nx, g.Ny))
    path = fivo2d.save_fields(tmp_path / "run" / "fields.npz", f, model=m, meta={"event": 3, "note": "m2 on"})
    d = fivo2d.load_fields(path)
    assert set(d["fields"]) == set(f)
    for k, v in f.items():
        assert np.array_equal(d["fields"][k].view(np.int64), np.asarray(v).view(np.int64)), k
    assert d["solver"] == "FiVo 2+1D"
    assert d["terms"]["m2_vorticity"] is True and d["terms"]["shear_vorticity"] is False
    assert d["model_fields"]["consistent_m2"] == "True" and d["model_fields"]["eos"] == "LatticeHRGEOS"
    assert "[x] m2_vorticity" in d["model"]
    assert d["meta"] == {"event": 3, "note": "m2 on"}
    assert d["created"] and d["fivo_revision"]
