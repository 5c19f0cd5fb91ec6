"""Host-side mirror of the reference's 2+1D model construction.

Same names, keyword arguments, defaults and refusals as the Julia API:

  make_grid2d          src2d/grid2d.jl:52-71
  make_layout2d        src2d/state_layout2d.jl:61-84
  ConformalHQEOS       src/eos.jl:39-47
  LatticeHRGEOS        src/eos.jl:318-345
  build_model_2d       main2D.jl:85-123 (+ IdealDiffVisc2DModel, src2d/primitives2d.jl:41-210)
  allocate_state       main2D.jl:125-126

A model flattens into the C struct `fivo_params` (include/fivo2d.h).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

# src/constants.jl
HBARC = 0.1973269804
T_MIN = 1e-20
E_FLOOR = 1e-20


@dataclass
class Grid2D:
    """Cartesian box [-xmax, xmax] x [-ymax, ymax] with `nghost` ghost layers
    (src2d/grid2d.jl:19-38). Flat index i = ix*Nytot + iy (0-based, y fast)."""
    Nx: int
    Ny: int
    nghost: int
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    dx: float
    dy: float
    Nxtot: int
    Nytot: int
    Ntot: int
    xC: np.ndarray
    yC: np.ndarray

    def lin(self, ix, iy):
        return ix * self.Nytot + iy

    def interior(self):
        """(ix, iy) slices of the physical cells in a (Nxtot, Nytot) view."""
        ng = self.nghost
        return slice(ng, ng + self.Nx), slice(ng, ng + self.Ny)


def make_grid2d(Nx: int, Ny: int, *, xmax: float = 20.0, ymax: float = 20.0, nghost: int = 3) -> Grid2D:
    """src2d/grid2d.jl:52-71."""
    if not (Nx > 8 and Ny > 8):
        raise ValueError("make_grid2d: Nx and Ny must exceed 8")
    if not (xmax > 0 and ymax > 0):
        raise ValueError("make_grid2d: xmax and ymax must be positive")
    if nghost != 3:
        raise ValueError("make_grid2d: the stage is built for nghost = 3")
    xmin, ymin = -xmax, -ymax
    dx = (xmax - xmin) / Nx
    dy = (ymax - ymin) / Ny
    Nxtot, Nytot = Nx + 2 * nghost, Ny + 2 * nghost
    xC = np.array([xmin + ((i + 1 - nghost) - 0.5) * dx for i in range(Nxtot)])
    yC = np.array([ymin + ((j + 1 - nghost) - 0.5) * dy for j in range(Nytot)])
    return Grid2D(Nx, Ny, nghost, xmin, xmax, ymin, ymax, dx, dy, Nxtot, Nytot, Nxtot * Nytot, xC, yC)


make_grid_2d = make_grid2d


@dataclass
class StateLayout2D:
    """Dense field order Dtau, Sx, Sy, E, [nux, nuy], [Pi], [pixx, pixy, piyy, pieta],
    [pQxx, pQxy, pQyy, pQeta, PiQ] (src2d/state_layout2d.jl:61-84); indices are 0-based."""
    names: list
    hasNu: bool
    hasPi: bool
    hasShear: bool
    hasM2: bool = False

    @property
    def nv(self):
        return len(self.names)

    def idx(self, name):
        return self.names.index(name)


def make_layout2d(*, with_charge=True, with_bulk=True, with_shear=True, with_m2=False) -> StateLayout2D:
    names = ["Dtau", "Sx", "Sy", "E"]
    if with_charge:
        names += ["nux", "nuy"]
    if with_bulk:
        names += ["Pi"]
    if with_shear:
        names += ["pixx", "pixy", "piyy", "pieta"]
    if with_m2:
        names += ["pQxx", "pQxy", "pQyy", "pQeta", "PiQ"]
    return StateLayout2D(names, with_charge, with_bulk, with_shear, with_m2)


@dataclass
class ConformalHQEOS:
    """src/eos.jl:39-47."""
    g_eff: float = 40.0
    m_hq: float = 1.5
    g_hq: float = 6.0
    hq_times_fmGeV3: bool = False


# I1(21.55/2)/I0(21.55/2), the reference's _LHRG_CCBAR_FACT (src/eos.jl:347-348),
# evaluated once with AMOS-based scipy.special.iv.
_LHRG_CCBAR_FACT = 0.9524014587885937


@dataclass
class LatticeHRGEOS:
    """src/eos.jl:318-345."""
    a1: float = -15.526548963383643
    a2: float = 18.6159584620131
    a3: float = -10.731808109698516
    a4: float = 2.7413302179949346
    b1: float = -3.3147904483107595
    b2: float = 5.310983721567554
    b3: float = -4.653922019495976
    b4: float = 1.8600649533271152
    c: float = -1.0465330501411811
    d: float = 0.09551531822245873
    m_hq: float = 1.5
    g_hq: float = 6.0
    hq_times_fmGeV3: bool = True
    canon_factor: float = _LHRG_CCBAR_FACT


def canonical_factor(N: float) -> float:
    """I1(N/2)/I0(N/2) (src/eos.jl:349)."""
    from scipy.special import ive
    return float(ive(1, N / 2) / ive(0, N / 2))


# Knobs the 2-D solver refuses away from their defaults (src2d/primitives2d.jl:232-237).
_UNWIRED_KNOBS_2D = (("diffusion_drive", "alpha"), ("diff_dt_coeff", 0.0),
                     ("shear_dt_coeff", 0.0), ("bulk_dt_coeff", 0.0))

# IdealDiffVisc2DModel keyword defaults (src2d/primitives2d.jl:41-210)
_MODEL_DEFAULTS = dict(
    enable_diff=False, diffusion_drive="alpha", kappa_coeff=0.0, transport_mass=0.0,
    tauN_coeff=1.0, deltaN_factor=0.0, diff_dt_coeff=0.0, advect_nu=False, relax_advect_nu=True,
    nu_clip_factor=-1.0, vacuum_n_lo=1e-6, vacuum_n_hi=2e-3, vacuum_ramp_relax=True,
    consistent_fm=False, consistent_m2=False,
    enable_shear=False, deltaShear_factor=4 / 3, taupi_pi_factor=0.0, shear_dt_coeff=0.0,
    advect_pi=False, relax_advect_pi=True, pi_clip_factor=-1.0,
    enable_bulk=False, deltaPi_factor=0.0, lambda_Pi_pi_factor=0.0, lambda_pi_Pi_factor=0.0,
    bulk_dt_coeff=0.0, advect_Pi=False, relax_advect_Pi=True, relax_advect_m2=True,
    Pi_clip_factor=-1.0, r_domain=math.inf, T_vac_cut=0.05, E_vac_cut=-1.0,
    shear_projected_deriv=True, diff_projected_deriv=True, shear_constraint="project",
)

# Sector each term belongs to (src/terms.jl TERM_REGISTER)
_TERM_SECTOR = {n: ("enable_diff" if n == "nu_gradalpha" else
                    "enable_shear" if n == "shear_vorticity" else
                    "consistent_fm" if n.startswith("fm_") else "consistent_m2")
                for n in A.TERM_NAMES}


def _resolve_terms(spec, sector_on) -> int:
    """A subset of resolve_terms (src/terms.jl): None/'default', an int mask, or a
    dict {term: bool}; then check_terms' refusal of switches that cannot act."""
    mask = A.FIVO_TERMS_DEFAULT
    if spec is None or spec == "default" or spec == ":default":
        pass
    elif isinstance(spec, int):
        mask = spec
    elif isinstance(spec, dict):
        for k, v in spec.items():
            if k not in A.TERM_BIT:
                raise ValueError(f"unknown term {k!r}; valid: {', '.join(A.TERM_NAMES)}")
            mask = (mask | A.TERM_BIT[k]) if v else (mask & ~A.TERM_BIT[k])
    else:
        raise ValueError(f"unsupported terms spec {spec!r}")
    for name in A.TERM_NAMES:
        bit = A.TERM_BIT[name]
        default_on = bool(A.FIVO_TERMS_DEFAULT & bit)
        on = bool(mask & bit)
        if on != default_on and not sector_on(_TERM_SECTOR[name]):
            raise ValueError(f"Terms2D: `{name}` is switched but its sector `{_TERM_SECTOR[name]}` is off")
    return mask


@dataclass
class IdealDiffVisc2DModel:
    eos: object
    layout: StateLayout2D
    params: A.FivoParams
    knobs: dict = field(default_factory=dict)

    @property
    def nv(self):
        return self.layout.nv


def eos_params(eos, p: A.FivoParams | None = None) -> A.FivoParams:
    """Fill the EOS block of a fivo_params."""
    p = p if p is not None else A.FivoParams()
    if isinstance(eos, ConformalHQEOS):
        lh = LatticeHRGEOS()                # unused by this EOS; fivo_params_default's values
        for k, v in enumerate((lh.a1, lh.a2, lh.a3, lh.a4)):
            p.lhrg_a[k] = v
        for k, v in enumerate((lh.b1, lh.b2, lh.b3, lh.b4)):
            p.lhrg_b[k] = v
        p.lhrg_c, p.lhrg_d, p.canon_factor = lh.c, lh.d, lh.canon_factor
        p.eos_kind = A.FIVO_EOS_CONFORMAL_HQ
        p.g_eff, p.m_hq, p.g_hq = eos.g_eff, eos.m_hq, eos.g_hq
        p.hq_times_fmGeV3 = int(eos.hq_times_fmGeV3)
    elif isinstance(eos, LatticeHRGEOS):
        p.eos_kind = A.FIVO_EOS_LATTICE_HRG
        p.g_eff = ConformalHQEOS.g_eff      # unused by this EOS; fivo_params_default's value
        for k, v in enumerate((eos.a1, eos.a2, eos.a3, eos.a4)):
            p.lhrg_a[k] = v
        for k, v in enumerate((eos.b1, eos.b2, eos.b3, eos.b4)):
            p.lhrg_b[k] = v
        p.lhrg_c, p.lhrg_d = eos.c, eos.d
        p.m_hq, p.g_hq = eos.m_hq, eos.g_hq
        p.hq_times_fmGeV3 = int(eos.hq_times_fmGeV3)
        p.canon_factor = eos.canon_factor
    else:
        raise TypeError(f"unsupported EOS {type(eos).__name__}")
    return p


def build_model_2d(*, eos=None, r_domain: float = math.inf, enable_shear: bool = False,
                   enable_bulk: bool = False, enable_diff: bool = False, with_charge: bool = True,
                   eta_over_s: float = 0.1, tauShear_coeff: float = 0.2,
                   zeta_over_s: float = 0.1, tauPi_coeff: float = 15.0,
                   bulk_model: str = "lorentzian", bulk_T0: float = 0.175, bulk_width: float = 0.024,
                   terms=None, primrec_maxit: int = 80, primrec_tol: float = 1e-12,
                   **kwargs) -> IdealDiffVisc2DModel:
    """main2D.jl:85-123. `bulk_model` selects the BulkViscosity subtype:
    "lorentzian" = SimpleBulkViscosity (peak at 0.175 GeV, half-width 0.024 GeV),
    "gaussian" = GaussianBulkViscosity, zeta/s = peak * exp(-(T-T0)^2/(2 width^2))."""
    eos = LatticeHRGEOS() if eos is None else eos
    unknown = set(kwargs) - set(_MODEL_DEFAULTS)
    if unknown:
        raise TypeError(f"build_model_2d: unknown keyword(s) {sorted(unknown)}")
    knobs = dict(_MODEL_DEFAULTS)
    knobs.update(kwargs)
    knobs.update(enable_shear=enable_shear, enable_bulk=enable_bulk, enable_diff=enable_diff,
                 r_domain=r_domain)
    # reject_unwired_knobs_2d, src2d/primitives2d.jl:246-272
    for knob, default in _UNWIRED_KNOBS_2D:
        if knobs[knob] != default:
            raise ValueError(f"IdealDiffVisc2DModel: `{knob} = {knobs[knob]}` is NOT implemented in the "
                             f"2-D solver; use the default ({default}).")
    if knobs["consistent_fm"] and knobs["tauN_coeff"] != 1.0:
        raise ValueError("IdealDiffVisc2DModel: `tauN_coeff` cannot be combined with `consistent_fm = true`.")
    if knobs["shear_constraint"] not in ("project", "monitor"):
        raise ValueError("shear_constraint must be 'project' or 'monitor'")

    L = make_layout2d(with_charge=with_charge, with_bulk=enable_bulk, with_shear=enable_shear,
                      with_m2=bool(knobs["consistent_m2"]))
    p = eos_params(eos)
    p.with_charge = int(with_charge)
    p.enable_diff, p.enable_shear, p.enable_bulk = int(enable_diff), int(enable_shear), int(enable_bulk)
    p.shear_kind = A.FIVO_SHEAR_QGP if enable_shear else A.FIVO_SHEAR_ZERO
    p.eta_over_s, p.tauShear_coeff = eta_over_s, tauShear_coeff
    if enable_bulk:
        if bulk_model == "lorentzian":
            p.bulk_kind = A.FIVO_BULK_LORENTZ
            bulk_T0, bulk_width = 0.175, 0.024
        elif bulk_model == "gaussian":
            p.bulk_kind = A.FIVO_BULK_GAUSS
        else:
            raise ValueError(f"unknown bulk_model {bulk_model!r}")
    else:
        p.bulk_kind = A.FIVO_BULK_ZERO
    p.zeta_over_s, p.tauPi_coeff, p.bulk_T0, p.bulk_width = zeta_over_s, tauPi_coeff, bulk_T0, bulk_width
    for name in ("kappa_coeff", "tauN_coeff", "deltaN_factor", "nu_clip_factor", "vacuum_n_lo",
                 "vacuum_n_hi", "deltaShear_factor", "taupi_pi_factor", "lambda_pi_Pi_factor",
                 "pi_clip_factor", "deltaPi_factor", "lambda_Pi_pi_factor", "Pi_clip_factor",
                 "r_domain", "T_vac_cut", "E_vac_cut", "transport_mass"):
        setattr(p, name, float(knobs[name]))
    for name in ("advect_nu", "relax_advect_nu", "advect_pi", "relax_advect_pi", "advect_Pi",
                 "relax_advect_Pi", "vacuum_ramp_relax", "shear_projected_deriv",
                 "diff_projected_deriv", "consistent_fm", "consistent_m2", "relax_advect_m2"):
        setattr(p, name, int(bool(knobs[name])))
    p.shear_constraint_project = int(knobs["shear_constraint"] == "project")
    p.primrec_maxit, p.primrec_tol = int(primrec_maxit), float(primrec_tol)
    sectors = dict(enable_diff=enable_diff, enable_shear=enable_shear, consistent_fm=bool(knobs["consistent_fm"]),
                   consistent_m2=bool(knobs["consistent_m2"]))
    p.terms = _resolve_terms(terms, lambda s: sectors[s])
    return IdealDiffVisc2DModel(eos=eos, layout=L, params=p, knobs=knobs)


def allocate_state(g: Grid2D, model: IdealDiffVisc2DModel) -> np.ndarray:
    """main2D.jl:125-126: zeros(nv, Ntot), stored here as an (Ntot, nv) C-order array,
    which is the same bytes as Julia's column-major (nv, Ntot)."""
    return np.zeros((g.Ntot, model.nv), dtype=np.float64)
