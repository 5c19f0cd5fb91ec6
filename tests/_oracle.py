"""ctypes wrapper of the CPU oracle (oracle/liboracle_fivo2d.so) for the tests.

The oracle is test infrastructure: only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "fivohydro.jl_b200"))

from fivo2d import _abi as A  # noqa: E402

ORACLE_DIR = ROOT / "oracle"
ORACLE_SO = ORACLE_DIR / "liboracle_fivo2d.so"

_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)
_lib = None


def _ptr(a):
    if a is None:
        return None
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_U8)
    return a.ctypes.data_as(_D)


def build_oracle():
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        P = C.POINTER(A.FivoParams)
        sig = {
            "oracle_last_error": (C.c_char_p, []),
            "oracle_ctx_create": (C.c_void_p, [P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]),
            "oracle_ctx_destroy": (None, [C.c_void_p]),
            "oracle_ctx_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64), _D]),
            "oracle_set_state": (None, [C.c_void_p, _D]),
            "oracle_get_state": (None, [C.c_void_p, _D]),
            "oracle_set_history": (None, [C.c_void_p] + [_D] * 8),
            "oracle_get_history": (None, [C.c_void_p] + [_D] * 8),
            "oracle_reset_history": (None, [C.c_void_p]),
            "oracle_get_primitives": (None, [C.c_void_p] + [_D] * 9 + [_U8]),
            "oracle_get_counters": (None, [C.c_void_p, C.POINTER(A.FivoCounters)]),
            "oracle_rhs": (None, [C.c_void_p, C.c_double, C.c_int, _U8, _D]),
            "oracle_step": (None, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                   _D, C.POINTER(C.c_int)]),
            "oracle_update_primitives": (C.c_int64, [C.c_void_p, C.c_double, C.c_int]),
            "oracle_relax": (None, [C.c_void_p, C.c_double, C.c_double]),
            "oracle_project_shear": (None, [C.c_void_p, _D, _D]),
            "oracle_compute_dt": (C.c_double, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
            "oracle_run": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                  C.c_int, C.c_int64, C.c_int, C.POINTER(A.FivoRunResult)]),
            "oracle_finalize_ic": (None, [C.c_void_p, C.c_double, C.c_int]),
            "oracle_advance": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                      C.c_int, C.c_int64, C.POINTER(A.FivoRunResult)]),
            "oracle_set_cells": (C.c_int, [P, C.c_int64, C.c_double] + [_D] * 10 + [_D, _U8]),
            "oracle_eos_Pne": (None, [P, C.c_int64, _D, _D, _D, _D, _D]),
            "oracle_eos_cs2": (None, [P, C.c_int64, _D, _D, _D]),
            "oracle_cons_to_prim": (None, [P, C.c_int64, C.c_double, _D, _D, _D, _U8, _U8]),
            "oracle_besselkx": (None, [C.c_int, C.c_int64, _D, _D]),
            "oracle_exp": (None, [C.c_int64, _D, _D]),
            "oracle_log": (None, [C.c_int64, _D, _D]),
            "oracle_pow4": (None, [C.c_int64, _D, _D]),
            "oracle_hypot": (None, [C.c_int64, _D, _D, _D]),
            "oracle_cfm_source": (None, [_D, C.c_uint32, _D, _D]),
            "oracle_cfm_h_hprime": (None, [P, C.c_double, _D, _D]),
            "oracle_cfm_dn_dT": (C.c_double, [P, C.c_double, C.c_double]),
            "oracle_diff_coeffs": (None, [P, C.c_double, C.c_double, C.c_double, _D, _D, _D]),
            "oracle_fo_record": (None, [C.c_void_p, C.c_double, C.c_double, C.c_double, _D, _D, _D, _D, _U8,
                                        C.POINTER(C.c_int64)]),
            "oracle_pion_yield": (None, [C.c_int, C.c_int, C.c_double, _D, _D, _D, _D, C.POINTER(C.c_int), _D]),
            "oracle_ref_bjorken_bulk": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64, _D]),
            "oracle_ref_bjorken_shear": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64, _D]),
            "oracle_ref_bjorken_dnmr": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64, _D,
                                               _D]),
            "oracle_ref_gubser_viscous": (None, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64,
                                                 C.c_int, _D, _D]),
            "oracle_shear_coeffs": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _D]),
            "oracle_bulk_coeffs": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _D]),
            "oracle_diff_tauN": (None, [P, C.c_double, C.c_double, C.c_double, C.c_double, _D]),
            "oracle_vacuum_weight": (C.c_double, [P, C.c_double]),
            "oracle_entropy": (C.c_double, [C.c_double] * 5),
            "oracle_ns_shear_target": (None, [C.c_int64, _D, _D]),
            "oracle_project_traceless": (None, [C.c_int64, _D, _D]),
            "oracle_ns_diffusion_target": (None, [C.c_int64, _D, _D]),
            "oracle_pi_sigma": (None, [C.c_int64, _D, _D]),
            "oracle_shear_tensor": (None, [C.c_int64, _D, _D]),
            "oracle_set_nu_history": (None, [C.c_void_p, _D, _D]),
            "oracle_get_nu_history": (None, [C.c_void_p, _D, _D]),
            "oracle_m2_source": (None, [_D, C.c_uint32, _D]),
            "oracle_m2_coeffs": (None, [C.c_double] * 6 + [_D]),
            "oracle_m2_tauM": (C.c_double, [C.c_double] * 3),
            "oracle_m2_sigma_nu": (None, [_D, _D]),
            "oracle_m2_rank1_traceless": (None, [_D, _D]),
            "oracle_ref_m2_rhs_1d": (None, [_D, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def vec(fn, x, *more):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    args = [np.ascontiguousarray(m, dtype=np.float64) for m in more]
    fn(x.size, _ptr(x), *[_ptr(a) for a in args], _ptr(out))
    return out


def besselkx(nu, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().oracle_besselkx(nu, x.size, _ptr(x), _ptr(out))
    return out


def set_cells(params, tau, T, alpha, ux, uy, nv, Pi=None, pixx=None, pixy=None, piyy=None, nux=None, nuy=None):
    n = len(T)
    U = np.zeros((n, nv))
    ok = np.zeros(n, dtype=np.uint8)
    cv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
    arrs = [cv(a) for a in (T, alpha, ux, uy, Pi, pixx, pixy, piyy, nux, nuy)]
    st = lib().oracle_set_cells(C.byref(params), n, tau, *[_ptr(a) for a in arrs], _ptr(U), _ptr(ok))
    assert st == 0, lib().oracle_last_error()
    return U, ok


def eos_Pne(params, T, mu):
    T = np.ascontiguousarray(T, dtype=np.float64)
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    P, n, e = np.empty_like(T), np.empty_like(T), np.empty_like(T)
    lib().oracle_eos_Pne(C.byref(params), T.size, _ptr(T), _ptr(mu), _ptr(P), _ptr(n), _ptr(e))
    return P, n, e


def eos_cs2(params, T, mu):
    T = np.ascontiguousarray(T, dtype=np.float64)
    mu = np.ascontiguousarray(mu, dtype=np.float64)
    out = np.empty_like(T)
    lib().oracle_eos_cs2(C.byref(params), T.size, _ptr(T), _ptr(mu), _ptr(out))
    return out


def cons_to_prim(params, tau, cons, warm=None):
    cons = np.ascontiguousarray(cons, dtype=np.float64).reshape(-1, 11)
    n = cons.shape[0]
    prim = np.empty((n, 7))
    ok = np.zeros(n, dtype=np.uint8)
    reason = np.zeros(n, dtype=np.uint8)
    w = None if warm is None else np.ascontiguousarray(warm, dtype=np.float64).reshape(-1, 4)
    lib().oracle_cons_to_prim(C.byref(params), n, tau, _ptr(cons), _ptr(w), _ptr(prim), _ptr(ok), _ptr(reason))
    return prim, ok.astype(bool), reason


class OracleSolver:
    """Same surface as fivo2d.solver.GPUSolver, on the CPU oracle."""

    def __init__(self, model, g):
        self.model, self.g = model, g
        self.h = lib().oracle_ctx_create(C.byref(model.params), g.Nx, g.Ny, g.nghost, g.xmax, g.ymax)
        if not self.h:
            raise RuntimeError(lib().oracle_last_error().decode())
        self.nv = model.nv
        self.N = g.Ntot

    def close(self):
        if self.h:
            lib().oracle_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.size == self.nv * self.N
        lib().oracle_set_state(self.h, _ptr(U))

    def get_state(self):
        U = np.empty((self.N, self.nv))
        lib().oracle_get_state(self.h, _ptr(U))
        return U

    def set_history(self, **kw):
        names = ("x0_yT", "x0_phi", "x0_ux", "x0_uy", "ux_prev", "uy_prev", "alpha_prev", "T_prev")
        arrs = [None if kw.get(n) is None else np.ascontiguousarray(kw[n], dtype=np.float64) for n in names]
        lib().oracle_set_history(self.h, *[_ptr(a) for a in arrs])

    def get_history(self):
        names = ("x0_yT", "x0_phi", "x0_ux", "x0_uy", "ux_prev", "uy_prev", "alpha_prev", "T_prev")
        arrs = [np.empty(self.N) for _ in names]
        lib().oracle_get_history(self.h, *[_ptr(a) for a in arrs])
        return dict(zip(names, arrs))

    def reset_history(self):
        lib().oracle_reset_history(self.h)

    def set_nu_history(self, nux_prev=None, nuy_prev=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (nux_prev, nuy_prev)]
        lib().oracle_set_nu_history(self.h, *[_ptr(a) for a in arrs])

    def get_nu_history(self):
        arrs = [np.empty(self.N), np.empty(self.N)]
        lib().oracle_get_nu_history(self.h, *[_ptr(a) for a in arrs])
        return dict(nux_prev=arrs[0], nuy_prev=arrs[1])

    def primitives(self):
        names = ("yT", "phi", "mu", "alpha", "ux", "uy", "P", "n", "e")
        arrs = [np.empty(self.N) for _ in names]
        ok = np.empty(self.N, dtype=np.uint8)
        lib().oracle_get_primitives(self.h, *[_ptr(a) for a in arrs], _ptr(ok))
        d = dict(zip(names, arrs))
        d["ok"] = ok
        return d

    def counters(self):
        c = A.FivoCounters()
        lib().oracle_get_counters(self.h, C.byref(c))
        return c

    def rhs(self, tau, bc=0, mask=None):
        dU = np.empty((self.N, self.nv))
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        lib().oracle_rhs(self.h, tau, bc, _ptr(m), _ptr(dU))
        return dU

    def step(self, integrator, tau, dtau, max_halve=12, max_mood=2, bc=0):
        used = C.c_double(0)
        ok = C.c_int(0)
        lib().oracle_step(self.h, integrator, tau, dtau, max_halve, max_mood, bc, C.byref(used), C.byref(ok))
        return bool(ok.value), used.value

    def update_primitives(self, tau, bc=0):
        return lib().oracle_update_primitives(self.h, tau, bc)

    def relax(self, tau, dtau):
        lib().oracle_relax(self.h, tau, dtau)

    def project_shear(self):
        a, b = C.c_double(0), C.c_double(0)
        lib().oracle_project_shear(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def compute_dt(self, tau, cfl=0.2, cfltau=0.05):
        return lib().oracle_compute_dt(self.h, tau, cfl, cfltau)

    def run(self, tau0, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=0,
            max_steps=2_000_000, reset_history=True):
        r = A.FivoRunResult()
        lib().oracle_run(self.h, tau0, taufinal, cfl, cfltau, integrator, bc, max_steps, int(reset_history),
                         C.byref(r))
        return r.as_dict()

    def advance(self, tau, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=0, max_steps=1):
        r = A.FivoRunResult()
        lib().oracle_advance(self.h, tau, taufinal, cfl, cfltau, integrator, bc, max_steps, C.byref(r))
        return r.as_dict()

    def finalize_ic(self, tau0, bc=0):
        lib().oracle_finalize_ic(self.h, tau0, bc)


# ----------------------------------------------------------------- cell-level functions and referees


def _rows(fn, rows, width_out):
    rows = np.ascontiguousarray(rows, dtype=np.float64)
    k = rows.shape[0]
    out = np.empty((k, width_out)) if width_out > 1 else np.empty(k)
    fn(k, _ptr(rows), _ptr(out))
    return out


def ns_shear_target(rows12):
    """rows of (ux, uy, ut, tau, theta, ax, ay, dxux, dxuy, dyux, dyuy, eta) -> (xx, xy, yy, eta)"""
    return _rows(lib().oracle_ns_shear_target, rows12, 4)


def project_traceless(rows6):
    return _rows(lib().oracle_project_traceless, rows6, 1)


def ns_diffusion_target(rows7):
    return _rows(lib().oracle_ns_diffusion_target, rows7, 2)


def pi_sigma(rows10):
    return _rows(lib().oracle_pi_sigma, rows10, 4)


def shear_tensor(rows8):
    return _rows(lib().oracle_shear_tensor, rows8, 7)


# consistent_m2_source_2d's 44 positional arguments, in order (src2d/hq_consistent_m2_2d.jl:247-262)
M2_ARGS = ("ux", "uy", "ut", "tau", "T", "dxT", "dyT", "dtT", "nux", "nuy", "pxx", "pxy", "pyy", "peta", "PiQ",
           "dta", "dxa", "dya", "thnu", "anux", "anuy", "dtnux", "dtnuy", "dxnux", "dxnuy", "dynux", "dynuy",
           "th", "ax", "ay", "dtux", "dtuy", "dxux", "dxuy", "dyux", "dyuy", "n", "tn", "Ds", "h", "hp", "tM",
           "etaM", "m")


def m2_source(args, terms=A.FIVO_TERMS_DEFAULT):
    """consistent_m2_source_2d: a dict (or sequence) of the 44 arguments -> (dpxx, dpxy, dpyy, dPiQ, geo)"""
    a = np.array([args[k] for k in M2_ARGS] if isinstance(args, dict) else args, dtype=np.float64)
    assert a.size == 44
    out = np.empty(5)
    lib().oracle_m2_source(_ptr(a), terms, _ptr(out))
    return out


def m2_coeffs(T, n, tn, Ds, h, m):
    out = np.empty(5)
    lib().oracle_m2_coeffs(T, n, tn, Ds, h, m, _ptr(out))
    return dict(zip(("dlnC_dlnT", "etabar", "lambda_a", "Aco", "ABr"), out))


def m2_tauM(T, tn, m=1.5):
    return lib().oracle_m2_tauM(T, tn, m)


def m2_sigma_nu(*a18):
    a = np.array(a18, dtype=np.float64)
    out = np.empty(4)
    lib().oracle_m2_sigma_nu(_ptr(a), _ptr(out))
    return out


def m2_rank1_traceless(*a7):
    a = np.array(a7, dtype=np.float64)
    out = np.empty(3)
    lib().oracle_m2_rank1_traceless(_ptr(a), _ptr(out))
    return out


def ref_m2_rhs_1d(**kw):
    """hq_consistent_m2_rhs (src/hq_consistent_m2.jl:138-252), all terms on -> (dp_l, dp_phi, dPiQ)"""
    names = ("tau", "r", "ur", "T", "dtT", "drT", "drur", "dtur", "p_l", "p_phi", "PiQ", "nu", "dta", "dra",
             "dtnu", "drnu", "drp_l", "drp_phi", "drPiQ", "n", "tn", "Ds", "h", "hp", "tM", "etaM", "m")
    a = np.array([kw.get(k, 0.0) for k in names], dtype=np.float64)
    out = np.empty(3)
    lib().oracle_ref_m2_rhs_1d(_ptr(a), _ptr(out))
    return out


def shear_coeffs(params, T, mu, n, e, P):
    out = np.empty(3)
    lib().oracle_shear_coeffs(C.byref(params), T, mu, n, e, P, _ptr(out))
    return out


def bulk_coeffs(params, T, mu, n, e, P):
    out = np.empty(2)
    lib().oracle_bulk_coeffs(C.byref(params), T, mu, n, e, P, _ptr(out))
    return out


def diff_coeffs(params, T, mu, n):
    k, t, d = C.c_double(), C.c_double(), C.c_double()
    lib().oracle_diff_coeffs(C.byref(params), T, mu, n, C.byref(k), C.byref(t), C.byref(d))
    return k.value, t.value, d.value


def diff_tauN(params, T, alpha, DsT, tauD):
    out = np.empty(2)
    lib().oracle_diff_tauN(C.byref(params), T, alpha, DsT, tauD, _ptr(out))
    return out[0]


def vacuum_weight(params, n):
    return lib().oracle_vacuum_weight(C.byref(params), n)


def ref_bjorken_bulk(params, T0, alpha, tau0, tauf, n=40_000):
    out = np.empty(3)
    lib().oracle_ref_bjorken_bulk(C.byref(params), T0, alpha, tau0, tauf, n, _ptr(out))
    return out


def ref_bjorken_shear(params, T0, alpha, tau0, tauf, nsub=20_000):
    out = np.empty(3)
    lib().oracle_ref_bjorken_shear(C.byref(params), T0, alpha, tau0, tauf, nsub, _ptr(out))
    return out


def ref_bjorken_dnmr(params, T0, alpha, tau0, tau1, ratios=(0.0, 0.0, 0.0, 0.0, 0.0), n=20_000):
    r = np.ascontiguousarray(ratios, dtype=np.float64)
    out = np.empty(3)
    lib().oracle_ref_bjorken_dnmr(C.byref(params), T0, alpha, tau0, tau1, n, _ptr(r), _ptr(out))
    return out


def ref_gubser_viscous(etas, TH0=0.6, rhomin=-6.0, rhomax=2.0, n=400_000, seed_ns=True):
    Th = np.empty(n + 1)
    pb = np.empty(n + 1)
    lib().oracle_ref_gubser_viscous(etas, TH0, rhomin, rhomax, n, int(seed_ns), _ptr(Th), _ptr(pb))
    return np.linspace(rhomin, rhomax, n + 1), Th, pb
