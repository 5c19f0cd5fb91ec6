"""The 2-D freeze-out surface and its Cooper-Frye pion yield (freezeout2d.jl):
the host mirror of freeze_surface / pion_yield over the library's fivo_fo_* and
fivo_cooper_frye, and the axisymmetric control's initial profile.

freeze_surface evolves in chunks of dtau (run_sim_2d! on the same work, so the
history carries across), refreshes the primitives after each chunk and records
tau_fo(x, y), the last downward crossing of T_fo per cell, interpolated between
records (freezeout2d.jl:63-130). pion_yield integrates Cooper-Frye over that
surface (freezeout2d.jl:144-190).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi as A

T_FO = 0.156
T_MIN = 1e-20


def smoothstep01_5(x):
    """x^3 (10 - 15 x + 6 x^2) clamped to [0, 1] (src/utils.jl:27-29)"""
    if x <= 0:
        return 0.0
    if x >= 1:
        return 1.0
    return (x * x * x) * ((10 - 15 * x) + 6 * (x * x))


def load_initial_interpolants(path, taper_width: float = 1.0):
    """load_initial_interpolants(csv; fugacity_kind = :alpha, interp_kind = :linear)
    (src/io.jl:51-260): piecewise-linear T0(r) and alpha0(r) through the sorted,
    de-duplicated rows, tapered with smoothstep01_5 over the last taper_width fm
    to T_MIN and alpha = 0, and constant beyond the data. Returns (T(r), alpha(r), rmax)."""
    rows = []
    with open(path) as f:
        head = [h.strip() for h in f.readline().split(",")]
        ir, iT, ia = head.index("r"), head.index("T0"), head.index("alpha0")
        for line in f:
            if line.strip():
                p = line.split(",")
                rows.append((float(p[ir]), float(p[iT]), float(p[ia])))
    rows.sort(key=lambda t: t[0])
    keep = [rows[0]]
    for r in rows[1:]:
        if abs(r[0] - keep[-1][0]) > 0.0:
            keep.append(r)
    r = np.array([k[0] for k in keep])
    T0 = np.array([k[1] for k in keep])
    f0 = np.array([k[2] for k in keep])
    rmin, rmax = r[0], r[-1]
    tw = max(taper_width, 0.0)
    r_t0 = max(rmax - tw, rmin)
    inv_tw = 1.0 / tw if tw > 0 else 0.0

    def lin(v, rr):
        j = int(np.searchsorted(r, rr, side="right")) - 1
        j = min(max(j, 0), len(r) - 2)
        t = (rr - r[j]) / (r[j + 1] - r[j])
        return (1.0 - t) * v[j] + t * v[j + 1]

    def itpT(rr):
        if rr <= rmin:
            return max(T0[0], T_MIN)
        if rr <= rmax:
            if tw == 0.0 or rr < r_t0:
                return max(lin(T0, rr), T_MIN)
            w = 1.0 - smoothstep01_5((rr - r_t0) * inv_tw)
            return max(w * lin(T0, rr) + (1.0 - w) * T_MIN, T_MIN)
        return T_MIN

    def itpF(rr):
        if rr <= rmin:
            return f0[0]
        if rr <= rmax:
            if tw == 0.0 or rr < r_t0:
                return lin(f0, rr)
            w = 1.0 - smoothstep01_5((rr - r_t0) * inv_tw)
            return w * lin(f0, rr) + (1.0 - w) * 0.0
        return 0.0

    return itpT, itpF, float(rmax)


def axisym_fields(g, path):
    """T and alpha of every cell (ghosts included) from the radial profile, u = 0
    (the axisymmetric control of freezeout2d.jl:73-83)"""
    itpT, itpF, _ = load_initial_interpolants(path, taper_width=1.0)
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    R = np.hypot(X, Y).ravel()
    T = np.array([itpT(float(x)) for x in R])
    a = np.array([itpF(float(x)) for x in R])
    return T, a, np.zeros_like(T), np.zeros_like(T)


def freeze_model(**kw):
    """build_model_2d as freeze_surface builds it (freezeout2d.jl:65-70)"""
    from .model import LatticeHRGEOS, build_model_2d
    args = dict(eos=LatticeHRGEOS(), enable_shear=True, eta_over_s=0.10, tauShear_coeff=0.2,
                deltaShear_factor=4 / 3, enable_bulk=True, zeta_over_s=0.10, tauPi_coeff=15.0,
                enable_diff=True, kappa_coeff=0.1163, tauN_coeff=1.0, pi_clip_factor=1.0)
    args.update(kw)
    return build_model_2d(**args)


def cf_params(**kw):
    p = A.FivoCFParams()
    A.load_library().fivo_cf_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class FreezeOut:
    """A device freeze-out surface over a GPUWork2D's interior cells (fivo_fo)."""

    def __init__(self, work, T_fo: float = T_FO):
        self.lib = work.lib
        self.nx, self.ny = work.g.Nx, work.g.Ny
        h = C.c_void_p()
        A.check(self.lib, self.lib.fivo_fo_create(work.h, T_fo, C.byref(h)), "fivo_fo_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.fivo_fo_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def record(self, work, tau: float):
        A.check(self.lib, self.lib.fivo_fo_record(self.h, work.h, tau), "fivo_fo_record")

    def surface(self):
        n = self.nx * self.ny
        t, ux, uy = np.empty(n), np.empty(n), np.empty(n)
        cnt = np.zeros(3, dtype=np.int64)
        A.check(self.lib, self.lib.fivo_fo_surface(self.h, t.ctypes.data_as(A._D), ux.ctypes.data_as(A._D),
                                                   uy.ctypes.data_as(A._D),
                                                   cnt.ctypes.data_as(C.POINTER(C.c_int64))), "fivo_fo_surface")
        shape = (self.nx, self.ny)
        return dict(tau_fo=t.reshape(shape), uxf=ux.reshape(shape), uyf=uy.reshape(shape), nhot=int(cnt[0]),
                    nfroze=int(cnt[1]), refroze=int(cnt[2]))

    def set_surface(self, tau_fo, uxf, uyf):
        a = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (tau_fo, uxf, uyf)]
        A.check(self.lib, self.lib.fivo_fo_set_surface(self.h, *[x.ctypes.data_as(A._D) for x in a]),
                "fivo_fo_set_surface")

    def pion_yield(self, params=None):
        """(dN/dy Boltzmann, dN/dy Bose, negative-dSigma fraction)"""
        p = params if params is not None else cf_params()
        out = np.zeros(3)
        A.check(self.lib, self.lib.fivo_cooper_frye(self.h, C.byref(p), out.ctypes.data_as(A._D)), "fivo_cooper_frye")
        return float(out[0]), float(out[1]), float(out[2])


def freeze_surface(work, tau0: float, tau_max: float, dtau: float = 0.02, cfl: float = 0.15, cfltau: float = 0.05,
                   T_fo: float = T_FO, integrator=A.FIVO_SSPRK2):
    """freeze_surface's evolution and records on a prepared GPUWork2D (state set,
    finalize_ic done): returns (FreezeOut, chunks)"""
    fo = FreezeOut(work, T_fo)
    work.rhs(tau0)
    fo.record(work, tau0)
    tau, chunks = tau0, 0
    while tau < tau_max - 1e-9:
        r = work.run(tau, min(tau + dtau, tau_max), cfl, cfltau, integrator, reset_history=False)
        if not r["ok"]:
            raise RuntimeError(f"freeze_surface: the run failed at tau = {r['tau']}")
        tau = r["tau"]
        work.update_primitives(tau)
        fo.record(work, tau)
        chunks += 1
    return fo, chunks
