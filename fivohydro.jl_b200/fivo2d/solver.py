"""GPU-backed Work2D and the reference's driver entry points over the C ABI.

`GPUWork2D` owns a device context (fivo_ctx) holding the state, primitives,
warm starts and dtau history of one event. The functions below keep the Julia
names and argument meaning:

  rhs_2d!               -> GPUWork2D.rhs
  step_ssprk{2,3}_2d!   -> GPUWork2D.step
  update_primitives_2d! -> GPUWork2D.update_primitives
  relax_dissipative_2d! -> GPUWork2D.relax
  project_shear!        -> GPUWork2D.project_shear
  compute_dt_2d         -> GPUWork2D.compute_dt
  run_sim_2d!           -> run_sim_2d (returns the reference's NamedTuple fields)
  set_cell!/finalize_ic! -> set_cells / GPUWork2D.finalize_ic
  fields_2d             -> fields_2d

There is no CPU fallback: every call goes to libfivo2d.so and raises if the
library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A
from .model import Grid2D, IdealDiffVisc2DModel

_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)


def _ptr(a):
    if a is None:
        return None
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_U8)
    return a.ctypes.data_as(_D)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


HISTORY = ("x0_yT", "x0_phi", "x0_ux", "x0_uy", "ux_prev", "uy_prev", "alpha_prev", "T_prev")
PRIMS = ("yT", "phi", "mu", "alpha", "ux", "uy", "P", "n", "e")


class GPUWork2D:
    """A device-resident Work2D for one (grid, model) pair."""

    def __init__(self, model: IdealDiffVisc2DModel, g: Grid2D, lib=None, _handle=None):
        self.lib = lib or A.load_library()
        self.model, self.g = model, g
        self.nv, self.N = model.nv, g.Ntot
        self._owned = _handle is None
        if _handle is not None:          # an event of a GPUBatch2D: the batch owns the context
            self.h = _handle
            return
        h = C.c_void_p()
        A.check(self.lib, self.lib.fivo_ctx_create(C.byref(model.params), g.Nx, g.Ny, g.nghost, g.xmax,
                                                   g.ymax, C.byref(h)), "fivo_ctx_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value and getattr(self, "_owned", True):
            self.lib.fivo_ctx_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st, what):
        A.check(self.lib, st, what)

    # ---- state / history
    def set_state(self, U):
        U = _f64(U)
        if U.size != self.nv * self.N:
            raise ValueError("state size mismatch")
        self._ck(self.lib.fivo_upload_state(self.h, _ptr(U), self.nv, self.N), "fivo_upload_state")

    def get_state(self):
        U = np.empty((self.N, self.nv))
        self._ck(self.lib.fivo_download_state(self.h, _ptr(U), self.nv, self.N), "fivo_download_state")
        return U

    def set_history(self, **kw):
        arrs = [_f64(kw.get(n)) for n in HISTORY]
        self._ck(self.lib.fivo_upload_history(self.h, self.N, *[_ptr(a) for a in arrs]), "fivo_upload_history")

    def get_history(self):
        arrs = [np.empty(self.N) for _ in HISTORY]
        self._ck(self.lib.fivo_download_history(self.h, self.N, *[_ptr(a) for a in arrs]), "fivo_download_history")
        return dict(zip(HISTORY, arrs))

    def reset_history(self):
        self._ck(self.lib.fivo_reset_history(self.h), "fivo_reset_history")

    def set_nu_history(self, nux_prev=None, nuy_prev=None):
        """Work2D nux_prev / nuy_prev: the charge current after the previous relaxation
        (the charm second moment's d_tau nu, src2d/work2d.jl:46-47)"""
        a, b = _f64(nux_prev), _f64(nuy_prev)
        self._ck(self.lib.fivo_upload_nu_history(self.h, self.N, _ptr(a), _ptr(b)), "fivo_upload_nu_history")

    def get_nu_history(self):
        a, b = np.empty(self.N), np.empty(self.N)
        self._ck(self.lib.fivo_download_nu_history(self.h, self.N, _ptr(a), _ptr(b)), "fivo_download_nu_history")
        return dict(nux_prev=a, nuy_prev=b)

    def primitives(self):
        arrs = [np.empty(self.N) for _ in PRIMS]
        ok = np.empty(self.N, dtype=np.uint8)
        self._ck(self.lib.fivo_get_primitives(self.h, self.N, *[_ptr(a) for a in arrs], _ptr(ok)),
                 "fivo_get_primitives")
        d = dict(zip(PRIMS, arrs))
        d["ok"] = ok
        return d

    def counters(self):
        c = A.FivoCounters()
        self._ck(self.lib.fivo_get_counters(self.h, C.byref(c)), "fivo_get_counters")
        return c

    # ---- the stage
    def rhs(self, tau, bc=A.FIVO_BC_OUTFLOW, mask=None):
        dU = np.empty((self.N, self.nv))
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        self._ck(self.lib.fivo_rhs(self.h, tau, bc, _ptr(m), _ptr(dU)), "fivo_rhs")
        return dU

    def step(self, integrator, tau, dtau, max_halve=12, max_mood=2, bc=A.FIVO_BC_OUTFLOW):
        used = C.c_double(0.0)
        ok = C.c_int(0)
        self._ck(self.lib.fivo_step(self.h, integrator, tau, dtau, max_halve, max_mood, bc, C.byref(used),
                                    C.byref(ok)), "fivo_step")
        return bool(ok.value), used.value

    def update_primitives(self, tau, bc=A.FIVO_BC_OUTFLOW):
        n = C.c_int64(0)
        self._ck(self.lib.fivo_update_primitives(self.h, tau, bc, C.byref(n)), "fivo_update_primitives")
        return n.value

    def relax(self, tau, dtau):
        self._ck(self.lib.fivo_relax(self.h, tau, dtau), "fivo_relax")

    def project_shear(self):
        a, b = C.c_double(0.0), C.c_double(0.0)
        self._ck(self.lib.fivo_project_shear(self.h, C.byref(a), C.byref(b)), "fivo_project_shear")
        return a.value, b.value

    def compute_dt(self, tau, cfl=0.2, cfltau=0.05):
        dt = C.c_double(0.0)
        self._ck(self.lib.fivo_compute_dt(self.h, tau, cfl, cfltau, C.byref(dt)), "fivo_compute_dt")
        return dt.value

    def run(self, tau0, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=A.FIVO_BC_OUTFLOW,
            max_steps=2_000_000, reset_history=True):
        r = A.FivoRunResult()
        self._ck(self.lib.fivo_run(self.h, tau0, taufinal, cfl, cfltau, integrator, bc, max_steps,
                                   int(reset_history), C.byref(r)), "fivo_run")
        return r.as_dict()

    def advance(self, tau, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=A.FIVO_BC_OUTFLOW,
                max_steps=1):
        """run_sim_2d!'s loop body from tau for at most max_steps steps (a join)."""
        r = A.FivoRunResult()
        self._ck(self.lib.fivo_advance(self.h, tau, taufinal, cfl, cfltau, integrator, bc, max_steps,
                                       C.byref(r)), "fivo_advance")
        return r.as_dict()

    def run_diagnostics(self):
        """run_sim_2d!'s end-of-run interior pass (main2D.jl:532-556) on the resident
        state: (Q = sum of Dtau, maxu, minPtot)."""
        q, mu, mp = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
        self._ck(self.lib.fivo_run_diagnostics(self.h, C.byref(q), C.byref(mu), C.byref(mp)),
                 "fivo_run_diagnostics")
        return q.value, mu.value, mp.value

    def finalize_ic(self, tau0, bc=A.FIVO_BC_OUTFLOW):
        self._ck(self.lib.fivo_finalize_ic(self.h, tau0, bc), "fivo_finalize_ic")

    def set_graphs(self, mode=1):
        """fivo_ctx_set_graphs: run and advance through the lockstep launch sequences of
        this one context, replayed as CUDA graphs on the context's stream (mode 1 or
        True), launched kernel by kernel (2), or the context's own path (0 or False);
        the same bits in every mode"""
        self._ck(self.lib.fivo_ctx_set_graphs(self.h, int(mode)), "fivo_ctx_set_graphs")

    def lockstep_info(self):
        info = A.FivoLockstepInfo()
        self._ck(self.lib.fivo_ctx_lockstep_info(self.h, C.byref(info)), "fivo_ctx_lockstep_info")
        return info.as_dict()

    def set_precision(self, mode):
        """FIVO_PRECISION_FP64 (the reference's arithmetic), FIVO_PRECISION_FP32_FACES (the
        face pass of rhs_2d! in FP32, everything else FP64) or FIVO_PRECISION_FP32 (the
        face pass and the relaxation's sources in FP32; recovery, SSPRK combination,
        transport coefficients and the relaxation's implicit update FP64)"""
        self._ck(self.lib.fivo_ctx_set_precision(self.h, int(mode)), "fivo_ctx_set_precision")

    def set_face_pass(self, x_cfg, y_cfg=None):
        """Pin the kernel of the FP64 face pass (fivo_ctx_set_face_pass):
        A.FIVO_FACES_AUTO (timed choice, the default), A.FIVO_FACES_GLOBAL, or the
        index of a TMA tile shape in A.FACE_TILE_SHAPES; same bits either way."""
        y_cfg = x_cfg if y_cfg is None else y_cfg
        self._ck(self.lib.fivo_ctx_set_face_pass(self.h, int(x_cfg), int(y_cfg)), "fivo_ctx_set_face_pass")

    def face_pass(self):
        """(x, y) face-pass choice in force (-2 until the first stage has tuned it)"""
        x, y = C.c_int(0), C.c_int(0)
        self._ck(self.lib.fivo_ctx_face_pass(self.h, C.byref(x), C.byref(y)), "fivo_ctx_face_pass")
        return x.value, y.value

    def sync(self):
        self._ck(self.lib.fivo_sync(self.h), "fivo_sync")

    def glauber_ic(self, tau0, seed, *, Tpeak=0.450, ncharm=10.0, bmax=8.0, alpha_min=-20.0,
                   T_edge=None, alpha_edge=None, bc=A.FIVO_BC_OUTFLOW, fields=False):
        """The seeded MC-Glauber initial condition built on the device into this
        context's state (fivo_glauber_ic); the nucleon sampling is ic.glauber_event's
        and the edge state is ic.glauber_fields' (T_edge <= 0: on vacuum).
        Returns (T, alpha) planes when fields=True."""
        from .ic import EDGE_ALPHA, EDGE_T, SRC_WIDTH, glauber_event
        T_edge = EDGE_T if T_edge is None else T_edge
        alpha_edge = EDGE_ALPHA if alpha_edge is None else alpha_edge
        ev = glauber_event(seed, bmax)
        pts = np.ascontiguousarray(ev["participants"], dtype=np.float64)
        w = np.ascontiguousarray(ev["weights"], dtype=np.float64)
        bi = np.ascontiguousarray(ev["binary"], dtype=np.float64)
        T = np.empty(self.N) if fields else None
        a = np.empty(self.N) if fields else None
        self._ck(self.lib.fivo_glauber_ic(self.h, tau0, _ptr(pts), _ptr(w), len(w), _ptr(bi) if len(bi) else None,
                                          len(bi), SRC_WIDTH, Tpeak, ncharm, alpha_min, T_edge, alpha_edge, bc,
                                          _ptr(T), _ptr(a)),
                 "fivo_glauber_ic")
        return (T, a) if fields else None

    def clone_state_from(self, other: "GPUWork2D"):
        """Make this work object's next steps bitwise those of `other` (same model and grid)."""
        self._ck(self.lib.fivo_ctx_clone_state(self.h, other.h), "fivo_ctx_clone_state")


class GPUBatch2D:
    """Many independent events (one model, uneven grids) advanced together: one
    device context per event on its own stream, driven by `nworkers` host
    threads inside the library (fivo_batch_*). `events[k]` is event k's
    GPUWork2D (for its initial condition and readout); `run` and `advance` are
    run_sim_2d! and its loop body on every event at once."""

    def __init__(self, model: IdealDiffVisc2DModel, grids, nworkers=0, lib=None):
        self.lib = lib or A.load_library()
        self.model, self.grids = model, list(grids)
        n = len(self.grids)
        nx = (C.c_int * n)(*[g.Nx for g in self.grids])
        ny = (C.c_int * n)(*[g.Ny for g in self.grids])
        xm = (C.c_double * n)(*[g.xmax for g in self.grids])
        ym = (C.c_double * n)(*[g.ymax for g in self.grids])
        h = C.c_void_p()
        A.check(self.lib, self.lib.fivo_batch_create(C.byref(model.params), n, nx, ny, xm, ym, self.grids[0].nghost,
                                                     int(nworkers), C.byref(h)), "fivo_batch_create")
        self.h = h
        self.events = []
        for k, g in enumerate(self.grids):
            ck = C.c_void_p()
            A.check(self.lib, self.lib.fivo_batch_event(self.h, k, C.byref(ck)), "fivo_batch_event")
            self.events.append(GPUWork2D(model, g, lib=self.lib, _handle=ck))

    def __len__(self):
        return len(self.grids)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            for e in self.events:
                e.h = C.c_void_p()
            self.lib.fivo_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _results(self, res, st):
        return [dict(r.as_dict(), status=int(s)) for r, s in zip(res, st)]

    def set_lockstep(self, enable=True, graphs=True, tune=False):
        """Lockstep mode (fivo_batch_set_lockstep): every kernel of a step launched
        once over all events, optionally replayed from captured CUDA graphs, the
        schedule optionally chosen by timing the candidates on the first steps."""
        flags = (A.FIVO_LOCKSTEP_GRAPHS if graphs else 0) | (A.FIVO_LOCKSTEP_TUNE if tune else 0)
        A.check(self.lib, self.lib.fivo_batch_set_lockstep(self.h, int(bool(enable)), flags),
                "fivo_batch_set_lockstep")

    def lockstep_info(self):
        info = A.FivoLockstepInfo()
        A.check(self.lib, self.lib.fivo_batch_lockstep_info(self.h, C.byref(info)), "fivo_batch_lockstep_info")
        return info.as_dict()

    def run(self, tau0, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=A.FIVO_BC_OUTFLOW,
            max_steps=10**9, reset_history=True):
        n = len(self)
        res, st = (A.FivoRunResult * n)(), (C.c_int * n)()
        A.check(self.lib, self.lib.fivo_batch_run(self.h, tau0, taufinal, cfl, cfltau, integrator, bc, max_steps,
                                                  int(reset_history), res, st), "fivo_batch_run")
        return self._results(res, st)

    def advance(self, taus, taufinal, cfl=0.2, cfltau=0.05, integrator=A.FIVO_SSPRK2, bc=A.FIVO_BC_OUTFLOW,
                max_steps=1):
        n = len(self)
        t = (C.c_double * n)(*[float(x) for x in taus])
        res, st = (A.FivoRunResult * n)(), (C.c_int * n)()
        A.check(self.lib, self.lib.fivo_batch_advance(self.h, t, taufinal, cfl, cfltau, integrator, bc, max_steps,
                                                      res, st), "fivo_batch_advance")
        return self._results(res, st)


def set_cells(model: IdealDiffVisc2DModel, tau, T, alpha, ux, uy, *, Pi=None, pixx=None, pixy=None,
              piyy=None, nux=None, nuy=None, U=None, lib=None):
    """set_cell! (main2D.jl:142-154) for every cell at once, on the device.
    Returns (U, ok); cells whose forward map fails keep their input column."""
    lib = lib or A.load_library()
    n = len(T)
    U = np.zeros((n, model.nv)) if U is None else np.ascontiguousarray(U, dtype=np.float64)
    ok = np.zeros(n, dtype=np.uint8)
    arrs = [_f64(a) for a in (T, alpha, ux, uy, Pi, pixx, pixy, piyy, nux, nuy)]
    A.check(lib, lib.fivo_set_cells(C.byref(model.params), n, tau, *[_ptr(a) for a in arrs], _ptr(U), _ptr(ok)),
            "fivo_set_cells")
    return U, ok.astype(bool)


def eos_Pne(model_or_params, T, mu, lib=None):
    lib = lib or A.load_library()
    p = model_or_params.params if hasattr(model_or_params, "params") else model_or_params
    T, mu = _f64(T), _f64(mu)
    P, n, e = np.empty_like(T), np.empty_like(T), np.empty_like(T)
    A.check(lib, lib.fivo_eos_Pne(C.byref(p), T.size, _ptr(T), _ptr(mu), _ptr(P), _ptr(n), _ptr(e)), "fivo_eos_Pne")
    return P, n, e


def cons_to_prim(model_or_params, tau, cons, warm=None, lib=None):
    """cons_to_prim_2d! for many independent cells: cons (n, 11) = D, Sx, Sy, E,
    nux, nuy, Pi, pixx, pixy, piyy, pieta; warm (n, 4) = yT0, phi0, ux0, uy0."""
    lib = lib or A.load_library()
    p = model_or_params.params if hasattr(model_or_params, "params") else model_or_params
    cons = _f64(cons).reshape(-1, 11)
    n = cons.shape[0]
    prim = np.empty((n, 7))
    ok = np.zeros(n, dtype=np.uint8)
    reason = np.zeros(n, dtype=np.uint8)
    w = None if warm is None else _f64(warm).reshape(-1, 4)
    A.check(lib, lib.fivo_cons_to_prim(C.byref(p), n, tau, _ptr(cons), _ptr(w), _ptr(prim), _ptr(ok), _ptr(reason)),
            "fivo_cons_to_prim")
    return prim, ok.astype(bool), reason


def run_sim_2d(U, g: Grid2D, model: IdealDiffVisc2DModel, *, tau0=0.4, taufinal=13.0, CFL=0.2, CFLtau=0.05,
               integrator="ssprk2", bc="outflow", work: GPUWork2D | None = None,
               reset_history: bool | None = None, max_steps=2_000_000):
    """run_sim_2d! (main2D.jl:371-561): advance U (host array, updated in place)
    from tau0 to taufinal on the GPU. Returns the reference's result fields plus
    the work object (whose history survives for a restart-neutral join)."""
    integ = {"ssprk2": A.FIVO_SSPRK2, "ssprk3": A.FIVO_SSPRK3}[integrator]
    bcc = {"outflow": A.FIVO_BC_OUTFLOW, "periodic": A.FIVO_BC_PERIODIC}[bc]
    if reset_history is None:
        reset_history = work is None
    wk = work or GPUWork2D(model, g)
    wk.set_state(U)
    res = wk.run(tau0, taufinal, CFL, CFLtau, integ, bcc, max_steps, reset_history)
    U[...] = wk.get_state().reshape(U.shape)
    res["work"] = wk
    return res


def fields_2d(g: Grid2D, U, work: GPUWork2D, model: IdealDiffVisc2DModel):
    """fields_2d (main2D.jl:588-600): interior fields as (Nx, Ny) arrays."""
    pr = work.primitives()
    sx, sy = g.interior()
    grab = lambda v: np.asarray(v).reshape(g.Nxtot, g.Nytot)[sx, sy].copy()  # noqa: E731
    out = dict(x=g.xC[sx].copy(), y=g.yC[sy].copy(), T=np.exp(grab(pr["yT"])), mu=grab(pr["mu"]),
               alpha=grab(pr["alpha"]), n=grab(pr["n"]), e=grab(pr["e"]), P=grab(pr["P"]),
               ux=grab(pr["ux"]), uy=grab(pr["uy"]))
    Um = np.asarray(U).reshape(g.Nxtot, g.Nytot, model.nv)
    for k, name in enumerate(model.layout.names[4:], start=4):
        out[name] = Um[sx, sy, k].copy()
    return out
