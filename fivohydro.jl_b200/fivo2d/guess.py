"""The learned starting guess of the primitive recovery (fivo_guess_* in
include/fivo2d.h): an MLP 8 -> 64 -> 64 -> 3 (GELU; BF16 weights, FP32
accumulation on the tensor cores) from a cell's normalised conserved and
dissipative components to (log T - log(E)/4, u^x, u^y), trained on the GPU on
(features, primitives) pairs harvested from the solver's own runs.

A GPUWork2D with a guess attached (`attach`) starts each cell's Newton from it;
a cell whose residual is above 1e-10 after 3 updates falls back to the plain
warm-started recovery. The reference has no counterpart: its Newton starts from
the previous step's primitives or a closed-form seed (src2d/primrec2d.jl:300-347,
465-486).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A

NPARAM, NNORM, NSAMP = A.FIVO_GUESS_NPARAM, A.FIVO_GUESS_NNORM, A.FIVO_GUESS_NSAMP


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.size != int(np.prod(shape)):
        raise ValueError(f"expected {shape} floats, got {a.size}")
    return a


class RecoveryGuess:
    """A device-resident guess network (fivo_guess)."""

    def __init__(self, work=None, seed: int = 1, lib=None):
        self.lib = lib or (work.lib if work is not None else A.load_library())
        h = C.c_void_p()
        A.check(self.lib, self.lib.fivo_guess_create(work.h if work is not None else None, seed, C.byref(h)),
                "fivo_guess_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.fivo_guess_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st, what):
        A.check(self.lib, st, what)

    # ---- parameters
    def get_params(self):
        P = np.empty(NPARAM, dtype=np.float32)
        nm = np.empty(NNORM, dtype=np.float32)
        self._ck(self.lib.fivo_guess_get_params(self.h, _fp(P), _fp(nm)), "fivo_guess_get_params")
        return P, nm

    def set_params(self, params=None, norm=None):
        P = None if params is None else _f32(params, (NPARAM,))
        nm = None if norm is None else _f32(norm, (NNORM,))
        self._ck(self.lib.fivo_guess_set_params(self.h, _fp(P), _fp(nm)), "fivo_guess_set_params")

    # ---- samples
    def reserve(self, capacity: int):
        self._ck(self.lib.fivo_guess_reserve(self.h, int(capacity)), "fivo_guess_reserve")

    def nsamples(self) -> int:
        n = C.c_int64()
        self._ck(self.lib.fivo_guess_nsamples(self.h, C.byref(n)), "fivo_guess_nsamples")
        return int(n.value)

    def set_samples(self, samples):
        s = _f32(samples)
        if s.size % NSAMP:
            raise ValueError("samples must hold 11 floats each")
        self._ck(self.lib.fivo_guess_set_samples(self.h, _fp(s), s.size // NSAMP), "fivo_guess_set_samples")

    def get_samples(self, n: int | None = None):
        n = self.nsamples() if n is None else n
        s = np.empty((n, NSAMP), dtype=np.float32)
        self._ck(self.lib.fivo_guess_get_samples(self.h, _fp(s), n), "fivo_guess_get_samples")
        return s

    def harvest(self, work, tau: float, stride: int = 1, phase: int = 0):
        """append (features, targets) of work's interior cells recovered at its last
        primitive pass"""
        self._ck(self.lib.fivo_guess_harvest(work.h, self.h, tau, stride, phase), "fivo_guess_harvest")

    def fit_norm(self):
        self._ck(self.lib.fivo_guess_fit_norm(self.h), "fivo_guess_fit_norm")

    # ---- training and evaluation
    def train(self, steps: int, ctas_per_step: int = 148, lr: float = 1e-3, seed: int = 7):
        """Adam steps on the stored samples; returns (loss of the first step, of the last)"""
        out = np.zeros(2)
        self._ck(self.lib.fivo_guess_train(self.h, steps, ctas_per_step, lr, seed, out.ctypes.data_as(A._D)),
                 "fivo_guess_train")
        return float(out[0]), float(out[1])

    def grad(self, samples):
        """(gradient over NPARAM, loss) of the mean-squared error over the samples
        (a multiple of 128, taken in order)"""
        s = _f32(samples)
        g = np.empty(NPARAM, dtype=np.float32)
        loss = C.c_double()
        self._ck(self.lib.fivo_guess_grad(self.h, _fp(s), s.size // NSAMP, _fp(g), C.byref(loss)),
                 "fivo_guess_grad")
        return g, float(loss.value)

    def forward(self, raw):
        """normalised outputs (n, 3) for raw features (n, 8)"""
        r = _f32(raw)
        n = r.size // 8
        out = np.empty((n, 3), dtype=np.float32)
        self._ck(self.lib.fivo_guess_forward(self.h, _fp(r), n, _fp(out)), "fivo_guess_forward")
        return out

    # ---- use in a solver
    def attach(self, work, mode=A.FIVO_GUESS_EVERY_CELL):
        """use the network in `work`'s recovery: for every cell (FIVO_GUESS_EVERY_CELL, the
        warm start as the fallback) or for the cells the warm start leaves
        (FIVO_GUESS_DEFERRED)"""
        self._ck(self.lib.fivo_ctx_set_guess(work.h, self.h), "fivo_ctx_set_guess")
        self._ck(self.lib.fivo_ctx_set_guess_mode(work.h, int(mode)), "fivo_ctx_set_guess_mode")

    @staticmethod
    def detach(work):
        A.check(work.lib, work.lib.fivo_ctx_set_guess(work.h, None), "fivo_ctx_set_guess")


def newton_stats(work, reset: bool = False) -> dict:
    """Newton statistics of a GPUWork2D (fivo_newton_stats_read)"""
    s = A.FivoNewtonStats()
    A.check(work.lib, work.lib.fivo_newton_stats_read(work.h, C.byref(s), int(reset)), "fivo_newton_stats_read")
    return s.as_dict()
