"""ctypes mirror of include/fivo2d.h and the loader for the CUDA library.

The structs here are byte-for-byte the C ABI the Julia shim (julia/FivoGPU.jl)
binds with `ccall`; Python is the host language of this repository's tests and
benchmark because no Julia toolchain is installed where they run.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

FIVO_ABI_VERSION = 2

FIVO_OK, FIVO_ERR_ARG, FIVO_ERR_CONFIG, FIVO_ERR_CUDA, FIVO_ERR_NOMEM, FIVO_ERR_DEVICE = range(6)

FIVO_EOS_CONFORMAL_HQ = 0
FIVO_EOS_LATTICE_HRG = 1
FIVO_SHEAR_ZERO, FIVO_SHEAR_QGP = 0, 1
FIVO_BULK_ZERO, FIVO_BULK_LORENTZ, FIVO_BULK_GAUSS = 0, 1, 2
FIVO_BC_OUTFLOW, FIVO_BC_PERIODIC = 0, 1
FIVO_SSPRK2, FIVO_SSPRK3 = 2, 3

# Terms register (src/terms.jl:82-104), one bit per field in field order.
TERM_NAMES = (
    "nu_gradalpha", "fm_gradT", "fm_inertial", "fm_nu_gradu", "fm_expansion", "fm_dlnh",
    "m2_nu_gradient", "m2_bg_gradu", "m2_bg_DlnT", "m2_bg_Dalpha", "m2_expansion",
    "m2_pi_sigma", "m2_PiQ_sigma", "m2_vorticity", "m2_projector", "m2_accel_nu",
    "m2_nu_gradTh", "shear_vorticity",
)
TERM_BIT = {n: 1 << k for k, n in enumerate(TERM_NAMES)}
FIVO_TERMS_DEFAULT = 0x1DFFF
FIVO_NOALLOC_MAX_CELLS = 160000
FIVO_LOCKSTEP_GRAPHS, FIVO_LOCKSTEP_TUNE = 1, 2
FIVO_LOCKSTEP_MAXCAND = 16


class FivoParams(C.Structure):
    _fields_ = [
        ("g_eff", C.c_double), ("m_hq", C.c_double), ("g_hq", C.c_double),
        ("lhrg_a", C.c_double * 4), ("lhrg_b", C.c_double * 4),
        ("lhrg_c", C.c_double), ("lhrg_d", C.c_double), ("canon_factor", C.c_double),
        ("kappa_coeff", C.c_double), ("tauN_coeff", C.c_double), ("deltaN_factor", C.c_double),
        ("nu_clip_factor", C.c_double), ("vacuum_n_lo", C.c_double), ("vacuum_n_hi", C.c_double),
        ("eta_over_s", C.c_double), ("tauShear_coeff", C.c_double),
        ("deltaShear_factor", C.c_double), ("taupi_pi_factor", C.c_double),
        ("lambda_pi_Pi_factor", C.c_double), ("pi_clip_factor", C.c_double),
        ("zeta_over_s", C.c_double), ("tauPi_coeff", C.c_double), ("bulk_T0", C.c_double),
        ("bulk_width", C.c_double), ("deltaPi_factor", C.c_double),
        ("lambda_Pi_pi_factor", C.c_double), ("Pi_clip_factor", C.c_double),
        ("r_domain", C.c_double), ("T_vac_cut", C.c_double), ("E_vac_cut", C.c_double),
        ("primrec_tol", C.c_double), ("transport_mass", C.c_double),
        ("eos_kind", C.c_int32), ("hq_times_fmGeV3", C.c_int32), ("with_charge", C.c_int32),
        ("enable_diff", C.c_int32), ("enable_shear", C.c_int32), ("enable_bulk", C.c_int32),
        ("shear_kind", C.c_int32), ("bulk_kind", C.c_int32),
        ("advect_nu", C.c_int32), ("relax_advect_nu", C.c_int32),
        ("advect_pi", C.c_int32), ("relax_advect_pi", C.c_int32),
        ("advect_Pi", C.c_int32), ("relax_advect_Pi", C.c_int32),
        ("vacuum_ramp_relax", C.c_int32),
        ("shear_projected_deriv", C.c_int32), ("diff_projected_deriv", C.c_int32),
        ("shear_constraint_project", C.c_int32),
        ("consistent_fm", C.c_int32), ("consistent_m2", C.c_int32),
        ("primrec_maxit", C.c_int32), ("terms", C.c_uint32),
        ("relax_advect_m2", C.c_int32), ("reserved0", C.c_int32),
    ]


class FivoCounters(C.Structure):
    _fields_ = [
        ("nprimfail", C.c_int64), ("nvacuum", C.c_int64), ("primfail_index", C.c_int64),
        ("primfail_reason", C.c_int32), ("pad0", C.c_int32), ("primfail_resnorm", C.c_double),
        ("amax", C.c_double), ("nmood", C.c_int64), ("nhalve", C.c_int64),
    ]


class FivoRunResult(C.Structure):
    _fields_ = [
        ("ok", C.c_int32), ("pad0", C.c_int32), ("tau", C.c_double), ("nsteps", C.c_int64),
        ("nprimfail", C.c_int64), ("nvacuum", C.c_int64), ("max_shear_res", C.c_double),
        ("maxu", C.c_double), ("dQ", C.c_double), ("Q0", C.c_double), ("Q1", C.c_double),
        ("minPtot", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("pad")}


class FivoLockstepInfo(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32), ("flags", C.c_int32), ("ncand", C.c_int32), ("chosen", C.c_int32),
        ("cand_order", C.c_int32 * FIVO_LOCKSTEP_MAXCAND), ("cand_slow", C.c_int32 * FIVO_LOCKSTEP_MAXCAND),
        ("cand_fused", C.c_int32 * FIVO_LOCKSTEP_MAXCAND),
        ("cand_ms", C.c_double * FIVO_LOCKSTEP_MAXCAND), ("steps", C.c_int64), ("fallbacks", C.c_int64),
        ("ms_step", C.c_double), ("ms_post", C.c_double), ("kernels", C.c_int64),
    ]

    def as_dict(self):
        n = self.ncand
        return {"enabled": bool(self.enabled), "graphs": bool(self.flags & FIVO_LOCKSTEP_GRAPHS),
                "tune": bool(self.flags & FIVO_LOCKSTEP_TUNE), "chosen": self.chosen,
                "candidates": [{"order": ("batch", "largest_first")[self.cand_order[i]],
                                "slow_blocks_per_sm": self.cand_slow[i], "faces_one_launch": bool(self.cand_fused[i]),
                                "best_step_ms": self.cand_ms[i]}
                               for i in range(n)],
                "steps": self.steps, "fallbacks": self.fallbacks, "ms_step": self.ms_step,
                "ms_post": self.ms_post, "kernels": self.kernels}


FIVO_KCLASS_N = 8
KERNEL_CLASSES = ("prim_fast", "prim_slow", "faces", "update", "adm_slow", "relax", "other", "unused")
(FIVO_KCLASS_PRIM_FAST, FIVO_KCLASS_PRIM_SLOW, FIVO_KCLASS_FACES, FIVO_KCLASS_UPDATE, FIVO_KCLASS_ADM_SLOW,
 FIVO_KCLASS_RELAX, FIVO_KCLASS_OTHER) = range(7)


FIVO_GUESS_NPARAM, FIVO_GUESS_NNORM, FIVO_GUESS_NSAMP = 6288, 22, 11
FIVO_PRECISION_FP64, FIVO_PRECISION_FP32_FACES, FIVO_PRECISION_FP32 = 0, 1, 2
FIVO_FACES_AUTO, FIVO_FACES_GLOBAL = -2, -1
FIVO_GUESS_EVERY_CELL, FIVO_GUESS_DEFERRED = 0, 1
FACE_TILE_SHAPES = ((4, 32), (2, 64), (8, 16), (8, 32))


class FivoNewtonStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("it_fast", "n_fast", "it_learn", "n_learn", "ok_learn", "it_fb", "n_fb",
                                          "deferred")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class FivoCFParams(C.Structure):
    _fields_ = [("T_fo", C.c_double), ("m", C.c_double), ("pt_lo", C.c_double), ("pt_hi", C.c_double),
                ("eta_max", C.c_double), ("f_yield", C.c_double), ("n_eta", C.c_int32), ("n_pt", C.c_int32),
                ("n_phi", C.c_int32), ("pad", C.c_int32)]


class FivoKernelTimes(C.Structure):
    _fields_ = [("launches", C.c_int64 * FIVO_KCLASS_N), ("ms", C.c_double * FIVO_KCLASS_N),
                ("units", C.c_int64 * FIVO_KCLASS_N), ("total_launches", C.c_int64)]

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR.parent / "csrc" / "libfivo2d.so"

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U8 = C.POINTER(C.c_uint8)
_I64 = C.c_int64

# name -> (restype, argtypes), exactly the declarations of include/fivo2d.h
SIGNATURES = {
    "fivo_abi_version": (C.c_int, []),
    "fivo_last_error": (C.c_char_p, []),
    "fivo_params_default": (None, [C.POINTER(FivoParams)]),
    "fivo_ctx_create": (C.c_int, [C.POINTER(FivoParams), C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.c_double, C.POINTER(C.c_void_p)]),
    "fivo_ctx_destroy": (C.c_int, [C.c_void_p]),
    "fivo_ctx_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64), _D]),
    "fivo_ctx_clone_state": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fivo_glauber_ic": (C.c_int, [C.c_void_p, C.c_double, _D, _D, C.c_int64, _D, C.c_int64, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _D, _D]),
    "fivo_batch_create": (C.c_int, [C.POINTER(FivoParams), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, _D,
                                    C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "fivo_batch_destroy": (C.c_int, [C.c_void_p]),
    "fivo_batch_event": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "fivo_batch_run": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                 C.c_int64, C.c_int, C.POINTER(FivoRunResult), C.POINTER(C.c_int)]),
    "fivo_batch_advance": (C.c_int, [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_int64, C.POINTER(FivoRunResult), C.POINTER(C.c_int)]),
    "fivo_batch_set_lockstep": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "fivo_batch_lockstep_info": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fivo_ctx_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "fivo_ctx_lockstep_info": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fivo_upload_state": (C.c_int, [C.c_void_p, _D, C.c_int, _I64]),
    "fivo_download_state": (C.c_int, [C.c_void_p, _D, C.c_int, _I64]),
    "fivo_upload_history": (C.c_int, [C.c_void_p, _I64] + [_D] * 8),
    "fivo_download_history": (C.c_int, [C.c_void_p, _I64] + [_D] * 8),
    "fivo_upload_nu_history": (C.c_int, [C.c_void_p, _I64, _D, _D]),
    "fivo_ctx_set_guess_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "fivo_download_nu_history": (C.c_int, [C.c_void_p, _I64, _D, _D]),
    "fivo_reset_history": (C.c_int, [C.c_void_p]),
    "fivo_get_primitives": (C.c_int, [C.c_void_p, _I64] + [_D] * 9 + [_U8]),
    "fivo_get_counters": (C.c_int, [C.c_void_p, C.POINTER(FivoCounters)]),
    "fivo_rhs": (C.c_int, [C.c_void_p, C.c_double, C.c_int, _U8, _D]),
    "fivo_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                            _D, C.POINTER(C.c_int)]),
    "fivo_update_primitives": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_int64)]),
    "fivo_relax": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "fivo_project_shear": (C.c_int, [C.c_void_p, _D, _D]),
    "fivo_compute_dt": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, _D]),
    "fivo_run": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                           C.c_int, _I64, C.c_int, C.POINTER(FivoRunResult)]),
    "fivo_advance": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                               C.c_int, _I64, C.POINTER(FivoRunResult)]),
    "fivo_run_diagnostics": (C.c_int, [C.c_void_p, _D, _D, _D]),
    "fivo_finalize_ic": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "fivo_set_cells": (C.c_int, [C.POINTER(FivoParams), _I64, C.c_double] + [_D] * 10 + [_D, _U8]),
    "fivo_eos_Pne": (C.c_int, [C.POINTER(FivoParams), _I64, _D, _D, _D, _D, _D]),
    "fivo_cons_to_prim": (C.c_int, [C.POINTER(FivoParams), _I64, C.c_double, _D, _D, _D, _U8, _U8]),
    "fivo_sync": (C.c_int, [C.c_void_p]),
    "fivo_rhs_noalloc": (C.c_int, [C.POINTER(FivoParams), C.c_int, C.c_int, C.c_double, C.c_double,
                                   C.c_double, C.c_int, C.c_void_p, C.c_void_p, _D, C.POINTER(FivoCounters),
                                   C.c_void_p]),
    "fivo_ctx_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fivo_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "fivo_profile_read": (C.c_int, [C.c_void_p, C.POINTER(FivoKernelTimes), C.c_int]),
    "fivo_guess_create": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p)]),
    "fivo_guess_destroy": (C.c_int, [C.c_void_p]),
    "fivo_guess_set_params": (C.c_int, [C.c_void_p, _F, _F]),
    "fivo_guess_get_params": (C.c_int, [C.c_void_p, _F, _F]),
    "fivo_guess_reserve": (C.c_int, [C.c_void_p, _I64]),
    "fivo_guess_set_samples": (C.c_int, [C.c_void_p, _F, _I64]),
    "fivo_guess_get_samples": (C.c_int, [C.c_void_p, _F, _I64]),
    "fivo_guess_nsamples": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "fivo_guess_harvest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int]),
    "fivo_guess_fit_norm": (C.c_int, [C.c_void_p]),
    "fivo_guess_train": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_uint64, _D]),
    "fivo_guess_grad": (C.c_int, [C.c_void_p, _F, _I64, _F, _D]),
    "fivo_guess_forward": (C.c_int, [C.c_void_p, _F, _I64, _F]),
    "fivo_ctx_set_guess": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fivo_newton_stats_read": (C.c_int, [C.c_void_p, C.POINTER(FivoNewtonStats), C.c_int]),
    "fivo_ctx_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "fivo_ctx_set_face_pass": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "fivo_ctx_face_pass": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fivo_cf_params_default": (None, [C.POINTER(FivoCFParams)]),
    "fivo_fo_create": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_void_p)]),
    "fivo_fo_destroy": (C.c_int, [C.c_void_p]),
    "fivo_fo_reset": (C.c_int, [C.c_void_p]),
    "fivo_fo_record": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "fivo_fo_surface": (C.c_int, [C.c_void_p, _D, _D, _D, C.POINTER(C.c_int64)]),
    "fivo_fo_set_surface": (C.c_int, [C.c_void_p, _D, _D, _D]),
    "fivo_cooper_frye": (C.c_int, [C.c_void_p, C.POINTER(FivoCFParams), _D]),
}

_LIB = None


class FivoError(RuntimeError):
    """A C-ABI call returned a non-zero status (see fivo_last_error)."""


def load_library(path: str | os.PathLike | None = None):
    """Load libfivo2d.so (the CUDA build). Raises if it is missing: there is no
    CPU fallback for the stage."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise FivoError(f"libfivo2d.so not built at {p}; run __graft_entry__.build()")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if lib.fivo_abi_version() != FIVO_ABI_VERSION:
        raise FivoError("libfivo2d ABI version mismatch")
    if path is None:
        _LIB = lib
    return lib


def check(lib, status: int, what: str = ""):
    if status != FIVO_OK:
        msg = lib.fivo_last_error()
        raise FivoError(f"{what}: status {status}: {msg.decode() if msg else ''}")
