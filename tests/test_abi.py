"""The C ABI boundary, without a GPU: the library loads, exports every symbol
include/fivo2d.h declares, its structs match the ctypes mirror byte for byte,
and configuration errors come back as status codes (as the reference's
build_model_2d / reject_unwired_knobs_2d refuse them)."""
import ctypes as C
import pathlib
import re
import subprocess

import numpy as np
import pytest

import __graft_entry__ as GE
import fivo2d
from fivo2d import _abi as A

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "fivo2d.h"


@pytest.fixture(scope="module")
def lib():
    GE.build_library()
    return A.load_library()


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fivo_[A-Za-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/fivo2d.h but not exported"
    assert set(names) == set(A.SIGNATURES), "ctypes signature table out of step with the header"


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(fivo_params), '
                   'sizeof(fivo_counters), sizeof(fivo_run_result), offsetof(fivo_params, eos_kind), '
                   'offsetof(fivo_params, terms));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(A.FivoParams)
    assert int(out[1]) == C.sizeof(A.FivoCounters)
    assert int(out[2]) == C.sizeof(A.FivoRunResult)
    assert int(out[3]) == A.FivoParams.eos_kind.offset
    assert int(out[4]) == A.FivoParams.terms.offset


def test_lockstep_info_layout_matches_c(tmp_path):
    """fivo_lockstep_info, field for field (the batch's and a context's sequences)"""
    fields = ("enabled", "ncand", "chosen", "cand_order", "cand_slow", "cand_fused", "cand_ms", "steps",
              "fallbacks", "ms_step", "ms_post", "kernels")
    src = tmp_path / "li.c"
    body = " ".join(f'printf("%zu ", offsetof(fivo_lockstep_info, {f}));' for f in fields)
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   f'int main(void){{printf("%zu ", sizeof(fivo_lockstep_info)); {body} return 0;}}\n')
    exe = tmp_path / "li"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(A.FivoLockstepInfo)
    for f, off in zip(fields, out[1:]):
        assert off == getattr(A.FivoLockstepInfo, f).offset, f


def test_params_default_matches_build_model_2d(lib):
    """fivo_params_default == build_model_2d() defaults (main2D.jl:85-123)."""
    p = A.FivoParams()
    lib.fivo_params_default(C.byref(p))
    q = fivo2d.build_model_2d().params
    for name, _ in A.FivoParams._fields_:
        a, b = getattr(p, name), getattr(q, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        elif name in ("shear_kind", "bulk_kind"):
            continue   # set from enable_* by build_model_2d
        else:
            assert a == b, (name, a, b)


def test_abi_version(lib):
    assert lib.fivo_abi_version() == A.FIVO_ABI_VERSION


def test_config_refusals_are_status_codes(lib):
    """Refused knobs return FIVO_ERR_CONFIG before any device work."""
    g = fivo2d.make_grid2d(16, 16)
    base = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS()).params
    cases = []
    p = A.FivoParams.from_buffer_copy(base); p.consistent_fm = 1; p.tauN_coeff = 1.5; cases.append(p)
    p = A.FivoParams.from_buffer_copy(base); p.terms = A.FIVO_TERMS_DEFAULT | A.TERM_BIT["m2_vorticity"]; cases.append(p)
    p = A.FivoParams.from_buffer_copy(base); p.terms = A.FIVO_TERMS_DEFAULT & ~A.TERM_BIT["fm_dlnh"]; cases.append(p)
    p = A.FivoParams.from_buffer_copy(base); p.terms = A.FIVO_TERMS_DEFAULT | A.TERM_BIT["shear_vorticity"]; cases.append(p)
    p = A.FivoParams.from_buffer_copy(base); p.terms = A.FIVO_TERMS_DEFAULT & ~A.TERM_BIT["nu_gradalpha"]; cases.append(p)
    p = A.FivoParams.from_buffer_copy(base); p.primrec_maxit = 0; cases.append(p)
    for p in cases:
        h = C.c_void_p()
        st = lib.fivo_ctx_create(C.byref(p), g.Nx, g.Ny, 3, g.xmax, g.ymax, C.byref(h))
        assert st == A.FIVO_ERR_CONFIG and not h.value
        assert lib.fivo_last_error()


def test_bad_grid_is_an_argument_error(lib):
    p = fivo2d.build_model_2d().params
    h = C.c_void_p()
    assert lib.fivo_ctx_create(C.byref(p), 8, 16, 3, 10.0, 10.0, C.byref(h)) == A.FIVO_ERR_ARG
    assert lib.fivo_ctx_create(C.byref(p), 16, 16, 2, 10.0, 10.0, C.byref(h)) == A.FIVO_ERR_ARG


def test_no_device_fails_loudly(lib):
    """Without a GPU the library reports an error; nothing falls back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    g = fivo2d.make_grid2d(16, 16)
    m = fivo2d.build_model_2d()
    with pytest.raises(fivo2d.FivoError):
        from fivo2d.solver import GPUWork2D
        GPUWork2D(m, g, lib=lib)
    with pytest.raises(fivo2d.FivoError):
        from fivo2d.solver import eos_Pne
        eos_Pne(m, np.array([0.2]), np.array([0.0]), lib=lib)
