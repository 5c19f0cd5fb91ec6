"""The learned recovery guess's CPU oracle (oracle/guess_oracle.py), pinned on
the CPU before it checks the device: its backward pass against central finite
differences of its loss, its BF16 rounding against the format's definition, and
its device-rounded gradient against the float64 one."""
import sys
import pathlib

import numpy as np
import pytest

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "oracle"))
import guess_oracle as G  # noqa: E402


def _params(seed):
    rng = np.random.default_rng(seed)
    P = np.zeros(G.NPARAM)
    P[G.P_W1:G.P_B1] = (rng.uniform(-1, 1, (G.NH, G.K0)) / np.sqrt(8) * (np.arange(G.K0) < 8)).ravel()
    P[G.P_B1:G.P_W2] = rng.uniform(-0.1, 0.1, G.NH)
    P[G.P_W2:G.P_B2] = rng.uniform(-1, 1, G.NH * G.NH) / 8
    P[G.P_B2:G.P_W3] = rng.uniform(-0.1, 0.1, G.NH)
    W3 = rng.uniform(-1, 1, (G.N3, G.NH)) / 8
    W3[G.NOUT:] = 0
    P[G.P_W3:G.P_B3] = W3.ravel()
    P[G.P_B3:G.P_B3 + G.NOUT] = rng.uniform(-0.1, 0.1, G.NOUT)
    return P


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    P = _params(5)
    xn = rng.normal(size=(64, G.NIN))
    tn = rng.normal(size=(64, G.NOUT))
    g = G.grad64(P, xn, tn)
    idx = np.concatenate([rng.choice(np.arange(G.P_W1, G.P_B1).reshape(G.NH, G.K0)[:, :8].ravel(), 6),
                          rng.integers(G.P_B1, G.P_W2, 3), rng.integers(G.P_W2, G.P_B2, 6),
                          rng.integers(G.P_B2, G.P_W3, 3),
                          rng.choice(np.arange(G.P_W3, G.P_B3).reshape(G.N3, G.NH)[:3].ravel(), 6),
                          np.arange(G.P_B3, G.P_B3 + 3)])
    for p in idx:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[p] += h
        Pm[p] -= h
        fd = (G.loss64(Pp, xn, tn) - G.loss64(Pm, xn, tn)) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(g[p])), (p, fd, g[p])


def test_padding_gradients_are_zero():
    rng = np.random.default_rng(4)
    P = _params(6)
    g = G.grad64(P, rng.normal(size=(32, G.NIN)), rng.normal(size=(32, G.NOUT)))
    assert not g[G.P_W1:G.P_B1].reshape(G.NH, G.K0)[:, 8:].any()
    assert not g[G.P_W3:G.P_B3].reshape(G.N3, G.NH)[G.NOUT:].any()
    assert not g[G.P_B3 + G.NOUT:].any()


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-40, 65504.0, np.inf, -np.inf],
                 dtype=np.float32)
    r = G.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                         # tie to even
    assert r[2] == 1.0 + 2 ** -7               # above the tie: up
    assert abs(r[3] + 3.140625) < 1e-7
    assert np.isinf(r[6]) and np.isinf(r[7])
    # every result has a zero low half
    assert not (r.view(np.uint32) & 0xFFFF).any()


def test_device_rounded_gradient_tracks_float64():
    rng = np.random.default_rng(8)
    P = _params(9)
    norm = np.concatenate([np.zeros(8), np.ones(8), np.zeros(3), np.ones(3)]).astype(np.float32)
    raw = rng.normal(size=(256, 8)).astype(np.float32)
    tgt = rng.normal(size=(256, 3)).astype(np.float32)
    samples = np.hstack([raw, tgt])
    g, loss = G.grad(P, norm, samples)
    g64 = G.grad64(P, G.normalise(norm, samples).astype(np.float64), G.norm_targets(norm, samples))
    rel = np.linalg.norm(g - g64) / np.linalg.norm(g64)
    assert rel < 3e-2, rel
    assert abs(loss - G.loss64(P, G.normalise(norm, samples), G.norm_targets(norm, samples))) < 3e-2 * loss


def _cutlass_include():
    import site
    for sp in site.getsitepackages():
        p = pathlib.Path(sp) / "flashinfer" / "data" / "cutlass" / "include"
        if (p / "cute" / "arch" / "mma_sm100_desc.hpp").exists():
            return p
    return None


def test_tc05_descriptors_match_cutlass(tmp_path):
    """the tensor-core descriptor encoders (csrc/tc05.cuh) against CUTLASS's own
    bitfield definitions of the sm_100 UMMA descriptors, on the CPU"""
    import shutil
    import subprocess
    inc = _cutlass_include()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if inc is None or not pathlib.Path(nvcc).exists():
        pytest.skip("CUTLASS headers or nvcc not available")
    src = pathlib.Path(__file__).resolve().parent / "native" / "tc05_desc_check.cu"
    exe = tmp_path / "tc05_desc_check"
    subprocess.run([nvcc, "-std=c++17", "-Wno-deprecated-gpu-targets", f"-I{inc}", "-o", str(exe), str(src)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
