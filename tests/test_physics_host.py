"""The library's per-cell physics compiled for the CPU (tests/native/physics_host.cpp
includes fivohydro.jl_b200/csrc/physics.cuh as plain C++), compared bit for bit with
the oracle: the device code's arithmetic is IEEE-only and built without contraction,
so these are the same bits the GPU produces — checked here without a GPU.
"""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

import _oracle as O
import fivo2d

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "native" / "physics_host.cpp"
_D = C.POINTER(C.c_double)
_U8 = C.POINTER(C.c_uint8)


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    same = a.view(np.int64) == b.view(np.int64)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


@pytest.fixture(scope="module")
def ph(tmp_path_factory):
    so = tmp_path_factory.mktemp("physics_host") / "libphysics_host.so"
    subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                    "-shared", "-o", str(so), str(SRC)], check=True)
    lib = C.CDLL(str(so))
    for name in ("ph_exp", "ph_log", "ph_pow4"):
        getattr(lib, name).argtypes = [C.c_long, _D, _D]
    lib.ph_hypot.argtypes = [C.c_long, _D, _D, _D]
    lib.ph_besselkx.argtypes = [C.c_int, C.c_long, _D, _D]
    P = C.POINTER(fivo2d._abi.FivoParams)
    lib.ph_eos.argtypes = [P, C.c_long, _D, _D, _D, _D, _D, _D]
    lib.ph_cons_to_prim.argtypes = [P, C.c_long, C.c_double, _D, _D, _D, _U8, _U8]
    lib.ph_fast_vs_attempt.argtypes = [P, C.c_long, C.c_double, _D, _D, C.c_int]
    lib.ph_fast_vs_attempt.restype = C.c_long
    return lib


def _p(a):
    return a.ctypes.data_as(_D)


def test_scalar_math_bitwise(ph):
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-745, 709, 20000), rng.normal(0, 3, 20000), [0.0, -0.0, np.nan, np.inf]])
    for host, orc in (("ph_exp", "oracle_exp"),):
        a, b = np.empty_like(x), np.empty_like(x)
        getattr(ph, host)(x.size, _p(x), _p(a))
        b = O.vec(getattr(O.lib(), orc), x)
        assert bits_equal(a, b), host
    xp = np.abs(x[np.isfinite(x)]) * 10.0 ** rng.integers(-300, 300, np.isfinite(x).sum())
    for host, orc in (("ph_log", "oracle_log"), ("ph_pow4", "oracle_pow4")):
        a = np.empty_like(xp)
        getattr(ph, host)(xp.size, _p(xp), _p(a))
        assert bits_equal(a, O.vec(getattr(O.lib(), orc), xp)), host
    y = rng.normal(size=xp.size) * 10.0 ** rng.integers(-100, 100, xp.size)
    a = np.empty_like(xp)
    ph.ph_hypot(xp.size, _p(xp), _p(y), _p(a))
    assert bits_equal(a, O.vec(O.lib().oracle_hypot, xp, y))


@pytest.mark.parametrize("nu", [0, 1, 2, 3, 5])
def test_besselkx_bitwise(ph, nu):
    x = np.exp(np.linspace(np.log(1e-3), np.log(3e5), 4000))
    a = np.empty_like(x)
    ph.ph_besselkx(nu, x.size, _p(x), _p(a))
    assert bits_equal(a, O.besselkx(nu, x))


@pytest.mark.parametrize("eos", ["lhrg", "conformal"])
def test_eos_bitwise(ph, eos):
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS() if eos == "lhrg" else fivo2d.ConformalHQEOS())
    T, mu = np.meshgrid(np.exp(np.linspace(np.log(0.02), np.log(2.0), 120)), np.linspace(-3, 2, 50))
    T, mu = T.ravel(), mu.ravel()
    P, n, e, cs2 = (np.empty_like(T) for _ in range(4))
    ph.ph_eos(C.byref(m.params), T.size, _p(T), _p(mu), _p(P), _p(n), _p(e), _p(cs2))
    Po, no, eo = O.eos_Pne(m.params, T, mu)
    assert bits_equal(P, Po) and bits_equal(n, no) and bits_equal(e, eo)


def _viscous_states(n, seed):
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True)
    rng = np.random.default_rng(seed)
    T = rng.uniform(0.12, 0.5, n)
    alpha = rng.uniform(-8, -1, n)
    ux, uy = rng.normal(0, 0.6, n), rng.normal(0, 0.6, n)
    tau = 1.3
    U, ok = O.set_cells(m.params, tau, T, alpha, ux, uy, m.nv)
    cons = np.column_stack([U[:, 0] / tau] + [U[:, k] for k in range(1, 11)])
    # warm starts near the solution, as a previous pass leaves them
    warm = np.column_stack([np.log(T) + rng.normal(0, 0.02, n), alpha + rng.normal(0, 0.05, n),
                            ux + rng.normal(0, 0.01, n), uy + rng.normal(0, 0.01, n)])
    return m, tau, cons, warm


def test_recovery_bitwise(ph):
    m, tau, cons, warm = _viscous_states(600, 21)
    for w in (warm, None):
        prim, ok, reason = np.empty((len(cons), 7)), np.zeros(len(cons), np.uint8), np.zeros(len(cons), np.uint8)
        wp = None if w is None else np.ascontiguousarray(w)
        ph.ph_cons_to_prim(C.byref(m.params), len(cons), tau, _p(np.ascontiguousarray(cons)),
                           None if wp is None else _p(wp), _p(prim), ok.ctypes.data_as(_U8),
                           reason.ctypes.data_as(_U8))
        po, oko, ro = O.cons_to_prim(m.params, tau, cons, w)
        assert bits_equal(prim, po) and np.array_equal(ok.astype(bool), oko) and np.array_equal(reason, ro)


@pytest.mark.parametrize("budget", [6, 80])
def test_fast_recovery_equals_the_first_attempt(ph, budget):
    """recover_fast (the fast pass) returns the bits of recover_attempt for every cell it
    does not defer, with its budget and without one."""
    m, tau, cons, warm = _viscous_states(800, 33)
    bad = ph.ph_fast_vs_attempt(C.byref(m.params), len(cons), tau, _p(np.ascontiguousarray(cons)),
                                _p(np.ascontiguousarray(warm)), budget)
    assert bad == 0
