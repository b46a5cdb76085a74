"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle checks the CUDA product: only tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py import it.  The product
(ecmc-qcb_b200/) never does.  The restatement is pinned to the reference's own
hot-path code compiled unchanged into oracle/_ref (ref.py, tests/test_ref_pin.py)
and to analytic known answers (tests/test_oracle.py).

Fields are numpy complex128 arrays of shape (V, 4, 3, 3) in the AoS/ILDG
order: site index lexicographic with x fastest, then mu, then the row-major
3x3 matrix.  L is (Lx, Ly, Lz, Lt).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libqcb_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i4 = C.c_int * 4


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O2 -fopenmp)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "libqcb_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        l = C.CDLL(_LIB_PATH)
        u64, u32, i, d = C.c_uint64, C.c_uint32, C.c_int, C.c_double
        sig = {
            "orc_philox4x32_10": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "orc_set_threads": (None, [i]),
            "orc_get_threads": (i, []),
            "orc_exp_su3_luscher": (None, [_dp, d, _dp]),
            "orc_proj_lie_su3": (None, [_dp]),
            "orc_projection_su3": (None, [_dp]),
            "orc_cold_start": (None, [_dp, _i4]),
            "orc_hot_start": (None, [_dp, _i4, u64]),
            "orc_staple_field": (None, [_dp, _i4, i, _dp]),
            "orc_plaquette": (d, [_dp, _i4]),
            "orc_clover_qe": (None, [_dp, _i4, C.POINTER(d), C.POINTER(d)]),
            "orc_clover_qe_density": (None, [_dp, _i4, _fp, _fp]),
            "orc_flow_rk3": (None, [_dp, _i4, d, i]),
            "orc_flow_measure": (None, [_dp, _i4, d, i, i, _fp]),
            "orc_hb_subsweep": (None, [_dp, _i4, d, i, u64, u32, i, i]),
            "orc_hb_sweep": (None, [_dp, _i4, d, i, u64, u32]),
            "orc_hb_sweep_refcost": (None, [_dp, _i4, d, i, u64, u32]),
            "orc_hb_subsweep_refcost": (None, [_dp, _i4, d, i, u64, u32, i, i]),
            "orc_shift": (None, [_dp, _i4, _i4]),
            "orc_random_shift_draw": (None, [u64, u64, _i4, i, _i4]),
            "orc_reunitarize": (None, [_dp, _i4]),
            "orc_unitarity": (None, [_dp, _i4, C.POINTER(d), C.POINTER(d)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _L(L):
    return _i4(*[int(v) for v in L])


def volume(L) -> int:
    return int(L[0]) * int(L[1]) * int(L[2]) * int(L[3])


def empty_field(L) -> np.ndarray:
    return np.zeros((volume(L), 4, 3, 3), dtype=np.complex128)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [int(v) for v in o]


def exp_su3(Z: np.ndarray, coeff: float) -> np.ndarray:
    z = np.ascontiguousarray(Z, dtype=np.complex128)
    out = np.empty_like(z)
    lib().orc_exp_su3_luscher(z, float(coeff), out)
    return out


def proj_lie_su3(A: np.ndarray) -> np.ndarray:
    a = np.array(A, dtype=np.complex128, order="C")
    lib().orc_proj_lie_su3(a)
    return a


def projection_su3(U: np.ndarray) -> np.ndarray:
    a = np.array(U, dtype=np.complex128, order="C")
    lib().orc_projection_su3(a)
    return a


def cold_start(L) -> np.ndarray:
    U = empty_field(L)
    lib().orc_cold_start(U, _L(L))
    return U


def hot_start(L, seed: int) -> np.ndarray:
    U = empty_field(L)
    lib().orc_hot_start(U, _L(L), int(seed))
    return U


def staple_field(U, L, mu: int) -> np.ndarray:
    out = np.empty((volume(L), 3, 3), dtype=np.complex128)
    lib().orc_staple_field(U, _L(L), int(mu), out)
    return out


def plaquette(U, L) -> float:
    return lib().orc_plaquette(U, _L(L))


def clover_qe(U, L):
    q, e = C.c_double(), C.c_double()
    lib().orc_clover_qe(U, _L(L), C.byref(q), C.byref(e))
    return q.value, e.value


def clover_qe_density(U, L):
    V = volume(L)
    q = np.empty(V)
    e = np.empty(V)
    lib().orc_clover_qe_density(U, _L(L), q, e)
    return q, e


def flow_rk3(U, L, eps: float, n: int) -> np.ndarray:
    """Returns a flowed copy."""
    W = np.array(U, copy=True)
    lib().orc_flow_rk3(W, _L(L), float(eps), int(n))
    return W


def flow_measure(U, L, eps: float, n_steps: int, n_rk: int) -> np.ndarray:
    out = np.empty(3 * n_steps)
    lib().orc_flow_measure(U, _L(L), float(eps), int(n_steps), int(n_rk), out)
    return out.reshape(n_steps, 3)


def hb_subsweep(U, L, beta, n_hits, seed, sweep, parity, mu, refcost: bool = False) -> None:
    f = lib().orc_hb_subsweep_refcost if refcost else lib().orc_hb_subsweep
    f(U, _L(L), float(beta), int(n_hits), int(seed), int(sweep), int(parity), int(mu))


def hb_sweep(U, L, beta, n_hits, seed, sweep, refcost: bool = False) -> None:
    f = lib().orc_hb_sweep_refcost if refcost else lib().orc_hb_sweep
    f(U, _L(L), float(beta), int(n_hits), int(seed), int(sweep))


def shift(U, L, s) -> None:
    lib().orc_shift(U, _L(L), _i4(*[int(v) for v in s]))


def random_shift_draw(seed, idx, L, max_shift: int = 0):
    o = _i4()
    lib().orc_random_shift_draw(int(seed), int(idx), _L(L), int(max_shift), o)
    return [int(v) for v in o]


def reunitarize(U, L) -> None:
    lib().orc_reunitarize(U, _L(L))


def unitarity(U, L):
    mx, mn = C.c_double(), C.c_double()
    lib().orc_unitarity(U, _L(L), C.byref(mx), C.byref(mn))
    return mx.value, mn.value
