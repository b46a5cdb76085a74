"""ctypes binding of the reference oracle, oracle/_ref/libqcb_ref.so (test infrastructure only).

That library is the reference's own hot-path code (ECMC-QCB src/geometry, src/gauge, src/su3,
src/heatbath, src/flow, src/observables, src/mpi), compiled unchanged by `make -C oracle ref`
against the project-written stand-ins in oracle/refshim/ (a small Eigen-API matrix library, a
one-rank mpi.h and a Philox replay engine in place of std::mt19937_64).  It pins the restated
oracle and the CUDA path to what the reference itself computes.  Only tests/, the fixture script
in tests/golden/ and bench.py's CPU legs may load it; the product never does.

Building it needs the reference source tree (REF, by default the read-only mount the reference is
kept in); the built library itself travels with the repository's other built files.  `available()`
says whether it is present.

Fields are numpy complex128 arrays of shape (V, 4, 3, 3) in the AoS/ILDG order (sites x fastest,
then mu, then the row-major 3x3 matrix) on a periodic L^4 lattice (the reference is hypercubic).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libqcb_ref.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(ref_src: str | None = None) -> bool:
    """Compiles _ref/libqcb_ref.so when the reference tree exists; returns whether the library exists."""
    src = ref_src or os.environ.get("QCB_REF_SRC", "/root/reference/src")
    if os.path.isdir(src):
        subprocess.run(["make", "-C", _HERE, "ref", f"REF={src}", "-j8"], check=True, stdout=subprocess.DEVNULL)
    return os.path.exists(LIB_PATH)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built (make -C oracle ref)")
        l = C.CDLL(LIB_PATH)
        vp, u64, u32, i, d, lg = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_double, C.c_long
        sig = {
            "qref_create": (vp, [i]),
            "qref_destroy": (None, [vp]),
            "qref_set_threads": (None, [i]),
            "qref_set_aos": (None, [vp, _dp]),
            "qref_get_aos": (None, [vp, _dp]),
            "qref_staple_field": (None, [vp, i, _dp]),
            "qref_plaquette": (d, [vp]),
            "qref_clover_qe": (None, [vp, C.POINTER(d), C.POINTER(d)]),
            "qref_clover_density": (None, [vp, _fp, _fp]),
            "qref_clover_site": (None, [vp, lg, i, i, _dp]),
            "qref_flow_rk3": (None, [vp, d, i]),
            "qref_flow_passes": (None, [vp, d, C.POINTER(C.c_int), i]),
            "qref_flow_measure": (None, [vp, d, i, i, _fp]),
            "qref_hb_subsweep": (None, [vp, d, i, u64, u32, i, i]),
            "qref_hb_sweep": (None, [vp, d, i, u64, u32]),
            "qref_hb_link": (None, [vp, lg, i, d, i, u64, u32, _dp]),
            "qref_projection": (None, [vp]),
            "qref_shift": (None, [vp, C.c_int * 4]),
            "qref_ildg_write": (i, [vp, C.c_char_p, C.c_char_p]),
            "qref_ildg_read": (None, [vp, C.c_char_p, C.c_char_p]),
            "qref_exp_su3_luscher": (None, [_dp, d, _dp]),
            "qref_proj_lie_su3": (None, [_dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def set_threads(n: int) -> None:
    lib().qref_set_threads(int(n))


class RefLattice:
    """One periodic L^4 lattice held in the reference's own GaugeField / GeometryCB layout."""

    def __init__(self, L: int, U: np.ndarray | None = None):
        self.L = int(L)
        self.V = self.L ** 4
        self._h = lib().qref_create(self.L)
        if not self._h:
            raise ValueError(f"reference lattice needs an even L >= 2, got {L}")
        if U is not None:
            self.set(U)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.qref_destroy(h)
            self._h = None

    def set(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.complex128).reshape(self.V, 4, 3, 3)
        lib().qref_set_aos(self._h, U)

    def get(self) -> np.ndarray:
        U = np.empty((self.V, 4, 3, 3), dtype=np.complex128)
        lib().qref_get_aos(self._h, U)
        return U

    def staple_field(self, mu: int) -> np.ndarray:
        out = np.empty((self.V, 3, 3), dtype=np.complex128)
        lib().qref_staple_field(self._h, int(mu), out)
        return out

    def plaquette(self) -> float:
        return float(lib().qref_plaquette(self._h))

    def clover_qe(self) -> tuple[float, float]:
        Q, E = C.c_double(), C.c_double()
        lib().qref_clover_qe(self._h, C.byref(Q), C.byref(E))
        return Q.value, E.value

    def clover_density(self) -> tuple[np.ndarray, np.ndarray]:
        q = np.empty(self.V)
        e = np.empty(self.V)
        lib().qref_clover_density(self._h, q, e)
        return q, e

    def clover_site(self, lex: int, mu: int, nu: int) -> np.ndarray:
        out = np.empty((3, 3), dtype=np.complex128)
        lib().qref_clover_site(self._h, int(lex), int(mu), int(nu), out)
        return out

    def flow_rk3(self, eps: float, n: int = 1) -> None:
        lib().qref_flow_rk3(self._h, float(eps), int(n))

    def flow_passes(self, eps: float, seq) -> None:
        """GradientFlow's member passes in order (0/1 compute_force(0/1), 2/3/5 compute_w1/2/3,
        4 replace_force_0); the lattice becomes the flowed field_c."""
        arr = (C.c_int * len(seq))(*[int(v) for v in seq])
        lib().qref_flow_passes(self._h, float(eps), arr, len(seq))

    def flow_measure(self, eps: float, n_steps: int, n_rk: int) -> np.ndarray:
        out = np.empty(3 * n_steps)
        lib().qref_flow_measure(self._h, float(eps), int(n_steps), int(n_rk), out)
        return out.reshape(n_steps, 3)

    def hb_subsweep(self, beta: float, n_hits: int, seed: int, sweep: int, parity: int, mu: int) -> None:
        lib().qref_hb_subsweep(self._h, float(beta), int(n_hits), int(seed), int(sweep), int(parity), int(mu))

    def hb_sweep(self, beta: float, n_hits: int, seed: int, sweep: int) -> None:
        lib().qref_hb_sweep(self._h, float(beta), int(n_hits), int(seed), int(sweep))

    def hb_link(self, lex: int, mu: int, beta: float, n_hits: int, seed: int, sweep: int) -> np.ndarray:
        A = np.empty((3, 3), dtype=np.complex128)
        lib().qref_hb_link(self._h, int(lex), int(mu), float(beta), int(n_hits), int(seed), int(sweep), A)
        return A

    def projection(self) -> None:
        lib().qref_projection(self._h)

    def shift(self, s) -> None:
        lib().qref_shift(self._h, (C.c_int * 4)(*[int(v) for v in s]))

    def ildg_write(self, directory: str, name: str) -> str:
        """save_ildg_clime: writes directory/name/name and returns that path."""
        if lib().qref_ildg_write(self._h, directory.encode(), name.encode()) != 0:
            raise OSError(f"cannot create {directory}/{name}")
        return os.path.join(directory, name, name)

    def ildg_read(self, directory: str, name: str) -> None:
        """read_ildg_clime of directory/name/name (the reference aborts the process on a bad file)."""
        lib().qref_ildg_read(self._h, directory.encode(), name.encode())


def exp_su3_luscher(Z: np.ndarray, coeff: float) -> np.ndarray:
    Z = np.ascontiguousarray(Z, dtype=np.complex128)
    out = np.empty((3, 3), dtype=np.complex128)
    lib().qref_exp_su3_luscher(Z, float(coeff), out)
    return out


def proj_lie_su3(A: np.ndarray) -> np.ndarray:
    A = np.array(A, dtype=np.complex128, order="C", copy=True)
    lib().qref_proj_lie_su3(A)
    return A
