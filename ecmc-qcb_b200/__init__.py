"""Python binding of libqcb.so, the B200 gauge-field hot path of ECMC-QCB.

Mirrors the reference's C++ call surface (src/gauge/GaugeField.h, src/heatbath/heatbath_mpi.h,
src/flow/gradient_flow.h, src/observables/observables_mpi.h, src/io/ildg.h) over the C ABI in
include/qcb.h.  Every call runs the CUDA kernels of libqcb.so; there is no CPU path, and loading
fails loudly when the library is missing or no GPU is visible.

Host link arrays are numpy complex128 of shape (V, 4, 3, 3): sites lexicographic with x fastest
(the ILDG payload order), then mu = x,y,z,t, then the row-major 3x3 matrix.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqcb.so")
# the same library with every field index validated on the device (QCB_CHECKED)
CHECKED_LIB_PATH = os.path.join(HERE, "libqcb_checked.so")

PREC_F64, PREC_F32 = 64, 32
STORE_18, STORE_12 = 0, 1
K_HB, K_FLOW, K_PLAQ, K_CLOVER, K_OTHER = range(5)
ILDG_SCIDAC_CHECKSUM = 1

ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "EIO", -4: "EFORMAT", -5: "ECUDA", -6: "ETIMEOUT", -7: "ERANGE"}


class QcbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None

_i4 = C.c_int * 4
_dp = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def exported_symbols():
    """Names of the C ABI functions declared in include/qcb.h, with their ctypes signatures."""
    d, i, u32, u64, sz = C.c_double, C.c_int, C.c_uint32, C.c_uint64, C.c_size_t
    pd, pi = C.POINTER(C.c_double), C.POINTER(C.c_int)
    return {
        "qcb_last_error": (C.c_char_p, []),
        "qcb_version": (C.c_char_p, []),
        "qcb_launch_count": (u64, []),
        "qcb_field_create": (i, [_i4, i, i, C.POINTER(_vp)]),
        "qcb_field_destroy": (i, [_vp]),
        "qcb_field_info": (i, [_vp, _i4, pi, pi, C.POINTER(sz)]),
        "qcb_field_stream": (_vp, [_vp]),
        "qcb_field_set_stream": (i, [_vp, _vp]),
        "qcb_field_sync": (i, [_vp]),
        "qcb_field_upload_aos": (i, [_vp, _vp]),
        "qcb_field_download_aos": (i, [_vp, _vp]),
        "qcb_field_upload_aos_device": (i, [_vp, _vp]),
        "qcb_field_download_aos_device": (i, [_vp, _vp]),
        "qcb_field_copy": (i, [_vp, _vp]),
        "qcb_cold_start": (i, [_vp]),
        "qcb_hot_start": (i, [_vp, u64]),
        "qcb_reunitarize": (i, [_vp]),
        "qcb_unitarity": (i, [_vp, pd, pd]),
        "qcb_shift": (i, [_vp, _i4]),
        "qcb_random_shift": (i, [_vp, u64, u64, i, _i4]),
        "qcb_hb_subsweep": (i, [_vp, d, i, u64, u32, i, i]),
        "qcb_hb_sweep": (i, [_vp, d, i, u64, u32]),
        "qcb_hb_link": (i, [_vp, C.c_int64, i, d, i, u64, u32, _vp]),
        "qcb_plaquette": (i, [_vp, pd]),
        "qcb_clover_qe": (i, [_vp, pd, pd]),
        "qcb_flow_create": (i, [_vp, d, i, i, C.POINTER(_vp)]),
        "qcb_flow_destroy": (i, [_vp]),
        "qcb_flow_copy": (i, [_vp, _vp]),
        "qcb_flow_rk3": (i, [_vp, i]),
        "qcb_flow_measure": (i, [_vp, _vp, i, i, _vp, _vp]),
        "qcb_flow_field": (_vp, [_vp]),
        "qcb_flow_pass": (i, [_vp, i]),
        "qcb_clover_site": (i, [_vp, C.c_int64, i, i, _vp]),
        "qcb_local_qe": (i, [_vp, C.c_int64, pd, pd]),
        "qcb_ildg_write": (i, [_vp, C.c_char_p]),
        "qcb_ildg_read": (i, [_vp, C.c_char_p]),
        "qcb_ildg_probe": (i, [C.c_char_p, _i4, pi]),
        "qcb_ildg_write_ex": (i, [_vp, C.c_char_p, i]),
        "qcb_scidac_checksum": (i, [_vp, u64, u64, C.POINTER(u32), C.POINTER(u32)]),
        "qcb_debug_oob": (i, [pi, C.POINTER(u64), C.POINTER(u64)]),
        "qcb_field_prefetch_aos": (i, [_vp, _vp]),
        "qcb_field_commit_prefetch": (i, [_vp]),
        "qcb_debug_probe_link": (i, [_vp, i, i, C.c_int64]),
        "qcb_timing_enable": (i, [_vp, i]),
        "qcb_timing_read": (i, [_vp, i, C.POINTER(C.c_long), pd]),
        "qcb_timing_reset": (i, [_vp]),
        "qcb_diag_staple": (i, [_vp, i, _vp]),
        "qcb_diag_exp_su3": (i, [_vp, i, d, i, _vp]),
        "qcb_diag_philox": (i, [C.POINTER(u32), C.POINTER(u32), i, C.POINTER(u32)]),
        "qcb_diag_fma_rate": (i, [i, pd]),
        "qcb_plaquette_noalloc": (i, [_i4, _vp, _vp, _vp]),
        "qcb_batch_create": (i, [i, C.POINTER(C.c_int), pd, C.POINTER(u64), i, i, C.POINTER(_vp)]),
        "qcb_batch_destroy": (i, [_vp]),
        "qcb_batch_info": (i, [_vp, pi, pi, pi, pi, C.POINTER(u32)]),
        "qcb_batch_stream": (_vp, [_vp]),
        "qcb_batch_hot_start": (i, [_vp]),
        "qcb_batch_cold_start": (i, [_vp]),
        "qcb_batch_sweep": (i, [_vp, i, i]),
        "qcb_batch_sync": (i, [_vp]),
        "qcb_batch_plaquette": (i, [_vp, pd]),
        "qcb_batch_upload_aos": (i, [_vp, i, _vp]),
        "qcb_batch_download_aos": (i, [_vp, i, _vp]),
        "qcb_batch_set_variant": (i, [_vp, i]),
        "qcb_batch_tune": (i, [_vp, i, i, i, pi, pd]),
        "qcb_serve_create": (i, [sz, i, i, i, i, C.POINTER(_vp)]),
        "qcb_serve_destroy": (i, [_vp]),
        "qcb_serve_now": (d, [_vp]),
        "qcb_serve_set_option": (i, [_vp, i, i]),
        "qcb_serve_submit": (i, [_vp, u64, _i4, _vp, d, i]),
        "qcb_serve_poll": (i, [_vp, C.POINTER(u64), pd, i, pi, pd]),
        "qcb_serve_wait": (i, [_vp, d]),
        "qcb_serve_stats": (i, [_vp, pd]),
    }


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libqcb.so and binds every C ABI symbol (no GPU needed to load)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"libqcb.so not built at {path}: run ecmc-qcb_b200/build.py")
        lib = C.CDLL(path)
        for name, (res, args) in exported_symbols().items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def lib() -> C.CDLL:
    return load_library()


def _check(code: int) -> None:
    if code != 0:
        raise QcbError(code, lib().qcb_last_error().decode())


def launch_count() -> int:
    return int(lib().qcb_launch_count())


def volume(L) -> int:
    return int(L[0]) * int(L[1]) * int(L[2]) * int(L[3])


class GaugeField:
    """Device-resident periodic gauge field (reference GaugeField + GeometryCB, one GPU)."""

    def __init__(self, L, prec: int = PREC_F64, store: int = STORE_18, _handle=None, _owner=None):
        self.L = tuple(int(v) for v in L)
        self.V = volume(self.L)
        self.prec, self.store = prec, store
        self._owner = _owner
        if _handle is not None:
            self.h = _handle
            self._owns = False
        else:
            h = _vp()
            _check(lib().qcb_field_create(_i4(*self.L), int(prec), int(store), C.byref(h)))
            self.h = h
            self._owns = True

    def close(self) -> None:
        if getattr(self, "_owns", False) and self.h:
            lib().qcb_field_destroy(self.h)
            self.h = None
            self._owns = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- transfers
    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        assert U.size == self.V * 36, "expected V*4*3*3 complex entries"
        _check(lib().qcb_field_upload_aos(self.h, U.ctypes.data))

    def download(self) -> np.ndarray:
        out = np.empty((self.V, 4, 3, 3), dtype=np.complex128)
        _check(lib().qcb_field_download_aos(self.h, out.ctypes.data))
        return out

    def prefetch(self, U: np.ndarray) -> None:
        """Starts the pipelined upload of U (pageable: staged before this returns); the links
        change at commit_prefetch()."""
        U = np.ascontiguousarray(U, dtype=np.complex128)
        _check(lib().qcb_field_prefetch_aos(self.h, U.ctypes.data))

    def prefetch_ptr(self, host_ptr: int) -> None:
        """Pipelined upload from a host pointer (pinned memory: asynchronous; keep the buffer
        unchanged until a synchronising call after the commit)."""
        _check(lib().qcb_field_prefetch_aos(self.h, _vp(host_ptr)))

    def commit_prefetch(self) -> None:
        _check(lib().qcb_field_commit_prefetch(self.h))

    def upload_device_ptr(self, ptr: int) -> None:
        _check(lib().qcb_field_upload_aos_device(self.h, _vp(ptr)))

    def download_device_ptr(self, ptr: int) -> None:
        _check(lib().qcb_field_download_aos_device(self.h, _vp(ptr)))

    def copy_from(self, other: "GaugeField") -> None:
        _check(lib().qcb_field_copy(self.h, other.h))

    @property
    def stream(self) -> int:
        return lib().qcb_field_stream(self.h) or 0

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().qcb_field_set_stream(self.h, _vp(stream_ptr)))

    def sync(self) -> None:
        _check(lib().qcb_field_sync(self.h))

    def device_bytes(self) -> int:
        n = C.c_size_t()
        _check(lib().qcb_field_info(self.h, _i4(), None, None, C.byref(n)))
        return n.value

    # -- starts, projections
    def cold_start(self) -> None:
        _check(lib().qcb_cold_start(self.h))

    def hot_start(self, seed: int) -> None:
        _check(lib().qcb_hot_start(self.h, int(seed)))

    def reunitarize(self) -> None:
        _check(lib().qcb_reunitarize(self.h))

    def unitarity(self):
        mx, mn = C.c_double(), C.c_double()
        _check(lib().qcb_unitarity(self.h, C.byref(mx), C.byref(mn)))
        return mx.value, mn.value

    # -- shift
    def shift(self, s) -> None:
        _check(lib().qcb_shift(self.h, _i4(*[int(v) for v in s])))

    def random_shift(self, seed: int, idx: int, max_shift: int = 0):
        o = _i4()
        _check(lib().qcb_random_shift(self.h, int(seed), int(idx), int(max_shift), o))
        return [int(v) for v in o]

    # -- heatbath
    def hb_subsweep(self, beta, n_hits, seed, sweep, parity, mu) -> None:
        _check(lib().qcb_hb_subsweep(self.h, float(beta), int(n_hits), int(seed), int(sweep), int(parity), int(mu)))

    def hb_sweep(self, beta, n_hits, seed, sweep) -> None:
        _check(lib().qcb_hb_sweep(self.h, float(beta), int(n_hits), int(seed), int(sweep)))

    def hb_link(self, site, mu, beta, n_hits, seed, sweep) -> np.ndarray:
        """n_hits hits of one link (lexicographic site index); returns the link's staple (3x3)."""
        A = np.empty((3, 3), dtype=np.complex128)
        _check(lib().qcb_hb_link(self.h, int(site), int(mu), float(beta), int(n_hits), int(seed), int(sweep),
                                 A.ctypes.data))
        return A

    # -- observables
    def plaquette(self) -> float:
        p = C.c_double()
        _check(lib().qcb_plaquette(self.h, C.byref(p)))
        return p.value

    def clover_qe(self):
        q, e = C.c_double(), C.c_double()
        _check(lib().qcb_clover_qe(self.h, C.byref(q), C.byref(e)))
        return q.value, e.value

    def clover_site(self, site: int, mu: int, nu: int) -> np.ndarray:
        """clover_site: F_mu_nu (3x3) at one lexicographic site."""
        F = np.empty((3, 3), dtype=np.complex128)
        _check(lib().qcb_clover_site(self.h, int(site), int(mu), int(nu), F.ctypes.data))
        return F

    def local_qe(self, site: int):
        """local_q_e_clover at one lexicographic site: (q, e)."""
        q, e = C.c_double(), C.c_double()
        _check(lib().qcb_local_qe(self.h, int(site), C.byref(q), C.byref(e)))
        return q.value, e.value

    def staple(self, mu: int) -> np.ndarray:
        out = np.empty((self.V, 3, 3), dtype=np.complex128)
        _check(lib().qcb_diag_staple(self.h, int(mu), out.ctypes.data))
        return out

    def debug_probe_link(self, mu: int, parity: int, h: int) -> None:
        _check(lib().qcb_debug_probe_link(self.h, int(mu), int(parity), int(h)))

    # -- ILDG
    def save_ildg(self, path: str, scidac_checksum: bool = False) -> None:
        if scidac_checksum:
            _check(lib().qcb_ildg_write_ex(self.h, os.fsencode(path), ILDG_SCIDAC_CHECKSUM))
        else:
            _check(lib().qcb_ildg_write(self.h, os.fsencode(path)))

    def read_ildg(self, path: str) -> None:
        _check(lib().qcb_ildg_read(self.h, os.fsencode(path)))

    # -- instrumentation
    def timing(self, on: bool = True) -> None:
        _check(lib().qcb_timing_enable(self.h, 1 if on else 0))

    def timing_read(self, kclass: int):
        n, ms = C.c_long(), C.c_double()
        _check(lib().qcb_timing_read(self.h, int(kclass), C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def timing_reset(self) -> None:
        _check(lib().qcb_timing_reset(self.h))


class Batch:
    """Many independent heatbath chains of uneven size and beta on one GPU (CUDA-graph sweeps)."""

    def __init__(self, Ls, betas, seeds, prec: int = PREC_F64, store: int = STORE_18):
        n = len(Ls)
        assert len(betas) == n and len(seeds) == n
        self.Ls = [tuple(int(v) for v in L) for L in Ls]
        Lflat = (C.c_int * (4 * n))(*[v for L in self.Ls for v in L])
        b = (C.c_double * n)(*[float(x) for x in betas])
        sd = (C.c_uint64 * n)(*[int(x) for x in seeds])
        h = _vp()
        _check(lib().qcb_batch_create(n, Lflat, b, sd, int(prec), int(store), C.byref(h)))
        self.h, self.n = h, n

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return lib().qcb_batch_stream(self.h) or 0

    def info(self):
        n, p, st, v = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        sw = C.c_uint32()
        _check(lib().qcb_batch_info(self.h, C.byref(n), C.byref(p), C.byref(st), C.byref(v), C.byref(sw)))
        return {"n": n.value, "prec": p.value, "store": st.value, "variant": v.value, "sweep": sw.value}

    def hot_start(self) -> None:
        _check(lib().qcb_batch_hot_start(self.h))

    def cold_start(self) -> None:
        _check(lib().qcb_batch_cold_start(self.h))

    def sweep(self, n_hits: int, n_sweeps: int = 1) -> None:
        _check(lib().qcb_batch_sweep(self.h, int(n_hits), int(n_sweeps)))

    def sync(self) -> None:
        _check(lib().qcb_batch_sync(self.h))

    def plaquette(self) -> np.ndarray:
        out = np.empty(self.n)
        _check(lib().qcb_batch_plaquette(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def upload(self, i: int, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        _check(lib().qcb_batch_upload_aos(self.h, int(i), U.ctypes.data))

    def download(self, i: int) -> np.ndarray:
        out = np.empty((volume(self.Ls[i]), 4, 3, 3), dtype=np.complex128)
        _check(lib().qcb_batch_download_aos(self.h, int(i), out.ctypes.data))
        return out

    def set_variant(self, v: int) -> None:
        _check(lib().qcb_batch_set_variant(self.h, int(v)))

    def tune(self, n_hits: int, n_trial: int = 2, allow_store_change: bool = False):
        v = C.c_int()
        ms = (C.c_double * 4)()
        _check(lib().qcb_batch_tune(self.h, int(n_hits), int(n_trial), 1 if allow_store_change else 0, C.byref(v), ms))
        return v.value, list(ms)


class Server:
    """Continuous-batching flow-measurement server (its own scheduler thread in libqcb.so)."""

    def __init__(self, budget_bytes: int, prec: int = PREC_F32, store: int = STORE_18, n_rk: int = 1,
                 max_active: int = 0):
        h = _vp()
        _check(lib().qcb_serve_create(int(budget_bytes), int(prec), int(store), int(n_rk), int(max_active),
                                      C.byref(h)))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def now(self) -> float:
        return lib().qcb_serve_now(self.h)

    def set_graphs(self, on: bool) -> None:
        """Replay the small requests' shared launches from CUDA graphs while the resident set is unchanged."""
        _check(lib().qcb_serve_set_option(self.h, 1, 1 if on else 0))

    def submit(self, rid: int, L, U: np.ndarray, eps: float, n_steps: int) -> None:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        _check(lib().qcb_serve_submit(self.h, int(rid), _i4(*[int(v) for v in L]), U.ctypes.data, float(eps),
                                      int(n_steps)))

    def poll(self, max_steps: int = 1 << 16):
        """Returns (id, tQE (n,3), (t_submit, t_admit, t_done)) or None."""
        rid = C.c_uint64()
        buf = np.empty(3 * max_steps)
        n = C.c_int()
        t = (C.c_double * 3)()
        r = lib().qcb_serve_poll(self.h, C.byref(rid), buf.ctypes.data_as(C.POINTER(C.c_double)), int(max_steps),
                                 C.byref(n), t)
        if r < 0:
            _check(r)
        if r == 0:
            return None
        return rid.value, buf[:3 * n.value].reshape(n.value, 3).copy(), tuple(t)

    def wait(self, timeout_s: float = 600.0) -> None:
        _check(lib().qcb_serve_wait(self.h, float(timeout_s)))

    def stats(self):
        o = (C.c_double * 8)()
        _check(lib().qcb_serve_stats(self.h, o))
        keys = ["submitted", "completed", "ticks", "peak_resident", "peak_bytes", "bytes_in_use", "busy_s", "queued"]
        return dict(zip(keys, list(o)))


def ildg_probe(path: str):
    L = _i4()
    p = C.c_int()
    _check(lib().qcb_ildg_probe(os.fsencode(path), L, C.byref(p)))
    return tuple(int(v) for v in L), p.value


def debug_oob():
    """(checked build?, out-of-bounds access count, first bad access) since the last call."""
    c, n, f = C.c_int(), C.c_uint64(), C.c_uint64()
    _check(lib().qcb_debug_oob(C.byref(c), C.byref(n), C.byref(f)))
    return bool(c.value), n.value, f.value


def scidac_checksum(payload, site_bytes: int):
    """SciDAC (suma, sumb) of a payload laid out as records of site_bytes bytes in rank order."""
    buf = memoryview(payload).cast("B")
    if len(buf) % site_bytes:
        raise ValueError("payload is not a whole number of site records")
    a, b = C.c_uint32(), C.c_uint32()
    arr = (C.c_ubyte * len(buf)).from_buffer_copy(buf) if buf.readonly else (C.c_ubyte * len(buf)).from_buffer(buf)
    _check(lib().qcb_scidac_checksum(arr, len(buf) // site_bytes, site_bytes, C.byref(a), C.byref(b)))
    return a.value, b.value


class GradientFlow:
    """Wilson flow state (reference GradientFlow, src/flow/gradient_flow.h:11-27)."""

    def __init__(self, field: GaugeField, eps: float = 0.02, prec: int | None = None, store: int | None = None):
        prec = field.prec if prec is None else prec
        store = field.store if store is None else store
        h = _vp()
        _check(lib().qcb_flow_create(field.h, float(eps), int(prec), int(store), C.byref(h)))
        self.h = h
        self.eps = eps
        self.field = GaugeField(field.L, prec, store, _handle=lib().qcb_flow_field(h), _owner=self)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def copy(self, field: GaugeField) -> None:
        _check(lib().qcb_flow_copy(self.h, field.h))

    def rk3_step(self, n: int = 1) -> None:
        _check(lib().qcb_flow_rk3(self.h, int(n)))

    # the reference's separate member passes (compute_force, compute_w1/2/3, replace_force_0)
    FORCE0, FORCE1, W1, W2, REPLACE_F0, W3 = range(6)

    def run_pass(self, p: int) -> None:
        _check(lib().qcb_flow_pass(self.h, int(p)))

    def measure(self, field: GaugeField, n_steps: int, n_rk: int = 1, plaquette: bool = False):
        """topo_charge_flowed: returns an (n_steps, 3) array of (t, Q, E), and plaquettes if asked."""
        out = np.empty(3 * n_steps)
        pl = np.empty(n_steps) if plaquette else None
        _check(lib().qcb_flow_measure(self.h, field.h, int(n_steps), int(n_rk), out.ctypes.data,
                                      pl.ctypes.data if pl is not None else None))
        tqe = out.reshape(n_steps, 3)
        return (tqe, pl) if plaquette else tqe


def plaquette_noalloc(L, d_links: int, d_out: int, stream: int = 0) -> None:
    """Mean plaquette of caller-owned device links (parity-split FP64 layout) into d_out[0],
    enqueued on `stream`; the library allocates nothing (see qcb_plaquette_noalloc in qcb.h)."""
    _check(lib().qcb_plaquette_noalloc(_i4(*[int(v) for v in L]), _vp(d_links), _vp(d_out), _vp(stream)))


def exp_su3(Z: np.ndarray, coeff: float, prec: int = PREC_F64) -> np.ndarray:
    z = np.ascontiguousarray(Z, dtype=np.complex128).reshape(-1, 3, 3)
    out = np.empty_like(z)
    _check(lib().qcb_diag_exp_su3(z.ctypes.data, z.shape[0], float(coeff), int(prec), out.ctypes.data))
    return out


def fma_rate(prec: int = PREC_F64) -> float:
    """Measured FMA throughput of the current device, FLOP/s (FP64 or FP32)."""
    r = C.c_double()
    _check(lib().qcb_diag_fma_rate(int(prec), C.byref(r)))
    return r.value


def philox(ctr, key, n: int = 1) -> np.ndarray:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * (4 * n))()
    _check(lib().qcb_diag_philox(c, k, int(n), out))
    return np.frombuffer(out, dtype=np.uint32).reshape(n, 4).copy()
