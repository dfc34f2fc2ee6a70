"""ctypes binding of libnkgpu.so (include/nkgpu.h).

This plays the role of the Cython declarations a NetworKit build would use
(``cdef extern from "nkgpu.h"``; the compiled form of those is
``_nkgpu.pxd`` / ``_cypagerank.pyx``). The library is loaded from the
package's ``_lib`` directory; if it is missing, or was built for another ABI
version, loading fails loudly - there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libnkgpu.so")

NKG_OK = 0
NKG_ERR_INVALID_ARG = -1
NKG_ERR_CUDA = -2
NKG_ERR_OOM = -3
NKG_ERR_CANCELLED = -4
NKG_ERR_TIMEOUT = -5
NKG_ERR_NOT_RUN = -6
NKG_ERR_NO_DEVICE = -7

NKG_PREC_FP64 = 0
NKG_PREC_FP32_REFINE = 1
NKG_PREC_FP32 = 2

UINT64_MAX = 2**64 - 1
NKG_DEVICE_PTRS = 1
# include/nkgpu.h NKG_ABI_VERSION this binding's structures follow.
ABI_VERSION = 2


class PRParams(C.Structure):
    _fields_ = [
        ("damp", C.c_double),
        ("tol", C.c_double),
        ("norm", C.c_int32),
        ("normalized", C.c_int32),
        ("distribute_sinks", C.c_int32),
        ("precision", C.c_int32),
        ("max_iterations", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64),
        ("residual", C.c_double),
        ("sink_mass", C.c_double),
        ("ms_total", C.c_double),
        ("ms_iterations", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("fp64_sweeps", C.c_uint64),
        ("fp32_sweeps", C.c_uint64),
        ("bytes_per_sweep_fp64", C.c_uint64),
        ("bytes_per_sweep_fp32", C.c_uint64),
        ("residual_trace", C.POINTER(C.c_double)),
        ("trace_capacity", C.c_uint64),
        ("trace_length", C.c_uint64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "residual_trace"}

    @classmethod
    def with_trace(cls, capacity: int):
        """Stats whose residual trace goes to a new float64 array of
        `capacity` entries (returned beside it)."""
        st = cls()
        buf = np.zeros(max(int(capacity), 0), np.float64)
        if capacity > 0:
            st.residual_trace = buf.ctypes.data_as(C.POINTER(C.c_double))
            st.trace_capacity = int(capacity)
        return st, buf


class GraphInfo(C.Structure):
    _fields_ = [
        ("z", C.c_uint64),
        ("n", C.c_uint64),
        ("arcs", C.c_uint64),
        ("sinks", C.c_uint64),
        ("slots", C.c_uint64),
        ("split_rows", C.c_uint64),
        ("weighted", C.c_int32),
        ("directed", C.c_int32),
        ("device", C.c_int32),
        ("row_order", C.c_int32),
        ("ms_create", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class GraphOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("sweep_shape", C.c_int32), ("arc_order", C.c_int32),
                ("row_order", C.c_int32), ("hot_tier_kb", C.c_int32)]

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        if "hot_tier_kb" not in kw and len(a) < 5:
            self.hot_tier_kb = -1


class BatchTuning(C.Structure):
    _fields_ = [("cluster", C.c_uint32), ("threads", C.c_uint32), ("split", C.c_uint32),
                ("variant", C.c_uint32), ("ms", C.c_double)]

    def as_dict(self):
        return {"cluster": self.cluster, "threads": self.threads, "split": self.split,
                "variant": self.variant, "ms": self.ms}


class LocalStats(C.Structure):
    _fields_ = [("pushes", C.c_uint64), ("arc_visits", C.c_uint64), ("support", C.c_uint64),
                ("slots", C.c_uint64), ("table_entries", C.c_uint64), ("reruns", C.c_uint64),
                ("ms_push", C.c_double), ("ms_sweep", C.c_double), ("ms_total", C.c_double),
                ("kernel_launches", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


NKG_LOCAL_NIBBLE = 2

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_f64p = C.POINTER(C.c_double)
_vp = C.c_void_p

# name -> (restype, argtypes); the exported surface of include/nkgpu.h
SIGNATURES = {
    "nkg_abi_version": (C.c_int, []),
    "nkg_last_error": (C.c_char_p, []),
    "nkg_graph_create": (C.c_int, [C.POINTER(_vp), C.c_uint64, C.c_uint64, _u64p, _u32p, _f64p,
                                   _f64p, _u8p, C.c_int]),
    "nkg_graph_create_ex": (C.c_int, [C.POINTER(_vp), C.c_uint64, C.c_uint64, _u64p, _u32p,
                                      _f64p, _f64p, _u8p, C.c_int, C.POINTER(GraphOptions)]),
    "nkg_graph_create_from_edges": (C.c_int, [C.POINTER(_vp), C.c_uint64, C.c_uint64, _vp, _vp,
                                              _vp, _vp, C.c_int, C.c_int,
                                              C.POINTER(GraphOptions)]),
    "nkg_graph_destroy": (None, [_vp]),
    "nkg_graph_get_info": (C.c_int, [_vp, C.POINTER(GraphInfo)]),
    "nkg_pagerank_run": (C.c_int, [_vp, C.POINTER(PRParams), _f64p, _u64p, _f64p,
                                   C.POINTER(Stats)]),
    "nkg_pagerank_run_device": (C.c_int, [_vp, C.POINTER(PRParams), _vp, _u64p, _f64p,
                                          C.POINTER(Stats)]),
    "nkg_pagerank_run_teleport": (C.c_int, [_vp, C.POINTER(PRParams), _f64p, _f64p, _u64p,
                                            _f64p, C.POINTER(Stats)]),
    "nkg_ranking": (C.c_int, [_vp, _f64p, _u64p, _f64p]),
    "nkg_cancel": (None, [_vp]),
    "nkg_sigint_cancels": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "nkg_profile_sweeps": (C.c_int, [_vp, C.c_int, C.c_int, _f64p, _f64p]),
    "nkg_profile_gathers": (C.c_int, [_vp, C.c_int, C.c_int, _f64p]),
    "nkg_pagerank_csr_noalloc": (C.c_int, [C.c_uint64, C.c_uint64, _vp, _vp, C.POINTER(PRParams),
                                           _vp, _u64p, _vp]),
    "nkg_ppr_run": (C.c_int, [_vp, C.POINTER(PRParams), C.c_uint32, _u32p, _vp, C.c_int, _u64p,
                              C.POINTER(Stats)]),
    "nkg_pagerank_run_ex": (C.c_int, [_vp, C.POINTER(PRParams), _vp, _vp, C.c_int, _u64p, _f64p,
                                      C.POINTER(Stats)]),
    "nkg_graph_set_weights": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "nkg_pagerank_adjoint": (C.c_int, [_vp, C.POINTER(PRParams), _vp, _vp, _vp, _vp, _vp, C.c_int,
                                       _u64p, C.POINTER(Stats)]),
    "nkg_eigenvector_run": (C.c_int, [_vp, C.c_double, C.c_uint64, _vp, C.c_int, _u64p,
                                      C.POINTER(Stats)]),
    "nkg_katz_run": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint64, _vp,
                               C.c_int, _u64p, C.POINTER(Stats)]),
    "nkg_batch_create": (C.c_int, [C.POINTER(_vp), C.c_uint32, _u64p, _u64p, _u32p, C.c_int]),
    "nkg_batch_destroy": (None, [_vp]),
    "nkg_batch_get_tuning": (C.c_int, [_vp, C.POINTER(BatchTuning)]),
    "nkg_batch_set_tuning": (C.c_int, [_vp, C.POINTER(BatchTuning)]),
    "nkg_batch_tune": (C.c_int, [_vp, C.POINTER(PRParams), C.c_uint32, C.POINTER(BatchTuning),
                                 C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(BatchTuning)]),
    "nkg_batch_run": (C.c_int, [_vp, C.POINTER(PRParams), _vp, C.c_int, _u64p,
                                C.POINTER(C.c_uint32), C.POINTER(Stats)]),
    "nkg_batch_graph_times": (C.c_int, [_vp, _f64p, _f64p]),
    "nkg_release_cached_memory": (C.c_int, [C.c_int]),
    "nkg_local_create": (C.c_int, [C.POINTER(_vp), C.c_uint64, _u64p, _u32p, _f64p, _u8p, C.c_int,
                                   C.c_int, C.c_uint64]),
    "nkg_local_destroy": (None, [_vp]),
    "nkg_local_run": (C.c_int, [_vp, C.c_double, C.c_double, C.c_uint64, _u64p, _u32p, C.c_int,
                                C.c_uint64, _u64p, _u64p, C.POINTER(LocalStats)]),
    "nkg_local_support": (C.c_int, [_vp, _u32p, _f64p]),
    "nkg_local_sets": (C.c_int, [_vp, _u32p]),
    "nkg_graph_create_from_nkbg": (C.c_int, [C.POINTER(_vp), _vp, C.c_uint64, C.c_int,
                                             C.POINTER(GraphOptions), _f64p]),
    "nkg_graph_create_from_nkbg_file": (C.c_int, [C.POINTER(_vp), C.c_char_p, C.c_uint64,
                                                  C.POINTER(GraphOptions), _f64p, _f64p]),
    "nkg_nkbg_decode": (C.c_int, [_vp, C.c_uint64, C.c_int, C.c_int, _u64p, _u64p,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), _u64p, _u32p, _f64p,
                                  _f64p, _u32p, _u8p, _f64p]),
    "nkg_part_create": (C.c_int, [C.POINTER(_vp), C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                                  _u64p, _u32p, _f64p, _u32p, _f64p, C.c_int]),
    "nkg_part_destroy": (None, [_vp]),
    "nkg_part_begin": (C.c_int, [_vp, C.POINTER(PRParams), C.c_uint64, _vp, _vp]),
    "nkg_part_sweep": (C.c_int, [_vp, _vp, C.c_double, _vp, _f64p, _f64p, _vp]),
    "nkg_part_sums": (C.c_int, [_vp, _vp, _f64p, _f64p, _f64p, _vp]),
    "nkg_part_scores": (C.c_int, [_vp, _vp, C.c_double, _vp, _vp]),
}

_lib = None


def lib():
    """Load libnkgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m networkit_b200.build` "
                "(the PageRank path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.nkg_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} has ABI version {L.nkg_abi_version()}, this binding "
                               f"expects {ABI_VERSION}: rebuild with `python -m networkit_b200.build`")
        _lib = L
    return _lib


class NkgError(RuntimeError):
    """A failed libnkgpu call (RuntimeError, like the reference's `except +`)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def check(rc: int) -> None:
    if rc != NKG_OK:
        msg = lib().nkg_last_error().decode(errors="replace")
        raise NkgError(rc, msg)


def ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


class DeviceGraph:
    """Owning wrapper of an nkg_graph handle."""

    def __init__(self, csr, device: int = -1, sweep_shape: int = -1, arc_order: int = 0,
                 row_order: int = -1, hot_tier_kb: int = -1):
        L = lib()
        h = _vp()
        in_ptr = np.ascontiguousarray(csr.in_ptr, np.uint64)
        in_col = np.ascontiguousarray(csr.in_col, np.uint32)
        in_w = None if csr.in_w is None else np.ascontiguousarray(csr.in_w, np.float64)
        wdeg = np.ascontiguousarray(csr.wdeg, np.float64)
        ex = None if csr.exists is None else np.ascontiguousarray(csr.exists, np.uint8)
        opts = GraphOptions()
        opts.device = int(device)
        opts.sweep_shape = int(sweep_shape)
        opts.arc_order = int(arc_order)
        opts.row_order = int(row_order)
        opts.hot_tier_kb = int(hot_tier_kb)
        check(L.nkg_graph_create_ex(C.byref(h), int(csr.z), int(in_col.shape[0]),
                                    ptr(in_ptr, _u64p), ptr(in_col, _u32p), ptr(in_w, _f64p),
                                    ptr(wdeg, _f64p), ptr(ex, _u8p), int(bool(csr.directed)),
                                    C.byref(opts)))
        self.h = h
        self.z = int(csr.z)
        self.n = int(csr.n)

    @classmethod
    def from_edges(cls, z, src, dst, w=None, directed=False, exists=None, device: int = -1,
                   sweep_shape: int = -1, row_order: int = -1):
        """Build the graph on the device from host edge arrays in insertion
        order (nkg_graph_create_from_edges)."""
        s = np.ascontiguousarray(src, np.uint32)
        d = np.ascontiguousarray(dst, np.uint32)
        if s.shape != d.shape:
            raise ValueError("src and dst differ in length")
        ww = None if w is None else np.ascontiguousarray(w, np.float64)
        ex = None if exists is None else np.ascontiguousarray(exists, np.uint8)
        return cls._from_edge_pointers(
            z, int(s.shape[0]), s.ctypes.data, d.ctypes.data, 0 if ww is None else ww.ctypes.data,
            0 if ex is None else ex.ctypes.data, directed, False, device, sweep_shape, row_order)

    @classmethod
    def from_nkbg(cls, data, device: int = -1, row_order: int = -1, on_device: bool = False,
                  size: int = 0):
        """Build the graph from a NetworkitBinaryGraph file's bytes, decoded on
        the device (nkg_graph_create_from_nkbg): `data` is a bytes-like host
        buffer, or with on_device a device pointer of `size` bytes. The decode's
        device time is in .ms_decode."""
        self = cls.__new__(cls)
        h = _vp()
        opts = GraphOptions()
        opts.device = int(device)
        opts.row_order = int(row_order)
        ms = C.c_double(0.0)
        if on_device:
            buf, nbytes, flags = _vp(int(data)), int(size), NKG_DEVICE_PTRS
        else:
            arr = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
            arr = np.ascontiguousarray(arr, np.uint8)
            buf, nbytes, flags = _vp(arr.ctypes.data), int(arr.shape[0]), 0
        check(lib().nkg_graph_create_from_nkbg(C.byref(h), buf, nbytes, flags, C.byref(opts),
                                               C.byref(ms)))
        self.h = h
        info = self.info()
        self.z = int(info["z"])
        self.n = int(info["n"])
        self.ms_decode = float(ms.value)
        return self

    @classmethod
    def from_nkbg_file(cls, path, device: int = -1, row_order: int = -1, staging_bytes: int = 0):
        """Build the graph from a NetworkitBinaryGraph file on disk
        (nkg_graph_create_from_nkbg_file): read in pieces by reader threads,
        each piece copied to the device as it arrives, then decoded there.
        .ms_decode: device time of the decode; .s_load: host seconds to get
        the whole file onto the device."""
        self = cls.__new__(cls)
        h = _vp()
        opts = GraphOptions()
        opts.device = int(device)
        opts.row_order = int(row_order)
        ms, sl = C.c_double(0.0), C.c_double(0.0)
        check(lib().nkg_graph_create_from_nkbg_file(C.byref(h), os.fsencode(path),
                                                    int(staging_bytes), C.byref(opts),
                                                    C.byref(ms), C.byref(sl)))
        self.h = h
        info = self.info()
        self.z = int(info["z"])
        self.n = int(info["n"])
        self.ms_decode = float(ms.value)
        self.s_load = float(sl.value)
        return self

    @classmethod
    def from_device_edges(cls, z, m, src_ptr, dst_ptr, w_ptr=0, exists_ptr=0, directed=False,
                          device: int = -1, sweep_shape: int = -1, row_order: int = -1):
        """The same from device arrays (raw pointers; uint32 src/dst, float64
        w, uint8 exists)."""
        return cls._from_edge_pointers(z, m, src_ptr, dst_ptr, w_ptr, exists_ptr, directed, True,
                                       device, sweep_shape, row_order)

    @classmethod
    def _from_edge_pointers(cls, z, m, src_p, dst_p, w_p, ex_p, directed, on_device, device,
                            sweep_shape, row_order=-1):
        self = cls.__new__(cls)
        h = _vp()
        opts = GraphOptions()
        opts.device = int(device)
        opts.row_order = int(row_order)
        opts.sweep_shape = int(sweep_shape)
        check(lib().nkg_graph_create_from_edges(
            C.byref(h), int(z), int(m), _vp(src_p or None), _vp(dst_p or None), _vp(w_p or None),
            _vp(ex_p or None), int(bool(directed)), NKG_DEVICE_PTRS if on_device else 0,
            C.byref(opts)))
        self.h = h
        self.z = int(z)
        self.n = int(self.info()["n"])
        return self

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().nkg_graph_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        gi = GraphInfo()
        check(lib().nkg_graph_get_info(self.h, C.byref(gi)))
        return gi.as_dict()

    @staticmethod
    def params(damp, tol, norm, normalized, distribute_sinks, precision, max_iterations):
        return PRParams(float(damp), float(tol), int(norm), int(bool(normalized)),
                        int(bool(distribute_sinks)), int(precision), int(max_iterations))

    def run(self, p: PRParams, teleport=None, out=None, trace: int = 0):
        """Run to convergence; returns (scores[z], iterations, maximum, stats).
        `out`: optional float64[z] host array to receive the scores (pinned
        memory makes the read-back a direct DMA). trace > 0: stats also holds
        "residual_trace", the residual of every sweep with a stopping test
        (at most `trace` of them)."""
        L = lib()
        if out is not None:
            if out.dtype != np.float64 or out.shape != (self.z,) or not out.flags.c_contiguous:
                raise ValueError("out must be a contiguous float64 array of z entries")
            scores = out
        else:
            scores = np.empty(self.z, np.float64)
        it = C.c_uint64(0)
        mx = C.c_double(0.0)
        st, tbuf = Stats.with_trace(trace)
        if teleport is None:
            check(L.nkg_pagerank_run(self.h, C.byref(p), ptr(scores, _f64p), C.byref(it),
                                     C.byref(mx), C.byref(st)))
        else:
            t = np.ascontiguousarray(teleport, np.float64)
            if t.shape != (self.z,):
                raise ValueError("teleport must have upperNodeIdBound() entries")
            check(L.nkg_pagerank_run_teleport(self.h, C.byref(p), ptr(t, _f64p),
                                              ptr(scores, _f64p), C.byref(it), C.byref(mx),
                                              C.byref(st)))
        d = st.as_dict()
        if trace > 0:
            d["residual_trace"] = tbuf[:min(int(st.trace_length), int(trace))].copy()
        return scores, int(it.value), float(mx.value), d

    def run_device(self, p: PRParams, d_out_ptr: int):
        """Run with the scores written to device memory at d_out_ptr."""
        it = C.c_uint64(0)
        mx = C.c_double(0.0)
        st = Stats()
        check(lib().nkg_pagerank_run_device(self.h, C.byref(p), _vp(d_out_ptr), C.byref(it),
                                            C.byref(mx), C.byref(st)))
        return int(it.value), float(mx.value), st.as_dict()

    def run_ex(self, p: PRParams, teleport_ptr: int, out_ptr: int, on_device: bool):
        """nkg_pagerank_run_ex on raw pointers (host or device, per on_device);
        teleport_ptr 0 = uniform. Returns (iterations, maximum, stats)."""
        it = C.c_uint64(0)
        mx = C.c_double(0.0)
        st = Stats()
        check(lib().nkg_pagerank_run_ex(self.h, C.byref(p), _vp(teleport_ptr or None),
                                        _vp(out_ptr), NKG_DEVICE_PTRS if on_device else 0,
                                        C.byref(it), C.byref(mx), C.byref(st)))
        return int(it.value), float(mx.value), st.as_dict()

    def set_weights(self, in_w, out_wdeg=None):
        """New arc weights (numpy, in in_col order); out_wdeg None = summed on
        the device."""
        w = np.ascontiguousarray(in_w, np.float64)
        d = None if out_wdeg is None else np.ascontiguousarray(out_wdeg, np.float64)
        check(lib().nkg_graph_set_weights(self.h, _vp(w.ctypes.data),
                                          None if d is None else _vp(d.ctypes.data), 0))

    def set_weights_device(self, w_ptr: int, wdeg_ptr: int = 0):
        check(lib().nkg_graph_set_weights(self.h, _vp(w_ptr), _vp(wdeg_ptr or None),
                                          NKG_DEVICE_PTRS))

    def adjoint(self, p: PRParams, scores, grad, teleport=None, arcs=None):
        """Backward pass on host arrays: returns (grad_w[arcs], grad_t[z],
        sweeps, stats)."""
        s = np.ascontiguousarray(scores, np.float64)
        g = np.ascontiguousarray(grad, np.float64)
        t = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
        m = int(self.info()["arcs"] if arcs is None else arcs)
        gw = np.empty(max(m, 1), np.float64)
        gt = np.empty(self.z, np.float64)
        it = C.c_uint64(0)
        st = Stats()
        check(lib().nkg_pagerank_adjoint(self.h, C.byref(p),
                                         None if t is None else _vp(t.ctypes.data),
                                         _vp(s.ctypes.data), _vp(g.ctypes.data),
                                         _vp(gw.ctypes.data), _vp(gt.ctypes.data), 0,
                                         C.byref(it), C.byref(st)))
        return gw[:m], gt, int(it.value), st.as_dict()

    def adjoint_device(self, p: PRParams, scores_ptr: int, grad_ptr: int, gw_ptr: int,
                       gt_ptr: int, teleport_ptr: int = 0):
        """Backward pass on device pointers (0 = NULL); returns (sweeps, stats)."""
        it = C.c_uint64(0)
        st = Stats()
        check(lib().nkg_pagerank_adjoint(self.h, C.byref(p), _vp(teleport_ptr or None),
                                         _vp(scores_ptr), _vp(grad_ptr), _vp(gw_ptr or None),
                                         _vp(gt_ptr or None), NKG_DEVICE_PTRS, C.byref(it),
                                         C.byref(st)))
        return int(it.value), st.as_dict()

    def eigenvector(self, tol=1e-9, max_iterations=UINT64_MAX):
        """EigenvectorCentrality scores (z), iterations, stats."""
        out = np.empty(self.z, np.float64)
        it = C.c_uint64(0)
        st = Stats()
        check(lib().nkg_eigenvector_run(self.h, float(tol), int(max_iterations),
                                        _vp(out.ctypes.data), 0, C.byref(it), C.byref(st)))
        return out, int(it.value), st.as_dict()

    def katz(self, alpha=0.0, beta=0.1, tol=1e-8, edge_direction=0, max_iterations=UINT64_MAX):
        """KatzCentrality scores (z), iterations, stats."""
        out = np.empty(self.z, np.float64)
        it = C.c_uint64(0)
        st = Stats()
        check(lib().nkg_katz_run(self.h, float(alpha), float(beta), float(tol),
                                 int(edge_direction), int(max_iterations), _vp(out.ctypes.data),
                                 0, C.byref(it), C.byref(st)))
        return out, int(it.value), st.as_dict()

    def ppr(self, seeds, p: PRParams, d_out_ptr: int = 0):
        """Batched personalised PageRank (one column per seed). Returns
        (scores float32[k, z] or None when written to d_out_ptr on the device,
        iterations uint64[k], stats)."""
        s = np.ascontiguousarray(seeds, np.uint32)
        k = int(s.shape[0])
        it = np.zeros(k, np.uint64)
        st = Stats()
        if d_out_ptr:
            check(lib().nkg_ppr_run(self.h, C.byref(p), k, ptr(s, _u32p), _vp(d_out_ptr), 1,
                                    ptr(it, _u64p), C.byref(st)))
            return None, it, st.as_dict()
        out = np.empty((k, self.z), np.float32)
        check(lib().nkg_ppr_run(self.h, C.byref(p), k, ptr(s, _u32p),
                                _vp(out.ctypes.data), 0, ptr(it, _u64p), C.byref(st)))
        return out, it, st.as_dict()

    def ranking(self, scores):
        s = np.ascontiguousarray(scores, np.float64)
        ids = np.empty(self.n, np.uint64)
        vals = np.empty(self.n, np.float64)
        check(lib().nkg_ranking(self.h, ptr(s, _f64p), ptr(ids, _u64p), ptr(vals, _f64p)))
        return ids, vals

    def cancel(self):
        lib().nkg_cancel(self.h)

    def sigint_cancels(self, enable: bool) -> bool:
        """Route SIGINT to cancel() (enable) or give it back to the handler
        it had; on disable, returns whether a SIGINT arrived meanwhile."""
        got = C.c_int(0)
        check(lib().nkg_sigint_cancels(self.h, int(bool(enable)), C.byref(got)))
        return bool(got.value)

    def profile_sweeps(self, precision: int, sweeps: int):
        """(ms per sweep-kernel launch, ms per iteration) from CUDA events."""
        a, b = C.c_double(0.0), C.c_double(0.0)
        check(lib().nkg_profile_sweeps(self.h, int(precision), int(sweeps), C.byref(a),
                                       C.byref(b)))
        return float(a.value), float(b.value)

    def profile_gathers(self, precision: int, reps: int = 20) -> float:
        """ms per launch of the gathers-only diagnostic kernel (the random
        gather bound of the sweep on this graph)."""
        a = C.c_double(0.0)
        check(lib().nkg_profile_gathers(self.h, int(precision), int(reps), C.byref(a)))
        return float(a.value)


class DeviceBatch:
    """Owning wrapper of an nkg_batch handle: many graphs given as one
    block-diagonal in-CSR plus node_offsets (graph i = nodes
    [node_offsets[i], node_offsets[i+1]))."""

    def __init__(self, csr, node_offsets, device: int = -1):
        L = lib()
        h = _vp()
        offs = np.ascontiguousarray(node_offsets, np.uint64)
        in_ptr = np.ascontiguousarray(csr.in_ptr, np.uint64)
        in_col = np.ascontiguousarray(csr.in_col, np.uint32)
        check(L.nkg_batch_create(C.byref(h), int(offs.shape[0] - 1), ptr(offs, _u64p),
                                 ptr(in_ptr, _u64p), ptr(in_col, _u32p), int(device)))
        self.h = h
        self.count = int(offs.shape[0] - 1)
        self.total = int(offs[-1])
        self.node_offsets = offs

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().nkg_batch_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self) -> dict:
        t = BatchTuning()
        check(lib().nkg_batch_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, cluster: int, threads: int, split: int, variant: int = 0):
        t = BatchTuning(int(cluster), int(threads), int(split), int(variant), 0.0)
        check(lib().nkg_batch_set_tuning(self.h, C.byref(t)))

    def tune(self, p: PRParams, sweeps: int = 8, capacity: int = 64):
        """Time every candidate launch shape; returns (best, [all timed])."""
        res = (BatchTuning * capacity)()
        nres = C.c_uint32(0)
        best = BatchTuning()
        check(lib().nkg_batch_tune(self.h, C.byref(p), int(sweeps), res, capacity, C.byref(nres),
                                   C.byref(best)))
        return best.as_dict(), [res[i].as_dict() for i in range(min(nres.value, capacity))]

    def graph_times(self):
        """(start_ms, end_ms) of every graph in the last launch."""
        a = np.empty(self.count, np.float64)
        b = np.empty(self.count, np.float64)
        check(lib().nkg_batch_graph_times(self.h, ptr(a, _f64p), ptr(b, _f64p)))
        return a, b

    def run(self, p: PRParams, d_out_ptr: int = 0):
        """Returns (scores float64[total] or None when written to d_out_ptr,
        iterations uint64[count], floor_stops, stats)."""
        its = np.zeros(self.count, np.uint64)
        fl = C.c_uint32(0)
        st = Stats()
        if d_out_ptr:
            check(lib().nkg_batch_run(self.h, C.byref(p), _vp(d_out_ptr), NKG_DEVICE_PTRS,
                                      ptr(its, _u64p), C.byref(fl), C.byref(st)))
            return None, its, int(fl.value), st.as_dict()
        out = np.empty(self.total, np.float64)
        check(lib().nkg_batch_run(self.h, C.byref(p), _vp(out.ctypes.data), 0, ptr(its, _u64p),
                                  C.byref(fl), C.byref(st)))
        return out, its, int(fl.value), st.as_dict()


class DeviceLocal:
    """Owning wrapper of an nkg_local handle: the neighbour CSR (forNeighborsOf
    order) for ApproximatePageRank / PageRankNibble runs."""

    def __init__(self, z, row_ptr, col, w=None, exists=None, directed=False, device: int = -1,
                 memory_budget: int = 0):
        L = lib()
        h = _vp()
        self._ptr = np.ascontiguousarray(row_ptr, np.uint64)
        self._col = np.ascontiguousarray(col, np.uint32)
        self._w = None if w is None else np.ascontiguousarray(w, np.float64)
        self._ex = None if exists is None else np.ascontiguousarray(exists, np.uint8)
        check(L.nkg_local_create(C.byref(h), int(z), ptr(self._ptr, _u64p), ptr(self._col, _u32p),
                                 ptr(self._w, _f64p), ptr(self._ex, _u8p), int(bool(directed)),
                                 int(device), int(memory_budget)))
        self.h = h
        self.z = int(z)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().nkg_local_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, seed_sets, alpha, epsilon, nibble=False, max_pushes=UINT64_MAX):
        """seed_sets: a 1-D integer array (one single-seed problem per entry) or
        a list of seed collections (each made a sorted set). Returns
        (supports, sets, stats): supports = [(nodes, values)] per problem
        (ascending ids); sets = [nodes] per problem or None."""
        if isinstance(seed_sets, np.ndarray) and seed_sets.ndim == 1:
            if seed_sets.size and seed_sets.min() < 0:
                raise NkgError(NKG_ERR_INVALID_ARG, "negative seed id")
            seeds = np.ascontiguousarray(seed_sets, np.uint32)
            seed_ptr = np.arange(seeds.shape[0] + 1, dtype=np.uint64)
        else:
            sets_ = [np.unique(np.atleast_1d(np.asarray(list(x) if isinstance(x, (set, frozenset))
                                                        else x, np.int64))) for x in seed_sets]
            if any(x.size and x.min() < 0 for x in sets_):
                raise NkgError(NKG_ERR_INVALID_ARG, "negative seed id")
            seed_ptr = np.zeros(len(sets_) + 1, np.uint64)
            np.cumsum([x.shape[0] for x in sets_], out=seed_ptr[1:])
            seeds = (np.concatenate(sets_) if sets_ else np.zeros(0)).astype(np.uint32)
        k = seed_ptr.shape[0] - 1
        sup = np.zeros(k, np.uint64)
        setc = np.zeros(k, np.uint64)
        st = LocalStats()
        check(lib().nkg_local_run(self.h, float(alpha), float(epsilon), k, ptr(seed_ptr, _u64p),
                                  ptr(seeds, _u32p), NKG_LOCAL_NIBBLE if nibble else 0,
                                  int(max_pushes), ptr(sup, _u64p),
                                  ptr(setc, _u64p) if nibble else None, C.byref(st)))
        tot = int(sup.sum())
        nodes = np.empty(max(tot, 1), np.uint32)
        vals = np.empty(max(tot, 1), np.float64)
        check(lib().nkg_local_support(self.h, ptr(nodes, _u32p), ptr(vals, _f64p)))
        cut = np.cumsum(sup.astype(np.int64))[:-1]
        supports = list(zip(np.split(nodes[:tot], cut), np.split(vals[:tot], cut)))
        sets_out = None
        if nibble:
            ts = int(setc.sum())
            sn = np.empty(max(ts, 1), np.uint32)
            check(lib().nkg_local_sets(self.h, ptr(sn, _u32p)))
            sets_out = np.split(sn[:ts], np.cumsum(setc.astype(np.int64))[:-1])
        return supports, sets_out, st.as_dict()
