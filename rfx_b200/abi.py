"""ctypes binding of the C ABI (include/rfx_b200.h) — the call path the parity
tests and bench.py use.  It is the kind of ctypes stub a maintainer of the
reference would add to call the library from Python.

Device outputs may be given as torch CUDA tensors (or raw device addresses);
host outputs as numpy arrays.  There is no CPU fallback: if the library or a
CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from .forest import Forest

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librfx_b200.so")

RFX_OK = 0
STATUS_NAMES = {0: "RFX_OK", 1: "RFX_ERR_INVALID", 2: "RFX_ERR_CUDA", 3: "RFX_ERR_OOM", 4: "RFX_ERR_STATE",
                5: "RFX_ERR_UNSUPPORTED", 6: "RFX_ERR_TIMEOUT", 7: "RFX_ERR_FOREST", 8: "RFX_ERR_NO_DEVICE"}

# Every symbol include/rfx_b200.h declares (checked by the CPU tests).
EXPORTS = ["rfx_last_error", "rfx_ctx_create", "rfx_ctx_destroy", "rfx_ctx_stream", "rfx_synchronize",
           "rfx_forest_load", "rfx_forest_load_device", "rfx_route_oob", "rfx_oob_summary", "rfx_proximity_upper_i32", "rfx_pair_updates",
           "rfx_finishprox", "rfx_varimp", "rfx_localimp", "rfx_predict", "rfx_mds3d_full", "rfx_lowrank", "rfx_lowrank_operator",
           "rfx_lowrank_quantize", "rfx_mds_from_factors", "rfx_factor_mds_operator", "rfx_outlier_scores", "rfx_pair_counts_noalloc",
           "rfx_profile_enable", "rfx_profile_read", "rfx_grow_forest", "rfx_free_forest", "rfx_graph_capture_batch",
           "rfx_graph_launch", "rfx_graph_destroy", "rfx_tuned_shapes", "rfx_casewise_votes",
           "rfx_proximity_upper_f64", "rfx_finishprox_f64", "rfx_proximity_rfgap"]

STAGES = ["route", "leaf_lists", "pair_counts", "finishprox", "varimp_tree", "varimp_sample", "varimp_feature",
          "predict", "oob_summary", "localimp", "pair_ranges", "lowrank_product", "lowrank_orth", "mds_factors",
          "mds_full", "pair_hubs"]


class RfxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class _Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("use_casewise", ctypes.c_int32), ("n_threads_cpu", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 5)]


class _ForestView(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("p", ctypes.c_int32), ("nclass", ctypes.c_int32), ("maxcat", ctypes.c_int32),
                ("ntree", ctypes.c_int32), ("offs", ctypes.c_void_p), ("nodestatus", ctypes.c_void_p),
                ("bestvar", ctypes.c_void_p), ("xbestsplit", ctypes.c_void_p), ("treemap", ctypes.c_void_p),
                ("nodeclass", ctypes.c_void_p), ("catgoleft", ctypes.c_void_p), ("nin", ctypes.c_void_p),
                ("X", ctypes.c_void_p), ("y", ctypes.c_void_p), ("cat", ctypes.c_void_p)]


class _ForestDeviceView(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("p", ctypes.c_int32), ("nclass", ctypes.c_int32), ("maxcat", ctypes.c_int32),
                ("ntree", ctypes.c_int32), ("maxnode", ctypes.c_int32), ("nnode", ctypes.c_void_p),
                ("nodestatus", ctypes.c_void_p), ("bestvar", ctypes.c_void_p), ("xbestsplit", ctypes.c_void_p),
                ("treemap", ctypes.c_void_p), ("nodeclass", ctypes.c_void_p), ("catgoleft", ctypes.c_void_p),
                ("nin", ctypes.c_void_p), ("X", ctypes.c_void_p), ("y", ctypes.c_void_p), ("cat", ctypes.c_void_p)]


class _LowrankOpts(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int32), ("oversample", ctypes.c_int32), ("power_iters", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("seed", ctypes.c_uint64), ("trees_per_pass", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class _BatchItem(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("votes", ctypes.c_void_p), ("nout", ctypes.c_void_p),
                ("oob_error", ctypes.c_void_p), ("oob_pred", ctypes.c_void_p), ("S", ctypes.c_void_p),
                ("avimp", ctypes.c_void_p), ("sqsd", ctypes.c_void_p), ("qimp", ctypes.c_void_p),
                ("qimpm", ctypes.c_void_p), ("impn", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class _Grown(ctypes.Structure):
    _fields_ = [("ntree", ctypes.c_int32), ("offs", ctypes.POINTER(ctypes.c_int64)),
                ("nodestatus", ctypes.POINTER(ctypes.c_int32)), ("bestvar", ctypes.POINTER(ctypes.c_int32)),
                ("xbestsplit", ctypes.POINTER(ctypes.c_float)), ("treemap", ctypes.POINTER(ctypes.c_int32)),
                ("nodeclass", ctypes.POINTER(ctypes.c_int32)), ("nin", ctypes.POINTER(ctypes.c_int32))]


_LIB = None


def lib():
    """Load librfx_b200.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RfxError(8, f"native library missing: {LIB_PATH} (run python -m rfx_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        L.rfx_last_error.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def _check(st: int):
    if st != RFX_OK:
        raise RfxError(st, lib().rfx_last_error().decode())


def _ptr(a) -> Optional[int]:
    """Address of a numpy array, a torch tensor, or an int device address."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)}")


def _vp(a):
    p = _ptr(a)
    return None if p is None else ctypes.c_void_p(p)


def grow_forest(X, y, ntree: int, mtry: int, minndsize: int = 1, maxnode: int = 0, iseed: int = 12345,
                n_threads: int = 0, nclass: Optional[int] = None, cat=None, maxcat: int = 10) -> Forest:
    """Grow a forest with the library's restatement of the reference grower."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.int32)
    n, p = X.shape
    c = int(nclass if nclass is not None else np.unique(y).size)
    g = _Grown()
    _check(lib().rfx_grow_forest(_vp(X), _vp(y), n, p, c, ntree, mtry, minndsize, maxnode, iseed, n_threads,
                                 ctypes.byref(g)))
    try:
        offs = np.ctypeslib.as_array(g.offs, shape=(ntree + 1,)).copy()
        N = int(offs[-1])
        arr = lambda ptr, k: np.ctypeslib.as_array(ptr, shape=(k,)).copy()
        f = Forest(n=n, p=p, nclass=c, maxcat=maxcat, nnode=np.diff(offs).astype(np.int32), offs=offs,
                   nodestatus=arr(g.nodestatus, N), bestvar=arr(g.bestvar, N), xbestsplit=arr(g.xbestsplit, N),
                   treemap=arr(g.treemap, 2 * N), nodeclass=arr(g.nodeclass, N),
                   nin=arr(g.nin, ntree * n).reshape(ntree, n),
                   cat=np.ascontiguousarray(cat if cat is not None else np.ones(p), dtype=np.int32))
    finally:
        lib().rfx_free_forest(ctypes.byref(g))
    return f


class BatchGraph:
    """Many loaded contexts analysed by one CUDA graph (rfx_graph_capture_batch).

    ``items`` is a list of dicts with key ``ctx`` (a :class:`Context` with a
    loaded forest) and any of the device buffers ``votes``, ``nout``,
    ``oob_error``, ``oob_pred``, ``S``, ``avimp``, ``sqsd``, ``qimp``,
    ``qimpm`` (torch CUDA tensors or device addresses) plus ``impn``."""

    KEYS = ("votes", "nout", "oob_error", "oob_pred", "S", "avimp", "sqsd", "qimp", "qimpm")

    def __init__(self, items):
        arr = (_BatchItem * len(items))()
        self._keep = items
        for k, it in enumerate(items):
            arr[k].ctx = it["ctx"]._h.value
            for key in self.KEYS:
                setattr(arr[k], key, _ptr(it.get(key)))
            arr[k].impn = int(bool(it.get("impn", False)))
        h = ctypes.c_void_p()
        kn = ctypes.c_int64(0)
        _check(lib().rfx_graph_capture_batch(arr, len(items), ctypes.byref(h), ctypes.byref(kn)))
        self._h = h
        self.kernel_nodes = int(kn.value)

    def launch(self, stream: int = 0):
        _check(lib().rfx_graph_launch(self._h, ctypes.c_void_p(stream)))

    def close(self):
        if self._h is not None and self._h.value:
            lib().rfx_graph_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


TUNED_STAGES = {0: "route", 1: "pair_counts", 2: "varimp_walk", 3: "route_leaf_order", 4: "pair_counts_hub",
                5: "lowrank_leaf_sums_fp32", 6: "lowrank_leaf_sums_bf16", 7: "lowrank_leaf_sums_fp8",
                8: "varimp_sample"}
# launch shapes per stage, in the library's shape order
TUNED_SHAPES = {0: ["256x1", "128x1", "512x1", "256x2 trees", "256x4 trees", "256x2 trees, 2 walks in flight",
                    "256x4 trees, 2 walks in flight", "128x4 trees, 2 walks in flight",
                    "256x8 samples, 2048 staged nodes", "256x4 samples, 1024 staged nodes"],
                1: ["row16 256", "row16 512", "row16 1024", "row2 256", "row2 512", "row2 1024", "row3 512",
                    "row3 1024"],
                2: ["64", "128", "256", "64 staged rows", "128 staged rows", "256 staged rows",
                    "64 child prefetch", "128 child prefetch", "256 child prefetch"],
                3: ["128", "256", "512", "64 staged rows", "128 staged rows", "256 staged rows",
                    "128 child prefetch", "256 child prefetch", "512 child prefetch"],
                4: ["row2 256", "row2 512", "row2 1024", "row2 256 start-mask", "row2 512 start-mask",
                    "row2 1024 start-mask", "row3 512", "row3 1024"],
                5: ["warp per key", "slots"], 6: ["warp per key", "slots"], 7: ["warp per key", "slots"],
                8: ["tree loop", "per-sample OOB tree lists"]}


def _shape_name(kernel: int, shape: int) -> str:
    names = TUNED_SHAPES.get(kernel, [])
    return names[shape] if 0 <= shape < len(names) else str(shape)


def tuned_shapes():
    """Launch shapes the autotuner has picked in this process, as dicts."""
    cnt = ctypes.c_int32(0)
    _check(lib().rfx_tuned_shapes(None, 0, ctypes.byref(cnt)))
    buf = np.zeros(6 * max(cnt.value, 1), np.int32)
    _check(lib().rfx_tuned_shapes(_vp(buf), cnt.value, ctypes.byref(cnt)))
    out = []
    for r in buf[: 6 * cnt.value].reshape(-1, 6):
        st = int(r[0])
        out.append({"stage": TUNED_STAGES.get(st, str(st)), "device": int(r[1]), "log2_n": int(r[2]),
                    "log2_ntree": int(r[3]), "log2_p": int(r[4]), "shape": _shape_name(st, int(r[5]))})
    return out


def pair_counts_noalloc(leaf, inbag, n: int, ntree: int, max_leaves: int, S, stream: int = 0) -> None:
    """Allocation-free pair counts into the device buffer S (see include/rfx_b200.h)."""
    _check(lib().rfx_pair_counts_noalloc(_vp(leaf), _vp(inbag), int(n), int(ntree), int(max_leaves), _vp(S),
                                         ctypes.c_size_t(n * (n + 1) // 2), ctypes.c_void_p(stream)))


class Context:
    """One rfx_ctx: a device, a stream, and (after load) a resident forest."""

    def __init__(self, device: int = 0, use_casewise: bool = False):
        cfg = _Config(device=device, use_casewise=int(use_casewise), n_threads_cpu=0)
        h = ctypes.c_void_p()
        _check(lib().rfx_ctx_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.forest: Optional[Forest] = None

    def close(self):
        if self._h:
            lib().rfx_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().rfx_ctx_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    def synchronize(self):
        _check(lib().rfx_synchronize(self._h))

    def profile(self, enable: bool = True):
        _check(lib().rfx_profile_enable(self._h, int(bool(enable))))

    def profile_read(self):
        """(dict stage -> ms of its last launch, kernel launches so far)."""
        ms = np.zeros(len(STAGES), np.float32)
        cnt = ctypes.c_int64(0)
        _check(lib().rfx_profile_read(self._h, _vp(ms), ctypes.byref(cnt)))
        return {s: float(v) for s, v in zip(STAGES, ms)}, int(cnt.value)

    def load(self, forest: Forest, X, y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.int32)
        f = forest
        keep = [np.ascontiguousarray(a) for a in (f.offs, f.nodestatus, f.bestvar, f.xbestsplit, f.treemap,
                                                  f.nodeclass, f.nin, f.cat)]
        cg = None if f.catgoleft is None else np.ascontiguousarray(f.catgoleft, dtype=np.int32)
        v = _ForestView(n=f.n, p=f.p, nclass=f.nclass, maxcat=f.maxcat, ntree=f.ntree,
                        offs=_ptr(keep[0].astype(np.int64, copy=False)), nodestatus=_ptr(keep[1]),
                        bestvar=_ptr(keep[2]), xbestsplit=_ptr(keep[3]), treemap=_ptr(keep[4]),
                        nodeclass=_ptr(keep[5]), catgoleft=_ptr(cg), nin=_ptr(keep[6]), X=_ptr(X), y=_ptr(y),
                        cat=_ptr(keep[7]))
        _check(lib().rfx_forest_load(self._h, ctypes.byref(v)))
        self.forest = f
        self.n, self.p, self.nclass, self.ntree = f.n, f.p, f.nclass, f.ntree

    def load_device(self, forest: Forest, arrays: dict, maxnode: int):
        """Load a forest held in device memory in the padded per-tree layout
        (rfx_forest_load_device).  ``arrays`` maps nodestatus, bestvar,
        xbestsplit, treemap, nodeclass, nin, X, y, cat (and optionally
        catgoleft) to device buffers (torch CUDA tensors or addresses); node
        counts come from ``forest.nnode`` (host)."""
        nnode = np.ascontiguousarray(forest.nnode, dtype=np.int32)
        g = lambda k: _ptr(arrays.get(k))
        v = _ForestDeviceView(n=forest.n, p=forest.p, nclass=forest.nclass, maxcat=forest.maxcat,
                              ntree=forest.ntree, maxnode=int(maxnode), nnode=_ptr(nnode),
                              nodestatus=g("nodestatus"), bestvar=g("bestvar"), xbestsplit=g("xbestsplit"),
                              treemap=g("treemap"), nodeclass=g("nodeclass"), catgoleft=g("catgoleft"),
                              nin=g("nin"), X=g("X"), y=g("y"), cat=g("cat"))
        _check(lib().rfx_forest_load_device(self._h, ctypes.byref(v)))
        self.forest = forest
        self.n, self.p, self.nclass, self.ntree = forest.n, forest.p, forest.nclass, forest.ntree

    # --- analysis ---------------------------------------------------------
    def route_oob(self, q=None, nout=None, leaf=None):
        """Integer OOB votes q (n, c), doubled nout (n,), optional leaf (T, n)."""
        if q is None:
            q = np.zeros((self.n, self.nclass), np.int32)
        if nout is None:
            nout = np.zeros(self.n, np.int32)
        _check(lib().rfx_route_oob(self._h, _vp(q), _vp(nout), _vp(leaf)))
        return q, nout, leaf

    def casewise_votes(self, q=None, nout=None):
        """Case-wise weighted OOB votes q (n, c) float32 and doubled nout."""
        if q is None:
            q = np.zeros((self.n, self.nclass), np.float32)
        if nout is None:
            nout = np.zeros(self.n, np.int32)
        _check(lib().rfx_casewise_votes(self._h, _vp(q), _vp(nout)))
        return q, nout

    def proximity_upper_f64(self, S=None):
        """FP64 pair sums C + C^T, packed upper triangle (n(n+1)/2,)."""
        L = self.n * (self.n + 1) // 2
        if S is None:
            S = np.zeros(L, np.float64)
        _check(lib().rfx_proximity_upper_f64(self._h, _vp(S), ctypes.c_size_t(L)))
        return S

    def finishprox_f64(self, S, P=None, full=True):
        """finishprox of FP64 sums (host or device buffers)."""
        if P is None:
            P = np.zeros((self.n, self.n) if full else (self.n * (self.n + 1) // 2,), np.float32)
        _check(lib().rfx_finishprox_f64(self._h, _vp(S), _vp(P), int(bool(full))))
        return P

    def proximity_rfgap(self, P=None):
        """RF-GAP proximity, packed upper triangle FP64 (n(n+1)/2,)."""
        L = self.n * (self.n + 1) // 2
        if P is None:
            P = np.zeros(L, np.float64)
        _check(lib().rfx_proximity_rfgap(self._h, _vp(P), ctypes.c_size_t(L)))
        return P

    def oob_summary(self, err=None, pred=None, proba=None):
        """OOB error, predictions and probabilities; with any output given
        (host or device buffers) only the given ones are written and returned."""
        if err is None and pred is None and proba is None:
            err = np.zeros(1, np.float32)
            pred = np.zeros(self.n, np.int32)
            proba = np.zeros((self.n, self.nclass), np.float32)
            _check(lib().rfx_oob_summary(self._h, _vp(err), _vp(pred), _vp(proba)))
            return float(err[0]), pred, proba
        _check(lib().rfx_oob_summary(self._h, _vp(err), _vp(pred), _vp(proba)))
        return err, pred, proba

    def proximity_upper(self, S=None):
        """Packed upper-triangle INT32 pair counts (n(n+1)/2,)."""
        L = self.n * (self.n + 1) // 2
        if S is None:
            S = np.zeros(L, np.int32)
        _check(lib().rfx_proximity_upper_i32(self._h, _vp(S), ctypes.c_size_t(L)))
        return S

    def pair_updates(self) -> int:
        c = ctypes.c_int64(0)
        _check(lib().rfx_pair_updates(self._h, ctypes.byref(c)))
        return int(c.value)

    def finishprox(self, S, P=None, full=True):
        if P is None:
            P = np.zeros((self.n, self.n) if full else self.n * (self.n + 1) // 2, np.float32)
        _check(lib().rfx_finishprox(self._h, _vp(S), _vp(P), int(bool(full))))
        return P

    def varimp(self, impn=True, avimp=None, sqsd=None, qimp=None, qimpm=None):
        if avimp is None:
            avimp = np.zeros(self.p, np.float32)
        if sqsd is None:
            sqsd = np.zeros(self.p, np.float32)
        if impn and qimp is None:
            qimp = np.zeros(self.n, np.float32)
        if impn and qimpm is None:
            qimpm = np.zeros(self.n * self.p, np.float32)
        _check(lib().rfx_varimp(self._h, int(bool(impn)), _vp(avimp), _vp(sqsd), _vp(qimp), _vp(qimpm)))
        return avimp, sqsd, qimp, qimpm

    def localimp(self, qimp, qimpm, out=None):
        if out is None:
            out = np.zeros((self.n, self.p), np.float32)
        _check(lib().rfx_localimp(self._h, _vp(qimp), _vp(qimpm), _vp(out)))
        return out

    def mds3d_full(self, P, coords=None):
        """compute_mds_3d_cpu on the full float32 proximity matrix: (coords n x 3, eigenvalues)."""
        if coords is None:
            coords = np.zeros((self.n, 3), np.float64)
        ev = np.zeros(3, np.float64)
        _check(lib().rfx_mds3d_full(self._h, _vp(P), _vp(coords), _vp(ev)))
        return coords, ev

    def lowrank(self, rank, oversample=16, power_iters=1, precision=0, seed=12345, A=None, trees_per_pass=0):
        """Factors A (n x rank float32, P ~= I + A A^T) and the rank eigenvalues."""
        self._rank_guess = rank
        if A is None:
            A = np.zeros((self.n, rank), np.float32)
        ev = np.zeros(rank, np.float32)
        o = _LowrankOpts(rank=rank, oversample=oversample, power_iters=power_iters, precision=precision, seed=seed,
                         trees_per_pass=trees_per_pass)
        _check(lib().rfx_lowrank(self._h, ctypes.byref(o), _vp(A), _vp(ev)))
        return A, ev

    def lowrank_operator(self, V, precision=0):
        """M V for the low-rank operator M = P - I (V: n x w float32, w a
        multiple of 8 up to 120), as the range finder computes it."""
        V = np.ascontiguousarray(V, dtype=np.float32)
        MV = np.zeros_like(V)
        _check(lib().rfx_lowrank_operator(self._h, int(V.shape[1]), int(precision), _vp(V), _vp(MV)))
        return MV

    def lowrank_quantize(self, fmt):
        """fmt 1 = INT8, 2 = FP8 e4m3 (q: n x rank bytes), 3 = NF4 (q:
        ceil(n * rank / 2) bytes, two codes per byte), 4 = FP16 (q: n x rank
        uint16); returns (q, per-column scales)."""
        r = self._rank_guess
        if fmt == 3:
            q = np.zeros((self.n * r + 1) // 2, np.uint8)
        elif fmt == 4:
            q = np.zeros((self.n, r), np.uint16)
        else:
            q = np.zeros((self.n, r), np.uint8)
        sc = np.zeros(r, np.float32)
        _check(lib().rfx_lowrank_quantize(self._h, int(fmt), _vp(q), _vp(sc)))
        return q, sc

    def mds_from_factors(self, k=3, use_quantized=False, precision=0):
        coords = np.zeros((self.n, k), np.float64)
        ev = np.zeros(k, np.float64)
        _check(lib().rfx_mds_from_factors(self._h, int(k), int(bool(use_quantized)), int(precision), _vp(coords),
                                          _vp(ev)))
        return coords, ev

    def factor_operator(self, V, use_quantized=False, precision=0):
        """W = B V for an n x 16 FP64 block (the factor MDS operator)."""
        V = np.ascontiguousarray(V, np.float64)
        W = np.zeros_like(V)
        _check(lib().rfx_factor_mds_operator(self._h, int(bool(use_quantized)), int(precision), _vp(V), _vp(W)))
        return W

    def outlier_scores(self, use_quantized=False):
        out = np.zeros(self.n, np.float32)
        _check(lib().rfx_outlier_scores(self._h, int(bool(use_quantized)), _vp(out)))
        return out

    def predict_votes(self, Xt, votes=None):
        m = int(Xt.shape[0])
        if isinstance(Xt, np.ndarray):
            Xt = np.ascontiguousarray(Xt, dtype=np.float32)
        if votes is None:
            votes = np.zeros((m, self.nclass), np.int32)
        _check(lib().rfx_predict(self._h, _vp(Xt), m, _vp(votes)))
        return votes
