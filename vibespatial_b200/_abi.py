"""ctypes binding of ``libvsjoin.so`` (the C-ABI declared in ``include/vsjoin.h``).

Device buffers are torch CUDA tensors: torch provides device memory and the
stream, the library does the work.  There is no CPU fallback: if the library
or a GPU is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "_lib" / "libvsjoin.so"

VS_OK, VS_E_ARG, VS_E_OOM, VS_E_CAPACITY, VS_E_CUDA, VS_E_TIMEOUT, VS_E_STATE = range(7)
PRED_BBOX, PRED_INTERSECTS, PRED_WITHIN, PRED_COVERED_BY, PRED_TOUCHES = range(5)
METHOD_RTREE, METHOD_LEARNED, METHOD_BRUTE = range(3)
JOIN_SORT = 1
JOIN_BULK_LEAVES = 2
JOIN_LEARNED_BSEARCH = 4
JOIN_LEARNED_FP64_WALK = 8
JOIN_LEARNED_NO_STAGE = 16
JOIN_LEARNED_NO_INTERIOR = 32

# Every function the header declares; tests check the library exports them.
EXPORTED = (
    "vs_version", "vs_last_error", "vs_context_create", "vs_context_destroy",
    "vs_context_synchronize", "vs_index_build", "vs_index_info_get", "vs_index_free",
    "vs_join", "vs_locate_aligned", "vs_sort_pairs", "vs_radix_sort_pairs", "vs_hilbert_keys",
    "vs_join_brute_noalloc", "vs_batch_plan_create", "vs_batch_run", "vs_batch_plan_free",
    "vs_wkb_plan_create", "vs_wkb_plan_decode", "vs_wkb_plan_free", "vs_join_host",
    "vs_thread_kernel_launches", "vs_join_dwithin", "vs_join_nearest", "vs_join_export",
    "vs_distance_aligned", "vs_join_nearest_polygons", "vs_row_counts", "vs_row_sums", "vs_select_rows",
    "vs_pairs_member",
)


class VsError(RuntimeError):
    """A C-ABI call returned a status other than VS_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[vsjoin status {status}] {message}")
        self.status = status


class CapacityError(VsError, MemoryError):
    """Pair buffer too small (mirrors the reference's CandidateRelationCapacityError)."""

    def __init__(self, status, message, required):
        super().__init__(status, message)
        self.required = required


class Polygons(ctypes.Structure):
    _fields_ = [
        ("d_x", ctypes.c_void_p), ("d_y", ctypes.c_void_p),
        ("d_ring_off", ctypes.c_void_p), ("d_part_off", ctypes.c_void_p),
        ("d_geom_off", ctypes.c_void_p), ("d_valid", ctypes.c_void_p),
        ("n_coords", ctypes.c_int64), ("n_rings", ctypes.c_int32),
        ("n_parts", ctypes.c_int32), ("n_geoms", ctypes.c_int32),
    ]


class Points(ctypes.Structure):
    _fields_ = [("d_x", ctypes.c_void_p), ("d_y", ctypes.c_void_p),
                ("d_valid", ctypes.c_void_p), ("n", ctypes.c_int64)]


class IndexOptions(ctypes.Structure):
    _fields_ = [("method_mask", ctypes.c_int32), ("cell_level", ctypes.c_int32),
                ("rmi_leaves", ctypes.c_int32), ("rmi_train_steps", ctypes.c_int32),
                ("ring_bin_min_vertices", ctypes.c_int32)]


class JoinStats(ctypes.Structure):
    _fields_ = [
        ("candidates", ctypes.c_int64), ("exact_fallbacks", ctypes.c_int64),
        ("fp32_edges", ctypes.c_int64), ("fp64_edges", ctypes.c_int64),
        ("rmi_fallbacks", ctypes.c_int64), ("kernel_ms", ctypes.c_float),
        ("sort_ms", ctypes.c_float), ("kernel_launches", ctypes.c_int64),
        ("phase_ms", ctypes.c_float * 4),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["phase_ms"] = [float(v) for v in self.phase_ms]
        return d


class BatchOptions(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32), ("packets_per_grab", ctypes.c_int32),
                ("sort_levels", ctypes.c_int32), ("method", ctypes.c_int32),
                ("learned_map_blocks_per_sm", ctypes.c_int32), ("learned_refine_blocks_per_sm", ctypes.c_int32),
                ("learned_grab", ctypes.c_int32), ("learned_flags", ctypes.c_uint32),
                ("learned_map_packets", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class WkbSizes(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("n_rows", "n_points", "n_polygons", "n_multipolygons", "n_null",
                                               "n_unsupported", "n_malformed", "n_parts", "n_rings", "n_coords")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class WkbOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("d_tags", "d_px", "d_py", "d_geom_off", "d_part_off", "d_ring_off",
                                                "d_x", "d_y")]


class IndexInfo(ctypes.Structure):
    _fields_ = [
        ("n_geoms", ctypes.c_int32), ("fanout", ctypes.c_int32), ("levels", ctypes.c_int32),
        ("cell_level", ctypes.c_int32), ("n_cells", ctypes.c_int64),
        ("n_cell_entries", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
        ("build_ms", ctypes.c_float), ("rmi_train_ms", ctypes.c_float),
        ("rmi_mean_window", ctypes.c_float), ("rmi_max_window", ctypes.c_int32),
        ("n_binned_rings", ctypes.c_int64), ("n_bin_edges", ctypes.c_int64),
        ("rmi_leaves", ctypes.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_lock = threading.Lock()


def load(path: Path | str | None = None):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise RuntimeError(
                f"{p} is missing: build it with `python -m vibespatial_b200._build` "
                "(the join has no CPU fallback)"
            )
        L = ctypes.CDLL(str(p))
        vp, i32, i64, u32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
        sig = {
            "vs_version": (ctypes.c_int, []),
            "vs_last_error": (ctypes.c_char_p, []),
            "vs_thread_kernel_launches": (ctypes.c_longlong, []),
            "vs_context_create": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(vp)]),
            "vs_context_destroy": (ctypes.c_int, [vp]),
            "vs_context_synchronize": (ctypes.c_int, [vp]),
            "vs_index_build": (ctypes.c_int, [vp, ctypes.POINTER(Polygons), ctypes.POINTER(IndexOptions), ctypes.POINTER(vp)]),
            "vs_index_info_get": (ctypes.c_int, [vp, ctypes.POINTER(IndexInfo)]),
            "vs_index_free": (ctypes.c_int, [vp]),
            "vs_join": (ctypes.c_int, [vp, vp, ctypes.POINTER(Points), i32, i32, u32, vp, vp, i64,
                                       ctypes.POINTER(i64), ctypes.POINTER(JoinStats)]),
            "vs_join_dwithin": (ctypes.c_int, [vp, vp, ctypes.POINTER(Points), vp, vp, ctypes.c_double, u32, vp, vp,
                                               i64, ctypes.POINTER(i64), ctypes.POINTER(JoinStats)]),
            "vs_join_nearest": (ctypes.c_int, [vp, vp, ctypes.POINTER(Points), ctypes.c_double, u32, vp, vp, vp,
                                               i64, ctypes.POINTER(i64), ctypes.POINTER(JoinStats)]),
            "vs_join_nearest_polygons": (ctypes.c_int, [vp, vp, ctypes.POINTER(Polygons), ctypes.c_double, u32, vp,
                                                        vp, vp, i64, ctypes.POINTER(i64), ctypes.POINTER(JoinStats)]),
            "vs_distance_aligned": (ctypes.c_int, [vp, ctypes.POINTER(Points), ctypes.POINTER(Polygons), vp, vp]),
            "vs_join_export": (ctypes.c_int, [vp, vp, vp, i64, i64, i64, i32, vp, vp, vp, vp, vp, i64,
                                              ctypes.POINTER(i64)]),
            "vs_locate_aligned": (ctypes.c_int, [vp, ctypes.POINTER(Points), ctypes.POINTER(Polygons), vp]),
            "vs_sort_pairs": (ctypes.c_int, [vp, vp, vp, i64]),
            "vs_radix_sort_pairs": (ctypes.c_int, [vp, vp, vp, i64, i32]),
            "vs_hilbert_keys": (ctypes.c_int, [vp, vp, vp, i64, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, vp]),
            "vs_join_brute_noalloc": (ctypes.c_int, [ctypes.POINTER(Points), ctypes.POINTER(Polygons), i32, vp, vp,
                                                     i64, ctypes.POINTER(i64), vp]),
            "vs_batch_plan_create": (ctypes.c_int, [vp, ctypes.POINTER(vp), i32, ctypes.POINTER(Points),
                                                    ctypes.POINTER(i64), ctypes.POINTER(BatchOptions),
                                                    ctypes.POINTER(vp)]),
            "vs_batch_run": (ctypes.c_int, [vp, i32, vp, vp, i64, i32, ctypes.POINTER(i64),
                                            ctypes.POINTER(JoinStats)]),
            "vs_batch_plan_free": (ctypes.c_int, [vp]),
            "vs_wkb_plan_create": (ctypes.c_int, [vp, vp, vp, vp, i64, ctypes.POINTER(WkbOut), ctypes.POINTER(vp),
                                                  ctypes.POINTER(WkbSizes)]),
            "vs_wkb_plan_decode": (ctypes.c_int, [vp, ctypes.POINTER(WkbOut)]),
            "vs_wkb_plan_free": (ctypes.c_int, [vp]),
            "vs_join_host": (ctypes.c_int, [vp, vp, vp, vp, vp, i64, i32, i32, u32, vp, vp, i64, ctypes.POINTER(i64),
                                            ctypes.POINTER(JoinStats)]),
            "vs_row_counts": (ctypes.c_int, [vp, vp, vp, i64, i64, vp]),
            "vs_row_sums": (ctypes.c_int, [vp, vp, vp, i64, i64, vp, i64, vp]),
            "vs_select_rows": (ctypes.c_int, [vp, vp, i64, i32, vp, ctypes.POINTER(i64)]),
            "vs_pairs_member": (ctypes.c_int, [vp, vp, vp, i64, vp, vp, i64, i64, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = L
        return L


def last_error() -> str:
    msg = load().vs_last_error()
    return msg.decode() if msg else ""


def check(status: int, required: int | None = None) -> None:
    if status == VS_OK:
        return
    msg = last_error()
    if status == VS_E_CAPACITY:
        raise CapacityError(status, msg, required)
    if status == VS_E_ARG:
        raise ValueError(f"[vsjoin] {msg}")
    if status == VS_E_OOM:
        raise MemoryError(f"[vsjoin] {msg}")
    raise VsError(status, msg)


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


class Context:
    """One device + one stream (torch's current stream by default)."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("vsjoin needs a CUDA device; none is visible")
        self.device = int(device)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        self.torch_stream = stream
        # torch reports its legacy default stream as handle 0, which the C-ABI
        # reads as "create a private stream"; pass cudaStreamLegacy (0x1)
        # instead so the join is ordered after torch's own copies.
        handle = stream.cuda_stream or 0x1
        h = ctypes.c_void_p()
        check(load().vs_context_create(self.device, ctypes.c_void_p(handle), ctypes.byref(h)))
        self.handle = h

    def synchronize(self):
        check(load().vs_context_synchronize(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            load().vs_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: dict[int, Context] = {}


def default_context(device: int = 0) -> Context:
    ctx = _default_ctx.get(device)
    if ctx is None:
        ctx = _default_ctx[device] = Context(device)
    return ctx


def make_points(x, y, valid=None) -> Points:
    return Points(_ptr(x), _ptr(y), _ptr(valid), int(x.numel()))


def make_polygons(x, y, ring_off, part_off, geom_off, valid=None) -> Polygons:
    return Polygons(_ptr(x), _ptr(y), _ptr(ring_off), _ptr(part_off), _ptr(geom_off), _ptr(valid),
                    int(x.numel()), int(ring_off.numel()) - 1, int(part_off.numel()) - 1,
                    int(geom_off.numel()) - 1)


class DeviceIndex:
    """Owned handle of a built index (vs_index*)."""

    def __init__(self, ctx: Context, polys: Polygons, *, learned: bool = False, cell_level: int = 0,
                 rmi_leaves: int = 0, rmi_train_steps: int = 0, ring_bin_min_vertices: int = 0):
        self.ctx = ctx
        opts = IndexOptions(1 | (2 if learned else 0), int(cell_level), int(rmi_leaves), int(rmi_train_steps),
                            int(ring_bin_min_vertices))
        h = ctypes.c_void_p()
        check(load().vs_index_build(ctx.handle, ctypes.byref(polys), ctypes.byref(opts), ctypes.byref(h)))
        self.handle = h
        self.learned = learned

    def info(self) -> dict:
        inf = IndexInfo()
        check(load().vs_index_info_get(self.handle, ctypes.byref(inf)))
        return inf.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            load().vs_index_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def join_into(self, pts: Points, predicate: int, method: int, left, right, *, sort: bool = False,
                  flags: int = 0):
        """One vs_join call into caller buffers; returns (n_pairs, stats dict).

        Raises CapacityError (with .required) if the buffers are too small.
        """
        n = ctypes.c_int64(0)
        st = JoinStats()
        cap = 0 if left is None else int(left.numel())
        status = load().vs_join(self.ctx.handle, self.handle, ctypes.byref(pts), int(predicate), int(method),
                                (JOIN_SORT if sort else 0) | int(flags), _ptr(left), _ptr(right), cap,
                                ctypes.byref(n), ctypes.byref(st))
        check(status, required=int(n.value))
        return int(n.value), st.as_dict()

    def join_host(self, x, y, predicate: int, method: int, left, right, *, valid=None, sort: bool = False):
        """vs_join_host: host (CPU) point buffers in, host pair buffers out; returns (n_pairs, stats).

        x, y: float64 and valid: uint8 (or None) CPU tensors or numpy arrays;
        left, right: int32 CPU tensors or numpy arrays (pinned tensors let the
        copies overlap the join).  Raises CapacityError (with .required).
        """
        def ptr(a):
            if a is None:
                return None
            return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data

        def size(a):
            return int(a.numel()) if hasattr(a, "numel") else int(a.size)

        n = ctypes.c_int64(0)
        st = JoinStats()
        cap = 0 if left is None else size(left)
        status = load().vs_join_host(self.ctx.handle, self.handle, ptr(x), ptr(y), ptr(valid), size(x),
                                     int(predicate), int(method), JOIN_SORT if sort else 0, ptr(left), ptr(right),
                                     cap, ctypes.byref(n), ctypes.byref(st))
        check(status, required=int(n.value))
        return int(n.value), st.as_dict()

    def dwithin_into(self, pts: Points, left, right, *, distance: float = 0.0, point_distance=None,
                     geom_distance=None, sort: bool = False):
        """vs_join_dwithin into caller buffers; returns (n_pairs, stats).

        The distance is ``point_distance`` (float64 CUDA tensor, one per
        point), ``geom_distance`` (one per polygon row) or the scalar
        ``distance``.  Raises CapacityError (with .required).
        """
        n = ctypes.c_int64(0)
        st = JoinStats()
        cap = 0 if left is None else int(left.numel())
        status = load().vs_join_dwithin(self.ctx.handle, self.handle, ctypes.byref(pts), _ptr(point_distance),
                                        _ptr(geom_distance), float(distance), JOIN_SORT if sort else 0, _ptr(left),
                                        _ptr(right), cap, ctypes.byref(n), ctypes.byref(st))
        check(status, required=int(n.value))
        return int(n.value), st.as_dict()

    def nearest_into(self, pts: Points, left, right, distance=None, *, max_distance: float = float("inf"),
                     sort: bool = False):
        """vs_join_nearest into caller buffers (``distance``: float64 CUDA
        tensor for the pair distances, or None); returns (n_pairs, stats)."""
        n = ctypes.c_int64(0)
        st = JoinStats()
        cap = 0 if left is None else int(left.numel())
        status = load().vs_join_nearest(self.ctx.handle, self.handle, ctypes.byref(pts), float(max_distance),
                                        JOIN_SORT if sort else 0, _ptr(left), _ptr(right), _ptr(distance), cap,
                                        ctypes.byref(n), ctypes.byref(st))
        check(status, required=int(n.value))
        return int(n.value), st.as_dict()

    def _grow(self, pts: Points, run, capacity, with_distance=False):
        import torch

        dev = torch.device("cuda", self.ctx.device)
        cap = int(capacity) if capacity is not None else max(1024, int(pts.n))
        for _ in range(2):
            left = torch.empty(cap, dtype=torch.int32, device=dev)
            right = torch.empty(cap, dtype=torch.int32, device=dev)
            dist = torch.empty(cap, dtype=torch.float64, device=dev) if with_distance else None
            try:
                n, stats = run(left, right, dist)
                return left[:n], right[:n], (dist[:n] if dist is not None else None), stats
            except CapacityError as e:
                cap = max(e.required, 1)
        raise RuntimeError("pair buffer sizing did not converge")

    def dwithin(self, pts: Points, *, distance: float = 0.0, point_distance=None, geom_distance=None,
                sort: bool = True, capacity: int | None = None):
        """Pairs within the distance, into fresh int32 device tensors (left, right, stats)."""
        left, right, _, st = self._grow(
            pts, lambda l, r, d: self.dwithin_into(pts, l, r, distance=distance, point_distance=point_distance,
                                                   geom_distance=geom_distance, sort=sort), capacity)
        return left, right, st

    def nearest(self, pts: Points, *, max_distance: float = float("inf"), sort: bool = True,
                capacity: int | None = None):
        """Nearest polygons (all ties): (left, right, distance, stats) device tensors."""
        return self._grow(pts, lambda l, r, d: self.nearest_into(pts, l, r, d, max_distance=max_distance,
                                                                 sort=sort), capacity, with_distance=True)

    def join(self, pts: Points, predicate: int, method: int = METHOD_RTREE, *, sort: bool = True,
             capacity: int | None = None, flags: int = 0):
        """Join into freshly allocated int32 device tensors, growing them once if needed."""
        import torch

        dev = torch.device("cuda", self.ctx.device)
        cap = int(capacity) if capacity is not None else max(1024, int(pts.n))
        for _ in range(2):
            left = torch.empty(cap, dtype=torch.int32, device=dev)
            right = torch.empty(cap, dtype=torch.int32, device=dev)
            try:
                n, stats = self.join_into(pts, predicate, method, left, right, sort=sort, flags=flags)
                return left[:n], right[:n], stats
            except CapacityError as e:
                cap = max(e.required, 1)
        raise RuntimeError("pair buffer sizing did not converge")


class BatchPlan:
    """Owned handle of a batched join plan (vs_batch_plan*).

    Job j joins points ``job_start[j]:job_start[j+1]`` of ``pts`` against
    ``indexes[j]``.  The plan borrows the point buffers and the indexes: keep
    them alive while the plan is used (this object holds references).
    """

    def __init__(self, ctx: Context, indexes, pts: Points, job_start, *, options: dict | None = None,
                 keepalive=()):
        self.ctx = ctx
        self.indexes = list(indexes)
        self.pts = pts
        self._keepalive = keepalive
        js = np.ascontiguousarray(np.asarray(job_start, dtype=np.int64))
        if len(js) != len(self.indexes) + 1:
            raise ValueError("job_start needs one entry more than there are jobs")
        self.job_start = js
        o = BatchOptions(**(options or {}))
        self.options = o.as_dict()
        arr = (ctypes.c_void_p * len(self.indexes))(*[ix.handle.value for ix in self.indexes])
        h = ctypes.c_void_p()
        check(load().vs_batch_plan_create(ctx.handle, arr, len(self.indexes), ctypes.byref(pts),
                                          js.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(o),
                                          ctypes.byref(h)))
        self.handle = h

    def run_into(self, predicate: int, left, right, *, use_graph: bool = True):
        """One batched join into caller buffers; returns (n_pairs, stats dict)."""
        n = ctypes.c_int64(0)
        st = JoinStats()
        cap = 0 if left is None else int(left.numel())
        status = load().vs_batch_run(self.handle, int(predicate), _ptr(left), _ptr(right), cap,
                                     1 if use_graph else 0, ctypes.byref(n), ctypes.byref(st))
        check(status, required=int(n.value))
        return int(n.value), st.as_dict()

    def run(self, predicate: int, *, use_graph: bool = True, capacity: int | None = None):
        """Batched join into fresh int32 device tensors (grown once if too small)."""
        import torch

        dev = torch.device("cuda", self.ctx.device)
        cap = int(capacity) if capacity is not None else max(1024, int(self.pts.n))
        for _ in range(2):
            left = torch.empty(cap, dtype=torch.int32, device=dev)
            right = torch.empty(cap, dtype=torch.int32, device=dev)
            try:
                n, stats = self.run_into(predicate, left, right, use_graph=use_graph)
                return left[:n], right[:n], stats
            except CapacityError as e:
                cap = max(e.required, 1)
        raise RuntimeError("pair buffer sizing did not converge")

    def close(self):
        if getattr(self, "handle", None):
            load().vs_batch_plan_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wkb_decode(ctx: Context, data, offsets, valid=None):
    """Decode WKB rows on the device (see vs_wkb_plan_create).

    ``data``: uint8 CUDA tensor of the concatenated WKB values, ``offsets``:
    int64 CUDA tensor of n + 1 byte offsets, ``valid``: optional uint8 CUDA
    tensor.  Returns (sizes dict, dict of CUDA tensors tags, px, py,
    geom_off, part_off, ring_off, x, y).
    """
    import torch

    n = int(offsets.numel()) - 1
    dev = offsets.device
    out = dict(tags=torch.empty(n, dtype=torch.int8, device=dev),
               px=torch.empty(n, dtype=torch.float64, device=dev),
               py=torch.empty(n, dtype=torch.float64, device=dev),
               geom_off=torch.empty(n + 1, dtype=torch.int32, device=dev))
    rows = WkbOut(_ptr(out["tags"]), _ptr(out["px"]), _ptr(out["py"]), _ptr(out["geom_off"]), None, None, None, None)
    sizes = WkbSizes()
    h = ctypes.c_void_p()
    check(load().vs_wkb_plan_create(ctx.handle, _ptr(data), _ptr(offsets), _ptr(valid), n, ctypes.byref(rows),
                                    ctypes.byref(h), ctypes.byref(sizes)))
    try:
        sz = sizes.as_dict()
        out.update(part_off=torch.empty(sz["n_parts"] + 1, dtype=torch.int32, device=dev),
                   ring_off=torch.empty(sz["n_rings"] + 1, dtype=torch.int32, device=dev),
                   x=torch.empty(sz["n_coords"], dtype=torch.float64, device=dev),
                   y=torch.empty(sz["n_coords"], dtype=torch.float64, device=dev))
        o = WkbOut(*[_ptr(out[k]) for k in ("tags", "px", "py", "geom_off", "part_off", "ring_off", "x", "y")])
        check(load().vs_wkb_plan_decode(h, ctypes.byref(o)))
        return sz, out
    finally:
        load().vs_wkb_plan_free(h)


HOW_CODES = {"inner": 0, "left": 1, "right": 2, "outer": 3}


def point_index(ctx: Context, x, y, valid=None) -> "DeviceIndex":
    """An index over points (float64 CUDA tensors) for vs_join_nearest_polygons:
    each point a polygon of one ring of one vertex."""
    import torch

    n = int(x.numel())
    offs = torch.arange(n + 1, dtype=torch.int32, device=x.device)
    P = make_polygons(x, y, offs, offs, offs, valid)
    return DeviceIndex(ctx, P, learned=False)


def nearest_polygons(ctx: Context, point_index: "DeviceIndex", polys: Polygons, *, max_distance: float = float("inf"),
                     sort: bool = True, capacity: int | None = None):
    """vs_join_nearest_polygons: (polygon rows, point rows, distances, stats), CUDA tensors."""
    import torch

    dev = torch.device("cuda", ctx.device)
    cap = int(capacity) if capacity is not None else max(1024, int(polys.n_geoms))
    for _ in range(2):
        left = torch.empty(cap, dtype=torch.int32, device=dev)
        right = torch.empty(cap, dtype=torch.int32, device=dev)
        dist = torch.empty(cap, dtype=torch.float64, device=dev)
        n = ctypes.c_int64(0)
        st = JoinStats()
        status = load().vs_join_nearest_polygons(ctx.handle, point_index.handle, ctypes.byref(polys),
                                                 float(max_distance), JOIN_SORT if sort else 0, _ptr(left),
                                                 _ptr(right), _ptr(dist), cap, ctypes.byref(n), ctypes.byref(st))
        try:
            check(status, required=int(n.value))
        except CapacityError as e:
            cap = max(e.required, 1)
            continue
        k = int(n.value)
        return left[:k], right[:k], dist[:k], st.as_dict()
    raise RuntimeError("pair buffer sizing did not converge")


def join_export(ctx: Context, left, right, n_left: int, n_right: int, how: str, left_code=None, right_code=None):
    """vs_join_export: (left rows, right rows, source pair) int64 CUDA tensors
    of the join's output rows (-1 = no row on that side / an added row).

    ``left``/``right``: int32 CUDA tensors of pairs sorted by (left, right);
    ``left_code``/``right_code``: optional int64 CUDA tensors of attribute
    codes per row (pairs kept where equal; negative codes never match).
    """
    import torch

    dev = left.device
    n = int(left.numel())
    cap = n + int(n_left) + int(n_right)
    out_l = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
    out_r = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
    out_s = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
    m = ctypes.c_int64(0)
    check(load().vs_join_export(ctx.handle, _ptr(left), _ptr(right), n, int(n_left), int(n_right), HOW_CODES[how],
                                _ptr(left_code), _ptr(right_code), _ptr(out_l), _ptr(out_r), _ptr(out_s), cap,
                                ctypes.byref(m)), required=int(m.value))
    k = int(m.value)
    return out_l[:k], out_r[:k], out_s[:k]


def wkb_plan_sizes(ctx: Context, data, offsets, valid, rows) -> dict:
    """Only the plan step of a WKB decode (the size pass): fills the row
    outputs ``rows`` (dict of CUDA tensors tags, px, py, geom_off) and returns
    the sizes; the plan is freed without decoding."""
    n = int(offsets.numel()) - 1
    o = WkbOut(_ptr(rows["tags"]), _ptr(rows["px"]), _ptr(rows["py"]), _ptr(rows["geom_off"]), None, None, None,
               None)
    sizes = WkbSizes()
    h = ctypes.c_void_p()
    check(load().vs_wkb_plan_create(ctx.handle, _ptr(data), _ptr(offsets), _ptr(valid), n, ctypes.byref(o),
                                    ctypes.byref(h), ctypes.byref(sizes)))
    load().vs_wkb_plan_free(h)
    return sizes.as_dict()


def kernel_launches() -> int:
    """Kernels the library has launched from this thread so far."""
    return int(load().vs_thread_kernel_launches())


def distance_aligned(ctx: Context, pts: Points, polys: Polygons, dist, env=None) -> None:
    check(load().vs_distance_aligned(ctx.handle, ctypes.byref(pts), ctypes.byref(polys), _ptr(dist), _ptr(env)))


def locate_aligned(ctx: Context, pts: Points, polys: Polygons, out) -> None:
    check(load().vs_locate_aligned(ctx.handle, ctypes.byref(pts), ctypes.byref(polys), _ptr(out)))


def join_brute_noalloc(pts: Points, polys: Polygons, predicate: int, left, right, stream: int = 0) -> int:
    """Allocation-free brute-force join (see vs_join_brute_noalloc); returns the pair count.

    For callers that cannot allocate device memory: the pairs go to the
    caller's ``left`` / ``right`` buffers and the library's only scratch is a
    fixed device array (at most 65,536 polygons).  Pairs are unordered.
    """
    n = ctypes.c_int64(0)
    cap = 0 if left is None else int(left.numel())
    status = load().vs_join_brute_noalloc(ctypes.byref(pts), ctypes.byref(polys), int(predicate), _ptr(left),
                                          _ptr(right), cap, ctypes.byref(n), ctypes.c_void_p(stream))
    check(status, required=int(n.value))
    return int(n.value)


def _i32_dev(a):
    """The int32 contiguous form of a device row array (no copy when it already is)."""
    import torch

    return a.contiguous() if a.dtype == torch.int32 else a.to(torch.int32).contiguous()


def row_counts(ctx: Context, rows, n_rows: int, mask=None):
    """int64 device tensor: pairs per row 0..n_rows-1, over the pairs where ``mask`` (bool / uint8 device
    tensor) is set when given (vs_row_counts)."""
    import torch

    r = _i32_dev(rows)
    m = None if mask is None else mask.to(torch.uint8).contiguous()
    out = torch.empty(max(int(n_rows), 0), dtype=torch.int64, device=r.device)
    check(load().vs_row_counts(ctx.handle, _ptr(r), _ptr(m), int(r.numel()), int(n_rows), _ptr(out)))
    return out


def row_sums(ctx: Context, rows, cols, values, n_rows: int):
    """float64 device tensor: per row, the sum of values[cols] over its pairs in pair order (rows ascending;
    vs_row_sums)."""
    import torch

    r, c = _i32_dev(rows), _i32_dev(cols)
    v = values.to(device=r.device, dtype=torch.float64).contiguous()
    out = torch.empty(max(int(n_rows), 0), dtype=torch.float64, device=r.device)
    check(load().vs_row_sums(ctx.handle, _ptr(r), _ptr(c), int(r.numel()), int(n_rows), _ptr(v), int(v.numel()),
                             _ptr(out)))
    return out


def select_rows(ctx: Context, counts, matched: bool = True):
    """int32 device tensor: ascending rows whose count is > 0 (matched) or == 0 (vs_select_rows)."""
    import torch

    c = counts.to(torch.int64).contiguous()
    out = torch.empty(max(int(c.numel()), 1), dtype=torch.int32, device=c.device)
    n = ctypes.c_int64(0)
    check(load().vs_select_rows(ctx.handle, _ptr(c), int(c.numel()), 1 if matched else 0, _ptr(out), ctypes.byref(n)))
    return out[:n.value]


def pairs_member(ctx: Context, a_left, a_right, b_left, b_right, n_left_rows: int):
    """bool device tensor: pair k of a is also a pair of b (b sorted by (left, right); vs_pairs_member)."""
    import torch

    al, ar, bl, br = (_i32_dev(t) for t in (a_left, a_right, b_left, b_right))
    flags = torch.empty(max(int(al.numel()), 1), dtype=torch.uint8, device=al.device)
    check(load().vs_pairs_member(ctx.handle, _ptr(al), _ptr(ar), int(al.numel()), _ptr(bl), _ptr(br),
                                 int(bl.numel()), int(n_left_rows), _ptr(flags)))
    return flags[:al.numel()].bool()


def sort_pairs(ctx: Context, left, right) -> None:
    check(load().vs_sort_pairs(ctx.handle, _ptr(left), _ptr(right), int(left.numel())))


def radix_sort_pairs(ctx: Context, keys, vals, key_bits: int = 64) -> None:
    check(load().vs_radix_sort_pairs(ctx.handle, _ptr(keys), _ptr(vals), int(keys.numel()), int(key_bits)))


def hilbert_keys(ctx: Context, x, y, frame, out) -> None:
    minx, miny, maxx, maxy = (float(v) for v in frame)
    check(load().vs_hilbert_keys(ctx.handle, _ptr(x), _ptr(y), int(x.numel()), minx, miny, maxx, maxy, _ptr(out)))


def hilbert_key_host(x: int, y: int, levels: int = 32) -> int:
    """Host restatement of the device Hilbert key (used by tests)."""
    d = 0
    mask = 0xFFFFFFFF
    for lv in range(31, 31 - levels, -1):
        rx = (x >> lv) & 1
        ry = (y >> lv) & 1
        d = (d << 2) | ((3 * rx) ^ ry)
        if ry == 0:
            if rx == 1:
                x = ~x & mask
                y = ~y & mask
            x, y = y, x
    return d


def _np_to_torch(a: np.ndarray, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(device)
