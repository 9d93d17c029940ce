"""cublox_b200 — B200-native map-integration path of cublox's OccupancyGrid.

Python view of the C ABI in include/cublox_b200.h (libcublox_b200.so, built
in-tree for sm_100a).  `OccupancyGrid` mirrors the reference's class
(include/cublox/OccupancyGrid.hpp:29-169): same method names, argument
meaning and defaults; snake_case aliases are provided as well.

There is no CPU fallback: constructing a grid without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes
import enum
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcublox_b200.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_RANGE, ERR_DEVICE, ERR_CANCELLED = -1, -2, -3, -4, -5, -6
LAYOUT_SOA, LAYOUT_AOS = 0, 1
DEPTH_U16_MM, DEPTH_F32_M = 0, 1
OPT_RAYCAST, OPT_CUBE, OPT_MATCH, OPT_SORT, OPT_SEGMENT, OPT_FOLD, OPT_BLOCK, OPT_CONTIGUOUS = (
    1, 2, 3, 4, 5, 6, 7, 8)
OPT_LAYOUT = 9
OPT_FLAT_CUBE = 10
LAYOUTS = (320, 230, 221, 0)  # 8x4x1, 4x8x1, 4x4x2 bricks; the reference's hash order


class VoxelState(enum.IntEnum):
    UNKNOWN = 0
    FREE = 1
    OCCUPIED = 2


class CubloxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class ScanStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_int64), ("op_incs", ctypes.c_int64),
                ("hit_incs", ctypes.c_int64), ("touched", ctypes.c_int64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    """cublox_server_config."""
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_tick_points", ctypes.c_int),
                ("max_tick_maps", ctypes.c_int), ("max_inflight_ticks", ctypes.c_int),
                ("graphs", ctypes.c_int), ("pinned_pool_bytes", ctypes.c_uint64),
                ("max_fetch_centres", ctypes.c_int), ("max_fetch_samples", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    """cublox_server_stats."""
    _fields_ = [("ticks", ctypes.c_int64), ("scans", ctypes.c_int64), ("fetches", ctypes.c_int64),
                ("points", ctypes.c_int64), ("admissions", ctypes.c_int64),
                ("evictions", ctypes.c_int64), ("resident_bytes", ctypes.c_uint64),
                ("peak_resident_bytes", ctypes.c_uint64), ("resident_maps", ctypes.c_int),
                ("cancelled", ctypes.c_int64)]


_lib = None


def lib():
    """Load libcublox_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python cublox_b200/build.py` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        G = ctypes.c_void_p
        f = ctypes.POINTER(ctypes.c_float)
        i = ctypes.POINTER(ctypes.c_int)
        i64 = ctypes.POINTER(ctypes.c_int64)
        u8 = ctypes.POINTER(ctypes.c_uint8)
        sig = {
            "cublox_last_error": ([], ctypes.c_char_p),
            "cublox_version": ([], ctypes.c_char_p),
            "cublox_binary_version": ([i], ctypes.c_int),
            "cublox_grid_create": ([i, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_double, f,
                                    ctypes.c_void_p, ctypes.POINTER(G)], ctypes.c_int),
            "cublox_grid_destroy": ([G], ctypes.c_int),
            "cublox_grid_reset": ([G], ctypes.c_int),
            "cublox_grid_reset_voxel": ([G, ctypes.c_int], ctypes.c_int),
            "cublox_grid_set_max_range": ([G, ctypes.c_float], ctypes.c_int),
            "cublox_grid_get_max_range": ([G, f], ctypes.c_int),
            "cublox_grid_set_log_odds": ([G] + [ctypes.c_float] * 6, ctypes.c_int),
            "cublox_grid_set_fp_mode": ([G, ctypes.c_uint], ctypes.c_int),
            "cublox_grid_get_fp_mode": ([G, ctypes.POINTER(ctypes.c_uint)], ctypes.c_int),
            "cublox_grid_update": ([G, f, f, f, ctypes.c_int, f], ctypes.c_int),
            "cublox_grid_update_xyz": ([G, f, ctypes.c_int, ctypes.c_int, f], ctypes.c_int),
            "cublox_grid_recenter": ([G, f, i], ctypes.c_int),
            "cublox_grid_set_recenter_mode": ([G, ctypes.c_int], ctypes.c_int),
            "cublox_grid_fetch": ([G, f, ctypes.c_float, ctypes.c_int, ctypes.c_int, f, u8, ctypes.c_int64,
                                   i64], ctypes.c_int),
            "cublox_grid_fetch_batch": ([G, f, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int, i64,
                                         f, u8, ctypes.c_int64], ctypes.c_int),
            "cublox_grid_fetch_counts": ([G, f, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                          i64], ctypes.c_int),
            "cublox_grid_query_states": ([G, f, ctypes.c_int, u8], ctypes.c_int),
            "cublox_grid_stored_at": ([G, ctypes.c_int, f], ctypes.c_int),
            "cublox_grid_origin": ([G, i, f], ctypes.c_int),
            "cublox_grid_geometry": ([G, i, i, i, f, i], ctypes.c_int),
            "cublox_grid_first_run": ([G, i], ctypes.c_int),
            "cublox_grid_set_origin_index": ([G, i], ctypes.c_int),
            "cublox_grid_export": ([G, f], ctypes.c_int),
            "cublox_grid_import": ([G, f], ctypes.c_int),
            "cublox_grid_stream": ([G, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
            "cublox_grid_synchronize": ([G], ctypes.c_int),
            "cublox_grid_enable_stats": ([G, ctypes.c_int], ctypes.c_int),
            "cublox_grid_last_stats": ([G, ctypes.POINTER(ScanStats)], ctypes.c_int),
            "cublox_grid_check": ([G, ctypes.POINTER(ctypes.c_uint32)], ctypes.c_int),
            "cublox_grid_count_scan": ([G, f, ctypes.c_int, f, i, i], ctypes.c_int),
            "cublox_grid_last_clear": ([G, i64], ctypes.c_int),
            "cublox_grid_update_pose": ([G, f, ctypes.c_int, ctypes.c_int, f, f], ctypes.c_int),
            "cublox_grid_fetch_viz": ([G, f, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_int64, f, f, ctypes.c_int64, i64],
                                      ctypes.c_int),
            "cublox_grid_update_depth": ([G, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int64, f, f, f], ctypes.c_int),
            "cublox_batch_create": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
            "cublox_batch_destroy": ([ctypes.c_void_p], ctypes.c_int),
            "cublox_batch_add_grid": ([ctypes.c_void_p, i, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, f, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
            "cublox_batch_set_option": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "cublox_batch_get_option": ([ctypes.c_void_p, ctypes.c_int, i], ctypes.c_int),
            "cublox_batch_update": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), f, i64, f],
                                    ctypes.c_int),
            "cublox_batch_recenter": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), f, i],
                                      ctypes.c_int),
            "cublox_batch_synchronize": ([ctypes.c_void_p], ctypes.c_int),
            "cublox_batch_last_timing": ([ctypes.c_void_p, f, f], ctypes.c_int),
            "cublox_batch_stream": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
            "cublox_server_create": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)],
                                     ctypes.c_int),
            "cublox_server_destroy": ([ctypes.c_void_p], ctypes.c_int),
            "cublox_server_add_map": ([ctypes.c_void_p, i, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, f, ctypes.c_float, f, i], ctypes.c_int),
            "cublox_server_submit_scan": ([ctypes.c_void_p, ctypes.c_int, f, ctypes.c_int, f, ctypes.c_int,
                                           i64], ctypes.c_int),
            "cublox_server_submit_fetch": ([ctypes.c_void_p, ctypes.c_int, f, ctypes.c_int, ctypes.c_float,
                                            ctypes.c_int, ctypes.c_int, i64], ctypes.c_int),
            "cublox_server_wait": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, i], ctypes.c_int),
            "cublox_server_drain": ([ctypes.c_void_p], ctypes.c_int),
            "cublox_server_request_times": ([ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
            "cublox_server_fetch_result": ([ctypes.c_void_p, ctypes.c_int64, i64, f,
                                            ctypes.POINTER(ctypes.c_uint8), ctypes.c_int64, i64], ctypes.c_int),
            "cublox_server_release": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
            "cublox_server_export": ([ctypes.c_void_p, ctypes.c_int, f, i], ctypes.c_int),
            "cublox_server_get_stats": ([ctypes.c_void_p, ctypes.POINTER(ServerStats)], ctypes.c_int),
            "cublox_server_cancel": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
            "cublox_server_scratch_bytes": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_uint64)],
                                            ctypes.c_int),
            "cublox_runtime_counters": ([i64, ctypes.c_int], ctypes.c_int),
            "cublox_test_fail_allocations": ([ctypes.c_int64, ctypes.c_int64], ctypes.c_int),
            "cublox_probe_red_rate": ([ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
            "cublox_batch_reserve_maps": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64],
                                          ctypes.c_int),
            "cublox_grid_enable_timing": ([G, ctypes.c_int], ctypes.c_int),
            "cublox_grid_set_option": ([G, ctypes.c_int, ctypes.c_int], ctypes.c_int),
            "cublox_grid_get_option": ([G, ctypes.c_int, i], ctypes.c_int),
            "cublox_grid_last_timing": ([G, f], ctypes.c_int),
            "cublox_grid_reference_steps": ([G, f, ctypes.c_int, f, i64], ctypes.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != OK:
        msg = lib().cublox_last_error().decode(errors="replace")
        raise CubloxError(rc, f"{what}: {msg}")


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f3(v):
    return (ctypes.c_float * 3)(*[float(x) for x in v])


def _dev_ptr(obj):
    """Device pointer of a CUDA array-like (torch tensor or
    __cuda_array_interface__), else None."""
    if hasattr(obj, "__cuda_array_interface__"):
        return obj.__cuda_array_interface__["data"][0]
    if hasattr(obj, "is_cuda") and getattr(obj, "is_cuda"):
        return obj.data_ptr()
    return None


class OccupancyGrid:
    """Drop-in for cublox::OccupancyGrid (OccupancyGrid.hpp:29-169)."""

    VoxelState = VoxelState

    def __init__(self, half_map_size_i, resolution: float, origin_at_center: bool = False,
                 recenter_threshold: float | None = None, origin=(0.0, 0.0, 0.0), stream=None,
                 _handle=None):
        L = lib()
        if _handle is None:
            h = ctypes.c_void_p()
            rc = L.cublox_grid_create((ctypes.c_int * 3)(*[int(v) for v in half_map_size_i]),
                                      float(resolution), int(bool(origin_at_center)),
                                      int(recenter_threshold is not None),
                                      float(recenter_threshold or 0.0), _f3(origin),
                                      ctypes.c_void_p(stream or 0), ctypes.byref(h))
            _check(rc, "OccupancyGrid")
            self._owned = True
        else:
            h = _handle
            self._owned = False
        self._h = h
        m = (ctypes.c_int * 3)()
        hf = (ctypes.c_int * 3)()
        vn = ctypes.c_int()
        res = ctypes.c_float()
        oc = ctypes.c_int()
        _check(L.cublox_grid_geometry(h, m, hf, ctypes.byref(vn), ctypes.byref(res), ctypes.byref(oc)),
               "geometry")
        self.map_size_i = tuple(m)
        self.half_map_size_i = tuple(hf)
        self.voxel_num = vn.value
        self.resolution = res.value
        self.resolution_inv = np.float32(1.0) / np.float32(self.resolution)
        self.origin_at_center = bool(oc.value)
        self.recenter_threshold = recenter_threshold
        self.l_params = dict(l_hit=0.847, l_miss=-0.405, l_min=-1.992, l_max=3.476,
                             l_free=-0.0004, l_occupied=1.7346)

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                lib().cublox_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- configuration (OccupancyGrid.hpp:68-85) ----
    def setMaxRaycastRange(self, r: float):
        _check(lib().cublox_grid_set_max_range(self._h, float(r)), "setMaxRaycastRange")

    def getMaxRaycastRange(self) -> float:
        v = ctypes.c_float()
        _check(lib().cublox_grid_get_max_range(self._h, ctypes.byref(v)), "getMaxRaycastRange")
        return v.value

    def setLogOddsParams(self, l_hit, l_miss, l_min, l_max, l_free, l_occupied):
        _check(lib().cublox_grid_set_log_odds(self._h, l_hit, l_miss, l_min, l_max, l_free,
                                              l_occupied), "setLogOddsParams")
        self.l_params = dict(l_hit=l_hit, l_miss=l_miss, l_min=l_min, l_max=l_max, l_free=l_free,
                             l_occupied=l_occupied)

    def set_fp_mode(self, mode: int):
        _check(lib().cublox_grid_set_fp_mode(self._h, int(mode)), "set_fp_mode")

    def fp_mode(self) -> int:
        v = ctypes.c_uint()
        _check(lib().cublox_grid_get_fp_mode(self._h, ctypes.byref(v)), "fp_mode")
        return v.value

    def set_recenter_mode(self, mode: int):
        _check(lib().cublox_grid_set_recenter_mode(self._h, int(mode)), "set_recenter_mode")

    # ---- path ----
    def update(self, cloud, sensor_origin):
        """update(cloud, sensor_origin) — OccupancyGrid.cpp:181-238.

        `cloud`: (N, 3) float32 host array (any order; copied), or a CUDA
        (N, 3) row-major tensor, or a CUDA (3, N) tensor (SoA)."""
        so = _f3(sensor_origin)
        ptr = _dev_ptr(cloud)
        if ptr is not None:
            shape = tuple(cloud.shape)
            if len(shape) != 2 or 3 not in shape:
                raise ValueError("device cloud must be (N, 3) or (3, N)")
            if shape[1] == 3 and shape[0] != 3:
                layout, n = LAYOUT_AOS, shape[0]
            else:
                layout, n = LAYOUT_SOA, shape[1]
            rc = lib().cublox_grid_update_xyz(self._h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)),
                                              layout, int(n), so)
            _check(rc, "update")
            return
        p = np.asarray(cloud, dtype=np.float32)
        if p.ndim != 2 or p.shape[1] != 3:
            raise ValueError("cloud must be (N, 3)")
        p = np.ascontiguousarray(p)
        _check(lib().cublox_grid_update_xyz(self._h, _fp(p), LAYOUT_AOS, p.shape[0], so), "update")

    def update_soa(self, x, y, z, sensor_origin):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        z = np.ascontiguousarray(z, dtype=np.float32)
        _check(lib().cublox_grid_update(self._h, _fp(x), _fp(y), _fp(z), x.shape[0],
                                        _f3(sensor_origin)), "update")

    def recenter(self, pos) -> int:
        """recenter(pos) — OccupancyGrid.cpp:141-179.  Returns the action."""
        a = ctypes.c_int(0)
        _check(lib().cublox_grid_recenter(self._h, _f3(pos), ctypes.byref(a)), "recenter")
        return a.value

    def fetchOccupancyAround(self, center, radius: float, state_filter=None, max_results: int = 0):
        """fetchOccupancyAround — OccupancyGrid.cpp:240-356.

        Returns (positions (n, 3) float32, states (n,) uint8), ordered by
        ascending (x, y, z) global voxel index."""
        flt = -1 if state_filter is None else int(state_filter)
        c = _f3(center)
        counts = np.zeros(1, dtype=np.int64)
        _check(lib().cublox_grid_fetch_counts(self._h, c, 1, float(radius), flt, int(max_results),
                                              counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
               "fetchOccupancyAround")
        n = int(counts[0])
        pos = np.empty((max(n, 1), 3), dtype=np.float32)
        st = np.empty(max(n, 1), dtype=np.uint8)
        got = ctypes.c_int64(0)
        _check(lib().cublox_grid_fetch(self._h, c, float(radius), flt, int(max_results), _fp(pos),
                                       st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n,
                                       ctypes.byref(got)), "fetchOccupancyAround")
        return pos[: got.value], st[: got.value]

    def fetch_batch(self, centers, radius: float, state_filter=None, max_results: int = 0):
        """All centres in one launch: (offsets (n+1,), positions, states)."""
        flt = -1 if state_filter is None else int(state_filter)
        c = np.ascontiguousarray(np.asarray(centers, dtype=np.float32).reshape(-1, 3))
        nq = c.shape[0]
        counts = np.zeros(max(nq, 1), dtype=np.int64)
        _check(lib().cublox_grid_fetch_counts(self._h, _fp(c), nq, float(radius), flt, int(max_results),
                                              counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
               "fetch_batch")
        total = int(counts[:nq].sum())
        off = np.zeros(nq + 1, dtype=np.int64)
        pos = np.empty((max(total, 1), 3), dtype=np.float32)
        st = np.empty(max(total, 1), dtype=np.uint8)
        _check(lib().cublox_grid_fetch_batch(self._h, _fp(c), nq, float(radius), flt, int(max_results),
                                             off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _fp(pos),
                                             st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), total),
               "fetch_batch")
        return off, pos[:total], st[:total]

    def fetch_viz(self, center, radius: float, state_filter=None, max_results: int = 0,
                  subsample_step: int = 1, max_viz_radius: float = 25.0, max_points: int = 200000,
                  robot_pos=None) -> np.ndarray:
        """The driver's visualisation cloud of one fetch: (n, 4) float32
        rows x, y, z, rgb (rgb's bits are 0x00RRGGBB)."""
        flt = -1 if state_filter is None else int(state_filter)
        rp = center if robot_pos is None else robot_pos
        out = np.empty((max(int(max_points), 1), 4), dtype=np.float32)
        n = ctypes.c_int64()
        _check(lib().cublox_grid_fetch_viz(self._h, _f3(center), float(radius), flt, int(max_results),
                                           int(subsample_step), float(max_viz_radius), int(max_points),
                                           _f3(rp), _fp(out), out.shape[0], ctypes.byref(n)),
               "fetch_viz")
        return out[: n.value]

    def fetch_counts(self, centers, radius: float, state_filter=None, max_results: int = 0):
        flt = -1 if state_filter is None else int(state_filter)
        c = np.ascontiguousarray(np.asarray(centers, dtype=np.float32).reshape(-1, 3))
        out = np.zeros(max(c.shape[0], 1), dtype=np.int64)
        _check(lib().cublox_grid_fetch_counts(self._h, _fp(c), c.shape[0], float(radius), flt,
                                              int(max_results),
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
               "fetch_counts")
        return out[: c.shape[0]]

    # ---- queries (OccupancyGrid.cpp:358-429) ----
    def query_states(self, points) -> np.ndarray:
        p = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1, 3))
        out = np.empty(max(p.shape[0], 1), dtype=np.uint8)
        _check(lib().cublox_grid_query_states(self._h, _fp(p), p.shape[0],
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))),
               "query_states")
        return out[: p.shape[0]]

    def isOccupied(self, pos) -> bool:
        return int(self.query_states([pos])[0]) == VoxelState.OCCUPIED

    def isFree(self, pos) -> bool:
        return int(self.query_states([pos])[0]) == VoxelState.FREE

    def isUnknown(self, pos) -> bool:
        return int(self.query_states([pos])[0]) == VoxelState.UNKNOWN

    def storedAt(self, hash_id: int) -> float:
        v = ctypes.c_float()
        _check(lib().cublox_grid_stored_at(self._h, int(hash_id), ctypes.byref(v)), "storedAt")
        return v.value

    # ---- Grid (Grid.hpp:22-57) ----
    def getOriginIndex(self):
        o = (ctypes.c_int * 3)()
        of = (ctypes.c_float * 3)()
        _check(lib().cublox_grid_origin(self._h, o, of), "getOriginIndex")
        return tuple(o)

    def getOriginPosition(self):
        o = (ctypes.c_int * 3)()
        of = (ctypes.c_float * 3)()
        _check(lib().cublox_grid_origin(self._h, o, of), "getOriginPosition")
        return tuple(of)

    def first_run(self) -> bool:
        v = ctypes.c_int()
        _check(lib().cublox_grid_first_run(self._h, ctypes.byref(v)), "first_run")
        return bool(v.value)

    def set_origin_index(self, o):
        _check(lib().cublox_grid_set_origin_index(self._h, (ctypes.c_int * 3)(*[int(v) for v in o])),
               "set_origin_index")

    def reset(self):
        _check(lib().cublox_grid_reset(self._h), "reset")

    def resetVoxel(self, hash_id: int):
        _check(lib().cublox_grid_reset_voxel(self._h, int(hash_id)), "resetVoxel")

    # ---- state transfer ----
    def export(self) -> np.ndarray:
        out = np.empty(self.voxel_num, dtype=np.float32)
        _check(lib().cublox_grid_export(self._h, _fp(out)), "export")
        return out

    def import_(self, occ):
        a = np.ascontiguousarray(occ, dtype=np.float32)
        if a.size != self.voxel_num:
            raise ValueError("occ must hold voxel_num floats")
        _check(lib().cublox_grid_import(self._h, _fp(a)), "import")

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().cublox_grid_stream(self._h, ctypes.byref(s)), "stream")
        return s.value or 0

    def synchronize(self):
        _check(lib().cublox_grid_synchronize(self._h), "synchronize")

    def enable_stats(self, on: bool = True):
        _check(lib().cublox_grid_enable_stats(self._h, int(on)), "enable_stats")

    def last_stats(self) -> dict:
        s = ScanStats()
        _check(lib().cublox_grid_last_stats(self._h, ctypes.byref(s)), "last_stats")
        return s.as_dict()

    def count_scan(self, cloud, sensor_origin):
        """Per-voxel (op, hit) counts of one scan, without folding them."""
        p = np.ascontiguousarray(np.asarray(cloud, dtype=np.float32).reshape(-1, 3))
        op = np.empty(self.voxel_num, dtype=np.int32)
        hit = np.empty(self.voxel_num, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        _check(lib().cublox_grid_count_scan(self._h, _fp(p), p.shape[0], _f3(sensor_origin),
                                            op.ctypes.data_as(ip), hit.ctypes.data_as(ip)),
               "count_scan")
        return op, hit

    def set_option(self, key: int, value: int):
        _check(lib().cublox_grid_set_option(self._h, int(key), int(value)), "set_option")

    def get_option(self, key: int) -> int:
        v = ctypes.c_int()
        _check(lib().cublox_grid_get_option(self._h, int(key), ctypes.byref(v)), "get_option")
        return v.value

    def enable_timing(self, on: bool = True):
        _check(lib().cublox_grid_enable_timing(self._h, int(on)), "enable_timing")

    def last_timing(self):
        """Device ms of the last (raycast, fold, recenter clear); -1 = none."""
        ms = (ctypes.c_float * 3)()
        _check(lib().cublox_grid_last_timing(self._h, ms), "last_timing")
        return tuple(ms)

    def last_clear(self) -> int:
        """Voxels the last recenter cleared."""
        v = ctypes.c_int64()
        _check(lib().cublox_grid_last_clear(self._h, ctypes.byref(v)), "last_clear")
        return v.value

    def reference_steps(self, cloud, sensor_origin) -> int:
        """The reference's work units for one scan (DDA iterations + endpoint)."""
        p = np.ascontiguousarray(np.asarray(cloud, dtype=np.float32).reshape(-1, 3))
        v = ctypes.c_int64()
        _check(lib().cublox_grid_reference_steps(self._h, _fp(p), p.shape[0], _f3(sensor_origin),
                                                 ctypes.byref(v)), "reference_steps")
        return v.value

    def update_pose(self, cloud_sensor, rotation, translation):
        """update() from a sensor-frame (N, 3) cloud (host array or CUDA
        tensor) and the sensor pose (3x3 rotation, translation): the
        reference driver's range filter and transform run on the device."""
        R = np.ascontiguousarray(np.asarray(rotation, dtype=np.float32).reshape(9))
        t = np.ascontiguousarray(np.asarray(translation, dtype=np.float32).reshape(3))
        dp = _dev_ptr(cloud_sensor)
        if dp is not None:
            n = int(cloud_sensor.shape[0])
            ptr = ctypes.cast(dp, ctypes.POINTER(ctypes.c_float))
        else:
            p = np.ascontiguousarray(np.asarray(cloud_sensor, dtype=np.float32).reshape(-1, 3))
            n, ptr = p.shape[0], _fp(p)
        _check(lib().cublox_grid_update_pose(self._h, ptr, LAYOUT_AOS, n, _fp(R), _fp(t)), "update_pose")

    def update_depth(self, image, intrinsics, rotation, translation):
        """update() from an (H, W) depth image — uint16 millimetres
        (16UC1) or float32 metres (32FC1), host array or CUDA tensor — with
        intrinsics (fx, fy, cx, cy) and the camera pose, as the reference
        driver's depthCallback + buildCloudInOdomFrame do."""
        K = np.ascontiguousarray(np.asarray(intrinsics, dtype=np.float32).reshape(4))
        R = np.ascontiguousarray(np.asarray(rotation, dtype=np.float32).reshape(9))
        t = np.ascontiguousarray(np.asarray(translation, dtype=np.float32).reshape(3))
        dp = _dev_ptr(image)
        if dp is not None:
            h, w = int(image.shape[0]), int(image.shape[1])
            es = image.element_size()
            enc = DEPTH_U16_MM if es == 2 else DEPTH_F32_M
            step, ptr, keep = int(image.stride(0)) * es, dp, None
        else:
            keep = np.asarray(image)
            if keep.dtype not in (np.uint16, np.float32):
                keep = keep.astype(np.float32)
            if keep.strides[1] != keep.itemsize:
                keep = np.ascontiguousarray(keep)
            h, w = keep.shape
            enc = DEPTH_U16_MM if keep.dtype == np.uint16 else DEPTH_F32_M
            step, ptr = keep.strides[0], keep.ctypes.data
        _check(lib().cublox_grid_update_depth(self._h, ctypes.c_void_p(ptr), enc, w, h, step, _fp(K),
                                              _fp(R), _fp(t)), "update_depth")
        del keep

    def update_ptr(self, ptr: int, n: int, sensor_origin, layout: int = LAYOUT_SOA):
        """update() from a raw pointer (device, pinned or pageable host)."""
        _check(lib().cublox_grid_update_xyz(self._h, ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)),
                                            layout, int(n), _f3(sensor_origin)), "update")

    def check(self) -> int:
        w = ctypes.c_uint32()
        _check(lib().cublox_grid_check(self._h, ctypes.byref(w)), "check")
        return w.value

    # snake_case aliases
    set_max_raycast_range = setMaxRaycastRange
    get_max_raycast_range = getMaxRaycastRange
    set_log_odds_params = setLogOddsParams
    fetch_occupancy_around = fetchOccupancyAround
    is_occupied = isOccupied
    is_free = isFree
    is_unknown = isUnknown
    stored_at = storedAt
    get_origin_index = getOriginIndex
    get_origin_position = getOriginPosition
    reset_voxel = resetVoxel


BATCH_OPT_GRAPHS, BATCH_OPT_AUTOTUNE, BATCH_OPT_SHAPE, BATCH_OPT_TIMING, BATCH_OPT_NUM_SHAPES = 1, 2, 3, 4, 5
BATCH_OPT_FOLD = 6
BATCH_OPT_TUNING = 7
BATCH_OPT_LAYOUT = 8
BATCH_OPT_WAIT_LIMIT, BATCH_OPT_INJECT_MISSING_WALK = 9, 10
BATCH_OPT_HOST_READ = 11
DEVICE_WAIT_TIMEOUT = 1 << 3


class Batch:
    """Many grids integrated together (cublox_batch_*): one walk launch and
    one fold launch per update, optional CUDA-graph replay, online choice of
    the launch shape.  Grids made by add_grid belong to the batch."""

    def __init__(self, stream=None):
        self._b = ctypes.c_void_p()
        _check(lib().cublox_batch_create(ctypes.c_void_p(stream or 0), ctypes.byref(self._b)),
               "Batch")
        self.grids = []

    def close(self):
        if getattr(self, "_b", None):
            for g in self.grids:
                g._h = None
            lib().cublox_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_grid(self, half_map_size_i, resolution, origin_at_center=False,
                 recenter_threshold=None, origin=(0.0, 0.0, 0.0)) -> OccupancyGrid:
        h = ctypes.c_void_p()
        _check(lib().cublox_batch_add_grid(self._b, (ctypes.c_int * 3)(*[int(v) for v in half_map_size_i]),
                                           float(resolution), int(bool(origin_at_center)),
                                           int(recenter_threshold is not None),
                                           float(recenter_threshold or 0.0), _f3(origin),
                                           ctypes.byref(h)), "add_grid")
        g = OccupancyGrid(half_map_size_i, resolution, origin_at_center, recenter_threshold, origin,
                          _handle=h)
        self.grids.append(g)
        return g

    def set_option(self, key, value):
        _check(lib().cublox_batch_set_option(self._b, int(key), int(value)), "batch set_option")

    def get_option(self, key) -> int:
        v = ctypes.c_int()
        _check(lib().cublox_batch_get_option(self._b, int(key), ctypes.byref(v)), "batch get_option")
        return v.value

    def tuning(self) -> bool:
        """True while the launch-shape tuner is still timing candidates."""
        return bool(self.get_option(BATCH_OPT_TUNING))

    def update(self, grids, clouds, sensors, offsets=None):
        """One scan into each grid.  `clouds`: a list of (N_i, 3) float32 host
        arrays, or one concatenated (sum N_i, 3) host array / CUDA tensor with
        `offsets` (n+1 int64)."""
        n = len(grids)
        handles = (ctypes.c_void_p * n)(*[g._h.value if isinstance(g._h, ctypes.c_void_p) else g._h
                                           for g in grids])
        if offsets is None:
            arrs = [np.ascontiguousarray(np.asarray(c, dtype=np.float32).reshape(-1, 3)) for c in clouds]
            offsets = np.zeros(n + 1, dtype=np.int64)
            offsets[1:] = np.cumsum([a.shape[0] for a in arrs])
            xyz = np.ascontiguousarray(np.concatenate(arrs, axis=0)) if arrs else np.zeros((0, 3), np.float32)
            ptr = _fp(xyz)
        else:
            offsets = np.ascontiguousarray(offsets, dtype=np.int64)
            dp = _dev_ptr(clouds)
            if dp is not None:
                ptr = ctypes.cast(dp, ctypes.POINTER(ctypes.c_float))
            else:
                xyz = np.ascontiguousarray(np.asarray(clouds, dtype=np.float32))
                ptr = _fp(xyz)
        so = np.ascontiguousarray(np.asarray(sensors, dtype=np.float32).reshape(-1, 3))
        _check(lib().cublox_batch_update(self._b, n, handles, ptr,
                                         offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _fp(so)),
               "batch update")

    def recenter(self, grids, positions):
        n = len(grids)
        handles = (ctypes.c_void_p * n)(*[g._h.value if isinstance(g._h, ctypes.c_void_p) else g._h
                                           for g in grids])
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
        acts = np.zeros(max(n, 1), dtype=np.int32)
        _check(lib().cublox_batch_recenter(self._b, n, handles, _fp(pos),
                                           acts.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "batch recenter")
        return acts[:n]

    def synchronize(self):
        _check(lib().cublox_batch_synchronize(self._b), "batch synchronize")

    def last_timing(self):
        a = ctypes.c_float()
        b = ctypes.c_float()
        _check(lib().cublox_batch_last_timing(self._b, ctypes.byref(a), ctypes.byref(b)), "batch timing")
        return a.value, b.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().cublox_batch_stream(self._b, ctypes.byref(s)), "batch stream")
        return s.value or 0


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Server:
    """The served form (cublox_server_*): many robots' maps kept on the
    device under an HBM budget, scans and fetches submitted from any thread
    and integrated in continuously formed batches by a worker thread."""

    def __init__(self, hbm_budget_bytes: int = 120 << 30, max_tick_points: int = 1 << 20,
                 max_tick_maps: int = 0, max_inflight_ticks: int = 2, graphs: bool = False,
                 pinned_pool_bytes: int = 0, max_fetch_centres: int = 0, max_fetch_samples: int = 0):
        cfg = ServerConfig(int(hbm_budget_bytes), int(max_tick_points), int(max_tick_maps),
                           int(max_inflight_ticks), int(bool(graphs)), int(pinned_pool_bytes),
                           int(max_fetch_centres), int(max_fetch_samples))
        self._s = ctypes.c_void_p()
        _check(lib().cublox_server_create(ctypes.byref(cfg), ctypes.byref(self._s)), "Server")
        self.maps = []

    def close(self):
        if getattr(self, "_s", None):
            lib().cublox_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_map(self, half_map_size_i, resolution, origin_at_center=False, recenter_threshold=None,
                origin=(0.0, 0.0, 0.0), max_range=25.0, log_odds=None) -> int:
        mid = ctypes.c_int()
        lo = None if log_odds is None else (ctypes.c_float * 6)(*[float(v) for v in log_odds])
        _check(lib().cublox_server_add_map(self._s, (ctypes.c_int * 3)(*[int(v) for v in half_map_size_i]),
                                           float(resolution), int(bool(origin_at_center)),
                                           int(recenter_threshold is not None),
                                           float(recenter_threshold or 0.0), _f3(origin), float(max_range),
                                           lo, ctypes.byref(mid)), "add_map")
        self.maps.append(mid.value)
        return mid.value

    def submit_scan(self, map_id: int, points, sensor_origin, recenter: bool = True) -> int:
        p = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1, 3))
        rid = ctypes.c_int64()
        _check(lib().cublox_server_submit_scan(self._s, int(map_id), _fp(p), p.shape[0], _f3(sensor_origin),
                                               int(bool(recenter)), ctypes.byref(rid)), "submit_scan")
        return rid.value

    def submit_fetch(self, map_id: int, centers, radius: float, state_filter=None,
                     max_results: int = 0) -> int:
        c = np.ascontiguousarray(np.asarray(centers, dtype=np.float32).reshape(-1, 3))
        rid = ctypes.c_int64()
        flt = -1 if state_filter is None else int(state_filter)
        _check(lib().cublox_server_submit_fetch(self._s, int(map_id), _fp(c), c.shape[0], float(radius), flt,
                                                int(max_results), ctypes.byref(rid)), "submit_fetch")
        return rid.value

    def wait(self, request_id: int, timeout_s: float = -1.0) -> int:
        st = ctypes.c_int()
        _check(lib().cublox_server_wait(self._s, int(request_id), float(timeout_s), ctypes.byref(st)),
               "wait")
        return st.value

    def drain(self):
        _check(lib().cublox_server_drain(self._s), "drain")

    def times(self, request_id: int):
        """(submission-to-start ms, submission-to-done ms) of a finished request."""
        q, l = ctypes.c_double(), ctypes.c_double()
        _check(lib().cublox_server_request_times(self._s, int(request_id), ctypes.byref(q), ctypes.byref(l)),
               "request_times")
        return q.value, l.value

    def fetch_result(self, request_id: int, n_centers: int):
        """(offsets (n+1,), positions, states) of a finished fetch."""
        n = ctypes.c_int64()
        off = np.zeros(n_centers + 1, dtype=np.int64)
        L = lib()
        _check(L.cublox_server_fetch_result(self._s, int(request_id),
                                            off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), None, None, 0,
                                            ctypes.byref(n)), "fetch_result")
        pos = np.empty((max(n.value, 1), 3), dtype=np.float32)
        st = np.empty(max(n.value, 1), dtype=np.uint8)
        _check(L.cublox_server_fetch_result(self._s, int(request_id),
                                            off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _fp(pos),
                                            st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n.value,
                                            ctypes.byref(n)), "fetch_result")
        return off, pos[: n.value], st[: n.value]

    def release(self, request_id: int):
        _check(lib().cublox_server_release(self._s, int(request_id)), "release")

    def export(self, map_id: int, voxel_num: int):
        """(stored log-odds (voxel_num,), window origin index) after draining."""
        occ = np.empty(voxel_num, dtype=np.float32)
        o = (ctypes.c_int * 3)()
        _check(lib().cublox_server_export(self._s, int(map_id), _fp(occ), o), "server export")
        return occ, tuple(o)

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().cublox_server_get_stats(self._s, ctypes.byref(st)), "server stats")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def cancel(self, request_id: int):
        """Withdraw a request still queued (it ends FAILED, ERR_CANCELLED)."""
        _check(lib().cublox_server_cancel(self._s, int(request_id)), "cancel")

    @staticmethod
    def scratch_bytes(max_tick_points: int = 1 << 20, max_fetch_centres: int = 0,
                      max_fetch_samples: int = 0) -> int:
        """Device bytes a server holds besides its maps (the least budget)."""
        cfg = ServerConfig(0, int(max_tick_points), 0, 0, 0, 0, int(max_fetch_centres),
                           int(max_fetch_samples))
        v = ctypes.c_uint64()
        _check(lib().cublox_server_scratch_bytes(ctypes.byref(cfg), ctypes.byref(v)), "scratch_bytes")
        return v.value


def red_rate(buffer_bytes: int, total_ops: int = 1 << 30, stream: int = 0) -> float:
    """Atomic adds per second (results unused) to distinct pseudo-random
    addresses of a buffer_bytes buffer (cublox_probe_red_rate)."""
    v = ctypes.c_double()
    _check(lib().cublox_probe_red_rate(int(buffer_bytes), int(total_ops), ctypes.c_void_p(stream),
                                       ctypes.byref(v)), "probe_red_rate")
    return v.value


COUNTER_NAMES = ("device_allocs", "device_frees", "pinned_allocs", "pinned_frees", "graph_builds")


def fail_allocations(skip: int, count: int):
    """Test hook (cublox_test_fail_allocations): after `skip` more device or
    pinned allocations, the next `count` fail as if memory were exhausted;
    count 0 turns it off."""
    _check(lib().cublox_test_fail_allocations(int(skip), int(count)), "test_fail_allocations")


def runtime_counters() -> dict:
    """Process-wide counts of this library's allocations, frees and CUDA
    graph builds (cublox_runtime_counters)."""
    out = (ctypes.c_int64 * len(COUNTER_NAMES))()
    _check(lib().cublox_runtime_counters(out, len(COUNTER_NAMES)), "runtime_counters")
    return dict(zip(COUNTER_NAMES, list(out)))


_libm = None


def binary_version() -> int:
    """The loaded kernels' binary version on the current device (100 for
    sm_100a)."""
    v = ctypes.c_int(0)
    _check(lib().cublox_binary_version(ctypes.byref(v)), "binary_version")
    return v.value


def logit(p: float) -> float:
    """utils.hpp:185-188 in float32: clamp to [1e-6, 1 - 1e-6], then the C
    library's logf of pc / (1 - pc)."""
    global _libm
    if _libm is None:
        _libm = ctypes.CDLL("libm.so.6")
        _libm.logf.argtypes = [ctypes.c_float]
        _libm.logf.restype = ctypes.c_float
    lo, hi = np.float32(1.0e-6), np.float32(1.0) - np.float32(1.0e-6)
    pc = np.float32(p)
    pc = lo if pc < lo else (hi if hi < pc else pc)
    return float(_libm.logf(float(np.float32(pc / (np.float32(1.0) - pc)))))


def yaml_log_odds():
    """Log-odds of the reference's config/cublox_driver.yaml probabilities
    (hit 0.9, miss 0.49, min 0.12, max 0.98, free 0.499, occupied 0.85)."""
    return tuple(logit(p) for p in (0.9, 0.49, 0.12, 0.98, 0.499, 0.85))


__all__ = ["OccupancyGrid", "Batch", "Server", "VoxelState", "CubloxError", "lib", "logit", "LIB_PATH"]
