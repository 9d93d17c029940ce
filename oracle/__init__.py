"""Checkers for the cublox map-integration path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this package, and only as the checker or the baseline
being compared against.  The product (cublox_b200/) never imports it.

  OracleGrid — ctypes view of libcublox_oracle.so, the CPU restatement of
               the reference's algorithm (cublox_oracle.c).
  RefGrid    — ctypes view of _ref/libcublox_ref.so: the reference's own
               src/kernels.cu built for sm_100a, driven in the sequence of
               its OccupancyGrid host class (ref_glue.cu).  Needs a GPU.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libcublox_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcublox_ref.so")
# The reference arm's inputs: this oracle and the scan synthesiser compiled
# into one library beside the reference harness, so that a process timing
# the reference maps no library of the product.
REF_INPUTS_SO = os.path.join(HERE, "_ref", "libcublox_refinputs.so")
# The reference tree: $CUBLOX_REFERENCE_TREE, else a directory named
# `reference` beside the repository.
REFERENCE_TREE = os.environ.get("CUBLOX_REFERENCE_TREE") or os.path.normpath(
    os.path.join(HERE, "..", "..", "reference"))

# contraction-site selectors, mirrored from cublox_oracle.h
SOS_PLAIN, SOS_FY_FZ, SOS_FX_FZ, SOS_P_FZ, SOS_FY_P, SOS_FX_P = range(6)
FP_RAY_SOS_SHIFT = 0
FP_CLIP_FMA = 1 << 3
FP_BOUND_FMA = 1 << 4
FP_CENTER_FMA = 1 << 5
FP_MISS_FMA = 1 << 6
FP_HIT_FMA = 1 << 7
FP_REC_SOS_SHIFT = 8
FP_FETCH_SOS_SHIFT = 11
FP_FETCH_DFMA = 1 << 14
FP_PINNED = ((SOS_FX_FZ << FP_RAY_SOS_SHIFT) | FP_CENTER_FMA | FP_MISS_FMA | FP_HIT_FMA
             | (SOS_FX_FZ << FP_REC_SOS_SHIFT) | (SOS_FX_FZ << FP_FETCH_SOS_SHIFT))


def fp_mode(ray_sos=SOS_FX_FZ, clip=False, bound=False, center=True, miss=True, hit=True,
            rec_sos=SOS_FX_FZ, fetch_sos=SOS_FX_FZ, fetch_d=False) -> int:
    m = (ray_sos << FP_RAY_SOS_SHIFT) | (rec_sos << FP_REC_SOS_SHIFT) | (fetch_sos << FP_FETCH_SOS_SHIFT)
    m |= FP_CLIP_FMA if clip else 0
    m |= FP_BOUND_FMA if bound else 0
    m |= FP_CENTER_FMA if center else 0
    m |= FP_MISS_FMA if miss else 0
    m |= FP_HIT_FMA if hit else 0
    m |= FP_FETCH_DFMA if fetch_d else 0
    return m


def build(ref: bool | None = None) -> None:
    """Build the oracle (always) and the reference harness (when the
    reference tree is present).  Uses oracle/Makefile."""
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle", "refinputs"])
    if ref is None:
        ref = os.path.isdir(REFERENCE_TREE)
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_TREE}"])


class OrcStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_int64), ("voxel_steps", ctypes.c_int64),
                ("op_incs", ctypes.c_int64), ("hit_incs", ctypes.c_int64),
                ("touched", ctypes.c_int64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class _OrcGrid(ctypes.Structure):
    _fields_ = [
        ("half", ctypes.c_int * 3), ("map", ctypes.c_int * 3), ("voxel_num", ctypes.c_int),
        ("res", ctypes.c_float), ("res_inv", ctypes.c_float), ("origin_at_center", ctypes.c_int),
        ("has_thr", ctypes.c_int), ("thr", ctypes.c_float), ("thr_sq", ctypes.c_float),
        ("origin_i", ctypes.c_int * 3), ("origin_f", ctypes.c_float * 3), ("first_run", ctypes.c_int),
        ("max_range", ctypes.c_float),
        ("l_hit", ctypes.c_float), ("l_miss", ctypes.c_float), ("l_min", ctypes.c_float),
        ("l_max", ctypes.c_float), ("l_free", ctypes.c_float), ("l_occ", ctypes.c_float),
        ("l_unknown", ctypes.c_float), ("fp_mode", ctypes.c_uint),
        ("occ", ctypes.POINTER(ctypes.c_float)), ("op", ctypes.POINTER(ctypes.c_int)),
        ("hit", ctypes.POINTER(ctypes.c_int)),
    ]


_olibs: dict = {}


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def oracle_lib(path: str | None = None):
    """The oracle's C library: libcublox_oracle.so, or the same code in the
    reference arm's inputs library (REF_INPUTS_SO)."""
    path = path or ORACLE_SO
    if path not in _olibs:
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        G = ctypes.POINTER(_OrcGrid)
        f3 = ctypes.POINTER(ctypes.c_float)
        i3 = ctypes.POINTER(ctypes.c_int)
        L.orc_grid_init.argtypes = [G, i3, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_double, f3]
        L.orc_grid_free.argtypes = [G]
        L.orc_grid_reset.argtypes = [G]
        L.orc_set_log_odds.argtypes = [G] + [ctypes.c_float] * 6
        L.orc_set_max_range.argtypes = [G, ctypes.c_float]
        L.orc_set_fp_mode.argtypes = [G, ctypes.c_uint]
        L.orc_set_origin_i.argtypes = [G, i3]
        L.orc_pos_to_global.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_uint]
        L.orc_global_to_local.argtypes = [ctypes.c_int] * 3
        L.orc_local_to_global.argtypes = [ctypes.c_int] * 4
        L.orc_global_to_hash.argtypes = [i3, i3, i3]
        L.orc_hash_to_local.argtypes = [ctypes.c_int, i3, i3, i3]
        L.orc_hash_to_local.restype = None
        L.orc_global_to_pos.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.orc_global_to_pos.restype = ctypes.c_float
        L.orc_logit.argtypes = [ctypes.c_float]
        L.orc_logit.restype = ctypes.c_float
        L.orc_ingest.argtypes = [f3, ctypes.c_int, f3, f3, ctypes.c_float, f3]
        L.orc_ingest.restype = ctypes.c_int
        L.orc_depth_cloud.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_longlong, f3, f3]
        L.orc_depth_cloud.restype = None
        L.orc_viz.argtypes = [f3, ctypes.c_longlong, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                              ctypes.c_float, ctypes.c_longlong, f3, f3]
        L.orc_viz.restype = ctypes.c_longlong
        st = ctypes.POINTER(OrcStats)
        L.orc_raycast.argtypes = [G, f3, f3, f3, ctypes.c_int, f3, st, ctypes.c_int]
        L.orc_apply.argtypes = [G, st, ctypes.c_int]
        L.orc_update.argtypes = [G, f3, f3, f3, ctypes.c_int, f3, st, ctypes.c_int]
        L.orc_trace_ray.argtypes = [G, ctypes.c_float, ctypes.c_float, ctypes.c_float, f3, i3, ctypes.c_int,
                                    i3, i3, i3]
        L.orc_recenter.argtypes = [G, f3, ctypes.c_int, i3, i3, ctypes.POINTER(i3), i3]
        L.orc_fetch.argtypes = [G, f3, ctypes.c_float, ctypes.c_int, ctypes.c_int, f3,
                                ctypes.POINTER(ctypes.c_uint8), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        L.orc_fetch.restype = ctypes.c_int64
        L.orc_is_state_pos.argtypes = [G, f3, ctypes.c_int]
        L.orc_sos.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint]
        L.orc_sos.restype = ctypes.c_float
        L.orc_fetch_sos.argtypes = [f3, i3, ctypes.c_float, ctypes.c_int, ctypes.c_uint]
        L.orc_fetch_sos.restype = ctypes.c_float
        L.orc_find_trace_diff.argtypes = [G, ctypes.c_uint, ctypes.c_uint, f3, ctypes.c_int, f3, i3,
                                          ctypes.c_int]
        L.orc_count_steps.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_uint,
                                      f3, f3, f3, ctypes.c_int, f3, ctypes.c_int]
        L.orc_count_steps.restype = ctypes.c_int64
        _olibs[path] = L
    return _olibs[path]


def count_steps(points, sensor, resolution, origin_at_center=False, max_range=25.0, fp=None,
                threads=None, lib_path=None) -> int:
    """The reference's voxel steps of one scan: its loop's iterations that did
    not break + 1 endpoint per ray it keeps (src/kernels.cu:44-137).  The
    count does not depend on the window, so no grid is needed."""
    L = oracle_lib(lib_path)
    x, y, z = _soa(points)
    s = (ctypes.c_float * 3)(*[float(v) for v in np.asarray(sensor, np.float32)])
    return int(L.orc_count_steps(float(np.float32(resolution)), int(origin_at_center),
                                 float(np.float32(max_range)), FP_PINNED if fp is None else fp,
                                 _fp(x), _fp(y), _fp(z), len(x), s,
                                 threads or (os.cpu_count() or 1)))


def _soa(points):
    p = np.asarray(points, dtype=np.float32)
    if p.ndim != 2 or p.shape[1] != 3:
        raise ValueError("points must be (N, 3)")
    return (np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]),
            np.ascontiguousarray(p[:, 2]))


class OracleGrid:
    """CPU restatement of the reference OccupancyGrid (host + device semantics)."""

    def __init__(self, half, resolution, origin_at_center=False, recenter_threshold=None,
                 origin=(0.0, 0.0, 0.0), fp=None):
        self._L = oracle_lib()
        self._g = _OrcGrid()
        h = (ctypes.c_int * 3)(*half)
        o = (ctypes.c_float * 3)(*origin)
        rc = self._L.orc_grid_init(ctypes.byref(self._g), h, resolution, int(origin_at_center),
                                   int(recenter_threshold is not None),
                                   float(recenter_threshold or 0.0), o)
        if rc != 0:
            raise RuntimeError(f"orc_grid_init failed ({rc})")
        if fp is not None:
            self._L.orc_set_fp_mode(ctypes.byref(self._g), fp)

    def __del__(self):
        try:
            self._L.orc_grid_free(ctypes.byref(self._g))
        except Exception:
            pass

    # ---- configuration ----
    @property
    def voxel_num(self):
        return self._g.voxel_num

    @property
    def map_size(self):
        return tuple(self._g.map)

    @property
    def half(self):
        return tuple(self._g.half)

    def set_fp_mode(self, m):
        self._L.orc_set_fp_mode(ctypes.byref(self._g), m)

    def set_max_range(self, r):
        self._L.orc_set_max_range(ctypes.byref(self._g), r)

    def set_log_odds(self, l_hit, l_miss, l_min, l_max, l_free, l_occ):
        self._L.orc_set_log_odds(ctypes.byref(self._g), l_hit, l_miss, l_min, l_max, l_free, l_occ)

    def set_origin_index(self, o):
        self._L.orc_set_origin_i(ctypes.byref(self._g), (ctypes.c_int * 3)(*o))
        self._g.first_run = 0

    def origin(self):
        return tuple(self._g.origin_i), tuple(self._g.origin_f)

    def reset(self):
        self._L.orc_grid_reset(ctypes.byref(self._g))

    # ---- state views (no copies) ----
    def set_state(self, occ=None, op=None, hit=None):
        if occ is not None:
            self.occ()[:] = occ
        if op is not None:
            self.op()[:] = op
        if hit is not None:
            self.hit()[:] = hit

    def occ(self):
        return np.ctypeslib.as_array(self._g.occ, shape=(self._g.voxel_num,))

    def op(self):
        return np.ctypeslib.as_array(self._g.op, shape=(self._g.voxel_num,))

    def hit(self):
        return np.ctypeslib.as_array(self._g.hit, shape=(self._g.voxel_num,))

    # ---- path ----
    def update(self, points, sensor, threads=1):
        x, y, z = _soa(points)
        st = OrcStats()
        s = (ctypes.c_float * 3)(*sensor)
        self._L.orc_update(ctypes.byref(self._g), _fp(x), _fp(y), _fp(z), x.shape[0], s,
                           ctypes.byref(st), threads)
        return st.as_dict()

    def raycast(self, points, sensor, threads=1):
        x, y, z = _soa(points)
        st = OrcStats()
        s = (ctypes.c_float * 3)(*sensor)
        self._L.orc_raycast(ctypes.byref(self._g), _fp(x), _fp(y), _fp(z), x.shape[0], s,
                            ctypes.byref(st), threads)
        return st.as_dict()

    def apply(self, threads=1):
        st = OrcStats()
        self._L.orc_apply(ctypes.byref(self._g), ctypes.byref(st), threads)
        return st.as_dict()

    def trace(self, point, sensor, cap=1 << 16):
        out = np.empty(cap, dtype=np.int32)
        nt = ctypes.c_int(0)
        ein = ctypes.c_int(0)
        ehit = ctypes.c_int(0)
        s = (ctypes.c_float * 3)(*sensor)
        n = self._L.orc_trace_ray(ctypes.byref(self._g), float(point[0]), float(point[1]),
                                  float(point[2]), s, _ip(out), cap, ctypes.byref(nt),
                                  ctypes.byref(ein), ctypes.byref(ehit))
        if n < 0:
            return None
        return out[:n].copy(), bool(ein.value), bool(ehit.value)

    def recenter(self, pos, compat=True):
        bufs = [np.zeros(m, dtype=np.int32) for m in self.map_size]
        ptrs = (ctypes.POINTER(ctypes.c_int) * 3)(*[_ip(b) for b in bufs])
        ns = (ctypes.c_int * 3)()
        no = (ctypes.c_int * 3)()
        skip = ctypes.c_int(0)
        p = (ctypes.c_float * 3)(*pos)
        act = self._L.orc_recenter(ctypes.byref(self._g), p, int(compat), ctypes.byref(skip), no, ptrs, ns)
        slabs = [bufs[a][: ns[a]].copy() for a in range(3)]
        return dict(action=act, host_skip=bool(skip.value), new_origin=tuple(no), slabs=slabs)

    def fetch(self, center, radius, state_filter=-1, max_results=0, cap=None):
        if cap is None:
            cap = max_results if max_results > 0 else 500000
        pos = np.empty((max(cap, 1), 3), dtype=np.float32)
        st = np.empty(max(cap, 1), dtype=np.uint8)
        npass = ctypes.c_int64(0)
        c = (ctypes.c_float * 3)(*center)
        n = self._L.orc_fetch(ctypes.byref(self._g), c, radius, state_filter, max_results,
                              _fp(pos), st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), cap,
                              ctypes.byref(npass))
        return pos[:n].copy(), st[:n].copy(), int(npass.value)

    def find_trace_diff(self, mode_a, mode_b, points, sensor, cap=1 << 20):
        p = np.ascontiguousarray(np.asarray(points, dtype=np.float32).reshape(-1, 3))
        out = np.empty(cap, dtype=np.int32)
        n = self._L.orc_find_trace_diff(ctypes.byref(self._g), mode_a, mode_b, _fp(p), p.shape[0],
                                        (ctypes.c_float * 3)(*sensor), _ip(out), cap)
        return out[:n].copy()

    def is_state(self, pos, state):
        return bool(self._L.orc_is_state_pos(ctypes.byref(self._g), (ctypes.c_float * 3)(*pos), state))


# ---------------------------------------------------------------------------
_rlib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _rlib
    if _rlib is None:
        L = ctypes.CDLL(REF_SO)
        f3 = ctypes.POINTER(ctypes.c_float)
        i3 = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.ref_pageable_access.argtypes = [ctypes.c_int]
        L.ref_create.argtypes = [i3, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_double, f3,
                                 ctypes.POINTER(vp)]
        L.ref_destroy.argtypes = [vp]
        L.ref_destroy.restype = None
        L.ref_set_max_range.argtypes = [vp, ctypes.c_float]
        L.ref_set_max_range.restype = None
        L.ref_set_log_odds.argtypes = [vp] + [ctypes.c_float] * 6
        L.ref_set_log_odds.restype = None
        L.ref_set_origin_i.argtypes = [vp, i3]
        L.ref_set_origin_i.restype = None
        L.ref_get_origin.argtypes = [vp, i3, f3]
        L.ref_get_origin.restype = None
        L.ref_raycast_only.argtypes = [vp, f3, f3, f3, ctypes.c_int, f3]
        L.ref_apply_only.argtypes = [vp]
        L.ref_update.argtypes = [vp, f3, f3, f3, ctypes.c_int, f3]
        L.ref_recenter.argtypes = [vp, f3, i3, i3, i3]
        L.ref_recenter_device_gate.argtypes = [vp, f3, ctypes.c_float, i3]
        L.ref_fetch.argtypes = [vp, f3, ctypes.c_float, ctypes.c_int, ctypes.c_int, f3,
                                ctypes.POINTER(ctypes.c_uint8), ctypes.c_int64]
        L.ref_fetch.restype = ctypes.c_int64
        L.ref_download.argtypes = [vp, f3, i3, i3]
        L.ref_upload.argtypes = [vp, f3, i3, i3]
        L.ref_voxel_num.argtypes = [vp]
        _rlib = L
    return _rlib


class RefGrid:
    """The reference's own CUDA kernels behind its OccupancyGrid call sequence."""

    def __init__(self, half, resolution, origin_at_center=False, recenter_threshold=None,
                 origin=(0.0, 0.0, 0.0)):
        self._L = ref_lib()
        self._h = ctypes.c_void_p()
        rc = self._L.ref_create((ctypes.c_int * 3)(*half), resolution, int(origin_at_center),
                                int(recenter_threshold is not None), float(recenter_threshold or 0.0),
                                (ctypes.c_float * 3)(*origin), ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"ref_create failed ({rc})")
        self.voxel_num = self._L.ref_voxel_num(self._h)

    def close(self):
        if self._h:
            self._L.ref_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_max_range(self, r):
        self._L.ref_set_max_range(self._h, r)

    def set_log_odds(self, *v):
        self._L.ref_set_log_odds(self._h, *v)

    def set_origin_index(self, o):
        self._L.ref_set_origin_i(self._h, (ctypes.c_int * 3)(*o))

    def origin(self):
        o = (ctypes.c_int * 3)()
        of = (ctypes.c_float * 3)()
        self._L.ref_get_origin(self._h, o, of)
        return tuple(o), tuple(of)

    def _call(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc})")

    def update(self, points, sensor, xyz=None):
        x, y, z = xyz if xyz is not None else _soa(points)
        self._call(self._L.ref_update(self._h, _fp(x), _fp(y), _fp(z), x.shape[0],
                                      (ctypes.c_float * 3)(*sensor)), "ref_update")

    def raycast(self, points, sensor):
        x, y, z = _soa(points)
        self._call(self._L.ref_raycast_only(self._h, _fp(x), _fp(y), _fp(z), x.shape[0],
                                            (ctypes.c_float * 3)(*sensor)), "ref_raycast_only")

    def apply(self):
        self._call(self._L.ref_apply_only(self._h), "ref_apply_only")

    def recenter(self, pos):
        a = ctypes.c_int(0)
        skip = ctypes.c_int(0)
        no = (ctypes.c_int * 3)()
        self._call(self._L.ref_recenter(self._h, (ctypes.c_float * 3)(*pos), ctypes.byref(a),
                                        ctypes.byref(skip), no), "ref_recenter")
        return dict(action=a.value, host_skip=bool(skip.value), new_origin=tuple(no))

    def device_gate(self, pos, thr_sq):
        a = ctypes.c_int(0)
        self._call(self._L.ref_recenter_device_gate(self._h, (ctypes.c_float * 3)(*pos), thr_sq,
                                                    ctypes.byref(a)), "ref_recenter_device_gate")
        return a.value

    def fetch(self, center, radius, state_filter=-1, max_results=0, cap=None):
        if cap is None:
            cap = max_results if max_results > 0 else 500000
        pos = np.empty((max(cap, 1), 3), dtype=np.float32)
        st = np.empty(max(cap, 1), dtype=np.uint8)
        n = self._L.ref_fetch(self._h, (ctypes.c_float * 3)(*center), radius, state_filter,
                              max_results, _fp(pos), st.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                              cap)
        if n < 0:
            raise RuntimeError("ref_fetch failed")
        return pos[:n].copy(), st[:n].copy()

    def download(self):
        occ = np.empty(self.voxel_num, dtype=np.float32)
        op = np.empty(self.voxel_num, dtype=np.int32)
        hit = np.empty(self.voxel_num, dtype=np.int32)
        self._call(self._L.ref_download(self._h, _fp(occ), _ip(op), _ip(hit)), "ref_download")
        return occ, op, hit

    def upload(self, occ=None, op=None, hit=None):
        keep = [np.ascontiguousarray(a, dtype=d) if a is not None else None
                for a, d in ((occ, np.float32), (op, np.int32), (hit, np.int32))]
        ptrs = [f(a) if a is not None else None for a, f in zip(keep, (_fp, _ip, _ip))]
        self._call(self._L.ref_upload(self._h, *ptrs), "ref_upload")


def ingest(points_sensor, rotation, translation, max_range):
    """World-frame cloud the reference driver builds from a sensor-frame one
    (src/main.cpp:640-693): filtered, transformed, in input order."""
    L = oracle_lib()
    p = np.ascontiguousarray(np.asarray(points_sensor, dtype=np.float32).reshape(-1, 3))
    R = np.ascontiguousarray(np.asarray(rotation, dtype=np.float32).reshape(9))
    t = np.ascontiguousarray(np.asarray(translation, dtype=np.float32).reshape(3))
    out = np.empty_like(p)
    r = np.float32(max_range)
    k = L.orc_ingest(_fp(p), p.shape[0], _fp(R), _fp(t), float(r * r), _fp(out))
    return out[:k].copy()


def depth_cloud(image, intrinsics):
    """Camera-frame cloud the reference driver makes from a depth image
    (src/main.cpp:558-632): (H*W, 3) float32, NaN rows for invalid pixels.
    `image`: (H, W) uint16 millimetres or float32 metres."""
    L = oracle_lib()
    img = np.ascontiguousarray(image)
    enc = 0 if img.dtype == np.uint16 else 1
    if enc == 1:
        img = img.astype(np.float32, copy=False)
    h, w = img.shape
    K = np.ascontiguousarray(np.asarray(intrinsics, dtype=np.float32).reshape(4))
    out = np.empty((h * w, 3), dtype=np.float32)
    L.orc_depth_cloud(img.ctypes.data, enc, w, h, img.strides[0], _fp(K), _fp(out))
    return out


def viz(samples_pos, resolution, origin_at_center, step, max_viz_radius, max_points, robot):
    """(n, 4) float32 x, y, z, rgb of the driver's visualisation cloud."""
    L = oracle_lib()
    p = np.ascontiguousarray(np.asarray(samples_pos, dtype=np.float32).reshape(-1, 3))
    out = np.empty((max(min(p.shape[0], int(max_points)), 1), 4), dtype=np.float32)
    inv = np.float32(1.0) / np.float32(resolution)
    k = L.orc_viz(_fp(p), p.shape[0], float(inv), int(bool(origin_at_center)), int(step),
                  float(max_viz_radius), int(max_points),
                  (ctypes.c_float * 3)(*[float(v) for v in robot]), _fp(out))
    return out[:k].copy()
