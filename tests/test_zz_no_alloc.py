"""The allocation-free integration entry point, checked against the normal one.

cublox_integrate_noalloc serves callers that must not allocate device memory
while they run (a real-time mapping loop that reserves its GPU memory up
front, or code inside a host framework that only hands it a stream and its
own buffers).  Those callers own the map buffers; the entry point's only
scratch is a fixed device array.  Here the same two scans go through
cublox_grid_update (which allocates its own buffers) and, through the C ABI,
through cublox_integrate_noalloc on buffers this test owns; after each call
the stored log-odds must match bit for bit, the caller's counters must be
back at zero, and an oversized cloud must be refused.

The file is named to be collected last, so a stop-at-first-failure run has
run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import cublox_b200 as C
from cublox_b200 import synth

pytestmark = pytest.mark.gpu


class MapView(ctypes.Structure):
    _fields_ = [
        ("occ", ctypes.c_void_p), ("cnt", ctypes.c_void_p), ("hit", ctypes.c_void_p),
        ("half_map_size", ctypes.c_int * 3), ("origin_index", ctypes.c_int * 3),
        ("resolution", ctypes.c_float), ("origin_at_center", ctypes.c_int),
        ("max_range", ctypes.c_float), ("l_hit", ctypes.c_float), ("l_miss", ctypes.c_float),
        ("l_min", ctypes.c_float), ("l_max", ctypes.c_float),
    ]


def _entry():
    L = C.lib()
    fn = L.cublox_integrate_noalloc
    fn.argtypes = [ctypes.POINTER(MapView), ctypes.c_void_p, ctypes.c_int,
                   ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    L.cublox_noalloc_last_error.restype = ctypes.c_char_p
    return fn, L


def test_noalloc_matches_grid_update_on_two_calls():
    import torch

    fn, L = _entry()
    w = synth.plain_small()
    lo = C.yaml_log_odds()
    g = C.OccupancyGrid(w.half, w.resolution, False, None)
    g.setLogOddsParams(*lo)
    g.setMaxRaycastRange(w.sensor.max_range)
    scans = [w.scan(0), (w.scan(0) + np.float32([0.37, -0.21, 0.05])).astype(np.float32)]
    sensors = [w.sensor_origin(0), (w.sensor_origin(0) + np.float32([0.37, -0.21, 0.05]))]
    V = g.voxel_num
    occ = torch.zeros(V, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(V, dtype=torch.int32, device="cuda")
    hit = torch.zeros(V, dtype=torch.int32, device="cuda")
    view = MapView()
    view.occ, view.cnt, view.hit = occ.data_ptr(), cnt.data_ptr(), hit.data_ptr()
    view.half_map_size[:] = list(w.half)
    view.resolution = w.resolution
    view.origin_at_center = 0
    view.max_range = w.sensor.max_range
    view.l_hit, view.l_miss, view.l_min, view.l_max = lo[0], lo[1], lo[2], lo[3]
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(2):
        g.update(scans[k], sensors[k])
        want = g.export()
        if k == 0:  # the normal entry snapped the window to the sensor voxel
            view.origin_index[:] = list(g.getOriginIndex())
        pts = torch.from_numpy(np.ascontiguousarray(scans[k].T)).cuda()
        so = (ctypes.c_float * 3)(*[float(v) for v in sensors[k]])
        rc = fn(ctypes.byref(view), pts.data_ptr(), scans[k].shape[0], so, stream)
        assert rc == 0, L.cublox_noalloc_last_error()
        torch.cuda.synchronize()
        got = occ.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), k
        assert not cnt.any().item() and not hit.any().item()


def test_noalloc_refuses_oversized_clouds():
    fn, L = _entry()
    view = MapView()
    view.occ = view.cnt = view.hit = 1  # never dereferenced: refused first
    view.half_map_size[:] = [4, 4, 4]
    view.resolution = 0.1
    so = (ctypes.c_float * 3)(0.0, 0.0, 0.0)
    rc = fn(ctypes.byref(view), 1, 262145, so, None)
    assert rc == C.ERR_INVALID
    assert b"at most 262144" in L.cublox_noalloc_last_error()


def test_noalloc_at_the_point_cap_matches_grid_update():
    """A cloud of exactly CUBLOX_NOALLOC_MAX_POINTS (262,144) points: four
    README-scale scans from one pose, concatenated, twice in a row."""
    import torch

    fn, L = _entry()
    w = synth.readme_scale(4)
    pts = np.concatenate([w.scan(k) for k in range(4)]).astype(np.float32)
    assert pts.shape[0] == 262144
    sensor = w.sensor_origin(0)
    lo = C.yaml_log_odds()
    g = C.OccupancyGrid(w.half, w.resolution, False, None)
    g.setLogOddsParams(*lo)
    g.setMaxRaycastRange(w.sensor.max_range)
    V = g.voxel_num
    occ = torch.zeros(V, dtype=torch.float32, device="cuda")
    cnt = torch.zeros(V, dtype=torch.int32, device="cuda")
    hit = torch.zeros(V, dtype=torch.int32, device="cuda")
    view = MapView()
    view.occ, view.cnt, view.hit = occ.data_ptr(), cnt.data_ptr(), hit.data_ptr()
    view.half_map_size[:] = list(w.half)
    view.resolution = w.resolution
    view.origin_at_center = 0
    view.max_range = w.sensor.max_range
    view.l_hit, view.l_miss, view.l_min, view.l_max = lo[0], lo[1], lo[2], lo[3]
    stream = torch.cuda.current_stream().cuda_stream
    dev = torch.from_numpy(np.ascontiguousarray(pts.T)).cuda()
    so = (ctypes.c_float * 3)(*[float(v) for v in sensor])
    for k in range(2):
        g.update(pts, sensor)
        if k == 0:
            view.origin_index[:] = list(g.getOriginIndex())
        rc = fn(ctypes.byref(view), dev.data_ptr(), pts.shape[0], so, stream)
        assert rc == 0, L.cublox_noalloc_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(occ.cpu().numpy().view(np.uint32), g.export().view(np.uint32)), k
        assert not cnt.any().item() and not hit.any().item()
    g.close()
