"""The oracle's restatement of the reference path, on hand-checked cases."""
import numpy as np

import oracle as O
from cublox_b200 import synth

LO = [O.oracle_lib().orc_logit(p) for p in (0.9, 0.49, 0.12, 0.98, 0.499, 0.85)]


def grid(half=(10, 10, 10), res=0.1, ctr=False, thr=None):
    g = O.OracleGrid(half, res, ctr, thr)
    g.set_log_odds(*LO)
    g.set_origin_index((0, 0, 0))
    return g


def test_axis_aligned_ray_visits_each_voxel_once():
    g = grid()
    g.set_max_range(5.0)
    s = np.float32([0.05, 0.05, 0.05])  # centre of voxel (0, 0, 0)
    hs, e_in, e_hit = g.trace([0.55, 0.05, 0.05], s)
    # voxels x = 0..4 by the loop, endpoint x = 5
    want = [O.oracle_lib().orc_global_to_hash((__import__("ctypes").c_int * 3)(x, 0, 0),
                                              (__import__("ctypes").c_int * 3)(*g.map_size),
                                              (__import__("ctypes").c_int * 3)(*g.half))
            for x in range(6)]
    assert list(hs) == want and e_in and e_hit


def test_clipped_ray_marks_free_only():
    g = grid()
    g.set_max_range(0.3)
    s = np.float32([0.05, 0.05, 0.05])
    hs, e_in, e_hit = g.trace([0.95, 0.05, 0.05], s)
    assert e_in and not e_hit
    assert len(hs) == 4  # x = 0, 1, 2 and the clip point's voxel x = 3


def test_dropped_rays():
    g = grid()
    s = np.float32([0.0, 0.0, 0.0])
    for p in ([np.nan, 0, 0], [np.inf, 0, 0], [0, 0, 0], [1e-8, 0, 0]):
        assert g.trace(p, s) is None


def test_update_counts_and_fold():
    g = grid(thr=None)
    g.set_max_range(10.0)
    s = np.float32([0.05, 0.05, 0.05])
    pts = np.float32([[0.55, 0.05, 0.05]] * 3)
    st = g.update(pts, s)
    assert st["rays"] == 3 and st["hit_incs"] == 3 and st["op_incs"] == 18
    occ = g.occ()
    assert np.count_nonzero(occ) == 6
    # endpoint: 3 hits -> l = 3 * l_hit clamped to l_max; free: 3 * l_miss
    assert np.float32(LO[3]) in occ
    assert np.isclose(occ[occ < 0], 3 * np.float32(LO[1])).all()


def test_recenter_slab_plan_compat_and_exiting_only():
    g = grid(half=(5, 5, 5), thr=0.1)
    g.occ()[:] = 1.0
    r = g.recenter(np.float32([0.35, 0.05, 0.05]))  # shift +3 on x
    assert r["action"] == 1 and r["new_origin"] == (3, 0, 0)
    # exiting: local slots of globals -5..-3 = -5,-4,-3; entering band 5,4,3
    assert list(r["slabs"][0]) == [-5, -4, -3, 3, 4, 5]
    g2 = grid(half=(5, 5, 5), thr=0.1)
    r2 = g2.recenter(np.float32([0.35, 0.05, 0.05]), compat=False)
    assert list(r2["slabs"][0]) == [-5, -4, -3]


def test_recenter_host_gate_and_threshold_none():
    g = grid(thr=None)
    assert g.recenter([5.0, 0, 0])["action"] == 0
    g = grid(thr=4.0)
    r = g.recenter([0.05 + 0.5, 0.05, 0.05])
    assert r["action"] == 0 and r["host_skip"]


def test_recenter_large_shift_is_bounded():
    """|shift| > half on one axis overflows the reference's slab list
    (kernels.cu:375-396); the oracle clears the defined union instead."""
    g = grid(half=(5, 5, 40), thr=0.1)
    r = g.recenter(np.float32([0.95, 0.05, 0.05]))  # +9 on x, map_x = 11
    assert r["action"] == 1
    assert len(r["slabs"][0]) == 11


def test_fetch_radius_shrinks_to_window_margin():
    g = grid(half=(10, 10, 10))
    g.occ()[:] = 5.0
    # centre 3 voxels from the x edge: radius limited to 0.3 m (Grid.cpp:67-78)
    c = np.float32([0.75, 0.05, 0.05])
    pos, st, n = g.fetch(c, 1.0)
    d = np.linalg.norm(pos - c, axis=1)
    assert d.max() <= 0.3 + 1e-6 and n == len(pos)
    assert (st == 2).all()
    pos, st, n = g.fetch(np.float32([1.05, 0.05, 0.05]), 1.0)  # margin 0
    assert n == 0


def test_fetch_order_and_cap():
    g = grid(half=(10, 10, 10))
    g.occ()[:] = -1.0
    pos, st, n = g.fetch(np.float32([0.05, 0.05, 0.05]), 0.5, -1, 10)
    assert len(pos) == 10 and n > 10
    key = [tuple(p) for p in pos]
    assert key == sorted(key)


def test_synth_is_deterministic():
    w = synth.plain_small()
    a, b = w.scan(0), w.scan(0)
    assert np.array_equal(a, b) and a.shape == (16384, 3) and a.dtype == np.float32
    r = np.linalg.norm(a - w.sensor_origin(0), axis=1)
    assert (r <= 30.0 + 1e-3).all() and (np.isclose(r, 30.0, atol=1e-3)).any()
