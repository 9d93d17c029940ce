"""cublox_b200 on the GPU against the oracle and the reference's own kernels.

Bit-exact bars (integer/index work and the FP32 path, whose operation order
and contraction are reproduced): per-voxel traversal and hit counts, stored
log-odds, recenter action/origin/cleared slabs, fetch samples.
"""
import numpy as np
import pytest

import cublox_b200 as C
import oracle as O
from cublox_b200 import synth

pytestmark = pytest.mark.gpu

LO = C.yaml_log_odds()


def pair(half, res, ctr=False, thr=None, origin=(0.0, 0.0, 0.0), max_range=None):
    g = C.OccupancyGrid(half, res, ctr, thr, origin)
    o = O.OracleGrid(half, res, ctr, thr, origin)
    g.setLogOddsParams(*LO)
    o.set_log_odds(*LO)
    if max_range is not None:
        g.setMaxRaycastRange(max_range)
        o.set_max_range(max_range)
    return g, o


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def ref_grid(half, res, ctr=False, thr=None, origin=(0.0, 0.0, 0.0), max_range=None):
    if not O.ref_available():
        return None
    r = O.RefGrid(half, res, ctr, thr, origin)
    r.set_log_odds(*LO)
    if max_range is not None:
        r.set_max_range(max_range)
    return r


@pytest.fixture(scope="module")
def small():
    w = synth.plain_small()
    return w, w.scan(0), w.sensor_origin(0)


def test_counts_match_oracle_plain_small(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.set_origin_index((0, 0, 18))
    o.set_origin_index((0, 0, 18))
    op, hit = g.count_scan(pts, s)
    st = o.raycast(pts, s)
    assert np.array_equal(op, o.op())
    assert np.array_equal(hit, o.hit())
    assert int(op.sum()) == st["op_incs"] and int(hit.sum()) == st["hit_incs"]
    assert g.check() == 0


def test_update_matches_oracle_and_reference(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, thr=4.0, max_range=w.sensor.max_range)
    assert g.first_run()
    g.update(pts, s)
    st = o.update(pts, s)
    assert not g.first_run()
    assert g.getOriginIndex() == o.origin()[0]
    assert same_bits(g.export(), o.occ())
    assert st["touched"] > 0
    r = ref_grid(w.half, w.resolution, thr=4.0, max_range=w.sensor.max_range)
    if r is not None:
        r.update(pts, s)
        occ, op, hit = r.download()
        assert same_bits(occ, o.occ())
        assert not op.any() and not hit.any()
        assert r.origin()[0] == o.origin()[0]


def test_update_stats(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.enable_stats(True)
    g.update(pts, s)
    st = o.update(pts, s)
    gs = g.last_stats()
    assert gs["rays"] == st["rays"]
    assert gs["op_incs"] == st["op_incs"]
    assert gs["hit_incs"] == st["hit_incs"]
    assert gs["touched"] == st["touched"]


def test_repeated_scans_and_clamp(small):
    """Many scans drive voxels into both clamps; every stored value exact."""
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    for k in range(6):
        sk = s + np.float32([0.013 * k, -0.021 * k, 0.0])
        g.update(pts, sk)
        o.update(pts, sk)
    occ = g.export()
    assert same_bits(occ, o.occ())
    assert (occ == np.float32(LO[3])).any() and (occ == np.float32(LO[2])).any()


@pytest.mark.parametrize("thr,expect_action", [(4.0, 0), (1.0, 1)])
def test_recenter_plain_small(small, thr, expect_action):
    """The (37,-12,3)-voxel shift is 3.901 m: below the 4 m yaml threshold
    (a no-op in the reference), above 1 m (slabs on all three axes)."""
    w, pts, s = small
    g, o = pair(w.half, w.resolution, thr=thr, max_range=w.sensor.max_range)
    g.update(pts, s)
    o.update(pts, s)
    oi, of = o.origin()
    shift = np.array(w.extra["recenter_shift"], dtype=np.float32)
    pos = (np.float32(of) + shift * np.float32(w.resolution)).astype(np.float32)
    a = g.recenter(pos)
    ro = o.recenter(pos)
    assert a == ro["action"] == expect_action
    assert g.getOriginIndex() == o.origin()[0]
    assert same_bits(g.export(), o.occ())
    # cleared-voxel accounting: the union of the oracle's slabs
    maps = [2 * h + 1 for h in w.half]
    keep = np.prod([maps[k] - len(set(ro["slabs"][k].tolist())) for k in range(3)])
    assert g.last_clear() == (int(np.prod(maps)) - keep if a == 1 else 0)
    r = ref_grid(w.half, w.resolution, thr=thr, max_range=w.sensor.max_range)
    if r is not None:
        r.update(pts, s)
        rr = r.recenter(pos)
        assert rr["action"] == expect_action
        assert r.origin()[0] == o.origin()[0]
        assert same_bits(r.download()[0], o.occ())
    # integrate again after the move
    g.update(pts, pos)
    o.update(pts, pos)
    assert same_bits(g.export(), o.occ())


def test_recenter_full_reset_and_mode1(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, thr=0.5, max_range=w.sensor.max_range)
    g.update(pts, s)
    o.update(pts, s)
    far = np.float32([500.0, 0.0, 1.8])  # shift >= largest map side
    assert g.recenter(far) == 2 == o.recenter(far)["action"]
    assert not g.export().any()
    assert g.last_clear() == g.voxel_num
    assert g.getOriginIndex() == o.origin()[0]
    # exiting-slabs-only mode clears a subset of compat mode's slabs
    g2, o2 = pair(w.half, w.resolution, thr=0.5, max_range=w.sensor.max_range)
    g2.set_recenter_mode(1)
    g2.update(pts, s)
    o2.update(pts, s)
    pos = np.float32(s + np.float32([1.2, -0.7, 0.3]))
    assert g2.recenter(pos) == 1
    r = o2.recenter(pos, compat=False)
    assert same_bits(g2.export(), o2.occ())
    assert r["action"] == 1


def test_fetch_plain_small(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.update(pts, s)
    o.update(pts, s)
    rng = np.random.default_rng(5)
    oi, of = o.origin()
    ext = np.float32(w.half) * np.float32(w.resolution)
    centres = (np.float32(of) + rng.uniform(-1, 1, (1000, 3)) * ext).astype(np.float32)
    off, pos, st = g.fetch_batch(centres, w.fetch_radius)
    r = ref_grid(w.half, w.resolution, max_range=w.sensor.max_range)
    if r is not None:
        r.update(pts, s)
    for q in range(len(centres)):
        opos, ost, _ = o.fetch(centres[q], w.fetch_radius)
        gp, gs = pos[off[q]:off[q + 1]], st[off[q]:off[q + 1]]
        assert same_bits(gp, opos) and np.array_equal(gs, ost), q
        if r is not None and q < 200:
            rp, rs = r.fetch(centres[q], w.fetch_radius)
            key = lambda p, t: sorted(map(tuple, np.concatenate(
                [p.view(np.uint32), t[:, None].astype(np.uint32)], axis=1).tolist()))
            assert key(rp, rs) == key(gp, gs), q


@pytest.mark.parametrize("flt,maxr", [(2, 0), (1, 0), (0, 0), (-1, 50), (2, 7)])
def test_fetch_filters_and_caps(small, flt, maxr):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.update(pts, s)
    o.update(pts, s)
    rng = np.random.default_rng(6)
    centres = (s + rng.uniform(-6, 6, (64, 3)) * np.float32([1, 1, 0.2])).astype(np.float32)
    for c in centres:
        gp, gs = g.fetchOccupancyAround(c, 1.5, None if flt < 0 else flt, maxr)
        opos, ost, npass = o.fetch(c, 1.5, flt, maxr)
        assert same_bits(gp, opos) and np.array_equal(gs, ost)
        if maxr:
            assert len(gp) == min(npass, maxr)


def test_point_queries(small):
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.update(pts, s)
    o.update(pts, s)
    rng = np.random.default_rng(7)
    q = np.concatenate([pts[::7], rng.uniform(-12, 12, (4000, 3)).astype(np.float32)])
    st = g.query_states(q)
    for i in range(0, len(q), 3):
        want = [k for k in (0, 1, 2) if o.is_state(q[i], k)]
        assert want == [int(st[i])], i
    assert g.isUnknown([1000.0, 0.0, 0.0])
    h = int(np.flatnonzero(o.occ())[0])
    assert g.storedAt(h) == o.occ()[h]
    assert g.storedAt(-1) == 0.0 and g.storedAt(g.voxel_num) == 0.0


def test_edge_case_rays():
    """Non-finite points, zero-length rays, clipped rays, axis-aligned and
    face-aligned rays, negative coordinates, sensor outside the window."""
    half, res = (20, 16, 12), 0.1
    sensors = [np.float32([0.0, 0.0, 0.0]), np.float32([-0.35, 0.2, -0.1]),
               np.float32([3.0, 0.05, 0.0])]  # the last is outside in x
    rng = np.random.default_rng(8)
    special = [
        [np.nan, 0, 0], [np.inf, 1, 1], [0, -np.inf, 0],
        [0.0, 0.0, 0.0], [1e-8, 0, 0],
        [1.0, 0.0, 0.0], [0.0, -1.3, 0.0], [0.0, 0.0, 0.9], [-1.7, 0, 0],
        [0.5, 0.5, 0.5], [-0.5, -0.5, -0.5], [0.3, -0.3, 0.0], [0.1, 0.2, 0.3],
        [100.0, 0.0, 0.0], [-30.0, 40.0, 1.0], [0.7, 0.7, 0.0],
    ]
    for s in sensors:
        pts = np.concatenate([np.float32(special) + 0 * s,
                              (s + rng.uniform(-4, 4, (3000, 3))).astype(np.float32),
                              (s + np.round(rng.uniform(-20, 20, (500, 3))) * np.float32(res)).astype(np.float32)])
        g, o = pair(half, res, max_range=2.5)
        g.set_origin_index((0, 0, 0))
        o.set_origin_index((0, 0, 0))
        op, hit = g.count_scan(pts, s)
        o.raycast(pts, s)
        assert np.array_equal(op, o.op()) and np.array_equal(hit, o.hit())


@pytest.mark.parametrize("fx", [((200, 200, 100), (17, -42, 8), 0.05, True),
                                ((350, 350, 75), (-120, 55, 0), 0.1, False),
                                ((3, 5, 7), (2, -1, 4), 0.25, True)])
def test_reference_fixture_grids(fx):
    """The three geometries of the reference's index tests
    (test/test_utils_index_roundtrip.cpp:44-53): a scan integrated into each,
    window origin as in the fixture, against the oracle."""
    half, origin, res, ctr = fx
    g, o = pair(half, res, ctr=ctr, max_range=8.0)
    g.set_origin_index(origin)
    o.set_origin_index(origin)
    c = np.float32(origin) * np.float32(res)
    pts = (c + synth.perf_test_cloud(20000, 0.3, 9.0, seed=42)).astype(np.float32)
    g.update(pts, c)
    o.update(pts, c)
    assert same_bits(g.export(), o.occ())


def test_trajectory_with_recenters():
    """A 40-scan drive on a 241x241x81 grid at 0.1 m, recentering at 1.5 m."""
    sensor = synth.Sensor(32, 512, -20.0, 20.0, 15.0, 0.02)
    scene = synth.make_scene(21, 150, 30.0, keepout=synth._keepout_line(0.0, 1.5))
    poses = synth.line_trajectory(40, 4.0, 10.0, 1.8, start=(-8.0, 0.0))
    half = (120, 120, 40)
    g, o = pair(half, 0.1, thr=1.5, max_range=sensor.max_range)
    actions = []
    for k, (x, y, z, yaw) in enumerate(poses):
        pts = synth.scan(scene, sensor, (x, y, z), yaw, seed=900 + k)
        so = np.float32([x, y, z])
        g.update(pts, so)
        o.update(pts, so)
        a = g.recenter(so)
        assert a == o.recenter(so)["action"]
        actions.append(a)
        assert g.getOriginIndex() == o.origin()[0]
        if k % 8 == 7:
            assert same_bits(g.export(), o.occ()), k
    assert same_bits(g.export(), o.occ())
    assert actions.count(1) >= 3


def test_empty_and_invalid_inputs():
    g = C.OccupancyGrid((4, 4, 4), 0.1, False, None)
    g.update(np.zeros((0, 3), np.float32), [0, 0, 0])
    assert g.first_run()  # an empty cloud returns before the first-run snap
    with pytest.raises(C.CubloxError):
        C.OccupancyGrid((40000, 40000, 40000), 0.1, False, None)
    with pytest.raises(C.CubloxError):
        C.OccupancyGrid((4, 4, 4), 0.0, False, None)
    with pytest.raises(ValueError):
        g.update(np.zeros((5, 2), np.float32), [0, 0, 0])
    pos, st = g.fetchOccupancyAround([0, 0, 0], -1.0)
    assert len(pos) == 0
    g.reset()
    assert g.first_run()


def test_stress_scale_drive_exact():
    """The largest configuration: 1025x1025x257 voxels at 0.05 m, 262,144-point
    scans to 100 m, recentering every scan — map and OCCUPIED fetches equal
    the oracle's after the drive."""
    sw = synth.stress(5)
    g, o = pair(sw.half, sw.resolution, thr=sw.threshold, max_range=sw.sensor.max_range)
    for k in range(5):
        pts, so = sw.scan(k), sw.sensor_origin(k)
        g.update(pts, so)
        g.recenter(so)
        o.update(pts, so, threads=8)
        o.recenter(so)
        assert tuple(g.getOriginIndex()) == tuple(o.origin()[0]), k
    assert same_bits(g.export(), o.occ())
    rng = np.random.default_rng(5)
    org = np.asarray(g.getOriginPosition(), np.float32)
    cen = (org + rng.uniform(-20, 20, (12, 3)) * np.float32([1, 1, 0.1])).astype(np.float32)
    off, pos, _ = g.fetch_batch(cen, sw.fetch_radius, C.VoxelState.OCCUPIED)
    for i in range(len(cen)):
        p, _, _ = o.fetch(cen[i], sw.fetch_radius, int(C.VoxelState.OCCUPIED))
        got = np.unique(np.asarray(pos[off[i]:off[i + 1]], np.float32).view(np.uint32), axis=0)
        want = np.unique(np.asarray(p, np.float32).view(np.uint32), axis=0)
        assert np.array_equal(got, want), i
    assert g.check() == 0


def test_readme_scale_scan_exact():
    """One full-size 64x1024 scan on the 701x701x151 (74.2M voxel) grid."""
    w = synth.readme_scale(2)
    g, o = pair(w.half, w.resolution, thr=4.0, max_range=w.sensor.max_range)
    for k in range(2):
        pts, so = w.scan(k), w.sensor_origin(k)
        g.update(pts, so)
        o.update(pts, so, threads=8)
    occ = g.export()
    assert same_bits(occ, o.occ())


@pytest.mark.parametrize("fold", [0, 1, 2, 3])
def test_fold_variants_exact(small, fold):
    """Every fold (full sweeps, flagged lines through registers or staged in
    shared memory) gives the oracle's map over scans that move the sensor,
    and leaves no line flagged behind."""
    w, pts, s = small
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.set_option(C.OPT_FOLD, fold)
    assert g.get_option(C.OPT_FOLD) == fold
    for k in range(3):
        so = (s + np.float32([1.7 * k, -0.9 * k, 0.1 * k])).astype(np.float32)
        g.update(pts, so)
        o.update(pts, so)
        assert same_bits(g.export(), o.occ()), k
    assert g.check() == 0


VARIANTS = [dict(raycast=0), dict(raycast=1, cube=32, match=1, sort=1),
            dict(raycast=1, cube=16, match=0, sort=1), dict(raycast=1, cube=0, match=1, sort=0),
            dict(raycast=2, cube=32, seg=48), dict(raycast=2, cube=0, seg=4, sort=0),
            dict(raycast=2, cube=16, seg=7, contig=0), dict(raycast=2, cube=8, seg=16, sort=1),
            dict(raycast=2, cube=32, seg=64, flat=1), dict(raycast=2, cube=32, seg=5, flat=1)]


def set_variant(g, v):
    g.set_option(C.OPT_RAYCAST, v["raycast"])
    if v["raycast"]:
        g.set_option(C.OPT_CUBE, v["cube"])
    if v["raycast"] == 1:
        g.set_option(C.OPT_MATCH, v["match"])
        g.set_option(C.OPT_SORT, v["sort"])
    if v["raycast"] == 2:
        g.set_option(C.OPT_SEGMENT, v["seg"])
        g.set_option(C.OPT_SORT, v.get("sort", 1))
        g.set_option(C.OPT_CONTIGUOUS, v.get("contig", 1))
        g.set_option(C.OPT_FLAT_CUBE, v.get("flat", 0))
        assert g.get_option(C.OPT_FLAT_CUBE) == v.get("flat", 0)


@pytest.mark.parametrize("v", VARIANTS, ids=lambda v: "-".join(f"{k}{x}" for k, x in v.items()))
def test_raycast_variants_exact(small, v):
    """Every kernel variant gives the oracle's counts, stats and map."""
    w, pts, s = small
    rng = np.random.default_rng(11)
    extra = (s + rng.uniform(-25, 25, (5000, 3))).astype(np.float32)
    extra[:100] = s  # zero-length rays
    extra[100:200] = s + np.float32([0.01, 0.0, 0.0])
    cloud = np.concatenate([pts, extra, np.float32([[np.nan, 0, 0], [np.inf, 0, 1]])])
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    set_variant(g, v)
    g.set_origin_index((3, -2, 18))
    o.set_origin_index((3, -2, 18))
    op, hit = g.count_scan(cloud, s)
    o.raycast(cloud, s)
    assert np.array_equal(op, o.op()) and np.array_equal(hit, o.hit())
    o.op()[:] = 0  # count_scan leaves the map untouched: drop the counts
    o.hit()[:] = 0
    g.enable_stats(True)
    g.update(cloud, s)
    st = o.update(cloud, s)
    assert same_bits(g.export(), o.occ())
    gs = g.last_stats()
    assert gs["rays"] == st["rays"] and gs["op_incs"] == st["op_incs"]
    assert gs["hit_incs"] == st["hit_incs"] and gs["touched"] == st["touched"]
    assert g.check() == 0


@pytest.mark.parametrize("v", [VARIANTS[1], VARIANTS[4], VARIANTS[5]],
                         ids=["binned32", "split48", "split4"])
def test_raycast_variants_readme_scale(v):
    w = synth.readme_scale(1)
    pts, so = w.scan(0), w.sensor_origin(0)
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    set_variant(g, v)
    g.set_origin_index((250, 0, 18))
    o.set_origin_index((250, 0, 18))
    op, hit = g.count_scan(pts, so)
    o.raycast(pts, so, threads=8)
    assert np.array_equal(op, o.op()) and np.array_equal(hit, o.hit())


def test_split_walk_many_geometries():
    """The split walk on tiny segments over varied grids, resolutions and
    binnings: every ray is cut at many exact time points."""
    rng = np.random.default_rng(12)
    # the last two put the sensor outside the window: rays enter it late,
    # so early segments walk nothing in it
    for half, res, ctr, org in [((40, 40, 40), 0.1, False, (1, -2, 0)),
                                ((30, 50, 20), 0.07, True, (1, -2, 0)),
                                ((64, 64, 16), 0.05, False, (1, -2, 0)),
                                ((25, 25, 25), 0.3, True, (1, -2, 0)),
                                ((25, 25, 25), 0.1, False, (40, 3, -2)),
                                ((20, 30, 10), 0.1, True, (-30, -35, 12))]:
        g, o = pair(half, res, ctr=ctr, max_range=float(np.float32(res) * 60))
        g.set_option(C.OPT_RAYCAST, 2)
        g.set_option(C.OPT_SEGMENT, 4)
        s = rng.uniform(-1, 1, 3).astype(np.float32) * np.float32(res) * 3
        g.set_origin_index(org)
        o.set_origin_index(org)
        d = rng.normal(size=(20000, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = rng.uniform(0.01, 1.0, (20000, 1)) * float(np.float32(res) * 90)
        pts = (s + d * r).astype(np.float32)
        op, hit = g.count_scan(pts, s)
        o.raycast(pts, s)
        assert np.array_equal(op, o.op()) and np.array_equal(hit, o.hit()), (half, res, ctr)
        assert g.check() == 0


def test_loaded_kernels_are_sm100a():
    assert C.binary_version() == 100


@pytest.mark.parametrize("cfg", ["plain_small", "readme_scale"])
def test_reference_steps_equal_oracle_count(cfg):
    """The work unit every voxel-steps/s figure divides by: the GPU count
    (cublox_grid_reference_steps) equals the oracle's exact count of the
    reference loop's iterations + 1 endpoint per kept ray, scan by scan, on
    the plain-small config and on README-scale scans along the trajectory."""
    if cfg == "plain_small":
        w = synth.plain_small()
        idx = [0]
    else:
        w = synth.readme_scale(60)
        idx = [0, 7, 31, 59]
    g = C.OccupancyGrid(w.half, w.resolution, False, w.threshold)
    g.setMaxRaycastRange(w.sensor.max_range)
    for k in idx:
        pts, so = w.scan(k), w.sensor_origin(k)
        want = O.count_steps(pts, so, w.resolution, False, w.sensor.max_range)
        assert g.reference_steps(pts, so) == want, k
        o = O.OracleGrid(w.half, w.resolution, False, w.threshold,
                         origin=tuple(float(v) for v in so))
        o.set_max_range(w.sensor.max_range)
        if cfg == "plain_small":  # the oracle's own per-scan accounting agrees
            assert o.raycast(pts, so, threads=8)["voxel_steps"] == want
    g.close()


@pytest.mark.parametrize("layout", C.LAYOUTS)
@pytest.mark.parametrize("raycast", [0, 1, 2])
def test_every_layout_exact(layout, raycast):
    """Every voxel layout (8x4x1, 4x8x1 and 4x4x2 bricks, the reference's
    hash order) with every walk: counts, stored log-odds, recenters (slab
    clears through partially and fully marked brick columns), fetches and
    point queries equal the oracle's, and exports stay in the reference's
    hash order."""
    sensor = synth.Sensor(16, 512, -20.0, 20.0, 12.0, 0.02)
    scene = synth.make_scene(31, 120, 25.0, keepout=synth._keepout_line(0.0, 1.5))
    poses = synth.line_trajectory(14, 6.0, 10.0, 1.8, start=(-4.0, 0.5))
    half = (90, 70, 22)  # 181 x 141 x 45: every axis ragged against the bricks
    g, o = pair(half, 0.1, thr=1.0, max_range=sensor.max_range)
    g.set_option(C.OPT_LAYOUT, layout)
    assert g.get_option(C.OPT_LAYOUT) == layout
    g.set_option(C.OPT_RAYCAST, raycast)
    rng = np.random.default_rng(40 + raycast)
    for k, (x, y, z, yaw) in enumerate(poses):
        pts = synth.scan(scene, sensor, (x, y, z), yaw, seed=1300 + k)
        so = np.float32([x, y, z + 0.13 * (k % 3)])  # z shifts exercise z slabs
        g.update(pts, so)
        o.update(pts, so)
        assert g.recenter(so) == o.recenter(so)["action"]
        if k % 5 == 4:
            assert same_bits(g.export(), o.occ()), k
            c = (so + rng.uniform(-3, 3, 3)).astype(np.float32)
            gp, gs = g.fetchOccupancyAround(c, 1.2)
            op_, os_, _ = o.fetch(c, 1.2)
            assert same_bits(gp, op_) and np.array_equal(gs, os_)
            q = (so + rng.uniform(-12, 12, (500, 3))).astype(np.float32)
            want = np.array([2 if o.is_state(p, 2) else (1 if o.is_state(p, 1) else 0)
                             for p in q], np.uint8)
            assert np.array_equal(g.query_states(q), want)
            h = int(rng.integers(0, o.voxel_num))
            assert np.float32(g.storedAt(h)).view(np.uint32) == np.float32(o.occ()[h]).view(np.uint32)
    assert same_bits(g.export(), o.occ())
    # count_scan reports counts in the reference's hash order
    pts = synth.scan(scene, sensor, poses[-1][:3], poses[-1][3], seed=1399)
    op, hit = g.count_scan(pts, np.float32(poses[-1][:3]))
    o.raycast(pts, np.float32(poses[-1][:3]))
    assert np.array_equal(op, o.op()) and np.array_equal(hit, o.hit())
    assert g.check() == 0


def test_layout_switch_keeps_the_map_and_import_export_round_trip():
    w = synth.plain_small()
    pts, so = w.scan(0), w.sensor_origin(0)
    g, o = pair(w.half, w.resolution, max_range=w.sensor.max_range)
    g.update(pts, so)
    o.update(pts, so)
    for layout in (230, 0, 221, 320):
        g.set_option(C.OPT_LAYOUT, layout)
        assert same_bits(g.export(), o.occ()), layout
        g.update(pts, so)
        o.update(pts, so)
        assert same_bits(g.export(), o.occ()), layout
    occ = o.occ().copy()
    occ[::97] = np.float32(1.25)
    g.import_(occ)
    assert same_bits(g.export(), occ)
    g.resetVoxel(97)
    assert g.storedAt(97) == 0.0
    with pytest.raises(C.CubloxError):
        g.set_option(C.OPT_LAYOUT, 321)  # 64-voxel bricks are not lines
