"""Sensor-frame ingest (cublox_grid_update_pose): the reference driver's
buildCloudInOdomFrame (src/main.cpp:640-693) — finite and range filter, then
the sensor-to-world isometry — followed by update().

CPU: the oracle's restatement against the same arithmetic written out in
numpy float32 (IEEE, no fused multiply-add).  GPU: update_pose equals
update() of the oracle-built world cloud, bit for bit, for host and device
inputs, and a cloud with no point left leaves the grid untouched.
"""
import numpy as np
import pytest

import cublox_b200 as C
import oracle as O
from cublox_b200 import synth


def pose(yaw=0.7, roll=0.05):
    cy, sy, cr, sr = np.cos(yaw), np.sin(yaw), np.cos(roll), np.sin(roll)
    Rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    Rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    return (Rz @ Rx).astype(np.float32)


def sensor_cloud(w, R, t, n_bad=64, seed=0):
    world = w.scan(0).astype(np.float64)
    local = ((world - t.astype(np.float64)) @ R.astype(np.float64)).astype(np.float32)
    rng = np.random.default_rng(seed)
    idx = rng.choice(local.shape[0], n_bad, replace=False)
    local[idx[: n_bad // 2], rng.integers(0, 3)] = np.nan
    local[idx[n_bad // 2:]] *= np.float32(40.0)  # beyond the range filter
    return local


def numpy_ingest(p, R, t, max_range):
    f = np.float32
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    keep = np.isfinite(p).all(axis=1)
    r2 = (x * x + y * y) + z * z
    keep &= ~(r2 > f(max_range) * f(max_range))
    out = np.stack([((R[a, 0] * x + R[a, 1] * y) + R[a, 2] * z) + t[a] for a in range(3)], axis=1)
    return out[keep].astype(np.float32)


def test_oracle_ingest_matches_explicit_float32():
    O.build()
    w = synth.plain_small()
    R, t = pose(), np.float32([0.4, -1.1, 1.8])
    p = sensor_cloud(w, R, t)
    got = O.ingest(p, R, t, w.sensor.max_range)
    want = numpy_ingest(p, R, t, w.sensor.max_range)
    assert got.shape == want.shape and got.shape[0] < p.shape[0]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the filter keeps r^2 == max^2 and drops anything beyond
    edge = np.float32([[20.0, 0.0, 0.0], [20.000002, 0.0, 0.0]])
    assert O.ingest(edge, np.eye(3, dtype=np.float32), np.zeros(3, np.float32), 20.0).shape[0] == 1


@pytest.mark.gpu
@pytest.mark.parametrize("where", ["host", "device"])
def test_update_pose_equals_update_of_driver_cloud(where):
    import torch
    w = synth.plain_small()
    lo = C.yaml_log_odds()
    R, t = pose(), np.float32([0.4, -1.1, 1.8])
    p = sensor_cloud(w, R, t)
    world = O.ingest(p, R, t, w.sensor.max_range)
    a = C.OccupancyGrid(w.half, w.resolution, False, 4.0)
    b = C.OccupancyGrid(w.half, w.resolution, False, 4.0)
    o = O.OracleGrid(w.half, w.resolution, False, 4.0)
    for g in (a, b):
        g.setLogOddsParams(*lo)
        g.setMaxRaycastRange(w.sensor.max_range)
    o.set_log_odds(*lo)
    o.set_max_range(w.sensor.max_range)
    src = torch.from_numpy(p).cuda() if where == "device" else p
    for k in range(2):  # first run (snap) and a second scan from a moved pose
        tk = t + np.float32([0.3 * k, 0.1 * k, 0.0])
        wk = O.ingest(p, R, tk, w.sensor.max_range)
        a.update_pose(src, R, tk)
        b.update(wk, tk)
        o.update(wk, tk)
        assert a.getOriginIndex() == b.getOriginIndex()
        assert np.array_equal(a.export().view(np.uint32), b.export().view(np.uint32)), k
        assert np.array_equal(a.export().view(np.uint32), o.occ().view(np.uint32)), k
    assert world.shape[0] < p.shape[0]


@pytest.mark.gpu
def test_update_pose_with_nothing_left_is_a_no_op():
    w = synth.plain_small()
    g = C.OccupancyGrid(w.half, w.resolution, False, 4.0, origin=(5.0, 5.0, 0.0))
    g.setMaxRaycastRange(w.sensor.max_range)
    before = g.getOriginIndex()
    far = np.full((100, 3), 1000.0, np.float32)  # all beyond the range filter
    g.update_pose(far, np.eye(3, dtype=np.float32), np.float32([0.0, 0.0, 1.8]))
    assert g.getOriginIndex() == before  # no first-run snap: update() was never due
    assert not g.export().any()


# ---------------------------------------------------------------------------
# depth images (depthCallback, src/main.cpp:558-638)
# ---------------------------------------------------------------------------
K = np.float32([240.0, 238.5, 159.5, 119.25])


def depth_images(seed=3, h=120, w=160):
    rng = np.random.default_rng(seed)
    mm = rng.integers(300, 9000, size=(h, w)).astype(np.uint16)
    mm[rng.random((h, w)) < 0.05] = 0
    m = (mm.astype(np.float32) * np.float32(0.001)) + rng.normal(0, 0.01, (h, w)).astype(np.float32)
    m[rng.random((h, w)) < 0.03] = np.nan
    m[rng.random((h, w)) < 0.03] = -1.0
    return mm, m.astype(np.float32)


def numpy_depth(img):
    h, w = img.shape
    v, u = np.mgrid[0:h, 0:w]
    u = u.astype(np.float32)
    v = v.astype(np.float32)
    if img.dtype == np.uint16:
        valid = img != 0
        z = img.astype(np.float32) * np.float32(0.001)
    else:
        z = img
        valid = np.isfinite(z) & (z > 0)
    x = ((u - K[2]) * z) / K[0]
    y = ((v - K[3]) * z) / K[1]
    out = np.stack([x, y, z], axis=-1).reshape(-1, 3).astype(np.float32)
    out[~valid.reshape(-1)] = np.nan
    return out


def test_oracle_depth_cloud_matches_explicit_float32():
    O.build()
    for img in depth_images():
        got, want = O.depth_cloud(img, K), numpy_depth(img)
        same = (got.view(np.uint32) == want.view(np.uint32)) | (np.isnan(got) & np.isnan(want))
        assert same.all()


@pytest.mark.gpu
@pytest.mark.parametrize("enc", [0, 1], ids=["16UC1", "32FC1"])
@pytest.mark.parametrize("where", ["host", "device"])
def test_update_depth_equals_driver_cloud(enc, where):
    import torch
    img = depth_images()[enc]
    R, t = pose(yaw=0.3, roll=-0.4), np.float32([1.0, 0.5, 1.2])
    lo = C.yaml_log_odds()
    a = C.OccupancyGrid((60, 60, 20), 0.05, False, 4.0)
    b = C.OccupancyGrid((60, 60, 20), 0.05, False, 4.0)
    for g in (a, b):
        g.setLogOddsParams(*lo)
        g.setMaxRaycastRange(6.0)
    cloud = O.ingest(O.depth_cloud(img, K), R, t, 6.0)
    if where == "device":
        src = torch.from_numpy(img.view(np.int16) if enc == 0 else img).cuda()
    else:
        src = img
    a.update_depth(src, K, R, t)
    b.update(cloud, t)
    assert a.getOriginIndex() == b.getOriginIndex()
    assert np.array_equal(a.export().view(np.uint32), b.export().view(np.uint32))
    assert a.export().any()


# ---------------------------------------------------------------------------
# visualisation cloud (publishOccupancyCloudAsync, src/main.cpp:740-790)
# ---------------------------------------------------------------------------
def numpy_viz(pos, res, step, d_max, max_points, robot):
    f = np.float32
    inv = f(1.0) / f(res)
    gi = np.floor(pos * inv).astype(np.int64).astype(np.uint32)
    keep = np.ones(pos.shape[0], bool) if step <= 1 else ((gi[:, 0] ^ gi[:, 1] ^ gi[:, 2]) % step) == 0
    q = pos[keep][:max_points]
    d = q - np.float32(robot)
    dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    t = np.clip(dist / max(f(d_max), f(1.0)), f(0), f(1)).astype(np.float32)
    lo = t <= f(0.5)
    k = np.where(lo, t * f(2), (t - f(0.5)) * f(2)).astype(np.float32)
    r = np.where(lo, f(0), k)
    g = np.where(lo, f(1) - k, f(0))
    b = np.where(lo, k, f(1) - k)
    c8 = lambda c: (np.clip(c, 0, 1).astype(np.float32) * f(255)).astype(np.uint32)
    rgb = ((c8(r) << 16) | (c8(g) << 8) | c8(b)).view(np.float32)
    return np.concatenate([q, rgb[:, None]], axis=1)


def test_oracle_viz_matches_explicit_float32():
    O.build()
    rng = np.random.default_rng(4)
    pos = ((rng.integers(-200, 200, size=(5000, 3)) + np.float32(0.5)) * np.float32(0.1)).astype(np.float32)
    for step, mp in ((1, 10**6), (3, 10**6), (2, 700)):
        got = O.viz(pos, 0.1, False, step, 12.0, mp, (0.3, -0.2, 1.8))
        want = numpy_viz(pos, 0.1, step, 12.0, mp, (0.3, -0.2, 1.8))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), step


@pytest.mark.gpu
@pytest.mark.parametrize("step,max_points,flt", [(1, 10**6, None), (3, 10**6, C.VoxelState.OCCUPIED),
                                                 (2, 500, None)])
def test_fetch_viz_equals_driver_loop(step, max_points, flt):
    w = synth.plain_small()
    g = C.OccupancyGrid(w.half, w.resolution, False, 4.0)
    g.setLogOddsParams(*C.yaml_log_odds())
    g.setMaxRaycastRange(w.sensor.max_range)
    g.update(w.scan(0), w.sensor_origin(0))
    robot = w.sensor_origin(0)
    pos, _ = g.fetchOccupancyAround(robot, 3.0, flt)
    want = O.viz(pos, w.resolution, False, step, 12.0, max_points, robot)
    got = g.fetch_viz(robot, 3.0, flt, 0, step, 12.0, max_points)
    assert got.shape[0] == want.shape[0] > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
