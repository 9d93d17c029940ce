"""The served form (cublox_server_*): results alone and in the mix.

Robots submit scans and fetches concurrently, from one thread each; the
server batches whatever is pending into shared launches, evicts maps to host
memory when the HBM budget is short, and brings them back.  None of that may
change a result: every robot's map and every fetch must equal, bit for bit,
what the same requests give on a lone OccupancyGrid fed in the same order.
"""
import threading

import numpy as np
import pytest

import cublox_b200 as C
from cublox_b200 import synth

pytestmark = pytest.mark.gpu

LO = C.yaml_log_odds()
DIMS = ((20, 20, 5), (32, 32, 8))
SENSORS = ((8, 64, 15.0), (16, 128, 15.0), (16, 256, 15.0))


def workload(n_robots=4, seconds=0.3, seed=11):
    return synth.serving(n_robots=n_robots, seconds=seconds, scan_rate=400.0, fetch_rate=100.0,
                         dims=DIMS, sensors=SENSORS, poses=3, max_range=6.0, threshold=0.5,
                         n_boxes=40, fetch_n=16, fetch_radius=0.6, seed=seed)


def voxels(half):
    return int(np.prod([2 * h + 1 for h in half]))


def serve(w, server):
    """Submit every robot's requests from its own thread; return per-robot
    lists of (kind, request id, centres)."""
    ids = [server.add_map(w.halves[r], w.resolution, False, w.threshold, max_range=w.max_range,
                          log_odds=LO) for r in range(w.n_robots)]
    per = [[] for _ in range(w.n_robots)]
    for i, (t, kind, r, c, j) in enumerate(w.events):
        per[r].append((i, kind, c, j))
    out = [[] for _ in range(w.n_robots)]

    def robot(r):
        for i, kind, c, j in per[r]:
            if kind == "scan":
                pts, origin = w.pool[r][c][j]
                out[r].append(("scan", server.submit_scan(ids[r], pts, origin, True), None))
            else:
                origin = w.pool[r][0][0][1]
                cen = w.fetch_centres(i, r, origin)
                out[r].append(("fetch", server.submit_fetch(ids[r], cen, w.fetch_radius), cen))

    th = [threading.Thread(target=robot, args=(r,)) for r in range(w.n_robots)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    server.drain()
    return ids, out


def check_alone(w, server, ids, out):
    for r in range(w.n_robots):
        g = C.OccupancyGrid(w.halves[r], w.resolution, False, w.threshold)
        g.setLogOddsParams(*LO)
        g.setMaxRaycastRange(w.max_range)
        k = 0
        for (t, kind, rr, c, j) in w.events:
            if rr != r:
                continue
            what, rid, cen = out[r][k]
            k += 1
            assert what == kind
            assert server.wait(rid) == C.REQ_DONE
            if kind == "scan":
                pts, origin = w.pool[r][c][j]
                g.update(pts, origin)
                g.recenter(origin)
            else:
                want = g.fetch_batch(cen, w.fetch_radius)
                got = server.fetch_result(rid, cen.shape[0])
                assert np.array_equal(got[0], want[0]), (r, k)
                assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2]), (r, k)
        occ, origin = server.export(ids[r], voxels(w.halves[r]))
        assert origin == tuple(g.getOriginIndex()), r
        assert np.array_equal(occ.view(np.uint32), g.export().view(np.uint32)), r


def test_served_maps_equal_lone_grids():
    w = workload()
    s = C.Server(hbm_budget_bytes=1 << 30, max_tick_points=1 << 16)
    ids, out = serve(w, s)
    check_alone(w, s, ids, out)
    st = s.stats()
    n_scans = sum(1 for e in w.events if e[1] == "scan")
    assert st["scans"] == n_scans and st["fetches"] == len(w.events) - n_scans
    assert 0 < st["ticks"] <= n_scans
    assert st["evictions"] == 0
    q, lat = s.times(out[0][0][1])
    assert 0.0 <= q <= lat
    s.release(out[0][0][1])
    with pytest.raises(C.CubloxError):
        s.times(out[0][0][1])
    s.close()


def test_tight_budget_evicts_and_restores_bit_for_bit():
    w = workload(seed=12)
    big = 12 * voxels(DIMS[1])
    scratch = 12 * 4096 + (1 << 20)
    s = C.Server(hbm_budget_bytes=scratch + big + 12 * voxels(DIMS[0]) + (64 << 10),
                 max_tick_points=4096)
    ids, out = serve(w, s)
    check_alone(w, s, ids, out)
    st = s.stats()
    assert st["evictions"] > 0 and st["admissions"] > w.n_robots
    # maps and tick scratch stay within the budget; a fetch in flight may add
    # its own output buffers until it ends
    assert st["peak_resident_bytes"] <= scratch + big + 12 * voxels(DIMS[0]) + (1 << 20)
    s.close()


def test_map_larger_than_budget_fails_alone():
    w = workload(n_robots=2, seconds=0.05, seed=13)
    s = C.Server(hbm_budget_bytes=12 * 4096 + (1 << 20) + 12 * voxels((20, 20, 5)) + (64 << 10),
                 max_tick_points=4096)
    small = s.add_map((20, 20, 5), 0.1, False, 0.5, max_range=6.0, log_odds=LO)
    huge = s.add_map((64, 64, 16), 0.1, False, 0.5, max_range=6.0, log_odds=LO)
    pts, origin = w.pool[0][0][0]
    bad = s.submit_scan(huge, pts, origin)
    good = s.submit_scan(small, pts, origin)
    with pytest.raises(C.CubloxError, match="budget"):
        s.wait(bad)
    assert s.wait(good) == C.REQ_DONE
    g = C.OccupancyGrid((20, 20, 5), 0.1, False, 0.5)
    g.setLogOddsParams(*LO)
    g.setMaxRaycastRange(6.0)
    g.update(pts, origin)
    g.recenter(origin)
    occ, _ = s.export(small, voxels((20, 20, 5)))
    assert np.array_equal(occ.view(np.uint32), g.export().view(np.uint32))
    s.close()
