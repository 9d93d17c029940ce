"""Out-of-memory paths, driven by the allocation-failure test hook.

cublox_test_fail_allocations makes the library's next device or pinned
allocations fail as if memory were exhausted, without exhausting the GPU and
without any CUDA call.  Every entry point that allocates must then return
CUBLOX_ERR_NOMEM, free what it had allocated so far, and leave the object
usable: the next call, with memory back, must give the same result as if the
failure had never happened.  (The reference aborts the process instead:
CUDA_OK, src/OccupancyGrid.cpp:32-49.)
"""
import contextlib

import numpy as np
import pytest

import cublox_b200 as C
import oracle as O
from cublox_b200 import synth

pytestmark = pytest.mark.gpu

LO = C.yaml_log_odds()


@contextlib.contextmanager
def failing(skip, count):
    C.fail_allocations(skip, count)
    try:
        yield
    finally:
        C.fail_allocations(0, 0)


def balance(before, after):
    """Allocations made minus frees made between two counter readings."""
    return ((after["device_allocs"] - before["device_allocs"]) -
            (after["device_frees"] - before["device_frees"]),
            (after["pinned_allocs"] - before["pinned_allocs"]) -
            (after["pinned_frees"] - before["pinned_frees"]))


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def small():
    w = synth.plain_small()
    return w, w.scan(0), w.sensor_origin(0)


@pytest.mark.parametrize("skip", [0, 1, 3, 5, 7])
def test_grid_create_out_of_memory_frees_what_it_allocated(skip):
    """The k-th allocation of cublox_grid_create fails: the call reports
    CUBLOX_ERR_NOMEM and every allocation it had made is freed."""
    w, _, _ = small()
    before = C.runtime_counters()
    with failing(skip, 1):
        with pytest.raises(C.CubloxError) as e:
            C.OccupancyGrid(w.half, w.resolution, False, None)
    assert e.value.code == C.ERR_NOMEM
    assert balance(before, C.runtime_counters()) == (0, 0)
    g = C.OccupancyGrid(w.half, w.resolution, False, None)  # memory is back
    g.close()


@pytest.mark.parametrize("skip", [0, 1, 2])
def test_update_out_of_memory_leaves_the_map_untouched(skip):
    """A scan whose working buffers cannot be allocated is rejected with
    CUBLOX_ERR_NOMEM before it touches the map; the same scan then
    integrates as on a grid that never failed."""
    w, pts, s = small()
    g = C.OccupancyGrid(w.half, w.resolution, False, None)
    g.setLogOddsParams(*LO)
    g.setMaxRaycastRange(w.sensor.max_range)
    with failing(skip, 1000):
        with pytest.raises(C.CubloxError) as e:
            g.update(pts, s)
    assert e.value.code == C.ERR_NOMEM
    assert not np.any(g.export().view(np.uint32))
    g.update(pts, s)
    o = O.OracleGrid(w.half, w.resolution, False, None)
    o.set_log_odds(*LO)
    o.set_max_range(w.sensor.max_range)
    o.update(pts, s)
    assert same_bits(g.export(), o.occ())
    assert g.check() == 0
    g.close()


def test_batch_update_out_of_memory_then_recovers():
    """The batch's first update cannot size its work items: it fails with
    CUBLOX_ERR_NOMEM, and the next updates (which size them again) give the
    maps lone grids give."""
    w = synth.plain_small()
    b = C.Batch()
    b.set_option(C.BATCH_OPT_GRAPHS, 1)
    bg, solo = [], []
    for _ in range(3):
        g = b.add_grid(w.half, w.resolution, False, None)
        g.setLogOddsParams(*LO)
        g.setMaxRaycastRange(w.sensor.max_range)
        bg.append(g)
        h = C.OccupancyGrid(w.half, w.resolution, False, None)
        h.setLogOddsParams(*LO)
        h.setMaxRaycastRange(w.sensor.max_range)
        solo.append(h)
    rng = np.random.default_rng(3)
    base, so = w.scan(0), w.sensor_origin(0)
    clouds = [base[rng.permutation(base.shape[0])[: 4000 * (m + 1)]] for m in range(3)]
    sensors = np.stack([so] * 3).astype(np.float32)
    with failing(0, 1000):
        with pytest.raises(C.CubloxError) as e:
            b.update(bg, clouds, sensors)
    assert e.value.code == C.ERR_NOMEM
    for step in range(2):
        b.update(bg, clouds, sensors)
        b.synchronize()
        for m in range(3):
            solo[m].update(clouds[m], sensors[m])
    for m in range(3):
        assert same_bits(bg[m].export(), solo[m].export()), m
        solo[m].close()
    b.close()


def test_server_request_fails_alone_when_its_map_cannot_be_allocated():
    """A served map whose arrays cannot be allocated at its first scan: that
    request fails with CUBLOX_ERR_NOMEM, another map's scan is served, and
    once memory is back the map's next scan is served as on a lone grid."""
    w = synth.plain_small()
    s = C.Server(hbm_budget_bytes=1 << 30, max_tick_points=1 << 16,
                 max_fetch_centres=16, max_fetch_samples=1 << 16)
    ids = [s.add_map(w.half, w.resolution, False, None, max_range=w.sensor.max_range,
                     log_odds=LO) for _ in range(2)]
    pts, so = w.scan(0), w.sensor_origin(0)
    with failing(0, 1 << 20):
        rid = s.submit_scan(ids[0], pts, so, False)
        with pytest.raises(C.CubloxError) as e:
            s.wait(rid)
    assert e.value.code == C.ERR_NOMEM
    assert s.wait(s.submit_scan(ids[1], pts, so, False)) == C.REQ_DONE
    assert s.wait(s.submit_scan(ids[0], pts, so, False)) == C.REQ_DONE
    s.drain()
    g = C.OccupancyGrid(w.half, w.resolution, False, None)
    g.setLogOddsParams(*LO)
    g.setMaxRaycastRange(w.sensor.max_range)
    g.update(pts, so)
    for m in ids:
        occ, origin = s.export(m, g.export().shape[0])
        assert origin == tuple(g.getOriginIndex())
        assert same_bits(occ, g.export()), m
    g.close()
    s.close()


def test_hook_rejects_negative_arguments():
    with pytest.raises(C.CubloxError):
        C.fail_allocations(-1, 1)
