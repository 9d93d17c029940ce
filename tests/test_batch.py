"""Batched integration (cublox_batch_*) against the same grids updated one by one.

Every grid of a batch must end each step bit-identical to a grid that got the
same scans through OccupancyGrid.update and the same recenters: the batch
changes only how the work is launched (one walk and one fold launch for all
maps, graph replay, launch shapes rotated by the tuner), never what a map
stores.  Maps differ in size, point counts are uneven (zero included), and
one map's voxel count is not a multiple of four.
"""
import numpy as np
import pytest

import cublox_b200 as C
from cublox_b200 import synth

pytestmark = pytest.mark.gpu

LO = C.yaml_log_odds()
DIMS = ((40, 40, 10), (64, 64, 16), (30, 50, 12), (3, 3, 3))


def same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def small_workload(n_maps=6, n_steps=6, seed=5):
    w = synth.batching(n_maps=n_maps, n_steps=n_steps, dims=DIMS, n_min=512, n_max=4096,
                       beams=16, max_range=8.0, speed=4.0, threshold=0.6, n_boxes=60, seed=seed)
    w.counts[1, 2] = 16  # one tiny scan
    return w


def setup(w, batch):
    bg, solo = [], []
    for m in range(w.n_maps):
        for make, out in ((lambda: batch.add_grid(w.halves[m], w.resolution, False, w.threshold), bg),
                          (lambda: C.OccupancyGrid(w.halves[m], w.resolution, False, w.threshold), solo)):
            g = make()
            g.setLogOddsParams(*LO)
            g.setMaxRaycastRange(w.max_range)
            out.append(g)
    return bg, solo


def run_and_compare(w, batch, bg, solo, feed, skip=()):
    for k in range(w.counts.shape[1]):
        clouds, sensors = w.step(k)
        clouds = [c if (m, k) not in skip else np.zeros((0, 3), np.float32)
                  for m, c in enumerate(clouds)]
        feed(batch, bg, clouds, sensors)
        for m in range(w.n_maps):
            solo[m].update(clouds[m], sensors[m])
        acts = batch.recenter(bg, sensors)
        for m in range(w.n_maps):
            assert acts[m] == solo[m].recenter(sensors[m]), (k, m)
        batch.synchronize()
        for m in range(w.n_maps):
            assert tuple(bg[m].getOriginIndex()) == tuple(solo[m].getOriginIndex()), (k, m)
            assert same_bits(bg[m].export(), solo[m].export()), (k, m)
    for m in range(w.n_maps):
        assert bg[m].check() == 0, m


def feed_lists(batch, bg, clouds, sensors):
    batch.update(bg, clouds, sensors)


def feed_device(batch, bg, clouds, sensors):
    import torch
    off = np.zeros(len(clouds) + 1, np.int64)
    off[1:] = np.cumsum([c.shape[0] for c in clouds])
    xyz = torch.from_numpy(np.concatenate(clouds, axis=0)).cuda()
    batch.update(bg, xyz, sensors, offsets=off)
    torch.cuda.synchronize()


def feed_pinned(batch, bg, clouds, sensors):
    import torch
    off = np.zeros(len(clouds) + 1, np.int64)
    off[1:] = np.cumsum([c.shape[0] for c in clouds])
    host = torch.from_numpy(np.concatenate(clouds, axis=0)).pin_memory()
    batch.update(bg, host.numpy(), sensors, offsets=off)
    batch.synchronize()  # the walk (or the copy ahead of it) reads the pinned buffer


@pytest.mark.parametrize("graphs", [False, True])
def test_batch_matches_solo_updates_through_tuning(graphs):
    w = small_workload(n_steps=32)  # 15 candidates x 2 tuning rounds, then the chosen one
    b = C.Batch()
    b.set_option(C.BATCH_OPT_GRAPHS, int(graphs))
    bg, solo = setup(w, b)
    run_and_compare(w, b, bg, solo, feed_lists, skip={(3, 4), (0, 0)})
    assert not b.tuning()
    assert 0 <= b.get_option(C.BATCH_OPT_SHAPE) < b.get_option(C.BATCH_OPT_NUM_SHAPES)
    assert b.get_option(C.BATCH_OPT_LAYOUT) in C.LAYOUTS
    assert all(g.get_option(C.OPT_LAYOUT) == b.get_option(C.BATCH_OPT_LAYOUT) for g in bg)
    b.close()


@pytest.mark.parametrize("layout", C.LAYOUTS)
def test_every_layout_gives_the_same_maps(layout):
    w = small_workload(n_maps=4, n_steps=4, seed=8)
    b = C.Batch()
    b.set_option(C.BATCH_OPT_SHAPE, 12)  # fused: folds read flags other CTAs wrote
    b.set_option(C.BATCH_OPT_LAYOUT, layout)
    b.set_option(C.BATCH_OPT_GRAPHS, 1)
    bg, solo = setup(w, b)
    run_and_compare(w, b, bg, solo, feed_lists)
    assert all(g.get_option(C.OPT_LAYOUT) == layout for g in bg)
    b.close()


@pytest.mark.parametrize("shape", [6, 12])
def test_fused_wait_runs_out_and_the_context_stays_usable(shape):
    """A fused launch whose first map's folds wait for a walk item that
    does not exist (the test hook): the bounded wait (shortened here to
    about a millisecond) gives up, the launch ends, the map's error word
    says CUBLOX_DEVICE_WAIT_TIMEOUT, and the same batch, after the maps are
    reset, integrates correctly again."""
    w = small_workload(n_maps=3, n_steps=3, seed=10)
    b = C.Batch()
    b.set_option(C.BATCH_OPT_SHAPE, shape)
    b.set_option(C.BATCH_OPT_WAIT_LIMIT, 4000)
    b.set_option(C.BATCH_OPT_INJECT_MISSING_WALK, 1)
    bg, solo = setup(w, b)
    clouds, sensors = w.step(0)
    b.update(bg, clouds, sensors)
    b.synchronize()
    words = [g.check() for g in bg]
    assert words[0] & C.DEVICE_WAIT_TIMEOUT, words
    b.set_option(C.BATCH_OPT_INJECT_MISSING_WALK, 0)
    b.set_option(C.BATCH_OPT_WAIT_LIMIT, 1 << 23)
    for g in bg:
        g.reset()
    run_and_compare(w, b, bg, solo, feed_lists)
    b.close()


@pytest.mark.parametrize("shape", range(16))
def test_every_shape_gives_the_same_maps(shape):
    w = small_workload(n_maps=4, n_steps=3, seed=7)
    b = C.Batch()
    assert b.get_option(C.BATCH_OPT_NUM_SHAPES) == 16
    b.set_option(C.BATCH_OPT_SHAPE, shape)
    b.set_option(C.BATCH_OPT_FOLD, shape % 3)
    b.set_option(C.BATCH_OPT_GRAPHS, 1)
    bg, solo = setup(w, b)
    run_and_compare(w, b, bg, solo, feed_lists)
    b.close()


@pytest.mark.parametrize("host_read", [1, 0], ids=["read-in-place", "copied"])
@pytest.mark.parametrize("feed", [feed_device, feed_pinned, feed_lists],
                         ids=["device", "pinned", "pageable"])
def test_batch_inputs_device_pinned_pageable(feed, host_read):
    """Device points are walked where they are; host points are read in
    place by the walk (pinned, or staged in the batch's pinned buffer) or
    copied to the device first: the maps are the same."""
    w = small_workload(n_maps=5, n_steps=3, seed=9)
    b = C.Batch()
    b.set_option(C.BATCH_OPT_GRAPHS, 1)
    b.set_option(C.BATCH_OPT_HOST_READ, host_read)
    assert b.get_option(C.BATCH_OPT_HOST_READ) == host_read
    bg, solo = setup(w, b)
    run_and_compare(w, b, bg, solo, feed)
    b.close()


def test_batch_subsets_and_stats():
    w = small_workload(n_maps=4, n_steps=4, seed=11)
    b = C.Batch()
    b.set_option(C.BATCH_OPT_SHAPE, 0)
    bg, solo = setup(w, b)
    for g in bg + solo:
        g.enable_stats(True)
    for k in range(4):
        clouds, sensors = w.step(k)
        idx = [m for m in range(w.n_maps) if (m + k) % 3]  # a different subset each step
        b.update([bg[m] for m in idx], [clouds[m] for m in idx], sensors[idx])
        for m in idx:
            solo[m].update(clouds[m], sensors[m])
        b.synchronize()
        for m in idx:
            assert bg[m].last_stats() == solo[m].last_stats(), (k, m)
        for m in range(w.n_maps):
            assert same_bits(bg[m].export(), solo[m].export()), (k, m)
    b.close()


def test_batch_rejects_bad_calls():
    b = C.Batch()
    g = b.add_grid((8, 8, 4), 0.1)
    other = C.OccupancyGrid((8, 8, 4), 0.1)
    pts = np.zeros((4, 3), np.float32) + 0.3
    so = np.zeros((1, 3), np.float32)
    with pytest.raises(C.CubloxError):
        b.update([other], [pts], so)  # not created by this batch
    with pytest.raises(C.CubloxError):
        b.update([g, g], [pts, pts], np.zeros((2, 3), np.float32))
    with pytest.raises(C.CubloxError):
        b.update([g], pts, so, offsets=np.array([4, 0], np.int64))
    with pytest.raises(C.CubloxError):
        b.set_option(C.BATCH_OPT_SHAPE, 99)
    with pytest.raises(C.CubloxError):
        b.set_option(C.BATCH_OPT_FOLD, 99)
    b.update([], [], np.zeros((0, 3), np.float32))
    b.close()
