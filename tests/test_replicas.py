"""Map-sharded replicas, on CPU with the gloo backend (world size 2).

Each rank integrates only the maps its shard owns, with no exchange; the
union of the ranks' maps must equal what one process gives for all of them,
and the job rate must use the slowest rank's time.  The maps are integrated
by the CPU oracle so the test needs no GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from cublox_b200 import replicas, synth

MAPS = 5


def _maps(indices):
    w = synth.plain_small()
    out = {}
    for m in indices:
        g = O.OracleGrid((20, 20, 6), 0.1, False, None)
        shift = np.float32([0.3 * m, -0.2 * m, 0.0])
        pts = (w.scan(0)[::64] * np.float32(0.3) + shift).astype(np.float32)
        g.update(pts, w.sensor_origin(0) * np.float32(0.3) + shift, threads=1)
        out[m] = g.occ().copy()
    return out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.shard(MAPS, rank, world)
        res = _maps(mine)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), **{str(k): v for k, v in res.items()})
        rate = replicas.job_rate(units=100.0 * (rank + 1), seconds=1.0 + rank, dist=dist)
        np.save(os.path.join(outdir, f"rate{rank}.npy"), np.float64(rate))
    finally:
        dist.destroy_process_group()


def test_shards_cover_maps_once():
    for world in (1, 2, 3, 8):
        got = [m for r in range(world) for m in replicas.shard(11, r, world)]
        assert got == list(range(11))
        sizes = [len(replicas.shard(11, r, world)) for r in range(world)]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_two_gloo_ranks_equal_one_process(tmp_path):
    O.build()
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    union = {}
    for r in range(2):
        with np.load(tmp_path / f"rank{r}.npz") as z:
            for k in z.files:
                assert int(k) not in union
                union[int(k)] = z[k]
    alone = _maps(range(MAPS))
    assert sorted(union) == list(range(MAPS))
    for m in range(MAPS):
        assert np.array_equal(union[m].view(np.uint32), alone[m].view(np.uint32))
    # all ranks' units (100 + 200) over the slowest rank's 2 s
    for r in range(2):
        assert float(np.load(tmp_path / f"rate{r}.npy")) == pytest.approx(150.0)
