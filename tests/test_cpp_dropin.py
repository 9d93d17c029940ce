"""The C++ drop-in class, compiled and run against libcublox_b200.so.

tests/cpp/dropin_replay.cpp drives include/cublox/OccupancyGrid.hpp the way
the reference's C++ callers drive theirs (construct, update, recenter,
fetchOccupancyAround, the is* queries, resetVoxel, reset) on the small plain
workload; every answer is compared with the oracle.  A second run restates
the reference's own perf test (test/test_occupancy_grid_perf.cpp:54-100)
through the same class.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import cublox_b200 as C
import oracle as O
from cublox_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LO = C.yaml_log_odds()


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "dropin_replay"
    libdir = os.path.dirname(C.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           "-o", str(out), os.path.join(HERE, "cpp", "dropin_replay.cpp"),
                           "-L", libdir, "-lcublox_b200", f"-Wl,-rpath,{libdir}"])
    return str(out)


class Out:
    def __init__(self, data):
        self.b = data
        self.i = 0

    def get(self, fmt):
        v = struct.unpack_from(fmt, self.b, self.i)
        self.i += struct.calcsize(fmt)
        return v if len(v) > 1 else v[0]

    def vec(self, dtype):
        n = self.get("<q")
        a = np.frombuffer(self.b, dtype=dtype, count=n, offset=self.i)
        self.i += n * np.dtype(dtype).itemsize
        return a


def classify(stored):
    s = np.asarray(stored, np.float32)
    return np.where(s >= np.float32(LO[5]), 2, np.where(s < np.float32(LO[4]), 1, 0))


def test_cpp_dropin_replay_matches_oracle(exe, tmp_path):
    w = synth.plain_small(threshold=1.0)
    pts, s0 = w.scan(0), w.sensor_origin(0)
    half, res, thr, mr = w.half, w.resolution, 1.0, w.sensor.max_range
    rng = np.random.default_rng(7)
    o = O.OracleGrid(half, res, False, thr)
    o.set_log_odds(*LO)
    o.set_max_range(mr)
    o.update(pts, s0)
    oi_upd, of_upd = o.origin()
    rc_pos = (np.float32(of_upd) + np.float32([37, -12, 3]) * np.float32(res)).astype(np.float32)
    o.recenter(rc_pos)
    oi, of = o.origin()
    hw = np.asarray(half, np.float64) * res
    cen = np.stack([of[0] + rng.uniform(-0.8, 0.8, 12) * hw[0],
                    of[1] + rng.uniform(-0.8, 0.8, 12) * hw[1],
                    rng.uniform(0.2, 2.5, 12)], axis=1).astype(np.float32)
    qs = np.stack([of[0] + rng.uniform(-1.1, 1.1, 3000) * hw[0],
                   of[1] + rng.uniform(-1.1, 1.1, 3000) * hw[1],
                   rng.uniform(-2.0, 4.0, 3000)], axis=1).astype(np.float32)
    radius = 1.0
    blob = struct.pack("<iiifi", *half, res, 0) + struct.pack("<d", thr) + struct.pack("<f", mr)
    blob += np.float32(LO).tobytes() + struct.pack("<q", len(pts)) + pts.astype(np.float32).tobytes()
    blob += np.float32(s0).tobytes() + rc_pos.tobytes()
    blob += struct.pack("<q", len(cen)) + cen.tobytes() + struct.pack("<f", radius)
    blob += struct.pack("<q", len(qs)) + qs.tobytes()
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    fin.write_bytes(blob)
    r = subprocess.run([exe, "replay", str(fin), str(fout)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = Out(fout.read_bytes())
    assert out.get("<f") == np.float32(mr)
    assert out.get("<i") == o.voxel_num
    assert out.get("<iii") == (0, 0, 0)
    out.get("<fff")
    assert out.get("<iii") == tuple(oi_upd)
    assert np.array_equal(np.float32(out.get("<fff")), np.float32(of_upd))
    assert out.get("<iii") == tuple(oi)
    assert np.array_equal(np.float32(out.get("<fff")), np.float32(of))
    occ = o.occ()
    inv = np.float32(1.0) / np.float32(res)
    for c in cen:
        for flt, cap in ((-1, 0), (2, 0), (-1, 7)):
            pos, st = out.vec(np.float32).reshape(-1, 3), out.vec(np.uint8)
            wp, ws, _ = o.fetch(c, radius, state_filter=flt, max_results=cap)
            assert np.array_equal(pos.view(np.uint32), wp.view(np.uint32)) and np.array_equal(st, ws)
        # Grid.cpp:67-78: min of the x and y margins, in metres
        g = [int(np.floor(np.float32(c[a]) * inv)) for a in range(2)]
        mx, my = half[0] - abs(g[0] - oi[0]), half[1] - abs(g[1] - oi[1])
        want = 0.0 if (mx < 0 or my < 0) else np.float32(min(mx, my)) * np.float32(res)
        assert out.get("<f") == np.float32(want)
    by_pos, by_idx, inside, by_hash = (out.vec(np.uint8) for _ in range(4))
    for k, p in enumerate(qs):
        st = 2 if o.is_state(p, 2) else (1 if o.is_state(p, 1) else 0)
        assert (by_pos[k] & 3) == st and bool(by_pos[k] & 4) == o.is_state(p, 0), k
    gi = np.floor(qs.astype(np.float32) * inv).astype(np.int64)
    ins = np.all(np.abs(gi - np.asarray(oi)) <= np.asarray(half), axis=1)
    assert np.array_equal(inside.astype(bool), ins)
    ms = 2 * np.asarray(half) + 1
    for k in range(len(qs)):
        if not ins[k]:
            assert by_idx[k] == 4
            continue
        loc = [(int(gi[k, a]) % int(ms[a])) for a in range(3)]
        loc = [v - ms[a] if v > half[a] else v for a, v in enumerate(loc)]
        h = ((loc[0] + half[0]) * ms[1] + (loc[1] + half[1])) * ms[2] + (loc[2] + half[2])
        st = int(classify(occ[h]))
        assert (by_idx[k] & 3) == st and bool(by_idx[k] & 4) == (st == 0), k
    sx = half[0]
    slab = occ[sx * ms[1] * ms[2]:(sx + 1) * ms[1] * ms[2]]
    assert np.array_equal(by_hash, classify(slab).astype(np.uint8))
    first = out.get("<i")
    if first >= 0:
        assert classify(occ[first]) == 2
        assert out.get("<B") == 1
    assert out.get("<q") == 0  # reset() leaves every voxel unknown


def test_cpp_reference_perf_test_restated(exe):
    r = subprocess.run([exe, "perf", "20"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "401 x 401 x 201 voxels (32321001 total) at 0.05 m" in r.stdout, r.stdout
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("steady-state")][0]
    mean = float(line.split("mean=")[1].split(" ms")[0])
    print(r.stdout)
    assert 0.0 < mean < 50.0
