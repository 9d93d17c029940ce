"""Generate the golden fixtures from the reference's own kernels.

Runs the reference harness (oracle/_ref/libcublox_ref.so: the reference's
src/kernels.cu for sm_100a, driven in its OccupancyGrid call sequence) on a
GPU and stores its outputs for seeded inputs of the small plain workload
(201 x 201 x 41 voxels at 0.1 m, 16 x 1024 scan from (0, 0, 1.8)):

  ref_plain_small.npz
    points (4096 x 3 wedge of the scan), sensor
    occ_hash/occ_bits   every nonzero stored log-odds after update()
    origin              window origin after the first-run snap
    rc_pos, rc_action, rc_origin, rc_hash/rc_bits   after recenter() by the
                        (37,-12,3)-voxel shift with a 1 m threshold
    fetch_c, fetch_r, fetch_off, fetch_pos_bits, fetch_state
                        sorted samples of 24 sphere fetches (r = 1 m)
    full_sha256, full_nonzero   digest of the whole stored grid after one
                        update with the full 16,384-point scan

tests/test_oracle_golden.py replays the same inputs through the CPU oracle
and requires identical results.  Usage: python tests/golden/make_golden.py OUT_DIR
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import cublox_b200 as C  # noqa: E402
import oracle as O  # noqa: E402
from cublox_b200 import synth  # noqa: E402


def sparse(occ):
    h = np.flatnonzero(occ).astype(np.int32)
    return h, occ[h].view(np.uint32)


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    w = synth.plain_small(threshold=1.0)
    full = w.scan(0)
    s = w.sensor_origin(0)
    pts = np.ascontiguousarray(full[:4096])
    lo = C.yaml_log_odds()
    r = O.RefGrid(w.half, w.resolution, False, 1.0)
    r.set_log_odds(*lo)
    r.set_max_range(w.sensor.max_range)
    r.update(pts, s)
    occ = r.download()[0]
    oh, ob = sparse(occ)
    oi, of = r.origin()
    shift = np.float32(w.extra["recenter_shift"])
    pos = (np.float32(of) + shift * np.float32(w.resolution)).astype(np.float32)
    rc = r.recenter(pos)
    occ2 = r.download()[0]
    rh, rb = sparse(occ2)
    rng = np.random.default_rng(3)
    no, nf = r.origin()
    cs = (np.float32(nf) + rng.uniform(-3, 3, (24, 3)) * np.float32([1, 1, 0.3])).astype(np.float32)
    offs, pb, stt = [0], [], []
    for c in cs:
        p, st = r.fetch(c, 1.0)
        key = np.concatenate([p.view(np.uint32), st[:, None].astype(np.uint32)], axis=1)
        key = key[np.lexsort(key.T[::-1])] if len(key) else key.reshape(0, 4)
        pb.append(key[:, :3])
        stt.append(key[:, 3].astype(np.uint8))
        offs.append(offs[-1] + len(key))
    r.close()
    r2 = O.RefGrid(w.half, w.resolution, False, 1.0)
    r2.set_log_odds(*lo)
    r2.set_max_range(w.sensor.max_range)
    r2.update(full, s)
    occf = r2.download()[0]
    r2.close()
    np.savez_compressed(
        os.path.join(out_dir, "ref_plain_small.npz"),
        points=pts, sensor=s, occ_hash=oh, occ_bits=ob, origin=np.int32(oi),
        rc_pos=pos, rc_action=np.int32(rc["action"]), rc_origin=np.int32(rc["new_origin"]),
        rc_hash=rh, rc_bits=rb, fetch_c=cs, fetch_r=np.float32(1.0),
        fetch_off=np.int64(offs), fetch_pos_bits=np.concatenate(pb) if pb else np.zeros((0, 3), np.uint32),
        fetch_state=np.concatenate(stt) if stt else np.zeros(0, np.uint8),
        full_sha256=np.frombuffer(hashlib.sha256(occf.tobytes()).digest(), dtype=np.uint8),
        full_nonzero=np.int64(np.count_nonzero(occf)),
        pageable_access=np.int32(O.ref_lib().ref_pageable_access(0)),
    )
    print("golden written:", os.path.join(out_dir, "ref_plain_small.npz"), len(oh), len(rh), offs[-1])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py OUTPUT_DIR")
    main(sys.argv[1])
