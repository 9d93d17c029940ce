"""The oracle against golden fixtures produced by the reference's own kernels.

tests/golden/ref_plain_small.npz was written by tests/golden/make_golden.py
running the reference's src/kernels.cu (sm_100a build, via oracle/_ref) on a
B200: the stored log-odds after update(), the recenter result and grid, and
24 sphere fetches of the small plain workload.  The CPU oracle must
reproduce every bit.  This pins the oracle to the reference itself.
"""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from cublox_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
LO = [O.oracle_lib().orc_logit(p) for p in (0.9, 0.49, 0.12, 0.98, 0.499, 0.85)]


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "ref_plain_small.npz"))


def sparse(occ):
    h = np.flatnonzero(occ).astype(np.int32)
    return h, occ[h].view(np.uint32)


def test_reference_has_no_pageable_access_on_the_box(gold):
    # Why the reference's slab kernels are rebuilt with by-value parameters.
    assert int(gold["pageable_access"]) == 0


def test_oracle_matches_reference_update_recenter_fetch(gold):
    w = synth.plain_small(threshold=1.0)
    g = O.OracleGrid(w.half, w.resolution, False, 1.0)
    g.set_log_odds(*LO)
    g.set_max_range(w.sensor.max_range)
    g.update(gold["points"], gold["sensor"])
    assert tuple(g.origin()[0]) == tuple(gold["origin"])
    h, b = sparse(g.occ())
    assert np.array_equal(h, gold["occ_hash"]) and np.array_equal(b, gold["occ_bits"])
    r = g.recenter(gold["rc_pos"])
    assert r["action"] == int(gold["rc_action"])
    assert tuple(r["new_origin"]) == tuple(gold["rc_origin"])
    h, b = sparse(g.occ())
    assert np.array_equal(h, gold["rc_hash"]) and np.array_equal(b, gold["rc_bits"])
    off = gold["fetch_off"]
    for q, c in enumerate(gold["fetch_c"]):
        pos, st, _ = g.fetch(c, float(gold["fetch_r"]))
        key = np.concatenate([pos.view(np.uint32), st[:, None].astype(np.uint32)], axis=1)
        key = key[np.lexsort(key.T[::-1])] if len(key) else key.reshape(0, 4)
        assert np.array_equal(key[:, :3], gold["fetch_pos_bits"][off[q]:off[q + 1]]), q
        assert np.array_equal(key[:, 3], gold["fetch_state"][off[q]:off[q + 1]]), q


def test_oracle_matches_reference_full_scan_digest(gold):
    w = synth.plain_small(threshold=1.0)
    full = w.scan(0)
    assert np.array_equal(full[:4096], gold["points"])  # the scan itself is reproducible
    g = O.OracleGrid(w.half, w.resolution, False, 1.0)
    g.set_log_odds(*LO)
    g.set_max_range(w.sensor.max_range)
    g.update(full, gold["sensor"])
    occ = g.occ()
    assert int(np.count_nonzero(occ)) == int(gold["full_nonzero"])
    assert hashlib.sha256(occ.tobytes()).digest() == bytes(gold["full_sha256"])
