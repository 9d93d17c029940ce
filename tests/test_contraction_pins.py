"""The FP32 contraction pattern is pinned against the reference's own kernels.

For every site the probes (tests/fp_probe.py) contain inputs on which the
fused and unfused readings differ observably.  The reference's sm_100a build
must match exactly the pinned pattern among all candidates, and cublox_b200
must reproduce the reference's outputs on the same probes.
"""
import numpy as np
import pytest

import oracle as O
import fp_probe as P

pytestmark = pytest.mark.gpu

CENTER_AGNOSTIC = O.FP_CENTER_FMA  # fused and unfused agree except at exact ties


def _ray_bits(m):
    return m & ((7 << O.FP_RAY_SOS_SHIFT) | O.FP_CLIP_FMA | O.FP_BOUND_FMA | O.FP_CENTER_FMA)


@pytest.fixture(scope="module")
def ray_scenarios():
    return P.build_ray_scenarios()


def test_ref_ray_sites_pinned(ray_scenarios):
    if not O.ref_available():
        pytest.skip("reference harness not built")
    for sc in ray_scenarios:
        op, hit = P.run_ray_scenario_ref(sc)
        got = P.matching_ray_modes(sc, op, hit)
        names = [P.describe(m) for m in got]
        assert got, f"{sc.name}: no candidate pattern reproduces the reference"
        pinned = _ray_bits(O.FP_PINNED)
        assert {_ray_bits(m) & ~CENTER_AGNOSTIC for m in got} == {pinned & ~CENTER_AGNOSTIC}, names


def test_ref_apply_sites_pinned():
    if not O.ref_available():
        pytest.skip("reference harness not built")
    pr = P.build_apply_probe()
    got = P.matching_apply_modes(pr, P.run_apply_ref(pr))
    want = O.FP_PINNED & (O.FP_MISS_FMA | O.FP_HIT_FMA)
    assert [m & (O.FP_MISS_FMA | O.FP_HIT_FMA) for m in got] == [want], [P.describe(m) for m in got]


def test_ref_recenter_gate_pinned():
    if not O.ref_available():
        pytest.skip("reference harness not built")
    pr = P.build_gate_probe()
    got = P.matching_gate_shapes(pr, P.run_gate_ref(pr))
    assert got == [(O.FP_PINNED >> O.FP_REC_SOS_SHIFT) & 7], got


def test_ref_fetch_sites_pinned():
    if not O.ref_available():
        pytest.skip("reference harness not built")
    pr = P.build_fetch_probe()
    assert len(pr["queries"]) >= 8
    got = P.matching_fetch_modes(pr, P.run_fetch_ref(pr))
    mask = (7 << O.FP_FETCH_SOS_SHIFT) | O.FP_FETCH_DFMA
    assert [m & mask for m in got] == [O.FP_PINNED & mask], [P.describe(m) for m in got]


def test_cublox_reproduces_ray_probes(ray_scenarios):
    import cublox_b200 as C

    for sc in ray_scenarios:
        want_op, want_hit = P.oracle_ray_counts(sc, O.FP_PINNED)
        g = C.OccupancyGrid(sc.half, sc.res, sc.ctr, None)
        g.set_origin_index((0, 0, 0))
        g.setMaxRaycastRange(float(sc.max_range))
        op, hit = g.count_scan(sc.points, sc.sensor)
        assert np.array_equal(op, want_op), sc.name
        assert np.array_equal(hit, want_hit), sc.name
        assert g.check() == 0


def test_cublox_reproduces_fetch_probe():
    import cublox_b200 as C

    pr = P.build_fetch_probe()
    key = O.fp_mode(fetch_sos=(O.FP_PINNED >> O.FP_FETCH_SOS_SHIFT) & 7,
                    fetch_d=bool(O.FP_PINNED & O.FP_FETCH_DFMA))
    og = pr["grids"][key]
    g = C.OccupancyGrid(pr["half"], 0.1, False, None)
    g.set_origin_index((0, 0, 0))
    g.setLogOddsParams(*pr["lo"])
    g.import_(pr["occ"])
    for c, r in pr["queries"]:
        pos, st = g.fetchOccupancyAround(c, r)
        got = sorted(map(tuple, np.concatenate([pos.view(np.uint32), st[:, None].astype(np.uint32)],
                                               axis=1).tolist()))
        assert got == P._fetch_set(og, c, r)
