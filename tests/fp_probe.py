"""Black-box pinning of the reference build's FP32 multiply-add contraction.

nvcc compiles the reference's kernels with its default -fmad=true, so some
`a*b + c` expressions become one fused multiply-add.  Which ones is not
visible in the source, and reading compiled code is not an option, so this
module pins it from outputs alone:

  * for every contraction site, inputs are searched on the CPU (with the
    oracle) for which the fused and unfused readings give different
    observable results (visited voxels, hit flags, stored log-odds, recenter
    action, fetch membership);
  * the reference's own kernels are run on those inputs;
  * every candidate pattern is replayed in the oracle, and the patterns whose
    outputs equal the reference's, bit for bit, are returned.

The same probes are then run through cublox_b200 to show that the pinned
pattern is the one it reproduces.  Sites (see oracle/cublox_oracle.h):
ray length sum of squares (kernels.cu:50), clip point (:60-62), boundary
distance (:89-100), centre binning (utils.cuh:27-29), apply terms
(kernels.cu:188-189), recenter gate (:329), fetch sphere test (:532-535).
"""
from __future__ import annotations

import itertools

import numpy as np

import oracle as O

SHAPES = list(range(6))


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _jitter(rng, a: np.ndarray, k: int) -> np.ndarray:
    out = a.copy()
    steps = rng.integers(-k, k + 1, size=a.shape)
    for s in range(1, k + 1):
        out = np.where(steps >= s, np.nextafter(out, np.float32(np.inf)), out)
        out = np.where(steps <= -s, np.nextafter(out, np.float32(-np.inf)), out)
    return out.astype(np.float32)


# ---------------------------------------------------------------------------
# Ray sites
# ---------------------------------------------------------------------------
class RayScenario:
    def __init__(self, name, half, res, ctr, sensor, max_range, points, modes):
        self.name = name
        self.half = half
        self.res = res
        self.ctr = ctr
        self.sensor = np.asarray(sensor, dtype=np.float32)
        self.max_range = np.float32(max_range)
        self.points = points
        self.modes = modes  # candidate patterns (ray bits only)


def _ray_mode(sos, clip, bound, center):
    return O.fp_mode(ray_sos=sos, clip=clip, bound=bound, center=center)


def _collect(g, base, variants, pool, sensor, per_pair):
    keep = []
    for v in variants:
        if v == base:
            continue
        idx = g.find_trace_diff(base, v, pool, sensor, cap=per_pair)
        keep.extend(idx.tolist())
    return keep


def build_ray_scenarios(seed: int = 11, per_pair: int = 24):
    rng = np.random.default_rng(seed)
    scen = []
    for ctr in (False, True):
        half = (64, 64, 64)
        res = np.float32(0.1)
        # Sensor just off voxel faces, so that the first boundary distance
        # b*res - o cancels and its fused/unfused readings part ways.
        if ctr:
            sensor = np.float32([0.05 + 3e-8, -0.15 + 2e-8, 0.25 - 3e-8])
        else:
            sensor = np.float32([0.3 + 2e-8, -0.2 + 3e-8, 0.1 + 1e-8])
        M = np.float32(3.0)
        g = O.OracleGrid(half, float(res), ctr, None)
        g.set_origin_index((0, 0, 0))
        g.set_max_range(float(M))
        base = _ray_mode(O.SOS_FX_FZ, False, False, True)
        # Pool 1: endpoints at |d| ~ M, a few ulps either side (clip decision).
        u = _unit(rng, 200000)
        e = (sensor[None, :].astype(np.float64) + float(M) * u).astype(np.float32)
        pool_len = _jitter(rng, e, 6)
        # Pool 2: clipped rays whose clip point sits on a voxel face.
        u = _unit(rng, 400000)
        tgt = sensor[None, :].astype(np.float64) + float(M) * u
        ax = rng.integers(0, 3, size=len(u))
        tgt[np.arange(len(u)), ax] = np.round(tgt[np.arange(len(u)), ax] / 0.1) * 0.1 + (0.05 if ctr else 0.0)
        d = tgt - sensor[None, :]
        pool_clip = (sensor[None, :] + d * rng.uniform(1.2, 2.0, size=(len(u), 1))).astype(np.float32)
        # Pool 3: unclipped rays of random length (traversal order).
        u = _unit(rng, 400000)
        pool_walk = (sensor[None, :] + u * rng.uniform(0.3, 2.9, size=(len(u), 1))).astype(np.float32)
        # Pool 4 (centre binning): endpoints with p*inv near k + 0.5.
        pools = [pool_len, pool_clip, pool_walk]
        if ctr:
            # p*inv + 0.5 fused or not only differs where the sum crosses a
            # binade, i.e. |p*inv| near 2^k - 0.5.
            u = _unit(rng, 200000)
            e = sensor[None, :] + u * rng.uniform(0.5, 2.5, size=(len(u), 1))
            ax = rng.integers(0, 3, size=len(u))
            k = rng.integers(1, 6, size=len(u))
            sg = np.where(rng.uniform(size=len(u)) < 0.5, -1.0, 1.0)
            e[np.arange(len(u)), ax] = sg * (2.0 ** k - 0.5) * 0.1
            pools.append(_jitter(rng, e.astype(np.float32), 12))
        variants = []
        for s in SHAPES:
            variants.append(_ray_mode(s, False, False, True))
        variants.append(_ray_mode(O.SOS_FX_FZ, True, False, True))
        variants.append(_ray_mode(O.SOS_FX_FZ, False, True, True))
        variants.append(_ray_mode(O.SOS_FX_FZ, True, True, True))
        # Also discriminate against the all-plain reading.
        variants.append(_ray_mode(O.SOS_PLAIN, False, False, False))
        sel = []
        for pool in pools:
            idx = _collect(g, base, variants, pool, sensor, per_pair)
            sel.append(pool[np.unique(np.asarray(idx, dtype=np.int64))] if idx else pool[:0])
        pts = np.concatenate(sel + [pool_walk[:256]], axis=0)
        modes = [_ray_mode(s, c, b, ce) for s in SHAPES for c in (False, True)
                 for b in (False, True) for ce in ((False, True) if ctr else (True,))]
        scen.append(RayScenario("center" if ctr else "corner", half, float(res), ctr, sensor, M,
                                pts, modes))
    return scen


def oracle_ray_counts(sc: RayScenario, mode: int):
    g = O.OracleGrid(sc.half, sc.res, sc.ctr, None, fp=mode)
    g.set_origin_index((0, 0, 0))
    g.set_max_range(float(sc.max_range))
    g.raycast(sc.points, sc.sensor)
    return g.op().copy(), g.hit().copy()


def matching_ray_modes(sc: RayScenario, op: np.ndarray, hit: np.ndarray):
    out = []
    for m in sc.modes:
        o, h = oracle_ray_counts(sc, m)
        if np.array_equal(o, op) and np.array_equal(h, hit):
            out.append(m)
    return out


def run_ray_scenario_ref(sc: RayScenario):
    r = O.RefGrid(sc.half, sc.res, sc.ctr, None)
    r.set_origin_index((0, 0, 0))
    r.set_max_range(float(sc.max_range))
    r.raycast(sc.points, sc.sensor)
    _, op, hit = r.download()
    r.close()
    return op, hit


# ---------------------------------------------------------------------------
# Apply sites
# ---------------------------------------------------------------------------
def build_apply_probe(seed: int = 12):
    rng = np.random.default_rng(seed)
    half = (10, 10, 10)
    n = 21 ** 3
    occ = rng.uniform(-1.99, 3.89, n).astype(np.float32)
    op = rng.integers(1, 3000, n).astype(np.int32)
    hit = (op * rng.uniform(0, 1, n)).astype(np.int32)
    hit[rng.uniform(size=n) < 0.5] = 0
    lo = [O.oracle_lib().orc_logit(p) for p in (0.9, 0.49, 0.12, 0.98, 0.499, 0.85)]
    return dict(half=half, occ=occ, op=op, hit=hit, lo=lo)


def oracle_apply(pr, mode):
    g = O.OracleGrid(pr["half"], 0.1, False, None, fp=mode)
    g.set_log_odds(*pr["lo"])
    g.set_state(pr["occ"], pr["op"], pr["hit"])
    g.apply()
    return g.occ().copy()


def apply_modes():
    return [O.fp_mode(miss=a, hit=b) for a in (False, True) for b in (False, True)]


def matching_apply_modes(pr, occ_out):
    return [m for m in apply_modes() if np.array_equal(oracle_apply(pr, m).view(np.uint32),
                                                       occ_out.view(np.uint32))]


def run_apply_ref(pr):
    r = O.RefGrid(pr["half"], 0.1, False, None)
    r.set_log_odds(*pr["lo"])
    r.upload(pr["occ"], pr["op"], pr["hit"])
    r.apply()
    occ, _, _ = r.download()
    r.close()
    return occ


# ---------------------------------------------------------------------------
# Recenter gate
# ---------------------------------------------------------------------------
def build_gate_probe(seed: int = 13, want: int = 64):
    rng = np.random.default_rng(seed)
    L = O.oracle_lib()
    origin_f = np.float32([0.05, 0.05, 0.05])  # voxel (0,0,0), corner binning
    thr = np.float32(0.5)
    thr_sq = np.float32(thr * thr)
    u = _unit(rng, 200000)
    pos = (origin_f[None, :] + 0.5 * u).astype(np.float32)
    pos = _jitter(rng, pos, 4)
    keep = []
    for p in pos:
        d = (p - origin_f).astype(np.float32)
        res = {s: bool(L.orc_sos(float(d[0]), float(d[1]), float(d[2]), s) < thr_sq) for s in SHAPES}
        if len(set(res.values())) > 1:
            keep.append(p)
        if len(keep) >= want:
            break
    return dict(origin_f=origin_f, thr_sq=thr_sq, pos=np.asarray(keep, dtype=np.float32))


def gate_expect(pr, shape):
    L = O.oracle_lib()
    out = []
    for p in pr["pos"]:
        d = (p - pr["origin_f"]).astype(np.float32)
        out.append(0 if L.orc_sos(float(d[0]), float(d[1]), float(d[2]), shape) < pr["thr_sq"] else 1)
    return np.asarray(out)


def run_gate_ref(pr):
    r = O.RefGrid((64, 64, 64), 0.1, False, 0.5)
    r.set_origin_index((0, 0, 0))
    acts = [1 if r.device_gate(p, float(pr["thr_sq"])) != 0 else 0 for p in pr["pos"]]
    r.close()
    return np.asarray(acts)


def matching_gate_shapes(pr, acts):
    return [s for s in SHAPES if np.array_equal(gate_expect(pr, s), acts)]


# ---------------------------------------------------------------------------
# Fetch sphere test
# ---------------------------------------------------------------------------
def fetch_modes():
    return [O.fp_mode(fetch_sos=s, fetch_d=d) for s in SHAPES for d in (False, True)]


def _fetch_set(g, c, r):
    pos, st, _ = g.fetch(c, r, -1, 0)
    return sorted(map(tuple, np.concatenate([pos.view(np.uint32), st[:, None].astype(np.uint32)],
                                            axis=1).tolist()))


def build_fetch_probe(seed: int = 14, want: int = 48, tries: int = 200000):
    """Queries whose sphere boundary passes within an ulp of a voxel centre,
    so that the fetch-site readings disagree on that voxel's membership."""
    rng = np.random.default_rng(seed)
    L = O.oracle_lib()
    half = (30, 30, 30)
    n = 61 ** 3
    occ = rng.uniform(-2.5, 4.0, n).astype(np.float32)
    lo = [L.orc_logit(p) for p in (0.9, 0.49, 0.12, 0.98, 0.499, 0.85)]
    grids = {}
    for m in fetch_modes():
        g = O.OracleGrid(half, 0.1, False, None, fp=m)
        g.set_origin_index((0, 0, 0))
        g.set_log_odds(*lo)
        g.set_state(occ)
        grids[m] = g
    queries = []
    import ctypes
    for _ in range(tries):
        c = rng.uniform(-1.5, 1.5, 3).astype(np.float32)
        gv = np.floor(c / 0.1).astype(np.int64) + rng.integers(-4, 5, size=3)
        cf = (ctypes.c_float * 3)(*[float(v) for v in c])
        gi = (ctypes.c_int * 3)(*[int(v) for v in gv])
        sums = sorted({np.float32(L.orc_fetch_sos(cf, gi, np.float32(0.1), 0, m)) for m in fetch_modes()})
        if len(sums) < 2 or sums[0] <= 0:
            continue
        r = np.float32(np.sqrt(np.float64(sums[0])))
        found = None
        for _k in range(8):
            r2 = np.float32(r * r)
            if sums[0] <= r2 < sums[-1]:
                found = r
                break
            r = np.nextafter(r, np.float32(np.inf)) if r2 < sums[0] else np.nextafter(r, np.float32(-np.inf))
        if found is None or found <= 0.05:
            continue
        sets = {m: _fetch_set(g, c, float(found)) for m, g in grids.items()}
        if len({tuple(v) for v in sets.values()}) > 1:
            queries.append((c, float(found)))
        if len(queries) >= want:
            break
    return dict(half=half, occ=occ, lo=lo, queries=queries, grids=grids)


def run_fetch_ref(pr):
    r = O.RefGrid(pr["half"], 0.1, False, None)
    r.set_origin_index((0, 0, 0))
    r.set_log_odds(*pr["lo"])
    r.upload(pr["occ"])
    out = []
    for c, rad in pr["queries"]:
        pos, st = r.fetch(c, rad, -1, 0)
        out.append(sorted(map(tuple, np.concatenate(
            [pos.view(np.uint32), st[:, None].astype(np.uint32)], axis=1).tolist())))
    r.close()
    return out


def matching_fetch_modes(pr, results):
    ok = []
    for m, g in pr["grids"].items():
        if all(_fetch_set(g, c, r) == res for (c, r), res in zip(pr["queries"], results)):
            ok.append(m)
    return ok


def describe(mode: int) -> str:
    names = ["plain", "fy_fz", "fx_fz", "p_fz", "fy_p", "fx_p"]
    return (f"ray_sos={names[mode & 7]} clip={bool(mode & O.FP_CLIP_FMA)} "
            f"bound={bool(mode & O.FP_BOUND_FMA)} center={bool(mode & O.FP_CENTER_FMA)} "
            f"miss={bool(mode & O.FP_MISS_FMA)} hit={bool(mode & O.FP_HIT_FMA)} "
            f"rec_sos={names[(mode >> 8) & 7]} fetch_sos={names[(mode >> 11) & 7]} "
            f"fetch_d={bool(mode & O.FP_FETCH_DFMA)}")
