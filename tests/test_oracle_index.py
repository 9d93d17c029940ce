"""Index-map properties of the oracle, on the reference's own fixtures.

Re-expresses test/test_utils_index_roundtrip.cpp:44-180 (host) and
test/test_utils_index_roundtrip.cu:66-147 (host utils.cuh): local->global->
local, local->hash->local, global->hash->global, pos->global->pos->global,
pos->hash->pos->hash over the three map fixtures, 500 seeded samples each.
"""
import ctypes

import numpy as np
import pytest

import oracle as O

FIXTURES = [((200, 200, 100), (17, -42, 8), 0.05, True),
            ((350, 350, 75), (-120, 55, 0), 0.1, False),
            ((3, 5, 7), (2, -1, 4), 0.25, True)]
L = O.oracle_lib()


def i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def l2g(l, m, h, o):
    return [L.orc_local_to_global(l[a], m[a], h[a], o[a]) for a in range(3)]


def g2l(g, m, h):
    return [L.orc_global_to_local(g[a], m[a], h[a]) for a in range(3)]


def g2h(g, m, h):
    return L.orc_global_to_hash(i3(g), i3(m), i3(h))


def h2l(hh, m, h):
    out = (ctypes.c_int * 3)()
    L.orc_hash_to_local(hh, i3(m), i3(h), out)
    return list(out)


def p2g(p, inv, ctr, host=1):
    return [L.orc_pos_to_global(float(p[a]), inv, int(ctr), host, O.FP_PINNED) for a in range(3)]


def g2p(g, res, ctr):
    return [L.orc_global_to_pos(int(g[a]), res, int(ctr)) for a in range(3)]


@pytest.mark.parametrize("fx", FIXTURES, ids=["center200", "corner350", "center3"])
def test_roundtrips(fx):
    half, origin, res, ctr = fx
    m = [2 * h + 1 for h in half]
    res = float(np.float32(res))
    inv = float(np.float32(1.0) / np.float32(res))
    rng = np.random.default_rng(42)
    for _ in range(500):
        l = [int(rng.integers(-half[a], half[a] + 1)) for a in range(3)]
        g = l2g(l, m, half, origin)
        assert g2l(g, m, half) == l
        hh = int(L.orc_global_to_hash(i3(g), i3(m), i3(half)))
        assert 0 <= hh < m[0] * m[1] * m[2]
        assert h2l(hh, m, half) == l
        assert l2g(h2l(hh, m, half), m, half, origin) == g
    for host in (1, 0):
        for _ in range(500):
            p = rng.uniform(-20, 20, 3).astype(np.float32)
            g = p2g(p, inv, ctr, host)
            pb = np.float32(g2p(g, res, ctr))
            assert p2g(pb, inv, ctr, host) == g
            hh = g2h(g, m, half)
            back = l2g(h2l(hh, m, half), m, half, origin)
            pb2 = np.float32(g2p(back, res, ctr))
            assert g2h(p2g(pb2, inv, ctr, host), m, half) == hh


def test_c_remainder_semantics():
    # C `%` truncates toward zero; negative globals wrap into [-h, h]
    assert L.orc_global_to_local(-1, 5, 2) == -1
    assert L.orc_global_to_local(-3, 5, 2) == 2
    assert L.orc_global_to_local(3, 5, 2) == -2
    assert L.orc_global_to_local(-7, 5, 2) == -2


def test_device_float_to_int_saturates_and_host_does_not():
    assert L.orc_pos_to_global(float("nan"), 10.0, 0, 0, 0) == 0
    assert L.orc_pos_to_global(3e9, 10.0, 0, 0, 0) == 2**31 - 1
    assert L.orc_pos_to_global(3e9, 10.0, 0, 1, 0) == -(2**31)
    assert L.orc_pos_to_global(float("nan"), 10.0, 0, 1, 0) == -(2**31)
