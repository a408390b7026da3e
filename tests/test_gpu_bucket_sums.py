"""The batched-affine bucket summation (bucket_sum.cuh) on the special cases that
random proof inputs never reach: doubling, cancellation, infinity, many copies."""
import numpy as np
import pytest

import vkzg_b200

pytestmark = pytest.mark.gpu

P_MOD = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
INF = bytes(96)


def neg(xy):
    if xy == INF:
        return INF
    y = int.from_bytes(xy[48:], "big")
    return xy[:48] + ((P_MOD - y) % P_MOD).to_bytes(48, "big")


def test_bucket_sums_special_cases(oracle, mainnet_setup):
    comp = [mainnet_setup[48 * i:48 * (i + 1)] for i in range(40)]
    xy = [oracle.g1_decompress(c)[1] for c in comp]
    P, Q = xy[1], xy[2]
    buckets = {
        0: [P, P],
        1: [P, neg(P)],
        2: [INF, P],
        3: [P] * 5,
        4: [P, neg(P), Q],
        5: [P] * 33,
        6: [INF, INF],
        7: [Q, P, neg(P), P],
        8: xy[3:33],
        9: [P, Q, neg(Q), neg(P), P, P, Q],
        127: [neg(Q)] * 17 + [Q] * 3,
    }
    pts, idx = [], []
    for k, lst in buckets.items():
        pts += lst
        idx += [k] * len(lst)
    out = vkzg_b200.bucket_sums_selftest(b"".join(pts), idx)

    def compress(p):
        rc, c = oracle.lib.orc_g1_compress, None
        buf = np.zeros(48, np.uint8)
        a = np.frombuffer(p, np.uint8).copy()
        oracle.lib.orc_g1_compress(a.ctypes.data, buf.ctypes.data)
        return buf.tobytes()

    inf_c = bytes([0xC0]) + bytes(47)
    for k in range(128):
        want = inf_c
        for p in buckets.get(k, []):
            c = compress(p)
            want = c if want == inf_c else (want if c == inf_c else oracle.g1_add(want, c)[1])
        assert compress(out[96 * k:96 * (k + 1)]) == want, k


def test_tree_sums_special_cases(oracle, mainnet_setup):
    """The grid-wide tree rounds (plan 3) on equal-length lists holding the
    special cases, with odd lengths so that elements move up unchanged."""
    comp = [mainnet_setup[48 * i:48 * (i + 1)] for i in range(40)]
    xy = [oracle.g1_decompress(c)[1] for c in comp]
    P, Q = xy[1], xy[2]
    m = 7
    lists = [
        [P, P, INF, INF, INF, INF, INF],
        [P, neg(P), Q, Q, neg(Q), INF, P],
        [INF] * 7,
        [P] * 7,
        [Q, P, neg(P), P, neg(Q), neg(P), INF],
        xy[3:10],
        [neg(Q), neg(Q), Q, Q, Q, neg(Q), Q],
        [INF, INF, INF, INF, INF, INF, P],
    ] * 40  # 320 lists: pairs spread over several lanes and warps
    sums, _ = vkzg_b200.tree_sums_selftest(b"".join(b"".join(l) for l in lists), len(lists), m)

    def compress(p):
        buf = np.zeros(48, np.uint8)
        a = np.frombuffer(p, np.uint8).copy()
        oracle.lib.orc_g1_compress(a.ctypes.data, buf.ctypes.data)
        return buf.tobytes()

    inf_c = bytes([0xC0]) + bytes(47)
    for o, lst in enumerate(lists[:8]):
        want = inf_c
        for p in lst:
            c = compress(p)
            want = c if want == inf_c else (want if c == inf_c else oracle.g1_add(want, c)[1])
        for rep in range(40):
            k = o + 8 * rep
            assert compress(sums[96 * k:96 * (k + 1)]) == want, (o, rep)


def test_tree_sums_seeded_workload_runs():
    _, ms = vkzg_b200.tree_sums_selftest(None, 4096, 64, seed=3)
    assert ms > 0
