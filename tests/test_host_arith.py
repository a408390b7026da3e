"""The device arithmetic headers (field.cuh, curve.cuh) built for the host --
the PTX carry-chain multiply runs with its carry flag emulated -- checked
against Python integers and the oracle (CPU only)."""
import ctypes
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P_MOD = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R_MOD = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "libshim.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-o", out,
                           os.path.join(ROOT, "tests", "host_shim.cpp")])
    return ctypes.CDLL(out)


def words(x, n):
    return (ctypes.c_uint32 * n)(*[(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)])


def value(a, n):
    return sum(a[i] << (32 * i) for i in range(n))


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_ops(shim, field):
    mod, n, radix = (P_MOD, 12, 1 << 384) if field == "fp" else (R_MOD, 8, 1 << 256)
    rinv = pow(radix, -1, mod)
    rng = random.Random(7)
    top = mod.bit_length() - 1
    edge = [0, 1, 2, mod - 1, mod - 2, radix % mod, radix * radix % mod, mod // 2, (mod + 1) // 2,
            (1 << top) - 1, mod - (1 << 32), mod - (1 << 200) - 1, ((1 << top) - 1) ^ (0xFFFF << 64)]
    edge += [mod - 1 - rng.randrange(1 << 64) for _ in range(50)]  # long runs of high words
    half = 16 * n  # Karatsuba halves: equal, one apart, all-ones low half
    edge += [(x << half) | x for x in (1, (1 << (top - half)) - 1, rng.randrange(1 << (top - half)))]
    edge += [(x << half) | (x + 1) for x in (0, rng.randrange(1 << (top - half)))]
    edge += [(x << half) | ((1 << half) - 1) for x in (0, 1, (1 << (top - half)) - 1)]
    quarter = 8 * n  # second Karatsuba level: equal quarters
    edge += [sum(x << (quarter * k) for k in range(4)) % mod for x in (1, (1 << quarter) - 1, rng.randrange(1 << quarter))]
    edge += [((1 << quarter) - 1) | (x << (2 * quarter)) for x in (0, 1, rng.randrange(1 << (top - 2 * quarter)))]
    vals = edge + [rng.randrange(mod) for _ in range(2000)]
    out = (ctypes.c_uint32 * n)()
    for k, a in enumerate(vals):
        b = vals[(7 * k + 3) % len(vals)]
        getattr(shim, f"shim_{field}_mul")(words(a, n), words(b, n), out)
        assert value(out, n) == a * b * rinv % mod
        getattr(shim, f"shim_{field}_mul_ks")(words(a, n), words(b, n), out)
        assert value(out, n) == a * b * rinv % mod
        getattr(shim, f"shim_{field}_mul_ks2")(words(a, n), words(b, n), out)
        assert value(out, n) == a * b * rinv % mod
        getattr(shim, f"shim_{field}_sqr")(words(a, n), words(b, n), out)
        assert value(out, n) == a * a * rinv % mod
        getattr(shim, f"shim_{field}_sqr_ks")(words(a, n), words(b, n), out)
        assert value(out, n) == a * a * rinv % mod
        getattr(shim, f"shim_{field}_add")(words(a, n), words(b, n), out)
        assert value(out, n) == (a + b) % mod
        getattr(shim, f"shim_{field}_sub")(words(a, n), words(b, n), out)
        assert value(out, n) == (a - b) % mod
    for a in vals[1:60]:
        if a == 0:
            continue
        getattr(shim, f"shim_{field}_inv")(words(a * radix % mod, n), out)
        assert value(out, n) == pow(a, -1, mod) * radix % mod


def test_fp_products_on_the_fp64_pipe(shim):
    """field_f64.cuh's products (50-bit limbs, exact FMA splits) equal a b / 2^384 mod p,
    including limbs at their extremes (all-ones 50-bit limbs, zero limbs, p - 1)."""
    rng = random.Random(11)
    mask50 = (1 << 50) - 1
    edge = [0, 1, P_MOD - 1, P_MOD - 2, (1 << 380) - 1, P_MOD >> 1, (1 << 384) % P_MOD]
    edge += [sum(mask50 << (50 * i) for i in range(k)) % P_MOD for k in range(1, 9)]
    edge += [(mask50 << (50 * i)) % P_MOD for i in range(8)]
    edge += [P_MOD - 1 - (mask50 << (50 * i)) for i in range(7)]
    edge += [P_MOD - 1 - rng.randrange(1 << 64) for _ in range(20)]
    vals = edge + [rng.randrange(P_MOD) for _ in range(3000)]
    rinv = pow(1 << 384, -1, P_MOD)
    out = (ctypes.c_uint32 * 12)()
    for k, a in enumerate(vals):
        for b in (vals[(7 * k + 3) % len(vals)], a, P_MOD - 1, vals[-1 - k % len(vals)]):
            shim.shim_fp_mul_f64(words(a, 12), words(b, 12), out)
            assert value(out, 12) == a * b * rinv % P_MOD, (hex(a), hex(b))
        shim.shim_fp_sqr_f64(words(a, 12), words(a, 12), out)
        assert value(out, 12) == a * a * rinv % P_MOD, hex(a)


def test_fr_from_raw_noncanonical(shim):
    """Raw 256-bit words (cells are not canonicity-checked) reduce mod r."""
    rng = random.Random(3)
    out = (ctypes.c_uint32 * 8)()
    for v in [R_MOD, R_MOD + 5, (1 << 256) - 1, 2 * R_MOD - 1] + [rng.randrange(1 << 256) for _ in range(500)]:
        shim.shim_fr_from_raw(words(v, 8), out)
        assert value(out, 8) == v % R_MOD * (1 << 256) % R_MOD


def test_curve_ops(shim, oracle, mainnet_setup):
    pts = [mainnet_setup[48 * i:48 * (i + 1)] for i in (0, 1, 17, 4095)]
    for p in pts:
        for q in pts:
            o1 = ctypes.create_string_buffer(48)
            o2 = ctypes.create_string_buffer(48)
            assert shim.shim_g1_ops(p, q, o1, o2) == 0
            _, two_p = oracle.g1_mul(p, (2).to_bytes(32, "big"))
            _, want = oracle.g1_add(two_p, q)
            assert o1.raw == want and o2.raw == want
    rng = random.Random(5)
    for _ in range(5):
        k = rng.randrange(R_MOD)
        o = ctypes.create_string_buffer(48)
        assert shim.shim_g1_mul(pts[1], words(k, 8), o) == 0
        _, want = oracle.g1_mul(pts[1], k.to_bytes(32, "big"))
        assert o.raw == want


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_divstep_inverse(shim, field):
    """Batched-divstep inversion (Montgomery in, Montgomery out) equals x^-1, with
    fixed 30-divstep batches (the default) and, for Fp, in variable time."""
    mod, n, radix = (P_MOD, 12, 1 << 384) if field == "fp" else (R_MOD, 8, 1 << 256)
    rng = random.Random(11)
    vals = [1, 2, 3, mod - 1, mod - 2, (mod - 1) // 2, 1 << 200, (1 << 250) + 1, radix % mod]
    vals += [rng.randrange(1, mod) for _ in range(3000)]
    out = (ctypes.c_uint32 * n)()
    fns = [getattr(shim, f"shim_{field}_inv_fast")]
    if field == "fp":
        fns.append(shim.shim_fp_inv_var)  # the variable-time divstep batches
    for fn in fns:
        for x in vals:
            fn(words(x * radix % mod, n), out)
            assert value(out, n) == pow(x, -1, mod) * radix % mod, hex(x)
        fn(words(0, n), out)
        assert value(out, n) == 0


def test_comb_window_layout(shim):
    """The digit table's windows (CombWindows, the device's layout) for every
    window count 18..32: widths of W and W + 1 bits summing to exactly 256,
    each window at the sum of the widths below it, each window's 2^(width - 1)
    entries after those of the windows below it; and the same table sizes as the
    Python helper the tests and the bench use."""
    import vkzg_b200
    fn = shim.shim_comb_windows
    for d in range(18, 33):
        width = (ctypes.c_int * 32)()
        bit = (ctypes.c_int * 32)()
        entry = (ctypes.c_uint32 * 32)()
        entries = ctypes.c_uint32()
        fn(d, width, bit, entry, ctypes.byref(entries))
        widths = list(width[:d])
        assert sum(widths) == 256 and max(widths) - min(widths) <= 1
        assert widths == vkzg_b200.comb_windows(d)
        assert list(bit[:d]) == [sum(widths[:k]) for k in range(d)]
        assert list(entry[:d]) == [sum(1 << (w - 1) for w in widths[:k]) for k in range(d)]
        assert entries.value == sum(1 << (w - 1) for w in widths)
        assert vkzg_b200.comb_table_bytes(d) == 128 * 64 * entries.value * 96
        assert max(widths) <= 15  # digits up to 2^14 in magnitude fit int16


def test_divsteps_grouped_equal_serial(shim):
    """The table-driven divstep groups (seven of 4 steps and one of 2, as the
    proof rounds' four-lane inversion runs them) give the same delta and
    transition matrix as 30 single divsteps, for deltas inside and far outside
    the tables' clamped range."""
    fn = shim.shim_divsteps_grouped_differs
    fn.argtypes = [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32]
    fn.restype = ctypes.c_int
    rng = random.Random(5)
    for k in range(40000):
        delta = rng.randint(-6, 6) if k % 2 else rng.randint(-900, 900)
        f = rng.getrandbits(32) | 1
        g = rng.getrandbits(32) if k % 7 else rng.getrandbits(32) & ~0x3FF  # long runs of even g
        assert fn(delta, f, g) == 0, (delta, hex(f), hex(g))


Z2 = 0xD201000000010000 ** 2


def test_endomorphism_and_tap_split(shim, oracle, mainnet_setup):
    """phi(x, y) = (beta x, y) equals (-z^2) P on setup points, and the tap split
    k = k1 + k2 z^2 (mod r) with both halves in 16 signed base-256 digits, which
    the proof ladder relies on."""
    lam = (-Z2) % R_MOD
    pts = [bytes(mainnet_setup[48 * i:48 * i + 48]) for i in (0, 1, 2, 4095)]
    for p in pts:
        o = ctypes.create_string_buffer(48)
        assert shim.shim_g1_phi(p, o) == 0
        _, want = oracle.g1_mul(p, lam.to_bytes(32, "big"))
        assert o.raw == want
    rng = random.Random(13)
    ks = [0, 1, 2, R_MOD - 1, R_MOD - 2, Z2 - 1, Z2, Z2 + 1, Z2 // 2, Z2 // 2 + 1, Z2 * (Z2 // 2),
          Z2 * (Z2 // 2 + 1), Z2 * (Z2 // 2 + 1) + Z2 // 2 + 1, (Z2 - 1) * Z2 + Z2 - 1, R_MOD // 2]
    ks += [rng.randrange(R_MOD) for _ in range(3000)]
    mag = (ctypes.c_uint32 * 8)()
    neg = (ctypes.c_int * 2)()
    dig = (ctypes.c_int * 32)()
    for k in ks:
        k %= R_MOD
        assert shim.shim_glv_split(words(k, 8), mag, neg, dig) == 0, hex(k)
        m1, m2 = value(mag, 4), sum(mag[4 + i] << (32 * i) for i in range(4))
        c1, c2 = (-m1 if neg[0] else m1), (-m2 if neg[1] else m2)
        assert max(m1, m2) <= Z2 // 2 + 1
        assert (c1 + c2 * lam - k) % R_MOD == 0, hex(k)
        assert sum(dig[d] << (8 * d) for d in range(16)) == c1
        assert sum(dig[16 + d] << (8 * d) for d in range(16)) == c2
        assert all(-128 <= v <= 128 for v in dig)
