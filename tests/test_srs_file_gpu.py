"""SRS file reading on the B200 (ParamsKZG::read_custom, SerdeFormat::
Processed, params.rs:283-350) and G1Affine::from_compressed on the device,
against the oracle: valid points, the identity, bad encodings, points off
the curve and points on the curve outside G1."""
import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu

P_MOD = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def encodings():
    pts = O.gen_bases(41, 40)
    pts[7] = 0
    enc = [bytes(O.g1_compress(p)) for p in pts]
    bad = bytearray(enc[0])
    bad[0] &= 0x7f                                   # compression flag cleared
    enc.append(bytes(bad))
    over = bytearray((P_MOD + 5).to_bytes(48, "big"))
    over[0] |= 0x80                                  # x >= p
    enc.append(bytes(over))
    ident_pad = bytearray(48)
    ident_pad[0], ident_pad[20] = 0xc0, 1            # identity with a stray bit
    enc.append(bytes(ident_pad))
    for x in range(1, 40):                           # small x: off the curve or outside G1
        b = bytearray(48)
        b[47], b[0] = x, 0x80 | (0x20 if x % 2 else 0)
        enc.append(bytes(b))
    return enc


@pytest.mark.parametrize("check", [True, False])
def test_decompress_matches_oracle(ctx, check):
    enc = encodings()
    n = len(enc)
    raw = np.frombuffer(b"".join(enc), np.uint8)
    d_in, d_out, d_st = ctx.alloc(raw.nbytes), ctx.alloc(n * 96), ctx.alloc(n)
    d_in.upload(raw)
    bad = ctx.g1_decompress_device(d_in, n, d_out, d_st, check_subgroup=check)
    got = d_out.download((n, 12))
    st = d_st.download((n,), np.uint8)
    want = [O.g1_decompress(e, check) for e in enc]
    assert [int(s) for s in st] == [w[0] for w in want]
    assert bad == sum(1 for w in want if w[0])
    for i, (s, p) in enumerate(want):
        assert np.array_equal(got[i], p if s == 0 else np.zeros(12, np.uint64)), i
    assert {int(s) for s in st} >= ({0, 1, 2, 3} if check else {0, 1, 2})


def srs_file(k, s):
    g, lag, _, _ = O.srs_setup(s, k)
    body = b"".join(bytes(O.g1_compress(p)) for p in g) + b"".join(bytes(O.g1_compress(p)) for p in lag)
    return k.to_bytes(4, "little") + body + bytes(192)  # the G2 elements are not read


def test_read_processed_matches_setup(ctx):
    k = 7
    s = O.rand_fr(99, 1)[0]
    data = srs_file(k, s)
    n = 1 << k
    bufs = [ctx.alloc(n * 96) for _ in range(4)]
    assert ctx.srs_read_processed(data, n, *bufs) == k
    for b, w in zip(bufs, O.srs_setup(s, k)):
        assert np.array_equal(b.download((n, 12)), w)


def test_read_processed_rejects(ctx):
    k = 4
    n = 1 << k
    data = bytearray(srs_file(k, O.rand_fr(98, 1)[0]))
    bufs = [ctx.alloc(n * 96) for _ in range(4)]
    with pytest.raises(mzk.MzkError):
        ctx.srs_read_processed(bytes(data[:100]), n, *bufs)          # short buffer
    with pytest.raises(mzk.MzkError):
        ctx.srs_read_processed(bytes(data), n // 2, *bufs)           # capacity below 2^k
    data[4 + 3 * 48 + 47] ^= 1                                       # corrupt one point of g
    with pytest.raises(mzk.MzkError):
        ctx.srs_read_processed(bytes(data), n, *bufs)


# ---- the subgroup check against points with a torsion component of every
# prime-power order dividing the G1 cofactor (plain Python curve arithmetic) ----
R_ORDER = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
COFACTOR_PRIMES = [(3, 1), (11, 2), (10177, 2), (859267, 2), (52437899, 2)]  # (l, e): l^e | h
COFACTOR = 3 * 11 ** 2 * 10177 ** 2 * 859267 ** 2 * 52437899 ** 2
GEN = (0x17F1D3A73197D7942695638C4FA9AC0FC3688C4F9774B905A14E3A3F171BAC586C55E83FF97A1AEFFB3AF00ADB22C6BB,
       0x08B3F481E3AAA0F1A09E30ED741D8AE4FCF5E095D5D00AF600DB18CB2C04B3EDD03CC744A2888AE40CAA232946C5E7E1)


def ec_add(a, b):
    if a is None:
        return b
    if b is None:
        return a
    (x1, y1), (x2, y2) = a, b
    if x1 == x2:
        if (y1 + y2) % P_MOD == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, P_MOD) % P_MOD
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, P_MOD) % P_MOD
    x3 = (lam * lam - x1 - x2) % P_MOD
    return x3, (lam * (x1 - x3) - y1) % P_MOD


def ec_mul(a, k):
    acc = None
    for bit in bin(k)[2:]:
        acc = ec_add(acc, acc)
        if bit == "1":
            acc = ec_add(acc, a)
    return acc


def curve_point(x):
    rhs = (x ** 3 + 4) % P_MOD
    y = pow(rhs, (P_MOD + 1) // 4, P_MOD)
    return (x, y) if y * y % P_MOD == rhs else None


def compress(pt):
    x, y = pt
    b = bytearray(x.to_bytes(48, "big"))
    b[0] |= 0x80 | (0x20 if y > P_MOD - y else 0)
    return bytes(b)


def torsion_cases():
    """(encoding, in G1) pairs: for every prime l | h, a point T of the
    l-Sylow subgroup (order l or l^2), T plus a G1 point, [l] T when that is
    not the identity, and G1 points."""
    assert COFACTOR * R_ORDER == P_MOD + 1 - (1 - 0xD201000000010000)  # #E(Fp) = p + 1 - t
    raw = [pt for pt in (curve_point(x) for x in range(2, 60)) if pt]
    cases = []
    for i, (l, e) in enumerate(COFACTOR_PRIMES):
        t = next(t for t in (ec_mul(pt, COFACTOR * R_ORDER // l ** e) for pt in raw) if t is not None)
        assert ec_mul(t, l ** e) is None
        g = ec_mul(GEN, 7 + 1000 * i)
        cases += [(compress(t), False), (compress(ec_add(g, t)), False), (compress(g), True)]
        lt = ec_mul(t, l)
        if lt is not None:
            cases += [(compress(lt), False), (compress(ec_add(g, lt)), False)]
    return cases


def test_subgroup_check_on_torsion_components(ctx):
    cases = torsion_cases()
    enc = [c for c, _ in cases]
    n = len(enc)
    raw = np.frombuffer(b"".join(enc), np.uint8)
    d_in, d_out, d_st = ctx.alloc(raw.nbytes), ctx.alloc(n * 96), ctx.alloc(n)
    d_in.upload(raw)
    bad = ctx.g1_decompress_device(d_in, n, d_out, d_st, check_subgroup=True)
    st = [int(s) for s in d_st.download((n,), np.uint8)]
    want = [O.g1_decompress(e, True)[0] for e in enc]
    assert want == [0 if ok else 3 for _, ok in cases]
    assert st == want
    assert bad == sum(1 for _, ok in cases if not ok)


def test_compress_matches_oracle_and_round_trips(ctx):
    """G1Affine::to_compressed on the device: the oracle's encoding for
    random points, the identity and a point with y and p - y swapped, and
    decompression of the result gives the points back."""
    pts = O.gen_bases(71, 300)
    pts[5] = 0                                        # the identity
    pts[6, 6:] = O.fp_op("sub", np.zeros(6, np.uint64), pts[6, 6:])  # -P: the other sign
    n = pts.shape[0]
    d_pts, d_out = ctx.alloc(pts.nbytes), ctx.alloc(n * 48)
    d_pts.upload(pts)
    ctx.g1_compress_device(d_pts, n, d_out)
    enc = d_out.download((n * 48,), np.uint8)
    want = b"".join(bytes(O.g1_compress(p)) for p in pts)
    assert enc.tobytes() == want
    d_back, d_st = ctx.alloc(n * 96), ctx.alloc(n)
    assert ctx.g1_decompress_device(d_out, n, d_back, d_st, check_subgroup=True) == 0
    assert np.array_equal(d_back.download((n, 12)), pts)


def test_write_then_read_processed(ctx):
    k = 6
    n = 1 << k
    s = O.rand_fr(123, 1)[0]
    g, lag, delta, ddelta = O.srs_setup(s, k)
    d_g, d_l = ctx.alloc(g.nbytes), ctx.alloc(lag.nbytes)
    d_g.upload(g)
    d_l.upload(lag)
    data = ctx.srs_write_processed(d_g, d_l, n)
    assert data == srs_file(k, s)[:4 + 96 * n]      # the oracle-built file, G1 part
    bufs = [ctx.alloc(n * 96) for _ in range(4)]
    assert ctx.srs_read_processed(data + bytes(192), n, *bufs) == k
    for b, w in zip(bufs, (g, lag, delta, ddelta)):
        assert np.array_equal(b.download((n, 12)), w)
    with pytest.raises(mzk.MzkError):
        ctx.srs_write_processed(d_g, d_l, 48)           # not a power of two
