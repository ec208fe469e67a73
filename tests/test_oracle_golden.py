"""Pin the C oracle against the reference's own known-answer vectors.

Every vector comes from tests/golden/reference_kats.json, which
tests/golden/make_golden.py extracts from the midnight-zk sources (file:line
recorded per vector).  CPU only.
"""
import numpy as np
import pytest

from oracle import oracle as O

R_INT = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
P_INT = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB


def L(entry):
    return O.u64s(entry["limbs"])


def fr_can(x):
    return O.to_int(O.fr_op("to_canonical", x))


def fr_mont(v):
    return O.fr_op("from_canonical", O.from_int(v % R_INT, 4))


def fp_mont(v):
    return O.fp_op("from_canonical", O.from_int(v % P_INT, 6))


# ---------------------------------------------------------------- Fr ----
def test_fr_modulus_and_montgomery_constants(kats):
    fr = kats["fr"]
    assert O.to_int(L(fr["MODULUS"])) == R_INT
    assert np.array_equal(O.fr_const(0), L(fr["R"]))
    assert np.array_equal(O.fr_const(1), L(fr["R2"]))
    assert O.to_int(L(fr["R3"])) == pow(2, 768, R_INT)
    assert (-pow(R_INT, -1, 2**64)) % 2**64 == int(fr["INV"]["value"], 16)
    for name, which in [("ROOT_OF_UNITY", 2), ("ZETA", 3), ("ROOT_OF_UNITY_INV", 4), ("DELTA", 5), ("GENERATOR", 6)]:
        assert np.array_equal(O.fr_const(which), L(fr[name])), name


def test_fr_constant_relations(kats):
    fr = kats["fr"]
    s = fr["S"]["value"]
    root = fr_can(L(fr["ROOT_OF_UNITY"]))
    assert pow(root, 2**s, R_INT) == 1 and pow(root, 2 ** (s - 1), R_INT) != 1
    assert fr_can(L(fr["GENERATOR"])) == 7
    assert pow(7, (R_INT - 1) >> s, R_INT) == root
    assert root * fr_can(L(fr["ROOT_OF_UNITY_INV"])) % R_INT == 1
    assert pow(7, 2**s, R_INT) == fr_can(L(fr["DELTA"]))
    zeta = fr_can(L(fr["ZETA"]))
    assert zeta != 1 and pow(zeta, 3, R_INT) == 1
    assert 2 * fr_can(L(fr["TWO_INV"])) % R_INT == 1


def test_fr_mul_kat(kats):
    k = kats["fr"]["kat_mul"]
    assert np.array_equal(O.fr_op("mul", L(k["a"]), L(k["b"])), L(k["expected"]))


def test_fr_add_kats(kats):
    largest = L(kats["fr"]["LARGEST"])
    assert np.array_equal(O.fr_op("add", largest, largest), L(kats["fr"]["kat_largest_plus_largest"]["expected"]))
    one_raw = O.from_int(1, 4)
    assert O.to_int(O.fr_op("add", largest, one_raw)) == 0
    assert np.array_equal(O.fr_op("neg", largest), one_raw)
    assert np.array_equal(O.fr_op("neg", one_raw), largest)


def test_fr_to_bytes_kats(kats):
    tb = kats["fr"]["kat_to_bytes"]
    def le_bytes(x):
        return list(O.to_int(O.fr_op("to_canonical", x)).to_bytes(32, "little"))
    assert le_bytes(np.zeros(4, np.uint64)) == tb["zero"]["bytes"]
    assert le_bytes(O.fr_const(0)) == tb["one"]["bytes"]
    assert le_bytes(O.fr_const(1)) == tb["r2"]["bytes"]
    assert le_bytes(O.fr_op("neg", O.fr_const(0))) == tb["minus_one"]["bytes"]
    for enc in kats["fr"]["kat_from_bytes_invalid"]:
        assert int.from_bytes(bytes(enc["bytes"]), "little") >= R_INT


def test_fr_random_algebra():
    xs = O.rand_fr(11, 64)
    for i in range(0, 60, 3):
        a, b, c = xs[i], xs[i + 1], xs[i + 2]
        ai, bi, ci = fr_can(a), fr_can(b), fr_can(c)
        assert fr_can(O.fr_op("mul", a, b)) == ai * bi % R_INT
        assert fr_can(O.fr_op("add", a, c)) == (ai + ci) % R_INT
        assert fr_can(O.fr_op("sub", a, c)) == (ai - ci) % R_INT
        assert fr_can(O.fr_op("inv", a)) == pow(ai, -1, R_INT)


def test_rand_fr_is_canonical_and_deterministic():
    a = O.rand_fr(5, 1000)
    b = O.rand_fr(5, 500, first=500)
    assert np.array_equal(a[500:], b)
    assert all(O.to_int(x) < R_INT for x in a)
    assert len({O.to_int(x) for x in a}) == 1000


# ---------------------------------------------------------------- Fp ----
def test_fp_constants(kats):
    fp = kats["fp"]
    assert O.to_int(L(fp["MODULUS"])) == P_INT
    assert np.array_equal(O.fp_const(0), L(fp["R"]))
    assert O.to_int(O.fp_const(1)) == pow(2, 768, P_INT)


def test_fp_mul_and_square_kats(kats):
    fp = kats["fp"]
    k = fp["kat_mul"]
    assert np.array_equal(O.fp_op("mul", L(k["a"]), L(k["b"])), L(k["expected"]))
    k = fp["kat_square"]
    a = L(k["a"])
    expected = O.fp_op("from_canonical", L(k["expected_canonical"]))
    assert np.array_equal(O.fp_op("mul", a, a), expected)


def test_fp_add_sub_kats(kats):
    for k in kats["fp"]["kat_add"]:
        got = O.fp_op("add", L(k["a"]), L(k["b"]))
        if k.get("expected_zero"):
            assert O.to_int(got) == 0
        else:
            assert np.array_equal(got, L(k["expected"]))
    for k in kats["fp"]["kat_sub"]:
        assert np.array_equal(O.fp_op("sub", L(k["a"]), L(k["b"])), L(k["expected"]))


def test_fp_inverse():
    rng = np.random.default_rng(3)
    for _ in range(20):
        v = int.from_bytes(rng.bytes(48), "little") % P_INT
        a = fp_mont(v)
        assert O.to_int(O.fp_op("to_canonical", O.fp_op("inv", a))) == pow(v, -1, P_INT)


# ---------------------------------------------------------------- G1 ----
def test_g1_generator_and_b(kats):
    g = kats["g1"]
    assert np.array_equal(O.fp_const(2), L(g["B"]))
    gx, gy = int(g["generator"]["x"]), int(g["generator"]["y"])
    gen = O.g1_generator()
    assert O.to_int(O.fp_op("to_canonical", gen[:6])) == gx
    assert O.to_int(O.fp_op("to_canonical", gen[6:])) == gy
    assert O.g1_is_on_curve(gen)


def test_g1_double_kat(kats):
    k = kats["g1"]["kat_double_generator"]
    jac = O.g1_jac_double(O.g1_from_affine(O.g1_generator()))
    aff = O.g1_to_affine(jac)
    assert np.array_equal(aff[:6], L(k["x"])) and np.array_equal(aff[6:], L(k["y"]))


def test_g1_add_kats(kats):
    k = kats["g1"]["kat_add"]
    gen = O.g1_generator()
    # identity + (G with a non-trivial z) == G   (g1.rs:1199-1221)
    z = L(k["z"])
    z2 = O.fp_op("mul", z, z)
    z3 = O.fp_op("mul", z2, z)
    gz = np.concatenate([O.fp_op("mul", gen[:6], z2), O.fp_op("mul", gen[6:], z3), z])
    c = O.g1_jac_add(np.zeros(18, np.uint64), gz)
    assert np.array_equal(O.g1_to_affine(c), gen)
    # degenerate case: 4G + (beta^2 x, -y, z)   (g1.rs:1257-1294)
    a = O.g1_jac_double(O.g1_jac_double(O.g1_from_affine(gen)))
    beta = L(k["beta"])
    beta2 = O.fp_op("mul", beta, beta)
    b = np.concatenate([O.fp_op("mul", a[:6], beta2), O.fp_op("sub", np.zeros(6, np.uint64), a[6:12]), a[12:]])
    c = O.g1_to_affine(O.g1_jac_add(a, b))
    assert np.array_equal(c[:6], L(k["expected_x"])) and np.array_equal(c[6:], L(k["expected_y"]))


def test_g1_scalar_mul_kat(kats):
    k = kats["g1"]["kat_scalar_mul"]
    a, b = L(k["a"]), L(k["b"])
    gen = O.g1_generator()
    lhs = O.g1_mul(O.g1_mul(gen, a), b)
    rhs = O.g1_mul(gen, O.fr_op("mul", a, b))
    assert np.array_equal(lhs, rhs)
    assert O.g1_is_on_curve(lhs)


def test_g1_compress_generator():
    # the compressed generator is x with the compression flag set
    gen = O.g1_generator()
    c = O.g1_compress(gen)
    x = O.to_int(O.fp_op("to_canonical", gen[:6]))
    assert c[0] & 0x80 and not c[0] & 0x40
    assert int.from_bytes(bytes([c[0] & 0x1F]) + c[1:], "big") == x
    assert O.g1_compress(np.zeros(12, np.uint64))[0] == 0xC0


def test_gen_bases_are_r_times_g():
    bases = O.gen_bases(77, 16)
    rs = O.rand_fr(77, 16)
    gen = O.g1_generator()
    for i in range(16):
        assert np.array_equal(bases[i], O.g1_mul(gen, rs[i]))
        assert O.g1_is_on_curve(bases[i])


# ---------------------------------------------------------------- MSM ----
def test_booth_index_recomposes_scalar():
    """Same property as test_booth_encoding (curves/src/msm.rs:548-590)."""
    xs = O.rand_fr(9, 10)
    for x in xs:
        v = fr_can(x)
        rep = v.to_bytes(32, "little")
        for c in range(1, 18):
            nwin = 255 // c + 1
            tot = sum(O.booth_index(w, c, rep) * (1 << (c * w)) for w in range(nwin))
            assert tot == v, (c, v)
            assert all(abs(O.booth_index(w, c, rep)) <= 1 << (c - 1) for w in range(nwin))


@pytest.mark.parametrize("n", [0, 1, 2, 3, 5, 31, 33, 100])
def test_msm_best_matches_naive(n):
    s = O.rand_fr(1000 + n, max(n, 1))[:n]
    b = O.gen_bases(2000 + n, max(n, 1))[:n]
    assert np.array_equal(O.msm_best(s, b), O.msm_naive(s, b))


def test_msm_best_edge_cases():
    n = 40
    s = O.rand_fr(5, n)
    b = O.gen_bases(6, n)
    s[3] = 0                      # zero scalar
    s[4] = O.fr_const(0)          # one
    b[5] = 0                      # identity base
    b[7] = b[6]                   # duplicate point
    s[7] = s[6]
    b[9] = b[8].copy()            # P and -P with the same scalar
    b[9][6:] = O.fp_op("sub", np.zeros(6, np.uint64), b[8][6:])
    s[9] = s[8]
    assert np.array_equal(O.msm_best(s, b), O.msm_naive(s, b))
    assert np.array_equal(O.msm_specific(s, b), O.msm_naive(s, b))


def test_msm_best_large_window_path_matches_closed_form():
    """n >= 8104 takes the c >= 10 batch-affine path (msm.rs:472-532).

    Bases are [r_i]G, so the MSM equals [sum s_i r_i]G."""
    n = 9000
    s = O.rand_fr(31, n)
    r = O.rand_fr(32, n)
    b = O.gen_bases(32, n)
    t = O.fr_inner_product(s, r)
    assert np.array_equal(O.msm_best(s, b), O.g1_mul(O.g1_generator(), t))


# ---------------------------------------------------------------- FFT ----
@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 8])
def test_best_fft_matches_dft(log_n):
    n = 1 << log_n
    d = O.Domain(2, log_n)
    omega = d.get(0)
    a = O.rand_fr(40 + log_n, n)
    tw = O.compute_twiddles(omega, log_n)
    for threads in (1, 8):
        assert np.array_equal(O.best_fft(a, tw, log_n, threads), O.dft_naive(a, omega))


@pytest.mark.parametrize("log_n,n_real", [(3, 2), (6, 16), (8, 64), (8, 50)])
def test_pruned_dif_matches_dit(log_n, n_real):
    n = 1 << log_n
    d = O.Domain(2, log_n)
    tw = O.compute_twiddles(d.get(0), log_n)
    a = np.zeros((n, 4), np.uint64)
    a[:n_real] = O.rand_fr(60 + n_real, n_real)
    assert np.array_equal(O.fft_dif_pruned(a, tw, log_n, n_real), O.best_fft(a, tw, log_n))


@pytest.mark.parametrize("k", [3, 6, 10])
def test_domain_roundtrips_and_coset_definition(k):
    d = O.Domain(5, k)
    assert d.extended_k == k + 2
    n = 1 << k
    a = O.rand_fr(70 + k, n)
    assert np.array_equal(d.lagrange_to_coeff(d.coeff_to_lagrange(a)), a)
    ext = d.coeff_to_extended(a)
    back = d.extended_to_coeff(ext)
    assert np.array_equal(back[:n], a) and not back[n:].any()
    assert np.array_equal(d.extended_to_lagrange(ext), d.coeff_to_lagrange(a))
    if k <= 6:
        zeta = O.fr_const(3)
        scaled = np.zeros((d.extended_len, 4), np.uint64)
        zp = O.fr_const(0)
        for i in range(n):
            scaled[i] = O.fr_op("mul", a[i], zp)
            zp = O.fr_op("mul", zp, zeta)
        assert np.array_equal(ext, O.dft_naive(scaled, d.get(2)))


def test_divide_by_vanishing_poly():
    k = 4
    d = O.Domain(5, k)
    # t(X) = X^n - 1 on the extended coset, divided by itself, is 1
    n, en = d.n, d.extended_len
    t = np.zeros((n, 4), np.uint64)
    t[0] = O.fr_op("neg", O.fr_const(0))
    tn = np.zeros((en, 4), np.uint64)
    tn[:n] = t
    # X^n - 1 has degree n: build it on the extended domain directly
    coeffs = np.zeros((en, 4), np.uint64)
    coeffs[0] = t[0]
    coeffs[n] = O.fr_const(0)
    zeta = O.fr_const(3)
    scaled = coeffs.copy()
    scaled[n] = O.fr_op("mul", coeffs[n], O.fr_op("mul", zeta, zeta) if n % 3 == 2 else (zeta if n % 3 == 1 else O.fr_const(0)))
    evals = O.dft_naive(scaled, d.get(2))
    q = d.divide_by_vanishing_poly(evals)
    assert all(np.array_equal(row, O.fr_const(0)) for row in q)


def test_eval_polynomial_matches_horner_and_dft():
    a = O.rand_fr(91, 1000)
    x = O.rand_fr(92, 1)[0]
    acc = np.zeros(4, np.uint64)
    for c in a[::-1]:
        acc = O.fr_op("add", O.fr_op("mul", acc, x), c)
    for threads in (1, 3, 8):
        assert np.array_equal(O.eval_polynomial(a, x, threads), acc)
    d = O.Domain(2, 6)
    b = O.rand_fr(93, 64)
    lag = d.coeff_to_lagrange(b)
    assert np.array_equal(lag[5], O.eval_polynomial(b, O.fr_pow(d.get(0), 5)))


def test_g1_decompress_inverts_compress():
    """from_compressed of to_compressed: the generator (the reference's README
    coordinates), random points and the identity; a cleared compression flag,
    x >= p and set padding bits of the identity are rejected."""
    pts = O.gen_bases(31, 16)
    pts[2] = 0
    pts = np.concatenate([pts, O.g1_generator().reshape(1, 12)])
    for p in pts:
        st, q = O.g1_decompress(O.g1_compress(p))
        assert st == 0 and np.array_equal(q, p)
    c = bytearray(O.g1_compress(O.g1_generator()))
    c[0] &= 0x7f
    assert O.g1_decompress(c)[0] == 1
    p_bytes = bytearray((0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab).to_bytes(48, "big"))
    p_bytes[0] |= 0x80
    assert O.g1_decompress(p_bytes)[0] == 1
    ident = bytearray(48)
    ident[0] = 0xc0
    assert O.g1_decompress(ident)[0] == 0
    ident[47] = 1
    assert O.g1_decompress(ident)[0] == 1
