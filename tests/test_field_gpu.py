"""The dedicated Fp squaring on the B200 equals the general Montgomery
multiplication a * a limb for limb, on random lazily reduced values in
[0, 2p) and on the carry extremes: 0, 1, p - 1, p, p + 1, 2p - 1, 2^381 - 1,
limbs of all ones, and values whose limbs alternate between 0 and 2^32 - 1."""
import numpy as np
import pytest

from _loader import load
from oracle import oracle as O

mzk = load()
pytestmark = pytest.mark.gpu

P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB


def limbs(v):
    return np.array([(v >> (64 * i)) & ((1 << 64) - 1) for i in range(6)], np.uint64)


def edge_values():
    vals = [0, 1, 2, P - 1, P, P + 1, 2 * P - 2, 2 * P - 1, (1 << 381) - 1, (1 << 380) - 1, (1 << 352) - 1,
            (1 << 64) - 1, 1 << 380]
    alt = sum(((1 << 32) - 1) << (64 * i) for i in range(6))        # words 0, 2, 4 ... all ones
    vals += [alt, alt << 32 & ((1 << 381) - 1), 2 * P - 1 - alt]
    return np.stack([limbs(v) for v in vals if 0 <= v < 2 * P])


@pytest.fixture(scope="module")
def ctx():
    c = mzk.Context(0)
    yield c
    c.close()


def test_square_matches_multiplication(ctx):
    # point coordinates are canonical Montgomery values; adding p gives the
    # lazily reduced representatives in [p, 2p)
    pts = O.gen_bases(91, 1 << 16)
    coords = pts.reshape(-1, 6)
    lazy = np.stack([limbs(int.from_bytes(c.tobytes(), "little") + P) for c in coords[:4096]])
    vals = np.concatenate([edge_values(), coords, lazy])
    buf = ctx.alloc(vals.nbytes)
    buf.upload(vals)
    assert ctx.probe_fp_sqr_check(buf, vals.shape[0]) == 0
    assert ctx.probe_fp_sqr_check(buf, 0) == 0


def test_binary_inverse_matches_fermat(ctx):
    """The binary extended Euclidean inversion (the batch inversion's per-block
    step uses it over Fr) equals the Fermat power over Fp and gives a^-1 a = 1,
    on point coordinates, their lazily reduced representatives and the edge
    values (zeros are skipped)."""
    pts = O.gen_bases(92, 1 << 12)
    coords = pts.reshape(-1, 6)
    lazy = np.stack([limbs(int.from_bytes(c.tobytes(), "little") + P) for c in coords[:512]])
    vals = np.concatenate([edge_values(), coords, lazy])
    buf = ctx.alloc(vals.nbytes)
    buf.upload(vals)
    assert ctx.probe_fp_inv_check(buf, vals.shape[0]) == 0


def test_batch_affine_probe_runs(ctx):
    """The batch-affine microbenchmark reports a rate for every batch size and
    inversion (its figures are recorded with the MSM design)."""
    rates = ctx.probe_batch_affine()
    assert len(rates) == 8 and all(r > 0 for r in rates.values())
