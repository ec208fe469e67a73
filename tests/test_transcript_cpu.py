"""The library's Fiat-Shamir transcript and VK hash (host code, no GPU)
against the oracle's restatement over CPython's BLAKE2b: the same absorbs,
writes and squeezes give the same challenges and proof bytes, across the
128-byte block boundaries of the hash, identity points included."""
import numpy as np

from _loader import load
from oracle import oracle as O
from oracle import plonk as OP

mzk = load()


def point18(aff):
    """affine (12 u64 Montgomery, identity all-zero) -> the 18-u64 layout"""
    out = np.zeros(18, np.uint64)
    if np.any(aff):
        out[:12] = aff
        out[12:] = O.fp_const(0)
    return out


def test_transcript_matches_oracle():
    rng = np.random.default_rng(3)
    pts = O.gen_bases(11, 24)
    scal = O.rand_fr(12, 64)
    lib_t, ora_t = mzk.Transcript(), OP.Transcript()
    lib_t.common_fr(scal[0])
    ora_t.common_fr(OP.to_int(scal[0]))
    for step in range(160):
        op = rng.integers(0, 4)
        if op == 0:
            v = scal[rng.integers(0, 64)]
            lib_t.write_fr(v)
            ora_t.write_fr(OP.to_int(v))
        elif op == 1:
            p = pts[rng.integers(0, 24)] if rng.random() < 0.9 else np.zeros(12, np.uint64)
            lib_t.write_point(point18(p))
            ora_t.write_point(p)
        elif op == 2:
            v = scal[rng.integers(0, 64)]
            lib_t.common_fr(v)
            ora_t.common_fr(OP.to_int(v))
        else:
            assert OP.to_int(lib_t.squeeze_challenge()) == ora_t.squeeze(), step
    assert lib_t.finalize() == bytes(ora_t.proof)
    assert OP.to_int(lib_t.squeeze_challenge()) == ora_t.squeeze()


def test_squeeze_twice_differs_and_is_canonical():
    t = mzk.Transcript()
    a, b = t.squeeze_challenge(), t.squeeze_challenge()
    assert not np.array_equal(a, b)
    for v in (a, b):
        assert OP.to_int(v) < OP.R


def test_vk_transcript_repr_matches_oracle():
    fixed = O.gen_bases(21, 7)
    perm = O.gen_bases(22, 3)
    fixed[2] = 0                      # an identity commitment (the 0x40 encoding)
    pinned = b"PinnedEvaluationDomain { k: 5, extended_k: 7, omega: 0x.. } " * 9  # several hash blocks
    got = mzk.vk_transcript_repr(5, np.stack([point18(p) for p in fixed]), np.stack([point18(p) for p in perm]),
                                 pinned)
    assert OP.to_int(got) == OP.vk_transcript_repr(5, list(fixed), list(perm), pinned)
    empty = mzk.vk_transcript_repr(3, np.zeros((0, 18), np.uint64), np.zeros((0, 18), np.uint64), b"")
    assert OP.to_int(empty) == OP.vk_transcript_repr(3, [], [], b"")


def test_compressed_point_encoding_matches_oracle():
    pts = O.gen_bases(31, 40)
    t, o = mzk.Transcript(), OP.Transcript()
    for p in pts:
        t.write_point(point18(p))
        o.write_point(p)
        neg = p.copy()
        neg[6:] = O.fp_op("sub", np.zeros(6, np.uint64), p[6:])   # -P: the other sign flag
        t.write_point(point18(neg))
        o.write_point(neg)
    assert t.finalize() == bytes(o.proof)
