"""Host-side helpers of bench.py on the CPU: the ZCash compression used to
prepare the decompression workload agrees with the oracle's encoder, and the
replica step time is the slowest rank's."""
import importlib.util
from pathlib import Path

import numpy as np

from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent


def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def test_compress_g1_matches_oracle():
    b = bench()
    pts = O.gen_bases(17, 24)
    pts[5] = 0
    for p in pts:
        assert b.compress_g1(p) == bytes(O.g1_compress(p))


def test_single_rank_max_is_identity():
    assert bench().max_over_ranks_of(3.5, 1, "cpu") == 3.5
