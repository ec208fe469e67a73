"""Host side of the benchmark's synthetic config-3 instances (no GPU): the
copy cycles form a permutation of the cells whose cycles have 2 to 4 cells
among the a and b cells of the usable rows, and the cycle ids agree with it."""
import numpy as np

from _loader import load

mzk = load()


def test_copy_cycles_form_a_permutation():
    n, u = 1 << 10, (1 << 10) - 8
    mapping, cycle_of = mzk.copy_cycles(n, u, seed=5)
    flat = mapping[:, :, 0].astype(np.int64) * n + mapping[:, :, 1]
    assert sorted(flat.ravel().tolist()) == list(range(3 * n))          # a bijection on the cells
    moved = np.argwhere(flat.reshape(3, n) != np.arange(3 * n).reshape(3, n))
    assert len(moved) >= int(0.1 * 2 * u) - 4
    assert set(moved[:, 0].tolist()) <= {0, 1} and moved[:, 1].max() < u   # a and b cells of usable rows
    # follow every cycle: length 2..4, one cycle id for all its cells
    seen = set()
    for c, r in moved:
        if (c, r) in seen:
            continue
        cyc, cur = [], (int(c), int(r))
        while cur not in cyc:
            cyc.append(cur)
            cur = tuple(int(v) for v in mapping[cur[0], cur[1]])
        assert cur == cyc[0] and 2 <= len(cyc) <= 4
        ids = {int(cycle_of[cc * n + rr]) for cc, rr in cyc}
        assert len(ids) == 1 and 0xFFFFFFFF not in ids
        seen.update(cyc)
    assert np.count_nonzero(cycle_of != 0xFFFFFFFF) == len(seen)


def test_config3_circuit_shape():
    c = mzk.config3_circuit(18)
    assert c["degree"] == 5 and c["blinding_factors"] == 7 and c["n_advice"] == 3 and c["n_fixed"] == 7


def test_prover_table_width_grows_with_k():
    widths = [mzk.prover_table_width(k) for k in range(4, 27)]
    assert widths == sorted(widths) and all(5 <= c <= 24 for c in widths)
    assert all(mzk.Context.msm_table_rows(c) * c >= 256 for c in set(widths))
