"""The multi-process paths on the CPU (gloo, world size 2): the slowest
rank's time is the step time of a replica run; the reference arm under
torchrun prints exactly one line (rank 0) while the other rank exits
cleanly; the point-split MSM (one all-gather of 144-byte partials, then the
host add) equals the MSM over all points on every rank."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    w, r, _ = bench.dist_init("gloo")
    got = bench.max_over_ranks_of(10.0 + 5 * r, w, "cpu")
    import torch.distributed as dist
    dist.destroy_process_group()
    q.put((r, got))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_reference_arm_under_torchrun_two_ranks():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-sample-log-n", "8"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def _split_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    from _loader import load
    from oracle import oracle as O
    mzk = load()
    w, r, _ = bench.dist_init("gloo")
    n = 1000
    s, b = O.rand_fr(31, n), O.gen_bases(32, n)
    s[5] = 0                                   # a zero scalar and an identity base in the mix
    b[700] = 0

    def msm_slice(begin, end):                 # this rank's MSM (the oracle standing in for the device)
        out = np.zeros(18, np.uint64)
        aff = O.msm_best(s[begin:end], b[begin:end])
        if np.any(aff):
            out[:12] = aff
            out[12:] = O.fp_const(0)
        return out

    got = mzk.msm_point_split(msm_slice, n, r, w, lambda a: bench.all_gather_u64(a, "cpu"))
    import torch.distributed as dist
    dist.destroy_process_group()
    q.put((r, got[:12].tolist(), O.msm_best(s, b).tolist()))


def test_point_split_msm_gloo():
    """The point-split MSM (each rank a slice of the points, one all-gather of
    the 144-byte partials, the host add) on two gloo ranks equals the MSM over
    all points, on every rank."""
    import numpy as np  # noqa: F401  (the ranks import it)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_split_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = [q.get(timeout=10) for _ in range(2)]
    for r, got, want in res:
        assert got == want, r


def test_g1_sum_host_edge_cases():
    from _loader import load
    from oracle import oracle as O
    mzk = load()
    import numpy as np
    pts = O.gen_bases(40, 3)
    p18 = np.zeros((4, 18), np.uint64)
    for i in range(3):
        p18[i, :12] = pts[i]
        p18[i, 12:] = O.fp_const(0)
    want = O.g1_to_affine(O.g1_jac_add(O.g1_jac_add(O.g1_from_affine(pts[0]), O.g1_from_affine(pts[1])),
                                       O.g1_from_affine(pts[2])))
    assert np.array_equal(mzk.g1_sum(p18)[:12], want)          # the all-zero fourth point is the identity
    neg = p18[0].copy()
    neg[6:12] = O.fp_op("sub", np.zeros(6, np.uint64), p18[0, 6:12])
    assert not mzk.g1_sum(np.stack([p18[0], neg])).any()        # P + (-P)
    dbl = O.g1_to_affine(O.g1_jac_double(O.g1_from_affine(pts[0])))
    assert np.array_equal(mzk.g1_sum(np.stack([p18[0], p18[0]]))[:12], dbl)
    assert not mzk.g1_sum(np.zeros((0, 18), np.uint64)).any()
    bad = p18[0].copy()
    bad[12] += 1                                                # z not normalised
    import pytest
    with pytest.raises(mzk.MzkError):
        mzk.g1_sum(bad)
