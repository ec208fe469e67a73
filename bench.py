#!/usr/bin/env python3
"""Headline benchmark: BLS12-381 G1 MSM throughput (Mpts/s) at n = 2^24.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full MSM (digit sort, bucket accumulation, bucket reduction,
window combination, normalisation) over n seeded synthetic points: bases
[r_i]G and uniform Fr scalars in Montgomery form, generated on the device.
`value` times K steps with the inputs resident in HBM (2.1 GB of inputs, far
above the 126 MB L2, so no flush is needed); `e2e` times the same MSM through
the reference-facing C ABI call with pinned HOST buffers (host->device copies
inside the timed region).  With N > 1 (torchrun) every rank runs its own MSM
on its own GPU (replicas, weak scaling; the MSM has no exchange step) and the
step time is the max over ranks.

Before anything is timed, the autotuner picks the MSM window widths and NTT
pass splits for the sizes the run uses (`--no-tune` keeps the cost model).
The same JSON line then carries the other configurations: the NTT sweep, the
k = 18 quotient (built-in and as flattened programs), 64 batched MSMs over a
2^22 SRS (plain and over a fixed-base window table), the proof core per k,
serving (plain / batched / served, closed loop and Poisson), and the column
scans and SRS set-up path (`--no-extras`, `--no-prover` skip them).

`--impl reference` times the CPU restatement of the reference's msm_best
(curves/src/msm.rs:460-532; the reference is Rust whose arithmetic lives in the
un-vendored blst crate, so it cannot be built here) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "G1 MSM Mpts/s at 2^24"
UNIT = "Mpts/s"
IMAD_PER_FP_MUL = 600        # CIOS, 12 limbs: 2*12^2+12 = 300 products x (lo, hi)
FP_MUL_PER_MIXED_ADD = 10    # madd-2008-s: 8M + 2S
IMAD_PER_POINT_REF = 97.0e3  # reference schedule c=17, W=16 at 2^24: 1.628e12 IMAD / 2^24


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--log-n", type=int, default=24)
    p.add_argument("--window", type=int, default=0, help="force the MSM window width c (0: autotuned / cost model)")
    p.add_argument("--no-tune", action="store_true", help="skip the autotuner (cost-model window, even NTT split)")
    p.add_argument("--cpu-sample-log-n", type=int, default=20)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the NTT and quotient lines")
    p.add_argument("--ntt-log-n", type=int, default=24)
    p.add_argument("--no-prover", action="store_true", help="skip the proof-core, batched-MSM and serving lines")
    p.add_argument("--create-proof-only", type=int, default=0, metavar="K",
                   help="only time create_proof of the single-proof configuration at 2^K rows (profiling)")
    p.add_argument("--prover-batch", type=int, default=8, help="proofs per call in --create-proof-only")
    p.add_argument("--ntt-only", type=int, default=0, metavar="LOG_N",
                   help="only time coeff_to_lagrange and lagrange_to_coeff at 2^LOG_N (profiling; even "
                        "pass split, W + K transforms each, three passes each at 2^24)")
    p.add_argument("--serve-requests", type=int, default=400)
    p.add_argument("--serve-reps", type=int, default=3)
    return p.parse_args()


def workload(log_n):
    return f"G1 MSM n=2^{log_n}: bases [r_i]G and scalars uniform in Fr (Montgomery), seeded"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_id), "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]), "power": float(parts[3]),
                             "hw_slowdown": parts[5], "hw_thermal": parts[6], "sw_thermal": parts[7],
                             "sw_power_cap": parts[8]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = sorted({name for r in rows for name, key in
                          (("hw_slowdown", "hw_slowdown"), ("hw_thermal_slowdown", "hw_thermal"),
                           ("sw_thermal_slowdown", "sw_thermal"), ("sw_power_cap", "sw_power_cap"))
                          if r[key].lower() == "active"})
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["max"] for r in rows),
                "power_w_max": max(r["power"] for r in rows), "samples": len(rows), "reasons": reasons}


def traffic_from_profiles(c):
    """DRAM bytes per bucket entry of the accumulate kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "msm_accumulate.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_entry:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


IMAD_PER_FR_MUL = 272  # CIOS, 8 limbs: 2*8^2+8 = 136 products x (lo, hi)


def measure_ntt(mzk, ctx, stream, log_n, reps):
    """EvaluationDomain NTTs at n = 2^log_n (extended 2^(log_n+2)), inputs resident."""
    import torch
    n, en = 1 << log_n, 1 << (log_n + 2)
    dom = mzk.EvaluationDomain(ctx, 5, log_n)
    da = ctx.gen_rand_fr(0x7007, n)
    de = ctx.alloc(en * 32)
    ops = [  # name, in, out, transform size, algorithmic bytes
        ("coeff_to_lagrange", da, da, n, 64 * n),
        ("lagrange_to_coeff", da, da, n, 64 * n),
        ("coeff_to_extended", da, de, en, 32 * n + 32 * en),
        ("extended_to_coeff", de, de, en, 64 * en),
    ]
    out = {}
    for name, src, dst, size, nbytes in ops:
        dom.op_device(name, src, dst)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            dom.op_device(name, src, dst)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        lg = size.bit_length() - 1
        imad = (size // 2) * lg * IMAD_PER_FR_MUL
        out[name] = {"n": size, "ms": round(ms, 3), "elements_per_s": round(size / (ms / 1e3), 1),
                     "hbm_gbs_algorithmic": round(nbytes / (ms / 1e3) / 1e9, 1),
                     "imad_t_per_s": round(imad / (ms / 1e3) / 1e12, 3)}
    dom.close()
    return out


QUOTIENT_FR_MUL_PER_ROW = 37   # counted on the oracle's evaluate_numerator restatement (tests/test_plonk_oracle.py)
IMAD_PER_FR_MUL = 272          # CIOS, 8 limbs: 2*8^2+8 = 136 products x (lo, hi)


def measure_quotient(mzk, ctx, stream, k, reps, imad_peak):
    """Fused quotient evaluation for the k-row proof circuit (extended 2^(k+2) rows)."""
    import torch
    E = 1 << (k + 2)
    dom = mzk.EvaluationDomain(ctx, 5, k)
    seed = iter(range(1000, 2000))
    col = lambda: ctx.gen_rand_fr(next(seed), E)
    cols = {
        "advice": [col() for _ in range(3)], "fixed": [col() for _ in range(7)],
        "gate_fixed": [0, 1, 2, 3, 4], "gate_advice": [0, 1, 2],
        "perm_cols": [(0, 0), (0, 1), (0, 2)], "perm_sigma": [col() for _ in range(3)], "perm_z": [col()],
        "chunk_len": 3, "blinding_factors": 7, "l0": col(), "l_last": col(), "l_active": col(),
        "lookup": {"input": 0, "table": 5, "selector": -1, "h": col(), "z": col(), "m": col()},
    }
    import numpy as np
    for name in ("y", "beta", "gamma", "theta"):
        cols[name] = np.array([7, 0, 0, 0], np.uint64)
    desc = mzk.build_quotient_desc(cols, k, k + 2, lambda b: b.ptr)
    out = ctx.alloc(E * 32)
    dom.quotient_eval_device(desc, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        dom.quotient_eval_device(desc, out)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    ncols = 3 + 7 + 3 + 1 + 3 + 3
    # the same circuit (its lookup selector read from a fixed column) with the
    # gate and the lookup given as flattened programs
    # (FlatGraphEvaluator layout: constants [0, 1], slots beta 2, theta 3,
    # trash 4, y 5, previous value 6), run by the program interpreters
    zero, one = np.zeros(4, np.uint64), np.array(FR_ONE_MONT, np.uint64)
    gate = mzk.build_flat_graph(
        [zero, one], [0], [(0, i, 0, 7 + i) for i in range(5)] + [(1, i, 0, 12 + i) for i in range(3)],
        [(2, 15, 7, 12, 0), (2, 16, 8, 13, 0), (0, 17, 15, 16, 0), (2, 18, 12, 13, 0), (2, 19, 18, 9, 0),
         (0, 20, 17, 19, 0), (2, 21, 10, 14, 0), (0, 22, 20, 21, 0), (0, 23, 22, 11, 0), (6, 24, 6, 5, 23)],
        25, 2, 3, 4, 5, 6, 24)
    lookup = mzk.build_flat_graph(
        [zero, one], [0], [(1, 0, 0, 7), (0, 5, 0, 8), (0, 6, 0, 9)],
        [(6, 10, 0, 3, 7), (0, 11, 10, 2, 0), (6, 12, 0, 3, 8), (0, 13, 12, 2, 0)], 14, 2, 3, 4, 5, 6, 13)
    lk = cols["lookup"]
    pcols = dict(cols)
    del pcols["lookup"]
    pcols["fixed"] = cols["fixed"][:6] + [ctx.gen_rand_fr(1999, E)]  # the program reads selector column 6
    pcols["gates"] = gate
    pcols["lookup_programs"] = [{"programs": [lookup], "outputs": [(1, 11, 13, 9)], "helpers": [lk["h"]],
                                 "aggregator": lk["z"], "multiplicities": lk["m"]}]
    pdesc = mzk.build_quotient_desc(pcols, k, k + 2, lambda b: b.ptr)
    dom.quotient_eval_device(pdesc, out)
    e0.record(stream)
    for _ in range(reps):
        dom.quotient_eval_device(pdesc, out)
    e1.record(stream)
    e1.synchronize()
    ms_prog = e0.elapsed_time(e1) / reps
    dom.close()
    imad = QUOTIENT_FR_MUL_PER_ROW * IMAD_PER_FR_MUL * E / (ms / 1e3)
    return {"rows": E, "ms": round(ms, 3), "rows_per_s": round(E / (ms / 1e3), 1),
            "fr_mul_per_row": QUOTIENT_FR_MUL_PER_ROW, "imad_t_per_s": round(imad / 1e12, 3),
            "imad_frac": round(imad / imad_peak, 4),
            "hbm_gbs_algorithmic": round((ncols + 1) * 32 * E / (ms / 1e3) / 1e9, 1),
            "columns_read": ncols,
            "as_programs_ms": round(ms_prog, 3),
            "as_programs": "the gate and the lookup as flattened programs (interpreted per row) instead of "
                           "the built-in fast path"}


# fixed-base window table of the resident SRS for the batched MSMs: width 20,
# used by items of 2^18 points and more.  Prover keys take the width
# prover_table_width(k) of their own SRS instead.
TABLE_C, TABLE_MIN_N = 20, 1 << 18
FR_ONE_MONT = [0x00000001fffffffe, 0x5884b7fa00034802, 0x998c4fefecbc4ff5, 0x1824b159acc5056f]  # R mod r
SERVE_KS = (14, 16, 18, 20)
SERVE_WEIGHTS = (0.4, 0.3, 0.2, 0.1)


class PlonkKeys:
    """Proving keys of the single-proof configuration's circuit (standard gate,
    copy cycles over 10 % of the a and b cells, range lookup of a into a 2^16
    table) for several k.  Each k has its own device SRS (the KZG test setup
    for one seeded secret: g, lagrange, delta and double-delta bases of 2^k
    points, as ParamsKZG downsized to k holds them) stored as row 0 of a
    fixed-base window table of width prover_table_width(k) that every MSM of
    the proof uses.  One seeded Config3Instance per k gives the fixed columns,
    the key (device keygen) and fresh satisfying witnesses per request."""

    def __init__(self, mzk, ctx, ks, table=True):
        self.mzk, self.ctx, self.ks = mzk, ctx, tuple(sorted(ks))
        secret = ctx.gen_rand_fr(0x5EC2E7, 1).download((1, 4))[0]
        self.doms, self.inst, self.srs, self.table = {}, {}, {}, {}
        setup_s = build_s = key_s = 0.0
        for k in self.ks:
            n = 1 << k
            c = mzk.prover_table_width(k) if table else 0
            rows = mzk.Context.msm_table_rows(c) if c else 1
            buf = ctx.alloc(rows * 4 * n * 96)
            p = buf.ptr
            t0 = time.perf_counter()
            dom = mzk.EvaluationDomain(ctx, mzk.CONFIG3_DEGREE, k)
            dom.srs_setup_device(secret, p, p + n * 96, p + 2 * n * 96, p + 3 * n * 96)
            t1 = time.perf_counter()
            if c:
                ctx.msm_window_table(buf, 4 * n, c, rows)
            t2 = time.perf_counter()
            desc = mzk.SrsDesc(p, 4 * n, 0, n, 2 * n, 3 * n, c, rows, n if c else 0)
            self.inst[k] = mzk.Config3Instance(ctx, dom, desc, seed=0xC0F3 + k)
            setup_s, build_s, key_s = setup_s + t1 - t0, build_s + t2 - t1, key_s + time.perf_counter() - t2
            self.doms[k], self.srs[k] = dom, buf
            self.table[str(k)] = {"c": c, "rows": rows, "bytes": rows * 4 * n * 96}
        self.table.update({"build_s": round(build_s, 2), "srs_setup_s": round(setup_s, 2),
                           "min_n": "2^k (every MSM of the proof)"})
        self.keygen_s = round(key_s, 2)

    def request(self, k, seed):
        inst = self.inst[k]
        return inst.key, inst.witness(seed), inst.blinds(seed ^ 0xB11D)

    def close(self):
        self.inst.clear()
        for d in self.doms.values():
            d.close()
        self.srs.clear()


def measure_proofs(mzk, ctx, keys, k, reps, batch):
    """create_proof of the single-proof configuration at 2^k rows, transcript
    on the host: plain (one proof per call, every MSM its own call, kernels
    launched one by one), one proof per call with each phase's MSMs batched,
    and `batch` proofs in one call.  The first proof runs with the self-check
    (L'(x) = -C), so the witnesses are known to satisfy the circuit."""
    reqs = [keys.request(k, 0x9000 + i) for i in range(batch)]
    mzk.create_proofs(ctx, [reqs[0]], flags=mzk.PROVE_SELF_CHECK)
    mzk.create_proofs(ctx, [reqs[0]], flags=mzk.PROVE_PLAIN)          # warm-up (scratch allocation)
    mzk.create_proofs(ctx, [reqs[0]])
    mzk.create_proofs(ctx, reqs)

    def timed(fn, calls):
        t0 = time.perf_counter()
        for i in range(calls):
            fn(i)
        return (time.perf_counter() - t0) / calls * 1e3

    plain_ms = timed(lambda i: mzk.create_proofs(ctx, [reqs[i % batch]], flags=mzk.PROVE_PLAIN), reps)
    one_ms = timed(lambda i: mzk.create_proofs(ctx, [reqs[i % batch]]), reps)
    calls = max(1, reps // batch)
    batch_ms = timed(lambda i: mzk.create_proofs(ctx, reqs), calls)
    key = keys.inst[k].key
    return {"k": k, "rows": 1 << k, "proof_bytes": key.proof_len, "msms_per_proof": 13,
            "plain_ms_per_proof": round(plain_ms, 2), "one_proof_batched_msms_ms": round(one_ms, 2),
            "batch": batch, "batched_ms_per_call": round(batch_ms, 2),
            "batched_proofs_per_s": round(batch * 1e3 / batch_ms, 2), "plain_proofs_per_s": round(1e3 / plain_ms, 2),
            "witness": "satisfying (self-checked); a in the 2^16 table, b uniform, c solved; copy cycles",
            "transcript": "Blake2b Fiat-Shamir, phases in the reference's order"}


def measure_batched_msm(mzk, ctx, reps):
    """64 MSMs, sizes 2^U(12,22) log-uniform, over one shared 2^22-point SRS;
    one in four sparse (90% of scalars in {0, 1}).  One batched call versus
    the same MSMs one call each."""
    import numpy as np
    rng = np.random.default_rng(0xBA7C4)
    sizes = [int(2 ** rng.uniform(12, 22)) for _ in range(64)]
    srs = ctx.gen_bases(0x5125, 1 << 22)
    bufs, items = [], []
    one = np.array(FR_ONE_MONT, np.uint64)
    for i, n in enumerate(sizes):
        b = ctx.gen_rand_fr(0xB000 + i, n)
        if i % 4 == 3:
            s = b.download((n, 4))
            u = rng.random(n)
            s[u < 0.45] = 0
            s[(u >= 0.45) & (u < 0.9)] = one
            b.upload(s)
        bufs.append(b)
        items.append((b, 0, n))
    total = sum(sizes)
    together = ctx.msm_batch_device(srs, 1 << 22, items)
    single = np.stack([ctx.msm_device(b, srs, n) for b, _, n in items])
    t0 = time.perf_counter()
    for _ in range(reps):
        ctx.msm_batch_device(srs, 1 << 22, items)
    t_batch = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        for b, _, n in items:
            ctx.msm_device(b, srs, n)
    t_seq = (time.perf_counter() - t0) / reps
    # the same batch over a fixed-base window table of the SRS (built once,
    # untimed, like the SRS itself): items of 2^18 points and more use it
    c, min_n = TABLE_C, TABLE_MIN_N
    rows = mzk.Context.msm_table_rows(c)
    del srs
    table = ctx.alloc(rows * (1 << 22) * 96)
    ctx.gen_bases(0x5125, 1 << 22, out=table)
    t0 = time.perf_counter()
    ctx.msm_window_table(table, 1 << 22, c, rows)
    t_build = time.perf_counter() - t0
    tabled = ctx.msm_batch_table_device(table, 1 << 22, c, rows, min_n, items)
    t0 = time.perf_counter()
    for _ in range(reps):
        ctx.msm_batch_table_device(table, 1 << 22, c, rows, min_n, items)
    t_table = (time.perf_counter() - t0) / reps
    del table
    return {"msms": 64, "points": total, "sparse_msms": 16, "batched_ms": round(t_batch * 1e3, 2),
            "batched_mpts_per_s": round(total / t_batch / 1e6, 2), "one_call_each_ms": round(t_seq * 1e3, 2),
            "one_call_each_mpts_per_s": round(total / t_seq / 1e6, 2),
            "batched_equals_one_call_each": bool(np.array_equal(together, single)),
            "window_table": {"c": c, "rows": rows, "min_n": min_n, "bytes": rows * (1 << 22) * 96,
                             "build_s": round(t_build, 2), "batched_ms": round(t_table * 1e3, 2),
                             "batched_mpts_per_s": round(total / t_table / 1e6, 2),
                             "equals_batched": bool(np.array_equal(tabled, together))}}


def measure_serving(mzk, ctx, keys, n_requests, reps, max_batch, lanes, mem_budget, max_wave_rows):
    """A stream of create_proof requests, k drawn from SERVE_KS with
    SERVE_WEIGHTS, a fresh seeded witness per request.  Closed loop (all
    requests queued at once): every mode `reps` times, median and spread of
    proofs/s.  Then open-loop Poisson arrivals at 0.8x and 1.5x the plain
    prover's closed-loop rate, twice each.  Latency = submit to transcript on
    the host.  One server per mode serves all of that mode's runs, after a
    warm-up (untimed) that gives every lane full waves of every k, so the
    lanes' scratch arenas have reached their working size and the NTT graphs
    of every proof slot are captured before anything is timed."""
    import threading

    import numpy as np
    rng = np.random.default_rng(0x5E7E)
    ks = [int(k) for k in rng.choice(SERVE_KS, size=n_requests, p=SERVE_WEIGHTS)]
    reqs = [keys.request(k, 0x20000 + i) for i, k in enumerate(ks)]

    def warm_up(srv, a):
        nl, mb, rows = a.get("lanes", 1), a.get("max_batch", 1), a.get("max_wave_rows", 0)
        for _ in range(2):
            for k in SERVE_KS:
                wave = min(mb, max(1, rows >> k)) if rows else mb
                r = reqs[ks.index(k)]
                for t in [srv.submit(*r) for _ in range(nl * wave)]:
                    srv.wait(t)

    def run(srv, arrivals):
        waves0 = srv.stats()["waves"]
        lat = [None] * len(reqs)
        tickets = [None] * len(reqs)
        ready = threading.Semaphore(0)

        def collector():
            for i in range(len(reqs)):
                ready.acquire()
                lat[i] = srv.wait(tickets[i])[1]

        th = threading.Thread(target=collector)
        th.start()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            if arrivals is not None:
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            tickets[i] = srv.submit(*r)
            ready.release()
        th.join()
        wall = time.perf_counter() - t0
        lat = np.array(lat)
        return {"proofs_per_s": round(len(reqs) / wall, 2), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2), "waves": srv.stats()["waves"] - waves0,
                "wall_s": round(wall, 2)}

    modes = {
        "plain": {"max_batch": 1, "lanes": 1, "per_call": True},           # one proof, one MSM per call
        "one_proof_batched_msms": {"max_batch": 1, "lanes": 1},            # one proof, its MSMs batched
        "served": {"max_batch": max_batch, "lanes": lanes, "mem_budget_bytes": mem_budget,
                   "max_wave_rows": max_wave_rows},
    }
    out = {"requests": n_requests, "k_mix": dict(zip(map(str, SERVE_KS), SERVE_WEIGHTS)), "modes": modes,
           "repetitions": reps}
    servers = {}
    for name, a in modes.items():
        servers[name] = mzk.ProvingServer(ctx, **a)
        warm_up(servers[name], a)
    closed = {}
    for name in modes:
        runs = [run(servers[name], None) for _ in range(reps)]
        rates = sorted(r["proofs_per_s"] for r in runs)
        closed[name] = {"proofs_per_s_median": rates[len(rates) // 2], "proofs_per_s_min": rates[0],
                        "proofs_per_s_max": rates[-1],
                        "p50_ms_median": sorted(r["p50_ms"] for r in runs)[len(runs) // 2],
                        "p99_ms_median": sorted(r["p99_ms"] for r in runs)[len(runs) // 2],
                        "wall_s": [r["wall_s"] for r in runs], "waves": [r["waves"] for r in runs]}
    out["closed_loop"] = closed
    rate = closed["plain"]["proofs_per_s_median"]
    out["served_over_plain_closed_loop"] = round(closed["served"]["proofs_per_s_median"] / rate, 3)
    for f in (0.8, 1.5):
        res = {"rate_per_s": round(f * rate, 2)}
        for rep in range(2):
            arr = np.cumsum(rng.exponential(1.0 / (f * rate), size=n_requests))
            for name in ("plain", "served"):
                res.setdefault(name, []).append(run(servers[name], arr))
        for name in ("plain", "served"):
            res[name + "_p99_ms_max"] = max(r["p99_ms"] for r in res[name])
        out[f"poisson_{f}x_plain"] = res
    for srv in servers.values():
        srv.close()
    return out


P_FP = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R_INV_FP = pow(1 << 384, -1, P_FP)


def compress_g1(p):
    """ZCash compressed encoding of an affine point (12 x u64 Montgomery),
    as G1Affine::to_compressed writes it (input preparation for the bench)."""
    if not any(int(v) for v in p):
        return bytes([0xC0]) + bytes(47)
    x = sum(int(v) << (64 * i) for i, v in enumerate(p[:6])) * R_INV_FP % P_FP
    y = sum(int(v) << (64 * i) for i, v in enumerate(p[6:])) * R_INV_FP % P_FP
    b = bytearray(x.to_bytes(48, "big"))
    b[0] |= 0x80 | (0x20 if y > P_FP - y else 0)
    return bytes(b)


def measure_setup_and_scans(mzk, ctx, stream):
    """The prover's column scans and the KZG setup path at production sizes,
    device time (CUDA events on the library's stream); inputs resident."""
    import numpy as np
    import torch

    def timed(fn, reps=3):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {}
    n24 = 1 << 24
    a = ctx.gen_rand_fr(0xA1, n24)
    x = np.array([12345, 0, 0, 0], np.uint64)
    ms = timed(lambda: ctx.batch_invert_device(a, n24))
    out["batch_invert_2^24"] = {"ms": round(ms, 3), "elements_per_s": round(n24 / ms * 1e3, 1)}
    ms = timed(lambda: ctx.eval_polynomial_device(a, n24, x))
    out["eval_polynomial_2^24"] = {"ms": round(ms, 3), "elements_per_s": round(n24 / ms * 1e3, 1)}
    q = ctx.alloc(n24 * 32)
    ms = timed(lambda: ctx.kate_division_device(a, n24, x, q))
    out["kate_division_2^24"] = {"ms": round(ms, 3), "elements_per_s": round(n24 / ms * 1e3, 1)}
    del q
    k = 20
    n = 1 << k
    dom = mzk.EvaluationDomain(ctx, 5, k)
    cols = [ctx.gen_rand_fr(0xB0 + i, n) for i in range(9)]
    z = ctx.alloc(n * 32)
    beta, gamma = np.array([7, 0, 0, 0], np.uint64), np.array([11, 0, 0, 0], np.uint64)
    blinds = np.zeros((1, 7, 4), np.uint64)
    ms = timed(lambda: dom.permutation_z_device(cols[:3], cols[3:6], 3, 7, blinds, beta, gamma, [z]))
    out["permutation_z_k20_3cols"] = {"ms": round(ms, 3), "rows_per_s": round(n / ms * 1e3, 1)}
    h, agg = ctx.alloc(n * 32), ctx.alloc(n * 32)
    ms = timed(lambda: dom.logup_device([[cols[0]]], cols[6], cols[7], cols[8], 7, blinds[0], beta, [h], agg))
    out["logup_k20_1input"] = {"ms": round(ms, 3), "rows_per_s": round(n / ms * 1e3, 1)}
    bufs = [ctx.alloc(n * 96) for _ in range(4)]
    s = np.array([0x1234567, 0x89, 0, 0], np.uint64)
    ms = timed(lambda: dom.srs_setup_device(s, *bufs), reps=1)
    out["srs_setup_k20"] = {"ms": round(ms, 2), "points_per_s": round(4 * n / ms * 1e3, 1),
                            "note": "g, g_lagrange, delta, double delta (4 x 2^20 points)"}
    small = mzk.EvaluationDomain(ctx, 5, 16)
    ms = timed(lambda: small.g1_to_lagrange_device(bufs[0], bufs[1]), reps=1)
    out["g_to_lagrange_k16"] = {"ms": round(ms, 2), "points_per_s": round((1 << 16) / ms * 1e3, 1),
                                "note": "inverse FFT over G1, one GLV scalar multiplication per butterfly"}
    # compressed points: 2^12 of the setup's g, compressed on the host, repeated
    m = 1 << 12
    pts = bufs[0].download((m, 12))
    comp = np.frombuffer(b"".join(compress_g1(p) for p in pts) * (n // m), np.uint8)
    d_comp = ctx.alloc(comp.nbytes)
    d_comp.upload(comp)
    ms = timed(lambda: ctx.g1_decompress_device(d_comp, n, bufs[2]), reps=1)
    out["g1_decompress_2^20"] = {"ms": round(ms, 2), "points_per_s": round(n / ms * 1e3, 1),
                                 "note": "square root, sign and the G1 membership test phi(P) = -[u^2]P per point"}
    small.close()
    dom.close()
    return out


def dist_init(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks_of(x, world, device):
    """The maximum of x over the ranks of the job (the step time of a replica
    run is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_gather_u64(arr, device):
    """torch.distributed all-gather of a small uint64 array (as int64), the
    exchange step of the point-split MSM; the list of every rank's array."""
    import numpy as np
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(arr, np.uint64).view(np.int64)).to(device)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [o.cpu().numpy().view(np.uint64) for o in out]


def run_reference(args):
    world, rank, _ = dist_init("gloo")
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    n = 1 << args.cpu_sample_log_n
    s = O.rand_fr(0xC0FFEE, n, threads=threads)
    b = O.gen_bases(0xBA5E, n, threads=threads)
    for _ in range(args.warmup):
        O.msm_best(s, b, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.msm_best(s, b, threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = n / (ms / 1e3) / 1e6
    sample = (f"n=2^{args.cpu_sample_log_n} points of the 2^{args.log_n} workload per step (bounded sample); "
              f"C restatement of msm_best, windows in parallel on {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 limbs (CPU)", "data": "synthetic (seeded)",
        "config": {"workload": workload(args.log_n), "n": 1 << args.log_n, "parallelism": "cpu threads"},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_create_proof_only(args):
    """create_proof of config 3 at 2^K rows, one proof per call and batches of
    --prover-batch (a short run for profilers); prints one JSON line."""
    from _loader import load
    mzk = load()
    ctx = mzk.Context(0)
    if not args.no_tune:
        ds = ctx.gen_rand_fr(0xC0FFEE, 1 << args.create_proof_only)
        db = ctx.gen_bases(0xBA5E, 1 << args.create_proof_only)
        ctx.autotune(ds, db, msm_log_n=list(range(12, args.create_proof_only + 1)),
                     ntt_log_n=list(range(12, args.create_proof_only + 3)), reps=2)
        del ds, db
    keys = PlonkKeys(mzk, ctx, (args.create_proof_only,))
    r = measure_proofs(mzk, ctx, keys, args.create_proof_only, max(2, args.steps), args.prover_batch)
    ph, calls = ctx.prove_phase_stats()
    r["phase_ms_total"] = {k: round(v, 2) for k, v in ph.items()}
    r["calls"] = calls
    print(json.dumps({"create_proof": r}), flush=True)
    keys.close()
    ctx.close()


def run_ntt_only(args):
    """The domain's two size-n transforms at 2^LOG_N, in place on seeded
    inputs (a short run for profilers); prints one JSON line."""
    import torch
    from _loader import load
    mzk = load()
    ctx = mzk.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    n = 1 << args.ntt_only
    dom = mzk.EvaluationDomain(ctx, 2, args.ntt_only)   # j = 2: the extended domain is n, no 4n tables
    da = ctx.gen_rand_fr(0x7007, n)
    out = {}
    for name in ("coeff_to_lagrange", "lagrange_to_coeff"):
        for _ in range(args.warmup):
            dom.op_device(name, da, da)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            dom.op_device(name, da, da)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        imad = (n // 2) * args.ntt_only * IMAD_PER_FR_MUL
        out[name] = {"n": n, "ms": round(ms, 3), "imad_t_per_s": round(imad / (ms / 1e3) / 1e12, 3)}
    print(json.dumps({"ntt": out}), flush=True)
    dom.close()
    ctx.close()


def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_init("nccl")
    torch.cuda.set_device(local)
    from _loader import load
    mzk = load()
    ctx = mzk.Context(local)
    n = 1 << args.log_n
    if args.window:
        ctx.set_msm_window(args.window)
    ds = ctx.gen_rand_fr(0xC0FFEE + rank, n)
    db = ctx.gen_bases(0xBA5E + rank, n)
    imad_peak, fp_mul_rate, imad_variants = ctx.probe_imad_peak()
    # the 12-limb Montgomery multiplication in a tight register loop (every operand
    # per-thread) is the fastest form of this work measured on the part: its rate
    # x 600 half-products is the denominator unless a plain IMAD probe beats it
    madd_rate = imad_variants.pop("madd_regs")
    # batch-affine additions (one shared inversion per batch) against the
    # mixed XYZZ addition, both without memory traffic (the MSM design record)
    batch_affine = {f"b{b}_{inv}": round(v / 1e9, 3) for (b, inv), v in ctx.probe_batch_affine().items()}
    imad_peak = max(imad_peak, max(imad_variants.values()), fp_mul_rate * IMAD_PER_FP_MUL)
    # the autotuner, before anything is timed: MSM window widths for every
    # log2 size the bench runs (the headline and the prover's MSMs) on the
    # headline inputs, NTT pass splits for 2^12 .. 2^26
    tune = None
    if not args.window and not args.no_tune:
        t0 = time.perf_counter()
        res = ctx.autotune(ds, db, msm_log_n=list(range(12, args.log_n + 1)), ntt_log_n=list(range(12, 27)), reps=2)
        tune = {"msm_c": {str(L): v[0] for L, v in res["msm"].items()},
                "ntt_split": {str(L): v[0] for L, v in res["ntt"].items()},
                "ntt_split_modes": "1 even, 2 largest passes first, 3 largest passes last",
                "seconds": round(time.perf_counter() - t0, 2)}
    stream = torch.cuda.ExternalStream(ctx.stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        return max_over_ranks_of(x, world, "cuda")

    for _ in range(args.warmup):
        ctx.msm_device(ds, db, n)
    ctx.synchronize()
    barrier()
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    launches0 = ctx.launches
    gpu_id = local
    try:
        uuid = torch.cuda.get_device_properties(local).uuid
        gpu_id = f"GPU-{uuid}"
    except Exception:
        pass
    sampler = ClockSampler(gpu_id)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.msm_device(ds, db, n)
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop()
    ctx.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    phases = ctx.phase_stats()
    ctx.set_profiling(False)
    c, windows, entries = ctx.msm_last_shape()
    value = world * n / (ms / 1e3) / 1e6

    acc_ms, acc_cnt = phases["accumulate"]
    acc_avg_ms = acc_ms / max(acc_cnt, 1)
    imad_acc = entries * FP_MUL_PER_MIXED_ADD * IMAD_PER_FP_MUL
    achieved = imad_acc / (acc_avg_ms / 1e3)
    tpe = traffic_from_profiles(c)
    roofline = {
        "kernel": "k_accumulate (bucket accumulation)", "bound": "imad",
        "achieved": round(achieved / 1e12, 3), "peak": round(imad_peak / 1e12, 3), "unit": "TIMAD/s",
        "frac": round(achieved / imad_peak, 4),
        "traffic": None if tpe is None else round(tpe * entries),
        "peak_source": "measured in this run: max of mzk_probe_imad_peak's IMAD microbenchmarks and "
                       "600 x the measured 12-limb Montgomery multiplication rate (per-thread operands)",
        "work": f"{entries} bucket entries x {FP_MUL_PER_MIXED_ADD} Fp mul x {IMAD_PER_FP_MUL} IMAD",
        "launch_ms": round(acc_avg_ms, 3),
    }
    msm_roof = {
        "achieved": round(IMAD_PER_POINT_REF * n / (ms / 1e3) / 1e12, 3), "unit": "TIMAD/s",
        "frac": round(IMAD_PER_POINT_REF * n / (ms / 1e3) / imad_peak, 4),
        "work": "97.0k IMAD per point (reference schedule c=17, 16 windows)",
    }

    # strong scaling (N > 1): one 2^log_n MSM split across the ranks by
    # points, the partials all-gathered over NCCL and added on the host
    point_split = None
    if world > 1:
        def msm_slice(b, e):
            return ctx.msm_device(mzk.DevicePtr(ds, b * 32), mzk.DevicePtr(db, b * 96), e - b)

        def split_once():
            return mzk.msm_point_split(msm_slice, n, rank, world, lambda a: all_gather_u64(a, "cuda"))

        for _ in range(2):
            split_once()
        times = []
        for _ in range(max(3, args.steps // 4)):
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            split_once()
            torch.cuda.synchronize()
            times.append(max_over_ranks((time.perf_counter() - t0) * 1e3))
        sms = statistics.median(times)
        point_split = {"n": n, "ranks": world, "ms": round(sms, 3), "mpts_per_s": round(n / (sms / 1e3) / 1e6, 2),
                       "scaling": "strong", "exchange": "one all-gather of 144-byte partials (NCCL), host add",
                       "timing": "wall clock per split MSM, max over ranks, median of runs"}

    e2e = None
    if not args.no_e2e:
        hs = torch.empty(n * 4, dtype=torch.int64, pin_memory=True)
        hb = torch.empty(n * 12, dtype=torch.int64, pin_memory=True)
        lib = mzk.lib()
        mzk._check(lib.mzk_memcpy_d2h(ctx.h, hs.data_ptr(), ds.ptr, n * 32))
        mzk._check(lib.mzk_memcpy_d2h(ctx.h, hb.data_ptr(), db.ptr, n * 96))
        s_host = hs.numpy().view(np.uint64).reshape(n, 4)
        b_host = hb.numpy().view(np.uint64).reshape(n, 12)
        for _ in range(2):
            ctx.msm_best(s_host, b_host)
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            ctx.msm_best(s_host, b_host)
        f1.record(stream)
        f1.synchronize()
        ems = max_over_ranks(f0.elapsed_time(f1) / args.steps)
        e2e = {"value": round(world * n / (ems / 1e3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(ems, 3),
               "h2d_bytes_per_step": n * 32 + n * 96, "d2h_bytes_per_step": windows * 192 + 4 * (3 if n >= 1 << 20 else 1),
               "api": "mzk_msm_g1 (host pointers, pinned)"}

    extra_ntt = extra_q = None
    extra_prover = {}
    if not args.no_extras:
        del ds, db
        extra_ntt = measure_ntt(mzk, ctx, stream, args.ntt_log_n, 5)
        extra_q = measure_quotient(mzk, ctx, stream, 18, 5, imad_peak)
        if not args.no_prover:
            extra_prover["batched_msm"] = measure_batched_msm(mzk, ctx, 3)
            keys = PlonkKeys(mzk, ctx, SERVE_KS)
            extra_prover["create_proof_k18"] = measure_proofs(mzk, ctx, keys, 18, 8, 8)
            extra_prover["create_proof_by_k"] = {str(k): measure_proofs(mzk, ctx, keys, k, reps, b)
                                                 for k, reps, b in ((14, 32, 16), (16, 32, 16), (20, 4, 2))}
            # served: 3 lanes, waves of at most 16 proofs and 2^21 rows (a lane
            # sweep on the B200 put 3 lanes and the row cap ahead of 2 lanes
            # and uncapped waves, in throughput and in p99)
            extra_prover["serving"] = measure_serving(mzk, ctx, keys, args.serve_requests, args.serve_reps, 16, 4,
                                                      48 << 30, 1 << 21)
            extra_prover["prover_srs_window_table"] = keys.table
            extra_prover["prover_keygen_s"] = keys.keygen_s
            keys.close()
            del keys
            extra_prover["setup_and_scans"] = measure_setup_and_scans(mzk, ctx, stream)
        ds = ctx.gen_rand_fr(0xC0FFEE + rank, n)
        db = ctx.gen_bases(0xBA5E + rank, n)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        m = 1 << args.cpu_sample_log_n
        s_cpu = ds.download((m, 4))
        b_cpu = db.download((m, 12))
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.msm_best(s_cpu, b_cpu, threads)
        dt = time.perf_counter() - t0
        cpu = {"value": round(m / dt / 1e6, 4), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"first 2^{args.cpu_sample_log_n} points of the timed inputs, one msm_best call "
                         f"(C restatement of curves/src/msm.rs:460-532), windows in parallel"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 (12-limb Fp / 8-limb Fr Montgomery)",
            "data": "synthetic (seeded, generated on device)",
            "config": {"workload": workload(args.log_n), "n": n, "window_c": c, "windows": windows,
                       "bucket_entries": entries, "l2": "inputs 2.1 GB > 126 MB L2 (no flush)",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "roofline_msm": msm_roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clocks, "autotune": tune,
            "phases_ms": {k: round(v[0] / max(v[1], 1), 3) for k, v in phases.items()},
            "fp_mul_rate_g_per_s": round(fp_mul_rate / 1e9, 2),
            "imad_probe_t_per_s": {k: round(v / 1e12, 3) for k, v in imad_variants.items()},
            "madd_in_registers_g_per_s": round(madd_rate / 1e9, 3),
            "batch_affine_adds_g_per_s": batch_affine,
            "ntt": extra_ntt, "quotient_k18": extra_q, "point_split_msm": point_split, **extra_prover,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.create_proof_only:
        run_create_proof_only(args)
    elif args.ntt_only:
        run_ntt_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
