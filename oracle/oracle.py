"""ctypes wrapper over the C oracle (oracle/libmzk_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import
this module.

Arrays are numpy uint64 arrays in the reference's in-memory layouts:
Fr elements shape (n, 4) Montgomery, G1 affine points shape (n, 12)
(x limbs 0..5, y limbs 6..11, Montgomery, identity all-zero).
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmzk_oracle.so"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _load():
    if not LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    sz = ctypes.c_size_t
    i32 = ctypes.c_int
    u32 = ctypes.c_uint32
    u64 = ctypes.c_uint64
    sigs = {
        "or_fr_mul": (None, [_u64p, _u64p, _u64p]),
        "or_fr_batch_invert": (None, [_u64p, sz]),
        "or_permutation_z": (None, [ctypes.c_void_p, ctypes.c_void_p, u32, u32, u32, _u64p, _u64p, _u64p, u32,
                                    _u64p, ctypes.c_void_p]),
        "or_logup": (None, [ctypes.c_void_p, ctypes.POINTER(u32), u32, _u64p, _u64p, _u64p, sz, _u64p, u32, _u64p,
                            ctypes.c_void_p, _u64p]),
        "or_kate_division": (None, [_u64p, sz, _u64p, _u64p]),
        "or_fr_mul_vec": (None, [_u64p, _u64p, _u64p, sz]),
        "or_fr_mul_counter": (ctypes.c_ulonglong, [i32]),
        "or_g1_suffix_sum": (None, [_u64p, sz, _u64p]),
        "or_g1_decompress": (i32, [_u64p, _u8p, i32]),
        "or_srs_setup": (None, [_u64p, u32, _u64p, _u64p, _u64p, _u64p, _u64p]),
        "or_poly_inner_product": (None, [ctypes.c_void_p, ctypes.POINTER(sz), sz, _u64p, _u64p, sz]),
        "or_fr_add": (None, [_u64p, _u64p, _u64p]),
        "or_fr_sub": (None, [_u64p, _u64p, _u64p]),
        "or_fr_neg": (None, [_u64p, _u64p]),
        "or_fr_inv": (None, [_u64p, _u64p]),
        "or_fr_from_canonical": (None, [_u64p, _u64p]),
        "or_fr_to_canonical": (None, [_u64p, _u64p]),
        "or_fr_const": (None, [i32, _u64p]),
        "or_fp_mul": (None, [_u64p, _u64p, _u64p]),
        "or_fp_add": (None, [_u64p, _u64p, _u64p]),
        "or_fp_sub": (None, [_u64p, _u64p, _u64p]),
        "or_fp_inv": (None, [_u64p, _u64p]),
        "or_fp_from_canonical": (None, [_u64p, _u64p]),
        "or_fp_to_canonical": (None, [_u64p, _u64p]),
        "or_fp_const": (None, [i32, _u64p]),
        "or_g1_generator": (None, [_u64p]),
        "or_g1_add": (None, [_u64p, _u64p, _u64p]),
        "or_g1_double": (None, [_u64p, _u64p]),
        "or_g1_to_affine": (None, [_u64p, _u64p]),
        "or_g1_from_affine": (None, [_u64p, _u64p]),
        "or_g1_is_on_curve_affine": (i32, [_u64p]),
        "or_g1_mul": (None, [_u64p, _u64p, _u64p]),
        "or_g1_compress": (None, [_u8p, _u64p]),
        "or_msm_naive": (None, [_u64p, _u64p, _u64p, sz]),
        "or_msm_best": (None, [_u64p, _u64p, _u64p, sz, i32]),
        "or_msm_specific": (None, [_u64p, _u64p, _u64p, sz, i32]),
        "or_booth_index": (i32, [sz, sz, _u8p]),
        "or_fr_inner_product": (None, [_u64p, _u64p, _u64p, sz, i32]),
        "or_rand64": (u64, [u64, u64]),
        "or_rand_fr": (None, [_u64p, u64, u64, sz, i32]),
        "or_gen_bases": (None, [_u64p, u64, u64, sz, i32]),
        "or_compute_twiddles": (None, [_u64p, _u64p, u32]),
        "or_best_fft": (None, [_u64p, _u64p, u32, i32]),
        "or_fft_dif_pruned": (None, [_u64p, _u64p, u32, sz, i32]),
        "or_dft_naive": (None, [_u64p, _u64p, _u64p, sz]),
        "or_eval_polynomial": (None, [_u64p, _u64p, sz, _u64p, i32]),
        "or_domain_new": (ctypes.c_void_p, [u32, u32]),
        "or_domain_free": (None, [ctypes.c_void_p]),
        "or_domain_k": (u32, [ctypes.c_void_p]),
        "or_domain_extended_k": (u32, [ctypes.c_void_p]),
        "or_domain_get": (None, [ctypes.c_void_p, i32, i32, _u64p]),
        "or_domain_lagrange_to_coeff": (None, [ctypes.c_void_p, _u64p, i32]),
        "or_domain_coeff_to_lagrange": (None, [ctypes.c_void_p, _u64p, i32]),
        "or_domain_coeff_to_extended": (None, [ctypes.c_void_p, _u64p, _u64p, i32]),
        "or_domain_extended_to_coeff": (None, [ctypes.c_void_p, _u64p, i32]),
        "or_domain_extended_to_lagrange": (None, [ctypes.c_void_p, _u64p, _u64p, i32]),
        "or_domain_divide_by_vanishing_poly": (None, [ctypes.c_void_p, _u64p, i32]),
        "or_quotient_eval": (None, [ctypes.c_void_p, ctypes.c_void_p, i32, _u64p, i32]),
        "or_quotient_eval_gates": (None, [ctypes.c_void_p, ctypes.c_void_p, i32, _u64p, _u64p, i32]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


class QuotientDesc(ctypes.Structure):
    """or_quotient_desc (oracle/mzk_oracle.h), host pointers."""
    _fields_ = [
    ("k", ctypes.c_uint32), ("extended_k", ctypes.c_uint32),
    ("advice", ctypes.POINTER(ctypes.c_void_p)), ("n_advice", ctypes.c_uint32),
    ("fixed", ctypes.POINTER(ctypes.c_void_p)), ("n_fixed", ctypes.c_uint32),
    ("gate_fixed", ctypes.c_uint32 * 5), ("gate_advice", ctypes.c_uint32 * 3),
    ("n_perm_cols", ctypes.c_uint32),
    ("perm_col_kind", ctypes.POINTER(ctypes.c_uint32)), ("perm_col_index", ctypes.POINTER(ctypes.c_uint32)),
    ("perm_sigma", ctypes.POINTER(ctypes.c_void_p)),
    ("n_perm_sets", ctypes.c_uint32), ("perm_z", ctypes.POINTER(ctypes.c_void_p)),
    ("chunk_len", ctypes.c_uint32), ("blinding_factors", ctypes.c_uint32),
    ("has_lookup", ctypes.c_int), ("lookup_input_advice", ctypes.c_uint32), ("lookup_table_fixed", ctypes.c_uint32),
    ("lookup_selector_fixed", ctypes.c_int32),
    ("lookup_h", ctypes.c_void_p), ("lookup_z", ctypes.c_void_p), ("lookup_m", ctypes.c_void_p),
    ("l0", ctypes.c_void_p), ("l_last", ctypes.c_void_p), ("l_active", ctypes.c_void_p),
    ("y", ctypes.c_uint64 * 4), ("beta", ctypes.c_uint64 * 4), ("gamma", ctypes.c_uint64 * 4),
    ("theta", ctypes.c_uint64 * 4), ("extended_omega", ctypes.c_uint64 * 4), ("g_coset", ctypes.c_uint64 * 4),
    ("instance", ctypes.POINTER(ctypes.c_void_p)), ("n_instance", ctypes.c_uint32),
]


def _run_program(graph, cols, idx, E, scale, challenges):
    """One row of a flattened program (FlatGraphEvaluator::evaluate,
    proofs/src/plonk/evaluation.rs:530-651) with the previous value zero;
    returns the whole values buffer.  challenges = (beta, theta, trash, y)."""
    zero = np.zeros(4, np.uint64)
    vals = [zero] * graph["values_len"]
    for i, c in enumerate(graph["constants"]):
        vals[i] = np.asarray(c, np.uint64)
    for slot, v in zip(("beta_idx", "theta_idx", "trash_challenge_idx", "y_idx"), challenges):
        vals[graph[slot]] = np.asarray(v, np.uint64)
    vals[graph["previous_value_idx"]] = zero
    for t, c, r, dst in graph["reads"]:
        vals[dst] = cols[t][c][(idx + (graph["rotations"][r] << scale)) % E]
    for kind, dst, a, b, c in graph["ops"]:
        if kind == 0:
            v = fr_op("add", vals[a], vals[b])
        elif kind == 1:
            v = fr_op("sub", vals[a], vals[b])
        elif kind == 2:
            v = fr_op("mul", vals[a], vals[b])
        elif kind == 3:
            v = fr_op("mul", vals[a], vals[a])
        elif kind == 4:
            v = fr_op("add", vals[a], vals[a])
        elif kind == 5:
            v = fr_op("neg", vals[a])
        else:
            v = fr_op("add", fr_op("mul", vals[a], vals[b]), vals[c])
        vals[dst] = v
    return vals


def flat_gates_eval(graph, fixed, advice, instance, k, extended_k, beta, theta, trash_challenge, y):
    """The custom-gate values of every row of the extended coset, restating
    FlatGraphEvaluator::evaluate_chunk (proofs/src/plonk/evaluation.rs:530-651)
    with the previous value zero (the gates are the first pass of
    evaluate_numerator, :846-856).  `graph` is a dict with the FlatGraph fields:
    constants, rotations, reads [(col_type, col_idx, rot_idx, dst)], ops
    [(kind, dst, a, b, c)], values_len and the slot indices; kinds in
    FlatOpKind order (:134-143).  Pure Python over single-element oracle field
    operations: small domains only."""
    E, scale = 1 << extended_k, extended_k - k
    cols, ch = (fixed, advice, instance), (beta, theta, trash_challenge, y)
    out = np.zeros((E, 4), np.uint64)
    for idx in range(E):
        out[idx] = _run_program(graph, cols, idx, E, scale, ch)[graph["result_idx"]]
    return out


def flat_tail_eval(v_in, fixed, advice, instance, k, extended_k, beta, theta, trash_challenge, y, l0, l_last,
                   l_active, lookups=(), trashcans=()):
    """The lookup terms (evaluation.rs:1034-1090) and trash terms (:1093-1109)
    of any shape continuing each row's y-Horner accumulator v_in (the gate and
    permutation terms).  lookups: [{"programs": [graph], "outputs":
    [(sum_partial_products, product, table, selector)], "helpers": [col],
    "aggregator": col, "multiplicities": col}]; trashcans: [{"program": graph,
    "selector": fixed index, "trash": col}].  Pure Python, small domains."""
    E, scale = 1 << extended_k, extended_k - k
    cols, ch = (fixed, advice, instance), (beta, theta, trash_challenge, y)
    one = fr_const(0)
    out = np.zeros((E, 4), np.uint64)
    for idx in range(E):
        r_next = (idx + (1 << scale)) % E
        v = v_in[idx]
        for lk in lookups:
            Z = lk["aggregator"][idx]
            v = fr_op("add", fr_op("mul", v, y), fr_op("mul", Z, fr_op("add", l0[idx], l_last[idx])))
            sum_h = np.zeros(4, np.uint64)
            table = sel = None
            for fi, prog in enumerate(lk["programs"]):
                vals = _run_program(prog, cols, idx, E, scale, ch)
                spp, prod, tbl, sl = lk["outputs"][fi]
                if fi == 0:
                    table, sel = vals[tbl], vals[sl]
                h = lk["helpers"][fi][idx]
                v = fr_op("sub", fr_op("add", fr_op("mul", v, y), fr_op("mul", h, vals[prod])), vals[spp])
                sum_h = fr_op("add", sum_h, h)
            u = fr_op("sub", fr_op("sub", lk["aggregator"][r_next], Z), fr_op("mul", sel, sum_h))
            u = fr_op("add", fr_op("mul", u, table), lk["multiplicities"][idx])
            v = fr_op("add", fr_op("mul", v, y), fr_op("mul", l_active[idx], u))
        for tc in trashcans:
            comp = _run_program(tc["program"], cols, idx, E, scale, ch)[tc["program"]["result_idx"]]
            q = fixed[tc["selector"]][idx]
            v = fr_op("add", fr_op("mul", v, y), fr_op("sub", comp, fr_op("mul", fr_op("sub", one, q), tc["trash"][idx])))
        out[idx] = v
    return out


def threads_default():
    return int(os.environ.get("MZK_ORACLE_THREADS", os.cpu_count() or 1))


def P(a):
    """uint64 pointer to a C-contiguous numpy array."""
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def u64s(limbs):
    return np.array([int(x, 16) if isinstance(x, str) else int(x) for x in limbs], dtype=np.uint64)


# ---- integers <-> limbs ----
def to_int(limbs):
    return sum(int(v) << (64 * i) for i, v in enumerate(np.asarray(limbs, dtype=np.uint64).tolist()))


def from_int(v, n):
    return np.array([(v >> (64 * i)) & (2**64 - 1) for i in range(n)], dtype=np.uint64)


# ---- Fr ----
def fr_const(which):
    o = np.zeros(4, np.uint64)
    lib.or_fr_const(which, P(o))
    return o


def fr_op(name, *args):
    o = np.zeros(4, np.uint64)
    args = [np.ascontiguousarray(a, dtype=np.uint64) for a in args]
    getattr(lib, "or_fr_" + name)(P(o), *[P(a) for a in args])
    return o


def fp_op(name, *args):
    o = np.zeros(6, np.uint64)
    args = [np.ascontiguousarray(a, dtype=np.uint64) for a in args]
    getattr(lib, "or_fp_" + name)(P(o), *[P(a) for a in args])
    return o


def fp_const(which):
    o = np.zeros(6, np.uint64)
    lib.or_fp_const(which, P(o))
    return o


# ---- G1 ----
def g1_generator():
    o = np.zeros(12, np.uint64)
    lib.or_g1_generator(P(o))
    return o


def g1_mul(aff, scalar_mont):
    o = np.zeros(12, np.uint64)
    lib.or_g1_mul(P(o), P(np.ascontiguousarray(aff, np.uint64)), P(np.ascontiguousarray(scalar_mont, np.uint64)))
    return o


def g1_jac_add(a, b):
    o = np.zeros(18, np.uint64)
    lib.or_g1_add(P(o), P(np.ascontiguousarray(a, np.uint64)), P(np.ascontiguousarray(b, np.uint64)))
    return o


def g1_jac_double(a):
    o = np.zeros(18, np.uint64)
    lib.or_g1_double(P(o), P(np.ascontiguousarray(a, np.uint64)))
    return o


def g1_to_affine(jac):
    o = np.zeros(12, np.uint64)
    lib.or_g1_to_affine(P(o), P(np.ascontiguousarray(jac, np.uint64)))
    return o


def g1_from_affine(aff):
    o = np.zeros(18, np.uint64)
    lib.or_g1_from_affine(P(o), P(np.ascontiguousarray(aff, np.uint64)))
    return o


def g1_is_on_curve(aff):
    return bool(lib.or_g1_is_on_curve_affine(P(np.ascontiguousarray(aff, np.uint64))))


def g1_compress(aff):
    o = np.zeros(48, np.uint8)
    lib.or_g1_compress(o.ctypes.data_as(_u8p), P(np.ascontiguousarray(aff, np.uint64)))
    return bytes(o)


# ---- MSM ----
def msm_naive(scalars, bases):
    o = np.zeros(12, np.uint64)
    lib.or_msm_naive(P(o), P(scalars), P(bases), scalars.shape[0])
    return o


def msm_best(scalars, bases, threads=None):
    o = np.zeros(12, np.uint64)
    lib.or_msm_best(P(o), P(scalars), P(bases), scalars.shape[0], threads or threads_default())
    return o


def msm_specific(scalars, bases, threads=None):
    o = np.zeros(12, np.uint64)
    lib.or_msm_specific(P(o), P(scalars), P(bases), scalars.shape[0], threads or threads_default())
    return o


def booth_index(window_index, window_size, repr32):
    b = np.ascontiguousarray(np.frombuffer(bytes(repr32), dtype=np.uint8))
    return lib.or_booth_index(window_index, window_size, b.ctypes.data_as(_u8p))


def fr_inner_product(s, r, threads=None):
    o = np.zeros(4, np.uint64)
    lib.or_fr_inner_product(P(o), P(s), P(r), s.shape[0], threads or threads_default())
    return o


# ---- seeded inputs ----
def rand_fr(seed, n, first=0, threads=None):
    o = np.zeros((n, 4), np.uint64)
    lib.or_rand_fr(P(o), seed, first, n, threads or threads_default())
    return o


def gen_bases(seed, n, first=0, threads=None):
    o = np.zeros((n, 12), np.uint64)
    lib.or_gen_bases(P(o), seed, first, n, threads or threads_default())
    return o


# ---- FFT ----
def compute_twiddles(omega, log_n):
    o = np.zeros(((1 << log_n) // 2, 4), np.uint64)
    lib.or_compute_twiddles(P(o), P(np.ascontiguousarray(omega, np.uint64)), log_n)
    return o


def best_fft(a, twiddles, log_n, threads=None):
    a = np.ascontiguousarray(a, np.uint64).copy()
    lib.or_best_fft(P(a), P(twiddles), log_n, threads or threads_default())
    return a


def fft_dif_pruned(a, twiddles, log_n, n_real, threads=None):
    a = np.ascontiguousarray(a, np.uint64).copy()
    lib.or_fft_dif_pruned(P(a), P(twiddles), log_n, n_real, threads or threads_default())
    return a


def dft_naive(a, omega):
    o = np.zeros_like(a)
    lib.or_dft_naive(P(o), P(np.ascontiguousarray(a, np.uint64)), P(np.ascontiguousarray(omega, np.uint64)), a.shape[0])
    return o


def eval_polynomial(poly, point, threads=None):
    o = np.zeros(4, np.uint64)
    poly = np.ascontiguousarray(poly, np.uint64)
    lib.or_eval_polynomial(P(o), P(poly), poly.shape[0], P(np.ascontiguousarray(point, np.uint64)),
                           threads or threads_default())
    return o


def _ptr_array(arrays):
    arr = (ctypes.c_void_p * max(1, len(arrays)))(*[a.ctypes.data for a in arrays])
    return arr


def batch_invert(a):
    """ff BatchInvert: every non-zero element inverted, zeros left as zero."""
    o = np.ascontiguousarray(a, np.uint64).copy()
    lib.or_fr_batch_invert(P(o), o.shape[0])
    return o


def permutation_z(values, sigmas, chunk_len, k, omega, beta, gamma, blinding_factors, blinds):
    """permutation/prover.rs:81-255: z of every set (Lagrange form).  blinds:
    (n_sets, blinding_factors, 4)."""
    n = 1 << k
    values = [np.ascontiguousarray(v, np.uint64) for v in values]
    sigmas = [np.ascontiguousarray(v, np.uint64) for v in sigmas]
    n_sets = (len(values) + chunk_len - 1) // chunk_len
    zs = [np.zeros((n, 4), np.uint64) for _ in range(n_sets)]
    bl = np.ascontiguousarray(blinds, np.uint64).reshape(-1, 4)
    lib.or_permutation_z(_ptr_array(values), _ptr_array(sigmas), len(values), chunk_len, k,
                         P(np.ascontiguousarray(omega, np.uint64)), P(np.ascontiguousarray(beta, np.uint64)),
                         P(np.ascontiguousarray(gamma, np.uint64)), blinding_factors, P(bl), _ptr_array(zs))
    return zs


def logup(chunks, table, selector, multiplicities, beta, blinding_factors, blinds):
    """logup/prover.rs:195-300: (helper per chunk, aggregator).  chunks: list
    of lists of compressed input columns."""
    n = table.shape[0]
    cols = [np.ascontiguousarray(c, np.uint64) for ch in chunks for c in ch]
    counts = (ctypes.c_uint32 * max(1, len(chunks)))(*[len(ch) for ch in chunks])
    helpers = [np.zeros((n, 4), np.uint64) for _ in chunks]
    agg = np.zeros((n, 4), np.uint64)
    lib.or_logup(_ptr_array(cols), counts, len(chunks), P(np.ascontiguousarray(table, np.uint64)),
                 P(np.ascontiguousarray(selector, np.uint64)), P(np.ascontiguousarray(multiplicities, np.uint64)),
                 n, P(np.ascontiguousarray(beta, np.uint64)), blinding_factors,
                 P(np.ascontiguousarray(blinds, np.uint64).reshape(-1, 4)), _ptr_array(helpers), P(agg))
    return helpers, agg


def poly_inner_product(polys, scalars):
    """kzg/mod.rs:125-147: sum_p scalars[p] polys[p], zero-extended."""
    polys = [np.ascontiguousarray(p, np.uint64) for p in polys]
    out_len = max((p.shape[0] for p in polys), default=0)
    lens = (ctypes.c_size_t * max(1, len(polys)))(*[p.shape[0] for p in polys])
    out = np.zeros((out_len, 4), np.uint64)
    sc = np.ascontiguousarray(scalars, np.uint64).reshape(-1, 4)
    lib.or_poly_inner_product(_ptr_array(polys), lens, len(polys), P(sc), P(out), out_len)
    return out


def g1_decompress(b48, check_subgroup=True):
    """(status, affine point): 0 ok, 1 bad encoding, 2 not on the curve, 3 not in G1."""
    buf = np.frombuffer(bytes(b48), np.uint8).copy()
    out = np.zeros(12, np.uint64)
    st = lib.or_g1_decompress(P(out), buf.ctypes.data_as(_u8p), 1 if check_subgroup else 0)
    return st, out


def g1_suffix_sum(points):
    """params.rs:47-57: out[i] = sum_{j >= i} points[j] (affine)."""
    p = np.ascontiguousarray(points, np.uint64)
    out = np.zeros_like(p)
    lib.or_g1_suffix_sum(P(p), p.shape[0], P(out))
    return out


def srs_setup(s, k):
    """params.rs:160-209 (G1 part): (g, g_lagrange, g_lagrange_delta, g_lagrange_double_delta)."""
    n = 1 << k
    omega = Domain(5, k).get(0) if k >= 1 else fr_const(0)
    outs = [np.zeros((n, 12), np.uint64) for _ in range(4)]
    lib.or_srs_setup(P(np.ascontiguousarray(s, np.uint64)), k, P(omega), *[P(o) for o in outs])
    return outs


def count_fr_muls(fn, *args, **kwargs):
    """(result of fn, Fr multiplications the C oracle made while it ran);
    run fn single-threaded for an exact count."""
    lib.or_fr_mul_counter(1)
    try:
        out = fn(*args, **kwargs)
    finally:
        count = lib.or_fr_mul_counter(0)
    return out, int(count)


def fr_mul_vec(a, b):
    """element-wise product of two Fr arrays of the same length"""
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    out = np.zeros_like(a)
    lib.or_fr_mul_vec(P(a), P(b), P(out), a.shape[0])
    return out


def kate_division(a, b):
    """utils/arithmetic.rs:106-125: coefficients of a(X) / (X - b), n - 1 of them."""
    a = np.ascontiguousarray(a, np.uint64)
    q = np.zeros((max(0, a.shape[0] - 1), 4), np.uint64)
    lib.or_kate_division(P(a), a.shape[0], P(np.ascontiguousarray(b, np.uint64)), P(q))
    return q


def fr_pow(x, e):
    r = fr_const(0)
    b = np.ascontiguousarray(x, np.uint64).copy()
    while e:
        if e & 1:
            r = fr_op("mul", r, b)
        b = fr_op("mul", b, b)
        e >>= 1
    return r


class Domain:
    """EvaluationDomain restatement (proofs/src/poly/domain.rs:54-414)."""

    def __init__(self, j, k):
        self.h = lib.or_domain_new(j, k)
        self.k = lib.or_domain_k(self.h)
        self.extended_k = lib.or_domain_extended_k(self.h)
        self.n = 1 << self.k
        self.extended_len = 1 << self.extended_k

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_domain_free(self.h)
            self.h = None

    def get(self, which, idx=0):
        o = np.zeros(4, np.uint64)
        lib.or_domain_get(self.h, which, idx, P(o))
        return o

    def lagrange_to_coeff(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64).copy()
        lib.or_domain_lagrange_to_coeff(self.h, P(a), threads or threads_default())
        return a

    def coeff_to_lagrange(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64).copy()
        lib.or_domain_coeff_to_lagrange(self.h, P(a), threads or threads_default())
        return a

    def coeff_to_extended(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64)
        o = np.zeros((self.extended_len, 4), np.uint64)
        lib.or_domain_coeff_to_extended(self.h, P(a), P(o), threads or threads_default())
        return o

    def extended_to_coeff(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64).copy()
        lib.or_domain_extended_to_coeff(self.h, P(a), threads or threads_default())
        return a

    def extended_to_lagrange(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64).copy()
        o = np.zeros((self.n, 4), np.uint64)
        lib.or_domain_extended_to_lagrange(self.h, P(a), P(o), threads or threads_default())
        return o

    def quotient_eval(self, desc, divide=True, threads=None, gate_values=None):
        o = np.zeros((self.extended_len, 4), np.uint64)
        if gate_values is None:
            lib.or_quotient_eval(ctypes.byref(desc), self.h, 1 if divide else 0, P(o), threads or threads_default())
        else:
            g = np.ascontiguousarray(gate_values, np.uint64)
            lib.or_quotient_eval_gates(ctypes.byref(desc), self.h, 1 if divide else 0, P(g), P(o),
                                       threads or threads_default())
        return o

    def divide_by_vanishing_poly(self, a, threads=None):
        a = np.ascontiguousarray(a, np.uint64).copy()
        lib.or_domain_divide_by_vanishing_poly(self.h, P(a), threads or threads_default())
        return a
