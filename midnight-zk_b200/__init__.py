"""Host-side mirror of the midnight-zk prover-core interface over the B200 C ABI.

The product is the CUDA library ``lib/libmzkgpu.so`` (sources in ``csrc/``,
ABI in ``include/mzk.h``).  This module binds it with ctypes and offers the
reference's operations under the reference's names:

    ctx = Context(0)
    ctx.msm_best(scalars, bases)        # curves::msm::msm_best      (curves/src/msm.rs:460)
    ctx.msm_specific(scalars, bases)    # kzg::msm::msm_specific     (proofs/src/poly/kzg/msm.rs:174)

Arrays use the reference's in-memory layouts as numpy uint64: Fr (``Fq``)
elements shape (n, 4) Montgomery, G1Affine shape (n, 12), G1Projective
shape (18,) (blst_p1 Jacobian; results come back with z = 1 or all-zero for
the identity).  There is no CPU fallback: when the library or a CUDA device is
missing every call raises ``MzkError``.

The directory name is not a Python identifier; ``_loader.load()`` at the
repository root imports it as ``mzk_b200``.
"""
import ctypes
import weakref
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libmzkgpu.so"
HEADER = PKG.parent / "include" / "mzk.h"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_i32 = ctypes.c_int
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32

# name -> (restype, argtypes); every symbol declared in include/mzk.h
SIGNATURES = {
    "mzk_ctx_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "mzk_ctx_destroy": (_i32, [_vp]),
    "mzk_last_error": (ctypes.c_char_p, []),
    "mzk_version": (ctypes.c_char_p, []),
    "mzk_ctx_launch_count": (_u64, [_vp]),
    "mzk_ctx_stream": (_vp, [_vp]),
    "mzk_ctx_synchronize": (_i32, [_vp]),
    "mzk_ctx_set_profiling": (_i32, [_vp, _i32]),
    "mzk_ctx_phase_stats": (_i32, [_vp, ctypes.POINTER(ctypes.c_double), _u64p, _i32]),
    "mzk_ctx_prove_phase_stats": (_i32, [_vp, ctypes.POINTER(ctypes.c_double), _u64p, _i32, _i32]),
    "mzk_probe_batch_affine": (_i32, [_vp, ctypes.POINTER(ctypes.c_double)]),
    "mzk_probe_fp_inv_check": (_i32, [_vp, _vp, _sz, _u64p]),
    "mzk_probe_imad_peak": (_i32, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]),
    "mzk_msm_last_shape": (_i32, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32), _u64p]),
    "mzk_device_alloc": (_i32, [_vp, _sz, ctypes.POINTER(_vp)]),
    "mzk_device_free": (_i32, [_vp, _vp]),
    "mzk_memcpy_h2d": (_i32, [_vp, _vp, _vp, _sz]),
    "mzk_memcpy_d2h": (_i32, [_vp, _vp, _vp, _sz]),
    "mzk_probe_fp_sqr_check": (_i32, [_vp, _vp, _sz, _u64p]),
    "mzk_autotune": (_i32, [_vp, _vp, _vp, ctypes.POINTER(_u32), _sz, ctypes.POINTER(_u32), _sz, _i32,
                            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "mzk_autotune_get": (_i32, [_vp, _i32, _u32, ctypes.POINTER(_i32)]),
    "mzk_g1_compress_device": (_i32, [_vp, _vp, _sz, _vp]),
    "mzk_msm_table_rows": (_i32, [_i32]),
    "mzk_msm_window_table": (_i32, [_vp, _vp, _sz, _i32, _sz]),
    "mzk_msm_g1_batch_table_device": (_i32, [_vp, _vp, _sz, _i32, _sz, _sz, _vp, _sz, _u64p]),
    "mzk_srs_write_processed": (_i32, [_vp, _vp, _vp, _sz, _vp, _sz]),
    "mzk_ctx_graph_stats": (_i32, [_vp, _u64p, _u64p]),
    "mzk_autotune_set": (_i32, [_vp, _i32, _u32, _i32]),
    "mzk_autotune_save": (_i32, [_vp, ctypes.c_char_p]),
    "mzk_autotune_load": (_i32, [_vp, ctypes.c_char_p]),
    "mzk_msm_g1": (_i32, [_vp, _u64p, _u64p, _sz, _u64p]),
    "mzk_msm_g1_device": (_i32, [_vp, _vp, _vp, _sz, _u64p]),
    "mzk_g1_sum_host": (_i32, [_u64p, _sz, _u64p]),
    "mzk_msm_g1_noalloc": (_i32, [_vp, _vp, _sz, _u64p, _vp]),
    "mzk_msm_g1_batch_device": (_i32, [_vp, _vp, _sz, _vp, _sz, _u64p]),
    "mzk_msm_set_window": (_i32, [_vp, _i32]),
    "mzk_msm_pick_window": (_i32, [_sz]),
    "mzk_domain_create": (_i32, [_vp, _u32, _u32, ctypes.POINTER(_vp)]),
    "mzk_domain_destroy": (_i32, [_vp]),
    "mzk_domain_shape": (_i32, [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u32)]),
    "mzk_domain_constant": (_i32, [_vp, _i32, _i32, _u64p]),
    "mzk_domain_op": (_i32, [_vp, _vp, _i32, _u64p, _u64p]),
    "mzk_domain_op_device": (_i32, [_vp, _vp, _i32, _vp, _vp]),
    "mzk_domain_op_batch_device": (_i32, [_vp, _vp, _i32, _vp, _vp, _sz]),
    "mzk_quotient_eval_device": (_i32, [_vp, _vp, ctypes.c_void_p, _i32, _vp]),
    "mzk_compute_h_poly_device": (_i32, [_vp, _vp, ctypes.c_void_p, _vp, _sz, _u64p, _u64p, _vp]),
    "mzk_prove_core_device": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, _sz, _u32, _u64p]),
    "mzk_batch_invert_device": (_i32, [_vp, ctypes.c_void_p, _sz]),
    "mzk_eval_polynomial_device": (_i32, [_vp, ctypes.c_void_p, _sz, _u64p, _u64p]),
    "mzk_kate_division_device": (_i32, [_vp, ctypes.c_void_p, _sz, _u64p, ctypes.c_void_p]),
    "mzk_permutation_z_device": (_i32, [_vp, _vp, ctypes.c_void_p]),
    "mzk_srs_setup_device": (_i32, [_vp, _vp, _u64p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "mzk_g1_suffix_sum_device": (_i32, [_vp, ctypes.c_void_p, _sz, ctypes.c_void_p]),
    "mzk_g1_to_lagrange_device": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p]),
    "mzk_srs_downsize_device": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mzk_g1_decompress_device": (_i32, [_vp, ctypes.c_void_p, _sz, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        _u64p]),
    "mzk_srs_read_processed": (_i32, [_vp, ctypes.c_void_p, _sz, _sz, ctypes.POINTER(_u32), ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mzk_poly_inner_product_device": (_i32, [_vp, ctypes.c_void_p, ctypes.c_void_p, _sz, _u64p, ctypes.c_void_p, _sz]),
    "mzk_logup_device": (_i32, [_vp, _vp, ctypes.c_void_p]),
    "mzk_server_create": (_i32, [_vp, _u32, _u32, _u64, _u32, ctypes.POINTER(_vp)]),
    "mzk_server_set_wave_rows": (_i32, [_vp, _u64]),
    "mzk_server_submit": (_i32, [_vp, ctypes.c_void_p, _u64p]),
    "mzk_server_wait": (_i32, [_vp, _u64, ctypes.POINTER(ctypes.c_double)]),
    "mzk_server_stats": (_i32, [_vp, _u64p, _u64p, ctypes.POINTER(ctypes.c_double)]),
    "mzk_server_destroy": (_i32, [_vp]),
    "mzk_transcript_create": (_i32, [ctypes.POINTER(_vp)]),
    "mzk_transcript_destroy": (_i32, [_vp]),
    "mzk_transcript_common_fr": (_i32, [_vp, _u64p]),
    "mzk_transcript_write_fr": (_i32, [_vp, _u64p]),
    "mzk_transcript_write_point": (_i32, [_vp, _u64p]),
    "mzk_transcript_squeeze": (_i32, [_vp, _u64p]),
    "mzk_transcript_proof": (_i32, [_vp, ctypes.c_void_p, _sz, ctypes.POINTER(_sz)]),
    "mzk_vk_transcript_repr": (_i32, [_u32, ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, _u64p]),
    "mzk_keygen": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p, _sz, ctypes.POINTER(_vp)]),
    "mzk_keygen_from_values": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, _sz, ctypes.POINTER(_vp)]),
    "mzk_plonk_key_transcript_layout": (_i32, [_vp, ctypes.c_void_p, _sz, ctypes.POINTER(_sz)]),
    "mzk_vk_write": (_i32, [_vp, _i32, ctypes.c_void_p, _sz, ctypes.POINTER(_sz)]),
    "mzk_pk_write": (_i32, [_vp, _vp, _i32, ctypes.c_void_p, _sz, ctypes.POINTER(_sz)]),
    "mzk_pk_read": (_i32, [_vp, _vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _sz, _i32, ctypes.c_void_p,
                           _sz, ctypes.POINTER(_vp)]),
    "mzk_plonk_key_destroy": (_i32, [_vp]),
    "mzk_plonk_key_info": (_i32, [_vp, _u64p, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]),
    "mzk_plonk_key_commitments": (_i32, [_vp, ctypes.c_void_p, ctypes.c_void_p]),
    "mzk_plonk_key_srs": (_i32, [_vp, ctypes.c_void_p]),
    "mzk_create_proofs": (_i32, [_vp, ctypes.c_void_p, _sz, _u32]),
    "mzk_gen_config3_fixed_device": (_i32, [_vp, _u32, _u32, _u32, _u64, _vp]),
    "mzk_gen_config3_witness_device": (_i32, [_vp, _u32, _u32, _u32, _u64, _vp, _vp, _vp, _vp]),
    "mzk_gen_rand_fr_device": (_i32, [_vp, _u64, _u64, _sz, _vp]),
    "mzk_gen_bases_g1_device": (_i32, [_vp, _u64, _u64, _sz, _vp]),
}

class MsmBatchItem(ctypes.Structure):
    """mzk_msm_batch_item (include/mzk.h)."""
    _fields_ = [("d_scalars", ctypes.c_void_p), ("base_offset", ctypes.c_uint64), ("n", ctypes.c_uint64)]


class ProvingKeyDesc(ctypes.Structure):
    """mzk_proving_key_desc (include/mzk.h)."""
    _fields_ = [("k", ctypes.c_uint32), ("fixed_ext", ctypes.c_void_p * 7), ("sigma_ext", ctypes.c_void_p * 3),
                ("l0_ext", ctypes.c_void_p), ("l_last_ext", ctypes.c_void_p), ("l_active_ext", ctypes.c_void_p),
                ("srs", ctypes.c_void_p), ("srs_len", ctypes.c_uint64), ("off_g", ctypes.c_uint64),
                ("off_lagrange", ctypes.c_uint64), ("off_lagrange_delta", ctypes.c_uint64),
                ("off_lagrange_double_delta", ctypes.c_uint64), ("blinding_factors", ctypes.c_uint32),
                ("sigma_lagrange", ctypes.c_void_p * 3), ("table_lagrange", ctypes.c_void_p),
                ("selector_lagrange", ctypes.c_void_p), ("srs_table_c", ctypes.c_int32),
                ("srs_table_rows", ctypes.c_uint32), ("srs_table_min_n", ctypes.c_uint64)]


class ProofJob(ctypes.Structure):
    """mzk_proof_job (include/mzk.h)."""
    _fields_ = [("advice", ctypes.c_void_p * 3), ("perm_z", ctypes.c_void_p), ("lookup_m", ctypes.c_void_p),
                ("lookup_h", ctypes.c_void_p), ("lookup_Z", ctypes.c_void_p), ("y", ctypes.c_uint64 * 4),
                ("beta", ctypes.c_uint64 * 4), ("gamma", ctypes.c_uint64 * 4), ("theta", ctypes.c_uint64 * 4),
                ("quotient_blinds", (ctypes.c_uint64 * 4) * 3), ("perm_blinds", (ctypes.c_uint64 * 4) * 8),
                ("lookup_blinds", (ctypes.c_uint64 * 4) * 8)]


SERDE_PROCESSED, SERDE_RAW, SERDE_RAW_UNCHECKED = 0, 1, 2  # SerdeFormat (MZK_SERDE_*)
PROVE_MSM_PER_CALL = 1  # MZK_PROVE_MSM_PER_CALL
PROVE_NO_GRAPHS = 2  # MZK_PROVE_NO_GRAPHS
PROVE_SELF_CHECK = 4  # MZK_PROVE_SELF_CHECK
# the plain one-call-at-a-time form: every MSM its own call, every kernel its own launch
PROVE_PLAIN = PROVE_MSM_PER_CALL | PROVE_NO_GRAPHS
PROOF_CORE_COMMITMENTS = ["a", "b", "c", "m_delta", "z_delta", "Z_double_delta", "h", "H0", "H1", "H2", "H3"]


class QuotientDesc(ctypes.Structure):
    """mzk_quotient_desc (include/mzk.h): columns of the quotient evaluation."""
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
    ("gates", ctypes.c_void_p), ("instance", ctypes.POINTER(ctypes.c_void_p)), ("n_instance", ctypes.c_uint32),
    ("trash_challenge", ctypes.c_uint64 * 4),
    ("n_lookups", ctypes.c_uint32), ("lookups", ctypes.c_void_p), ("n_trash", ctypes.c_uint32),
    ("trash", ctypes.c_void_p),
]

# FlatOpKind (proofs/src/plonk/evaluation.rs:134-143), MZK_FLAT_* in include/mzk.h
FLAT_ADD, FLAT_SUB, FLAT_MUL, FLAT_SQUARE, FLAT_DOUBLE, FLAT_NEGATE, FLAT_MULADD = range(7)
COL_FIXED, COL_ADVICE, COL_INSTANCE = 0, 1, 2


class ColumnRead(ctypes.Structure):
    _fields_ = [("col_type", ctypes.c_uint32), ("col_idx", ctypes.c_uint32), ("rot_idx", ctypes.c_uint32),
                ("dst", ctypes.c_uint32)]


class FlatOp(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("dst", ctypes.c_uint32), ("a", ctypes.c_uint32), ("b", ctypes.c_uint32),
                ("c", ctypes.c_uint32)]


class FlatGraph(ctypes.Structure):
    """mzk_flat_graph: the custom gates as the reference's FlatGraphEvaluator
    (proofs/src/plonk/evaluation.rs:148-213)."""
    _fields_ = [
        ("constants", ctypes.c_void_p), ("n_constants", ctypes.c_uint32),
        ("rotations", ctypes.POINTER(ctypes.c_int32)), ("n_rotations", ctypes.c_uint32),
        ("reads", ctypes.POINTER(ColumnRead)), ("n_reads", ctypes.c_uint32),
        ("ops", ctypes.POINTER(FlatOp)), ("n_ops", ctypes.c_uint32),
        ("values_len", ctypes.c_uint32),
        ("beta_idx", ctypes.c_uint32), ("theta_idx", ctypes.c_uint32), ("trash_challenge_idx", ctypes.c_uint32),
        ("y_idx", ctypes.c_uint32), ("previous_value_idx", ctypes.c_uint32), ("result_idx", ctypes.c_uint32),
    ]


def build_flat_graph(constants, rotations, reads, ops, values_len, beta_idx, theta_idx, trash_challenge_idx, y_idx,
                     previous_value_idx, result_idx):
    """A FlatGraph from plain Python data: constants (m, 4) uint64 Montgomery,
    rotations [int], reads [(col_type, col_idx, rot_idx, dst)], ops
    [(kind, dst, a, b, c)].  Keeps its arrays alive on the returned object."""
    g = FlatGraph()
    consts = np.ascontiguousarray(np.asarray(constants, np.uint64).reshape(-1, 4))
    rots = (ctypes.c_int32 * max(1, len(rotations)))(*rotations)
    rd = (ColumnRead * max(1, len(reads)))(*[ColumnRead(*r) for r in reads])
    op = (FlatOp * max(1, len(ops)))(*[FlatOp(*(tuple(o) + (0,) * (5 - len(o)))) for o in ops])
    g.constants, g.n_constants = consts.ctypes.data, consts.shape[0]
    g.rotations, g.n_rotations = ctypes.cast(rots, ctypes.POINTER(ctypes.c_int32)), len(rotations)
    g.reads, g.n_reads = ctypes.cast(rd, ctypes.POINTER(ColumnRead)), len(reads)
    g.ops, g.n_ops = ctypes.cast(op, ctypes.POINTER(FlatOp)), len(ops)
    g.values_len = values_len
    g.beta_idx, g.theta_idx, g.trash_challenge_idx = beta_idx, theta_idx, trash_challenge_idx
    g.y_idx, g.previous_value_idx, g.result_idx = y_idx, previous_value_idx, result_idx
    g._keep = (consts, rots, rd, op)
    return g


class LookupArg(ctypes.Structure):
    """mzk_lookup_arg: a logup argument of any shape as one program per helper."""
    _fields_ = [("n_helpers", ctypes.c_uint32), ("programs", ctypes.POINTER(FlatGraph)),
                ("outputs", ctypes.POINTER(ctypes.c_uint32)), ("helpers", ctypes.POINTER(ctypes.c_void_p)),
                ("aggregator", ctypes.c_void_p), ("multiplicities", ctypes.c_void_p)]


class TrashArg(ctypes.Structure):
    """mzk_trash_arg: a trash argument (program, selector column, trash polynomial)."""
    _fields_ = [("program", FlatGraph), ("selector_fixed", ctypes.c_uint32), ("trash", ctypes.c_void_p)]


def build_quotient_desc(cols, k, extended_k, addr):
    """Fill a QuotientDesc from `cols` (a dict of column objects and parameters);
    addr(x) turns each column object into an address (device pointer or host
    array).  Keeps the pointer arrays alive on the returned object."""
    d = QuotientDesc()
    keep = []

    def ptr_array(items):
        arr = (ctypes.c_void_p * max(1, len(items)))(*[addr(x) for x in items])
        keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p))

    def u32_array(items):
        arr = (ctypes.c_uint32 * max(1, len(items)))(*items)
        keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_uint32))

    d.k, d.extended_k = k, extended_k
    d.advice, d.n_advice = ptr_array(cols["advice"]), len(cols["advice"])
    d.fixed, d.n_fixed = ptr_array(cols["fixed"]), len(cols["fixed"])
    d.gate_fixed[:] = cols.get("gate_fixed", [0] * 5)
    d.gate_advice[:] = cols.get("gate_advice", [0] * 3)
    pc = cols.get("perm_cols", [])
    d.n_perm_cols = len(pc)
    d.perm_col_kind = u32_array([kind for kind, _ in pc])
    d.perm_col_index = u32_array([idx for _, idx in pc])
    d.perm_sigma = ptr_array(cols.get("perm_sigma", []))
    d.n_perm_sets = len(cols.get("perm_z", []))
    d.perm_z = ptr_array(cols.get("perm_z", []))
    d.chunk_len = cols.get("chunk_len", 3)
    d.blinding_factors = cols.get("blinding_factors", 7)
    lk = cols.get("lookup")
    d.has_lookup = 1 if lk else 0
    if lk:
        d.lookup_input_advice, d.lookup_table_fixed, d.lookup_selector_fixed = lk["input"], lk["table"], lk["selector"]
        d.lookup_h, d.lookup_z, d.lookup_m = addr(lk["h"]), addr(lk["z"]), addr(lk["m"])
    d.l0, d.l_last, d.l_active = addr(cols["l0"]), addr(cols["l_last"]), addr(cols["l_active"])
    for name in ("y", "beta", "gamma", "theta", "extended_omega", "g_coset", "trash_challenge"):
        if name in cols:
            getattr(d, name)[:] = [int(v) for v in cols[name]]
    if cols.get("gates") is not None:
        keep.append(cols["gates"])
        d.gates = ctypes.addressof(cols["gates"])
    inst = cols.get("instance", [])
    d.instance, d.n_instance = ptr_array(inst), len(inst)
    # lookups / trashcans as programs: [{"programs": [FlatGraph], "outputs": [(spp, prod, table, sel)],
    # "helpers": [col], "aggregator": col, "multiplicities": col}], [{"program": FlatGraph, "selector": i,
    # "trash": col}]
    lps = cols.get("lookup_programs", [])
    if lps:
        arr = (LookupArg * len(lps))()
        for n, lp in enumerate(lps):
            progs = (FlatGraph * len(lp["programs"]))(*lp["programs"])
            outs = (ctypes.c_uint32 * (4 * len(lp["outputs"])))(*[v for o in lp["outputs"] for v in o])
            keep.extend([progs, outs] + list(lp["programs"]))
            arr[n].n_helpers = len(lp["programs"])
            arr[n].programs = ctypes.cast(progs, ctypes.POINTER(FlatGraph))
            arr[n].outputs = ctypes.cast(outs, ctypes.POINTER(ctypes.c_uint32))
            arr[n].helpers = ptr_array(lp["helpers"])
            arr[n].aggregator, arr[n].multiplicities = addr(lp["aggregator"]), addr(lp["multiplicities"])
        keep.append(arr)
        d.n_lookups, d.lookups = len(lps), ctypes.addressof(arr)
    tcs = cols.get("trash", [])
    if tcs:
        arr = (TrashArg * len(tcs))()
        for n, tc in enumerate(tcs):
            arr[n].program = tc["program"]
            arr[n].selector_fixed, arr[n].trash = tc["selector"], addr(tc["trash"])
            keep.append(tc["program"])
        keep.append(arr)
        d.n_trash, d.trash = len(tcs), ctypes.addressof(arr)
    d._keep = keep
    return d


STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_CUDA", 4: "ERR_TIMEOUT", 5: "ERR_STATE"}


class MzkError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """The loaded CUDA library (raises MzkError when it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise MzkError(5, f"{LIB_PATH} is missing: run __graft_entry__.build() (no CPU fallback exists)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise MzkError(status, lib().mzk_last_error().decode(errors="replace"))


def _ptr(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "expect C-contiguous uint64 arrays"
    return a.ctypes.data_as(_u64p)


class DeviceBuffer:
    """Device memory owned through the library (plumbing for tests/bench)."""

    def __init__(self, ctx, nbytes):
        self.ctx = ctx
        self.nbytes = int(nbytes)
        p = _vp()
        _check(lib().mzk_device_alloc(ctx.h, self.nbytes, ctypes.byref(p)))
        self.ptr = p.value
        ctx._buffers.add(self)

    def free(self):
        if self.ptr and self.ctx.h:
            _check(lib().mzk_device_free(self.ctx.h, self.ptr))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def upload(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        _check(lib().mzk_memcpy_h2d(self.ctx.h, self.ptr, arr.ctypes.data, arr.nbytes))

    def download(self, shape, dtype=np.uint64):
        out = np.empty(shape, dtype)
        assert out.nbytes <= self.nbytes
        _check(lib().mzk_memcpy_d2h(self.ctx.h, out.ctypes.data, self.ptr, out.nbytes))
        return out


class PermutationDesc(ctypes.Structure):
    """mzk_permutation_desc (include/mzk.h)."""
    _fields_ = [("n_cols", ctypes.c_uint32), ("values", ctypes.c_void_p), ("sigmas", ctypes.c_void_p),
                ("chunk_len", ctypes.c_uint32), ("blinding_factors", ctypes.c_uint32), ("blinds", ctypes.c_void_p),
                ("beta", ctypes.c_uint64 * 4), ("gamma", ctypes.c_uint64 * 4), ("z_out", ctypes.c_void_p)]


class LogupDesc(ctypes.Structure):
    """mzk_logup_desc (include/mzk.h)."""
    _fields_ = [("n_chunks", ctypes.c_uint32), ("chunk_cols", ctypes.c_void_p), ("inputs", ctypes.c_void_p),
                ("table", ctypes.c_void_p), ("selector", ctypes.c_void_p), ("multiplicities", ctypes.c_void_p),
                ("blinding_factors", ctypes.c_uint32), ("blinds", ctypes.c_void_p), ("beta", ctypes.c_uint64 * 4),
                ("helpers_out", ctypes.c_void_p), ("aggregator_out", ctypes.c_void_p)]


def _dptr(x):
    return x.ptr if hasattr(x, "ptr") else int(x)


def _ptrs(xs):
    return (ctypes.c_void_p * max(1, len(xs)))(*[_dptr(x) for x in xs])


class Context:
    """One device context (streams, scratch arena) on GPU `device`."""

    def __init__(self, device=0):
        h = _vp()
        _check(lib().mzk_ctx_create(device, ctypes.byref(h)))
        self.h = h.value
        self.device = device
        # objects that hold library handles tied to this context: closed
        # (servers first, then proving keys, domains, buffers) before the
        # context goes
        self._servers, self._keys = weakref.WeakSet(), weakref.WeakSet()
        self._domains, self._buffers = weakref.WeakSet(), weakref.WeakSet()

    def close(self):
        if getattr(self, "h", None):
            for group in (self._servers, self._keys, self._domains):
                for obj in list(group):
                    obj.close()
            for buf in list(self._buffers):
                try:
                    buf.free()
                except MzkError:
                    pass
            lib().mzk_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self):
        return int(lib().mzk_ctx_launch_count(self.h))

    @property
    def stream(self):
        return lib().mzk_ctx_stream(self.h)

    def synchronize(self):
        _check(lib().mzk_ctx_synchronize(self.h))

    def alloc(self, nbytes):
        return DeviceBuffer(self, nbytes)

    def set_profiling(self, on=True):
        _check(lib().mzk_ctx_set_profiling(self.h, 1 if on else 0))

    PHASES = ["histogram", "scan", "scatter", "accumulate", "fixup", "reduce"]

    def phase_stats(self):
        """{phase: (total_ms, count)} of the device time recorded while profiling."""
        ms = (ctypes.c_double * 16)()
        cnt = np.zeros(16, np.uint64)
        _check(lib().mzk_ctx_phase_stats(self.h, ms, _ptr(cnt), 16))
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(self.PHASES)}

    PROVE_PHASES = ["setup", "advice", "multiplicities", "products", "quotient", "evaluations", "f",
                    "q_evaluations", "pi", "msm"]

    def prove_phase_stats(self, reset=False):
        """create_proof wall time per phase (ms, summed) and the calls made."""
        ms = (ctypes.c_double * len(self.PROVE_PHASES))()
        calls = np.zeros(1, np.uint64)
        _check(lib().mzk_ctx_prove_phase_stats(self.h, ms, _ptr(calls), len(ms), 1 if reset else 0))
        return {name: ms[i] for i, name in enumerate(self.PROVE_PHASES)}, int(calls[0])

    def probe_imad_peak(self):
        """(IMAD/s, 12-limb Montgomery multiplications/s, {variant: IMAD/s}) of this GPU."""
        a, b = ctypes.c_double(), ctypes.c_double()
        v = (ctypes.c_double * 4)()
        _check(lib().mzk_probe_imad_peak(self.h, ctypes.byref(a), ctypes.byref(b), v))
        return a.value, b.value, {"mad_lo_hi": v[0], "mad_cc_chain": v[1], "mad_lo": v[2], "madd_regs": v[3]}

    def graph_stats(self):
        """(captures, replays) of the context's CUDA graphs."""
        c, r = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        _check(lib().mzk_ctx_graph_stats(self.h, _ptr(c), _ptr(r)))
        return int(c[0]), int(r[0])

    TUNE_MSM_WINDOW, TUNE_NTT_SPLIT = 0, 1

    def autotune(self, d_scalars=None, d_bases=None, msm_log_n=(), ntt_log_n=(), reps=2):
        """Time the MSM window widths (on the first 2^L device scalars/bases) and
        the NTT pass splits per log2 size and keep the fastest.  Returns
        {"msm": {L: (c, ms)}, "ntt": {L: (split, ms)}}."""
        ml = (_u32 * max(1, len(msm_log_n)))(*msm_log_n)
        nl = (_u32 * max(1, len(ntt_log_n)))(*ntt_log_n)
        mms = (ctypes.c_double * max(1, len(msm_log_n)))()
        nms = (ctypes.c_double * max(1, len(ntt_log_n)))()
        ds = 0 if d_scalars is None else (d_scalars.ptr if isinstance(d_scalars, DeviceBuffer) else int(d_scalars))
        db = 0 if d_bases is None else (d_bases.ptr if isinstance(d_bases, DeviceBuffer) else int(d_bases))
        _check(lib().mzk_autotune(self.h, ds or None, db or None, ml, len(msm_log_n), nl, len(ntt_log_n), int(reps),
                                  mms, nms))
        return {"msm": {int(L): (self.tuned(self.TUNE_MSM_WINDOW, L), mms[i]) for i, L in enumerate(msm_log_n)},
                "ntt": {int(L): (self.tuned(self.TUNE_NTT_SPLIT, L), nms[i]) for i, L in enumerate(ntt_log_n)}}

    def tuned(self, kind, log_n):
        v = _i32()
        _check(lib().mzk_autotune_get(self.h, int(kind), int(log_n), ctypes.byref(v)))
        return v.value

    def set_tuned(self, kind, log_n, value):
        _check(lib().mzk_autotune_set(self.h, int(kind), int(log_n), int(value)))

    def save_tuning(self, path):
        _check(lib().mzk_autotune_save(self.h, str(path).encode()))

    def load_tuning(self, path):
        _check(lib().mzk_autotune_load(self.h, str(path).encode()))

    def probe_fp_sqr_check(self, d_values, n):
        """Values among n device Fp elements whose dedicated square differs from a*a."""
        out = np.zeros(1, np.uint64)
        ptr = d_values.ptr if isinstance(d_values, DeviceBuffer) else int(d_values)
        _check(lib().mzk_probe_fp_sqr_check(self.h, ptr, int(n), _ptr(out)))
        return int(out[0])

    def probe_fp_inv_check(self, d_values, n):
        """Values among n device Fp elements whose binary-Euclid inverse differs
        from the Fermat power or fails a^-1 a = 1."""
        out = np.zeros(1, np.uint64)
        ptr = d_values.ptr if isinstance(d_values, DeviceBuffer) else int(d_values)
        _check(lib().mzk_probe_fp_inv_check(self.h, ptr, int(n), _ptr(out)))
        return int(out[0])

    def probe_batch_affine(self):
        """Batch-affine additions per second: {(batch, "fermat" | "binary"): rate}."""
        v = (ctypes.c_double * 8)()
        _check(lib().mzk_probe_batch_affine(self.h, v))
        return {(b, inv): v[4 * j + i] for j, inv in enumerate(("fermat", "binary"))
                for i, b in enumerate((16, 32, 64, 128))}

    def msm_last_shape(self):
        c, w, e = _i32(), _i32(), np.zeros(1, np.uint64)
        _check(lib().mzk_msm_last_shape(self.h, ctypes.byref(c), ctypes.byref(w), _ptr(e)))
        return c.value, w.value, int(e[0])

    # ---- MSM ----
    def set_msm_window(self, c):
        _check(lib().mzk_msm_set_window(self.h, int(c)))

    def msm_best(self, scalars, bases):
        """sum_i scalars[i] * bases[i] (host arrays) -> G1Projective (18,) uint64."""
        scalars = np.ascontiguousarray(scalars, np.uint64).reshape(-1, 4)
        bases = np.ascontiguousarray(bases, np.uint64).reshape(-1, 12)
        if scalars.shape[0] != bases.shape[0]:
            # the reference asserts equal lengths (curves/src/msm.rs:461)
            raise MzkError(1, "msm: coeffs and bases have different lengths")
        out = np.zeros(18, np.uint64)
        _check(lib().mzk_msm_g1(self.h, _ptr(scalars), _ptr(bases), scalars.shape[0], _ptr(out)))
        return out

    msm_specific = msm_best

    def msm_device(self, d_scalars, d_bases, n):
        """MSM over device-resident inputs (pointers or DeviceBuffers)."""
        out = np.zeros(18, np.uint64)
        _check(lib().mzk_msm_g1_device(self.h, _dptr(d_scalars), _dptr(d_bases), int(n), _ptr(out)))
        return out

    def msm_batch_device(self, d_bases, bases_len, items):
        """items: [(d_scalars, base_offset, n)] -> (len(items), 18) uint64 G1Projective."""
        arr = (MsmBatchItem * max(1, len(items)))()
        for i, (ds, off, n) in enumerate(items):
            arr[i].d_scalars = ds.ptr if isinstance(ds, DeviceBuffer) else int(ds)
            arr[i].base_offset, arr[i].n = int(off), int(n)
        db = d_bases.ptr if isinstance(d_bases, DeviceBuffer) else int(d_bases)
        out = np.zeros((max(1, len(items)), 18), np.uint64)
        _check(lib().mzk_msm_g1_batch_device(self.h, db, int(bases_len), ctypes.addressof(arr), len(items), _ptr(out)))
        return out[:len(items)]

    # ---- fixed-base window tables ----
    @staticmethod
    def msm_table_rows(c):
        return int(lib().mzk_msm_table_rows(int(c)))

    def msm_window_table(self, d_table, length, c, rows):
        """Fill rows 1 .. rows-1 of a window table whose row 0 (length points) is in place."""
        _check(lib().mzk_msm_window_table(self.h, _dptr(d_table), int(length), int(c), int(rows)))

    def msm_batch_table_device(self, d_table, length, c, rows, min_n, items):
        """msm_batch_device over a window table: items of at least min_n points use it."""
        arr = (MsmBatchItem * max(1, len(items)))()
        for i, (ds, off, n) in enumerate(items):
            arr[i].d_scalars = ds.ptr if isinstance(ds, DeviceBuffer) else int(ds)
            arr[i].base_offset, arr[i].n = int(off), int(n)
        out = np.zeros((max(1, len(items)), 18), np.uint64)
        _check(lib().mzk_msm_g1_batch_table_device(self.h, _dptr(d_table), int(length), int(c), int(rows), int(min_n),
                                                   ctypes.addressof(arr), len(items), _ptr(out)))
        return out[:len(items)]

    # ---- column scans ----
    def batch_invert_device(self, buf, n):
        """ff BatchInvert in place on n device Fr (zeros stay zero)."""
        _check(lib().mzk_batch_invert_device(self.h, _dptr(buf), int(n)))

    def eval_polynomial_device(self, buf, n, point):
        out = np.zeros(4, np.uint64)
        _check(lib().mzk_eval_polynomial_device(self.h, _dptr(buf), int(n), _ptr(np.ascontiguousarray(point, np.uint64)),
                                                _ptr(out)))
        return out

    def g1_compress_device(self, d_points, n, d_out):
        """G1Affine::to_compressed of n device points into n x 48 device bytes."""
        _check(lib().mzk_g1_compress_device(self.h, _dptr(d_points), int(n), _dptr(d_out)))

    def srs_write_processed(self, d_g, d_g_lagrange, n):
        """write_custom (Processed), G1 part: bytes k | g | g_lagrange (the caller adds G2)."""
        out = np.zeros(4 + 96 * int(n), np.uint8)
        _check(lib().mzk_srs_write_processed(self.h, _dptr(d_g), _dptr(d_g_lagrange), int(n),
                                             ctypes.c_void_p(out.ctypes.data), out.size))
        return out.tobytes()

    def g1_decompress_device(self, d_in, n, d_out, d_status=None, check_subgroup=True):
        """G1Affine::from_compressed of n device encodings; returns the invalid count."""
        bad = np.zeros(1, np.uint64)
        _check(lib().mzk_g1_decompress_device(self.h, _dptr(d_in), int(n), 1 if check_subgroup else 0, _dptr(d_out),
                                              None if d_status is None else _dptr(d_status), _ptr(bad)))
        return int(bad[0])

    def srs_read_processed(self, data, capacity, g=None, g_lagrange=None, g_lagrange_delta=None,
                           g_lagrange_double_delta=None):
        """ParamsKZG::read_custom (Processed) from host bytes into device buffers; returns k."""
        buf = np.frombuffer(bytes(data), np.uint8)
        k = _u32()
        opt = lambda b: None if b is None else _dptr(b)
        _check(lib().mzk_srs_read_processed(self.h, buf.ctypes.data, buf.size, int(capacity), ctypes.byref(k), opt(g),
                                            opt(g_lagrange), opt(g_lagrange_delta), opt(g_lagrange_double_delta)))
        return k.value

    def g1_suffix_sum_device(self, d_in, n, d_out):
        """suffix_sum (params.rs:47-57) of n device affine points."""
        _check(lib().mzk_g1_suffix_sum_device(self.h, _dptr(d_in), int(n), _dptr(d_out)))

    def poly_inner_product_device(self, polys, lens, scalars, out, out_len):
        """out = sum_p scalars[p] polys[p] (kzg/mod.rs:125-147)."""
        pp = _ptrs(polys)
        ll = (ctypes.c_size_t * max(1, len(lens)))(*[int(x) for x in lens])
        sc = np.ascontiguousarray(scalars, np.uint64).reshape(-1)
        _check(lib().mzk_poly_inner_product_device(self.h, ctypes.addressof(pp), ctypes.addressof(ll), len(polys),
                                                   _ptr(sc) if sc.size else None, _dptr(out), int(out_len)))

    def kate_division_device(self, a, n, b, q):
        _check(lib().mzk_kate_division_device(self.h, _dptr(a), int(n), _ptr(np.ascontiguousarray(b, np.uint64)),
                                              _dptr(q)))

    # ---- synthetic inputs ----
    def gen_rand_fr(self, seed, n, first=0, out=None):
        buf = out or self.alloc(n * 32)
        _check(lib().mzk_gen_rand_fr_device(self.h, seed, first, n, buf.ptr))
        return buf

    def gen_bases(self, seed, n, first=0, out=None):
        buf = out or self.alloc(n * 96)
        _check(lib().mzk_gen_bases_g1_device(self.h, seed, first, n, buf.ptr))
        return buf


class EvaluationDomain:
    """EvaluationDomain (proofs/src/poly/domain.rs:34) with its NTTs on the GPU.

    Methods take and return (len, 4) uint64 arrays of Fr in Montgomery form,
    like the reference's Polynomial values; inputs are not modified.
    """

    OPS = {"coeff_to_lagrange": 0, "lagrange_to_coeff": 1, "coeff_to_extended": 2,
           "extended_to_coeff": 3, "extended_to_lagrange": 4, "divide_by_vanishing_poly": 5}

    def __init__(self, ctx, j, k):
        self.ctx = ctx
        h = _vp()
        _check(lib().mzk_domain_create(ctx.h, j, k, ctypes.byref(h)))
        self.h = h.value
        ctx._domains.add(self)
        kk, ek = _u32(), _u32()
        _check(lib().mzk_domain_shape(self.h, ctypes.byref(kk), ctypes.byref(ek)))
        self.k, self.extended_k = kk.value, ek.value
        self.n, self.extended_len = 1 << self.k, 1 << self.extended_k
        self.quotient_poly_degree = j - 1

    def close(self):
        if getattr(self, "h", None):
            lib().mzk_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def constant(self, which, idx=0):
        out = np.zeros(4, np.uint64)
        _check(lib().mzk_domain_constant(self.h, which, idx, _ptr(out)))
        return out

    def _lens(self, op):
        n, en = self.n, self.extended_len
        return {0: (n, n), 1: (n, n), 2: (n, en), 3: (en, en), 4: (en, n), 5: (en, en)}[op]

    def _run(self, name, a):
        op = self.OPS[name]
        lin, lout = self._lens(op)
        a = np.ascontiguousarray(a, np.uint64).reshape(-1, 4)
        if a.shape[0] != lin:
            # the reference asserts the length (domain.rs:250, :286, :313, :339, :365)
            raise MzkError(1, f"{name}: expected {lin} elements, got {a.shape[0]}")
        out = np.zeros((lout, 4), np.uint64)
        _check(lib().mzk_domain_op(self.ctx.h, self.h, op, _ptr(a), _ptr(out)))
        return out

    def coeff_to_lagrange(self, a):
        return self._run("coeff_to_lagrange", a)

    def lagrange_to_coeff(self, a):
        return self._run("lagrange_to_coeff", a)

    def coeff_to_extended(self, a):
        return self._run("coeff_to_extended", a)

    def extended_to_coeff(self, a):
        return self._run("extended_to_coeff", a)

    def extended_to_lagrange(self, a):
        return self._run("extended_to_lagrange", a)

    def divide_by_vanishing_poly(self, a):
        return self._run("divide_by_vanishing_poly", a)

    def quotient_eval_device(self, desc, d_out, divide=True):
        """h(X) (divide) or nu(X) on the extended coset into d_out (device)."""
        do = d_out.ptr if isinstance(d_out, DeviceBuffer) else int(d_out)
        _check(lib().mzk_quotient_eval_device(self.ctx.h, self.h, ctypes.byref(desc), 1 if divide else 0, do))

    def compute_h_poly_device(self, desc, d_srs_g, srs_len, blinds, d_limbs_out=None):
        """compute_h_poly on the device: (qdeg, 18) limb commitments."""
        qdeg = self.quotient_poly_degree
        blinds = np.ascontiguousarray(blinds, np.uint64).reshape(-1, 4)
        assert blinds.shape[0] == qdeg - 1
        out = np.zeros((qdeg, 18), np.uint64)
        dg = d_srs_g.ptr if isinstance(d_srs_g, DeviceBuffer) else int(d_srs_g)
        dl = 0 if d_limbs_out is None else (d_limbs_out.ptr if isinstance(d_limbs_out, DeviceBuffer) else int(d_limbs_out))
        _check(lib().mzk_compute_h_poly_device(self.ctx.h, self.h, ctypes.byref(desc), dg, int(srs_len),
                                               _ptr(blinds), _ptr(out), dl or None))
        return out

    def prove_core_device(self, pk_desc, jobs, per_call=False, graphs=None):
        """Device part of create_proof for a list of ProofJob: (len, 11, 18) commitments.
        per_call: the plain form (every MSM its own call, the NTT sequence launched
        kernel by kernel) instead of batched MSMs and a replayed CUDA graph;
        graphs: override the graph choice."""
        arr = (ProofJob * max(1, len(jobs)))(*jobs)
        out = np.zeros((max(1, len(jobs)), len(PROOF_CORE_COMMITMENTS), 18), np.uint64)
        flags = PROVE_PLAIN if per_call else 0
        if graphs is not None:
            flags = (flags & ~PROVE_NO_GRAPHS) | (0 if graphs else PROVE_NO_GRAPHS)
        _check(lib().mzk_prove_core_device(self.ctx.h, self.h, ctypes.byref(pk_desc), ctypes.addressof(arr),
                                           len(jobs), flags, _ptr(out)))
        return out[:len(jobs)]

    def srs_setup_device(self, s, g=None, g_lagrange=None, g_lagrange_delta=None, g_lagrange_double_delta=None):
        """G1 part of ParamsKZG::unsafe_setup (params.rs:160-209) for secret s
        into device buffers of n affine points (any may be None)."""
        opt = lambda b: None if b is None else _dptr(b)
        _check(lib().mzk_srs_setup_device(self.ctx.h, self.h, _ptr(np.ascontiguousarray(s, np.uint64)), opt(g),
                                          opt(g_lagrange), opt(g_lagrange_delta), opt(g_lagrange_double_delta)))

    def g1_to_lagrange_device(self, g, out):
        """g_to_lagrange (utils/arithmetic.rs:34-54) of the first n device points of g."""
        _check(lib().mzk_g1_to_lagrange_device(self.ctx.h, self.h, _dptr(g), _dptr(out)))

    def srs_downsize_device(self, g, g_lagrange=None, g_lagrange_delta=None, g_lagrange_double_delta=None):
        """ParamsKZG::downsize (params.rs:96-107) to this domain's k."""
        opt = lambda b: None if b is None else _dptr(b)
        _check(lib().mzk_srs_downsize_device(self.ctx.h, self.h, _dptr(g), opt(g_lagrange), opt(g_lagrange_delta),
                                             opt(g_lagrange_double_delta)))

    def permutation_z_device(self, values, sigmas, chunk_len, blinding_factors, blinds, beta, gamma, z_out):
        """z of every permutation set (permutation/prover.rs:81-255) into the
        device buffers z_out; blinds: host (n_sets, blinding_factors, 4)."""
        d = PermutationDesc()
        vp, sp, zp = _ptrs(values), _ptrs(sigmas), _ptrs(z_out)
        bl = np.ascontiguousarray(blinds, np.uint64).reshape(-1)
        d.n_cols, d.values, d.sigmas = len(values), ctypes.addressof(vp), ctypes.addressof(sp)
        d.chunk_len, d.blinding_factors = chunk_len, blinding_factors
        d.blinds = bl.ctypes.data if bl.size else None
        d.beta[:] = [int(v) for v in beta]
        d.gamma[:] = [int(v) for v in gamma]
        d.z_out = ctypes.addressof(zp)
        _check(lib().mzk_permutation_z_device(self.ctx.h, self.h, ctypes.byref(d)))

    def logup_device(self, chunks, table, selector, multiplicities, blinding_factors, blinds, beta, helpers_out,
                     aggregator_out):
        """helpers and aggregator of one logup argument (logup/prover.rs:195-300);
        chunks: list of lists of device columns; blinds: host (blinding_factors, 4)."""
        d = LogupDesc()
        cols = [c for ch in chunks for c in ch]
        counts = (ctypes.c_uint32 * max(1, len(chunks)))(*[len(ch) for ch in chunks])
        ip, hp = _ptrs(cols), _ptrs(helpers_out)
        bl = np.ascontiguousarray(blinds, np.uint64).reshape(-1)
        d.n_chunks, d.chunk_cols, d.inputs = len(chunks), ctypes.addressof(counts), ctypes.addressof(ip)
        d.table, d.selector, d.multiplicities = _dptr(table), _dptr(selector), _dptr(multiplicities)
        d.blinding_factors = blinding_factors
        d.blinds = bl.ctypes.data if bl.size else None
        d.beta[:] = [int(v) for v in beta]
        d.helpers_out, d.aggregator_out = ctypes.addressof(hp), _dptr(aggregator_out)
        _check(lib().mzk_logup_device(self.ctx.h, self.h, ctypes.byref(d)))

    def op_device(self, name, d_in, d_out):
        """Operation on device buffers (pointers or DeviceBuffers)."""
        di = d_in.ptr if isinstance(d_in, DeviceBuffer) else int(d_in)
        do = d_out.ptr if isinstance(d_out, DeviceBuffer) else int(d_out)
        _check(lib().mzk_domain_op_device(self.ctx.h, self.h, self.OPS[name], di, do))

    def op_batch_device(self, name, d_ins, d_outs):
        """The same operation on many device buffers, launched together."""
        ptr = lambda b: b.ptr if isinstance(b, DeviceBuffer) else int(b)
        ins = (ctypes.c_void_p * max(1, len(d_ins)))(*[ptr(b) for b in d_ins])
        outs = (ctypes.c_void_p * max(1, len(d_outs)))(*[ptr(b) for b in d_outs])
        if len(d_ins) != len(d_outs):
            raise MzkError(1, "domain op batch: inputs and outputs differ in number")
        _check(lib().mzk_domain_op_batch_device(self.ctx.h, self.h, self.OPS[name], ins, outs, len(d_ins)))


class ProvingServer:
    """Proving service with continuous batching over create_proof (mzk_server_*)."""

    def __init__(self, ctx, max_batch=16, lanes=2, mem_budget_bytes=0, per_call=False, flags=0, max_wave_rows=0):
        self.ctx = ctx
        h = _vp()
        fl = flags | (PROVE_PLAIN if per_call else 0)
        _check(lib().mzk_server_create(ctx.h, int(max_batch), int(lanes), int(mem_budget_bytes), fl,
                                       ctypes.byref(h)))
        self.h = h.value
        if max_wave_rows:
            _check(lib().mzk_server_set_wave_rows(self.h, int(max_wave_rows)))
        ctx._servers.add(self)
        self._held = {}

    def submit(self, key, advice, blinds, instance=None):
        """Queue one proof of `key` (a PlonkKey) over the advice columns (host
        arrays or DeviceBuffers), the blinding values and the instance columns'
        values; wait() returns its transcript."""
        req, keep, out = _proof_request(key, advice, blinds, instance)
        t = np.zeros(1, np.uint64)
        _check(lib().mzk_server_submit(self.h, ctypes.byref(req), _ptr(t)))
        self._held[int(t[0])] = (req, keep, out)
        return int(t[0])

    def wait(self, ticket):
        lat = ctypes.c_double()
        try:
            _check(lib().mzk_server_wait(self.h, ticket, ctypes.byref(lat)))
        finally:
            held = self._held.pop(int(ticket), None)
        return bytes(held[2]), lat.value

    def stats(self):
        w, p = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
        busy = ctypes.c_double()
        _check(lib().mzk_server_stats(self.h, _ptr(w), _ptr(p), ctypes.byref(busy)))
        return {"waves": int(w[0]), "proofs": int(p[0]), "busy_ms": busy.value}

    def close(self):
        if getattr(self, "h", None):
            lib().mzk_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Query(ctypes.Structure):
    """mzk_query (include/mzk.h)."""
    _fields_ = [("column", ctypes.c_uint32), ("rotation", ctypes.c_int32)]


class LookupShape(ctypes.Structure):
    """mzk_lookup_shape (include/mzk.h)."""
    _fields_ = [("input_advice", ctypes.c_uint32), ("table_fixed", ctypes.c_uint32),
                ("selector_fixed", ctypes.c_int32)]


class CircuitDesc(ctypes.Structure):
    """mzk_circuit_desc (include/mzk.h)."""
    _fields_ = [("degree", ctypes.c_uint32), ("blinding_factors", ctypes.c_uint32),
                ("n_advice", ctypes.c_uint32), ("n_fixed", ctypes.c_uint32),
                ("advice_queries", ctypes.c_void_p), ("n_advice_queries", ctypes.c_uint32),
                ("fixed_queries", ctypes.c_void_p), ("n_fixed_queries", ctypes.c_uint32),
                ("gate_fixed", ctypes.c_uint32 * 5), ("gate_advice", ctypes.c_uint32 * 3),
                ("gates", ctypes.c_void_p),
                ("n_perm_cols", ctypes.c_uint32), ("perm_col_kind", ctypes.c_void_p),
                ("perm_col_index", ctypes.c_void_p), ("n_lookups", ctypes.c_uint32), ("lookups", ctypes.c_void_p),
                ("n_instance", ctypes.c_uint32), ("instance_queries", ctypes.c_void_p),
                ("n_instance_queries", ctypes.c_uint32), ("n_trash", ctypes.c_uint32), ("trash", ctypes.c_void_p),
                ("n_gate_polys", ctypes.c_uint32), ("gate_poly_values", ctypes.c_void_p),
                ("gate_poly_selector", ctypes.c_void_p), ("lookup_tuples", ctypes.c_void_p),
                ("lookup_input_programs", ctypes.c_void_p)]


class LookupTuple(ctypes.Structure):
    """mzk_lookup_tuple (include/mzk.h)."""
    _fields_ = [("width", ctypes.c_uint32), ("n_inputs", ctypes.c_uint32),
                ("input_advice", (ctypes.c_uint32 * 4) * 8), ("table_fixed", ctypes.c_uint32 * 4)]


def lookup_columns(lk):
    """(input tuples, table tuple) of a lookup dict: "input" a column or a
    tuple (list) of columns, or "inputs" a list of such tuples (parallel
    inputs); "table" a column or a tuple.  An input element is an advice
    column or an expression: a flattened program (dict with the FlatGraph
    fields, or a FlatGraph) whose result_idx holds its value."""
    one = lambda v: list(v) if isinstance(v, (list, tuple)) else [v]
    ins = [one(t) for t in lk["inputs"]] if "inputs" in lk else [one(lk["input"])]
    return ins, one(lk["table"])


def _program(g):
    """A FlatGraph from a program dict (a FlatGraph is returned as it is)."""
    if isinstance(g, FlatGraph):
        return g
    return build_flat_graph(g["constants"], g["rotations"], g["reads"], g["ops"], g["values_len"], g["beta_idx"],
                            g["theta_idx"], g["trash_challenge_idx"], g["y_idx"], g["previous_value_idx"],
                            g["result_idx"])


def _column_program(col):
    """The program of a plain lookup input: advice column `col` at rotation 0."""
    return build_flat_graph(np.zeros((0, 4), np.uint64), [0], [(1, col, 0, 5)], [], 6, 0, 1, 2, 3, 4, 5)


class SrsDesc(ctypes.Structure):
    """mzk_srs_desc (include/mzk.h)."""
    _fields_ = [("srs", ctypes.c_void_p), ("srs_len", ctypes.c_uint64), ("off_g", ctypes.c_uint64),
                ("off_lagrange", ctypes.c_uint64), ("off_lagrange_delta", ctypes.c_uint64),
                ("off_lagrange_double_delta", ctypes.c_uint64), ("table_c", ctypes.c_int32),
                ("table_rows", ctypes.c_uint32), ("table_min_n", ctypes.c_uint64)]


def prover_table_width(k):
    """Width c of the fixed-base window table that made create_proof fastest
    at 2^k rows on a B200 (config-3 circuit, 8 proofs per call; k = 18: no
    table 33.0 ms per proof, c = 15 / 16 / 17 / 18: 28.4 / 27.5 / 27.9 / 29.2
    ms; k = 20, 2 per call: no table 121.7, c = 17 / 18 / 19 / 20: 92.5 / 94.9
    / 99.6 / 113.8 ms; 16 per call, k = 14: c = 11 / 12 / 13 / 14 / 16: 52.9 /
    52.4 / 52.0 / 52.5 / 56.6 ms per call, k = 16: c = 14 / 15 / 16 / 17 / 18:
    124.1 / 123.6 / 122.7 / 131.0 / 146.4 ms).  Each MSM of
    2^k points then adds ceil(255 / c) + 1 table rows of points into one window
    of 2^(c-1) buckets: wider tables mean fewer entries per point but more
    buckets to reduce, and the best width grows with the point count."""
    if k <= 14:
        return 12
    if k <= 18:
        return 16
    if k <= 20:
        return 17
    return 20


class ProofRequest(ctypes.Structure):
    """mzk_proof_request (include/mzk.h)."""
    _fields_ = [("key", ctypes.c_void_p), ("advice", ctypes.c_void_p), ("advice_on_device", ctypes.c_int),
                ("blinds", ctypes.c_void_p), ("proof_out", ctypes.c_void_p), ("instance", ctypes.c_void_p),
                ("instance_len", ctypes.c_void_p)]




class Transcript:
    """CircuitTranscript<Blake2bState> (proofs/src/transcript/mod.rs:83-150)
    as the library implements it: common / write of Fr (4 u64 Montgomery) and
    G1 points (18 u64, z = 1 or all zero), squeeze_challenge, finalize."""

    def __init__(self):
        h = _vp()
        _check(lib().mzk_transcript_create(ctypes.byref(h)))
        self.h = h.value

    def close(self):
        if getattr(self, "h", None):
            lib().mzk_transcript_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def common_fr(self, v):
        _check(lib().mzk_transcript_common_fr(self.h, _ptr(np.ascontiguousarray(v, np.uint64))))

    def write_fr(self, v):
        _check(lib().mzk_transcript_write_fr(self.h, _ptr(np.ascontiguousarray(v, np.uint64))))

    def write_point(self, p18):
        _check(lib().mzk_transcript_write_point(self.h, _ptr(np.ascontiguousarray(p18, np.uint64))))

    def squeeze_challenge(self):
        out = np.zeros(4, np.uint64)
        _check(lib().mzk_transcript_squeeze(self.h, _ptr(out)))
        return out

    def finalize(self):
        n = _sz()
        _check(lib().mzk_transcript_proof(self.h, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_uint8 * max(1, n.value))()
        _check(lib().mzk_transcript_proof(self.h, buf, n.value, ctypes.byref(n)))
        return bytes(buf[:n.value])


def vk_transcript_repr(k, fixed_coms, perm_coms, pinned=b""):
    """VerifyingKey::from_parts's transcript_repr (proofs/src/plonk/mod.rs:227-284)
    over commitments in the 18-u64 point layout."""
    f = np.ascontiguousarray(fixed_coms, np.uint64).reshape(-1, 18)
    pm = np.ascontiguousarray(perm_coms, np.uint64).reshape(-1, 18)
    out = np.zeros(4, np.uint64)
    pin = ctypes.create_string_buffer(bytes(pinned), max(1, len(pinned)))
    _check(lib().mzk_vk_transcript_repr(k, f.ctypes.data if f.size else None, f.shape[0],
                                        pm.ctypes.data if pm.size else None, pm.shape[0], pin, len(pinned),
                                        _ptr(out)))
    return out


class PlonkKey:
    """keygen_vk + keygen_pk (proofs/src/plonk/keygen.rs:227-359) on the device.

    circuit: dict with degree, blinding_factors, n_advice, n_fixed,
    advice_queries / fixed_queries [(column, rotation)], gate_fixed (5),
    gate_advice (3), perm_cols [(kind 0 advice | 1 fixed | 2 instance,
    column)], lookups [{"input", "table", "selector" (None: constant one)}]
    (input and table a column or a list of up to four columns, compressed with
    theta; or "inputs", a list of up to eight such input tuples; an input
    element may be an expression, a flattened program dict),
    n_instance and instance_queries [(column, rotation)] (optional),
    trashcans [{"program": flattened program, "selector": fixed column}]
    (optional), gate_polys [(value slot, simple selector fixed column or
    None)] per gate polynomial (optional, with "gates").  fixed_values:
    host (n, 4) arrays; mapping: (n_perm_cols, n, 2) uint32 or None; srs:
    an SrsDesc.  The domain and the SRS buffer must outlive the key."""

    def __init__(self, ctx, domain, circuit, srs, fixed_values=None, mapping=None, pinned=b"", perm_values=None,
                 pk_bytes=None, pk_format=SERDE_PROCESSED):
        """fixed_values (+ mapping or perm_values): keygen; pk_bytes: a key
        read from a ProvingKey file (ProvingKey::read) in pk_format."""
        self.ctx, self.domain, self.circuit = ctx, domain, circuit
        keep = []

        def arr(ctype, items):
            a = (ctype * max(1, len(items)))(*items)
            keep.append(a)
            return ctypes.addressof(a)

        cs = CircuitDesc()
        cs.degree, cs.blinding_factors = circuit["degree"], circuit["blinding_factors"]
        cs.n_advice, cs.n_fixed = circuit["n_advice"], circuit["n_fixed"]
        cs.advice_queries = arr(Query, [Query(c, r) for c, r in circuit["advice_queries"]])
        cs.n_advice_queries = len(circuit["advice_queries"])
        cs.fixed_queries = arr(Query, [Query(c, r) for c, r in circuit["fixed_queries"]])
        cs.n_fixed_queries = len(circuit["fixed_queries"])
        cs.gate_fixed[:] = circuit.get("gate_fixed", [0] * 5)
        cs.gate_advice[:] = circuit.get("gate_advice", [0] * 3)
        if circuit.get("gates") is not None:
            g = circuit["gates"]
            fg = g if isinstance(g, FlatGraph) else build_flat_graph(
                g["constants"], g["rotations"], g["reads"], g["ops"], g["values_len"], g["beta_idx"],
                g["theta_idx"], g["trash_challenge_idx"], g["y_idx"], g["previous_value_idx"], g["result_idx"])
            keep.append(fg)
            cs.gates = ctypes.addressof(fg)
        pc = circuit["perm_cols"]
        cs.n_perm_cols = len(pc)
        cs.perm_col_kind = arr(ctypes.c_uint32, [kd for kd, _ in pc])
        cs.perm_col_index = arr(ctypes.c_uint32, [ci for _, ci in pc])
        lks = circuit["lookups"]
        cs.n_lookups = len(lks)
        shapes = [lookup_columns(lk) for lk in lks]
        col = lambda el: el if isinstance(el, (int, np.integer)) else 0   # a program's slot in the column fields
        cs.lookups = arr(LookupShape, [LookupShape(col(ins[0][0]), tab[0], -1 if lk["selector"] is None else lk["selector"])
                                       for lk, (ins, tab) in zip(lks, shapes)])
        if any(len(ins) > 1 or len(tab) > 1 for ins, tab in shapes):
            tuples = []
            for ins, tab in shapes:
                if not 1 <= len(tab) <= 4 or not 1 <= len(ins) <= 8 or any(len(t) != len(tab) for t in ins):
                    raise MzkError(1, "keygen: a lookup takes 1..8 input tuples of the table tuple's 1..4 columns")
                t = LookupTuple()
                t.width, t.n_inputs = len(tab), len(ins)
                for i, tup in enumerate(ins):
                    t.input_advice[i][:len(tup)] = [col(el) for el in tup]
                t.table_fixed[:len(tab)] = tab
                tuples.append(t)
            cs.lookup_tuples = arr(LookupTuple, tuples)
        elements = [el for ins, _ in shapes for tup in ins for el in tup]
        if any(not isinstance(el, (int, np.integer)) for el in elements):
            progs = [_column_program(int(el)) if isinstance(el, (int, np.integer)) else _program(el)
                     for el in elements]
            keep.extend(progs)
            cs.lookup_input_programs = arr(FlatGraph, progs)
        cs.n_instance = circuit.get("n_instance", 0)
        iq = circuit.get("instance_queries", [])
        cs.instance_queries = arr(Query, [Query(c, r) for c, r in iq])
        cs.n_instance_queries = len(iq)
        tcs = circuit.get("trashcans", [])
        if tcs:
            targs = (TrashArg * len(tcs))()
            for i, tc in enumerate(tcs):
                g = tc["program"]
                fg = g if isinstance(g, FlatGraph) else build_flat_graph(
                    g["constants"], g["rotations"], g["reads"], g["ops"], g["values_len"], g["beta_idx"],
                    g["theta_idx"], g["trash_challenge_idx"], g["y_idx"], g["previous_value_idx"], g["result_idx"])
                keep.append(fg)
                targs[i].program = fg
                targs[i].selector_fixed = tc["selector"]
            keep.append(targs)
            cs.n_trash, cs.trash = len(tcs), ctypes.addressof(targs)
        gpolys = circuit.get("gate_polys", [])
        if gpolys:
            cs.n_gate_polys = len(gpolys)
            cs.gate_poly_values = arr(ctypes.c_uint32, [slot for slot, _ in gpolys])
            cs.gate_poly_selector = arr(ctypes.c_int32, [-1 if sel is None else sel for _, sel in gpolys])
        pin = ctypes.create_string_buffer(bytes(pinned), max(1, len(pinned)))
        h = _vp()
        if pk_bytes is not None:
            data = bytes(pk_bytes)
            _check(lib().mzk_pk_read(ctx.h, domain.h, ctypes.byref(cs), ctypes.byref(srs), data, len(data), pk_format,
                                     pin, len(pinned), ctypes.byref(h)))
            self._finish(h)
            return
        cols = [np.ascontiguousarray(v, np.uint64) for v in fixed_values]
        if any(c.shape != (domain.n, 4) for c in cols):
            raise MzkError(1, "keygen: every fixed column needs n Fr values")
        fptrs = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        mp = None if mapping is None else np.ascontiguousarray(mapping, np.uint32)
        if perm_values is not None:
            pv = [np.ascontiguousarray(v, np.uint64) for v in perm_values]
            keep.append(pv)
            pptrs = (ctypes.c_void_p * max(1, len(pv)))(*[v.ctypes.data for v in pv])
            _check(lib().mzk_keygen_from_values(ctx.h, domain.h, ctypes.byref(cs), ctypes.byref(srs), fptrs, pptrs,
                                                pin, len(pinned), ctypes.byref(h)))
        else:
            _check(lib().mzk_keygen(ctx.h, domain.h, ctypes.byref(cs), ctypes.byref(srs), fptrs,
                                    None if mp is None else mp.ctypes.data, pin, len(pinned), ctypes.byref(h)))
        self._finish(h)

    def _finish(self, h):
        ctx, circuit = self.ctx, self.circuit
        pc = circuit["perm_cols"]
        self.h = h.value
        ctx._keys.add(self)
        repr_, plen, nbl = np.zeros(4, np.uint64), _sz(), _sz()
        _check(lib().mzk_plonk_key_info(self.h, _ptr(repr_), ctypes.byref(plen), ctypes.byref(nbl)))
        self.repr, self.proof_len, self.n_blinds = repr_, plen.value, nbl.value
        self.fixed_coms = np.zeros((circuit["n_fixed"], 18), np.uint64)
        self.perm_coms = np.zeros((len(pc), 18), np.uint64)
        _check(lib().mzk_plonk_key_commitments(self.h, self.fixed_coms.ctypes.data, self.perm_coms.ctypes.data))

    def vk_bytes(self, fmt=SERDE_PROCESSED):
        """VerifyingKey::write (plonk/mod.rs:95-113) of this key."""
        n = _sz()
        _check(lib().mzk_vk_write(self.h, fmt, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_uint8 * max(1, n.value))()
        _check(lib().mzk_vk_write(self.h, fmt, buf, n.value, ctypes.byref(n)))
        return bytes(buf[:n.value])

    def pk_bytes(self, fmt=SERDE_PROCESSED):
        """ProvingKey::write (plonk/mod.rs:391-399) of this key."""
        n = _sz()
        _check(lib().mzk_pk_write(self.ctx.h, self.h, fmt, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_uint8 * max(1, n.value))()
        _check(lib().mzk_pk_write(self.ctx.h, self.h, fmt, buf, n.value, ctypes.byref(n)))
        return bytes(buf[:n.value])

    def transcript_layout(self):
        """The MZK_TR_* operation codes of one proof, in order."""
        n = _sz()
        _check(lib().mzk_plonk_key_transcript_layout(self.h, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_uint8 * max(1, n.value))()
        _check(lib().mzk_plonk_key_transcript_layout(self.h, buf, n.value, ctypes.byref(n)))
        return bytes(buf[:n.value])

    def close(self):
        if getattr(self, "h", None):
            lib().mzk_plonk_key_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DevicePtr:
    """A device address inside a larger DeviceBuffer (kept alive with it)."""

    def __init__(self, buf, offset_bytes=0):
        self.buf, self.ptr = buf, _dptr(buf) + int(offset_bytes)


def _proof_request(key, advice, blinds, instance=None):
    """A ProofRequest with the buffers it points to (kept alive by the caller).
    instance: one host array of Fr values (m, 4) per instance column of the key."""
    on_dev = isinstance(advice[0], (DeviceBuffer, DevicePtr))
    keep = [key]
    if on_dev:
        ptrs = (ctypes.c_void_p * len(advice))(*[a.ptr for a in advice])
        keep.extend(advice)
    else:
        cols = [np.ascontiguousarray(a, np.uint64) for a in advice]
        keep.extend(cols)
        ptrs = (ctypes.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    if len(advice) != key.circuit["n_advice"]:
        raise MzkError(1, f"create_proof: {key.circuit['n_advice']} advice columns expected, got {len(advice)}")
    bl = np.ascontiguousarray(blinds, np.uint64).reshape(-1, 4)
    if bl.shape[0] != key.n_blinds:
        raise MzkError(1, f"create_proof: {key.n_blinds} blinding values expected, got {bl.shape[0]}")
    out = (ctypes.c_uint8 * key.proof_len)()
    keep.extend([ptrs, bl])
    req = ProofRequest()
    req.key, req.advice, req.advice_on_device = key.h, ctypes.addressof(ptrs), 1 if on_dev else 0
    req.blinds, req.proof_out = bl.ctypes.data, ctypes.addressof(out)
    ni = key.circuit.get("n_instance", 0)
    inst = list(instance) if instance is not None else []
    if len(inst) != ni:
        raise MzkError(1, f"create_proof: {ni} instance columns expected, got {len(inst)}")
    if ni:
        icols = [np.ascontiguousarray(v, np.uint64).reshape(-1, 4) for v in inst]
        iptrs = (ctypes.c_void_p * ni)(*[c.ctypes.data if c.shape[0] else None for c in icols])
        ilen = np.array([c.shape[0] for c in icols], np.uint64)
        keep.extend([icols, iptrs, ilen])
        req.instance, req.instance_len = ctypes.addressof(iptrs), ilen.ctypes.data
    return req, keep, out


def create_proofs(ctx, jobs, flags=0):
    """create_proof (proofs/src/plonk/prover.rs:432-473) for many proofs in
    one call.  jobs: [(PlonkKey, advice columns, blinds[, instance columns])]
    where the advice columns are host (n, 4) arrays or DeviceBuffers, blinds an
    (n_blinds, 4) host array in the reference's draw order (include/mzk.h) and
    the instance columns host arrays of their values.  Returns the proofs as
    bytes."""
    reqs = (ProofRequest * max(1, len(jobs)))()
    keep, outs = [], []
    for i, job in enumerate(jobs):
        req, kp, out = _proof_request(*job)
        reqs[i] = req
        keep.append(kp)
        outs.append(out)
    _check(lib().mzk_create_proofs(ctx.h, reqs, len(jobs), flags))
    return [bytes(o) for o in outs]


CONFIG3_DEGREE = 5


def config3_circuit(k):
    """The single-proof configuration's constraint system (standard gate over
    advice a, b, c and fixed q_l, q_r, q_m, q_o, q_c; permutation over a, b, c;
    one lookup of a into the fixed table column 5 with the fixed selector 6;
    degree 5, set_minimum_degree(5) of proofs/benches/plonk.rs:191) as the
    dict PlonkKey takes; blinding_factors as ConstraintSystem::blinding_factors
    (plonk/circuit.rs:2203-2245) gives it: max(3, 1) + 1 helper + 3 = 7."""
    return {"k": k, "degree": CONFIG3_DEGREE, "blinding_factors": 7, "n_advice": 3, "n_fixed": 7,
            "advice_queries": [(0, 0), (1, 0), (2, 0)], "fixed_queries": [(i, 0) for i in range(7)],
            "gate_fixed": [0, 1, 2, 3, 4], "gate_advice": [0, 1, 2],
            "perm_cols": [(0, 0), (0, 1), (0, 2)], "lookups": [{"input": 0, "table": 5, "selector": 6}]}


def copy_cycles(n, usable, seed, fraction=0.10):
    """Seeded copy cycles of 2 to 4 cells over `fraction` of the a and b cells
    of the usable rows: (mapping (3, n, 2) uint32, each cell's (column, row)
    successor in its cycle, identity elsewhere, as Assembly::mapping gives
    build_pk; cycle_of (2n,) uint32, the cycle of each a then b cell,
    0xffffffff outside cycles)."""
    rng = np.random.default_rng(seed)
    m = int(fraction * 2 * usable)
    cells = rng.permutation(2 * usable)[:m]
    lens = rng.integers(2, 5, size=m // 2 + 1)
    ends = np.cumsum(lens)
    lens = lens[ends <= m]
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    total = int(lens.sum())
    cyc = np.repeat(np.arange(len(lens)), lens)
    first = np.repeat(starts, lens)
    pos = np.arange(total) - first
    nxt = cells[first + (pos + 1) % np.repeat(lens, lens)]
    cur = cells[:total]
    mapping = np.zeros((3, n, 2), np.uint32)
    mapping[:, :, 0] = np.arange(3, dtype=np.uint32)[:, None]
    mapping[:, :, 1] = np.arange(n, dtype=np.uint32)[None, :]
    mapping[cur // usable, cur % usable, 0] = nxt // usable
    mapping[cur // usable, cur % usable, 1] = nxt % usable
    cycle_of = np.full(2 * n, 0xFFFFFFFF, np.uint32)
    cycle_of[(cur // usable) * n + cur % usable] = cyc
    return mapping, cycle_of


class Config3Instance:
    """A seeded instance of the single-proof configuration's circuit on the
    device (benchmarks): the fixed columns (mzk_gen_config3_fixed_device), copy
    cycles, the proving key over `srs` (an SrsDesc), and fresh satisfying
    witnesses per request (mzk_gen_config3_witness_device)."""

    def __init__(self, ctx, domain, srs, seed, table_rows=1 << 16, pinned=b"config-3 circuit"):
        k = domain.k
        self.ctx, self.domain, self.k, self.n = ctx, domain, k, domain.n
        self.circuit = config3_circuit(k)
        bf = self.bf = self.circuit["blinding_factors"]
        n, self.table_rows = domain.n, table_rows
        self.fixed = ctx.alloc(7 * n * 32)
        _check(lib().mzk_gen_config3_fixed_device(ctx.h, k, bf, table_rows, seed, self.fixed.ptr))
        host = self.fixed.download((7, n, 4))
        self.inv_qo = ctx.alloc(n * 32)
        self.inv_qo.upload(host[3])
        ctx.batch_invert_device(self.inv_qo, n)
        mapping, cycle_of = copy_cycles(n, n - bf - 1, seed)
        self.cycle_of = ctx.alloc(cycle_of.nbytes)
        self.cycle_of.upload(cycle_of)
        self.key = PlonkKey(ctx, domain, self.circuit, srs, [host[i] for i in range(7)], mapping, pinned)

    def witness(self, seed):
        """A fresh witness: a DeviceBuffer of a | b | c and the three column pointers."""
        buf = self.ctx.alloc(3 * self.n * 32)
        _check(lib().mzk_gen_config3_witness_device(self.ctx.h, self.k, self.bf, self.table_rows, seed,
                                                    self.fixed.ptr, self.inv_qo.ptr, self.cycle_of.ptr, buf.ptr))
        return [DevicePtr(buf, i * self.n * 32) for i in range(3)]

    def blinds(self, seed):
        """n_blinds uniform Fr (Montgomery) from a seeded stream."""
        out = np.empty((self.key.n_blinds, 4), np.uint64)
        buf = self.ctx.alloc(out.nbytes)
        self.ctx.gen_rand_fr(seed, self.key.n_blinds, out=buf)
        return buf.download(out.shape)


def g1_sum(points):
    """Sum of points in the (count, 18) MSM result layout, normalised (host)."""
    p = np.ascontiguousarray(points, np.uint64).reshape(-1, 18)
    out = np.zeros(18, np.uint64)
    _check(lib().mzk_g1_sum_host(_ptr(p) if p.size else None, p.shape[0], _ptr(out)))
    return out


def point_split_slice(n, rank, world):
    """The contiguous point range [begin, end) rank `rank` of `world` takes."""
    return n * rank // world, n * (rank + 1) // world


def msm_point_split(msm_slice, n, rank, world, all_gather):
    """One MSM of n points split across `world` ranks: this rank computes the
    partial sum of its slice (msm_slice(begin, end) -> 18-u64 point, e.g. an
    MSM over device-resident scalars and bases), one all-gather exchanges the
    144-byte partials (all_gather(array) -> list of the ranks' arrays, e.g.
    torch.distributed over NCCL or gloo), and every rank adds them on the
    host.  Same point as the MSM over all n points."""
    begin, end = point_split_slice(n, rank, world)
    part = np.ascontiguousarray(msm_slice(begin, end), np.uint64).reshape(18)
    parts = all_gather(part)
    return g1_sum(np.stack(parts))


def msm_pick_window(n):
    return int(lib().mzk_msm_pick_window(n))


def affine(jac18):
    """G1Projective with z in {0, 1} -> G1Affine (12,) layout."""
    return np.ascontiguousarray(jac18[:12])
