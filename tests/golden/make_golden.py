#!/usr/bin/env python3
"""Extract the reference's known-answer vectors into tests/golden/reference_kats.json.

Reads the midnight-zk sources AS TEXT (nothing of the reference is executed:
it is Rust, and no Rust toolchain exists in this image).  Every vector records
the file and line it came from.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/midnight-zk

(or set MZK_REFERENCE to the reference tree).
The generated JSON is committed; the tests only read the JSON, so they run
where the reference tree is absent.
"""
import json
import os
import re
import sys
from pathlib import Path

if len(sys.argv) > 1:
    REF = Path(sys.argv[1])
elif os.environ.get("MZK_REFERENCE"):
    REF = Path(os.environ["MZK_REFERENCE"])
else:
    sys.exit("usage: make_golden.py <path to the midnight-zk sources> (or set MZK_REFERENCE)")
OUT = Path(__file__).resolve().parent / "reference_kats.json"

NUM = r"(?:0x[0-9a-fA-F_]+|\d+)"


def parse_int(tok):
    tok = tok.replace("_", "")
    return int(tok, 16) if tok.lower().startswith("0x") else int(tok)


def read(rel):
    return (REF / rel).read_text()


def line_of(text, pos):
    return text.count("\n", 0, pos) + 1


def fn_body(text, name):
    """Text span of `fn name(` up to the next test/function at the same indent."""
    m = re.search(r"\n(\s*)fn " + re.escape(name) + r"\(", text)
    if not m:
        raise KeyError(name)
    indent = m.group(1)
    start = m.start() + 1
    nxt = re.search(r"\n" + indent + r"(#\[test\]|fn |\})", text[m.end():])
    end = m.end() + (nxt.start() if nxt else len(text) - m.end())
    return start, end


def arrays_in(text, start, end, prefix):
    """All `prefix[ ... ]` integer arrays in text[start:end], in order."""
    out = []
    for m in re.finditer(prefix + r"\s*\[\s*((?:" + NUM + r"\s*,\s*)*" + NUM + r")\s*,?\s*\]", text[start:end]):
        vals = [parse_int(t) for t in re.findall(NUM, m.group(1))]
        out.append({"limbs": ["0x%016x" % v for v in vals], "line": line_of(text, start + m.start())})
    return out


def const_array(text, name, prefix=r"l:"):
    m = re.search(r"const " + re.escape(name) + r"\s*:[^=]*=", text)
    if not m:
        raise KeyError(name)
    arr = arrays_in(text, m.end(), m.end() + 600, prefix)[0]
    arr["line"] = line_of(text, m.start())
    return arr


def byte_arrays_in(text, start, end):
    out = []
    for m in re.finditer(r"\[\s*((?:\d+\s*,\s*){31}\d+)\s*,?\s*\]", text[start:end]):
        vals = [int(t) for t in re.findall(r"\d+", m.group(1))]
        out.append({"bytes": vals, "line": line_of(text, start + m.start())})
    return out


def main():
    kats = {"source": "midnightntwrk/midnight-zk (read as text by tests/golden/make_golden.py)"}
    fq_path = "curves/src/bls12_381/fq.rs"
    fp_path = "curves/src/bls12_381/fp.rs"
    g1_path = "curves/src/bls12_381/g1.rs"
    fq = read(fq_path)
    fp = read(fp_path)
    g1 = read(g1_path)

    # ---- Fr (midnight's Fq) constants, Montgomery form ----
    fr = {"file": fq_path}
    for name in ["GENERATOR", "ROOT_OF_UNITY", "R", "R3", "LARGEST"]:
        fr[name] = const_array(fq, name)
    fr["R2"] = const_array(fq, "R2_LIMBS", prefix="")
    fr["MODULUS"] = const_array(fq, "MODULUS", prefix="")
    for name in ["ROOT_OF_UNITY_INV", "DELTA", "ZETA", "TWO_INV"]:
        fr[name] = const_array(fq, name)
    m = re.search(r"const INV: u64 = (0x[0-9a-fA-F_]+);", fq)
    fr["INV"] = {"value": "0x%016x" % parse_int(m.group(1)), "line": line_of(fq, m.start())}
    m = re.search(r"pub const S: u32 = (\d+);", fq)
    fr["S"] = {"value": int(m.group(1)), "line": line_of(fq, m.start())}

    s, e = fn_body(fq, "test_multiplication")
    a = arrays_in(fq, s, e, r"l:")
    fr["kat_mul"] = {"a": a[0], "b": a[1], "expected": a[2]}
    s, e = fn_body(fq, "test_addition")
    a = arrays_in(fq, s, e, r"l:")
    fr["kat_largest_plus_largest"] = {"expected": a[0]}
    s, e = fn_body(fq, "test_to_bytes")
    b = byte_arrays_in(fq, s, e)
    # order in the test: ZERO, ONE, R2 (canonical bytes of R2 = R mod r), -ONE
    fr["kat_to_bytes"] = {"zero": b[0], "one": b[1], "r2": b[2], "minus_one": b[3]}
    s, e = fn_body(fq, "test_from_bytes")
    b = byte_arrays_in(fq, s, e)
    # order: 0, 1, R2 bytes, -1 (valid), then three invalid encodings
    fr["kat_from_bytes_invalid"] = [b[4], b[5], b[6]]
    kats["fr"] = fr

    # ---- Fp constants and KATs ----
    fpk = {"file": fp_path}
    fpk["MODULUS"] = const_array(fp, "MODULUS", prefix="")
    fpk["R"] = const_array(fp, "R")
    s, e = fn_body(fp, "test_fp_mul_assign")
    a = arrays_in(fp, s, e, r"l:")
    fpk["kat_mul"] = {"a": a[0], "b": a[1], "expected": a[2]}
    s, e = fn_body(fp, "test_fp_squaring")
    a = arrays_in(fp, s, e, r"l:")
    c = arrays_in(fp, s, e, r"from_u64s_le\(&")
    fpk["kat_square"] = {"a": a[0], "expected_canonical": c[0]}
    s, e = fn_body(fp, "test_fp_add_assign")
    a = arrays_in(fp, s, e, r"l:")
    fpk["kat_add"] = [
        {"a": a[0], "b": a[2], "expected": a[3]},
        {"a": a[3], "b": a[4], "expected": a[5]},
        {"a": a[6], "b": a[7], "expected_zero": True},
        {"a": a[8], "b": a[9], "expected": a[10]},
    ]
    s, e = fn_body(fp, "test_fp_sub_assign")
    a = arrays_in(fp, s, e, r"l:")
    fpk["kat_sub"] = [
        {"a": a[0], "b": a[1], "expected": a[2]},
        {"a": a[3], "b": a[4], "expected": a[5]},
    ]
    kats["fp"] = fpk

    # ---- G1 ----
    g = {"file": g1_path}
    g["B"] = const_array(g1, "B")
    s, e = fn_body(g1, "test_doubling")
    a = arrays_in(g1, s, e, r"from_mont_unchecked\(")
    g["kat_double_generator"] = {"x": a[0], "y": a[1]}
    s, e = fn_body(g1, "test_projective_addition")
    a = arrays_in(g1, s, e, r"from_mont_unchecked\(")
    # z (twice), beta, expected x, expected y
    g["kat_add"] = {"z": a[0], "beta": a[2], "expected_x": a[3], "expected_y": a[4]}
    s, e = fn_body(g1, "test_projective_scalar_multiplication")
    a = arrays_in(g1, s, e, r"l:")
    g["kat_scalar_mul"] = {"a": a[0], "b": a[1]}
    readme = read("curves/README.md")
    m = re.search(r"##### G1\s*```\s*x = (\d+)\s*y = (\d+)", readme)
    g["generator"] = {"x": str(int(m.group(1))), "y": str(int(m.group(2))),
                      "file": "curves/README.md", "line": line_of(readme, m.start())}
    kats["g1"] = g

    OUT.write_text(json.dumps(kats, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
