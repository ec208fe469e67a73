"""The ctypes mirrors of the C ABI structs (midnight-zk_b200/__init__.py)
have the size and field offsets of the structs in include/mzk.h: a small C
program compiled against the header prints sizeof / offsetof of every field,
and each must equal the ctypes value.  CPU only (gcc)."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from _loader import load

mzk = load()
ROOT = Path(__file__).resolve().parent.parent

# ctypes class -> C struct name
PAIRS = [
    (mzk.MsmBatchItem, "mzk_msm_batch_item"),
    (mzk.ProvingKeyDesc, "mzk_proving_key_desc"),
    (mzk.ProofJob, "mzk_proof_job"),
    (mzk.QuotientDesc, "mzk_quotient_desc"),
    (mzk.ColumnRead, "mzk_column_read"),
    (mzk.FlatOp, "mzk_flat_op"),
    (mzk.FlatGraph, "mzk_flat_graph"),
    (mzk.LookupArg, "mzk_lookup_arg"),
    (mzk.TrashArg, "mzk_trash_arg"),
    (mzk.PermutationDesc, "mzk_permutation_desc"),
    (mzk.LogupDesc, "mzk_logup_desc"),
]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_the_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mzk.h"', "int main(void) {"]
    for cls, cname in PAIRS:
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field in cls._fields_:
            lines.append(f'printf("{cname} {field[0]} %zu\\n", offsetof({cname}, {field[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cls, cname in PAIRS:
        assert ctypes.sizeof(cls) == got[(cname, "size")], cname
        for field in cls._fields_:
            assert getattr(cls, field[0]).offset == got[(cname, field[0])], (cname, field[0])
