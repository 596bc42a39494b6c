"""The ctypes mirrors of the C-ABI structs must match the header's layout field by
field (offsets and total size), checked by compiling a probe against include/jxb.h."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO
from jaxley_pytorch_b200 import _lib

STRUCTS = [_lib.JxbTreeSchedule, _lib.JxbRegSchedule, _lib.JxbSimArgs, _lib.JxbSynArgs]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is not available")
def test_ctypes_structs_match_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "jxb.h"', "int main(void) {"]
    for st in STRUCTS:
        name = st.__name__
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for st in STRUCTS:
        name = st.__name__
        assert got[(name, "sizeof")] == C.sizeof(st), name
        for field, _ in st._fields_:
            assert got[(name, field)] == getattr(st, field).offset, (name, field)


def _int32_fields(body: str) -> int:
    n = 0
    for ln in body.split("\n")[1:]:
        if "int32_t" in ln:
            decl = ln.split(";")[0].replace("int32_t", "")
            n += len([x for x in decl.split(",") if x.strip()])
    return n


def test_block_and_item_records_match_header():
    # JxbBlock is 12 int32 and JxbItem 4 int32: the host packs them as int32 arrays.
    hdr = open(os.path.join(REPO, "include", "jxb.h")).read()
    blk = hdr[hdr.index("typedef struct {\n  int32_t node0"):hdr.index("} JxbBlock;")]
    item = hdr[hdr.index("typedef struct {\n  int32_t block;"):hdr.index("} JxbItem;")]
    assert _int32_fields(blk) == 12
    assert _int32_fields(item) == 4
    from jaxley_pytorch_b200 import synth
    from jaxley_pytorch_b200.lower import lower

    low = lower(synth.config_small())
    assert low.blocks.dtype == np.int32 and low.blocks.shape[1] == 12
