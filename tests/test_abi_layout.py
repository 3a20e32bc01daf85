"""The ctypes mirrors of the C ABI structs (helix_b200/capi.py) against the
header itself: a small C program compiled with gcc prints sizeof and the
offset of every field of every public struct in include/helix_b200.h."""
import json
import os
import shutil
import subprocess
import ctypes as C

import pytest

from helix_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "hx_csr": capi._Csr,
    "hx_bath": capi._Bath,
    "hx_problem": capi._Problem,
    "hx_info": capi.Info,
    "hx_counters": capi.Counters,
    "hx_batch_options": capi.BatchOptions,
    "hx_batch_stats": capi.BatchStats,
}


def _probe_source() -> str:
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "helix_b200.h"', "int main(void) {",
             '    printf("{");']
    first = True
    for name, cls in STRUCTS.items():
        parts = [f'\\"size\\": %zu'] + [f'\\"{f}\\": %zu' for f, _ in cls._fields_]
        args = [f"sizeof({name})"] + [f"offsetof({name}, {f})" for f, _ in cls._fields_]
        sep = "" if first else ", "
        first = False
        lines.append(f'    printf("{sep}\\"{name}\\": {{{", ".join(parts)}}}", {", ".join(args)});')
    lines += ['    printf("}\\n");', "    return 0;", "}"]
    return "\n".join(lines) + "\n"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is not installed")
def test_ctypes_structs_match_the_header(tmp_path):
    src = tmp_path / "probe.c"
    exe = tmp_path / "probe"
    src.write_text(_probe_source())
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    layout = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    for name, cls in STRUCTS.items():
        got = layout[name]
        assert got["size"] == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert got[f] == getattr(cls, f).offset, f"{name}.{f}"
