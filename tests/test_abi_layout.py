"""The binding's ctypes structures have the C header's layout: a small C
program compiled against include/dcore_b200.h prints every struct's size and
field offsets, which must equal the ctypes ones (no GPU needed)."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> binding class name
STRUCTS = {"dc_graph_opts": "GraphOpts", "dc_decomp_info": "DecompInfo", "dc_maint_stats": "MaintStats",
           "dc_server_info": "ServerInfo", "dc_tuning": "Tuning"}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_header(dc, tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dcore_b200.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(dc, pyname)
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            name, field, val = line.split()
            got[(name, field)] = int(val)
    for cname, pyname in STRUCTS.items():
        cls = getattr(dc, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)


def test_tuning_as_dict(dc):
    t = dc.Tuning(3, 2, 128, (ctypes.c_int32 * 7)(150, 200, 450))
    assert t.as_dict() == {"peel_blocks_per_sm": 3, "rows_blocks_per_sm": 2, "peel_chunk": 128,
                           "rows_split_permille": [150, 200, 450, 0, 0, 0, 0]}
