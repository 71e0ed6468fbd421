"""The ctypes mirrors of the C-ABI structs (sphpc_b200/_lib.py) against the
header itself: a small C program compiled with gcc against
include/sphpc_types.h prints sizeof and offsetof of every field the binding
declares, and each must match ctypes.  A field added on one side only fails
to compile or shifts an offset."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from sphpc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ctypes class -> C struct tag
STRUCTS = {
    _lib.Params: "Params", _lib.AABB: "AABB", _lib.Particles: "Particles",
    _lib.NeighborBucket: "NeighborBucket", _lib.Neighbors: "Neighbors",
    _lib.Obstacle: "Obstacle", _lib.Solver: "SphpcSolver", _lib.FileIO: "FileIO",
    _lib.Diag: "SphpcDiag", _lib.StepInfo: "SphpcStepInfo", _lib.KernelTime: "SphpcKernelTime",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_layout_matches_header(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "sphpc_types.h"',
             "int main(void) {"]
    expect = []
    for cls, tag in STRUCTS.items():
        lines.append(f'  printf("%zu\\n", sizeof(struct {tag}));')
        expect.append((f"sizeof {tag}", C.sizeof(cls)))
        for name, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof(struct {tag}, {name}));')
            expect.append((f"{tag}.{name}", getattr(cls, name).offset))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert len(got) == len(expect)
    bad = [(what, want, g) for (what, want), g in zip(expect, got) if want != g]
    assert not bad, bad
