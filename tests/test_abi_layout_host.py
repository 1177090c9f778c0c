"""The ctypes mirrors of the C ABI's structures have the C layout.

A small C program compiled against include/simpfem.h with the host compiler
prints sizeof and every field's offset of simpfem_gmg_opts, simpfem_gmg_props,
simpfem_policy_opts, simpfem_policy_result and simpfem_policy_state; the ctypes
structures in gpu_fem._lib must agree field by field (no GPU needed)."""

import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "simpfem_gmg_opts": "GmgOpts",
    "simpfem_gmg_props": "GmgProps",
    "simpfem_policy_opts": "PolicyOpts",
    "simpfem_policy_result": "PolicyResult",
    "simpfem_policy_state": "PolicyState",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_struct_layouts_match(tmp_path):
    from gpu_fem import _lib

    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "simpfem.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(_lib, pyname)
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line.strip():
            a, b, v = line.split()
            got[(a, b)] = int(v)
    for cname, pyname in STRUCTS.items():
        cls = getattr(_lib, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
