"""The ctypes mirrors of the Arrow C Data Interface structures and of
ursa_gpu_output_column (ursa_b200/result.py) match include/ursa_gpu.h: sizes
and every field offset, checked against a C program compiled here."""

import ctypes as C
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_layout(tmp_path, structs):
    src = ['#include <stddef.h>', '#include <stdio.h>', '#include "ursa_gpu.h"', "int main(void) {"]
    for ctype, fields in structs:
        src.append(f'  printf("{ctype} %zu\\n", sizeof({ctype}));')
        for f in fields:
            src.append(f'  printf("{ctype}.{f} %zu\\n", offsetof({ctype}, {f}));')
    src += ["  return 0;", "}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = str(tmp_path / "layout")
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (line.rsplit(None, 1) for line in out.splitlines())}


def test_struct_layouts_match_header(tmp_path):
    from ursa_b200.result import ArrowArray, ArrowSchema, _Column

    pairs = [("struct ArrowSchema", ArrowSchema), ("struct ArrowArray", ArrowArray),
             ("ursa_gpu_output_column", _Column)]
    got = _c_layout(tmp_path, [(c, [f for f, _ in py._fields_]) for c, py in pairs])
    for cname, py in pairs:
        assert got[cname] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[f"{cname}.{f}"] == getattr(py, f).offset, (cname, f)
