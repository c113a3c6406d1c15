"""CPU-side check that the Python binding's structures and constants match include/bem_b200.h: a
small C program compiled against the header prints the size and field offsets of every structure
the binding mirrors, and the #define constants are read from the header text."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from bem_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bem_b200.h")

STRUCTS = {"bem_params": L.Params, "bem_stats": L.Stats, "bem_profile": L.Profile}


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "bem_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([shutil.which("gcc"), "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_structures_match_the_header(tmp_path):
    lay = _c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert C.sizeof(py) == lay[(cname, "size")], cname
        for fname, _ in py._fields_:
            assert getattr(py, fname).offset == lay[(cname, fname)], (cname, fname)


def test_constants_match_the_header():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    defines = {m.group(1): int(m.group(2), 0) for m in re.finditer(r"#define\s+(BEM_\w+)\s+(-?\w+)\b", text)
               if re.fullmatch(r"-?(0x[0-9a-fA-F]+|\d+)", m.group(2))}
    # enumerators (status codes, solver ids)
    defines.update({m.group(1): int(m.group(2)) for m in re.finditer(r"\b(BEM_\w+)\s*=\s*(\d+)", text)})
    assert defines["BEM_OK"] == L.BEM_OK and defines["BEM_ERR_STATE"] == L.BEM_ERR_STATE
    assert defines["BEM_FLAG_BICGSTAB_MULTIKERNEL"] == L.FLAG_BICGSTAB_MULTIKERNEL
    assert defines["BEM_FLAG_NO_STAGE_PREDICTOR"] == L.FLAG_NO_STAGE_PREDICTOR
    # every status code and solver id the binding names
    for name, value in defines.items():
        short = name[len("BEM_"):]
        if hasattr(L, name):
            assert getattr(L, name) == value, name
        elif short.startswith("SOLVER_") and hasattr(L, short):
            assert getattr(L, short) == value, name
