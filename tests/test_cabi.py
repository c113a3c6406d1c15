"""CPU-side checks of the C ABI: the library builds, loads, and exports every entry point that
include/bem_b200.h declares, with the reference's default parameters.  No compute call is made
here (there is no GPU in the build container)."""
import ctypes as C
import os
import re

import pytest

from bem_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bem_[a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    # every declared function has a ctypes signature in the binding (and vice versa)
    names = declared_symbols()
    assert names <= set(L.SIGNATURES) | {"bem_solve_into"}, names - set(L.SIGNATURES)


def test_default_params_follow_reference():
    lib = L.load()
    p = L.Params()
    lib.bem_default_params(C.byref(p))
    # Simulation ctor defaults (Simulation.hpp:29-39), LinLinSim eps (LinLinSim.hpp:24)
    assert (p.p_inf, p.epsilon, p.sigma, p.gamma) == (1.0, 1.0, 0.0, 1.0)
    assert p.min_dt == -1.0 and p.dp_balance == 3.0 and p.nopen_eps == 1e-2
    assert p.solver == L.SOLVER_BICGSTAB and p.mirror == 0
    assert C.sizeof(L.Params) == 8 * 11 + 4 * 2 + 8 + 4 * 2


def test_null_context_is_rejected():
    lib = L.load()
    assert lib.bem_destroy(None) == L.BEM_OK
    assert lib.bem_set_phi(None, None) == L.BEM_ERR_ARG


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.load()
    h = C.c_void_p()
    rc = lib.bem_create(C.byref(h), 0, None)
    assert rc == L.BEM_ERR_CUDA and not h.value
