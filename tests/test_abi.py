"""The C-ABI library: it loads, exports every function include/*.h declares,
validates arguments and reports errors through status codes.  CPU only (no
compute call needs a GPU here)."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

import pytest

from conftest import LIB_SO, ROOT, have_gpu
from origami_b200 import _ffi as F


def declared_functions() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(og_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_SO), "build the library first: python -m origami_b200.build"
    lib = C.CDLL(LIB_SO)
    declared = declared_functions()
    assert len(declared) > 30
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers exactly the declared set
    assert {n for n, _, _ in F.SIGNATURES} == declared


def test_status_strings(origami):
    lib = origami.lib()
    assert lib.og_status_string(0) == b"ok"
    assert b"diverged" in lib.og_status_string(2)
    assert lib.og_version().startswith(b"origami-b200")


def test_bad_arguments_return_status(origami):
    lib = origami.lib()
    h = C.c_void_p()
    assert lib.og_chain_build(b"", 0.0, 0.0, 0.0, C.byref(h)) == 1
    assert lib.og_chain_build(b"AXZ", 0.0, 0.0, 0.0, C.byref(h)) == 1
    assert b"amino" in lib.og_last_error()
    assert lib.og_chain_build(None, 0.0, 0.0, 0.0, C.byref(h)) == 1
    p = F.og_params()
    lib.og_params_default(C.byref(p))
    assert p.nb_cutoff == 10.0 and p.born_cutoff == 20.0 and p.gb_force_cutoff == 10.0
    assert lib.og_engine_create(None, C.byref(h)) == 1
    assert lib.og_step(None, 1) == 1


@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_engine_without_gpu_fails_loudly(origami):
    lib = origami.lib()
    p = F.og_params()
    lib.og_params_default(C.byref(p))
    h = C.c_void_p()
    st = lib.og_engine_create(C.byref(p), C.byref(h))
    assert st == 5  # OG_E_CUDA: there is no CPU fallback
    with pytest.raises(origami.OrigamiError):
        origami.Engine()
