"""The C ABI library (CPU checks, no GPU calls): it loads, it exports every
function include/ufem_gpu.h declares, and without a GPU it fails loudly
instead of falling back to the CPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof") or name.isupper():
                continue
            names.add(name)
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from ufem_b200 import _lib, build
    build.build()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from ufem_b200 import _lib
    assert set(declared_functions()) == set(_lib.EXPORTED)


def test_no_gpu_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    rv = lib.ufem_device_info(None, None, None, None)
    assert rv == -1
    assert b"no CPU fallback" in lib.ufem_last_error()
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200._lib import UfemError
    with pytest.raises(UfemError):
        GpuModel(mg.beam_brick(2, 1, 1))
    assert lib.monte_init_lib_stuff(b"/nonexistent.fem") == -1


def test_monte_interface_type(lib):
    assert lib.monte_dlib_interface_type() == 2
