"""The engine's shared library: builds, loads and exports every C-ABI symbol
that include/*.h declares (no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//.*", "", src)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(qg_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["qg_context_create", "qg_hamiltonian_create", "qg_hamiltonian_apply_d",
              "qg_hamiltonian_apply_f", "qg_hamiltonian_apply_host_d", "qg_status_string"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from qumasun_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_no_device_errors_are_loud():
    from qumasun_b200 import engine
    L = engine.lib()
    assert L.qg_status_string(0) == b"ok"
    assert L.qg_status_string(-4) == b"Gram matrix not positive definite"
    assert L.qg_version() == 1
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(engine.QGError):
            engine.Context(0)
