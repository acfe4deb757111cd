"""The C-ABI library loads and exports every function include/frep.h declares;
its error paths return status codes (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import frep
from frep import _lib

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (REPO / "include" / "frep.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(frep_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_function_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], check=True, capture_output=True,
                         text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    assert len(declared_functions()) >= 25


def test_python_binding_covers_the_header():
    assert set(declared_functions()) == set(_lib.declared_symbols())


def test_error_paths_without_a_gpu():
    lib = _lib.lib()
    # null arguments
    assert lib.frep_tape_compile(None, None) == _lib.ERR_INVALID_ARG
    assert b"null" in lib.frep_last_error()
    assert lib.frep_tape_get_info(None, None) == _lib.ERR_INVALID_ARG
    # a bad reference tape
    bad = (C.c_uint32 * 1)(0xFF)
    h = C.c_void_p()
    assert lib.frep_tape_from_reference(bad, 1, None, 0, C.byref(h)) == _lib.ERR_INVALID_ARG


@pytest.mark.skipif(__import__("conftest").has_gpu(), reason="checks the no-device path")
def test_context_without_a_device_reports_cuda_error():
    with pytest.raises(frep.FrepError) as e:
        frep.Context(0)
    assert e.value.status == _lib.ERR_CUDA
