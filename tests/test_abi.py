"""The C ABI library loads without a GPU and exports every symbol of include/*.h."""
import ctypes
import glob
import os
import re

import pytest

from ctc_b200 import _lib
from ctc_b200.build import build

from .conftest import ROOT


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*(ctc_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_the_abi():
    names = declared_functions()
    assert "ctc_clist_build" in names and "ctc_sim_step" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_status_strings_without_gpu():
    L = _lib.lib()
    assert L.ctc_status_string(0) == b"ok"
    assert L.ctc_status_string(3) == b"capacity exceeded"
    assert abs(L.ctc_dpd_sigma(0.0444, 8.0, 5e-4) - 37.6935) < 1e-3


def test_argument_errors_are_reported_not_fatal():
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.ctc_fluforces_ini(2, 8, 8, 10, ctypes.byref(h))   # box must be >= 3 cells
    assert rc == _lib.CTC_ERR_ARG
    assert b"box" in L.ctc_last_error()


def test_binding_constants_match_the_header():
    """The Python mirror of the header's #defines (array sizes the binding
    allocates for the library to fill)."""
    src = open(os.path.join(ROOT, "include", "ctc_b200.h")).read()
    for name in ("CTC_SIM_PHASES", "CTC_RNG_REFERENCE", "CTC_RNG_STABLE"):
        m = re.search(r"#define\s+%s\s+(\d+)" % name, src)
        if m is None:
            m = re.search(r"\b%s\s*=\s*(\d+)" % name, src)
        assert m is not None, name
        assert getattr(_lib, name) == int(m.group(1)), name
    assert len(_lib.SIM_PHASE_NAMES) == _lib.CTC_SIM_PHASES
