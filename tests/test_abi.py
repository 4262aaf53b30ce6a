"""The C ABI: libmpp.so loads without a GPU and exports every entry point include/mpp.h
declares; the host-only entry points behave as documented. No device calls here."""
import ctypes
import os
import re

import pytest

from mpp import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mpp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mpp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_symbols()
    for need in ("mpp_ctx_create", "mpp_ctx_destroy", "mpp_project", "mpp_pressure", "mpp_vcycle", "mpp_volume"):
        assert need in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_opts_default_matches_reference_defaults():
    lib = _lib.load()
    o = _lib.Opts()
    lib.mpp_opts_default(ctypes.byref(o))
    # pressure!(s; tol = 1f-4, maxiter = 60, sweeps = 2), vcycle!(...; coarse = 40)
    assert o.tol == pytest.approx(1e-4) and o.maxiter == 60 and o.sweeps == 2 and o.coarse == 40
    assert o.precision == 0 and o.restart == 8


@pytest.mark.parametrize("n,levels", [((64, 64, 64), 4), ((256, 256, 256), 6), ((384, 384, 256), 7),
                                      ((48, 48, 24), 3), ((30, 30, 30), -1)])
def test_levels_for(n, levels):
    lib = _lib.load()
    arr = (ctypes.c_int32 * 3)(*n)
    assert lib.mpp_levels_for(arr) == levels


def test_version_string():
    assert b"sm_100a" in _lib.load().mpp_version()
