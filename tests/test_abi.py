"""The C-ABI library loads and exports every entry point include/*.h declares
(CPU only: no compute call is made)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        syms |= set(re.findall(r"\b(icarat_[A-Za-z0-9_]+)\s*\(", src))
    return sorted(syms)


def test_header_declares_the_api():
    syms = declared_symbols()
    for s in ["icarat_ctx_create", "icarat_solve", "icarat_apply_K",
              "icarat_density_filter", "icarat_oc_update", "icarat_mma_update",
              "icarat_loop_step"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    import icarat2_b200 as G
    if not os.path.exists(G.LIBPATH):
        G_build = __import__("icarat2_b200.build", fromlist=["build"])
        G_build.build()
    lib = ctypes.CDLL(G.LIBPATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    import icarat2_b200 as G
    assert set(declared_symbols()) == set(G.SIGNATURES)


def test_status_strings_without_gpu():
    import icarat2_b200 as G
    L = G.load_library()
    assert L.icarat_status_string(0) == b"ok"
    assert L.icarat_status_string(G.ERR_STATE) == b"call order violated"
    assert L.icarat_version() >= 10100  # option structs with filter_kind
