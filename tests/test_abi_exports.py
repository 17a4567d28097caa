"""The C ABI library loads without a GPU and exports every function that
include/trex_b200.h declares; the ctypes table (trex_b200/_lib.py) covers the
same set. No compute call is made."""

import ctypes
import re
import shutil
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


def _declared():
    text = (REPO / "include" / "trex_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M)))


def test_header_declares_the_reference_abis():
    names = _declared()
    for n in ("monoid_batch_engine_init", "prefix_engine_dispatch", "monoid_engine_dispatch_batch",
              "nfa_tc_engine_dispatch", "trex_dfa_batch_run", "trex_dfa_batch_run_static",
              "trex_dfa_set_kgram", "trex_pnfa_run", "trex_nfa_run", "trex_dfa_scan_run"):
        assert n in names


@pytest.mark.skipif(shutil.which("nvcc") is None and not (REPO / "build" / "libtrex_b200.so").exists(),
                    reason="needs nvcc (to build) or a built library")
def test_library_exports_every_declared_symbol():
    from trex_b200 import _lib
    from trex_b200.build import build
    lib_path = build()
    L = ctypes.CDLL(str(lib_path))
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(_declared()) == set(_lib.SIGNATURES), set(_declared()) ^ set(_lib.SIGNATURES)
