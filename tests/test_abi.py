"""The C-ABI library loads and exports every symbol include/icarat_b200.h
declares (no compute calls: runs without a GPU)."""
import ctypes as C
import os

import icarat_b200 as icb


def test_library_built_and_loads():
    assert os.path.exists(icb.LIB_PATH), "run python icarat-contact_b200/build.py"
    L = icb.lib()
    assert L.icb_version().decode().startswith("icarat-b200")


def test_every_header_symbol_is_exported():
    syms = icb.header_symbols()
    assert len(syms) >= 25
    L = C.CDLL(icb.LIB_PATH)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(icb.header_symbols()) <= set(icb._SIGS), set(icb.header_symbols()) - set(icb._SIGS)


def test_no_torch_in_the_abi():
    txt = open(icb.HEADER).read()
    assert "torch" not in txt.lower() or "no torch" in txt.lower()
