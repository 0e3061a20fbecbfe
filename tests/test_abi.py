"""The C-ABI library loads and exports every entry point the header declares
(no compute calls; runs without a GPU)."""
import ctypes as C
import os

from dust_b200 import _lib, abi


def test_library_exists_and_loads():
    assert os.path.exists(_lib.SO_PATH)
    L = _lib.lib()
    assert L.dust_status_string(0) == b"ok"


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    syms = _lib.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_struct_sizes_match_header():
    L = _lib.lib()
    sizes = (C.c_int64 * 16)()
    n = L.dust_abi_sizes(sizes, 16)
    mine = [C.sizeof(t) for t in (abi.FmmParams, abi.Panels, abi.Lines, abi.Elements,
                                   abi.FmmStats, abi.SolveReport, abi.WakeRows,
                                   abi.UpdateParams, abi.PaParams, abi.WakeParams, abi.Te)]
    assert n == len(mine)
    assert list(sizes)[:n] == mine


def test_library_targets_sm100a_only():
    # the build recipe compiles for sm_100a only
    mk = open(os.path.join(os.path.dirname(_lib._HERE), "dust_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
