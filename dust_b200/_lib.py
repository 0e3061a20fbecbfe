"""Loader of the compiled C-ABI library (dust_b200/_lib/libdust_b200.so).

There is no fallback: if the library is missing or no sm_100 device is
usable, the calls raise.
"""
import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
# DUST_B200_LIB selects another build of the same library (same ABI)
SO_PATH = os.environ.get("DUST_B200_LIB") or os.path.join(_HERE, "_lib", "libdust_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "dust_b200.h")

_lib = None


class DustError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = f"{where}: status {status}"
        try:
            msg += f" ({lib().dust_status_string(status).decode()})"
            le = lib().dust_last_error().decode()
            if le:
                msg += f" [{le}]"
        except Exception:  # pragma: no cover - diagnostics only
            pass
        super().__init__(msg)


def header_symbols():
    """Function names declared in include/dust_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"DUST_API\s+(?:const\s+char\s*\*|int)\s*(dust_\w+)\s*\(", txt)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise RuntimeError(
                f"{SO_PATH} is missing: build it with __graft_entry__.build() "
                "(make -C dust_b200/csrc)")
        L = C.CDLL(SO_PATH)
        for name in header_symbols():
            if hasattr(L, name):
                getattr(L, name).restype = C.c_int
        L.dust_status_string.restype = C.c_char_p
        L.dust_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(status, where):
    if status != 0:
        raise DustError(status, where)
