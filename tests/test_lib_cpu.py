"""CPU checks of the C ABI library: it loads, exports every function include/hdgx.h
declares, and the Python binding declares matching argument counts."""
import ctypes as ct
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared():
    txt = (ROOT / "include" / "hdgx.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|const char \*|void)\s*\**\s*(hdgx_\w+)\s*\(([^;]*?)\)\s*;", txt, re.S):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def test_library_exports_every_declared_symbol():
    from hdg_b200 import _lib
    L = _lib.lib()
    decl = declared()
    assert len(decl) >= 5
    for name in decl:
        assert hasattr(L, name), name


def test_binding_argument_counts_match_header():
    from hdg_b200 import _lib
    L = _lib.lib()
    for name, n in declared().items():
        f = getattr(L, name)
        if f.argtypes is not None:
            assert len(f.argtypes) == n, (name, len(f.argtypes), n)


def test_version_and_status_strings():
    from hdg_b200 import _lib
    L = _lib.lib()
    assert L.hdgx_version() >= 10000
    assert L.hdgx_status_str(0) == b"ok"
    assert b"unsupported" in L.hdgx_status_str(-3)


def test_host_wait_mode_round_trip():
    from hdg_b200 import _lib
    L = _lib.lib()
    prev = L.hdgx_get_host_wait()
    assert prev in (0, 1)
    assert L.hdgx_set_host_wait(2) == -1 and L.hdgx_set_host_wait(-1) == -1
    assert L.hdgx_set_host_wait(1) == 0 and L.hdgx_get_host_wait() == 1
    assert L.hdgx_set_host_wait(0) == 0 and L.hdgx_get_host_wait() == 0
    L.hdgx_set_host_wait(prev)
