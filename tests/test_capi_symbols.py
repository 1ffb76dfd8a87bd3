"""The C-ABI library loads and exports every entry point its header declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(viprs_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "viprs_plan_execute" in names and "viprs_reduceh" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from viprs_b200 import _native
    lib = _native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_signature_table_covers_header():
    from viprs_b200 import _native
    missing = [n for n in declared_functions() if n not in _native.SIGNATURES]
    assert not missing, f"no ctypes signature for: {missing}"


def test_status_strings():
    from viprs_b200 import _native
    lib = _native.lib()
    assert lib.viprs_status_string(0) == b"ok"
    assert b"taps" in lib.viprs_status_string(3)
