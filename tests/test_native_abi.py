"""The C-ABI library loads and exports every entry point declared in include/zlatko_b200.h (no GPU needed)."""
import os
import re
import subprocess

from zlatko_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(zk_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_the_documented_entry_points():
    assert declared_symbols() == set(_native.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (zk_\w+)", out))
    assert declared_symbols() <= exported


def test_abi_version():
    assert _native.lib().zk_abi_version() == 1
