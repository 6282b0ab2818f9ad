"""The C-ABI library loads and exports every function include/*.h declares (no GPU calls)."""
import ctypes
import os
import re

from custingeralg_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(tc_[a-z_0-9]+)\s*\(", text, flags=re.M))


def test_every_declared_symbol_is_exported():
    lib = N.lib()
    decl = declared_functions("custinger_tc.h")
    assert len(decl) >= 10
    for name in decl:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, f"{name} missing from native.SIGNATURES"


def test_generator_library_exports():
    lib = ctypes.CDLL(os.path.join(ROOT, "custingeralg_b200", "libtcgen.so"))
    text = open(os.path.join(ROOT, "include", "tc_gen.h")).read()
    for name in re.findall(r"\b(tcgen_[a-z_]+)\s*\(", text):
        assert hasattr(lib, name), name


def test_default_sched_and_strings():
    s = N.default_sched()
    assert 2 <= s.warp_max_deg <= 256
    assert N.lib().tc_status_string(N.TC_ERR_NOT_SYMMETRIC) == b"graph not symmetric"
