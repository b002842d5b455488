"""The C ABI library loads without a GPU, exports every entry point the
public header declares, and agrees with the Python mirror of its structs."""
import ctypes as C
import os
import re

from asterx_b200 import abi
from asterx_b200.engine import LIB_PATH, load_library

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "asterx_b200.h")


def declared_entry_points():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"AXB_API\s+[\w\s\*]+?\b(axb_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = load_library()
    names = declared_entry_points()
    assert len(names) >= 5
    for n in names:
        assert hasattr(lib, n), n


def test_param_defaults_match_reference_param_ccl():
    lib = load_library()
    p = abi.Params()
    lib.axb_params_default(C.byref(p))
    q = abi.default_params()
    for name, _ in abi.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name


def test_grid_function_names():
    lib = load_library()
    for i, n in enumerate(abi.GF_NAMES):
        assert lib.axb_gf_name(i).decode() == n
    assert lib.axb_gf_name(abi.NUM_GF) is None
