"""The C-ABI library loads and exports every symbol its headers declare, and
its argument checks fail loudly (no GPU needed)."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT

import zerork_b200 as zb


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(zrk_\w+|zerork_reactor_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    syms = declared_symbols()
    assert "zrk_rates_jac_dev" in syms and "zrk_mech_create" in syms


@pytest.mark.parametrize("sym", declared_symbols())
def test_library_exports(sym):
    L = zb.lib()
    assert hasattr(L, sym), f"{sym} not exported by {zb.LIB_PATH}"


def test_null_handle_and_pointer_errors(c1):
    L = zb.lib()
    assert L.zrk_mech_sizes(None, None, None, None, None) == 1
    assert L.zrk_mech_free(None) == 1
    h = C.c_void_p()
    assert L.zrk_mech_parse(None, b"x", C.byref(h)) == 2
    pm = zb.Mechanism(*c1[1], device=False)
    rc = L.zrk_rates_jac_dev(pm.handle, 4, 4, None, None, None, None, None, None, None)
    assert rc != 0
    assert L.zrk_mech_set_double_option(pm.handle, b"no_such_option", 1.0) == 5
    pm.set_option("step_limiter", 1e20)
    assert pm.get_option("step_limiter") == 1e20
