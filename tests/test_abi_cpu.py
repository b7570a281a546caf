"""CPU checks of the C ABI: the library loads, exports every function include/tild.h declares,
and rejects invalid configurations before touching a device."""
import ctypes as C
import os
import re

import pytest

import tild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "tild.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int32_t|const char\*)\s+(tild_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    L = tild.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_abi_version_and_status_strings():
    L = tild.lib()
    assert L.tild_abi_version() == 1
    assert L.tild_status_string(tild.OK) == b"ok"
    assert L.tild_status_string(tild.ERR_BAD_INPUT) == b"bad input"


@pytest.mark.parametrize("field,value", [("dim", 4), ("pmeorder", 5), ("ns", 0), ("ntypes", 0)])
def test_invalid_config_rejected_before_device(field, value):
    from helpers import small_diblock
    cfg = small_diblock(3, 1).config()
    setattr(cfg, field, value)
    h = C.c_void_p()
    assert tild.lib().tild_create(C.byref(cfg), 0, C.byref(h)) == tild.ERR_BAD_INPUT
    assert not h.value


def test_bad_style_type_and_unsupported_integrator_order():
    from helpers import small_diblock
    L = tild.lib()
    cfg = small_diblock(3, 1).config()
    cfg.styles[0].type2 = 5
    h = C.c_void_p()
    assert L.tild_create(C.byref(cfg), 0, C.byref(h)) == tild.ERR_BAD_INPUT
    cfg = small_diblock(3, 1).config()
    cfg.n_integrators = 2
    cfg.integrators[0].kind, cfg.integrators[0].group_type = tild.INTEGRATOR_EM, -1
    cfg.integrators[1].kind, cfg.integrators[1].group_type = tild.INTEGRATOR_GJF, 0
    assert L.tild_create(C.byref(cfg), 0, C.byref(h)) == tild.ERR_UNSUPPORTED


def test_null_arguments():
    L = tild.lib()
    assert L.tild_create(None, 0, None) == tild.ERR_BAD_INPUT
    assert L.tild_destroy(None) == tild.ERR_BAD_INPUT
    assert L.tild_step(None, 1) == tild.ERR_BAD_INPUT
