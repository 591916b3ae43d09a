"""The C-ABI library loads without a GPU and exports every entry point that
include/emustack_gsm.h declares; host-only entry points are checked here."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, 'include')):
        if fn.endswith('.h'):
            src = open(os.path.join(ROOT, 'include', fn)).read()
            src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
            names |= set(re.findall(r'\b(emu_[a-z0-9_]+)\s*\(', src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from emustack_b200 import _lib
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 6
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    from emustack_b200 import _lib
    L = _lib.lib()
    assert L.emu_version() >= 100
    for s in range(0, 9):
        assert L.emu_status_string(s)


@pytest.mark.parametrize('max_order,period,period_y', [(1, 1.0, 1.0), (3, 600.0, 600.0), (5, 500.0, 500.0),
                                                      (10, 700.0, 700.0), (10, 500.0, 500.0),
                                                      (4, 940.0, 940.0), (6, 760.0, 380.0),
                                                      (7, 450.0, 610.0)])
def test_grating_orders_match_reference_rounding(max_order, period, period_y):
    """Order sets equal backend/mode_calcs.py:61-74 bit for bit, including the
    orders dropped on the circle by rounding (period 700, max order 10)."""
    from emustack_b200.films import grating_orders
    from oracle import gsm_oracle as O
    px, py = grating_orders(max_order, period, period_y)
    rx, ry = O.grating_orders_2d(max_order, period, period_y)
    np.testing.assert_array_equal(px, rx)
    np.testing.assert_array_equal(py, ry)
    if (max_order, period) == (10, 700.0):
        assert len(px) == 309
    if (max_order, period) == (10, 500.0):
        assert len(px) == 317


def test_grating_orders_1d_and_errors():
    from emustack_b200.films import grating_orders
    from emustack_b200 import _lib
    px, py = grating_orders(6, 760.0, world_1d=True)
    np.testing.assert_array_equal(px, np.arange(-6, 7))
    assert not py.any()
    import ctypes as C
    n = C.c_int(0)
    assert _lib.lib().emu_grating_orders(-1, 1.0, 1.0, 0, None, None, 0, C.byref(n)) == 1
