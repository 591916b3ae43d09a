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


STRUCTS = ('EmuFilmStackBatch', 'EmuAnalloModes', 'EmuLayer', 'EmuStackDense', 'EmuOverlap',
           'EmuNormalise', 'EmuFilmPoint', 'EmuFilmVarBatch', 'EmuVarLayer', 'EmuStackPoint',
           'EmuStackVarBatch', 'EmuOverlap1D', 'EmuNormalise1D', 'EmuMaterial', 'EmuFilmRingRequest',
           'EmuFilmRingResult', 'EmuPwFields', 'EmuBlochFieldsPlane', 'EmuFemTopology', 'EmuFemElements',
           'EmuFemFields', 'EmuFem1dTopology', 'EmuFem1dElements', 'EmuFem1dFields')


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror of a descriptor struct has the C layout of
    include/emustack_gsm.h (size and the offset of every field)."""
    import ctypes as C
    import shutil
    import subprocess
    from emustack_b200 import _lib
    gcc = shutil.which('gcc')
    if gcc is None:
        pytest.skip('gcc not available')
    src = tmp_path / 'layout.c'
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "emustack_gsm.h"', 'int main(void){']
    for name in STRUCTS:
        lines.append('printf("%%zu", sizeof(%s));' % name)
        lines += ['printf(" %%zu", offsetof(%s, %s));' % (name, f) for f, _ in getattr(_lib, name)._fields_]
        lines.append('printf("\\n");')
    lines.append('return 0; }')
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'layout'
    subprocess.check_call([gcc, '-I' + os.path.join(ROOT, 'include'), str(src), '-o', str(exe)])
    out = subprocess.check_output([str(exe)]).decode().strip().split('\n')
    assert len(out) == len(STRUCTS)
    for name, line in zip(STRUCTS, out):
        st = getattr(_lib, name)
        got = list(map(int, line.split()))
        assert got[0] == C.sizeof(st), name
        assert got[1:] == [getattr(st, f).offset for f, _ in st._fields_], name


def test_film_var_plan_offsets_and_order():
    """emu_film_var_plan packs outputs point after point, sizes the workspace
    (one slot per point, Npw slots for caller-given incoming vectors) and
    orders points costliest first (stable on ties)."""
    import ctypes as C
    from emustack_b200 import _lib, films
    shapes = [(3, 5, 0), (12, 25, 0), (2, 1, 0), (12, 25, -1), (5, 9, 2)]
    desc = np.zeros(len(shapes), films._POINT_DTYPE)
    for i, (L, npw, pol) in enumerate(shapes):
        desc[i]['n_layers'], desc[i]['n_pw'], desc[i]['pol'] = L, npw, pol
        desc[i]['period'] = desc[i]['period_y'] = 600.0
    order = np.zeros(len(shapes), np.int32)
    rt, li, npl = C.c_int64(), C.c_int64(), C.c_int64()
    ws, ml, mp = C.c_size_t(), C.c_int(), C.c_int()
    st = _lib.lib().emu_film_var_plan(desc.ctypes.data_as(C.c_void_p), len(shapes),
                                      order.ctypes.data_as(C.c_void_p), C.byref(rt), C.byref(li),
                                      C.byref(npl), C.byref(ws), C.byref(ml), C.byref(mp))
    assert st == 0
    assert rt.value == sum(2 * s[1] for s in shapes)
    assert li.value == sum(s[0] - 1 for s in shapes)
    assert npl.value == sum(s[0] + 1 for s in shapes)
    assert (ml.value, mp.value) == (12, 25)
    np.testing.assert_array_equal(desc['rt_off'], np.cumsum([0] + [2 * s[1] for s in shapes])[:-1])
    np.testing.assert_array_equal(desc['list_off'], np.cumsum([0] + [s[0] - 1 for s in shapes])[:-1])
    per = [(s[1] if s[2] == -1 else 1) * s[0] * 2 * 5 * 16 for s in shapes]
    np.testing.assert_array_equal(desc['ws_off'], np.cumsum([0] + per)[:-1])
    assert ws.value == sum(per)
    assert list(order[:2]) == [1, 3] and order[-1] == 2
    desc[2]['n_layers'] = 1
    assert _lib.lib().emu_film_var_plan(desc.ctypes.data_as(C.c_void_p), len(shapes), None,
                                        None, None, None, None, None, None) == 2


def test_argument_checks_need_no_gpu():
    """Descriptors the library must refuse are refused on the host, before
    any device work: status codes as the header documents them."""
    import ctypes as C
    from emustack_b200 import _lib
    L = _lib.lib()
    # uneven dense batch
    assert L.emu_stack_var_batch(None, None, 0, None) == 1                 # EMU_E_ARG
    d = _lib.EmuStackVarBatch()
    d.n_stacks = 3
    d.max_P, d.max_D, d.max_L = 26, 30, 4
    assert L.emu_stack_var_workspace_size(C.byref(d)) == 0                 # no buffers: invalid
    assert L.emu_stack_var_batch(C.byref(d), None, 0, None) == 1
    for nm in ('d_points', 'd_layers', 'd_R_net', 'd_T_net', 'd_a_list', 'd_t_list', 'd_r_list', 'd_flags',
               'd_info'):
        setattr(d, nm, 256)
    d.max_L = 65                                                           # above the 64-layer limit
    assert L.emu_stack_var_batch(C.byref(d), None, 0, None) == 2           # EMU_E_SHAPE
    d.max_L, d.max_D = 4, 20                                               # max_D below max_P
    assert L.emu_stack_var_batch(C.byref(d), None, 0, None) == 2
    d.max_D, d.n_slots = 30, 2
    assert L.emu_stack_var_slots(C.byref(d)) == 2
    assert L.emu_stack_var_batch(C.byref(d), None, 0, None) == 5           # EMU_E_WORKSPACE
    d.n_stacks = 0
    assert L.emu_stack_var_batch(C.byref(d), None, 0, None) == 0           # nothing to do
    # overlap: complex64 fields only on the tensor-core path
    o = _lib.EmuOverlap()
    o.batch, o.nval, o.nel, o.npt, o.n_pw, o.max_order = 1, 4, 2, 4, 5, 1
    for nm in ('d_px', 'd_py', 'd_x', 'd_table_nod', 'd_bloch', 'd_k0', 'd_sol1', 'd_J'):
        setattr(o, nm, 256)
    o.d, o.dy, o.area_norm = 1.0, 1.0, 1.0
    o.field_c64, o.precision = 1, 0
    assert L.emu_overlap_batch(C.byref(o), None, 0, None) == 8            # EMU_E_UNSUPPORTED
    o.field_c64 = 2
    assert L.emu_overlap_batch(C.byref(o), None, 0, None) == 1
    # uneven film batch: register-budget variant out of range
    f = _lib.EmuFilmVarBatch()
    f.variant = 2
    assert L.emu_film_var_batch(C.byref(f), None, 0, None) != 0


def test_film_sources_build_with_exact_rounding():
    """The film kernels' launch shapes return the same bits only when their
    sources are compiled without compiler-chosen multiply-add contraction."""
    from emustack_b200 import build
    assert {'film_stack.cu', 'film_varlen.cu'} <= build.EXACT_ROUNDING


@pytest.mark.parametrize('max_order', [0, 1, 3, 4, 6, 9, 15, 20])
def test_pw_order_1d_matches_the_oracle(max_order):
    """emu_pw_order_1d ranks the 1D plane waves as the oracle's restatement
    of pw_ordering_1d / z_indexx does, tied keys included (zero Bloch
    vector: +-px tie)."""
    import ctypes as C
    from emustack_b200 import _lib
    from oracle import overlap1d_oracle as O
    L = _lib.lib()
    rng = np.random.default_rng(max_order)
    cases = [(0.0, 0.0, 2 * np.pi / 1.3), (0.0, 0.0, 2 * np.pi / 0.61)] + \
        [(rng.uniform(-1, 1), rng.uniform(-1, 1), 2 * np.pi / rng.uniform(0.5, 2.5)) for _ in range(4)]
    for period_x in (1.0, 0.83):
        for bx, by, k0 in cases:
            out = np.empty(2 * max_order + 1, np.int32)
            assert L.emu_pw_order_1d(max_order, period_x, bx, by, k0, out.ctypes.data_as(C.c_void_p)) == 0
            _, inv = O.pw_order_1d(max_order, period_x, bx, by, k0)
            np.testing.assert_array_equal(out, inv)


@pytest.mark.parametrize('max_order', [1, 3, 4, 6, 10])
def test_pw_embed_1d_to_2d_matches_the_oracle(max_order):
    """emu_pw_embed_1d_to_2d places each 1D order where the oracle's
    restatement of pw_matrix_1d_to_2d puts its J row."""
    import ctypes as C
    from emustack_b200 import _lib
    from oracle import overlap1d_oracle as O
    L = _lib.lib()
    for period_x, bx, by, k0 in ((1.0, 0.0, 0.0, 2 * np.pi / 1.1), (1.0, 0.31, -0.2, 7.3),
                                 (0.7, 0.0, 0.0, 4.0)):
        n2 = C.c_int(0)
        assert L.emu_pw_embed_1d_to_2d(max_order, period_x, bx, by, k0, None, 0, C.byref(n2)) == 0
        rows = np.empty(2 * max_order + 1, np.int32)
        assert L.emu_pw_embed_1d_to_2d(max_order, period_x, bx, by, k0, rows.ctypes.data_as(C.c_void_p),
                                       len(rows), C.byref(n2)) == 0
        _, inv = O.pw_order_1d(max_order, period_x, bx, by, k0)
        npw1 = 2 * max_order + 1
        J = np.zeros((2 * npw1, 1), complex)
        J[:npw1, 0] = 1 + np.arange(npw1)          # label each sorted 1D row
        J2, _, (p2, _) = O.pw_matrix_1d_to_2d(J, J.T.copy(), period_x, bx, by, max_order, k0, inv)
        assert n2.value == len(p2)
        for o in range(npw1):
            assert J2[rows[o], 0] == 1 + inv[o]


def test_field_entry_points_check_their_arguments_on_the_host():
    """emu_pw_fields and emu_bloch_fields_plane refuse bad descriptors before
    touching the device: order counts out of range, a grid without its
    workspace, a plane outside the layer; emu_pw_fields_workspace_size is
    the tables' size for grids and 0 for points."""
    import ctypes as C
    from emustack_b200 import _lib
    L = _lib.lib()
    d = _lib.EmuPwFields()
    d.n_stacks, d.n_pw, d.grid, d.nx, d.ny, d.nz = 2, 81, 1, 51, 51, 4
    assert L.emu_pw_fields_workspace_size(C.byref(d)) == 2 * (51 + 51 + 3 * 4) * 81 * 16
    d.grid = 0
    assert L.emu_pw_fields_workspace_size(C.byref(d)) == 0
    d.n_pw = 0
    assert L.emu_pw_fields(C.byref(d), None) == _lib.EMU_E_ARG
    d.n_pw = _lib.PW_FIELDS_MAX_ORDERS + 1
    assert L.emu_pw_fields(C.byref(d), None) == _lib.EMU_E_ARG
    # a grid with every input present but no workspace
    d.n_pw, d.grid = 81, 1
    for f in ('d_alphas', 'd_betas', 'd_sort', 'd_kz', 'd_n', 'd_vec_coef_down', 'd_x', 'd_y', 'd_z', 'd_E'):
        setattr(d, f, 256)
    d.vcd_stride = 162
    assert L.emu_pw_fields(C.byref(d), None) == _lib.EMU_E_WORKSPACE
    b = _lib.EmuBlochFieldsPlane()
    b.n_stacks, b.n_modes, b.n_elements, b.h, b.hz = 1, 10, 5, 0.3, 0.31
    assert L.emu_bloch_fields_plane(C.byref(b), None) == _lib.EMU_E_ARG
    b.hz = -0.01
    assert L.emu_bloch_fields_plane(C.byref(b), None) == _lib.EMU_E_ARG


def test_ring_entry_points_check_their_arguments_on_the_host():
    """The request-loop calls refuse a null ring and bad arguments with
    negative (poll) or positive (submit) statuses before any device work."""
    import ctypes as C
    from emustack_b200 import _lib
    L = _lib.lib()
    k = C.c_int(7)
    assert L.emu_film_ring_submit_many(None, None, 0, None, C.byref(k)) == _lib.EMU_E_ARG
    assert L.emu_film_ring_poll(None, 0, None) < 0
    assert L.emu_film_ring_poll_many(None, None, 0, None, None) < 0
    assert L.emu_film_ring_ready(None, 0) < 0
