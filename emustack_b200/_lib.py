"""ctypes binding of libemustack_gsm.so (declarations: include/emustack_gsm.h).

The CUDA library is the only compute path of this package: if it is missing
or cannot be loaded, every solve raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libemustack_gsm.so')

EMU_OK = 0
EMU_E_ARG = 1
EMU_E_SHAPE = 2
EMU_E_SINGULAR = 3
EMU_E_WORKSPACE = 5
STATUS_NAMES = {
    0: 'EMU_OK', 1: 'EMU_E_ARG', 2: 'EMU_E_SHAPE', 3: 'EMU_E_SINGULAR',
    4: 'EMU_E_NONFINITE', 5: 'EMU_E_WORKSPACE', 6: 'EMU_E_TIMEOUT',
    7: 'EMU_E_CUDA', 8: 'EMU_E_UNSUPPORTED',
}

POL = {'TE': 0, 'TM': 1, 'un': 2, 'R Circ': 3, 'L Circ': 4}
POL_INCOMING = -1

PT_WOOD_AIR = 1
PT_WOOD_LAYER = 2
PT_NO_PROP_SUB = 4
PT_NO_PROP_SUP = 8
PT_NONFINITE = 16

vp = C.c_void_p


class EmuFilmStackBatch(C.Structure):
    _fields_ = [
        ('n_points', C.c_int), ('n_layers', C.c_int), ('n_pw', C.c_int), ('world_1d', C.c_int),
        ('period', C.c_double), ('period_y', C.c_double),
        ('d_px', vp), ('d_py', vp), ('d_wl_nm', vp), ('d_k_pll', vp), ('d_n', vp),
        ('d_heights_nm', vp), ('heights_per_point', C.c_int), ('pol', C.c_int),
        ('d_incoming', vp), ('d_shears', vp), ('shear_ncoord', C.c_int),
        ('d_R_net', vp), ('d_T_net', vp), ('d_a_list', vp), ('d_t_list', vp), ('d_r_list', vp),
        ('d_flags', vp),
        ('d_kz', vp), ('d_layer_rt', vp), ('d_vec_coef_down', vp), ('d_vec_coef_up', vp),
        ('d_fluxes', vp), ('d_sort_order', vp), ('d_specular', vp), ('d_num_prop', vp),
        ('variant', C.c_int),
    ]

FILM_VARIANTS = (0, 1, 2, 3, 4, 5)


class EmuError(RuntimeError):
    def __init__(self, status, what=''):
        self.status = status
        super().__init__('%s failed: %s' % (what, STATUS_NAMES.get(status, status)))


_lib = None


def lib():
    """Load the CUDA library (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError('libemustack_gsm.so is not built (run emustack_b200.build.build_library()); '
                           'emustack_b200 has no CPU fallback')
    L = C.CDLL(LIB_PATH)
    L.emu_version.restype = C.c_int
    L.emu_status_string.restype = C.c_char_p
    L.emu_status_string.argtypes = [C.c_int]
    L.emu_launch_count.restype = C.c_longlong
    L.emu_set_dense_mode.restype = C.c_int
    L.emu_set_dense_mode.argtypes = [C.c_int]
    L.emu_grating_orders.restype = C.c_int
    L.emu_grating_orders.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, vp, vp, C.c_int,
                                     C.POINTER(C.c_int)]
    L.emu_film_stack_workspace_size.restype = C.c_size_t
    L.emu_film_stack_workspace_size.argtypes = [C.POINTER(EmuFilmStackBatch)]
    L.emu_film_stack_batch.restype = C.c_int
    L.emu_film_stack_batch.argtypes = [C.POINTER(EmuFilmStackBatch), vp, C.c_size_t, vp]
    _extra_signatures(L)
    _lib = L
    return L


def _extra_signatures(L):
    """Signatures of the entry points added beyond the film path."""
    for name, res, args in EXTRA_SIGNATURES:
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args


EXTRA_SIGNATURES = []


def check(status, what):
    if status != EMU_OK:
        raise EmuError(status, what)


def ptr(t):
    """Device (or host) address of a torch tensor, None for None."""
    return None if t is None else C.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class EmuAnalloModes(C.Structure):
    _fields_ = [
        ('n_points', C.c_int), ('n_pw', C.c_int), ('world_1d', C.c_int),
        ('period', C.c_double), ('period_y', C.c_double),
        ('d_px', vp), ('d_py', vp), ('d_wl_nm', vp), ('d_k_pll', vp), ('d_n', vp),
        ('d_sort_in', vp), ('d_kz', vp), ('d_alphas', vp), ('d_betas', vp),
        ('d_sort_out', vp), ('d_specular', vp), ('d_num_prop', vp), ('d_wood', vp),
    ]


EXTRA_SIGNATURES.append(('emu_anallo_modes', C.c_int, [C.POINTER(EmuAnalloModes), vp]))


class EmuLayer(C.Structure):
    _fields_ = [
        ('M', C.c_int), ('dense', C.c_int),
        ('d_R12', vp), ('d_T12', vp), ('d_R21', vp), ('d_T21', vp),
        ('stride_R12', C.c_longlong), ('stride_T12', C.c_longlong),
        ('stride_R21', C.c_longlong), ('stride_T21', C.c_longlong),
        ('d_kz', vp), ('stride_kz', C.c_longlong), ('height_norm', C.c_double),
        ('d_height_norm', vp),
    ]


class EmuStackDense(C.Structure):
    _fields_ = [
        ('batch', C.c_int), ('n_layers', C.c_int), ('P', C.c_int),
        ('h_layers', C.POINTER(EmuLayer)), ('h_shears', C.POINTER(C.c_double)),
        ('shear_ncoord', C.c_int), ('d_air_alphas', vp), ('d_air_betas', vp),
        ('calc_fluxes', C.c_int), ('pol', C.c_int), ('d_incoming', vp), ('d_specular', vp),
        ('d_num_prop', vp), ('d_R_net', vp), ('d_T_net', vp), ('d_fluxes', vp),
        ('d_a_list', vp), ('d_t_list', vp), ('d_r_list', vp), ('d_flags', vp), ('d_info', vp),
        ('d_vec_coef_down', vp), ('d_vec_coef_up', vp),
        ('vec_coef_down_stride', C.c_longlong), ('vec_coef_up_stride', C.c_longlong),
        ('save_lists', C.c_int), ('d_tnet_list', vp), ('d_rnet_list', vp),
        ('mode', C.c_int),
    ]


class EmuC128(C.Structure):
    _fields_ = [('re', C.c_double), ('im', C.c_double)]


EXTRA_SIGNATURES.extend([
    ('emu_zgemm_batched', C.c_int, [C.c_int, C.c_int, C.c_int, EmuC128, vp, C.c_int, C.c_longlong,
                                    vp, C.c_int, C.c_longlong, EmuC128, vp, C.c_int, C.c_longlong,
                                    C.c_int, vp]),
    ('emu_zgesv_batched', C.c_int, [C.c_int, C.c_int, vp, C.c_int, C.c_longlong, vp, vp, C.c_int,
                                    C.c_longlong, vp, C.c_int, vp]),
    ('emu_film_interface_batch', C.c_int, [C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]),
    ('emu_interface_dense_workspace_size', C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    ('emu_interface_dense_batch', C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp,
                                            vp, vp, vp, vp, C.c_size_t, vp]),
    ('emu_stack_dense_workspace_size', C.c_size_t, [C.POINTER(EmuStackDense)]),
    ('emu_stack_dense_list_stride', C.c_longlong, [C.POINTER(EmuStackDense)]),
    ('emu_stack_dense_batch', C.c_int, [C.POINTER(EmuStackDense), vp, C.c_size_t, vp]),
])


class EmuOverlap(C.Structure):
    _fields_ = [
        ('batch', C.c_int), ('nval', C.c_int), ('nel', C.c_int), ('npt', C.c_int),
        ('n_pw', C.c_int), ('max_order', C.c_int),
        ('d_px', vp), ('d_py', vp), ('d_x', vp), ('d_table_nod', vp),
        ('d', C.c_double), ('dy', C.c_double), ('d_bloch', vp), ('d_k0', vp),
        ('d_sol1', vp), ('d_sol2', vp), ('d_scale2', vp), ('d_perm2', vp),
        ('area_norm', C.c_double), ('d_J', vp), ('d_J_dag', vp), ('d_index_pw_inv', vp),
        ('elements_per_chunk', C.c_int), ('precision', C.c_int), ('d_error', vp),
        ('tc_splits', C.c_int), ('field_c64', C.c_int),
    ]


class EmuNormalise(C.Structure):
    _fields_ = [
        ('batch', C.c_int), ('nval', C.c_int), ('nel', C.c_int), ('npt', C.c_int),
        ('d_x', vp), ('d_table_nod', vp), ('d_type_el', vp), ('d_pp', vp), ('d_k0', vp),
        ('d_beta1', vp), ('d_sol1', vp), ('d_sol2', vp), ('d_diag', vp), ('d_scale', vp),
        ('d_n_small', vp),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_overlap_workspace_size', C.c_size_t, [C.POINTER(EmuOverlap)]),
    ('emu_overlap_batch', C.c_int, [C.POINTER(EmuOverlap), vp, C.c_size_t, vp]),
    ('emu_mode_overlap_workspace_size', C.c_size_t, [C.POINTER(EmuNormalise)]),
    ('emu_mode_overlap_diag', C.c_int, [C.POINTER(EmuNormalise), vp, C.c_size_t, vp]),
    ('emu_mode_overlap_reorder_workspace_size', C.c_size_t, [C.POINTER(EmuNormalise)]),
    ('emu_mode_overlap_reorder', C.c_int, [C.POINTER(EmuNormalise), vp, vp, vp, C.c_size_t, vp]),
    ('emu_tc_gemm_workspace_size', C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ('emu_tc_gemm_tf32x3', C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, vp, C.c_size_t, vp]),
])

PT_BAD_POINT = 32


class EmuFilmPoint(C.Structure):
    _fields_ = [
        ('n_layers', C.c_int32), ('n_pw', C.c_int32), ('world_1d', C.c_int32), ('pol', C.c_int32),
        ('order_off', C.c_int64), ('n_off', C.c_int64), ('h_off', C.c_int64),
        ('inc_off', C.c_int64), ('rt_off', C.c_int64), ('list_off', C.c_int64),
        ('np_off', C.c_int64), ('ws_off', C.c_int64),
        ('period', C.c_double), ('period_y', C.c_double), ('wl_nm', C.c_double),
        ('kx', C.c_double), ('ky', C.c_double),
    ]


class EmuFilmVarBatch(C.Structure):
    _fields_ = [
        ('n_points', C.c_int), ('max_layers', C.c_int), ('max_pw', C.c_int),
        ('d_points', vp), ('d_order', vp), ('d_px', vp), ('d_py', vp), ('d_n', vp),
        ('d_heights_nm', vp), ('d_incoming', vp), ('d_R_net', vp), ('d_T_net', vp),
        ('d_a_list', vp), ('d_t_list', vp), ('d_r_list', vp), ('d_flags', vp),
        ('d_specular', vp), ('d_num_prop', vp),
        ('order_len', C.c_int64), ('n_len', C.c_int64), ('h_len', C.c_int64),
        ('inc_len', C.c_int64), ('rt_len', C.c_int64), ('list_len', C.c_int64),
        ('np_len', C.c_int64), ('warps_per_cta', C.c_int), ('variant', C.c_int),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_film_var_plan', C.c_int, [vp, C.c_int, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ('emu_film_var_batch', C.c_int, [C.POINTER(EmuFilmVarBatch), vp, C.c_size_t, vp]),
])


class EmuVarLayer(C.Structure):
    _fields_ = [
        ('M', C.c_int), ('dense', C.c_int),
        ('d_R12', vp), ('d_T12', vp), ('d_R21', vp), ('d_T21', vp), ('d_kz', vp),
        ('height_norm', C.c_double),
    ]


class EmuStackPoint(C.Structure):
    _fields_ = [
        ('n_layers', C.c_int32), ('P', C.c_int32), ('pol', C.c_int32), ('spec', C.c_int32),
        ('num_prop', C.c_int32 * 3), ('_pad', C.c_int32),
        ('layer_off', C.c_int64), ('inc_off', C.c_int64), ('rnet_off', C.c_int64),
        ('tnet_off', C.c_int64), ('list_off', C.c_int64), ('flux_off', C.c_int64),
    ]


class EmuStackVarBatch(C.Structure):
    _fields_ = [
        ('n_stacks', C.c_int), ('d_points', vp), ('d_order', vp), ('d_layers', vp),
        ('n_layer_desc', C.c_int64),
        ('d_incoming', vp), ('incoming_len', C.c_int64),
        ('d_R_net', vp), ('rnet_len', C.c_int64),
        ('d_T_net', vp), ('tnet_len', C.c_int64),
        ('d_a_list', vp), ('d_t_list', vp), ('list_len', C.c_int64),
        ('d_fluxes', vp), ('flux_len', C.c_int64),
        ('d_r_list', vp), ('d_flags', vp), ('d_info', vp),
        ('max_P', C.c_int), ('max_D', C.c_int), ('max_L', C.c_int), ('n_slots', C.c_int),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_stack_var_slots', C.c_int, [C.POINTER(EmuStackVarBatch)]),
    ('emu_stack_var_workspace_size', C.c_size_t, [C.POINTER(EmuStackVarBatch)]),
    ('emu_stack_var_batch', C.c_int, [C.POINTER(EmuStackVarBatch), vp, C.c_size_t, vp]),
])


class EmuOverlap1D(C.Structure):
    _fields_ = [
        ('batch', C.c_int), ('nval', C.c_int), ('nel', C.c_int), ('npt', C.c_int),
        ('max_order', C.c_int), ('d_x', vp), ('d_table_nod', vp), ('period_x', C.c_double),
        ('d_bloch', vp), ('d_index_pw_inv', vp), ('d_sol1', vp), ('d_sol2', vp),
        ('d_scale', vp), ('d_perm2', vp), ('d_J', vp), ('d_J_dag', vp),
        ('npw_2d', C.c_int), ('d_row_2d', vp), ('d_J_2d', vp), ('d_J_dag_2d', vp), ('d_error', vp),
    ]


class EmuNormalise1D(C.Structure):
    _fields_ = [
        ('batch', C.c_int), ('nval', C.c_int), ('nel', C.c_int), ('npt', C.c_int),
        ('n_types', C.c_int), ('d_x', vp), ('d_table_nod', vp), ('d_type_el', vp), ('d_pp', vp),
        ('d_k0', vp), ('d_bloch', vp), ('d_beta1', vp), ('d_sol1', vp), ('d_sol2', vp),
        ('d_perm2', vp), ('d_out', vp), ('d_scale', vp), ('d_n_small', vp), ('d_error', vp),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_pw_order_1d', C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, vp]),
    ('emu_pw_embed_1d_to_2d', C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, vp,
                                        C.c_int, C.POINTER(C.c_int)]),
    ('emu_overlap1d_batch', C.c_int, [C.POINTER(EmuOverlap1D), vp]),
    ('emu_mode_overlap_1d', C.c_int, [C.POINTER(EmuNormalise1D), C.c_int, vp]),
])


MAT_CONSTANT, MAT_TABLE, MAT_DRUDE, MAT_TABLE_REAL = 0, 1, 2, 3


class EmuMaterial(C.Structure):
    _fields_ = [
        ('kind', C.c_int), ('n_rows', C.c_int), ('d_wl', vp), ('d_n', vp), ('n_const', EmuC128),
        ('drude', C.c_double * 3), ('loss', C.c_int),
    ]


EXTRA_SIGNATURES.append(('emu_material_n_batch', C.c_int, [C.POINTER(EmuMaterial), C.c_int, C.c_int, vp, vp,
                                                           vp, vp]))


class EmuFilmRingRequest(C.Structure):
    _fields_ = [
        ('n_layers', C.c_int), ('n_pw', C.c_int), ('world_1d', C.c_int), ('pol', C.c_int),
        ('period', C.c_double), ('period_y', C.c_double), ('wl_nm', C.c_double), ('k_pll', C.c_double * 2),
        ('h_px', vp), ('h_py', vp), ('h_n', vp), ('h_heights_nm', vp),
    ]


class EmuFilmRingResult(C.Structure):
    _fields_ = [('h_R_net', vp), ('h_T_net', vp), ('h_a_list', vp), ('h_t_list', vp), ('h_r_list', vp),
                ('h_flags', vp)]


RING_MAX_PW, RING_MAX_LAYERS = 512, 16

EXTRA_SIGNATURES.extend([
    ('emu_film_ring_slot_bytes', C.c_size_t, []),
    ('emu_film_ring_create', C.c_int, [C.c_int, C.c_double, C.POINTER(vp)]),
    ('emu_film_ring_submit', C.c_int, [vp, C.POINTER(EmuFilmRingRequest), C.POINTER(C.c_longlong)]),
    ('emu_film_ring_poll', C.c_int, [vp, C.c_longlong, C.POINTER(EmuFilmRingResult)]),
    ('emu_film_ring_submit_many', C.c_int, [vp, vp, C.c_int, vp, C.POINTER(C.c_int)]),
    ('emu_film_ring_poll_many', C.c_int, [vp, vp, C.c_int, vp, vp]),
    ('emu_film_ring_wait', C.c_int, [vp, C.c_longlong, C.c_double, C.POINTER(EmuFilmRingResult)]),
    ('emu_film_ring_ready', C.c_int, [vp, C.c_longlong]),
    ('emu_film_ring_running', C.c_int, [vp]),
    ('emu_film_ring_stop', C.c_int, [vp]),
    ('emu_film_ring_destroy', C.c_int, [vp]),
])


class EmuPwFields(C.Structure):
    _fields_ = [
        ('n_stacks', C.c_int), ('n_pw', C.c_int), ('substrate', C.c_int), ('grid', C.c_int),
        ('nx', C.c_int), ('ny', C.c_int), ('nz', C.c_int),
        ('d_alphas', vp), ('d_betas', vp), ('d_sort', vp), ('d_kz', vp), ('d_n', vp), ('d_height', vp),
        ('d_vec_coef_down', vp), ('d_vec_coef_up', vp), ('vcd_stride', C.c_longlong),
        ('vcu_stride', C.c_longlong), ('d_x', vp), ('d_y', vp), ('d_z', vp), ('d_E', vp), ('d_E_abs', vp),
        ('d_workspace', vp), ('workspace_bytes', C.c_size_t),
    ]


class EmuBlochFieldsPlane(C.Structure):
    _fields_ = [
        ('n_stacks', C.c_int), ('n_modes', C.c_int), ('n_elements', C.c_int), ('d_sol', vp),
        ('sol_stride', C.c_longlong), ('d_k_z', vp), ('d_vec_coef', vp), ('h', C.c_double),
        ('hz', C.c_double), ('d_E', vp),
    ]


PW_FIELDS_MAX_ORDERS = 1536

EXTRA_SIGNATURES.extend([
    ('emu_pw_fields_workspace_size', C.c_size_t, [C.POINTER(EmuPwFields)]),
    ('emu_pw_fields', C.c_int, [C.POINTER(EmuPwFields), vp]),
    ('emu_bloch_fields_plane', C.c_int, [C.POINTER(EmuBlochFieldsPlane), vp]),
])


class EmuFemTopology(C.Structure):
    _fields_ = [
        ('npt', C.c_int), ('nel', C.c_int), ('h_x', vp), ('h_type_nod', vp), ('h_table_nod', vp),
        ('h_dof', vp), ('h_shift', vp), ('h_ends', vp), ('h_row_ptr', vp), ('h_col', vp),
        ('h_src_ptr', vp), ('h_src', vp), ('neq', C.c_int), ('nnz', C.c_int),
    ]


class EmuFemElements(C.Structure):
    _fields_ = [
        ('nel', C.c_int), ('n_types', C.c_int), ('d_x', vp), ('d_table_nod', vp), ('d_type_el', vp),
        ('d_shift', vp), ('d_ends', vp), ('n_eff', EmuC128 * 8), ('k0', C.c_double),
        ('bloch', C.c_double * 2), ('d_Ke', vp), ('d_Me', vp),
    ]


class EmuFemFields(C.Structure):
    _fields_ = [
        ('nel', C.c_int), ('neq', C.c_int), ('nval', C.c_int), ('d_x', vp), ('d_table_nod', vp),
        ('d_shift', vp), ('d_ends', vp), ('d_dof', vp), ('bloch', C.c_double * 2), ('d_vec', vp),
        ('ldv', C.c_int), ('d_sol', vp),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_fem_topology', C.c_int, [C.POINTER(EmuFemTopology)]),
    ('emu_fem_element_matrices', C.c_int, [C.POINTER(EmuFemElements), vp]),
    ('emu_fem_assemble', C.c_int, [C.c_int, vp, vp, vp, vp, vp, vp, vp]),
    ('emu_fem_shifted_dense', C.c_int, [C.c_int, vp, vp, vp, vp, EmuC128, vp, C.c_int, vp]),
    ('emu_fem_lu', C.c_int, [C.c_int, vp, C.c_int, vp, vp, vp]),
    ('emu_fem_inverse', C.c_int, [C.c_int, vp, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp]),
    ('emu_fem_apply_op', C.c_int, [C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_int, vp, vp,
                                   C.c_int, vp]),
    ('emu_fem_mode_order', C.c_int, [C.c_int, vp, vp]),
    ('emu_fem_fields_workspace_size', C.c_size_t, [C.POINTER(EmuFemFields)]),
    ('emu_fem_nodal_fields', C.c_int, [C.POINTER(EmuFemFields), vp, C.c_size_t, vp]),
])


class EmuFem1dTopology(C.Structure):
    _fields_ = [
        ('npt', C.c_int), ('nel', C.c_int), ('h_x', vp), ('h_table_nod', vp), ('h_dof', vp), ('h_shift', vp),
        ('h_row_ptr', vp), ('h_col', vp), ('h_src_ptr', vp), ('h_src', vp), ('neq', C.c_int), ('nnz', C.c_int),
        ('period', C.c_double),
    ]


class EmuFem1dElements(C.Structure):
    _fields_ = [
        ('nel', C.c_int), ('n_types', C.c_int), ('d_x', vp), ('d_table_nod', vp), ('d_type_el', vp),
        ('d_shift', vp), ('n_eff', EmuC128 * 8), ('k0', C.c_double), ('bloch', C.c_double * 2),
        ('d_Ke', vp), ('d_Me', vp),
    ]


class EmuFem1dFields(C.Structure):
    _fields_ = [
        ('nel', C.c_int), ('neq', C.c_int), ('nval', C.c_int), ('d_x', vp), ('d_table_nod', vp),
        ('d_shift', vp), ('d_dof', vp), ('bloch_x', C.c_double), ('adjoint', C.c_int), ('d_vec', vp),
        ('ldv', C.c_int), ('d_sol', vp),
    ]


EXTRA_SIGNATURES.extend([
    ('emu_fem1d_topology', C.c_int, [C.POINTER(EmuFem1dTopology)]),
    ('emu_fem1d_element_matrices', C.c_int, [C.POINTER(EmuFem1dElements), vp]),
    ('emu_fem1d_fields_workspace_size', C.c_size_t, [C.POINTER(EmuFem1dFields)]),
    ('emu_fem1d_nodal_fields', C.c_int, [C.POINTER(EmuFem1dFields), vp, C.c_size_t, vp]),
])
