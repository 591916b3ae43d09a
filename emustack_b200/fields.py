"""Fields reconstructed from the GSM amplitudes, and the spectra / reference
data writers (mirror of the data side of backend/plotting.py and of
tests/testing.py).

Device entry points (libemustack_gsm.so):

* ``pw_fields`` -- E inside a homogeneous layer from its plane-wave
  amplitudes, for a batch of solved stacks, at points or on a grid
  (emu_pw_fields: the arithmetic of field_values, backend/plotting.py:
  2857-2996, and of the ThinFilm branch of fields_in_plane, 1759-1833);
* ``bloch_fields_plane`` -- E at the P2 nodes of a 2D nanostructured layer
  from its Bloch-mode amplitudes (emu_bloch_fields_plane: field_value_plane,
  backend/fortran/field_value_plane.f:6-132).

Reference-facing functions with the reference's names and arguments:
``field_values``, ``fields_in_plane``, ``fields_vertically``, ``t_r_a_write_files``,
``layers_print``, ``zeros_int_str``, ``save_reference_data``.  They write the
reference's data files (.txt / .npz, same names and formats); figures
(matplotlib PDFs) and gmsh files are not produced -- ``fields_in_plane``
saves the field arrays it would have plotted as .npz instead.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError('emustack_b200 needs a CUDA device (no CPU fallback)')
    return torch.device('cuda', torch.cuda.current_device())


def _t(a, dtype, dev):
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)


# ------------------------------------------------------------ device calls
def pw_fields(alphas, betas, sort_order, kz, n, vec_coef_down, vec_coef_up, x, y, z,
              height_norm=None, substrate=False, grid=False, stream=None):
    """E inside one homogeneous layer of B solved stacks.

    alphas, betas, sort_order, kz: [B, Npw] (unsorted alphas / betas as
    ``Anallo.alphas`` / ``betas`` hold them, betas repeated for 1D worlds;
    the air reference's sort order; the sorted k_z); n: [B] complex (loss
    flag applied); vec_coef_down / vec_coef_up: [B, 2 Npw] (TE then TM) or
    vec_coef_up None; height_norm: [B] heights / period, None or 0 for a
    semi-infinite layer; substrate: layer 0 (z -> -z, no up amplitudes).
    x, y, z in units of the period: points (grid False, equal lengths Q) or
    the axes of a grid (Q = nx ny nz, [x][y][z] order).

    Returns (E [B, 3, Q] complex128, |E| [B, Q] float64) on the device."""
    dev = _dev()
    f64, c128 = torch.float64, torch.complex128
    alphas = _t(alphas, f64, dev)
    if alphas.dim() == 1:
        alphas = alphas[None]
    B, S = alphas.shape
    if S > _lib.PW_FIELDS_MAX_ORDERS:
        raise ValueError('at most %d orders per polarisation' % _lib.PW_FIELDS_MAX_ORDERS)
    betas = _t(betas, f64, dev).reshape(B, -1)
    if betas.shape[1] == 1:
        betas = betas.expand(B, S).contiguous()
    sort_order = _t(sort_order, torch.int32, dev).reshape(B, S)
    kz = _t(kz, c128, dev).reshape(B, S)
    n = _t(n, c128, dev).reshape(B)
    vcd = _t(vec_coef_down, c128, dev).reshape(B, 2 * S)
    vcu = None if (vec_coef_up is None or substrate) else _t(vec_coef_up, c128, dev).reshape(B, 2 * S)
    h = None if height_norm is None else _t(height_norm, f64, dev).reshape(-1).expand(B).contiguous()
    x, y, z = (_t(v, f64, dev).reshape(-1) for v in (x, y, z))
    if grid:
        Q = x.numel() * y.numel() * z.numel()
    else:
        if not (x.numel() == y.numel() == z.numel()):
            raise ValueError('points need equal numbers of x, y and z')
        Q = x.numel()
    E = torch.empty((B, 3, Q), dtype=c128, device=dev)
    Eabs = torch.empty((B, Q), dtype=f64, device=dev)
    d = _lib.EmuPwFields()
    d.n_stacks, d.n_pw, d.substrate, d.grid = B, S, int(bool(substrate)), int(bool(grid))
    d.nx, d.ny, d.nz = x.numel(), (y.numel() if grid else 0), (z.numel() if grid else 0)
    d.d_alphas, d.d_betas, d.d_sort, d.d_kz, d.d_n = ptr(alphas), ptr(betas), ptr(sort_order), ptr(kz), ptr(n)
    d.d_height = ptr(h)
    d.d_vec_coef_down, d.vcd_stride = ptr(vcd), 2 * S
    d.d_vec_coef_up, d.vcu_stride = ptr(vcu), 2 * S
    d.d_x, d.d_y, d.d_z = ptr(x), ptr(y), ptr(z)
    d.d_E, d.d_E_abs = ptr(E), ptr(Eabs)
    ws = None
    nbytes = lib().emu_pw_fields_workspace_size(C.byref(d))
    if nbytes:
        ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        d.d_workspace, d.workspace_bytes = ptr(ws), nbytes
    check(lib().emu_pw_fields(C.byref(d), stream_ptr(stream)), 'emu_pw_fields')
    return E, Eabs


def bloch_fields_plane(sol, k_z, vec_coef, h_norm, hz_norm, stream=None):
    """m_E[b, el, node, component] at the six P2 nodes of every element of a
    2D nanostructured layer, at the plane hz_norm (from the top of the
    layer, units of the period; 0 <= hz_norm <= h_norm).

    sol: [B, nel, M, 13, 3] or [nel, M, 13, 3] complex128 (Fortran
    sol(3, 13, M, nel)); k_z: [B, M]; vec_coef: [B, 2M] (vec_coef_down then
    vec_coef_up of the layer).  Returns a device tensor [B, nel, 6, 3]."""
    dev = _dev()
    c128 = torch.complex128
    sol = _t(sol, c128, dev)
    if sol.dim() == 4:
        sol = sol[None]
    if sol.dim() != 5 or tuple(sol.shape[3:]) != (13, 3):
        raise ValueError('sol must be [B, nel, M, 13, 3]')
    B, nel, M = sol.shape[:3]
    k_z = _t(k_z, c128, dev).reshape(B, M)
    vc = _t(vec_coef, c128, dev).reshape(B, 2 * M)
    if not (0.0 <= float(hz_norm) <= float(h_norm)):
        raise ValueError('field_value_plane: hz should be in the interval [0, h]')
    E = torch.empty((B, nel, 6, 3), dtype=c128, device=dev)
    d = _lib.EmuBlochFieldsPlane()
    d.n_stacks, d.n_modes, d.n_elements = B, M, nel
    d.d_sol, d.sol_stride = ptr(sol), nel * M * 39
    d.d_k_z, d.d_vec_coef = ptr(k_z), ptr(vc)
    d.h, d.hz = float(h_norm), float(hz_norm)
    d.d_E = ptr(E)
    check(lib().emu_bloch_fields_plane(C.byref(d), stream_ptr(stream)), 'emu_bloch_fields_plane')
    return E


def film_batch_fields(solver, out, k_pll, n, layer, x, y, z, heights_nm=None, grid=False, stream=None):
    """Fields in one layer of every point of a batched all-film solve
    (``FilmStackSolver.solve(..., want=('kz', 'vec_coef', 'sort_order'))``):
    out is that call's outputs, k_pll [B, 2] (nm^-1) and n [B, L] its
    inputs, heights_nm [L-2] or [B, L-2] (nm).  The orders' alphas and betas
    are formed on the device as Anallo.calc_kz forms them
    (backend/mode_calcs.py:131-140).  Points flagged with a Wood anomaly
    (their orders were shifted by 1e-9 in the solve) are refused."""
    dev = solver.device
    for k in ('kz', 'vec_coef_down', 'vec_coef_up', 'sort_order'):
        if k not in out:
            raise ValueError("the solve needs want=('kz', 'vec_coef', 'sort_order')")
    flags = out['flags']
    if bool(((flags & (_lib.PT_WOOD_AIR | _lib.PT_WOOD_LAYER)) != 0).any()):
        raise ValueError('points with a Wood anomaly are not supported; drop them from the batch')
    L = solver.L
    if not 0 <= layer < L:
        raise ValueError('layer out of range')
    B = out['kz'].shape[0]
    kp = _t(k_pll, torch.float64, dev).reshape(B, 2) * solver.period
    two_pi = 2 * np.pi
    alphas = kp[:, 0:1] + solver.d_px.to(torch.float64)[None] * two_pi
    dy = solver.period_y / solver.period
    if solver.world_1d:
        betas = kp[:, 1:2].expand(B, solver.npw)
    else:
        betas = kp[:, 1:2] + solver.d_py.to(torch.float64)[None] * two_pi / dy
    row = L - 1 - layer
    h = None
    if 0 < layer < L - 1:
        hs = _t(heights_nm, torch.float64, dev)
        h = (hs[..., layer - 1] if hs.dim() == 2 else hs[layer - 1].expand(B)) / solver.period
    nn = _t(n, torch.complex128, dev).reshape(B, L)[:, layer]
    return pw_fields(alphas.contiguous(), betas.contiguous(), out['sort_order'], out['kz'][:, layer], nn,
                     out['vec_coef_down'][:, row], None if layer == 0 else out['vec_coef_up'][:, row],
                     x, y, z, height_norm=h, substrate=(layer == 0), grid=grid, stream=stream)


# ------------------------------------------------- stack-level helpers
def _layer_pw_inputs(pstack, lay_interest):
    """The film layer's order data and amplitudes, as the reference reads
    them (backend/plotting.py:2890-2913)."""
    lay = pstack.layers[lay_interest]
    num_lays = len(pstack.layers)
    S = int(lay.structure.num_pw_per_pol)
    kz = np.asarray(lay.k_z)[:S]
    betas = np.atleast_1d(np.asarray(lay.betas, float))
    if betas.size == 1:
        betas = np.full(S, betas[0])
    vcd = np.asarray(pstack.vec_coef_down[num_lays - 1 - lay_interest]).ravel()
    vcu = None if lay_interest == 0 else np.asarray(pstack.vec_coef_up[num_lays - 1 - lay_interest]).ravel()
    h = lay.structure.height_nm
    h_norm = None if h == 'semi_inf' else float(h) / float(pstack.layers[-1].structure.period)
    return dict(alphas=np.asarray(lay.alphas, float), betas=betas, sort_order=np.asarray(lay.sort_order),
                kz=kz, n=complex(np.asarray(lay.n()).item()), vec_coef_down=vcd, vec_coef_up=vcu,
                height_norm=h_norm, substrate=(lay_interest == 0))


def _is_film(lay):
    from .mode_calcs import is_film
    return is_film(lay)


def layer_fields(pstack, lay_interest, x, y, z, grid=False):
    """E (3 complex arrays) and |E| in a film layer of one solved stack at
    points / on a grid in units of the period (see pw_fields)."""
    a = _layer_pw_inputs(pstack, lay_interest)
    if a['height_norm'] is None:
        a['height_norm'] = 0.0
    E, Eabs = pw_fields(x=x, y=y, z=z, grid=grid, **a)
    E, Eabs = E[0].cpu().numpy(), Eabs[0].cpu().numpy()
    if grid:
        shape = (np.size(x), np.size(y), np.size(z))
        return tuple(e.reshape(shape) for e in E), Eabs.reshape(shape)
    return tuple(E), Eabs


def field_values(stacks_list, lay_interest=0, xyz_values=[(0.1, 0.1, 0.1)]):
    """Electric field at x-y-z points (units of the period) inside a ThinFilm
    layer, saved as field_values/<stack>_E_calc_points_<layer>_wl_<wl>.npz
    and .txt (rows Re Ex, Im Ex, Re Ey, Im Ey, Re Ez, Im Ez, |E|), as
    backend/plotting.py:2857-2996 saves them.  z is the distance from the
    top of the layer below (into the substrate for lay_interest 0).

    Returns [[E_x, E_y, E_z, E_tot], ...].  Every stack of the list is
    evaluated (the reference returns after the first one)."""
    dir_name = 'field_values'
    if not os.path.exists(dir_name):
        os.mkdir(dir_name)
    super_points = []
    for stack_num, pstack in enumerate(stacks_list):
        lay = pstack.layers[lay_interest]
        if not _is_film(lay):
            print("field_values can only calculate field values in ThinFilms."
                  "\nPlease select a different lay_interest.\n")
            continue
        num_lays = len(pstack.layers)
        wl = np.around(pstack.layers[-1].light.wl_nm, decimals=2)
        if lay_interest == 0:
            name_lay = "0_Substrate"
        elif lay_interest == num_lays - 1:
            name_lay = "%i_Superstrate" % (num_lays - 1)
        else:
            name_lay = "%i_Thin_Film" % lay_interest
        xyz = np.asarray(xyz_values, dtype=float).reshape(-1, 3).copy()
        if lay.structure.world_1d is True:
            xyz[:, 1] = 0.0
        (Ex, Ey, Ez), Eabs = layer_fields(pstack, lay_interest, xyz[:, 0], xyz[:, 1], xyz[:, 2])
        Etot = Eabs.astype(complex)
        base = '%(dir_name)s/%(stack_num)s_E_calc_points_%(name)s_wl_%(wl)s' % {
            'dir_name': dir_name, 'wl': wl, 'name': name_lay, 'stack_num': stack_num}
        np.savez(base, calc_E_x_array=Ex, calc_E_y_array=Ey, calc_E_z_array=Ez, calc_E_tot_array=Etot)
        np.savetxt(base + '.txt', np.array([Ex.real, Ex.imag, Ey.real, Ey.imag, Ez.real, Ez.imag, Etot.real]))
        super_points.append([Ex, Ey, Ez, Etot])
    return super_points


def fields_in_plane(stacks_list, lay_interest=1, z_values=[0.1, 3.6], nu_calc_pts=51):
    """Fields in x-y planes at heights z_values (nm from the bottom of the
    layer; from the top of the substrate into it for lay_interest 0), on a
    nu_calc_pts^2 grid over the unit cell (backend/plotting.py:1663-1941).

    Film layers: E_x, E_y, E_z, |E| arrays indexed [x, y, z] (the arrays the
    reference contours), saved to in_plane_fields/stack_<n>_E_<layer>_wl=<wl>.npz.
    2D nanostructured layers: m_E [nel, 6, 3] at each z (the values the
    reference writes to gmsh), saved to in_plane_fields/stack_<n>_E_<layer>_slice=<z>.npz.
    Returns one dict per stack."""
    dir_name = "in_plane_fields"
    if not os.path.exists(dir_name):
        os.mkdir(dir_name)
    if nu_calc_pts % 2 == 0:
        nu_calc_pts += 1
    out = []
    for stack_num, pstack in enumerate(stacks_list):
        lay = pstack.layers[lay_interest]
        num_lays = len(pstack.layers)
        zs = np.array(z_values, dtype=float) / float(lay.structure.period)
        if not _is_film(lay):
            if getattr(lay.structure, 'periodicity', '2D_array') != '2D_array':
                print("fields_in_plane cannot plot fields in 1D-arrays."
                      "\nPlease select a different lay_interest.\n")
                continue
            sol = getattr(lay, 'sol1', None)
            if sol is None:
                raise ValueError('the nanostructured layer carries no Bloch-mode fields (sol1)')
            h_normed = float(lay.structure.height_nm) / float(lay.structure.period)
            vec_index = num_lays - lay_interest - 1
            vc = np.concatenate((np.asarray(pstack.vec_coef_down[vec_index]).ravel(),
                                 np.asarray(pstack.vec_coef_up[vec_index]).ravel()))
            res = {}
            for zv in zs:
                mE = bloch_fields_plane(sol, np.asarray(lay.k_z)[None], vc[None], h_normed,
                                        h_normed - zv)[0].cpu().numpy()
                res[float(zv)] = mE
                np.savez('%s/stack_%s_E_Lay%s_slice=%s.npz' % (dir_name, stack_num, zeros_int_str(lay_interest),
                                                                zv), m_E=mE)
            out.append(res)
            continue
        wl = np.around(pstack.layers[-1].light.wl_nm, decimals=2)
        if lay_interest == 0:
            name_lay = "0_Substrate"
        elif lay_interest == num_lays - 1:
            name_lay = "%(i)s_Superstrate" % {'i': num_lays - 1}
        else:
            name_lay = "Thin_Film_%(i)s" % {'i': lay_interest}
        h = lay.structure.height_nm
        if h != 'semi_inf' and lay_interest != 0 and np.any(np.abs(zs) > float(h) / float(lay.structure.period)):
            raise ValueError("fields_in_plane: z_value exceeds thickness of layer, reduce it. ")
        r = np.linspace(0.0, 1.0, nu_calc_pts)
        (Ex, Ey, Ez), Eabs = layer_fields(pstack, lay_interest, r, r, zs, grid=True)
        res = {'x': r, 'y': r, 'z': zs, 'E_x': Ex, 'E_y': Ey, 'E_z': Ez, 'E_abs': Eabs}
        np.savez('%(d)s/stack_%(n)s_E_%(name)s_wl=%(wl)s.npz' % {'d': dir_name, 'n': stack_num, 'name': name_lay,
                                                                 'wl': wl}, **res)
        out.append(res)
    return out


# E_y / E_z at an element's middle from its four P3 values (array_sol_P2_1d.f:20-40)
_P3_MID = (-1.0 / 16.0, -1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0)


def grating_slice_1d(sol1, k_z, vec_coef, h_norm, z_range):
    """E_x, E_y, E_z [2 nel + 1][nz] on the x-z slice through a 1D grating
    layer from its Bloch-mode nodal values ``sol1`` ([nel][M][11], device or
    host) and amplitudes ``vec_coef`` (2M, down then up), as fields_vertically
    builds it (backend/plotting.py:2244-2282 with array_sol_P2_1d.f): per
    element the P2 values (x_min, x_max, middle) placed at slice entries 0
    (first element's x_min), 2e + 1 (x_max) and 2e + 2 (middle), and each
    mode weighted by vec_coef_down e^{i beta (h - z)} + vec_coef_up e^{i beta z}
    (E_z: their difference over beta).  One GEMM per component on the GPU."""
    dev = torch.device('cuda', torch.cuda.current_device())
    s = sol1 if isinstance(sol1, torch.Tensor) else torch.as_tensor(np.asarray(sol1, np.complex128))
    s = s.to(device=dev, dtype=torch.complex128)
    nel, M = s.shape[0], s.shape[1]
    beta = np.asarray(k_z, np.complex128).ravel()
    vc = np.asarray(vec_coef, np.complex128).ravel()
    z = np.asarray(z_range, np.float64).ravel()
    cd = vc[:M, None] * np.exp(1j * beta[:, None] * (h_norm - z[None, :]))
    cu = vc[M:, None] * np.exp(1j * beta[:, None] * z[None, :])
    coef_t = torch.as_tensor(cu + cd, device=dev)
    coef_z = torch.as_tensor((cu - cd) / beta[:, None], device=dev)
    w = torch.tensor(_P3_MID, dtype=torch.complex128, device=dev)
    out = []
    for comp in range(3):
        if comp == 0:
            p2 = s[:, :, 0:3]
        else:
            lo = 3 if comp == 1 else 7
            p2 = torch.stack([s[:, :, lo], s[:, :, lo + 1], s[:, :, lo:lo + 4] @ w], dim=2)
        nodes = torch.empty((2 * nel + 1, M), dtype=torch.complex128, device=dev)
        nodes[0] = p2[0, :, 0]
        nodes[1::2] = p2[:, :, 1]
        nodes[2::2] = p2[:, :, 2]
        out.append((nodes @ (coef_z if comp == 2 else coef_t)).cpu().numpy())
    return tuple(out)


def fields_vertically(stacks_list, factor_pts_vert=31, nu_pts_hori=41, semi_inf_height=1.0, gradient=None,
                      no_incoming=False, add_name='', force_eq_ratio=False, colour_res=30, plot_boundaries=True):
    """Fields on the x-z slice (y = 0) through every ThinFilm layer of each
    stack, on the grids of backend/plotting.py:2074-2856: nu_pts_hori x
    points over the cell, round(factor_pts_vert Re(eps) h / wl) z points per
    layer (at least 11), semi_inf_height (units of the period) into the
    substrate and superstrate; no_incoming drops the incident field in the
    superstrate.  Saved to fields_vertically/stack_<n><add_name>.npz (for
    layer i: E_x_<i>, E_y_<i>, E_z_<i> [x, z], z_<i> on the stack's height
    axis, x) and returned as one dict per stack.  1D gratings whose Bloch-mode
    fields are known (``sol1``, from calc_modes) give their slice on the
    mesh's nodes as the routine assembles it (grating_slice_1d; x_<i> the
    node coordinates); 2D nanostructured layers (gmsh files in the
    reference) are skipped; the plotting arguments are accepted for
    compatibility and not used."""
    dir_name = "fields_vertically"
    if not os.path.exists(dir_name):
        os.mkdir(dir_name)
    if nu_pts_hori % 2 == 0:
        nu_pts_hori += 1
    out = []
    for stack_num, pstack in enumerate(stacks_list):
        num_lays = len(pstack.layers)
        wl_normed = pstack.layers[0].wl_norm()
        ind_h_list = list(pstack.heights_norm())
        h_list = [-semi_inf_height, 0]
        for h in ind_h_list:
            h_list.append(h_list[-1] + h)
        h_list.append(h_list[-1] + semi_inf_height)
        ind_h_list.append(semi_inf_height)
        ind_h_list.insert(0, semi_inf_height)
        x_range = np.linspace(0.0, 1.0, nu_pts_hori)
        res = {'x': x_range}
        for lay in range(num_lays):
            layer = pstack.layers[lay]
            if not _is_film(layer):
                st = getattr(layer, 'structure', None)
                sol1 = getattr(layer, 'sol1', None)
                if (getattr(st, 'periodicity', None) == '1D_array' and sol1 is not None
                        and getattr(st, 'mesh', None) is not None):
                    eps = np.asarray(getattr(layer, 'n_effs', [1.0])) ** 2
                    nz = max(int(np.round(factor_pts_vert * (np.real(np.max(eps)) * ind_h_list[lay] / wl_normed))),
                             11)
                    z_range = np.linspace(0.0, ind_h_list[lay], nz)
                    vi = num_lays - lay - 1
                    vc = np.concatenate([np.asarray(pstack.vec_coef_down[vi]).ravel(),
                                         np.asarray(pstack.vec_coef_up[vi]).ravel()])
                    ex, ey, ez = grating_slice_1d(sol1, layer.k_z, vc, ind_h_list[lay], z_range)
                    res['E_x_%d' % lay], res['E_y_%d' % lay], res['E_z_%d' % lay] = ex, ey, ez
                    xm = np.sort(np.asarray(st.mesh.x, float))
                    res['x_%d' % lay] = (xm - xm[0]) / (xm[-1] - xm[0])
                    res['z_%d' % lay] = np.linspace(h_list[lay], h_list[lay + 1], nz)
                continue
            eps = np.asarray(layer.n()) ** 2
            nz = int(np.round(factor_pts_vert * (np.real(np.max(eps)) * ind_h_list[lay] / wl_normed)))
            nz = max(nz, 11)
            if lay == 0:
                z_range = np.linspace(h_list[lay], 0.0, nz)
            else:
                z_range = np.linspace(0.0, ind_h_list[lay], nz)
            a = _layer_pw_inputs(pstack, lay)
            if lay == num_lays - 1 and no_incoming:
                a['vec_coef_down'] = np.zeros_like(a['vec_coef_down'])
            if a['height_norm'] is None:
                a['height_norm'] = 0.0
            # the routine's z below the stack is negative; the kernel takes the
            # distance into the substrate
            zk = -z_range if lay == 0 else z_range
            E, _ = pw_fields(x=x_range, y=np.zeros(1), z=zk, grid=True, **a)
            E = E[0].cpu().numpy().reshape(3, nu_pts_hori, 1, nz)[:, :, 0, :]
            res['E_x_%d' % lay], res['E_y_%d' % lay], res['E_z_%d' % lay] = E[0], E[1], E[2]
            res['z_%d' % lay] = np.linspace(h_list[lay], 0.0 if lay == 0 else h_list[lay + 1], nz)
        np.savez('%s/stack_%d%s.npz' % (dir_name, stack_num, add_name), **res)
        out.append(res)
    return out


# ------------------------------------------------------------- writers
def zeros_int_str(zero_int):
    """Integer as a 4-character string with '0' for ' ' (backend/plotting.py:69-78)."""
    string = '%4.0f' % zero_int
    return string.replace(' ', '0')


def t_r_a_write_files(stacks_list, wavelengths, stack_label=1, add_name=''):
    """Save t, r, a of each layer and the totals in text files
    (backend/plotting.py:735-775): Lay_Absorb_<i>_stack<label>.txt ...,
    Absorptance_stack<label>.txt, Transmittance_..., Reflectance_..., each
    row 'wavelength value total_height' in '%18.11f'."""
    stack_label = zeros_int_str(stack_label)
    a_list, t_list, r_list = [], [], []
    for stack in stacks_list:
        a_list.extend(stack.a_list)
        t_list.extend(stack.t_list)
        r_list.extend(stack.r_list)
    total_h = sum(stacks_list[0].heights_nm())
    layers_print('Lay_Absorb', a_list, wavelengths, total_h, stack_label)
    layers_print('Lay_Trans', t_list, wavelengths, total_h, stack_label)
    layers_print('Lay_Reflec', r_list, wavelengths, total_h, stack_label)


def layers_print(spectra_name, spec_list, wavelengths, total_h, stack_label=1, add_name=''):
    """One text file per layer and one for the total
    (backend/plotting.py:778-809)."""
    nu_layers = int(len(spec_list) / len(wavelengths))
    h_array = np.ones(len(wavelengths)) * total_h
    names = {'Lay_Absorb': 'Absorptance', 'Lay_Trans': 'Transmittance', 'Lay_Reflec': 'Reflectance'}
    for i in range(nu_layers):
        layer_spec = np.array([float(np.real(np.asarray(spec_list[wl * nu_layers + i])).ravel()[0])
                               for wl in range(len(wavelengths))])
        av_array = list(zip(wavelengths, layer_spec, h_array))
        if i != nu_layers - 1:
            np.savetxt('%(s)s_%(i)i_stack%(bon)s%(add)s.txt' % {'s': spectra_name, 'i': i, 'bon': stack_label,
                                                               'add': add_name}, av_array, fmt='%18.11f')
        else:
            np.savetxt('%(s)s_stack%(bon)s%(add)s.txt' % {'s': names[spectra_name], 'bon': stack_label,
                                                         'add': add_name}, av_array, fmt='%18.11f')


def save_reference_data(casefile_name, stack_list, directory='ref'):
    """Save each stack's layer matrices (R12, T12, R21, T21, k_z) and net
    R_net / T_net to <directory>/<casefile_name>.npz in the layout of
    tests/testing.py:7-24 (an object array of dicts under 'stack_list');
    returns the path.  (The reference also copies *.txt there and then fails
    the calling test on purpose; neither is done here.)"""
    ref_stack_list = []
    for stack in stack_list:
        rstack = {'layers': []}
        for lay in stack.layers:
            rstack['layers'].append({k: getattr(lay, k) for k in ('R12', 'T12', 'R21', 'T21', 'k_z')})
        rstack['R_net'] = stack.R_net
        rstack['T_net'] = stack.T_net
        ref_stack_list.append(rstack)
    if directory and not os.path.exists(directory):
        os.makedirs(directory)
    path = os.path.join(directory, '%s.npz' % casefile_name)
    np.savez_compressed(path, stack_list=np.array(ref_stack_list, dtype=object))
    return path
