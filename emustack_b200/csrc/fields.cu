// Electric fields from the GSM amplitudes (vec_coef_down / vec_coef_up of a
// solved stack):
//
//  * plane-wave basis inside a homogeneous layer: the ThinFilm branch of
//    fields_in_plane (backend/plotting.py:1759-1833) and field_values
//    (backend/plotting.py:2857-2996).  For the orders s of the layer (sorted
//    by the air reference's order) with alpha_s, beta_s, gamma_s = k_z,s and
//    index n:
//        norm = sqrt(alpha^2 + beta^2),  k = sqrt(alpha^2 + beta^2 + gamma^2)
//        chi_TE = sqrt(n gamma / k),     chi_TM = sqrt(n k / gamma)
//        e_TE = (beta, -alpha, 0) / norm, e_TM = (alpha / norm, beta / norm,
//        -norm / gamma)
//        eta_{TE,TM} = c_{TE,TM} e_{TE,TM} / chi_{TE,TM}   (c: the amplitude)
//        E(x, y, z) = sum_s eta_down exp(i(alpha x + beta y - gamma (z1 - h)))
//                         + eta_up   exp(i(alpha x + beta y + gamma z1))
//    with z1 = -z in the substrate (layer 0, whose upward amplitudes are
//    zero) and |z| elsewhere, h the layer's height over the period and 0 for
//    a semi-infinite layer.  The TE and TM terms of one order share their
//    exponentials, so they are summed into one coefficient per component.
//
//  * Bloch-mode basis at the six P2 nodes of every element of a 2D
//    nanostructured layer, at one plane hz (measured from the top of the
//    layer, 0 <= hz <= h): field_value_plane
//    (backend/fortran/field_value_plane.f:6-132),
//        E_j(el, i) = sum_m sol(j, i, m, el) c_j(m),
//        c_{x,y} = d_m + u_m, c_z = (u_m - d_m) / beta_m,
//        d_m = v_m exp(i beta_m hz), u_m = v_{m+M} exp(i beta_m (h - hz)).
//
// Both are evaluated in FP64; sums run in another order than the
// reference's, so results agree to rounding, not bit for bit.
#include <cuda_runtime.h>

#include "emu_cplx.cuh"
#include "emu_internal.h"

namespace {

// ------------------------------------------------------ plane-wave basis
struct PwOrder {  // one order in shared memory (128 bytes)
  double a, b, gr, gi;
  cd d[3], u[3];
};

constexpr int kPwThreads = 256;
constexpr int kPwMaxOrders = 1536;  // 192 KB of shared memory

struct PwArgs {
  int S, Q, grid, nx, ny, nz, substrate, has_up;
  const double *alphas, *betas;
  const int32_t *sort;
  const cd *kz, *n;
  const double *height;
  const cd *vcd, *vcu;
  long long vcd_stride, vcu_stride;
  const double *x, *y, *z;
  cd *E;
  double *E_abs;
};

__device__ __forceinline__ void pw_coefs(cd c_te, cd c_tm, const double ete[3], const cd etm[3],
                                         cd chi_te, cd chi_tm, cd out[3]) {
  for (int j = 0; j < 3; ++j) {
    const cd te = cdiv(cd{c_te.x * ete[j], c_te.y * ete[j]}, chi_te);
    const cd tm = cdiv(cmul(c_tm, etm[j]), chi_tm);
    out[j] = cadd(te, tm);
  }
}

// Order s of stack b: sorted alpha, beta, k_z and the TE + TM coefficients
// of the down and up amplitudes (backend/plotting.py:2896-2941).
__device__ __forceinline__ PwOrder pw_order(const PwArgs &a, int b, int s, cd n) {
  const int S = a.S;
  const int j = a.sort[(size_t)b * S + s];
  const bool ok = j >= 0 && j < S;  // a sort order that is not a permutation gives NaN fields
  const double al = ok ? a.alphas[(size_t)b * S + j] : nan(""), be = ok ? a.betas[(size_t)b * S + j] : nan("");
  const cd g = a.kz[(size_t)b * S + s];
  const double ab2 = al * al + be * be;
  const double norm = sqrt(ab2);
  const cd k = csqrt_p(cd{ab2 + (g.x * g.x - g.y * g.y), 2.0 * g.x * g.y});
  const cd chi_te = csqrt_p(cdiv(cmul(n, g), k));
  const cd chi_tm = csqrt_p(cdiv(cmul(n, k), g));
  const double ete[3] = {be / norm, -al / norm, 0.0};
  const cd etm[3] = {cd{al / norm, 0.0}, cd{be / norm, 0.0}, cdiv(cd{-norm, 0.0}, g)};
  PwOrder o;
  o.a = al;
  o.b = be;
  o.gr = g.x;
  o.gi = g.y;
  const cd *vd = a.vcd + (size_t)b * a.vcd_stride;
  pw_coefs(vd[s], vd[S + s], ete, etm, chi_te, chi_tm, o.d);
  if (a.has_up) {
    const cd *vu = a.vcu + (size_t)b * a.vcu_stride;
    pw_coefs(vu[s], vu[S + s], ete, etm, chi_te, chi_tm, o.u);
  } else {
    for (int c = 0; c < 3; ++c) o.u[c] = cd{0.0, 0.0};
  }
  return o;
}

// Points (x[q], y[q], z[q]): every term evaluated directly.
__global__ void __launch_bounds__(kPwThreads) pw_fields_kernel(PwArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PwOrder *ord = (PwOrder *)smem_raw;
  const int b = blockIdx.y;
  const int S = a.S;
  const cd n = a.n[b];
  const double h = a.height ? a.height[b] : 0.0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) ord[s] = pw_order(a, b, s, n);
  __syncthreads();

  cd *E = a.E + (size_t)b * 3 * a.Q;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.Q;
       q += (long long)gridDim.x * blockDim.x) {
    double x, y, z;
    if (a.grid) {
      const int iz = (int)(q % a.nz);
      const long long r = q / a.nz;
      x = a.x[r / a.ny];
      y = a.y[r % a.ny];
      z = a.z[iz];
    } else {
      x = a.x[q];
      y = a.y[q];
      z = a.z[q];
    }
    const double z1 = a.substrate ? -z : fabs(z);
    const double dzd = z1 - h;
    cd e[3] = {cd{0.0, 0.0}, cd{0.0, 0.0}, cd{0.0, 0.0}};
    for (int s = 0; s < S; ++s) {
      const PwOrder &o = ord[s];
      const double ph = o.a * x + o.b * y;
      // exp(i (ph - gamma (z1 - h))) = exp(gi (z1 - h)) (cos, sin)(ph - gr (z1 - h))
      double sd, cdn;
      sincos(ph - o.gr * dzd, &sd, &cdn);
      const double md = exp(o.gi * dzd);
      const cd ed{md * cdn, md * sd};
      for (int c = 0; c < 3; ++c) e[c] = cadd(e[c], cmul(o.d[c], ed));
      if (a.has_up) {
        double su, cu;
        sincos(ph + o.gr * z1, &su, &cu);
        const double mu = exp(-o.gi * z1);
        const cd eu{mu * cu, mu * su};
        for (int c = 0; c < 3; ++c) e[c] = cadd(e[c], cmul(o.u[c], eu));
      }
    }
    for (int c = 0; c < 3; ++c) E[(size_t)c * a.Q + q] = e[c];
    if (a.E_abs) a.E_abs[(size_t)b * a.Q + q] = sqrt(cabs2(e[0]) + cabs2(e[1]) + cabs2(e[2]));
  }
}

// Grid x[nx] x y[ny] x z[nz]: the exponential of every term factors as
// exp(i alpha x) exp(i beta y) times a z factor, so per stack three tables
// are formed once,
//   X[ix][s] = exp(i alpha_s x_ix),  Y[iy][s] = exp(i beta_s y_iy),
//   Z[iz][s][c] = eta_down,c exp(-i gamma_s (z1 - h)) + eta_up,c exp(i gamma_s z1),
// and E_c(ix, iy, iz) = sum_s X Y Z is a contraction with no transcendental
// function per term.
constexpr int kZc = 4;   // z values per pass (accumulators in registers)
__device__ __forceinline__ cd ldg_c(const cd *p) {
  const double2 v = __ldg((const double2 *)p);
  return cd{v.x, v.y};
}
constexpr int kSc = 64;  // orders per shared-memory stage of Z

__global__ void __launch_bounds__(kPwThreads) pw_tables_kernel(PwArgs a, cd *ws, long long ws_stride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PwOrder *ord = (PwOrder *)smem_raw;
  const int b = blockIdx.x;
  const int S = a.S;
  const cd n = a.n[b];
  const double h = a.height ? a.height[b] : 0.0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) ord[s] = pw_order(a, b, s, n);
  __syncthreads();
  cd *X = ws + (size_t)b * ws_stride;
  cd *Y = X + (size_t)a.nx * S;
  cd *Z = Y + (size_t)a.ny * S;
  for (int i = threadIdx.x; i < a.nx * S; i += blockDim.x) {
    double sn, cs;
    sincos(ord[i % S].a * a.x[i / S], &sn, &cs);
    X[i] = cd{cs, sn};
  }
  for (int i = threadIdx.x; i < a.ny * S; i += blockDim.x) {
    double sn, cs;
    sincos(ord[i % S].b * a.y[i / S], &sn, &cs);
    Y[i] = cd{cs, sn};
  }
  for (int i = threadIdx.x; i < a.nz * S; i += blockDim.x) {
    const PwOrder &o = ord[i % S];
    const double z = a.z[i / S];
    const double z1 = a.substrate ? -z : fabs(z);
    const double dzd = z1 - h;
    double sd, cdn;
    sincos(-o.gr * dzd, &sd, &cdn);
    const double md = exp(o.gi * dzd);
    const cd ed{md * cdn, md * sd};
    cd zc[3];
    for (int c = 0; c < 3; ++c) zc[c] = cmul(o.d[c], ed);
    if (a.has_up) {
      double su, cu;
      sincos(o.gr * z1, &su, &cu);
      const double mu = exp(-o.gi * z1);
      const cd eu{mu * cu, mu * su};
      for (int c = 0; c < 3; ++c) zc[c] = cadd(zc[c], cmul(o.u[c], eu));
    }
    for (int c = 0; c < 3; ++c) Z[(size_t)i * 3 + c] = zc[c];
  }
}

__global__ void __launch_bounds__(kPwThreads) pw_grid_kernel(PwArgs a, const cd *ws, long long ws_stride) {
  __shared__ cd zs[kZc][kSc][3];
  const int b = blockIdx.y;
  const int S = a.S, nxy = a.nx * a.ny;
  const cd *X = ws + (size_t)b * ws_stride;
  const cd *Y = X + (size_t)a.nx * S;
  const cd *Z = Y + (size_t)a.ny * S;
  cd *E = a.E + (size_t)b * 3 * a.Q;
  for (int t0 = blockIdx.x * blockDim.x; t0 < nxy; t0 += gridDim.x * blockDim.x) {
    const int t = t0 + threadIdx.x;
    const bool live = t < nxy;
    const int ix = live ? t / a.ny : 0, iy = live ? t % a.ny : 0;
    const cd *xr = X + (size_t)ix * S, *yr = Y + (size_t)iy * S;
    for (int z0 = 0; z0 < a.nz; z0 += kZc) {
      const int zc = min(kZc, a.nz - z0);
      cd acc[kZc][3];
#pragma unroll
      for (int k = 0; k < kZc; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[k][c] = cd{0.0, 0.0};
      for (int s0 = 0; s0 < S; s0 += kSc) {
        const int sc = min(kSc, S - s0);
        __syncthreads();
        for (int i = threadIdx.x; i < zc * sc * 3; i += blockDim.x) {
          const int k = i / (sc * 3), r = i % (sc * 3);
          zs[k][r / 3][r % 3] = Z[((size_t)(z0 + k) * S + s0 + r / 3) * 3 + r % 3];
        }
        __syncthreads();
        if (live) {
          // the next order's table entries are loaded while this one is summed
          cd xn = ldg_c(xr + s0), yn = ldg_c(yr + s0);
          for (int s = 0; s < sc; ++s) {
            const cd xy = cmul(xn, yn);
            if (s + 1 < sc) {
              xn = ldg_c(xr + s0 + s + 1);
              yn = ldg_c(yr + s0 + s + 1);
            }
#pragma unroll
            for (int k = 0; k < kZc; ++k)
              if (k < zc)
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[k][c] = cadd(acc[k][c], cmul(xy, zs[k][s][c]));
          }
        }
      }
      if (live) {
#pragma unroll
        for (int k = 0; k < kZc; ++k) {
          if (k < zc) {
            const size_t q = (size_t)t * a.nz + z0 + k;
            for (int c = 0; c < 3; ++c) E[(size_t)c * a.Q + q] = acc[k][c];
            if (a.E_abs)
              a.E_abs[(size_t)b * a.Q + q] = sqrt(cabs2(acc[k][0]) + cabs2(acc[k][1]) + cabs2(acc[k][2]));
          }
        }
      }
    }
  }
}

// ------------------------------------------------------- Bloch-mode basis
constexpr int kNodeVals = 18;  // 6 P2 nodes x 3 components
constexpr int kGroups = 8;     // mode groups per element (partial sums)
constexpr int kBlochThreads = kNodeVals * kGroups;
constexpr int kSolRow = 13 * 3;  // complex values per (element, mode) row

struct BlochArgs {
  int M, nel;
  const cd *sol;
  long long sol_stride;
  const cd *beta, *vc;
  double h, hz;
  cd *E;
};

__global__ void __launch_bounds__(kBlochThreads) bloch_plane_kernel(BlochArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd *ct = (cd *)smem_raw;  // [M] coefficient of the transverse components
  cd *cz = ct + a.M;        // [M] coefficient of E_z
  cd *red = cz + a.M;       // [kGroups][kNodeVals]
  const int b = blockIdx.y;
  const cd *beta = a.beta + (size_t)b * a.M;
  const cd *vc = a.vc + (size_t)b * 2 * a.M;
  for (int m = threadIdx.x; m < a.M; m += blockDim.x) {
    const cd bm = beta[m];
    const cd dn = cmul(vc[m], cexp_ikh(bm, a.hz));
    const cd up = cmul(vc[m + a.M], cexp_ikh(bm, a.h - a.hz));
    ct[m] = cadd(up, dn);
    cz[m] = cdiv(csub(up, dn), bm);
  }
  __syncthreads();
  const int o = threadIdx.x % kNodeVals, g = threadIdx.x / kNodeVals;
  const cd *coef = (o % 3 == 2) ? cz : ct;
  const cd *sol_b = a.sol + (size_t)b * a.sol_stride;
  for (int el = blockIdx.x; el < a.nel; el += gridDim.x) {
    const cd *row = sol_b + (size_t)el * a.M * kSolRow + o;
    cd acc{0.0, 0.0};
#pragma unroll 4
    for (int m = g; m < a.M; m += kGroups) acc = cadd(acc, cmul(row[(size_t)m * kSolRow], coef[m]));
    red[g * kNodeVals + o] = acc;
    __syncthreads();
    if (g == 0) {
      cd s = red[o];
      for (int k = 1; k < kGroups; ++k) s = cadd(s, red[k * kNodeVals + o]);
      a.E[((size_t)b * a.nel + el) * kNodeVals + o] = s;
    }
    __syncthreads();
  }
}

}  // namespace

namespace {
long long pw_ws_stride(const EmuPwFields *p) {
  return ((long long)p->nx + p->ny + 3LL * p->nz) * p->n_pw;  // complex values per stack
}
}  // namespace

extern "C" size_t emu_pw_fields_workspace_size(const EmuPwFields *p) {
  if (!p || !p->grid || p->n_stacks <= 0 || p->n_pw < 1 || p->nx < 0 || p->ny < 0 || p->nz < 0) return 0;
  return (size_t)p->n_stacks * (size_t)pw_ws_stride(p) * sizeof(cd);
}

extern "C" int emu_pw_fields(const EmuPwFields *p, void *stream) {
  if (!p || p->n_stacks < 0 || p->n_pw < 1 || p->n_pw > kPwMaxOrders) return EMU_E_ARG;
  if (p->nx < 0 || (p->grid && (p->ny < 0 || p->nz < 0))) return EMU_E_ARG;
  const long long Q = p->grid ? (long long)p->nx * p->ny * p->nz : (long long)p->nx;
  if (Q > 0x7fffffffLL || p->n_stacks > 65535) return EMU_E_SHAPE;
  if (p->n_stacks == 0 || Q == 0) return EMU_OK;
  if (!p->d_alphas || !p->d_betas || !p->d_sort || !p->d_kz || !p->d_n || !p->d_vec_coef_down ||
      !p->d_x || !p->d_y || !p->d_z || !p->d_E)
    return EMU_E_ARG;
  if (p->vcd_stride < 2LL * p->n_pw) return EMU_E_ARG;
  const bool has_up = !p->substrate && p->d_vec_coef_up;
  if (has_up && p->vcu_stride < 2LL * p->n_pw) return EMU_E_ARG;
  PwArgs a;
  a.S = p->n_pw;
  a.Q = (int)Q;
  a.grid = p->grid ? 1 : 0;
  a.nx = p->nx;
  a.ny = p->ny;
  a.nz = p->nz;
  a.substrate = p->substrate ? 1 : 0;
  a.has_up = has_up ? 1 : 0;
  a.alphas = p->d_alphas;
  a.betas = p->d_betas;
  a.sort = p->d_sort;
  a.kz = (const cd *)p->d_kz;
  a.n = (const cd *)p->d_n;
  a.height = p->d_height;
  a.vcd = (const cd *)p->d_vec_coef_down;
  a.vcu = (const cd *)p->d_vec_coef_up;
  a.vcd_stride = p->vcd_stride;
  a.vcu_stride = p->vcu_stride;
  a.x = p->d_x;
  a.y = p->d_y;
  a.z = p->d_z;
  a.E = (cd *)p->d_E;
  a.E_abs = p->d_E_abs;
  const size_t smem = sizeof(PwOrder) * (size_t)p->n_pw;
  cudaStream_t st = (cudaStream_t)stream;
  if (p->grid) {
    const size_t need = emu_pw_fields_workspace_size(p);
    if (!p->d_workspace || p->workspace_bytes < need) return EMU_E_WORKSPACE;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(pw_tables_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
      return EMU_E_CUDA;
    cd *ws = (cd *)p->d_workspace;
    const long long stride = pw_ws_stride(p);
    pw_tables_kernel<<<(unsigned)p->n_stacks, kPwThreads, smem, st>>>(a, ws, stride);
    emu::note_launch();
    long long tiles = ((long long)p->nx * p->ny + kPwThreads - 1) / kPwThreads;
    long long want = (8LL * emu::sm_count() + p->n_stacks - 1) / p->n_stacks;
    if (want < 1) want = 1;
    if (tiles > want) tiles = want;
    pw_grid_kernel<<<dim3((unsigned)tiles, (unsigned)p->n_stacks), kPwThreads, 0, st>>>(a, ws, stride);
    emu::note_launch();
    return emu::check_launch();
  }
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(pw_fields_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return EMU_E_CUDA;
  // enough blocks per stack to fill the device a few times over, each one
  // sweeping several tiles of points (its order table is built once)
  long long tiles = (Q + kPwThreads - 1) / kPwThreads;
  long long want = (4LL * emu::sm_count() + p->n_stacks - 1) / p->n_stacks;
  if (want < 1) want = 1;
  if (tiles > want) tiles = want;
  pw_fields_kernel<<<dim3((unsigned)tiles, (unsigned)p->n_stacks), kPwThreads, smem, st>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_bloch_fields_plane(const EmuBlochFieldsPlane *p, void *stream) {
  if (!p || p->n_stacks < 0 || p->n_modes < 1 || p->n_elements < 0) return EMU_E_ARG;
  if (!(p->hz >= 0.0 && p->hz <= p->h)) return EMU_E_ARG;  // the routine's own check
  if (p->n_stacks > 65535) return EMU_E_SHAPE;
  if (p->n_stacks == 0 || p->n_elements == 0) return EMU_OK;
  if (!p->d_sol || !p->d_k_z || !p->d_vec_coef || !p->d_E) return EMU_E_ARG;
  if (p->n_stacks > 1 && p->sol_stride < (long long)p->n_elements * p->n_modes * kSolRow) return EMU_E_ARG;
  BlochArgs a;
  a.M = p->n_modes;
  a.nel = p->n_elements;
  a.sol = (const cd *)p->d_sol;
  a.sol_stride = p->sol_stride;
  a.beta = (const cd *)p->d_k_z;
  a.vc = (const cd *)p->d_vec_coef;
  a.h = p->h;
  a.hz = p->hz;
  a.E = (cd *)p->d_E;
  const size_t smem = sizeof(cd) * (2 * (size_t)p->n_modes + kGroups * kNodeVals);
  if (smem > 200 * 1024) return EMU_E_SHAPE;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(bloch_plane_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return EMU_E_CUDA;
  long long blocks = p->n_elements;
  const long long cap = (16LL * emu::sm_count() + p->n_stacks - 1) / p->n_stacks;
  if (blocks > cap) blocks = cap;
  bloch_plane_kernel<<<dim3((unsigned)blocks, (unsigned)p->n_stacks), kBlochThreads, smem,
                       (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}
