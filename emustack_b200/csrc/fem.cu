// FEM Bloch modes of a 2D nanostructured layer (row f1): the mode solve of
// calc_modes_2d (backend/fortran/py_calc_modes.f:243-700) for the E-field
// formulation with periodic boundaries.
//
//   emu_fem_topology          host: periodic pairing (periodic_node.f:60-120),
//                             DOF numbering (periodic_cond.f: face / edge 3
//                             DOFs, P3 node 1), CSR pattern and the element
//                             entries each CSR entry sums
//   emu_fem_element_matrices  one CTA per element: K_e, M_e of asmbly.f:130-320
//   emu_fem_assemble          one thread per CSR entry, element order
//   emu_fem_shifted_dense     A = K - shift M, dense
//   emu_fem_lu / _apply_op    multi-CTA LU of A (FP64 tensor-core GEMM tiles)
//                             and Y = A^-1 M X for a block of vectors
//   emu_fem_nodal_fields      array_sol.f:88-300
//
// The element: per triangle a face and 3 edges, each with 3 transverse basis
// vectors phi2(m) grad(lambda) (basis_ls.f, basis_vec.f), and 10 P3 nodes
// with one E_z value (phi3_2d_mat.f); straight elements (curved_elem_tri.f
// returns "straight" for every element), 16-point rule (quad_triangle.f).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "dense_la.cuh"
#include "dense_multi.cuh"
#include "emu_cplx.cuh"
#include "emu_internal.h"

namespace {

constexpr int kLoc = 22;           // local DOFs: 12 transverse + 10 E_z
constexpr int kLoc2 = kLoc * kLoc;
constexpr int kElemThreads = 128;

// 16-point rule on the reference triangle (weights include the area 1/2)
__constant__ double c_qw[16];
__constant__ double c_qx[16];
__constant__ double c_qy[16];

void quad_rule(double *w, double *x, double *y) {
  const double wbar = 1.443156076777862e-1 / 2.0, w1 = 2.852749028018549e-1 / 6.0,
               w2 = 9.737549286959440e-2 / 6.0, w3 = 3.096521116041552e-1 / 6.0,
               w4 = 1.633818850466092e-1 / 12.0, cb = 1.0 / 3.0;
  const double a1 = 4.592925882927229e-1, b1 = 8.141482341455413e-2;
  const double a2 = 5.054722831703103e-2, b2 = 8.989055433659379e-1;
  const double a3 = 1.705693077517601e-1, b3 = 6.588613844964797e-1;
  const double a4 = 7.284923929554041e-1, b4 = 2.63112829634638689e-1, c4 = 8.394777409957211e-3;
  const double X[16] = {cb, a1, a1, b1, a2, a2, b2, a3, a3, b3, a4, b4, b4, c4, c4, a4};
  const double Y[16] = {cb, a1, b1, a1, a2, b2, a2, a3, b3, a3, b4, a4, c4, b4, a4, c4};
  const double W[16] = {wbar, w1, w1, w1, w2, w2, w2, w3, w3, w3, w4, w4, w4, w4, w4, w4};
  for (int i = 0; i < 16; ++i) {
    w[i] = W[i];
    x[i] = X[i];
    y[i] = Y[i];
  }
}

int upload_quad() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done[dev]) return EMU_OK;
  double w[16], x[16], y[16];
  quad_rule(w, x, y);
  if (cudaMemcpyToSymbol(c_qw, w, sizeof w) != cudaSuccess ||
      cudaMemcpyToSymbol(c_qx, x, sizeof x) != cudaSuccess ||
      cudaMemcpyToSymbol(c_qy, y, sizeof y) != cudaSuccess)
    return EMU_E_CUDA;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return EMU_OK;
}

// ------------------------------------------------------------ bases
__device__ __forceinline__ void phi2_vg(double x, double y, double v[6], double gx[6], double gy[6]) {
  v[0] = (-1 + x + y) * (-1 + 2 * x + 2 * y);
  v[1] = x * (-1 + 2 * x);
  v[2] = y * (-1 + 2 * y);
  v[3] = -4 * x * (-1 + x + y);
  v[4] = 4 * x * y;
  v[5] = -4 * y * (-1 + x + y);
  gx[0] = -3 + 4 * x + 4 * y;
  gy[0] = -3 + 4 * x + 4 * y;
  gx[1] = -1 + 4 * x;
  gy[1] = 0;
  gx[2] = 0;
  gy[2] = -1 + 4 * y;
  gx[3] = 4 - 8 * x - 4 * y;
  gy[3] = -4 * x;
  gx[4] = 4 * y;
  gy[4] = 4 * x;
  gx[5] = -4 * y;
  gy[5] = 4 - 4 * x - 8 * y;
}

__device__ __forceinline__ double phi3_v(int i, double x, double y) {
  switch (i) {
    case 0: return -((-1 + x + y) * (-2 + 3 * x + 3 * y) * (-1 + 3 * x + 3 * y)) / 2.;
    case 1: return (x * (-2 + 3 * x) * (-1 + 3 * x)) / 2.;
    case 2: return (y * (-2 + 3 * y) * (-1 + 3 * y)) / 2.;
    case 3: return (9 * x * (-1 + x + y) * (-2 + 3 * x + 3 * y)) / 2.;
    case 4: return (-9 * x * (-1 + 3 * x) * (-1 + x + y)) / 2.;
    case 5: return (9 * x * (-1 + 3 * x) * y) / 2.;
    case 6: return (9 * x * y * (-1 + 3 * y)) / 2.;
    case 7: return (-9 * y * (-1 + x + y) * (-1 + 3 * y)) / 2.;
    case 8: return (9 * y * (-1 + x + y) * (-2 + 3 * x + 3 * y)) / 2.;
    default: return -27 * x * y * (-1 + x + y);
  }
}

__device__ __forceinline__ void phi3_g(int i, double x, double y, double &gx, double &gy) {
  switch (i) {
    case 0: {
      const double t = (-11 - 27 * x * x + x * (36 - 54 * y) + 36 * y - 27 * y * y) / 2.;
      gx = t;
      gy = t;
      break;
    }
    case 1: gx = 1 - 9 * x + (27 * x * x) / 2.; gy = 0; break;
    case 2: gx = 0; gy = 1 - 9 * y + (27 * y * y) / 2.; break;
    case 3:
      gx = (9 * (2 + 9 * x * x - 5 * y + 3 * y * y + 2 * x * (-5 + 6 * y))) / 2.;
      gy = (9 * x * (-5 + 6 * x + 6 * y)) / 2.;
      break;
    case 4:
      gx = (-9 * (1 + 9 * x * x - y + x * (-8 + 6 * y))) / 2.;
      gy = (-9 * x * (-1 + 3 * x)) / 2.;
      break;
    case 5: gx = (9 * (-1 + 6 * x) * y) / 2.; gy = (9 * x * (-1 + 3 * x)) / 2.; break;
    case 6: gx = (9 * y * (-1 + 3 * y)) / 2.; gy = (9 * x * (-1 + 6 * y)) / 2.; break;
    case 7:
      gx = (-9 * y * (-1 + 3 * y)) / 2.;
      gy = (-9 * (1 - 8 * y + 9 * y * y + x * (-1 + 6 * y))) / 2.;
      break;
    case 8:
      gx = (9 * y * (-5 + 6 * x + 6 * y)) / 2.;
      gy = (9 * (2 + 3 * x * x - 10 * y + 9 * y * y + x * (-5 + 12 * y))) / 2.;
      break;
    default:
      gx = -27 * y * (-1 + 2 * x + y);
      gy = -27 * x * (-1 + x + 2 * y);
  }
}

struct ElemGeom {
  double T[2][2];  // B^-1, B = [x2 - x1, x3 - x1] (jacobian_p1_2d.f)
  double det;
};

__device__ __forceinline__ ElemGeom elem_geom(const double *x, const int64_t *tn) {
  const int64_t n0 = tn[0] - 1, n1 = tn[1] - 1, n2 = tn[2] - 1;
  const double B00 = x[2 * n1] - x[2 * n0], B01 = x[2 * n2] - x[2 * n0];
  const double B10 = x[2 * n1 + 1] - x[2 * n0 + 1], B11 = x[2 * n2 + 1] - x[2 * n0 + 1];
  ElemGeom g;
  g.det = B00 * B11 - B01 * B10;
  g.T[0][0] = B11 / g.det;
  g.T[0][1] = -B01 / g.det;
  g.T[1][0] = -B10 / g.det;
  g.T[1][1] = B00 / g.det;
  return g;
}

// physical gradient T^T g0
__device__ __forceinline__ void tgrad(const ElemGeom &G, double g0x, double g0y, double &gx, double &gy) {
  gx = G.T[0][0] * g0x + G.T[1][0] * g0y;
  gy = G.T[0][1] * g0x + G.T[1][1] * g0y;
}

// P1 gradients on the element: lambda_1 = 1 - x - y, lambda_2 = x, lambda_3 = y
__device__ __forceinline__ void p1_grads(const ElemGeom &G, double gx[3], double gy[3]) {
  tgrad(G, -1.0, -1.0, gx[0], gy[0]);
  tgrad(G, 1.0, 0.0, gx[1], gy[1]);
  tgrad(G, 0.0, 1.0, gx[2], gy[2]);
}

// transverse function i (0..11): the P2 node it lives on (basis_list(2, ., .))
// and its P1-gradient factor (basis_vec.f)
__device__ __forceinline__ void tfun(int i, const int8_t ends[3][2], const double g1x[3], const double g1y[3],
                                     int &m, double &px, double &py) {
  if (i < 3) {  // face: phi2(mid j) grad(lambda of the opposite vertex)
    m = 3 + i;
    const int n1 = (i + 2) % 3;
    px = g1x[n1];
    py = g1y[n1];
    return;
  }
  const int k = (i - 3) / 3, r = (i - 3) % 3;
  const int j1 = ends[k][0], j2 = ends[k][1];
  if (r == 0) {
    m = j1;
    px = g1x[j2];
    py = g1y[j2];
  } else if (r == 1) {
    m = j2;
    px = g1x[j1];
    py = g1y[j1];
  } else {
    m = 3 + k;
    px = g1x[j1] - g1x[j2];
    py = g1y[j1] - g1y[j2];
  }
}

// entity (0..13) of local DOF a
__device__ __forceinline__ int entity_of(int a) { return a < 12 ? a / 3 : a - 8; }

struct ElemArgs {
  int nel, n_types;
  const double *x;
  const int64_t *tn;
  const int64_t *type_el;
  const double *shift;
  const int8_t *ends;
  cd pp[8], qq[8];
  double bloch0, bloch1;
  cd *Ke, *Me;
};

__global__ void __launch_bounds__(kElemThreads) fem_element_kernel(ElemArgs a) {
  const int e = blockIdx.x;
  __shared__ double s_vx[12], s_vy[12], s_c[12], s_gx[10], s_gy[10], s_v3[10];
  __shared__ cd s_ph[14];
  const int tid = threadIdx.x;
  const ElemGeom G = elem_geom(a.x, a.tn + (size_t)e * 6);
  int8_t ends[3][2];
  for (int k = 0; k < 3; ++k) {
    ends[k][0] = a.ends[(size_t)e * 6 + 2 * k];
    ends[k][1] = a.ends[(size_t)e * 6 + 2 * k + 1];
  }
  if (tid < 14) {
    const double arg = a.bloch0 * a.shift[((size_t)e * 14 + tid) * 2] +
                       a.bloch1 * a.shift[((size_t)e * 14 + tid) * 2 + 1];
    double sn, cs;
    sincos(arg, &sn, &cs);
    s_ph[tid] = cd{cs, sn};
  }
  const int te = (int)a.type_el[e] - 1;
  const cd pp = a.pp[te], qq = a.qq[te];
  const double wdet = fabs(G.det);
  double g1x[3], g1y[3];
  p1_grads(G, g1x, g1y);
  constexpr int kPer = (kLoc2 + kElemThreads - 1) / kElemThreads;
  cd kacc[kPer], macc[kPer];
#pragma unroll
  for (int t = 0; t < kPer; ++t) kacc[t] = macc[t] = cd{0.0, 0.0};
  for (int q = 0; q < 16; ++q) {
    const double xq = c_qx[q], yq = c_qy[q];
    if (tid < 12) {
      double v2[6], g2x0[6], g2y0[6];
      phi2_vg(xq, yq, v2, g2x0, g2y0);
      int m;
      double px, py;
      tfun(tid, ends, g1x, g1y, m, px, py);
      double g2x, g2y;
      tgrad(G, g2x0[m], g2y0[m], g2x, g2y);
      s_vx[tid] = v2[m] * px;
      s_vy[tid] = v2[m] * py;
      s_c[tid] = g2x * py - g2y * px;
    } else if (tid >= 32 && tid < 42) {
      const int i = tid - 32;
      double g0x, g0y;
      phi3_g(i, xq, yq, g0x, g0y);
      tgrad(G, g0x, g0y, s_gx[i], s_gy[i]);
      s_v3[i] = phi3_v(i, xq, yq);
    }
    __syncthreads();
    const double w = c_qw[q] * wdet;
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
      const int idx = tid + t * kElemThreads;
      if (idx < kLoc2) {
        const int ai = idx / kLoc, bi = idx % kLoc;  // trial, test
        if (ai < 12 && bi < 12) {
          const double dtt = s_vx[bi] * s_vx[ai] + s_vy[bi] * s_vy[ai];
          const double cc = s_c[bi] * s_c[ai];
          kacc[t].x += w * (cc * pp.x - dtt * qq.x);
          kacc[t].y += w * (cc * pp.y - dtt * qq.y);
          macc[t].x -= w * dtt * pp.x;
          macc[t].y -= w * dtt * pp.y;
        } else if (ai < 12) {
          const int j = bi - 12;
          const double d = s_gx[j] * s_vx[ai] + s_gy[j] * s_vy[ai];
          macc[t].x += w * d * pp.x;
          macc[t].y += w * d * pp.y;
        } else if (bi < 12) {
          const int i = ai - 12;
          const double d = s_vx[bi] * s_gx[i] + s_vy[bi] * s_gy[i];
          kacc[t].x += w * d * pp.x;
          kacc[t].y += w * d * pp.y;
        } else {
          const int i = ai - 12, j = bi - 12;
          const double gg = s_gx[j] * s_gx[i] + s_gy[j] * s_gy[i];
          const double vv = s_v3[j] * s_v3[i];
          kacc[t].x += w * (vv * qq.x - gg * pp.x);
          kacc[t].y += w * (vv * qq.y - gg * pp.y);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < kPer; ++t) {
    const int idx = tid + t * kElemThreads;
    if (idx < kLoc2) {
      const int ai = idx / kLoc, bi = idx % kLoc;
      const cd pa = s_ph[entity_of(ai)], pb = s_ph[entity_of(bi)];
      const cd fac = cmul(cd{pa.x, -pa.y}, pb);
      a.Ke[(size_t)e * kLoc2 + idx] = cmul(kacc[t], fac);
      a.Me[(size_t)e * kLoc2 + idx] = cmul(macc[t], fac);
    }
  }
}

__global__ void fem_gather_kernel(int nnz, const int32_t *src_ptr, const int32_t *src, const cd *Ke,
                                  const cd *Me, cd *K, cd *M) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += gridDim.x * blockDim.x) {
    cd k{0.0, 0.0}, m{0.0, 0.0};
    for (int s = src_ptr[i]; s < src_ptr[i + 1]; ++s) {
      const int j = src[s];
      k.x += Ke[j].x;
      k.y += Ke[j].y;
      m.x += Me[j].x;
      m.y += Me[j].y;
    }
    K[i] = k;
    M[i] = m;
  }
}

__global__ void fem_dense_kernel(int n, const int32_t *row_ptr, const int32_t *col, const cd *K, const cd *M,
                                 cd shift, cd *A, int lda) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int i = row_ptr[r]; i < row_ptr[r + 1]; ++i) {
      const cd sm = cmul(shift, M[i]);
      A[(size_t)r * lda + col[i]] = cd{K[i].x - sm.x, K[i].y - sm.y};
    }
}

// T = (M X) restricted to rows[0..nr) (all rows when rows is null), one warp
// per row, lanes over the block's vectors
__global__ void fem_spmm_kernel(int nr, const int32_t *rows, int nrhs, const int32_t *row_ptr, const int32_t *col,
                                const cd *M, const cd *X, int ldx, cd *Y, int ldy) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nr; j += warps) {
    const int r = rows ? rows[j] : j;
    for (int c = lane; c < nrhs; c += 32) {
      cd y{0.0, 0.0};
      for (int i = row_ptr[r]; i < row_ptr[r + 1]; ++i) {
        const cd xv = X[(size_t)col[i] * ldx + c];
        const cd mv = M[i];
        y.x += mv.x * xv.x - mv.y * xv.y;
        y.y += mv.x * xv.y + mv.y * xv.x;
      }
      Y[(size_t)j * ldy + c] = y;
    }
  }
}

// ------------------------------------------------------------ nodal fields
struct FieldArgs {
  int nel, nval, ldv;
  const double *x;
  const int64_t *tn;
  const double *shift;
  const int8_t *ends;
  const int32_t *dof;
  double bloch0, bloch1;
  const cd *vec;
  cd *sol;
};

__global__ void fem_nodal_kernel(FieldArgs a) {
  const int e = blockIdx.x;
  __shared__ int s_dof[kLoc];
  __shared__ cd s_ph[14];
  __shared__ int s_node[12];
  __shared__ double s_px[12], s_py[12];
  __shared__ double s_p3[6][10];
  const int tid = threadIdx.x;
  if (tid < kLoc) s_dof[tid] = a.dof[(size_t)e * kLoc + tid];
  if (tid < 14) {
    const double arg = a.bloch0 * a.shift[((size_t)e * 14 + tid) * 2] +
                       a.bloch1 * a.shift[((size_t)e * 14 + tid) * 2 + 1];
    double sn, cs;
    sincos(arg, &sn, &cs);
    s_ph[tid] = cd{cs, sn};
  }
  if (tid < 12) {
    const ElemGeom G = elem_geom(a.x, a.tn + (size_t)e * 6);
    double g1x[3], g1y[3];
    p1_grads(G, g1x, g1y);
    int8_t ends[3][2];
    for (int k = 0; k < 3; ++k) {
      ends[k][0] = a.ends[(size_t)e * 6 + 2 * k];
      ends[k][1] = a.ends[(size_t)e * 6 + 2 * k + 1];
    }
    int m;
    double px, py;
    tfun(tid, ends, g1x, g1y, m, px, py);
    s_node[tid] = m;
    s_px[tid] = px;  // phi2(m) = 1 at its own node
    s_py[tid] = py;
  }
  if (tid >= 32 && tid < 92) {
    const int k = tid - 32, nd = k / 10, i = k % 10;
    const double xs[6] = {0, 1, 0, 0.5, 0.5, 0}, ys[6] = {0, 0, 1, 0, 0.5, 0.5};
    s_p3[nd][i] = phi3_v(i, xs[nd], ys[nd]);
  }
  __syncthreads();
  for (int m = blockIdx.y * blockDim.x + tid; m < a.nval; m += gridDim.y * blockDim.x) {
    cd u[kLoc];
#pragma unroll
    for (int i = 0; i < kLoc; ++i) u[i] = cmul(a.vec[(size_t)s_dof[i] * a.ldv + m], s_ph[entity_of(i)]);
    cd *out = a.sol + ((size_t)e * a.nval + m) * 39;
    for (int nd = 0; nd < 6; ++nd) {
      cd ex{0.0, 0.0}, ey{0.0, 0.0}, ez{0.0, 0.0};
      for (int i = 0; i < 12; ++i)
        if (s_node[i] == nd) {
          ex.x += u[i].x * s_px[i];
          ex.y += u[i].y * s_px[i];
          ey.x += u[i].x * s_py[i];
          ey.y += u[i].y * s_py[i];
        }
      for (int i = 0; i < 10; ++i) {
        ez.x += u[12 + i].x * s_p3[nd][i];
        ez.y += u[12 + i].y * s_p3[nd][i];
      }
      out[nd * 3] = ex;
      out[nd * 3 + 1] = ey;
      out[nd * 3 + 2] = ez;
    }
    for (int k = 0; k < 7; ++k) {
      out[(6 + k) * 3] = cd{0.0, 0.0};
      out[(6 + k) * 3 + 1] = cd{0.0, 0.0};
      out[(6 + k) * 3 + 2] = u[15 + k];
    }
  }
}

// first largest-modulus P2-node component of each mode (one CTA per mode)
__global__ void fem_argmax_kernel(int nel, int nval, const cd *sol, cd *zmax) {
  const int m = blockIdx.x;
  double best = -1.0;
  long long bi = 0;
  const long long total = (long long)nel * 18;
  for (long long f = threadIdx.x; f < total; f += blockDim.x) {
    const long long e = f / 18, r = f % 18;
    const cd v = sol[((size_t)e * nval + m) * 39 + r];
    const double mag = hypot(v.x, v.y);
    if (mag > best) {  // f ascends per thread: the first of equal values stays
      best = mag;
      bi = f;
    }
  }
  __shared__ double s_b[256];
  __shared__ long long s_i[256];
  s_b[threadIdx.x] = best;
  s_i[threadIdx.x] = bi;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      const double ob = s_b[threadIdx.x + st];
      const long long oi = s_i[threadIdx.x + st];
      if (ob > s_b[threadIdx.x] || (ob == s_b[threadIdx.x] && oi < s_i[threadIdx.x])) {
        s_b[threadIdx.x] = ob;
        s_i[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long f = s_i[0];
    zmax[m] = sol[((size_t)(f / 18) * nval + m) * 39 + f % 18];
  }
}

__global__ void fem_scale_kernel(int nel, int nval, cd *sol, const cd *zmax) {
  const long long total = (long long)nel * nval * 39;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int m = (int)((i / 39) % nval);
    sol[i] = cdiv(sol[i], zmax[m]);
  }
}

inline int grid_for(long long work, int threads) {
  long long g = (work + threads - 1) / threads;
  const long long cap = 32LL * emu::sm_count();
  if (g > cap) g = cap;
  return (int)std::max(1LL, g);
}

// CSR pattern of element matrices with nloc local DOFs (row = trial DOF,
// column = test DOF, columns ascending) and, for every CSR entry, the flat
// element-matrix entries e*nloc*nloc + a*nloc + b it sums, in element order.
void csr_pattern(int nel, int nloc, const int32_t *dof, int neq, int32_t *row_ptr, int32_t *col, int32_t *src_ptr,
                 int32_t *src, int *nnz_out) {
  const size_t nloc2 = (size_t)nloc * nloc;
  const size_t total = (size_t)nel * nloc2;
  std::vector<unsigned long long> rc(total);
  for (int e = 0; e < nel; ++e) {
    const int32_t *d = &dof[(size_t)e * nloc];
    for (int a = 0; a < nloc; ++a)
      for (int b = 0; b < nloc; ++b)
        rc[(size_t)e * nloc2 + (size_t)a * nloc + b] = ((unsigned long long)d[a] << 32) | (unsigned)d[b];
  }
  std::vector<int32_t> order(total);
  for (size_t i = 0; i < total; ++i) order[i] = (int32_t)i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t p, int32_t q) { return rc[p] < rc[q]; });
  int nnz = 0;
  for (int r = 0; r <= neq; ++r) row_ptr[r] = 0;
  unsigned long long prev = ~0ULL;
  for (size_t i = 0; i < total; ++i) {
    const unsigned long long v = rc[order[i]];
    if (v != prev) {
      col[nnz] = (int32_t)(v & 0xffffffffULL);
      src_ptr[nnz] = (int32_t)i;
      row_ptr[(v >> 32) + 1] += 1;
      ++nnz;
      prev = v;
    }
    src[i] = order[i];
  }
  src_ptr[nnz] = (int32_t)total;
  for (int r = 0; r < neq; ++r) row_ptr[r + 1] += row_ptr[r];
  *nnz_out = nnz;
}

}  // namespace

// ---------------------------------------------------------------- host topology
extern "C" int emu_fem_topology(EmuFemTopology *t) {
  if (!t || t->npt < 3 || t->nel < 1 || !t->h_x || !t->h_type_nod || !t->h_table_nod || !t->h_dof ||
      !t->h_shift || !t->h_ends || !t->h_row_ptr || !t->h_col || !t->h_src_ptr || !t->h_src)
    return EMU_E_ARG;
  const int npt = t->npt, nel = t->nel;
  if ((long long)nel * kLoc2 > 0x7fffffffLL) return EMU_E_SHAPE;
  const double *x = t->h_x;
  const int64_t *tab = t->h_table_nod;
  for (long long i = 0; i < (long long)nel * 6; ++i)
    if (tab[i] < 1 || tab[i] > npt) return EMU_E_ARG;
  // periodic pairing (periodic_node.f:60-120)
  double xmin = x[0], xmax = x[0], ymin = x[1], ymax = x[1];
  for (int i = 0; i < npt; ++i) {
    xmin = std::min(xmin, x[2 * i]);
    xmax = std::max(xmax, x[2 * i]);
    ymin = std::min(ymin, x[2 * i + 1]);
    ymax = std::max(ymax, x[2 * i + 1]);
  }
  const double ax = xmax - xmin, ay = ymax - ymin;
  std::vector<int> ip(npt, -1), bnd;
  for (int i = 0; i < npt; ++i)
    if (t->h_type_nod[i] != 0) bnd.push_back(i);
  for (size_t ii = 0; ii + 1 < bnd.size(); ++ii) {
    const int i = bnd[ii];
    for (size_t jj = ii + 1; jj < bnd.size(); ++jj) {
      const int j = bnd[jj];
      if (ip[j] != -1) continue;
      const double dx = x[2 * j] - x[2 * i], dy = x[2 * j + 1] - x[2 * i + 1];
      bool lat = false;
      for (int ix = -1; ix <= 1 && !lat; ++ix)
        for (int iy = -1; iy <= 1 && !lat; ++iy)
          lat = fabs(dx - ix * ax) + fabs(dy - iy * ay) < 1e-6;
      if (lat) {
        if (ip[i] == -1) {
          ip[i] = i;
          ip[j] = i;
        } else {
          ip[j] = ip[i];
        }
      }
    }
  }
  for (int i : bnd)
    if (ip[i] == -1) return EMU_E_ARG;
  std::vector<int> origin(npt);
  for (int i = 0; i < npt; ++i) origin[i] = ip[i] >= 0 ? ip[i] : i;
  // entities, numbered in order of first appearance (element by element:
  // face, edges, vertices, P3 edge nodes, interior node)
  std::unordered_map<unsigned long long, int> ids;
  std::vector<int> width;
  auto num = [&](unsigned long long key, int w) {
    auto it = ids.find(key);
    if (it != ids.end()) return it->second;
    const int id = (int)width.size();
    ids.emplace(key, id);
    width.push_back(w);
    return id;
  };
  auto key = [](unsigned long long kind, unsigned long long p, unsigned long long q) {
    return (kind << 60) | (p << 30) | q;
  };
  static const int kEdge[3][2] = {{0, 1}, {1, 2}, {0, 2}};
  static const int kP3Edge[6][2] = {{0, 0}, {0, 1}, {1, 1}, {1, 2}, {2, 2}, {2, 0}};
  std::vector<int> ent((size_t)nel * 14);
  for (int e = 0; e < nel; ++e) {
    int tn[6], tm[6];
    for (int k = 0; k < 6; ++k) {
      tn[k] = (int)tab[(size_t)e * 6 + k] - 1;
      tm[k] = origin[tn[k]];
    }
    int *en = &ent[(size_t)e * 14];
    double *sh = &t->h_shift[(size_t)e * 28];
    auto put_shift = [&](int slot, int node) {
      sh[2 * slot] = x[2 * node] - x[2 * origin[node]];
      sh[2 * slot + 1] = x[2 * node + 1] - x[2 * origin[node] + 1];
    };
    en[0] = num(key(1, (unsigned)e, 0), 3);
    sh[0] = sh[1] = 0.0;
    for (int k = 0; k < 3; ++k) {
      const int mid = tn[3 + k], p = kEdge[k][0], q = kEdge[k][1];
      en[1 + k] = num(key(2, (unsigned)origin[mid], 0), 3);
      put_shift(1 + k, mid);
      if (tm[p] == tm[q]) return EMU_E_ARG;
      const bool lo = tm[p] <= tm[q];
      t->h_ends[(size_t)e * 6 + 2 * k] = (int8_t)(lo ? p : q);
      t->h_ends[(size_t)e * 6 + 2 * k + 1] = (int8_t)(lo ? q : p);
    }
    for (int v = 0; v < 3; ++v) {
      en[4 + v] = num(key(3, (unsigned)tm[v], 0), 1);
      put_shift(4 + v, tn[v]);
    }
    for (int n = 0; n < 6; ++n) {
      const int mid = tn[3 + kP3Edge[n][0]];
      en[7 + n] = num(key(4, (unsigned)origin[mid], (unsigned)tm[kP3Edge[n][1]]), 1);
      put_shift(7 + n, mid);
    }
    en[13] = num(key(5, (unsigned)e, 0), 1);
    sh[26] = sh[27] = 0.0;
  }
  std::vector<long long> first(width.size() + 1, 0);
  for (size_t i = 0; i < width.size(); ++i) first[i + 1] = first[i] + width[i];
  if (first.back() > 0x7fffffffLL) return EMU_E_SHAPE;
  const int neq = (int)first.back();
  for (int e = 0; e < nel; ++e) {
    const int *en = &ent[(size_t)e * 14];
    int32_t *d = &t->h_dof[(size_t)e * kLoc];
    for (int k = 0; k < 4; ++k)
      for (int q = 0; q < 3; ++q) d[3 * k + q] = (int32_t)(first[en[k]] + q);
    for (int i = 0; i < 10; ++i) d[12 + i] = (int32_t)first[en[4 + i]];
  }
  csr_pattern(nel, kLoc, t->h_dof, neq, t->h_row_ptr, t->h_col, t->h_src_ptr, t->h_src, &t->nnz);
  t->neq = neq;
  return EMU_OK;
}

// ---------------------------------------------------------------- device entries
extern "C" int emu_fem_element_matrices(const EmuFemElements *p, void *stream) {
  if (!p || p->nel < 1 || p->n_types < 1 || p->n_types > 8) return EMU_E_ARG;
  if (!p->d_x || !p->d_table_nod || !p->d_type_el || !p->d_shift || !p->d_ends || !p->d_Ke || !p->d_Me)
    return EMU_E_ARG;
  int rc = upload_quad();
  if (rc != EMU_OK) return rc;
  ElemArgs a;
  a.nel = p->nel;
  a.n_types = p->n_types;
  a.x = p->d_x;
  a.tn = p->d_table_nod;
  a.type_el = p->d_type_el;
  a.shift = p->d_shift;
  a.ends = p->d_ends;
  for (int i = 0; i < 8; ++i) {
    const cd n{p->n_eff[i].re, p->n_eff[i].im};
    const cd eps = cmul(n, n);
    a.pp[i] = cd{1.0, 0.0};
    a.qq[i] = cd{eps.x * p->k0 * p->k0, eps.y * p->k0 * p->k0};
  }
  a.bloch0 = p->bloch[0];
  a.bloch1 = p->bloch[1];
  a.Ke = (cd *)p->d_Ke;
  a.Me = (cd *)p->d_Me;
  fem_element_kernel<<<p->nel, kElemThreads, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_fem_assemble(int nnz, const int32_t *d_src_ptr, const int32_t *d_src, const emu_c128 *d_Ke,
                                const emu_c128 *d_Me, emu_c128 *d_K, emu_c128 *d_M, void *stream) {
  if (nnz < 0) return EMU_E_SHAPE;
  if (nnz == 0) return EMU_OK;
  if (!d_src_ptr || !d_src || !d_Ke || !d_Me || !d_K || !d_M) return EMU_E_ARG;
  fem_gather_kernel<<<grid_for(nnz, 256), 256, 0, (cudaStream_t)stream>>>(
      nnz, d_src_ptr, d_src, (const cd *)d_Ke, (const cd *)d_Me, (cd *)d_K, (cd *)d_M);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_fem_shifted_dense(int neq, const int32_t *d_row_ptr, const int32_t *d_col, const emu_c128 *d_K,
                                     const emu_c128 *d_M, emu_c128 shift, emu_c128 *d_A, int lda, void *stream) {
  if (neq < 1 || lda < neq) return EMU_E_SHAPE;
  if (!d_row_ptr || !d_col || !d_K || !d_M || !d_A) return EMU_E_ARG;
  const cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(d_A, 0, (size_t)neq * lda * sizeof(emu_c128), s) != cudaSuccess) return EMU_E_CUDA;
  fem_dense_kernel<<<grid_for(neq, 128), 128, 0, s>>>(neq, d_row_ptr, d_col, (const cd *)d_K, (const cd *)d_M,
                                                      cd{shift.re, shift.im}, (cd *)d_A, lda);
  emu::note_launch();
  return emu::check_launch();
}

namespace {

// In-place LU with partial pivoting, blocked twice: panels of kNB columns
// factored as in getrf_multi (same panel kernels, full-row interchanges)
// inside outer blocks of kOuterNB columns, whose trailing matrix is updated
// once per outer block by a GEMM of depth kOuterNB.  The matrix is read and
// written kOuterNB / kNB times less than by getrf_multi's per-panel updates.
constexpr int kOuterNB = 256;

void getrf_blocked(int n, cd *A, int lda, int *ipiv, int *info, cudaStream_t s) {
  for (int J = 0; J < n; J += kOuterNB) {
    const int JB = std::min(kOuterNB, n - J);
    for (int j0 = J; j0 < J + JB; j0 += kNB) {
      const int jb = std::min(kNB, J + JB - j0);
      if (!panel_cluster(A, 0, lda, n, j0, jb, ipiv, 0, info, 0, 1, s, 16)) {
        cudaGetLastError();
        panel_kernel<<<1, kPanelThreads, 0, s>>>(A, 0, lda, n, j0, jb, ipiv, 0, info, 0);
        emu::note_launch();
      }
      const int c0 = j0 + jb, nc = J + JB - c0;
      if (nc > 0) {
        trsm_lower_kernel<<<col_grid(nc, 1), 128, 0, s>>>(A, 0, lda, j0, jb, A, 0, lda, c0, nc);
        emu::note_launch();
        bgemm(n - c0, nc, jb, cd{-1.0, 0.0}, A + (size_t)c0 * lda + j0, 0, lda, A + (size_t)j0 * lda + c0, 0, lda,
              cd{1.0, 0.0}, A + (size_t)c0 * lda + c0, 0, lda, 1, s);
      }
    }
    const int c1 = J + JB, rest = n - c1;
    if (rest <= 0) continue;
    for (int r0 = J; r0 < c1; r0 += kNB) {  // U12 = L11^-1 A12, by blocks of kNB rows
      const int rb = std::min(kNB, c1 - r0);
      trsm_lower_kernel<<<col_grid(rest, 1), 128, 0, s>>>(A, 0, lda, r0, rb, A, 0, lda, c1, rest);
      emu::note_launch();
      const int below = c1 - (r0 + rb);
      if (below > 0)
        bgemm(below, rest, rb, cd{-1.0, 0.0}, A + (size_t)(r0 + rb) * lda + r0, 0, lda, A + (size_t)r0 * lda + c1, 0,
              lda, cd{1.0, 0.0}, A + (size_t)(r0 + rb) * lda + c1, 0, lda, 1, s);
    }
    bgemm(rest, rest, JB, cd{-1.0, 0.0}, A + (size_t)c1 * lda + J, 0, lda, A + (size_t)J * lda + c1, 0, lda,
          cd{1.0, 0.0}, A + (size_t)c1 * lda + c1, 0, lda, 1, s);
  }
}

// Y = A^-1 T for a narrow block T [n][nrhs] (A^-1 rows x n, T n x nrhs;
// n here is the inner extent, the columns of A^-1 kept): one row of A^-1
// per warp, streamed once per COLS vectors; T staged in shared memory 128
// rows at a time (read row by row, stored column-major with one pad entry
// per column so that both the staging writes and the lanes' reads avoid
// bank conflicts); the next chunk's A entries are loaded while the current
// one is summed; lanes split the k range and a butterfly sums each output.
// COLS = 16 for wide blocks (2 CTAs per SM), 4 for the Krylov iteration's
// blocks of up to 4 vectors (no multiply-adds and shared-memory reads for
// empty columns; 78 registers, so 3 CTAs per SM keep more loads in flight).
constexpr int kSkRows = 8, kSkK = 128, kSkPer = kSkK / 32;

template <int COLS>
__global__ void __launch_bounds__(256, COLS <= 4 ? 3 : 2) fem_skinny_kernel(int n, int nrhs, const cd *__restrict__ A, int lda,
                                                            const cd *__restrict__ T, int ldt, cd *Y, int ldy,
                                                            int rows) {
  __shared__ cd Ts[COLS][kSkK + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kSkRows + warp;
  const bool live = r < rows;
  const cd *Ar = A + (size_t)(live ? r : 0) * lda;
  for (int c0 = 0; c0 < nrhs; c0 += COLS) {
    const int nc = min(COLS, nrhs - c0);
    cd acc[COLS];
#pragma unroll
    for (int c = 0; c < COLS; ++c) acc[c] = cd{0.0, 0.0};
    cd a[kSkPer];
#pragma unroll
    for (int j = 0; j < kSkPer; ++j) {
      const int k = lane + 32 * j;
      a[j] = (live && k < n) ? Ar[k] : cd{0.0, 0.0};
    }
    for (int k0 = 0; k0 < n; k0 += kSkK) {
      __syncthreads();
      for (int e = threadIdx.x; e < kSkK * COLS; e += blockDim.x) {
        const int kk = e / COLS, c = e % COLS;
        Ts[c][kk] = (k0 + kk < n && c < nc) ? T[(size_t)(k0 + kk) * ldt + c0 + c] : cd{0.0, 0.0};
      }
      cd an[kSkPer];
#pragma unroll
      for (int j = 0; j < kSkPer; ++j) {
        const int k = k0 + kSkK + lane + 32 * j;
        an[j] = (live && k < n) ? Ar[k] : cd{0.0, 0.0};
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kSkPer; ++j) {
        const int kk = lane + 32 * j;
#pragma unroll
        for (int c = 0; c < COLS; ++c) {
          const cd t = Ts[c][kk];
          acc[c].x += a[j].x * t.x - a[j].y * t.y;
          acc[c].y += a[j].x * t.y + a[j].y * t.x;
        }
      }
#pragma unroll
      for (int j = 0; j < kSkPer; ++j) a[j] = an[j];
    }
#pragma unroll
    for (int c = 0; c < COLS; ++c) {
      for (int o = 16; o > 0; o >>= 1) {
        acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
        acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
      }
      if (lane == c && c < nc && live) Y[(size_t)r * ldy + c0 + c] = acc[c];
    }
  }
}

// X [n][nc]: column j = unit vector e_{cols[j]} (cols null: the identity)
__global__ void fem_identity_kernel(int n, int nc, const int32_t *cols, cd *X, int ldx) {
  const long long total = (long long)n * nc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / nc, c = i % nc;
    const long long one = cols ? cols[c] : c;
    X[r * ldx + c] = cd{r == one ? 1.0 : 0.0, 0.0};
  }
}

}  // namespace

extern "C" int emu_fem_lu(int n, emu_c128 *d_A, int lda, int32_t *d_ipiv, int32_t *d_info, void *stream) {
  if (n < 1 || lda < n) return EMU_E_SHAPE;
  if (!d_A || !d_ipiv || !d_info) return EMU_E_ARG;
  const cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(d_info, 0, sizeof(int32_t), s) != cudaSuccess) return EMU_E_CUDA;
  getrf_blocked(n, (cd *)d_A, lda, (int *)d_ipiv, (int *)d_info, s);
  return emu::check_launch();
}

extern "C" int emu_fem_inverse(int n, const emu_c128 *d_LU, int lda, const int32_t *d_ipiv, int ncols,
                               const int32_t *d_cols, emu_c128 *d_Ainv, int ldi, void *stream) {
  if (n < 1 || lda < n || ncols < 1 || ncols > n || ldi < ncols) return EMU_E_SHAPE;
  if (!d_LU || !d_ipiv || !d_Ainv || (const void *)d_LU == (const void *)d_Ainv) return EMU_E_ARG;
  if (!d_cols && ncols != n) return EMU_E_ARG;
  const cudaStream_t s = (cudaStream_t)stream;
  fem_identity_kernel<<<grid_for((long long)n * ncols, 256), 256, 0, s>>>(n, ncols, d_cols, (cd *)d_Ainv, ldi);
  emu::note_launch();
  getrs_multi(n, ncols, (const cd *)d_LU, 0, lda, (const int *)d_ipiv, 0, (cd *)d_Ainv, 0, ldi, 1, s);
  return emu::check_launch();
}

extern "C" int emu_fem_apply_op(int n, int nrhs, const emu_c128 *d_Ainv, int ldi, int ncols, const int32_t *d_cols,
                                const int32_t *d_row_ptr, const int32_t *d_col, const emu_c128 *d_M,
                                const emu_c128 *d_X, int ldx, emu_c128 *d_T, emu_c128 *d_Y, int ldy, void *stream) {
  if (n < 1 || nrhs < 0 || ncols < 1 || ncols > n || ldi < ncols || ldx < nrhs || ldy < nrhs) return EMU_E_SHAPE;
  if (nrhs == 0) return EMU_OK;
  if (!d_Ainv || !d_row_ptr || !d_col || !d_M || !d_X || !d_T || !d_Y) return EMU_E_ARG;
  if (!d_cols && ncols != n) return EMU_E_ARG;
  if (d_X == d_Y || d_T == d_Y || d_T == d_X) return EMU_E_ARG;
  const cudaStream_t s = (cudaStream_t)stream;
  fem_spmm_kernel<<<grid_for((long long)ncols * 32, 256), 256, 0, s>>>(
      ncols, d_cols, nrhs, d_row_ptr, d_col, (const cd *)d_M, (const cd *)d_X, ldx, (cd *)d_T, nrhs);
  emu::note_launch();
  const int grid = (n + kSkRows - 1) / kSkRows;
  if (nrhs <= 4)
    fem_skinny_kernel<4><<<grid, 256, 0, s>>>(ncols, nrhs, (const cd *)d_Ainv, ldi, (const cd *)d_T, nrhs,
                                              (cd *)d_Y, ldy, n);
  else
    fem_skinny_kernel<16><<<grid, 256, 0, s>>>(ncols, nrhs, (const cd *)d_Ainv, ldi, (const cd *)d_T, nrhs,
                                               (cd *)d_Y, ldy, n);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" size_t emu_fem_fields_workspace_size(const EmuFemFields *p) {
  if (!p || p->nval < 1) return 0;
  return emu::align_up((size_t)p->nval * sizeof(emu_c128), 256);
}

extern "C" int emu_fem_nodal_fields(const EmuFemFields *p, void *d_workspace, size_t workspace_bytes,
                                    void *stream) {
  if (!p || p->nel < 1 || p->neq < 1 || p->nval < 1 || p->ldv < p->nval) return EMU_E_ARG;
  if (!p->d_x || !p->d_table_nod || !p->d_shift || !p->d_ends || !p->d_dof || !p->d_vec || !p->d_sol)
    return EMU_E_ARG;
  if (!d_workspace || workspace_bytes < emu_fem_fields_workspace_size(p)) return EMU_E_WORKSPACE;
  const cudaStream_t s = (cudaStream_t)stream;
  FieldArgs a;
  a.nel = p->nel;
  a.nval = p->nval;
  a.ldv = p->ldv;
  a.x = p->d_x;
  a.tn = p->d_table_nod;
  a.shift = p->d_shift;
  a.ends = p->d_ends;
  a.dof = p->d_dof;
  a.bloch0 = p->bloch[0];
  a.bloch1 = p->bloch[1];
  a.vec = (const cd *)p->d_vec;
  a.sol = (cd *)p->d_sol;
  dim3 grid((unsigned)p->nel, (unsigned)std::min(8, (p->nval + 127) / 128));
  fem_nodal_kernel<<<grid, 128, 0, s>>>(a);
  emu::note_launch();
  cd *zmax = (cd *)d_workspace;
  fem_argmax_kernel<<<p->nval, 256, 0, s>>>(p->nel, p->nval, a.sol, zmax);
  emu::note_launch();
  fem_scale_kernel<<<grid_for((long long)p->nel * p->nval * 39, 256), 256, 0, s>>>(p->nel, p->nval, a.sol, zmax);
  emu::note_launch();
  return emu::check_launch();
}

// =============================================================== 1D gratings
// The mode solve of calc_modes_1d (backend/fortran/py_calc_modes_1d.f:
// 330-500) for the E-field formulation: per element E_x at its three P2
// nodes (discontinuous from element to element), E_y and E_z at its four P3
// nodes (x_min, x_max, x_min + h/3, x_min + 2h/3; continuous, the last
// element's x_max values the periodic images of the first element's x_min
// values), the element matrices of asmbly_1d.f, then the same assembly,
// factorisation and operator as the 2D solve.
namespace {

constexpr int kLoc1 = 11;
constexpr int kLoc1Sq = kLoc1 * kLoc1;

// Lagrange basis polynomials on [0, 1] (monomial coefficients, degree < 4)
void lagrange_coeffs(const double *nodes, int n, double c[4][4]) {
  for (int i = 0; i < n; ++i) {
    double p[4] = {1.0, 0.0, 0.0, 0.0};
    double den = 1.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double q[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < 3; ++k) {
        q[k + 1] += p[k];
        q[k] -= nodes[j] * p[k];
      }
      for (int k = 0; k < 4; ++k) p[k] = q[k];
      den *= nodes[i] - nodes[j];
    }
    for (int k = 0; k < 4; ++k) c[i][k] = p[k] / den;
  }
}

// int_0^1 f g dt for monomial coefficient vectors
double poly_int(const double *f, const double *g) {
  double s = 0.0;
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) s += f[a] * g[b] / (a + b + 1);
  return s;
}

struct Elem1dIntegrals {
  double Mxx[3][3], Kxy[3][4], Kyy[4][4], Myy[4][4];
};

// The reference element's integrals (the closed forms of matrix_mxx_1d.f,
// matrix_kxy_1d.f, matrix_kyy_1d.f, matrix_myy_1d.f on [0, 1]): P2 mass,
// P2 times P3 derivative, P3 stiffness, P3 mass.
Elem1dIntegrals elem1d_integrals() {
  const double n2[3] = {0.0, 1.0, 0.5}, n3[4] = {0.0, 1.0, 1.0 / 3.0, 2.0 / 3.0};
  double c2[4][4] = {}, c3[4][4] = {}, d3[4][4] = {};
  lagrange_coeffs(n2, 3, c2);
  lagrange_coeffs(n3, 4, c3);
  for (int i = 0; i < 4; ++i)
    for (int k = 1; k < 4; ++k) d3[i][k - 1] = k * c3[i][k];
  Elem1dIntegrals r;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) r.Mxx[i][j] = poly_int(c2[i], c2[j]);
    for (int j = 0; j < 4; ++j) r.Kxy[i][j] = poly_int(c2[i], d3[j]);
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      r.Kyy[i][j] = poly_int(d3[i], d3[j]);
      r.Myy[i][j] = poly_int(c3[i], c3[j]);
    }
  return r;
}

struct Elem1dArgs {
  int nel;
  const double *x;
  const int64_t *tn;
  const int64_t *type_el;
  const double *shift;
  cd qq[8];
  double by, bx;
  Elem1dIntegrals I;
  cd *Ke, *Me;
};

// one CTA per element, one thread per (trial, test) entry (asmbly_1d.f:
// 150-250 with pp = 1): groups X = 0..2 (E_x), Y = 3..6 (E_y), Z = 7..10 (E_z)
__global__ void fem1d_element_kernel(Elem1dArgs a) {
  const int e = blockIdx.x, idx = threadIdx.x;
  if (idx >= kLoc1Sq) return;
  const int ai = idx / kLoc1, bi = idx % kLoc1;   // trial, test
  const double xmin = a.x[a.tn[(size_t)e * 3] - 1], xmax = a.x[a.tn[(size_t)e * 3 + 1] - 1];
  const double h = xmax - xmin;
  const cd q = a.qq[a.type_el[e] - 1];
  const double by = a.by;
  const int ga = ai < 3 ? 0 : (ai < 7 ? 1 : 2), gb = bi < 3 ? 0 : (bi < 7 ? 1 : 2);
  const int la = ga == 0 ? ai : (ga == 1 ? ai - 3 : ai - 7), lb = gb == 0 ? bi : (gb == 1 ? bi - 3 : bi - 7);
  cd k{0.0, 0.0}, m{0.0, 0.0};
  const cd xx{by * by - q.x, -q.y};  // pp by^2 - qq
  if (ga == 0 && gb == 0) {
    const double v = a.I.Mxx[la][lb] * h;
    k = cd{xx.x * v, xx.y * v};
    m = cd{-v, 0.0};
  } else if (ga == 1 && gb == 0) {
    k = cd{0.0, -by * a.I.Kxy[lb][la]};   // -i by Kyx, Kyx = Kxy^T
  } else if (ga == 2 && gb == 0) {
    k = cd{-a.I.Kxy[lb][la], 0.0};
  } else if (ga == 0 && gb == 1) {
    k = cd{0.0, by * a.I.Kxy[la][lb]};
  } else if (ga == 1 && gb == 1) {
    const double kyy = a.I.Kyy[la][lb] / h, myy = a.I.Myy[la][lb] * h;
    k = cd{kyy - q.x * myy, -q.y * myy};
    m = cd{-myy, 0.0};
  } else if (ga == 2 && gb == 1) {
    k = cd{0.0, by * a.I.Myy[la][lb] * h};
  } else if (ga == 0 && gb == 2) {
    m = cd{a.I.Kxy[la][lb], 0.0};
  } else if (ga == 1 && gb == 2) {
    m = cd{0.0, by * a.I.Myy[la][lb] * h};
  } else {
    const double kyy = a.I.Kyy[la][lb] / h, myy = a.I.Myy[la][lb] * h;
    k = cd{kyy + xx.x * myy, xx.y * myy};
  }
  double sa, ca, sb, cb;
  sincos(a.bx * a.shift[(size_t)e * kLoc1 + ai], &sa, &ca);
  sincos(a.bx * a.shift[(size_t)e * kLoc1 + bi], &sb, &cb);
  const cd fac = cmul(cd{ca, -sa}, cd{cb, sb});
  a.Ke[(size_t)e * kLoc1Sq + idx] = cmul(k, fac);
  a.Me[(size_t)e * kLoc1Sq + idx] = cmul(m, fac);
}

struct Field1dArgs {
  int nel, nval, ldv;
  const int32_t *dof;
  const double *shift;
  double bx;
  const cd *vec;
  cd *sol;
};

__global__ void fem1d_nodal_kernel(Field1dArgs a) {
  const long long total = (long long)a.nel * a.nval;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i / a.nval), m = (int)(i % a.nval);
    cd *out = a.sol + ((size_t)e * a.nval + m) * kLoc1;
    for (int j = 0; j < kLoc1; ++j) {
      double sn, cs;
      sincos(a.bx * a.shift[(size_t)e * kLoc1 + j], &sn, &cs);
      out[j] = cmul(a.vec[(size_t)a.dof[(size_t)e * kLoc1 + j] * a.ldv + m], cd{cs, sn});
    }
  }
}

// x of local DOF j of an element (periodic_cond_1d.f's x_ddl)
__device__ __forceinline__ double dof1d_x(int j, double xmin, double xmax) {
  const double h = xmax - xmin;
  switch (j) {
    case 0: case 3: case 7: return xmin;
    case 1: case 4: case 8: return xmax;
    case 2: return xmin + h / 2.0;
    case 5: case 9: return xmin + h / 3.0;
    default: return xmin + 2.0 * h / 3.0;
  }
}

// array_sol_1d.f's choice of the value each mode is divided by: the first
// largest value within dx/4 of the cell's middle when it is at least 0.95 of
// the first largest value anywhere, else the first largest value right of
// the middle (prime modes) or left of it (adjoint modes).  One CTA per mode.
__global__ void fem1d_norm_kernel(int nel, int nval, const double *x, const int64_t *tn, int adjoint,
                                  const cd *sol, cd *zsel) {
  const int m = blockIdx.x;
  const double x0 = x[tn[0] - 1], x1 = x[tn[(size_t)(nel - 1) * 3 + 1] - 1];
  const double xm = 0.5 * (x0 + x1), dx = (x1 - x0) / nel;
  double best[4] = {-1.0, -1.0, -1.0, -1.0};  // all, middle, right, left
  long long bi[4] = {0, 0, 0, 0};
  const long long total = (long long)nel * kLoc1;
  for (long long f = threadIdx.x; f < total; f += blockDim.x) {
    const int e = (int)(f / kLoc1), j = (int)(f % kLoc1);
    const double xx = dof1d_x(j, x[tn[(size_t)e * 3] - 1], x[tn[(size_t)e * 3 + 1] - 1]);
    const cd v = sol[((size_t)e * nval + m) * kLoc1 + j];
    const double mag = hypot(v.x, v.y);
    const bool in[4] = {true, fabs(xx - xm) < dx / 4.0, xx > xm, xx < xm};
    for (int c = 0; c < 4; ++c)
      if (in[c] && mag > best[c]) {
        best[c] = mag;
        bi[c] = f;
      }
  }
  __shared__ double s_b[4][256];
  __shared__ long long s_i[4][256];
  for (int c = 0; c < 4; ++c) {
    s_b[c][threadIdx.x] = best[c];
    s_i[c][threadIdx.x] = bi[c];
  }
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int c = 0; c < 4; ++c) {
        const double ob = s_b[c][threadIdx.x + st];
        const long long oi = s_i[c][threadIdx.x + st];
        if (ob > s_b[c][threadIdx.x] || (ob == s_b[c][threadIdx.x] && ob >= 0.0 && oi < s_i[c][threadIdx.x])) {
          s_b[c][threadIdx.x] = ob;
          s_i[c][threadIdx.x] = oi;
        }
      }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    cd z[4];
    for (int c = 0; c < 4; ++c) {
      const long long f = s_i[c][0];
      z[c] = s_b[c][0] >= 0.0 ? sol[((size_t)(f / kLoc1) * nval + m) * kLoc1 + f % kLoc1] : cd{0.0, 0.0};
    }
    const double r = (z[0].x == 0.0 && z[0].y == 0.0) ? 0.0 : hypot(z[1].x, z[1].y) / hypot(z[0].x, z[0].y);
    zsel[m] = r >= 0.95 ? z[1] : (adjoint ? z[3] : z[2]);
  }
}

__global__ void fem1d_scale_kernel(int nel, int nval, cd *sol, const cd *z) {
  const long long total = (long long)nel * nval * kLoc1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    sol[i] = cdiv(sol[i], z[(i / kLoc1) % nval]);
}

}  // namespace

extern "C" int emu_fem1d_topology(EmuFem1dTopology *t) {
  if (!t || t->nel < 2 || t->npt < 3 || !t->h_x || !t->h_table_nod || !t->h_dof || !t->h_shift || !t->h_row_ptr ||
      !t->h_col || !t->h_src_ptr || !t->h_src)
    return EMU_E_ARG;
  const int nel = t->nel;
  const int64_t *tab = t->h_table_nod;
  for (long long i = 0; i < (long long)nel * 3; ++i)
    if (tab[i] < 1 || tab[i] > t->npt) return EMU_E_ARG;
  const double *x = t->h_x;
  const double x0 = x[tab[0] - 1], x1 = x[tab[(size_t)(nel - 1) * 3 + 1] - 1];
  const double span = x1 - x0;
  if (!(span > 0.0)) return EMU_E_ARG;
  for (int e = 0; e < nel; ++e) {
    const double a = x[tab[(size_t)e * 3] - 1], b = x[tab[(size_t)e * 3 + 1] - 1];
    if (!(b > a)) return EMU_E_ARG;  // elements run left to right
    if (e + 1 < nel && fabs(x[tab[(size_t)(e + 1) * 3] - 1] - b) > 1e-12 * span) return EMU_E_ARG;
  }
  // equations element by element: E_x (3), E_y at x_min, h/3, 2h/3, E_z the same
  for (int e = 0; e < nel; ++e) {
    int32_t *d = &t->h_dof[(size_t)e * kLoc1];
    const int b = 9 * e;
    d[0] = b;
    d[1] = b + 1;
    d[2] = b + 2;
    d[3] = b + 3;
    d[5] = b + 4;
    d[6] = b + 5;
    d[7] = b + 6;
    d[9] = b + 7;
    d[10] = b + 8;
  }
  for (int e = 0; e < nel; ++e) {
    const int nx = (e + 1) % nel;
    t->h_dof[(size_t)e * kLoc1 + 4] = t->h_dof[(size_t)nx * kLoc1 + 3];
    t->h_dof[(size_t)e * kLoc1 + 8] = t->h_dof[(size_t)nx * kLoc1 + 7];
    for (int j = 0; j < kLoc1; ++j) t->h_shift[(size_t)e * kLoc1 + j] = 0.0;
  }
  t->h_shift[(size_t)(nel - 1) * kLoc1 + 4] = span;
  t->h_shift[(size_t)(nel - 1) * kLoc1 + 8] = span;
  t->neq = 9 * nel;
  t->period = span;
  csr_pattern(nel, kLoc1, t->h_dof, t->neq, t->h_row_ptr, t->h_col, t->h_src_ptr, t->h_src, &t->nnz);
  return EMU_OK;
}

extern "C" int emu_fem1d_element_matrices(const EmuFem1dElements *p, void *stream) {
  if (!p || p->nel < 2 || p->n_types < 1 || p->n_types > 8) return EMU_E_ARG;
  if (!p->d_x || !p->d_table_nod || !p->d_type_el || !p->d_shift || !p->d_Ke || !p->d_Me) return EMU_E_ARG;
  Elem1dArgs a;
  a.nel = p->nel;
  a.x = p->d_x;
  a.tn = p->d_table_nod;
  a.type_el = p->d_type_el;
  a.shift = p->d_shift;
  for (int i = 0; i < 8; ++i) {
    const cd n{p->n_eff[i].re, p->n_eff[i].im};
    const cd eps = cmul(n, n);
    a.qq[i] = cd{eps.x * p->k0 * p->k0, eps.y * p->k0 * p->k0};
  }
  a.bx = p->bloch[0];
  a.by = p->bloch[1];
  a.I = elem1d_integrals();
  a.Ke = (cd *)p->d_Ke;
  a.Me = (cd *)p->d_Me;
  fem1d_element_kernel<<<p->nel, 128, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" size_t emu_fem1d_fields_workspace_size(const EmuFem1dFields *p) {
  if (!p || p->nval < 1) return 0;
  return emu::align_up((size_t)p->nval * sizeof(emu_c128), 256);
}

extern "C" int emu_fem1d_nodal_fields(const EmuFem1dFields *p, void *d_workspace, size_t workspace_bytes,
                                      void *stream) {
  if (!p || p->nel < 2 || p->neq < 1 || p->nval < 1 || p->ldv < p->nval) return EMU_E_ARG;
  if (!p->d_x || !p->d_table_nod || !p->d_shift || !p->d_dof || !p->d_vec || !p->d_sol) return EMU_E_ARG;
  if (!d_workspace || workspace_bytes < emu_fem1d_fields_workspace_size(p)) return EMU_E_WORKSPACE;
  const cudaStream_t s = (cudaStream_t)stream;
  Field1dArgs a{p->nel, p->nval, p->ldv, p->d_dof, p->d_shift, p->bloch_x, (const cd *)p->d_vec, (cd *)p->d_sol};
  fem1d_nodal_kernel<<<grid_for((long long)p->nel * p->nval, 128), 128, 0, s>>>(a);
  emu::note_launch();
  cd *z = (cd *)d_workspace;
  fem1d_norm_kernel<<<p->nval, 256, 0, s>>>(p->nel, p->nval, p->d_x, p->d_table_nod, p->adjoint, a.sol, z);
  emu::note_launch();
  fem1d_scale_kernel<<<grid_for((long long)p->nel * p->nval * kLoc1, 256), 256, 0, s>>>(p->nel, p->nval, a.sol, z);
  emu::note_launch();
  return emu::check_launch();
}
