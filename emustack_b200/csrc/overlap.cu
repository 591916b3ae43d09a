// Bloch-mode / plane-wave overlap integrals J and J_dag
// (backend/fortran/J_overlap.f:92-198, J_dagger_overlap.f:93-199) and the
// Bloch-mode orthogonality / normalisation factors
// (backend/fortran/orthogonal.f:84-248, normalisation.f:15-31).
//
// The reference loops element x quadrature point x plane wave x mode and
// re-interpolates the P2 field for every plane wave.  Here the quadrature
// is folded into a plane-wave table first:
//   E~_s(el, node) = sum_q w_q |det_el| exp(-i k_s . x_q) phi_node(xi_q)
// (16 quadrature points, affine element map), so that
//   G_c[s, n] = sum_{el,node} E~_s(el, node) sol(c, node, n, el),  c = x, y
// is one complex GEMM with K = 6 nel, and
//   J_E = (beta o G_x - alpha o G_y) / |k_s|,  J_K = (alpha o G_x + beta o G_y) / |k_s|
// in the epilogue (rows in the sorted plane-wave order of pw_ordering.f).
// J_dag uses conj(E~) (exp(+i k.x)) and the adjoint fields.
// The exponentials factor as exp(-i(a0 x + b0 y)) (exp(-i 2 pi x / d))^px
// (exp(-i 2 pi y / dy))^py: per quadrature point one base phase and two
// short power tables replace a sine/cosine per plane wave.
#include <cuda_runtime.h>

#include "dense_la.cuh"
#include "emu_internal.h"

namespace {

using namespace emu;

__constant__ double c_wq[16], c_xq[16], c_yq[16];
__constant__ double c_phi2[16][6];       // P2 basis at the quadrature points
__constant__ float c_phi2f[16][6];       // the same, rounded to FP32 (tensor-core operand path)
__constant__ double c_g3[16][2][10];     // P3 gradients (reference triangle)

// 16-point symmetric rule of Lyness & Jespersen (J. Inst. Math. Appl. 15,
// 1975), as tabulated in backend/fortran/quad_triangle.f:56-145.
void quad_table(double *w, double *x, double *y) {
  const double wbar = 1.443156076777862e-1 / 2.0, w1 = 2.852749028018549e-1 / 6.0;
  const double w2 = 9.737549286959440e-2 / 6.0, w3 = 3.096521116041552e-1 / 6.0;
  const double w4 = 1.633818850466092e-1 / 12.0;
  const double cb = 1.0 / 3.0, a1 = 4.592925882927229e-1, b1 = 8.141482341455413e-2;
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

int upload_tables() {
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done[dev]) return EMU_OK;
  double w[16], x[16], y[16], phi[16][6], g[16][2][10];
  float phif[16][6];
  quad_table(w, x, y);
  for (int q = 0; q < 16; ++q) {
    const double x0 = x[q], y0 = y[q];
    // P2 basis (backend/fortran/phi2_2d_mat_J.f:17-30)
    phi[q][0] = (-1 + x0 + y0) * (-1 + 2 * x0 + 2 * y0);
    phi[q][1] = x0 * (-1 + 2 * x0);
    phi[q][2] = y0 * (-1 + 2 * y0);
    phi[q][3] = -4 * x0 * (-1 + x0 + y0);
    phi[q][4] = 4 * x0 * y0;
    phi[q][5] = -4 * y0 * (-1 + x0 + y0);
    for (int k = 0; k < 6; ++k) phif[q][k] = (float)phi[q][k];
    // P3 gradients (backend/fortran/phi3_2d_mat.f:17-64)
    const double t = (-11 - 27 * x0 * x0 + x0 * (36 - 54 * y0) + 36 * y0 - 27 * y0 * y0) / 2.;
    g[q][0][0] = t; g[q][1][0] = t;
    g[q][0][1] = 1 - 9 * x0 + (27 * x0 * x0) / 2.; g[q][1][1] = 0;
    g[q][0][2] = 0; g[q][1][2] = 1 - 9 * y0 + (27 * y0 * y0) / 2.;
    g[q][0][3] = (9 * (2 + 9 * x0 * x0 - 5 * y0 + 3 * y0 * y0 + 2 * x0 * (-5 + 6 * y0))) / 2.;
    g[q][1][3] = (9 * x0 * (-5 + 6 * x0 + 6 * y0)) / 2.;
    g[q][0][4] = (-9 * (1 + 9 * x0 * x0 - y0 + x0 * (-8 + 6 * y0))) / 2.;
    g[q][1][4] = (-9 * x0 * (-1 + 3 * x0)) / 2.;
    g[q][0][5] = (9 * (-1 + 6 * x0) * y0) / 2.;
    g[q][1][5] = (9 * x0 * (-1 + 3 * x0)) / 2.;
    g[q][0][6] = (9 * y0 * (-1 + 3 * y0)) / 2.;
    g[q][1][6] = (9 * x0 * (-1 + 6 * y0)) / 2.;
    g[q][0][7] = (-9 * y0 * (-1 + 3 * y0)) / 2.;
    g[q][1][7] = (-9 * (1 - 8 * y0 + 9 * y0 * y0 + x0 * (-1 + 6 * y0))) / 2.;
    g[q][0][8] = (9 * y0 * (-5 + 6 * x0 + 6 * y0)) / 2.;
    g[q][1][8] = (9 * (2 + 3 * x0 * x0 - 10 * y0 + 9 * y0 * y0 + x0 * (-5 + 12 * y0))) / 2.;
    g[q][0][9] = -27 * y0 * (-1 + 2 * x0 + y0);
    g[q][1][9] = -27 * x0 * (-1 + x0 + 2 * y0);
  }
  if (cudaMemcpyToSymbol(c_wq, w, sizeof(w)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_xq, x, sizeof(x)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_yq, y, sizeof(y)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_phi2, phi, sizeof(phi)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_phi2f, phif, sizeof(phif)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_g3, g, sizeof(g)) != cudaSuccess)
    return EMU_E_CUDA;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return EMU_OK;
}

// Element geometry: vertices, affine map x = B xi + x1, |det B| and T = B^-1
// (backend/fortran/jacobian_p1_2d.f:68-133).
struct Geo {
  double x1, y1, B00, B01, B10, B11, adet, T00, T01, T10, T11;
};

__device__ __forceinline__ Geo element_geo(const double *x, const int64_t *tn, long el) {
  const int64_t n1 = tn[el * 6 + 0] - 1, n2 = tn[el * 6 + 1] - 1, n3 = tn[el * 6 + 2] - 1;
  Geo g;
  g.x1 = x[2 * n1];
  g.y1 = x[2 * n1 + 1];
  g.B00 = x[2 * n2] - g.x1;
  g.B01 = x[2 * n3] - g.x1;
  g.B10 = x[2 * n2 + 1] - g.y1;
  g.B11 = x[2 * n3 + 1] - g.y1;
  const double det = g.B00 * g.B11 - g.B01 * g.B10;
  g.adet = fabs(det);
  g.T00 = g.B11 / det;
  g.T01 = -g.B01 / det;
  g.T10 = -g.B10 / det;
  g.T11 = g.B00 / det;
  return g;
}

// ---------------------------------------------------------------- setup
// Plane-wave data per problem: sorted position (pw_ordering.f:54-78 with the
// z_indexx.f key -Re(kz^2)), alpha, beta and 1/|k| by sorted row.
struct PwArgs {
  int batch, npw;
  const int32_t *px, *py;
  double d, dy;
  const double *bloch, *k0;
  int32_t *pos;       // [batch][npw] sorted position of generation-order s
  double *tab;        // [batch][npw][3]: alpha, beta, 1/|k| by sorted row
  int32_t *out_inv;   // optional copy of pos
};

__global__ void pw_setup_kernel(PwArgs a) {
  extern __shared__ double keys[];
  const int b = blockIdx.x;
  const double bx = a.bloch[2 * b], by = a.bloch[2 * b + 1], k0 = a.k0[b];
  const double vkx = 2.0 * 3.141592653589793 / a.d, vky = 2.0 * 3.141592653589793 / a.dy;
  for (int s = threadIdx.x; s < a.npw; s += blockDim.x) {
    const double al = bx + vkx * a.px[s], be = by + vky * a.py[s];
    const cd bz = csqrt_p(cd{k0 * k0 - al * al - be * be, 0.0});
    keys[s] = -(bz.x * bz.x - bz.y * bz.y);
  }
  __syncthreads();
  for (int s = threadIdx.x; s < a.npw; s += blockDim.x) {
    const double ks = keys[s];
    int r = 0;
    for (int v = 0; v < a.npw; ++v) r += (keys[v] < ks) || (keys[v] == ks && v < s);
    a.pos[(size_t)b * a.npw + s] = r;
    if (a.out_inv) a.out_inv[(size_t)b * a.npw + s] = r;
    const double al = bx + vkx * a.px[s], be = by + vky * a.py[s];
    double *t = a.tab + ((size_t)b * a.npw + r) * 3;
    t[0] = al;
    t[1] = be;
    t[2] = 1.0 / sqrt(al * al + be * be);
  }
}

// ---------------------------------------------------------------- E~ table
// One warp per element: lanes build the per-quadrature-point phase tables in
// shared memory, then each lane owns plane waves s and accumulates the six
// node sums E~_s(el, node).  Output row = sorted position of s, column
// (el - e0) * 6 + node; rows padded to ldE.
struct EtArgs {
  int npw, mo, e0, ne;
  const int32_t *px, *py, *pos;
  const double *x;
  const int64_t *tn;
  double d, dy;
  const double *bloch;  // this problem's k_parallel * period (2 values)
  cd *E;
  long long ldE;
  // tensor-core path: instead of E, the real embedding A (FP32,
  // [2 npw][2 K], K = 6 ne), columns in (element, node, re/im) order:
  // row s = (Re E, -Im E) pairs, row npw + s = (Im E, Re E) pairs
  float *A32;
  // tensor-core path, several problems per launch (blockIdx.y = problem):
  // per-problem strides of pos (ints) and A32 (floats); bloch advances by 2
  int spos;
  long long sA32;
};

constexpr int kEtWarps = 4;
constexpr int kMaxOrd = 24;  // |px|, |py| <= kMaxOrd

// dynamic shared memory per warp: base[16], tx[16][no], ty[16][no] (cd), cq[16]
__host__ __device__ inline size_t et_warp_bytes(int mo) {
  return sizeof(cd) * (16 + 2 * 16 * (size_t)(2 * mo + 1)) + sizeof(double) * 16;
}

// FP32 tables of the tensor-core operand path: bc[16] (base x weight),
// tx[16][no], ty[16][no] as float2
__host__ __device__ inline size_t et_warp_bytes_f32(int mo) {
  return sizeof(float2) * (16 + 2 * 16 * (size_t)(2 * mo + 1));
}

// kF32: tensor-core operand path.  The phase tables of each element are
// computed in FP64 (arguments, sincos, powers) and stored rounded to FP32
// (relative 6e-8 per entry); the phase products and the 16-point x 6-node
// sums then run in FP32 (~3e-7 relative), below the ~2^-21 relative error of
// the split-TF32 products they feed.  Half the table bytes of the FP64 path,
// so twice the resident warps.
template <bool kF32>
__global__ void __launch_bounds__(32 * kEtWarps) etable_kernel(EtArgs a) {
  extern __shared__ __align__(16) unsigned char et_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int no = 2 * a.mo + 1;
  if constexpr (kF32) {
    float2 *bc = (float2 *)(et_smem + (size_t)w * et_warp_bytes_f32(a.mo));  // [16]
    float2 *fx = bc + 16;                                                      // [16][no]
    float2 *fy = fx + 16 * no;                                                 // [16][no]
    const int prob = blockIdx.y;
    const double bx = a.bloch[2 * prob], by = a.bloch[2 * prob + 1];
    const int32_t *pos = a.pos + (size_t)prob * a.spos;
    float *A32 = a.A32 + (size_t)prob * a.sA32;
    const long long K = 6LL * a.ne;
    for (long el0 = (long)blockIdx.x * kEtWarps; el0 < a.ne; el0 += (long)gridDim.x * kEtWarps) {
      const long el = el0 + w;
      const bool ok = el < a.ne;
      if (ok && lane < 16) {
        const Geo g = element_geo(a.x, a.tn, a.e0 + el);
        const int q = lane;
        const double xg = g.x1 + g.B00 * c_xq[q] + g.B01 * c_yq[q];
        const double yg = g.y1 + g.B10 * c_xq[q] + g.B11 * c_yq[q];
        const double wq = c_wq[q] * g.adet;
        double s, c;
        sincos(-(bx * xg + by * yg), &s, &c);
        bc[q] = make_float2((float)(c * wq), (float)(s * wq));
        double sx, cx, sy, cy;
        sincos(-2.0 * 3.141592653589793 / a.d * xg, &sx, &cx);
        sincos(-2.0 * 3.141592653589793 / a.dy * yg, &sy, &cy);
        const cd ux = cd{cx, sx}, uy = cd{cy, sy};
        cd px = cd{1.0, 0.0}, py = cd{1.0, 0.0};
        fx[q * no + a.mo] = make_float2(1.f, 0.f);
        fy[q * no + a.mo] = make_float2(1.f, 0.f);
        for (int p = 1; p <= a.mo; ++p) {
          px = cmul(px, ux);
          py = cmul(py, uy);
          fx[q * no + a.mo + p] = make_float2((float)px.x, (float)px.y);
          fx[q * no + a.mo - p] = make_float2((float)px.x, (float)-px.y);
          fy[q * no + a.mo + p] = make_float2((float)py.x, (float)py.y);
          fy[q * no + a.mo - p] = make_float2((float)py.x, (float)-py.y);
        }
      }
      __syncwarp();
      if (ok) {
        for (int s = lane; s < a.npw; s += 32) {
          const int ix = a.px[s] + a.mo, iy = a.py[s] + a.mo;
          float2 acc[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) acc[k] = make_float2(0.f, 0.f);
#pragma unroll 4
          for (int q = 0; q < 16; ++q) {
            const float2 b = bc[q], u = fx[q * no + ix], v = fy[q * no + iy];
            const float2 t = make_float2(b.x * u.x - b.y * u.y, b.x * u.y + b.y * u.x);
            const float ex = t.x * v.x - t.y * v.y, ey = t.x * v.y + t.y * v.x;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
              acc[k].x = fmaf(ex, c_phi2f[q][k], acc[k].x);
              acc[k].y = fmaf(ey, c_phi2f[q][k], acc[k].y);
            }
          }
          // K order (element, node, re/im): 12 contiguous floats per row
          float4 *r0 = (float4 *)(A32 + (size_t)pos[s] * 2 * K + (size_t)el * 12);
          float4 *r1 = (float4 *)((float *)r0 + (size_t)a.npw * 2 * K);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            r0[k] = make_float4(acc[2 * k].x, -acc[2 * k].y, acc[2 * k + 1].x, -acc[2 * k + 1].y);
            r1[k] = make_float4(acc[2 * k].y, acc[2 * k].x, acc[2 * k + 1].y, acc[2 * k + 1].x);
          }
        }
      }
      __syncwarp();
    }
    return;
  }
  cd *wb = (cd *)(et_smem + (size_t)w * et_warp_bytes(a.mo));
  cd *base = wb;                 // [16]
  cd *tx = base + 16;            // [16][no]
  cd *ty = tx + 16 * no;         // [16][no]
  double *cq = (double *)(ty + 16 * no);
  const double bx = a.bloch[0], by = a.bloch[1];
  for (long el0 = (long)blockIdx.x * kEtWarps; el0 < a.ne; el0 += (long)gridDim.x * kEtWarps) {
    const long el = el0 + w;
    const bool ok = el < a.ne;
    if (ok && lane < 16) {
      const Geo g = element_geo(a.x, a.tn, a.e0 + el);
      const int q = lane;
      const double xg = g.x1 + g.B00 * c_xq[q] + g.B01 * c_yq[q];
      const double yg = g.y1 + g.B10 * c_xq[q] + g.B11 * c_yq[q];
      cq[q] = c_wq[q] * g.adet;
      double s, c;
      sincos(-(bx * xg + by * yg), &s, &c);
      base[q] = cd{c, s};
      // powers of exp(-i 2 pi x / d) and exp(-i 2 pi y / dy), exponents -mo..mo
      double sx, cx, sy, cy;
      sincos(-2.0 * 3.141592653589793 / a.d * xg, &sx, &cx);
      sincos(-2.0 * 3.141592653589793 / a.dy * yg, &sy, &cy);
      const cd ux = cd{cx, sx}, uy = cd{cy, sy};
      cd px = cd{1.0, 0.0}, py = cd{1.0, 0.0};
      tx[q * no + a.mo] = px;
      ty[q * no + a.mo] = py;
      for (int p = 1; p <= a.mo; ++p) {
        px = cmul(px, ux);
        py = cmul(py, uy);
        tx[q * no + a.mo + p] = px;
        tx[q * no + a.mo - p] = cconj(px);
        ty[q * no + a.mo + p] = py;
        ty[q * no + a.mo - p] = cconj(py);
      }
    }
    __syncwarp();
    if (ok) {
      for (int s = lane; s < a.npw; s += 32) {
        const int ix = a.px[s] + a.mo, iy = a.py[s] + a.mo;
        {
          cd acc[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) acc[k] = cd{0.0, 0.0};
#pragma unroll 4
          for (int q = 0; q < 16; ++q) {
            const cd e = cscale(cmul(cmul(base[q], tx[q * no + ix]), ty[q * no + iy]), cq[q]);
#pragma unroll
            for (int k = 0; k < 6; ++k) {
              acc[k].x = fma(e.x, c_phi2[q][k], acc[k].x);
              acc[k].y = fma(e.y, c_phi2[q][k], acc[k].y);
            }
          }
          cd *row = a.E + (size_t)a.pos[s] * a.ldE + (size_t)el * 6;
#pragma unroll
          for (int k = 0; k < 6; ++k) row[k] = acc[k];
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- repack
// S[(el - e0) * 6 + node][c * nval + n] = sol[el][n][node][c], c = 0, 1
// (the transverse field of the reference layout sol(3, 13, nval, nel)).
__global__ void repack_kernel(const cd *sol, int nval, long e0, long ne, cd *S) {
  const long total = ne * 6 * 2 * (long)nval;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int n = (int)(i % nval);
    long r = i / nval;
    const int c = (int)(r % 2);
    r /= 2;
    const int node = (int)(r % 6);
    const long el = r / 6;
    S[(size_t)(el * 6 + node) * 2 * nval + (size_t)c * nval + n] =
        sol[((size_t)(e0 + el) * nval + n) * 39 + node * 3 + c];
  }
}

// ---------------------------------------------------------------- GEMM
// G[b] (+)= op(E) S with op = identity or conjugation, row-major; grid
// (n-tiles, m-tiles, chunks), chunk c writes G_part[c].
struct OvGemm {
  int m, n, k;
  const cd *E;
  long long ldE;
  const cd *S;
  cd *G;
  long long sG;
  int conjA;
  int kchunk;
};

// The contraction on the FP64 tensor cores: one 64 x 64 complex tile of
// G_part[c] per CTA through cta_gemm_tile (mma.sync m8n8k4 f64).
__global__ void __launch_bounds__(kDLThreads) ov_gemm_tc_kernel(OvGemm g) {
  __shared__ GemmSmem sm;
  const int c = blockIdx.z;
  const int k0 = c * g.kchunk;
  const int kk = min(g.kchunk, g.k - k0);
  if (kk <= 0) return;
  cta_gemm_tile(g.m, g.n, kk, cd{1.0, 0.0}, g.E + k0, (int)g.ldE, g.S + (size_t)k0 * g.n, g.n, cd{0.0, 0.0},
                g.G + (size_t)c * g.sG, g.n, blockIdx.y * kTM, blockIdx.x * kTN, sm, nullptr, nullptr,
                g.conjA != 0);
}

// Sum the chunk partials into the accumulator (fixed order: deterministic).
__global__ void reduce_parts_kernel(const cd *parts, int nparts, long long stride, cd *acc, long long n,
                                    int first) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    cd s = first ? cd{0.0, 0.0} : acc[i];
    for (int p = 0; p < nparts; ++p) s = cadd(s, parts[(size_t)p * stride + i]);
    acc[i] = s;
  }
}

// ---------------------------------------------------------------- epilogue
// J[row][n]: rows 0..npw-1 = J_E, npw..2npw-1 = J_K (sorted order), divided
// by area_norm; J_dag[i][row] uses adjoint column perm[i] scaled by scale[i].
__global__ void epilogue_kernel(const cd *G, const double *tab, int npw, int nval, double inv_area,
                                int dagger, const cd *scale, const int32_t *perm, cd *out) {
  // problem blockIdx.y: every array advances by its per-problem size
  const long long y = blockIdx.y;
  G += y * 2 * npw * (long long)nval;
  tab += y * 3 * npw;
  if (scale) scale += y * nval;
  if (perm) perm += y * nval;
  out += y * 2 * npw * (long long)nval;
  const long total = (long)npw * nval;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nval), n = (int)(i % nval);
    const double al = tab[3 * r], be = tab[3 * r + 1], nm = tab[3 * r + 2];
    const int src = (dagger && perm) ? perm[n] : n;
    const cd gx = G[(size_t)r * 2 * nval + src], gy = G[(size_t)r * 2 * nval + nval + src];
    cd je = cscale(cd{be * gx.x - al * gy.x, be * gx.y - al * gy.y}, nm);
    cd jk = cscale(cd{al * gx.x + be * gy.x, al * gx.y + be * gy.y}, nm);
    if (!dagger) {
      out[(size_t)r * nval + n] = cscale(je, inv_area);
      out[(size_t)(npw + r) * nval + n] = cscale(jk, inv_area);
    } else {
      if (scale) {
        je = cmul(je, scale[n]);
        jk = cmul(jk, scale[n]);
      }
      out[(size_t)n * 2 * npw + r] = je;
      out[(size_t)n * 2 * npw + npw + r] = jk;
    }
  }
}

// ---------------------------------------------------------------- orthogonality
// Per element, the 12 x 22 real matrix of orthogonal.f:110-193 without the
// pp(type_el) / k0 factor: rows (component, P2 node), columns P2 mass part
// (12) then -grad P3 part (10).
__device__ void element_scal(const Geo &g, double ms[12][22]) {
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 22; ++j) ms[i][j] = 0.0;
  for (int q = 0; q < 16; ++q) {
    const double c = c_wq[q] * g.adet;
    double g3[2][10];
    for (int j = 0; j < 10; ++j) {
      g3[0][j] = g.T00 * c_g3[q][0][j] + g.T10 * c_g3[q][1][j];
      g3[1][j] = g.T01 * c_g3[q][0][j] + g.T11 * c_g3[q][1][j];
    }
    for (int it = 0; it < 6; ++it) {
      const double pi = c_phi2[q][it] * c;
      for (int jt = 0; jt < 6; ++jt) {
        const double v = pi * c_phi2[q][jt];
        ms[2 * it][2 * jt] += v;
        ms[2 * it + 1][2 * jt + 1] += v;
      }
      for (int jt = 0; jt < 10; ++jt) {
        ms[2 * it][12 + jt] -= pi * g3[0][jt];
        ms[2 * it + 1][12 + jt] -= pi * g3[1][jt];
      }
    }
  }
}

// sol_el_1 entry j of mode n (orthogonal.f:205-227), without the beta factor
__device__ __forceinline__ cd sol1_entry(const cd *s1, int j) {
  if (j < 12) return s1[(j >> 1) * 3 + (j & 1)];
  const int t = j - 12;  // P3 nodes: vertices 0..2, then nodes 6..12
  return s1[(t < 3 ? t : t + 3) * 3 + 2];
}

// Diagonal of the orthogonality matrix for a batch: block (chunk c, problem
// b) stages the element matrices of kDiagChunk elements in shared memory
// (precomputed once per mesh by elem_scal_kernel), then each thread takes
// modes n = tid, tid + 128, ... and sums its chunk's contribution.
constexpr int kDiagChunk = 16;

struct DiagArgs {
  int nval;
  long nel;
  const double *ms_all;  // [nel][12][22]
  const int64_t *type_el;
  const cd *pp, *sol1, *sol2;  // sol: [B][nel][nval][13][3]
  const double *k0;            // [B]
  cd *part;                    // [B][nchunks][nval]
};

__global__ void __launch_bounds__(128) diag_kernel(DiagArgs a) {
  __shared__ double ms[kDiagChunk][264];
  __shared__ cd ppk[kDiagChunk];
  const long c = blockIdx.x, nch = gridDim.x;
  const int b = blockIdx.y;
  const long e0 = c * kDiagChunk;
  const int ne = (int)min((long)kDiagChunk, a.nel - e0);
  for (int i = threadIdx.x; i < ne * 264; i += blockDim.x)
    ms[i / 264][i % 264] = a.ms_all[(size_t)e0 * 264 + i];
  if (threadIdx.x < ne) {
    const cd p = a.pp[a.type_el[e0 + threadIdx.x] - 1];
    ppk[threadIdx.x] = cd{p.x / a.k0[b], p.y / a.k0[b]};
  }
  __syncthreads();
  const size_t sb = (size_t)b * a.nel * a.nval * 39;
  for (int n = threadIdx.x; n < a.nval; n += blockDim.x) {
    cd acc = cd{0.0, 0.0};
    for (int e = 0; e < ne; ++e) {
      const cd *s1 = a.sol1 + sb + ((size_t)(e0 + e) * a.nval + n) * 39;
      const cd *s2 = a.sol2 + sb + ((size_t)(e0 + e) * a.nval + n) * 39;
      cd s1v[22];
#pragma unroll
      for (int j = 0; j < 22; ++j) s1v[j] = sol1_entry(s1, j);
      const double *m = ms[e];
      cd v_e = cd{0.0, 0.0};
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        cd v = cd{0.0, 0.0};
#pragma unroll
        for (int j = 0; j < 22; ++j) {
          v.x = fma(m[i * 22 + j], s1v[j].x, v.x);
          v.y = fma(m[i * 22 + j], s1v[j].y, v.y);
        }
        v_e = cadd(v_e, cmul(v, s2[(i >> 1) * 3 + (i & 1)]));
      }
      acc = cadd(acc, cmul(v_e, ppk[e]));
    }
    a.part[((size_t)b * nch + c) * a.nval + n] = acc;
  }
}

// diag(n) = beta1(n) sum_chunks part ; scale = 1/sqrt(diag)^2 (or 1); one
// thread per (problem, mode)
__global__ void diag_finish_kernel(const cd *part, int nchunks, int nval, int batch, const cd *beta1,
                                   cd *diag, cd *scale, int *n_small) {
  const long total = (long)batch * nval;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int b = (int)(t / nval), n = (int)(t % nval);
    cd s = cd{0.0, 0.0};
    for (int c = 0; c < nchunks; ++c) s = cadd(s, part[((size_t)b * nchunks + c) * nval + n]);
    s = cmul(s, beta1[t]);
    diag[t] = s;
    if (hypot(s.x, s.y) <= 1e-7) atomicAdd(n_small + b, 1);
    const cd z = csqrt_p(s);
    scale[t] = (hypot(z.x, z.y) > 1e-8) ? crecip(cmul(z, z)) : cd{1.0, 0.0};
  }
}

// ---------------------------------------------------------------- tensor-core operands
// Tensor-core path: the complex contractions G = E~ . S1 and
// G_dag = conj(E~) . S2 = conj(E~ . conj(S2)) share one real GEMM
//   C[2 npw][Nb] = A[2 npw][2 K] . B[Nb][2 K]^T
// with A from etable_kernel (A32 output) and B rows, K in (element, node,
// re/im) order,
//   c * M + m          = (Re S1, Im S1) pairs   (c = 0, 1: x, y component)
//   off1 + c * M + m   = (Re S2, -Im S2) pairs  (off1 = 2 M when S1 is present)
// B tile builder: 8 modes x 16 elements per CTA; the 12 transverse values
// (node 0-5, component 0-1) of each (element, mode) record are read with
// consecutive lanes, staged in shared memory and written as rows of
// 192 contiguous floats.
// Field records may be complex128 (the reference's layout) or complex64 in
// the same layout (half the bytes; the B operand is FP32 either way).
constexpr int kBModes = 8, kBElems = 16;
struct cf32 {
  float x, y;
};
__device__ __forceinline__ cd to_cd(const cd &v) { return v; }
__device__ __forceinline__ cd to_cd(const cf32 &v) { return cd{(double)v.x, (double)v.y}; }

template <class Rec>
__global__ void __launch_bounds__(256) make_B_kernel(const Rec *sol_, long long ssol, int nval, long e0, long ne,
                                                     int conj, int row0, float *B_, long long sB) {
  __shared__ cd v[kBModes][kBElems][12];
  const Rec *sol = sol_ + (size_t)blockIdx.z * ssol;  // problem blockIdx.z
  float *B = B_ + (size_t)blockIdx.z * sB;
  const long long K = 6LL * ne;
  const int m0 = blockIdx.x * kBModes;
  const long el0 = (long)blockIdx.y * kBElems;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // load: warp w takes mode m0 + w, two elements per step (lanes 0-23)
  const int m = m0 + w;
  if (lane < 24) {
    const int j = lane % 12, eo = lane / 12;
    const int node = j >> 1, c = j & 1;
#pragma unroll
    for (int e = eo; e < kBElems; e += 2) {
      const long el = el0 + e;
      cd x = cd{0.0, 0.0};
      if (m < nval && el < ne) x = to_cd(sol[((size_t)(e0 + el) * nval + m) * 39 + node * 3 + c]);
      v[w][e][j] = x;
    }
  }
  __syncthreads();
  // write: 16 rows (c, mode) x 192 floats (element, node, re/im)
  const int nel_here = (int)(ne - el0 < kBElems ? ne - el0 : kBElems);
  for (int i = threadIdx.x; i < 2 * kBModes * 192; i += 256) {
    const int within = i % 192, r = i / 192;
    const int c = r / kBModes, mm = r % kBModes;
    const int e = within / 12, node = (within % 12) >> 1, ri = within & 1;
    if (m0 + mm >= nval || e >= nel_here) continue;
    const cd x = v[mm][e][node * 2 + c];
    const float val = ri == 0 ? (float)x.x : (float)(conj ? -x.y : x.y);
    B[(size_t)(row0 + c * nval + m0 + mm) * 2 * K + (size_t)(el0 + e) * 12 + node * 2 + ri] = val;
  }
}

// G (+)= C[:, 0:2M] ; G_dag (+)= conj(C[:, off1:off1+2M]), C = FP64 sum of
// the tensor-core K-split partials Cp[prob][split][2 npw][nb]; problem
// blockIdx.y; G, Gd advance by gsz per problem.
__global__ void pack_G_parts_kernel(const float *Cp, int nsplit, int npw, int nb, int n2, cd *G_, cd *Gd_,
                                    long long gsz, int off1, int first) {
  const long long prob = blockIdx.y;
  const float *C = Cp + prob * nsplit * (long long)2 * npw * nb;
  cd *G = G_ ? G_ + prob * gsz : nullptr;
  cd *Gd = Gd_ ? Gd_ + prob * gsz : nullptr;
  const long long total = (long long)npw * n2, step = (long long)2 * npw * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i / n2), n = (int)(i % n2);
    double a0 = 0.0, a1 = 0.0, d0 = 0.0, d1 = 0.0;
    for (int sp = 0; sp < nsplit; ++sp) {
      const float *r0 = C + sp * step + (size_t)s * nb, *r1 = C + sp * step + (size_t)(npw + s) * nb;
      if (G) {
        a0 += (double)r0[n];
        a1 += (double)r1[n];
      }
      if (Gd) {
        d0 += (double)r0[off1 + n];
        d1 += (double)r1[off1 + n];
      }
    }
    if (G) G[i] = first ? cd{a0, a1} : cadd(G[i], cd{a0, a1});
    if (Gd) Gd[i] = first ? cd{d0, -d1} : cadd(Gd[i], cd{d0, -d1});
  }
}


// ---------------------------------------------------------------- pair reordering
// Full adjoint x prime matrix for the conjugate-pair reordering of
// orthogonal.f:252-301 (only run when a diagonal entry vanishes).
__global__ void elem_scal_kernel(const double *x, const int64_t *tn, long nel, double *ms_all) {
  for (long el = blockIdx.x * (long)blockDim.x + threadIdx.x; el < nel; el += (long)gridDim.x * blockDim.x) {
    double ms[12][22];
    element_scal(element_geo(x, tn, el), ms);
    double *o = ms_all + (size_t)el * 264;
    for (int i = 0; i < 12; ++i)
      for (int j = 0; j < 22; ++j) o[i * 22 + j] = ms[i][j];
  }
}

// ovl[i][j] = sum_el (pp_e / k0) sol2_el(:, i)^T ms_el (beta1(j) sol1_el(:, j)); one thread per (i, j).
__global__ void ovl_full_kernel(const double *ms_all, int nval, long nel, const int64_t *type_el,
                                const cd *pp, const double *k0, const cd *beta1, const cd *sol1,
                                const cd *sol2, cd *ovl) {
  const long total = (long)nval * nval;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nval), j = (int)(t % nval);
    cd acc = cd{0.0, 0.0};
    for (long el = 0; el < nel; ++el) {
      const double *ms = ms_all + (size_t)el * 264;
      const cd *s1 = sol1 + ((size_t)el * nval + j) * 39;
      const cd *s2 = sol2 + ((size_t)el * nval + i) * 39;
      cd e = cd{0.0, 0.0};
      for (int r = 0; r < 12; ++r) {
        cd v = cd{0.0, 0.0};
        for (int c = 0; c < 22; ++c) {
          const cd s = sol1_entry(s1, c);
          v.x = fma(ms[r * 22 + c], s.x, v.x);
          v.y = fma(ms[r * 22 + c], s.y, v.y);
        }
        e = cadd(e, cmul(v, s2[(r >> 1) * 3 + (r & 1)]));
      }
      const cd p = pp[type_el[el] - 1];
      acc = cadd(acc, cmul(e, cd{p.x / k0[0], p.y / k0[0]}));
    }
    ovl[t] = cmul(acc, beta1[j]);
  }
}

// The reordering loop itself (one thread): swaps of adjoint modes recorded
// as a permutation; the recomputed diagonal is ovl[perm[i]][i].
__global__ void pair_swap_kernel(const cd *ovl, int nval, int32_t *perm, cd *diag, cd *scale, int32_t *warn) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < nval; ++i) perm[i] = i;
  int skip = 0, w = 0;
  for (int j = 0; j < nval; ++j) {
    const cd djj = ovl[(size_t)j * nval + j];
    if (hypot(djj.x, djj.y) > 1e-7) continue;
    if (skip == 0) {
      if (j == nval - 1) ++w;
      for (int j2 = j + 1; j2 < nval; ++j2) {
        const cd o = ovl[(size_t)j2 * nval + j];
        if (hypot(o.x, o.y) > 1e-7) {
          const int t = perm[j];
          perm[j] = perm[j2];
          perm[j2] = t;
        }
      }
      skip = 1;
    } else {
      skip = 0;
    }
  }
  for (int i = 0; i < nval; ++i) {
    const cd d = ovl[(size_t)perm[i] * nval + i];
    diag[i] = d;
    const cd z = csqrt_p(d);
    scale[i] = (hypot(z.x, z.y) > 1e-8) ? crecip(cmul(z, z)) : cd{1.0, 0.0};
  }
  *warn = w;
}

}  // namespace

// =============================================================== C ABI
// K splits of the FP64 overlap GEMM: 4, or enough CTAs for two waves when
// the output has few 64 x 64 tiles (few plane waves or modes)
static int ov_nparts(int npw, int M) {
  const int tiles = ((2 * M + kTN - 1) / kTN) * ((npw + kTM - 1) / kTM);
  if (tiles >= 32) return 4;
  const int n = (2 * emu::sm_count() + tiles - 1) / tiles;
  return n < 4 ? 4 : (n > 64 ? 64 : n);
}

// ---- tensor-core path: problems in groups, one launch per step for a group
struct TcPlan {
  long nec;        // elements per chunk
  long long K2;    // 12 nec: GEMM K of one chunk
  int nb, off1;    // B rows (2M per field set), row of the adjoint set
  int group;       // problems per launch
  int splits;      // K splits of the GEMM
};

constexpr size_t kTcGroupBytes = (size_t)4 << 30;  // scratch budget of one group
// The tensor cores accumulate in FP32 and the sum drifts toward zero by
// about 7e-9 x K relative (measured: 1.9e-6 rms at K = 256, 7.3e-6 at 1024,
// 1.8e-3 at 262144, for random operands).  The GEMM kernel therefore starts
// a fresh tensor-memory accumulation every 256 K values and sums those
// chunk results in FP32 (round to nearest) inside the CTA; a CTA's K range
// holds at most kTcMaxChunksPerCta chunks, and the K splits (CTAs) are
// summed in FP64.
constexpr long long kTcChunkK = 256;
constexpr long long kTcMaxChunksPerCta = 32;
constexpr int kTcMaxSplits = 256;
// element chunk (12 K values per element) of one GEMM
constexpr long kTcMaxChunk = 32768;

static size_t tc_problem_bytes(const EmuOverlap *p, const TcPlan &t) {
  const size_t npw = p->n_pw, M = p->nval;
  return align_up(sizeof(int32_t) * npw, 16) + align_up(sizeof(double) * 3 * npw, 16) +
         2 * align_up(sizeof(cd) * npw * 2 * M, 16) + sizeof(float) * 2 * npw * t.K2 +
         sizeof(float) * t.nb * t.K2 + sizeof(float) * t.splits * 2 * npw * t.nb;
}

static TcPlan tc_plan(const EmuOverlap *p) {
  TcPlan t;
  long chunk = p->elements_per_chunk > 0 ? p->elements_per_chunk : 4096;
  if (chunk > kTcMaxChunk) chunk = kTcMaxChunk;
  t.nec = chunk < p->nel ? chunk : p->nel;
  t.K2 = 12 * (long long)t.nec;
  t.nb = (p->d_sol1 ? 2 * p->nval : 0) + (p->d_sol2 ? 2 * p->nval : 0);
  if (t.nb == 0) t.nb = 2 * p->nval;
  t.off1 = p->d_sol1 ? 2 * p->nval : 0;
  // largest group within the budget (at one split), then splits so that
  // tiles x splits x group fills one wave of CTAs
  t.splits = 1;
  const size_t per = tc_problem_bytes(p, t);
  long long g = (long long)(kTcGroupBytes / (per > 0 ? per : 1));
  if (g < 1) g = 1;
  if (g > p->batch) g = p->batch;
  if (g > 1024) g = 1024;
  t.group = (int)g;
  const int tiles = emu::tc_tiles(2 * p->n_pw, t.nb) * t.group;
  int sp = (emu::sm_count() + tiles - 1) / tiles;
  const int maxsp = (int)(t.K2 / kTcChunkK > 0 ? t.K2 / kTcChunkK : 1);
  if (sp > maxsp) sp = maxsp;
  if (p->tc_splits > 0) sp = p->tc_splits;
  // accuracy floor, also under an explicit choice: no CTA sums more than
  // kTcMaxChunksPerCta chunk results in FP32
  const int need = (int)((t.K2 + kTcChunkK * kTcMaxChunksPerCta - 1) / (kTcChunkK * kTcMaxChunksPerCta));
  if (sp < need) sp = need;
  if (sp > kTcMaxSplits) sp = kTcMaxSplits;
  if (sp * t.group > 65535) sp = 65535 / t.group;
  t.splits = sp < 1 ? 1 : sp;
  return t;
}

extern "C" size_t emu_overlap_workspace_size(const EmuOverlap *p) {
  if (!p || p->n_pw < 1 || p->nval < 1 || p->nel < 1 || p->batch < 0) return 0;
  const long long npw = p->n_pw, M = p->nval;
  if (p->precision == 1) {
    const TcPlan t = tc_plan(p);
    return (size_t)t.group * tc_problem_bytes(p, t) + 16 * 256 + 256;
  }
  const long long chunk = p->elements_per_chunk > 0 ? p->elements_per_chunk : 4096;
  const long long ne = chunk < p->nel ? chunk : p->nel;
  const long long nparts = ov_nparts(p->n_pw, p->nval);
  size_t b = 0;
  b += align_up(sizeof(int32_t) * npw, 256);                 // pos
  b += align_up(sizeof(double) * 3 * npw, 256);              // tab
  b += align_up(sizeof(cd) * npw * 6 * ne, 256);             // E~ chunk
  b += align_up(sizeof(cd) * 6 * ne * 2 * M, 256);           // S chunk
  b += 2 * align_up(sizeof(cd) * npw * 2 * M, 256);          // G, Gd
  b += align_up(sizeof(cd) * nparts * npw * 2 * M, 256);     // partials
  return b + 256;
}

// Tensor-core J / J_dag for all problems, `group` problems per launch: plane
// waves, per element chunk the E~ table (as the FP32 A operand) and B (both
// field sets), one batched tcgen05 GEMM, the split sums folded into G / G_dag,
// then the epilogues.
static int overlap_tc(const EmuOverlap *p, void *ws, cudaStream_t s) {
  const TcPlan t = tc_plan(p);
  const int npw = p->n_pw, M = p->nval, Gp = t.group;
  const long long gsz = (long long)npw * 2 * M;
  char *w = (char *)ws;
  auto take = [&](size_t bytes) {
    char *r = w;
    w += align_up(bytes, 256);
    return (void *)r;
  };
  int32_t *pos = (int32_t *)take(sizeof(int32_t) * npw * Gp);
  double *tab = (double *)take(sizeof(double) * 3 * npw * Gp);
  cd *G = (cd *)take(sizeof(cd) * gsz * Gp);
  cd *Gd = (cd *)take(sizeof(cd) * gsz * Gp);
  float *A32 = (float *)take(sizeof(float) * 2 * npw * t.K2 * Gp);
  float *B32 = (float *)take(sizeof(float) * t.nb * t.K2 * Gp);
  float *Cpart = (float *)take(sizeof(float) * t.splits * 2 * npw * (size_t)t.nb * Gp);
  int *terr = p->d_error ? (int *)p->d_error : (int *)take(256);
  if (!p->d_error && cudaMemsetAsync(terr, 0, sizeof(int), s) != cudaSuccess) return EMU_E_CUDA;
  const int sms = emu::sm_count();
  const size_t et_smem32 = kEtWarps * et_warp_bytes_f32(p->max_order);
  if (et_smem32 > 48 * 1024 &&
      cudaFuncSetAttribute(etable_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)et_smem32) !=
          cudaSuccess)
    return EMU_E_CUDA;
  const long long ssol = (long long)p->nel * M * 39;
  const cd *sol1 = (const cd *)p->d_sol1, *sol2 = (const cd *)p->d_sol2;
  for (int g0 = 0; g0 < p->batch; g0 += Gp) {
    const int ng = (p->batch - g0) < Gp ? (p->batch - g0) : Gp;
    PwArgs pa;
    pa.batch = ng;
    pa.npw = npw;
    pa.px = p->d_px;
    pa.py = p->d_py;
    pa.d = p->d;
    pa.dy = p->dy;
    pa.bloch = p->d_bloch + 2 * (size_t)g0;
    pa.k0 = p->d_k0 + g0;
    pa.pos = pos;
    pa.tab = tab;
    pa.out_inv = p->d_index_pw_inv ? p->d_index_pw_inv + (size_t)g0 * npw : nullptr;
    pw_setup_kernel<<<ng, 256, sizeof(double) * npw, s>>>(pa);
    emu::note_launch();
    int first = 1;
    for (long e0 = 0; e0 < p->nel; e0 += t.nec) {
      const long ne = (p->nel - e0) < t.nec ? (p->nel - e0) : t.nec;
      const long long K2 = 12 * (long long)ne;
      EtArgs ea;
      ea.npw = npw;
      ea.mo = p->max_order;
      ea.e0 = (int)e0;
      ea.ne = (int)ne;
      ea.px = p->d_px;
      ea.py = p->d_py;
      ea.pos = pos;
      ea.x = p->d_x;
      ea.tn = p->d_table_nod;
      ea.d = p->d;
      ea.dy = p->dy;
      ea.bloch = p->d_bloch + 2 * (size_t)g0;
      ea.E = nullptr;
      ea.ldE = 6 * ne;
      ea.A32 = A32;
      ea.spos = npw;
      ea.sA32 = 2LL * npw * K2;
      long long eg = (ne + kEtWarps - 1) / kEtWarps;
      const long long egmax = (16LL * sms + ng - 1) / ng;
      if (eg > egmax) eg = egmax;
      etable_kernel<true><<<dim3((unsigned)eg, (unsigned)ng), 32 * kEtWarps, et_smem32, s>>>(ea);
      const dim3 bg((M + kBModes - 1) / kBModes, (unsigned)((ne + kBElems - 1) / kBElems), (unsigned)ng);
      const long long sB = (long long)t.nb * K2;
      if (p->field_c64) {
        const cf32 *f1 = (const cf32 *)p->d_sol1, *f2 = (const cf32 *)p->d_sol2;
        if (f1) make_B_kernel<cf32><<<bg, 256, 0, s>>>(f1 + (size_t)g0 * ssol, ssol, M, e0, ne, 0, 0, B32, sB);
        if (f2)
          make_B_kernel<cf32><<<bg, 256, 0, s>>>(f2 + (size_t)g0 * ssol, ssol, M, e0, ne, 1, t.off1, B32, sB);
      } else {
        if (sol1) make_B_kernel<cd><<<bg, 256, 0, s>>>(sol1 + (size_t)g0 * ssol, ssol, M, e0, ne, 0, 0, B32, sB);
        if (sol2)
          make_B_kernel<cd><<<bg, 256, 0, s>>>(sol2 + (size_t)g0 * ssol, ssol, M, e0, ne, 1, t.off1, B32, sB);
      }
      emu::note_launch(1 + (sol1 ? 1 : 0) + (sol2 ? 1 : 0));
      int used = 0;
      const int tst = emu::tc_gemm_tf32x3_parts(A32, 2LL * npw * K2, B32, sB, 2 * npw, t.nb, (int)K2, ng, t.splits,
                                                Cpart, terr, &used, s);
      if (tst != EMU_OK) return tst;
      long long rgs = (gsz + 255) / 256;
      if (rgs > 1024) rgs = 1024;
      pack_G_parts_kernel<<<dim3((unsigned)rgs, (unsigned)ng), 256, 0, s>>>(
          Cpart, used, npw, t.nb, 2 * M, sol1 ? G : nullptr, sol2 ? Gd : nullptr, gsz, t.off1, first);
      emu::note_launch();
      first = 0;
    }
    long long eb = ((long long)npw * M + 255) / 256;
    if (eb > 1024) eb = 1024;
    if (sol1) {
      epilogue_kernel<<<dim3((unsigned)eb, (unsigned)ng), 256, 0, s>>>(
          G, tab, npw, M, 1.0 / p->area_norm, 0, nullptr, nullptr, (cd *)p->d_J + (size_t)g0 * 2 * npw * M);
      emu::note_launch();
    }
    if (sol2) {
      epilogue_kernel<<<dim3((unsigned)eb, (unsigned)ng), 256, 0, s>>>(
          Gd, tab, npw, M, 1.0, 1, p->d_scale2 ? (const cd *)p->d_scale2 + (size_t)g0 * M : nullptr,
          p->d_perm2 ? p->d_perm2 + (size_t)g0 * M : nullptr, (cd *)p->d_J_dag + (size_t)g0 * 2 * npw * M);
      emu::note_launch();
    }
  }
  return emu::check_launch();
}

extern "C" int emu_overlap_batch(const EmuOverlap *p, void *d_workspace, size_t workspace_bytes,
                                 void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->batch < 0 || p->nval < 1 || p->nel < 1 || p->npt < 3 || p->n_pw < 1) return EMU_E_SHAPE;
  if (!p->d_px || !p->d_py || !p->d_x || !p->d_table_nod || !p->d_bloch || !p->d_k0) return EMU_E_ARG;
  if (!(p->d > 0) || !(p->dy > 0) || !(p->area_norm > 0)) return EMU_E_ARG;
  if ((p->d_sol1 == nullptr) != (p->d_J == nullptr) || (p->d_sol2 == nullptr) != (p->d_J_dag == nullptr))
    return EMU_E_ARG;
  if (p->max_order < 0 || p->max_order > kMaxOrd) return EMU_E_UNSUPPORTED;
  if (p->precision != 0 && p->precision != 1) return EMU_E_ARG;
  if (p->tc_splits < 0) return EMU_E_ARG;
  if (p->field_c64 != 0 && p->field_c64 != 1) return EMU_E_ARG;
  if (p->field_c64 && p->precision != 1) return EMU_E_UNSUPPORTED;  // the FP64 path reads complex128
  if (p->batch == 0) return EMU_OK;
  if (!d_workspace || workspace_bytes < emu_overlap_workspace_size(p)) return EMU_E_WORKSPACE;
  int st = upload_tables();
  if (st != EMU_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (p->precision == 1) return overlap_tc(p, d_workspace, s);
  const int npw = p->n_pw, M = p->nval;
  const long chunk = p->elements_per_chunk > 0 ? p->elements_per_chunk : 4096;
  const long nec = chunk < p->nel ? chunk : p->nel;
  const int nparts = ov_nparts(npw, M);
  char *w = (char *)d_workspace;
  auto take = [&](size_t bytes) {
    char *r = w;
    w += align_up(bytes, 256);
    return (void *)r;
  };
  int32_t *pos = (int32_t *)take(sizeof(int32_t) * npw);
  double *tab = (double *)take(sizeof(double) * 3 * npw);
  cd *E = (cd *)take(sizeof(cd) * (size_t)npw * 6 * nec);
  cd *S = (cd *)take(sizeof(cd) * 6 * (size_t)nec * 2 * M);
  cd *G = (cd *)take(sizeof(cd) * (size_t)npw * 2 * M);
  cd *Gd = (cd *)take(sizeof(cd) * (size_t)npw * 2 * M);
  cd *parts = (cd *)take(sizeof(cd) * (size_t)nparts * npw * 2 * M);
  const long long gsz = (long long)npw * 2 * M;
  const int sms = emu::sm_count();
  const size_t et_smem = kEtWarps * et_warp_bytes(p->max_order);
  if (et_smem > 48 * 1024 &&
      cudaFuncSetAttribute(etable_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)et_smem) !=
          cudaSuccess)
    return EMU_E_CUDA;
  for (int b = 0; b < p->batch; ++b) {
    PwArgs pa;
    pa.batch = 1;
    pa.npw = npw;
    pa.px = p->d_px;
    pa.py = p->d_py;
    pa.d = p->d;
    pa.dy = p->dy;
    pa.bloch = p->d_bloch + 2 * b;
    pa.k0 = p->d_k0 + b;
    pa.pos = pos;
    pa.tab = tab;
    pa.out_inv = p->d_index_pw_inv ? p->d_index_pw_inv + (size_t)b * npw : nullptr;
    pw_setup_kernel<<<1, 256, sizeof(double) * npw, s>>>(pa);
    emu::note_launch();
    const cd *sol1 = p->d_sol1 ? (const cd *)p->d_sol1 + (size_t)b * p->nel * M * 39 : nullptr;
    const cd *sol2 = p->d_sol2 ? (const cd *)p->d_sol2 + (size_t)b * p->nel * M * 39 : nullptr;
    for (int pass = 0; pass < 2; ++pass) {
      const cd *sol = pass == 0 ? sol1 : sol2;
      if (!sol) continue;
      cd *acc = pass == 0 ? G : Gd;
      int first = 1;
      for (long e0 = 0; e0 < p->nel; e0 += nec) {
        const long ne = (p->nel - e0) < nec ? (p->nel - e0) : nec;
        EtArgs ea;
        ea.npw = npw;
        ea.mo = p->max_order;
        ea.e0 = (int)e0;
        ea.ne = (int)ne;
        ea.px = p->d_px;
        ea.py = p->d_py;
        ea.pos = pos;
        ea.x = p->d_x;
        ea.tn = p->d_table_nod;
        ea.d = p->d;
        ea.dy = p->dy;
        ea.bloch = p->d_bloch + 2 * b;
        ea.E = E;
        ea.ldE = 6 * ne;
        ea.A32 = nullptr;
        ea.spos = 0;
        ea.sA32 = 0;
        const int eg = (int)((ne + kEtWarps - 1) / kEtWarps);
        etable_kernel<false><<<eg < 8 * sms ? eg : 8 * sms, 32 * kEtWarps, et_smem, s>>>(ea);
        const long long rn = ne * 6 * 2 * (long long)M;
        const long long rg = (rn + 255) / 256;
        repack_kernel<<<(int)(rg < 16 * sms ? rg : 16 * sms), 256, 0, s>>>(sol, M, e0, ne, S);
        OvGemm g;
        g.m = npw;
        g.n = 2 * M;
        g.k = (int)(6 * ne);
        g.E = E;
        g.ldE = 6 * ne;
        g.S = S;
        g.G = parts;
        g.sG = gsz;
        g.conjA = pass;
        g.kchunk = (int)(((6 * ne + nparts - 1) / nparts + kTK - 1) / kTK * kTK);
        const int used = (g.k + g.kchunk - 1) / g.kchunk;
        dim3 grid((2 * M + kTN - 1) / kTN, (npw + kTM - 1) / kTM, used);
        ov_gemm_tc_kernel<<<grid, kDLThreads, 0, s>>>(g);
        const long long rgs = (gsz + 255) / 256;
        reduce_parts_kernel<<<(int)(rgs < 8 * sms ? rgs : 8 * sms), 256, 0, s>>>(parts, used, gsz, acc, gsz,
                                                                                  first);
        emu::note_launch(4);
        first = 0;
      }
      const long long et = (long long)npw * M;
      const int eb = (int)((et + 255) / 256 < 8 * sms ? (et + 255) / 256 : 8 * sms);
      if (pass == 0) {
        epilogue_kernel<<<eb, 256, 0, s>>>(G, tab, npw, M, 1.0 / p->area_norm, 0, nullptr, nullptr,
                                           (cd *)p->d_J + (size_t)b * 2 * npw * M);
      } else {
        epilogue_kernel<<<eb, 256, 0, s>>>(
            Gd, tab, npw, M, 1.0, 1, p->d_scale2 ? (const cd *)p->d_scale2 + (size_t)b * M : nullptr,
            p->d_perm2 ? p->d_perm2 + (size_t)b * M : nullptr, (cd *)p->d_J_dag + (size_t)b * 2 * npw * M);
      }
      emu::note_launch();
    }
  }
  return emu::check_launch();
}

// ---------------------------------------------------------------- normalisation
extern "C" size_t emu_mode_overlap_workspace_size(const EmuNormalise *p) {
  if (!p || p->nval < 1 || p->nel < 1 || p->batch < 0) return 0;
  const long long nch = (p->nel + kDiagChunk - 1) / kDiagChunk;
  const long long B = p->batch > 0 ? p->batch : 1;
  return align_up(sizeof(double) * 264 * (size_t)p->nel, 256) +
         align_up(sizeof(cd) * B * nch * p->nval, 256) + 256;
}

extern "C" int emu_mode_overlap_diag(const EmuNormalise *p, void *d_workspace, size_t workspace_bytes,
                                     void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->batch < 0 || p->nval < 1 || p->nel < 1) return EMU_E_SHAPE;
  if (!p->d_x || !p->d_table_nod || !p->d_type_el || !p->d_pp || !p->d_k0 || !p->d_beta1 ||
      !p->d_sol1 || !p->d_sol2 || !p->d_diag || !p->d_scale || !p->d_n_small)
    return EMU_E_ARG;
  if (p->batch == 0) return EMU_OK;
  if (p->batch > 65535) return EMU_E_SHAPE;
  if (!d_workspace || workspace_bytes < emu_mode_overlap_workspace_size(p)) return EMU_E_WORKSPACE;
  int st = upload_tables();
  if (st != EMU_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const long nch = (p->nel + kDiagChunk - 1) / kDiagChunk;
  double *ms_all = (double *)d_workspace;
  cd *part = (cd *)((char *)d_workspace + align_up(sizeof(double) * 264 * (size_t)p->nel, 256));
  if (cudaMemsetAsync(p->d_n_small, 0, sizeof(int32_t) * p->batch, s) != cudaSuccess) return EMU_E_CUDA;
  const int sms = emu::sm_count();
  const long eb = (p->nel + 127) / 128;
  elem_scal_kernel<<<(int)(eb < 8 * sms ? eb : 8 * sms), 128, 0, s>>>(p->d_x, p->d_table_nod, p->nel, ms_all);
  DiagArgs a;
  a.nval = p->nval;
  a.nel = p->nel;
  a.ms_all = ms_all;
  a.type_el = p->d_type_el;
  a.pp = (const cd *)p->d_pp;
  a.sol1 = (const cd *)p->d_sol1;
  a.sol2 = (const cd *)p->d_sol2;
  a.k0 = p->d_k0;
  a.part = part;
  diag_kernel<<<dim3((unsigned)nch, (unsigned)p->batch), 128, 0, s>>>(a);
  const long nt = (long)p->batch * p->nval;
  const long fb = (nt + 127) / 128;
  diag_finish_kernel<<<(int)(fb < 8 * sms ? fb : 8 * sms), 128, 0, s>>>(
      part, (int)nch, p->nval, p->batch, (const cd *)p->d_beta1, (cd *)p->d_diag, (cd *)p->d_scale,
      p->d_n_small);
  emu::note_launch(3);
  return emu::check_launch();
}

extern "C" size_t emu_mode_overlap_reorder_workspace_size(const EmuNormalise *p) {
  if (!p || p->nval < 1 || p->nel < 1) return 0;
  return align_up(sizeof(double) * 264 * (size_t)p->nel, 256) +
         align_up(sizeof(cd) * (size_t)p->nval * p->nval, 256) + 256;
}

extern "C" int emu_mode_overlap_reorder(const EmuNormalise *p, int32_t *d_perm, int32_t *d_warn,
                                        void *d_workspace, size_t workspace_bytes, void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->batch < 0 || p->nval < 1 || p->nel < 1) return EMU_E_SHAPE;
  if (!p->d_x || !p->d_table_nod || !p->d_type_el || !p->d_pp || !p->d_k0 || !p->d_beta1 ||
      !p->d_sol1 || !p->d_sol2 || !p->d_diag || !p->d_scale || !d_perm || !d_warn)
    return EMU_E_ARG;
  if (p->batch == 0) return EMU_OK;
  if (!d_workspace || workspace_bytes < emu_mode_overlap_reorder_workspace_size(p)) return EMU_E_WORKSPACE;
  int st = upload_tables();
  if (st != EMU_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  double *ms_all = (double *)d_workspace;
  cd *ovl = (cd *)((char *)d_workspace + align_up(sizeof(double) * 264 * (size_t)p->nel, 256));
  const int sms = emu::sm_count();
  elem_scal_kernel<<<(int)((p->nel + 127) / 128 < 8 * sms ? (p->nel + 127) / 128 : 8 * sms), 128, 0, s>>>(
      p->d_x, p->d_table_nod, p->nel, ms_all);
  emu::note_launch();
  for (int b = 0; b < p->batch; ++b) {
    const size_t off = (size_t)b * p->nel * p->nval * 39;
    const long tot = (long)p->nval * p->nval;
    ovl_full_kernel<<<(int)((tot + 127) / 128 < 16 * sms ? (tot + 127) / 128 : 16 * sms), 128, 0, s>>>(
        ms_all, p->nval, p->nel, p->d_type_el, (const cd *)p->d_pp, p->d_k0 + b,
        (const cd *)p->d_beta1 + (size_t)b * p->nval, (const cd *)p->d_sol1 + off,
        (const cd *)p->d_sol2 + off, ovl);
    pair_swap_kernel<<<1, 32, 0, s>>>(ovl, p->nval, d_perm + (size_t)b * p->nval,
                                       (cd *)p->d_diag + (size_t)b * p->nval,
                                       (cd *)p->d_scale + (size_t)b * p->nval, d_warn + b);
    emu::note_launch(2);
  }
  return emu::check_launch();
}
