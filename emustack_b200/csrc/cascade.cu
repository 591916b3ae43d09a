// Dense GSM cascade and energy fluxes for stacks with nanostructured layers
// (backend/stack.py:162-426), batched: one CTA per spectral point walks the
// stack bottom to top with LU solves and GEMMs in FP64, keeps the matrices
// the flux pass needs in its workspace, then walks top to bottom with
// matrix-vector products and the U-weighted air-gap fluxes.
//
// Film layers (diagonal interfaces) take diagonal-aware steps: their
// products are row scalings and their right-hand sides diagonal matrices.
#include <cuda_runtime.h>

#include <cstring>

#include "dense_la.cuh"
#include "dense_multi.cuh"
#include "emu_internal.h"

namespace {

using namespace emu;

constexpr int kMaxLayers = 64;

struct DLayer {
  const cd *R12, *T12, *R21, *T21, *kz;
  long long sR12, sT12, sR21, sT21, skz;
  int M, dense;
  double hn, sh0, sh1;
  const double *hnp;  // per-point height / period [b], or null: hn for all
};

struct StackArgs {
  DLayer lay[kMaxLayers];
  int B, L, P, npw, D, ncoord, has_shear, calc_fluxes, pol, save_lists;
  const double *alphas, *betas;
  const cd *incoming;
  const int *spec, *nprop;
  cd *R_net, *T_net;
  double *fluxes, *a_list, *t_list, *r_list;
  unsigned *flags;
  int *info;
  cd *vcd, *vcu;
  long long vcd_stride, vcu_stride;
  cd *tnl, *rnl;
  cd *ws;
  long long ws_stride;
  int *ipiv;
  double inv_sqrt2;
  int flux_only;  // the cascade was run by stack_dense_multi: outputs and fluxes only
};

struct Smem {
  GemmSmem gs;
  LuSmem ls;
  double red[2 * kDLThreads / 32];
};

// ---- small CTA helpers ------------------------------------------------------
__device__ void copy_mat(cd *dst, int ldd, const cd *src, int lds, int rows, int cols) {
  for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
    const int r = e / cols, c = e % cols;
    dst[(size_t)r * ldd + c] = src[(size_t)r * lds + c];
  }
}

__device__ void diag_to_dense(cd *dst, int n, const cd *d) {
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e % n;
    dst[e] = (r == c) ? d[r] : cd{0.0, 0.0};
  }
}

// y = A x, A rows x cols (lda); one warp per row.
__device__ void matvec(cd *y, const cd *A, int lda, const cd *x, int rows, int cols) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = w; r < rows; r += nw) {
    cd s = cd{0.0, 0.0};
    for (int c = lane; c < cols; c += 32) s = cadd(s, cmul(A[(size_t)r * lda + c], x[c]));
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_down_sync(0xffffffffu, s.x, o);
      s.y += __shfl_down_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) y[r] = s;
  }
}

__device__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  __syncthreads();
  if (threadIdx.x == 0) red[0] = s;
  __syncthreads();
  const double out = red[0];
  __syncthreads();
  return out;
}

__device__ __forceinline__ cd shear_q(const StackArgs &a, int b, int pos, double c0, double c1) {
  const int u = pos % a.npw;  // unsorted air order of the same index (reference behaviour)
  const double al = a.alphas[(size_t)b * a.npw + u];
  const double be = a.betas ? a.betas[(size_t)b * a.npw + u] : 0.0;
  const double th = (a.ncoord == 1) ? al * c0 : al * c0 + be * c1;
  double s, c;
  sincos(th, &s, &c);
  return cd{c, s};
}

__device__ __forceinline__ cd incidence(const StackArgs &a, int b, int pos, int spec) {
  if (a.pol == EMU_POL_INCOMING) return a.incoming[(size_t)b * a.P + pos];
  const bool te = pos == spec, tm = pos == spec + a.npw;
  switch (a.pol) {
    case EMU_POL_TE: return te ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_TM: return tm ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_UN: return (te || tm) ? cd{a.inv_sqrt2, 0.0} : cd{0.0, 0.0};
    case EMU_POL_RCIRC: return te ? cd{a.inv_sqrt2, 0.0} : (tm ? cd{0.0, a.inv_sqrt2} : cd{0.0, 0.0});
    case EMU_POL_LCIRC: return te ? cd{a.inv_sqrt2, 0.0} : (tm ? cd{0.0, -a.inv_sqrt2} : cd{0.0, 0.0});
  }
  return cd{0.0, 0.0};
}

// One spectral point, the whole cascade and flux pass, by one CTA.  `a` is
// the uniform batch's kernel parameter (point b) or, for the uneven batch,
// a per-stack copy in shared memory whose pointers are already offset to the
// stack (b = 0).
__device__ __forceinline__ void stack_body(const StackArgs &a, const int b, Smem &sm) {
  const int L = a.L, P = a.P, D = a.D, npw = a.npw;
  const int tid = threadIdx.x, nt = blockDim.x;
  const size_t DD = (size_t)D * D;
  cd *base = a.ws + (size_t)b * a.ws_stride;
  cd *Rl = base;                              // rnet_list: 2L-2 slots
  cd *X1l = Rl + (size_t)(2 * L - 2) * DD;    // inv_t21_list: L-1 slots (P x M_i)
  cd *X2l = X1l + (size_t)(L - 1) * DD;       // inv_t12_list: L-2 slots (M_i x P)
  cd *Pl = X2l + (size_t)(L > 2 ? L - 2 : 0) * DD;  // P_list: L-2 vectors
  cd *tnet = Pl + (size_t)(L > 2 ? L - 2 : 0) * D;
  cd *T = tnet + DD;
  cd *Y = T + DD;
  cd *Z = Y + DD;
  cd *V = Z + DD;  // 6 vectors of D
  int *ipiv = a.ipiv + (size_t)b * D;
  int info = 0;
  const int M0 = a.lay[0].M;

  auto lay_ptr = [&](const cd *p, long long s) { return p + (size_t)b * s; };

  int slot = 0;       // index of the current rnet in Rl
  int tcols = P;      // columns of tnet
  if (a.flux_only) {
    slot = 2 * L - 3;
  } else {
  // ---- substrate: tnet = T12_0, rnet = R12_0
  {
    const DLayer &l0 = a.lay[0];
    if (l0.dense) {
      copy_mat(tnet, P, lay_ptr(l0.T12, l0.sT12), P, M0, P);
      copy_mat(Rl, P, lay_ptr(l0.R12, l0.sR12), P, P, P);
    } else {
      diag_to_dense(tnet, P, lay_ptr(l0.T12, l0.sT12));
      diag_to_dense(Rl, P, lay_ptr(l0.R12, l0.sR12));
    }
    __syncthreads();
    if (a.save_lists) {
      copy_mat(a.tnl + (size_t)b * (2 * L - 2) * DD, P, tnet, P, M0, P);
      copy_mat(a.rnl + (size_t)b * (2 * L - 2) * DD, P, Rl, P, P, P);
    }
  }
  for (int i = 1; i < L; ++i) {
    const DLayer &ly = a.lay[i];
    const int M = ly.M;
    cd *rnet = Rl + (size_t)slot * DD;      // P x P here
    cd *X1 = X1l + (size_t)(i - 1) * DD;     // P x M
    cd *rn1 = Rl + (size_t)(slot + 1) * DD;  // M x M after the gap
    // ---------------- air gap below layer i (stack.py:229-247, 263-278)
    // shear: rnet' = Qinv rnet Q, tnet' = tnet Q
    const cd *rg = rnet;
    if (a.has_shear) {
      double c0, c1;
      if (i < L - 1) {
        c0 = a.lay[i - 1].sh0 - ly.sh0;
        c1 = a.lay[i - 1].sh1 - ly.sh1;
      } else {
        c0 = ly.sh0;
        c1 = ly.sh1;
      }
      for (int e = tid; e < P * P; e += nt) {
        const int r = e / P, c = e % P;
        Z[e] = cmul(cmul(shear_q(a, b, r, -1 * c0, -1 * c1), rnet[e]), shear_q(a, b, c, c0, c1));
      }
      for (int e = tid; e < M0 * tcols; e += nt) {
        const int c = e % tcols;
        tnet[e] = cmul(tnet[e], shear_q(a, b, c, c0, c1));
      }
      __syncthreads();
      rg = Z;
    }
    // T = I - R12 rnet'
    if (ly.dense) {
      for (int e = tid; e < P * P; e += nt) T[e] = cd{(e / P == e % P) ? 1.0 : 0.0, 0.0};
      __syncthreads();
      cta_gemm(P, P, P, cd{-1.0, 0.0}, lay_ptr(ly.R12, ly.sR12), P, rg, P, cd{1.0, 0.0}, T, P, sm.gs);
      copy_mat(X1, M, lay_ptr(ly.T21, ly.sT21), M, P, M);
    } else {
      const cd *r12 = lay_ptr(ly.R12, ly.sR12);
      for (int e = tid; e < P * P; e += nt) {
        const int r = e / P, c = e % P;
        T[e] = csub(cd{(r == c) ? 1.0 : 0.0, 0.0}, cmul(r12[r], rg[e]));
      }
      diag_to_dense(X1, P, lay_ptr(ly.T21, ly.sT21));
    }
    __syncthreads();
    int inf = cta_getrf(P, T, P, ipiv, sm.ls, sm.gs);
    if (inf && !info) info = (2 * i - 1) * 100000 + inf;
    __syncthreads();
    cta_getrs(P, M, T, P, ipiv, X1, M, sm.gs);
    // tnet = tnet X1 ; rnet_new = R21 + T12 rnet' X1
    cta_gemm(M0, M, P, cd{1.0, 0.0}, tnet, tcols, X1, M, cd{0.0, 0.0}, Y, M, sm.gs);
    __syncthreads();
    copy_mat(tnet, M, Y, M, M0, M);
    tcols = M;
    if (ly.dense) {
      cta_gemm(M, P, P, cd{1.0, 0.0}, lay_ptr(ly.T12, ly.sT12), P, rg, P, cd{0.0, 0.0}, Y, P, sm.gs);
      copy_mat(rn1, M, lay_ptr(ly.R21, ly.sR21), M, M, M);
      __syncthreads();
      cta_gemm(M, M, P, cd{1.0, 0.0}, Y, P, X1, M, cd{1.0, 0.0}, rn1, M, sm.gs);
    } else {
      cta_gemm(P, P, P, cd{1.0, 0.0}, rg, P, X1, P, cd{0.0, 0.0}, Y, P, sm.gs);
      __syncthreads();
      const cd *t12 = lay_ptr(ly.T12, ly.sT12);
      const cd *r21 = lay_ptr(ly.R21, ly.sR21);
      for (int e = tid; e < P * P; e += nt) {
        const int r = e / P, c = e % P;
        const cd v = cmul(t12[r], Y[e]);
        rn1[e] = (r == c) ? cadd(r21[r], v) : v;
      }
    }
    __syncthreads();
    slot += 1;
    if (a.save_lists) {
      copy_mat(a.tnl + ((size_t)b * (2 * L - 2) + slot) * DD, tcols, tnet, tcols, M0, tcols);
      copy_mat(a.rnl + ((size_t)b * (2 * L - 2) + slot) * DD, M, rn1, M, M, M);
    }
    if (i == L - 1) break;
    // ---------------- through layer i (stack.py:249-262)
    cd *pd = Pl + (size_t)(i - 1) * D;
    const cd *kz = lay_ptr(ly.kz, ly.skz);
    const double hn = ly.hnp ? ly.hnp[b] : ly.hn;
    for (int r = tid; r < M; r += nt) pd[r] = cexp_ikh(kz[r], hn);
    __syncthreads();
    cd *X2 = X2l + (size_t)(i - 1) * DD;      // M x P
    cd *rn2 = Rl + (size_t)(slot + 1) * DD;   // P x P
    // T = I - R21 (Pd rnet Pd)
    if (ly.dense) {
      for (int e = tid; e < M * M; e += nt) {
        const int r = e / M, c = e % M;
        Z[e] = cmul(cmul(pd[r], rn1[e]), pd[c]);
        T[e] = cd{(r == c) ? 1.0 : 0.0, 0.0};
      }
      __syncthreads();
      cta_gemm(M, M, M, cd{-1.0, 0.0}, lay_ptr(ly.R21, ly.sR21), M, Z, M, cd{1.0, 0.0}, T, M, sm.gs);
      copy_mat(X2, P, lay_ptr(ly.T12, ly.sT12), P, M, P);
    } else {
      const cd *r21 = lay_ptr(ly.R21, ly.sR21);
      for (int e = tid; e < M * M; e += nt) {
        const int r = e / M, c = e % M;
        T[e] = csub(cd{(r == c) ? 1.0 : 0.0, 0.0}, cmul(cmul(cmul(r21[r], pd[r]), rn1[e]), pd[c]));
      }
      diag_to_dense(X2, P, lay_ptr(ly.T12, ly.sT12));
    }
    __syncthreads();
    inf = cta_getrf(M, T, M, ipiv, sm.ls, sm.gs);
    if (inf && !info) info = (2 * i) * 100000 + inf;
    __syncthreads();
    cta_getrs(M, P, T, M, ipiv, X2, P, sm.gs);
    // PX2 = Pd X2 (into Z) ; tnet = tnet PX2
    for (int e = tid; e < M * P; e += nt) Z[e] = cmul(pd[e / P], X2[e]);
    __syncthreads();
    cta_gemm(M0, P, M, cd{1.0, 0.0}, tnet, tcols, Z, P, cd{0.0, 0.0}, Y, P, sm.gs);
    __syncthreads();
    copy_mat(tnet, P, Y, P, M0, P);
    tcols = P;
    __syncthreads();
    // rnet = R12 + (T21 Pd) rnet PX2
    if (ly.dense) {
      cta_gemm(P, M, M, cd{1.0, 0.0}, lay_ptr(ly.T21, ly.sT21), M, rn1, M, cd{0.0, 0.0}, Y, M, sm.gs,
               pd, nullptr);
      copy_mat(rn2, P, lay_ptr(ly.R12, ly.sR12), P, P, P);
      __syncthreads();
      cta_gemm(P, P, M, cd{1.0, 0.0}, Y, M, Z, P, cd{1.0, 0.0}, rn2, P, sm.gs);
    } else {
      cta_gemm(P, P, P, cd{1.0, 0.0}, rn1, P, Z, P, cd{0.0, 0.0}, Y, P, sm.gs, nullptr, nullptr);
      __syncthreads();
      const cd *t21 = lay_ptr(ly.T21, ly.sT21);
      const cd *r12 = lay_ptr(ly.R12, ly.sR12);
      for (int e = tid; e < P * P; e += nt) {
        const int r = e / P, c = e % P;
        const cd v = cmul(cmul(t21[r], pd[r]), Y[e]);
        rn2[e] = (r == c) ? cadd(r12[r], v) : v;
      }
    }
    __syncthreads();
    slot += 1;
    if (a.save_lists) {
      copy_mat(a.tnl + ((size_t)b * (2 * L - 2) + slot) * DD, P, tnet, P, M0, P);
      copy_mat(a.rnl + ((size_t)b * (2 * L - 2) + slot) * DD, P, rn2, P, P, P);
    }
  }
  }  // cascade
  // outputs R_net (P x P), T_net (M0 x P)
  const cd *Rtop = Rl + (size_t)slot * DD;
  copy_mat(a.R_net + (size_t)b * P * P, P, Rtop, P, P, P);
  copy_mat(a.T_net + (size_t)b * M0 * P, P, tnet, P, M0, P);
  __syncthreads();
  if (tid == 0 && a.info && !a.flux_only) a.info[b] = info;
  if (!a.calc_fluxes) return;

  // ---------------- fluxes, top to bottom (stack.py:289-426)
  cd *d = V, *f1m = V + D, *f1p = V + 2 * D, *f2m = V + 3 * D, *f2p = V + 4 * D, *tmp = V + 5 * D;
  const int spec = a.spec[b];
  const int np_air = a.nprop[3 * b + 0], np_in = a.nprop[3 * b + 1], np_out = a.nprop[3 * b + 2];
  for (int j = tid; j < P; j += nt) d[j] = incidence(a, b, j, spec);
  __syncthreads();
  matvec(f1p, Rtop, P, d, P, P);  // d_plus
  matvec(f1m, X1l + (size_t)(L - 2) * DD, P, d, P, P);
  __syncthreads();
  cd *vcd = a.vcd ? a.vcd + (size_t)b * a.vcd_stride : nullptr;
  cd *vcu = a.vcu ? a.vcu + (size_t)b * a.vcu_stride : nullptr;
  size_t od = 0, ou = 0;
  double s_in = 0.0, s_up = 0.0;
  for (int j = tid; j < P; j += nt) {
    if ((j % npw) < np_in) {
      s_in += cabs2(d[j]);
      s_up += cabs2(f1p[j]);
    }
    if (vcd) vcd[j] = d[j];
    if (vcu) vcu[j] = f1p[j];
  }
  od = P;
  ou = P;
  const double df0 = block_sum(s_in, sm.red);
  const double up0 = block_sum(s_up, sm.red);
  double *fo = a.fluxes ? a.fluxes + (size_t)b * (L + 1) * 2 : nullptr;
  double gre[kMaxLayers], gim[kMaxLayers];
  for (int q = 0; q < L - 2; ++q) {
    const int k = L - 2 - q;
    const int M = a.lay[k].M;
    const cd *pd = Pl + (size_t)(k - 1) * D;
    matvec(f1p, Rl + (size_t)(2 * k) * DD, P, f1m, P, P);
    __syncthreads();
    double sr = 0.0, si = 0.0;
    for (int j = tid; j < P; j += nt) {
      const cd fm = f1m[j], fp = f1p[j];
      const bool prop = (j % npw) < np_air;
      const bool tm = j >= npw;
      if (prop) {
        sr += cabs2(fm) - cabs2(fp);
      } else {
        const cd u = cmul(cconj(fm), fp), v = cmul(cconj(fp), fm);
        cd dd = csub(v, u);
        cd t = cd{-dd.y, dd.x};
        if (tm) t = cneg(t);
        sr += t.x;
        si += t.y;
      }
    }
    gre[q] = block_sum(sr, sm.red);
    gim[q] = block_sum(si, sm.red);
    matvec(f2m, X2l + (size_t)(k - 1) * DD, P, f1m, M, P);
    __syncthreads();
    for (int j = tid; j < M; j += nt) tmp[j] = cmul(pd[j], f2m[j]);
    __syncthreads();
    matvec(f2p, Rl + (size_t)(2 * k - 1) * DD, M, tmp, M, M);
    matvec(f1m, X1l + (size_t)(k - 1) * DD, M, tmp, P, M);
    __syncthreads();
    for (int j = tid; j < M; j += nt) {
      if (vcd) vcd[od + j] = f2m[j];
      if (vcu) vcu[ou + j] = f2p[j];
    }
    od += M;
    ou += M;
    __syncthreads();
  }
  // bottom: f2m = tnet_list[0] f1m = T12_0 f1m
  {
    const DLayer &l0 = a.lay[0];
    if (l0.dense) {
      matvec(f2m, lay_ptr(l0.T12, l0.sT12), P, f1m, M0, P);
    } else {
      const cd *t12 = lay_ptr(l0.T12, l0.sT12);
      for (int j = tid; j < P; j += nt) f2m[j] = cmul(t12[j], f1m[j]);
    }
    __syncthreads();
    double so = 0.0;
    for (int j = tid; j < M0; j += nt) {
      if (vcd) vcd[od + j] = f2m[j];
      if (!l0.dense && (j % npw) < np_out) so += cabs2(f2m[j]);
    }
    const double dsub = block_sum(so, sm.red);
    if (tid == 0) {
      if (fo) {
        fo[0] = df0;
        fo[1] = 0.0;
        for (int q = 0; q < L - 2; ++q) {
          fo[2 * (q + 1)] = gre[q];
          fo[2 * (q + 1) + 1] = gim[q];
        }
        fo[2 * (L - 1)] = dsub;
        fo[2 * (L - 1) + 1] = 0.0;
        fo[2 * L] = up0;
        fo[2 * L + 1] = 0.0;
      }
      uint32_t flags = 0;
      if (np_in == 0) flags |= EMU_PT_NO_PROP_SUP;
      if (!l0.dense && np_out == 0) flags |= EMU_PT_NO_PROP_SUB;
      if (a.a_list && !l0.dense) {
        double *al = a.a_list + (size_t)b * (L - 1);
        double *tl = a.t_list + (size_t)b * (L - 1);
        auto dfa = [&](int i) -> double {
          if (i == 0) return fabs(df0);
          if (i == L - 1) return fabs(dsub);
          return hypot(gre[i - 1], gim[i - 1]);
        };
        if (np_out != 0) {
          for (int i = 1; i <= L - 2; ++i) al[i - 1] = fabs(dfa(i) - dfa(i + 1));
          al[L - 2] = fabs(df0 - dsub - up0);
          for (int i = 0; i <= L - 3; ++i) tl[i] = fabs(dfa(i + 2) / dfa(i));
          tl[L - 2] = fabs(dsub / df0);
          a.r_list[b] = fabs(up0 / df0);
        } else {
          for (int i = 0; i < L - 1; ++i) al[i] = tl[i] = 0.0;
          a.r_list[b] = 0.0;
        }
        bool fin = isfinite(a.r_list[b]);
        for (int i = 0; i < L - 1; ++i) fin = fin && isfinite(al[i]) && isfinite(tl[i]);
        if (!fin) flags |= EMU_PT_NONFINITE;
      }
      if (a.flags) a.flags[b] = flags;
    }
  }
}

__global__ void __launch_bounds__(kDLThreads) stack_dense_kernel(StackArgs a) {
  __shared__ Smem sm;
  stack_body(a, blockIdx.x, sm);
}

// ---------------------------------------------------------------------------
// Multi-CTA cascade.  The same steps as stack_dense_kernel, in the same
// order and with the same arithmetic (results are bit-identical), but each
// step is a launch over all solves of the batch that spreads the matrices
// over many CTAs: batched tiled GEMMs, getrf_multi / getrs_multi and
// elementwise kernels.  The workspace holds exactly what the one-CTA kernel
// keeps (rnet / inv_t21 / inv_t12 lists, propagation vectors, tnet and
// scratch), so the flux pass runs afterwards as stack_dense_kernel with
// flux_only set.  Large matrices (P, M in the hundreds) then use the whole
// GPU even for a handful of solves.

struct MultiWs {
  long long stride, DD;
  int D, L;
  cd *ws;
  __host__ __device__ cd *base(long long b) const { return ws + b * stride; }
  __host__ __device__ cd *Rl(int slot) const { return ws + (long long)slot * DD; }  // add b * stride
  __host__ __device__ cd *X1(int i) const { return ws + (long long)(2 * L - 2 + i) * DD; }
  __host__ __device__ cd *X2(int i) const { return ws + (long long)(2 * L - 2 + L - 1 + i) * DD; }
  __host__ __device__ cd *Pl(int i) const {
    return ws + (long long)(2 * L - 2 + L - 1 + (L > 2 ? L - 2 : 0)) * DD + (long long)i * D;
  }
  __host__ __device__ cd *tnet() const {
    return ws + (long long)(2 * L - 2 + L - 1 + (L > 2 ? L - 2 : 0)) * DD + (long long)(L > 2 ? L - 2 : 0) * D;
  }
  __host__ __device__ cd *T() const { return tnet() + DD; }
  __host__ __device__ cd *Y() const { return tnet() + 2 * DD; }
  __host__ __device__ cd *Z() const { return tnet() + 3 * DD; }
};

#define EW_LOOP(total)                                                                        \
  const long long b = blockIdx.y;                                                             \
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (total);           \
       e += (long long)gridDim.x * blockDim.x)

inline dim3 ew_grid(long long n, int batch) {
  long long g = (n + 255) / 256;
  if (g > 1024) g = 1024;
  return dim3((unsigned)(g < 1 ? 1 : g), (unsigned)batch);
}

// dst[b] (rows x cols, ldd) = src[b] (lds)
__global__ void ew_copy(cd *dst, long long sd, int ldd, const cd *src, long long ss, int lds, int rows, int cols) {
  EW_LOOP((long long)rows * cols) {
    const int r = (int)(e / cols), c = (int)(e % cols);
    dst[b * sd + (long long)r * ldd + c] = src[b * ss + (long long)r * lds + c];
  }
}

// dst[b] = diag(d[b]) (n x n)
__global__ void ew_diag(cd *dst, long long sd, const cd *d, long long sdd, int n) {
  EW_LOOP((long long)n * n) {
    const int r = (int)(e / n), c = (int)(e % n);
    dst[b * sd + e] = (r == c) ? d[b * sdd + r] : cd{0.0, 0.0};
  }
}

// dst[b] = I (n x n)
__global__ void ew_eye(cd *dst, long long sd, int n) {
  EW_LOOP((long long)n * n) dst[b * sd + e] = cd{(e / n == e % n) ? 1.0 : 0.0, 0.0};
}

// shear: Z = Qinv rnet Q (P x P), tnet[:, c] *= Q(c) (M0 x tcols)
__global__ void ew_shear(StackArgs a, MultiWs w, int slot, double c0, double c1, int M0, int tcols) {
  const int P = a.P;
  EW_LOOP((long long)P * P + (long long)M0 * tcols) {
    cd *base = w.base(b);
    if (e < (long long)P * P) {
      const int r = (int)(e / P), c = (int)(e % P);
      const cd *rnet = base + (w.Rl(slot) - w.ws);
      cd *Z = base + (w.Z() - w.ws);
      Z[e] = cmul(cmul(shear_q(a, (int)b, r, -1 * c0, -1 * c1), rnet[e]), shear_q(a, (int)b, c, c0, c1));
    } else {
      const long long f = e - (long long)P * P;
      const int c = (int)(f % tcols);
      cd *tn = base + (w.tnet() - w.ws);
      tn[f] = cmul(tn[f], shear_q(a, (int)b, c, c0, c1));
    }
  }
}

// T = I - diag(r12) rg  (P x P)
__global__ void ew_t_gap_diag(cd *T, long long sT, const cd *r12, long long sr, const cd *rg, long long sg, int P) {
  EW_LOOP((long long)P * P) {
    const int r = (int)(e / P), c = (int)(e % P);
    T[b * sT + e] = csub(cd{(r == c) ? 1.0 : 0.0, 0.0}, cmul(r12[b * sr + r], rg[b * sg + e]));
  }
}

// rn1 = diag(t12) Y + diag(r21)  (P x P)
__global__ void ew_rn_gap_diag(cd *rn, long long sn, const cd *t12, long long st, const cd *Y, long long sy,
                               const cd *r21, long long sr, int P) {
  EW_LOOP((long long)P * P) {
    const int r = (int)(e / P), c = (int)(e % P);
    const cd v = cmul(t12[b * st + r], Y[b * sy + e]);
    rn[b * sn + e] = (r == c) ? cadd(r21[b * sr + r], v) : v;
  }
}

// pd = exp(i kz h)  (M)
__global__ void ew_prop(cd *pd, long long sp, const cd *kz, long long skz, double hn, const double *hnp,
                        int M) {
  EW_LOOP(M) pd[b * sp + e] = cexp_ikh(kz[b * skz + e], hnp ? hnp[b] : hn);
}

// Z = diag(pd) rn1 diag(pd), T = I  (M x M)
__global__ void ew_layer_dense(cd *Z, cd *T, long long sw, const cd *pd, long long sp, const cd *rn1, int M) {
  EW_LOOP((long long)M * M) {
    const int r = (int)(e / M), c = (int)(e % M);
    const cd *p = pd + b * sp;
    Z[b * sw + e] = cmul(cmul(p[r], rn1[b * sw + e]), p[c]);
    T[b * sw + e] = cd{(r == c) ? 1.0 : 0.0, 0.0};
  }
}

// T = I - diag(r21) diag(pd) rn1 diag(pd)  (M x M)
__global__ void ew_t_layer_diag(cd *T, long long sw, const cd *r21, long long sr, const cd *pd, long long sp,
                                const cd *rn1, int M) {
  EW_LOOP((long long)M * M) {
    const int r = (int)(e / M), c = (int)(e % M);
    const cd *p = pd + b * sp;
    T[b * sw + e] = csub(cd{(r == c) ? 1.0 : 0.0, 0.0},
                         cmul(cmul(cmul(r21[b * sr + r], p[r]), rn1[b * sw + e]), p[c]));
  }
}

// Z = diag(pd) X2  (M x P)
__global__ void ew_rowscale(cd *Z, long long sw, const cd *pd, long long sp, const cd *X2, int M, int P) {
  EW_LOOP((long long)M * P) Z[b * sw + e] = cmul(pd[b * sp + e / P], X2[b * sw + e]);
}

// rn2 = diag(t21) diag(pd) Y + diag(r12)  (P x P)
__global__ void ew_rn_layer_diag(cd *rn, long long sw, const cd *t21, long long st, const cd *pd, long long sp,
                                 const cd *Y, const cd *r12, long long sr, int P) {
  EW_LOOP((long long)P * P) {
    const int r = (int)(e / P), c = (int)(e % P);
    const cd v = cmul(cmul(t21[b * st + r], pd[b * sp + r]), Y[b * sw + e]);
    rn[b * sw + e] = (r == c) ? cadd(r12[b * sr + r], v) : v;
  }
}

int stack_dense_multi(const StackArgs &a, cudaStream_t s) {
  const int B = a.B, L = a.L, P = a.P, D = a.D;
  MultiWs w;
  w.stride = a.ws_stride;
  w.DD = (long long)D * D;
  w.D = D;
  w.L = L;
  w.ws = a.ws;
  const long long S = w.stride;       // batch stride of every workspace object
  const long long sip = D;            // ipiv batch stride
  const int M0 = a.lay[0].M;
  const cd one{1.0, 0.0}, zero{0.0, 0.0}, mone{-1.0, 0.0};
  const long long DD = w.DD, LS = (long long)(2 * L - 2) * DD;  // saved-list stride in tnl / rnl
  int n_launch = 0;
  auto ew = [&](long long n) {
    ++n_launch;
    return ew_grid(n, B);
  };
  if (a.info && cudaMemsetAsync(a.info, 0, sizeof(int) * B, s) != cudaSuccess) return EMU_E_CUDA;
  cd *tnet = w.tnet(), *T = w.T(), *Y = w.Y(), *Z = w.Z();
  // ---- substrate
  {
    const DLayer &l0 = a.lay[0];
    if (l0.dense) {
      ew_copy<<<ew(M0 * P), 256, 0, s>>>(tnet, S, P, l0.T12, l0.sT12, P, M0, P);
      ew_copy<<<ew(P * P), 256, 0, s>>>(w.Rl(0), S, P, l0.R12, l0.sR12, P, P, P);
    } else {
      ew_diag<<<ew(P * P), 256, 0, s>>>(tnet, S, l0.T12, l0.sT12, P);
      ew_diag<<<ew(P * P), 256, 0, s>>>(w.Rl(0), S, l0.R12, l0.sR12, P);
    }
    if (a.save_lists) {
      ew_copy<<<ew(M0 * P), 256, 0, s>>>(a.tnl, LS, P, tnet, S, P, M0, P);
      ew_copy<<<ew(P * P), 256, 0, s>>>(a.rnl, LS, P, w.Rl(0), S, P, P, P);
    }
  }
  int slot = 0, tcols = P;
  for (int i = 1; i < L; ++i) {
    const DLayer &ly = a.lay[i];
    const int M = ly.M;
    cd *rnet = w.Rl(slot), *X1 = w.X1(i - 1), *rn1 = w.Rl(slot + 1);
    const cd *rg = rnet;
    if (a.has_shear) {
      double c0, c1;
      if (i < L - 1) {
        c0 = a.lay[i - 1].sh0 - ly.sh0;
        c1 = a.lay[i - 1].sh1 - ly.sh1;
      } else {
        c0 = ly.sh0;
        c1 = ly.sh1;
      }
      ew_shear<<<ew((long long)P * P + (long long)M0 * tcols), 256, 0, s>>>(a, w, slot, c0, c1, M0, tcols);
      rg = Z;
    }
    if (ly.dense) {
      ew_eye<<<ew(P * P), 256, 0, s>>>(T, S, P);
      bgemm(P, P, P, mone, ly.R12, ly.sR12, P, rg, S, P, one, T, S, P, B, s);
      ew_copy<<<ew(P * M), 256, 0, s>>>(X1, S, M, ly.T21, ly.sT21, M, P, M);
    } else {
      ew_t_gap_diag<<<ew(P * P), 256, 0, s>>>(T, S, ly.R12, ly.sR12, rg, S, P);
      ew_diag<<<ew(P * P), 256, 0, s>>>(X1, S, ly.T21, ly.sT21, P);
    }
    getrf_multi(P, T, S, P, a.ipiv, sip, a.info, (2 * i - 1) * 100000, B, s);
    getrs_multi(P, M, T, S, P, a.ipiv, sip, X1, S, M, B, s);
    bgemm(M0, M, P, one, tnet, S, tcols, X1, S, M, zero, Y, S, M, B, s);
    ew_copy<<<ew(M0 * M), 256, 0, s>>>(tnet, S, M, Y, S, M, M0, M);
    tcols = M;
    if (ly.dense) {
      bgemm(M, P, P, one, ly.T12, ly.sT12, P, rg, S, P, zero, Y, S, P, B, s);
      ew_copy<<<ew(M * M), 256, 0, s>>>(rn1, S, M, ly.R21, ly.sR21, M, M, M);
      bgemm(M, M, P, one, Y, S, P, X1, S, M, one, rn1, S, M, B, s);
    } else {
      bgemm(P, P, P, one, rg, S, P, X1, S, P, zero, Y, S, P, B, s);
      ew_rn_gap_diag<<<ew(P * P), 256, 0, s>>>(rn1, S, ly.T12, ly.sT12, Y, S, ly.R21, ly.sR21, P);
    }
    slot += 1;
    if (a.save_lists) {
      ew_copy<<<ew(M0 * tcols), 256, 0, s>>>(a.tnl + slot * DD, LS, tcols, tnet, S, tcols, M0, tcols);
      ew_copy<<<ew(M * M), 256, 0, s>>>(a.rnl + slot * DD, LS, M, rn1, S, M, M, M);
    }
    if (i == L - 1) break;
    cd *pd = w.Pl(i - 1);
    ew_prop<<<ew(M), 256, 0, s>>>(pd, S, ly.kz, ly.skz, ly.hn, ly.hnp, M);
    cd *X2 = w.X2(i - 1), *rn2 = w.Rl(slot + 1);
    if (ly.dense) {
      ew_layer_dense<<<ew(M * M), 256, 0, s>>>(Z, T, S, pd, S, rn1, M);
      bgemm(M, M, M, mone, ly.R21, ly.sR21, M, Z, S, M, one, T, S, M, B, s);
      ew_copy<<<ew(M * P), 256, 0, s>>>(X2, S, P, ly.T12, ly.sT12, P, M, P);
    } else {
      ew_t_layer_diag<<<ew(M * M), 256, 0, s>>>(T, S, ly.R21, ly.sR21, pd, S, rn1, M);
      ew_diag<<<ew(P * P), 256, 0, s>>>(X2, S, ly.T12, ly.sT12, P);
    }
    getrf_multi(M, T, S, M, a.ipiv, sip, a.info, (2 * i) * 100000, B, s);
    getrs_multi(M, P, T, S, M, a.ipiv, sip, X2, S, P, B, s);
    ew_rowscale<<<ew(M * P), 256, 0, s>>>(Z, S, pd, S, X2, M, P);
    bgemm(M0, P, M, one, tnet, S, tcols, Z, S, P, zero, Y, S, P, B, s);
    ew_copy<<<ew(M0 * P), 256, 0, s>>>(tnet, S, P, Y, S, P, M0, P);
    tcols = P;
    if (ly.dense) {
      bgemm(P, M, M, one, ly.T21, ly.sT21, M, rn1, S, M, zero, Y, S, M, B, s, pd, S);
      ew_copy<<<ew(P * P), 256, 0, s>>>(rn2, S, P, ly.R12, ly.sR12, P, P, P);
      bgemm(P, P, M, one, Y, S, M, Z, S, P, one, rn2, S, P, B, s);
    } else {
      bgemm(P, P, P, one, rn1, S, P, Z, S, P, zero, Y, S, P, B, s);
      ew_rn_layer_diag<<<ew(P * P), 256, 0, s>>>(rn2, S, ly.T21, ly.sT21, pd, S, Y, ly.R12, ly.sR12, P);
    }
    slot += 1;
    if (a.save_lists) {
      ew_copy<<<ew(M0 * P), 256, 0, s>>>(a.tnl + slot * DD, LS, P, tnet, S, P, M0, P);
      ew_copy<<<ew(P * P), 256, 0, s>>>(a.rnl + slot * DD, LS, P, rn2, S, P, P, P);
    }
  }
  note_launch(n_launch);
  // outputs and fluxes from the saved state
  StackArgs f = a;
  f.flux_only = 1;
  stack_dense_kernel<<<B, kDLThreads, 0, s>>>(f);
  note_launch();
  return check_launch();
}

}  // namespace

namespace {

int max_dim(const EmuStackDense *p) {
  int D = p->P;
  for (int i = 0; i < p->n_layers; ++i) D = p->h_layers[i].M > D ? p->h_layers[i].M : D;
  return D;
}

long long per_solve_elems(const EmuStackDense *p) {
  const long long L = p->n_layers, D = max_dim(p);
  const long long Lf = L > 2 ? L - 2 : 0;
  return (2 * L - 2 + L - 1 + Lf + 4) * D * D + Lf * D + 6 * D;
}

int validate(const EmuStackDense *p) {
  if (!p || !p->h_layers) return EMU_E_ARG;
  if (p->batch < 0 || p->n_layers < 2 || p->n_layers > kMaxLayers || p->P < 2 || (p->P % 2))
    return EMU_E_SHAPE;
  for (int i = 0; i < p->n_layers; ++i) {
    const EmuLayer &l = p->h_layers[i];
    if (l.M < 1) return EMU_E_SHAPE;
    if (!l.dense && l.M != p->P) return EMU_E_SHAPE;
    if (!l.d_R12 || !l.d_T12 || !l.d_R21 || !l.d_T21) return EMU_E_ARG;
    if (i > 0 && i < p->n_layers - 1 && !l.d_kz) return EMU_E_ARG;
  }
  if (p->h_layers[p->n_layers - 1].M != p->P) return EMU_E_SHAPE;
  if (!p->d_R_net || !p->d_T_net) return EMU_E_ARG;
  if (p->calc_fluxes) {
    if (p->h_layers[p->n_layers - 1].dense) return EMU_E_UNSUPPORTED;  // needs a film on top
    if (!p->d_specular || !p->d_num_prop) return EMU_E_ARG;
    if (p->pol == EMU_POL_INCOMING && !p->d_incoming) return EMU_E_ARG;
    if (p->pol < EMU_POL_INCOMING || p->pol > EMU_POL_LCIRC) return EMU_E_ARG;
  }
  if (p->h_shears && (!p->d_air_alphas || (p->shear_ncoord == 2 && !p->d_air_betas))) return EMU_E_ARG;
  if (p->save_lists && (!p->d_tnet_list || !p->d_rnet_list)) return EMU_E_ARG;
  if (p->mode < 0 || p->mode > 2) return EMU_E_ARG;
  if (p->batch > 65535) return EMU_E_SHAPE;
  return EMU_OK;
}

}  // namespace

extern "C" size_t emu_stack_dense_workspace_size(const EmuStackDense *p) {
  if (validate(p) != EMU_OK) return 0;
  const long long D = max_dim(p);
  return (size_t)p->batch * ((size_t)per_solve_elems(p) * sizeof(cd) + align_up((size_t)D * 4, 16)) + 256;
}

extern "C" long long emu_stack_dense_list_stride(const EmuStackDense *p) {
  if (validate(p) != EMU_OK) return 0;
  const long long D = max_dim(p);
  return D * D;
}

extern "C" int emu_stack_dense_batch(const EmuStackDense *p, void *d_workspace,
                                     size_t workspace_bytes, void *stream) {
  int st = validate(p);
  if (st != EMU_OK) return st;
  if (p->batch == 0) return EMU_OK;
  if (!d_workspace || workspace_bytes < emu_stack_dense_workspace_size(p)) return EMU_E_WORKSPACE;
  StackArgs a;
  memset(&a, 0, sizeof(a));
  a.B = p->batch;
  a.L = p->n_layers;
  a.P = p->P;
  a.npw = p->P / 2;
  a.D = max_dim(p);
  for (int i = 0; i < p->n_layers; ++i) {
    const EmuLayer &l = p->h_layers[i];
    DLayer &d = a.lay[i];
    d.R12 = (const cd *)l.d_R12;
    d.T12 = (const cd *)l.d_T12;
    d.R21 = (const cd *)l.d_R21;
    d.T21 = (const cd *)l.d_T21;
    d.kz = (const cd *)l.d_kz;
    d.sR12 = l.stride_R12;
    d.sT12 = l.stride_T12;
    d.sR21 = l.stride_R21;
    d.sT21 = l.stride_T21;
    d.skz = l.stride_kz;
    d.M = l.M;
    d.dense = l.dense;
    d.hn = l.height_norm;
    d.hnp = l.d_height_norm;
    d.sh0 = p->h_shears ? p->h_shears[2 * i] : 0.0;
    d.sh1 = p->h_shears ? p->h_shears[2 * i + 1] : 0.0;
  }
  a.ncoord = p->shear_ncoord;
  a.has_shear = p->h_shears != nullptr;
  a.alphas = p->d_air_alphas;
  a.betas = p->d_air_betas;
  a.calc_fluxes = p->calc_fluxes;
  a.pol = p->pol;
  a.incoming = (const cd *)p->d_incoming;
  a.spec = p->d_specular;
  a.nprop = p->d_num_prop;
  a.R_net = (cd *)p->d_R_net;
  a.T_net = (cd *)p->d_T_net;
  a.fluxes = p->d_fluxes;
  a.a_list = p->d_a_list;
  a.t_list = p->d_t_list;
  a.r_list = p->d_r_list;
  a.flags = p->d_flags;
  a.info = p->d_info;
  a.vcd = (cd *)p->d_vec_coef_down;
  a.vcu = (cd *)p->d_vec_coef_up;
  a.vcd_stride = p->vec_coef_down_stride;
  a.vcu_stride = p->vec_coef_up_stride;
  a.save_lists = p->save_lists;
  a.tnl = (cd *)p->d_tnet_list;
  a.rnl = (cd *)p->d_rnet_list;
  a.ws = (cd *)d_workspace;
  a.ws_stride = per_solve_elems(p);
  a.ipiv = (int *)((char *)d_workspace + align_up((size_t)p->batch * a.ws_stride * sizeof(cd), 16));
  a.inv_sqrt2 = 1.0 / sqrt(2.0);
  a.flux_only = 0;
  // one CTA per solve while the batch fills the GPU and matrices are small;
  // the multi-CTA cascade for large matrices or few solves
  int mode = p->mode ? p->mode : emu::dense_mode();
  if (mode == 0) mode = (a.D >= 256 || (a.D >= 96 && p->batch < emu::sm_count())) ? 2 : 1;
  if (mode == 2) return stack_dense_multi(a, (cudaStream_t)stream);
  stack_dense_kernel<<<p->batch, kDLThreads, 0, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

// ---------------------------------------------------------------------------
// Uneven batch of dense stacks in one launch (emu_stack_var_batch).
//
// A persistent kernel: each CTA owns one workspace slot and repeatedly takes
// the next stack from an atomic counter (in the caller's processing order),
// copies the stack's descriptor into a StackArgs in shared memory with every
// pointer offset to the stack, checks it against the packed arrays, and runs
// stack_body on it -- the one-CTA cascade and flux pass of the uniform batch,
// so a stack gives the same result here as in emu_stack_dense_batch.  No CTA
// waits on another: a CTA that finds the counter past the end returns.

namespace {

struct VarStackArgs {
  int n;
  const EmuStackPoint *pts;
  const int *order;
  const EmuVarLayer *lays;
  long long n_lays;
  const cd *inc;
  long long inc_len;
  cd *R_net, *T_net;
  long long rnet_len, tnet_len;
  double *a_list, *t_list, *fluxes, *r_list;
  long long list_len, flux_len;
  unsigned *flags;
  int *info;
  int max_P, max_D, max_L;
  int *counter;
  cd *ws;
  long long ws_stride;
  int *ipiv;
  double inv_sqrt2;
};

__global__ void __launch_bounds__(kDLThreads) stack_var_kernel(VarStackArgs v) {
  __shared__ Smem sm;
  __shared__ StackArgs sa;
  __shared__ int s_next, s_bad;
  const int tid = threadIdx.x;
  cd *ws = v.ws + (size_t)blockIdx.x * v.ws_stride;
  int *ipiv = v.ipiv + (size_t)blockIdx.x * v.max_D;
  for (;;) {
    if (tid == 0) {
      s_next = atomicAdd(v.counter, 1);
      s_bad = 0;
    }
    __syncthreads();
    const int k = s_next;
    if (k >= v.n) break;
    const int s = v.order ? v.order[k] : k;
    if (s < 0 || s >= v.n) {  // a bad order entry: nothing to flag
      __syncthreads();
      continue;
    }
    const EmuStackPoint &pt = v.pts[s];
    const int L = pt.n_layers, P = pt.P;
    bool ok = L >= 2 && L <= v.max_L && L <= kMaxLayers && P >= 2 && (P % 2) == 0 && P <= v.max_P &&
              pt.pol >= EMU_POL_INCOMING && pt.pol <= EMU_POL_LCIRC && pt.spec >= 0 && pt.spec < P / 2 &&
              pt.layer_off >= 0 && pt.layer_off + L <= v.n_lays;
    for (int q = 0; q < 3; ++q) ok = ok && pt.num_prop[q] >= 0 && pt.num_prop[q] <= P / 2;
    ok = ok && pt.rnet_off >= 0 && pt.rnet_off + (long long)P * P <= v.rnet_len;
    ok = ok && pt.tnet_off >= 0 && pt.tnet_off + (long long)P * P <= v.tnet_len;
    ok = ok && pt.list_off >= 0 && pt.list_off + L - 1 <= v.list_len;
    ok = ok && (!v.fluxes || (pt.flux_off >= 0 && pt.flux_off + 2LL * (L + 1) <= v.flux_len));
    ok = ok && (pt.pol != EMU_POL_INCOMING || (v.inc && pt.inc_off >= 0 && pt.inc_off + P <= v.inc_len));
    if (!ok && tid == 0) s_bad = 1;
    __syncthreads();
    if (!s_bad && tid < L) {
      const EmuVarLayer &l = v.lays[pt.layer_off + tid];
      const bool fin = tid > 0 && tid < L - 1;
      bool lok = l.M >= 1 && l.M <= v.max_D && l.d_R12 && l.d_T12 && l.d_R21 && l.d_T21 &&
                 (!fin || l.d_kz) && (l.dense || l.M == P) && (fin || !l.dense);
      if (!lok) atomicOr(&s_bad, 1);
      DLayer &d = sa.lay[tid];
      d.R12 = (const cd *)l.d_R12;
      d.T12 = (const cd *)l.d_T12;
      d.R21 = (const cd *)l.d_R21;
      d.T21 = (const cd *)l.d_T21;
      d.kz = (const cd *)l.d_kz;
      d.sR12 = d.sT12 = d.sR21 = d.sT21 = d.skz = 0;
      d.M = l.M;
      d.dense = l.dense;
      d.hn = l.height_norm;
      d.sh0 = d.sh1 = 0.0;
      d.hnp = nullptr;
    }
    __syncthreads();
    if (s_bad) {
      if (tid == 0) {
        v.flags[s] = EMU_PT_BAD_POINT;
        v.info[s] = 0;
      }
      __syncthreads();
      continue;
    }
    if (tid == 0) {
      int D = P;
      for (int i = 0; i < L; ++i) D = sa.lay[i].M > D ? sa.lay[i].M : D;
      sa.B = 1;
      sa.L = L;
      sa.P = P;
      sa.npw = P / 2;
      sa.D = D;
      sa.ncoord = 1;
      sa.has_shear = 0;
      sa.calc_fluxes = 1;
      sa.pol = pt.pol;
      sa.save_lists = 0;
      sa.alphas = sa.betas = nullptr;
      sa.incoming = pt.pol == EMU_POL_INCOMING ? v.inc + pt.inc_off : nullptr;
      sa.spec = &pt.spec;
      sa.nprop = pt.num_prop;
      sa.R_net = v.R_net + pt.rnet_off;
      sa.T_net = v.T_net + pt.tnet_off;
      sa.fluxes = v.fluxes ? v.fluxes + pt.flux_off : nullptr;
      sa.a_list = v.a_list + pt.list_off;
      sa.t_list = v.t_list + pt.list_off;
      sa.r_list = v.r_list + s;
      sa.flags = v.flags + s;
      sa.info = v.info + s;
      sa.vcd = sa.vcu = nullptr;
      sa.vcd_stride = sa.vcu_stride = 0;
      sa.tnl = sa.rnl = nullptr;
      sa.ws = ws;
      sa.ws_stride = 0;
      sa.ipiv = ipiv;
      sa.inv_sqrt2 = v.inv_sqrt2;
      sa.flux_only = 0;
    }
    __syncthreads();
    stack_body(sa, 0, sm);
    __syncthreads();
  }
}

long long var_slot_elems(int L, int D) {
  const long long Lf = L > 2 ? L - 2 : 0, DD = (long long)D * D;
  return (2LL * L - 2 + L - 1 + Lf + 4) * DD + Lf * D + 6LL * D;
}

int var_validate(const EmuStackVarBatch *p) {
  if (!p) return EMU_E_ARG;
  if (p->n_stacks < 0 || p->n_slots < 0) return EMU_E_SHAPE;
  if (p->n_stacks == 0) return EMU_OK;
  if (p->max_P < 2 || p->max_D < p->max_P || p->max_L < 2 || p->max_L > kMaxLayers) return EMU_E_SHAPE;
  if (!p->d_points || !p->d_layers || !p->d_R_net || !p->d_T_net || !p->d_a_list || !p->d_t_list ||
      !p->d_r_list || !p->d_flags || !p->d_info)
    return EMU_E_ARG;
  return EMU_OK;
}

}  // namespace

extern "C" int emu_stack_var_slots(const EmuStackVarBatch *p) {
  if (var_validate(p) != EMU_OK) return 0;
  if (p->n_slots > 0) return p->n_slots < p->n_stacks ? p->n_slots : p->n_stacks;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stack_var_kernel, kDLThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long slots = (long long)emu::sm_count() * per_sm;
  return (int)(slots < p->n_stacks ? slots : p->n_stacks);
}

extern "C" size_t emu_stack_var_workspace_size(const EmuStackVarBatch *p) {
  if (var_validate(p) != EMU_OK) return 0;
  const long long slots = emu_stack_var_slots(p);
  return 256 + (size_t)slots * var_slot_elems(p->max_L, p->max_D) * sizeof(cd) +
         align_up((size_t)slots * p->max_D * sizeof(int), 16);
}

extern "C" int emu_stack_var_batch(const EmuStackVarBatch *p, void *d_workspace, size_t workspace_bytes,
                                   void *stream) {
  const int st = var_validate(p);
  if (st != EMU_OK) return st;
  if (p->n_stacks == 0) return EMU_OK;
  const size_t need = emu_stack_var_workspace_size(p);
  if (!d_workspace || workspace_bytes < need) return EMU_E_WORKSPACE;
  const int slots = emu_stack_var_slots(p);
  cudaStream_t s = (cudaStream_t)stream;
  VarStackArgs v;
  v.n = p->n_stacks;
  v.pts = p->d_points;
  v.order = p->d_order;
  v.lays = p->d_layers;
  v.n_lays = p->n_layer_desc;
  v.inc = (const cd *)p->d_incoming;
  v.inc_len = p->incoming_len;
  v.R_net = (cd *)p->d_R_net;
  v.T_net = (cd *)p->d_T_net;
  v.rnet_len = p->rnet_len;
  v.tnet_len = p->tnet_len;
  v.a_list = p->d_a_list;
  v.t_list = p->d_t_list;
  v.list_len = p->list_len;
  v.fluxes = p->d_fluxes;
  v.flux_len = p->flux_len;
  v.r_list = p->d_r_list;
  v.flags = p->d_flags;
  v.info = p->d_info;
  v.max_P = p->max_P;
  v.max_D = p->max_D;
  v.max_L = p->max_L;
  v.counter = (int *)d_workspace;
  v.ws = (cd *)((char *)d_workspace + 256);
  v.ws_stride = var_slot_elems(p->max_L, p->max_D);
  v.ipiv = (int *)((char *)d_workspace + 256 + (size_t)slots * v.ws_stride * sizeof(cd));
  v.inv_sqrt2 = 1.0 / sqrt(2.0);
  if (cudaMemsetAsync(v.counter, 0, sizeof(int), s) != cudaSuccess) return EMU_E_CUDA;
  stack_var_kernel<<<slots, kDLThreads, 0, s>>>(v);
  emu::note_launch();
  return emu::check_launch();
}
