// Fused all-film GSM kernel: k_z, sort order, impedances, Fresnel interfaces,
// cascade and energy fluxes for a batch of spectral points in one launch.
//
// When every layer of a stack is a homogeneous film (reference: Anallo),
// every matrix of backend/stack.py:162-426 is diagonal, so the reference's
// dense solves and products collapse to independent scalar recursions, one
// per plane-wave order and polarisation.  The reference still runs them as
// dense P x P LAPACK solves; here each order is one thread.
//
// Mapping: a CTA of 256 threads holds `ppc` points at a time, a team of
// `team` threads per point, one thread per order (looping when Npw > team).
// Both polarisations of an order share one thread (they share k_z).
//
// Phases per CTA iteration (all threads take every __syncthreads):
//   0  per-point constants in shared memory: each layer's n, k = 2 pi n / wl,
//      1/n, 1/k and the heights
//   1  air k_z with the Wood-anomaly check (backend/mode_calcs.py:147-162),
//      sort keys -Re k_z + Im k_z (backend/mode_calcs.py:164-171) and the
//      air's propagating-order count
//   2  (only if the air hit a Wood anomaly) air k_z again with k_parallel
//      scaled by 1 - 1e-9
//   3  rank of each order = its position in the sorted order (stable on
//      ties; ties only occur at exactly degenerate orders, whose values are
//      identical), specular order = rank of (0, 0), propagating counts of
//      substrate and superstrate
//   4  Wood check of every layer (k^2 - alpha^2 - beta^2 == 0), then per
//      order: bottom-to-top cascade for both polarisations (R_net, T_net)
//      and, for the order(s) that carry incident light, the top-to-bottom
//      flux pass over the scalars saved in the workspace, summed per level
//      in shared memory
//   5  (only if a layer hit a Wood anomaly) phase 4 again for those points
//      with k_parallel scaled by 1 - 1e-9 in the marked layers
//   6  a_list / t_list / r_list (backend/stack.py:368-426)
// Divisions use the Newton reciprocal of emu_fastmath.cuh; k_z itself uses
// IEEE square roots and quotients so that exact zeros (Wood anomalies) and
// exactly real k_z (propagating orders) are decided as numpy decides them.
#include <cuda_runtime.h>

#include "emu_cplx.cuh"
#include "emu_fastmath.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"

namespace {

using namespace emu;

constexpr int kThreads = 256;
constexpr int kSave = 5;  // saved scalars per (layer, polarisation)

struct FilmArgs {
  EmuFilmStackBatch p;
  int team;        // threads per point
  int ppc;         // points per CTA iteration
  int n_act;       // active-order slots per point in the workspace
  cd *ws;          // [B][n_act][L][2][kSave]
  double dy;       // period_y / period
  double inv_sqrt2;
};

struct LayerC {
  cd k, zcr, ik;  // wavenumber, 1/n, 1/k
};

struct SlotSmem {
  int keys, rank, wood, nprop, acc, lay, h, misc, stride;
};

__host__ __device__ inline SlotSmem slot_layout(int npw, int L) {
  SlotSmem s;
  int o = 0;
  s.lay = o; o += (int)sizeof(LayerC) * L;
  s.acc = o; o += 16 * (L + 1);
  s.keys = o; o += 8 * npw;
  s.h = o; o += 8 * (L > 2 ? L - 2 : 1);
  s.rank = o; o += 4 * npw;
  s.nprop = o; o += 4 * (L + 1);
  s.wood = o; o += 4 * ((L + 1 + 31) / 32);
  s.misc = o; o += 16;  // [0] specular order, [1] layer-Wood flag
  s.stride = (o + 15) / 16 * 16;
  return s;
}

__device__ __forceinline__ cd incidence(const FilmArgs &a, int b, int pos, int spec, int npw) {
  const int pol = a.p.pol;
  if (pol == EMU_POL_INCOMING) {
    const emu_c128 v = a.p.d_incoming[(size_t)b * 2 * npw + pos];
    return cd{v.re, v.im};
  }
  const bool te = (pos == spec), tm = (pos == spec + npw);
  switch (pol) {
    case EMU_POL_TE: return te ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_TM: return tm ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_UN: return (te || tm) ? cd{a.inv_sqrt2, 0.0} : cd{0.0, 0.0};
    case EMU_POL_RCIRC: return te ? cd{a.inv_sqrt2, 0.0} : (tm ? cd{0.0, a.inv_sqrt2} : cd{0.0, 0.0});
    case EMU_POL_LCIRC: return te ? cd{a.inv_sqrt2, 0.0} : (tm ? cd{0.0, -a.inv_sqrt2} : cd{0.0, 0.0});
  }
  return cd{0.0, 0.0};
}

__device__ __forceinline__ void store_c(emu_c128 *p, size_t i, cd v) {
  p[i] = emu_c128{v.x, v.y};
}

// U-weighted flux contribution of one order and polarisation
// (backend/stack.py:311-321, 351): propagating orders give |f-|^2 - |f+|^2,
// evanescent ones the cross terms with -+i.
__device__ __forceinline__ cd flux_term(cd fm, cd fp, bool prop, bool tm) {
  if (prop) return cd{cabs2(fm) - cabs2(fp), 0.0};
  // TE: conj(fm)(-i)fp + conj(fp)(i)fm ; TM: conj(fm)(i)fp + conj(fp)(-i)fm
  const cd a = cmul(cconj(fm), fp);
  const cd b = cmul(cconj(fp), fm);
  const cd d = csub(b, a);
  const cd te = cd{-d.y, d.x};
  return tm ? cneg(te) : te;
}

__device__ __forceinline__ cd shear_phase(double alpha, double beta, double c0, double c1, int ncoord) {
  const double th = (ncoord == 1) ? alpha * c0 : alpha * c0 + beta * c1;
  double s, c;
  sincos(th, &s, &c);
  return cd{c, s};
}

// Cascade of one order (both polarisations) bottom to top, then, if the
// order carries incident light, its flux pass top to bottom.
__device__ void solve_order(const FilmArgs &a, int b, int u, int j, int spec, const LayerC *lay,
                            const double *hsm, const unsigned *wood, bool wood_air, double a0,
                            double b0, double sa0, double sb0, double wln, int np_air, int np_in,
                            int np_out, cd *acc, int *nprop, bool count) {
  const EmuFilmStackBatch &p = a.p;
  const int L = p.n_layers, npw = p.n_pw, P = 2 * npw;
  const int px = p.d_px[u], py = p.d_py[u];
  double al_air, be_air;
  order_ab(p.world_1d, a.dy, px, py, wood_air ? sa0 : a0, wood_air ? sb0 : b0, al_air, be_air);
  const cd kair = wavenumber(cd{1.0, 0.0}, wln);
  const cd kz_air = csqrt_p(kz_arg(kair, al_air, be_air));
  // air impedances (1/n = 1): Z_TE = k/kz, Z_TM = kz/k
  const cd z1[2] = {cmul(kair, crcp_nr(kz_air)), cmul(kz_air, crcp_nr(kair))};
  const cd sz1[2] = {csqrt_nr(z1[0]), csqrt_nr(z1[1])};
  const double *sh = p.d_shears;
  double al_sh = 0.0, be_sh = 0.0;
  if (sh)
    order_ab(p.world_1d, a.dy, p.d_px[j], p.d_py[j], wood_air ? sa0 : a0, wood_air ? sb0 : b0,
             al_sh, be_sh);
  const cd din[2] = {incidence(a, b, j, spec, npw), incidence(a, b, j + npw, spec, npw)};
  const bool active = !cis_zero(din[0]) || !cis_zero(din[1]);
  const int aslot = (p.pol == EMU_POL_INCOMING) ? u : 0;
  cd *wsv = a.ws + (((size_t)b * a.n_act + aslot) * L) * 2 * kSave;
  cd tnet[2], rnet[2];
  for (int l = 0; l < L; ++l) {
    const bool wl_l = (wood[l >> 5] >> (l & 31)) & 1u;
    double al, be;
    order_ab(p.world_1d, a.dy, px, py, wl_l ? sa0 : a0, wl_l ? sb0 : b0, al, be);
    const LayerC c = lay[l];
    const cd kz = csqrt_p(kz_arg(c.k, al, be));
    const bool fin = (l >= 1 && l < L - 1);
    if (count && fin && kz.y == 0.0) atomicAdd(&nprop[l], 1);
    if (p.d_kz) store_c(p.d_kz, ((size_t)b * L + l) * npw + j, kz);
    // Z_TE = (1/n) k / kz ; Z_TM = (1/n) kz / k
    const cd z2[2] = {cmul(c.zcr, cmul(c.k, crcp_nr(kz))), cmul(c.zcr, cmul(kz, c.ik))};
    const cd pr = fin ? cexp_ikh(kz, hsm[l - 1] / p.period) : cd{1.0, 0.0};
    cd Q = cd{1.0, 0.0}, Qi = cd{1.0, 0.0};
    if (sh && l >= 1) {
      double c0, c1;
      if (l < L - 1) {
        c0 = sh[2 * (l - 1)] - sh[2 * l];
        c1 = sh[2 * (l - 1) + 1] - sh[2 * l + 1];
      } else {
        c0 = sh[2 * l];
        c1 = sh[2 * l + 1];
      }
      Q = shear_phase(al_sh, be_sh, c0, c1, p.shear_ncoord);
      Qi = shear_phase(al_sh, be_sh, -1 * c0, -1 * c1, p.shear_ncoord);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const cd is = crcp_nr(cadd(z2[q], z1[q]));
      const cd R12 = cmul(csub(z2[q], z1[q]), is);
      const cd T12 = cmul(cscale(cmul(csqrt_nr(z2[q]), sz1[q]), 2.0), is);
      const cd R21 = cneg(R12), T21 = T12;
      if (p.d_layer_rt) {
        const size_t o = ((size_t)b * L + l) * 2 * P;
        store_c(p.d_layer_rt, o + j + q * npw, R12);
        store_c(p.d_layer_rt, o + P + j + q * npw, T12);
      }
      cd *sv = wsv + ((size_t)l * 2 + q) * kSave;
      if (l == 0) {
        tnet[q] = T12;
        rnet[q] = R12;
        if (active) {
          sv[0] = rnet[q];
          sv[1] = tnet[q];
        }
        continue;
      }
      // air gap below layer l (backend/stack.py:229-247, 263-278)
      cd x1;
      if (sh) {
        const cd rq = cmul(cmul(Qi, rnet[q]), Q);
        x1 = cmul(T21, crcp_nr(csub(cd{1.0, 0.0}, cmul(R12, rq))));
        tnet[q] = cmul(cmul(tnet[q], Q), x1);
        rnet[q] = cadd(R21, cmul(cmul(T12, rq), x1));
      } else {
        x1 = cmul(T21, crcp_nr(csub(cd{1.0, 0.0}, cmul(R12, rnet[q]))));
        tnet[q] = cmul(tnet[q], x1);
        rnet[q] = cadd(R21, cmul(cmul(T12, rnet[q]), x1));
      }
      if (active) {
        sv[0] = x1;
        sv[1] = rnet[q];
      }
      if (!fin) continue;
      // through layer l (backend/stack.py:249-262)
      const cd x2 = cmul(T12, crcp_nr(csub(cd{1.0, 0.0}, cmul(cmul(cmul(R21, pr), rnet[q]), pr))));
      const cd px2 = cmul(pr, x2);
      tnet[q] = cmul(tnet[q], px2);
      rnet[q] = cadd(R12, cmul(cmul(cmul(T21, pr), rnet[q]), px2));
      if (active) {
        sv[2] = pr;
        sv[3] = x2;
        sv[4] = rnet[q];
      }
    }
  }
  store_c(p.d_R_net, (size_t)b * P + j, rnet[0]);
  store_c(p.d_R_net, (size_t)b * P + j + npw, rnet[1]);
  store_c(p.d_T_net, (size_t)b * P + j, tnet[0]);
  store_c(p.d_T_net, (size_t)b * P + j + npw, tnet[1]);

  // ---- flux pass (backend/stack.py:323-366)
  const bool want_vec = p.d_vec_coef_down != nullptr;
  if (!active) {
    if (want_vec) {
      for (int lv = 0; lv < L; ++lv)
        for (int q = 0; q < 2; ++q)
          store_c(p.d_vec_coef_down, ((size_t)b * L + lv) * P + j + q * npw, cd{0.0, 0.0});
      for (int lv = 0; lv < L - 1; ++lv)
        for (int q = 0; q < 2; ++q)
          store_c(p.d_vec_coef_up, ((size_t)b * (L - 1) + lv) * P + j + q * npw, cd{0.0, 0.0});
    }
    return;
  }
  const bool prop = j < np_air;
  double in_sum = 0.0, up_sum = 0.0, out_sum = 0.0;
  for (int q = 0; q < 2; ++q) {
    const int pos = j + q * npw;
    const cd *top = wsv + ((size_t)(L - 1) * 2 + q) * kSave;
    const cd dp = cmul(top[1], din[q]);  // d_plus = r_top d
    if (j < np_in) {
      in_sum += cabs2(din[q]);
      up_sum += cabs2(dp);
    }
    if (want_vec) {
      store_c(p.d_vec_coef_down, ((size_t)b * L + 0) * P + pos, din[q]);
      store_c(p.d_vec_coef_up, ((size_t)b * (L - 1) + 0) * P + pos, dp);
    }
    cd f1m = cmul(top[0], din[q]);
    for (int i = 0; i < L - 2; ++i) {
      const int k = L - 2 - i;
      const cd *s = wsv + ((size_t)k * 2 + q) * kSave;
      const cd f1p = cmul(s[4], f1m);
      const cd fl = flux_term(f1m, f1p, prop, q == 1);
      atomicAdd(&acc[1 + i].x, fl.x);
      atomicAdd(&acc[1 + i].y, fl.y);
      const cd f2m = cmul(s[3], f1m);
      const cd f2p = cmul(cmul(s[1], s[2]), f2m);
      if (want_vec) {
        store_c(p.d_vec_coef_down, ((size_t)b * L + 1 + i) * P + pos, f2m);
        store_c(p.d_vec_coef_up, ((size_t)b * (L - 1) + 1 + i) * P + pos, f2p);
      }
      f1m = cmul(cmul(s[0], s[2]), f2m);
    }
    const cd *s0 = wsv + ((size_t)0 * 2 + q) * kSave;
    const cd f2m = cmul(s0[1], f1m);
    if (want_vec) store_c(p.d_vec_coef_down, ((size_t)b * L + L - 1) * P + pos, f2m);
    if (j < np_out) out_sum += cabs2(f2m);
  }
  atomicAdd(&acc[0].x, in_sum);
  atomicAdd(&acc[L].x, up_sum);
  atomicAdd(&acc[L - 1].x, out_sum);
}

__global__ void __launch_bounds__(kThreads, 2) film_stack_kernel(FilmArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const EmuFilmStackBatch &p = a.p;
  const int B = p.n_points, L = p.n_layers, npw = p.n_pw;
  const int team = a.team, ppc = a.ppc;
  const int slot = threadIdx.x / team;
  const int lt = threadIdx.x % team;
  const bool in_slot = slot < ppc;
  const SlotSmem S = slot_layout(npw, L);
  unsigned char *base = smem + (in_slot ? slot : 0) * S.stride;
  LayerC *lay = (LayerC *)(base + S.lay);
  cd *acc = (cd *)(base + S.acc);
  double *keys = (double *)(base + S.keys);
  double *hsm = (double *)(base + S.h);
  int *rank = (int *)(base + S.rank);
  int *nprop = (int *)(base + S.nprop);
  unsigned *wood = (unsigned *)(base + S.wood);
  int *misc = (int *)(base + S.misc);
  const int wood_words = (L + 1 + 31) / 32;
  const bool count = p.d_num_prop != nullptr;

  for (int bb = blockIdx.x * ppc; bb < B; bb += gridDim.x * ppc) {
    const int b = bb + slot;
    const bool valid = in_slot && b < B;
    double wln = 1.0, a0 = 0.0, b0 = 0.0;
    if (valid) {
      wln = wl_norm(p.d_wl_nm[b], p.period);
      a0 = p.d_k_pll[2 * (size_t)b] * p.period;
      b0 = p.d_k_pll[2 * (size_t)b + 1] * p.period;
    }
    const double sa0 = (1 - 1e-9) * a0, sb0 = (1 - 1e-9) * b0;
    // ---------------------------------------------------------- phase 0
    if (valid) {
      for (int i = lt; i < L; i += team) {
        const emu_c128 v = p.d_n[(size_t)b * L + i];
        const cd n = cd{v.re, v.im};
        LayerC c;
        c.k = wavenumber(n, wln);
        c.zcr = crecip(n);
        c.ik = crecip(c.k);
        lay[i] = c;
      }
      for (int i = lt; i < L - 2; i += team)
        hsm[i] = p.d_heights_nm[(p.heights_per_point ? (size_t)b * (L - 2) : 0) + i];
      for (int i = lt; i < L + 1; i += team) {
        acc[i] = cd{0.0, 0.0};
        nprop[i] = 0;
      }
      for (int i = lt; i < wood_words; i += team) wood[i] = 0u;
      if (lt == 0) {
        misc[0] = -1;
        misc[1] = 0;
      }
    }
    __syncthreads();
    // ---------------------------------------------------------- phase 1
    if (valid) {
      const cd kair = wavenumber(cd{1.0, 0.0}, wln);
      for (int u = lt; u < npw; u += team) {
        double al, be;
        order_ab(p.world_1d, a.dy, p.d_px[u], p.d_py[u], a0, b0, al, be);
        const cd kz = csqrt_p(kz_arg(kair, al, be));
        if (cis_zero(kz)) atomicOr(&wood[L >> 5], 1u << (L & 31));
        keys[u] = -1 * kz.x + kz.y;
        if (kz.y == 0.0) atomicAdd(&nprop[L], 1);
      }
    }
    __syncthreads();
    // ---------------------------------------------------------- phase 2
    const bool wood_air = valid && ((wood[L >> 5] >> (L & 31)) & 1u);
    if (__syncthreads_or(wood_air)) {
      if (wood_air && lt == 0) nprop[L] = 0;
      __syncthreads();
      if (wood_air) {
        const cd kair = wavenumber(cd{1.0, 0.0}, wln);
        for (int u = lt; u < npw; u += team) {
          double al, be;
          order_ab(p.world_1d, a.dy, p.d_px[u], p.d_py[u], sa0, sb0, al, be);
          const cd kz = csqrt_p(kz_arg(kair, al, be));
          keys[u] = -1 * kz.x + kz.y;
          if (kz.y == 0.0) atomicAdd(&nprop[L], 1);
        }
      }
      __syncthreads();
    }
    // ---------------------------------------------------------- phase 3
    if (valid) {
      for (int u = lt; u < npw; u += team) {
        const double ku = keys[u];
        int r = 0;
        for (int v = 0; v < npw; ++v) {
          const double kv = keys[v];
          r += (kv < ku) || (kv == ku && v < u);
        }
        rank[u] = r;
        const bool zero_order = (p.d_px[u] == 0) && (p.world_1d || p.d_py[u] == 0);
        if (zero_order) misc[0] = r;
        if (p.d_sort_order) p.d_sort_order[(size_t)b * npw + r] = u;
        double al, be;
        order_ab(p.world_1d, a.dy, p.d_px[u], p.d_py[u], a0, b0, al, be);
        if (csqrt_p(kz_arg(lay[0].k, al, be)).y == 0.0) atomicAdd(&nprop[0], 1);
        if (csqrt_p(kz_arg(lay[L - 1].k, al, be)).y == 0.0) atomicAdd(&nprop[L - 1], 1);
        // Wood check of every layer: k_z == 0 exactly iff its argument is 0
        for (int l = 0; l < L; ++l) {
          const cd arg = kz_arg(lay[l].k, al, be);
          if (arg.x == 0.0 && arg.y == 0.0) {
            atomicOr(&wood[l >> 5], 1u << (l & 31));
            misc[1] = 1;
          }
        }
      }
    }
    __syncthreads();
    // ---------------------------------------------------------- phase 4
    const bool layer_wood = valid && misc[1] != 0;
    if (valid && !layer_wood) {
      const int spec = misc[0];
      const int np_air = nprop[L], np_in = nprop[L - 1], np_out = nprop[0];
      for (int u = lt; u < npw; u += team)
        solve_order(a, b, u, rank[u], spec, lay, hsm, wood, wood_air, a0, b0, sa0, sb0, wln,
                    np_air, np_in, np_out, acc, nprop, count);
    }
    // ---------------------------------------------------------- phase 5
    if (__syncthreads_or(layer_wood)) {
      // recount substrate / superstrate with the scaled k_parallel where marked
      if (layer_wood && lt == 0) {
        nprop[0] = 0;
        nprop[L - 1] = 0;
      }
      __syncthreads();
      if (layer_wood) {
        for (int u = lt; u < npw; u += team) {
          for (int t = 0; t < 2; ++t) {
            const int l = t ? L - 1 : 0;
            const bool wl_l = (wood[l >> 5] >> (l & 31)) & 1u;
            double al, be;
            order_ab(p.world_1d, a.dy, p.d_px[u], p.d_py[u], wl_l ? sa0 : a0, wl_l ? sb0 : b0, al, be);
            if (csqrt_p(kz_arg(lay[l].k, al, be)).y == 0.0) atomicAdd(&nprop[l], 1);
          }
        }
      }
      __syncthreads();
      if (layer_wood) {
        const int spec = misc[0];
        const int np_air = nprop[L], np_in = nprop[L - 1], np_out = nprop[0];
        for (int u = lt; u < npw; u += team)
          solve_order(a, b, u, rank[u], spec, lay, hsm, wood, wood_air, a0, b0, sa0, sb0, wln,
                      np_air, np_in, np_out, acc, nprop, count);
      }
    }
    __syncthreads();
    // ---------------------------------------------------------- phase 6
    if (valid && lt == 0) {
      uint32_t flags = 0;
      if (wood_air) flags |= EMU_PT_WOOD_AIR;
      if (layer_wood) flags |= EMU_PT_WOOD_LAYER;
      const int np_in = nprop[L - 1], np_out = nprop[0];
      if (np_out == 0) flags |= EMU_PT_NO_PROP_SUB;
      if (np_in == 0) flags |= EMU_PT_NO_PROP_SUP;
      double *al = p.d_a_list + (size_t)b * (L - 1);
      double *tl = p.d_t_list + (size_t)b * (L - 1);
      const double df0 = acc[0].x, up0 = acc[L].x, dsub = acc[L - 1].x;
      // |down_fluxes[i]| with down_fluxes = [df0, gap_1..gap_{L-2}, dsub]
      auto dfa = [&](int i) -> double {
        if (i == 0) return fabs(df0);
        if (i == L - 1) return fabs(dsub);
        return hypot(acc[i].x, acc[i].y);
      };
      double rr = 0.0;
      if (np_out != 0) {
        for (int i = 1; i <= L - 2; ++i) al[i - 1] = fabs(dfa(i) - dfa(i + 1));
        al[L - 2] = fabs(df0 - dsub - up0);
        for (int i = 0; i <= L - 3; ++i) tl[i] = fabs(dfa(i + 2) / dfa(i));
        tl[L - 2] = fabs(dsub / df0);
        rr = fabs(up0 / df0);
      } else {
        for (int i = 0; i < L - 1; ++i) {
          al[i] = 0.0;
          tl[i] = 0.0;
        }
      }
      p.d_r_list[b] = rr;
      bool fin = isfinite(rr);
      for (int i = 0; i < L - 1; ++i) fin = fin && isfinite(al[i]) && isfinite(tl[i]);
      if (!fin) flags |= EMU_PT_NONFINITE;
      p.d_flags[b] = flags;
      if (p.d_specular) p.d_specular[b] = misc[0];
      if (p.d_num_prop)
        for (int i = 0; i <= L; ++i) p.d_num_prop[(size_t)b * (L + 1) + i] = nprop[i];
      if (p.d_fluxes) {
        double *fo = p.d_fluxes + (size_t)b * (L + 1) * 2;
        for (int i = 0; i <= L; ++i) {
          fo[2 * i] = acc[i].x;
          fo[2 * i + 1] = acc[i].y;
        }
      }
    }
    __syncthreads();
  }
}

struct Launch {
  int team, ppc, n_act;
  size_t smem;
};

Launch plan(const EmuFilmStackBatch *p) {
  Launch l;
  l.team = p->n_pw <= kThreads ? p->n_pw : kThreads;
  l.ppc = kThreads / l.team;
  l.n_act = (p->pol == EMU_POL_INCOMING) ? p->n_pw : 1;
  l.smem = (size_t)slot_layout(p->n_pw, p->n_layers).stride * l.ppc;
  return l;
}

int validate(const EmuFilmStackBatch *p) {
  if (!p) return EMU_E_ARG;
  if (p->n_points < 0 || p->n_layers < 2 || p->n_pw < 1) return EMU_E_SHAPE;
  if (!(p->period > 0) || !(p->period_y > 0)) return EMU_E_ARG;
  if (p->pol < EMU_POL_INCOMING || p->pol > EMU_POL_LCIRC) return EMU_E_ARG;
  if (p->pol == EMU_POL_INCOMING && !p->d_incoming) return EMU_E_ARG;
  if (p->n_points > 0 &&
      (!p->d_px || !p->d_py || !p->d_wl_nm || !p->d_k_pll || !p->d_n || !p->d_R_net ||
       !p->d_T_net || !p->d_a_list || !p->d_t_list || !p->d_r_list || !p->d_flags))
    return EMU_E_ARG;
  if (p->n_layers > 2 && p->n_points > 0 && !p->d_heights_nm) return EMU_E_ARG;
  if ((p->d_vec_coef_down == nullptr) != (p->d_vec_coef_up == nullptr)) return EMU_E_ARG;
  if (p->d_shears && p->shear_ncoord != 1 && p->shear_ncoord != 2) return EMU_E_ARG;
  if (slot_layout(p->n_pw, p->n_layers).stride > 200 * 1024) return EMU_E_SHAPE;
  return EMU_OK;
}

}  // namespace

extern "C" size_t emu_film_stack_workspace_size(const EmuFilmStackBatch *p) {
  if (validate(p) != EMU_OK) return 0;
  const Launch l = plan(p);
  return (size_t)p->n_points * l.n_act * p->n_layers * 2 * kSave * sizeof(cd);
}

extern "C" int emu_film_stack_batch(const EmuFilmStackBatch *p, void *d_workspace,
                                    size_t workspace_bytes, void *stream) {
  int st = validate(p);
  if (st != EMU_OK) return st;
  if (p->n_points == 0) return EMU_OK;
  const size_t need = emu_film_stack_workspace_size(p);
  if (!d_workspace || workspace_bytes < need) return EMU_E_WORKSPACE;
  const Launch l = plan(p);
  FilmArgs a;
  a.p = *p;
  a.team = l.team;
  a.ppc = l.ppc;
  a.n_act = l.n_act;
  a.ws = (cd *)d_workspace;
  a.dy = p->period_y / p->period;
  a.inv_sqrt2 = 1.0 / sqrt(2.0);
  if (l.smem > 48 * 1024) {
    if (cudaFuncSetAttribute(film_stack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)l.smem) != cudaSuccess)
      return EMU_E_CUDA;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, film_stack_kernel, kThreads, l.smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long groups = ((long long)p->n_points + l.ppc - 1) / l.ppc;
  long long grid = (long long)emu::sm_count() * per_sm;
  if (grid > groups) grid = groups;
  film_stack_kernel<<<(int)grid, kThreads, l.smem, (cudaStream_t)stream>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the point where they solve:
// a host thread inside a latency-critical loop (cudaMalloc and cudaFree
// synchronise the device), code that runs while another framework owns the
// device heap through its own caching allocator, or an embedding that must
// not fail on memory pressure after start-up.  For them the film solve can
// use a fixed scratch array compiled into this library instead of a
// caller-provided workspace.  The array lives in every GPU that loads the
// library, for the life of the process.
#include <mutex>

namespace {

constexpr size_t kStaticScratchBytes = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_film_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[64] = {nullptr};

}  // namespace

extern "C" size_t emu_film_stack_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int emu_film_stack_batch_noalloc(const EmuFilmStackBatch *p, void *stream) {
  int st = validate(p);
  if (st != EMU_OK) return st;
  if (p->n_points == 0) return EMU_OK;
  if (emu_film_stack_workspace_size(p) > kStaticScratchBytes) return EMU_E_WORKSPACE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return EMU_E_CUDA;
  void *addr = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      // the host-side name of the array is not a device address: ask the
      // runtime for this device's copy once, with the device current
      if (cudaGetSymbolAddress(&g_scratch_addr[dev], g_film_scratch) != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        cudaGetLastError();
        return EMU_E_CUDA;
      }
    }
    addr = g_scratch_addr[dev];
  }
  return emu_film_stack_batch(p, addr, kStaticScratchBytes, stream);
}
