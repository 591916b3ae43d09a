// Per-order film recursion shared by the film kernels (uniform batches in
// film_stack.cu, heterogeneous batches in film_varlen.cu): impedances,
// Fresnel interfaces, the bottom-to-top cascade of one plane-wave order for
// both polarisations and, for orders carrying incident light, the
// top-to-bottom flux pass (backend/mode_calcs.py:199-218, 451-477;
// backend/stack.py:196-366).
#pragma once
#include "emu_cplx.cuh"
#include "emu_fastmath.cuh"
#include "emu_internal.h"
#include "emu_modes.cuh"

namespace emu {

constexpr int kSave = 5;  // saved scalars per (layer, polarisation)

struct LayerC {
  cd k, zcr, ik;  // wavenumber, 1/n, 1/k
  cd zk, zka;     // k / n and k_air / n (k_air real)
  cd kk;          // k^2, rounded as kz_arg rounds it
};

// Shared-memory layout of one point's slot (byte offsets); a slot sized for
// (npw, L) also holds any point with fewer orders and layers.
struct SlotSmem {
  int keys, rank, wood, nprop, acc, lay, h, misc, ws, stride;
};

// with_ws: room for the flux-pass scalars of the one order that carries
// light ([L][2][kSave]), for every polarisation but incoming amplitudes
// (whose scalars, one set per order, stay in the global workspace).
__host__ __device__ inline SlotSmem slot_layout(int npw, int L, bool with_ws = true) {
  SlotSmem s;
  int o = 0;
  s.lay = o; o += (int)sizeof(LayerC) * L;
  s.ws = o; o += with_ws ? (int)sizeof(cd) * L * 2 * kSave : 0;
  s.acc = o; o += 16 * (L + 1);
  s.keys = o; o += 8 * npw;
  s.h = o; o += 8 * (L > 2 ? L - 2 : 1);
  s.rank = o; o += 4 * npw;
  s.nprop = o; o += 4 * (L + 1);
  s.wood = o; o += 4 * ((L + 1 + 31) / 32);
  s.misc = o; o += 16;  // [0] specular order, [1] layer-Wood flag, [2] non-finite list entry
  s.stride = (o + 15) / 16 * 16;
  return s;
}

// Thread teams that solve one point together: a whole CTA's slot (uniform
// batches, barriers over the CTA) or one warp (heterogeneous batches).
struct CtaTeam {
  int lt, size;
  __device__ void sync() const { __syncthreads(); }
  __device__ bool any(bool v) const { return __syncthreads_or(v) != 0; }
};
struct WarpTeam {
  int lt;
  static constexpr int size = 32;
  __device__ void sync() const { __syncwarp(); }
  __device__ bool any(bool v) const { return __any_sync(0xffffffffu, v) != 0; }
};

// A point accessor P (FilmPointCtx-like) exposes, as member functions:
//   L() npw() world_1d() pol() ncoord() slot_per_order() dy() period()
//   inv_sqrt2(), px() py() (order lists), incoming() ([P] or unused),
//   shears() ([L][2] or NULL), ws() ([n_slots][L][2][kSave] workspace),
//   R_net() T_net() ([P]), kz() ([L][npw] or NULL), layer_rt() ([L][2][P]
//   or NULL), vcd() vcu() ([L][P], [L-1][P] or NULL).
// Accessors compute these from kernel parameters on demand, so the
// recursion holds no per-point pointers in registers.
template <class Pt>
__device__ __forceinline__ cd incidence(const Pt &c, int pos, int spec) {
  const int pol = c.pol(), npw = c.npw();
  if (pol == EMU_POL_INCOMING) {
    const emu_c128 v = c.incoming()[pos];
    return cd{v.re, v.im};
  }
  const bool te = (pos == spec), tm = (pos == spec + npw);
  switch (pol) {
    case EMU_POL_TE: return te ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_TM: return tm ? cd{1.0, 0.0} : cd{0.0, 0.0};
    case EMU_POL_UN: return (te || tm) ? cd{c.inv_sqrt2(), 0.0} : cd{0.0, 0.0};
    case EMU_POL_RCIRC: return te ? cd{c.inv_sqrt2(), 0.0} : (tm ? cd{0.0, c.inv_sqrt2()} : cd{0.0, 0.0});
    case EMU_POL_LCIRC: return te ? cd{c.inv_sqrt2(), 0.0} : (tm ? cd{0.0, -c.inv_sqrt2()} : cd{0.0, 0.0});
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

// Transmission coefficient T12 = T21 of the air / layer interface for
// polarisation q (0 TE, 1 TM): 2 sqrt(z2) sqrt(z1) / (z2 + z1) with the
// impedances z1 of air and z2 of the layer (backend/mode_calcs.py:199-218,
// 451-477), principal square roots as numpy takes them.
__device__ __forceinline__ cd t12_exact(const LayerC &c, cd kz, double kair, cd kz_air, int q) {
  cd z1, z2;
  if (q == 0) {
    z1 = cscale(crcp_nr(kz_air), kair);
    z2 = cmul(c.zcr, cmul(c.k, crcp_nr(kz)));
  } else {
    z1 = cscale(kz_air, 1.0 / kair);
    z2 = cmul(c.zcr, cmul(kz, c.ik));
  }
  const cd is = crcp_nr(cadd(z2, z1));
  return cmul(cscale(cmul(csqrt_k(z2), csqrt_k(z1)), 2.0), is);
}

// R12 and T12 T21 of the air / layer interface for polarisation q from the
// scaled impedances A, B (the scaling is described at solve_order).
__device__ __forceinline__ void iface_scaled(const LayerC &c, cd kz, double kair, cd kz_air, int q,
                                             cd &R12, cd &TT) {
  const cd A = q ? cmul(c.zka, kz) : cmul(c.zk, kz_air);
  const cd Bz = q ? cmul(kz_air, c.k) : cscale(kz, kair);
  const cd is = crcp_nr(cadd(A, Bz));
  R12 = cmul(csub(A, Bz), is);
  TT = cmul(cscale(cmul(A, Bz), 4.0), cmul(is, is));
}

// Cascade of one order (both polarisations) bottom to top, then, if the
// order carries incident light, its flux pass top to bottom.
//
// The reference builds each interface from z1, z2 as R12 = (z2 - z1)/(z2 + z1)
// and T12 = T21 = 2 sqrt(z2 z1)/(z2 + z1) and runs the recursion of
// backend/stack.py:229-278 on them.  Here, for a layer between two air gaps:
//  * z1 and z2 are scaled by k_z k_z,air (TE) or k k_air (TM), which leaves
//    R12 unchanged and removes the quotient inside each impedance:
//    R12 = (A - B)/(A + B) with A = k k_z,air / n, B = k_air k_z (TE) and
//    A = k_air k_z / n, B = k k_z,air (TM);
//  * T12 enters the reflection recursion only as T12 T21 = 4 A B/(A + B)^2,
//    and the transmission and the downward gap fields of the flux pass only
//    as the product over one layer x1 p x2 = T12 T21 p / (d1 d2), with
//    d1 = 1 - R12 r (gap) and d2 = 1 + R12 p^2 r (film, p = exp(i k_z h)),
//    so no square root is taken for them.
// The outer layers (substrate, superstrate) and the optional per-layer
// outputs (layer_rt, vec_coef) take T12 itself from t12_exact.  Every
// result is the same whichever optional outputs are requested.
template <class Pt>
__device__ __forceinline__ void solve_order(const Pt &p, int u, int j, int spec, const LayerC *lay,
                            const double *hsm, const unsigned *wood, bool wood_air, double a0,
                            double b0, double sa0, double sb0, double wln, int np_air, int np_in,
                            int np_out, cd *acc, int *nprop, bool count, cd *ws_smem) {
  const int L = p.L(), npw = p.npw(), P = 2 * npw;
  const int px = p.px()[u], py = p.py()[u];
  // alpha^2 and beta^2 of the order, with k_parallel as given and scaled by
  // 1 - 1e-9 (layers at a Wood anomaly)
  double al2, be2, al2w, be2w;
  {
    double al, be;
    order_ab(p.world_1d(), p.dy(), px, py, a0, b0, al, be);
    al2 = __dmul_rn(al, al);
    be2 = __dmul_rn(be, be);
    order_ab(p.world_1d(), p.dy(), px, py, sa0, sb0, al, be);
    al2w = __dmul_rn(al, al);
    be2w = __dmul_rn(be, be);
  }
  const double kair = wavenumber(cd{1.0, 0.0}, wln).x;
  const cd kz_air = csqrt_k(kz_arg_sq(k_squared(cd{kair, 0.0}), wood_air ? al2w : al2,
                                      wood_air ? be2w : be2));
  const double *sh = p.shears();
  double al_sh = 0.0, be_sh = 0.0;
  if (sh)
    order_ab(p.world_1d(), p.dy(), p.px()[j], p.py()[j], wood_air ? sa0 : a0, wood_air ? sb0 : b0, al_sh,
             be_sh);
  const cd din[2] = {incidence(p, j, spec), incidence(p, j + npw, spec)};
  const bool active = !cis_zero(din[0]) || !cis_zero(din[1]);
  const bool want_vec = p.vcd() != nullptr;
  const bool all_t = want_vec || p.layer_rt() != nullptr;
  // flux-pass scalars: in the point's shared-memory slot when one order
  // carries light, else per order in the global workspace
  cd *wsv = p.slot_per_order() ? p.ws() + ((size_t)u * L) * 2 * kSave : ws_smem;
  // k_z of the order in layer l (also stored when requested)
  auto layer_kz = [&](int l) -> cd {
    const int wl = (wood[l >> 5] >> (l & 31)) & 1u;
    const cd kz = csqrt_k(kz_arg_sq(lay[l].kk, wl ? al2w : al2, wl ? be2w : be2));
    if (p.kz()) store_c(p.kz(), (size_t)l * npw + j, kz);
    return kz;
  };
  // shear phase Q of the gap below layer l and its inverse (backend/stack.py:236-244, 267-275)
  auto shear_q = [&](int l, cd &Q, cd &Qi) {
    Q = cd{1.0, 0.0};
    Qi = cd{1.0, 0.0};
    if (!sh) return;
    double c0, c1;
    if (l < L - 1) {
      c0 = sh[2 * (l - 1)] - sh[2 * l];
      c1 = sh[2 * (l - 1) + 1] - sh[2 * l + 1];
    } else {
      c0 = sh[2 * l];
      c1 = sh[2 * l + 1];
    }
    Q = shear_phase(al_sh, be_sh, c0, c1, p.ncoord());
    Qi = shear_phase(al_sh, be_sh, -1 * c0, -1 * c1, p.ncoord());
  };
  auto store_rt = [&](int l, int q, cd R12, cd T12) {
    if (!p.layer_rt()) return;
    const size_t o = (size_t)l * 2 * P;
    store_c(p.layer_rt(), o + j + q * npw, R12);
    store_c(p.layer_rt(), o + P + j + q * npw, T12);
  };
  cd tnet[2], rnet[2];
  // substrate (l = 0)
  {
    const LayerC c = lay[0];
    const cd kz = layer_kz(0);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      cd R12, TT;
      iface_scaled(c, kz, kair, kz_air, q, R12, TT);
      const cd T12 = t12_exact(c, kz, kair, kz_air, q);
      store_rt(0, q, R12, T12);
      tnet[q] = T12;
      rnet[q] = R12;
      if (active) {
        cd *sv = wsv + (size_t)q * kSave;
        sv[0] = R12;
        sv[1] = T12;
      }
    }
  }
  // films between air gaps (backend/stack.py:229-262).  With s = A + B and
  // d = A - B the interface is R12 = d/s, T12 T21 = 4AB/s^2, and
  // T12 T21 + R12^2 = 1, so the gap and layer steps of the reference,
  //   rg = T12 (1 - R12 rq)^-1 T21 rq - R12,   (air gap, rq = rnet below)
  //   rnet' = R12 + T12 p rg p (1 + R12 p rg p)^-1 T21,
  // are Moebius maps: rg = v/u and rnet' = N/D with
  //   u = s - d rq,  v = s rq - d,  D = s u + d p^2 v,  N = d u + s p^2 v,
  // and the transmission through gap and layer, x1 p x2 = 4AB p / D, shares
  // the one quotient 1/D (x1 = T12 (1 - R12 rq)^-1, x2 the layer's
  // (1 + R12 p rg p)^-1 T21 = s u / D with T21 folded in).
  for (int l = 1; l < L - 1; ++l) {
    const LayerC c = lay[l];
    const cd kz = layer_kz(l);
    if (count && kz.y == 0.0) atomicAdd(&nprop[l], 1);
    const cd pr = cexp_ikh(kz, hsm[l - 1]);
    const cd pr2 = cmul(pr, pr);
    cd Q, Qi;
    shear_q(l, Q, Qi);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const cd A = q ? cmul(c.zka, kz) : cmul(c.zk, kz_air);
      const cd Bz = q ? cmul(kz_air, c.k) : cscale(kz, kair);
      const cd s = cadd(A, Bz), d = csub(A, Bz);
      cd T12 = cd{0.0, 0.0};
      if (all_t) {
        T12 = t12_exact(c, kz, kair, kz_air, q);
        store_rt(l, q, cmul(d, crcp_nr(s)), T12);
      }
      const cd rq = sh ? cmul(cmul(Qi, rnet[q]), Q) : rnet[q];
      const cd u = csub(s, cmul(d, rq));
      const cd v = csub(cmul(s, rq), d);
      const cd w = cmul(pr2, v);
      const cd Dn = cadd(cmul(s, u), cmul(d, w));
      const cd Nn = cadd(cmul(d, u), cmul(s, w));
      const cd iD = crcp_nr(Dn);
      const cd g = cmul(cscale(cmul(cmul(A, Bz), pr), 4.0), iD);  // x1 p x2
      tnet[q] = cmul(sh ? cmul(tnet[q], Q) : tnet[q], g);
      rnet[q] = cmul(Nn, iD);
      if (active) {
        cd *sv = wsv + ((size_t)l * 2 + q) * kSave;
        sv[0] = g;
        sv[2] = pr;
        if (want_vec) {
          sv[1] = cmul(v, crcp_nr(u));               // rg
          sv[3] = cmul(cmul(T12, cmul(s, u)), iD);  // T12 x2 / T21 = T12 (1 + R12 p rg p)^-1
        }
        sv[4] = rnet[q];
      }
    }
  }
  // superstrate (l = L - 1): the air gap below it (backend/stack.py:263-278)
  {
    const int l = L - 1;
    const LayerC c = lay[l];
    const cd kz = layer_kz(l);
    cd Q, Qi;
    shear_q(l, Q, Qi);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      cd R12, TT;
      iface_scaled(c, kz, kair, kz_air, q, R12, TT);
      const cd T12 = t12_exact(c, kz, kair, kz_air, q);
      store_rt(l, q, R12, T12);
      const cd rq = sh ? cmul(cmul(Qi, rnet[q]), Q) : rnet[q];
      const cd d1 = crcp_nr(csub(cd{1.0, 0.0}, cmul(R12, rq)));
      const cd x1 = cmul(T12, d1);
      tnet[q] = cmul(sh ? cmul(tnet[q], Q) : tnet[q], x1);
      rnet[q] = csub(cmul(cmul(TT, d1), rq), R12);
      if (active) {
        cd *sv = wsv + ((size_t)l * 2 + q) * kSave;
        sv[0] = x1;
        sv[1] = rnet[q];
      }
    }
  }
  store_c(p.R_net(), j, rnet[0]);
  store_c(p.R_net(), j + npw, rnet[1]);
  store_c(p.T_net(), j, tnet[0]);
  store_c(p.T_net(), j + npw, tnet[1]);

  // ---- flux pass (backend/stack.py:323-366)
  if (!active) {
    if (want_vec) {
      for (int lv = 0; lv < L; ++lv)
        for (int q = 0; q < 2; ++q) store_c(p.vcd(), (size_t)lv * P + j + q * npw, cd{0.0, 0.0});
      for (int lv = 0; lv < L - 1; ++lv)
        for (int q = 0; q < 2; ++q) store_c(p.vcu(), (size_t)lv * P + j + q * npw, cd{0.0, 0.0});
    }
    return;
  }
  const bool prop = j < np_air;
  double in_sum = 0.0, up_sum = 0.0, out_sum = 0.0;
  for (int q = 0; q < 2; ++q) {
    // a polarisation without incident light (TE or TM incidence) carries
    // zero amplitudes through every layer and adds nothing to the fluxes,
    // unless its saved scalars are not finite (0 times them is NaN, as in
    // the reference's dense products): then it runs like the other
    if (!want_vec && cis_zero(din[q])) {
      double chk = 0.0;
      for (int k = 0; k < L; ++k) {
        const cd *sk = wsv + ((size_t)k * 2 + q) * kSave;
        chk += sk[0].x + sk[0].y + sk[1].x + sk[1].y + sk[4].x + sk[4].y;
      }
      if (isfinite(chk)) continue;
    }
    const int pos = j + q * npw;
    const cd *top = wsv + ((size_t)(L - 1) * 2 + q) * kSave;
    const cd dp = cmul(top[1], din[q]);  // d_plus = r_top d
    if (j < np_in) {
      in_sum += cabs2(din[q]);
      up_sum += cabs2(dp);
    }
    if (want_vec) {
      store_c(p.vcd(), pos, din[q]);
      store_c(p.vcu(), pos, dp);
    }
    cd f1m = cmul(top[0], din[q]);
    for (int i = 0; i < L - 2; ++i) {
      const int k = L - 2 - i;
      const cd *s = wsv + ((size_t)k * 2 + q) * kSave;
      const cd f1p = cmul(s[4], f1m);
      const cd fl = flux_term(f1m, f1p, prop, q == 1);
      if (p.slot_per_order()) {  // several orders carry light: they add concurrently
        atomicAdd(&acc[1 + i].x, fl.x);
        atomicAdd(&acc[1 + i].y, fl.y);
      } else {                   // the one order that carries light adds alone
        acc[1 + i].x += fl.x;
        acc[1 + i].y += fl.y;
      }
      if (want_vec) {
        const cd f2m = cmul(s[3], f1m);
        const cd f2p = cmul(cmul(s[1], s[2]), f2m);
        store_c(p.vcd(), (size_t)(1 + i) * P + pos, f2m);
        store_c(p.vcu(), (size_t)(1 + i) * P + pos, f2p);
      }
      f1m = cmul(s[0], f1m);
    }
    const cd *s0 = wsv + ((size_t)0 * 2 + q) * kSave;
    const cd f2m = cmul(s0[1], f1m);
    if (want_vec) store_c(p.vcd(), (size_t)(L - 1) * P + pos, f2m);
    if (j < np_out) out_sum += cabs2(f2m);
  }
  atomicAdd(&acc[0].x, in_sum);
  atomicAdd(&acc[L].x, up_sum);
  atomicAdd(&acc[L - 1].x, out_sum);
}

// Sort key of -Re k_z + Im k_z as an unsigned integer with the order of the
// doubles (sign bit flipped for positive values, all bits for negative
// ones; -0 taken as +0, as the double comparison does).
__device__ __forceinline__ unsigned long long sort_key(double k) {
  const long long b = __double_as_longlong(k + 0.0);
  return b < 0 ? ~(unsigned long long)b : (unsigned long long)b | 0x8000000000000000ull;
}

// One point, phases 0-6 (the film kernels' header comments describe them).
// Every thread of the team calls this with the same `valid`, and with
// `valid` false takes the same barriers without touching memory.  The point
// accessor adds, to the fields solve_order uses: wl_nm() kx() ky() (k_pll),
// n(i), height(i), and the optional outputs sort_order() specular()
// num_prop() fluxes() (NULL to skip), and the required a_list() t_list()
// r_list() flags().
template <class Team, class Pt>
__device__ __forceinline__ void film_point(const Team &tm, const Pt &p, bool valid,
                                           unsigned char *base, const SlotSmem &S) {
  LayerC *lay = (LayerC *)(base + S.lay);
  cd *acc = (cd *)(base + S.acc);
  unsigned long long *keys = (unsigned long long *)(base + S.keys);
  double *hsm = (double *)(base + S.h);
  int *rank = (int *)(base + S.rank);
  int *nprop = (int *)(base + S.nprop);
  unsigned *wood = (unsigned *)(base + S.wood);
  cd *ws_smem = (cd *)(base + S.ws);
  int *misc = (int *)(base + S.misc);
  const int lt = tm.lt, team = tm.size;
  const int L = valid ? p.L() : 2, npw = valid ? p.npw() : 1;
  const int wood_words = (L + 1 + 31) / 32;
  const bool count = valid && p.num_prop() != nullptr;
  double wln = 1.0, a0 = 0.0, b0 = 0.0;
  if (valid) {
    wln = wl_norm(p.wl_nm(), p.period());
    a0 = p.kx() * p.period();
    b0 = p.ky() * p.period();
  }
  const double sa0 = (1 - 1e-9) * a0, sb0 = (1 - 1e-9) * b0;
  // ---------------------------------------------------------- phase 0
  if (valid) {
    for (int i = lt; i < L; i += team) {
      const emu_c128 v = p.n(i);
      const cd n = cd{v.re, v.im};
      LayerC c;
      c.k = wavenumber(n, wln);
      c.zcr = crcp_nr(n);
      c.ik = crcp_nr(c.k);
      c.zk = cmul(c.zcr, c.k);
      c.zka = cscale(c.zcr, wavenumber(cd{1.0, 0.0}, wln).x);
      c.kk = k_squared(c.k);
      lay[i] = c;
    }
    for (int i = lt; i < L - 2; i += team) hsm[i] = p.height(i) / p.period();
    for (int i = lt; i < L + 1; i += team) {
      acc[i] = cd{0.0, 0.0};
      nprop[i] = 0;
    }
    for (int i = lt; i < wood_words; i += team) wood[i] = 0u;
    if (lt == 0) {
      misc[0] = -1;
      misc[1] = 0;
      misc[2] = 0;
    }
  }
  tm.sync();
  // ---------------------------------------------------------- phase 1
  if (valid) {
    const cd kair = wavenumber(cd{1.0, 0.0}, wln);
    for (int u = lt; u < npw; u += team) {
      double al, be;
      order_ab(p.world_1d(), p.dy(), p.px()[u], p.py()[u], a0, b0, al, be);
      const cd kz = csqrt_p(kz_arg(kair, al, be));
      if (cis_zero(kz)) atomicOr(&wood[L >> 5], 1u << (L & 31));
      keys[u] = sort_key(-1 * kz.x + kz.y);
      if (kz.y == 0.0) atomicAdd(&nprop[L], 1);
    }
  }
  tm.sync();
  // ---------------------------------------------------------- phase 2
  const bool wood_air = valid && ((wood[L >> 5] >> (L & 31)) & 1u);
  if (tm.any(wood_air)) {
    if (wood_air && lt == 0) nprop[L] = 0;
    tm.sync();
    if (wood_air) {
      const cd kair = wavenumber(cd{1.0, 0.0}, wln);
      for (int u = lt; u < npw; u += team) {
        double al, be;
        order_ab(p.world_1d(), p.dy(), p.px()[u], p.py()[u], sa0, sb0, al, be);
        const cd kz = csqrt_p(kz_arg(kair, al, be));
        keys[u] = sort_key(-1 * kz.x + kz.y);
        if (kz.y == 0.0) atomicAdd(&nprop[L], 1);
      }
    }
    tm.sync();
  }
  // ---------------------------------------------------------- phase 3
  if (valid) {
    int32_t *so = p.sort_order();
    for (int u = lt; u < npw; u += team) {
      const unsigned long long ku = keys[u];
      int r = 0;
#pragma unroll 4
      for (int v = 0; v < npw; ++v) {
        const unsigned long long kv = keys[v];
        r += (kv < ku) | ((kv == ku) & (v < u));
      }
      rank[u] = r;
      const int pxu = p.px()[u], pyu = p.py()[u];
      const bool zero_order = (pxu == 0) && (p.world_1d() || pyu == 0);
      if (zero_order) misc[0] = r;
      if (so) so[r] = u;
      double al, be;
      order_ab(p.world_1d(), p.dy(), pxu, pyu, a0, b0, al, be);
      const double al2 = __dmul_rn(al, al), be2 = __dmul_rn(be, be);
      if (sqrt_is_real(kz_arg_sq(lay[0].kk, al2, be2))) atomicAdd(&nprop[0], 1);
      if (sqrt_is_real(kz_arg_sq(lay[L - 1].kk, al2, be2))) atomicAdd(&nprop[L - 1], 1);
      // Wood check of every layer: k_z == 0 exactly iff its argument is 0
      for (int l = 0; l < L; ++l) {
        const cd arg = kz_arg_sq(lay[l].kk, al2, be2);
        if (arg.x == 0.0 && arg.y == 0.0) {
          atomicOr(&wood[l >> 5], 1u << (l & 31));
          misc[1] = 1;
        }
      }
    }
  }
  tm.sync();
  // ---------------------------------------------------------- phase 4
  const bool layer_wood = valid && misc[1] != 0;
  if (valid && !layer_wood) {
    const int spec = misc[0];
    const int np_air = nprop[L], np_in = nprop[L - 1], np_out = nprop[0];
    for (int u = lt; u < npw; u += team)
      solve_order(p, u, rank[u], spec, lay, hsm, wood, wood_air, a0, b0, sa0, sb0, wln, np_air,
                  np_in, np_out, acc, nprop, count, ws_smem);
  }
  // ---------------------------------------------------------- phase 5
  if (tm.any(layer_wood)) {
    // recount substrate / superstrate with the scaled k_parallel where marked
    if (layer_wood && lt == 0) {
      nprop[0] = 0;
      nprop[L - 1] = 0;
    }
    tm.sync();
    if (layer_wood) {
      for (int u = lt; u < npw; u += team) {
        for (int t = 0; t < 2; ++t) {
          const int l = t ? L - 1 : 0;
          const bool wl_l = (wood[l >> 5] >> (l & 31)) & 1u;
          double al, be;
          order_ab(p.world_1d(), p.dy(), p.px()[u], p.py()[u], wl_l ? sa0 : a0, wl_l ? sb0 : b0,
                   al, be);
          if (sqrt_is_real(kz_arg(lay[l].k, al, be))) atomicAdd(&nprop[l], 1);
        }
      }
    }
    tm.sync();
    if (layer_wood) {
      const int spec = misc[0];
      const int np_air = nprop[L], np_in = nprop[L - 1], np_out = nprop[0];
      for (int u = lt; u < npw; u += team)
        solve_order(p, u, rank[u], spec, lay, hsm, wood, wood_air, a0, b0, sa0, sb0, wln, np_air,
                    np_in, np_out, acc, nprop, count, ws_smem);
    }
  }
  tm.sync();
  // ---------------------------------------------------------- phase 6
  // a_list / t_list / r_list (backend/stack.py:368-426), one entry per
  // thread of the team; the flags word once every entry is checked
  int nprop_in0 = 0, nprop_out0 = 0;
  if (valid) {
    const int np_in = nprop[L - 1], np_out = nprop[0];
    nprop_in0 = np_in;
    nprop_out0 = np_out;
    const double df0 = acc[0].x, up0 = acc[L].x, dsub = acc[L - 1].x;
    // |down_fluxes[i]| with down_fluxes = [df0, gap_1..gap_{L-2}, dsub]
    auto dfa = [&](int i) -> double {
      if (i == 0) return fabs(df0);
      if (i == L - 1) return fabs(dsub);
      return hypot(acc[i].x, acc[i].y);
    };
    double *al = p.a_list();
    double *tl = p.t_list();
    bool fin = true;
    for (int i = lt; i < L - 1; i += team) {
      double a = 0.0, t = 0.0;
      if (np_out != 0) {
        a = (i < L - 2) ? fabs(dfa(i + 1) - dfa(i + 2)) : fabs(df0 - dsub - up0);
        t = (i < L - 2) ? fabs(dfa(i + 2) / dfa(i)) : fabs(dsub / df0);
      }
      al[i] = a;
      tl[i] = t;
      fin = fin && isfinite(a) && isfinite(t);
    }
    if (lt == 0) {
      const double rr = (np_out != 0) ? fabs(up0 / df0) : 0.0;
      *p.r_list() = rr;
      fin = fin && isfinite(rr);
      if (p.specular()) *p.specular() = misc[0];
    }
    if (!fin) atomicOr(&misc[2], 1);
    if (int32_t *np = p.num_prop())
      for (int i = lt; i <= L; i += team) np[i] = nprop[i];
    if (double *fo = p.fluxes()) {
      for (int i = lt; i <= L; i += team) {
        fo[2 * i] = acc[i].x;
        fo[2 * i + 1] = acc[i].y;
      }
    }
  }
  tm.sync();
  // only misc[2] is read after the barrier, by the thread that resets it in
  // phase 0 of the team's next point
  if (valid && lt == 0) {
    uint32_t flags = 0;
    if (wood_air) flags |= EMU_PT_WOOD_AIR;
    if (layer_wood) flags |= EMU_PT_WOOD_LAYER;
    if (nprop_out0 == 0) flags |= EMU_PT_NO_PROP_SUB;
    if (nprop_in0 == 0) flags |= EMU_PT_NO_PROP_SUP;
    if (misc[2]) flags |= EMU_PT_NONFINITE;
    *p.flags() = flags;
  }
}

}  // namespace emu
