// Overlap integrals of 1D-grating layers (rows a11 / a12 for
// periodicity '1D_array'): J and J_dag between the P2 (Ex) / P3 (Ey) Bloch
// modes of a 1D FEM mesh and the plane waves exp(-+ i alpha x), the
// plane-wave order of the 1D set, and the embedding of both matrices into the
// 2D order set of the same maximum order.
//
// Reference (paths relative to the EMUstack source tree):
//   J_overlap_1d         backend/fortran/J_overlap_1d.f:8-225
//   J_dagger_overlap_1d  backend/fortran/J_dagger_overlap_1d.f:1-225
//   element integrals    backend/fortran/vector_p2_exp_1d.f, vector_p3_exp_1d.f
//   plane-wave order     backend/fortran/pw_ordering_1d.f:1-80, z_indexx.f
//   2D embedding         backend/fortran/pw_matrix_1d_to_2d.f:1-200
//   call sequence        backend/fortran/py_calc_modes_1d.f:583-620,
//                        backend/mode_calcs.py:323-355
//
// Element integrals.  On an element [xmin, xmax] with h = xmax - xmin and
// x = xmin + h t, int L_i(x) exp(i b x) dx = h exp(i b xmin) sum_k c_ik M_k,
// where l_i(t) = sum_k c_ik t^k is the Lagrange basis polynomial of the
// element's nodes in t (P2: t = 0, 1, 1/2; P3: t = 0, 1, 1/3, 2/3) and
// M_k = int_0^1 t^k exp(i theta t) dt, theta = b h.  M_k comes from its power
// series sum_j (i theta)^j / (j! (k + j + 1)) for |theta| <= 1 and from the
// recurrence M_0 = (e - 1)/(i theta), M_k = (e - k M_{k-1})/(i theta),
// e = exp(i theta), above (its error grows at most as k!/|theta|^k <= 6).
// The reference evaluates the same integrals in closed form with a Taylor
// switch at |alpha h| = 1e-3; both are the exact integral, to rounding.
// The plane waves of J_dag are the complex conjugates (+i alpha x) and the
// basis is real, so J_dag's element integrals are the conjugates of J's.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "emu_cplx.cuh"
#include "emu_internal.h"

namespace {

constexpr double kPi1 = 3.141592653589793;
constexpr int kChunk = 128;   // elements staged in shared memory at a time
constexpr int kThreads = 128; // Bloch modes per pass of a block

// ----------------------------------------------------------------- host
// Numerical Recipes' indexx (W. H. Press et al., Numerical Recipes, 2nd ed.,
// section 8.4): ascending index sort by median-of-three quicksort with
// straight insertion for sub-arrays of fewer than 7 elements, and an explicit
// stack.  The reference ranks plane waves with this algorithm (z_indexx.f);
// the order it gives to tied keys is part of its result, so the same
// partitioning steps are followed here.  Returns 0-based indices.
bool nr_indexx(int n, const double *key, std::vector<int> &out) {
  const int M = 7, NSTACK = 50;
  std::vector<long long> indx(n + 1);
  long long istack[NSTACK + 1];
  for (int j = 1; j <= n; ++j) indx[j] = j;
  auto a0 = [&](long long p) { return key[indx[p] - 1]; };
  auto swp = [&](long long p, long long q) {
    const long long t = indx[p];
    indx[p] = indx[q];
    indx[q] = t;
  };
  int jstack = 0;
  long long l = 1, ir = n;
  for (;;) {
    if (ir - l < M) {
      for (long long j = l + 1; j <= ir; ++j) {
        const long long indxt = indx[j];
        const double a = key[indxt - 1];
        long long i = j - 1;
        for (; i >= l; --i) {
          if (key[indx[i] - 1] <= a) break;
          indx[i + 1] = indx[i];
        }
        indx[i + 1] = indxt;
      }
      if (jstack == 0) break;
      ir = istack[jstack];
      l = istack[jstack - 1];
      jstack -= 2;
    } else {
      const long long k = (l + ir) / 2;
      swp(k, l + 1);
      if (a0(l) > a0(ir)) swp(l, ir);
      if (a0(l + 1) > a0(ir)) swp(l + 1, ir);
      if (a0(l) > a0(l + 1)) swp(l, l + 1);
      long long i = l + 1, j = ir;
      const long long indxt = indx[l + 1];
      const double a = key[indxt - 1];
      for (;;) {
        do ++i; while (a0(i) < a);
        do --j; while (a0(j) > a);
        if (j < i) break;
        swp(i, j);
      }
      indx[l + 1] = indx[j];
      indx[j] = indxt;
      jstack += 2;
      if (jstack > NSTACK) return false;
      if (ir - i + 1 >= j - l) {
        istack[jstack] = ir;
        istack[jstack - 1] = i;
        ir = j - 1;
      } else {
        istack[jstack] = j - 1;
        istack[jstack - 1] = l;
        l = i;
      }
    }
  }
  out.resize(n);
  for (int j = 0; j < n; ++j) out[j] = (int)(indx[j + 1] - 1);
  return true;
}

// Sort key of one plane wave: -Re(kz^2) with kz = sqrt(k0^2 - alpha^2 -
// beta^2) taken as a complex square root and squared in complex arithmetic
// (pw_ordering_1d.f:64-69, z_indexx.f:26-28).  For the real argument z the
// root is (sqrt z, 0) or (0, sqrt -z), so the key is -+ fl(s * s) with
// s = fl(sqrt |z|).
double pw_key(double k0, double alpha, double beta) {
  const double z = (k0 * k0 - alpha * alpha) - beta * beta;
  const double s = std::sqrt(std::fabs(z));
  const double s2 = s * s;
  return z >= 0.0 ? -s2 : s2;
}

// Inverse permutation of the ranking: pos[s] = rank of generation index s.
bool rank_positions(int n, const std::vector<double> &key, int32_t *pos) {
  std::vector<int> idx;
  if (!nr_indexx(n, key.data(), idx)) return false;
  for (int r = 0; r < n; ++r) pos[idx[r]] = r;
  return true;
}

// ---------------------------------------------------------------- device
struct Ov1Args {
  int nval, nel, npt, npw, max_order, npw2d;
  double vk;                    // 2 pi / period_x
  const double *x;              // [npt]
  const int64_t *tn;            // [nel][3], 1-based
  const double *bloch;          // [batch][2]
  const int32_t *pos;           // [batch][npw]
  const int32_t *row2d;         // [batch][npw] or NULL
  const emu_c128 *sol1, *sol2;  // [batch][nel][nval][11] or NULL
  const emu_c128 *scale;        // [batch][nval] mode normalisation or NULL
  const int32_t *perm2;         // [batch][nval] adjoint mode of row n or NULL
  emu_c128 *J, *Jd, *J2, *Jd2;
  int32_t *err;
};

// M_k = int_0^1 t^k exp(i th t) dt, k = 0..3 (see the file comment).
__device__ __forceinline__ void moments4(double th, cd M[4]) {
  if (fabs(th) <= 1.0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) M[k] = cd{0.0, 0.0};
    cd term{1.0, 0.0};
#pragma unroll
    for (int j = 0; j < 22; ++j) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double w = 1.0 / (double)(k + j + 1);
        M[k].x += term.x * w;
        M[k].y += term.y * w;
      }
      const double f = th / (double)(j + 1);
      term = cd{-term.y * f, term.x * f};
    }
  } else {
    double s, c;
    sincos(th, &s, &c);
    const double r = 1.0 / th;
    // (t) / (i th) = (t.y r, -t.x r)
    cd t{c - 1.0, s};
    M[0] = cd{t.y * r, -t.x * r};
#pragma unroll
    for (int k = 1; k < 4; ++k) {
      t = cd{c - k * M[k - 1].x, s - k * M[k - 1].y};
      M[k] = cd{t.y * r, -t.x * r};
    }
  }
}

// Lagrange coefficients c_ik of l_i(t) = sum_k c_ik t^k.
__constant__ double kP2c[3][3] = {{1.0, -3.0, 2.0}, {0.0, -1.0, 2.0}, {0.0, 4.0, -4.0}};
__constant__ double kP3c[4][4] = {{1.0, -5.5, 9.0, -4.5},
                                  {0.0, 1.0, -4.5, 4.5},
                                  {0.0, 9.0, -22.5, 13.5},
                                  {0.0, -4.5, 18.0, -13.5}};

// One block per (order, problem): element integrals of a chunk of elements
// in shared memory, then each thread accumulates J's E and K rows (and
// J_dag's) for one Bloch mode over the chunk.
__global__ void __launch_bounds__(kThreads) overlap1d_kernel(Ov1Args a) {
  __shared__ cd I2s[kChunk][3];
  __shared__ cd I3s[kChunk][4];
  __shared__ int okS[kChunk];
  const int o = blockIdx.x, b = blockIdx.y;
  const int px = o - a.max_order;
  const double bx = a.bloch[2 * (size_t)b], by = a.bloch[2 * (size_t)b + 1];
  const double alpha = bx + a.vk * px;
  // unit transverse vectors of the plane wave (J_overlap_1d.f:146-166)
  double rk0, rk1, re0, re1;
  if (alpha != 0.0 || by != 0.0) {
    const double nrm = 1.0 / sqrt(alpha * alpha + by * by);
    rk0 = alpha * nrm;
    rk1 = by * nrm;
    re0 = by * nrm;
    re1 = -alpha * nrm;
  } else {
    rk0 = 0.0;
    rk1 = 1.0;
    re0 = 1.0;
    re1 = 0.0;
  }
  const size_t fstride = (size_t)a.nel * a.nval * 11;
  const cd *s1 = a.sol1 ? (const cd *)a.sol1 + (size_t)b * fstride : nullptr;
  const cd *s2 = a.sol2 ? (const cd *)a.sol2 + (size_t)b * fstride : nullptr;
  for (int n0 = 0; n0 < a.nval; n0 += kThreads) {
    const int n = n0 + threadIdx.x;
    int n2 = n;
    if (a.perm2 && n < a.nval) {
      n2 = a.perm2[(size_t)b * a.nval + n];
      if (n2 < 0 || n2 >= a.nval) {
        if (a.err) atomicExch(a.err, 1);
        n2 = n;
      }
    }
    cd e1{0, 0}, k1{0, 0}, e2{0, 0}, k2{0, 0};
    for (int c0 = 0; c0 < a.nel; c0 += kChunk) {
      const int cn = min(kChunk, a.nel - c0);
      for (int q = threadIdx.x; q < cn; q += kThreads) {
        const int64_t *t = a.tn + 3 * (size_t)(c0 + q);
        const int64_t g0 = t[0], g1 = t[1];
        const bool ok = g0 >= 1 && g0 <= a.npt && g1 >= 1 && g1 <= a.npt;
        okS[q] = ok;
        if (!ok) {
          if (a.err) atomicExch(a.err, 1);
          continue;
        }
        const double xmin = a.x[g0 - 1], xmax = a.x[g1 - 1];
        const double h = xmax - xmin;
        // plane wave exp(-i alpha x): b = -alpha
        cd M[4];
        moments4(-alpha * h, M);
        double sp, cp;
        sincos(-alpha * xmin, &sp, &cp);
        const cd pre{h * cp, h * sp};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          cd acc{0, 0};
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            acc.x += kP2c[i][k] * M[k].x;
            acc.y += kP2c[i][k] * M[k].y;
          }
          I2s[q][i] = cmul(pre, acc);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          cd acc{0, 0};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            acc.x += kP3c[i][k] * M[k].x;
            acc.y += kP3c[i][k] * M[k].y;
          }
          I3s[q][i] = cmul(pre, acc);
        }
      }
      __syncthreads();
      if (n < a.nval) {
        for (int q = 0; q < cn; ++q) {
          if (!okS[q]) continue;
          const size_t off = ((size_t)(c0 + q) * a.nval + n) * 11;
          if (s1) {
            cd fx{0, 0}, fy{0, 0};
#pragma unroll
            for (int i = 0; i < 3; ++i) fx = cadd(fx, cmul(s1[off + i], I2s[q][i]));
#pragma unroll
            for (int i = 0; i < 4; ++i) fy = cadd(fy, cmul(s1[off + 3 + i], I3s[q][i]));
            e1 = cadd(e1, cadd(cscale(fx, re0), cscale(fy, re1)));
            k1 = cadd(k1, cadd(cscale(fx, rk0), cscale(fy, rk1)));
          }
          if (s2) {
            const size_t off2 = ((size_t)(c0 + q) * a.nval + n2) * 11;
            cd fx{0, 0}, fy{0, 0};
#pragma unroll
            for (int i = 0; i < 3; ++i) fx = cadd(fx, cmul(s2[off2 + i], cconj(I2s[q][i])));
#pragma unroll
            for (int i = 0; i < 4; ++i) fy = cadd(fy, cmul(s2[off2 + 3 + i], cconj(I3s[q][i])));
            e2 = cadd(e2, cadd(cscale(fx, re0), cscale(fy, re1)));
            k2 = cadd(k2, cadd(cscale(fx, rk0), cscale(fy, rk1)));
          }
        }
      }
      __syncthreads();
    }
    if (n >= a.nval) continue;
    if (a.scale) {
      // normalisation_1d.f: prime and adjoint mode n both divided by sqrt(<n|n>)
      const emu_c128 sc = a.scale[(size_t)b * a.nval + n];
      const cd z{sc.re, sc.im};
      e1 = cmul(e1, z);
      k1 = cmul(k1, z);
      e2 = cmul(e2, z);
      k2 = cmul(k2, z);
    }
    const int r = a.pos[(size_t)b * a.npw + o];
    const int P = 2 * a.npw;
    if (s1) {
      cd *J = (cd *)a.J + (size_t)b * P * a.nval;
      J[(size_t)r * a.nval + n] = e1;
      J[(size_t)(r + a.npw) * a.nval + n] = k1;
    }
    if (s2) {
      cd *Jd = (cd *)a.Jd + (size_t)b * a.nval * P;
      Jd[(size_t)n * P + r] = e2;
      Jd[(size_t)n * P + r + a.npw] = k2;
    }
    if (a.row2d) {
      const int r2 = a.row2d[(size_t)b * a.npw + o];
      const int P2 = 2 * a.npw2d;
      if (s1 && a.J2) {
        cd *J2 = (cd *)a.J2 + (size_t)b * P2 * a.nval;
        J2[(size_t)r2 * a.nval + n] = e1;
        J2[(size_t)(r2 + a.npw2d) * a.nval + n] = k1;
      }
      if (s2 && a.Jd2) {
        cd *Jd2 = (cd *)a.Jd2 + (size_t)b * a.nval * P2;
        Jd2[(size_t)n * P2 + r2] = e2;
        Jd2[(size_t)n * P2 + r2 + a.npw2d] = k2;
      }
    }
  }
}

// ------------------------------------------------ 1D mode orthogonality
// Element matrices of the 1D orthogonality integral (orthogonal_1d.f:75-140),
// from the Lagrange coefficients of the element's P2 and P3 bases on t in
// [0, 1]: Mxx = h int l2_i l2_j, Myy = h int l3_i l3_j, Kxy = int l2_i
// (d l3_j / dt) (the derivative's 1/h cancels the h of dx).
struct ElemMats {
  double mxx[3][3], myy[4][4], kxy[3][4];
};

__device__ void reference_element_matrices(ElemMats &m) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) v += kP2c[i][p] * kP2c[j][q] / (double)(p + q + 1);
      m.mxx[i][j] = v;
    }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double v = 0.0;
      for (int p = 0; p < 4; ++p)
        for (int q = 0; q < 4; ++q) v += kP3c[i][p] * kP3c[j][q] / (double)(p + q + 1);
      m.myy[i][j] = v;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) {
      double v = 0.0;
      for (int p = 0; p < 3; ++p)
        for (int q = 1; q < 4; ++q) v += kP2c[i][p] * q * kP3c[j][q] / (double)(p + q);
      m.kxy[i][j] = v;
    }
}

struct Or1Args {
  int nval, nel, npt, n_types;
  const double *x;
  const int64_t *tn, *type_el;
  const emu_c128 *pp;       // [n_types]
  const double *k0;         // [batch]
  const double *bloch;      // [batch][2] (bloch_vec_y enters M_yz)
  const emu_c128 *beta1;    // [batch][nval]
  const emu_c128 *sol1, *sol2;
  const int32_t *perm2;     // [batch][nval] or NULL
  emu_c128 *out;            // diag [batch][nval] or full [batch][nval][nval]
  emu_c128 *scale;          // [batch][nval] or NULL (diagonal pass only)
  int32_t *n_small;         // [batch] or NULL
  int32_t *err;
};

// <adjoint u | prime v> over one element, before the factor beta / k0:
// pp (u_x Mxx v_x + u_y Myy v_y - u_x Kxy v_z - i by u_y Myy v_z)
// (orthogonal_1d.f:75-158; entries 0-2 Ex, 3-6 Ey, 7-10 Ez).
__device__ __forceinline__ cd elem_form(const ElemMats &m, double h, double by, const cd *u,
                                        const cd *v) {
  cd sx{0, 0}, sy{0, 0}, sxz{0, 0}, syz{0, 0};
  for (int i = 0; i < 3; ++i) {
    cd w{0, 0}, wz{0, 0};
    for (int j = 0; j < 3; ++j) w = cadd(w, cscale(v[j], m.mxx[i][j]));
    for (int j = 0; j < 4; ++j) wz = cadd(wz, cscale(v[7 + j], m.kxy[i][j]));
    sx = cadd(sx, cmul(u[i], w));
    sxz = cadd(sxz, cmul(u[i], wz));
  }
  for (int i = 0; i < 4; ++i) {
    cd w{0, 0}, wz{0, 0};
    for (int j = 0; j < 4; ++j) {
      w = cadd(w, cscale(v[3 + j], m.myy[i][j]));
      wz = cadd(wz, cscale(v[7 + j], m.myy[i][j]));
    }
    sy = cadd(sy, cmul(u[3 + i], w));
    syz = cadd(syz, cmul(u[3 + i], wz));
  }
  // h scales the mass matrices, not Kxy
  const cd mass = cscale(cadd(sx, sy), h);
  const cd iby_syz = cscale(cd{-syz.y, syz.x}, by * h);
  return csub(csub(mass, sxz), iby_syz);
}

__device__ __forceinline__ bool elem_span(const Or1Args &a, int el, double &h, cd &pp) {
  const int64_t *t = a.tn + 3 * (size_t)el;
  const int64_t g0 = t[0], g1 = t[1], ty = a.type_el[el];
  if (g0 < 1 || g0 > a.npt || g1 < 1 || g1 > a.npt || ty < 1 || ty > a.n_types) {
    if (a.err) atomicExch(a.err, 1);
    return false;
  }
  h = a.x[g1 - 1] - a.x[g0 - 1];
  pp = cd{a.pp[ty - 1].re, a.pp[ty - 1].im};
  return true;
}

// Diagonal <adjoint m | prime m> beta1(m) / k0 and, with `scale`, the
// normalisation factor 1/sqrt of it (1 where |sqrt| <= 1e-8,
// normalisation_1d.f:18-31).  One thread per mode.
__global__ void ortho1d_diag_kernel(Or1Args a) {
  const int b = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nval) return;
  ElemMats em;
  reference_element_matrices(em);
  int m2 = a.perm2 ? a.perm2[(size_t)b * a.nval + m] : m;
  if (m2 < 0 || m2 >= a.nval) {
    if (a.err) atomicExch(a.err, 1);
    m2 = m;
  }
  const double by = a.bloch[2 * (size_t)b + 1];
  const size_t fs = (size_t)a.nel * a.nval * 11;
  const cd *s1 = (const cd *)a.sol1 + (size_t)b * fs, *s2 = (const cd *)a.sol2 + (size_t)b * fs;
  cd acc{0, 0};
  for (int el = 0; el < a.nel; ++el) {
    double h;
    cd pp;
    if (!elem_span(a, el, h, pp)) continue;
    const cd f = elem_form(em, h, by, s2 + ((size_t)el * a.nval + m2) * 11, s1 + ((size_t)el * a.nval + m) * 11);
    acc = cadd(acc, cmul(pp, f));
  }
  const emu_c128 bt = a.beta1[(size_t)b * a.nval + m];
  const cd d = cscale(cmul(cd{bt.re, bt.im}, acc), 1.0 / a.k0[b]);
  a.out[(size_t)b * a.nval + m] = emu_c128{d.x, d.y};
  if (a.n_small && hypot(d.x, d.y) <= 1e-7) atomicAdd(&a.n_small[b], 1);
  if (a.scale) {
    const cd z = csqrt_p(d);
    cd sc{1.0, 0.0};
    if (hypot(z.x, z.y) > 1e-8) sc = cdiv(cd{1.0, 0.0}, z);
    a.scale[(size_t)b * a.nval + m] = emu_c128{sc.x, sc.y};
  }
}

// Full matrix <adjoint i | prime j> beta1(j) / k0: one block per row i,
// threads over the columns j.
__global__ void ortho1d_full_kernel(Or1Args a) {
  const int b = blockIdx.y, i = blockIdx.x;
  ElemMats em;
  reference_element_matrices(em);
  const double by = a.bloch[2 * (size_t)b + 1];
  const size_t fs = (size_t)a.nel * a.nval * 11;
  const cd *s1 = (const cd *)a.sol1 + (size_t)b * fs, *s2 = (const cd *)a.sol2 + (size_t)b * fs;
  int i2 = a.perm2 ? a.perm2[(size_t)b * a.nval + i] : i;
  if (i2 < 0 || i2 >= a.nval) i2 = i;
  for (int j = threadIdx.x; j < a.nval; j += blockDim.x) {
    cd acc{0, 0};
    for (int el = 0; el < a.nel; ++el) {
      double h;
      cd pp;
      if (!elem_span(a, el, h, pp)) continue;
      const cd f = elem_form(em, h, by, s2 + ((size_t)el * a.nval + i2) * 11, s1 + ((size_t)el * a.nval + j) * 11);
      acc = cadd(acc, cmul(pp, f));
    }
    const emu_c128 bt = a.beta1[(size_t)b * a.nval + j];
    const cd d = cscale(cmul(cd{bt.re, bt.im}, acc), 1.0 / a.k0[b]);
    a.out[((size_t)b * a.nval + i) * a.nval + j] = emu_c128{d.x, d.y};
  }
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" int emu_pw_order_1d(int max_order, double period_x, double bloch_x, double bloch_y,
                               double k0, int32_t *h_index_pw_inv) {
  if (max_order < 0 || !(period_x > 0) || !h_index_pw_inv) return EMU_E_ARG;
  const int n = 2 * max_order + 1;
  const double vk = 2.0 * kPi1 / period_x;
  std::vector<double> key(n);
  for (int s = 0; s < n; ++s) key[s] = pw_key(k0, bloch_x + vk * (s - max_order), bloch_y);
  return rank_positions(n, key, h_index_pw_inv) ? EMU_OK : EMU_E_SHAPE;
}

extern "C" int emu_pw_embed_1d_to_2d(int max_order, double period_x, double bloch_x, double bloch_y,
                                     double k0, int32_t *h_row_2d, int capacity, int *h_npw_2d) {
  if (max_order < 0 || !(period_x > 0) || !h_npw_2d) return EMU_E_ARG;
  const double vk = 2.0 * kPi1 / period_x;
  // the 2D order set of pw_matrix_1d_to_2d.f:74-90: px outer, py inner,
  // (px/d)^2 + (py/d)^2 <= (max_order/max(d, d))^2 with d = period_x
  volatile double rq = (double)max_order / period_x;
  const double r2 = rq * rq;
  std::vector<double> key;
  std::vector<int> gen_of_1d(2 * max_order + 1, -1);
  for (int px = -max_order; px <= max_order; ++px) {
    for (int py = -max_order; py <= max_order; ++py) {
      volatile double ax = (double)px / period_x, ay = (double)py / period_x;
      volatile double sx = ax * ax, sy = ay * ay;
      volatile double lhs = sx + sy;
      if (lhs <= r2) {
        if (py == 0) gen_of_1d[px + max_order] = (int)key.size();
        key.push_back(pw_key(k0, bloch_x + vk * px, bloch_y + vk * py));
      }
    }
  }
  const int n2 = (int)key.size();
  *h_npw_2d = n2;
  if (!h_row_2d) return EMU_OK;
  if (capacity < 2 * max_order + 1) return EMU_E_ARG;
  std::vector<int32_t> pos2(n2);
  if (!rank_positions(n2, key, pos2.data())) return EMU_E_SHAPE;
  for (int o = 0; o < 2 * max_order + 1; ++o) {
    if (gen_of_1d[o] < 0) return EMU_E_SHAPE;
    h_row_2d[o] = pos2[gen_of_1d[o]];
  }
  return EMU_OK;
}

extern "C" int emu_overlap1d_batch(const EmuOverlap1D *p, void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->batch < 0 || p->nval < 1 || p->nel < 1 || p->npt < 2 || p->max_order < 0 ||
      p->max_order > 1000)
    return EMU_E_SHAPE;
  if (!(p->period_x > 0) || !p->d_x || !p->d_table_nod || !p->d_bloch || !p->d_index_pw_inv)
    return EMU_E_ARG;
  if (!p->d_sol1 && !p->d_sol2) return EMU_E_ARG;
  if ((p->d_sol1 && !p->d_J) || (p->d_sol2 && !p->d_J_dag)) return EMU_E_ARG;
  if (p->d_row_2d && (p->npw_2d < 2 * p->max_order + 1 || (p->d_sol1 && !p->d_J_2d) ||
                      (p->d_sol2 && !p->d_J_dag_2d)))
    return EMU_E_ARG;
  if (p->batch == 0) return EMU_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int npw = 2 * p->max_order + 1;
  if (p->d_row_2d) {
    // the 2D matrices are zero outside the rows of the (px, 0) orders
    const size_t m = (size_t)p->batch * 2 * p->npw_2d * p->nval * sizeof(emu_c128);
    if (p->d_sol1 && cudaMemsetAsync(p->d_J_2d, 0, m, s) != cudaSuccess) return EMU_E_CUDA;
    if (p->d_sol2 && cudaMemsetAsync(p->d_J_dag_2d, 0, m, s) != cudaSuccess) return EMU_E_CUDA;
  }
  Ov1Args a;
  a.nval = p->nval;
  a.nel = p->nel;
  a.npt = p->npt;
  a.npw = npw;
  a.max_order = p->max_order;
  a.npw2d = p->npw_2d;
  a.vk = 2.0 * kPi1 / p->period_x;
  a.x = p->d_x;
  a.tn = p->d_table_nod;
  a.bloch = p->d_bloch;
  a.pos = p->d_index_pw_inv;
  a.row2d = p->d_row_2d;
  a.sol1 = p->d_sol1;
  a.sol2 = p->d_sol2;
  a.scale = p->d_scale;
  a.perm2 = p->d_perm2;
  a.J = p->d_J;
  a.Jd = p->d_J_dag;
  a.J2 = p->d_J_2d;
  a.Jd2 = p->d_J_dag_2d;
  a.err = p->d_error;
  const dim3 grid(npw, p->batch);
  overlap1d_kernel<<<grid, kThreads, 0, s>>>(a);
  emu::note_launch();
  return emu::check_launch();
}

extern "C" int emu_mode_overlap_1d(const EmuNormalise1D *p, int full, void *stream) {
  if (!p) return EMU_E_ARG;
  if (p->batch < 0 || p->nval < 1 || p->nel < 1 || p->npt < 2 || p->n_types < 1) return EMU_E_SHAPE;
  if (!p->d_x || !p->d_table_nod || !p->d_type_el || !p->d_pp || !p->d_k0 || !p->d_bloch ||
      !p->d_beta1 || !p->d_sol1 || !p->d_sol2 || !p->d_out)
    return EMU_E_ARG;
  if (p->batch == 0) return EMU_OK;
  cudaStream_t s = (cudaStream_t)stream;
  Or1Args a;
  a.nval = p->nval;
  a.nel = p->nel;
  a.npt = p->npt;
  a.n_types = p->n_types;
  a.x = p->d_x;
  a.tn = p->d_table_nod;
  a.type_el = p->d_type_el;
  a.pp = p->d_pp;
  a.k0 = p->d_k0;
  a.bloch = p->d_bloch;
  a.beta1 = p->d_beta1;
  a.sol1 = p->d_sol1;
  a.sol2 = p->d_sol2;
  a.perm2 = p->d_perm2;
  a.out = p->d_out;
  a.scale = full ? nullptr : p->d_scale;
  a.n_small = full ? nullptr : p->d_n_small;
  a.err = p->d_error;
  if (full) {
    ortho1d_full_kernel<<<dim3(p->nval, p->batch), 128, 0, s>>>(a);
  } else {
    if (p->d_n_small && cudaMemsetAsync(p->d_n_small, 0, sizeof(int32_t) * p->batch, s) != cudaSuccess)
      return EMU_E_CUDA;
    ortho1d_diag_kernel<<<dim3((p->nval + 127) / 128, p->batch), 128, 0, s>>>(a);
  }
  emu::note_launch();
  return emu::check_launch();
}

// Order of Bloch modes after the eigen-solve (py_calc_modes.f:683): z_indexx
// on the key -Re(beta^2) (z_indexx.f:26-28), 0-based.
extern "C" int emu_fem_mode_order(int n, const emu_c128 *h_beta, int32_t *h_index) {
  if (n < 0) return EMU_E_SHAPE;
  if (n == 0) return EMU_OK;
  if (!h_beta || !h_index) return EMU_E_ARG;
  std::vector<double> key(n);
  for (int i = 0; i < n; ++i) key[i] = -(h_beta[i].re * h_beta[i].re - h_beta[i].im * h_beta[i].im);
  std::vector<int> idx;
  if (!nr_indexx(n, key.data(), idx)) return EMU_E_SHAPE;
  for (int i = 0; i < n; ++i) h_index[i] = idx[i];
  return EMU_OK;
}
