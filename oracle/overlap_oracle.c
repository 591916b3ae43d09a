/*
 * CPU oracle for the Bloch-mode / plane-wave overlap integrals and the
 * Bloch-mode normalisation of EMUstack.  TEST INFRASTRUCTURE ONLY: used by
 * tests/ and bench.py's CPU baseline as the checker, never by the product.
 *
 * A plain-C restatement (the Fortran of the reference cannot be compiled
 * here: there is no Fortran compiler) of, relative to the EMUstack tree:
 *   quad_triangle      backend/fortran/quad_triangle.f:42-145
 *                      (16-point rule of Lyness & Jespersen, J. Inst. Math.
 *                      Appl. 15 (1975) 19-32)
 *   phi2_2d_mat(_J)    backend/fortran/phi2_2d_mat.f:9-43,
 *                      backend/fortran/phi2_2d_mat_J.f:9-34   (P2 basis)
 *   phi3_2d_mat        backend/fortran/phi3_2d_mat.f:9-65      (P3 basis)
 *   jacobian_p1_2d     backend/fortran/jacobian_p1_2d.f:33-133 (affine map)
 *   pw_ordering        backend/fortran/pw_ordering.f:2-91
 *   J_overlap          backend/fortran/J_overlap.f:92-198
 *   J_dagger_overlap   backend/fortran/J_dagger_overlap.f:93-199
 *   orthogonal         backend/fortran/orthogonal.f:75-301
 *   normalisation      backend/fortran/normalisation.f:15-31
 *
 * Layouts follow the reference arrays in memory (Fortran column-major seen
 * as C row-major with the indices reversed):
 *   x          [npt][2]           coordinates (unit cell)
 *   table_nod  [nel][6]           1-based node numbers
 *   type_el    [nel]              1-based material index
 *   sol        [nel][nval][13][3] complex (re, im interleaved) mode fields
 *   J          [2 npw][nval]      J_E rows then J_K rows (row-major)
 *   J_dag      [nval][2 npw]
 * Element curvature: curved_elem_tri (backend/fortran/curved_elem_tri.f:62)
 * always returns "straight", so every element uses the affine map.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

static const double PI_F = 3.141592653589793;

/* ----------------------------------------------------- quadrature */
void ora_quad_triangle(double *wq, double *xq, double *yq) {
  const double wbar = 1.443156076777862e-1 / 2.0;
  const double w1 = 2.852749028018549e-1 / 6.0;
  const double w2 = 9.737549286959440e-2 / 6.0;
  const double w3 = 3.096521116041552e-1 / 6.0;
  const double w4 = 1.633818850466092e-1 / 12.0;
  const double cbar = 1.0 / 3.0;
  const double a1 = 4.592925882927229e-1, b1 = 8.141482341455413e-2;
  const double a2 = 5.054722831703103e-2, b2 = 8.989055433659379e-1;
  const double a3 = 1.705693077517601e-1, b3 = 6.588613844964797e-1;
  const double a4 = 7.284923929554041e-1, b4 = 2.63112829634638689e-1, c4 = 8.394777409957211e-3;
  double X[16] = {cbar, a1, a1, b1, a2, a2, b2, a3, a3, b3, a4, b4, b4, c4, c4, a4};
  double Y[16] = {cbar, a1, b1, a1, a2, b2, a2, a3, b3, a3, b4, a4, c4, b4, a4, c4};
  double W[16] = {wbar, w1, w1, w1, w2, w2, w2, w3, w3, w3, w4, w4, w4, w4, w4, w4};
  for (int i = 0; i < 16; ++i) {
    xq[i] = X[i];
    yq[i] = Y[i];
    wq[i] = W[i];
  }
}

/* ----------------------------------------------------- basis functions */
void ora_phi2(double x0, double y0, double *phi) {
  phi[0] = (-1 + x0 + y0) * (-1 + 2 * x0 + 2 * y0);
  phi[1] = x0 * (-1 + 2 * x0);
  phi[2] = y0 * (-1 + 2 * y0);
  phi[3] = -4 * x0 * (-1 + x0 + y0);
  phi[4] = 4 * x0 * y0;
  phi[5] = -4 * y0 * (-1 + x0 + y0);
}

/* gradients of the 10 P3 basis functions on the reference triangle, [2][10] */
void ora_phi3_grad(double x0, double y0, double g[2][10]) {
  double t = (-11 - 27 * x0 * x0 + x0 * (36 - 54 * y0) + 36 * y0 - 27 * y0 * y0) / 2.;
  g[0][0] = t;
  g[1][0] = t;
  g[0][1] = 1 - 9 * x0 + (27 * x0 * x0) / 2.;
  g[1][1] = 0;
  g[0][2] = 0;
  g[1][2] = 1 - 9 * y0 + (27 * y0 * y0) / 2.;
  g[0][3] = (9 * (2 + 9 * x0 * x0 - 5 * y0 + 3 * y0 * y0 + 2 * x0 * (-5 + 6 * y0))) / 2.;
  g[1][3] = (9 * x0 * (-5 + 6 * x0 + 6 * y0)) / 2.;
  g[0][4] = (-9 * (1 + 9 * x0 * x0 - y0 + x0 * (-8 + 6 * y0))) / 2.;
  g[1][4] = (-9 * x0 * (-1 + 3 * x0)) / 2.;
  g[0][5] = (9 * (-1 + 6 * x0) * y0) / 2.;
  g[1][5] = (9 * x0 * (-1 + 3 * x0)) / 2.;
  g[0][6] = (9 * y0 * (-1 + 3 * y0)) / 2.;
  g[1][6] = (9 * x0 * (-1 + 6 * y0)) / 2.;
  g[0][7] = (-9 * y0 * (-1 + 3 * y0)) / 2.;
  g[1][7] = (-9 * (1 - 8 * y0 + 9 * y0 * y0 + x0 * (-1 + 6 * y0))) / 2.;
  g[0][8] = (9 * y0 * (-5 + 6 * x0 + 6 * y0)) / 2.;
  g[1][8] = (9 * (2 + 3 * x0 * x0 - 10 * y0 + 9 * y0 * y0 + x0 * (-5 + 12 * y0))) / 2.;
  g[0][9] = -27 * y0 * (-1 + 2 * x0 + y0);
  g[1][9] = -27 * x0 * (-1 + x0 + 2 * y0);
}

/* Affine map of an element: x_g = B xi + x_1, B columns = (x2-x1, x3-x1);
 * T = B^-1; returns det(B) (the LU-based determinant of jacobian_p1_2d). */
static double jac_p1(const double xel[6][2], double xi0, double xi1, double *xg, double T[2][2]) {
  const double B00 = xel[1][0] - xel[0][0], B01 = xel[2][0] - xel[0][0];
  const double B10 = xel[1][1] - xel[0][1], B11 = xel[2][1] - xel[0][1];
  xg[0] = xel[0][0] + B00 * xi0 + B01 * xi1;
  xg[1] = xel[0][1] + B10 * xi0 + B11 * xi1;
  const double det = B00 * B11 - B01 * B10;
  T[0][0] = B11 / det;
  T[0][1] = -B01 / det;
  T[1][0] = -B10 / det;
  T[1][1] = B00 / det;
  return det;
}

static void element_nodes(const double *x, const int64_t *table_nod, long iel, double xel[6][2]) {
  for (int k = 0; k < 6; ++k) {
    const int64_t g = table_nod[iel * 6 + k] - 1;
    xel[k][0] = x[2 * g];
    xel[k][1] = x[2 * g + 1];
  }
}

/* ----------------------------------------------------- pw ordering */
/* index_pw_inv (0-based): sorted position of each plane wave, by
 * -Re(kz^2) ascending with kz = sqrt(k0^2 - alpha^2 - beta^2)
 * (pw_ordering.f:54-78, key of z_indexx.f:26-28).  Ties keep the
 * generation order (the reference's quicksort leaves them unspecified). */
int ora_pw_ordering(int ordre_ls, double d, double dy, const double *bloch, double k0,
                    int32_t *index_pw_inv, int32_t *px_out, int32_t *py_out) {
  const double vkx = 2.0 * PI_F / d, vky = 2.0 * PI_F / dy;
  const double mx = d > dy ? d : dy;
  int n = 0;
  double *key = (double *)malloc(sizeof(double) * (2 * ordre_ls + 1) * (2 * ordre_ls + 1));
  for (int px = -ordre_ls; px <= ordre_ls; ++px)
    for (int py = -ordre_ls; py <= ordre_ls; ++py) {
      const double a = (double)px / d, b = (double)py / dy, r = (double)ordre_ls / mx;
      if (a * a + b * b <= r * r) {
        const double alpha = bloch[0] + vkx * px, beta = bloch[1] + vky * py;
        zc z = k0 * k0 - alpha * alpha - beta * beta;
        zc bz = csqrt(z);
        key[n] = -creal(bz * bz);
        if (px_out) px_out[n] = px;
        if (py_out) py_out[n] = py;
        ++n;
      }
    }
  for (int s = 0; s < n; ++s) {
    int r = 0;
    for (int v = 0; v < n; ++v) r += (key[v] < key[s]) || (key[v] == key[s] && v < s);
    index_pw_inv[s] = r;
  }
  free(key);
  return n;
}

/* ----------------------------------------------------- J and J^dagger */
/* sign = -1: J_overlap (exp(-i k.x)), output J [2npw][nval];
 * sign = +1: J_dagger_overlap (exp(+i k.x)), output Jd [nval][2npw]. */
static void overlap(int sign, long nval, long nel, const double *x, const int64_t *table_nod,
                    const zc *sol, double d, double dy, const double *bloch,
                    const int32_t *index_pw_inv, int ordre_ls, int npw, zc *out) {
  double wq[16], xq[16], yq[16];
  ora_quad_triangle(wq, xq, yq);
  const double vkx = 2.0 * PI_F / d, vky = 2.0 * PI_F / dy;
  const double mx = d > dy ? d : dy;
  zc *OK = (zc *)calloc((size_t)npw * nval, sizeof(zc));
  zc *OE = (zc *)calloc((size_t)npw * nval, sizeof(zc));
  zc *RK = (zc *)malloc(sizeof(zc) * npw * 2);
  zc *RE = (zc *)malloc(sizeof(zc) * npw * 2);
  for (long iel = 0; iel < nel; ++iel) {
    double xel[6][2];
    element_nodes(x, table_nod, iel, xel);
    for (int iq = 0; iq < 16; ++iq) {
      double phi[6], xg[2], T[2][2];
      ora_phi2(xq[iq], yq[iq], phi);
      const double det = jac_p1(xel, xq[iq], yq[iq], xg, T);
      int s = 0;
      for (int px = -ordre_ls; px <= ordre_ls; ++px)
        for (int py = -ordre_ls; py <= ordre_ls; ++py) {
          const double a = (double)px / d, b = (double)py / dy, r = (double)ordre_ls / mx;
          if (a * a + b * b <= r * r) {
            const double alpha = bloch[0] + vkx * px, beta = bloch[1] + vky * py;
            const double norm = 1.0 / sqrt(alpha * alpha + beta * beta);
            const double rt = alpha * xg[0] + beta * xg[1];
            const zc ve = cexp(sign * I * rt) * norm;
            const int s2 = index_pw_inv[s];
            RK[2 * s2] = alpha * ve;
            RK[2 * s2 + 1] = beta * ve;
            RE[2 * s2] = beta * ve;
            RE[2 * s2 + 1] = -alpha * ve;
            ++s;
          }
        }
      const double c1 = wq[iq] * fabs(det);
      for (int s = 0; s < npw; ++s) {
        for (long n = 0; n < nval; ++n) {
          zc vx = 0, vy = 0;
          const zc *se = sol + ((size_t)iel * nval + n) * 39;
          for (int k = 0; k < 6; ++k) {
            vx += se[k * 3 + 0] * phi[k];
            vy += se[k * 3 + 1] * phi[k];
          }
          OK[(size_t)s * nval + n] += c1 * (vx * RK[2 * s] + vy * RK[2 * s + 1]);
          OE[(size_t)s * nval + n] += c1 * (vx * RE[2 * s] + vy * RE[2 * s + 1]);
        }
      }
    }
  }
  for (int t = 0; t < 2 * npw; ++t)
    for (long n = 0; n < nval; ++n) {
      const zc v = (t < npw) ? OE[(size_t)t * nval + n] : OK[(size_t)(t - npw) * nval + n];
      if (sign < 0)
        out[(size_t)t * nval + n] = v;
      else
        out[(size_t)n * 2 * npw + t] = v;
    }
  free(OK);
  free(OE);
  free(RK);
  free(RE);
}

void ora_J_overlap(long nval, long nel, const double *x, const int64_t *table_nod, const double *sol,
                   double d, double dy, const double *bloch, const int32_t *index_pw_inv,
                   int ordre_ls, int npw, double *J) {
  overlap(-1, nval, nel, x, table_nod, (const zc *)sol, d, dy, bloch, index_pw_inv, ordre_ls, npw,
          (zc *)J);
}

void ora_J_dagger_overlap(long nval, long nel, const double *x, const int64_t *table_nod,
                          const double *sol, double d, double dy, const double *bloch,
                          const int32_t *index_pw_inv, int ordre_ls, int npw, double *Jd) {
  overlap(+1, nval, nel, x, table_nod, (const zc *)sol, d, dy, bloch, index_pw_inv, ordre_ls, npw,
          (zc *)Jd);
}

/* ----------------------------------------------------- orthogonality */
/* mat_overlap (ival adjoint, jval prime) [nval][nval] (orthogonal.f:84-248). */
static void overlap_matrix(long nval, long nel, const double *x, const int64_t *table_nod,
                           const int64_t *type_el, const zc *pp, const zc *beta1, const zc *sol1,
                           const zc *sol2, double k0, zc *ovl) {
  double wq[16], xq[16], yq[16];
  ora_quad_triangle(wq, xq, yq);
  memset(ovl, 0, sizeof(zc) * nval * nval);
  for (long iel = 0; iel < nel; ++iel) {
    double xel[6][2];
    element_nodes(x, table_nod, iel, xel);
    zc ms[12][22];
    memset(ms, 0, sizeof(ms));
    const zc ppe = pp[type_el[iel] - 1];
    for (int iq = 0; iq < 16; ++iq) {
      double phi2[6], g30[2][10], g3[2][10], xg[2], T[2][2];
      ora_phi2(xq[iq], yq[iq], phi2);
      ora_phi3_grad(xq[iq], yq[iq], g30);
      const double det = jac_p1(xel, xq[iq], yq[iq], xg, T);
      for (int j = 0; j < 10; ++j)
        for (int r = 0; r < 2; ++r) g3[r][j] = T[0][r] * g30[0][j] + T[1][r] * g30[1][j];
      const zc coeff = wq[iq] * fabs(det) * ppe;
      for (int it = 0; it < 6; ++it)
        for (int ie = 0; ie < 2; ++ie) {
          const int ip = ie + 2 * it;
          for (int jt = 0; jt < 6; ++jt)
            for (int je = 0; je < 2; ++je) {
              const int jp = je + 2 * jt;
              const double dot = (ie == je) ? phi2[it] * phi2[jt] : 0.0;
              ms[ip][jp] += coeff * dot / k0;
            }
          for (int jt = 0; jt < 10; ++jt) {
            const double dot = phi2[it] * (-g3[ie][jt]);
            ms[ip][jt + 12] += coeff * dot / k0;
          }
        }
    }
    for (long iv = 0; iv < nval; ++iv) {
      const zc *s2 = sol2 + ((size_t)iel * nval + iv) * 39;
      zc se2[12];
      for (int i = 0; i < 6; ++i)
        for (int c = 0; c < 2; ++c) se2[c + 2 * i] = s2[i * 3 + c];
      for (long jv = 0; jv < nval; ++jv) {
        const zc *s1 = sol1 + ((size_t)iel * nval + jv) * 39;
        const zc b1 = beta1[jv];
        zc se1[22];
        for (int i = 0; i < 6; ++i)
          for (int c = 0; c < 2; ++c) se1[c + 2 * i] = s1[i * 3 + c] * b1;
        for (int i = 0; i < 3; ++i) se1[12 + i] = s1[i * 3 + 2] * b1;
        for (int i = 6; i < 13; ++i) se1[i + 9] = s1[i * 3 + 2] * b1;
        zc acc = 0;
        for (int i = 0; i < 12; ++i) {
          zc v = 0;
          for (int j = 0; j < 22; ++j) v += se1[j] * ms[i][j];
          acc += v * se2[i];
        }
        ovl[(size_t)iv * nval + jv] += acc;
      }
    }
  }
}

/* orthogonal + normalisation: reorders mis-ordered complex-conjugate pairs
 * of the adjoint modes (swapping sol2 modes and beta2), recomputes the
 * overlap matrix, then scales each adjoint mode by 1/sqrt(ovl(i,i))^2.
 * Returns the number of pair warnings; ovl receives the recomputed matrix;
 * perm[i] = adjoint mode now at position i; scale[i] = the factor applied. */
int ora_orthogonal_normalise(long nval, long nel, const double *x, const int64_t *table_nod,
                             const int64_t *type_el, const double *pp, const double *beta1,
                             double *beta2, const double *sol1, double *sol2, double k0,
                             double *ovl_out, int32_t *perm, double *scale) {
  zc *ovl = (zc *)ovl_out;
  zc *s2 = (zc *)sol2;
  zc *b2 = (zc *)beta2;
  int warn = 0;
  overlap_matrix(nval, nel, x, table_nod, type_el, (const zc *)pp, (const zc *)beta1,
                 (const zc *)sol1, s2, k0, ovl);
  for (long i = 0; i < nval; ++i) perm[i] = (int32_t)i;
  long j = 0;
  int skip = 0;
  int swapped = 0;
  while (j < nval) {
    if (cabs(ovl[(size_t)j * nval + j]) > 1e-7) {
      ++j;
    } else if (skip == 0) {
      if (j == nval - 1) ++warn;
      for (long j2 = j + 1; j2 < nval; ++j2) {
        if (cabs(ovl[(size_t)j2 * nval + j]) > 1e-7) {
          zc t = b2[j];
          b2[j] = b2[j2];
          b2[j2] = t;
          int32_t tp = perm[j];
          perm[j] = perm[j2];
          perm[j2] = tp;
          for (long e = 0; e < nel; ++e)
            for (int k = 0; k < 39; ++k) {
              zc a = s2[((size_t)e * nval + j) * 39 + k];
              s2[((size_t)e * nval + j) * 39 + k] = s2[((size_t)e * nval + j2) * 39 + k];
              s2[((size_t)e * nval + j2) * 39 + k] = a;
            }
          swapped = 1;
        }
      }
      skip = 1;
      ++j;
    } else {
      skip = 0;
      ++j;
    }
  }
  if (swapped)
    overlap_matrix(nval, nel, x, table_nod, type_el, (const zc *)pp, (const zc *)beta1,
                   (const zc *)sol1, s2, k0, ovl);
  /* normalisation.f:15-31 */
  zc *sc = (zc *)scale;
  for (long i = 0; i < nval; ++i) {
    const zc z1 = csqrt(ovl[(size_t)i * nval + i]);
    if (cabs(z1) > 1e-8) {
      sc[i] = 1.0 / (z1 * z1);
    } else {
      sc[i] = 1.0;
    }
  }
  for (long e = 0; e < nel; ++e)
    for (long i = 0; i < nval; ++i)
      for (int k = 0; k < 39; ++k) s2[((size_t)e * nval + i) * 39 + k] *= sc[i];
  return warn;
}
