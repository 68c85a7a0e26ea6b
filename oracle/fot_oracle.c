/*
 * fot_oracle.c -- CPU oracle for the indirect-increment loops.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see fot_oracle.h).  Compiled with
 * -O2 -ffp-contract=off so that no multiply-add is fused and every operation
 * rounds as written, in the reference's order.
 */
#include "fot_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Per-cell increment functions.  Each computes the increments of one cell   */
/* exactly as the reference's StepSeq + user functor, then adds them to the  */
/* target rows slot by slot.                                                 */
/* ------------------------------------------------------------------------ */

/* res_calc user functor, res_calc_func.hpp:9-60 (float literals 1.0f, 0.5f
 * promote to double). */
static void res_calc_func(const double *x1, const double *x2, const double *q1,
                          const double *q2, const double *adt1,
                          const double *adt2, double *res1, double *res2,
                          uint32_t xs, uint32_t qs) {
  const double gm1 = 0.4, eps = 0.05;
  double dx, dy, mu, ri, p1, vol1, p2, vol2, f;
  dx = x1[0 * xs] - x2[0 * xs];
  dy = x1[1 * xs] - x2[1 * xs];
  ri = 1.0 / q1[0 * qs];
  p1 = gm1 * (q1[3 * qs] -
              0.5 * ri * (q1[1 * qs] * q1[1 * qs] + q1[2 * qs] * q1[2 * qs]));
  vol1 = ri * (q1[1 * qs] * dy - q1[2 * qs] * dx);
  ri = 1.0 / q2[0 * qs];
  p2 = gm1 * (q2[3 * qs] -
              0.5 * ri * (q2[1 * qs] * q2[1 * qs] + q2[2 * qs] * q2[2 * qs]));
  vol2 = ri * (q2[1 * qs] * dy - q2[2 * qs] * dx);
  mu = 0.5 * ((*adt1) + (*adt2)) * eps;
  f = 0.5 * (vol1 * q1[0 * qs] + vol2 * q2[0 * qs]) + mu * (q1[0 * qs] - q2[0 * qs]);
  res1[0] = f;
  res2[0] = -f;
  f = 0.5 * (vol1 * q1[1 * qs] + p1 * dy + vol2 * q2[1 * qs] + p2 * dy) +
      mu * (q1[1 * qs] - q2[1 * qs]);
  res1[1] = f;
  res2[1] = -f;
  f = 0.5 * (vol1 * q1[2 * qs] - p1 * dx + vol2 * q2[2 * qs] - p2 * dx) +
      mu * (q1[2 * qs] - q2[2 * qs]);
  res1[2] = f;
  res2[2] = -f;
  f = 0.5 * (vol1 * (q1[3 * qs] + p1) + vol2 * (q2[3 * qs] + p2)) +
      mu * (q1[3 * qs] - q2[3 * qs]);
  res1[3] = f;
  res2[3] = -f;
}

/* mini_aero helpers, mini_aero_utils.hpp:6-373. */
static void ma_primitives(const double *U, double *V) {
  const double gamma = 1.4, Rgas = 287.05;
  double r, u, v, w, T, ri, k, e;
  r = U[0];
  ri = 1.0 / r;
  u = U[1] * ri;
  v = U[2] * ri;
  w = U[3] * ri;
  k = 0.5 * (u * u + v * v + w * w);
  e = U[4] * ri - k;
  T = e * (gamma - 1.0) / Rgas;
  V[0] = r;
  V[1] = u;
  V[2] = v;
  V[3] = w;
  V[4] = T;
}

static double ma_pressure(const double *V) { return V[0] * 287.05 * V[4]; }
static double ma_enthalpy(const double *V) { return 1004.0 * V[4]; }

static void ma_matvec5(const double *A, const double *x, double *y) {
  /* MatVec5(1.0, A, x, 0.0, y): y = y*beta, then y += alpha*A*x in j order */
  for (int i = 0; i < 5; ++i) {
    y[i] *= 0.0;
    for (int j = 0; j < 5; ++j) y[i] += 1.0 * A[5 * i + j] * x[j];
  }
}

static void ma_inviscid(const double *pl, const double *pr, double *flux,
                        const double *n, const double *t, const double *b,
                        uint32_t fs) {
  const double efix_u = 0.1, efix_c = 0.1, gm1 = 0.4;
  const double rho_l = pl[0], u_l = pl[1], v_l = pl[2], w_l = pl[3];
  const double p_l = ma_pressure(pl), h_l = ma_enthalpy(pl);
  const double H_l = h_l + 0.5 * (u_l * u_l + v_l * v_l + w_l * w_l);
  const double mf_l = rho_l * (n[0 * fs] * u_l + n[1 * fs] * v_l + n[2 * fs] * w_l);
  const double rho_r = pr[0], u_r = pr[1], v_r = pr[2], w_r = pr[3];
  const double p_r = ma_pressure(pr), h_r = ma_enthalpy(pr);
  const double H_r = h_r + 0.5 * (u_r * u_r + v_r * v_r + w_r * w_r);
  const double mf_r = rho_r * (n[0 * fs] * u_r + n[1 * fs] * v_r + n[2 * fs] * w_r);
  const double psum = p_l + p_r;
  flux[0] = 0.5 * (mf_l + mf_r);
  flux[1] = 0.5 * (mf_l * u_l + mf_r * u_r + n[0 * fs] * psum);
  flux[2] = 0.5 * (mf_l * v_l + mf_r * v_r + n[1 * fs] * psum);
  flux[3] = 0.5 * (mf_l * w_l + mf_r * w_r + n[2 * fs] * psum);
  flux[4] = 0.5 * (mf_l * H_l + mf_r * H_r);

  const double nn = sqrt(n[0 * fs] * n[0 * fs] + n[1 * fs] * n[1 * fs] + n[2 * fs] * n[2 * fs]);
  const double tn = sqrt(t[0 * fs] * t[0 * fs] + t[1 * fs] * t[1 * fs] + t[2 * fs] * t[2 * fs]);
  const double bn = sqrt(b[0 * fs] * b[0 * fs] + b[1 * fs] * b[1 * fs] + b[2 * fs] * b[2 * fs]);
  const double nu[3] = {n[0 * fs] / nn, n[1 * fs] / nn, n[2 * fs] / nn};
  const double tu[3] = {t[0 * fs] / tn, t[1 * fs] / tn, t[2 * fs] / tn};
  const double bu[3] = {b[0 * fs] / bn, b[1 * fs] / bn, b[2 * fs] / bn};

  const double denom = 1.0 / (sqrt(rho_l) + sqrt(rho_r));
  const double alpha = sqrt(rho_l) * denom;
  const double beta = 1.0 - alpha;
  const double ur = alpha * u_l + beta * u_r;
  const double vr = alpha * v_l + beta * v_r;
  const double wr = alpha * w_l + beta * w_r;
  const double hr = alpha * h_l + beta * h_r +
                    0.5 * alpha * beta *
                        ((u_r - u_l) * (u_r - u_l) + (v_r - v_l) * (v_r - v_l) +
                         (w_r - w_l) * (w_r - w_l));
  const double c = sqrt(gm1 * hr);
  double M[25];
  const double nv = ur * nu[0] + vr * nu[1] + wr * nu[2];
  const double tv = ur * tu[0] + vr * tu[1] + wr * tu[2];
  const double bv = ur * bu[0] + vr * bu[1] + wr * bu[2];
  const double ke = 0.5 * (ur * ur + vr * vr + wr * wr);
  const double c2i = 1.0 / (c * c);
  const double hc2i = 0.5 * c2i;
  double dq[5];
  dq[0] = rho_r - rho_l;
  dq[1] = rho_r * u_r - rho_l * u_l;
  dq[2] = rho_r * v_r - rho_l * v_l;
  dq[3] = rho_r * w_r - rho_l * w_l;
  dq[4] = (rho_r * H_r - p_r) - (rho_l * H_l - p_l);
  const double cbar = c * nn;
  const double ubar = ur * n[0 * fs] + vr * n[1 * fs] + wr * n[2 * fs];
  const double cfl = fabs(ubar) + cbar;
  const double e1 = ubar + cbar, e2 = ubar - cbar, e3 = ubar;
  double a1 = fabs(e1), a2 = fabs(e2), a3 = fabs(e3);
  const double epuc = efix_u * cfl, epcc = efix_c * cfl;
  if (a1 < epcc) a1 = 0.5 * (e1 * e1 + epcc * epcc) / epcc;
  if (a2 < epcc) a2 = 0.5 * (e2 * e2 + epcc * epcc) / epcc;
  if (a3 < epuc) a3 = 0.5 * (e3 * e3 + epuc * epuc) / epuc;
  double ep[5] = {0.5 * (e1 + a1), 0.5 * (e2 + a2), 0.5 * (e3 + a3), 0.0, 0.0};
  ep[3] = ep[4] = ep[2];
  double em[5] = {0.5 * (e1 - a1), 0.5 * (e2 - a2), 0.5 * (e3 - a3), 0.0, 0.0};
  em[3] = em[4] = em[2];
  double ldq[5] = {0, 0, 0, 0, 0};
  double rl[5] = {0, 0, 0, 0, 0};
  /* left eigenvector matrix, mini_aero_utils.hpp:231-261 */
  M[0] = gm1 * (ke - hr) + c * (c - nv);
  M[1] = c * nu[0] - gm1 * ur;
  M[2] = c * nu[1] - gm1 * vr;
  M[3] = c * nu[2] - gm1 * wr;
  M[4] = gm1;
  M[5] = gm1 * (ke - hr) + c * (c + nv);
  M[6] = -c * nu[0] - gm1 * ur;
  M[7] = -c * nu[1] - gm1 * vr;
  M[8] = -c * nu[2] - gm1 * wr;
  M[9] = gm1;
  M[10] = ke - hr;
  M[11] = -ur;
  M[12] = -vr;
  M[13] = -wr;
  M[14] = 1.0;
  M[15] = -tv;
  M[16] = tu[0];
  M[17] = tu[1];
  M[18] = tu[2];
  M[19] = 0.0;
  M[20] = -bv;
  M[21] = bu[0];
  M[22] = bu[1];
  M[23] = bu[2];
  M[24] = 0.0;
  ma_matvec5(M, dq, ldq);
  for (int j = 0; j < 5; ++j) ldq[j] = (ep[j] - em[j]) * ldq[j];
  /* right eigenvector matrix, mini_aero_utils.hpp:266-313 */
  M[0] = hc2i;
  M[1] = hc2i;
  M[2] = -gm1 * c2i;
  M[3] = 0.0;
  M[4] = 0.0;
  M[5] = (ur + nu[0] * c) * hc2i;
  M[6] = (ur - nu[0] * c) * hc2i;
  M[7] = -gm1 * ur * c2i;
  M[8] = tu[0];
  M[9] = bu[0];
  M[10] = (vr + nu[1] * c) * hc2i;
  M[11] = (vr - nu[1] * c) * hc2i;
  M[12] = -gm1 * vr * c2i;
  M[13] = tu[1];
  M[14] = bu[1];
  M[15] = (wr + nu[2] * c) * hc2i;
  M[16] = (wr - nu[2] * c) * hc2i;
  M[17] = -gm1 * wr * c2i;
  M[18] = tu[2];
  M[19] = bu[2];
  M[20] = (hr + ke + c * nv) * hc2i;
  M[21] = (hr + ke - c * nv) * hc2i;
  M[22] = (c * c - gm1 * (hr + ke)) * c2i;
  M[23] = tv;
  M[24] = bv;
  ma_matvec5(M, ldq, rl);
  for (int i = 0; i < 5; ++i) flux[i] -= 0.5 * rl[i];
}

static void ma_viscous(const double g[5][3], const double *prim,
                       const double *a, double *vflux, uint32_t as) {
  const double T = prim[4];
  const double visc = 1.458e-6 * T * sqrt(T) / (T + 110.4);
  const double tc = visc * 1006.0 / 0.71;
  double div = 0;
  for (int i = 0; i < 5; ++i) vflux[i] = 0.0;
  for (int i = 0; i < 3; i++) div += g[i + 1][i];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      const double delta = (i == j) ? 1 : 0;
      const double S = 0.5 * (g[i + 1][j] + g[j + 1][i]);
      const double tij = S - div * delta / 3.;
      vflux[1 + i] += (2 * visc * tij) * a[j * as];
      vflux[4] += (2 * visc * tij) * prim[i + 1] * a[j * as];
    }
    vflux[4] += tc * g[4][i] * a[i * as];
  }
}

/* mini_aero user functor, mini_aero_func.hpp:11-85. */
static void mini_aero_func(double flux[5], const double *vl, const double *vr,
                           const double *cl, const double *cr,
                           const double *gl, const double *gr,
                           const double *ll, const double *lr,
                           const double *fc, const double *fn,
                           const double *ft, const double *fb, uint32_t cs,
                           uint32_t fs) {
  double Ul[5], Ur[5], Pl[5], Pr[5];
  for (int k = 0; k < 5; ++k) {
    Ul[k] = vl[k * cs];
    Ur[k] = vr[k * cs];
  }
  ma_primitives(Ul, Pl);
  ma_primitives(Ur, Pr);
  for (int k = 0; k < 5; ++k) {
    double tl = 0, tr = 0;
    for (int d = 0; d < 3; ++d) {
      tl += (fc[d * fs] - cl[d * cs]) * gl[(k * 3 + d) * cs];
      tr += (fc[d * fs] - cr[d * cs]) * gr[(k * 3 + d) * cs];
    }
    Pl[k] += tl * ll[k * cs];
    Pr[k] += tr * lr[k * cs];
  }
  ma_inviscid(Pl, Pr, flux, fn, ft, fb, fs);
  double pf[5], gf[5][3];
  for (int k = 0; k < 5; ++k) {
    pf[k] = 0.5 * (Pl[k] + Pr[k]);
    for (int d = 0; d < 3; ++d)
      gf[k][d] = 0.5 * (gl[(k * 3 + d) * cs] + gr[(k * 3 + d) * cs]);
  }
  double vf[5];
  ma_viscous((const double(*)[3])gf, pf, fn, vf, fs);
  for (int k = 0; k < 5; ++k) flux[k] -= vf[k];
}

/* LULESH helpers, lulesh_utils.hpp:4-200. */
static double lu_shape_volume(const double *x, const double *y,
                              const double *z) {
  /* Only the volume of CalcElemShapeFunctionDerivatives survives: its b[][]
   * is overwritten by CalcElemNodeNormals in the functor. */
  double fjxxi, fjxet, fjxze, fjyxi, fjyet, fjyze, fjzxi, fjzet, fjzze;
  double cjxet, cjyet, cjzet;
  fjxxi = .125 * ((x[6] - x[0]) + (x[5] - x[3]) - (x[7] - x[1]) - (x[4] - x[2]));
  fjxet = .125 * ((x[6] - x[0]) - (x[5] - x[3]) + (x[7] - x[1]) - (x[4] - x[2]));
  fjxze = .125 * ((x[6] - x[0]) + (x[5] - x[3]) + (x[7] - x[1]) + (x[4] - x[2]));
  fjyxi = .125 * ((y[6] - y[0]) + (y[5] - y[3]) - (y[7] - y[1]) - (y[4] - y[2]));
  fjyet = .125 * ((y[6] - y[0]) - (y[5] - y[3]) + (y[7] - y[1]) - (y[4] - y[2]));
  fjyze = .125 * ((y[6] - y[0]) + (y[5] - y[3]) + (y[7] - y[1]) + (y[4] - y[2]));
  fjzxi = .125 * ((z[6] - z[0]) + (z[5] - z[3]) - (z[7] - z[1]) - (z[4] - z[2]));
  fjzet = .125 * ((z[6] - z[0]) - (z[5] - z[3]) + (z[7] - z[1]) - (z[4] - z[2]));
  fjzze = .125 * ((z[6] - z[0]) + (z[5] - z[3]) + (z[7] - z[1]) + (z[4] - z[2]));
  cjxet = -(fjyxi * fjzze) + (fjzxi * fjyze);
  cjyet = (fjxxi * fjzze) - (fjzxi * fjxze);
  cjzet = -(fjxxi * fjyze) + (fjyxi * fjxze);
  return 8. * (fjxet * cjxet + fjyet * cjyet + fjzet * cjzet);
}

static void lu_face(double *px, double *py, double *pz, int a, int b, int c,
                    int d, const double *x, const double *y, const double *z) {
  /* SumElemFaceNormal with nodes (a, b, c, d) as (0, 1, 2, 3) */
  const double bx0 = 0.5 * (x[d] + x[c] - x[b] - x[a]);
  const double by0 = 0.5 * (y[d] + y[c] - y[b] - y[a]);
  const double bz0 = 0.5 * (z[d] + z[c] - z[b] - z[a]);
  const double bx1 = 0.5 * (x[c] + x[b] - x[d] - x[a]);
  const double by1 = 0.5 * (y[c] + y[b] - y[d] - y[a]);
  const double bz1 = 0.5 * (z[c] + z[b] - z[d] - z[a]);
  const double ax = 0.25 * (by0 * bz1 - bz0 * by1);
  const double ay = 0.25 * (bz0 * bx1 - bx0 * bz1);
  const double az = 0.25 * (bx0 * by1 - by0 * bx1);
  px[a] += ax; px[b] += ax; px[c] += ax; px[d] += ax;
  py[a] += ay; py[b] += ay; py[c] += ay; py[d] += ay;
  pz[a] += az; pz[b] += az; pz[c] += az; pz[d] += az;
}

/* LULESH user functor, lulesh_func.hpp:11-37: f_out[i*8+j] = force component
 * i on node j; writes the element volume into *determ. */
static void lulesh_func(double *f_out, const double *const *xyz,
                        const double *sig, double *determ, uint32_t xs,
                        uint32_t ds) {
  double x[8], y[8], z[8], B[3][8];
  for (int j = 0; j < 8; ++j) {
    x[j] = xyz[j][0];
    y[j] = xyz[j][xs];
    z[j] = xyz[j][2 * xs];
  }
  const double sxx = sig[0], syy = sig[1 * ds], szz = sig[2 * ds];
  *determ = lu_shape_volume(x, y, z);
  for (int j = 0; j < 8; ++j) B[0][j] = B[1][j] = B[2][j] = 0.0;
  lu_face(B[0], B[1], B[2], 0, 1, 2, 3, x, y, z);
  lu_face(B[0], B[1], B[2], 0, 4, 5, 1, x, y, z);
  lu_face(B[0], B[1], B[2], 1, 5, 6, 2, x, y, z);
  lu_face(B[0], B[1], B[2], 2, 6, 7, 3, x, y, z);
  lu_face(B[0], B[1], B[2], 3, 7, 4, 0, x, y, z);
  lu_face(B[0], B[1], B[2], 4, 7, 6, 5, x, y, z);
  for (int j = 0; j < 8; j++) {
    f_out[0 * 8 + j] = -(sxx * B[0][j]);
    f_out[1 * 8 + j] = -(syy * B[1][j]);
    f_out[2 * 8 + j] = -(szz * B[2][j]);
  }
}

/* volna user functor, volna_func.hpp:16-35 (float arithmetic). */
static void volna_func(const float *vol0, const float *vol1, float *left,
                       float *right, const float *fl, const float *bs,
                       const float *nm, const int *isb, uint32_t cs) {
  left[0] -= (fl[0 * cs]) / vol0[0];
  left[1] -= (fl[1 * cs] + bs[0 * cs] * nm[0 * cs]) / vol0[0];
  left[2] -= (fl[2 * cs] + bs[0 * cs] * nm[1 * cs]) / vol0[0];
  if (!*isb) {
    right[0] += fl[0 * cs] / vol1[0];
    right[1] += (fl[1 * cs] + bs[1 * cs] * nm[0 * cs]) / vol1[0];
    right[2] += (fl[2 * cs] + bs[1 * cs] * nm[1 * cs]) / vol1[0];
  }
}

/* getacc user functor, getacc_scatter_func.hpp:18-96. */
static void getacc_func(const double *cnmass, const double *rho,
                        const double *cnwt, const double *cnfx,
                        const double *cnfy, double *const *pt, uint32_t cs) {
  const double zerocut = 1.0e-40;
  for (int jj = 0; jj < 4; ++jj) {
    double *p = pt[jj];
    if (cnmass[jj * cs] > zerocut) {
      p[0] += cnmass[jj * cs];
    } else {
      int ii = jj - 1;
      if (ii == -1) ii = 3;
      if (cnmass[ii * cs] > zerocut) {
        p[0] += cnmass[ii * cs];
      } else {
        p[0] += *rho * cnwt[jj * cs];
      }
    }
    p[1] += cnwt[jj * cs];
    p[2] += cnfx[jj * cs];
    p[3] += cnfy[jj * cs];
  }
}

/* ------------------------------------------------------------------------ */
/* Loop descriptions (initProblem of each driver)                            */
/* ------------------------------------------------------------------------ */

typedef struct loop_desc {
  int n_maps, mesh_dim;
  int out_dim;   /* dim of point_data[0] */
  int out_f32;   /* point_data[0] is float */
} loop_desc;

static int get_desc(int loop, loop_desc *d) {
  switch (loop) {
  case ORC_RES_CALC: *d = (loop_desc){4, 2, 4, 0}; return 0;
  case ORC_MINI_AERO: *d = (loop_desc){2, 2, 5, 0}; return 0;
  case ORC_LULESH: *d = (loop_desc){2, 8, 3, 0}; return 0;
  case ORC_VOLNA: *d = (loop_desc){2, 2, 4, 1}; return 0;
  case ORC_GETACC: *d = (loop_desc){1, 4, 4, 0}; return 0;
  default: return -1;
  }
}

/* Computes the increments of cell `c` into inc[slot*out_dim + k] (float
 * loops use incf).  Direct outputs (lulesh determ) are written in place. */
static void cell_increment(int loop, int soa, uint32_t n_cells,
                           const uint32_t *n_points, const uint32_t *const *maps,
                           void *const *pd, void *const *cd, uint32_t c,
                           double *inc, float *incf) {
  switch (loop) {
  case ORC_RES_CALC: {
    /* res_calc.hpp:29-89: x through mapping 1; q, adt and res through mapping 0 */
    const double *x = (const double *)pd[1], *q = (const double *)pd[2],
                 *adt = (const double *)pd[3];
    const uint32_t dx = soa ? 1 : 2, dq = soa ? 1 : 4;
    const uint32_t n0 = maps[0][2 * c + 0], n1 = maps[0][2 * c + 1];
    const uint32_t m0 = maps[1][2 * c + 0], m1 = maps[1][2 * c + 1];
    const uint32_t xs = soa ? n_points[1] : 1, qs = soa ? n_points[2] : 1;
    res_calc_func(x + dx * m0, x + dx * m1, q + dq * n0, q + dq * n1, adt + n0,
                  adt + n1, inc, inc + 4, xs, qs);
    break;
  }
  case ORC_MINI_AERO: {
    /* mini_aero.hpp:43-111: cell records through mapping 0 */
    const double *co = (const double *)pd[1], *face = (const double *)cd[0];
    const uint32_t d1 = soa ? 1 : 28, s1 = soa ? n_points[1] : 1;
    const uint32_t l = maps[0][2 * c + 0], r = maps[0][2 * c + 1];
    const double *L = co + d1 * l, *R = co + d1 * r;
    const double *f = face + c;
    double flux[5];
    mini_aero_func(flux, L, R, L + 5 * s1, R + 5 * s1, L + 8 * s1, R + 8 * s1,
                   L + 23 * s1, R + 23 * s1, f + 0 * n_cells, f + 3 * n_cells,
                   f + 6 * n_cells, f + 9 * n_cells, s1, n_cells);
    /* left -= flux, right += flux: stored as signed increments */
    for (int k = 0; k < 5; ++k) {
      inc[k] = -flux[k];
      inc[5 + k] = flux[k];
    }
    break;
  }
  case ORC_LULESH: {
    /* lulesh.hpp:23-58 */
    const double *xyz = (const double *)pd[1], *sig = (const double *)cd[0];
    double *determ = (double *)cd[1];
    const uint32_t d = soa ? 1 : 3, xs = soa ? n_points[1] : 1;
    const double *rows[8];
    for (int j = 0; j < 8; ++j) rows[j] = xyz + d * maps[0][8 * c + j];
    double f[24];
    lulesh_func(f, rows, sig + c, &determ[c], xs, n_cells);
    for (int j = 0; j < 8; ++j)
      for (int i = 0; i < 3; ++i) inc[j * 3 + i] = f[i * 8 + j];
    break;
  }
  case ORC_VOLNA: {
    /* volna.hpp:30-75 */
    const float *vol = (const float *)pd[1];
    const float *fl = (const float *)cd[0], *bs = (const float *)cd[1],
                *nm = (const float *)cd[2];
    const int *isb = (const int *)cd[3];
    const uint32_t l = maps[0][2 * c + 0], r = maps[0][2 * c + 1];
    for (int i = 0; i < 8; ++i) incf[i] = 0;
    volna_func(vol + l, vol + r, incf, incf + 4, fl + c, bs + c, nm + c,
               isb + c, n_cells);
    break;
  }
  case ORC_GETACC: {
    /* getacc_scatter.hpp:29-75 */
    const double *const *D = (const double *const *)cd;
    for (int i = 0; i < 16; ++i) inc[i] = 0;
    double *pt[4] = {inc, inc + 4, inc + 8, inc + 12};
    getacc_func(D[0] + c, D[1] + c, D[2] + c, D[3] + c, D[4] + c, pt, n_cells);
    break;
  }
  }
}

static size_t out_index(int soa, uint32_t np0, uint32_t p, int dim, int k) {
  return soa ? (size_t)k * np0 + p : (size_t)p * dim + k;
}

int orc_loop_serial(int loop, int soa, uint32_t n_cells,
                    const uint32_t *n_points, const uint32_t *const *maps,
                    void *const *point_data, void *const *cell_data,
                    uint32_t iters) {
  loop_desc d;
  if (get_desc(loop, &d)) return -1;
  double inc[24];
  float incf[8];
  const uint32_t np0 = n_points[0];
  for (uint32_t it = 0; it < iters; ++it) {
    for (uint32_t c = 0; c < n_cells; ++c) {
      cell_increment(loop, soa, n_cells, n_points, maps, point_data, cell_data,
                     c, inc, incf);
      for (int s = 0; s < d.mesh_dim; ++s) {
        const uint32_t p = maps[0][(size_t)d.mesh_dim * c + s];
        for (int k = 0; k < d.out_dim; ++k) {
          const size_t o = out_index(soa, np0, p, d.out_dim, k);
          if (d.out_f32)
            ((float *)point_data[0])[o] += incf[s * d.out_dim + k];
          else
            ((double *)point_data[0])[o] += inc[s * d.out_dim + k];
        }
      }
    }
  }
  return 0;
}

int orc_replay_hier(int loop, int soa, uint32_t n_cells,
                    const uint32_t *n_points, const uint32_t *const *maps,
                    void *const *point_data, void *const *cell_data,
                    uint32_t iters, const orc_plan *P) {
  loop_desc d;
  if (get_desc(loop, &d)) return -1;
  if (P->n_cells != n_cells || (int)P->mesh_dim != d.mesh_dim) return -2;
  uint32_t max_pts = 0;
  for (uint32_t b = 0; b < P->n_blocks; ++b) {
    const uint32_t n = P->pts_off[b + 1] - P->pts_off[b];
    if (n > max_pts) max_pts = n;
  }
  double *cache = (double *)malloc(sizeof(double) * (max_pts + 1) * d.out_dim);
  float *cachef = (float *)malloc(sizeof(float) * (max_pts + 1) * d.out_dim);
  double inc[24];
  float incf[8];
  const uint32_t np0 = n_points[0];
  for (uint32_t it = 0; it < iters; ++it) {
    for (uint32_t b = 0; b < P->n_blocks; ++b) {
      const uint32_t npts = P->pts_off[b + 1] - P->pts_off[b];
      const uint32_t *pts = P->pts + P->pts_off[b];
      for (uint32_t i = 0; i < npts * (uint32_t)d.out_dim; ++i) {
        cache[i] = 0.0;
        cachef[i] = 0.0f;
      }
      /* thread colours in ascending order; inside one colour no two cells
       * share a written point, so their order does not matter */
      for (uint32_t col = 0; col < P->block_ntcol[b]; ++col) {
        for (uint32_t pos = P->block_start[b]; pos < P->block_start[b + 1]; ++pos) {
          if (P->tcol[pos] != col) continue;
          const uint32_t c = P->cell_id[pos];
          cell_increment(loop, soa, n_cells, n_points, maps, point_data,
                         cell_data, c, inc, incf);
          for (int s = 0; s < d.mesh_dim; ++s) {
            const uint32_t l = P->lidx[(size_t)s * n_cells + pos];
            for (int k = 0; k < d.out_dim; ++k) {
              if (d.out_f32)
                cachef[l * d.out_dim + k] += incf[s * d.out_dim + k];
              else
                cache[l * d.out_dim + k] += inc[s * d.out_dim + k];
            }
          }
        }
      }
      for (uint32_t i = 0; i < npts; ++i) {
        for (int k = 0; k < d.out_dim; ++k) {
          const size_t o = out_index(soa, np0, pts[i], d.out_dim, k);
          if (d.out_f32)
            ((float *)point_data[0])[o] += cachef[i * d.out_dim + k];
          else
            ((double *)point_data[0])[o] += cache[i * d.out_dim + k];
        }
      }
    }
  }
  free(cache);
  free(cachef);
  return 0;
}

/* The Airfoil iteration around res_calc (fot_airfoil_run's kernels in
 * csrc/airfoil.cu, operation for operation). */
int orc_airfoil_run(int soa, uint32_t n_edges, const uint32_t *n_points,
                    const uint32_t *const *maps, void *const *point_data,
                    const orc_airfoil *A, uint32_t iters, const orc_plan *P,
                    double *rms) {
  const double gam = 1.4, gm1 = 0.4, eps = 0.05;
  const uint32_t nc = n_points[0], nn = n_points[1];
  double *res = (double *)point_data[0], *q = (double *)point_data[2];
  double *adt = (double *)point_data[3];
  const double *x = (const double *)point_data[1];
  double *qold = (double *)malloc(sizeof(double) * 4 * (size_t)nc);
  if (!qold) return -1;
#define AT(n, i, dim, k) (soa ? (size_t)(k) * (n) + (i) : (size_t)(i) * (dim) + (k))
  double sum = 0.0;
  for (uint32_t it = 0; it < iters; ++it) {
    memcpy(qold, q, sizeof(double) * 4 * (size_t)nc);
    for (int stage = 0; stage < 2; ++stage) {
      /* adt_calc */
      for (uint32_t c = 0; c < nc; ++c) {
        double px[4], py[4];
        for (int j = 0; j < 4; ++j) {
          const uint32_t n = A->cell_to_node[4 * (size_t)c + j];
          px[j] = x[AT(nn, n, 2, 0)];
          py[j] = x[AT(nn, n, 2, 1)];
        }
        const double ri = 1.0 / q[AT(nc, c, 4, 0)];
        const double u = ri * q[AT(nc, c, 4, 1)], v = ri * q[AT(nc, c, 4, 2)];
        const double snd = sqrt(gam * gm1 * (ri * q[AT(nc, c, 4, 3)] - 0.5 * (u * u + v * v)));
        double s = 0.0;
        for (int j = 0; j < 4; ++j) {
          const double dx = px[(j + 1) & 3] - px[j];
          const double dy = py[(j + 1) & 3] - py[j];
          s += fabs(u * dy - v * dx) + snd * sqrt(dx * dx + dy * dy);
        }
        adt[c] = s / A->cfl;
      }
      /* res_calc */
      const int rc = P ? orc_replay_hier(ORC_RES_CALC, soa, n_edges, n_points, maps,
                                         point_data, NULL, 1, P)
                       : orc_loop_serial(ORC_RES_CALC, soa, n_edges, n_points, maps,
                                         point_data, NULL, 1);
      if (rc) {
        free(qold);
        return rc;
      }
      /* bres_calc */
      for (uint32_t e = 0; e < A->n_bedges; ++e) {
        const uint32_t c = A->bedge_to_cell[e];
        const uint32_t n1 = A->bedge_to_node[2 * (size_t)e], n2 = A->bedge_to_node[2 * (size_t)e + 1];
        const double dx = x[AT(nn, n1, 2, 0)] - x[AT(nn, n2, 2, 0)];
        const double dy = x[AT(nn, n1, 2, 1)] - x[AT(nn, n2, 2, 1)];
        double q1[4];
        for (int k = 0; k < 4; ++k) q1[k] = q[AT(nc, c, 4, k)];
        const double ri = 1.0 / q1[0];
        const double p1 = gm1 * (q1[3] - 0.5 * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
        double *r0 = &res[AT(nc, c, 4, 0)], *r1 = &res[AT(nc, c, 4, 1)];
        double *r2 = &res[AT(nc, c, 4, 2)], *r3 = &res[AT(nc, c, 4, 3)];
        if (A->bound[e] == 1) {
          *r1 += p1 * dy;
          *r2 += -p1 * dx;
        } else {
          const double *qi = A->qinf;
          const double vol1 = ri * (q1[1] * dy - q1[2] * dx);
          const double ri2 = 1.0 / qi[0];
          const double p2 = gm1 * (qi[3] - 0.5 * ri2 * (qi[1] * qi[1] + qi[2] * qi[2]));
          const double vol2 = ri2 * (qi[1] * dy - qi[2] * dx);
          const double mu = adt[c] * eps;
          *r0 += 0.5 * (vol1 * q1[0] + vol2 * qi[0]) + mu * (q1[0] - qi[0]);
          *r1 += 0.5 * (vol1 * q1[1] + p1 * dy + vol2 * qi[1] + p2 * dy) + mu * (q1[1] - qi[1]);
          *r2 += 0.5 * (vol1 * q1[2] - p1 * dx + vol2 * qi[2] - p2 * dx) + mu * (q1[2] - qi[2]);
          *r3 += 0.5 * (vol1 * (q1[3] + p1) + vol2 * (qi[3] + p2)) + mu * (q1[3] - qi[3]);
        }
      }
      /* update */
      sum = 0.0;
      for (uint32_t c = 0; c < nc; ++c) {
        const double adti = 1.0 / adt[c];
        for (int k = 0; k < 4; ++k) {
          const size_t o = AT(nc, c, 4, k);
          const double del = adti * res[o];
          q[o] = qold[o] - del;
          res[o] = 0.0;
          sum += del * del;
        }
      }
    }
  }
#undef AT
  if (rms) *rms = sqrt(sum / (double)nc);
  free(qold);
  return 0;
}

int orc_is_permutation(const uint32_t *perm, uint32_t n) {
  unsigned char *seen = (unsigned char *)calloc(n ? n : 1, 1);
  int ok = 1;
  for (uint32_t i = 0; i < n && ok; ++i) {
    if (perm[i] >= n || seen[perm[i]]) ok = 0;
    else seen[perm[i]] = 1;
  }
  free(seen);
  return ok;
}

#define PLAN_FAIL(code, ...)                                                   \
  do {                                                                         \
    if (err && err_len) snprintf(err, err_len, __VA_ARGS__);                   \
    rc = code;                                                                 \
    goto done;                                                                 \
  } while (0)

int orc_check_plan(const orc_plan *P, const uint32_t *map0, uint32_t n_points0,
                   uint32_t block_size, char *err, uint32_t err_len) {
  int rc = 0;
  const uint32_t n = P->n_cells, D = P->mesh_dim;
  uint32_t *owner = (uint32_t *)malloc(sizeof(uint32_t) * (n_points0 ? n_points0 : 1));
  uint32_t *stamp = (uint32_t *)malloc(sizeof(uint32_t) * (n_points0 ? n_points0 : 1));
  uint64_t *tmask = NULL;
  if (err && err_len) err[0] = 0;
  for (uint32_t i = 0; i < n_points0; ++i) owner[i] = stamp[i] = 0xFFFFFFFFu;
  /* 1: positions are a bijection onto the cells */
  if (!orc_is_permutation(P->cell_id, n)) PLAN_FAIL(1, "cell_id is not a permutation");
  /* 2: block and colour offsets are consistent */
  if (P->block_start[0] != 0 || P->block_start[P->n_blocks] != n)
    PLAN_FAIL(2, "block_start does not cover [0, n_cells)");
  if (P->colour_offsets[0] != 0 || P->colour_offsets[P->n_colours] != P->n_blocks)
    PLAN_FAIL(2, "colour_offsets do not cover the blocks");
  for (uint32_t b = 0; b < P->n_blocks; ++b) {
    const uint32_t sz = P->block_start[b + 1] - P->block_start[b];
    if (sz == 0 || sz > block_size) PLAN_FAIL(3, "block %u has size %u", b, sz);
  }
  for (uint32_t c = 0; c < P->n_colours; ++c)
    if (P->colour_offsets[c + 1] < P->colour_offsets[c]) PLAN_FAIL(2, "colour offsets decrease");
  tmask = (uint64_t *)malloc(sizeof(uint64_t) * (n_points0 ? n_points0 : 1));
  for (uint32_t col = 0; col < P->n_colours; ++col) {
    for (uint32_t b = P->colour_offsets[col]; b < P->colour_offsets[col + 1]; ++b) {
      const uint32_t *pts = P->pts + P->pts_off[b];
      const uint32_t npts = P->pts_off[b + 1] - P->pts_off[b];
      /* 4: point list strictly ascending (unique) */
      for (uint32_t i = 1; i < npts; ++i)
        if (pts[i] <= pts[i - 1]) PLAN_FAIL(4, "block %u point list not unique/ascending", b);
      for (uint32_t i = 0; i < npts; ++i) {
        if (pts[i] >= n_points0) PLAN_FAIL(4, "block %u point out of range", b);
        tmask[pts[i]] = 0;
      }
      uint32_t prev_col = 0;
      for (uint32_t pos = P->block_start[b]; pos < P->block_start[b + 1]; ++pos) {
        const uint32_t c = P->cell_id[pos];
        const uint32_t tc = P->tcol[pos];
        /* 6: thread colours sorted and below the block's count */
        if (tc < prev_col || tc >= P->block_ntcol[b] || tc >= 64)
          PLAN_FAIL(6, "block %u thread colours not sorted or out of range", b);
        prev_col = tc;
        for (uint32_t s = 0; s < D; ++s) {
          const uint32_t l = P->lidx[(size_t)s * n + pos];
          const uint32_t p = map0[(size_t)c * D + s];
          /* 5: local index resolves to the cell's point */
          if (l >= npts || pts[l] != p) PLAN_FAIL(5, "block %u pos %u slot %u bad local index", b, pos, s);
          /* 7: no two cells of one thread colour share a point (a cell may
           * list the same point in two slots) */
          if (tmask[p] & (1ull << tc)) {
            int same_cell = 0;
            for (uint32_t s2 = 0; s2 < s; ++s2)
              if (map0[(size_t)c * D + s2] == p) same_cell = 1;
            if (!same_cell)
              PLAN_FAIL(7, "block %u: thread colour %u writes point %u twice", b, tc, p);
          }
          tmask[p] |= 1ull << tc;
          /* 8: no point written by two blocks of one block colour */
          if (stamp[p] == col && owner[p] != b)
            PLAN_FAIL(8, "colour %u: blocks %u and %u both write point %u", col, owner[p], b, p);
          stamp[p] = col;
          owner[p] = b;
        }
      }
      /* every listed point is used by the block */
      for (uint32_t i = 0; i < npts; ++i)
        if (owner[pts[i]] != b) PLAN_FAIL(4, "block %u lists unused point %u", b, pts[i]);
    }
  }
done:
  free(owner);
  free(stamp);
  free(tmask);
  return rc;
}

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

uint32_t orc_point_graph(uint32_t n_points, uint32_t n_cells, uint32_t dim,
                         const uint32_t *map, uint32_t *indices,
                         uint32_t *endpoints) {
  /* count candidate neighbours per point, then fill, sort and unique */
  uint32_t *cnt = (uint32_t *)calloc((size_t)n_points + 1, sizeof(uint32_t));
  for (uint32_t c = 0; c < n_cells; ++c)
    for (uint32_t i = 0; i < dim; ++i)
      for (uint32_t j = 0; j < dim; ++j)
        if (map[c * dim + i] != map[c * dim + j]) cnt[map[c * dim + i] + 1]++;
  for (uint32_t p = 0; p < n_points; ++p) cnt[p + 1] += cnt[p];
  uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)n_points + 1));
  memcpy(fill, cnt, sizeof(uint32_t) * ((size_t)n_points + 1));
  for (uint32_t c = 0; c < n_cells; ++c)
    for (uint32_t i = 0; i < dim; ++i)
      for (uint32_t j = 0; j < dim; ++j)
        if (map[c * dim + i] != map[c * dim + j])
          endpoints[fill[map[c * dim + i]]++] = map[c * dim + j];
  uint32_t out = 0;
  indices[0] = 0;
  for (uint32_t p = 0; p < n_points; ++p) {
    const uint32_t a = cnt[p], b = cnt[p + 1];
    qsort(endpoints + a, b - a, sizeof(uint32_t), cmp_u32);
    for (uint32_t k = a; k < b; ++k)
      if (k == a || endpoints[k] != endpoints[k - 1]) endpoints[out++] = endpoints[k];
    indices[p + 1] = out;
  }
  free(cnt);
  free(fill);
  return out;
}

void orc_bandwidth_profile(uint32_t n_points, uint32_t n_cells, uint32_t dim,
                           const uint32_t *map, uint64_t *bandwidth,
                           uint64_t *profile) {
  uint32_t *lowest = (uint32_t *)malloc(sizeof(uint32_t) * (n_points ? n_points : 1));
  for (uint32_t p = 0; p < n_points; ++p) lowest[p] = p;
  uint64_t bw = 0;
  for (uint32_t c = 0; c < n_cells; ++c) {
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    for (uint32_t i = 0; i < dim; ++i) {
      const uint32_t p = map[c * dim + i];
      if (p < lo) lo = p;
      if (p > hi) hi = p;
    }
    if (hi - lo > bw) bw = hi - lo;
    for (uint32_t i = 0; i < dim; ++i)
      if (lowest[map[c * dim + i]] > lo) lowest[map[c * dim + i]] = lo;
  }
  uint64_t prof = 0;
  for (uint32_t p = 0; p < n_points; ++p) prof += p - lowest[p];
  *bandwidth = bw;
  *profile = prof;
  free(lowest);
}
