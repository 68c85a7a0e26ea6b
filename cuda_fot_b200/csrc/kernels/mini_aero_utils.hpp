// Helper physics of the miniAero face flux: primitive variables, Roe upwind
// inviscid flux with the eigenvalue fix, and the viscous flux.  The
// arithmetic follows the reference's kernels/mini_aero_utils.hpp:6-373
// operation for operation so that results are bit-identical to its serial
// loop when neither side fuses multiply-adds.
#ifndef FOT_MINI_AERO_UTILS_HPP
#define FOT_MINI_AERO_UTILS_HPP

#ifndef FOT_HD
#define FOT_HD __host__ __device__ __forceinline__
#endif

// conserved (rho, rho u, rho v, rho w, E) -> primitive (rho, u, v, w, T)
FOT_HD void ma_primitives(const double *U, double *V) {
  const double gamma = 1.4, Rgas = 287.05;
  const double r = U[0];
  const double ri = 1.0 / r;
  const double u = U[1] * ri, v = U[2] * ri, w = U[3] * ri;
  const double k = 0.5 * (u * u + v * v + w * w);
  const double e = U[4] * ri - k;
  V[0] = r;
  V[1] = u;
  V[2] = v;
  V[3] = w;
  V[4] = e * (gamma - 1.0) / Rgas;
}

// y = A x for a 5x5 row-major A; y starts at y*0 and sums in column order
FOT_HD void ma_matvec5(const double *A, const double *x, double *y) {
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double acc = y[i] * 0.0;
#pragma unroll
    for (int j = 0; j < 5; ++j) acc += 1.0 * A[5 * i + j] * x[j];
    y[i] = acc;
  }
}

FOT_HD void ma_inviscid_flux(const double *pl, const double *pr, double *flux,
                             const double *n, const double *t, const double *b,
                             unsigned fs) {
  const double efix_u = 0.1, efix_c = 0.1, gm1 = 0.4;
  const double n0 = n[0], n1 = n[fs], n2 = n[2 * fs];
  const double t0 = t[0], t1 = t[fs], t2 = t[2 * fs];
  const double b0 = b[0], b1 = b[fs], b2 = b[2 * fs];
  const double rho_l = pl[0], u_l = pl[1], v_l = pl[2], w_l = pl[3];
  const double p_l = rho_l * 287.05 * pl[4], h_l = 1004.0 * pl[4];
  const double H_l = h_l + 0.5 * (u_l * u_l + v_l * v_l + w_l * w_l);
  const double mf_l = rho_l * (n0 * u_l + n1 * v_l + n2 * w_l);
  const double rho_r = pr[0], u_r = pr[1], v_r = pr[2], w_r = pr[3];
  const double p_r = rho_r * 287.05 * pr[4], h_r = 1004.0 * pr[4];
  const double H_r = h_r + 0.5 * (u_r * u_r + v_r * v_r + w_r * w_r);
  const double mf_r = rho_r * (n0 * u_r + n1 * v_r + n2 * w_r);
  const double psum = p_l + p_r;
  flux[0] = 0.5 * (mf_l + mf_r);
  flux[1] = 0.5 * (mf_l * u_l + mf_r * u_r + n0 * psum);
  flux[2] = 0.5 * (mf_l * v_l + mf_r * v_r + n1 * psum);
  flux[3] = 0.5 * (mf_l * w_l + mf_r * w_r + n2 * psum);
  flux[4] = 0.5 * (mf_l * H_l + mf_r * H_r);

  const double nn = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  const double tn = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
  const double bn = sqrt(b0 * b0 + b1 * b1 + b2 * b2);
  const double nu0 = n0 / nn, nu1 = n1 / nn, nu2 = n2 / nn;
  const double tu0 = t0 / tn, tu1 = t1 / tn, tu2 = t2 / tn;
  const double bu0 = b0 / bn, bu1 = b1 / bn, bu2 = b2 / bn;

  const double sl = sqrt(rho_l);
  const double denom = 1.0 / (sl + sqrt(rho_r));
  const double alpha = sl * denom;
  const double beta = 1.0 - alpha;
  const double ur = alpha * u_l + beta * u_r;
  const double vr = alpha * v_l + beta * v_r;
  const double wr = alpha * w_l + beta * w_r;
  const double hr = alpha * h_l + beta * h_r +
                    0.5 * alpha * beta *
                        ((u_r - u_l) * (u_r - u_l) + (v_r - v_l) * (v_r - v_l) +
                         (w_r - w_l) * (w_r - w_l));
  const double c = sqrt(gm1 * hr);
  const double nv = ur * nu0 + vr * nu1 + wr * nu2;
  const double tv = ur * tu0 + vr * tu1 + wr * tu2;
  const double bv = ur * bu0 + vr * bu1 + wr * bu2;
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
  const double ubar = ur * n0 + vr * n1 + wr * n2;
  const double cfl = fabs(ubar) + cbar;
  const double e1 = ubar + cbar, e2 = ubar - cbar, e3 = ubar;
  double a1 = fabs(e1), a2 = fabs(e2), a3 = fabs(e3);
  const double epuc = efix_u * cfl, epcc = efix_c * cfl;
  if (a1 < epcc) a1 = 0.5 * (e1 * e1 + epcc * epcc) / epcc;
  if (a2 < epcc) a2 = 0.5 * (e2 * e2 + epcc * epcc) / epcc;
  if (a3 < epuc) a3 = 0.5 * (e3 * e3 + epuc * epuc) / epuc;
  const double ep0 = 0.5 * (e1 + a1), ep1 = 0.5 * (e2 + a2), ep2 = 0.5 * (e3 + a3);
  const double em0 = 0.5 * (e1 - a1), em1 = 0.5 * (e2 - a2), em2 = 0.5 * (e3 - a3);
  const double gk = gm1 * (ke - hr);
  // left eigenvectors, one row per wave
  const double L[25] = {gk + c * (c - nv), c * nu0 - gm1 * ur, c * nu1 - gm1 * vr,
                        c * nu2 - gm1 * wr, gm1,
                        gk + c * (c + nv), -c * nu0 - gm1 * ur, -c * nu1 - gm1 * vr,
                        -c * nu2 - gm1 * wr, gm1,
                        ke - hr, -ur, -vr, -wr, 1.0,
                        -tv, tu0, tu1, tu2, 0.0,
                        -bv, bu0, bu1, bu2, 0.0};
  double ldq[5] = {0, 0, 0, 0, 0};
  ma_matvec5(L, dq, ldq);
  ldq[0] = (ep0 - em0) * ldq[0];
  ldq[1] = (ep1 - em1) * ldq[1];
  ldq[2] = (ep2 - em2) * ldq[2];
  ldq[3] = (ep2 - em2) * ldq[3];
  ldq[4] = (ep2 - em2) * ldq[4];
  // right eigenvectors
  const double hk = hr + ke;
  const double R[25] = {hc2i, hc2i, -gm1 * c2i, 0.0, 0.0,
                        (ur + nu0 * c) * hc2i, (ur - nu0 * c) * hc2i, -gm1 * ur * c2i, tu0, bu0,
                        (vr + nu1 * c) * hc2i, (vr - nu1 * c) * hc2i, -gm1 * vr * c2i, tu1, bu1,
                        (wr + nu2 * c) * hc2i, (wr - nu2 * c) * hc2i, -gm1 * wr * c2i, tu2, bu2,
                        (hk + c * nv) * hc2i, (hk - c * nv) * hc2i, (c * c - gm1 * hk) * c2i,
                        tv, bv};
  double rl[5] = {0, 0, 0, 0, 0};
  ma_matvec5(R, ldq, rl);
#pragma unroll
  for (int i = 0; i < 5; ++i) flux[i] -= 0.5 * rl[i];
}

FOT_HD void ma_viscous_flux(const double g[5][3], const double *prim,
                            const double *a, double *vflux, unsigned as) {
  const double T = prim[4];
  const double visc = 1.458e-6 * T * sqrt(T) / (T + 110.4);
  const double tc = visc * 1006.0 / 0.71;
  const double a0 = a[0], a1 = a[as], a2 = a[2 * as];
  const double av[3] = {a0, a1, a2};
  double div = 0;
#pragma unroll
  for (int i = 0; i < 5; ++i) vflux[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; i++) div += g[i + 1][i];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double delta = (i == j) ? 1 : 0;
      const double S = 0.5 * (g[i + 1][j] + g[j + 1][i]);
      const double tij = S - div * delta / 3.;
      vflux[1 + i] += (2 * visc * tij) * av[j];
      vflux[4] += (2 * visc * tij) * prim[i + 1] * av[j];
    }
    vflux[4] += tc * g[4][i] * av[i];
  }
}

#endif
