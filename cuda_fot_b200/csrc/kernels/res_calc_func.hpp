// Airfoil res_calc edge flux (the per-edge user function).
//
// Drop-in format of the reference's kernels/res_calc_func.hpp: the includer
// defines USER_FUNCTION_SIGNATURE (return type, qualifiers and name) and
// RESTRICT before including this file, once per compilation target.  The
// arithmetic is the reference's operation for operation (res_calc_func.hpp:9-60;
// its float literals promote to double); a replacement file with the same
// signature can be dropped in through FOT_FUNCTOR_DIR.
//
// x1, x2: node coordinates (2, stride x_stride); q1, q2: cell states (4,
// stride q_stride); adt1, adt2: cell time steps; res1, res2: the flux added
// to the first cell and subtracted from the second.
#ifndef USER_FUNCTION_SIGNATURE
#define USER_FUNCTION_SIGNATURE void user_func
#endif
#ifndef RESTRICT
#define RESTRICT
#endif

USER_FUNCTION_SIGNATURE(const double *RESTRICT x1, const double *RESTRICT x2,
                        const double *RESTRICT q1, const double *RESTRICT q2,
                        const double *RESTRICT adt1, const double *RESTRICT adt2,
                        double *RESTRICT res1, double *RESTRICT res2,
                        unsigned x_stride, unsigned q_stride) {
  const double gm1 = 0.4, eps = 0.05;
  const double dx = x1[0] - x2[0];
  const double dy = x1[x_stride] - x2[x_stride];
  const double a0 = q1[0], a1 = q1[q_stride], a2 = q1[2 * q_stride], a3 = q1[3 * q_stride];
  const double b0 = q2[0], b1 = q2[q_stride], b2 = q2[2 * q_stride], b3 = q2[3 * q_stride];
  double ri = 1.0 / a0;
  const double p1 = gm1 * (a3 - 0.5 * ri * (a1 * a1 + a2 * a2));
  const double vol1 = ri * (a1 * dy - a2 * dx);
  ri = 1.0 / b0;
  const double p2 = gm1 * (b3 - 0.5 * ri * (b1 * b1 + b2 * b2));
  const double vol2 = ri * (b1 * dy - b2 * dx);
  const double mu = 0.5 * ((*adt1) + (*adt2)) * eps;
  double f;
  f = 0.5 * (vol1 * a0 + vol2 * b0) + mu * (a0 - b0);
  res1[0] = f;
  res2[0] = -f;
  f = 0.5 * (vol1 * a1 + p1 * dy + vol2 * b1 + p2 * dy) + mu * (a1 - b1);
  res1[1] = f;
  res2[1] = -f;
  f = 0.5 * (vol1 * a2 - p1 * dx + vol2 * b2 - p2 * dx) + mu * (a2 - b2);
  res1[2] = f;
  res2[2] = -f;
  f = 0.5 * (vol1 * (a3 + p1) + vol2 * (b3 + p2)) + mu * (a3 - b3);
  res1[3] = f;
  res2[3] = -f;
}

#undef USER_FUNCTION_SIGNATURE
#undef RESTRICT
