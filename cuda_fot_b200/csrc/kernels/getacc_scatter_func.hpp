// BookLeaf getacc element -> node scatter (the per-element user function).
//
// Drop-in format of the reference's kernels/getacc_scatter_func.hpp (same
// include protocol as res_calc_func.hpp); arithmetic and branch structure as
// getacc_scatter_func.hpp:18-96.  For corner jj of the quad the node mass is
// cnmass[jj] when above zerocut, else the previous corner's cnmass, else
// rho*cnwt[jj]; then cnwt, cnfx, cnfy are added.
#ifndef USER_FUNCTION_SIGNATURE
#define USER_FUNCTION_SIGNATURE void user_func
#endif
#ifndef RESTRICT
#define RESTRICT
#endif

USER_FUNCTION_SIGNATURE(const double *RESTRICT cnmass, const double *RESTRICT rho,
                        const double *RESTRICT cnwt, const double *RESTRICT cnfx,
                        const double *RESTRICT cnfy, double *point1,
                        double *point2, double *point3, double *point4,
                        unsigned cell_stride) {
  const double zerocut = 1.0e-40;
  double *const pts[4] = {point1, point2, point3, point4};
#pragma unroll
  for (int jj = 0; jj < 4; ++jj) {
    double *p = pts[jj];
    const double m = cnmass[jj * cell_stride];
    if (m > zerocut) {
      p[0] += m;
    } else {
      const int ii = jj == 0 ? 3 : jj - 1;
      const double mp = cnmass[ii * cell_stride];
      if (mp > zerocut) {
        p[0] += mp;
      } else {
        p[0] += *rho * cnwt[jj * cell_stride];
      }
    }
    p[1] += cnwt[jj * cell_stride];
    p[2] += cnfx[jj * cell_stride];
    p[3] += cnfy[jj * cell_stride];
  }
}

#undef USER_FUNCTION_SIGNATURE
#undef RESTRICT
