// miniAero face flux (the per-face user function).
//
// Drop-in format of the reference's kernels/mini_aero_func.hpp (same include
// protocol as res_calc_func.hpp); arithmetic as mini_aero_func.hpp:11-85.
// Cell records (stride cell_stride): conserved values (5), centre (3),
// gradients (15), limiters (5); face record (stride face_stride): centre,
// normal, tangent, binormal.  flux receives the inviscid minus the viscous
// flux through the face.
#ifndef USER_FUNCTION_SIGNATURE
#define USER_FUNCTION_SIGNATURE void user_func
#endif
#ifndef RESTRICT
#define RESTRICT
#endif

#include "mini_aero_utils.hpp"

USER_FUNCTION_SIGNATURE(double flux[5], const double *RESTRICT cell_values_left,
                        const double *RESTRICT cell_values_right,
                        const double *RESTRICT cell_coordinates_left,
                        const double *RESTRICT cell_coordinates_right,
                        const double *RESTRICT cell_gradients_left,
                        const double *RESTRICT cell_gradients_right,
                        const double *RESTRICT cell_limiters_left,
                        const double *RESTRICT cell_limiters_right,
                        const double *RESTRICT face_coordinates,
                        const double *RESTRICT face_normal,
                        const double *RESTRICT face_tangent,
                        const double *RESTRICT face_binormal,
                        MY_SIZE cell_stride, MY_SIZE face_stride) {
  double Ul[5], Ur[5], Pl[5], Pr[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    Ul[k] = cell_values_left[k * cell_stride];
    Ur[k] = cell_values_right[k * cell_stride];
  }
  ma_primitives(Ul, Pl);
  ma_primitives(Ur, Pr);
  // linear extrapolation to the face, limited
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double tl = 0, tr = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fc = face_coordinates[d * face_stride];
      tl += (fc - cell_coordinates_left[d * cell_stride]) *
            cell_gradients_left[(k * 3 + d) * cell_stride];
      tr += (fc - cell_coordinates_right[d * cell_stride]) *
            cell_gradients_right[(k * 3 + d) * cell_stride];
    }
    Pl[k] += tl * cell_limiters_left[k * cell_stride];
    Pr[k] += tr * cell_limiters_right[k * cell_stride];
  }
  // The viscous flux is evaluated before the inviscid one (the two are
  // independent, so every value is the same): the gradients then die before
  // the Roe flux's eigenvector matrices are live.
  double pf[5], gf[5][3];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    pf[k] = 0.5 * (Pl[k] + Pr[k]);
#pragma unroll
    for (int d = 0; d < 3; ++d)
      gf[k][d] = 0.5 * (cell_gradients_left[(k * 3 + d) * cell_stride] +
                        cell_gradients_right[(k * 3 + d) * cell_stride]);
  }
  double vf[5];
  ma_viscous_flux(gf, pf, face_normal, vf, face_stride);
  ma_inviscid_flux(Pl, Pr, flux, face_normal, face_tangent, face_binormal,
                   face_stride);
#pragma unroll
  for (int k = 0; k < 5; ++k) flux[k] -= vf[k];
}

#undef USER_FUNCTION_SIGNATURE
#undef RESTRICT
