// LULESH element stress -> node forces (the per-element user function).
//
// Drop-in format of the reference's kernels/lulesh_func.hpp (same include
// protocol as res_calc_func.hpp; MESH_DIM = 8 comes from the including
// namespace); arithmetic as lulesh_func.hpp:11-37.  xyz[j] points at node j's
// coordinates (stride xyz_stride), sig at the element's stress (stride
// direct_stride).  f_out[i*8 + j] receives force component i on node j and
// determ the element volume.
#ifndef USER_FUNCTION_SIGNATURE
#define USER_FUNCTION_SIGNATURE void user_func
#endif
#ifndef RESTRICT
#define RESTRICT
#endif

#include "lulesh_utils.hpp"

USER_FUNCTION_SIGNATURE(double *RESTRICT f_out, const double *RESTRICT xyz[MESH_DIM],
                        const double *RESTRICT sig, double &determ,
                        unsigned xyz_stride, unsigned direct_stride) {
  double x[8], y[8], z[8], bx[8], by[8], bz[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    x[j] = xyz[j][0];
    y[j] = xyz[j][xyz_stride];
    z[j] = xyz[j][2 * xyz_stride];
  }
  const double sxx = sig[0], syy = sig[direct_stride], szz = sig[2 * direct_stride];
  determ = lu_element_volume(x, y, z);
  lu_node_normals(bx, by, bz, x, y, z);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    f_out[0 * MESH_DIM + j] = -(sxx * bx[j]);
    f_out[1 * MESH_DIM + j] = -(syy * by[j]);
    f_out[2 * MESH_DIM + j] = -(szz * bz[j]);
  }
}

#undef USER_FUNCTION_SIGNATURE
#undef RESTRICT
