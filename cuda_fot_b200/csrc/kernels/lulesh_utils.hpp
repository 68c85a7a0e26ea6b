// Helpers of the LULESH element force: the element volume from the
// shape-function Jacobian, the node normals summed over the six faces, and the
// stress -> node force product.  Arithmetic as the reference's
// kernels/lulesh_utils.hpp:4-200, operation for operation.
#ifndef FOT_LULESH_UTILS_HPP
#define FOT_LULESH_UTILS_HPP

#ifndef FOT_HD
#define FOT_HD __host__ __device__ __forceinline__
#endif

// Jacobian determinant (volume) of the hex; the shape-function derivatives the
// reference also computes here are overwritten by the node normals in the
// functor, so only the cofactors the volume needs are formed.
FOT_HD double lu_element_volume(const double x[8], const double y[8], const double z[8]) {
  const double fjxxi = .125 * ((x[6] - x[0]) + (x[5] - x[3]) - (x[7] - x[1]) - (x[4] - x[2]));
  const double fjxet = .125 * ((x[6] - x[0]) - (x[5] - x[3]) + (x[7] - x[1]) - (x[4] - x[2]));
  const double fjxze = .125 * ((x[6] - x[0]) + (x[5] - x[3]) + (x[7] - x[1]) + (x[4] - x[2]));
  const double fjyxi = .125 * ((y[6] - y[0]) + (y[5] - y[3]) - (y[7] - y[1]) - (y[4] - y[2]));
  const double fjyet = .125 * ((y[6] - y[0]) - (y[5] - y[3]) + (y[7] - y[1]) - (y[4] - y[2]));
  const double fjyze = .125 * ((y[6] - y[0]) + (y[5] - y[3]) + (y[7] - y[1]) + (y[4] - y[2]));
  const double fjzxi = .125 * ((z[6] - z[0]) + (z[5] - z[3]) - (z[7] - z[1]) - (z[4] - z[2]));
  const double fjzet = .125 * ((z[6] - z[0]) - (z[5] - z[3]) + (z[7] - z[1]) - (z[4] - z[2]));
  const double fjzze = .125 * ((z[6] - z[0]) + (z[5] - z[3]) + (z[7] - z[1]) + (z[4] - z[2]));
  const double cjxet = -(fjyxi * fjzze) + (fjzxi * fjyze);
  const double cjyet = (fjxxi * fjzze) - (fjzxi * fjxze);
  const double cjzet = -(fjxxi * fjyze) + (fjyxi * fjxze);
  return 8. * (fjxet * cjxet + fjyet * cjyet + fjzet * cjzet);
}

// quarter of the face normal of the quad (a, b, c, d), added to its 4 nodes
FOT_HD void lu_face_normal(double *px, double *py, double *pz, int a, int b,
                           int c, int d, const double *x, const double *y,
                           const double *z) {
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

FOT_HD void lu_node_normals(double px[8], double py[8], double pz[8],
                            const double x[8], const double y[8], const double z[8]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) px[i] = py[i] = pz[i] = 0.0;
  lu_face_normal(px, py, pz, 0, 1, 2, 3, x, y, z);
  lu_face_normal(px, py, pz, 0, 4, 5, 1, x, y, z);
  lu_face_normal(px, py, pz, 1, 5, 6, 2, x, y, z);
  lu_face_normal(px, py, pz, 2, 6, 7, 3, x, y, z);
  lu_face_normal(px, py, pz, 3, 7, 4, 0, x, y, z);
  lu_face_normal(px, py, pz, 4, 7, 6, 5, x, y, z);
}

#endif
