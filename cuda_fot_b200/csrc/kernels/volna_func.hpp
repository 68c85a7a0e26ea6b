// Volna shallow-water edge update (the per-edge user function), FP32.
//
// Drop-in format of the reference's kernels/volna_func.hpp (same include
// protocol as res_calc_func.hpp); arithmetic as volna_func.hpp:16-35.
// cellVolumes0/1: areas of the two cells; left/right: the 4-component cell
// increments (3 used); edgeFluxes (3), bathySource (2), edgeNormals (2) and
// isRightBoundary are per-edge data with stride cell_stride.
#ifndef USER_FUNCTION_SIGNATURE
#define USER_FUNCTION_SIGNATURE void user_func
#endif
#ifndef RESTRICT
#define RESTRICT
#endif

USER_FUNCTION_SIGNATURE(const float *RESTRICT cellVolumes0,
                        const float *RESTRICT cellVolumes1,
                        float *RESTRICT left, float *RESTRICT right,
                        const float *RESTRICT edgeFluxes,
                        const float *RESTRICT bathySource,
                        const float *RESTRICT edgeNormals,
                        const int *RESTRICT isRightBoundary,
                        unsigned cell_stride) {
  const float f0 = edgeFluxes[0], f1 = edgeFluxes[cell_stride],
              f2 = edgeFluxes[2 * cell_stride];
  const float nx = edgeNormals[0], ny = edgeNormals[cell_stride];
  const float bl = bathySource[0], br = bathySource[cell_stride];
  left[0] -= f0 / cellVolumes0[0];
  left[1] -= (f1 + bl * nx) / cellVolumes0[0];
  left[2] -= (f2 + bl * ny) / cellVolumes0[0];
  if (!*isRightBoundary) {
    right[0] += f0 / cellVolumes1[0];
    right[1] += (f1 + br * nx) / cellVolumes1[0];
    right[2] += (f2 + br * ny) / cellVolumes1[0];
  }
}

#undef USER_FUNCTION_SIGNATURE
#undef RESTRICT
