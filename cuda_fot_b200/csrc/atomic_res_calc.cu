// Atomic executor instantiated for the res_calc loop, with multiply-add
// contraction (see loop_atomic_impl.cuh).
#define FOT_ADAPTER FOT_LOOP_RES_CALC
#define FOT_ADAPTER_NS res_calc
#include "loop_atomic_impl.cuh"
