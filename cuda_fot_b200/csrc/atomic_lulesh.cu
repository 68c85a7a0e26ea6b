// Atomic executor instantiated for the lulesh loop, with multiply-add
// contraction (see loop_atomic_impl.cuh).
#define FOT_ADAPTER FOT_LOOP_LULESH
#define FOT_ADAPTER_NS lulesh
#include "loop_atomic_impl.cuh"
