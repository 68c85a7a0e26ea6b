// Atomic executor instantiated for the getacc loop, with multiply-add
// contraction (see loop_atomic_impl.cuh).
#define FOT_ADAPTER FOT_LOOP_GETACC
#define FOT_ADAPTER_NS getacc
#include "loop_atomic_impl.cuh"
