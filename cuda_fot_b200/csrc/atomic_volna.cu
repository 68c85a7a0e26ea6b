// Atomic executor instantiated for the volna loop, with multiply-add
// contraction (see loop_atomic_impl.cuh).
#define FOT_ADAPTER FOT_LOOP_VOLNA
#define FOT_ADAPTER_NS volna
#include "loop_atomic_impl.cuh"
