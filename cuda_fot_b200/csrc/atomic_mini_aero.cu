// Atomic executor instantiated for the mini_aero loop, with multiply-add
// contraction (see loop_atomic_impl.cuh).
#define FOT_ADAPTER FOT_LOOP_MINI_AERO
#define FOT_ADAPTER_NS mini_aero
#include "loop_atomic_impl.cuh"
