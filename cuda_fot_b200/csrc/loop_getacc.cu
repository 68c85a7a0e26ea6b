// Executors instantiated for the getacc loop.
#define FOT_ADAPTER FOT_LOOP_GETACC
#define FOT_ADAPTER_NS getacc
#define FOT_OPS_NAME k_ops_getacc
#include "loop_impl.cuh"
