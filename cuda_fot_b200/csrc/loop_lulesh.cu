// Executors instantiated for the lulesh loop.
#define FOT_ADAPTER FOT_LOOP_LULESH
#define FOT_ADAPTER_NS lulesh
#define FOT_OPS_NAME k_ops_lulesh
#include "loop_impl.cuh"
