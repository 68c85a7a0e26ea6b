// Executors instantiated for the volna loop.
#define FOT_ADAPTER FOT_LOOP_VOLNA
#define FOT_ADAPTER_NS volna
#define FOT_OPS_NAME k_ops_volna
#include "loop_impl.cuh"
