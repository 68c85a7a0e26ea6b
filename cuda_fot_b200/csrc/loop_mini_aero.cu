// Executors instantiated for the mini_aero loop.
#define FOT_ADAPTER FOT_LOOP_MINI_AERO
#define FOT_ADAPTER_NS mini_aero
#define FOT_OPS_NAME k_ops_mini_aero
#include "loop_impl.cuh"
