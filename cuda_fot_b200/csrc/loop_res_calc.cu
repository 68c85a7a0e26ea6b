// Executors instantiated for the res_calc loop.
#define FOT_ADAPTER FOT_LOOP_RES_CALC
#define FOT_ADAPTER_NS res_calc
#define FOT_OPS_NAME k_ops_res_calc
#include "loop_impl.cuh"
