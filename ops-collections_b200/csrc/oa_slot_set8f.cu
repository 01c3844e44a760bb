// Open-addressing launchers for the fp64-key set layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsSet8F, 8, 0, true)
