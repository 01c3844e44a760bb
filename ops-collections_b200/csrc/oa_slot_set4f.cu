// Open-addressing launchers for the fp32-key set layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsSet4F, 4, 0, true)
