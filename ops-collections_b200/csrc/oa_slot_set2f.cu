// Open-addressing launchers for the fp16-key set layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsSet2F, 2, 0, true)
