// Open-addressing launchers for the 2-byte-key set layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsSet2, 2, 0, false)
