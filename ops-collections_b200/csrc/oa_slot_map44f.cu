// Open-addressing launchers for the fp32-key / 4-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap44F, 4, 4, true)
