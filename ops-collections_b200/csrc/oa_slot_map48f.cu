// Open-addressing launchers for the fp32-key / 8-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap48F, 4, 8, true)
