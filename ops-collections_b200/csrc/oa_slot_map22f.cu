// Open-addressing launchers for the fp16-key / 2-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap22F, 2, 2, true)
