// Open-addressing launchers for the 2-byte-key / 2-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap22, 2, 2, false)
