// Open-addressing launchers for the fp64-key / 4-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap84F, 8, 4, true)
