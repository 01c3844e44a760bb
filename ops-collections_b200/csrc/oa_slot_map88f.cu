// Open-addressing launchers for the fp64-key / 8-byte-payload map layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS_ONLY(kOpsMap88F, 8, 8, true)
