// Open-addressing launchers for the 4-byte-key / 4-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsMap44, kGroupMap44, 4, 4)
