// Open-addressing launchers for the 4-byte-key / 8-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsMap48, kGroupMap48, 4, 8)
