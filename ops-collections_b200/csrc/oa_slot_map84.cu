// Open-addressing launchers for the 8-byte-key / 4-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsMap84, kGroupMap84, 8, 4)
