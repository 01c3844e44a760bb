// Open-addressing launchers for the 4-byte-key / 0-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsSet4, kGroupSet4, 4, 0)
