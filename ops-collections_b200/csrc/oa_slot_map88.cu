// Open-addressing launchers for the 8-byte-key / 8-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsMap88, kGroupMap88, 8, 8)
