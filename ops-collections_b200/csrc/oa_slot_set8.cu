// Open-addressing launchers for the 8-byte-key / 0-byte-payload slot layout.
#include "oa_inst.cuh"

B2CO_DEFINE_OA_OPS(kOpsSet8, kGroupSet8, 8, 0)
