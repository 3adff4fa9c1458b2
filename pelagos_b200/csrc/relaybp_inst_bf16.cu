// Instantiations of the decode kernel for __nv_bfloat16 message storage.
#include "relaybp_kernel.cuh"

RBPK_DEFINE_PICK(pick_bf16, __nv_bfloat16)
