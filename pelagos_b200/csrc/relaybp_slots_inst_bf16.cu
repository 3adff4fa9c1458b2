// Instantiations of the block-per-group decode kernel for __nv_bfloat16 message storage.
#include "relaybp_slots.cuh"

RBPK_DEFINE_PICK_SLOTS(pick_slots_bf16, __nv_bfloat16)
