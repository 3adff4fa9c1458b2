// Instantiations of the block-per-group decode kernel for __half message storage.
#include "relaybp_slots.cuh"

RBPK_DEFINE_PICK_SLOTS(pick_slots_f16, __half)
