// Instantiations of the block-per-group decode kernel for float message storage.
#include "relaybp_slots.cuh"

RBPK_DEFINE_PICK_SLOTS(pick_slots_f32, float)
