// Instantiations of the block-per-group decode kernel for double message storage.
#include "relaybp_slots.cuh"

RBPK_DEFINE_PICK_SLOTS(pick_slots_f64, double)
