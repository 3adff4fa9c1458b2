// Instantiations of the decode kernel for float message storage.
#include "relaybp_kernel.cuh"

RBPK_DEFINE_PICK(pick_f32, float)
RBPK_DEFINE_PICK_MIXED(pick_mixed_f32, float)
