// Instantiations of the decode kernel for __half message storage.
#include "relaybp_kernel.cuh"

RBPK_DEFINE_PICK(pick_f16, __half)
