// Instantiations of the decode kernel for double message storage.
#include "relaybp_kernel.cuh"

RBPK_DEFINE_PICK(pick_f64, double)
