// Instantiation unit of the tracking kernel for register rows of 32
// complex entries (systems with N = n + 1 <= 32 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(32)
