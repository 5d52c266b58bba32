// Instantiation unit of the tracking kernel for register rows of 24
// complex entries (systems with N = n + 1 <= 24 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(24)
