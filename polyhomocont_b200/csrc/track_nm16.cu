// Instantiation unit of the tracking kernel for register rows of 16
// complex entries (systems with N = n + 1 <= 16 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(16)
