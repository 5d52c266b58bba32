// Instantiation unit of the tracking kernel for register rows of 6
// complex entries (systems with N = n + 1 <= 6 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(6)
