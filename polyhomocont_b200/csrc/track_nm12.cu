// Instantiation unit of the tracking kernel for register rows of 12
// complex entries (systems with N = n + 1 <= 12 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(12)
