// Instantiation unit of the tracking kernel for register rows of 8
// complex entries (systems with N = n + 1 <= 8 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(8)
