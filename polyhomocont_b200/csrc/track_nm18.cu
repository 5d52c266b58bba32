// Instantiation unit of the tracking kernel for register rows of 18
// complex entries (systems with N = n + 1 <= 18 unknowns).
#include "phc_track.cuh"

PHC_DEFINE_NM(18)
