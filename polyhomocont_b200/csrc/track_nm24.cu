// Instantiation unit of the tracking kernel for register rows of 24
// complex entries (systems of n <= 24 equations: the rows of the reduced
// system, the patch row eliminated first).
#include "phc_track.cuh"

PHC_DEFINE_NM(24)
