// Instantiation unit of the tracking kernel for register rows of 6
// complex entries (systems of n <= 6 equations: the rows of the reduced
// system, the patch row eliminated first).
#include "phc_track.cuh"

PHC_DEFINE_NM(6)
