// Instantiation unit of the tracking kernel for register rows of 12
// complex entries (systems of n <= 12 equations: the rows of the reduced
// system, the patch row eliminated first).
#include "phc_track.cuh"

PHC_DEFINE_NM(12)
