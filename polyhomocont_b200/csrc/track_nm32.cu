// Instantiation unit of the tracking kernel for register rows of 32
// complex entries (systems of n <= 32 equations: the rows of the reduced
// system, the patch row eliminated first).
#include "phc_track.cuh"

PHC_DEFINE_NM(32)
