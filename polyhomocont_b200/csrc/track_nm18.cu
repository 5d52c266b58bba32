// Instantiation unit of the tracking kernel for register rows of 18
// complex entries (systems whose eliminated rows -- the N = n + 1 rows, or
// the n equation rows when the patch row is eliminated first -- number at
// most 18).
#include "phc_track.cuh"

PHC_DEFINE_NM(18)
