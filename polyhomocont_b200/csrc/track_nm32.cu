// Instantiation unit of the tracking kernel for register rows of 32
// complex entries (systems whose eliminated rows -- the N = n + 1 rows, or
// the n equation rows when the patch row is eliminated first -- number at
// most 32).
#include "phc_track.cuh"

PHC_DEFINE_NM(32)
