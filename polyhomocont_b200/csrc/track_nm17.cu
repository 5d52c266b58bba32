// Instantiation unit of the tracking kernel for n = 16 with the patch row
// eliminated first: register rows of 16 complex entries holding the 16 rows
// of the reduced system (width id kNmReduced16).
#include "phc_track.cuh"

PHC_DEFINE_NM(17)
