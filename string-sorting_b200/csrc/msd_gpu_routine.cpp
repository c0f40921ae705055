// msd_gpu_routine.cpp -- registers the B200 sort as one more routine of the
// reference's registry.  This file is compiled against the reference's own
// routine.h (rantala/string-sorting src/routine.h) and linked into its
// sortstring and unit-test programs together with libssort_b200.so; it is the
// only piece a maintainer adds to the reference's source lists.
//
// ROUTINE_REGISTER_SINGLECORE (src/routine.h:55-56) builds a static
// struct routine {f = msd_gpu, name = "msd_gpu", ...} and registers it from a
// load-time constructor, exactly as src/msd_ce.cpp:418-419 registers msd_CE6.
#include "routine.h"
#include "ssort_b200.h"

ROUTINE_REGISTER_SINGLECORE(msd_gpu,
	"B200 GPU MSD radix sort: 16-byte keys per round, sample partition + on-chip segment sorts")
