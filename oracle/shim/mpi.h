/* Empty stand-in: the reference includes <mpi.h>
 * (include/Utils/PatchInterpolation.hpp:18) but never calls MPI.
 * Test infrastructure only, used to compile the reference oracle. */
#pragma once
