/* Test-only: the host-process MPI stand-in (../shim/mpi.h) for the GPU build
 * of the reference executables, whose include path must reach the real
 * <cuda.h> and <cufftw.h> (the CPU build's shim directory replaces both). */
#include "../shim/mpi.h"
