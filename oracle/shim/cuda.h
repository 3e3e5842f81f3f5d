/* Test-only empty stand-in for <cuda.h>: the reference filter source includes
 * it but calls nothing from it on the CPU path compiled into the oracle. */
#ifndef ORACLE_SHIM_CUDA_H
#define ORACLE_SHIM_CUDA_H
#endif
