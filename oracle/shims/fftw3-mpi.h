/* Test infrastructure only (oracle): the reference includes this header but
 * calls nothing from it on the single-rank path. */
#ifndef ISDF_ORACLE_SHIM_FFTW3_MPI_H
#define ISDF_ORACLE_SHIM_FFTW3_MPI_H
#include "fftw3.h"
#endif
