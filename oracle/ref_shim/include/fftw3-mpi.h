/* Declarations of the fftw3-mpi calls the reference makes (FFTW 3.3 MPI API), over the one-rank
   MPI stand-in: one rank holds the whole grid.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_FFTW3_MPI_H
#define RG_SHIM_FFTW3_MPI_H
#include <stddef.h>
#include "fftw3.h"
#include "mpi.h"
#ifdef __cplusplus
extern "C" {
#endif

void fftwf_mpi_init(void);
void fftwf_mpi_cleanup(void);
ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm, ptrdiff_t* local_n0,
                                  ptrdiff_t* local_0_start);
fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, float* in, fftwf_complex* out,
                                     MPI_Comm comm, unsigned flags);
fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftwf_complex* in, float* out,
                                     MPI_Comm comm, unsigned flags);
void fftwf_mpi_gather_wisdom(MPI_Comm comm);
void fftwf_mpi_broadcast_wisdom(MPI_Comm comm);

#ifdef __cplusplus
}
#endif
#endif
