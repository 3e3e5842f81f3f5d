/* Test-only stand-in for <cufftw.h> (the FFTW3 single-precision API that the
 * reference WBP filter calls, filter/filter_prj.cpp:683-692, 725).
 *
 * The reference links NVIDIA's cufftw, i.e. its R-weighting filter runs its
 * FFTs on the GPU.  The oracle build replaces the five entry points it uses
 * with an exact real DFT evaluated in double precision on the host
 * (oracle/shim/fftw_dft.cpp), so the reference CPU path runs without a GPU.
 * Only the semantics the reference relies on are implemented: 1-D transforms,
 * howmany batches, element strides and batch distances, unnormalised c2r that
 * ignores the imaginary parts of the DC and (even N) Nyquist bins. */
#ifndef ORACLE_SHIM_CUFFTW_H
#define ORACLE_SHIM_CUFFTW_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct oracle_fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                   float *in, const int *inembed, int istride,
                                   int idist, fftwf_complex *out,
                                   const int *onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                   fftwf_complex *in, const int *inembed,
                                   int istride, int idist, float *out,
                                   const int *onembed, int ostride, int odist,
                                   unsigned flags);
void fftwf_execute(const fftwf_plan plan);
void fftwf_destroy_plan(fftwf_plan plan);

#ifdef __cplusplus
}
#endif
#endif
