/*
 * Test infrastructure only (oracle). The subset of the FFTW3 API that the
 * reference's src/common/fourier.cpp and src/common/checkcode.cpp call,
 * implemented over a small mixed-radix FFT in minifft.cpp. Conventions follow
 * FFTW: row-major n0 x n1 x n2 (n2 fastest), unnormalised transforms, the
 * forward sign is -1, r2c keeps n2/2+1 entries of the last dimension.
 */
#ifndef ISDF_ORACLE_SHIM_FFTW3_H
#define ISDF_ORACLE_SHIM_FFTW3_H

typedef double fftw_complex[2];
typedef struct isdf_minifft_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_UNALIGNED (1U << 1)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#endif
