// Test infrastructure only (oracle): a plain mixed-radix Cooley-Tukey FFT
// behind the FFTW3 subset declared in fftw3.h. It is written for clarity, not
// speed; the oracle only transforms grids of a few 10^4..10^5 points.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

typedef std::complex<double> cplx;

namespace {

// Unnormalised 1-D DFT of x (length n, stride 1) with exponent sign*2*pi*i*jk/n.
void fft1d(cplx* x, int n, int sign, std::vector<cplx>& scratch) {
  if (n <= 1) return;
  int p = 0;
  for (int f = 2; f * f <= n; ++f)
    if (n % f == 0) { p = f; break; }
  const double two_pi = 6.283185307179586476925286766559;
  if (p == 0) {  // prime length: direct sum
    std::vector<cplx> out(n);
    for (int k = 0; k < n; ++k) {
      cplx acc(0.0, 0.0);
      for (int j = 0; j < n; ++j) {
        long long e = (long long)j * k % n;
        double ang = sign * two_pi * (double)e / n;
        acc += x[j] * cplx(std::cos(ang), std::sin(ang));
      }
      out[k] = acc;
    }
    for (int k = 0; k < n; ++k) x[k] = out[k];
    return;
  }
  const int m = n / p;
  // Decimation in time: p sub-sequences x[r], x[r+p], ... each of length m.
  std::vector<cplx> sub((size_t)n);
  for (int r = 0; r < p; ++r)
    for (int j = 0; j < m; ++j) sub[(size_t)r * m + j] = x[(size_t)j * p + r];
  for (int r = 0; r < p; ++r) fft1d(&sub[(size_t)r * m], m, sign, scratch);
  for (int k = 0; k < n; ++k) {
    cplx acc(0.0, 0.0);
    for (int r = 0; r < p; ++r) {
      long long e = (long long)r * k % n;
      double ang = sign * two_pi * (double)e / n;
      acc += sub[(size_t)r * m + (k % m)] * cplx(std::cos(ang), std::sin(ang));
    }
    x[k] = acc;
  }
}

void fft3d(cplx* a, int n0, int n1, int n2, int sign) {
  std::vector<cplx> line, scratch;
  const size_t s1 = (size_t)n2, s0 = (size_t)n1 * n2;
  line.resize((size_t)std::max(n0, std::max(n1, n2)));
  for (int i0 = 0; i0 < n0; ++i0)
    for (int i1 = 0; i1 < n1; ++i1) fft1d(a + i0 * s0 + i1 * s1, n2, sign, scratch);
  for (int i0 = 0; i0 < n0; ++i0)
    for (int i2 = 0; i2 < n2; ++i2) {
      for (int i1 = 0; i1 < n1; ++i1) line[i1] = a[i0 * s0 + i1 * s1 + i2];
      fft1d(line.data(), n1, sign, scratch);
      for (int i1 = 0; i1 < n1; ++i1) a[i0 * s0 + i1 * s1 + i2] = line[i1];
    }
  for (int i1 = 0; i1 < n1; ++i1)
    for (int i2 = 0; i2 < n2; ++i2) {
      for (int i0 = 0; i0 < n0; ++i0) line[i0] = a[i0 * s0 + i1 * s1 + i2];
      fft1d(line.data(), n0, sign, scratch);
      for (int i0 = 0; i0 < n0; ++i0) a[i0 * s0 + i1 * s1 + i2] = line[i0];
    }
}

}  // namespace

struct isdf_minifft_plan {
  int kind;  // 0 complex, 1 r2c, 2 c2r
  int n0, n1, n2, sign;
  void* in;
  void* out;
};

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned) {
  return new isdf_minifft_plan{0, n0, n1, n2, sign, in, out};
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned) {
  return new isdf_minifft_plan{1, n0, n1, n2, FFTW_FORWARD, in, out};
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned) {
  return new isdf_minifft_plan{2, n0, n1, n2, FFTW_BACKWARD, in, out};
}
void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2;
  const size_t n = (size_t)n0 * n1 * n2;
  const int h2 = n2 / 2 + 1;
  std::vector<cplx> a(n);
  if (p->kind == 0) {
    std::memcpy(a.data(), p->in, n * sizeof(cplx));
    fft3d(a.data(), n0, n1, n2, p->sign);
    std::memcpy(p->out, a.data(), n * sizeof(cplx));
  } else if (p->kind == 1) {
    const double* in = (const double*)p->in;
    for (size_t i = 0; i < n; ++i) a[i] = cplx(in[i], 0.0);
    fft3d(a.data(), n0, n1, n2, FFTW_FORWARD);
    cplx* out = (cplx*)p->out;
    for (int i0 = 0; i0 < n0; ++i0)
      for (int i1 = 0; i1 < n1; ++i1)
        for (int i2 = 0; i2 < h2; ++i2)
          out[((size_t)i0 * n1 + i1) * h2 + i2] = a[((size_t)i0 * n1 + i1) * n2 + i2];
  } else {
    const cplx* in = (const cplx*)p->in;
    for (int i0 = 0; i0 < n0; ++i0)
      for (int i1 = 0; i1 < n1; ++i1)
        for (int i2 = 0; i2 < n2; ++i2) {
          if (i2 < h2) {
            a[((size_t)i0 * n1 + i1) * n2 + i2] = in[((size_t)i0 * n1 + i1) * h2 + i2];
          } else {
            int j0 = (n0 - i0) % n0, j1 = (n1 - i1) % n1, j2 = n2 - i2;
            a[((size_t)i0 * n1 + i1) * n2 + i2] = std::conj(in[((size_t)j0 * n1 + j1) * h2 + j2]);
          }
        }
    fft3d(a.data(), n0, n1, n2, FFTW_BACKWARD);
    double* out = (double*)p->out;
    for (size_t i = 0; i < n; ++i) out[i] = a[i].real();
  }
}
