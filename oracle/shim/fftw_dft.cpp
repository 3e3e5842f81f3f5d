// Host implementation of the FFTW entry points declared in shim/cufftw.h.
// Oracle infrastructure: an exact O(N^2) real DFT in double precision,
// threaded over the batch ("howmany") dimension.
#include "cufftw.h"

#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <thread>
#include <vector>

struct oracle_fftwf_plan_s {
  int r2c;  // 1: real -> half complex, 0: half complex -> real
  int n, howmany;
  float *rbuf;
  fftwf_complex *cbuf;
  int rstride, rdist, cstride, cdist;
};

namespace {

// Twiddles e^{-2 pi i j / n} for j in [0, n), computed in double.
void twiddles(int n, std::vector<double> &c, std::vector<double> &s) {
  c.resize(n);
  s.resize(n);
  const double w = 2.0 * 3.14159265358979323846 / n;
  for (int j = 0; j < n; ++j) {
    c[j] = cos(w * j);
    s[j] = -sin(w * j);
  }
}

void run_rows(const oracle_fftwf_plan_s *p, int b0, int b1,
              const std::vector<double> &c, const std::vector<double> &s) {
  const int n = p->n, nb = n / 2 + 1;
  std::vector<double> tmp(2 * (size_t)std::max(n, nb));
  for (int b = b0; b < b1; ++b) {
    float *r = p->rbuf + (size_t)b * p->rdist;
    fftwf_complex *z = p->cbuf + (size_t)b * p->cdist;
    if (p->r2c) {
      for (int k = 0; k < nb; ++k) {
        double re = 0, im = 0;
        for (int m = 0; m < n; ++m) {
          const int j = (int)(((long long)k * m) % n);
          const double x = r[(size_t)m * p->rstride];
          re += x * c[j];
          im += x * s[j];
        }
        tmp[2 * k] = re;
        tmp[2 * k + 1] = im;
      }
      for (int k = 0; k < nb; ++k) {
        z[(size_t)k * p->cstride][0] = (float)tmp[2 * k];
        z[(size_t)k * p->cstride][1] = (float)tmp[2 * k + 1];
      }
    } else {
      // y[m] = sum_k Y[k] e^{+2 pi i k m / n} with Hermitian symmetry.
      const int kmax = (n % 2 == 0) ? n / 2 - 1 : (n - 1) / 2;
      for (int m = 0; m < n; ++m) {
        double acc = z[0][0];
        for (int k = 1; k <= kmax; ++k) {
          const int j = (int)(((long long)k * m) % n);
          const double yr = z[(size_t)k * p->cstride][0];
          const double yi = z[(size_t)k * p->cstride][1];
          // Re(Y e^{+i t}) with e^{+i t} = (c, -s)
          acc += 2.0 * (yr * c[j] + yi * s[j]);
        }
        if (n % 2 == 0) {
          const double yr = z[(size_t)(n / 2) * p->cstride][0];
          acc += (m % 2 == 0) ? yr : -yr;
        }
        tmp[m] = acc;
      }
      for (int m = 0; m < n; ++m) r[(size_t)m * p->rstride] = (float)tmp[m];
    }
  }
}

}  // namespace

extern "C" {

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                   float *in, const int *, int istride,
                                   int idist, fftwf_complex *out, const int *,
                                   int ostride, int odist, unsigned) {
  if (rank != 1) abort();
  oracle_fftwf_plan_s *p = new oracle_fftwf_plan_s;
  *p = {1, n[0], howmany, in, out, istride, idist, ostride, odist};
  return p;
}

fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                   fftwf_complex *in, const int *, int istride,
                                   int idist, float *out, const int *,
                                   int ostride, int odist, unsigned) {
  if (rank != 1) abort();
  oracle_fftwf_plan_s *p = new oracle_fftwf_plan_s;
  *p = {0, n[0], howmany, out, in, ostride, odist, istride, idist};
  return p;
}

void fftwf_execute(const fftwf_plan p) {
  std::vector<double> c, s;
  twiddles(p->n, c, s);
  int nt = (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, p->howmany));
  std::vector<std::thread> th;
  const int per = (p->howmany + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int b0 = t * per, b1 = std::min(p->howmany, b0 + per);
    if (b0 >= b1) break;
    th.emplace_back(run_rows, p, b0, b1, std::cref(c), std::cref(s));
  }
  for (auto &x : th) x.join();
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }

}  // extern "C"
