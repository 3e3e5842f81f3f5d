/* CPU restatement of the reference TiltRec path (the oracle).
 * TEST INFRASTRUCTURE: see tiltrec_oracle.h for who may load it and how it
 * is pinned against the reference. */
#include "tiltrec_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* PI_180 and D2R exactly as main/main-mpi.cpp:9,15 (a float constant, so the
 * degree-to-radian product is formed in float). */
#define ORC_PI_180 0.01745329252f

/* TranslateAngleToCoefficients (main/main-mpi.cpp:85-106) followed by the
 * linear part of DecorateCoefficients (:110-183).  The reference also carries
 * quadratic terms a[4..9], b[4..9]; they start at zero and every decorated
 * quadratic term is a sum of products of them, so they stay zero and the
 * z-shift step reduces to the terms kept here. */
void orc_coeffs(const float *angles, int nt, float offset, float pitch,
                float zshift, double *out) {
  const double alpha = -(pitch * ORC_PI_180), beta = offset * ORC_PI_180,
               t = -zshift;
  const double ca = cos(alpha), sa = sin(alpha), cb = cos(beta),
               sb = sin(beta);
  for (int i = 0; i < nt; ++i) {
    /* The reference calls cos/sin on a float argument, which in C++ selects
     * the float overloads: the angle terms carry float precision. */
    const float tb = angles[i] * ORC_PI_180;
    double a[4] = {0, cosf(tb), 0, -sinf(tb)};
    double b[4] = {0, 0, 1, 0};
    double A[4], B[4];
    A[0] = a[0];
    A[1] = (a[2] * sa * sb + a[3] * ca * sb + a[1] * cb);
    A[2] = (a[2] * ca - a[3] * sa);
    A[3] = (a[3] * ca * cb + a[2] * cb * sa - a[1] * sb);
    B[0] = b[0];
    B[1] = (b[2] * sa * sb + b[3] * ca * sb + b[1] * cb);
    B[2] = (b[2] * ca - b[3] * sa);
    B[3] = (b[3] * ca * cb + b[2] * cb * sa - b[1] * sb);
    /* z shift (:167-182) with the quadratic terms equal to zero */
    double *o = out + 8 * (size_t)i;
    o[0] = A[0] + A[3] * t + 0.0 * t * t;
    o[1] = A[1] + 0.0 * t;
    o[2] = A[2] + 0.0 * t;
    o[3] = A[3] + 2 * 0.0 * t;
    o[4] = B[0] + B[3] * t + 0.0 * t * t;
    o[5] = B[1] + 0.0 * t;
    o[6] = B[2] + 0.0 * t;
    o[7] = B[3] + 2 * 0.0 * t;
  }
}

/* R-weighting filter, mode 2 (filter/filter_prj.cpp:636-736).
 * Per row: pad from nx to N = nx + nx/10 samples with a linear ramp running
 * from the last sample back to the first (buf2fft_padding_1D, :652-672),
 * weight the half spectrum by W[k] (k=0: 0.2; k<=r: k; else
 * r*exp(-(k-r)^2/sigma^2), r = floor(N*0.05f), sigma = N*0.5f; :694-723),
 * inverse transform without normalisation, keep the first nx samples and
 * divide by nx (:726-731).  Forward transform, weighting and unnormalised
 * inverse together are a circular convolution of the padded row with
 * h[d] = sum_k W_sym[k] cos(2 pi k d / N); it is evaluated here directly in
 * double precision. */
void orc_filter_rweight(int nx, long nrows, float *rows) {
  const int N = nx + nx / 10;
  const int nxp = N - nx + 1;
  const int r = (int)floor((float)N * 0.05f);
  const float sg = (float)N * 0.5f;
  const int nb = N / 2 + 1;
  double *W = (double *)malloc(sizeof(double) * nb);
  for (int k = 0; k < nb; ++k) {
    if (k == 0)
      W[k] = 0.2;
    else if (k <= r)
      W[k] = k;
    else
      W[k] = (double)(float)r *
             (double)expf(-(float)((k - r) * (k - r)) / (sg * sg));
  }
  double *cs = (double *)malloc(sizeof(double) * N);
  for (int j = 0; j < N; ++j) cs[j] = cos(2.0 * 3.14159265358979323846 * j / N);
  double *h = (double *)malloc(sizeof(double) * N);
  const int kmax = (N % 2 == 0) ? N / 2 - 1 : (N - 1) / 2;
  for (int d = 0; d < N; ++d) {
    double acc = W[0];
    for (int k = 1; k <= kmax; ++k) acc += 2.0 * W[k] * cs[(long)k * d % N];
    if (N % 2 == 0) acc += (d % 2 == 0) ? W[N / 2] : -W[N / 2];
    h[d] = acc;
  }
#pragma omp parallel
  {
    float *xp = (float *)malloc(sizeof(float) * N);
#pragma omp for schedule(static)
    for (long row = 0; row < nrows; ++row) {
      float *x = rows + (size_t)row * nx;
      for (int j = 0; j < nx; ++j) xp[j] = x[j];
      for (int j = nx; j < N; ++j)
        xp[j] = ((float)(j - nx + 1) / (float)nxp) * x[0] +
                ((float)(N - j) / (float)nxp) * x[nx - 1];
      for (int j = 0; j < nx; ++j) {
        double acc = 0;
        for (int m = 0; m < N; ++m) {
          int d = j - m;
          if (d < 0) d += N;
          acc += h[d] * (double)xp[m];
        }
        x[j] = (float)(acc / nx);
      }
    }
    free(xp);
  }
  free(W);
  free(cs);
  free(h);
}

#define PFX orc_
#define REAL float
#include "tiltrec_oracle_impl.h"
#undef PFX
#undef REAL

#define PFX orc64_
#define REAL double
#include "tiltrec_oracle_impl.h"
#undef PFX
#undef REAL

int orc_optimal_dft_size(int n) {
  for (int m = n > 1 ? n : 1;; ++m) {
    int r = m;
    while (r % 2 == 0) r /= 2;
    while (r % 3 == 0) r /= 3;
    while (r % 5 == 0) r /= 5;
    if (r == 1) return m;
  }
}

/* The filter kernels as filter_prj.cpp forms them (float arithmetic):
 * RamLak(251): n = -125..125, pi/4 at n = 0, -1/(pi n^2) at odd n, 0 at even
 * n (:137-155); SheppLogan(251): -2/(pi (4 n^2 - 1)) with float n (:158-178).
 *
 * FileterProjectionSymmetrize per row (the y padding rows are filtered and
 * cropped away, so rows are independent): the row is padded by one sample on
 * each side with its edge values (the 2-D symmetrisation about the centred
 * ROI, :301-316 with :209-263); that padded row of n = nx + 2 samples is
 * extended to L = optimal(251 + n - 1) by mirroring about its right end
 * (x[i] = x[2n - 1 - i], up to 2n, zeros beyond; :370-389); the kernel sits at
 * [0, 251) of an L-sample buffer; forward DFTs, a spectrum product and the
 * scaled inverse give the circular convolution y = kernel (*) x; samples
 * [125, 125 + n) of y are the filtered padded row (:397-401), whose centre
 * [1, 1 + nx) is the output (:403-413).  So out[i] = sum_k f[k] x[(126 + i -
 * k) mod L]. */
int orc_filter_fbp(int mode, int nx, long nrows, float *rows) {
  const int len = 251, half = len / 2;
  float f[251];
  if (mode == 1) {
    int n = -(len - 1) / 2;
    for (int i = 0; i < len; ++i, ++n) {
      if (n == 0)
        f[i] = (float)(3.14159265358979323846 / 4);
      else if (abs(n % 2) == 1)
        f[i] = (float)(-1.0 / (3.14159265358979323846 * n * n));
      else
        f[i] = 0;
    }
  } else {
    float n = -((float)len - 1.0f) / 2.0f;
    for (int i = 0; i < len; ++i) {
      f[i] = (float)(-2.0 / (3.14159265358979323846 * (4.0 * n * n - 1.0)));
      n = n + 1.0f;
    }
  }
  const int np = nx + 2;
  const int L = orc_optimal_dft_size(len + np - 1);
#pragma omp parallel
  {
    float *x = (float *)calloc((size_t)L, sizeof(float));
#pragma omp for schedule(static)
    for (long row = 0; row < nrows; ++row) {
      float *r = rows + (size_t)row * nx;
      for (int i = 0; i < L; ++i) x[i] = 0;
      x[0] = r[0];
      for (int i = 0; i < nx; ++i) x[1 + i] = r[i];
      x[np - 1] = r[nx - 1];
      const int end = np >= L - np ? L : 2 * np;
      for (int i = np; i < end; ++i) x[i] = x[2 * np - 1 - i];
      for (int i = 0; i < nx; ++i) {
        double acc = 0;
        for (int k = 0; k < len; ++k) {
          int m = (half + 1 + i - k) % L;
          if (m < 0) m += L;
          acc += (double)f[k] * (double)x[m];
        }
        r[i] = (float)acc;
      }
    }
    free(x);
  }
  return L;
}

/* Overlap weights of one axis: output cell d covers [d*scale, (d+1)*scale)
 * of n input pixels; w[k] is the covered part of input pixel first + k,
 * divided by the cell width (clipped at the image end). */
static int orc_area_axis(int n, int dn, int d, int *first, double *w) {
  const double scale = (double)n / dn;
  const double a = d * scale, b = a + scale > n ? (double)n : a + scale;
  const int i0 = (int)floor(a), i1 = (int)ceil(b);
  const double width = b - a;
  int k = 0;
  for (int i = i0; i < i1; ++i, ++k) {
    const double lo = i > a ? i : a, hi = i + 1 < b ? i + 1 : b;
    w[k] = (hi - lo) / width;
  }
  *first = i0;
  return k;
}

void orc_resample_bin(const float *src, int nx, int ny, int nt, int bin, float *dst) {
  const int dnx = nx / bin, dny = ny / bin;
  double *wx = (double *)malloc(sizeof(double) * (bin + 2));
  double *wy = (double *)malloc(sizeof(double) * (bin + 2));
  for (int t = 0; t < nt; ++t)
    for (int j = 0; j < dny; ++j) {
      int y0, x0;
      const int ky = orc_area_axis(ny, dny, j, &y0, wy);
      for (int i = 0; i < dnx; ++i) {
        const int kx = orc_area_axis(nx, dnx, i, &x0, wx);
        double acc = 0;
        for (int b = 0; b < ky; ++b) {
          const float *row = src + ((size_t)t * ny + y0 + b) * nx + x0;
          double r = 0;
          for (int a = 0; a < kx; ++a) r += wx[a] * (double)row[a];
          acc += wy[b] * r;
        }
        dst[((size_t)t * dny + j) * dnx + i] = (float)acc;
      }
    }
  free(wx);
  free(wy);
}
