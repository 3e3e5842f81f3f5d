// Host-side construction of the R-weighting filter's kernel spectrum
// (ApplyFilterInplace mode 2, filter/filter_prj.cpp:674-736): the filter is
// applied on the device as a linear convolution through a power-of-two FFT,
// whose kernel spectrum is formed here in double precision.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace trb {

// Iterative radix-2 FFT in double (host), forward sign -1.
inline void fft_host(std::vector<std::complex<double>> &x) {
  const size_t n = x.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * M_PI / (double)len;
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        const std::complex<double> w(cos(ang * k), sin(ang * k));
        const std::complex<double> u = x[i + k], v = x[i + k + len / 2] * w;
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
  }
}

// FFT sizes the device filter handles: M = 2^4 .. 2^14 (nx up to about 7800).
constexpr int kRweightMinLog2 = 4;
constexpr int kRweightMaxLog2 = 14;

struct RweightSpectrum {
  int npad = 0;   // padded row length nx + nx/10 of the reference
  int log2m = 0;  // FFT size 2^log2m >= npad + nx - 1
  std::vector<float2> ghat;  // kernel spectrum, natural order, scaled 1/(M nx)
  // Twiddles of the radix-16 Stockham passes with sub-transform size
  // Ns = 2^ls > 1 (ls = log2m mod 4, then every 4th value below log2m), one
  // table per pass in that order: entry [r - 1][k] = e^{-2 pi i r k / (16 Ns)}
  // for r = 1..15, k < Ns.
  std::vector<float2> tw;
};

// False when the FFT (M points plus one pad entry per 16) would not fit
// `smem_max` bytes of shared memory.
inline bool rweight_spectrum(int nx, size_t smem_max, RweightSpectrum *out) {
  const int N = nx + nx / 10;
  int log2m = kRweightMinLog2;
  while ((1 << log2m) < N + nx - 1) ++log2m;
  const int M = 1 << log2m;
  out->npad = N;
  out->log2m = log2m;
  if ((size_t)(M + M / 16) * sizeof(float2) > smem_max || log2m > kRweightMaxLog2) return false;
  // Weights exactly as filter_prj.cpp:694-723 forms them (float arithmetic).
  const int r = (int)floor((float)N * 0.05f);
  const float sg = (float)N * 0.5f;
  const int nb = N / 2 + 1;
  std::vector<double> W(nb);
  for (int k = 0; k < nb; ++k) {
    if (k == 0)
      W[k] = 0.2;
    else if (k <= r)
      W[k] = k;
    else
      W[k] = (double)(float)r * (double)expf(-(float)((k - r) * (k - r)) / (sg * sg));
  }
  // h[d] = sum over the Hermitian-extended spectrum of W cos(2 pi k d / N).
  std::vector<double> cs(N), h(N);
  for (int j = 0; j < N; ++j) cs[j] = cos(2.0 * M_PI * j / N);
  const int kmax = (N % 2 == 0) ? N / 2 - 1 : (N - 1) / 2;
  for (int d = 0; d < N; ++d) {
    double acc = W[0];
    for (int k = 1; k <= kmax; ++k) acc += 2.0 * W[k] * cs[(long long)k * d % N];
    if (N % 2 == 0) acc += (d % 2 == 0) ? W[N / 2] : -W[N / 2];
    h[d] = acc;
  }
  std::vector<std::complex<double>> g(M, 0.0);
  for (int e = -(N - 1); e <= nx - 1; ++e) g[(e % M + M) % M] = h[(e % N + N) % N];
  fft_host(g);
  out->ghat.resize(M);
  const double scale = 1.0 / ((double)M * nx);
  for (int i = 0; i < M; ++i)
    out->ghat[i] = make_float2((float)(g[i].real() * scale), (float)(g[i].imag() * scale));
  out->tw.clear();
  for (int ls = log2m & 3; ls < log2m; ls += 4) {
    if (ls == 0) continue;
    const int ns = 1 << ls;
    for (int r = 1; r < 16; ++r)
      for (int k = 0; k < ns; ++k) {
        const double a = -2.0 * M_PI * r * k / (16.0 * ns);
        out->tw.push_back(make_float2((float)cos(a), (float)sin(a)));
      }
  }
  if (out->tw.empty()) out->tw.push_back(make_float2(1.f, 0.f));  // keep the buffer non-empty
  return true;
}

}  // namespace trb
