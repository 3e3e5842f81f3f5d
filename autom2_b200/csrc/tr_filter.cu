// WBP R-weighting filter (filter/filter_prj.cpp:636-736, ApplyFilterInplace
// mode 2, :787-795) as one shared-memory FFT convolution per pair of rows.
//
// The reference pads each row of nx samples to N = nx + nx/10 with a linear
// ramp from the last sample back to the first, takes a real FFT of length N,
// scales bin k by W[k] (0.2 at k = 0, k up to r = floor(0.05 N), then a
// Gaussian roll-off r exp(-(k-r)^2 / (N/2)^2)), inverse transforms without
// normalisation, keeps the first nx samples and divides by nx.  That whole
// chain is a circular convolution of the padded row with a fixed real kernel
// h (length N).  N is generally not a power of two (281, 1126, 2252, 4505 for
// nx = 256..4096), so the circular convolution is evaluated as a linear one on
// a power-of-two length M >= N + nx - 1 with the kernel laid out for
// lags -(N-1)..nx-1; no wrap-around reaches the kept outputs.  The kernel's
// spectrum (already scaled by 1/(M nx) and permuted to bit-reversed order) is
// built once on the host in double precision.
//
// Per CTA: rows r and r+1 become the real and imaginary parts of one complex
// sequence of M points in shared memory; a Stockham autosort FFT (radix-4
// passes, one radix-2 pass first when log2 M is odd; each thread holds its
// butterflies' points in registers between a load and a store phase), a
// pointwise product with the spectrum, and the inverse transform give both
// filtered rows at once because the kernel is real.
#include <cuda_runtime.h>

#include <algorithm>

#include "tr_internal.cuh"

namespace trb {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

constexpr int kFftMaxB = 4;  // butterflies per thread and pass (launcher sizes the block)

// One Stockham pass of radix R over buf[0..M) (M = 2^log2m), sub-transform
// size Ns = 2^log2ns before the pass: butterfly j reads points j + r M/R,
// multiplies point r by w^{r (j mod Ns)} with w = e^{DIR 2 pi i / (Ns R)},
// transforms the R points and writes them to (j / Ns) Ns R + (j mod Ns) +
// r Ns.  DIR = -1 forward, +1 inverse (unscaled).  tw[t] = e^{-2 pi i t / M}.
template <int R, int DIR>
__device__ __forceinline__ void stockham_pass(float2 *buf, int log2m, int log2ns,
                                              const float2 *__restrict__ tw) {
  const int M = 1 << log2m, nb = M / R, Ns = 1 << log2ns;
  constexpr int lr = R == 4 ? 2 : 1;
  float2 v[kFftMaxB][R];
#pragma unroll
  for (int b = 0; b < kFftMaxB; ++b) {
    const int j = threadIdx.x + b * blockDim.x;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = buf[j + r * nb];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < kFftMaxB; ++b) {
    const int j = threadIdx.x + b * blockDim.x;
    if (j < nb) {
      const int k = j & (Ns - 1);
      const int step = k << (log2m - log2ns - lr);  // k M / (Ns R)
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(tw + ((r * step) & (M - 1)));
        if (DIR > 0) w.y = -w.y;
        v[b][r] = cmul(v[b][r], w);
      }
      float2 o[R];
      if (R == 2) {
        o[0] = cadd(v[b][0], v[b][1]);
        o[1] = csub(v[b][0], v[b][1]);
      } else {
        const float2 y0 = cadd(v[b][0], v[b][2]), y1 = csub(v[b][0], v[b][2]);
        const float2 y2 = cadd(v[b][1], v[b][3]), d = csub(v[b][1], v[b][3]);
        // forward: -i d; inverse: +i d
        const float2 y3 = DIR < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
        o[0] = cadd(y0, y2);
        o[1] = cadd(y1, y3);
        o[2] = csub(y0, y2);
        o[3] = csub(y1, y3);
      }
      const int base = ((j - k) << lr) + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[base + r * Ns] = o[r];
    }
  }
  __syncthreads();
}

template <int DIR>
__device__ __forceinline__ void stockham_fft(float2 *buf, int log2m, const float2 *tw) {
  int ls = 0;
  if (log2m & 1) {
    stockham_pass<2, DIR>(buf, log2m, 0, tw);
    ls = 1;
  }
  for (; ls < log2m; ls += 2) stockham_pass<4, DIR>(buf, log2m, ls, tw);
}

__global__ void __launch_bounds__(1024) rweight_kernel(const FilterArgs f) {
  extern __shared__ float2 buf[];
  const int M = 1 << f.log2m;
  const long long r0 = 2ll * blockIdx.x;
  const bool has1 = r0 + 1 < f.nrows;
  const float *x0 = f.rows + r0 * f.nx;
  const float *x1 = has1 ? x0 + f.nx : nullptr;
  const int nx = f.nx, N = f.n_pad;
  const int nxp = N - nx + 1;
  const float a0 = x0[0], b0 = x0[nx - 1];
  const float a1 = has1 ? x1[0] : 0.f, b1 = has1 ? x1[nx - 1] : 0.f;

  // Padded rows (buf2fft_padding_1D, filter_prj.cpp:652-672), zero beyond N.
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    float re = 0.f, im = 0.f;
    if (j < nx) {
      re = x0[j];
      im = has1 ? x1[j] : 0.f;
    } else if (j < N) {
      const float wa = (float)(j - nx + 1) / (float)nxp;
      const float wb = (float)(N - j) / (float)nxp;
      re = wa * a0 + wb * b0;
      im = wa * a1 + wb * b1;
    }
    buf[j] = make_float2(re, im);
  }
  __syncthreads();
  stockham_fft<-1>(buf, f.log2m, f.tw);
  for (int j = threadIdx.x; j < M; j += blockDim.x) buf[j] = cmul(buf[j], __ldg(f.ghat + j));
  __syncthreads();
  stockham_fft<1>(buf, f.log2m, f.tw);
  float *y0 = f.rows + r0 * f.nx;
  for (int j = threadIdx.x; j < nx; j += blockDim.x) {
    const float2 z = buf[j];
    y0[j] = z.x;
    if (has1) y0[f.nx + j] = z.y;
  }
}

cudaError_t launch_rweight(const FilterArgs &f, cudaStream_t s) {
  const int M = 1 << f.log2m;
  const size_t smem = (size_t)M * sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(
      rweight_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long pairs = (f.nrows + 1) / 2;
  // At most kFftMaxB butterflies per thread in a radix-2 pass (M/2 of them).
  const int threads = std::min(1024, std::max(64, M / (2 * kFftMaxB)));
  rweight_kernel<<<(unsigned)pairs, threads, smem, s>>>(f);
  return cudaGetLastError();
}

// ------------------------------------------------------------- FBP filters
//
// FBP row filters, ApplyFilterInplace modes 0 (Shepp-Logan) and 1 (Ram-Lak)
// (filter/filter_prj.cpp:755-786): FileterProjectionSymmetrize (:265-446)
// convolves each row, padded by one edge sample on each side and extended by
// mirroring to the DFT length L = optimal(251 + nx + 1), with a 251-tap kernel
// through forward DFTs, a spectrum product and a scaled inverse, and keeps
// samples [126, 126 + nx) of the circular result.  That is
//   out[i] = sum_{k<251} f[k] x[(126 + i - k) mod L],
// evaluated here as a direct sum in double precision (251 products per
// output; the kernel's many small taps make float accumulation lose ~1e-6).
// One CTA per row: the row's extended samples e[t] = x[(t - 124) mod L],
// t in [0, nx + 250], and the taps live in shared memory.

constexpr int kFbpTaps = 251;

__global__ void __launch_bounds__(256) fbp_filter_kernel(float *rows, int nx, int L, int mode) {
  extern __shared__ double fsm[];
  double *f = fsm;                                     // [251]
  float *e = reinterpret_cast<float *>(fsm + kFbpTaps);  // [nx + 250]
  const int half = kFbpTaps / 2;
  for (int k = threadIdx.x; k < kFbpTaps; k += blockDim.x) {
    // The reference's kernels, formed in the same precision (:137-178).
    const double pi = 3.14159265358979323846;
    float v;
    if (mode == 1) {
      const int n = k - half;
      v = n == 0 ? (float)(pi / 4) : ((n % 2) != 0 ? (float)(-1.0 / (pi * n * n)) : 0.f);
    } else {
      const double n = (double)((float)(k - half));
      v = (float)(-2.0 / (pi * (4.0 * n * n - 1.0)));
    }
    f[k] = (double)v;
  }
  float *r = rows + (size_t)blockIdx.x * nx;
  const int np = nx + 2;
  const int end = np >= L - np ? L : 2 * np;  // mirrored extension, zeros after
  for (int t = threadIdx.x; t < nx + kFbpTaps - 1; t += blockDim.x) {
    int m = t - (half - 1);
    if (m < 0) m += L;
    // x[m] of the padded, extended row
    int src;  // index into the padded row [0, np)
    if (m < np) src = m;
    else if (m < end) src = 2 * np - 1 - m;
    else src = -1;
    float v = 0.f;
    if (src >= 0) v = r[min(max(src - 1, 0), nx - 1)];
    e[t] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    double acc = 0.0;
    const float *w = e + i + kFbpTaps - 1;
#pragma unroll 8
    for (int k = 0; k < kFbpTaps; ++k) acc = fma(f[k], (double)w[-k], acc);
    // All reads of the row precede this write: e is a private copy.
    r[i] = (float)acc;
  }
}

cudaError_t launch_fbp_filter(float *rows, long long nrows, int nx, int L, int mode,
                              cudaStream_t s) {
  const size_t smem = kFbpTaps * sizeof(double) + (size_t)(nx + kFbpTaps) * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(fbp_filter_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  for (long long r0 = 0; r0 < nrows; r0 += 2147483647ll) {
    const unsigned n = (unsigned)std::min<long long>(nrows - r0, 2147483647ll);
    fbp_filter_kernel<<<n, 256, smem, s>>>(rows + (size_t)r0 * nx, nx, L, mode);
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------ area binning
//
// The GUI chain's `resample -b bin` step before TiltRec
// (resample/src/main/main.cpp:14-58, 67-147) shrinks every image to
// (nx/bin) x (ny/bin) with OpenCV's area resize: output pixel (i, j) is the
// mean of the input over [i sx, (i+1) sx) x [j sy, (j+1) sy), sx = nx/(nx/bin),
// partial pixels weighted by their overlap (an exact block mean when bin
// divides the size).  One thread per output pixel, separable sums in FP64.

__device__ __forceinline__ int area_axis(int n, int dn, int d, int *first, double *w, int cap) {
  const double scale = (double)n / dn;
  const double a = d * scale, b = a + scale > n ? (double)n : a + scale;
  const int i0 = (int)floor(a), i1 = (int)ceil(b);
  const double width = b - a;
  int k = 0;
  for (int i = i0; i < i1 && k < cap; ++i, ++k) {
    const double lo = i > a ? i : a, hi = i + 1 < b ? i + 1 : b;
    w[k] = (hi - lo) / width;
  }
  *first = i0;
  return k;
}

constexpr int kBinMax = 64;  // largest bin factor (weights per axis: bin + 1)

__global__ void resample_bin_kernel(const float *__restrict__ src, int nx, int ny, int nt,
                                    int dnx, int dny, float *__restrict__ dst) {
  const size_t total = (size_t)dnx * dny * nt;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < total;
       o += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(o % dnx);
    const size_t jt = o / dnx;
    const int j = (int)(jt % dny), t = (int)(jt / dny);
    double wx[kBinMax + 2], wy[kBinMax + 2];
    int x0, y0;
    const int kx = area_axis(nx, dnx, i, &x0, wx, kBinMax + 2);
    const int ky = area_axis(ny, dny, j, &y0, wy, kBinMax + 2);
    double acc = 0.0;
    for (int b = 0; b < ky; ++b) {
      const float *row = src + ((size_t)t * ny + y0 + b) * nx + x0;
      double r = 0.0;
      for (int a = 0; a < kx; ++a) r += wx[a] * (double)row[a];
      acc += wy[b] * r;
    }
    dst[o] = (float)acc;
  }
}

cudaError_t launch_resample_bin(const float *src, int nx, int ny, int nt, int bin, float *dst,
                                cudaStream_t s) {
  const int dnx = nx / bin, dny = ny / bin;
  const size_t total = (size_t)dnx * dny * nt;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
  resample_bin_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(src, nx, ny, nt, dnx, dny, dst);
  return cudaGetLastError();
}

}  // namespace trb
