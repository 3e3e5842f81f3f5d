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
// spectrum (already scaled by 1/(M nx), natural order) is built once on the
// host in double precision.
//
// Per row pair: rows r and r+1 become the real and imaginary parts of one
// complex sequence of M points in shared memory, transformed by a Stockham
// autosort FFT, multiplied by the spectrum and transformed back; both rows
// come out filtered at once because the kernel is real.  Each thread holds
// 16 P points in registers per pass (P = 1, or 2 for M = 16384 so that the
// block stays at 512 threads): radix-16 passes, after one radix-2/4/8 pass
// when log2 M is not a multiple of 4, so M = 4096 takes 3 passes each way.
// A pass is a shared-memory load, a barrier, twiddles and 16-point DFTs in
// registers, and a store.  Shared memory holds one pad entry after every 16
// points, which spreads the strided stores of the early passes over all
// banks.  Twiddles come from per-pass tables, [r - 1][k] for the radix-16
// pass with sub-transform size Ns (e^{-2 pi i r k / (16 Ns)}), read through
// L1 with consecutive threads on consecutive entries.  CTAs are persistent
// and loop over row pairs; the next pair's rows are copied into shared memory
// by asynchronous copies while the current pair is transformed, so the
// padding step reads shared memory only.
#include <cuda_runtime.h>

#include <algorithm>

#include "tr_filter_host.h"
#include "tr_internal.cuh"

namespace trb {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Shared-memory slot of point i: one pad entry after every 16 points.
__device__ __forceinline__ int fft_slot(int i) { return i + (i >> 4); }

// e^{DIR 2 pi i m / 16} for a compile-time m (after unrolling).
template <int DIR>
__device__ __forceinline__ float2 w16(int m) {
  constexpr float c[16] = {1.f, 0.92387953f, 0.70710678f, 0.38268343f, 0.f, -0.38268343f,
                           -0.70710678f, -0.92387953f, -1.f, -0.92387953f, -0.70710678f,
                           -0.38268343f, 0.f, 0.38268343f, 0.70710678f, 0.92387953f};
  m &= 15;
  return make_float2(c[m], (float)DIR * c[(m + 12) & 15]);  // sin(x) = cos(x - pi/2)
}

template <int DIR>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  const float2 y0 = cadd(a0, a2), y1 = csub(a0, a2), y2 = cadd(a1, a3), d = csub(a1, a3);
  const float2 y3 = DIR < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);  // DIR i d
  a0 = cadd(y0, y2);
  a1 = cadd(y1, y3);
  a2 = csub(y0, y2);
  a3 = csub(y1, y3);
}

// In-place R-point DFT of v[0..R) (R = 2, 4, 8, 16; sign DIR); output X[r]
// ends at v[dft_pos<R>(r)]: (R/4) (r % 4) + r / 4 for R = 8, 16 and r
// otherwise (Cooley-Tukey with n = (R/4) n1 + n2, k = k1 + 4 k2).
template <int R>
__device__ __forceinline__ constexpr int dft_pos(int r) {
  return R >= 8 ? (R / 4) * (r % 4) + r / 4 : r;
}
template <int R, int DIR>
__device__ __forceinline__ void dft_r(float2 *v) {
  if (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    dft4<DIR>(v[0], v[1], v[2], v[3]);
  } else {
    constexpr int Q = R / 4;  // 2 or 4
#pragma unroll
    for (int n2 = 0; n2 < Q; ++n2) dft4<DIR>(v[n2], v[Q + n2], v[2 * Q + n2], v[3 * Q + n2]);
    // now v[n2 + Q k1] = Y[n2][k1]; twiddle by e^{DIR 2 pi i n2 k1 / R}
#pragma unroll
    for (int n2 = 1; n2 < Q; ++n2)
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) v[n2 + Q * k1] = cmul(v[n2 + Q * k1], w16<DIR>(n2 * k1 * (16 / R)));
    // DFT over n2 for each k1: X[k1 + 4 k2] = sum_n2 Y[n2][k1] W_Q^{n2 k2}
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 *y = v + Q * k1;
      if (Q == 2) {
        const float2 a = y[0], b = y[1];
        y[0] = cadd(a, b);
        y[1] = csub(a, b);
      } else {
        dft4<DIR>(y[0], y[1], y[2], y[3]);
      }
    }
  }
}

// One Stockham pass of radix R over the M = 2^log2m points in buf, with
// sub-transform size Ns = 2^log2ns: butterfly j reads points j + r M/R,
// multiplies point r by w^{r (j mod Ns)} with w = e^{DIR 2 pi i / (Ns R)},
// transforms the R points and writes point r to (j / Ns) Ns R + (j mod Ns) +
// r Ns.  Each thread takes 16 P / R butterflies j = tid + b blockDim.x
// (blockDim.x = M / (16 P) exactly).  tw: this pass's table, [r - 1][k] for
// k < Ns (radix 16 only; passes with Ns = 1 have no twiddles).
template <int R, int DIR, int P>
__device__ __forceinline__ void stockham_pass(float2 *buf, int log2m, int log2ns,
                                              const float2 *__restrict__ tw) {
  constexpr int B = 16 * P / R;
  constexpr int lr = R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1;
  const int nb = (1 << log2m) >> lr, Ns = 1 << log2ns;
  float2 v[16 * P];
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int j = threadIdx.x + b * blockDim.x;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = buf[fft_slot(j + r * nb)];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; ++b) {
    const int j = threadIdx.x + b * blockDim.x;
    const int k = j & (Ns - 1);
    if (R == 16 && log2ns > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(tw + (r - 1) * Ns + k);
        if (DIR > 0) w.y = -w.y;
        v[b * R + r] = cmul(v[b * R + r], w);
      }
    }
    dft_r<R, DIR>(v + b * R);
    const int base = ((j - k) << lr) + k;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[fft_slot(base + r * Ns)] = v[b * R + dft_pos<R>(r)];
  }
  __syncthreads();
}

// R0: radix of the first pass (2, 4 or 8 = 2^(log2m mod 4)), or 16 when
// log2m is a multiple of 4.  A template parameter rather than a switch: one
// code path per instantiation keeps the register allocation at one pass's.
template <int DIR, int P, int R0>
__device__ __forceinline__ void stockham_fft(float2 *buf, int log2m, const float2 *tw) {
  int ls = 0;
  if (R0 < 16) {
    stockham_pass<R0, DIR, P>(buf, log2m, 0, tw);
    ls = log2m & 3;
  }
  for (; ls < log2m; ls += 4) {
    stockham_pass<16, DIR, P>(buf, log2m, ls, tw);
    if (ls > 0) tw += 15 << ls;
  }
}

__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(float *dst, const float *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Starts copying row pair `pair` (one row when the second is absent) into the
// staging area: 16-byte pieces when the rows allow, else 4-byte ones.
__device__ __forceinline__ void stage_rows(const FilterArgs &f, long long pair, float *dst,
                                           bool vec) {
  const long long r0 = 2 * pair;
  const int n = (r0 + 1 < f.nrows ? 2 : 1) * f.nx;
  const float *src = f.rows + r0 * f.nx;
  if (vec) {
    for (int i = 4 * threadIdx.x; i < n; i += 4 * blockDim.x) cp_async16(dst + i, src + i);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) cp_async4(dst + i, src + i);
  }
  cp_async_commit();
}

// Float2 offset of the row staging area (2 nx floats, 16-byte aligned) after
// the M padded points.
__host__ __device__ __forceinline__ int rweight_stage_offset(int M) {
  return (M + M / 16 + 1) & ~1;
}

template <int P, int R0>
__global__ void __launch_bounds__(512) rweight_kernel(const FilterArgs f) {
  extern __shared__ float2 buf[];
  const int M = 1 << f.log2m;
  const long long npairs = (f.nrows + 1) / 2;
  const int nx = f.nx, N = f.n_pad;
  const int nxp = N - nx + 1;
  float *stage = reinterpret_cast<float *>(buf + rweight_stage_offset(M));
  const bool vec = (nx & 3) == 0 && (reinterpret_cast<uintptr_t>(f.rows) & 15) == 0;
  // The next pair's rows are copied in while this pair is transformed.
  if (blockIdx.x < npairs) stage_rows(f, blockIdx.x, stage, vec);
  for (long long pair = blockIdx.x; pair < npairs; pair += gridDim.x) {
    const long long r0 = 2 * pair;
    const bool has1 = r0 + 1 < f.nrows;
    cp_async_wait_all();
    __syncthreads();
    const float *x0 = stage;
    const float *x1 = has1 ? x0 + nx : nullptr;
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
      buf[fft_slot(j)] = make_float2(re, im);
    }
    __syncthreads();
    if (pair + gridDim.x < npairs) stage_rows(f, pair + gridDim.x, stage, vec);
    stockham_fft<-1, P, R0>(buf, f.log2m, f.tw);
    for (int j = threadIdx.x; j < M; j += blockDim.x)
      buf[fft_slot(j)] = cmul(buf[fft_slot(j)], __ldg(f.ghat + j));
    __syncthreads();
    stockham_fft<1, P, R0>(buf, f.log2m, f.tw);
    float *y0 = f.rows + r0 * f.nx;
    for (int j = threadIdx.x; j < nx; j += blockDim.x) {
      const float2 z = buf[fft_slot(j)];
      y0[j] = z.x;
      if (has1) y0[f.nx + j] = z.y;
    }
    __syncthreads();  // buf is reused by the next pair
  }
}

template <int P, int R0>
static cudaError_t launch_rweight_p(const FilterArgs &f, cudaStream_t s) {
  const int M = 1 << f.log2m;
  const size_t smem =
      (size_t)rweight_stage_offset(M) * sizeof(float2) + 2 * (size_t)f.nx * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(
      rweight_kernel<P, R0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long pairs = (f.nrows + 1) / 2;
  const int threads = M / (16 * P);
  int dev = 0, nsm = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rweight_kernel<P, R0>, threads, smem);
  const long long grid = std::min<long long>(pairs, (long long)nsm * std::max(1, per_sm));
  rweight_kernel<P, R0><<<(unsigned)std::max<long long>(1, grid), threads, smem, s>>>(f);
  return cudaGetLastError();
}

cudaError_t launch_rweight(const FilterArgs &f, cudaStream_t s) {
  if (f.log2m < kRweightMinLog2 || f.log2m > kRweightMaxLog2) return cudaErrorInvalidValue;
  if (f.log2m == 14) return launch_rweight_p<2, 4>(f, s);
  switch (f.log2m & 3) {
    case 1: return launch_rweight_p<1, 2>(f, s);
    case 2: return launch_rweight_p<1, 4>(f, s);
    case 3: return launch_rweight_p<1, 8>(f, s);
    default: return launch_rweight_p<1, 16>(f, s);
  }
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
