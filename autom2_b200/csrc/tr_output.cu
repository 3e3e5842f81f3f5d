// Byte output of a reconstruction (--f2b) on the device.
//
// The reference maps its volume to bytes slab by slab on the GPU
// (TiltRec_cuda_y/recon_y.cu:164-181 with CufloatToByteKernel,
// basic.cu:442-475): for each slab of the volume it takes the slab's mean and
// standard deviation, folds them into exponentially averaged values
// (alpha 0.9, both starting at 0; the Z-layout drivers take the whole volume
// as one slab with its own statistics, alpha 0, TiltRec_cuda_z/recon_z.cu:
// 164-172), and maps every value of each complete group of four to
// (clamp((v - mean) / std, -10, 10) + 10) / 20 * 255, truncated to an
// unsigned byte.  Here the slab statistics are sums in FP64 over fixed
// partitions of each slab, added in a fixed order, so the bytes are the same
// from run to run; the mean is the float of sum / n, the deviation the float
// square root of the FP64 sum of the float squares of (v - mean), as the
// drop-in executables compute them on the host.
#include <cuda_runtime.h>
#include <math.h>

#include "tr_internal.cuh"

namespace trb {

// Per slab s and part b: the part's sum of x (pass 0) or of the float
// (x - mean[s])^2 (pass 1), in FP64.  grid = (kF2bParts, nslabs), 256 threads.
__global__ void f2b_partials_kernel(const float *__restrict__ v, size_t n, size_t slab,
                                    const float *__restrict__ mean, double *part, int pass) {
  const int s = blockIdx.y, b = blockIdx.x;
  const size_t s0 = (size_t)s * slab;
  const size_t len = min(slab, n - s0);
  const size_t per = (len + kF2bParts - 1) / kF2bParts;
  const size_t lo = min(len, (size_t)b * per), hi = min(len, lo + per);
  const float m = pass ? mean[s] : 0.f;
  double acc = 0.0;
  for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const float x = v[s0 + i];
    if (pass) {
      const float d = x - m;
      acc += (double)(d * d);
    } else {
      acc += (double)x;
    }
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(size_t)s * kF2bParts + b] = red[0];
}

// Pass 0, one thread per slab: the slab mean from its parts summed in order.
// Pass 1, one thread: each slab's deviation, and the exponential averages
// over the slabs in order (g = alpha g + (1 - alpha) stat) into gm / gs.
__global__ void f2b_slab_kernel(const double *part, size_t n, size_t slab, int nslabs,
                                float *mean, float *sd, float *gm, float *gs, float alpha,
                                int pass) {
  if (pass == 0) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslabs) return;
    const size_t len = min(slab, n - (size_t)s * slab);
    double acc = 0.0;
    for (int b = 0; b < kF2bParts; ++b) acc += part[(size_t)s * kF2bParts + b];
    mean[s] = (float)(acc / (double)len);
    return;
  }
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float g_mean = 0.f, g_std = 0.f;
  for (int s = 0; s < nslabs; ++s) {
    const size_t len = min(slab, n - (size_t)s * slab);
    double acc = 0.0;
    for (int b = 0; b < kF2bParts; ++b) acc += part[(size_t)s * kF2bParts + b];
    sd[s] = sqrtf((float)(acc / (double)len));
    g_mean = alpha * g_mean + (1.f - alpha) * mean[s];
    g_std = alpha * g_std + (1.f - alpha) * sd[s];
    gm[s] = g_mean;
    gs[s] = g_std;
  }
}

__global__ void f2b_map_kernel(const float *__restrict__ v, size_t n, size_t slab,
                               const float *__restrict__ gm, const float *__restrict__ gs,
                               unsigned char *out) {
  const float sf = 10.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t s = i / slab, w = i - s * slab;
    const size_t len = min(slab, n - s * slab);
    unsigned char b = 0;
    if ((w & ~(size_t)3) + 3 < len) {  // complete groups of four only
      float x = (v[i] - gm[s]) / gs[s];
      x = fmaxf(-sf, fminf(sf, x));
      b = (unsigned char)(((x + sf) / (2.0f * sf)) * 255.0f);
    }
    out[i] = b;
  }
}

cudaError_t launch_f2b(const float *vol, size_t n, size_t slab, float alpha, unsigned char *out,
                       double *part, float *stats, int nsm, cudaStream_t s) {
  const int nslabs = (int)((n + slab - 1) / slab);
  float *mean = stats, *sd = stats + nslabs, *gm = sd + nslabs, *gs = gm + nslabs;
  const dim3 pg(kF2bParts, nslabs);
  f2b_partials_kernel<<<pg, 256, 0, s>>>(vol, n, slab, mean, part, 0);
  f2b_slab_kernel<<<(nslabs + 127) / 128, 128, 0, s>>>(part, n, slab, nslabs, mean, sd, gm, gs,
                                                      alpha, 0);
  f2b_partials_kernel<<<pg, 256, 0, s>>>(vol, n, slab, mean, part, 1);
  f2b_slab_kernel<<<1, 1, 0, s>>>(part, n, slab, nslabs, mean, sd, gm, gs, alpha, 1);
  f2b_map_kernel<<<nsm * 8, 256, 0, s>>>(vol, n, slab, gm, gs, out);
  return cudaGetLastError();
}

}  // namespace trb
