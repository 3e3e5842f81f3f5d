// Elementwise and reduction kernels of ADMM (TiltRecZ's ADMM,
// main/main-mpiz.cpp:603-1013): the normalisation inside A^T D A, the mu
// terms, the conjugate-gradient updates with FP64 dot products, and the soft
// threshold.  The forward and back-projections are the engine's kernels.
//
// Dot products are deterministic: each block sums a fixed strided range in
// FP64 and a tree; one block then adds the block partials in order.  The CG
// scalars stay on the device (no host round trip per iteration): the update
// kernels read them from `scal`, [0] = r.r, [1] = h.p, [2] = r_new.h.
#include <cuda_runtime.h>

#include "tr_internal.cuh"

namespace trb {

namespace {

// Reproject_admm_atax's normalisation (main-mpiz.cpp:657-791, :752-783): a detector
// pixel contributes ax/w where |w| > 10e-6, nothing elsewhere.
__global__ void admm_normalize_kernel(float *val, const float *__restrict__ wt, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float w = wt[i];
    val[i] = (double)fabsf(w) > 10e-6 ? val[i] / w : 0.f;
  }
}

// ATAmuLTL (:819-841): out += mu * x.
__global__ void admm_add_scaled_kernel(float *out, const float *__restrict__ x, float mu,
                                       size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] += mu * x[i];
}

// ATbmuLT (:793-818): atb += (u - d) * mu.
__global__ void admm_atb_kernel(float *atb, const float *__restrict__ u,
                                const float *__restrict__ d, float mu, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    atb[i] += (u[i] - d[i]) * mu;
}

// applycg's start (:863-867): r = b - a, p = r.
__global__ void admm_cg_init_kernel(float *r, float *p, const float *__restrict__ b,
                                    const float *__restrict__ a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v = b[i] - a[i];
    r[i] = v;
    p[i] = v;
  }
}

// sum of the float products a[i]*b[i] in FP64 (the reference multiplies in
// float and accumulates in double, :886-891, :916), or with PROD64 the exact
// FP64 products: per-block partials.
template <bool PROD64>
__global__ void admm_dot_partial_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                        size_t n, double *part) {
  __shared__ double red[256];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    s += PROD64 ? (double)a[i] * (double)b[i] : (double)(a[i] * b[i]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void admm_dot_finish_kernel(const double *__restrict__ part, int nparts, double *out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// alpha = d0/d2 and beta = d1/d2 where |d2| > 10e-6, else 0 (:894-901, :920-927).
__device__ __forceinline__ double cg_ratio(double num, double d2) {
  return (d2 > 10e-6 || -d2 > 10e-6) ? num / d2 : 0.0;
}

// vol += alpha * p (:903-906), in double as the reference evaluates it.
__global__ void admm_x_update_kernel(float *vol, const float *__restrict__ p,
                                     const double *__restrict__ scal, size_t n) {
  const double alpha = cg_ratio(scal[0], scal[1]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    vol[i] = (float)((double)vol[i] + alpha * (double)p[i]);
}

// r = b - ax (:913-917).
__global__ void admm_r_update_kernel(float *r, const float *__restrict__ b,
                                     const float *__restrict__ ax, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    r[i] = b[i] - ax[i];
}

// p = r + beta * p (:929-932).
__global__ void admm_p_update_kernel(float *p, const float *__restrict__ r,
                                     const double *__restrict__ scal, size_t n) {
  const double beta = cg_ratio(scal[2], scal[1]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = (float)((double)r[i] + beta * (double)p[i]);
}

// soft_admm (:940-957) then the dual update d += x - u (:1002-1006).
__global__ void admm_soft_kernel(float *u, float *d, const float *__restrict__ x, float soft,
                                 size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v = x[i] + d[i];
    const float uu = v < -soft ? v + soft : (v > soft ? v - soft : 0.f);
    u[i] = uu;
    d[i] += x[i] - uu;
  }
}

unsigned grid_for(size_t n, int nsm) {
  const size_t want = (size_t)nsm * 8, need = (n + 255) / 256;
  return (unsigned)(need < want ? (need ? need : 1) : want);
}

}  // namespace

cudaError_t admm_normalize(float *val, const float *wt, size_t n, int nsm, cudaStream_t s) {
  admm_normalize_kernel<<<grid_for(n, nsm), 256, 0, s>>>(val, wt, n);
  return cudaGetLastError();
}

cudaError_t admm_add_scaled(float *out, const float *x, float mu, size_t n, int nsm,
                            cudaStream_t s) {
  admm_add_scaled_kernel<<<grid_for(n, nsm), 256, 0, s>>>(out, x, mu, n);
  return cudaGetLastError();
}

cudaError_t admm_atb(float *atb, const float *u, const float *d, float mu, size_t n, int nsm,
                     cudaStream_t s) {
  admm_atb_kernel<<<grid_for(n, nsm), 256, 0, s>>>(atb, u, d, mu, n);
  return cudaGetLastError();
}

cudaError_t admm_cg_init(float *r, float *p, const float *b, const float *a, size_t n, int nsm,
                         cudaStream_t s) {
  admm_cg_init_kernel<<<grid_for(n, nsm), 256, 0, s>>>(r, p, b, a, n);
  return cudaGetLastError();
}

// Deterministic FP64 dot product into *out; part holds kAdmmParts doubles.
cudaError_t admm_dot(const float *a, const float *b, size_t n, double *part, double *out,
                     cudaStream_t s) {
  admm_dot_partial_kernel<false><<<kAdmmParts, 256, 0, s>>>(a, b, n, part);
  admm_dot_finish_kernel<<<1, 256, 0, s>>>(part, kAdmmParts, out);
  return cudaGetLastError();
}

// |a|^2 with FP64 products and fixed-order FP64 sums into *out.
cudaError_t sumsq_f64(const float *a, size_t n, double *part, double *out, cudaStream_t s) {
  admm_dot_partial_kernel<true><<<kAdmmParts, 256, 0, s>>>(a, a, n, part);
  admm_dot_finish_kernel<<<1, 256, 0, s>>>(part, kAdmmParts, out);
  return cudaGetLastError();
}

cudaError_t admm_x_update(float *vol, const float *p, const double *scal, size_t n, int nsm,
                          cudaStream_t s) {
  admm_x_update_kernel<<<grid_for(n, nsm), 256, 0, s>>>(vol, p, scal, n);
  return cudaGetLastError();
}

cudaError_t admm_r_update(float *r, const float *b, const float *ax, size_t n, int nsm,
                          cudaStream_t s) {
  admm_r_update_kernel<<<grid_for(n, nsm), 256, 0, s>>>(r, b, ax, n);
  return cudaGetLastError();
}

cudaError_t admm_p_update(float *p, const float *r, const double *scal, size_t n, int nsm,
                          cudaStream_t s) {
  admm_p_update_kernel<<<grid_for(n, nsm), 256, 0, s>>>(p, r, scal, n);
  return cudaGetLastError();
}

cudaError_t admm_soft(float *u, float *d, const float *x, float soft, size_t n, int nsm,
                      cudaStream_t s) {
  admm_soft_kernel<<<grid_for(n, nsm), 256, 0, s>>>(u, d, x, soft, n);
  return cudaGetLastError();
}

}  // namespace trb
