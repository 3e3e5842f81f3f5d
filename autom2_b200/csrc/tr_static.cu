// tr_sirt_static: SIRT for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they reconstruct:
// a host application whose memory pool already owns the device memory it is
// allowed to use (a serving process holding a fixed HBM budget, a framework's
// caching allocator), or code that must not issue the device-wide
// synchronisation a cudaMalloc/cudaFree can imply in the middle of a
// stream-ordered pipeline.  This entry point needs no context and allocates
// nothing: its scratch (the per-tilt geometry, the reprojection, the
// projection weights and the voxel weights) lives in one file-scope static
// device array of kStaticScratchBytes (64 MiB).
//
// The array is reserved on a device when this file's device module is loaded
// there -- with CUDA's lazy module loading (the default), at the first call of
// this library's kernels on that device; with CUDA_MODULE_LOADING=EAGER, when
// the library is loaded, on every device the process uses, whether or not
// this entry point is ever called -- and stays reserved until the process
// exits.  The first call on a device also looks up the array's device address
// (cudaGetSymbolAddress, with the device current); make it before any stream
// capture.  Every call shares the one array and leaves the last call's
// contents in it: the buffers that must start at zero are cleared by each
// call, and calls whose work overlaps on the GPU (different streams, or
// different host threads) race on the scratch and must be serialised by the
// caller.
//
// The per-tilt geometry reaches the device as kernel arguments (a copy kernel
// per 32 tilts), so the call reads no host memory after it returns.  A
// back-projection whose bounded staging wait gives up sets a sticky word in
// the array that stays set until tr_static_take_timeout reads it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "tiltrec_b200.h"
#include "tr_geom.h"
#include "tr_internal.cuh"


using namespace trb;

namespace {

constexpr size_t kStaticScratchBytes = 64ull << 20;
constexpr int kStaticMaxTilts = 360;
constexpr int kStaticMaxDevices = 64;
constexpr size_t kStaticSmemBp = 64 * 1024;
constexpr size_t kStaticSmemFp = 44 * 1024;
constexpr size_t kStaticSmemMax = 200 * 1024;

}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

std::mutex g_static_mu;
void *g_static_addr[kStaticMaxDevices];

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of the static scratch on `device` (which is current).
cudaError_t static_scratch(int device, void **out) {
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_static_addr[device] = p;
  }
  *out = g_static_addr[device];
  return cudaSuccess;
}

struct StaticGeom {
  int fw, fh, ffw, ffh, chunk_bp, chunk_fp;
  float nbound;
  bool sep;
};

// Fixed-point steps and tile windows for the coefficients, as the context
// path derives them; returns the GeomStatus (GEOM_OK when the kernels can
// stage the geometry).
int derive(const double *coeff8, int nt, int nx, int ny, int th, TiltGeo *g,
           StaticGeom *out) {
  GeomInfo gi;
  int bad = -1;
  const int gs = derive_geometry(coeff8, nt, nx, ny, th, kStaticSmemMax, g, &gi, &bad);
  if (gs != GEOM_OK) return gs;
  out->fw = gi.fw;
  out->fh = gi.fh;
  out->ffw = gi.ffw;
  out->ffh = gi.ffh;
  out->sep = gi.sep;
  out->nbound = gi.nbound;
  out->chunk_bp = chunk_for(kStaticSmemBp, gi.bp_tilt_bytes);
  out->chunk_fp = chunk_for(kStaticSmemFp, gi.fp_tilt_bytes);
  return GEOM_OK;
}

// Up to kGeoPerLaunch tilts' geometry passed by value as a kernel argument
// (3.6 KB, under the 4 KB argument limit of every launch form).
constexpr int kGeoPerLaunch = 32;
struct GeoChunk {
  TiltGeo g[kGeoPerLaunch];
};

__global__ void geo_upload_kernel(const GeoChunk c, int n, TiltGeo *dst) {
  const int words = (int)(sizeof(TiltGeo) / sizeof(long long));
  const long long *src = reinterpret_cast<const long long *>(c.g);
  long long *out = reinterpret_cast<long long *>(dst);
  for (int i = threadIdx.x; i < n * words; i += blockDim.x) out[i] = src[i];
}

tr_status run(int device, int nx, int ny, int nt, int th, int layout,
              const double *coeff8, float ox, float oy, float oz,
              const float *proj, float *vol, int iters, float gamma,
              cudaStream_t s) {
  const size_t plane = (size_t)nx * ny * nt, nvox = (size_t)nx * ny * th;
  const size_t flag_b = 256;  // device-wait words of the back-projections
  const size_t geo_b = round256(sizeof(TiltGeo) * nt);
  const size_t plane_b = round256(plane * sizeof(float));
  const size_t vox_b = round256(nvox * sizeof(float));
  if (flag_b + geo_b + 2 * plane_b + vox_b > kStaticScratchBytes) return TR_ERR_BUDGET;

  TiltGeo g[kStaticMaxTilts];
  StaticGeom sg;
  const int gs = derive(coeff8, nt, nx, ny, th, g, &sg);
  if (gs == GEOM_NONFINITE) return TR_ERR_ARG;  // as tr_set_problem
  if (gs != GEOM_OK) return TR_ERR_UNSUPPORTED;

  void *base = nullptr;
  if (static_scratch(device, &base) != cudaSuccess) return TR_ERR_CUDA;
  int *flags = (int *)base;
  unsigned char *b = (unsigned char *)base + flag_b;
  TiltGeo *geo = (TiltGeo *)b;
  float *wt = (float *)(b + geo_b);
  float *val = (float *)(b + geo_b + plane_b);
  float *wtvol = (float *)(b + geo_b + 2 * plane_b);

  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  for (int t0 = 0; t0 < nt; t0 += kGeoPerLaunch) {
    GeoChunk c;
    const int n = std::min(kGeoPerLaunch, nt - t0);
    std::copy(g + t0, g + t0 + n, c.g);
    geo_upload_kernel<<<1, 128, 0, s>>>(c, n, geo + t0);
    if (cudaGetLastError() != cudaSuccess) return TR_ERR_CUDA;
  }

  VolView v;
  v.vol = vol;
  v.nx = nx;
  v.ny = ny;
  v.nz = th;
  v.zoff = 0;
  v.sy = layout == TR_LAYOUT_Y ? (long long)th * nx : nx;
  v.sz = layout == TR_LAYOUT_Y ? nx : (long long)ny * nx;

  FpArgs f{};
  f.v = v;
  f.tstride = (long long)nx * ny;
  f.pnx = nx;
  f.pny = ny;
  f.geo = geo;
  f.t0 = 0;
  f.nt = nt;
  f.ox = ox;
  f.oy = oy;
  f.oz = oz;
  f.fw = sg.ffw;
  f.fh = sg.ffh;
  f.chunk = sg.chunk_fp;
  f.nbound = sg.nbound;

  BpArgs bp{};
  bp.v = v;
  bp.img.nx = nx;
  bp.img.ny = ny;
  bp.img.tstride = (long long)nx * ny;
  bp.img.dtype = IMG_F32;
  bp.img.scale = nullptr;
  bp.geo = geo;
  bp.t0 = 0;
  bp.nt = nt;
  bp.ox = ox;
  bp.oy = oy;
  bp.oz = oz;
  bp.fw = sg.fw;
  bp.fh = sg.fh;
  bp.chunk = sg.chunk_bp;
  bp.wtvol = wtvol;
  bp.err = flags;

  // Geometry-only weights: splat of ones (projection side) and Σ_t c_t
  // (voxel side); the previous call's contents are cleared first.
  if (cudaMemsetAsync(wt, 0, plane * sizeof(float), s) != cudaSuccess) return TR_ERR_CUDA;
  FpArgs fw_ = f;
  fw_.v.vol = nullptr;
  fw_.val = wt;
  if (launch_fp(sg.sep, fw_, s) != cudaSuccess) return TR_ERR_CUDA;
  BpArgs bw = bp;
  bw.v.vol = wtvol;
  bw.img.p = nullptr;
  bw.gamma = 1.f;
  bw.out = wtvol;
  if (cudaMemsetAsync(flags, 0, sizeof(int), s) != cudaSuccess) return TR_ERR_CUDA;
  if (launch_bp(BP_WEIGHTS, sg.sep, bw, s) != cudaSuccess) return TR_ERR_CUDA;

  for (int it = 0; it < iters; ++it) {
    if (cudaMemsetAsync(val, 0, plane * sizeof(float), s) != cudaSuccess)
      return TR_ERR_CUDA;
    FpArgs fi = f;
    fi.val = val;
    if (launch_fp(sg.sep, fi, s) != cudaSuccess) return TR_ERR_CUDA;
    if (launch_resid(proj, val, wt, plane, nsm, s) != cudaSuccess) return TR_ERR_CUDA;
    BpArgs bi = bp;
    bi.img.p = val;
    bi.gamma = gamma;
    bi.out = nullptr;
    if (cudaMemsetAsync(flags, 0, sizeof(int), s) != cudaSuccess) return TR_ERR_CUDA;
    if (launch_bp(BP_SIRT, sg.sep, bi, s) != cudaSuccess) return TR_ERR_CUDA;
  }
  return TR_OK;
}

}  // namespace

extern "C" tr_status tr_sirt_static(int device, int nx, int ny, int ntilt,
                                    int thickness, int layout,
                                    const double *coeff8, float ox, float oy,
                                    float oz, const float *proj_dev,
                                    float *vol_dev, int iters, float gamma,
                                    void *stream) {
  if (nx < 2 || ny < 1 || ntilt < 1 || thickness < 1 || iters < 0 || !coeff8 ||
      !proj_dev || !vol_dev || ntilt > kStaticMaxTilts || device < 0 ||
      device >= kStaticMaxDevices || ny > 65535 * kTY ||
      (layout != TR_LAYOUT_Y && layout != TR_LAYOUT_Z))
    return TR_ERR_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return TR_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  const tr_status st = run(device, nx, ny, ntilt, thickness, layout, coeff8, ox, oy,
                           oz, proj_dev, vol_dev, iters, gamma, (cudaStream_t)stream);
  if (prev != device) cudaSetDevice(prev);
  return st;
}

extern "C" size_t tr_static_scratch_limit(void) { return kStaticScratchBytes; }

// Reads and clears the sticky device-wait word of the static scratch on
// `device` (after the caller has synchronised the streams of its calls).
extern "C" tr_status tr_static_take_timeout(int device) {
  if (device < 0 || device >= kStaticMaxDevices) return TR_ERR_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return TR_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  tr_status st = TR_OK;
  void *base = nullptr;
  int h = 0;
  if (static_scratch(device, &base) != cudaSuccess ||
      cudaMemcpy(&h, (int *)base + 1, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    st = TR_ERR_CUDA;
  } else if (h) {
    st = cudaMemset(base, 0, 2 * sizeof(int)) == cudaSuccess ? TR_ERR_TIMEOUT : TR_ERR_CUDA;
  }
  if (prev != device) cudaSetDevice(prev);
  return st;
}

// The bounded device wait on the static scratch's words: one CTA waits on a
// barrier nothing completes for budget_us of GPU clock, gives up and reports
// as a back-projection would; the report is then read back as a timeout.
extern "C" tr_status tr_static_selftest_wait(int device, int budget_us) {
  if (device < 0 || device >= kStaticMaxDevices || budget_us < 1 || budget_us > 10000000)
    return TR_ERR_ARG;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return TR_ERR_CUDA;
  if (prev != device && cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  void *base = nullptr;
  int khz = 0;
  tr_status st = TR_OK;
  if (static_scratch(device, &base) != cudaSuccess ||
      cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device) != cudaSuccess ||
      cudaMemset(base, 0, 2 * sizeof(int)) != cudaSuccess ||
      launch_bounded_wait_selftest((long long)khz * budget_us / 1000, (int *)base, nullptr) !=
          cudaSuccess ||
      cudaStreamSynchronize(nullptr) != cudaSuccess)
    st = TR_ERR_CUDA;
  if (prev != device) cudaSetDevice(prev);
  return st ? st : tr_static_take_timeout(device);
}
