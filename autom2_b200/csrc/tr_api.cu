// C-ABI of the TiltRec B200 engine (include/tiltrec_b200.h): context,
// geometry, scratch management and the BPT / WBP / SIRT / SART drivers.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <complex>
#include <map>
#include <string>
#include <vector>

#include "tiltrec_b200.h"
#include "tr_filter_host.h"
#include "tr_geom.h"
#include "tr_internal.cuh"


using namespace trb;

namespace {
constexpr size_t kSmemBp = 64 * 1024;  // interpolation tables per CTA
// Splat windows per CTA: with the kernel's ~8.4 KB of static bookkeeping, four
// CTAs fit on an SM.
constexpr size_t kSmemFp = 44 * 1024;
constexpr size_t kSmemMax = 200 * 1024;
}  // namespace

struct tr_ctx {
  int device = 0;
  int nsm = 148;
  size_t budget = 0;
  std::string err;
  cudaStream_t io_stream = nullptr;

  // problem
  bool have_problem = false;
  int nx = 0, ny = 0, nt = 0, th = 0, layout = 0;
  float ox = 0, oy = 0, oz = 0;
  bool sep = false;
  int fw = 0, fh = 0, chunk_bp = 1, chunk_fp = 1;
  int ffw = 0, ffh = 0;  // forward-projection tile window
  float fp_nbound = 0;   // most voxel contributions per forward window entry
  TiltGeo *geo_d = nullptr;

  // scratch: buffers are kept across problems and grown on demand; slot
  // records each buffer's capacity and the problem generation that last
  // claimed it (set_problem starts a new generation)
  struct Slot {
    size_t cap = 0;
    unsigned gen = 0;
  };
  std::map<void **, Slot> slots;
  unsigned gen = 0;
  size_t scratch = 0;
  float *val_d = nullptr, *wt_d = nullptr;
  // SIRT voxel weights in compact form (BpArgs::wslot): a slot per tile of
  // the view [w_z0, w_z0 + w_nz), the border tiles' weights, the separable
  // per-row weights
  float *wtvol_d = nullptr, *wrow_d = nullptr;
  int *wslot_d = nullptr;
  int w_z0 = -1, w_nz = -1;
  long long w_border = 0;
  void *res16_d = nullptr;      // 16-bit SIRT residual [ntilt][ny][nx]
  unsigned *maxbits_d = nullptr;  // per-tilt |p| maxima for tr_quantize
  float *rscale_d = nullptr;      // per-tilt scales of the FP16 SIRT residual
  float *admm_d = nullptr;        // ADMM: 7 volumes (A^T b, u, d, A x, r, p, h)
  double *admm_dot_d = nullptr;   // ADMM: dot partials + the 3 CG scalars
  bool wt_ready = false, wtvol_ready = false;
  int filt_nx = 0, filt_npad = 0, filt_log2m = 0;
  float2 *ghat_d = nullptr, *tw_d = nullptr;
  float *hproj_d = nullptr, *hvol_d = nullptr;
  // byte output: slab partial sums and statistics, the bytes themselves
  double *f2b_part_d = nullptr;
  float *f2b_stats_d = nullptr;
  unsigned char *bytes_d = nullptr;
  // streamed output: two pinned staging buffers and their copy events
  void *stage_h[2] = {nullptr, nullptr};
  size_t stage_n = 0;
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int *err_d = nullptr;  // [0] abort word of the current launch, [1] sticky report
  // z-slab SIRT: the next iteration's reprojection, the device staging slabs
  // of a host-resident volume, their copy streams and events
  float *val2_d = nullptr, *slab_d = nullptr;
  // deterministic forward projections (tr_set_deterministic): int64 sums
  // [ntilt][ny][nx] and the view's max |voxel|
  bool deterministic = false;
  unsigned long long *ival_d = nullptr;
  unsigned *gmax_d = nullptr;
  cudaStream_t cp_in = nullptr, cp_out = nullptr;
  cudaEvent_t ev_in[3] = {}, ev_comp[3] = {}, ev_free[3] = {}, ev_start = nullptr;
};

namespace {

tr_status fail(tr_ctx *c, tr_status s, const char *fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return s;
}

tr_status cuda_fail(tr_ctx *c, cudaError_t e, const char *what) {
  return fail(c, TR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Returns the tr_status of `call` when it is not TR_OK.
#define TR_TRY(call)                \
  do {                              \
    const tr_status s_ = (call);    \
    if (s_ != TR_OK) return s_;     \
  } while (0)

#define TR_CUDA(ctx, call)                                  \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

size_t vol_elems(const tr_ctx *c) { return (size_t)c->nx * c->ny * c->th; }
size_t proj_elems(const tr_ctx *c) { return (size_t)c->nx * c->ny * c->nt; }

void scratch_free(tr_ctx *c, void **p) {
  tr_ctx::Slot &sl = c->slots[p];
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
    c->scratch -= std::min(c->scratch, sl.cap);
  }
  sl.cap = 0;
}

// Frees the scratch buffers no call of the current problem has claimed.
void release_idle(tr_ctx *c) {
  for (auto &kv : c->slots)
    if (*kv.first && kv.second.gen != c->gen) scratch_free(c, kv.first);
}

// Claims scratch buffer *p with at least `bytes` for the current problem:
// reuses it when large enough, else reallocates it.  When the budget or the
// device runs short, buffers idle in this problem are released first.
tr_status scratch_alloc(tr_ctx *c, void **p, size_t bytes, const char *what) {
  tr_ctx::Slot &sl = c->slots[p];
  if (*p && sl.cap >= bytes) {
    sl.gen = c->gen;
    return TR_OK;
  }
  if (*p) scratch_free(c, p);
  if (c->budget && c->scratch + bytes > c->budget) release_idle(c);
  if (c->budget && c->scratch + bytes > c->budget)
    return fail(c, TR_ERR_BUDGET,
                "%s needs %zu bytes; %zu of the %zu-byte budget in use", what,
                bytes, c->scratch, c->budget);
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    release_idle(c);
    e = cudaMalloc(p, bytes);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(c, TR_ERR_OOM, "cudaMalloc(%zu) for %s: %s", bytes, what,
                cudaGetErrorString(e));
  }
  sl.cap = bytes;
  sl.gen = c->gen;
  c->scratch += bytes;
  return TR_OK;
}

// Ends the current problem.  Its scratch buffers stay allocated for the next
// problem to reuse (a new generation: they count as idle until claimed).
void release_problem(tr_ctx *c) {
  ++c->gen;
  if (c->geo_d) {
    cudaFree(c->geo_d);
    c->geo_d = nullptr;
  }
  c->wt_ready = c->wtvol_ready = false;
  c->have_problem = false;
}

VolView full_view(const tr_ctx *c, float *vol, int z0, int nz) {
  VolView v;
  v.vol = vol;
  v.nx = c->nx;
  v.ny = c->ny;
  v.nz = nz;
  v.zoff = z0;
  if (c->layout == TR_LAYOUT_Y) {
    v.sy = (long long)c->th * c->nx;
    v.sz = c->nx;
  } else {
    v.sy = c->nx;
    v.sz = (long long)c->ny * c->nx;
  }
  return v;
}

BpArgs bp_args(const tr_ctx *c, float *vol, int z0, int nz, const float *img,
               int t0, int nt, float gamma) {
  BpArgs a{};
  a.v = full_view(c, vol, z0, nz);
  a.img.p = img;
  a.img.nx = c->nx;
  a.img.ny = c->ny;
  a.img.tstride = (long long)c->nx * c->ny;
  a.img.dtype = IMG_F32;
  a.img.scale = nullptr;
  a.geo = c->geo_d;
  a.t0 = t0;
  a.nt = nt;
  a.ox = c->ox;
  a.oy = c->oy;
  a.oz = c->oz;
  a.fw = c->fw;
  a.fh = c->fh;
  a.chunk = c->chunk_bp;
  a.gamma = gamma;
  a.wtvol = nullptr;
  a.out = nullptr;
  a.err = c->err_d;
  return a;
}

// Back-projection launch: clears the launch-wide abort word first.
cudaError_t run_bp(tr_ctx *c, int mode, const BpArgs &a, cudaStream_t s) {
  if (c->err_d) {
    cudaError_t e = cudaMemsetAsync(c->err_d, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
  }
  return launch_bp(mode, c->sep, a, s);
}

// Reads and clears the sticky device-wait report (after a synchronisation).
tr_status take_timeout(tr_ctx *c) {
  if (!c->err_d) return TR_OK;
  int h = 0;
  if (cudaMemcpy(&h, c->err_d + 1, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return cuda_fail(c, cudaGetLastError(), "reading the device-wait flag");
  if (!h) return TR_OK;
  cudaMemset(c->err_d, 0, 2 * sizeof(int));
  return fail(c, TR_ERR_TIMEOUT,
              "a back-projection's staging copy did not arrive within its time limit; "
              "the volume of that launch was left unchanged");
}

FpArgs fp_args(const tr_ctx *c, const float *vol, int z0, int nz, float *val,
               int t0, int nt) {
  FpArgs a{};
  a.v = full_view(c, const_cast<float *>(vol), z0, nz);
  a.val = val;
  a.tstride = (long long)c->nx * c->ny;
  a.pnx = c->nx;
  a.pny = c->ny;
  a.geo = c->geo_d;
  a.t0 = t0;
  a.nt = nt;
  a.ox = c->ox;
  a.oy = c->oy;
  a.oz = c->oz;
  a.fw = c->ffw;
  a.fh = c->ffh;
  a.chunk = c->chunk_fp;
  a.nbound = c->fp_nbound;
  return a;
}

// A forward projection through the context: the float flush, or with
// tr_set_deterministic the int64 one (sums cleared first, converted after).
tr_status run_fp(tr_ctx *c, const FpArgs &a, cudaStream_t s) {
  if (!c->deterministic) {
    TR_CUDA(c, launch_fp(c->sep, a, s));
    return TR_OK;
  }
  tr_status st;
  if ((st = scratch_alloc(c, (void **)&c->ival_d, proj_elems(c) * sizeof(unsigned long long),
                          "deterministic projection sums")) ||
      (st = scratch_alloc(c, (void **)&c->gmax_d, sizeof(unsigned), "largest voxel")))
    return st;
  const size_t off = (size_t)a.t0 * a.tstride, n = (size_t)a.nt * a.tstride;
  TR_CUDA(c, cudaMemsetAsync(c->ival_d + off, 0, n * sizeof(unsigned long long), s));
  TR_CUDA(c, launch_fp_deterministic(c->sep, a, c->ival_d, c->gmax_d, c->nsm, s));
  return TR_OK;
}

// Kernel spectrum of the R-weighting filter for rows of nx samples.
tr_status build_filter(tr_ctx *c, int nx) {
  if (c->filt_nx == nx && c->ghat_d && c->tw_d) {  // cached: claim for this problem
    c->slots[(void **)&c->ghat_d].gen = c->slots[(void **)&c->tw_d].gen = c->gen;
    return TR_OK;
  }
  RweightSpectrum sp;
  if (!rweight_spectrum(nx, kSmemMax, &sp))
    return fail(c, TR_ERR_UNSUPPORTED, "row length %d needs an FFT of %d points", nx,
                1 << sp.log2m);
  const int M = 1 << sp.log2m;
  scratch_free(c, (void **)&c->ghat_d);
  scratch_free(c, (void **)&c->tw_d);
  tr_status s = scratch_alloc(c, (void **)&c->ghat_d, sizeof(float2) * M, "filter spectrum");
  if (s) return s;
  s = scratch_alloc(c, (void **)&c->tw_d, sizeof(float2) * sp.tw.size(), "filter twiddles");
  if (s) return s;
  TR_CUDA(c, cudaMemcpy(c->ghat_d, sp.ghat.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
  TR_CUDA(c, cudaMemcpy(c->tw_d, sp.tw.data(), sizeof(float2) * sp.tw.size(),
                        cudaMemcpyHostToDevice));
  c->filt_nx = nx;
  c->filt_npad = sp.npad;
  c->filt_log2m = sp.log2m;
  return TR_OK;
}

// Validates coefficients, derives the fixed-point steps and the per-tile
// detector window, and uploads them (ordered on `s`).  Invalidates the cached
// SIRT/SART weights, which depend on the geometry.
tr_status load_geometry(tr_ctx *c, const double *coeff8, cudaStream_t s) {
  const int nt = c->nt;
  std::vector<TiltGeo> g(nt);
  GeomInfo gi;
  int bad = -1;
  switch (derive_geometry(coeff8, nt, c->nx, c->ny, c->th, kSmemMax, g.data(), &gi, &bad)) {
    case GEOM_OK: break;
    case GEOM_NONFINITE: return fail(c, TR_ERR_ARG, "non-finite coefficient at tilt %d", bad);
    case GEOM_MAGNITUDE:
      return fail(c, TR_ERR_UNSUPPORTED, "coefficient magnitude above 1024 at tilt %d", bad);
    case GEOM_RANGE:
      return fail(c, TR_ERR_UNSUPPORTED, "detector coordinates out of range at tilt %d", bad);
    case GEOM_SMEM:
      return fail(c, TR_ERR_UNSUPPORTED, "detector window %dx%d per tile exceeds shared memory",
                  gi.ffw, gi.ffh);
    default:
      return fail(c, TR_ERR_UNSUPPORTED, "detector window %dx%d per tile exceeds %d",
                  std::max(gi.fw, gi.ffw), std::max(gi.fh, gi.ffh), kMaxWindow);
  }
  if (s) {
    TR_CUDA(c, cudaMemcpyAsync(c->geo_d, g.data(), sizeof(TiltGeo) * nt,
                               cudaMemcpyHostToDevice, s));
    TR_CUDA(c, cudaStreamSynchronize(s));
  } else {
    TR_CUDA(c, cudaMemcpy(c->geo_d, g.data(), sizeof(TiltGeo) * nt, cudaMemcpyHostToDevice));
  }
  c->fw = gi.fw;
  c->fh = gi.fh;
  c->ffw = gi.ffw;
  c->ffh = gi.ffh;
  c->fp_nbound = gi.nbound;
  c->sep = gi.sep;
  c->chunk_bp = chunk_for(kSmemBp, gi.bp_tilt_bytes);
  c->chunk_fp = chunk_for(kSmemFp, gi.fp_tilt_bytes);
  c->wt_ready = c->wtvol_ready = false;
  return TR_OK;
}

// Device copies of the host-buffer calls' stack and (with_vol) volume:
// scratch like the rest, kept across calls and counted against the budget.
tr_status host_buffers(tr_ctx *c, bool with_vol = true) {
  tr_status st = scratch_alloc(c, (void **)&c->hproj_d, proj_elems(c) * sizeof(float),
                               "device copy of the stack");
  if (!st && with_vol)
    st = scratch_alloc(c, (void **)&c->hvol_d, vol_elems(c) * sizeof(float),
                       "device copy of the volume");
  return st;
}

tr_status need_problem(tr_ctx *c) {
  if (!c) return TR_ERR_ARG;
  if (!c->have_problem) return fail(c, TR_ERR_NOPROBLEM, "tr_set_problem has not been called");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
  return TR_OK;
}

tr_status ensure_wt(tr_ctx *c, cudaStream_t s) {
  const size_t pb = proj_elems(c) * sizeof(float);
  tr_status st = scratch_alloc(c, (void **)&c->wt_d, pb, "projection weights");
  if (st) return st;
  if (!c->wt_ready) {
    TR_CUDA(c, cudaMemsetAsync(c->wt_d, 0, pb, s));
    FpArgs a = fp_args(c, nullptr, 0, c->th, c->wt_d, 0, c->nt);
    if ((st = run_fp(c, a, s))) return st;
    c->wt_ready = true;
  }
  return TR_OK;
}

// SIRT voxel weights of sections [z0, z0 + nz), compact: the view's tiles are
// classified on the device (one read of the border count), the border tiles'
// weights computed by the weight pass, interior ones implied (BpArgs::wslot).
tr_status ensure_wtvol(tr_ctx *c, int z0, int nz, cudaStream_t s) {
  if (c->wtvol_ready && c->w_z0 == z0 && c->w_nz == nz) {
    c->slots[(void **)&c->wtvol_d].gen = c->slots[(void **)&c->wslot_d].gen = c->gen;
    if (c->wrow_d) c->slots[(void **)&c->wrow_d].gen = c->gen;
    return TR_OK;
  }
  c->wtvol_ready = false;
  const VolView v = full_view(c, nullptr, z0, nz);
  const dim3 g = bp_tile_grid(v);
  const size_t ntiles = (size_t)g.x * g.y * g.z;
  tr_status st = scratch_alloc(c, (void **)&c->wslot_d, (ntiles + 1) * sizeof(int),
                               "voxel-weight tile slots");
  if (st) return st;
  int *count = c->wslot_d + ntiles;
  TR_CUDA(c, cudaMemsetAsync(count, 0, sizeof(int), s));
  TR_CUDA(c, launch_classify_tiles(c->geo_d, c->nt, v, c->ox, c->oy, c->oz, c->nx, c->ny, c->sep,
                                   c->wslot_d, count, s));
  int nborder = 0;
  TR_CUDA(c, cudaMemcpyAsync(&nborder, count, sizeof(int), cudaMemcpyDeviceToHost, s));
  TR_CUDA(c, cudaStreamSynchronize(s));
  if ((st = scratch_alloc(c, (void **)&c->wtvol_d,
                          std::max<size_t>(1, (size_t)nborder) * kTileVox * sizeof(float),
                          "border-tile voxel weights")))
    return st;
  if (c->sep) {
    if ((st = scratch_alloc(c, (void **)&c->wrow_d, (size_t)c->ny * sizeof(float),
                            "row voxel weights")))
      return st;
    TR_CUDA(c, launch_sep_row_weights(c->geo_d, c->nt, c->ny, c->oy, c->ny, c->wrow_d, s));
  }
  if (nborder > 0) {
    BpArgs a = bp_args(c, nullptr, z0, nz, nullptr, 0, c->nt, 1.f);
    a.out = c->wtvol_d;
    a.wslot = c->wslot_d;
    TR_CUDA(c, run_bp(c, BP_WEIGHTS, a, s));
  }
  c->w_z0 = z0;
  c->w_nz = nz;
  c->w_border = nborder;
  c->wtvol_ready = true;
  return TR_OK;
}

// The compact weights of the cached view for a BP_SIRT launch.
void set_weights(const tr_ctx *c, BpArgs *b) {
  b->wtvol = c->wtvol_d;
  b->wslot = c->wslot_d;
  b->wrow = c->wrow_d;
  b->wfull = (float)c->nt;
}

// ---------------------------------------------------------------- z-slabs
// SIRT over slabs of `depth` sections (TiltRecZ's split of the volume along
// z, main-mpiz.cpp:1054-1069, with CuSIRTZ's iteration, recon_z.cu:85-190).
// Each iteration is one sweep over the slabs: back-project the residual into
// slab k with the update, then forward-project the updated slab into the next
// iteration's reprojection sums.  A host-resident volume is staged slab by
// slab through three device buffers: the copy in of slab k+1 and the copy out
// of slab k-1 run on their own streams while slab k computes.
constexpr int kSlabBufs = 3;

struct SlabRun {
  const void *proj;
  int pdtype;
  const float *pscale;
  int rdtype;
  float *vol;
  bool host;
  int iters;
  float gamma;
  int depth;
};

// Slab depth used for `want` sections: the whole thickness, or a multiple of
// the tile depth (the slab boundaries are tile boundaries, so each slab's
// tiles are the whole volume's and share its compact voxel weights).
int slab_depth(const tr_ctx *c, int want) {
  if (want >= c->th) return c->th;
  return std::max(kTZ, want / kTZ * kTZ);
}

size_t slab_elems(const tr_ctx *c, int depth) { return (size_t)c->nx * c->ny * depth; }

// Volume view of sections [z0, z0 + nz): the caller's device volume, or a
// staging buffer holding just those sections ([ny][nz][nx] in the Y layout).
VolView slab_view(const tr_ctx *c, float *base, bool staged, int z0, int nz) {
  if (!staged) {
    const size_t off = c->layout == TR_LAYOUT_Y ? (size_t)z0 * c->nx
                                                : (size_t)z0 * c->nx * c->ny;
    return full_view(c, base + off, z0, nz);
  }
  VolView v = full_view(c, base, z0, nz);
  if (c->layout == TR_LAYOUT_Y) v.sy = (long long)nz * c->nx;
  return v;
}

cudaError_t slab_copy(const tr_ctx *c, float *dev, float *host, int z0, int nz, bool to_dev,
                      cudaStream_t s) {
  const size_t nx = c->nx, ny = c->ny;
  const cudaMemcpyKind k = to_dev ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (c->layout == TR_LAYOUT_Z) {
    float *h = host + (size_t)z0 * nx * ny;
    return to_dev ? cudaMemcpyAsync(dev, h, nx * ny * nz * sizeof(float), k, s)
                  : cudaMemcpyAsync(h, dev, nx * ny * nz * sizeof(float), k, s);
  }
  // Y layout: ny runs of nz rows, one strided copy.
  float *h = host + (size_t)z0 * nx;
  const size_t w = nx * nz * sizeof(float), hp = nx * (size_t)c->th * sizeof(float);
  return to_dev ? cudaMemcpy2DAsync(dev, w, h, hp, w, ny, k, s)
                : cudaMemcpy2DAsync(h, hp, dev, w, w, ny, k, s);
}

tr_status slab_streams(tr_ctx *c) {
  if (c->cp_in) return TR_OK;
  TR_CUDA(c, cudaStreamCreateWithFlags(&c->cp_in, cudaStreamNonBlocking));
  TR_CUDA(c, cudaStreamCreateWithFlags(&c->cp_out, cudaStreamNonBlocking));
  for (int i = 0; i < kSlabBufs; ++i) {
    TR_CUDA(c, cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming));
    TR_CUDA(c, cudaEventCreateWithFlags(&c->ev_comp[i], cudaEventDisableTiming));
    TR_CUDA(c, cudaEventCreateWithFlags(&c->ev_free[i], cudaEventDisableTiming));
  }
  TR_CUDA(c, cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming));
  return TR_OK;
}

// Scratch of the slab path: both reprojections, the 16-bit residual, the
// weights of the whole volume, and the staging slabs of a host volume.
tr_status slab_scratch(tr_ctx *c, const SlabRun &r, cudaStream_t s) {
  const size_t pn = proj_elems(c);
  tr_status st;
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection")) ||
      (st = scratch_alloc(c, (void **)&c->val2_d, pn * sizeof(float), "next reprojection")))
    return st;
  if (r.rdtype != TR_DTYPE_F32 &&
      (st = scratch_alloc(c, &c->res16_d, pn * 2, "16-bit residual")))
    return st;
  if (r.rdtype == TR_DTYPE_F16 &&
      ((st = scratch_alloc(c, (void **)&c->rscale_d, sizeof(float) * c->nt,
                           "residual scales")) ||
       (st = scratch_alloc(c, (void **)&c->maxbits_d, sizeof(unsigned) * c->nt,
                           "per-tilt maxima"))))
    return st;
  if (r.host &&
      (st = scratch_alloc(c, (void **)&c->slab_d,
                          kSlabBufs * slab_elems(c, r.depth) * sizeof(float), "z-slab staging")))
    return st;
  if ((st = ensure_wt(c, s))) return st;
  if ((st = ensure_wtvol(c, 0, c->th, s))) return st;
  return slab_streams(c);
}

// Residual of the reprojection `val` (in place) and its 16-bit copy; returns
// the image the back-projection reads.
tr_status slab_residual(tr_ctx *c, const SlabRun &r, float *val, cudaStream_t s,
                        const void **res, const float **rs) {
  const size_t plane = (size_t)c->nx * c->ny;
  const float *ps = r.pdtype == TR_DTYPE_F32 ? nullptr : r.pscale;
  if (r.rdtype == TR_DTYPE_F16) {
    TR_CUDA(c, launch_resid_lp(r.proj, r.pdtype, ps, val, c->wt_d, plane, c->nt, TR_DTYPE_F32,
                               val, nullptr, c->nsm, s));
    TR_CUDA(c, launch_quantize(val, plane, c->nt, TR_DTYPE_F16, c->res16_d, c->rscale_d,
                               c->maxbits_d, c->nsm, s));
    *res = c->res16_d;
    *rs = c->rscale_d;
  } else {
    void *out = r.rdtype == TR_DTYPE_F32 ? (void *)val : c->res16_d;
    TR_CUDA(c, launch_resid_lp(r.proj, r.pdtype, ps, val, c->wt_d, plane, c->nt, r.rdtype, out,
                               nullptr, c->nsm, s));
    *res = out;
    *rs = nullptr;
  }
  return TR_OK;
}

// One sweep over the slabs of sections [0, zend): with `res`, the SIRT
// update of each slab from that residual; with `fp_out`, the forward
// projection of each (updated) slab added into fp_out.  A host volume is
// copied in before and, after an update, out again.
tr_status slab_sweep(tr_ctx *c, const SlabRun &r, int zend, const void *res, const float *rs,
                     float *fp_out, cudaStream_t s) {
  const dim3 g = bp_tile_grid(full_view(c, nullptr, 0, c->th));
  const bool write_back = res != nullptr;
  if (r.host) {
    TR_CUDA(c, cudaEventRecord(c->ev_start, s));
    TR_CUDA(c, cudaStreamWaitEvent(c->cp_in, c->ev_start, 0));
  }
  int k = 0, used = 0;
  for (int z0 = 0; z0 < zend; z0 += r.depth, k = (k + 1) % kSlabBufs, ++used) {
    const int nz = std::min(r.depth, zend - z0);
    float *buf = r.host ? c->slab_d + k * slab_elems(c, r.depth) : r.vol;
    if (r.host) {
      if (used >= kSlabBufs) TR_CUDA(c, cudaStreamWaitEvent(c->cp_in, c->ev_free[k], 0));
      TR_CUDA(c, slab_copy(c, buf, r.vol, z0, nz, true, c->cp_in));
      TR_CUDA(c, cudaEventRecord(c->ev_in[k], c->cp_in));
      TR_CUDA(c, cudaStreamWaitEvent(s, c->ev_in[k], 0));
    }
    const VolView v = slab_view(c, buf, r.host, z0, nz);
    if (res) {
      BpArgs b = bp_args(c, nullptr, z0, nz, (const float *)res, 0, c->nt, r.gamma);
      b.v = v;
      b.img.dtype = r.rdtype;
      b.img.scale = rs;
      set_weights(c, &b);
      b.wslot = c->wslot_d + (size_t)(z0 / kTZ) * g.x * g.y;  // this slab's tiles
      TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
    }
    if (fp_out) {
      FpArgs f = fp_args(c, nullptr, z0, nz, fp_out, 0, c->nt);
      f.v = v;
      TR_TRY(run_fp(c, f, s));
    }
    if (r.host) {
      if (write_back) {
        TR_CUDA(c, cudaEventRecord(c->ev_comp[k], s));
        TR_CUDA(c, cudaStreamWaitEvent(c->cp_out, c->ev_comp[k], 0));
        TR_CUDA(c, slab_copy(c, buf, r.vol, z0, nz, false, c->cp_out));
        TR_CUDA(c, cudaEventRecord(c->ev_free[k], c->cp_out));
      } else {
        TR_CUDA(c, cudaEventRecord(c->ev_free[k], s));
      }
    }
  }
  if (r.host && write_back) {  // the volume is complete when `s` reaches here
    TR_CUDA(c, cudaEventRecord(c->ev_start, c->cp_out));
    TR_CUDA(c, cudaStreamWaitEvent(s, c->ev_start, 0));
  }
  return TR_OK;
}

tr_status slab_sirt(tr_ctx *c, const SlabRun &r, cudaStream_t s) {
  tr_status st = slab_scratch(c, r, s);
  if (st) return st;
  const size_t pn = proj_elems(c);
  float *cur = c->val_d, *next = c->val2_d;
  if (r.iters == 0) return TR_OK;
  TR_CUDA(c, cudaMemsetAsync(cur, 0, pn * sizeof(float), s));
  if ((st = slab_sweep(c, r, c->th, nullptr, nullptr, cur, s))) return st;
  for (int it = 0; it < r.iters; ++it) {
    const void *res;
    const float *rs;
    if ((st = slab_residual(c, r, cur, s, &res, &rs))) return st;
    const bool more = it + 1 < r.iters;
    if (more) TR_CUDA(c, cudaMemsetAsync(next, 0, pn * sizeof(float), s));
    if ((st = slab_sweep(c, r, c->th, res, rs, more ? next : nullptr, s))) return st;
    std::swap(cur, next);
  }
  if (r.host) TR_CUDA(c, cudaStreamSynchronize(s));
  return TR_OK;
}

}  // namespace

extern "C" {

int tr_version(void) { return 10000; }

const char *tr_status_string(int s) {
  switch (s) {
    case TR_OK: return "ok";
    case TR_ERR_ARG: return "invalid argument";
    case TR_ERR_OOM: return "device out of memory";
    case TR_ERR_BUDGET: return "HBM budget exceeded";
    case TR_ERR_CUDA: return "CUDA error";
    case TR_ERR_TIMEOUT: return "device wait timed out";
    case TR_ERR_NOPROBLEM: return "no problem set";
    case TR_ERR_UNSUPPORTED: return "unsupported geometry";
    default: return "unknown status";
  }
}

tr_status tr_geometry_from_angles(const float *angles, int nt, float offset,
                                  float pitch, float zshift, double *out) {
  if (!angles || !out || nt <= 0) return TR_ERR_ARG;
  // D2R with the reference's float constant (main-mpi.cpp:9,15): the
  // product is formed in float.  cos/sin of a float angle resolve to the
  // float overloads in the reference's C++ (TranslateAngleToCoefficients,
  // :94-98), of the double alpha/beta to the double ones (:112-113).
  const float kPi180 = 0.01745329252f;
  const double alpha = -(pitch * kPi180), beta = offset * kPi180, t = -zshift;
  const double ca = cos(alpha), sa = sin(alpha), cb = cos(beta), sb = sin(beta);
  for (int i = 0; i < nt; ++i) {
    const float tb = angles[i] * kPi180;
    const double a1 = cosf(tb), a3 = -sinf(tb);
    // DecorateCoefficients (:121-146) with a = (0, a1, 0, a3), b = (0, 0, 1, 0),
    // then the z shift (:173-181); the quadratic terms are all zero.
    const double A1 = 0.0 * sa * sb + a3 * ca * sb + a1 * cb;
    const double A2 = 0.0 * ca - a3 * sa;
    const double A3 = a3 * ca * cb + 0.0 * cb * sa - a1 * sb;
    const double B1 = 1.0 * sa * sb + 0.0 * ca * sb + 0.0 * cb;
    const double B2 = 1.0 * ca - 0.0 * sa;
    const double B3 = 0.0 * ca * cb + 1.0 * cb * sa - 0.0 * sb;
    double *o = out + 8 * (size_t)i;
    o[0] = 0.0 + A3 * t + 0.0 * t * t;
    o[1] = A1 + 0.0 * t;
    o[2] = A2 + 0.0 * t;
    o[3] = A3 + 2 * 0.0 * t;
    o[4] = 0.0 + B3 * t + 0.0 * t * t;
    o[5] = B1 + 0.0 * t;
    o[6] = B2 + 0.0 * t;
    o[7] = B3 + 2 * 0.0 * t;
  }
  return TR_OK;
}

tr_status tr_create(int device, size_t budget, tr_ctx **out) {
  if (!out) return TR_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return TR_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  tr_ctx *c = new tr_ctx;
  c->device = device;
  c->budget = budget;
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->io_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return TR_ERR_CUDA;
  }
  if (cudaMalloc(&c->err_d, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemset(c->err_d, 0, 2 * sizeof(int)) != cudaSuccess) {
    cudaStreamDestroy(c->io_stream);
    delete c;
    return TR_ERR_CUDA;
  }
  *out = c;
  return TR_OK;
}

tr_status tr_destroy(tr_ctx *c) {
  if (!c) return TR_ERR_ARG;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  release_problem(c);
  for (auto &kv : c->slots) scratch_free(c, kv.first);
  for (int i = 0; i < 2; ++i) {
    if (c->stage_h[i]) cudaFreeHost(c->stage_h[i]);
    if (c->stage_ev[i]) cudaEventDestroy(c->stage_ev[i]);
  }
  if (c->io_stream) cudaStreamDestroy(c->io_stream);
  if (c->cp_in) cudaStreamDestroy(c->cp_in);
  if (c->cp_out) cudaStreamDestroy(c->cp_out);
  for (int i = 0; i < 3; ++i)
    for (cudaEvent_t e : {c->ev_in[i], c->ev_comp[i], c->ev_free[i]})
      if (e) cudaEventDestroy(e);
  if (c->ev_start) cudaEventDestroy(c->ev_start);
  if (c->err_d) cudaFree(c->err_d);
  delete c;
  return TR_OK;
}

const char *tr_last_error(const tr_ctx *c) { return c ? c->err.c_str() : "null context"; }
size_t tr_scratch_bytes(const tr_ctx *c) { return c ? c->scratch : 0; }

tr_status tr_set_problem(tr_ctx *c, int nx, int ny, int nt, int th, int layout,
                         const double *coeff8, float ox, float oy, float oz) {
  if (!c) return TR_ERR_ARG;
  if (nx < 2 || ny < 1 || nt < 1 || th < 1 || !coeff8 ||
      (layout != TR_LAYOUT_Y && layout != TR_LAYOUT_Z))
    return fail(c, TR_ERR_ARG, "bad problem: nx=%d ny=%d ntilt=%d th=%d layout=%d",
                nx, ny, nt, th, layout);
  if ((double)nx * ny * th > 9.0e18 || ny > 65535 * kTY)
    return fail(c, TR_ERR_ARG, "problem too large");
  TR_CUDA(c, cudaSetDevice(c->device));
  TR_CUDA(c, cudaDeviceSynchronize());
  release_problem(c);
  c->nx = nx;
  c->ny = ny;
  c->nt = nt;
  c->th = th;
  TR_CUDA(c, cudaMalloc(&c->geo_d, sizeof(TiltGeo) * nt));
  tr_status st = load_geometry(c, coeff8, nullptr);
  if (st) {
    cudaFree(c->geo_d);
    c->geo_d = nullptr;
    return st;
  }
  c->layout = layout;
  c->ox = ox;
  c->oy = oy;
  c->oz = oz;
  c->have_problem = true;
  return TR_OK;
}

tr_status tr_update_geometry(tr_ctx *c, const double *coeff8, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!coeff8) return fail(c, TR_ERR_ARG, "null coefficients");
  // The old geometry may still be in use by queued kernels on `stream`.
  return load_geometry(c, coeff8, stream ? (cudaStream_t)stream : c->io_stream);
}

tr_status tr_filter_rweight(tr_ctx *c, float *proj, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj) return fail(c, TR_ERR_ARG, "null projections");
  st = build_filter(c, c->nx);
  if (st) return st;
  FilterArgs f;
  f.rows = proj;
  f.nrows = (long long)c->ny * c->nt;
  f.nx = c->nx;
  f.n_pad = c->filt_npad;
  f.log2m = c->filt_log2m;
  f.ghat = c->ghat_d;
  f.tw = c->tw_d;
  TR_CUDA(c, launch_rweight(f, (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_filter_fbp(tr_ctx *c, float *proj, int mode, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || (mode != 0 && mode != 1))
    return fail(c, TR_ERR_ARG, "bad FBP filter arguments (mode %d)", mode);
  // DFT length of the reference: the smallest 2^a 3^b 5^c >= 251 + (nx + 2) - 1
  // (cvGetOptimalDFTSize).
  int L = c->nx + 252;
  for (;; ++L) {
    int r = L;
    while (r % 2 == 0) r /= 2;
    while (r % 3 == 0) r /= 3;
    while (r % 5 == 0) r /= 5;
    if (r == 1) break;
  }
  TR_CUDA(c, launch_fbp_filter(proj, (long long)c->ny * c->nt, c->nx, L, mode,
                               (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_backproject(tr_ctx *c, const float *proj, float *vol, int z0, int nz,
                         void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || z0 < 0 || nz < 1 || z0 + nz > c->th)
    return fail(c, TR_ERR_ARG, "bad back-projection arguments (z0=%d nz=%d)", z0, nz);
  BpArgs a = bp_args(c, vol, z0, nz, proj, 0, c->nt, 1.f);
  TR_CUDA(c, run_bp(c, BP_NORM, a, (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_forward_project(tr_ctx *c, const float *vol, int z0, int nz, float *val,
                             float *wt, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!vol || !val || z0 < 0 || nz < 1 || z0 + nz > c->th)
    return fail(c, TR_ERR_ARG, "bad forward-projection arguments (z0=%d nz=%d)", z0, nz);
  FpArgs a = fp_args(c, vol, z0, nz, val, 0, c->nt);
  TR_TRY(run_fp(c, a, (cudaStream_t)stream));
  if (wt) {
    FpArgs w = fp_args(c, nullptr, z0, nz, wt, 0, c->nt);
    TR_TRY(run_fp(c, w, (cudaStream_t)stream));
  }
  return TR_OK;
}

tr_status tr_forward_project_tilts(tr_ctx *c, const float *vol, int z0, int nz, int t0,
                                   int ntilts, float *val, float *wt, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!vol || !val || z0 < 0 || nz < 1 || z0 + nz > c->th || t0 < 0 || ntilts < 1 ||
      t0 + ntilts > c->nt)
    return fail(c, TR_ERR_ARG, "bad forward-projection arguments (z0=%d nz=%d t0=%d nt=%d)",
                z0, nz, t0, ntilts);
  FpArgs a = fp_args(c, vol, z0, nz, val, 0, ntilts);
  a.geo = c->geo_d + t0;
  TR_TRY(run_fp(c, a, (cudaStream_t)stream));
  if (wt) {
    FpArgs w = fp_args(c, nullptr, z0, nz, wt, 0, ntilts);
    w.geo = c->geo_d + t0;
    TR_TRY(run_fp(c, w, (cudaStream_t)stream));
  }
  return TR_OK;
}

tr_status tr_residual(tr_ctx *c, const float *proj, float *val, const float *wt, int ntilts,
                      void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !val || !wt || ntilts < 1 || ntilts > c->nt)
    return fail(c, TR_ERR_ARG, "bad residual arguments (ntilts=%d)", ntilts);
  TR_CUDA(c, launch_resid(proj, val, wt, (size_t)c->nx * c->ny * ntilts, c->nsm,
                          (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_sirt_update(tr_ctx *c, const float *resid, float *vol, int z0, int nz,
                         float gamma, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!resid || !vol || z0 < 0 || nz < 1 || z0 + nz > c->th)
    return fail(c, TR_ERR_ARG, "bad SIRT update arguments (z0=%d nz=%d)", z0, nz);
  cudaStream_t s = (cudaStream_t)stream;
  if ((st = ensure_wtvol(c, z0, nz, s))) return st;
  BpArgs b = bp_args(c, vol, z0, nz, resid, 0, c->nt, gamma);
  set_weights(c, &b);
  TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
  return TR_OK;
}

tr_status tr_sart_update(tr_ctx *c, const float *resid_plane, int tilt, float *vol, int z0,
                         int nz, float gamma, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!resid_plane || !vol || tilt < 0 || tilt >= c->nt || z0 < 0 || nz < 1 ||
      z0 + nz > c->th)
    return fail(c, TR_ERR_ARG, "bad SART update arguments (tilt=%d z0=%d nz=%d)", tilt, z0,
                nz);
  BpArgs b = bp_args(c, vol, z0, nz, resid_plane, 0, 1, gamma);
  b.geo = c->geo_d + tilt;
  TR_CUDA(c, run_bp(c, BP_NORM, b, (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_sirt(tr_ctx *c, const float *proj, float *vol, int iters, float gamma,
                  void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || iters < 0) return fail(c, TR_ERR_ARG, "bad SIRT arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t pn = proj_elems(c);
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection"))) return st;
  if ((st = ensure_wt(c, s))) return st;
  if ((st = ensure_wtvol(c, 0, c->th, s))) return st;
  for (int it = 0; it < iters; ++it) {
    TR_CUDA(c, cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s));
    FpArgs f = fp_args(c, vol, 0, c->th, c->val_d, 0, c->nt);
    TR_TRY(run_fp(c, f, s));
    TR_CUDA(c, launch_resid(proj, c->val_d, c->wt_d, pn, c->nsm, s));
    BpArgs b = bp_args(c, vol, 0, c->th, c->val_d, 0, c->nt, gamma);
    set_weights(c, &b);
    TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
  }
  return TR_OK;
}

tr_status tr_sirt_gated(tr_ctx *c, const float *proj, float *vol, int max_iters, float gamma,
                        double rel_tol, double *norms, int *iters_done, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || max_iters < 0 || !(rel_tol >= 0))
    return fail(c, TR_ERR_ARG, "bad gated SIRT arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t pn = proj_elems(c);
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection")) ||
      (st = scratch_alloc(c, (void **)&c->admm_dot_d, (kAdmmParts + 3) * sizeof(double),
                          "residual norm")) ||
      (st = ensure_wt(c, s)) || (st = ensure_wtvol(c, 0, c->th, s)))
    return st;
  double *part = c->admm_dot_d, *dnorm = part + kAdmmParts;
  double prev = 0;
  int done = 0;
  for (int it = 0; it < max_iters; ++it) {
    TR_CUDA(c, cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s));
    TR_TRY(run_fp(c, fp_args(c, vol, 0, c->th, c->val_d, 0, c->nt), s));
    TR_CUDA(c, launch_resid(proj, c->val_d, c->wt_d, pn, c->nsm, s));
    // |r|^2 in FP64 with fixed-order partial sums, read back to gate
    TR_CUDA(c, sumsq_f64(c->val_d, pn, part, dnorm, s));
    double h = 0;
    TR_CUDA(c, cudaMemcpyAsync(&h, dnorm, sizeof(double), cudaMemcpyDeviceToHost, s));
    TR_CUDA(c, cudaStreamSynchronize(s));
    const double nrm = sqrt(h);
    if (norms) norms[it] = nrm;
    if (it > 0 && rel_tol > 0 && prev - nrm < rel_tol * prev) break;  // converged
    BpArgs b = bp_args(c, vol, 0, c->th, c->val_d, 0, c->nt, gamma);
    set_weights(c, &b);
    TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
    prev = nrm;
    done = it + 1;
  }
  if (iters_done) *iters_done = done;
  TR_CUDA(c, cudaStreamSynchronize(s));
  return take_timeout(c);
}

tr_status tr_sart(tr_ctx *c, const float *proj, float *vol, int iters, float gamma,
                  void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || iters < 0) return fail(c, TR_ERR_ARG, "bad SART arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t plane = (size_t)c->nx * c->ny;
  if ((st = scratch_alloc(c, (void **)&c->val_d, proj_elems(c) * sizeof(float),
                          "reprojection")))
    return st;
  if ((st = ensure_wt(c, s))) return st;
  for (int it = 0; it < iters; ++it)
    for (int t = 0; t < c->nt; ++t) {
      float *vt = c->val_d + plane * t;
      TR_CUDA(c, cudaMemsetAsync(vt, 0, plane * sizeof(float), s));
      FpArgs f = fp_args(c, vol, 0, c->th, c->val_d, t, 1);
      TR_TRY(run_fp(c, f, s));
      TR_CUDA(c, launch_resid(proj + plane * t, vt, c->wt_d + plane * t, plane, c->nsm, s));
      BpArgs b = bp_args(c, vol, 0, c->th, c->val_d, t, 1, gamma);
      TR_CUDA(c, run_bp(c, BP_NORM, b, s));
    }
  return TR_OK;
}

tr_status tr_quantize(tr_ctx *c, const float *proj, int dtype, void *out, float *scale,
                      void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !out || !scale || (dtype != TR_DTYPE_F16 && dtype != TR_DTYPE_BF16))
    return fail(c, TR_ERR_ARG, "bad quantize arguments (dtype=%d)", dtype);
  if ((st = scratch_alloc(c, (void **)&c->maxbits_d, sizeof(unsigned) * c->nt,
                          "per-tilt maxima")))
    return st;
  TR_CUDA(c, launch_quantize(proj, (size_t)c->nx * c->ny, c->nt, dtype, out, scale,
                             c->maxbits_d, c->nsm, (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_backproject_lp(tr_ctx *c, const void *proj, int dtype, const float *scale,
                            float *vol, int z0, int nz, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || z0 < 0 || nz < 1 || z0 + nz > c->th ||
      (dtype != TR_DTYPE_F32 && dtype != TR_DTYPE_F16 && dtype != TR_DTYPE_BF16))
    return fail(c, TR_ERR_ARG, "bad back-projection arguments (z0=%d nz=%d dtype=%d)", z0,
                nz, dtype);
  BpArgs a = bp_args(c, vol, z0, nz, (const float *)proj, 0, c->nt, 1.f);
  a.img.dtype = dtype;
  a.img.scale = scale;
  TR_CUDA(c, run_bp(c, BP_NORM, a, (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_sirt_lp(tr_ctx *c, const void *proj, int pdtype, const float *scale, int rdtype,
                     float *vol, int iters, float gamma, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  auto ok_dtype = [](int d) {
    return d == TR_DTYPE_F32 || d == TR_DTYPE_F16 || d == TR_DTYPE_BF16;
  };
  if (!proj || !vol || iters < 0 || !ok_dtype(pdtype) || !ok_dtype(rdtype) ||
      (pdtype != TR_DTYPE_F32 && !scale))
    return fail(c, TR_ERR_ARG, "bad SIRT arguments (proj dtype %d, residual dtype %d)",
                pdtype, rdtype);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t plane = (size_t)c->nx * c->ny, pn = proj_elems(c);
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection"))) return st;
  if (rdtype != TR_DTYPE_F32 &&
      (st = scratch_alloc(c, &c->res16_d, pn * 2, "16-bit residual")))
    return st;
  if (rdtype == TR_DTYPE_F16 &&
      ((st = scratch_alloc(c, (void **)&c->rscale_d, sizeof(float) * c->nt,
                           "residual scales")) ||
       (st = scratch_alloc(c, (void **)&c->maxbits_d, sizeof(unsigned) * c->nt,
                           "per-tilt maxima"))))
    return st;
  if ((st = ensure_wt(c, s))) return st;
  if ((st = ensure_wtvol(c, 0, c->th, s))) return st;
  const float *ps = pdtype == TR_DTYPE_F32 ? nullptr : scale;
  void *res = rdtype == TR_DTYPE_F32 ? (void *)c->val_d : c->res16_d;
  const float *rs = rdtype == TR_DTYPE_F16 ? c->rscale_d : nullptr;
  for (int it = 0; it < iters; ++it) {
    TR_CUDA(c, cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s));
    FpArgs f = fp_args(c, vol, 0, c->th, c->val_d, 0, c->nt);
    TR_TRY(run_fp(c, f, s));
    if (rdtype == TR_DTYPE_F16) {
      // The residual's range is not the stack's (a WBP start, for one, makes
      // it larger): form it in FP32, then store it with its own per-tilt
      // power-of-two scales.
      TR_CUDA(c, launch_resid_lp(proj, pdtype, ps, c->val_d, c->wt_d, plane, c->nt,
                                 TR_DTYPE_F32, c->val_d, nullptr, c->nsm, s));
      TR_CUDA(c, launch_quantize(c->val_d, plane, c->nt, TR_DTYPE_F16, c->res16_d, c->rscale_d,
                                 c->maxbits_d, c->nsm, s));
    } else {
      TR_CUDA(c, launch_resid_lp(proj, pdtype, ps, c->val_d, c->wt_d, plane, c->nt, rdtype,
                                 res, nullptr, c->nsm, s));
    }
    BpArgs b = bp_args(c, vol, 0, c->th, (const float *)res, 0, c->nt, gamma);
    b.img.dtype = rdtype;
    b.img.scale = rs;
    set_weights(c, &b);
    TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
  }
  return TR_OK;
}

tr_status tr_host_alloc(size_t bytes, void **out) {
  if (!out) return TR_ERR_ARG;
  *out = nullptr;
  if (cudaHostAlloc(out, std::max<size_t>(bytes, 1), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return TR_ERR_OOM;
  }
  return TR_OK;
}

tr_status tr_host_free(void *p) {
  if (p && cudaFreeHost(p) != cudaSuccess) {
    cudaGetLastError();
    return TR_ERR_CUDA;
  }
  return TR_OK;
}

tr_status tr_sirt_host_zslabs(tr_ctx *c, const float *proj_h, float *vol_h, int zero_start,
                              int iters, float gamma, int depth, int *depth_used) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj_h || !vol_h || iters < 0 || depth < 0)
    return fail(c, TR_ERR_ARG, "bad host z-slab SIRT arguments");
  scratch_free(c, (void **)&c->hvol_d);  // a device copy of the volume is what does not fit
  if ((st = host_buffers(c, false))) return st;  // the stack only: the volume stays here
  cudaStream_t s = c->io_stream;
  TR_CUDA(c, cudaMemcpyAsync(c->hproj_d, proj_h, proj_elems(c) * sizeof(float),
                             cudaMemcpyHostToDevice, s));
  TR_CUDA(c, cudaStreamSynchronize(s));
  if (zero_start) memset(vol_h, 0, vol_elems(c) * sizeof(float));
  if (depth == 0 && (st = tr_autotune_zslab(c, c->hproj_d, TR_DTYPE_F32, nullptr, TR_DTYPE_F32,
                                            vol_h, 1, &depth, nullptr)))
    return st;
  if (depth_used) *depth_used = slab_depth(c, depth);
  return tr_sirt_zslabs(c, c->hproj_d, TR_DTYPE_F32, nullptr, TR_DTYPE_F32, vol_h, 1, iters,
                        gamma, depth, s);
}

tr_status tr_set_deterministic(tr_ctx *c, int on) {
  if (!c) return TR_ERR_ARG;
  c->deterministic = on != 0;
  c->wt_ready = false;  // recompute the projection weights the same way
  return TR_OK;
}

tr_status tr_sirt_zslabs(tr_ctx *c, const void *proj, int pdtype, const float *scale,
                         int rdtype, float *vol, int vol_on_host, int iters, float gamma,
                         int depth, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  auto ok_dtype = [](int d) {
    return d == TR_DTYPE_F32 || d == TR_DTYPE_F16 || d == TR_DTYPE_BF16;
  };
  if (!proj || !vol || iters < 0 || depth < 1 || !ok_dtype(pdtype) || !ok_dtype(rdtype) ||
      (pdtype != TR_DTYPE_F32 && !scale))
    return fail(c, TR_ERR_ARG, "bad z-slab SIRT arguments (depth %d, dtypes %d/%d)", depth,
                pdtype, rdtype);
  SlabRun r{proj, pdtype, scale, rdtype, vol, vol_on_host != 0, iters, gamma,
            slab_depth(c, depth)};
  st = slab_sirt(c, r, (cudaStream_t)stream);
  if (!st && r.host) st = take_timeout(c);
  return st;
}

tr_status tr_autotune_zslab(tr_ctx *c, const void *proj, int pdtype, const float *scale,
                            int rdtype, float *vol, int vol_on_host, int *depth_out,
                            double *sweep_ms) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || !depth_out || (pdtype != TR_DTYPE_F32 && !scale))
    return fail(c, TR_ERR_ARG, "bad z-slab autotune arguments");
  cudaStream_t s = c->io_stream;
  cudaEvent_t e0, e1;
  TR_CUDA(c, cudaEventCreate(&e0));
  TR_CUDA(c, cudaEventCreate(&e1));
  int best = 0;
  double best_ms = 0;
  int last = 0;
  for (int want : {32, 64, 128, 256, 512}) {
    const int d = slab_depth(c, want);
    if (d == last) continue;
    last = d;
    // gamma 0 over a zero residual: the sweep does the full work (copies,
    // update, forward projection) and leaves the volume's values unchanged.
    SlabRun r{proj, pdtype, scale, rdtype, vol, vol_on_host != 0, 1, 0.f, d};
    if ((st = slab_scratch(c, r, s))) {
      if (st == TR_ERR_BUDGET || st == TR_ERR_OOM) continue;  // this depth does not fit
      break;
    }
    const size_t pn = proj_elems(c);
    const void *res = rdtype == TR_DTYPE_F32 ? (const void *)c->val_d : c->res16_d;
    const float *rs = rdtype == TR_DTYPE_F16 ? c->rscale_d : nullptr;
    cudaError_t e = cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s);
    if (e == cudaSuccess && rdtype != TR_DTYPE_F32) e = cudaMemsetAsync(c->res16_d, 0, pn * 2, s);
    if (e == cudaSuccess && rs) e = cudaMemsetAsync(c->rscale_d, 0, c->nt * sizeof(float), s);
    if (e != cudaSuccess) {
      st = cuda_fail(c, e, "clearing the autotune residual");
      break;
    }
    double ms = 0;
    for (int rep = 0; rep < 2 && !st; ++rep) {  // the first sweep warms up
      st = cudaEventRecord(e0, s) ? TR_ERR_CUDA : TR_OK;
      if (!st) st = slab_sweep(c, r, c->th, res, rs, c->val2_d, s);
      if (!st && cudaEventRecord(e1, s)) st = TR_ERR_CUDA;
      if (!st && cudaEventSynchronize(e1)) st = TR_ERR_CUDA;
      float f = 0;
      if (!st) cudaEventElapsedTime(&f, e0, e1);
      ms = f;
    }
    if (st) break;
    if (!best || ms < best_ms) {
      best = d;
      best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st && st != TR_ERR_BUDGET && st != TR_ERR_OOM) return st;
  if (!best) return fail(c, TR_ERR_BUDGET, "no slab depth fits the budget");
  if ((st = take_timeout(c))) return st;
  c->err.clear();
  *depth_out = best;
  if (sweep_ms) *sweep_ms = best_ms;
  return TR_OK;
}

tr_status tr_admm(tr_ctx *c, const float *proj, float *vol, int outer, int cg_iters, float mu,
                  float soft, void *stream) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj || !vol || outer < 0 || cg_iters < 0)
    return fail(c, TR_ERR_ARG, "bad ADMM arguments (outer %d, cg %d)", outer, cg_iters);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t pn = proj_elems(c), V = vol_elems(c);
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection")) ||
      (st = scratch_alloc(c, (void **)&c->admm_d, 7 * V * sizeof(float), "ADMM volumes")) ||
      (st = scratch_alloc(c, (void **)&c->admm_dot_d, (kAdmmParts + 3) * sizeof(double),
                          "ADMM scalars")))
    return st;
  if ((st = ensure_wt(c, s))) return st;
  float *atb = c->admm_d, *u = atb + V, *d = u + V, *ax = d + V, *r = ax + V, *p = r + V,
        *h = p + V;
  double *part = c->admm_dot_d, *scal = part + kAdmmParts;
  const int nsm = c->nsm;
  // out = (A^T D A + mu I) x, Reproject_admm_atax + ATAmuLTL (main-mpiz.cpp:657-841):
  // the forward splat, its normalisation by the projection weights, the
  // unnormalised gather over all tilts, plus mu x.
  auto apply = [&](const float *x, float *out) -> tr_status {
    TR_CUDA(c, cudaMemsetAsync(out, 0, V * sizeof(float), s));
    TR_CUDA(c, cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s));
    TR_TRY(run_fp(c, fp_args(c, x, 0, c->th, c->val_d, 0, c->nt), s));
    TR_CUDA(c, admm_normalize(c->val_d, c->wt_d, pn, nsm, s));
    TR_CUDA(c, run_bp(c, BP_SUM, bp_args(c, out, 0, c->th, c->val_d, 0, c->nt, 1.f), s));
    TR_CUDA(c, admm_add_scaled(out, x, mu, V, nsm, s));
    return TR_OK;
  };
  // A^T b (Reproject_admm_htb, :603-656), u = d = 0.
  TR_CUDA(c, cudaMemsetAsync(atb, 0, 3 * V * sizeof(float), s));
  TR_CUDA(c, run_bp(c, BP_SUM, bp_args(c, atb, 0, c->th, proj, 0, c->nt, 1.f), s));
  for (int it = 0; it < outer; ++it) {
    // The reference adds (u - d) mu to A^T b itself, so the term accumulates
    // over outer iterations (ATbmuLT on htb, :989).
    TR_CUDA(c, admm_atb(atb, u, d, mu, V, nsm, s));
    if ((st = apply(vol, ax))) return st;
    // applycg (:843-938)
    TR_CUDA(c, admm_cg_init(r, p, atb, ax, V, nsm, s));
    for (int k = 0; k < cg_iters; ++k) {
      if ((st = apply(p, h))) return st;
      TR_CUDA(c, admm_dot(r, r, V, part, scal + 0, s));
      TR_CUDA(c, admm_dot(h, p, V, part, scal + 1, s));
      TR_CUDA(c, admm_x_update(vol, p, scal, V, nsm, s));
      if ((st = apply(vol, ax))) return st;
      TR_CUDA(c, admm_r_update(r, atb, ax, V, nsm, s));
      TR_CUDA(c, admm_dot(r, h, V, part, scal + 2, s));
      TR_CUDA(c, admm_p_update(p, r, scal, V, nsm, s));
    }
    TR_CUDA(c, admm_soft(u, d, vol, soft, V, nsm, s));
  }
  return TR_OK;
}

tr_status tr_admm_host(tr_ctx *c, const float *proj_h, float *vol_h, int outer, int cg_iters,
                       float mu, float soft) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj_h || !vol_h) return fail(c, TR_ERR_ARG, "null host buffer");
  if ((st = host_buffers(c))) return st;
  cudaStream_t s = c->io_stream;
  const size_t pn = proj_elems(c), vn = vol_elems(c);
  TR_CUDA(c, cudaMemcpyAsync(c->hproj_d, proj_h, pn * sizeof(float), cudaMemcpyHostToDevice, s));
  TR_CUDA(c, cudaMemcpyAsync(c->hvol_d, vol_h, vn * sizeof(float), cudaMemcpyHostToDevice, s));
  if ((st = tr_admm(c, c->hproj_d, c->hvol_d, outer, cg_iters, mu, soft, s))) return st;
  TR_CUDA(c, cudaMemcpyAsync(vol_h, c->hvol_d, vn * sizeof(float), cudaMemcpyDeviceToHost, s));
  TR_CUDA(c, cudaStreamSynchronize(s));
  return take_timeout(c);
}

tr_status tr_wbp(tr_ctx *c, float *proj, float *vol, void *stream) {
  tr_status st = tr_filter_rweight(c, proj, stream);
  if (st) return st;
  return tr_backproject(c, proj, vol, 0, c->th, stream);
}

}  // extern "C"

namespace {

// Uploads the host stack (and the starting volume, or zeroes it) to the
// context's device copies and runs `method` on them, ordered on io_stream.
// Host memory the GPU can copy asynchronously (page-locked or registered).
bool host_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Copies sections [z0, z0 + nz) of the device volume into the host volume.
cudaError_t vol_sections_d2h(const tr_ctx *c, float *host, const float *dev, int z0, int nz,
                             cudaStream_t s) {
  const size_t nx = c->nx, ny = c->ny;
  if (c->layout == TR_LAYOUT_Z)
    return cudaMemcpyAsync(host + (size_t)z0 * nx * ny, dev + (size_t)z0 * nx * ny,
                           (size_t)nz * nx * ny * sizeof(float), cudaMemcpyDeviceToHost, s);
  const size_t pitch = nx * (size_t)c->th * sizeof(float);
  return cudaMemcpy2DAsync(host + (size_t)z0 * nx, pitch, dev + (size_t)z0 * nx, pitch,
                           (size_t)nz * nx * sizeof(float), ny, cudaMemcpyDeviceToHost, s);
}

// SIRT from page-locked host buffers with the copies overlapped: the stack's
// upload runs on a copy stream while the geometry-only weights are computed,
// and the last iteration's update runs in z-slabs (about four, tile-aligned)
// whose sections go back to the host while the next slab updates.  The same
// launches as tr_sirt, so the same volume.
tr_status sirt_host_overlapped(tr_ctx *c, const float *proj_h, float *vol_h, bool zero_start,
                               int iters, float gamma) {
  const size_t pn = proj_elems(c), vn = vol_elems(c);
  tr_status st = host_buffers(c);
  if (st || (st = slab_streams(c))) return st;
  cudaStream_t s = c->io_stream;
  TR_CUDA(c, cudaEventRecord(c->ev_start, s));
  TR_CUDA(c, cudaStreamWaitEvent(c->cp_in, c->ev_start, 0));
  TR_CUDA(c, cudaMemcpyAsync(c->hproj_d, proj_h, pn * sizeof(float), cudaMemcpyHostToDevice,
                             c->cp_in));
  if (!zero_start)
    TR_CUDA(c, cudaMemcpyAsync(c->hvol_d, vol_h, vn * sizeof(float), cudaMemcpyHostToDevice,
                               c->cp_in));
  TR_CUDA(c, cudaEventRecord(c->ev_in[0], c->cp_in));
  if (zero_start) TR_CUDA(c, cudaMemsetAsync(c->hvol_d, 0, vn * sizeof(float), s));
  if ((st = scratch_alloc(c, (void **)&c->val_d, pn * sizeof(float), "reprojection")) ||
      (st = ensure_wt(c, s)) || (st = ensure_wtvol(c, 0, c->th, s)))
    return st;
  TR_CUDA(c, cudaStreamWaitEvent(s, c->ev_in[0], 0));
  if (iters > 1 && (st = tr_sirt(c, c->hproj_d, c->hvol_d, iters - 1, gamma, s))) return st;
  if (iters > 0) {  // the last iteration: forward projection and residual as tr_sirt
    TR_CUDA(c, cudaMemsetAsync(c->val_d, 0, pn * sizeof(float), s));
    TR_TRY(run_fp(c, fp_args(c, c->hvol_d, 0, c->th, c->val_d, 0, c->nt), s));
    TR_CUDA(c, launch_resid(c->hproj_d, c->val_d, c->wt_d, pn, c->nsm, s));
  }
  const int depth = c->th >= 4 * kTZ ? slab_depth(c, c->th / 4) : c->th;
  const dim3 g = bp_tile_grid(full_view(c, nullptr, 0, c->th));
  int k = 0;
  for (int z0 = 0; z0 < c->th; z0 += depth, k = (k + 1) % kSlabBufs) {
    const int nz = std::min(depth, c->th - z0);
    if (iters > 0) {
      BpArgs b = bp_args(c, nullptr, z0, nz, c->val_d, 0, c->nt, gamma);
      b.v = slab_view(c, c->hvol_d, false, z0, nz);
      set_weights(c, &b);
      b.wslot = c->wslot_d + (size_t)(z0 / kTZ) * g.x * g.y;  // this slab's tiles
      TR_CUDA(c, run_bp(c, BP_SIRT, b, s));
    }
    TR_CUDA(c, cudaEventRecord(c->ev_comp[k], s));
    TR_CUDA(c, cudaStreamWaitEvent(c->cp_out, c->ev_comp[k], 0));
    TR_CUDA(c, vol_sections_d2h(c, vol_h, c->hvol_d, z0, nz, c->cp_out));
  }
  TR_CUDA(c, cudaStreamSynchronize(c->cp_out));
  TR_CUDA(c, cudaStreamSynchronize(s));
  return take_timeout(c);
}

tr_status run_host_method(tr_ctx *c, int method, const float *proj_h, const float *vol_h,
                          bool zero_start, int iters, float gamma) {
  const size_t pn = proj_elems(c), vn = vol_elems(c);
  tr_status st = host_buffers(c);
  if (st) return st;
  cudaStream_t s = c->io_stream;
  TR_CUDA(c, cudaMemcpyAsync(c->hproj_d, proj_h, pn * sizeof(float), cudaMemcpyHostToDevice, s));
  if (zero_start)
    TR_CUDA(c, cudaMemsetAsync(c->hvol_d, 0, vn * sizeof(float), s));
  else
    TR_CUDA(c, cudaMemcpyAsync(c->hvol_d, vol_h, vn * sizeof(float), cudaMemcpyHostToDevice, s));
  switch (method) {
    case TR_METHOD_BPT: return tr_backproject(c, c->hproj_d, c->hvol_d, 0, c->th, s);
    case TR_METHOD_WBP: return tr_wbp(c, c->hproj_d, c->hvol_d, s);
    case TR_METHOD_FBP:
      st = tr_filter_fbp(c, c->hproj_d, 0, s);
      return st ? st : tr_backproject(c, c->hproj_d, c->hvol_d, 0, c->th, s);
    case TR_METHOD_SIRT: return tr_sirt(c, c->hproj_d, c->hvol_d, iters, gamma, s);
    case TR_METHOD_SART: return tr_sart(c, c->hproj_d, c->hvol_d, iters, gamma, s);
    default: return fail(c, TR_ERR_ARG, "unknown method %d", method);
  }
}

}  // namespace

extern "C" {

tr_status tr_reconstruct_host(tr_ctx *c, int method, const float *proj_h, float *vol_h,
                              int iters, float gamma) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj_h || !vol_h) return fail(c, TR_ERR_ARG, "null host buffer");
  const bool zero_start = (method & TR_RECON_ZERO_START) != 0;
  if ((method & ~TR_RECON_ZERO_START) == TR_METHOD_SIRT && iters >= 0 && host_pinned(proj_h) &&
      host_pinned(vol_h))
    return sirt_host_overlapped(c, proj_h, vol_h, zero_start, iters, gamma);
  if ((st = run_host_method(c, method & ~TR_RECON_ZERO_START, proj_h, vol_h, zero_start, iters,
                            gamma)))
    return st;
  cudaStream_t s = c->io_stream;
  TR_CUDA(c, cudaMemcpyAsync(vol_h, c->hvol_d, vol_elems(c) * sizeof(float),
                             cudaMemcpyDeviceToHost, s));
  TR_CUDA(c, cudaStreamSynchronize(s));
  return take_timeout(c);
}

tr_status tr_volume_to_bytes(tr_ctx *c, const float *vol, size_t n, size_t slab, float alpha,
                             unsigned char *out, void *stream) {
  if (!c) return TR_ERR_ARG;
  if (!vol || !out || n == 0 || slab == 0 || (n + slab - 1) / slab > 65535)
    return fail(c, TR_ERR_ARG, "bad byte-output arguments (n=%zu slab=%zu)", n, slab);
  TR_CUDA(c, cudaSetDevice(c->device));
  const size_t nslabs = (n + slab - 1) / slab;
  tr_status st;
  if ((st = scratch_alloc(c, (void **)&c->f2b_part_d, nslabs * kF2bParts * sizeof(double),
                          "byte-output partial sums")) ||
      (st = scratch_alloc(c, (void **)&c->f2b_stats_d, 4 * nslabs * sizeof(float),
                          "byte-output statistics")))
    return st;
  TR_CUDA(c, launch_f2b(vol, n, slab, alpha, out, c->f2b_part_d, c->f2b_stats_d, c->nsm,
                        (cudaStream_t)stream));
  return TR_OK;
}

tr_status tr_reconstruct_to_sink(tr_ctx *c, int method, const float *proj_h,
                                 const float *vol_init_h, int iters, float gamma,
                                 size_t f2b_slab, float f2b_alpha, size_t block_bytes,
                                 tr_block_sink sink, void *user) {
  tr_status st = need_problem(c);
  if (st) return st;
  if (!proj_h || !sink || block_bytes == 0)
    return fail(c, TR_ERR_ARG, "bad streamed-output arguments");
  if ((st = run_host_method(c, method, proj_h, vol_init_h, vol_init_h == nullptr, iters, gamma)))
    return st;
  cudaStream_t s = c->io_stream;
  const size_t vn = vol_elems(c);
  const unsigned char *src = reinterpret_cast<const unsigned char *>(c->hvol_d);
  size_t total = vn * sizeof(float);
  if (f2b_slab) {
    if ((st = scratch_alloc(c, (void **)&c->bytes_d, vn, "byte volume"))) return st;
    if ((st = tr_volume_to_bytes(c, c->hvol_d, vn, f2b_slab, f2b_alpha, c->bytes_d, s)))
      return st;
    src = c->bytes_d;
    total = vn;
  }
  if (c->stage_n != block_bytes) {
    for (int i = 0; i < 2; ++i) {
      if (c->stage_h[i]) cudaFreeHost(c->stage_h[i]);
      c->stage_h[i] = nullptr;
    }
    c->stage_n = 0;
    for (int i = 0; i < 2; ++i) TR_CUDA(c, cudaHostAlloc(&c->stage_h[i], block_bytes, 0));
    c->stage_n = block_bytes;
  }
  for (int i = 0; i < 2; ++i)
    if (!c->stage_ev[i])
      TR_CUDA(c, cudaEventCreateWithFlags(&c->stage_ev[i], cudaEventDisableTiming));
  const size_t nblocks = (total + block_bytes - 1) / block_bytes;
  auto issue = [&](size_t k) -> cudaError_t {
    const size_t off = k * block_bytes, len = std::min(block_bytes, total - off);
    cudaError_t e = cudaMemcpyAsync(c->stage_h[k & 1], src + off, len, cudaMemcpyDeviceToHost, s);
    return e == cudaSuccess ? cudaEventRecord(c->stage_ev[k & 1], s) : e;
  };
  for (size_t k = 0; k < std::min<size_t>(2, nblocks); ++k) TR_CUDA(c, issue(k));
  for (size_t k = 0; k < nblocks; ++k) {
    TR_CUDA(c, cudaEventSynchronize(c->stage_ev[k & 1]));
    const size_t off = k * block_bytes, len = std::min(block_bytes, total - off);
    if (sink(user, c->stage_h[k & 1], off, len) != 0) {
      cudaStreamSynchronize(s);
      return fail(c, TR_ERR_ARG, "the output sink stopped the transfer at byte %zu", off);
    }
    if (k + 2 < nblocks) TR_CUDA(c, issue(k + 2));
  }
  TR_CUDA(c, cudaStreamSynchronize(s));
  return take_timeout(c);
}

tr_status tr_resample_bin(const float *src, int nx, int ny, int nt, int bin, float *dst,
                          void *stream) {
  if (!src || !dst || nx < 1 || ny < 1 || nt < 1 || bin < 1 || bin > 64 || nx / bin < 1 ||
      ny / bin < 1)
    return TR_ERR_ARG;
  if (launch_resample_bin(src, nx, ny, nt, bin, dst, (cudaStream_t)stream) != cudaSuccess)
    return TR_ERR_CUDA;
  return TR_OK;
}

tr_status tr_resample_bin_host(int device, const float *src, int nx, int ny, int nt, int bin,
                               float *dst) {
  if (!src || !dst || nx < 1 || ny < 1 || nt < 1 || bin < 1 || bin > 64 || nx / bin < 1 ||
      ny / bin < 1)
    return TR_ERR_ARG;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return TR_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  const size_t in_b = (size_t)nx * ny * nt * sizeof(float);
  const size_t out_b = (size_t)(nx / bin) * (ny / bin) * nt * sizeof(float);
  float *s_d = nullptr, *d_d = nullptr;
  tr_status st = TR_OK;
  if (cudaMalloc(&s_d, in_b) != cudaSuccess || cudaMalloc(&d_d, out_b) != cudaSuccess) {
    cudaGetLastError();
    st = TR_ERR_OOM;
  } else if (cudaMemcpy(s_d, src, in_b, cudaMemcpyHostToDevice) != cudaSuccess ||
             launch_resample_bin(s_d, nx, ny, nt, bin, d_d, nullptr) != cudaSuccess ||
             cudaMemcpy(dst, d_d, out_b, cudaMemcpyDeviceToHost) != cudaSuccess) {
    st = TR_ERR_CUDA;
  }
  if (s_d) cudaFree(s_d);
  if (d_d) cudaFree(d_d);
  return st;
}

tr_status tr_selftest_wait(tr_ctx *c, int budget_us) {
  if (!c || budget_us < 1 || budget_us > 10000000) return TR_ERR_ARG;
  TR_CUDA(c, cudaSetDevice(c->device));
  int khz = 0;
  TR_CUDA(c, cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, c->device));
  const long long cycles = (long long)khz * budget_us / 1000;
  TR_CUDA(c, cudaMemsetAsync(c->err_d, 0, 2 * sizeof(int), c->io_stream));
  TR_CUDA(c, launch_bounded_wait_selftest(cycles, c->err_d, c->io_stream));
  TR_CUDA(c, cudaStreamSynchronize(c->io_stream));
  return take_timeout(c);
}

tr_status tr_synchronize(tr_ctx *c) {
  if (!c) return TR_ERR_ARG;
  TR_CUDA(c, cudaSetDevice(c->device));
  TR_CUDA(c, cudaDeviceSynchronize());
  return take_timeout(c);
}

}  // extern "C"
