// Job scheduler: many reconstructions on one device, batched per step.
//
// The reference reconstructs one tilt series per process run (TiltRec-cuda /
// TiltRec-mpi launched by the GUI's command chain); it has no batching or
// serving.  This scheduler keeps many jobs device-resident and advances all of
// them together: every step is one table of work items run by four launches
// (zero, persistent forward projection, residual, FP16 residual maxima and
// conversion, persistent back-projection)
// captured once in a CUDA graph and replayed with a new table each step.  A
// job's SIRT iterations are consecutive steps; a WBP job (or the WBP start of
// a WBP-then-SIRT job) is one back-projection item.
//
// Jobs are admitted in submission order while their device memory fits the
// HBM budget.  Admission (upload, 16-bit quantisation of the projections,
// WBP filtering, projection and voxel weights) runs on a preparation stream
// and overlaps the steps of the jobs already running; a finished job's volume
// is copied back on a third stream.  A background thread drives the steps.
//
// Per-job results do not depend on the other jobs in the step: each voxel is
// written by one CTA summing its tilts in order, and each forward-projection
// tile adds its window into the job's own accumulators; only the order of the
// float atomic adds of different tiles into one detector pixel varies from run
// to run (as it does for a job run alone).
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "tiltrec_b200.h"
#include "tr_filter_host.h"
#include "tr_geom.h"
#include "tr_internal.cuh"

using namespace trb;

namespace {

constexpr size_t kSchedSmemFp = 44 * 1024;  // four FP CTAs per SM with the static bookkeeping
constexpr size_t kSchedSmemMax = 200 * 1024;

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t elem_size(int dtype) { return dtype == TR_DTYPE_F32 ? 4 : 2; }

enum JobState { J_QUEUED, J_LOADING, J_READY, J_DRAINING, J_COPYBACK, J_DONE };

struct Job {
  unsigned long long id = 0;
  tr_job d{};
  std::vector<double> coeff;
  GeomInfo gi{};
  size_t plane = 0, nvox = 0, bytes = 0;
  // device memory owned by the job (stream-ordered allocations)
  TiltGeo *geo = nullptr;
  float *val = nullptr, *wt = nullptr, *wtvol = nullptr, *vol_own = nullptr;
  float *wrow = nullptr;  // separable per-row voxel weights
  int *wslot = nullptr;   // compact voxel weights: a slot per tile, then the border count
  void *pstore = nullptr, *res = nullptr;
  float *pscale = nullptr, *rscale = nullptr;
  unsigned *maxbits = nullptr;
  // what the steps read
  float *vol = nullptr;
  const void *proj = nullptr;
  int pdtype = TR_DTYPE_F32, rdtype = TR_DTYPE_F32;
  const float *ps = nullptr, *rs = nullptr;
  BatchBp bp_norm{}, bp_sirt{};
  BatchFp fp{};
  BpArgs a_norm{}, a_sirt{};  // the same work for the per-job kernels
  double work = 0;            // remaining voxel-projection updates
  size_t smem_norm = 0, smem_sirt = 0;
  // progress
  JobState state = J_QUEUED;
  bool wbp_pending = false;
  int iters_left = 0;
  cudaEvent_t ev_ready = nullptr, ev_done = nullptr, ev_copied = nullptr;
  double t_submit = 0, t_ready = 0, t_done = 0;
  tr_status status = TR_OK;
};

}  // namespace

struct tr_sched {
  int device = 0, nsm = 148;
  size_t budget = 0, used = 0, peak = 0;
  int pdtype = TR_DTYPE_F32, rdtype = TR_DTYPE_F32;
  cudaStream_t s = nullptr, prep = nullptr, back = nullptr;
  int *err_d = nullptr;
  // step tables, double-buffered
  BatchTable *tab_d[2] = {nullptr, nullptr};
  BatchTable *tab_h[2] = {nullptr, nullptr};
  cudaEvent_t tab_ev[2] = {nullptr, nullptr};
  bool tab_used[2] = {false, false};
  int next_tab = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // launch configuration (autotuned)
  size_t smem_bp = 56 * 1024, smem_fp = kSchedSmemFp;
  int grid_bp = 0, grid_fp = 0;
  // R-weighting spectra per row length (device, shared by jobs)
  std::map<int, std::pair<float2 *, float2 *>> filt;
  std::map<int, RweightSpectrum> filt_h;
  // jobs
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<std::shared_ptr<Job>> queue;
  std::vector<std::shared_ptr<Job>> active;
  std::map<unsigned long long, std::shared_ptr<Job>> all;
  unsigned long long next_id = 1;
  bool stop = false;
  std::thread worker;
  std::string err;
  tr_status fatal = TR_OK;
  // TR_SCHED_BATCHED or TR_SCHED_SRPT, and the SRPT aging time (0: none)
  int policy = TR_SCHED_BATCHED;
  double aging_s = 0;
  // counters
  long long steps = 0, items_bp = 0, items_fp = 0;
};

namespace {

tr_status sched_fail(tr_sched *S, tr_status st, const std::string &msg) {
  if (!S->fatal) {
    S->fatal = st;
    S->err = msg;
  }
  return st;
}

#define SCHED_CUDA(S, call)                                                         \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return sched_fail(S, TR_ERR_CUDA,                                             \
                        std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

VolView job_view(const Job &j, float *vol) {
  VolView v;
  v.vol = vol;
  v.nx = j.d.nx;
  v.ny = j.d.ny;
  v.nz = j.d.thickness;
  v.zoff = 0;
  if (j.d.layout == TR_LAYOUT_Y) {
    v.sy = (long long)j.d.thickness * j.d.nx;
    v.sz = j.d.nx;
  } else {
    v.sy = j.d.nx;
    v.sz = (long long)j.d.ny * j.d.nx;
  }
  return v;
}

BpArgs job_bp(const tr_sched *S, const Job &j, const void *img, int dtype, const float *scale,
              float gamma) {
  BpArgs a{};
  a.v = job_view(j, j.vol);
  a.img.p = (const float *)img;
  a.img.nx = j.d.nx;
  a.img.ny = j.d.ny;
  a.img.tstride = (long long)j.d.nx * j.d.ny;
  a.img.dtype = dtype;
  a.img.scale = scale;
  a.geo = j.geo;
  a.t0 = 0;
  a.nt = j.d.ntilt;
  a.ox = j.d.ox;
  a.oy = j.d.oy;
  a.oz = j.d.oz;
  a.fw = j.gi.fw;
  a.fh = j.gi.fh;
  a.chunk = chunk_for(64 * 1024, j.gi.bp_tilt_bytes);
  a.gamma = gamma;
  a.wtvol = nullptr;
  a.out = nullptr;
  a.err = S->err_d;
  return a;
}

FpArgs job_fp(const tr_sched *S, const Job &j, const float *vol, float *out) {
  FpArgs a{};
  a.v = job_view(j, const_cast<float *>(vol));
  a.val = out;
  a.tstride = (long long)j.d.nx * j.d.ny;
  a.pnx = j.d.nx;
  a.pny = j.d.ny;
  a.geo = j.geo;
  a.t0 = 0;
  a.nt = j.d.ntilt;
  a.ox = j.d.ox;
  a.oy = j.d.oy;
  a.oz = j.d.oz;
  a.fw = j.gi.ffw;
  a.fh = j.gi.ffh;
  a.chunk = chunk_for(S->smem_fp, j.gi.fp_tilt_bytes);
  a.nbound = j.gi.nbound;
  return a;
}

size_t job_tiles(const Job &j) {
  const dim3 g = bp_tile_grid(job_view(j, nullptr));
  return (size_t)g.x * g.y * g.z;
}

// Device bytes a job holds while admitted.
size_t job_bytes(const tr_sched *S, const Job &j) {
  const size_t p = j.plane, v = j.nvox;
  size_t b = sizeof(TiltGeo) * j.d.ntilt + p * 4;  // geo, val
  if (j.d.sirt_iters > 0) {  // wt; compact voxel weights at their largest
    const size_t tiles = job_tiles(j);
    b += p * 4 + tiles * (kTileVox * 4 + 4) + 4 + (size_t)j.d.ny * 4;
  }
  if (S->pdtype != TR_DTYPE_F32 || j.d.host) b += p * elem_size(S->pdtype);  // stored stack
  b += sizeof(float) * j.d.ntilt * 3;                        // scales, maxima (16-bit)
  if (S->rdtype != TR_DTYPE_F32) b += p * 2;                               // 16-bit residual
  if (j.d.host) b += v * 4;                                                // volume
  return b;
}

template <typename T>
cudaError_t alloc(T **p, size_t bytes, cudaStream_t s) {
  return cudaMallocAsync((void **)p, std::max<size_t>(bytes, 16), s);
}

// R-weighting spectrum for rows of nx samples (built once per row length).
tr_status ensure_filter(tr_sched *S, int nx, std::pair<float2 *, float2 *> *out) {
  auto it = S->filt.find(nx);
  if (it != S->filt.end()) {
    *out = it->second;
    return TR_OK;
  }
  RweightSpectrum sp;
  if (!rweight_spectrum(nx, kSchedSmemMax, &sp))
    return sched_fail(S, TR_ERR_UNSUPPORTED, "row length too long for the filter");
  const int M = 1 << sp.log2m;
  float2 *g = nullptr, *t = nullptr;
  SCHED_CUDA(S, cudaMalloc(&g, sizeof(float2) * M));
  SCHED_CUDA(S, cudaMalloc(&t, sizeof(float2) * sp.tw.size()));
  SCHED_CUDA(S, cudaMemcpy(g, sp.ghat.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
  SCHED_CUDA(S, cudaMemcpy(t, sp.tw.data(), sizeof(float2) * sp.tw.size(),
                           cudaMemcpyHostToDevice));
  S->filt[nx] = {g, t};
  S->filt_h[nx] = sp;
  *out = {g, t};
  return TR_OK;
}

void fill_grid(BatchBp *b, dim3 g, int mode, bool sep) {
  b->mode = mode;
  b->sep = sep;
  b->gx = g.x;
  b->gy = g.y;
  b->gz = g.z;
}

// Admission: allocations and the preparation launches on the prep stream.
tr_status admit(tr_sched *S, Job &j) {
  cudaStream_t ps = S->prep;
  const int nt = j.d.ntilt;
  const size_t P = j.plane, V = j.nvox;
  j.pdtype = S->pdtype;
  j.rdtype = S->rdtype;
  std::pair<float2 *, float2 *> filt{nullptr, nullptr};
  if (j.d.wbp) {
    tr_status st = ensure_filter(S, j.d.nx, &filt);
    if (st) return st;
  }
  const bool sirt = j.d.sirt_iters > 0;
  const size_t tiles = job_tiles(j);
  SCHED_CUDA(S, alloc(&j.geo, sizeof(TiltGeo) * nt, ps));
  SCHED_CUDA(S, alloc(&j.val, P * 4, ps));
  if (sirt) {
    SCHED_CUDA(S, alloc(&j.wt, P * 4, ps));
    SCHED_CUDA(S, alloc(&j.wslot, (tiles + 1) * sizeof(int), ps));
    SCHED_CUDA(S, alloc(&j.wtvol, tiles * kTileVox * 4, ps));  // every tile a border tile
    SCHED_CUDA(S, alloc(&j.wrow, (size_t)j.d.ny * 4, ps));
  }
  if (j.pdtype != TR_DTYPE_F32 || j.d.host)
    SCHED_CUDA(S, alloc(&j.pstore, P * elem_size(j.pdtype), ps));
  if (j.pdtype != TR_DTYPE_F32) SCHED_CUDA(S, alloc(&j.pscale, sizeof(float) * nt, ps));
  if (j.pdtype != TR_DTYPE_F32 || j.rdtype == TR_DTYPE_F16)
    SCHED_CUDA(S, alloc(&j.maxbits, sizeof(unsigned) * nt, ps));
  if (j.rdtype == TR_DTYPE_F16) SCHED_CUDA(S, alloc(&j.rscale, sizeof(float) * nt, ps));
  if (j.rdtype != TR_DTYPE_F32) SCHED_CUDA(S, alloc(&j.res, P * 2, ps));
  if (j.d.host) SCHED_CUDA(S, alloc(&j.vol_own, V * 4, ps));
  j.vol = j.d.host ? j.vol_own : j.d.vol;

  std::vector<TiltGeo> g(nt);
  int bad = -1;
  derive_geometry(j.coeff.data(), nt, j.d.nx, j.d.ny, j.d.thickness, kSchedSmemMax, g.data(),
                  &j.gi, &bad);
  SCHED_CUDA(S, cudaMemcpyAsync(j.geo, g.data(), sizeof(TiltGeo) * nt, cudaMemcpyHostToDevice,
                                ps));
  // FP32 projections into val (upload or device copy), then the stored stack.
  const cudaMemcpyKind k_in = j.d.host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  SCHED_CUDA(S, cudaMemcpyAsync(j.val, j.d.proj, P * 4, k_in, ps));
  const size_t plane2 = (size_t)j.d.nx * j.d.ny;
  if (j.pdtype != TR_DTYPE_F32) {
    SCHED_CUDA(S, launch_quantize(j.val, plane2, nt, j.pdtype, j.pstore, j.pscale, j.maxbits,
                                  S->nsm, ps));
    j.proj = j.pstore;
    j.ps = j.pscale;
  } else if (j.d.host) {
    SCHED_CUDA(S, cudaMemcpyAsync(j.pstore, j.val, P * 4, cudaMemcpyDeviceToDevice, ps));
    j.proj = j.pstore;
  } else {
    j.proj = j.d.proj;
  }
  // FP16 residuals carry their own per-tilt scales, recomputed every step.
  j.rs = j.rdtype == TR_DTYPE_F16 ? j.rscale : nullptr;
  if (j.d.wbp) {
    const RweightSpectrum &sp = S->filt_h[j.d.nx];
    FilterArgs f;
    f.rows = j.val;
    f.nrows = (long long)j.d.ny * nt;
    f.nx = j.d.nx;
    f.n_pad = sp.npad;
    f.log2m = sp.log2m;
    f.ghat = filt.first;
    f.tw = filt.second;
    SCHED_CUDA(S, launch_rweight(f, ps));
  }
  if (!j.d.vol_in)
    SCHED_CUDA(S, cudaMemsetAsync(j.vol, 0, V * 4, ps));
  else if (j.d.host)
    SCHED_CUDA(S, cudaMemcpyAsync(j.vol_own, j.d.vol, V * 4, cudaMemcpyHostToDevice, ps));
  // Geometry-only weights of SIRT jobs: the splat of ones, and the voxel
  // sums of c in compact form (tiles classified on the device; the border
  // tiles' slots come from a device counter, so the worst-case buffer needs
  // no read-back of the count).
  if (sirt) {
    SCHED_CUDA(S, cudaMemsetAsync(j.wt, 0, P * 4, ps));
    SCHED_CUDA(S, launch_fp(j.gi.sep, job_fp(S, j, nullptr, j.wt), ps));
    SCHED_CUDA(S, cudaMemsetAsync(j.wslot + tiles, 0, sizeof(int), ps));
    SCHED_CUDA(S, launch_classify_tiles(j.geo, nt, job_view(j, nullptr), j.d.ox, j.d.oy, j.d.oz,
                                        j.d.nx, j.d.ny, j.gi.sep, j.wslot, j.wslot + tiles, ps));
    if (j.gi.sep)
      SCHED_CUDA(S, launch_sep_row_weights(j.geo, nt, j.d.ny, j.d.oy, j.d.ny, j.wrow, ps));
    BpArgs w = job_bp(S, j, nullptr, TR_DTYPE_F32, nullptr, 1.f);
    w.v.vol = nullptr;
    w.out = j.wtvol;
    w.wslot = j.wslot;
    w.err = nullptr;
    SCHED_CUDA(S, launch_bp(BP_WEIGHTS, j.gi.sep, w, ps));
  }

  // Step items (layouts fixed for the job's life).
  const dim3 gb = bp_tile_grid(job_view(j, j.vol)), gf = fp_tile_grid(job_view(j, j.vol));
  if (j.d.wbp) {
    BpArgs a = job_bp(S, j, j.val, TR_DTYPE_F32, nullptr, 1.f);
    j.a_norm = a;
    if (!batch_bp_layout(a, j.gi.sep, S->smem_bp, &j.bp_norm, &j.smem_norm) ||
        j.smem_norm > S->smem_bp)
      return sched_fail(S, TR_ERR_UNSUPPORTED, "tile window does not suit the step's layout");
    fill_grid(&j.bp_norm, gb, BP_NORM, j.gi.sep);
  }
  if (j.d.sirt_iters > 0) {
    j.fp.a = job_fp(S, j, j.vol, j.val);
    j.fp.sep = j.gi.sep;
    j.fp.gx = gf.x;
    j.fp.gy = gf.y;
    j.fp.gz = gf.z;
    const void *r = j.rdtype == TR_DTYPE_F32 ? (const void *)j.val : j.res;
    BpArgs a = job_bp(S, j, r, j.rdtype, j.rs, j.d.gamma);
    a.wtvol = j.wtvol;
    a.wslot = j.wslot;
    a.wrow = j.wrow;
    a.wfull = (float)nt;
    j.a_sirt = a;
    if (!batch_bp_layout(a, j.gi.sep, S->smem_bp, &j.bp_sirt, &j.smem_sirt) ||
        j.smem_sirt > S->smem_bp ||
        (size_t)j.fp.a.chunk * j.gi.fp_tilt_bytes > S->smem_fp)
      return sched_fail(S, TR_ERR_UNSUPPORTED, "tile window does not suit the step's layout");
    fill_grid(&j.bp_sirt, gb, BP_SIRT, j.gi.sep);
  }
  SCHED_CUDA(S, cudaEventCreateWithFlags(&j.ev_ready, cudaEventDisableTiming));
  SCHED_CUDA(S, cudaEventCreateWithFlags(&j.ev_done, cudaEventDisableTiming));
  SCHED_CUDA(S, cudaEventCreateWithFlags(&j.ev_copied, cudaEventDisableTiming));
  SCHED_CUDA(S, cudaEventRecord(j.ev_ready, ps));
  j.wbp_pending = j.d.wbp != 0;
  j.iters_left = j.d.sirt_iters;
  j.state = J_LOADING;
  return TR_OK;
}

void release(tr_sched *S, Job &j, cudaStream_t s) {
  void *ptrs[] = {j.geo,    j.val, j.wt,     j.wtvol,  j.vol_own, j.wrow,
                  j.wslot,  j.pstore, j.res, j.pscale, j.rscale, j.maxbits};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, s);
  j.geo = nullptr;
  j.wslot = nullptr;
  j.val = j.wt = j.wtvol = j.vol_own = j.pscale = j.rscale = j.wrow = nullptr;
  j.pstore = j.res = nullptr;
  j.maxbits = nullptr;
  S->used -= std::min(S->used, j.bytes);
}

// Captures the four launches of a step over table b.
tr_status capture(tr_sched *S, int b) {
  cudaGraph_t g = nullptr;
  SCHED_CUDA(S, cudaStreamBeginCapture(S->s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launch_batch_step(S->tab_d[b], S->rdtype, S->grid_fp, S->grid_bp,
                                    S->smem_fp, S->smem_bp, S->nsm, S->s);
  cudaError_t e2 = cudaStreamEndCapture(S->s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return sched_fail(S, TR_ERR_CUDA, std::string("step capture: ") +
                                          cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  if (S->graph[b]) cudaGraphExecDestroy(S->graph[b]);
  S->graph[b] = nullptr;
  e = cudaGraphInstantiate(&S->graph[b], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return sched_fail(S, TR_ERR_CUDA, "graph instantiate failed");
  return TR_OK;
}

tr_status configure(tr_sched *S, size_t smem_bp, int bp_per_sm) {
  int fp_per_sm = 0;
  const int occ = batch_occupancy(S->rdtype, smem_bp, S->smem_fp, &fp_per_sm);
  if (occ < 1 || fp_per_sm < 1) return sched_fail(S, TR_ERR_UNSUPPORTED, "no resident CTA");
  S->smem_bp = smem_bp;
  S->grid_bp = S->nsm * std::max(1, std::min(occ, bp_per_sm > 0 ? bp_per_sm : occ));
  S->grid_fp = S->nsm * fp_per_sm;
  for (int b = 0; b < 2; ++b) {
    tr_status st = capture(S, b);
    if (st) return st;
  }
  return TR_OK;
}

double job_work(const Job &j) {
  return ((j.wbp_pending ? 1.0 : 0.0) + 2.0 * j.iters_left) * j.d.ntilt * (double)j.nvox;
}

// SRPT order key: the work left, divided by 1 + (time since submission) /
// aging time, so that a long job's priority grows while it waits.
double srpt_key(const tr_sched *S, const Job &j, double now) {
  const double w = job_work(j);
  return S->aging_s > 0 ? w / (1.0 + (now - j.t_submit) / S->aging_s) : w;
}

// TR_SCHED_SRPT step: the next unit of the ready job with the least remaining
// work (its WBP back-projection, or one SIRT iteration) through the per-job
// kernels the context path runs.  At most two steps are in flight, so a job
// that becomes ready is considered within one step.
tr_status launch_job_step(tr_sched *S, bool *launched) {
  Job *j = nullptr;
  const double now = now_s();
  for (auto &jp : S->active)
    if (jp->state == J_READY && (jp->wbp_pending || jp->iters_left > 0) &&
        (!j || srpt_key(S, *jp, now) < srpt_key(S, *j, now)))
      j = jp.get();
  if (!j) return TR_OK;
  const int b = S->next_tab;
  if (S->tab_used[b]) {
    if (cudaEventQuery(S->tab_ev[b]) == cudaErrorNotReady) return TR_OK;  // try later
    S->tab_used[b] = false;
  }
  cudaStream_t s = S->s;
  if (j->wbp_pending) {
    SCHED_CUDA(S, cudaMemsetAsync(S->err_d, 0, sizeof(int), s));
    SCHED_CUDA(S, launch_bp(BP_NORM, j->gi.sep, j->a_norm, s));
    j->wbp_pending = false;
    ++S->items_bp;
  } else {
    const size_t plane = (size_t)j->d.nx * j->d.ny;
    const int nt = j->d.ntilt;
    SCHED_CUDA(S, cudaMemsetAsync(j->val, 0, j->plane * 4, s));
    SCHED_CUDA(S, launch_fp(j->gi.sep, j->fp.a, s));
    if (j->rdtype == TR_DTYPE_F16) {  // FP32 over val, then FP16 with own scales
      SCHED_CUDA(S, launch_resid_lp(j->proj, j->pdtype, j->ps, j->val, j->wt, plane, nt,
                                    TR_DTYPE_F32, j->val, nullptr, S->nsm, s));
      SCHED_CUDA(S, launch_quantize(j->val, plane, nt, TR_DTYPE_F16, j->res, j->rscale,
                                    j->maxbits, S->nsm, s));
    } else {
      void *r = j->rdtype == TR_DTYPE_F32 ? (void *)j->val : j->res;
      SCHED_CUDA(S, launch_resid_lp(j->proj, j->pdtype, j->ps, j->val, j->wt, plane, nt,
                                    j->rdtype, r, nullptr, S->nsm, s));
    }
    SCHED_CUDA(S, cudaMemsetAsync(S->err_d, 0, sizeof(int), s));
    SCHED_CUDA(S, launch_bp(BP_SIRT, j->gi.sep, j->a_sirt, s));
    --j->iters_left;
    ++S->items_bp;
    ++S->items_fp;
  }
  SCHED_CUDA(S, cudaEventRecord(S->tab_ev[b], s));
  S->tab_used[b] = true;
  S->next_tab = b ^ 1;
  ++S->steps;
  if (!j->wbp_pending && j->iters_left == 0) {
    SCHED_CUDA(S, cudaEventRecord(j->ev_done, s));
    j->state = J_DRAINING;
  }
  *launched = true;
  return TR_OK;
}

// Builds and launches one step over the ready jobs (nothing when none has
// work or the next table buffer is still being uploaded).
tr_status launch_step(tr_sched *S, bool *launched) {
  *launched = false;
  if (S->policy == TR_SCHED_SRPT) return launch_job_step(S, launched);
  std::vector<Job *> part;
  for (auto &jp : S->active)
    if (jp->state == J_READY && (jp->wbp_pending || jp->iters_left > 0)) part.push_back(jp.get());
  if (part.empty()) return TR_OK;
  const int b = S->next_tab;
  if (S->tab_used[b]) {
    if (cudaEventQuery(S->tab_ev[b]) == cudaErrorNotReady) return TR_OK;  // try later
    S->tab_used[b] = false;
  }
  BatchTable *T = S->tab_h[b];
  BatchHeader &h = T->h;
  memset(&h, 0, sizeof(h));
  h.err = S->err_d;
  long long bp_tiles = 0, fp_tiles = 0;
  std::vector<Job *> finishing;
  for (Job *j : part) {
    if (h.nbp >= kBatchMaxItems || h.nfp >= kBatchMaxItems || h.nzero + 2 > kBatchMaxItems)
      break;
    const bool wbp = j->wbp_pending;
    BatchBp &bi = T->bp[h.nbp++];
    bi = wbp ? j->bp_norm : j->bp_sirt;
    bi.first = bp_tiles;
    bp_tiles += (long long)bi.gx * bi.gy * bi.gz;
    if (wbp) {
      j->wbp_pending = false;
    } else {
      BatchFp &fi = T->fp[h.nfp++];
      fi = j->fp;
      fi.first = fp_tiles;
      fp_tiles += (long long)fi.gx * fi.gy * fi.gz;
      BatchZero &z = T->zero[h.nzero++];
      z.p = j->val;
      z.n = j->plane;
      BatchRes &r = T->res[h.nres++];
      r.p = j->proj;
      r.ps = j->ps;
      r.pdtype = j->pdtype;
      r.val = j->val;
      r.wt = j->wt;
      r.plane = (unsigned long long)j->d.nx * j->d.ny;
      r.nt = j->d.ntilt;
      if (j->rdtype == TR_DTYPE_F16) {  // FP32 over val, then FP16 with own scales
        r.r = j->val;
        r.rs = nullptr;
        r.rdtype = TR_DTYPE_F32;
        r.q = (__half *)j->res;
        r.qscale = j->rscale;
        r.qmax = j->maxbits;
        BatchZero &zm = T->zero[h.nzero++];
        zm.p = (float *)j->maxbits;
        zm.n = (unsigned long long)j->d.ntilt;
      } else {
        r.r = j->rdtype == TR_DTYPE_F32 ? (void *)j->val : j->res;
        r.rs = nullptr;
        r.rdtype = j->rdtype;
        r.q = nullptr;
        r.qscale = nullptr;
        r.qmax = nullptr;
      }
      --j->iters_left;
    }
    if (!j->wbp_pending && j->iters_left == 0) finishing.push_back(j);
  }
  h.bp_tiles = bp_tiles;
  h.fp_tiles = fp_tiles;
  // Upload the used parts of the table, then replay the step graph.
  BatchTable *D = S->tab_d[b];
  cudaStream_t s = S->s;
  SCHED_CUDA(S, cudaMemcpyAsync(&D->h, &T->h, sizeof(BatchHeader), cudaMemcpyHostToDevice, s));
  if (h.nbp)
    SCHED_CUDA(S, cudaMemcpyAsync(D->bp, T->bp, sizeof(BatchBp) * h.nbp,
                                  cudaMemcpyHostToDevice, s));
  if (h.nfp)
    SCHED_CUDA(S, cudaMemcpyAsync(D->fp, T->fp, sizeof(BatchFp) * h.nfp,
                                  cudaMemcpyHostToDevice, s));
  if (h.nres)
    SCHED_CUDA(S, cudaMemcpyAsync(D->res, T->res, sizeof(BatchRes) * h.nres,
                                  cudaMemcpyHostToDevice, s));
  if (h.nzero)
    SCHED_CUDA(S, cudaMemcpyAsync(D->zero, T->zero, sizeof(BatchZero) * h.nzero,
                                  cudaMemcpyHostToDevice, s));
  SCHED_CUDA(S, cudaEventRecord(S->tab_ev[b], s));
  S->tab_used[b] = true;
  SCHED_CUDA(S, cudaGraphLaunch(S->graph[b], s));
  S->next_tab = b ^ 1;
  ++S->steps;
  S->items_bp += h.nbp;
  S->items_fp += h.nfp;
  for (Job *j : finishing) {
    SCHED_CUDA(S, cudaEventRecord(j->ev_done, s));
    j->state = J_DRAINING;
  }
  *launched = true;
  return TR_OK;
}

// One pass of the scheduler (lock held): admit, advance, retire.
tr_status progress(tr_sched *S, bool *busy) {
  *busy = false;
  // Admit while a job fits: the queue's head in order (TR_SCHED_BATCHED), or
  // the queued job with the least work that fits (TR_SCHED_SRPT).  With
  // nothing admitted, the chosen job is admitted whatever its size.
  const double now = now_s();
  while (!S->queue.empty()) {
    auto pick = S->queue.begin();
    if (S->policy == TR_SCHED_SRPT)
      for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
        if (srpt_key(S, **it, now) < srpt_key(S, **pick, now) &&
            (!S->budget || S->used + (*it)->bytes <= S->budget))
          pick = it;
    Job &j = **pick;
    if (S->budget && S->used + j.bytes > S->budget && !S->active.empty()) break;
    S->used += j.bytes;
    S->peak = std::max(S->peak, S->used);
    S->active.push_back(*pick);
    S->queue.erase(pick);
    tr_status st = admit(S, j);
    if (st) return st;
    *busy = true;
  }
  for (auto &jp : S->active) {
    Job &j = *jp;
    if (j.state == J_LOADING && cudaEventQuery(j.ev_ready) == cudaSuccess) {
      j.state = J_READY;
      j.t_ready = now_s();
      if (!j.wbp_pending && j.iters_left == 0) {  // nothing to iterate: done once loaded
        SCHED_CUDA(S, cudaEventRecord(j.ev_done, S->prep));
        j.state = J_DRAINING;
      }
      *busy = true;
    }
  }
  bool launched = false;
  tr_status st = launch_step(S, &launched);
  if (st) return st;
  *busy |= launched;
  for (size_t i = 0; i < S->active.size();) {
    Job &j = *S->active[i];
    if (j.state == J_DRAINING && cudaEventQuery(j.ev_done) == cudaSuccess) {
      if (j.d.host)
        SCHED_CUDA(S, cudaMemcpyAsync(j.d.vol, j.vol_own, j.nvox * 4, cudaMemcpyDeviceToHost,
                                      S->back));
      SCHED_CUDA(S, cudaEventRecord(j.ev_copied, S->back));
      j.state = J_COPYBACK;
      *busy = true;
    }
    if (j.state == J_COPYBACK && cudaEventQuery(j.ev_copied) == cudaSuccess) {
      release(S, j, S->back);
      j.t_done = now_s();
      j.state = J_DONE;
      cudaEventDestroy(j.ev_ready);
      cudaEventDestroy(j.ev_done);
      cudaEventDestroy(j.ev_copied);
      j.ev_ready = j.ev_done = j.ev_copied = nullptr;
      S->active.erase(S->active.begin() + i);
      S->done_cv.notify_all();
      *busy = true;
      continue;
    }
    ++i;
  }
  return TR_OK;
}

void worker(tr_sched *S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (!S->stop) {
    bool busy = false;
    if (!S->fatal) {
      const tr_status st = progress(S, &busy);
      if (st) {
        // Fail every job still in flight; the scheduler stays unusable.
        for (auto &jp : S->active) {
          jp->status = st;
          jp->state = J_DONE;
        }
        for (auto &jp : S->queue) {
          jp->status = st;
          jp->state = J_DONE;
        }
        S->active.clear();
        S->queue.clear();
        S->done_cv.notify_all();
      }
    }
    if (!busy) S->cv.wait_for(lk, std::chrono::microseconds(100));
  }
}

// TR_ERR_TIMEOUT when a back-projection's bounded wait ran out (sticky word).
tr_status take_timeout(tr_sched *S) {
  int e[2] = {0, 0};
  if (cudaMemcpy(e, S->err_d, sizeof(e), cudaMemcpyDeviceToHost) != cudaSuccess)
    return TR_ERR_CUDA;
  if (e[1]) {
    cudaMemset(S->err_d + 1, 0, sizeof(int));
    return TR_ERR_TIMEOUT;
  }
  return TR_OK;
}

}  // namespace

extern "C" {

tr_status tr_sched_create(int device, size_t hbm_budget, int proj_dtype, int resid_dtype,
                          tr_sched **out) {
  if (!out) return TR_ERR_ARG;
  *out = nullptr;
  auto ok = [](int d) { return d == TR_DTYPE_F32 || d == TR_DTYPE_F16 || d == TR_DTYPE_BF16; };
  if (!ok(proj_dtype) || !ok(resid_dtype)) return TR_ERR_ARG;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return TR_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess) return TR_ERR_CUDA;
  std::unique_ptr<tr_sched> S(new tr_sched);
  S->device = device;
  S->budget = hbm_budget;
  S->pdtype = proj_dtype;
  S->rdtype = resid_dtype;
  cudaDeviceGetAttribute(&S->nsm, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&S->prep, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&S->back, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&S->err_d, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemset(S->err_d, 0, 2 * sizeof(int)) != cudaSuccess)
    return TR_ERR_CUDA;
  for (int b = 0; b < 2; ++b) {
    if (cudaMalloc(&S->tab_d[b], sizeof(BatchTable)) != cudaSuccess ||
        cudaMallocHost(&S->tab_h[b], sizeof(BatchTable)) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->tab_ev[b], cudaEventDisableTiming) != cudaSuccess)
      return TR_ERR_CUDA;
    memset(S->tab_h[b], 0, sizeof(BatchTable));
    if (cudaMemset(S->tab_d[b], 0, sizeof(BatchTable)) != cudaSuccess) return TR_ERR_CUDA;
  }
  if (configure(S.get(), S->smem_bp, 0)) return S->fatal;
  if (cudaStreamSynchronize(S->s) != cudaSuccess) return TR_ERR_CUDA;
  tr_sched *p = S.release();
  p->worker = std::thread(worker, p);
  *out = p;
  return TR_OK;
}

tr_status tr_sched_submit(tr_sched *S, const tr_job *job, unsigned long long *id) {
  if (!S || !job || !job->proj || !job->coeff8 || !job->vol) return TR_ERR_ARG;
  const tr_job &d = *job;
  if (d.nx < 2 || d.ny < 1 || d.ntilt < 1 || d.thickness < 1 || d.sirt_iters < 0 ||
      d.ny > 65535 * kTY || (d.layout != TR_LAYOUT_Y && d.layout != TR_LAYOUT_Z))
    return TR_ERR_ARG;
  auto j = std::make_shared<Job>();
  j->d = d;
  j->coeff.assign(d.coeff8, d.coeff8 + 8 * (size_t)d.ntilt);
  j->d.coeff8 = nullptr;
  j->plane = (size_t)d.nx * d.ny * d.ntilt;
  j->nvox = (size_t)d.nx * d.ny * d.thickness;
  j->wbp_pending = d.wbp != 0;  // the work left, for the SRPT order while queued
  j->iters_left = d.sirt_iters;
  std::vector<TiltGeo> g(d.ntilt);
  int bad = -1;
  const int gs = derive_geometry(j->coeff.data(), d.ntilt, d.nx, d.ny, d.thickness,
                                 kSchedSmemMax, g.data(), &j->gi, &bad);
  if (gs == GEOM_NONFINITE) return TR_ERR_ARG;
  if (gs != GEOM_OK) return TR_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return S->fatal;
  j->bytes = job_bytes(S, *j);
  if (S->budget && j->bytes > S->budget) return TR_ERR_BUDGET;
  j->id = S->next_id++;
  j->t_submit = now_s();
  S->queue.push_back(j);
  S->all[j->id] = j;
  if (id) *id = j->id;
  S->cv.notify_all();
  return TR_OK;
}

tr_status tr_sched_wait(tr_sched *S, unsigned long long id, double *latency_s) {
  if (!S) return TR_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->all.find(id);
  if (it == S->all.end()) return TR_ERR_ARG;
  std::shared_ptr<Job> j = it->second;
  S->done_cv.wait(lk, [&] { return j->state == J_DONE; });
  if (latency_s) *latency_s = j->t_done - j->t_submit;
  const tr_status st = j->status;
  S->all.erase(id);
  if (st) return st;
  return take_timeout(S);
}

tr_status tr_sched_drain(tr_sched *S) {
  if (!S) return TR_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  S->done_cv.wait(lk, [&] { return S->queue.empty() && S->active.empty(); });
  for (auto it = S->all.begin(); it != S->all.end();)
    it = it->second->state == J_DONE ? S->all.erase(it) : std::next(it);
  if (S->fatal) return S->fatal;
  return take_timeout(S);
}

tr_status tr_sched_stats(tr_sched *S, tr_sched_info *out) {
  if (!S || !out) return TR_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  out->steps = S->steps;
  out->bp_items = S->items_bp;
  out->fp_items = S->items_fp;
  out->peak_bytes = S->peak;
  out->grid_bp = S->grid_bp;
  out->grid_fp = S->grid_fp;
  out->smem_bp = S->smem_bp;
  out->queued = (int)S->queue.size();
  out->active = (int)S->active.size();
  return S->fatal;
}

const char *tr_sched_last_error(const tr_sched *S) { return S ? S->err.c_str() : "null"; }

tr_status tr_sched_set_policy(tr_sched *S, int policy) {
  if (!S || (policy != TR_SCHED_BATCHED && policy != TR_SCHED_SRPT)) return TR_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->policy = policy;
  return TR_OK;
}

tr_status tr_sched_set_aging(tr_sched *S, double aging_s) {
  if (!S || !(aging_s >= 0)) return TR_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  S->aging_s = aging_s;
  return TR_OK;
}

tr_status tr_sched_configure(tr_sched *S, size_t smem_bp, int bp_ctas_per_sm) {
  if (!S || smem_bp < 16 * 1024 || smem_bp > kSchedSmemMax || bp_ctas_per_sm < 0)
    return TR_ERR_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  // Reconfigure only while idle: admitted jobs hold layouts for the old budget.
  S->done_cv.wait(lk, [&] { return S->queue.empty() && S->active.empty(); });
  if (S->fatal) return S->fatal;
  cudaSetDevice(S->device);
  if (cudaStreamSynchronize(S->s) != cudaSuccess) return TR_ERR_CUDA;
  return configure(S, smem_bp, bp_ctas_per_sm);
}

tr_status tr_sched_autotune(tr_sched *S, const tr_job *probe, int iters, size_t *best_smem,
                            int *best_ctas) {
  if (!S || !probe || probe->host || !probe->vol || iters < 1) return TR_ERR_ARG;
  cudaSetDevice(S->device);
  // The probe runs on a scratch copy of its starting volume.
  const size_t V = (size_t)probe->nx * probe->ny * probe->thickness;
  float *tmp = nullptr;
  if (cudaMalloc(&tmp, V * 4) != cudaSuccess) {
    cudaGetLastError();
    return TR_ERR_OOM;
  }
  const size_t cand_smem[] = {40 * 1024, 56 * 1024, 80 * 1024, 112 * 1024};
  double best = 1e30;
  size_t bs = S->smem_bp;
  int bc = 0;
  tr_status st = TR_OK;
  for (int pass = 0; pass < 2 && !st; ++pass) {
    const size_t best_so_far = bs;
    for (size_t sm : cand_smem) {
      // pass 0: each budget at full residency; pass 1: one CTA fewer at the best
      if (pass == 1 && sm != best_so_far) continue;
      int fp_occ = 0;
      const int occ = batch_occupancy(S->rdtype, sm, S->smem_fp, &fp_occ);
      const int ctas = pass == 0 ? occ : occ - 1;
      if (ctas < 1) continue;
      if ((st = tr_sched_configure(S, sm, ctas))) break;
      double t = 0;
      for (int rep = 0; rep < 2 && !st; ++rep) {  // the first run warms the allocator
        if (cudaMemcpy(tmp, probe->vol, V * 4, cudaMemcpyDeviceToDevice) != cudaSuccess) {
          st = TR_ERR_CUDA;
          break;
        }
        tr_job j = *probe;
        j.vol = tmp;
        j.wbp = 0;
        j.sirt_iters = iters;
        const double t0 = now_s();
        unsigned long long id = 0;
        if ((st = tr_sched_submit(S, &j, &id))) break;
        if ((st = tr_sched_wait(S, id, nullptr))) break;
        t = now_s() - t0;
      }
      if (!st && t < best) {
        best = t;
        bs = sm;
        bc = ctas;
      }
    }
  }
  cudaFree(tmp);
  if (st) return st;
  if ((st = tr_sched_configure(S, bs, bc))) return st;
  if (best_smem) *best_smem = bs;
  if (best_ctas) *best_ctas = bc;
  return TR_OK;
}

tr_status tr_sched_destroy(tr_sched *S) {
  if (!S) return TR_ERR_ARG;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->done_cv.wait(lk, [&] { return S->queue.empty() && S->active.empty(); });
    S->stop = true;
    S->cv.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->device);
  cudaDeviceSynchronize();
  for (int b = 0; b < 2; ++b) {
    if (S->graph[b]) cudaGraphExecDestroy(S->graph[b]);
    if (S->tab_d[b]) cudaFree(S->tab_d[b]);
    if (S->tab_h[b]) cudaFreeHost(S->tab_h[b]);
    if (S->tab_ev[b]) cudaEventDestroy(S->tab_ev[b]);
  }
  for (auto &kv : S->filt) {
    cudaFree(kv.second.first);
    cudaFree(kv.second.second);
  }
  if (S->err_d) cudaFree(S->err_d);
  cudaStreamDestroy(S->s);
  cudaStreamDestroy(S->prep);
  cudaStreamDestroy(S->back);
  delete S;
  return TR_OK;
}

}  // extern "C"
