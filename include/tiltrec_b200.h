/* tiltrec_b200 -- C ABI of the B200 (sm_100a) TiltRec reconstruction engine.
 *
 * Drop-in boundary for the reference's reconstruction drivers.  The reference
 * binds its hot path as C++ calls that own device memory and write MRC files
 * (src/TiltRec/src/TiltRec_cuda_y/recon_y.cuh:25-40,
 *  src/TiltRec/src/TiltRec_cuda_z/recon_z.cuh:17-39) and as CPU routines in
 * src/TiltRec/src/main/main-mpi.cpp / main-mpiz.cpp.  This ABI exposes the
 * same operations on caller-owned buffers: plain pointers and sizes, no C++ or
 * CUDA types (streams are passed as void*, i.e. a cudaStream_t or NULL for
 * the legacy default stream).
 *
 * Data layout (all float32, C order):
 *   projections  [ntilt][ny][nx]            (MRC stack X, Y, Z = tilts)
 *   volume, Y    [ny][thickness][nx]        (TiltRec:  MRC (X, th, Y))
 *   volume, Z    [thickness][ny][nx]        (TiltRecZ: MRC (X, Y, th))
 *   coefficients [ntilt][8] double          a0 a1 a2 a3 b0 b1 b2 b3: a voxel
 *       at (x, y, z) projects to detector column
 *       u = a0 + a1 (x-ox) + a2 (y-oy) + a3 (z-oz) + ox and row
 *       v = b0 + b1 (x-ox) + b2 (y-oy) + b3 (z-oz) + oy
 *       (the linear part of the reference's struct Coeff, main-mpi.cpp:19-30,
 *       as evaluated by ValCoef, main-mpi.cpp:204-226).
 *
 * Conventions: every call returns a tr_status (0 = OK, negative = error; the
 * message is in tr_last_error).  No call exits the process.  Device calls are
 * asynchronous and ordered on the given stream.  A context is not safe for
 * concurrent use by several host threads; use one context per thread/stream.
 * The library owns only scratch memory, allocated within the context's HBM
 * budget (0 = unlimited). */
#ifndef TILTREC_B200_H
#define TILTREC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is an exported symbol of libtiltrec_b200.so (the
 * library is built with hidden visibility by default). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct tr_ctx tr_ctx;

typedef enum {
  TR_OK = 0,
  TR_ERR_ARG = -1,         /* invalid argument / state for this call */
  TR_ERR_OOM = -2,         /* device allocation failed */
  TR_ERR_BUDGET = -3,      /* scratch would exceed the HBM budget */
  TR_ERR_CUDA = -4,        /* CUDA runtime error (see tr_last_error) */
  TR_ERR_TIMEOUT = -5,     /* a bounded device wait ran out */
  TR_ERR_NOPROBLEM = -6,   /* tr_set_problem has not been called */
  TR_ERR_UNSUPPORTED = -7  /* geometry outside what the kernels stage */
} tr_status;

typedef enum { TR_LAYOUT_Y = 0, TR_LAYOUT_Z = 1 } tr_layout;

typedef enum {
  TR_METHOD_BPT = 0,   /* back-projection                    (--method BPT) */
  TR_METHOD_WBP = 1,   /* R-weighting filter + BPT           (--method WBP) */
  TR_METHOD_SIRT = 2,  /* SIRT,n,gamma                       */
  TR_METHOD_SART = 3,  /* SART,n,gamma                       */
  TR_METHOD_FBP = 4    /* Shepp-Logan FBP filter + BPT       (--method FBP) */
} tr_method;

/* Flag OR-ed into tr_reconstruct_host's method: start from a zero volume
 * (the reference's default without --initial); vol_host is then output only
 * and is not copied to the device. */
#define TR_RECON_ZERO_START 0x100

/* Element types of 16-bit storage (projections, SIRT residuals). */
typedef enum {
  TR_DTYPE_F32 = 0,
  TR_DTYPE_F16 = 1,  /* IEEE binary16 */
  TR_DTYPE_BF16 = 2  /* bfloat16 */
} tr_dtype;

/* Library version: major*10000 + minor*100 + patch. */
int tr_version(void);
const char *tr_status_string(int status);

/* Per-tilt coefficients from tilt angles and the --geometry
 * offset,pitch(XTILT),zshift values, bit-identical to the reference CPU path:
 * TranslateAngleToCoefficients + DecorateCoefficients
 * (src/TiltRec/src/main/main-mpi.cpp:85-106, 110-183).  Host only.
 * coeff8_out: ntilt*8 doubles. */
tr_status tr_geometry_from_angles(const float *angles_deg, int ntilt,
                                  float offset, float pitch, float zshift,
                                  double *coeff8_out);

/* Context on CUDA device `device` with a scratch budget in bytes (0 = none).
 * Replaces InitializeCuda (src/TiltRec/src/main/main-cuda.cpp:83-109) minus
 * its cudaDeviceReset.  Scratch buffers (reprojections, weights, filter
 * spectra, host-call staging) are kept across tr_set_problem calls and
 * reused when large enough, so a context that reconstructs many series
 * allocates only when a larger one arrives; under a budget, or when the
 * device is short of memory, buffers the current problem has not used are
 * released first.  tr_scratch_bytes reports the budgeted buffers held;
 * tr_destroy frees everything. */
tr_status tr_create(int device, size_t hbm_budget, tr_ctx **out);
tr_status tr_destroy(tr_ctx *ctx);
const char *tr_last_error(const tr_ctx *ctx);
size_t tr_scratch_bytes(const tr_ctx *ctx);

/* Problem geometry: projection stack nx*ny*ntilt, volume thickness, layout,
 * coefficients (ntilt*8 doubles) and the float origin the reference uses
 * (TiltRec-mpi: (nx/2, th/2, th/2), main-mpi.cpp:743-745;
 *  TiltRecZ:     (nx/2, ny/2, th/2), main-mpiz.cpp:1078-1080). */
tr_status tr_set_problem(tr_ctx *ctx, int nx, int ny, int ntilt,
                         int thickness, int layout, const double *coeff8,
                         float ox, float oy, float oz);

/* Replace the coefficients of the current problem (same sizes, e.g. the next
 * tilt series of the same shape).  Ordered after work already queued on
 * `stream` (NULL: the context's own stream); invalidates the cached SIRT/SART
 * weights.  Same validation as tr_set_problem. */
tr_status tr_update_geometry(tr_ctx *ctx, const double *coeff8, void *stream);

/* R-weighting filter in place over every row of the stack [ntilt][ny][nx]:
 * ApplyFilterInplace(..., mode 2) (src/TiltRec/src/filter/filter_prj.h:24,
 * filter_prj.cpp:674-736, 787-795). */
tr_status tr_filter_rweight(tr_ctx *ctx, float *proj_dev, void *stream);

/* FBP row filter in place over every row of the stack: ApplyFilterInplace
 * modes 0 (Shepp-Logan) and 1 (Ram-Lak) (filter_prj.cpp:755-786), i.e.
 * FileterProjectionSymmetrize (:265-446) with the 251-tap kernels of
 * :137-178: each row, edge-padded and mirror-extended to the reference's DFT
 * length, circularly convolved with the kernel; computed as a direct sum in
 * double precision. */
tr_status tr_filter_fbp(tr_ctx *ctx, float *proj_dev, int mode, void *stream);

/* vol += sum over tilts of s/c (normalised bilinear gather) on sections
 * [z0, z0+nz) of the volume; vol_dev points at section z0 of the layout's
 * volume.  BackProject (main-mpi.cpp:411-450; main-mpiz.cpp:322-363, which
 * zeroes the volume first) and CuBackProject / CuBackProjectZ
 * (recon_y.cuh:25, recon_z.cuh:17). */
tr_status tr_backproject(tr_ctx *ctx, const float *proj_dev, float *vol_dev,
                         int z0, int nz, void *stream);

/* Forward projection of sections [z0, z0+nz): val += splat(vol) and, if
 * wt_dev != NULL, wt += splat(1), for every tilt ([ntilt][ny][nx]).
 * Reproject (main-mpi.cpp:286-344; main-mpiz.cpp:197-254). */
tr_status tr_forward_project(tr_ctx *ctx, const float *vol_dev, int z0, int nz,
                             float *val_dev, float *wt_dev, void *stream);

/* SIRT, `iters` iterations with relaxation gamma, in place on vol_dev (the
 * starting volume, --initial semantics).  SIRT (main-mpi.cpp:614-664;
 * main-mpiz.cpp:548-601), CuSIRT / CuSIRTZ (recon_y.cuh:31, recon_z.cuh:22). */
tr_status tr_sirt(tr_ctx *ctx, const float *proj_dev, float *vol_dev,
                  int iters, float gamma, void *stream);

/* SIRT (as tr_sirt) with an FP64 convergence gate.  Each iteration's
 * residual r = p - val/wt has its L2 norm summed in FP64 on the device
 * (fixed-order partial sums, so the norms repeat exactly) and read back; the
 * iterations stop before applying an update once the norm fell by less than
 * rel_tol of the previous one (rel_tol 0: run all max_iters).  norms_out
 * (host, max_iters doubles, may be NULL) receives every residual norm
 * computed, including the one that stopped the loop; *iters_done the updates
 * applied.  Blocking. */
tr_status tr_sirt_gated(tr_ctx *ctx, const float *proj_dev, float *vol_dev,
                        int max_iters, float gamma, double rel_tol,
                        double *norms_out, int *iters_done, void *stream);

/* SART, in place.  SART (main-mpi.cpp:578-612; main-mpiz.cpp:502-546),
 * CuSART / CuSARTZ (recon_y.cuh:35, recon_z.cuh:26). */
tr_status tr_sart(tr_ctx *ctx, const float *proj_dev, float *vol_dev,
                  int iters, float gamma, void *stream);

/* Building blocks of SIRT / SART for callers that own the iteration, e.g.
 * one rank per GPU holding a z-slab of the volume and summing the forward
 * projections of all slabs between the two passes, as TiltRecZ-mpi does
 * with MPI_Allreduce (main-mpiz.cpp:548-601).
 *
 * tr_forward_project_tilts: as tr_forward_project for tilts
 * [t0, t0+ntilts) only; val_dev / wt_dev point at tilt t0's plane. */
tr_status tr_forward_project_tilts(tr_ctx *ctx, const float *vol_dev, int z0,
                                   int nz, int t0, int ntilts, float *val_dev,
                                   float *wt_dev, void *stream);

/* Residual in place over ntilts planes: val <- proj - (wt != 0 ? val/wt : val)
 * (main-mpi.cpp:640-647). */
tr_status tr_residual(tr_ctx *ctx, const float *proj_dev, float *val_dev,
                      const float *wt_dev, int ntilts, void *stream);

/* SIRT update from the residuals of all tilts on sections [z0, z0+nz):
 * vol += gamma * (sum_t s) / (sum_t c) where sum_t c != 0, the voxel weight
 * sums cached per geometry.  UpdateWeightsByProjDiff + UpdateVolumeByWeights
 * (main-mpi.cpp:526-576; main-mpiz.cpp:453-501). */
tr_status tr_sirt_update(tr_ctx *ctx, const float *resid_dev, float *vol_dev,
                         int z0, int nz, float gamma, void *stream);

/* SART update of one tilt from its residual plane on sections [z0, z0+nz):
 * vol += gamma * s/c where c != 0.  UpdateVolumeByProjDiff
 * (main-mpi.cpp:492-524; main-mpiz.cpp:419-451). */
tr_status tr_sart_update(tr_ctx *ctx, const float *resid_plane_dev, int tilt,
                         float *vol_dev, int z0, int nz, float gamma,
                         void *stream);

/* ADMM with a soft-threshold (l1) prior, in place on vol_dev (the starting
 * volume): TiltRecZ's ADMM (main-mpiz.cpp:958-1013, --method
 * ADMM,outer,cg,mu,soft), with the same algorithm and its quirks kept: A^T b
 * accumulates the (u - d) mu terms of every outer iteration; each CG
 * iteration applies (A^T D A + mu I) twice (D = 1/projection weights where
 * they exceed 1e-5); dot products in FP64.  Any layout. */
tr_status tr_admm(tr_ctx *ctx, const float *proj_dev, float *vol_dev, int outer,
                  int cg_iters, float mu, float soft, void *stream);
/* tr_admm from host buffers (as tr_reconstruct_host). */
tr_status tr_admm_host(tr_ctx *ctx, const float *proj_host, float *vol_host,
                       int outer, int cg_iters, float mu, float soft);

/* WBP: filter proj_dev in place, then vol += back-projection.
 * main-mpi.cpp:841-846 (ApplyFilterInplace mode 2 + BackProject), CuFBP with
 * filterMode 2 (recon_y.cuh:28). */
tr_status tr_wbp(tr_ctx *ctx, float *proj_dev, float *vol_dev, void *stream);

/* Host-buffer reconstruction, the path a drop-in CLI takes: copies the
 * projections from host memory, reconstructs with `method` starting from
 * vol_host (BPT/WBP add to it) -- or from zeros when method carries
 * TR_RECON_ZERO_START, without reading vol_host -- and copies the volume
 * back; returns when vol_host holds the result.  Pinned host buffers give the
 * fastest copies.  Device buffers are kept in the context and reused across
 * calls of the same size.  (main-cuda.cpp's read / CuSIRT / write sequence;
 * the reference starts from zeros unless --initial is given.) */
tr_status tr_reconstruct_host(tr_ctx *ctx, int method, const float *proj_host,
                              float *vol_host, int iters, float gamma);

/* Mixed precision.  No counterpart in the reference (whose projections and
 * residuals are float throughout).  A 16-bit stack holds element e of tilt t
 * for the value e * scale[t]; the per-tilt scales are powers of two.
 *
 * tr_quantize: FP32 stack proj_dev -> out_dev (ntilt*ny*nx elements of
 * `dtype`, TR_DTYPE_F16 or TR_DTYPE_BF16) and scale_dev[ntilt].  FP16 scales
 * put each tilt's largest magnitude in (2^13, 2^14], a factor of four under
 * the format's largest finite value; BF16 keeps scale 1. */
tr_status tr_quantize(tr_ctx *ctx, const float *proj_dev, int dtype,
                      void *out_dev, float *scale_dev, void *stream);

/* Back-projection (as tr_backproject) from a 16-bit stack; the FP32 sums
 * over tilts are compensated (Kahan) per voxel. */
tr_status tr_backproject_lp(tr_ctx *ctx, const void *proj_dev, int dtype,
                            const float *scale_dev, float *vol_dev, int z0,
                            int nz, void *stream);

/* SIRT (as tr_sirt) from a 16-bit stack (proj_dtype, scales from
 * tr_quantize; scale_dev may be NULL for TR_DTYPE_F32) with the residual
 * stored as resid_dtype: TR_DTYPE_F32; F16 with its own per-tilt
 * power-of-two scales, recomputed every iteration (the residual's range is
 * not the stack's: after a WBP start it can be far larger); or BF16 (float's
 * range, no scale).  The reprojection, weights and volume stay FP32; the
 * residual back-projection sums are compensated per voxel when the residual
 * is 16-bit. */
tr_status tr_sirt_lp(tr_ctx *ctx, const void *proj_dev, int proj_dtype,
                     const float *scale_dev, int resid_dtype, float *vol_dev,
                     int iters, float gamma, void *stream);

/* SIRT over z-slabs (TiltRecZ's split of the volume along z,
 * TR/main/main-mpiz.cpp:1054-1069, with CuSIRTZ's iteration,
 * TR/TiltRec_cuda_z/recon_z.cu:85-190), either layout, storage as
 * tr_sirt_lp.  Each iteration is one sweep over the slabs: the SIRT update of
 * slab k from the residual, then the forward projection of the updated slab
 * into the next iteration's sums, so every slab is touched once per
 * iteration.  vol_on_host != 0: `vol` is host memory (page-locked for the
 * copies to overlap; any size the host holds) staged through three device
 * slabs, slab k+1 copied in and slab k-1 copied out while slab k computes;
 * the call then returns when the volume is written back.  Otherwise `vol` is
 * the device volume and the call is ordered on `stream`.  depth: sections per
 * slab, rounded down to a multiple of 32 (at least 32; the whole thickness
 * when larger).  Results equal tr_sirt / tr_sirt_lp up to the order of the
 * forward projection's float atomic adds.  Device memory: two reprojections
 * (ntilt*ny*nx floats each), the weights, and with a host volume three slabs
 * of depth*ny*nx floats. */
tr_status tr_sirt_zslabs(tr_ctx *ctx, const void *proj_dev, int proj_dtype,
                         const float *scale_dev, int resid_dtype, float *vol,
                         int vol_on_host, int iters, float gamma, int depth,
                         void *stream);

/* Deterministic forward projections for this context (on != 0; off by
 * default).  The splat's window flush then adds each pixel's contributions
 * as int64 fixed point at one launch-wide scale (the largest power of two S
 * with S * voxels * max|v| <= 2^62, so no sum can overflow; each contribution
 * rounded from the same float value the default flush adds), and the sums are
 * converted and added into the output afterwards.  Integer addition is
 * associative, so tr_forward_project and every SIRT / SART / ADMM / z-slab
 * call of the context give bitwise-identical results run to run (the
 * back-projection is deterministic in both modes).  Costs a reduction over
 * the volume, int64 sums of twice the stack's bytes and a conversion pass per
 * forward projection.  Scheduler and tr_sirt_static calls are not affected. */
tr_status tr_set_deterministic(tr_ctx *ctx, int on);

/* SIRT over z-slabs from host buffers, the volume staying in host memory
 * (volumes larger than the device budget: TiltRecZ's managed-memory
 * streaming, TR/TiltRec_cuda_z/recon_z.cu:96-100).  The stack is copied to
 * the device (counted in the budget); vol_host (page-locked for overlapped
 * copies: tr_host_alloc) is the starting volume, or zeroed first when
 * zero_start; depth 0 autotunes the slab depth (tr_autotune_zslab), and
 * *depth_used (may be NULL) receives the depth run.  Blocking. */
tr_status tr_sirt_host_zslabs(tr_ctx *ctx, const float *proj_host, float *vol_host,
                              int zero_start, int iters, float gamma, int depth,
                              int *depth_used);

/* Page-locked host memory (cudaHostAlloc) for host-buffer calls, and its
 * release. */
tr_status tr_host_alloc(size_t bytes, void **out);
tr_status tr_host_free(void *p);

/* Picks the slab depth for tr_sirt_zslabs: times one full sweep (copies,
 * update with gamma 0 over a zero residual, forward projection; the volume's
 * values are unchanged) at depths 32, 64, 128, 256, 512 (those that fit the
 * HBM budget) and returns the fastest, with its sweep time in ms when
 * sweep_ms is not NULL.  Blocking. */
tr_status tr_autotune_zslab(tr_ctx *ctx, const void *proj_dev, int proj_dtype,
                            const float *scale_dev, int resid_dtype, float *vol,
                            int vol_on_host, int *depth_out, double *sweep_ms);

/* ---- Batched jobs and serving.  No counterpart in the reference, which
 * reconstructs one tilt series per process run.
 *
 * A scheduler owns one device and an HBM budget.  Submitted jobs are
 * admitted while their device memory fits the budget; admission (upload,
 * 16-bit storage of the projections, WBP filtering, the weights of SIRT
 * jobs) runs on its own stream and overlaps the running jobs, and a finished
 * job's volume is copied back on a third.  Two step policies:
 *  - TR_SCHED_BATCHED (default): jobs are admitted in submission order and
 *    all admitted jobs advance together, one step at a time: a step is one
 *    persistent forward-projection launch, one residual launch and one
 *    persistent back-projection launch over the tiles of every job (a WBP
 *    back-projection or one SIRT iteration each), replayed from a CUDA graph.
 *  - TR_SCHED_SRPT: shortest remaining work first.  Admission takes the
 *    queued job with the least work that fits; each step runs the next unit
 *    (WBP back-projection or SIRT iteration) of the ready job with the least
 *    work left, through the same per-job kernels as tr_sirt / tr_wbp
 *    (optionally aged: tr_sched_set_aging).
 * A background thread drives the steps; calls are thread-safe.
 * Results do not depend on the other jobs in the mix beyond the order of the
 * forward projection's float atomic adds (as for a job run alone).  Images
 * must suit the TMA staging: rows of a multiple of 16 bytes (nx % 4 == 0 for
 * FP32 storage, nx % 8 == 0 for 16-bit storage). */
typedef struct tr_sched tr_sched;

typedef struct {
  int nx, ny, ntilt, thickness, layout;
  const double *coeff8;  /* ntilt*8, copied at submission */
  float ox, oy, oz;      /* origin as for tr_set_problem */
  const float *proj;     /* FP32 stack [ntilt][ny][nx] */
  float *vol;            /* result (whole volume); also the starting volume
                            when vol_in is 1 */
  int vol_in;            /* 1: start from vol (--initial); 0: start from zeros */
  int host;              /* 1: proj and vol are host buffers (pinned for overlap);
                            0: device buffers, vol updated in place */
  int wbp;               /* 1: add the WBP reconstruction first (--method WBP) */
  int sirt_iters;        /* then SIRT iterations */
  float gamma;
} tr_job;

typedef struct {
  long long steps, bp_items, fp_items;
  size_t peak_bytes;     /* most job memory admitted at once */
  int grid_bp, grid_fp;  /* persistent CTAs of the step launches */
  size_t smem_bp;        /* back-projection shared-memory budget per CTA */
  int queued, active;
} tr_sched_info;

/* proj_dtype: storage of the stack between steps (TR_DTYPE_F32/F16/BF16,
 * 16-bit with per-tilt power-of-two scales); resid_dtype: SIRT residual
 * storage (FP16 in the stack's scales). */
tr_status tr_sched_create(int device, size_t hbm_budget, int proj_dtype,
                          int resid_dtype, tr_sched **out);
tr_status tr_sched_submit(tr_sched *s, const tr_job *job, unsigned long long *id);
/* Blocks until job `id` is done (its volume written); latency from
 * submission to completion in seconds. */
tr_status tr_sched_wait(tr_sched *s, unsigned long long id, double *latency_s);
/* Blocks until every submitted job is done. */
tr_status tr_sched_drain(tr_sched *s);
tr_status tr_sched_stats(tr_sched *s, tr_sched_info *out);
const char *tr_sched_last_error(const tr_sched *s);
/* Launch configuration of the steps (waits until idle): back-projection
 * shared-memory budget per CTA and resident CTAs per SM (0: as many as fit). */
tr_status tr_sched_configure(tr_sched *s, size_t smem_bp, int bp_ctas_per_sm);
#define TR_SCHED_BATCHED 0
#define TR_SCHED_SRPT 1
/* Step policy (TR_SCHED_BATCHED / TR_SCHED_SRPT); takes effect at the next
 * step or admission. */
tr_status tr_sched_set_policy(tr_sched *s, int policy);
/* TR_SCHED_SRPT aging: a job's remaining work counts divided by
 * 1 + (seconds since submission) / aging_s when jobs are ordered, so that a
 * long job's priority grows while it waits (bounding its delay behind a
 * stream of short ones).  0 (the default): pure shortest remaining work. */
tr_status tr_sched_set_aging(tr_sched *s, double aging_s);
/* Autotuner: times `iters` SIRT steps of a device-resident probe job (run on
 * a scratch copy of its volume) under candidate configurations -- shared
 * memory per back-projection CTA (40, 56, 80, 112 KiB) at full residency,
 * then one resident CTA fewer at the best -- and keeps the fastest. */
tr_status tr_sched_autotune(tr_sched *s, const tr_job *probe, int iters,
                            size_t *best_smem_bp, int *best_ctas_per_sm);
tr_status tr_sched_destroy(tr_sched *s);

/* SIRT that allocates no device memory and needs no context.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc
 * where they reconstruct: a process whose memory pool already owns the device
 * memory it may use, or a stream-ordered pipeline that must not take the
 * device-wide synchronisation an allocation can imply.  Arguments are those of
 * tr_set_problem followed by those of tr_sirt; `device` is made current for
 * the call and restored.  All scratch lives in one static device array of
 * tr_static_scratch_limit() bytes (64 MiB), held until the process exits.  It
 * is reserved when the library's device code is loaded on a device: under
 * CUDA's default lazy module loading at the first use of the library's kernels
 * there; under CUDA_MODULE_LOADING=EAGER as soon as the library is loaded, on
 * every device the process uses, whether or not this function is called.
 * Problems whose geometry (ntilt*112 B), reprojection and projection weights
 * (2*ntilt*ny*nx*4 B) and voxel weights (voxels*4 B), each rounded up to
 * 256 B, exceed it are rejected with TR_ERR_BUDGET, and ntilt is at most 360;
 * non-finite coefficients give TR_ERR_ARG.  The geometry is passed to the
 * device as kernel arguments, so nothing on the host is read after the call
 * returns.  The first call on a device also looks up the array's device
 * address (a synchronous runtime call).  Calls share the array: each clears what
 * must start at zero, and calls whose work overlaps on the GPU race.  A
 * back-projection whose bounded staging wait gives up leaves its volume
 * unchanged and sets a sticky report word in the array that later calls do
 * not clear: tr_static_take_timeout returns it. */
tr_status tr_sirt_static(int device, int nx, int ny, int ntilt, int thickness,
                         int layout, const double *coeff8, float ox, float oy,
                         float oz, const float *proj_dev, float *vol_dev,
                         int iters, float gamma, void *stream);
size_t tr_static_scratch_limit(void);
/* Reads and clears the static scratch's device-wait report on `device`:
 * TR_ERR_TIMEOUT when a tr_sirt_static back-projection gave up a wait since
 * the last read, else TR_OK.  Synchronise the streams of the calls first.  No
 * counterpart in the reference. */
tr_status tr_static_take_timeout(int device);
/* Self-test of the static path's device-wait report (no counterpart in the
 * reference): a bounded wait on a barrier nothing completes, with a budget of
 * budget_us microseconds of GPU clock, reporting through the static scratch;
 * returns TR_ERR_TIMEOUT (the expected outcome) as tr_static_take_timeout
 * would after a back-projection that gave up. */
tr_status tr_static_selftest_wait(int device, int budget_us);

/* Byte output of a float volume (--f2b), on the device: for each slab of
 * `slab` consecutive values (the last may be shorter) its mean and standard
 * deviation, exponentially averaged over the slabs in order (g = alpha g +
 * (1 - alpha) stat from g = 0: the Y-layout drivers use alpha 0.9 and 64-row
 * slabs, the Z-layout ones the whole volume as one slab with alpha 0,
 * src/TiltRec/src/TiltRec_cuda_z/recon_z.cu:164-172), then every value of
 * each complete group of four in a slab mapped to
 * (clamp((v - mean) / std, -10, 10) + 10) / 20 * 255, truncated to a byte
 * (0 for the values past the last complete group).  Replaces the reference's
 * per-slab thrust reductions and CufloatToByteKernel
 * (src/TiltRec/src/TiltRec_cuda_y/recon_y.cu:164-181, basic.cu:442-475);
 * the slab sums here are FP64 over fixed partitions, so repeated runs give
 * the same bytes.  vol_dev: n floats; out_dev: n bytes; at most 65535 slabs. */
tr_status tr_volume_to_bytes(tr_ctx *ctx, const float *vol_dev, size_t n, size_t slab,
                             float alpha, unsigned char *out_dev, void *stream);

/* Receives consecutive blocks of a reconstruction's output, in order; returns
 * 0 to continue, non-zero to stop the transfer (the call then fails with
 * TR_ERR_ARG). */
typedef int (*tr_block_sink)(void *user, const void *data, size_t offset, size_t bytes);

/* Host-buffer reconstruction whose output streams to the caller in blocks:
 * as tr_reconstruct_host (vol_init_host NULL: zero start), then, when
 * f2b_slab > 0, tr_volume_to_bytes on the device with that slab length and
 * f2b_alpha (the output is then one byte per voxel), and the output is copied
 * back through two pinned staging buffers of block_bytes each (kept by the
 * context): the copy of block k+1 is in flight while `sink` consumes block k,
 * as the reference writes each slab with MrcStackM::WriteBlock while the next
 * is transferred (src/TiltRec/src/mrcmx/mrcstack.cpp:472-521). */
tr_status tr_reconstruct_to_sink(tr_ctx *ctx, int method, const float *proj_host,
                                 const float *vol_init_host, int iters, float gamma,
                                 size_t f2b_slab, float f2b_alpha, size_t block_bytes,
                                 tr_block_sink sink, void *user);

/* Area binning of nt images [nt][ny][nx] to [nt][ny/bin][nx/bin] (bin 1..64),
 * the GUI chain's `resample -b bin` before TiltRec (resample/src/main/
 * main.cpp:14-58, OpenCV's area resize): each output pixel is the overlap-
 * weighted mean of its input cell.  Needs no context; runs on the current
 * device (tr_resample_bin) or copies host buffers through `device`. */
tr_status tr_resample_bin(const float *src_dev, int nx, int ny, int nt, int bin,
                          float *dst_dev, void *stream);
tr_status tr_resample_bin_host(int device, const float *src_host, int nx, int ny,
                               int nt, int bin, float *dst_host);

/* Self-test of the device-side wait limit (no counterpart in the reference):
 * one CTA waits on a barrier nothing completes, with a budget of budget_us
 * microseconds of GPU clock.  Returns TR_ERR_TIMEOUT when the wait gave up and
 * reported as a back-projection does (the expected outcome), after which the
 * context stays usable. */
tr_status tr_selftest_wait(tr_ctx *ctx, int budget_us);

/* Wait for all work the context issued. */
tr_status tr_synchronize(tr_ctx *ctx);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* TILTREC_B200_H */
