// Internal definitions shared by the TiltRec B200 kernels and the C-ABI.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace trb {

// Volume tile owned by one CTA: 32 voxels along x (the lanes of a warp), kTY
// voxel rows (one warp group each) and kZG groups of NV consecutive sections
// along z per row (NV voxels per thread, held in registers).
constexpr int kThreads = 256;
constexpr int kTX = 32;
constexpr int kTY = 4;
constexpr int kZG = kThreads / (kTX * kTY);  // 2
constexpr int kNV = 16;                       // voxels per thread along z
constexpr int kTZ = kZG * kNV;                // 32
constexpr int kMaxChunk = 32;                 // tilts staged per chunk (max)
constexpr int kTileVox = kTX * kTY * kTZ;     // voxels of a back-projection tile

// Forward-projection tile: each lane owns a pair of neighbouring x voxels, so
// a warp covers 64 x; rows and z groups as above.
constexpr int kFX = 2 * kTX;                  // 64
constexpr int kFNV = 16;                      // voxel pairs per thread along z
constexpr int kFTZ = kZG * kFNV;              // 32

// Largest tile window side (columns or rows): the kernels step window
// coordinates in Q9.23 fixed point, whose integer part is below 512.
constexpr int kMaxWindow = 511;

// Per-tilt projection geometry.  a/b are the reference's linear coefficients
// (detector x = a0 + a1 X + a2 Y + a3 Z + ox, y likewise with b, X/Y/Z the
// voxel offsets from the origin).  A/B are the same slopes in Q32.32 fixed
// point, the per-voxel coordinate steps along x, y and z.
struct TiltGeo {
  double a[4], b[4];
  long long A[3], B[3];
};

// A strided view of a float volume: voxel (x, y, z) of the view lives at
// vol[y*sy + z*sz + x]; its global section index (used for geometry) is
// z + zoff.  Y layout (TiltRec): sy = th*nx, sz = nx.  Z layout (TiltRecZ):
// sy = nx, sz = ny*nx.
struct VolView {
  float *vol;
  long long sy, sz;
  int nx, ny, nz;
  int zoff;
};

// Projection images [tilt][ny][nx].  dtype: IMG_F32 / IMG_F16 / IMG_BF16
// elements; value = element * scale[tilt] (scale == nullptr: 1).
enum { IMG_F32 = 0, IMG_F16 = 1, IMG_BF16 = 2 };
struct ImgView {
  const float *p;  // element pointer, reinterpreted per dtype
  int nx, ny;
  long long tstride;
  int dtype;
  const float *scale;
};

enum BpMode {
  BP_NORM = 0,     // vol += gamma * sum_t s/c      (BPT / WBP / SART update)
  BP_SIRT = 1,     // vol += gamma * (sum_t s) / wtvol where wtvol != 0
  BP_WEIGHTS = 2,  // out = sum_t c                 (SIRT voxel weights)
  BP_SUM = 3,      // vol += gamma * sum_t s        (unnormalised gather, A^T)
};

struct BpArgs {
  VolView v;
  ImgView img;
  const TiltGeo *geo;
  int t0, nt;
  float ox, oy, oz;
  int fw, fh, chunk;
  float gamma;
  const float *wtvol;  // BP_SIRT: per-voxel weight sums (same view strides)
  float *out;          // BP_WEIGHTS: output (same view strides)
  // Compact voxel weights (wslot != nullptr): tile (bz gy + by) gx + bx of
  // the view is interior when wslot[tile] < 0 -- every voxel has all four
  // bilinear neighbours inside the image for every tilt -- and its weight is
  // wfull (the tilt count; general geometry) or wrow[y] (separable: the
  // per-row sum of the in-image row weights); a border tile's kTileVox
  // weights live at wtvol / out + wslot[tile] * kTileVox, voxel
  // ((wz kNV + k) kTY + wy) kTX + lane.  The weight pass skips interior tiles.
  const int *wslot;
  const float *wrow;
  float wfull;
  int *err;            // err[0]: launch-wide abort word (zero at launch);
                       // err[1]: sticky report word; both set to 1 when a
                       // bounded device wait runs out.  nullptr: no TMA path.
  // TMA staging (filled by the launcher): raw window box, raw buffer stride in
  // floats and byte offset of the raw buffers in dynamic shared memory.
  int tma_bw, tma_bh, tma_raw_stride, tma_raw_offset;
};

struct FpArgs {
  VolView v;          // v.vol == nullptr: splat ones (the weight pass)
  float *val;         // [nt][ny][nx] accumulators (tilt t at val + t*tstride)
  long long tstride;
  int pnx, pny;       // projection size
  const TiltGeo *geo;
  int t0, nt;
  float ox, oy, oz;
  int fw, fh, chunk;
  float nbound;       // most voxel contributions one window entry can collect
  // Deterministic flush (ival != nullptr): each pixel accumulates int64 fixed
  // point at the launch-wide scale fp_gscale(gmax, gbound), so integer adds in
  // any order give the same sums; launch_ival_to_val then adds them into val.
  // gmax: the view's largest |voxel| as float bits (nullptr: ones, 1);
  // gbound: the view's voxel count, which bounds any pixel's sum / max|v|.
  unsigned long long *ival;
  const unsigned *gmax;
  double gbound;
};

// Footprint bookkeeping of one tilt for one tile, computed in FP64.
struct TileTilt {
  long long U0, V0;  // Q32.32 detector coordinates of the tile's first voxel,
                     // relative to (kmin, jmin)
  int kmin, jmin;    // detector column / row of table entry (0, 0)
  int check_rows;    // rows outside [-1, ny-1] are reachable (BP_NORM only)
  int nq, nr;        // columns / rows of the window this tile can reach
};

// Back-projection coordinate starts of one staged tilt, in Q9.23: the
// per-voxel steps and, per warp w (wy = w % kTY, wz = w / kTY), the
// coordinates of the warp's lane-0 first voxel, U0 + wy A1 + wz kNV A2
// (V likewise), so that a thread's start is one 32-bit multiply-add,
// u0 + lane du_x.
struct WarpStarts {
  unsigned dux, dvx;  // steps along x (one lane)
  unsigned du, dv;    // steps along z
  int jmin, check_rows;
  unsigned u0[kThreads / 32], v0[kThreads / 32];
};

// Forward-projection coordinate starts of one tilt: the x and z steps and,
// per warp, U0 + wy A1 + wz kFNV A2 (V likewise); lane l's voxel pair starts
// at W + 2 l A0.
struct FpStarts {
  long long A0, A2, B0, B2;
  long long Wu[kThreads / 32], Wv[kThreads / 32];
};

// Separable rows (b1 = b3 = 0, b2 = 1): per voxel row of the tile, the lower
// detector row and its weight, as the reference computes them.
struct SepRow {
  int y0;
  float dy;
};

// R-weighting filter of rows in place (tr_filter.cu).
struct FilterArgs {
  float *rows;          // [nrows][nx], filtered in place
  long long nrows;
  int nx, n_pad;        // row length and the reference's padded length N
  int log2m;            // M = 1 << log2m
  const float2 *ghat;   // [M] kernel spectrum, natural order, scaled
  const float2 *tw;     // two-level twiddles (tr_filter_host.h RweightSpectrum::tw)
};

// ------------------------------------------------------------ batched steps
//
// A batch step runs the same stage for many jobs in one launch: a table in
// device memory lists work items; the persistent forward and back-projection
// kernels pull tiles of all items from one atomic counter.  The same launches
// (captured once in a CUDA graph) serve every step: only the table changes.

constexpr int kBatchMaxItems = 256;  // per item kind

struct __align__(64) BatchBp {
  CUtensorMap map;  // TMA descriptor of the item's image stack
  BpArgs a;         // chunk / tma_* laid out for the step's shared budget
  int mode, sep;
  int gx, gy, gz;   // tile grid
  long long first;  // global index of the item's first tile
};

struct BatchFp {
  FpArgs a;
  int sep;
  int gx, gy, gz;
  long long first;
};

struct BatchRes {       // r = p*ps[t] - val/wt, stored as rdtype in units of rs[t]
  const void *p;
  const float *ps;
  const float *val, *wt;
  void *r;
  const float *rs;
  unsigned long long plane;
  int nt, pdtype, rdtype;
  // FP16 residuals: r is FP32 (over val), then stored at q as FP16 with
  // per-tilt power-of-two scales qscale from the maxima qmax (zeroed by the
  // zero stage); q == nullptr: none
  __half *q;
  float *qscale;
  unsigned *qmax;
};

struct BatchZero {
  float *p;
  unsigned long long n;
};

struct BatchHeader {
  int nbp, nfp, nres, nzero;
  int *err;                             // abort word of the step's waits, reset by zero
  long long bp_tiles, fp_tiles;
  unsigned long long bp_next, fp_next;  // work counters, reset by the zero stage
};

// Device table: header, then the item arrays at fixed offsets.
struct BatchTable {
  BatchHeader h;
  BatchBp bp[kBatchMaxItems];
  BatchFp fp[kBatchMaxItems];
  BatchRes res[kBatchMaxItems];
  BatchZero zero[kBatchMaxItems];
};

// ------------------------------------------------------------ launchers
// (tr_kernels.cu, tr_filter.cu)

cudaError_t launch_bp(int mode, bool sep, const BpArgs &a, cudaStream_t s);
// Compact voxel weights: classifies the tiles of view v (slot[tile] = -1
// interior, else a border slot from *count, which must start at 0), and the
// separable per-row weights wrow[0..ny) (rows of voxel view v.ny).
cudaError_t launch_classify_tiles(const TiltGeo *geo, int nt, const VolView &v, float ox, float oy,
                                  float oz, int pnx, int pny, bool sep, int *slot, int *count,
                                  cudaStream_t s);
cudaError_t launch_sep_row_weights(const TiltGeo *geo, int nt, int ny, float oy, int pny,
                                   float *wrow, cudaStream_t s);
cudaError_t launch_fp(bool sep, const FpArgs &a, cudaStream_t s);
// Deterministic forward projection into a.val: the view's max |voxel| into
// *gmax, the splat with the int64 flush into ival (all zero on entry, left
// zero), then the sums converted and added into a.val.
cudaError_t launch_fp_deterministic(bool sep, FpArgs a, unsigned long long *ival,
                                    unsigned *gmax, int nsm, cudaStream_t s);
cudaError_t launch_resid(const float *p, float *val, const float *wt, size_t n, int nsm,
                         cudaStream_t s);
cudaError_t launch_quantize(const float *p, size_t plane, int nt, int dtype, void *out,
                            float *scale, unsigned *maxbits, int nsm, cudaStream_t s);
cudaError_t launch_resid_lp(const void *p, int pdtype, const float *ps, const float *val,
                            const float *wt, size_t plane, int nt, int rdtype, void *r,
                            const float *rs, int nsm, cudaStream_t s);
cudaError_t launch_rweight(const FilterArgs &f, cudaStream_t s);
cudaError_t launch_bounded_wait_selftest(long long budget, int *err, cudaStream_t s);
cudaError_t launch_fbp_filter(float *rows, long long nrows, int nx, int L, int mode,
                              cudaStream_t s);
cudaError_t launch_resample_bin(const float *src, int nx, int ny, int nt, int bin, float *dst,
                                cudaStream_t s);

// ADMM pieces (tr_admm.cu)
constexpr int kAdmmParts = 592;  // blocks of a deterministic dot product
cudaError_t admm_normalize(float *val, const float *wt, size_t n, int nsm, cudaStream_t s);
cudaError_t admm_add_scaled(float *out, const float *x, float mu, size_t n, int nsm,
                            cudaStream_t s);
cudaError_t admm_atb(float *atb, const float *u, const float *d, float mu, size_t n, int nsm,
                     cudaStream_t s);
cudaError_t admm_cg_init(float *r, float *p, const float *b, const float *a, size_t n, int nsm,
                         cudaStream_t s);
// |a|^2 with FP64 products and fixed-order FP64 sums (kAdmmParts partials).
cudaError_t sumsq_f64(const float *a, size_t n, double *part, double *out, cudaStream_t s);
cudaError_t admm_dot(const float *a, const float *b, size_t n, double *part, double *out,
                     cudaStream_t s);
cudaError_t admm_x_update(float *vol, const float *p, const double *scal, size_t n, int nsm,
                          cudaStream_t s);
cudaError_t admm_r_update(float *r, const float *b, const float *ax, size_t n, int nsm,
                          cudaStream_t s);
cudaError_t admm_p_update(float *p, const float *r, const double *scal, size_t n, int nsm,
                          cudaStream_t s);
cudaError_t admm_soft(float *u, float *d, const float *x, float soft, size_t n, int nsm,
                      cudaStream_t s);
// Byte output (tr_output.cu): part[nslabs][kF2bParts] doubles and 4 * nslabs
// floats of statistics as scratch; nslabs = ceil(n / slab) <= 65535.
constexpr int kF2bParts = 64;
cudaError_t launch_f2b(const float *vol, size_t n, size_t slab, float alpha, unsigned char *out,
                       double *part, float *stats, int nsm, cudaStream_t s);

dim3 bp_tile_grid(const VolView &v);
dim3 fp_tile_grid(const VolView &v);
bool batch_bp_layout(const BpArgs &a0, bool sep, size_t budget, BatchBp *out, size_t *smem);
int batch_occupancy(int rdtype, size_t smem_bp, size_t smem_fp, int *fp_per_sm);
cudaError_t launch_batch_step(BatchTable *T, int rdtype, int grid_fp, int grid_bp,
                              size_t smem_fp, size_t smem_bp, int nsm, cudaStream_t s);

}  // namespace trb
