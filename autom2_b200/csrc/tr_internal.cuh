// Internal definitions shared by the TiltRec B200 kernels and the C-ABI.
#pragma once

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
};

// Footprint bookkeeping of one tilt for one tile, computed in FP64.
struct TileTilt {
  long long U0, V0;  // Q32.32 detector coordinates of the tile's first voxel,
                     // relative to (kmin, jmin)
  int kmin, jmin;    // detector column / row of table entry (0, 0)
  int check_rows;    // rows outside [-1, ny-1] are reachable (BP_NORM only)
  int nq, nr;        // columns / rows of the window this tile can reach
};

// Separable rows (b1 = b3 = 0, b2 = 1): per voxel row of the tile, the lower
// detector row and its weight, as the reference computes them.
struct SepRow {
  int y0;
  float dy;
};

}  // namespace trb
