// Host-side derivation of the kernels' per-tilt geometry: the Q32.32 voxel
// steps, the per-tile detector window sizes and the forward-projection
// fixed-point bound, shared by the context, the no-allocation entry point and
// the batch scheduler.
#pragma once

#include <algorithm>
#include <cmath>

#include "tr_internal.cuh"

namespace trb {

struct GeomInfo {
  int fw, fh;      // back-projection tile window (columns, rows)
  int ffw, ffh;    // forward-projection tile window
  float nbound;    // most voxel contributions one forward window entry collects
  bool sep;        // every tilt has b1 = b3 = 0, b2 = 1 (separable rows)
  size_t fp_tilt_bytes;  // shared memory of one staged tilt's splat window
  size_t bp_tilt_bytes;  // shared memory of one staged tilt's interpolation table
};

enum GeomStatus {
  GEOM_OK = 0,
  GEOM_NONFINITE,   // a coefficient is NaN or infinite
  GEOM_MAGNITUDE,   // a slope above 1024
  GEOM_RANGE,       // detector coordinates beyond the int range of the windows
  GEOM_SMEM,        // one tilt's window exceeds smem_max
  GEOM_WINDOW,      // a window side exceeds kMaxWindow
};

// Most voxels of one section of a forward-projection tile (kFX x kTY voxels)
// that can add to one window entry.  Entry (q, r) collects the voxels
// whose detector coordinates (u, v) lie in [q-1, q+1) x [r-1, r+1), a 2 x 2
// square; over one section (u, v) = M (x, y) + c with M = [[a1, a2], [b1, b2]],
// so those voxels are the lattice points of the square's preimage, a
// parallelogram of area 4/|det M| and perimeter 4 (|M^-1 e1| + |M^-1 e2|).  A
// convex planar region of area A and perimeter P holds at most A + P/2 + 1
// lattice points (Bokowski, Hadwiger and Wills, 1972); the square is widened
// by 2^-16 px for the fixed-point coordinates and one point is added.
inline double fp_section_bound(double a1, double a2, double b1, double b2) {
  const double cap = (double)kFX * kTY;
  const double det = a1 * b2 - a2 * b1;
  if (!(std::fabs(det) > 1e-9)) return cap;
  const double s = 2.0 + 1.0 / 65536.0;
  // M^-1 = [[b2, -a2], [-b1, a1]] / det
  const double c1 = std::hypot(b2, b1) / std::fabs(det), c2 = std::hypot(a2, a1) / std::fabs(det);
  const double n = s * s / std::fabs(det) + s * (c1 + c2) + 2.0;
  return std::min(cap, std::floor(n));
}

// Most voxels of one forward-projection tile that can add to one window
// entry.  Separable windows hold one voxel row per window row: along x a row
// steps the detector column by |a1|, so at most floor(2/|a1|) + 1 of its
// voxels (+1 for fixed-point rounding) have their lower column at q-1 or q,
// in each of the tile's kFTZ sections.  General geometry: kFTZ sections of at
// most fp_section_bound voxels each (the largest over the tilts).
inline float fp_entry_bound_sep(double min_a1) {
  double n = min_a1 > 2.0 / kFX ? std::floor(2.0 / min_a1) + 2.0 : (double)kFX;
  n = std::min(n, (double)kFX);
  return (float)(n * kFTZ);
}

// Fills g[0..nt) and *out from [nt][8] coefficients; *bad_tilt names the
// offending tilt for the per-tilt failures.
inline int derive_geometry(const double *coeff8, int nt, int nx, int ny, int th,
                           size_t smem_max, TiltGeo *g, GeomInfo *out, int *bad_tilt) {
  bool sep = true;
  double span_u = 0, span_v = 0, fspan_u = 0, fspan_v = 0, min_a1 = 1e30, sect = 0;
  const double two32 = 4294967296.0;
  const double ext = std::max(std::max(nx, ny), th) + 64.0;
  *bad_tilt = -1;
  for (int t = 0; t < nt; ++t) {
    const double *k = coeff8 + 8 * (size_t)t;
    *bad_tilt = t;
    for (int i = 0; i < 4; ++i) {
      if (!std::isfinite(k[i]) || !std::isfinite(k[4 + i])) return GEOM_NONFINITE;
      g[t].a[i] = k[i];
      g[t].b[i] = k[4 + i];
    }
    for (int i = 0; i < 3; ++i) {
      if (std::fabs(k[1 + i]) > 1024.0 || std::fabs(k[5 + i]) > 1024.0) return GEOM_MAGNITUDE;
      g[t].A[i] = std::llrint(k[1 + i] * two32);
      g[t].B[i] = std::llrint(k[5 + i] * two32);
    }
    // Detector coordinates must stay far inside the int range of the window
    // origins for every voxel of the volume.
    const double reach_u =
        std::fabs(k[0]) + (std::fabs(k[1]) + std::fabs(k[2]) + std::fabs(k[3])) * 2 * ext;
    const double reach_v =
        std::fabs(k[4]) + (std::fabs(k[5]) + std::fabs(k[6]) + std::fabs(k[7])) * 2 * ext;
    if (reach_u > 1.0e9 || reach_v > 1.0e9) return GEOM_RANGE;
    if (!(k[5] == 0.0 && k[7] == 0.0 && k[6] == 1.0)) sep = false;
    min_a1 = std::min(min_a1, std::fabs(k[1]));
    sect = std::max(sect, fp_section_bound(k[1], k[2], k[5], k[6]));
    span_u = std::max(span_u, std::fabs(k[1]) * (kTX - 1) + std::fabs(k[2]) * (kTY - 1) +
                                  std::fabs(k[3]) * (kTZ - 1));
    span_v = std::max(span_v, std::fabs(k[5]) * (kTX - 1) + std::fabs(k[6]) * (kTY - 1) +
                                  std::fabs(k[7]) * (kTZ - 1));
    fspan_u = std::max(fspan_u, std::fabs(k[1]) * (kFX - 1) + std::fabs(k[2]) * (kTY - 1) +
                                    std::fabs(k[3]) * (kFTZ - 1));
    fspan_v = std::max(fspan_v, std::fabs(k[5]) * (kFX - 1) + std::fabs(k[6]) * (kTY - 1) +
                                    std::fabs(k[7]) * (kFTZ - 1));
  }
  *bad_tilt = -1;
  out->fw = (int)std::ceil(span_u) + 4;
  out->fh = sep ? kTY : (int)std::ceil(span_v) + 5;
  // Forward windows start at a 4-column boundary (up to 3 extra columns) and
  // span whole 4-column groups, so that the flush adds 16-byte groups.
  // Coverage: a tile's window starts at column floor(umin) - 1 - o (o <= 3,
  // the alignment shift), and a voxel at fixed-point column u' (within eps
  // << 1/2 px of its FP64 column) writes columns floor(u') - start and one
  // more.  Over any tile position that index is at most
  // floor(span + 2 eps) + 6 <= ceil(span) + 6 < ceil(span) + 7 <= ffw, with
  // span = umax - umin <= fspan_u.  Rows start at floor(vmin) - 1 with no
  // shift: at most ceil(span_v) + 3 < ffh.
  out->ffw = ((int)std::ceil(fspan_u) + 4 + 3 + 3) & ~3;
  out->ffh = sep ? kTY : (int)std::ceil(fspan_v) + 5;
  out->nbound = sep ? fp_entry_bound_sep(min_a1) : (float)(sect * kFTZ);
  out->sep = sep;
  out->fp_tilt_bytes = (size_t)out->ffw * out->ffh * sizeof(int);
  out->bp_tilt_bytes = (size_t)out->fw * out->fh * sizeof(float2);
  if (out->bp_tilt_bytes > smem_max || out->fp_tilt_bytes > smem_max) return GEOM_SMEM;
  if (std::max(std::max(out->fw, out->fh), std::max(out->ffw, out->ffh)) > kMaxWindow)
    return GEOM_WINDOW;
  return GEOM_OK;
}

// Tilts staged per chunk when one tilt's window takes `entry` bytes of a
// `budget`-byte table.
inline int chunk_for(size_t budget, size_t entry) {
  return (int)std::max<size_t>(1, std::min<size_t>(kMaxChunk, budget / entry));
}

}  // namespace trb
