// TiltRec reconstruction kernels for sm_100a: back-projection (gather),
// forward projection (scatter with shared-memory pre-aggregation) and the
// SIRT residual.
//
// Geometry.  For voxel (x, y, z) and tilt t the reference computes, in double,
//   u = a0 + a1 (x-ox) + a2 (y-oy) + a3 (z-oz) + ox,   v = (same with b) + oy
// and interpolates the projection bilinearly at (u, v) with x0 = floor(u),
// dx = float(u - x0) (main/main-mpi.cpp:204-226).  Here the per-tilt, per-tile
// base coordinate is formed in FP64 exactly that way and then advanced per
// voxel in Q32.32 fixed point (64-bit integer adds): the integer word is the
// table column, the fraction word gives 1+dx as a float by bit assembly.  The
// worst-case coordinate error over a tile is ~1e-8 pixel.
//
// Interpolation tables.  For each tilt of a chunk a CTA stages the detector
// window its tile can reach into shared memory as entries
//   E(j, k) = (b - s, s),  b = P(j, k), s = P(j, k+1) - P(j, k)
// so that interpolating along x at 1+dx is a single FMA:
//   fma(1+dx, s, b-s) = b + dx*s.
// The boundary rules of the reference are folded into the entries:
//   * normalised back-projection (s/c per tilt, BackProject :411-450,
//     UpdateVolumeByProjDiff :492-524): s/c equals bilinear interpolation of
//     the edge-clamped image whenever the lower neighbour lies in
//     [-1, nx-1] x [-1, ny-1], and the voxel gets nothing otherwise.  Entries
//     use the clamped image inside that range and are zero outside it; rows
//     below -1 / at or above ny are masked per voxel when a tile can reach them.
//   * unnormalised gathers (UpdateWeightsByProjDiff :526-562, SIRT): taps
//     outside the image contribute zero, i.e. interpolation of the zero-padded
//     image.  Entries use the zero-padded image.
//   * the SIRT voxel weight sum c uses the indicator image (1 inside).
// Separable geometry (b1 = b3 = 0, b2 = 1: no XTILT, no in-plane rotation,
// any per-tilt y shift) interpolates in y with one weight per voxel row, so
// the two rows are blended while staging and the inner loop is one table
// read and one FMA per voxel and tilt.
#include "tr_internal.cuh"

namespace trb {

__device__ __forceinline__ float one_plus_frac(unsigned long long U) {
  // 1 + (low 32 bits / 2^32), truncated to the 23-bit float mantissa.
  return __uint_as_float(0x3F800000u | ((unsigned)U >> 9));
}

// Adds the scaled contribution x (|x| <= 2^21) to a fixed-point window entry,
// rounded to the nearest integer by the 1.5*2^23 float shift.
__device__ __forceinline__ void wadd(int *p, float x) {
  atomicAdd(p, __float_as_int(x + 12582912.0f) - 0x4B400000);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// Separable row weights for one (tilt, voxel row): lower detector row y0 and
// the in-image tap weights along y; inv = 1/(w0+w1), or 0 when both taps
// miss the image (the reference's c == 0 case).
struct SepW {
  int y0;
  float w0, w1, dy;
};

// FP64 setup of one tilt for one tile (thread-local; one thread per tilt).
// (ex, ey, ez) are the tile's extents minus one.  The window spans columns
// kmin .. kmin+nq-1 and rows jmin .. jmin+nr-1: every lower neighbour the
// tile's voxels can have, its upper neighbour, and one column/row of margin
// for the fixed-point rounding of the voxel coordinates.
__device__ void tile_setup(const TiltGeo &g, int xc, int yc, int zc, float ox,
                           float oy, float oz, int pny, bool sep, double ex,
                           double ey, double ez, TileTilt &tt, SepW *sw) {
  const double X = (double)((float)xc - ox);
  const double Y = (double)((float)yc - oy);
  const double Z = (double)((float)zc - oz);
  const double uc = g.a[0] + g.a[1] * X + g.a[2] * Y + g.a[3] * Z + (double)ox;
  const double umin = uc + fmin(0.0, g.a[1] * ex) + fmin(0.0, g.a[2] * ey) +
                      fmin(0.0, g.a[3] * ez);
  const double umax = uc + fmax(0.0, g.a[1] * ex) + fmax(0.0, g.a[2] * ey) +
                      fmax(0.0, g.a[3] * ez);
  const int kmin = (int)floor(umin) - 1;
  tt.kmin = kmin;
  tt.nq = (int)floor(umax) - (int)floor(umin) + 4;
  tt.U0 = __double2ll_rn((uc - (double)kmin) * 4294967296.0);
  if (!sep) {
    const double vc =
        g.b[0] + g.b[1] * X + g.b[2] * Y + g.b[3] * Z + (double)oy;
    const double vmin = vc + fmin(0.0, g.b[1] * ex) + fmin(0.0, g.b[2] * ey) +
                        fmin(0.0, g.b[3] * ez);
    const double vmax = vc + fmax(0.0, g.b[1] * ex) + fmax(0.0, g.b[2] * ey) +
                        fmax(0.0, g.b[3] * ez);
    const int jmin = (int)floor(vmin) - 1;
    tt.jmin = jmin;
    tt.nr = (int)floor(vmax) - (int)floor(vmin) + 4;
    tt.V0 = __double2ll_rn((vc - (double)jmin) * 4294967296.0);
    tt.check_rows = (floor(vmin) - 1.0 < -1.0) || (floor(vmax) + 1.0 > pny - 1);
  } else {
    tt.jmin = 0;
    tt.nr = kTY;
    tt.V0 = 0;
    tt.check_rows = 0;
    for (int r = 0; r < kTY; ++r) {
      // n1 = b0 + b1 X + b2 Y + b3 Z with b1 = b3 = 0, b2 = 1; y = n1 + oy.
      const double Yr = (double)((float)(yc + r) - oy);
      const double v = g.b[0] + g.b[1] * X + g.b[2] * Yr + g.b[3] * Z + (double)oy;
      const int y0 = (int)floor(v);
      const float dy = (float)(v - (double)y0);
      sw[r].y0 = y0;
      sw[r].dy = dy;
      sw[r].w0 = (y0 >= 0 && y0 < pny) ? (1 - dy) : 0.f;
      sw[r].w1 = (y0 + 1 >= 0 && y0 + 1 < pny) ? dy : 0.f;
    }
  }
}

// Image value for table staging.  MODE: BP_NORM clamped, BP_SIRT zero padded,
// BP_WEIGHTS indicator.
template <int MODE>
__device__ __forceinline__ float img_at(const float *p, int nx, int ny, int j,
                                        int k) {
  if (MODE == BP_NORM) {
    return __ldg(p + (size_t)clampi(j, 0, ny - 1) * nx + clampi(k, 0, nx - 1));
  } else {
    const bool in = (unsigned)j < (unsigned)ny && (unsigned)k < (unsigned)nx;
    if (MODE == BP_WEIGHTS) return in ? 1.f : 0.f;
    return in ? __ldg(p + (size_t)j * nx + k) : 0.f;
  }
}

// Separable staging: blended row value at column k (BP_NORM: k is clamped).
template <int MODE>
__device__ __forceinline__ float sep_at(const float *p, int nx, int ny,
                                        const SepW &s, int k) {
  if (MODE == BP_NORM) {
    const float c = s.w0 + s.w1;
    const int kc = clampi(k, 0, nx - 1);
    const float p0 = s.w0 != 0.f ? __ldg(p + (size_t)s.y0 * nx + kc) : 0.f;
    const float p1 = s.w1 != 0.f ? __ldg(p + (size_t)(s.y0 + 1) * nx + kc) : 0.f;
    return (s.w0 * p0 + s.w1 * p1) / c;
  } else {
    if ((unsigned)k >= (unsigned)nx) return 0.f;
    if (MODE == BP_WEIGHTS) return s.w0 + s.w1;
    const float p0 = s.w0 != 0.f ? __ldg(p + (size_t)s.y0 * nx + k) : 0.f;
    const float p1 = s.w1 != 0.f ? __ldg(p + (size_t)(s.y0 + 1) * nx + k) : 0.f;
    return s.w0 * p0 + s.w1 * p1;
  }
}

template <int MODE, bool SEP>
__global__ void __launch_bounds__(kThreads)
    bp_kernel(const BpArgs a) {
  extern __shared__ float2 tbl[];
  __shared__ TileTilt tt[kMaxChunk];
  __shared__ SepW sw[kMaxChunk][kTY];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wy = (tid >> 5) % kTY;
  const int wz = (tid >> 5) / kTY;
  const int xc = blockIdx.x * kTX, yc = blockIdx.y * kTY, zl = blockIdx.z * kTZ;
  const int zc = zl + a.v.zoff;
  const int fw = a.fw, fh = SEP ? kTY : a.fh;
  const int pnx = a.img.nx, pny = a.img.ny;

  float acc[kNV];
#pragma unroll
  for (int k = 0; k < kNV; ++k) acc[k] = 0.f;

  for (int c0 = 0; c0 < a.nt; c0 += a.chunk) {
    const int nc = min(a.chunk, a.nt - c0);
    if (tid < nc)
      tile_setup(a.geo[a.t0 + c0 + tid], xc, yc, zc, a.ox, a.oy, a.oz, pny, SEP,
                 kTX - 1, kTY - 1, kTZ - 1, tt[tid], sw[tid]);
    __syncthreads();
    // Stage the interpolation tables of the chunk.  One flat loop over the
    // chunk's entries keeps many independent image loads in flight per
    // thread; entries outside a tilt's reachable window are skipped.
    const int per = fh * fw;
    for (int e = tid; e < nc * per; e += kThreads) {
      const int i = e / per, rq = e - i * per;
      const int r = rq / fw, q = rq - r * fw;
      if (r >= tt[i].nr || q >= tt[i].nq) continue;
      const float *p = a.img.p ? a.img.p + (size_t)(a.t0 + c0 + i) * a.img.tstride
                               : nullptr;
      const int x0 = tt[i].kmin + q;
      float b, n;
      if (SEP) {
        const SepW s = sw[i][r];
        const bool valid = (MODE != BP_NORM) ||
                           ((s.w0 + s.w1) != 0.f && x0 >= -1 && x0 <= pnx - 1);
        b = valid ? sep_at<MODE>(p, pnx, pny, s, x0) : 0.f;
        n = valid ? sep_at<MODE>(p, pnx, pny, s, x0 + 1) : 0.f;
      } else {
        const int j = tt[i].jmin + r;
        const bool valid = (MODE != BP_NORM) ||
                           (x0 >= -1 && x0 <= pnx - 1 && j >= -1 && j <= pny);
        b = valid ? img_at<MODE>(p, pnx, pny, j, x0) : 0.f;
        n = valid ? img_at<MODE>(p, pnx, pny, j, x0 + 1) : 0.f;
      }
      const float sl = n - b;
      tbl[e] = make_float2(b - sl, sl);
    }
    __syncthreads();

    for (int i = 0; i < nc; ++i) {
      const TiltGeo &g = a.geo[a.t0 + c0 + i];
      const long long A0 = g.A[0], A1 = g.A[1], A2 = g.A[2];
      unsigned long long U = (unsigned long long)(tt[i].U0 + lane * A0 + wy * A1 +
                                                  (long long)(wz * kNV) * A2);
      if (SEP) {
        const float2 *T = tbl + (size_t)(i * kTY + wy) * fw;
#pragma unroll
        for (int k = 0; k < kNV; ++k) {
          const float2 t = T[(int)(U >> 32)];
          acc[k] += fmaf(one_plus_frac(U), t.y, t.x);
          U += (unsigned long long)A2;
        }
      } else {
        const long long B0 = g.B[0], B1 = g.B[1], B2 = g.B[2];
        unsigned long long V = (unsigned long long)(tt[i].V0 + lane * B0 + wy * B1 +
                                                    (long long)(wz * kNV) * B2);
        const float2 *T = tbl + (size_t)i * per;
        const bool chk = (MODE == BP_NORM) && tt[i].check_rows;
        const int jmin = tt[i].jmin;
#pragma unroll
        for (int k = 0; k < kNV; ++k) {
          const int q = (int)(U >> 32), r = (int)(V >> 32);
          const float2 *e = T + r * fw + q;
          const float2 t0 = e[0], t1 = e[fw];
          const float f = one_plus_frac(U);
          const float r0 = fmaf(f, t0.y, t0.x), r1 = fmaf(f, t1.y, t1.x);
          float val = fmaf(one_plus_frac(V) - 1.f, r1 - r0, r0);
          if (chk && (unsigned)(jmin + r + 1) > (unsigned)pny) val = 0.f;
          acc[k] += val;
          U += (unsigned long long)A2;
          V += (unsigned long long)B2;
        }
      }
    }
    __syncthreads();
  }

  // Epilogue: one coalesced read-modify-write per voxel.
  const int x = xc + lane, y = yc + wy;
  if (x >= a.v.nx || y >= a.v.ny) return;
#pragma unroll
  for (int k = 0; k < kNV; ++k) {
    const int z = zl + wz * kNV + k;
    if (z >= a.v.nz) break;
    const size_t idx = (size_t)y * a.v.sy + (size_t)z * a.v.sz + x;
    if (MODE == BP_NORM) {
      a.v.vol[idx] += a.gamma * acc[k];
    } else if (MODE == BP_SIRT) {
      const float w = a.wtvol[idx];
      if (w != 0.f) a.v.vol[idx] += acc[k] / w * a.gamma;
    } else {
      a.out[idx] = acc[k];
    }
  }
}

// Forward projection: voxel splat (Reproject, main/main-mpi.cpp:286-344) of
// one tile into per-tilt shared-memory windows, then one global atomic add per
// touched in-image detector pixel.  v.vol == nullptr splats ones (the
// per-pixel weight sums, reproj_wt).
//
// Each lane owns the voxel pair (x, x+1) with x = xc + 2*lane.  Their columns
// are q and q or q+1 (the x slope is at most 1), so the pair's splat folds
// into three columns per detector row in registers.
//
// The windows accumulate in 32-bit fixed point with native shared-memory
// integer atomics (fire-and-forget; float atomics on shared memory are a
// compare-and-swap loop whose round trips left the kernel latency-bound).  The
// tile's values are scaled by a power of two S chosen from the tile's largest
// |voxel| so that no window entry can overflow: an entry collects at most
// `nbound` voxel contributions (host bound from the x slope) of magnitude at
// most max|v|, and S <= 2^30 / (nbound max|v|); also S <= 2^20 / max|v| so a
// voxel pair's combined contribution stays within the exact range of the
// float-shift rounding (|x| < 2^22).  Each contribution is rounded
// to the nearest integer of its scaled value (a quantum of
// nbound * max|v| * 2^-30, ~1e-9 of the tile's largest value for tilts
// within +-60 degrees); the sums are exact and independent of atomic order.
// The flush converts back (x 1/S) and adds the in-image pixels to the global
// float accumulators.
template <bool SEP>
__global__ void __launch_bounds__(kThreads) fp_kernel(const FpArgs a) {
  extern __shared__ float accs[];
  __shared__ TileTilt tt[kMaxChunk];
  __shared__ SepW sw[kMaxChunk][kTY];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wy = (tid >> 5) % kTY;
  const int wz = (tid >> 5) / kTY;
  const int xc = blockIdx.x * kFX, yc = blockIdx.y * kTY, zl = blockIdx.z * kFTZ;
  const int zc = zl + a.v.zoff;
  const int fw = a.fw, fh = SEP ? kTY : a.fh;
  const int per = fh * fw;

  float va[kFNV], vb[kFNV];
  {
    const int x = xc + 2 * lane, y = yc + wy;
    const bool ina = x < a.v.nx && y < a.v.ny, inb = x + 1 < a.v.nx && y < a.v.ny;
#pragma unroll
    for (int k = 0; k < kFNV; ++k) {
      const int z = zl + wz * kFNV + k;
      const float *p = a.v.vol + (size_t)y * a.v.sy + (size_t)z * a.v.sz + x;
      const bool inz = z < a.v.nz;
      va[k] = !(ina && inz) ? 0.f : (a.v.vol ? __ldg(p) : 1.f);
      vb[k] = !(inb && inz) ? 0.f : (a.v.vol ? __ldg(p + 1) : 1.f);
    }
  }
  // Tile scale: largest |v| over the tile (as ordered float bits).
  __shared__ unsigned wmax[kThreads / 32];
  __shared__ float s_scale, s_inv;
  {
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < kFNV; ++k)
      m = max(m, max(__float_as_uint(fabsf(va[k])), __float_as_uint(fabsf(vb[k]))));
    m = __reduce_max_sync(0xffffffffu, m);
    if (lane == 0) wmax[tid >> 5] = m;
    __syncthreads();
    if (tid == 0) {
      unsigned mm = 0;
      for (int w = 0; w < kThreads / 32; ++w) mm = max(mm, wmax[w]);
      const float vmax = __uint_as_float(mm);
      float lim = vmax > 0.f ? fminf(1073741824.0f / (a.nbound * vmax), 1048576.0f / vmax)
                             : 1.f;
      int ex;
      frexpf(lim, &ex);  // lim = m 2^ex, m in [0.5, 1): 2^(ex-1) <= lim
      s_scale = ldexpf(1.f, ex - 1);
      s_inv = ldexpf(1.f, 1 - ex);
    }
    __syncthreads();
    const float S = s_scale;
#pragma unroll
    for (int k = 0; k < kFNV; ++k) {
      va[k] *= S;
      vb[k] *= S;
    }
  }
  int *const iacc = reinterpret_cast<int *>(accs);

  for (int c0 = 0; c0 < a.nt; c0 += a.chunk) {
    const int nc = min(a.chunk, a.nt - c0);
    if (tid < nc)
      tile_setup(a.geo[a.t0 + c0 + tid], xc, yc, zc, a.ox, a.oy, a.oz, a.pny,
                 SEP, kFX - 1, kTY - 1, kFTZ - 1, tt[tid], sw[tid]);
    for (int e = tid; e < nc * per; e += kThreads) iacc[e] = 0;
    __syncthreads();

    for (int i = 0; i < nc; ++i) {
      const TiltGeo &g = a.geo[a.t0 + c0 + i];
      const long long A0 = g.A[0], A1 = g.A[1], A2 = g.A[2];
      unsigned long long U = (unsigned long long)(tt[i].U0 + (2 * lane) * A0 +
                                                  wy * A1 + (long long)(wz * kFNV) * A2);
      if (SEP) {
        int *T = iacc + (size_t)(i * kTY + wy) * fw;
#pragma unroll
        for (int k = 0; k < kFNV; ++k) {
          const float vA = va[k], vB = vb[k];
          if (vA != 0.f || vB != 0.f) {
            const unsigned long long UB = U + (unsigned long long)A0;
            const int qa = (int)(U >> 32), qb = (int)(UB >> 32);
            const float dxa = one_plus_frac(U) - 1.f, dxb = one_plus_frac(UB) - 1.f;
            const float t1a = dxa * vA, t0a = vA - t1a;
            const float t1b = dxb * vB, t0b = vB - t1b;
            int *e = T + qa;
            if (qb == qa) {
              wadd(e, t0a + t0b);
              wadd(e + 1, t1a + t1b);
            } else if (qb == qa + 1) {
              wadd(e, t0a);
              wadd(e + 1, t1a + t0b);
              wadd(e + 2, t1b);
            } else {
              wadd(e, t0a);
              wadd(e + 1, t1a);
              int *f = T + qb;
              wadd(f, t0b);
              wadd(f + 1, t1b);
            }
          }
          U += (unsigned long long)A2;
        }
      } else {
        const long long B0 = g.B[0], B1 = g.B[1], B2 = g.B[2];
        unsigned long long V = (unsigned long long)(tt[i].V0 + (2 * lane) * B0 +
                                                    wy * B1 + (long long)(wz * kFNV) * B2);
        int *T = iacc + (size_t)i * per;
#pragma unroll
        for (int k = 0; k < kFNV; ++k) {
          const float vA = va[k], vB = vb[k];
          if (vA != 0.f || vB != 0.f) {
            const unsigned long long UB = U + (unsigned long long)A0;
            const unsigned long long VB = V + (unsigned long long)B0;
            const int qa = (int)(U >> 32), qb = (int)(UB >> 32);
            const int ra = (int)(V >> 32), rb = (int)(VB >> 32);
            const float dxa = one_plus_frac(U) - 1.f, dya = one_plus_frac(V) - 1.f;
            const float dxb = one_plus_frac(UB) - 1.f, dyb = one_plus_frac(VB) - 1.f;
            const float ya1 = dya * vA, ya0 = vA - ya1;
            const float a01 = dxa * ya0, a00 = ya0 - a01;
            const float a11 = dxa * ya1, a10 = ya1 - a11;
            const float yb1 = dyb * vB, yb0 = vB - yb1;
            const float b01 = dxb * yb0, b00 = yb0 - b01;
            const float b11 = dxb * yb1, b10 = yb1 - b11;
            int *e = T + ra * fw + qa;
            if (rb == ra && qb == qa) {
              wadd(e, a00 + b00);
              wadd(e + 1, a01 + b01);
              wadd(e + fw, a10 + b10);
              wadd(e + fw + 1, a11 + b11);
            } else if (rb == ra && qb == qa + 1) {
              wadd(e, a00);
              wadd(e + 1, a01 + b00);
              wadd(e + 2, b01);
              wadd(e + fw, a10);
              wadd(e + fw + 1, a11 + b10);
              wadd(e + fw + 2, b11);
            } else {
              wadd(e, a00);
              wadd(e + 1, a01);
              wadd(e + fw, a10);
              wadd(e + fw + 1, a11);
              int *f = T + rb * fw + qb;
              wadd(f, b00);
              wadd(f + 1, b01);
              wadd(f + fw, b10);
              wadd(f + fw + 1, b11);
            }
          }
          U += (unsigned long long)A2;
          V += (unsigned long long)B2;
        }
      }
    }
    __syncthreads();

    // Flush the windows: in-image pixels only, as the reference's splat.
    for (int i = 0; i < nc; ++i) {
      const int kmin = tt[i].kmin, nq = tt[i].nq, nr = tt[i].nr;
      const int *T = iacc + (size_t)i * per;
      float *base = a.val + (size_t)(a.t0 + c0 + i) * a.tstride;
      const float inv = s_inv;
      for (int r = tid >> 5; r < nr; r += kThreads / 32) {
        for (int q = lane; q < nq; q += 32) {
          const float s = (float)T[r * fw + q] * inv;
          const int k = kmin + q;
          if (s == 0.f || (unsigned)k >= (unsigned)a.pnx) continue;
          if (SEP) {
            const SepW w = sw[i][r];
            if ((unsigned)w.y0 < (unsigned)a.pny)
              atomicAdd(base + (size_t)w.y0 * a.pnx + k, s * (1 - w.dy));
            if (w.dy != 0.f && (unsigned)(w.y0 + 1) < (unsigned)a.pny)
              atomicAdd(base + (size_t)(w.y0 + 1) * a.pnx + k, s * w.dy);
          } else {
            const int j = tt[i].jmin + r;
            if ((unsigned)j < (unsigned)a.pny)
              atomicAdd(base + (size_t)j * a.pnx + k, s);
          }
        }
      }
    }
    __syncthreads();
  }
}

// SIRT residual (main/main-mpi.cpp:640-647): r = p - (wt != 0 ? val/wt : val),
// written over val.
__global__ void resid_kernel(const float *__restrict__ p, float *val,
                             const float *__restrict__ wt, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float r = val[i];
    const float w = wt[i];
    if (w != 0.f) r /= w;
    val[i] = p[i] - r;
  }
}

// ---------------------------------------------------------------- launchers

static dim3 tile_grid(const VolView &v) {
  return dim3((v.nx + kTX - 1) / kTX, (v.ny + kTY - 1) / kTY,
              (v.nz + kTZ - 1) / kTZ);
}

template <int MODE, bool SEP>
static cudaError_t launch_bp_t(const BpArgs &a, cudaStream_t s) {
  const int fh = SEP ? kTY : a.fh;
  const size_t smem = (size_t)a.chunk * fh * a.fw * sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(
      bp_kernel<MODE, SEP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)smem);
  if (e != cudaSuccess) return e;
  bp_kernel<MODE, SEP><<<tile_grid(a.v), kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bp(int mode, bool sep, const BpArgs &a, cudaStream_t s) {
  if (sep) {
    if (mode == BP_NORM) return launch_bp_t<BP_NORM, true>(a, s);
    if (mode == BP_SIRT) return launch_bp_t<BP_SIRT, true>(a, s);
    return launch_bp_t<BP_WEIGHTS, true>(a, s);
  }
  if (mode == BP_NORM) return launch_bp_t<BP_NORM, false>(a, s);
  if (mode == BP_SIRT) return launch_bp_t<BP_SIRT, false>(a, s);
  return launch_bp_t<BP_WEIGHTS, false>(a, s);
}

static dim3 fp_grid(const VolView &v) {
  return dim3((v.nx + kFX - 1) / kFX, (v.ny + kTY - 1) / kTY,
              (v.nz + kFTZ - 1) / kFTZ);
}

cudaError_t launch_fp(bool sep, const FpArgs &a, cudaStream_t s) {
  const int fh = sep ? kTY : a.fh;
  const size_t smem = (size_t)a.chunk * fh * a.fw * sizeof(float);
  cudaError_t e;
  if (sep) {
    e = cudaFuncSetAttribute(fp_kernel<true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fp_kernel<true><<<fp_grid(a.v), kThreads, smem, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(fp_kernel<false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fp_kernel<false><<<fp_grid(a.v), kThreads, smem, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_resid(const float *p, float *val, const float *wt, size_t n,
                         int nsm, cudaStream_t s) {
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  resid_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(p, val, wt, n);
  return cudaGetLastError();
}

}  // namespace trb
