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
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <type_traits>

#include <algorithm>

#include "tr_internal.cuh"

namespace trb {

__device__ __forceinline__ float one_plus_frac(unsigned long long U) {
  // 1 + (low 32 bits / 2^32), truncated to the 23-bit float mantissa: one
  // funnel shift of 0x7F:low by 9 puts 0x7F << 23 = 0x3F800000 above the
  // fraction's top 23 bits.
  return __uint_as_float(__funnelshift_r((unsigned)U, 0x7Fu, 9));
}

// Image element -> float.
__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

// The 1.5*2^23 float shift: its bits are 0x4B400000 + round(x) for
// |x| < 2^22, so the difference of two shifted values is the difference of
// the rounded ones (the forward splat's fixed-point windows).
constexpr int kFshiftBias = 0x4B400000;
__device__ __forceinline__ int fshift(float x) { return __float_as_int(x + 12582912.0f); }

// Paired FP32 arithmetic (sm_100 f32x2): two lanes of float math per
// instruction on 64-bit register pairs {lo, hi}.
using f32x2 = unsigned long long;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(f32x2 r, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
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
template <int MODE, typename IT>
__device__ __forceinline__ float img_at(const IT *p, float sc, int nx, int ny, int j,
                                        int k) {
  if (MODE == BP_NORM) {
    return to_f(__ldg(p + (size_t)clampi(j, 0, ny - 1) * nx + clampi(k, 0, nx - 1))) * sc;
  } else {
    const bool in = (unsigned)j < (unsigned)ny && (unsigned)k < (unsigned)nx;
    if (MODE == BP_WEIGHTS) return in ? 1.f : 0.f;
    return in ? to_f(__ldg(p + (size_t)j * nx + k)) * sc : 0.f;
  }
}

// Separable staging: blended row value at column k (BP_NORM: k is clamped).
template <int MODE, typename IT>
__device__ __forceinline__ float sep_at(const IT *p, float sc, int nx, int ny,
                                        const SepW &s, int k) {
  if (MODE == BP_NORM) {
    const float c = s.w0 + s.w1;
    const int kc = clampi(k, 0, nx - 1);
    const float p0 = s.w0 != 0.f ? to_f(__ldg(p + (size_t)s.y0 * nx + kc)) * sc : 0.f;
    const float p1 = s.w1 != 0.f ? to_f(__ldg(p + (size_t)(s.y0 + 1) * nx + kc)) * sc : 0.f;
    return (s.w0 * p0 + s.w1 * p1) / c;
  } else {
    if ((unsigned)k >= (unsigned)nx) return 0.f;
    if (MODE == BP_WEIGHTS) return s.w0 + s.w1;
    const float p0 = s.w0 != 0.f ? to_f(__ldg(p + (size_t)s.y0 * nx + k)) * sc : 0.f;
    const float p1 = s.w1 != 0.f ? to_f(__ldg(p + (size_t)(s.y0 + 1) * nx + k)) * sc : 0.f;
    return s.w0 * p0 + s.w1 * p1;
  }
}

// Position (tilt i, row r, column q) of table entry e in a chunk's tables laid
// out [tilt][fh rows][fw columns], for e = tid, tid + kThreads, ...: the
// divisions happen once per chunk and each step adds the precomputed
// decomposition of kThreads.
struct EntryWalk {
  int i, r, q, si, sr, sq;
  __device__ __forceinline__ EntryWalk(int e0, int fh, int fw) {
    const int per = fh * fw;
    i = e0 / per;
    const int rq = e0 - i * per;
    r = rq / fw;
    q = rq - r * fw;
    si = kThreads / per;
    const int rem = kThreads - si * per;
    sr = rem / fw;
    sq = rem - sr * fw;
  }
  __device__ __forceinline__ void next(int fh, int fw) {
    q += sq;
    r += sr;
    i += si;
    if (q >= fw) {
      q -= fw;
      ++r;
    }
    if (r >= fh) {
      r -= fh;
      ++i;
    }
  }
};

// Interpolation of one staged chunk of tilts into the thread's accumulators.
// Compensated (Kahan) addition of val to a voxel accumulator: the running
// compensation c carries the low-order bits each addition loses.
__device__ __forceinline__ void kahan_add(float &acc, float &c, float val) {
  const float y = val - c;
  const float t = acc + y;
  c = (t - acc) - y;
  acc = t;
}

// Window coordinates inside the z loop run in Q9.23 (32-bit): the integer
// part is the window column/row (< 512), the 23 fraction bits are exactly the
// float mantissa of 1 + dx.  Each warp's start is the exact Q32.32 value
// truncated and the lane and section steps are rounded to 2^-23, so a
// thread's coordinates (31 lane steps at most, then kNV - 1 section steps)
// stay within 24 * 2^-23 px of the exact ones.
__device__ __forceinline__ unsigned q23(unsigned long long U) { return (unsigned)(U >> 9); }
__device__ __forceinline__ unsigned q23_step(long long A) { return (unsigned)((A + 256) >> 9); }
__device__ __forceinline__ float one_plus_frac23(unsigned u) {
  return __uint_as_float(0x3F800000u | (u & 0x7FFFFFu));
}

// Threads tid < nc * (kThreads / 32) fill ws[0..nc) from the chunk's tile
// bookkeeping tt[0..nc) and geometry geo[0..nc).
__device__ __forceinline__ void fill_warp_starts(WarpStarts *ws, const TileTilt *tt,
                                                 const TiltGeo *geo, int nc, int tid) {
  constexpr int kW = kThreads / 32;
  if (tid >= nc * kW) return;
  const int i = tid / kW, w = tid % kW;
  const int wy = w % kTY, wz = w / kTY;
  const TiltGeo &g = geo[i];
  ws[i].u0[w] = q23((unsigned long long)(tt[i].U0 + wy * g.A[1] + (long long)(wz * kNV) * g.A[2]));
  ws[i].v0[w] = q23((unsigned long long)(tt[i].V0 + wy * g.B[1] + (long long)(wz * kNV) * g.B[2]));
  if (w == 0) {
    ws[i].dux = q23_step(g.A[0]);
    ws[i].dvx = q23_step(g.B[0]);
    ws[i].du = q23_step(g.A[2]);
    ws[i].dv = q23_step(g.B[2]);
    ws[i].jmin = tt[i].jmin;
    ws[i].check_rows = tt[i].check_rows;
  }
}

template <int MODE, bool SEP, bool KAHAN>
__device__ __forceinline__ void bp_accumulate(float (&acc)[kNV], float (&cmp)[kNV],
                                              const void *tblv, const WarpStarts *ws,
                                              int nc, int per, int fw, int pny,
                                              int lane, int wy, int wz) {
  const int w = wz * kTY + wy;  // the warp's index in the CTA
  // KAHAN: the chunk's tilts (at most kMaxChunk) sum into a plain partial,
  // which joins the voxel's total by one compensated addition per chunk.
  float part[kNV];
  float(&sum)[kNV] = KAHAN ? part : acc;
  if (KAHAN) {
#pragma unroll
    for (int k = 0; k < kNV; ++k) part[k] = 0.f;
  }
  for (int i = 0; i < nc; ++i) {
    const WarpStarts &st = ws[i];
    unsigned u = st.u0[w] + lane * st.dux;
    const unsigned du = st.du;
    if (SEP) {
      const float2 *T = reinterpret_cast<const float2 *>(tblv) + (size_t)(i * kTY + wy) * fw;
      // Two sections per step: the two sums advance in one f32x2 add (the
      // same roundings as two scalar adds).
#pragma unroll
      for (int k = 0; k < kNV; k += 2) {
        const float2 ta = T[u >> 23];
        const float ra = fmaf(one_plus_frac23(u), ta.y, ta.x);
        u += du;
        const float2 tb = T[u >> 23];
        const float rb = fmaf(one_plus_frac23(u), tb.y, tb.x);
        u += du;
        unpack2(add2(pack2(sum[k], sum[k + 1]), pack2(ra, rb)), sum[k], sum[k + 1]);
      }
    } else {
      unsigned v = st.v0[w] + lane * st.dvx;
      const unsigned dv = st.dv;
      const float2 *T = reinterpret_cast<const float2 *>(tblv) + (size_t)i * per;
      const int jmin = st.jmin;
      if (MODE == BP_NORM && st.check_rows) {
#pragma unroll
        for (int k = 0; k < kNV; ++k) {
          const int q = (int)(u >> 23), r = (int)(v >> 23);
          const float2 *e = T + r * fw + q;
          const float2 t0 = e[0], t1 = e[fw];
          const float f = one_plus_frac23(u);
          const float r0 = fmaf(f, t0.y, t0.x), r1 = fmaf(f, t1.y, t1.x);
          const float val = fmaf(one_plus_frac23(v) - 1.f, r1 - r0, r0);
          if ((unsigned)(jmin + r + 1) <= (unsigned)pny) sum[k] += val;
          u += du;
          v += dv;
        }
      } else {
        // Two sections per step: the row interpolation and the sums of both
        // run in f32x2 instructions (the same roundings as the scalar form
        // sum += fma(dy, r1 - r0, r0)).
        const f32x2 one2 = pack2(1.f, 1.f);
#pragma unroll
        for (int k = 0; k < kNV; k += 2) {
          float r0[2], r1[2], gy[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int q = (int)(u >> 23), r = (int)(v >> 23);
            const float2 *e = T + r * fw + q;
            const float2 t0 = e[0], t1 = e[fw];
            const float f = one_plus_frac23(u);
            r0[h] = fmaf(f, t0.y, t0.x);
            r1[h] = fmaf(f, t1.y, t1.x);
            gy[h] = one_plus_frac23(v);
            u += du;
            v += dv;
          }
          const f32x2 R0 = pack2(r0[0], r0[1]);
          const f32x2 d = sub2(pack2(r1[0], r1[1]), R0);
          const f32x2 dy = sub2(pack2(gy[0], gy[1]), one2);
          unpack2(add2(pack2(sum[k], sum[k + 1]), fma2(dy, d, R0)), sum[k], sum[k + 1]);
        }
      }
    }
  }
  if (KAHAN) {
#pragma unroll
    for (int k = 0; k < kNV; ++k) kahan_add(acc[k], cmp[k], part[k]);
  }
}

// Tile index of tile (bx, by, bz) in the compact weights' slot table.
__device__ __forceinline__ int bp_tile_index(const VolView &v, int bx, int by, int bz) {
  const int gx = (v.nx + kTX - 1) / kTX, gy = (v.ny + kTY - 1) / kTY;
  return (bz * gy + by) * gx + bx;
}

// Epilogue: one coalesced read-modify-write per voxel.  slot: the tile's
// compact-weight slot (see BpArgs::wslot), -1 interior; unused without them.
template <int MODE, bool SEP>
__device__ __forceinline__ void bp_epilogue(const BpArgs &a, const float (&acc)[kNV],
                                            int x, int y, int zbase, int slot) {
  if (x >= a.v.nx || y >= a.v.ny) return;
  // Voxel k of this thread in a tile's compact weights.
  const int local0 = (((threadIdx.x >> 5) / kTY) * kNV * kTY + (threadIdx.x >> 5) % kTY) * kTX +
                     (threadIdx.x & 31);
#pragma unroll
  for (int k = 0; k < kNV; ++k) {
    const int z = zbase + k;
    if (z >= a.v.nz) break;
    const size_t idx = (size_t)y * a.v.sy + (size_t)z * a.v.sz + x;
    const size_t cidx = (size_t)slot * kTileVox + local0 + k * (kTY * kTX);
    if (MODE == BP_NORM || MODE == BP_SUM) {
      a.v.vol[idx] += a.gamma * acc[k];
    } else if (MODE == BP_SIRT) {
      float w;
      if (!a.wslot) w = a.wtvol[idx];
      else if (slot < 0) w = SEP ? a.wrow[y] : a.wfull;
      else w = a.wtvol[cidx];
      if (w != 0.f) a.v.vol[idx] += acc[k] / w * a.gamma;
    } else {
      a.out[a.wslot ? cidx : idx] = acc[k];
    }
  }
}

// Slot of tile (bx, by, bz) in the compact weights, or -1.
__device__ __forceinline__ int bp_tile_slot(const BpArgs &a, int bx, int by, int bz) {
  return a.wslot ? __ldg(a.wslot + bp_tile_index(a.v, bx, by, bz)) : -1;
}

// Back-projection with tables staged by the threads from global memory (any
// image width; also the voxel-weight pass, which has no image).
template <int MODE, bool SEP, typename IT>
__global__ void __launch_bounds__(kThreads)
    bp_kernel(const BpArgs a) {
  constexpr bool KAHAN = !std::is_same<IT, float>::value;
  extern __shared__ float4 tbl_raw[];
  float2 *tbl2 = reinterpret_cast<float2 *>(tbl_raw);
  __shared__ TileTilt tt[kMaxChunk];
  __shared__ SepW sw[kMaxChunk][kTY];
  __shared__ WarpStarts ws[kMaxChunk];

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wy = (tid >> 5) % kTY;
  const int wz = (tid >> 5) / kTY;
  const int xc = blockIdx.x * kTX, yc = blockIdx.y * kTY, zl = blockIdx.z * kTZ;
  const int zc = zl + a.v.zoff;
  const int fw = a.fw, fh = SEP ? kTY : a.fh;
  const int pnx = a.img.nx, pny = a.img.ny;
  const int slot = bp_tile_slot(a, blockIdx.x, blockIdx.y, blockIdx.z);
  // Compact weights: interior tiles need no weight pass (uniform per CTA).
  if (MODE == BP_WEIGHTS && a.wslot && slot < 0) return;

  float acc[kNV], cmp[kNV];
#pragma unroll
  for (int k = 0; k < kNV; ++k) acc[k] = cmp[k] = 0.f;

  for (int c0 = 0; c0 < a.nt; c0 += a.chunk) {
    const int nc = min(a.chunk, a.nt - c0);
    if (tid < nc)
      tile_setup(a.geo[a.t0 + c0 + tid], xc, yc, zc, a.ox, a.oy, a.oz, pny, SEP,
                 kTX - 1, kTY - 1, kTZ - 1, tt[tid], sw[tid]);
    __syncthreads();
    fill_warp_starts(ws, tt, a.geo + a.t0 + c0, nc, tid);
    // Stage the interpolation tables of the chunk.  One flat loop over the
    // chunk's entries keeps many independent image loads in flight per
    // thread; entries outside a tilt's reachable window are skipped.
    const int per = fh * fw;
    EntryWalk w(tid, fh, fw);
    for (int e = tid; e < nc * per; e += kThreads, w.next(fh, fw)) {
      const int i = w.i, r = w.r, q = w.q;
      if (r >= tt[i].nr || q >= tt[i].nq) continue;
      const int tilt = a.t0 + c0 + i;
      const IT *p = a.img.p ? reinterpret_cast<const IT *>(a.img.p) + (size_t)tilt * a.img.tstride
                            : nullptr;
      const float sc = a.img.scale ? a.img.scale[tilt] : 1.f;
      const int x0 = tt[i].kmin + q;
      if (SEP) {
        const SepW s = sw[i][r];
        const bool valid = (MODE != BP_NORM) ||
                           ((s.w0 + s.w1) != 0.f && x0 >= -1 && x0 <= pnx - 1);
        const float b = valid ? sep_at<MODE>(p, sc, pnx, pny, s, x0) : 0.f;
        const float n = valid ? sep_at<MODE>(p, sc, pnx, pny, s, x0 + 1) : 0.f;
        const float sl = n - b;
        tbl2[e] = make_float2(b - sl, sl);
      } else {
        const int j = tt[i].jmin + r;
        const bool valid = (MODE != BP_NORM) ||
                           (x0 >= -1 && x0 <= pnx - 1 && j >= -1 && j <= pny);
        const float b = valid ? img_at<MODE>(p, sc, pnx, pny, j, x0) : 0.f;
        const float n = valid ? img_at<MODE>(p, sc, pnx, pny, j, x0 + 1) : 0.f;
        const float sl = n - b;
        tbl2[e] = make_float2(b - sl, sl);
      }
    }
    __syncthreads();
    bp_accumulate<MODE, SEP, KAHAN>(acc, cmp, tbl_raw, ws, nc, per, fw, pny, lane, wy, wz);
    __syncthreads();
  }
  bp_epilogue<MODE, SEP>(a, acc, xc + lane, yc + wy, zl + wz * kNV, slot);
}

// ------------------------------------------------------------- TMA staging
//
// One elected thread issues, per tilt, a 3-D bulk tensor copy (TMA,
// cp.async.bulk.tensor, no multicast) of the tile's raw detector window --
// columns [kmin rounded down to 16 bytes, +BW), rows [ys, +BH) of image
// `tilt` -- into a raw
// shared buffer; the copies of the next chunk land while the CTA interpolates
// the current one (two raw buffers, one mbarrier each).  TMA fills the parts
// of a box outside the image with zeros.  The threads then turn the raw window
// into interpolation-table entries with shared-memory reads only.  The global
// tensor needs 16-byte row strides, so this path serves images whose rows are
// a multiple of 16 bytes (width % 4 for float, % 8 for 16-bit elements); the
// others stage through bp_kernel.

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *m, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for a phase until it completes (true), `budget` clock cycles pass or
// the launch-wide abort word becomes non-zero (false).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *m, unsigned parity,
                                                  long long budget, const int *abort_word) {
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try_wait(m, parity)) return true;
    if (clock64() - t0 > budget) return false;
    if (abort_word && *(volatile const int *)abort_word) return false;
  }
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y,
                                            int z, unsigned long long *m) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(m))
      : "memory");
}

// Five consecutive raw window elements p[0..4] as floats; p is 16-byte aligned
// for 32-bit elements and 8-byte aligned for 16-bit ones.
__device__ __forceinline__ float bits16_to_f(unsigned b, const __half *) {
  return __half2float(__ushort_as_half((unsigned short)b));
}
__device__ __forceinline__ float bits16_to_f(unsigned b, const __nv_bfloat16 *) {
  return __bfloat162float(__ushort_as_bfloat16((unsigned short)b));
}
template <typename IT>
__device__ __forceinline__ void load5(const IT *p, float (&v)[5]) {
  if constexpr (std::is_same<IT, float>::value) {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
  } else {
    const uint2 a = *reinterpret_cast<const uint2 *>(p);
    v[0] = bits16_to_f(a.x & 0xFFFFu, p);
    v[1] = bits16_to_f(a.x >> 16, p);
    v[2] = bits16_to_f(a.y & 0xFFFFu, p);
    v[3] = bits16_to_f(a.y >> 16, p);
  }
  v[4] = to_f(p[4]);
}

// Writes the four table entries (b - s, s), s = n - b, of a group from the
// values b_m = p[m], n_m = p[m+1] (32-byte aligned destination).
__device__ __forceinline__ void store_group(float2 *dst, const float (&p)[5]) {
  float e[8];
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const float sl = p[m + 1] - p[m];
    e[2 * m] = p[m] - sl;
    e[2 * m + 1] = sl;
  }
  float4 *d = reinterpret_cast<float4 *>(dst);
  d[0] = make_float4(e[0], e[1], e[2], e[3]);
  d[1] = make_float4(e[4], e[5], e[6], e[7]);
}

// One volume tile (bx, by, bz) of a TMA-staged back-projection.  dsm is the
// CTA's dynamic shared memory laid out by the launcher, mbar its two
// initialised mbarriers, and uses[b] the completed phases of mbarrier b so far
// (a persistent CTA runs many tiles on the same mbarriers).  Returns false
// when a bounded wait ran out (err words set; the tile's voxels untouched).
//
// The tables are staged in groups of four entries per thread: a tilt's window
// starts at the raw window's first column (the tile's lowest reachable column
// rounded down to the 16-byte TMA granularity), so a group's five image values
// come from one aligned vector read and one scalar read of the raw window.
// Groups touching the image border in normalised mode take the per-entry
// clamping path; both paths give the same entries as per-entry staging.
template <int MODE, bool SEP, typename IT>
__device__ __forceinline__ bool bp_tma_tile(const BpArgs &a, const CUtensorMap *tmap, int bx,
                                            int by, int bz, unsigned char *dsm,
                                            unsigned long long *mbar, unsigned (&uses)[2]) {
  constexpr bool KAHAN = !std::is_same<IT, float>::value;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wy = (tid >> 5) % kTY;
  const int wz = (tid >> 5) / kTY;
  const int xc = bx * kTX, yc = by * kTY, zl = bz * kTZ;
  const int zc = zl + a.v.zoff;
  const int fw = a.fw, fh = SEP ? kTY : a.fh;
  const int pnx = a.img.nx, pny = a.img.ny;
  const int bw = a.tma_bw, bh = a.tma_bh, rs = a.tma_raw_stride;  // elements
  const int nt = a.nt, chunk = a.chunk, per = fh * fw;

  TileTilt *tt = reinterpret_cast<TileTilt *>(dsm);
  SepW(*sw)[kTY] = reinterpret_cast<SepW(*)[kTY]>(dsm + (size_t)nt * sizeof(TileTilt));
  IT *raw0 = reinterpret_cast<IT *>(dsm + a.tma_raw_offset);
  float *tblf = reinterpret_cast<float *>(raw0 + 2 * (size_t)chunk * rs);  // float2 entries
  WarpStarts *ws = reinterpret_cast<WarpStarts *>(tblf + 2 * (size_t)chunk * per);
  constexpr int kXAlign = 16 / (int)sizeof(IT);  // TMA x coordinates: 16-byte multiples
  float2 *tbl2 = reinterpret_cast<float2 *>(tblf);

  for (int i = tid; i < nt; i += kThreads) {
    tile_setup(a.geo[a.t0 + i], xc, yc, zc, a.ox, a.oy, a.oz, pny, SEP, kTX - 1, kTY - 1,
               kTZ - 1, tt[i], sw[i]);
    if (SEP) {  // raw rows start at the lowest detector row of the tile
      int y0 = sw[i][0].y0;
      for (int r = 1; r < kTY; ++r) y0 = min(y0, sw[i][r].y0);
      tt[i].jmin = y0;
    }
    // Table column 0 = raw column 0 = the aligned TMA x coordinate.
    const int xs = tt[i].kmin & ~(kXAlign - 1), o = tt[i].kmin - xs;
    tt[i].U0 += (long long)o << 32;
    tt[i].nq += o;
    tt[i].kmin = xs;
  }
  __syncthreads();

  const int nchunks = (nt + chunk - 1) / chunk;
  auto issue = [&](int c, int buf) {
    const int c0 = c * chunk, nc = min(chunk, nt - c0);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&mbar[buf], (unsigned)(nc * bw * bh * (int)sizeof(IT)));
    IT *dst = raw0 + (size_t)buf * chunk * rs;
    for (int i = 0; i < nc; ++i)
      tma_load_3d(dst + (size_t)i * rs, tmap, tt[c0 + i].kmin, tt[c0 + i].jmin, a.t0 + c0 + i,
                  &mbar[buf]);
  };
  if (tid == 0) {
    issue(0, 0);
    if (nchunks > 1) issue(1, 1);
  }

  float acc[kNV], cmp[kNV];
#pragma unroll
  for (int k = 0; k < kNV; ++k) acc[k] = cmp[k] = 0.f;

  for (int c = 0; c < nchunks; ++c) {
    const int buf = c & 1, c0 = c * chunk, nc = min(chunk, nt - c0);
    // ~1 s budget for a copy; a CTA that gives up raises the launch-wide
    // abort word (err[0]) and the sticky report word (err[1]) so that the
    // other CTAs stop waiting too.
    const unsigned par = (uses[buf] + (unsigned)(c >> 1)) & 1u;
    const bool ok = mbar_wait_bounded(&mbar[buf], par, 1ll << 31, a.err);
    if (__syncthreads_or(!ok)) {
      // Report, give the copies this CTA still has in flight a bounded
      // chance to land, and leave the volume untouched.
      if (tid == 0) {
        atomicExch(a.err, 1);
        atomicExch(a.err + 1, 1);
      }
      mbar_wait_bounded(&mbar[buf], par, 1ll << 28, nullptr);
      if (c + 1 < nchunks)
        mbar_wait_bounded(&mbar[buf ^ 1], (uses[buf ^ 1] + (unsigned)((c + 1) >> 1)) & 1u,
                          1ll << 28, nullptr);
      return false;
    }
    fill_warp_starts(ws, tt + c0, a.geo + a.t0 + c0, nc, tid);
    const IT *R0 = raw0 + (size_t)buf * chunk * rs;
    const int ng = fw >> 2;  // four-entry groups per table row
    if constexpr (SEP) {
      EntryWalk w(tid, fh, ng);
      for (int g = tid; g < nc * fh * ng; g += kThreads, w.next(fh, ng)) {
        const int i = w.i, r = w.r, q = w.q << 2;  // q: the group's first column
        const TileTilt &t = tt[c0 + i];
        if (r >= t.nr || q >= t.nq) continue;
        const IT *R = R0 + (size_t)i * rs;  // raw column = table column
        const float sc = a.img.scale ? a.img.scale[a.t0 + c0 + i] : 1.f;
        const int xs = t.kmin, ys = t.jmin;
        const int x0 = xs + q;  // image column of the group's first entry
        float p[5];
        const SepW s = sw[c0 + i][r];
        const IT *r0 = R + (s.y0 - ys) * bw, *r1 = r0 + bw;
        const float w0 = s.w0 * sc, w1 = s.w1 * sc;
        if (MODE != BP_NORM) {
          float p0[5], p1[5];
          load5(r0 + q, p0);
          load5(r1 + q, p1);
#pragma unroll
          for (int m = 0; m < 5; ++m) p[m] = w0 * p0[m] + w1 * p1[m];
          store_group(tbl2 + (size_t)g * 4, p);
        } else if ((s.w0 + s.w1) != 0.f && x0 >= 0 && x0 + 4 <= pnx - 1) {
          const float c = s.w0 + s.w1;
          float p0[5], p1[5];
          load5(r0 + q, p0);
          load5(r1 + q, p1);
#pragma unroll
          for (int m = 0; m < 5; ++m)
            p[m] = (w0 * (s.w0 != 0.f ? p0[m] : 0.f) + w1 * (s.w1 != 0.f ? p1[m] : 0.f)) / c;
          store_group(tbl2 + (size_t)g * 4, p);
        } else {  // border: per entry, clamped; zero outside the valid range
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int x = x0 + m;
            float b = 0.f, n = 0.f;
            if ((s.w0 + s.w1) != 0.f && x >= -1 && x <= pnx - 1) {
              const int kb = clampi(x, 0, pnx - 1) - xs, kn = clampi(x + 1, 0, pnx - 1) - xs;
              const float c = s.w0 + s.w1;
              b = (w0 * (s.w0 != 0.f ? to_f(r0[kb]) : 0.f) +
                   w1 * (s.w1 != 0.f ? to_f(r1[kb]) : 0.f)) / c;
              n = (w0 * (s.w0 != 0.f ? to_f(r0[kn]) : 0.f) +
                   w1 * (s.w1 != 0.f ? to_f(r1[kn]) : 0.f)) / c;
            }
            const float sl = n - b;
            tbl2[(size_t)g * 4 + m] = make_float2(b - sl, sl);
          }
        }
      }
    } else {
      // One four-entry group: tilt i of the chunk, table row r, first column q,
      // group index g in the chunk's tables.
      auto stage = [&](int i, int r, int q, int g) {
        const IT *R = R0 + (size_t)i * rs;  // raw column = table column
        float p[5];
        if (MODE != BP_NORM) load5(R + r * bw + q, p);  // in the raw box for any r < fh
        const TileTilt &t = tt[c0 + i];
        if (r >= t.nr || q >= t.nq) return;
        const float sc = a.img.scale ? a.img.scale[a.t0 + c0 + i] : 1.f;
        const int xs = t.kmin, ys = t.jmin;
        const int x0 = xs + q;  // image column of the group's first entry
        const int j = ys + r;
        if (MODE != BP_NORM || (x0 >= 0 && x0 + 4 <= pnx - 1 && j >= 0 && j <= pny - 1)) {
          if (MODE == BP_NORM) load5(R + r * bw + q, p);
#pragma unroll
          for (int m = 0; m < 5; ++m) p[m] *= sc;
          store_group(tbl2 + (size_t)g * 4, p);
        } else {  // border: per entry, clamped; zero outside the valid range
          const IT *row = R + (clampi(j, 0, pny - 1) - ys) * bw - xs;
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int x = x0 + m;
            float b = 0.f, n = 0.f;
            if (x >= -1 && x <= pnx - 1 && j >= -1 && j <= pny) {
              b = to_f(row[clampi(x, 0, pnx - 1)]) * sc;
              n = to_f(row[clampi(x + 1, 0, pnx - 1)]) * sc;
            }
            const float sl = n - b;
            tbl2[(size_t)g * 4 + m] = make_float2(b - sl, sl);
          }
        }
      };
      // Each thread keeps one (row, group) position and stages it for the
      // chunk's tilts, W tilts side by side when a table has fewer groups
      // than the CTA has threads: the tilts' reads are independent.
      const int P = fh * ng;  // groups per tilt
      const int W = max(1, kThreads / P);
      const int way = tid / P;
      for (int pos = tid - way * P; way < W && pos < P; pos += kThreads) {
        const int r = pos / ng, q = (pos - r * ng) << 2;
#pragma unroll 2
        for (int i = way; i < nc; i += W) stage(i, r, q, i * P + pos);
      }
    }
    __syncthreads();
    if (tid == 0 && c + 2 < nchunks) issue(c + 2, buf);
    bp_accumulate<MODE, SEP, KAHAN>(acc, cmp, tblf, ws, nc, per, fw, pny, lane, wy, wz);
    // No barrier here: the next chunk's tables and warp starts are written
    // only after the CTA-wide __syncthreads_or that follows its copy wait.
  }
  uses[0] += (unsigned)(nchunks + 1) / 2;
  uses[1] += (unsigned)nchunks / 2;
  bp_epilogue<MODE, SEP>(a, acc, xc + lane, yc + wy, zl + wz * kNV, bp_tile_slot(a, bx, by, bz));
  return true;
}

__device__ __forceinline__ void mbar_init_pair(unsigned long long *mbar) {
  if (threadIdx.x == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// 16-bit images: three CTAs per SM (80 registers) hold the compensated sums
// without spilling (FP16-storage SIRT iteration on cfg1: 31.7 -> 30.5 ms);
// FP32 images: four.
template <int MODE, bool SEP, typename IT>
__global__ void __launch_bounds__(kThreads, std::is_same<IT, float>::value ? 4 : 3)
    bp_tma_kernel(const BpArgs a, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long mbar[2];
  mbar_init_pair(mbar);
  unsigned uses[2] = {0u, 0u};
  bp_tma_tile<MODE, SEP, IT>(a, &tmap, blockIdx.x, blockIdx.y, blockIdx.z, dsm, mbar, uses);
}

// Forward projection: voxel splat (Reproject, main/main-mpi.cpp:286-344) of
// one tile into per-tilt shared-memory windows, then one global atomic add per
// touched in-image detector pixel.  v.vol == nullptr splats ones (the
// per-pixel weight sums, reproj_wt).
//
// Each lane owns the voxel pair (x, x+1) with x = xc + 2*lane and splats
// the two voxels in turn: lanes of one atomic instruction are then two voxels
// apart along x and land on distinct detector columns whenever |a1| >= 0.5.
//
// The windows accumulate in 32-bit fixed point with native shared-memory
// integer atomics (fire-and-forget; float atomics on shared memory are a
// compare-and-swap loop whose round trips left the kernel latency-bound).  The
// tile's values are scaled by a power of two S chosen from the tile's largest
// |voxel| so that no window entry can overflow: an entry collects at most
// `nbound` voxel contributions (host bound: the lattice points of the entry's
// 2 x 2 detector footprint in each section of the tile) of magnitude at
// most max|v|, and S <= 2^30 / (nbound max|v|); also S <= 2^21 / max|v| so
// every scaled contribution stays within the exact range of the float-shift
// rounding (|x| < 2^22).  Per voxel and window row, the row's scaled value y
// and its upper-column part t are each rounded to the nearest integer; the
// upper tap adds round(t) and the lower round(y) - round(t), so a tap is off
// by at most one quantum of max(nbound 2^-30, 2^-21) max|v| (nbound <= 512
// for tilts within +-60 degrees and small in-plane rotations: ~5e-7 of the
// tile's largest |v|) and a row's two taps by half a quantum together; the
// sums are exact and independent of atomic order.  The arithmetic of a
// lane's two voxels runs side by side in f32x2 instructions.
// The flush converts back (x 1/S) and adds the in-image pixels to the global
// float accumulators.
// Adds four floats to four consecutive global floats (16-byte aligned).
__device__ __forceinline__ void red_add_v4(float *p, float x, float y, float z, float w) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(__cvta_generic_to_global(p)),
               "f"(x), "f"(y), "f"(z), "f"(w)
               : "memory");
}

// Launch-wide fixed-point scale of the deterministic flush: the largest power
// of two S with S * gbound * max|v| <= 2^62, so no pixel's int64 sum can
// overflow (each voxel adds at most |v| to a pixel in total); 0 when the view
// is all zero.
__device__ __forceinline__ double fp_gscale(const unsigned *gmax, double gbound) {
  const float vmax = gmax ? __uint_as_float(*gmax) : 1.f;
  if (!(vmax > 0.f)) return 0.0;
  int e;
  frexp(4.611686018427387904e18 / (gbound * (double)vmax), &e);
  return ldexp(1.0, e - 1);
}

// A forward-projection CTA's shared bookkeeping.  Declared once per kernel and
// passed in, so that a kernel instantiating both fp_tile forms holds one copy.
struct FpShared {
  TileTilt tt[kMaxChunk];
  SepW sw[kMaxChunk][kTY];
  FpStarts fs[kMaxChunk];
  unsigned wmax[kThreads / 32];
  float scale, inv;
  int nonzero;
};

template <bool SEP, bool DET = false>
__device__ __forceinline__ void fp_tile(const FpArgs &a, int bx, int by, int bz,
                                        float *accs, FpShared &sh) {
  TileTilt *const tt = sh.tt;
  SepW(*const sw)[kTY] = sh.sw;
  FpStarts *const fs = sh.fs;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  // 16-byte pixel groups of the stack: rows and tilt planes of whole groups.
  const bool vec_ok = ((a.pnx | (int)a.tstride) & 3) == 0 &&
                      (reinterpret_cast<uintptr_t>(a.val) & 15) == 0;
  const int wy = (tid >> 5) % kTY;
  const int wz = (tid >> 5) / kTY;
  const int xc = bx * kFX, yc = by * kTY, zl = bz * kFTZ;
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
  unsigned *const wmax = sh.wmax;
  float &s_scale = sh.scale, &s_inv = sh.inv;
  int &s_nonzero = sh.nonzero;
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
      float lim = vmax > 0.f ? fminf(1073741824.0f / (a.nbound * vmax), 2097152.0f / vmax)
                             : 1.f;
      int ex;
      frexpf(lim, &ex);  // lim = m 2^ex, m in [0.5, 1): 2^(ex-1) <= lim
      s_scale = ldexpf(1.f, ex - 1);
      s_inv = ldexpf(1.f, 1 - ex);
      s_nonzero = vmax > 0.f;
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
  const bool s_scale_nonzero = s_nonzero != 0;  // an all-zero tile adds nothing
  // DET: the deterministic int64 flush (a.ival), a separate instantiation so
  // that the default flush carries none of it.
  const double gS = DET ? fp_gscale(a.gmax, a.gbound) : 0.0;

  for (int c0 = 0; c0 < a.nt; c0 += a.chunk) {
    const int nc = min(a.chunk, a.nt - c0);
    if (tid < nc) {
      const TiltGeo &g = a.geo[a.t0 + c0 + tid];
      tile_setup(g, xc, yc, zc, a.ox, a.oy, a.oz, a.pny, SEP, kFX - 1, kTY - 1, kFTZ - 1,
                 tt[tid], sw[tid]);
      // Window column 0 on a 4-column boundary (the flush adds 4-pixel groups).
      const int xs = tt[tid].kmin & ~3, o = tt[tid].kmin - xs;
      tt[tid].U0 += (long long)o << 32;
      tt[tid].nq += o;
      tt[tid].kmin = xs;
      FpStarts &st = fs[tid];
      st.A0 = g.A[0];
      st.A2 = g.A[2];
      st.B0 = g.B[0];
      st.B2 = g.B[2];
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) {
        const int ry = w % kTY, rz = w / kTY;
        st.Wu[w] = tt[tid].U0 + ry * g.A[1] + (long long)(rz * kFNV) * g.A[2];
        st.Wv[w] = tt[tid].V0 + ry * g.B[1] + (long long)(rz * kFNV) * g.B[2];
      }
    }
    for (int e = tid; e < nc * per; e += kThreads) iacc[e] = 0;
    __syncthreads();

    for (int i = 0; i < nc && s_scale_nonzero; ++i) {
      const FpStarts &st = fs[i];
      const long long A0 = st.A0, A2 = st.A2;
      // Lane coordinates of the pair's voxels: A at x = xc + 2 lane, B at x+1.
      unsigned long long UA = (unsigned long long)(st.Wu[warp] + (2 * lane) * A0);
      unsigned long long UB = UA + (unsigned long long)A0;
      if (SEP) {
        int *T = iacc + (size_t)(i * kTY + wy) * fw;
        const f32x2 one2 = pack2(1.f, 1.f), shift2 = pack2(12582912.0f, 12582912.0f);
#pragma unroll
        for (int k = 0; k < kFNV; ++k) {
          // The pair's voxels side by side in f32x2 arithmetic: t = v dx and
          // v rounded once each (float shift); the lower column gets
          // round(v) - round(t), the upper round(t).  The pair's lanes are two
          // x apart, so one instruction's lanes hit distinct columns.
          const f32x2 v2 = pack2(va[k], vb[k]);
          const f32x2 fx = sub2(pack2(one_plus_frac(UA), one_plus_frac(UB)), one2);
          float rva, rvb, rta, rtb;
          unpack2(add2(v2, shift2), rva, rvb);
          unpack2(add2(mul2(fx, v2), shift2), rta, rtb);
          const int ta = __float_as_int(rta), tb = __float_as_int(rtb);
          int *ea = T + (int)(UA >> 32), *eb = T + (int)(UB >> 32);
          atomicAdd(ea, __float_as_int(rva) - ta);
          atomicAdd(ea + 1, ta - kFshiftBias);
          atomicAdd(eb, __float_as_int(rvb) - tb);
          atomicAdd(eb + 1, tb - kFshiftBias);
          UA += (unsigned long long)A2;
          UB += (unsigned long long)A2;
        }
      } else {
        const long long B0 = st.B0, B2 = st.B2;
        unsigned long long VA = (unsigned long long)(st.Wv[warp] + (2 * lane) * B0);
        unsigned long long VB = VA + (unsigned long long)B0;
        int *T = iacc + (size_t)i * per;
        const f32x2 one2 = pack2(1.f, 1.f), two2 = pack2(2.f, 2.f);
        const f32x2 shift2 = pack2(12582912.0f, 12582912.0f);
#pragma unroll
        for (int k = 0; k < kFNV; ++k) {
          // The pair's voxels side by side in f32x2 arithmetic.  Rows:
          // y0 = v (1 - dy) with 1 - dy = 2 - (1 + dy) exact, y1 = v - y0.
          // Each row's pair of taps: the row's value y and its upper-column
          // part t = y dx are rounded once each (float shift), the lower
          // column gets round(y) - round(t), so the two taps add up to
          // round(y) exactly.
          const f32x2 v2 = pack2(va[k], vb[k]);
          const f32x2 y0 = mul2(sub2(two2, pack2(one_plus_frac(VA), one_plus_frac(VB))), v2);
          const f32x2 y1 = sub2(v2, y0);
          const f32x2 fx = sub2(pack2(one_plus_frac(UA), one_plus_frac(UB)), one2);
          float r0a, r0b, r01a, r01b, r1a, r1b, r11a, r11b;
          unpack2(add2(y0, shift2), r0a, r0b);
          unpack2(add2(mul2(fx, y0), shift2), r01a, r01b);
          unpack2(add2(y1, shift2), r1a, r1b);
          unpack2(add2(mul2(fx, y1), shift2), r11a, r11b);
          {
            const int r0 = __float_as_int(r0a), r01 = __float_as_int(r01a);
            const int r1 = __float_as_int(r1a), r11 = __float_as_int(r11a);
            int *e = T + (int)(VA >> 32) * fw + (int)(UA >> 32);
            atomicAdd(e, r0 - r01);
            atomicAdd(e + 1, r01 - kFshiftBias);
            atomicAdd(e + fw, r1 - r11);
            atomicAdd(e + fw + 1, r11 - kFshiftBias);
          }
          {
            const int r0 = __float_as_int(r0b), r01 = __float_as_int(r01b);
            const int r1 = __float_as_int(r1b), r11 = __float_as_int(r11b);
            int *e = T + (int)(VB >> 32) * fw + (int)(UB >> 32);
            atomicAdd(e, r0 - r01);
            atomicAdd(e + 1, r01 - kFshiftBias);
            atomicAdd(e + fw, r1 - r11);
            atomicAdd(e + fw + 1, r11 - kFshiftBias);
          }
          UA += (unsigned long long)A2;
          UB += (unsigned long long)A2;
          VA += (unsigned long long)B2;
          VB += (unsigned long long)B2;
        }
      }
    }
    __syncthreads();

    // Flush the windows: in-image pixels only, as the reference's splat.
    // Four columns per thread: a group inside the image goes out as one
    // 16-byte vector reduction when the stack's rows are 16-byte aligned;
    // border groups add their in-image pixels one by one.
    for (int i = 0; i < nc; ++i) {
      const int kmin = tt[i].kmin, nq = tt[i].nq, nr = tt[i].nr;
      const int *T = iacc + (size_t)i * per;
      float *base = a.val + (size_t)(a.t0 + c0 + i) * a.tstride;
      unsigned long long *ibase =
          DET ? a.ival + (size_t)(a.t0 + c0 + i) * a.tstride : nullptr;
      const float inv = s_inv;
      // Splat writes stay below column fw (the host's window width covers
      // the tile's reach); nq comes from this tile's FP64 extremes, which
      // rounding can put one column wider, so the flush stops at fw too.
      const int ngq = (min(nq, fw) + 3) >> 2;
      for (int e = tid; e < nr * ngq; e += kThreads) {
        const int r = e / ngq, q = (e - r * ngq) << 2;
        const int4 v = *reinterpret_cast<const int4 *>(T + r * fw + q);
        const float s[4] = {(float)v.x * inv, (float)v.y * inv, (float)v.z * inv,
                            (float)v.w * inv};
        if (s[0] == 0.f && s[1] == 0.f && s[2] == 0.f && s[3] == 0.f) continue;
        const int k = kmin + q;
        const bool inside = vec_ok && k >= 0 && k + 3 < a.pnx;
        auto add_row = [&](int j, float wgt) {
          if ((unsigned)j >= (unsigned)a.pny) return;
          if (DET) {  // deterministic: int64 adds at the launch-wide scale
            unsigned long long *ip = ibase + (size_t)j * a.pnx + k;
#pragma unroll
            for (int m = 0; m < 4; ++m)
              if (s[m] != 0.f && (unsigned)(k + m) < (unsigned)a.pnx)
                atomicAdd(ip + m,
                          (unsigned long long)__double2ll_rn((double)(s[m] * wgt) * gS));
            return;
          }
          float *p = base + (size_t)j * a.pnx + k;
          if (inside && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
            red_add_v4(p, s[0] * wgt, s[1] * wgt, s[2] * wgt, s[3] * wgt);
          } else {
#pragma unroll
            for (int m = 0; m < 4; ++m)
              if (s[m] != 0.f && (unsigned)(k + m) < (unsigned)a.pnx) atomicAdd(p + m, s[m] * wgt);
          }
        };
        if (SEP) {
          const SepW w = sw[i][r];
          add_row(w.y0, 1 - w.dy);
          if (w.dy != 0.f) add_row(w.y0 + 1, w.dy);
        } else {
          add_row(tt[i].jmin + r, 1.f);
        }
      }
    }

    __syncthreads();
  }
}

template <bool SEP, bool DET>
__global__ void __launch_bounds__(kThreads, SEP || DET ? 3 : 4) fp_kernel(const FpArgs a) {
  extern __shared__ __align__(16) float accs[];
  __shared__ FpShared sh;
  fp_tile<SEP, DET>(a, blockIdx.x, blockIdx.y, blockIdx.z, accs, sh);
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

// ------------------------------------------------------ 16-bit storage
//
// Measured projections and SIRT residuals may be stored as FP16 or BF16 to
// halve the bytes staged per tilt.  A stored element e of tilt t stands for
// e * scale[t]; the scales are powers of two, so scaling is exact and the
// only rounding is the 16-bit conversion itself.

template <typename T>
__device__ __forceinline__ T from_f(float x);
template <>
__device__ __forceinline__ float from_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) {
  return __float2bfloat16_rn(x);
}

// 2^e as a float for |e| < 127.
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }

// Per-tilt maximum of |p| as float bits (non-negative floats order like their
// bit patterns).  grid.y = tilt.
__global__ void absmax_kernel(const float *__restrict__ p, size_t plane,
                              unsigned *__restrict__ maxbits) {
  const float *pt = p + plane * blockIdx.y;
  float m = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v = fabsf(pt[i]);
    m = v > m ? v : m;  // NaN never replaces m
  }
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(maxbits + blockIdx.y, __float_as_uint(m));
}

// Exponent e of the power-of-two scale of a tilt whose largest magnitude has
// float bits mb: FP16 places the maximum in (2^13, 2^14], a factor of four
// below the format's largest finite value, so residuals up to four times the
// measured range stay finite; BF16 has float's range and keeps scale 1.
template <typename T>
__device__ __forceinline__ int scale_exp(unsigned mb) {
  if (!std::is_same<T, __half>::value || mb == 0u || mb >= 0x7f800000u) return 0;
  const int E = (int)(mb >> 23) - 127;  // m = 1.f * 2^E, f the fraction bits
  const int ceil_log2 = (mb & 0x7fffffu) ? E + 1 : E;
  return max(-126, min(126, ceil_log2 - 14));
}

template <typename T>
__global__ void quantize_kernel(const float *__restrict__ p, size_t plane,
                                const unsigned *__restrict__ maxbits, T *__restrict__ out,
                                float *__restrict__ scale) {
  const int t = blockIdx.y;
  const int e = scale_exp<T>(maxbits[t]);
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[t] = pow2f(e);
  const float inv = pow2f(-e);
  const float *pt = p + plane * t;
  T *ot = out + plane * t;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane;
       i += (size_t)gridDim.x * blockDim.x)
    ot[i] = from_f<T>(pt[i] * inv);
}

// SIRT residual from 16-bit measured projections: r = p*ps[t] - val/wt (val
// where wt == 0), stored as RT in units of rs[t] (rs == nullptr: 1).  With
// RT = float, r may alias val.  grid.y = tilt.
template <typename PT, typename RT>
__global__ void resid_lp_kernel(const PT *__restrict__ p, const float *__restrict__ ps,
                                const float *val, const float *__restrict__ wt, size_t plane,
                                RT *r, const float *__restrict__ rs) {
  const size_t off = plane * blockIdx.y;
  const float sp = ps ? ps[blockIdx.y] : 1.f;
  const float inv = rs ? 1.f / rs[blockIdx.y] : 1.f;  // exact: rs is a power of two
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane;
       i += (size_t)gridDim.x * blockDim.x) {
    float v = val[off + i];
    const float w = wt[off + i];
    if (w != 0.f) v /= w;
    r[off + i] = from_f<RT>((to_f(p[off + i]) * sp - v) * inv);
  }
}

// Self-test of the bounded device wait: one CTA waits on an mbarrier that
// nothing arrives at, with the budget given; the wait must give up and the
// CTA report through err[1], as a back-projection whose copies never land.
__global__ void bounded_wait_selftest_kernel(long long budget, int *err) {
  __shared__ __align__(8) unsigned long long m;
  if (threadIdx.x == 0) {
    mbar_init(&m, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(&m, 0u, budget, nullptr);
  if (!__syncthreads_or(ok) && threadIdx.x == 0) atomicExch(err + 1, 1);
}

cudaError_t launch_bounded_wait_selftest(long long budget, int *err, cudaStream_t s) {
  bounded_wait_selftest_kernel<<<1, 32, 0, s>>>(budget, err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- batches
//
// One batch step: zero the accumulators of the step's forward projections
// (and reset the work counters), forward-project every item, form every
// residual, back-project every item.  The forward and back-projection kernels
// are persistent: each CTA takes the next tile of any item from the table's
// counter until all are done, so small and large tilt series share the waves.

template <typename Item>
__device__ __forceinline__ int find_item(const Item *items, int n, long long t) {
  int lo = 0, hi = n - 1;  // last item whose first tile <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].first <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void zero_batch_kernel(BatchTable *T) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    T->h.bp_next = 0ull;
    T->h.fp_next = 0ull;
    if (T->h.err) T->h.err[0] = 0;
  }
  const int n = T->h.nzero;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int j = 0; j < n; ++j) {
    float *p = T->zero[j].p;
    const size_t cnt = T->zero[j].n;
    const size_t n4 = (reinterpret_cast<uintptr_t>(p) & 15) ? 0 : cnt / 4;
    float4 *p4 = reinterpret_cast<float4 *>(p);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += stride)
      p4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (size_t i = 4 * n4 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cnt; i += stride)
      p[i] = 0.f;
  }
}

__device__ __forceinline__ float load_elem(const void *p, int dtype, size_t i) {
  if (dtype == IMG_F16) return __half2float(reinterpret_cast<const __half *>(p)[i]);
  if (dtype == IMG_BF16) return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(p)[i]);
  return reinterpret_cast<const float *>(p)[i];
}

__device__ __forceinline__ void store_elem(void *p, int dtype, size_t i, float v) {
  if (dtype == IMG_F16) reinterpret_cast<__half *>(p)[i] = __float2half_rn(v);
  else if (dtype == IMG_BF16) reinterpret_cast<__nv_bfloat16 *>(p)[i] = __float2bfloat16_rn(v);
  else reinterpret_cast<float *>(p)[i] = v;
}

__global__ void resid_batch_kernel(const BatchTable *T) {
  const int n = T->h.nres;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int j = 0; j < n; ++j) {
    const BatchRes &R = T->res[j];
    for (int t = 0; t < R.nt; ++t) {
      const float sp = R.ps ? R.ps[t] : 1.f;
      const float inv = R.rs ? 1.f / R.rs[t] : 1.f;  // exact: powers of two
      const size_t off = R.plane * t;
      for (size_t i = off + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < off + R.plane;
           i += stride) {
        float v = R.val[i];
        const float w = R.wt[i];
        if (w != 0.f) v /= w;
        store_elem(R.r, R.rdtype, i, (load_elem(R.p, R.pdtype, i) * sp - v) * inv);
      }
    }
  }
}

// FP16 residual items: per-tilt maxima of the FP32 residual, then the
// conversion with power-of-two scales (as tr_quantize).
__global__ void absmax_batch_kernel(const BatchTable *T) {
  const int n = T->h.nres;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int j = 0; j < n; ++j) {
    const BatchRes &R = T->res[j];
    if (!R.q) continue;
    const float *v = reinterpret_cast<const float *>(R.r);
    for (int t = 0; t < R.nt; ++t) {
      const size_t off = R.plane * t;
      float m = 0.f;
      for (size_t i = off + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < off + R.plane;
           i += stride) {
        const float a = fabsf(v[i]);
        m = a > m ? a : m;
      }
      for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(R.qmax + t, __float_as_uint(m));
    }
  }
}

__global__ void quantize_batch_kernel(const BatchTable *T) {
  const int n = T->h.nres;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int j = 0; j < n; ++j) {
    const BatchRes &R = T->res[j];
    if (!R.q) continue;
    const float *v = reinterpret_cast<const float *>(R.r);
    for (int t = 0; t < R.nt; ++t) {
      const int e = scale_exp<__half>(R.qmax[t]);
      if (blockIdx.x == 0 && threadIdx.x == 0) R.qscale[t] = pow2f(e);
      const float inv = pow2f(-e);
      const size_t off = R.plane * t;
      for (size_t i = off + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < off + R.plane;
           i += stride)
        R.q[i] = __float2half_rn(v[i] * inv);
    }
  }
}

__global__ void __launch_bounds__(kThreads, 4) fp_batch_kernel(BatchTable *T) {
  extern __shared__ __align__(16) float accs[];
  __shared__ long long s_tile;
  __shared__ int s_item;
  __shared__ FpShared sh;
  const long long total = T->h.fp_tiles;
  const int n = T->h.nfp;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long t = (long long)atomicAdd(&T->h.fp_next, 1ull);
      s_tile = t;
      s_item = t < total ? find_item(T->fp, n, t) : -1;
    }
    __syncthreads();
    const long long t = s_tile;
    if (t >= total) break;
    const BatchFp &it = T->fp[s_item];
    long long l = t - it.first;
    const int bx = (int)(l % it.gx);
    l /= it.gx;
    const int by = (int)(l % it.gy), bz = (int)(l / it.gy);
    if (it.sep) fp_tile<true>(it.a, bx, by, bz, accs, sh);
    else fp_tile<false>(it.a, bx, by, bz, accs, sh);
  }
}

// Back-projection items: BP_NORM over FP32 images (filtered projections) and
// BP_SIRT over residuals of type RT.
template <typename RT>
__global__ void __launch_bounds__(kThreads, std::is_same<RT, float>::value ? 4 : 3)
    bp_batch_kernel(BatchTable *T) {
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ long long s_tile;
  __shared__ int s_item;
  mbar_init_pair(mbar);
  unsigned uses[2] = {0u, 0u};
  const long long total = T->h.bp_tiles;
  const int n = T->h.nbp;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long t = (long long)atomicAdd(&T->h.bp_next, 1ull);
      s_tile = t;
      s_item = t < total ? find_item(T->bp, n, t) : -1;
    }
    __syncthreads();
    const long long t = s_tile;
    if (t >= total) break;
    const BatchBp &it = T->bp[s_item];
    long long l = t - it.first;
    const int bx = (int)(l % it.gx);
    l /= it.gx;
    const int by = (int)(l % it.gy), bz = (int)(l / it.gy);
    bool ok;
    if (it.mode == BP_NORM)
      ok = it.sep ? bp_tma_tile<BP_NORM, true, float>(it.a, &it.map, bx, by, bz, dsm, mbar, uses)
                  : bp_tma_tile<BP_NORM, false, float>(it.a, &it.map, bx, by, bz, dsm, mbar, uses);
    else
      ok = it.sep ? bp_tma_tile<BP_SIRT, true, RT>(it.a, &it.map, bx, by, bz, dsm, mbar, uses)
                  : bp_tma_tile<BP_SIRT, false, RT>(it.a, &it.map, bx, by, bz, dsm, mbar, uses);
    if (!ok) break;
  }
}

// ------------------------------------------------------ compact voxel weights
//
// A back-projection tile is interior when, for every tilt, the detector
// coordinates its voxels can reach keep all four bilinear neighbours inside
// the image (lower neighbour in [0, nx-2] x [0, ny-2], with 1e-3 px of margin
// over the FP64 extremes for the fixed-point coordinates).  Then every
// voxel's per-tilt weight sum c is exactly 1 in the weight pass (general
// geometry: the indicator interpolates to 1.0), so its SIRT weight is the
// tilt count; with separable geometry the weight depends on the voxel row
// only (the row pair's in-image weights w0 + w1), so it is the float sum over
// the tilts, in tilt order, of those -- as the weight pass adds them.

__global__ void classify_tiles_kernel(const TiltGeo *__restrict__ geo, int nt, VolView v,
                                      float ox, float oy, float oz, int pnx, int pny, int sep,
                                      int *slot, int *count) {
  const int gx = (v.nx + kTX - 1) / kTX, gy = (v.ny + kTY - 1) / kTY;
  const int gz = (v.nz + kTZ - 1) / kTZ;
  const long long ntiles = (long long)gx * gy * gz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ntiles;
       t += (long long)gridDim.x * blockDim.x) {
    const int bx = (int)(t % gx), by = (int)((t / gx) % gy), bz = (int)(t / ((long long)gx * gy));
    const int xc = bx * kTX, yc = by * kTY, zc = bz * kTZ + v.zoff;
    const double X = (double)((float)xc - ox), Y = (double)((float)yc - oy),
                 Z = (double)((float)zc - oz);
    const double ex = kTX - 1, ey = kTY - 1, ez = kTZ - 1, m = 1e-3;
    bool interior = true;
    for (int i = 0; i < nt && interior; ++i) {
      const TiltGeo &g = geo[i];
      const double uc = g.a[0] + g.a[1] * X + g.a[2] * Y + g.a[3] * Z + (double)ox;
      const double umin = uc + fmin(0.0, g.a[1] * ex) + fmin(0.0, g.a[2] * ey) +
                          fmin(0.0, g.a[3] * ez);
      const double umax = uc + fmax(0.0, g.a[1] * ex) + fmax(0.0, g.a[2] * ey) +
                          fmax(0.0, g.a[3] * ez);
      interior = floor(umin - m) >= 0.0 && floor(umax + m) <= pnx - 2;
      if (!sep) {
        const double vc = g.b[0] + g.b[1] * X + g.b[2] * Y + g.b[3] * Z + (double)oy;
        const double vmin = vc + fmin(0.0, g.b[1] * ex) + fmin(0.0, g.b[2] * ey) +
                            fmin(0.0, g.b[3] * ez);
        const double vmax = vc + fmax(0.0, g.b[1] * ex) + fmax(0.0, g.b[2] * ey) +
                            fmax(0.0, g.b[3] * ez);
        interior = interior && floor(vmin - m) >= 0.0 && floor(vmax + m) <= pny - 2;
      }
    }
    slot[t] = interior ? -1 : atomicAdd(count, 1);
  }
}

// Separable per-row weights: wrow[y] = sum over tilts (in order, float) of
// w0 + w1 for voxel row y, with the rows and weights tile_setup forms.
__global__ void sep_row_weights_kernel(const TiltGeo *__restrict__ geo, int nt, int ny, float oy,
                                       int pny, float *wrow) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= ny) return;
  float acc = 0.f;
  for (int i = 0; i < nt; ++i) {
    const TiltGeo &g = geo[i];
    const double Yr = (double)((float)y - oy);
    // b1 = b3 = 0 for separable geometry: v = b0 + b2 Yr + oy (tile_setup).
    const double vv = g.b[0] + g.b[2] * Yr + (double)oy;
    const int y0 = (int)floor(vv);
    const float dy = (float)(vv - (double)y0);
    const float w0 = (y0 >= 0 && y0 < pny) ? (1 - dy) : 0.f;
    const float w1 = (y0 + 1 >= 0 && y0 + 1 < pny) ? dy : 0.f;
    acc += w0 + w1;
  }
  wrow[y] = acc;
}

cudaError_t launch_classify_tiles(const TiltGeo *geo, int nt, const VolView &v, float ox, float oy,
                                  float oz, int pnx, int pny, bool sep, int *slot, int *count,
                                  cudaStream_t s) {
  classify_tiles_kernel<<<1184, 128, 0, s>>>(geo, nt, v, ox, oy, oz, pnx, pny, sep ? 1 : 0, slot,
                                              count);
  return cudaGetLastError();
}

cudaError_t launch_sep_row_weights(const TiltGeo *geo, int nt, int ny, float oy, int pny,
                                   float *wrow, cudaStream_t s) {
  sep_row_weights_kernel<<<(ny + 127) / 128, 128, 0, s>>>(geo, nt, ny, oy, pny, wrow);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- launchers

static dim3 tile_grid(const VolView &v) {
  return dim3((v.nx + kTX - 1) / kTX, (v.ny + kTY - 1) / kTY,
              (v.nz + kTZ - 1) / kTZ);
}

template <int MODE, bool SEP, typename IT>
static cudaError_t launch_bp_t(const BpArgs &a, cudaStream_t s) {
  const int fh = SEP ? kTY : a.fh;
  const size_t smem = (size_t)a.chunk * fh * a.fw * sizeof(float2);
  cudaError_t e = cudaFuncSetAttribute(
      bp_kernel<MODE, SEP, IT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)smem);
  if (e != cudaSuccess) return e;
  bp_kernel<MODE, SEP, IT><<<tile_grid(a.v), kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

constexpr size_t kSmemTma = 56 * 1024;

// TMA-staged launch; returns false (nothing launched) when the image or the
// window does not fit the TMA path.
template <typename IT>
constexpr CUtensorMapDataType tma_type() {
  return std::is_same<IT, float>::value   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
         : std::is_same<IT, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                           : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}

// TMA staging layout of a back-projection within `budget` bytes of dynamic
// shared memory: tile bookkeeping, two raw window buffers per staged tilt and
// the interpolation tables.  Fills the tensor map, the chunk and the tma_*
// fields; false when the images or the window do not suit TMA.
template <typename IT>
static bool tma_layout(const BpArgs &a0, bool sep, size_t budget, BpArgs *out,
                       CUtensorMap *map, size_t *smem) {
  const ImgView &im = a0.img;
  constexpr int es = (int)sizeof(IT);
  constexpr int xal = 16 / es;  // TMA x coordinates and box widths: 16-byte multiples
  if (!im.p || !a0.err || (im.nx * es) % 16 != 0 ||
      (reinterpret_cast<uintptr_t>(im.p) & 15) != 0)
    return false;
  const int fh = sep ? kTY : a0.fh;
  // Table rows start at the aligned raw column: up to xal - 1 extra columns,
  // rounded up to whole four-entry groups; the raw window holds one more
  // column for the last group's slopes.
  const int fwt = (a0.fw + xal - 1 + 3) & ~3;
  const int bw = (fwt + 1 + xal - 1) / xal * xal;
  const int bh = sep ? kTY + 3 : fh + 1;
  if (bw > 256 || bh > 256) return false;
  const int rs = ((bw * bh * es + 127) & ~127) / es;  // elements; 128-byte aligned slots
  const size_t fixed =
      ((size_t)a0.nt * (sizeof(TileTilt) + kTY * sizeof(SepW)) + 127) & ~(size_t)127;
  const size_t per_tilt =
      2 * (size_t)rs * es + (size_t)fh * fwt * sizeof(float2) + sizeof(WarpStarts);
  if (fixed + per_tilt > budget + 64 * 1024) return false;
  int chunk = (int)std::max<size_t>(1, (budget > fixed ? budget - fixed : 0) / per_tilt);
  chunk = std::min(chunk, std::min(kMaxChunk, a0.nt));
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)im.nx, (cuuint64_t)im.ny,
                              (cuuint64_t)(a0.t0 + a0.nt)};
  const cuuint64_t strides[2] = {(cuuint64_t)im.nx * es, (cuuint64_t)im.tstride * es};
  const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (enc(map, tma_type<IT>(), 3, const_cast<float *>(im.p), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  *out = a0;
  out->fw = fwt;
  out->chunk = chunk;
  out->tma_bw = bw;
  out->tma_bh = bh;
  out->tma_raw_stride = rs;
  out->tma_raw_offset = (int)fixed;
  *smem = fixed + (size_t)chunk * per_tilt;
  return true;
}

template <int MODE, bool SEP, typename IT>
static bool try_launch_bp_tma(const BpArgs &a0, cudaStream_t s, cudaError_t *err) {
  BpArgs a;
  CUtensorMap map;
  size_t smem = 0;
  if (!tma_layout<IT>(a0, SEP, kSmemTma, &a, &map, &smem)) return false;
  cudaError_t e = cudaFuncSetAttribute(bp_tma_kernel<MODE, SEP, IT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    bp_tma_kernel<MODE, SEP, IT><<<tile_grid(a.v), kThreads, smem, s>>>(a, map);
    e = cudaGetLastError();
  }
  *err = e;
  return true;
}

template <int MODE, bool SEP, typename IT>
static cudaError_t launch_bp_any(const BpArgs &a, cudaStream_t s) {
  if (MODE != BP_WEIGHTS) {
    cudaError_t e;
    if (try_launch_bp_tma<MODE, SEP, IT>(a, s, &e)) return e;
  }
  return launch_bp_t<MODE, SEP, IT>(a, s);
}

template <typename IT>
static cudaError_t launch_bp_it(int mode, bool sep, const BpArgs &a, cudaStream_t s) {
  if (sep) {
    if (mode == BP_NORM) return launch_bp_any<BP_NORM, true, IT>(a, s);
    return launch_bp_any<BP_SIRT, true, IT>(a, s);
  }
  if (mode == BP_NORM) return launch_bp_any<BP_NORM, false, IT>(a, s);
  return launch_bp_any<BP_SIRT, false, IT>(a, s);
}

cudaError_t launch_bp(int mode, bool sep, const BpArgs &a, cudaStream_t s) {
  if (mode == BP_WEIGHTS)
    return sep ? launch_bp_any<BP_WEIGHTS, true, float>(a, s)
               : launch_bp_any<BP_WEIGHTS, false, float>(a, s);
  if (mode == BP_SUM)  // FP32 images only
    return sep ? launch_bp_any<BP_SUM, true, float>(a, s)
               : launch_bp_any<BP_SUM, false, float>(a, s);
  if (a.img.dtype == IMG_F16) return launch_bp_it<__half>(mode, sep, a, s);
  if (a.img.dtype == IMG_BF16) return launch_bp_it<__nv_bfloat16>(mode, sep, a, s);
  return launch_bp_it<float>(mode, sep, a, s);
}

static dim3 fp_grid(const VolView &v) {
  return dim3((v.nx + kFX - 1) / kFX, (v.ny + kTY - 1) / kTY,
              (v.nz + kFTZ - 1) / kFTZ);
}

template <bool SEP, bool DET>
static cudaError_t launch_fp_t(const FpArgs &a, size_t smem, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(fp_kernel<SEP, DET>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fp_kernel<SEP, DET><<<fp_grid(a.v), kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fp(bool sep, const FpArgs &a, cudaStream_t s) {
  const int fh = sep ? kTY : a.fh;
  const size_t smem = (size_t)a.chunk * fh * a.fw * sizeof(float);
  if (a.ival)
    return sep ? launch_fp_t<true, true>(a, smem, s) : launch_fp_t<false, true>(a, smem, s);
  return sep ? launch_fp_t<true, false>(a, smem, s) : launch_fp_t<false, false>(a, smem, s);
}

// Largest |voxel| of a view, as float bits, max-combined into *out (which
// starts at 0).  Walks x fastest, then the view's smaller-stride axis.
__global__ void absmax_view_kernel(const VolView v, unsigned *out) {
  const size_t n = (size_t)v.nx * v.ny * v.nz;
  const bool zy = v.sz < v.sy;  // [y][z][x] (Y layout): z before y
  unsigned m = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % v.nx);
    const size_t r = i / v.nx;
    const int a = zy ? (int)(r % v.nz) : (int)(r % v.ny);
    const int b = zy ? (int)(r / v.nz) : (int)(r / v.ny);
    const int z = zy ? a : b, y = zy ? b : a;
    m = max(m, __float_as_uint(fabsf(v.vol[(size_t)y * v.sy + (size_t)z * v.sz + x])));
  }
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Adds the deterministic flush's int64 sums into val and clears them.
__global__ void ival_to_val_kernel(unsigned long long *ival, float *val, size_t n,
                                   const unsigned *gmax, double gbound) {
  const double S = fp_gscale(gmax, gbound);
  const double inv = S > 0.0 ? 1.0 / S : 0.0;  // S is a power of two
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const long long q = (long long)ival[i];
    if (q) {
      val[i] += (float)((double)q * inv);
      ival[i] = 0ull;
    }
  }
}

cudaError_t launch_fp_deterministic(bool sep, FpArgs a, unsigned long long *ival,
                                    unsigned *gmax, int nsm, cudaStream_t s) {
  a.ival = ival;
  a.gbound = (double)a.v.nx * a.v.ny * a.v.nz;
  a.gmax = nullptr;
  cudaError_t e;
  if (a.v.vol) {
    if ((e = cudaMemsetAsync(gmax, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
    absmax_view_kernel<<<nsm * 4, 256, 0, s>>>(a.v, gmax);
    a.gmax = gmax;
  }
  if ((e = launch_fp(sep, a, s)) != cudaSuccess) return e;
  const size_t n = (size_t)a.nt * a.tstride, off = (size_t)a.t0 * a.tstride;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  ival_to_val_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(ival + off, a.val + off, n, a.gmax,
                                                            a.gbound);
  return cudaGetLastError();
}

cudaError_t launch_resid(const float *p, float *val, const float *wt, size_t n,
                         int nsm, cudaStream_t s) {
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  resid_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(p, val, wt, n);
  return cudaGetLastError();
}

static unsigned plane_blocks(size_t plane, int nt, int nsm) {
  // About 8 resident 256-thread blocks per SM in total across the tilts.
  const size_t want = ((size_t)nsm * 8 + nt - 1) / nt;
  const size_t need = (plane + 255) / 256;
  return (unsigned)std::max<size_t>(1, std::min(want, need));
}

cudaError_t launch_quantize(const float *p, size_t plane, int nt, int dtype, void *out,
                            float *scale, unsigned *maxbits, int nsm, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(maxbits, 0, sizeof(unsigned) * nt, s);
  if (e != cudaSuccess) return e;
  const dim3 grid(plane_blocks(plane, nt, nsm), nt);
  absmax_kernel<<<grid, 256, 0, s>>>(p, plane, maxbits);
  if (dtype == IMG_F16)
    quantize_kernel<__half><<<grid, 256, 0, s>>>(p, plane, maxbits, (__half *)out, scale);
  else
    quantize_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>(p, plane, maxbits,
                                                        (__nv_bfloat16 *)out, scale);
  return cudaGetLastError();
}

template <typename PT>
static void resid_lp_rt(const PT *p, const float *ps, const float *val, const float *wt,
                        size_t plane, int nt, int rdtype, void *r, const float *rs,
                        int nsm, cudaStream_t s) {
  const dim3 grid(plane_blocks(plane, nt, nsm), nt);
  if (rdtype == IMG_F16)
    resid_lp_kernel<PT, __half><<<grid, 256, 0, s>>>(p, ps, val, wt, plane, (__half *)r, rs);
  else if (rdtype == IMG_BF16)
    resid_lp_kernel<PT, __nv_bfloat16><<<grid, 256, 0, s>>>(p, ps, val, wt, plane,
                                                            (__nv_bfloat16 *)r, rs);
  else
    resid_lp_kernel<PT, float><<<grid, 256, 0, s>>>(p, ps, val, wt, plane, (float *)r, rs);
}

cudaError_t launch_resid_lp(const void *p, int pdtype, const float *ps, const float *val,
                            const float *wt, size_t plane, int nt, int rdtype, void *r,
                            const float *rs, int nsm, cudaStream_t s) {
  if (pdtype == IMG_F16)
    resid_lp_rt((const __half *)p, ps, val, wt, plane, nt, rdtype, r, rs, nsm, s);
  else if (pdtype == IMG_BF16)
    resid_lp_rt((const __nv_bfloat16 *)p, ps, val, wt, plane, nt, rdtype, r, rs, nsm, s);
  else
    resid_lp_rt((const float *)p, ps, val, wt, plane, nt, rdtype, r, rs, nsm, s);
  return cudaGetLastError();
}

// ------------------------------------------------------- batch host helpers

dim3 bp_tile_grid(const VolView &v) { return tile_grid(v); }
dim3 fp_tile_grid(const VolView &v) { return fp_grid(v); }

// TMA layout of one back-projection item within `budget` bytes of shared
// memory (image element type by a.img.dtype); false when unsuitable.
bool batch_bp_layout(const BpArgs &a0, bool sep, size_t budget, BatchBp *out, size_t *smem) {
  BpArgs a;
  bool ok;
  if (a0.img.dtype == IMG_F16) ok = tma_layout<__half>(a0, sep, budget, &a, &out->map, smem);
  else if (a0.img.dtype == IMG_BF16)
    ok = tma_layout<__nv_bfloat16>(a0, sep, budget, &a, &out->map, smem);
  else ok = tma_layout<float>(a0, sep, budget, &a, &out->map, smem);
  if (ok) out->a = a;
  return ok;
}

template <typename RT>
static cudaError_t set_bp_batch_smem(size_t smem) {
  return cudaFuncSetAttribute(bp_batch_kernel<RT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
}

// Resident CTAs per SM of the persistent kernels at the given shared memory.
int batch_occupancy(int rdtype, size_t smem_bp, size_t smem_fp, int *fp_per_sm) {
  int nb = 0, nf = 0;
  cudaFuncSetAttribute(fp_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem_fp);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nf, fp_batch_kernel, kThreads, smem_fp);
  if (rdtype == IMG_F16) {
    set_bp_batch_smem<__half>(smem_bp);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bp_batch_kernel<__half>, kThreads, smem_bp);
  } else if (rdtype == IMG_BF16) {
    set_bp_batch_smem<__nv_bfloat16>(smem_bp);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bp_batch_kernel<__nv_bfloat16>, kThreads,
                                                  smem_bp);
  } else {
    set_bp_batch_smem<float>(smem_bp);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bp_batch_kernel<float>, kThreads, smem_bp);
  }
  *fp_per_sm = nf;
  return nb;
}

// The six launches of one step over the table at T (device).  The kernels'
// shared-memory limits are set beforehand by batch_occupancy.
cudaError_t launch_batch_step(BatchTable *T, int rdtype, int grid_fp, int grid_bp,
                              size_t smem_fp, size_t smem_bp, int nsm, cudaStream_t s) {
  zero_batch_kernel<<<nsm * 4, 256, 0, s>>>(T);
  fp_batch_kernel<<<grid_fp, kThreads, smem_fp, s>>>(T);
  resid_batch_kernel<<<nsm * 4, 256, 0, s>>>(T);
  absmax_batch_kernel<<<nsm * 4, 256, 0, s>>>(T);
  quantize_batch_kernel<<<nsm * 4, 256, 0, s>>>(T);
  if (rdtype == IMG_F16)
    bp_batch_kernel<__half><<<grid_bp, kThreads, smem_bp, s>>>(T);
  else if (rdtype == IMG_BF16)
    bp_batch_kernel<__nv_bfloat16><<<grid_bp, kThreads, smem_bp, s>>>(T);
  else
    bp_batch_kernel<float><<<grid_bp, kThreads, smem_bp, s>>>(T);
  return cudaGetLastError();
}

}  // namespace trb
