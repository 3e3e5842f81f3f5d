// extern "C" entry points over the reference TiltRec CPU functions, compiled
// together with the unmodified reference sources (main/main-mpi.cpp for the
// Y layout, main/main-mpiz.cpp for the Z layout) by oracle/Makefile.
//
// Oracle infrastructure: used only by tests and the benchmark's CPU-baseline
// leg to run the reference's own arithmetic on host memory.
//
// The declarations below restate the reference's own signatures so that this
// translation unit can call them: struct Coeff (main/main-mpi.cpp:19-30),
// TranslateAngleToCoefficients (:85-106), DecorateCoefficients (:110-183),
// BackProject (:411-450), Reproject (:286-344), UpdateVolumeByProjDiff
// (:492-524), UpdateWeightsByProjDiff (:526-562), SART (:578-612),
// SIRT (:614-664); Z layout: main/main-mpiz.cpp BackProject (:322-363),
// FBP (:365-418), SART (:502-546), SIRT (:548-601);
// ApplyFilterInplace (filter/filter_prj.h:24).
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "filter/filter_prj.h"
#include "mrcmx/mrcstack.h"

struct Coeff {
  union {
    double p[20];
    struct {
      double a[10];
      double b[10];
    };
  };
};

void TranslateAngleToCoefficients(const std::vector<float> &angles,
                                  std::vector<Coeff> &coeffs);
void DecorateCoefficients(std::vector<Coeff> &coeffs, const Geometry &geo);

#ifdef REF_LAYOUT_Y
void BackProject(const Point3DF &origin, MrcStackM &projs, Volume &vol,
                 Coeff coeffv[], int start, int length, Slice &proj,
                 int thickness);
void Reproject(const Point3DF &origin, const Volume &vol, const Coeff &coeff,
               float *reproj_val, float *reproj_wt, int thickness, int length,
               int width);
void UpdateVolumeByProjDiff(const Point3DF &origin, float *diff, Volume &vol,
                            float gamma, const Coeff &coeff, int thickness,
                            int length, int width);
void UpdateWeightsByProjDiff(const Point3DF &origin, float *diff,
                             float *values, float *weights, const Coeff &coeff,
                             int thickness, int length, int width);
void SART(const Point3DF &origin, MrcStackM &projs, Volume &vol,
          Coeff coeffv[], int iteration, float gamma, int start, int length,
          Slice &proj, int thickness);
void SIRT(const Point3DF &origin, MrcStackM &projs, Volume &vol,
          Coeff coeffv[], int iteration, float gamma, int start, int length,
          Slice &proj, int thickness);
#endif

#ifdef REF_LAYOUT_Z
void BackProject(const Point3DF &origin, MrcStackM &projs, Volume &vol,
                 Coeff coeffv[]);
void FBP(const Point3DF &origin, MrcStackM &projs, Volume &vol,
         Coeff coeffv[], int filterMode);
void SART(const Point3DF &origin, MrcStackM &projs, Volume &vol,
          Coeff coeffv[], int iteration, float gamma);
void SIRT(const Point3DF &origin, MrcStackM &projs, Volume &vol,
          Coeff coeffv[], int iteration, float gamma);
void ADMM(const Point3DF &origin, MrcStackM &projs, Volume &vol, Coeff coeffv[],
          int maxOutIter, int numberIteration, float mu, float soft);
#endif

namespace {

// The reference prints progress per tilt and iteration; keep the caller's
// stdout clean by pointing fd 1 at /dev/null for the duration of a call.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
      dup2(devnull, 1);
      close(devnull);
    }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

std::vector<Coeff> to_coeffs(const double *c20, int nt) {
  std::vector<Coeff> v(nt);
  for (int t = 0; t < nt; ++t) memcpy(v[t].p, c20 + 20 * (size_t)t, 160);
  return v;
}

void header_only(MrcStackM &s, int nx, int ny, int nz) {
  memset(&s.header, 0, sizeof(s.header));
  s.header.nx = nx;
  s.header.ny = ny;
  s.header.nz = nz;
  s.header.mode = MrcStackM::MODE_FLOAT;
}

}  // namespace

extern "C" {

// Per-tilt coefficients exactly as the reference CPU path computes them:
// TranslateAngleToCoefficients then DecorateCoefficients; 20 doubles per tilt
// (a[0..9], b[0..9]).
void ref_coeffs(const float *angles, int nt, float offset, float pitch,
                float zshift, double *out20) {
  std::vector<float> ang(angles, angles + nt);
  std::vector<Coeff> c;
  TranslateAngleToCoefficients(ang, c);
  Geometry geo;
  geo.offset = offset;
  geo.pitch_angle = pitch;
  geo.zshift = zshift;
  DecorateCoefficients(c, geo);
  for (int t = 0; t < nt; ++t) memcpy(out20 + 20 * (size_t)t, c[t].p, 160);
}

// ApplyFilterInplace(mode 2): the WBP R-weighting of every row of every tilt.
// proj: [nt][ny][nx] float, filtered in place.
int ref_filter_rweight(int nx, int ny, int nt, float *proj) {
  MrcStackM s;
  header_only(s, nx, ny, nt);
  QuietStdout q;
  return ApplyFilterInplace(s, proj, (size_t)ny, 2);
}

// ApplyFilterInplace modes 0 (Shepp-Logan) and 1 (Ram-Lak): the FBP row
// filters, through the OpenCV C-API shim (exact DFTs).  proj: [nt][ny][nx].
int ref_filter_fbp(int mode, int nx, int ny, int nt, float *proj) {
  if (mode != 0 && mode != 1) return -2;
  MrcStackM s;
  header_only(s, nx, ny, nt);
  QuietStdout q;
  return ApplyFilterInplace(s, proj, (size_t)ny, mode);
}

#ifdef REF_LAYOUT_Y
// Y layout: proj [nt][ny][nx], vol [ny][th][nx]; one rank owning every row.

void ref_y_backproject(int nx, int ny, int nt, int th, const double *c20,
                       float ox, float oy, float oz, float *proj, float *vol) {
  MrcStackM s;
  header_only(s, nx, ny, nt);
  std::vector<Coeff> c = to_coeffs(c20, nt);
  Point3DF o{ox, oy, oz};
  Volume v(0, 0, 0, nx, th, ny, vol);
  Slice p(nx, ny, proj);
  QuietStdout q;
  BackProject(o, s, v, c.data(), 0, ny, p, th);
}

void ref_y_sirt(int nx, int ny, int nt, int th, const double *c20, float ox,
                float oy, float oz, float *proj, float *vol, int iters,
                float gamma, int sart) {
  MrcStackM s;
  header_only(s, nx, ny, nt);
  std::vector<Coeff> c = to_coeffs(c20, nt);
  Point3DF o{ox, oy, oz};
  Volume v(0, 0, 0, nx, th, ny, vol);
  Slice p(nx, ny, proj);
  QuietStdout q;
  if (sart)
    SART(o, s, v, c.data(), iters, gamma, 0, ny, p, th);
  else
    SIRT(o, s, v, c.data(), iters, gamma, 0, ny, p, th);
}

// One tilt's voxel splat (accumulates into val/wt, [ny][nx]).
void ref_y_reproject(int nx, int ny, int th, const double *c20, float ox,
                     float oy, float oz, const float *vol, float *val,
                     float *wt) {
  std::vector<Coeff> c = to_coeffs(c20, 1);
  Point3DF o{ox, oy, oz};
  Volume v(0, 0, 0, nx, th, ny, const_cast<float *>(vol));
  Reproject(o, v, c[0], val, wt, th, ny, nx);
}

// One tilt's unnormalised bilinear gather (valvol += s, wtvol += c).
void ref_y_update_weights(int nx, int ny, int th, const double *c20, float ox,
                          float oy, float oz, float *diff, float *valvol,
                          float *wtvol) {
  std::vector<Coeff> c = to_coeffs(c20, 1);
  Point3DF o{ox, oy, oz};
  UpdateWeightsByProjDiff(o, diff, valvol, wtvol, c[0], th, ny, nx);
}

// One tilt's normalised update vol += gamma * s / c (SART back-projection).
void ref_y_update_by_projdiff(int nx, int ny, int th, const double *c20,
                              float ox, float oy, float oz, float *diff,
                              float *vol, float gamma) {
  std::vector<Coeff> c = to_coeffs(c20, 1);
  Point3DF o{ox, oy, oz};
  Volume v(0, 0, 0, nx, th, ny, vol);
  UpdateVolumeByProjDiff(o, diff, v, gamma, c[0], th, ny, nx);
}

// Timed CPU baseline: the reference SIRT run on nthreads host threads, each
// owning an even share of the rows [row0, row0 + nrows) plus the reference's
// XTILT halo (ceil(|tan(pitch)| * th) rows each side, main-mpi.cpp:713-740),
// exactly as one MPI rank of TiltRec-mpi would process its block.  The
// reference's own rank partition hands every remaining row to each rank
// (main-mpi.cpp:732-735), so as written it does not scale with ranks; the even
// partition used here favours the reference.  Returns wall seconds of the
// reconstruction only (no file I/O).  proj: full [nt][ny][nx] stack.
double ref_y_sirt_threaded(int nthreads, int nx, int ny, int nt, int th,
                           const double *c20, float pitch, const float *proj,
                           int row0, int nrows, int iters, float gamma) {
  std::vector<Coeff> c = to_coeffs(c20, nt);
  const int halo =
      (int)ceil(fabsf(tan(pitch * 0.01745329252f)) * (float)th);
  struct Block {
    int s, e, hl, hr;
    std::vector<float> p, v;
  };
  std::vector<Block> blocks(nthreads);
  for (int r = 0; r < nthreads; ++r) {
    Block &b = blocks[r];
    const int base = nrows / nthreads, rem = nrows % nthreads;
    b.s = row0 + r * base + (r < rem ? r : rem);
    b.e = b.s + base + (r < rem ? 1 : 0);
    b.hl = std::min(halo, b.s);
    b.hr = std::min(halo, ny - b.e);
    const int len = b.e - b.s + b.hl + b.hr;
    b.p.resize((size_t)nt * len * nx);
    for (int t = 0; t < nt; ++t)
      memcpy(&b.p[(size_t)t * len * nx],
             proj + ((size_t)t * ny + (b.s - b.hl)) * nx,
             sizeof(float) * (size_t)len * nx);
    b.v.assign((size_t)len * th * nx, 0.f);
  }
  QuietStdout q;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (int r = 0; r < nthreads; ++r) {
    pool.emplace_back([&, r]() {
      Block &b = blocks[r];
      const int len = b.e - b.s + b.hl + b.hr;
      if (b.e <= b.s) return;
      MrcStackM s;
      header_only(s, nx, ny, nt);
      Point3DF o{nx * 0.5f, th * 0.5f - b.s + b.hl, th * 0.5f};
      Volume v(0, 0, 0, nx, th, len, b.v.data());
      Slice p(nx, ny, b.p.data());
      SIRT(o, s, v, c.data(), iters, gamma, b.s, len, p, th);
    });
  }
  for (auto &t : pool) t.join();
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

namespace {
// Reusable barrier for a fixed set of threads (C++17 has no std::barrier).
class Barrier {
 public:
  explicit Barrier(int n) : n_(n) {}
  void wait() {
    std::unique_lock<std::mutex> lk(m_);
    const unsigned long g = gen_;
    if (++count_ == n_) {
      count_ = 0;
      ++gen_;
      cv_.notify_all();
    } else {
      cv_.wait(lk, [&] { return gen_ != g; });
    }
  }

 private:
  std::mutex m_;
  std::condition_variable cv_;
  int n_, count_ = 0;
  unsigned long gen_ = 0;
};
}  // namespace

// Whole-volume SIRT of the reference (SIRT, main-mpi.cpp:614-664) on host
// threads, exact: the volume is split into z-slabs (thread r owns sections
// [z0, z1), copied to a [ny][z1-z0][nx] buffer with the origin moved by z0),
// and per tilt every thread runs the reference's Reproject on its slab into
// its own reprojection planes; the planes are summed in thread order, the
// residual is formed as the reference forms it, and every thread runs the
// reference's UpdateWeightsByProjDiff on its slab; after all tilts each slab
// takes the reference's update vol += valvol / wtvol * gamma.  Per voxel the
// arithmetic is the reference's; only the order in which the forward splat's
// contributions are added to a detector pixel differs (slab partial sums).
// vol [ny][th][nx] is updated in place.  Returns wall seconds.
double ref_y_sirt_zslabs(int nthreads, int nx, int ny, int nt, int th, const double *c20,
                         float ox, float oy, float oz, const float *proj, float *vol,
                         int iters, float gamma) {
  std::vector<Coeff> c = to_coeffs(c20, nt);
  nthreads = std::max(1, std::min(nthreads, th));
  const size_t plane = (size_t)ny * nx;
  struct Slab {
    int z0, nz;
    std::vector<float> v, valvol, wtvol, val, wt;
  };
  std::vector<Slab> sl(nthreads);
  for (int r = 0; r < nthreads; ++r) {
    Slab &s = sl[r];
    const int base = th / nthreads, rem = th % nthreads;
    s.z0 = r * base + std::min(r, rem);
    s.nz = base + (r < rem ? 1 : 0);
    s.v.resize(plane * s.nz);
    for (int y = 0; y < ny; ++y)
      memcpy(&s.v[(size_t)y * s.nz * nx], vol + ((size_t)y * th + s.z0) * nx,
             sizeof(float) * (size_t)s.nz * nx);
    s.valvol.resize(plane * s.nz);
    s.wtvol.resize(plane * s.nz);
    s.val.resize(plane);
    s.wt.resize(plane);
  }
  std::vector<float> resid(plane);
  Barrier bar(nthreads);
  QuietStdout q;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (int r = 0; r < nthreads; ++r) {
    pool.emplace_back([&, r]() {
      Slab &s = sl[r];
      Point3DF o{ox, oy, oz - (float)s.z0};
      Volume v(0, 0, 0, nx, s.nz, ny, s.v.data());
      const size_t n0 = plane * r / nthreads, n1 = plane * (r + 1) / nthreads;
      const size_t size = plane * s.nz;
      for (int it = 0; it < iters; ++it) {
        std::fill(s.valvol.begin(), s.valvol.end(), 0.f);
        std::fill(s.wtvol.begin(), s.wtvol.end(), 0.f);
        for (int idx = 0; idx < nt; ++idx) {
          std::fill(s.val.begin(), s.val.end(), 0.f);
          std::fill(s.wt.begin(), s.wt.end(), 0.f);
          Reproject(o, v, c[idx], s.val.data(), s.wt.data(), s.nz, ny, nx);
          bar.wait();
          const float *pd = proj + plane * idx;
          for (size_t n = n0; n < n1; ++n) {
            float val = 0.f, wt = 0.f;
            for (int k = 0; k < nthreads; ++k) {
              val += sl[k].val[n];
              wt += sl[k].wt[n];
            }
            if (wt) val /= wt;
            resid[n] = pd[n] - val;
          }
          bar.wait();
          UpdateWeightsByProjDiff(o, resid.data(), s.valvol.data(), s.wtvol.data(), c[idx],
                                  s.nz, ny, nx);
        }
        for (size_t i = size; i--;)
          if (s.wtvol[i]) s.v[i] += s.valvol[i] / s.wtvol[i] * gamma;
      }
    });
  }
  for (auto &t : pool) t.join();
  auto t1 = std::chrono::steady_clock::now();
  for (int r = 0; r < nthreads; ++r)
    for (int y = 0; y < ny; ++y)
      memcpy(vol + ((size_t)y * th + sl[r].z0) * nx, &sl[r].v[(size_t)y * sl[r].nz * nx],
             sizeof(float) * (size_t)sl[r].nz * nx);
  return std::chrono::duration<double>(t1 - t0).count();
}
#endif  // REF_LAYOUT_Y

#ifdef REF_LAYOUT_Z
// The Z-layout reference frees two of its owned Slice buffers twice: an
// explicit delete[] of slice.data followed by ~Slice() deleting it again
// (main/main-mpiz.cpp BackProject :361-362 with Slice(int,int) :324, SIRT
// :597-599 with :553-555; Slice owns data it allocated, mrcmx/mrcstack.h:252-
// 287), which aborts the process once the volume is complete.  libref_z.so is
// linked with --wrap for operator delete[] so that, inside ref_z_run, array
// deletes are deferred to the end of the call and each pointer is freed once.
static thread_local std::vector<void *> *g_deferred = nullptr;
extern "C" void __real__ZdaPv(void *p);
extern "C" void __wrap__ZdaPv(void *p) {
  if (g_deferred) {
    for (void *q : *g_deferred)
      if (q == p) return;
    g_deferred->push_back(p);
    return;
  }
  __real__ZdaPv(p);
}
extern "C" void __real__ZdaPvm(void *p, size_t n);
extern "C" void __wrap__ZdaPvm(void *p, size_t n) {
  if (g_deferred) {
    __wrap__ZdaPv(p);
    return;
  }
  __real__ZdaPvm(p, n);
}

// Z layout: proj [nt][ny][nx], vol [th][ny][nx].  The reference reads the
// projections from an MRC file inside these functions, so the stack is
// written to a scratch file under tmpdir first.
static int write_stack(const char *path, int nx, int ny, int nt,
                       const float *proj) {
  MRCheader h;
  memset(&h, 0, sizeof(h));
  h.nx = nx;
  h.ny = ny;
  h.nz = nt;
  h.mode = 2;
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  fwrite(&h, sizeof(h), 1, f);
  fwrite(proj, sizeof(float), (size_t)nx * ny * nt, f);
  fclose(f);
  return 0;
}

// mode: 0 = BPT (BackProject), 2 = WBP (FBP with filter mode 2),
//       3 = SIRT, 4 = SART.
int ref_z_run(int mode, int nx, int ny, int nt, int th, const double *c20,
              float ox, float oy, float oz, const float *proj, float *vol,
              int iters, float gamma, const char *tmpdir) {
  std::string path = std::string(tmpdir) + "/oracle_z_stack_" +
                     std::to_string((long)getpid()) + ".mrc";
  if (write_stack(path.c_str(), nx, ny, nt, proj)) return -1;
  std::vector<Coeff> c = to_coeffs(c20, nt);
  Point3DF o{ox, oy, oz};
  MrcStackM s;
  if (!s.ReadFile(path.c_str())) return -2;
  s.ReadHeader();
  Volume v(0, 0, 0, ny, nx, th, vol);
  std::vector<void *> deferred;
  {
    QuietStdout q;
    g_deferred = &deferred;
    if (mode == 0)
      BackProject(o, s, v, c.data());
    else if (mode == 2)
      FBP(o, s, v, c.data(), 2);
    else if (mode == 3)
      SIRT(o, s, v, c.data(), iters, gamma);
    else if (mode == 4)
      SART(o, s, v, c.data(), iters, gamma);
    g_deferred = nullptr;
  }
  for (void *p : deferred) __real__ZdaPv(p);
  s.Close();
  unlink(path.c_str());
  return 0;
}
// ADMM (main-mpiz.cpp:958-1013) on the Z layout, as ref_z_run.
int ref_z_admm(int nx, int ny, int nt, int th, const double *c20, float ox, float oy,
               float oz, const float *proj, float *vol, int outer, int cg, float mu,
               float soft, const char *tmpdir) {
  std::string path = std::string(tmpdir) + "/oracle_z_stack_" +
                     std::to_string((long)getpid()) + ".mrc";
  if (write_stack(path.c_str(), nx, ny, nt, proj)) return -1;
  std::vector<Coeff> c = to_coeffs(c20, nt);
  Point3DF o{ox, oy, oz};
  MrcStackM s;
  if (!s.ReadFile(path.c_str())) return -2;
  s.ReadHeader();
  Volume v(0, 0, 0, ny, nx, th, vol);
  std::vector<void *> deferred;
  {
    QuietStdout q;
    g_deferred = &deferred;
    ADMM(o, s, v, c.data(), outer, cg, mu, soft);
    g_deferred = nullptr;
  }
  for (void *p : deferred) __real__ZdaPv(p);
  s.Close();
  unlink(path.c_str());
  return 0;
}
#endif  // REF_LAYOUT_Z

}  // extern "C"
