/* Body of the oracle restatement, instantiated twice by tiltrec_oracle.c:
 *   PFX = orc_,   REAL = float   (the reference arithmetic)
 *   PFX = orc64_, REAL = double  (the FP64 oracle)
 * TEST INFRASTRUCTURE: see tiltrec_oracle.h.
 *
 * Each routine restates the reference CPU routine it cites, in the same
 * operation order, so the float instantiation reproduces the reference
 * bit for bit when both are compiled without FMA contraction (ISO mode). */

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC_FN(name) ORC_CAT(PFX, name)

/* Weight: int x_min,y_min; float x_min_del,y_min_del (mrcmx/mrcstack.h:291-298).
 * In the FP64 oracle the deltas are kept in double. */
typedef struct {
  int x0, y0;
  REAL dx, dy;
} ORC_CAT(PFX, weight);
#define ORC_W ORC_CAT(PFX, weight)

/* ValCoef (main/main-mpi.cpp:204-226; same in main-mpiz.cpp:173-195): voxel
 * offsets from the float origin are formed in float and widened to double,
 * the projected position is evaluated in double, floor gives the lower
 * neighbour and the fractional part is narrowed to the Weight type. */
static inline void ORC_FN(valcoef)(const orc_geom *g, const double *c, int x,
                                   int y, int z, ORC_W *w) {
  double X = (double)((float)x - g->ox);
  double Y = (double)((float)y - g->oy);
  double Z = (double)((float)z - g->oz);
  double n0 = c[0] + c[1] * X + c[2] * Y + c[3] * Z;
  double n1 = c[4] + c[5] * X + c[6] * Y + c[7] * Z;
  double px = n0 + (double)g->ox;
  double py = n1 + (double)g->oy;
  w->x0 = (int)floor(px);
  w->y0 = (int)floor(py);
  w->dx = (REAL)(px - w->x0);
  w->dy = (REAL)(py - w->y0);
}

/* BilinearValue (main/main-mpi.cpp:378-410): sum over the four neighbours
 * that fall inside the [width x height] image of weight*value, and of
 * weight alone. */
static inline void ORC_FN(bilinear)(int width, int height, const REAL *img,
                                    const ORC_W *w, REAL *val, REAL *vwt) {
  const int x0 = w->x0, y0 = w->y0;
  const REAL dx = w->dx, dy = w->dy;
  int n;
  if (x0 >= 0 && x0 < width && y0 >= 0 && y0 < height) {
    n = x0 + y0 * width;
    *val += (1 - dx) * (1 - dy) * img[n];
    *vwt += (1 - dx) * (1 - dy);
  }
  if ((x0 + 1) >= 0 && (x0 + 1) < width && y0 >= 0 && y0 < height) {
    n = x0 + 1 + y0 * width;
    *val += dx * (1 - dy) * img[n];
    *vwt += dx * (1 - dy);
  }
  if (x0 >= 0 && x0 < width && (y0 + 1) >= 0 && (y0 + 1) < height) {
    n = x0 + (y0 + 1) * width;
    *val += (1 - dx) * dy * img[n];
    *vwt += (1 - dx) * dy;
  }
  if ((x0 + 1) >= 0 && (x0 + 1) < width && (y0 + 1) >= 0 &&
      (y0 + 1) < height) {
    n = x0 + 1 + (y0 + 1) * width;
    *val += dx * dy * img[n];
    *vwt += dx * dy;
  }
}

/* Voxel index for (x, y, z) in either layout; z is the slab-local section. */
static inline size_t ORC_FN(vidx)(const orc_geom *g, int x, int y, int z) {
  if (g->layout == 0) return ((size_t)y * g->th + z) * g->nx + x;
  return ((size_t)z * g->ny + y) * g->nx + x;
}

/* BackProject (main/main-mpi.cpp:411-450, Y layout; main-mpiz.cpp:322-363,
 * Z layout): for each tilt, every voxel adds s/c when c != 0.  Adds to vol
 * (the Z-layout reference zeroes vol first; its callers do that here). */
void ORC_FN(backproject)(const orc_geom *g, const double *coeff8,
                         const REAL *proj, REAL *vol) {
  const size_t plane = (size_t)g->nx * g->ny;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < g->ny; ++y) {
    for (int t = 0; t < g->nt; ++t) {
      const REAL *p = proj + plane * t;
      for (int z = 0; z < g->th; ++z) {
        for (int x = 0; x < g->nx; ++x) {
          ORC_W w;
          REAL s = 0, c = 0;
          ORC_FN(valcoef)(g, coeff8 + 8 * t, x, y, z + g->z0, &w);
          ORC_FN(bilinear)(g->nx, g->ny, p, &w, &s, &c);
          if (c) vol[ORC_FN(vidx)(g, x, y, z)] += (REAL)(s / c);
        }
      }
    }
  }
}

/* Reproject (main/main-mpi.cpp:286-344 for the Y layout, loop order y,z,x;
 * main-mpiz.cpp:197-254 for the Z layout, loop order z,y,x): one tilt's
 * bilinear voxel splat into val (weight*voxel) and wt (weight). */
static void ORC_FN(splat)(const orc_geom *g, const double *c, const REAL *vol,
                          REAL *val, REAL *wt, int y, int z, int x) {
  ORC_W w;
  const int W = g->nx, L = g->ny;
  const REAL v = vol[ORC_FN(vidx)(g, x, y, z)];
  int n;
  ORC_FN(valcoef)(g, c, x, y, z + g->z0, &w);
  const int x0 = w.x0, y0 = w.y0;
  const REAL dx = w.dx, dy = w.dy;
  if (x0 >= 0 && x0 < W && y0 >= 0 && y0 < L) {
    n = x0 + y0 * W;
    val[n] += (1 - dx) * (1 - dy) * v;
    wt[n] += (1 - dx) * (1 - dy);
  }
  if ((x0 + 1) >= 0 && (x0 + 1) < W && y0 >= 0 && y0 < L) {
    n = x0 + 1 + y0 * W;
    val[n] += dx * (1 - dy) * v;
    wt[n] += dx * (1 - dy);
  }
  if (x0 >= 0 && x0 < W && (y0 + 1) >= 0 && (y0 + 1) < L) {
    n = x0 + (y0 + 1) * W;
    val[n] += (1 - dx) * dy * v;
    wt[n] += (1 - dx) * dy;
  }
  if ((x0 + 1) >= 0 && (x0 + 1) < W && (y0 + 1) >= 0 && (y0 + 1) < L) {
    n = (x0 + 1) + (y0 + 1) * W;
    val[n] += dx * dy * v;
    wt[n] += dx * dy;
  }
}

void ORC_FN(reproject)(const orc_geom *g, const double *coeff8,
                       const REAL *vol, REAL *val, REAL *wt) {
  if (g->layout == 0) {
    for (int y = 0; y < g->ny; ++y)
      for (int z = 0; z < g->th; ++z)
        for (int x = 0; x < g->nx; ++x)
          ORC_FN(splat)(g, coeff8, vol, val, wt, y, z, x);
  } else {
    for (int z = 0; z < g->th; ++z)
      for (int y = 0; y < g->ny; ++y)
        for (int x = 0; x < g->nx; ++x)
          ORC_FN(splat)(g, coeff8, vol, val, wt, y, z, x);
  }
}

/* UpdateWeightsByProjDiff (main/main-mpi.cpp:526-562; main-mpiz.cpp:453-486):
 * one tilt's unnormalised gather, valvol += s and wtvol += c. */
void ORC_FN(update_weights)(const orc_geom *g, const double *coeff8,
                            const REAL *diff, REAL *valvol, REAL *wtvol) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < g->ny; ++y)
    for (int z = 0; z < g->th; ++z)
      for (int x = 0; x < g->nx; ++x) {
        ORC_W w;
        REAL s = 0, c = 0;
        ORC_FN(valcoef)(g, coeff8, x, y, z + g->z0, &w);
        ORC_FN(bilinear)(g->nx, g->ny, diff, &w, &s, &c);
        const size_t i = ORC_FN(vidx)(g, x, y, z);
        valvol[i] += s;
        wtvol[i] += c;
      }
}

/* UpdateVolumeByProjDiff (main/main-mpi.cpp:492-524; main-mpiz.cpp:419-451):
 * the SART back-projection vol += (s/c)*gamma where c != 0. */
void ORC_FN(update_by_projdiff)(const orc_geom *g, const double *coeff8,
                                const REAL *diff, REAL *vol, REAL gamma) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < g->ny; ++y)
    for (int z = 0; z < g->th; ++z)
      for (int x = 0; x < g->nx; ++x) {
        ORC_W w;
        REAL s = 0, c = 0;
        ORC_FN(valcoef)(g, coeff8, x, y, z + g->z0, &w);
        ORC_FN(bilinear)(g->nx, g->ny, diff, &w, &s, &c);
        if (c) vol[ORC_FN(vidx)(g, x, y, z)] += (REAL)(s / c) * gamma;
      }
}

/* Residual of one tilt (main/main-mpi.cpp:640-647): reproj <- p - val/wt,
 * with val left unnormalised where wt == 0. */
static void ORC_FN(residual)(size_t n, const REAL *p, REAL *val,
                             const REAL *wt) {
  for (size_t i = 0; i < n; ++i) {
    if (wt[i]) val[i] /= wt[i];
    val[i] = p[i] - val[i];
  }
}

/* SIRT (main/main-mpi.cpp:614-664; main-mpiz.cpp:548-601).  Within an
 * iteration the volume is fixed, so the per-tilt splats run in parallel over
 * tilts; the gathers then add tilt by tilt in tilt order per voxel, which is
 * the reference's per-voxel summation order. */
void ORC_FN(sirt)(const orc_geom *g, const double *coeff8, const REAL *proj,
                  REAL *vol, int iters, REAL gamma) {
  const size_t plane = (size_t)g->nx * g->ny;
  const size_t nvox = plane * g->th;
  REAL *val = (REAL *)malloc(sizeof(REAL) * plane * g->nt);
  REAL *wt = (REAL *)malloc(sizeof(REAL) * plane * g->nt);
  REAL *valvol = (REAL *)malloc(sizeof(REAL) * nvox);
  REAL *wtvol = (REAL *)malloc(sizeof(REAL) * nvox);
  for (int it = 0; it < iters; ++it) {
    memset(valvol, 0, sizeof(REAL) * nvox);
    memset(wtvol, 0, sizeof(REAL) * nvox);
#pragma omp parallel for schedule(dynamic, 1)
    for (int t = 0; t < g->nt; ++t) {
      REAL *v = val + plane * t, *w = wt + plane * t;
      memset(v, 0, sizeof(REAL) * plane);
      memset(w, 0, sizeof(REAL) * plane);
      ORC_FN(reproject)(g, coeff8 + 8 * t, vol, v, w);
      ORC_FN(residual)(plane, proj + plane * t, v, w);
    }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < g->ny; ++y)
      for (int t = 0; t < g->nt; ++t)
        for (int z = 0; z < g->th; ++z)
          for (int x = 0; x < g->nx; ++x) {
            ORC_W w;
            REAL s = 0, c = 0;
            ORC_FN(valcoef)(g, coeff8 + 8 * t, x, y, z + g->z0, &w);
            ORC_FN(bilinear)(g->nx, g->ny, val + plane * t, &w, &s, &c);
            const size_t i = ORC_FN(vidx)(g, x, y, z);
            valvol[i] += s;
            wtvol[i] += c;
          }
    /* UpdateVolumeByWeights (main/main-mpi.cpp:652-658) */
    for (size_t i = nvox; i--;)
      if (wtvol[i]) vol[i] += valvol[i] / wtvol[i] * gamma;
  }
  free(val);
  free(wt);
  free(valvol);
  free(wtvol);
}

/* SART (main/main-mpi.cpp:578-612; main-mpiz.cpp:502-546): per tilt,
 * splat, residual, then the normalised update of the volume. */
void ORC_FN(sart)(const orc_geom *g, const double *coeff8, const REAL *proj,
                  REAL *vol, int iters, REAL gamma) {
  const size_t plane = (size_t)g->nx * g->ny;
  REAL *val = (REAL *)malloc(sizeof(REAL) * plane);
  REAL *wt = (REAL *)malloc(sizeof(REAL) * plane);
  for (int it = 0; it < iters; ++it)
    for (int t = 0; t < g->nt; ++t) {
      memset(val, 0, sizeof(REAL) * plane);
      memset(wt, 0, sizeof(REAL) * plane);
      ORC_FN(reproject)(g, coeff8 + 8 * t, vol, val, wt);
      ORC_FN(residual)(plane, proj + plane * t, val, wt);
      ORC_FN(update_by_projdiff)(g, coeff8 + 8 * t, val, vol, gamma);
    }
  free(val);
  free(wt);
}

#undef ORC_W
#undef ORC_FN
#undef ORC_CAT
#undef ORC_CAT2
