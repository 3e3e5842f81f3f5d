/* CPU restatement of the reference TiltRec reconstruction path.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this.  It is the checker, never the
 * product path.
 *
 * Parity pin: the reference ships no golden vectors or tests for TiltRec; the
 * restatement is pinned against the unmodified reference CPU sources compiled
 * by oracle/Makefile (`make ref`, outputs in oracle/_ref/) on seeded inputs,
 * and the reference-generated fixtures in tests/golden/.
 *
 * Every function is compiled twice from tiltrec_oracle_impl.h: orc_* computes
 * in float exactly as the reference does (double coordinates, float weights
 * and accumulators), orc64_* replaces every float in the data path by double
 * (the FP64 oracle used to score reduced-precision storage).
 */
#ifndef TILTREC_ORACLE_H
#define TILTREC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Volume geometry.  layout 0 = Y layout (TiltRec): vol[ny][th][nx];
 * layout 1 = Z layout (TiltRecZ): vol[th][ny][nx].  Projections are
 * [nt][ny][nx].  z0 is the global z index of the first volume section (Z
 * slabs); ox/oy/oz the float origin the reference passes to ValCoef. */
typedef struct {
  int nx, ny, nt, th;
  int layout;
  int z0;
  float ox, oy, oz;
} orc_geom;

/* Per-tilt linear coefficients a0..a3, b0..b3 (main-mpi.cpp:85-183). */
void orc_coeffs(const float *angles, int nt, float offset, float pitch,
                float zshift, double *coeff8);

/* WBP R-weighting filter, mode 2 (filter_prj.cpp:636-736), in place over
 * nrows rows of nx floats, evaluated as a double-precision circular
 * convolution on the padded row. */
void orc_filter_rweight(int nx, long nrows, float *rows);

/* FBP row filters, modes 0 (Shepp-Logan) and 1 (Ram-Lak) of
 * ApplyFilterInplace (filter_prj.cpp:755-786), in place over nrows rows of nx
 * floats: FileterProjectionSymmetrize (:265-446) with its 251-tap kernel
 * (RamLak :137-155, SheppLogan :158-178), evaluated as the circular
 * convolution its DFTs compute, in double precision.  Returns the DFT length
 * L the reference would use. */
int orc_filter_fbp(int mode, int nx, long nrows, float *rows);

/* Area binning of nt images of nx*ny floats by an integer factor (the GUI
 * chain's `resample -b bin`, resample/src/main/main.cpp:14-58, 67-147, which
 * calls OpenCV's area resize to (nx/bin) x (ny/bin)): output pixel (i, j)
 * is the mean of the input over [i*sx, (i+1)*sx) x [j*sy, (j+1)*sy) with
 * sx = nx/(nx/bin), sy likewise, partial pixels weighted by their overlap;
 * separable, in double.  Out: nt * (nx/bin) * (ny/bin). */
void orc_resample_bin(const float *src, int nx, int ny, int nt, int bin, float *dst);

/* Smallest integer >= n whose only prime factors are 2, 3 and 5 (the
 * sizes OpenCV's getOptimalDFTSize returns). */
int orc_optimal_dft_size(int n);

#define ORC_DECLARE(PFX, REAL)                                                \
  void PFX##backproject(const orc_geom *g, const double *coeff8,              \
                        const REAL *proj, REAL *vol);                          \
  void PFX##reproject(const orc_geom *g, const double *coeff8,                \
                      const REAL *vol, REAL *val, REAL *wt);                   \
  void PFX##update_weights(const orc_geom *g, const double *coeff8,           \
                           const REAL *diff, REAL *valvol, REAL *wtvol);       \
  void PFX##update_by_projdiff(const orc_geom *g, const double *coeff8,        \
                               const REAL *diff, REAL *vol, REAL gamma);       \
  void PFX##sirt(const orc_geom *g, const double *coeff8, const REAL *proj,   \
                 REAL *vol, int iters, REAL gamma);                            \
  void PFX##sart(const orc_geom *g, const double *coeff8, const REAL *proj,   \
                 REAL *vol, int iters, REAL gamma);

ORC_DECLARE(orc_, float)
ORC_DECLARE(orc64_, double)

#ifdef __cplusplus
}
#endif
#endif
