// TiltRec-cuda / TiltRecZ-cuda drop-in executables on the B200 engine.
//
// Same flags and files as the reference executables:
//   --input/-i <mrc>   --output/-o <mrc>   --tiltfile/-t <angles>
//   --geometry/-g offset,pitch,zshift,thickness
//   --method/-m BPT | FBP | WBP | SIRT,n,gamma | SART,n,gamma | ADMM,n,cg,mu,soft
//   --inital/-n <mrc> (cuda dialect, sic) or --initial <mrc> (mpi dialect)
//   --axis/-a y|z (parsed; the executable name selects the layout)
//   --f2b/-f (byte output)   --help/-h
// (option parsing: TR/opts/opts.cpp:126-359, TR/opts/opts-mpi.h:114-284).
//
// Compiled four times: TR_CLI_LAYOUT=0 gives TiltRec-cuda (Y layout, output
// MRC (X, thickness, Y), TR/main/main-cuda.cpp), TR_CLI_LAYOUT=1 gives
// TiltRecZ-cuda (Z layout, output MRC (X, Y, thickness),
// TR/main/main-cudaz.cpp, which forces XTILT to 0, :163); with
// TR_CLI_MPI_DIALECT=1 the same two layouts answer to the names the GUI also
// spawns, TiltRec-mpi and TiltRecZ-mpi (CommandChainManager.qml:167-170), and
// take the mpi executables' option table (TR/opts/opts-mpi.h:114-128): long
// --tiltfile only, --initial, no --f2b; the reference's -a / -x short options
// reach assert(false) there (:279-280) and are an error (status 1) here.
//
// Semantics follow the reference CPU path (TiltRec-mpi / TiltRecZ-mpi), the
// parity target: FP64 coefficients (main-mpi.cpp:85-183), the Y-layout origin
// (X/2, thickness/2, thickness/2) (main-mpi.cpp:743-745) and the whole volume
// reconstructed at once (no Y-slab halos).  Under mpirun only rank 0 works and
// the others exit, as in the reference GPU executables where rank 0 computes.
// Differences, all deliberate: --initial is honoured on the GPU path (the
// reference GPU code parses it and ignores it, recon_y.cu:345); a bare
// SIRT/SART without iterations is an error (the reference leaves them
// uninitialised, opts.cpp:112-123); ADMM (TiltRecZ-mpi only in the reference)
// runs in both layouts; errors exit with status 1.  FBP is the Shepp-Logan filter (ApplyFilterInplace
// mode 0, main-mpi.cpp:835-839) then the back-projection.
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <sstream>
#include <string>
#include <vector>

#include "mrc_io.h"
#include "tiltrec_b200.h"

#ifndef TR_CLI_LAYOUT
#define TR_CLI_LAYOUT 0
#endif
#ifndef TR_CLI_MPI_DIALECT
#define TR_CLI_MPI_DIALECT 0
#endif

namespace {

struct Options {
  std::string input, output, initial, angles, method, axis = "y";
  float offset = 0, pitch = 0, zshift = 0;
  int thickness = 0;
  int iteration = -1;
  float gamma = 0;
  int cgiter = -1;   // ADMM
  float soft = 0;    // ADMM
  bool f2b = false;
};

// ADMM has no tr_method code: it takes two more parameters (tr_admm_host).
constexpr int kMethodAdmm = -1;
const char *kProg = TR_CLI_MPI_DIALECT ? (TR_CLI_LAYOUT == 0 ? "TiltRec-mpi" : "TiltRecZ-mpi")
                                       : (TR_CLI_LAYOUT == 0 ? "TiltRec-cuda" : "TiltRecZ-cuda");

void usage() {
  printf(
      "%s -- TiltRec reconstruction on the B200 engine\n"
      "  --input(-i) <mrc>        tilt series\n"
      "  --output(-o) <mrc>       reconstruction\n"
      "  --tiltfile(-t) <file>    tilt angles, degrees\n"
      "  --inital(-n)/--initial <mrc>  starting volume\n"
      "  --geometry(-g) offset,pitch_angle,zshift,thickness\n"
      "  --method(-m) BPT | FBP | WBP | SIRT,iterations,relax | SART,iterations,relax\n"
      "               | ADMM,iterations,cgiter,relax,soft\n"
      "  --f2b(-f)                write bytes (0-255)\n"
      "  --help(-h)\n"
      "example: mpirun -n 1 ./%s --input a.mrc --output v.mrc --tiltfile a.rawtlt"
      " --geometry 0,0,0,300 --method WBP\n",
      kProg, kProg);
}

// 1 ok, 0 help, -1 error (GetOpts conventions).
int parse(int argc, char **argv, Options *o) {
#if TR_CLI_MPI_DIALECT
  static option longopts[] = {{"help", no_argument, nullptr, 'h'},
                              {"input", required_argument, nullptr, 'i'},
                              {"output", required_argument, nullptr, 'o'},
                              {"initial", required_argument, nullptr, 'n'},
                              {"tiltfile", required_argument, nullptr, 't'},
                              {"geometry", required_argument, nullptr, 'g'},
                              {"method", required_argument, nullptr, 'm'},
                              {nullptr, 0, nullptr, 0}};
  const char *shortopts = "hi:o:n:g:m:a:x:";
#else
  static option longopts[] = {{"help", no_argument, nullptr, 'h'},
                              {"input", required_argument, nullptr, 'i'},
                              {"output", required_argument, nullptr, 'o'},
                              {"inital", required_argument, nullptr, 'n'},
                              {"initial", required_argument, nullptr, 'n'},
                              {"tiltfile", required_argument, nullptr, 't'},
                              {"geometry", required_argument, nullptr, 'g'},
                              {"method", required_argument, nullptr, 'm'},
                              {"axis", required_argument, nullptr, 'a'},
                              {"f2b", no_argument, nullptr, 'f'},
                              {nullptr, 0, nullptr, 0}};
  const char *shortopts = "hi:o:n:t:g:m:a:f";
#endif
  int ch;
  while ((ch = getopt_long(argc, argv, shortopts, longopts, nullptr)) != -1) {
#if TR_CLI_MPI_DIALECT
    if (ch == 'a' || ch == 'x') {  // assert(false) in the reference's GetOpts
      fprintf(stderr, "%s: option -%c is not accepted\n", kProg, ch);
      return -1;
    }
#endif
    switch (ch) {
      case 'h':
        usage();
        return 0;
      case 'i':
        o->input = optarg;
        break;
      case 'o':
        o->output = optarg;
        break;
      case 'n':
        o->initial = optarg;
        break;
      case 't':
        o->angles = optarg;
        break;
      case 'a':
        o->axis = optarg;
        break;
      case 'f':
        o->f2b = true;
        break;
      case 'g': {
        std::stringstream iss(optarg);
        std::string t;
        getline(iss, t, ',');
        o->offset = (float)atof(t.c_str());
        getline(iss, t, ',');
        o->pitch = (float)atof(t.c_str());
        getline(iss, t, ',');
        o->zshift = (float)atof(t.c_str());
        getline(iss, t);
        o->thickness = atoi(t.c_str());
        if (!iss.eof()) {
          fprintf(stderr, "Too many arguments for geometry '%s'.\n", optarg);
          return -1;
        }
        break;
      }
      case 'm': {
        std::stringstream iss(optarg);
        std::string t;
        getline(iss, o->method, ',');
        if (o->method == "SIRT" || o->method == "SART") {
          if (getline(iss, t, ',')) o->iteration = atoi(t.c_str());
          if (getline(iss, t)) o->gamma = (float)atof(t.c_str());
        } else if (o->method == "ADMM") {
          // ADMM,iterations,cgiter,relax,soft (opts.cpp:301-311)
          if (getline(iss, t, ',')) o->iteration = atoi(t.c_str());
          if (getline(iss, t, ',')) o->cgiter = (int)atof(t.c_str());
          if (getline(iss, t, ',')) o->gamma = (float)atof(t.c_str());
          if (getline(iss, t)) o->soft = (float)atof(t.c_str());
        }
        break;
      }
      default:
        fprintf(stderr, "Unknown option: %s\n", argv[optind - 1]);
        return -1;
    }
  }
  return 1;
}

int rank_from_env() {
  for (const char *v : {"OMPI_COMM_WORLD_RANK", "PMI_RANK", "PMIX_RANK", "MV2_COMM_WORLD_RANK"})
    if (const char *s = getenv(v)) return atoi(s);
  return 0;
}

// --f2b: the reference maps each Y slab of (up to) 64 rows to bytes with an
// exponentially averaged mean and deviation (alpha 0.9, starting from 0),
// clamps the z-score to +-10 and scales to 0..255, converting complete groups
// of four values only (recon_y.cu:164-181, basic.cu:442-475); the Z-layout
// drivers map the whole volume with its own mean and deviation (recon_z.cu:
// 164-172).  Reconstructions other than ADMM do this on the device
// (tr_volume_to_bytes through tr_reconstruct_to_sink); ADMM's host volume is
// mapped here the same way.
std::vector<unsigned char> to_bytes(const std::vector<float> &vol, size_t slab, float alpha) {
  std::vector<unsigned char> out(vol.size(), 0);
  float gmean = 0, gstd = 0;
  const float sf = 10.f;
  for (size_t s0 = 0; s0 < vol.size(); s0 += slab) {
    const size_t n = std::min(slab, vol.size() - s0);
    double sum = 0;
    for (size_t i = 0; i < n; ++i) sum += vol[s0 + i];
    const float mean = (float)(sum / n);
    double ss = 0;
    for (size_t i = 0; i < n; ++i) {
      const float d = vol[s0 + i] - mean;
      ss += d * d;
    }
    const float sd = std::sqrt((float)(ss / n));
    gmean = alpha * gmean + (1 - alpha) * mean;
    gstd = alpha * gstd + (1 - alpha) * sd;
    for (size_t i = 0; i + 3 < n; i += 4)
      for (int k = 0; k < 4; ++k) {
        float v = (vol[s0 + i + k] - gmean) / gstd;
        v = std::fmax(-sf, std::fmin(sf, v));
        out[s0 + i + k] = (unsigned char)(((v + sf) / (2.0f * sf)) * 255.0f);
      }
  }
  return out;
}

// Output file written block by block as the engine streams the volume back:
// the header first (rewritten at the end with the statistics of the middle
// section, which is captured as it passes), then the data in order.
struct FileSink {
  FILE *f = nullptr;
  size_t es = 4;                  // bytes per voxel in the file
  size_t mid_off = 0, mid_n = 0;  // middle section: first byte, voxels
  std::vector<float> mid;
};

int file_sink(void *user, const void *data, size_t off, size_t len) {
  FileSink *k = static_cast<FileSink *>(user);
  if (fwrite(data, 1, len, k->f) != len) return 1;
  const size_t a = std::max(off, k->mid_off), b = std::min(off + len, k->mid_off + k->mid_n * k->es);
  for (size_t p = a; p < b; p += k->es) {
    const unsigned char *src = static_cast<const unsigned char *>(data) + (p - off);
    float v;
    if (k->es == 1) {
      v = (float)src[0];
    } else {
      memcpy(&v, src, sizeof v);
    }
    k->mid[(p - k->mid_off) / k->es] = v;
  }
  return 0;
}

int run(const Options &o) {
  std::string err;
  if (o.input.empty() || o.output.empty() || o.angles.empty())
    return fprintf(stderr, "%s: --input, --output and --tiltfile are required\n", kProg), 1;
  if (o.thickness <= 0)
    return fprintf(stderr, "%s: --geometry needs a positive thickness\n", kProg), 1;
  int method;
  if (o.method == "BPT")
    method = TR_METHOD_BPT;
  else if (o.method == "WBP")
    method = TR_METHOD_WBP;
  else if (o.method == "FBP")
    method = TR_METHOD_FBP;
  else if (o.method == "SIRT" || o.method == "SART") {
    if (o.iteration < 0)
      return fprintf(stderr, "%s: %s needs iterations and relaxation (%s,n,gamma)\n", kProg,
                     o.method.c_str(), o.method.c_str()),
             1;
    method = o.method == "SIRT" ? TR_METHOD_SIRT : TR_METHOD_SART;
  } else if (o.method == "ADMM") {
    if (o.iteration < 0 || o.cgiter < 0)
      return fprintf(stderr, "%s: ADMM needs ADMM,iterations,cgiter,relax,soft\n", kProg), 1;
    method = kMethodAdmm;
  } else {
    return fprintf(stderr, "%s: unknown method '%s'\n", kProg, o.method.c_str()), 1;
  }

  trcli::MrcHeader in;
  if (!trcli::read_header(o.input, &in, &err)) return fprintf(stderr, "%s\n", err.c_str()), 1;
  const int nx = in.nx, ny = in.ny, nt = in.nz, th = o.thickness;
  std::vector<float> angles;
  if (!trcli::read_angles(o.angles, &angles, &err)) return fprintf(stderr, "%s\n", err.c_str()), 1;
  if ((int)angles.size() < nt)
    return fprintf(stderr, "%s: %zu tilt angles for %d projections\n", kProg, angles.size(), nt),
           1;
  angles.resize(nt);
  const bool zlayout = TR_CLI_LAYOUT == 1;
  // TiltRecZ-cuda ignores XTILT (main-cudaz.cpp:163).
  const float pitch = zlayout ? 0.f : o.pitch;

  std::vector<float> proj((size_t)nx * ny * nt);
  // Byte stacks: the Y executables read through ReadBlock (signed); the Z
  // executables read BPT/SIRT/SART projections through ReadSliceZ
  // (unsigned) and WBP / FBP through ReadBlock (signed, main-mpiz.cpp:365-384).
  const bool signed_bytes = !zlayout || method == TR_METHOD_WBP || method == TR_METHOD_FBP;
  if (!trcli::read_sections(o.input, in, 0, nt, signed_bytes, proj.data(), &err))
    return fprintf(stderr, "%s\n", err.c_str()), 1;

  std::vector<double> coeff((size_t)nt * 8);
  if (tr_geometry_from_angles(angles.data(), nt, o.offset, pitch, o.zshift, coeff.data()))
    return fprintf(stderr, "%s: bad geometry\n", kProg), 1;
  const float ox = nx * 0.5f, oy = zlayout ? ny * 0.5f : th * 0.5f, oz = th * 0.5f;

  const size_t nvox = (size_t)nx * ny * th;
  std::vector<float> vol;  // the starting volume (--initial), or ADMM's output
  // The starting volume: TiltRec-mpi loads it for every method
  // (main-mpi.cpp:778-791); the Z-layout BPT/WBP start from zero
  // (main-mpiz.cpp BackProject/FBP zero the volume).
  const bool use_initial = !o.initial.empty() &&
                           !(zlayout && (method == TR_METHOD_BPT || method == TR_METHOD_WBP ||
                                         method == TR_METHOD_FBP));
  if (use_initial || method == kMethodAdmm) vol.assign(nvox, 0.f);
  if (use_initial) {
    trcli::MrcHeader ih;
    if (!trcli::read_header(o.initial, &ih, &err)) return fprintf(stderr, "%s\n", err.c_str()), 1;
    const int want_y = zlayout ? ny : th, want_z = zlayout ? th : ny;
    if (ih.nx != nx || ih.ny != want_y || ih.nz != want_z)
      return fprintf(stderr, "%s: initial volume is %dx%dx%d, expected %dx%dx%d\n", kProg, ih.nx,
                     ih.ny, ih.nz, nx, want_y, want_z),
             1;
    if (!trcli::read_sections(o.initial, ih, 0, want_z, true, vol.data(), &err))
      return fprintf(stderr, "%s\n", err.c_str()), 1;
  }

  tr_ctx *ctx = nullptr;
  int device = 0;
  if (const char *d = getenv("TILTREC_DEVICE")) device = atoi(d);
  // TILTREC_HBM_BUDGET: device-memory budget of the context in bytes (0: none)
  size_t budget = 0;
  if (const char *b = getenv("TILTREC_HBM_BUDGET")) budget = strtoull(b, nullptr, 10);
  if (tr_create(device, budget, &ctx) != TR_OK)
    return fprintf(stderr, "%s: no CUDA device %d\n", kProg, device), 1;
  int st = tr_set_problem(ctx, nx, ny, nt, th, zlayout ? TR_LAYOUT_Z : TR_LAYOUT_Y, coeff.data(),
                          ox, oy, oz);

  // Output: Y layout MRC (X, thickness, Y), Z layout MRC (X, Y, thickness).
  trcli::MrcHeader out = zlayout ? trcli::new_volume_header(nx, ny, th, o.f2b)
                                 : trcli::new_volume_header(nx, th, ny, o.f2b);
  const size_t plane = (size_t)out.nx * out.ny;
  const size_t mid = (size_t)(int)(out.nz * .5);
  // Byte slabs: 64 rows of the Y layout (EMA alpha 0.9; the reference's slab
  // height is at least 64 rows, more where its device memory allows), or the
  // whole Z volume (alpha 0).
  const size_t slab = zlayout ? nvox : (size_t)nx * th * 64;
  const float alpha = zlayout ? 0.f : 0.9f;
  bool ok = true;
  // A whole volume in host memory to the output file (float, or bytes).
  auto write_host = [&](const float *v) {
    if (o.f2b) {
      std::vector<float> copy(v, v + nvox);
      std::vector<unsigned char> b = to_bytes(copy, slab, alpha);
      std::vector<float> sec(plane);
      for (size_t i = 0; i < plane; ++i) sec[i] = (float)b[mid * plane + i];
      trcli::update_stats(&out, sec.data(), plane);
      return trcli::write_volume(o.output, out, b.data(), b.size(), &err);
    }
    trcli::update_stats(&out, v + mid * plane, plane);
    return trcli::write_volume(o.output, out, v, nvox * sizeof(float), &err);
  };
  if (st == TR_OK && method == kMethodAdmm) {
    st = tr_admm_host(ctx, proj.data(), vol.data(), o.iteration, o.cgiter, o.gamma, o.soft);
    if (st == TR_OK) ok = write_host(vol.data());
  } else if (st == TR_OK) {
    FileSink k;
    k.f = fopen(o.output.c_str(), "wb");
    if (!k.f) {
      tr_destroy(ctx);
      return fprintf(stderr, "%s: cannot create %s\n", kProg, o.output.c_str()), 1;
    }
    k.es = o.f2b ? 1 : sizeof(float);
    k.mid_off = mid * plane * k.es;
    k.mid_n = plane;
    k.mid.assign(plane, 0.f);
    ok = fwrite(&out, 1, sizeof out, k.f) == sizeof out;  // placeholder header
    if (ok)
      st = tr_reconstruct_to_sink(ctx, method, proj.data(), use_initial ? vol.data() : nullptr,
                                  o.iteration, o.gamma, o.f2b ? slab : 0, alpha, 64u << 20,
                                  file_sink, &k);
    if (ok && st == TR_OK) {
      trcli::update_stats(&out, k.mid.data(), plane);
      ok = fseek(k.f, 0, SEEK_SET) == 0 && fwrite(&out, 1, sizeof out, k.f) == sizeof out;
    }
    ok = (fclose(k.f) == 0) && ok;
    if (!ok) err = "write failed for " + o.output;
    if ((st == TR_ERR_OOM || st == TR_ERR_BUDGET) && method == TR_METHOD_SIRT) {
      // The volume does not fit the device (or its budget): keep it in host
      // memory and stream it through the device in z-slabs, as TiltRecZ
      // streams through managed memory (recon_z.cu:96-100).
      fprintf(stderr, "%s: the volume does not fit the device budget (%s); streaming it "
              "in z-slabs from host memory\n", kProg, tr_last_error(ctx));
      void *hv = nullptr;
      st = tr_host_alloc(nvox * sizeof(float), &hv);
      if (st == TR_OK) {
        float *v = static_cast<float *>(hv);
        if (use_initial) memcpy(v, vol.data(), nvox * sizeof(float));
        int depth = 0;
        st = tr_sirt_host_zslabs(ctx, proj.data(), v, !use_initial, o.iteration, o.gamma, 0,
                                 &depth);
        if (st == TR_OK) {
          printf("%s: z-slab depth %d\n", kProg, depth);
          ok = write_host(v);
        }
        tr_host_free(hv);
      }
    }
  }
  if (st != TR_OK) {
    fprintf(stderr, "%s: %s\n", kProg, tr_last_error(ctx));
    tr_destroy(ctx);
    return 1;
  }
  tr_destroy(ctx);
  if (!ok) return fprintf(stderr, "%s\n", err.c_str()), 1;
  printf("%s: %s %dx%dx%d tilts=%d -> %s\n", kProg, o.method.c_str(), nx, ny, th, nt,
         o.output.c_str());
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  Options o;
  const int r = parse(argc, argv, &o);
  if (r < 0) {
    printf("***WRONG INPUT.\n");
    return 1;
  }
  if (r == 0) return 0;
  if (rank_from_env() != 0) return 0;  // rank 0 reconstructs
  return run(o);
}
