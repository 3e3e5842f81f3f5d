// `resample` drop-in: area binning of an MRC stack on the B200 engine, the
// step the GUI's TiltRec chain runs first when its bin factor exceeds 1
// (src/qmlapp/Autom2qml/CommandChainManager.qml:147-160).
//
//   resample -i/--input <mrc> -o/--output <mrc> -b/--bin <factor>   (-h/--help)
// (resample/src/main/opts.h).  The reference (resample/src/main/main.cpp)
// reads every section as float (mode 0 bytes unsigned and divided by 255,
// mode 1 shorts as their value; mrcimg/mrc2img.cpp:47-108), shrinks it to
// (nx/bin) x (ny/bin) with OpenCV's area resize and writes a float MRC whose
// header is the input's with the new sizes in nx/ny/nz and mx/my/mz and mode
// 2.  Its closing header rewrite (new min/mean/max) goes to a stream that is
// still open (util::MrcStack::WriteHeaderToFile) and never reaches the file,
// so the statistics stay the input's; that is kept here.  The reference
// writes `next` bytes of uninitialised memory as the extended header; here
// they are zeros.
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "mrc_io.h"
#include "tiltrec_b200.h"

int main(int argc, char **argv) {
  std::string input, output;
  int bin = 0;
  const option longopts[] = {{"output", required_argument, nullptr, 'o'},
                             {"input", required_argument, nullptr, 'i'},
                             {"bin", required_argument, nullptr, 'b'},
                             {"help", no_argument, nullptr, 'h'},
                             {nullptr, 0, nullptr, 0}};
  int ch;
  while ((ch = getopt_long(argc, argv, "hi:o:b:", longopts, nullptr)) != -1) {
    switch (ch) {
      case 'i': input = optarg; break;
      case 'o': output = optarg; break;
      case 'b': bin = atoi(optarg); break;
      case 'h':
        printf("resample -i <input.mrc> -o <output.mrc> -b <bin factor >= 1>\n");
        return 0;
      default: return 1;
    }
  }
  if (input.empty() || output.empty() || bin < 1)
    return fprintf(stderr, "resample: --input, --output and --bin >= 1 are required\n"), 1;
  std::string err;
  trcli::MrcHeader h;
  if (!trcli::read_header(input, &h, &err)) return fprintf(stderr, "%s\n", err.c_str()), 1;
  const int nx = h.nx, ny = h.ny, nt = h.nz;
  if (nx / bin < 1 || ny / bin < 1 || bin > 64)
    return fprintf(stderr, "resample: bin %d too large for %dx%d\n", bin, nx, ny), 1;
  std::vector<float> src((size_t)nx * ny * nt);
  if (!trcli::read_sections(input, h, 0, nt, false, src.data(), &err))
    return fprintf(stderr, "%s\n", err.c_str()), 1;
  if (h.mode == trcli::MRC_BYTE)
    for (float &v : src) v = v / 255.0f;
  const int dnx = nx / bin, dny = ny / bin;
  std::vector<float> dst((size_t)dnx * dny * nt);
  int device = 0;
  if (const char *d = getenv("TILTREC_DEVICE")) device = atoi(d);
  const int st = tr_resample_bin_host(device, src.data(), nx, ny, nt, bin, dst.data());
  if (st != TR_OK)
    return fprintf(stderr, "resample: %s\n", tr_status_string(st)), 1;
  trcli::MrcHeader o = h;
  o.nx = dnx;
  o.ny = dny;
  o.nz = nt;
  o.mx = dnx;
  o.my = dny;
  o.mz = nt;
  o.mode = trcli::MRC_FLOAT;
  if (!trcli::write_with_extended(output, o, dst.data(), dst.size(), &err))
    return fprintf(stderr, "%s\n", err.c_str()), 1;
  printf("Binning completed! Output saved to: %s\n", output.c_str());
  return 0;
}
