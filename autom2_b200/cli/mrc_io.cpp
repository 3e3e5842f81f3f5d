// MRC file I/O for the TiltRec drop-in executables (see mrc_io.h).
#include "mrc_io.h"

#include <float.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <fstream>

namespace trcli {

namespace {
bool fail(std::string *err, const std::string &msg) {
  if (err) *err = msg;
  return false;
}
}  // namespace

bool read_header(const std::string &path, MrcHeader *h, std::string *err) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return fail(err, "cannot open " + path);
  const size_t got = fread(h, 1, sizeof(*h), f);
  fclose(f);
  if (got != sizeof(*h)) return fail(err, "short MRC header in " + path);
  if (h->nx <= 0 || h->ny <= 0 || h->nz <= 0)
    return fail(err, "bad MRC dimensions in " + path);
  if (h->mode != MRC_BYTE && h->mode != MRC_SHORT && h->mode != MRC_FLOAT)
    return fail(err, "unsupported MRC mode " + std::to_string(h->mode) + " in " + path);
  return true;
}

bool read_sections(const std::string &path, const MrcHeader &h, int z0, int z1,
                   bool signed_bytes, float *out, std::string *err) {
  const size_t psize = h.mode == MRC_FLOAT ? 4 : (h.mode == MRC_SHORT ? 2 : 1);
  const size_t plane = (size_t)h.nx * h.ny;
  const size_t n = plane * (size_t)(z1 - z0);
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return fail(err, "cannot open " + path);
  const long long off = (long long)sizeof(MrcHeader) + h.next + (long long)z0 * plane * psize;
  if (fseeko(f, off, SEEK_SET) != 0) {
    fclose(f);
    return fail(err, "seek failed in " + path);
  }
  bool ok = true;
  if (h.mode == MRC_FLOAT) {
    ok = fread(out, 4, n, f) == n;
  } else {
    std::vector<unsigned char> buf(n * psize);
    ok = fread(buf.data(), 1, buf.size(), f) == buf.size();
    for (size_t i = 0; ok && i < n; ++i) {
      if (h.mode == MRC_SHORT) {
        int16_t v;
        memcpy(&v, &buf[2 * i], 2);
        out[i] = (float)v;
      } else {
        out[i] = signed_bytes ? (float)(signed char)buf[i] : (float)buf[i];
      }
    }
  }
  fclose(f);
  if (!ok) return fail(err, "short read in " + path);
  return true;
}

MrcHeader new_volume_header(int nx, int ny, int nz, bool byte_mode) {
  MrcHeader h;
  memset(&h, 0, sizeof(h));
  h.mode = byte_mode ? MRC_BYTE : MRC_FLOAT;
  h.mx = h.my = h.mz = 1;
  h.xlen = h.ylen = h.zlen = 1;
  h.alpha = h.beta = h.gamma = 90;
  h.mapc = 1;
  h.mapr = 2;
  h.maps = 3;
  h.amin = 0;
  h.amax = 255;
  h.amean = 128;
  h.creatid = 1000;
  h.nx = nx;
  h.ny = ny;
  h.nz = nz;
  return h;
}

void update_stats(MrcHeader *h, const float *sec, size_t n) {
  float amin = FLT_MAX, amax = FLT_MIN;
  long double amean = 0;
  for (size_t i = n; i--;) {
    if (sec[i] > amax) amax = sec[i];
    if (sec[i] < amin) amin = sec[i];
    amean += sec[i];
  }
  amean /= n;
  h->amin = amin;
  h->amax = amax;
  h->amean = (float)amean;
  h->nlabl = 0;
}

bool write_volume(const std::string &path, const MrcHeader &h, const void *data,
                  size_t bytes, std::string *err) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return fail(err, "cannot create " + path);
  bool ok = fwrite(&h, 1, sizeof(h), f) == sizeof(h);
  const char *p = (const char *)data;
  size_t done = 0;
  while (ok && done < bytes) {
    const size_t chunk = std::min<size_t>(bytes - done, (size_t)1 << 30);
    ok = fwrite(p + done, 1, chunk, f) == chunk;
    done += chunk;
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(err, "write failed for " + path);
  return true;
}

bool write_with_extended(const std::string &path, const MrcHeader &h, const float *data,
                         size_t count, std::string *err) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return fail(err, "cannot create " + path);
  bool ok = fwrite(&h, 1, sizeof(h), f) == sizeof(h);
  if (ok && h.next > 0) {
    std::vector<char> zeros((size_t)h.next, 0);
    ok = fwrite(zeros.data(), 1, zeros.size(), f) == zeros.size();
  }
  if (ok) ok = fwrite(data, sizeof(float), count, f) == count;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(err, "write failed for " + path);
  return true;
}

bool read_angles(const std::string &path, std::vector<float> *angles, std::string *err) {
  std::ifstream in(path);
  if (!in.good()) return fail(err, "cannot open tilt file " + path);
  while (in.good()) {
    float v;
    in >> v;
    if (in.fail()) break;
    angles->push_back(v);
  }
  return true;
}

}  // namespace trcli
