// MRC file I/O for the TiltRec drop-in executables.
//
// The MRC format fixes a 1024-byte header of 56 32-bit words plus ten 80-byte
// labels; the field order below is that format's (as the reference's
// MRCheader, src/TiltRec/src/mrcmx/mrcheader.h:24-101, also lays it out).
// Data follow the header and `next` bytes of extended header.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

namespace trcli {

#pragma pack(push, 1)
struct MrcHeader {
  int32_t nx, ny, nz, mode;
  int32_t nxstart, nystart, nzstart;
  int32_t mx, my, mz;
  float xlen, ylen, zlen;
  float alpha, beta, gamma;
  int32_t mapc, mapr, maps;
  float amin, amax, amean;
  int16_t ispg, nsymbt;
  int32_t next;
  int16_t creatid;
  char blank[30];
  int16_t nint, nreal, sub, zfac;
  float min2, max2, min3, max3, min4, max4;
  int16_t idtype, lens, nd1, nd2, vd1, vd2;
  float tiltangles[6];
  float xorg, yorg, zorg;
  char cmap[4], stamp[4];
  float rms;
  int32_t nlabl;
  char labels[10][80];
};
#pragma pack(pop)
static_assert(sizeof(MrcHeader) == 1024, "MRC header must be 1024 bytes");

enum { MRC_BYTE = 0, MRC_SHORT = 1, MRC_FLOAT = 2 };

// Reads the header; false if the file cannot be read.
bool read_header(const std::string &path, MrcHeader *h, std::string *err);

// Reads sections [z0, z1) as float.  Mode 0 bytes are read as signed or
// unsigned per `signed_bytes` (the reference reads them signed through
// ReadBlock, mrcstack.cpp:255-262, and unsigned through ReadSlice, :227-231).
bool read_sections(const std::string &path, const MrcHeader &h, int z0, int z1,
                   bool signed_bytes, float *out, std::string *err);

// A new volume header as the reference's InitializeHeader (mrcstack.cpp:57-86)
// followed by SetSize: float (or byte) mode, unit grid and cell, 90-degree
// angles, axes 1/2/3, placeholder stats 0/255/128, creator id 1000.
MrcHeader new_volume_header(int nx, int ny, int nz, bool byte_mode);

// Header statistics as the reference's UpdateHeader (mrcstack.cpp:104-142):
// min, max and mean of the middle section nz/2 only; the running maximum
// starts at FLT_MIN (the smallest positive float), the mean accumulates in
// long double.
void update_stats(MrcHeader *h, const float *section, size_t n);

// Writes header + float data (or bytes when h.mode == MRC_BYTE).
bool write_volume(const std::string &path, const MrcHeader &h, const void *data,
                  size_t bytes, std::string *err);

// Writes header, h.next zero bytes of extended header, then float data.
bool write_with_extended(const std::string &path, const MrcHeader &h, const float *data,
                         size_t count, std::string *err);

// Tilt angles: whitespace-separated floats until the first that fails to
// parse (ReadAngles, main-mpi.cpp:62-83).
bool read_angles(const std::string &path, std::vector<float> *angles, std::string *err);

}  // namespace trcli
