// ref_emdata_min.cpp — TEST INFRASTRUCTURE ONLY.
//
// Minimal definitions of the reference's emdata image reader used when the reference
// search path (GisSPA_v2.0 src/main.cu, norm.cu, nonorm.cu, kernels.cu, ...) is
// compiled by oracle/ref_build.sh to generate golden pick lists.  The reference's
// own reader (src/EMReader/emdata.cpp) needs libhdf5, which this machine lacks;
// the search never reaches HDF5 when templates and micrographs are MRC files, so
// these definitions read little-endian MRC mode 2 (float32) only: section n when
// 0 <= n < nz, otherwise the whole map (emdata.cpp:511-521 semantics).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "emdata.h"

Euler::Euler() {}
Euler::~Euler() {}

emdata::emdata() {
  std::memset(&header, 0, sizeof(header));
  rdata = nullptr;
  mrch = nullptr;
  spiderH = nullptr;
  imagich = nullptr;
  fft = nullptr;
  rfp = nullptr;
}

emdata::~emdata() {
  if (rdata) std::free(rdata);
}

int emdata::readImage(const char* filespec, int n, int) {
  FILE* in = std::fopen(filespec, "rb");
  if (!in) {
    std::printf("Cannot open \"%s\"\n", filespec);
    std::exit(-1);
  }
  int hdr[256];
  if (std::fread(hdr, 4, 256, in) != 256 || hdr[3] != 2) {
    std::fclose(in);
    return -1;
  }
  const int nx = hdr[0], ny = hdr[1], nz = hdr[2], next = hdr[23];
  int z0 = 0, cnt = nz;
  if (n >= 0 && n < nz) {
    z0 = n;
    cnt = 1;
  }
  const size_t sec = (size_t)nx * ny;
  std::fseek(in, 1024L + next + (long)(z0 * sec * 4), SEEK_SET);
  rdata = (float*)std::realloc(rdata, sizeof(float) * sec * cnt);
  const size_t got = std::fread(rdata, sizeof(float), sec * cnt, in);
  std::fclose(in);
  header.nx = nx;
  header.ny = ny;
  header.nz = cnt;
  return got == sec * cnt ? 0 : -1;
}
