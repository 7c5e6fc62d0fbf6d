// Projection harness over the reference's own emdata::project3d (src/EMReader/emdata.cpp:
// 891-996), linked from the unmodified reference sources by oracle/ref_project.sh
// (TEST INFRASTRUCTURE ONLY: it produces golden projections).
//
//   ref_project <volume.mrc> <ri> <angles.txt> <out.raw>
//   angles.txt: one "alt az phi" line per projection, radians (project3d's units);
//   out.raw: float32 [n][ny][nx].
//
// project3d reads three members that the reference never sets on this path:
//  * nz, the volume depth (emdata.cpp:958): readMRC assigns locals that shadow the members
//    (emdata.cpp:426-428), so after readImage the member is stale.  applyMask with a type it
//    has no case for sets nx, ny, nz from the header and leaves the data alone
//    (emdata.cpp:998-1008): the harness calls it, as a caller of the reference must;
//  * dx, dy, the projection's translation (emdata.cpp:934-935): emdata::emdata() initialises
//    header.dx/dy only (emdata.cpp:133-158).  Every emdata here is built in zero-filled
//    storage: dx = dy = 0, the translation-free projection.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "emdata.h"

namespace {
emdata* make_zeroed() {
  void* p = ::operator new(sizeof(emdata));
  std::memset(p, 0, sizeof(emdata));
  return new (p) emdata();
}
}  // namespace

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s volume.mrc ri angles.txt out.raw\n", argv[0]);
    return 2;
  }
  emdata* vol = make_zeroed();
  if (vol->readImage(argv[1], -1) != 0) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 1;
  }
  vol->applyMask(1, 0, 0.f, 0.f, 0.f);  // type 0: members from the header, data unchanged
  const int ri = std::atoi(argv[2]);
  FILE* fa = std::fopen(argv[3], "r");
  FILE* fo = std::fopen(argv[4], "wb");
  if (!fa || !fo) return 1;
  float alt, az, phi;
  int n = 0;
  while (std::fscanf(fa, "%f %f %f", &alt, &az, &phi) == 3) {
    emdata* proj = make_zeroed();
    vol->project3d(proj, alt, az, phi, -6, 1.0f, ri);
    std::fwrite(proj->getData(), sizeof(float), (size_t)proj->xSize() * proj->ySize(), fo);
    ++n;
  }
  std::fclose(fo);
  std::fclose(fa);
  std::printf("%d projections of %dx%dx%d\n", n, vol->xSize(), vol->ySize(), vol->zSize());
  return 0;
}
