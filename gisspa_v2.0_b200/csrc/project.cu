// project.cu — template generation on the device: projections of a 3D map (the reference's
// emdata::project3d, EMReader/emdata.cpp:891-996, reproduced bit for bit).
//
// One thread per output pixel walks the masked column k = -rmax .. rmax-1 in the reference's
// order.  The in-plane source coordinates are truncated to int in the reference (x2, y2 are
// int, emdata.cpp:899), so its trilinear interpolation keeps only the weight along z:
// (1 - v) p(z) + v p(z + 1) in double (emdata.h:173-179), whose products are exact, summed,
// rounded to float and added in float.  Coordinates are evaluated with round-to-nearest
// intrinsics in the reference's operation order (no contraction into FMAs), so every
// truncation lands where the reference's does.
#include <cmath>

#include "project.cuh"

namespace gisspa {
namespace {

__global__ void project_kernel(const float* __restrict__ vol, ProjGeom g, const float* __restrict__ mx,
                               float* __restrict__ out) {
  const int q = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.nx * g.ny) return;
  const int px = t % g.nx, py = t / g.nx;
  const int i = px - g.nx / 2, j = py - g.ny / 2;
  float acc = 0.f;
  if (i >= g.imin && i < g.imax && j >= g.jmin && j < g.jmax) {
    const float* m = mx + 9 * q;
    const float m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3], m4 = m[4], m5 = m[5], m6 = m[6], m7 = m[7], m8 = m[8];
    const float ix = (float)i, jy = (float)j;
    const float cx = (float)(g.nx / 2), cy = (float)(g.ny / 2), cz = (float)(g.nz / 2);
    // the k-independent parts, in the reference's left-to-right order
    const float ax = __fadd_rn(__fmul_rn(m0, ix), __fmul_rn(m1, jy));
    const float ay = __fadd_rn(__fmul_rn(m3, ix), __fmul_rn(m4, jy));
    const float az = __fadd_rn(__fmul_rn(m6, ix), __fmul_rn(m7, jy));
    const float ij = __fadd_rn(__fmul_rn(ix, ix), __fmul_rn(jy, jy));
    const long long xy = (long long)g.nx * g.ny;
    for (int k = -g.rmax; k < g.rmax; ++k) {
      const float kz = (float)k;
      if (g.r2 < __fadd_rn(ij, __fmul_rn(kz, kz))) continue;
      const int x2 = (int)__fadd_rn(__fadd_rn(ax, __fmul_rn(m2, kz)), cx);
      const int y2 = (int)__fadd_rn(__fadd_rn(ay, __fmul_rn(m5, kz)), cy);
      const float z2 = __fadd_rn(__fadd_rn(az, __fmul_rn(m8, kz)), cz);
      if (x2 < 0 || y2 < 0 || z2 < 0.f || x2 >= g.nx - 1 || y2 >= g.ny - 1 || z2 >= (float)(g.nz - 1)) continue;
      const int z = (int)z2;
      const float v = __fsub_rn(z2, (float)z);
      const long long ii = x2 + (long long)y2 * g.nx + (long long)z * xy;
      const double s = __dadd_rn(__dmul_rn(1.0 - (double)v, (double)__ldg(vol + ii)),
                                 __dmul_rn((double)v, (double)__ldg(vol + ii + xy)));
      acc = __fadd_rn(acc, (float)s);
    }
  }
  out[(size_t)q * g.nx * g.ny + t] = acc;
}

}  // namespace

ProjGeom projection_geometry(int nx, int ny, int nz, int ri) {
  ProjGeom g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  // emdata.cpp:906-939 with scale 1 and no translation
  g.rmax = int((float)ri * 1.0f + 0.5);
  if (g.rmax <= 0) g.rmax = nx / 2;
  g.r2 = (float)(g.rmax * g.rmax);
  g.jmin = std::max(int(-g.rmax + 0.0f + 0.5), -ny / 2);
  g.jmax = std::min(int(g.rmax + 0.0f + 0.5), ny / 2);
  g.imin = std::max(int(-g.rmax + 0.0f + 0.5), -nx / 2);
  g.imax = std::min(int(g.rmax + 0.0f + 0.5), nx / 2);
  return g;
}

void projection_matrices(const float* angles, int n, std::vector<float>& mx) {
  for (int q = 0; q < n; ++q) {
    const double alt = angles[3 * q], az = angles[3 * q + 1], phi = angles[3 * q + 2];
    const double ca = std::cos(alt), sa = std::sin(alt), cz = std::cos(az), sz = std::sin(az), cp = std::cos(phi),
                 sp = std::sin(phi);
    mx.push_back((float)(cp * cz - ca * sz * sp));
    mx.push_back((float)(-(sp * cz + ca * sz * cp)));
    mx.push_back((float)(sa * sz));
    mx.push_back((float)(cp * sz + ca * cz * sp));
    mx.push_back((float)(-sp * sz + ca * cz * cp));
    mx.push_back((float)(-sa * cz));
    mx.push_back((float)(sa * sp));
    mx.push_back((float)(sa * cp));
    mx.push_back((float)ca);
  }
}

void project_volume(const float* d_vol, const ProjGeom& g, const float* d_mx, int n, float* d_out, cudaStream_t s) {
  constexpr int kT = 256;
  dim3 grid((unsigned)ceil_div((long long)g.nx * g.ny, kT), (unsigned)n);
  project_kernel<<<grid, kT, 0, s>>>(d_vol, g, d_mx, d_out);
  GISSPA_LAUNCH_CHECK();
}

}  // namespace gisspa
