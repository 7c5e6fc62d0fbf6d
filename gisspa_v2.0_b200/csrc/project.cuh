// project.cuh — projections of a 3D map along Euler angles (template generation on the
// device; emdata::project3d, EMReader/emdata.cpp:891-996).
#pragma once

#include <vector>

#include "common.cuh"

namespace gisspa {

// Geometry of one projection set: volume size, mask radius, pixel ranges (emdata.cpp:906-939).
struct ProjGeom {
  int nx, ny, nz;
  int rmax;                     // mask radius: ri, or nx/2 when ri <= 0
  int imin, imax, jmin, jmax;   // projected pixel ranges around the centre
  float r2;                     // rmax^2
};
ProjGeom projection_geometry(int nx, int ny, int nz, int ri);

// Row-major 3x3 rotation (float) per (alt, az, phi) in radians, from C's double cos/sin as the
// reference evaluates them (emdata.cpp:913-921); appended to mx, 9 floats per projection.
void projection_matrices(const float* angles, int n, std::vector<float>& mx);

// out[q][ny][nx] = projection q of vol[nz][ny][nx] with rotation d_mx[q] (device pointers).
void project_volume(const float* d_vol, const ProjGeom& g, const float* d_mx, int n, float* d_out, cudaStream_t s);

}  // namespace gisspa
