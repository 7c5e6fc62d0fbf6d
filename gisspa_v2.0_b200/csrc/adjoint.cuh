// adjoint.cuh — gradient of a pick's normalised score (see adjoint.cu).
#pragma once

#include "common.cuh"
#include "prep.cuh"

namespace gisspa {

struct GradPick {
  int b, n, px, py;        // window, template, window-local pixel of the pick
  float dx, dy, theta;     // shift (pixels) and search angle (degrees)
  float pad;
};

struct GradArgs {
  const float* prep;       // [nt][L][L] prepared templates (real space) at the CTF evaluated
  const float* dprep;      // [3][nt][L][L] d prep / d(dfu, dfv, dfang)
  // The same two arrays stored in the handle's template precision (GISSPA_SPEC_FP16 / BF16:
  // 2-byte values read in place of prep / dprep); precision GISSPA_SPEC_FP32 reads the above.
  const void* prep_lp;
  const void* dprep_lp;
  int precision;
  const float* img;        // [ny][nx] preprocessed micrograph
  int nx, ny;
  const int* offx;
  const int* offy;
  int bx;
  const double* win_m;     // per-window radial RMS factor
  const double* win_sum;   // per-window sum of the filtered window
  const float2* musig;     // [W][L][L] (mu, 1/sigma)
  int L, nt;
  float d_m, ehw;
};

// d(template weight)/d(dfu, dfv, dfang) tables, [3][l][l]
void ctf_dweight(float* dtab, int l, const DevParams& p, cudaStream_t s);
// out[t] = F[t] * tab / m[t]
void scale_by_table(const float2* F, const float* tab, const double* m, int nt, int l, float2* out, cudaStream_t s);
void window_sums(const float* img, int nx, int ny, const int* offx, const int* offy, int bx, int nwin, int l,
                 const double* win_m, double* out, cudaStream_t s);
// prep (n1 values) and dprep (n2) rounded to the template precision (1: FP16, 2: BF16) into out1,
// out2; FP16 first scales both by one power of two that fits their largest value (absmax: one
// unsigned of device scratch)
void round_templates(const float* prep, long long n1, const float* dprep, long long n2, int precision,
                     unsigned* absmax, void* out1, void* out2, cudaStream_t s);
// out: n x 7 floats (z, dz/d(dx, dy, theta, dfu, dfv, dfang))
void score_grads(const GradArgs& g, const GradPick* picks, int n, float* out, cudaStream_t s);

}  // namespace gisspa
