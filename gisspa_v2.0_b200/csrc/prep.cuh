// prep.cuh — per-micrograph preparation kernels (everything outside the hot loop).
#pragma once

#include "../../include/gisspa.h"
#include "common.cuh"

namespace gisspa {

// SetParams (norm.cu:183-192) and Parameters (DataReader2.h:73-83), in FP64.
struct DevParams {
  double apix, kk, cs, highres, lowres, d_m, thresh, ehw, ampconst, a, b, b2, bf, bf2, bf3;
  double lambda, dfu, dfv, dfdiff, dfang;
};
DevParams make_params(const gisspa_config& c, const gisspa_ctf& ctf);

// ---- templates
void tmpl_pad(const float* stack, int nt, int tw, int th, int l, float2* out, cudaStream_t s);
// edge mean over the ring + sigma over the padded window, then t <- (t - em) / sigma
void tmpl_edge_normalise(float2* tb, int nt, int l, double* scratch, cudaStream_t s);
// radial power over x <= nx/2, 0 <= r < max(nx, ny)/2: ra[b][r] += |F|^2, rb[r] += 1 (rb shared)
void radial_power(const float2* F, int batch, int nx, int ny, double* ra, unsigned* rb, int nbins, cudaStream_t s);
// F /= sqrt(ra / rb) on valid shells (whiten_Tmp kernels.cu:128-149)
void tmpl_whiten(float2* F, int batch, int l, const double* ra, const unsigned* rb, int nbins, cudaStream_t s);
// soft circular mask on the real part, imaginary part cleared (apply_mask kernels.cu:225-241)
void mask_real(float2* data, int batch, int l, float d_m, float ehw, cudaStream_t s);
// band-pass x |CTF| x SSNR weight table for templates (apply_weighting_function kernels.cu:243-288)
void tmpl_weight_table(float* table, int l, const DevParams& p, cudaStream_t s);
void apply_table(float2* F, int batch, int l, const float* table, cudaStream_t s);
// F /= m, m = sqrt(sum |F|^2 / count^2) over x <= l/2 and valid shells (kernels.cu:319-382 +
// host); m per batch entry is written to factors when not null
void rms_normalise(float2* F, int batch, int l, double* factors, cudaStream_t s);
void real_part(const float2* in, float* out, long long n, float scale, cudaStream_t s);
void to_complex(const float* in, float2* out, long long n, cudaStream_t s);

// ---- micrograph
// LoadImage statistics (norm.cu:157-167): stats = {avg, up_bound, low_bound, clamp}
void image_stats(const float* img, int nx, int ny, bool fp32_serial, float* stats, double* scratch, cudaStream_t s);
// clamp (norm) + invert, to complex
void image_load(const float* img, long long n, const float* stats, bool clamp, bool invert, float2* out,
                cudaStream_t s);
// phase flip (do_phase_flip kernels.cu:828-839)
void phase_flip(float2* G, int nx, int ny, const DevParams& p, cudaStream_t s);
// whiten_filter_weight_Img (kernels.cu:151-202) + optional DC = 0
void image_filter(float2* G, int nx, int ny, const DevParams& p, const double* ra, const unsigned* rb, int nbins,
                  bool zero_dc, cudaStream_t s);

// ---- windows
// out[b] = image[offy + y][offx + x] (0 outside); offsets per axis in offx/offy (device)
void gather_windows(const float* img, int nx, int ny, const int* offx, const int* offy, int bx, int nwin, int l,
                    float2* out, cudaStream_t s);

// ---- rotation (rotate_subIMG kernels.cu:534-603)
// out[n] = mask(rotate(in[n])) as complex (imag 0); sums[n] = {sum, sum of squares} (FP64)
// st (optional): read cos/sin from device memory instead of cose/sine (graph replays).
void rotate_batch(const float* in, int n, int l, float cose, float sine, bool mask, float d_m, float ehw, float2* out,
                  double* sums, cudaStream_t s, const AngleState* st = nullptr);
// Write spectra in the kx-major hot layout and storage precision:
// out[n][kx][ky] = X[n][kx][ky] * scale_n, scale_n = base/sqrt(var_n) when sums are given (and DC = 0:
// the reference subtracts the mean first), base otherwise.  X is [n][l/2+1][l].
// base_scale multiplies the result (1/l^2 for forward spectra of real images).
void finalize_spectra(const float2* X, int n, int l, const double* sums, int spec, void* out, double base_scale,
                      cudaStream_t s);
// Per-window radial RMS scale and repack: out[b][kx][ky] = F[b][ky][kx] / m_b (F is [b][l][l])
void scale_batch(float2* F, int batch, long long per, const double* factors, cudaStream_t s);

}  // namespace gisspa
