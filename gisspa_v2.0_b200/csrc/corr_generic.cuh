// corr_generic.cuh — correlation of (window, template) pairs for window sizes without
// hand-tuned kernels (any even L the reference accepts, e.g. its default 320).
#pragma once

#include "correlate.cuh"
#include "fft_generic.cuh"

namespace gisspa {

// Window sizes with the hand-written two-pass kernels (correlate.cu); every other multiple
// of 16 goes through correlate_generic.
bool correlate_fast(int L);

// Workspace of correlate_generic for P = E x D pairs: z holds P x (L/2+1) x L complex, x holds
// P x L x L complex.
size_t generic_z_elems(int L, int P);
size_t generic_x_elems(int L, int P);

// The same launch as correlate_launch (windows b0.., templates n0.., epilogue cl.epi with the
// same arguments and results), computed with the generic FFT engine: product of the half
// spectra, column inverse transforms, Hermitian row extension, row inverse transforms, and the
// epilogue on the real maps (zero lag moved to (L/2, L/2)).
void correlate_generic(const CorrLaunch& cl, const float2* I, const void* T, const CorrArgs& a, FftEngine& fft,
                       float2* z, float2* x, cudaStream_t s);

}  // namespace gisspa
