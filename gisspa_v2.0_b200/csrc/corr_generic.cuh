// corr_generic.cuh — correlation of (window, template) pairs for window sizes without
// hand-tuned kernels (any even L the reference accepts, e.g. its default 320).
#pragma once

#include "correlate.cuh"
#include "fft_generic.cuh"

namespace gisspa {

// Window sizes with the hand-written two-pass kernels (correlate.cu); every other multiple
// of 16 goes through correlate_generic.
bool correlate_fast(int L);

// True when correlate_generic runs its fused two-pass form for (L, epilogue): L's prime
// factors are 2, 3, 5 and 7 and the row pass's shared memory fits; otherwise it runs the
// unfused form (product, engine transforms, row extension, epilogue kernels).
bool generic_fused(int L, int epi);

// Workspace of correlate_generic for P = E x D pairs: z holds P x (L/2+1) x L complex, x holds
// P x L x L complex (unfused form only; 0 for the fused form).
size_t generic_z_elems(int L, int P);
size_t generic_x_elems(int L, int P, int epi);

// The same launch as correlate_launch (windows b0.., templates n0.., epilogue cl.epi with the
// same arguments and results).  Fused form: a column kernel (product of the half spectra and
// the inverse transforms along ky) and a row kernel (Hermitian rows two at a time through one
// complex transform, the epilogue over the launch's templates in shared memory).  Unfused
// form: product, column transforms on the generic FFT engine, Hermitian row extension, row
// transforms, and the epilogue on the real maps.  Zero lag at (L/2, L/2).  ev (optional,
// three events) brackets the column half and the row half (with the epilogue), as the pass A /
// pass B samples of correlate_launch.
void correlate_generic(const CorrLaunch& cl, const float2* I, const void* T, const CorrArgs& a, FftEngine& fft,
                       float2* z, float2* x, cudaStream_t s, cudaEvent_t* ev = nullptr);

}  // namespace gisspa
