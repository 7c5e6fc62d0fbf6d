// correlate.cuh — the hot loop: fused conjugate multiply + 2D C2R inverse FFT +
// per-pixel epilogue for a batch of (window, template) pairs at one angle.
//
// Spectra are stored as half spectra in column-major order, S[kx][ky] with
// kx in [0, L/2] and ky in [0, L) ("kx-major"), the layout the column pass reads.
//   pass A: for every pair and column kx: Z[ky] = I[kx][ky] conj(T[kx][ky]);
//           columns 0 and L/2 (whose inverse transforms are real) are packed into
//           one complex column; inverse FFT of length L along ky -> Q[pair][y][kx].
//   pass B: per output row y, a length-L/2 complex inverse FFT turns the L/2+1
//           Hermitian-half values into L real samples (even/odd interleave);
//           the zero lag is moved to (L/2, L/2) (the reference's (-1)^(kx+ky)
//           factor, kernels.cu:668-677) and the epilogue consumes the row.
// The result equals Re(IFFT2(I conj(T) (-1)^(kx+ky))) of the reference
// (compute_corner_CCG kernels.cu:645-678 + cufftExecC2C norm.cu:536/568).
#pragma once

#include "common.cuh"

namespace gisspa {

enum Epilogue : int {
  EPI_SUM = 0,     // sweep 1: S1 += c, S2 += c^2 (c = CC / L^2), FP64 state
  EPI_CHUNK = 1,   // sweep 2: z = (c - mu) / sigma, 256-pixel chunk max, threshold -> candidates
  EPI_TOPK = 2,    // one sweep: S1, S2 and per-pixel max c with its (angle, template)
  EPI_NONORM = 3,  // norm_type=0: per pair peak (border zeroed), sum, sum of squares of CC
  EPI_MAP = 4,     // write c maps (tests and the no-scratch entry point)
  EPI_SUMMAX = 5   // sweep 1 of a pruned search: S1, S2 and the per-pixel max c (peak key, no index)
};

// A picked chunk (or, for EPI_NONORM, nothing: per-pair reductions go to nn_*).
struct Cand {
  float score;
  int x, y;          // window-local pixel (zero lag at L/2)
  int window, templ, angle, chunk;
  int pad;
};

// Index of the (window, template, angle) pair in the per-pair arrays of a pruned search,
// template-major: the pairs of one launch (a few windows and consecutive templates at one angle)
// fall in different cache lines, and so in different L2 slices, for their atomic maxima.
__host__ __device__ __forceinline__ size_t pair_index(int win, int templ, int angle, int n_windows, int n_angles) {
  return ((size_t)templ * n_windows + win) * n_angles + angle;
}

// What the second sweep of a pruned search skips (null pointers: nothing).  Every pair's z at a
// pixel is at most the z of the pixel's best correlation over all pairs, and a pair's correlation
// is at most its maximum over the window: rows whose pixels cannot reach the threshold, windows
// without such rows and pairs whose maximum stays below every live pixel's bar hold no pick.
struct SkipMask {
  const unsigned char* rows;     // [W][L] by row y of Q (output row (y + L/2) mod L)
  const unsigned char* windows;  // [W]
  const unsigned char* pairs;    // [nt_total][W][n_angles] (pair_index)
  int nt_total, n_windows, n_angles;
  int angle;                      // the launch's angle (set by correlate_launch)
  const AngleState* angle_state;  // when set, the angle index is read here (graph replays)
  __device__ __forceinline__ bool pair_live(int win, int templ) const {
    if (!pairs) return true;
    const int a = angle_state ? angle_state->index : angle;
    return pairs[pair_index(win, templ, a, n_windows, n_angles)] != 0;
  }
};
// Pair masks apply to launches of at most this many templates (pass B lists the live ones).
constexpr int kMaxListedTemplates = 256;

struct CorrArgs {
  const float2* Q;          // pass A output, row-major [pairs][L][L/2] (slot 0 packs columns 0 and L/2)
  unsigned* err;            // set to 1 when a bounded wait gives up
  int D;                    // templates per window in this launch
  int b0, n0;               // first window / template of the launch
  int angle;                // index of the angle in the angle sequence
  const AngleState* angle_state;  // when set, the angle index is read here instead (graph replays)
  int nt_real;              // templates >= nt_real never produce picks
  int nt_total;             // N_T used in the (angle, template) combination index
  // EPI_SUM / EPI_TOPK state, [W][L][L]
  double* S1;
  double* S2;
  // EPI_TOPK: per pixel the best correlation and its index k = angle * nt_total + template,
  // (float_key(c) << 32) | (0xFFFFFFFF - k), 0 = none yet: an integer max keeps the larger c
  // and, on ties, the lower k (the first one a single sweep meets)
  unsigned long long* peak;
  // EPI_CHUNK
  const float2* musig;      // [W][L][L] (mu, 1/sigma or 0)
  float thresh;
  const int* offx;          // window offsets (x of window b % bx), (y of window b / bx)
  const int* offy;
  int bx, nx, ny;
  float dmin;               // centre must lie in [dmin, n - dmin)
  Cand* cand;
  unsigned* cand_count;
  unsigned cand_cap;
  // EPI_CHUNK (optional): rows, windows and pairs that are skipped (their nt_total, n_angles,
  // angle and angle_state are those of the launch)
  SkipMask skip;
  // EPI_SUMMAX (optional): each (window, template, angle) pair's maximum correlation over the
  // window, float_key(c) at pair_index(window, template, angle, n_windows, n_angles)
  unsigned* pair_max;
  int n_windows, n_angles;
  // EPI_NONORM, indexed [window][template] with nt_total templates per window
  unsigned long long* nn_key;
  double* nn_sum;           // [W][nt_total][2]
  float border;             // diameter / 4
  // EPI_MAP, [pairs][L][L]
  float* map_out;
};

struct CorrLaunch {
  int L;
  int E;              // windows in this launch
  int D;              // templates per window in this launch
  int spec;           // GISSPA_SPEC_*
  int epi;            // Epilogue
  int variant = 0;    // pass B shape (see correlate_variants)
  int a_variant = 0;  // pass A shape (see pass_a_variants)
  // Pass A directly follows the previous launch's pass B on the stream and reads nothing that
  // pass B writes: it then waits for it only before storing Q (programmatic dependent launch
  // overlaps the rest with pass B's last CTAs).  Otherwise pass A waits at its start.
  bool chained = false;
  // FP16 template spectra at L = 512: the column pass on the tensor cores (colmma.cu)
  bool tc = false;
};

// Launch pass A then pass B on stream s.  I: window spectra [W][L/2+1][L];
// T: template spectra [N][L/2+1][L] in the storage type of `spec`; Q: scratch.
// Returns the number of kernel launches issued.
// ev (optional): three events recorded before pass A, between the passes and after pass B.
int correlate_launch(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
                     const float2* twL, const float2* twNZ, cudaStream_t s, cudaEvent_t* ev = nullptr);

// The pair engine (pair_engine.cu): one launch runs pass A of one batch and pass B of the batch
// before it, so that the load-bound and the issue-bound pass share the SMs.  Window 512, epilogues
// EPI_SUM, EPI_SUMMAX, EPI_TOPK and EPI_CHUNK.
struct EngineBatch {
  int valid;          // 0: no such pass in this launch
  int b0, n0, d, e;   // first window, first template, templates, windows
  float2* Q;          // the batch's Q slot, row-major [d * e pairs][L][L/2]
};
bool engine_supported(int L, int epi);
// Counters one engine launch uses (zeroed before the launch sequence).
size_t engine_counter_ints();
// b_args: the epilogue's arguments (its Q, b0, n0 and D are taken from B).  chained: the launch
// before on the stream belongs to the same sequence (and its pass B reads the Q slot that this
// launch's pass A writes).
void engine_launch(int spec, int epi, const float2* I, const void* T, const EngineBatch& A, const EngineBatch& B,
                   const CorrArgs& b_args, int* ctr, bool chained, const float2* twL, const float2* twNZ,
                   cudaStream_t s);

// Number of pass A shapes compiled for a window size.
int pass_a_variants(int L);
// The pass B shape index that selects the pair engine at window size L (-1: none).
int engine_variant(int L);

// Whether a window size has compiled correlation kernels.
// One input of a row's half-length inverse transform: from the row's Hermitian half (slot 0
// packing the kx = 0 and kx = L/2 terms as its real and imaginary parts), Z[k] = E[k] +
// i W_L^-k O[k] with E, O the even and odd parts (tw_l: e^(-2 pi i k / L), k < NZ).
// MAYBE_ZERO = false: the caller knows k > 0 (every input of a lane but its first).
template <int NZ, bool MAYBE_ZERO = true>
__device__ __forceinline__ float2 row_unpack(const float2* row, const float2* tw_l, int k) {
  float2 xk, xm;
  if (MAYBE_ZERO && k == 0) {
    const float2 q = row[0];
    xk = make_float2(q.x, 0.f);
    xm = make_float2(q.y, 0.f);
  } else {
    xk = row[k];
    xm = row[NZ - k];
  }
  const float2 ev = make_float2(xk.x + xm.x, xk.y - xm.y);
  const float2 od = make_float2(xk.x - xm.x, xk.y + xm.y);
  float2 w = tw_l[k];
  w.y = -w.y;
  const float2 o = cmul(w, od);
  return make_float2(ev.x - o.y, ev.y + o.x);
}

// Pass A on the tensor cores (colmma.cu): FP16 template spectra at L = 512.
void launch_a_tc(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
                 const float2* twL, cudaStream_t s);
// Pass B on the tensor cores with the top-K epilogue (colmma.cu): FP16 template spectra at L = 512.
void launch_b_tc(const CorrLaunch& cl, const CorrArgs& args, const float2* twL, const float2* twNZ, cudaStream_t s);
bool correlate_supported(int L);
// Number of pass B shapes compiled for a window size (the autotuner's choices).
int correlate_variants(int L);
// Whether pass B shape `variant` has epilogue `epi`.
bool correlate_variant_ok(int L, int variant, int epi);

}  // namespace gisspa
