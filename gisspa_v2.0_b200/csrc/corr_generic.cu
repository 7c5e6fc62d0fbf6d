// corr_generic.cu — the correlation and its epilogues for window sizes without hand-tuned
// kernels.  Same results as pass A + pass B (correlate.cu) within FP32 rounding: the
// transforms run in shared memory (mixed radix 2/3/4/5/7) in a fused two-pass form, or on the
// generic FFT engine (Bluestein for other lengths) in an unfused form; the epilogues reproduce
// pass B's per-pixel sums and maxima, chunk picks with the reference's tie order, norm_type=0
// peaks and sums, and maps.  The reference's chunks are 256 consecutive pixels of the window's
// linear index (norm.cu:583-597), so for L that is not a multiple of 256 they straddle rows:
// the chunk scans work on linear indices.
#include "../../include/gisspa.h"
#include "corr_generic.cuh"
#include "fft_smooth.cuh"

namespace gisspa {
namespace {

constexpr int kT = 256;

// Z[p][kx][ky] = I[b0 + e][kx][ky] conj(T[n0 + d][kx][ky]), p = e D + d (half spectra, kx-major)
template <typename SPEC>
__global__ void gen_product_kernel(const float2* __restrict__ I, const typename SPEC::T* __restrict__ T, int b0,
                                   int n0, int D, long long H, float2* __restrict__ Z) {
  const int p = blockIdx.y, e = p / D, d = p - e * D;
  const float2* Ib = I + (size_t)(b0 + e) * H;
  const typename SPEC::T* Tn = T + (size_t)(n0 + d) * H;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < H; k += (long long)gridDim.x * blockDim.x)
    Z[(size_t)p * H + k] = cmulc(Ib[k], SPEC::load(Tn + k));
}

// After the column transforms Z[p][kx][y] holds row y's half spectrum over kx <= L/2; each
// row of a real map is Hermitian: X[p][y][k] = Z[p][k][y] (k <= L/2), conj(Z[p][L - k][y]).
__global__ void gen_hermitian_rows_kernel(const float2* __restrict__ Z, int L, float2* __restrict__ X) {
  const int p = blockIdx.y;
  const long long L2 = (long long)L * L, H = (long long)(L / 2 + 1) * L;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < L2; q += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(q / L), k = (int)(q - (long long)y * L);
    float2 v;
    if (k <= L / 2) {
      v = Z[(size_t)p * H + (size_t)k * L + y];
    } else {
      const float2 w = Z[(size_t)p * H + (size_t)(L - k) * L + y];
      v = make_float2(w.x, -w.y);
    }
    X[(size_t)p * L2 + q] = v;
  }
}

// raw correlation at the shifted window pixel (oy, ox): the zero lag sits at (L/2, L/2)
__device__ __forceinline__ float gen_raw(const float2* X, int p, int L, int oy, int ox) {
  const int y = oy + L / 2 - (oy + L / 2 >= L ? L : 0), x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
  return X[(size_t)p * L * L + (size_t)y * L + x].x;
}

// EPI_SUM / EPI_TOPK: per window pixel over the launch's D templates, folded into the state
__global__ void gen_sum_kernel(const float2* __restrict__ X, CorrArgs a, int L, int topk) {
  const int e = blockIdx.y;
  const long long L2 = (long long)L * L;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= L2) return;
  const int oy = (int)(q / L), ox = (int)(q - (long long)oy * L);
  const float inv = 1.0f / (float)L2;
  const int angle = a.angle_state ? a.angle_state->index : a.angle;
  float s1 = 0.f, s2 = 0.f, best = -INFINITY;
  int barg = -1;
  for (int d = 0; d < a.D; ++d) {
    const float c = gen_raw(X, e * a.D + d, L, oy, ox) * inv;
    s1 += c;
    s2 = fmaf(c, c, s2);
    if (c > best) {
      best = c;
      barg = angle * a.nt_total + a.n0 + d;
    }
  }
  const size_t pix = (size_t)(a.b0 + e) * L2 + q;
  atomicAdd(a.S1 + pix, (double)s1);
  atomicAdd(a.S2 + pix, (double)s2);
  if (topk && barg >= 0)
    atomicMax(a.peak + pix, ((unsigned long long)float_key(best) << 32) | (unsigned)(0xFFFFFFFFu - (unsigned)barg));
}

// block-wide max of a u64 key (blockDim.x == kT)
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long k, unsigned long long* sh) {
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xffffffffu, k, off);
    k = o > k ? o : k;
  }
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = k;
  __syncthreads();
  if (threadIdx.x < 32) {
    k = threadIdx.x < kT / 32 ? sh[threadIdx.x] : 0ull;
    for (int off = 16; off > 0; off >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, k, off);
      k = o > k ? o : k;
    }
  }
  return k;  // valid in thread 0
}

// EPI_CHUNK: one block per (chunk, pair): z-score, chunk max with the reference's tie order
// (the lowest bit-reversed position wins), threshold and centre test -> candidate
__global__ void gen_chunk_kernel(const float2* __restrict__ X, CorrArgs a, int L) {
  __shared__ unsigned long long sh[kT / 32];
  const int p = blockIdx.y, e = p / a.D, d = p - e * a.D, win = a.b0 + e;
  const int chunk = blockIdx.x, t = threadIdx.x;
  const long long L2 = (long long)L * L, q = (long long)chunk * 256 + t;
  const int oy = (int)(q / L), ox = (int)(q - (long long)oy * L);
  const float c = gen_raw(X, p, L, oy, ox) / (float)L2;
  const float2 m = a.musig[(size_t)win * L2 + q];
  const float z = (c - m.x) * m.y;
  const unsigned long long key = ((unsigned long long)float_key(z) << 32) | (unsigned)(255 - brev8(t));
  const unsigned long long best = block_max_u64(key, sh);
  if (threadIdx.x != 0) return;
  const float zb = key_float((uint32_t)(best >> 32));
  if (!(zb >= a.thresh)) return;
  const int tb = brev8(255 - (unsigned)(best & 0xffu));
  const int id = chunk * 256 + tb;
  const int px = id % L, py = id / L;
  const int cx = a.offx[win % a.bx] + px, cy = a.offy[win / a.bx] + py;
  if (!(cx >= a.dmin && cx < a.nx - a.dmin && cy >= a.dmin && cy < a.ny - a.dmin)) return;
  const unsigned slot = atomicAdd(a.cand_count, 1u);
  if (slot >= a.cand_cap) return;
  Cand cd;
  cd.score = zb;
  cd.x = px;
  cd.y = py;
  cd.window = win;
  cd.templ = a.n0 + d;
  cd.angle = a.angle_state ? a.angle_state->index : a.angle;
  cd.chunk = chunk;
  cd.pad = 0;
  a.cand[slot] = cd;
}

// EPI_NONORM: one block per (chunk, pair): peak with the border zeroed (the largest value,
// then the lowest chunk, then the reference's in-chunk order) and the sums of the raw map
__global__ void gen_nonorm_kernel(const float2* __restrict__ X, CorrArgs a, int L) {
  __shared__ unsigned long long sh[kT / 32];
  __shared__ double s1s[kT / 32], s2s[kT / 32];
  const int p = blockIdx.y, e = p / a.D, d = p - e * a.D, win = a.b0 + e;
  const int chunk = blockIdx.x, t = threadIdx.x;
  const long long q = (long long)chunk * 256 + t;
  const int oy = (int)(q / L), ox = (int)(q - (long long)oy * L);
  const float v = gen_raw(X, p, L, oy, ox);
  double s1 = v, s2 = (double)v * v;
  for (int off = 16; off > 0; off >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
  }
  if ((t & 31) == 0) {
    s1s[t >> 5] = s1;
    s2s[t >> 5] = s2;
  }
  float val = v;
  if (ox < a.border || ox > L - a.border || oy < a.border || oy > L - a.border) val = 0.f;
  const unsigned long long key = ((unsigned long long)float_key(val) << 32) | (unsigned)(255 - brev8(t));
  const unsigned long long best = block_max_u64(key, sh);  // includes a __syncthreads
  if (t != 0) return;
  double b1 = 0, b2 = 0;
  for (int w = 0; w < kT / 32; ++w) {
    b1 += s1s[w];
    b2 += s2s[w];
  }
  const size_t qq = (size_t)win * a.nt_total + a.n0 + d;
  atomicAdd(a.nn_sum + 2 * qq, b1);
  atomicAdd(a.nn_sum + 2 * qq + 1, b2);
  const float vb = key_float((uint32_t)(best >> 32));
  if (vb > 0.f) {
    const unsigned long long g =
        ((unsigned long long)float_key(vb) << 32) | ((unsigned long long)(0xFFFFFu - chunk) << 8) | (best & 0xffu);
    atomicMax(a.nn_key + qq, g);
  }
}

// EPI_MAP: c maps [pair][L][L], zero lag at (L/2, L/2)
__global__ void gen_map_kernel(const float2* __restrict__ X, CorrArgs a, int L) {
  const int p = blockIdx.y;
  const long long L2 = (long long)L * L;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= L2) return;
  const int oy = (int)(q / L), ox = (int)(q - (long long)oy * L);
  a.map_out[(size_t)p * L2 + q] = gen_raw(X, p, L, oy, ox) / (float)L2;
}

// ---- fused two-pass form for window sizes whose prime factors are 2, 3, 5 and 7

// Rows per CTA of gen_rows_kernel: even, a divisor of L, about 1280 pixels per CTA, and for
// the chunk scans (EPI_CHUNK, EPI_NONORM) RB L a multiple of 256; 0 when no such RB exists.
__host__ __device__ constexpr int gen_rows_rb(int L, int epi) {
  int rb0 = 1;
  if (epi == EPI_CHUNK || epi == EPI_NONORM) {
    int g = 256;
    while (L % g) g >>= 1;
    rb0 = 256 / g;
  }
  const int step = rb0 % 2 ? 2 * rb0 : rb0;
  int rb = step;
  while (rb * L < 1280 && rb + step <= L) rb += step;
  while (rb <= L && L % rb) rb += step;
  return rb <= L ? rb : 0;
}


// Column pass: rows gr = p (L/2+1) + kx of the launch's half-spectrum products
// I[b0 + e][kx][.] conj(T[n0 + d][kx][.]) (p = e D + d), each inverse-transformed along ky in
// shared memory: Z[p][kx][y].
template <int LC, typename SPEC>
__global__ void gen_cols_kernel(const float2* __restrict__ I, const typename SPEC::T* __restrict__ T, int b0, int n0,
                                int D, int L_, long long nrows, int rpc, SmoothPlan plan, const float2* __restrict__ tw,
                                float2* __restrict__ Z) {
  extern __shared__ float2 sm[];
  const int L = LC ? LC : L_;
  const int hz = L / 2 + 1;
  const long long H = (long long)hz * L;
  const long long row0 = (long long)blockIdx.x * rpc;
  const int rows_here = (int)min((long long)rpc, nrows - row0);
  float2* a = sm;
  float2* b = sm + (size_t)rpc * L;
  for (int i = threadIdx.x; i < rows_here * L; i += blockDim.x) {
    const int r = i / L, k = i - r * L;
    const long long gr = row0 + r;
    const int p = (int)(gr / hz), kx = (int)(gr - (long long)p * hz);
    const int e = p / D, d = p - e * D;
    a[i] = cmulc(I[(size_t)(b0 + e) * H + (size_t)kx * L + k],
                 SPEC::load(T + (size_t)(n0 + d) * H + (size_t)kx * L + k));
  }
  __syncthreads();
  const float2* f = smooth_stages_l<LC, 1>(a, b, rows_here, L, L, plan, tw);
  for (int i = threadIdx.x; i < rows_here * L; i += blockDim.x) Z[(size_t)row0 * L + i] = f[i];
}

// Row pass: one CTA per (block of RB window rows, window of the launch), over the launch's D
// templates.  Window (state) row Y0 + r is transform row (Y0 + r + L/2) mod L, and state
// column ox is transform column (ox + L/2) mod L (zero lag at (L/2, L/2)).  Rows r and
// r + RB/2 are real, so their Hermitian spectra X_r[k] (= Z[p][k][y] for k <= L/2,
// conj Z[p][L-k][y] above) go through one complex transform as X_r + i X_{r+RB/2}: the real
// and imaginary parts of the result are the two rows.  Thread t holds the CTA's pixels
// q = 256 i + t (state linear index Y0 L + q, q < RB L); for the chunk scans (EPI_CHUNK,
// EPI_NONORM) RB L is a multiple of 256, so these are whole chunks of the reference's
// 256-pixel scan and q = 256 i + t is pixel t of the CTA's chunk i.  The rows of up to TB
// templates go through one transform pass (fewer block barriers, more butterflies per thread);
// the epilogue then takes those templates in order.
template <int LC, int EPI>
__global__ void __launch_bounds__(256) gen_rows_kernel(const float2* __restrict__ Z, CorrArgs a, int L_, int RB_,
                                                       int TB, SmoothPlan plan, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int kRB = LC ? gen_rows_rb(LC, EPI) : 0;
  static_assert(LC == 0 || kRB > 0, "no row block for LC");
  const int L = LC ? LC : L_, RB = LC ? kRB : RB_, ld = L + 1;
  const int hr = RB / 2, npix = RB * L, nch = npix / 256, t = threadIdx.x, lane = t & 31, wid = t >> 5;
  float2* buf0 = sm;  // TB templates x hr complex rows, row stride ld
  float2* buf1 = sm + (size_t)TB * hr * ld;
  unsigned long long* red = reinterpret_cast<unsigned long long*>(sm + (size_t)2 * TB * hr * ld);  // [nch][8]
  double* dred = reinterpret_cast<double*>(red + (size_t)nch * 8);                            // [2][8]
  char* st = reinterpret_cast<char*>(dred + 16);
  const int e = blockIdx.y, win = a.b0 + e, Y0 = blockIdx.x * RB;
  const long long L2 = (long long)L * L, H = (long long)(L / 2 + 1) * L;
  const size_t wpix = (size_t)win * L2 + (size_t)Y0 * L;
  const float inv = 1.0f / (float)L2;
  const int angle = a.angle_state ? a.angle_state->index : a.angle;
  float* s1 = reinterpret_cast<float*>(st);  // SUM / TOPK per-pixel accumulators
  float* s2 = s1 + npix;
  float* bst = s2 + npix;
  int* barg = reinterpret_cast<int*>(bst + npix);
  float2* ms = reinterpret_cast<float2*>(st);  // CHUNK: (mu, 1/sigma) of the CTA's pixels
  if constexpr (EPI == EPI_SUM || EPI == EPI_TOPK) {
    for (int q = t; q < npix; q += 256) {
      s1[q] = 0.f;
      s2[q] = 0.f;
      if constexpr (EPI == EPI_TOPK) {
        bst[q] = -INFINITY;
        barg[q] = -1;
      }
    }
  }
  if constexpr (EPI == EPI_CHUNK)
    for (int q = t; q < npix; q += 256) ms[q] = a.musig[wpix + q];

  for (int d0 = 0; d0 < a.D; d0 += TB) {
    const int nd = min(TB, a.D - d0);
    for (int idx = t; idx < nd * hr * L; idx += 256) {
      const int g = idx / (hr * L), rem = idx - g * (hr * L);
      const int k = rem / hr, r2 = rem - k * hr;
      const float2* Zp = Z + (size_t)(e * a.D + d0 + g) * H;
      const int ya = (Y0 + r2 + L / 2) % L, yb = (Y0 + r2 + hr + L / 2) % L;
      float2 A, B;
      if (k <= L / 2) {
        A = Zp[(size_t)k * L + ya];
        B = Zp[(size_t)k * L + yb];
      } else {
        A = Zp[(size_t)(L - k) * L + ya];
        B = Zp[(size_t)(L - k) * L + yb];
        A.y = -A.y;
        B.y = -B.y;
      }
      buf0[(size_t)(g * hr + r2) * ld + k] = make_float2(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    const float2* fg = smooth_stages_l<LC, 1>(buf0, buf1, nd * hr, L, ld, plan, tw);

    // the group's templates in order, so every pixel folds them as the one-at-a-time sweep would
    for (int g = 0; g < nd; ++g) {
      const int d = d0 + g, p = e * a.D + d;
      const float2* f = fg + (size_t)g * hr * ld;

      if constexpr (EPI == EPI_SUM || EPI == EPI_TOPK) {
        for (int q = t; q < npix; q += 256) {
          const int r = q / L, ox = q - r * L, x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
          const float2 w = f[(size_t)(r < hr ? r : r - hr) * ld + x];
          const float c = (r < hr ? w.x : w.y) * inv;
          s1[q] += c;
          s2[q] = fmaf(c, c, s2[q]);
          if constexpr (EPI == EPI_TOPK) {
            if (c > bst[q]) {
              bst[q] = c;
              barg[q] = angle * a.nt_total + a.n0 + d;
            }
          }
        }
      } else if constexpr (EPI == EPI_CHUNK) {
        bool hit = false;
        for (int q = t; q < npix; q += 256) {
          const int r = q / L, ox = q - r * L, x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
          const float2 w = f[(size_t)(r < hr ? r : r - hr) * ld + x];
          const float z = ((r < hr ? w.x : w.y) * inv - ms[q].x) * ms[q].y;
          hit = hit || z >= a.thresh;
        }
        if (__syncthreads_or(hit)) {  // CTA-uniform
          for (int i = 0; i < nch; ++i) {
            const int q = 256 * i + t;
            const int r = q / L, ox = q - r * L, x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
            const float2 w = f[(size_t)(r < hr ? r : r - hr) * ld + x];
            const float z = ((r < hr ? w.x : w.y) * inv - ms[q].x) * ms[q].y;
            unsigned long long key = ((unsigned long long)float_key(z) << 32) | (unsigned)(255 - brev8(t));
            for (int off = 16; off > 0; off >>= 1) {
              const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
              key = o > key ? o : key;
            }
            if (lane == 0) red[i * 8 + wid] = key;
          }
          __syncthreads();
          for (int i = t; i < nch; i += 256) {
            unsigned long long best = 0;
            for (int w = 0; w < 8; ++w) best = red[i * 8 + w] > best ? red[i * 8 + w] : best;
            const float zb = key_float((uint32_t)(best >> 32));
            if (!(zb >= a.thresh)) continue;
            const int id = Y0 * L + i * 256 + brev8(255 - (unsigned)(best & 0xffu));
            const int px = id % L, py = id / L;
            const int cx = a.offx[win % a.bx] + px, cy = a.offy[win / a.bx] + py;
            if (!(cx >= a.dmin && cx < a.nx - a.dmin && cy >= a.dmin && cy < a.ny - a.dmin)) continue;
            const unsigned slot = atomicAdd(a.cand_count, 1u);
            if (slot >= a.cand_cap) continue;
            Cand cd;
            cd.score = zb;
            cd.x = px;
            cd.y = py;
            cd.window = win;
            cd.templ = a.n0 + d;
            cd.angle = angle;
            cd.chunk = id >> 8;
            cd.pad = 0;
            a.cand[slot] = cd;
          }
        }
      } else if constexpr (EPI == EPI_NONORM) {
        double t1 = 0.0, t2 = 0.0;
        for (int i = 0; i < nch; ++i) {
          const int q = 256 * i + t;
          const int r = q / L, ox = q - r * L, oy = Y0 + r, x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
          const float2 w = f[(size_t)(r < hr ? r : r - hr) * ld + x];
          const float v = r < hr ? w.x : w.y;
          t1 += v;
          t2 += (double)v * v;
          float val = v;
          if (ox < a.border || ox > L - a.border || oy < a.border || oy > L - a.border) val = 0.f;
          unsigned long long key = ((unsigned long long)float_key(val) << 32) | (unsigned)(255 - brev8(t));
          for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
            key = o > key ? o : key;
          }
          if (lane == 0) red[i * 8 + wid] = key;
        }
        for (int off = 16; off > 0; off >>= 1) {
          t1 += __shfl_xor_sync(0xffffffffu, t1, off);
          t2 += __shfl_xor_sync(0xffffffffu, t2, off);
        }
        if (lane == 0) {
          dred[wid] = t1;
          dred[8 + wid] = t2;
        }
        __syncthreads();
        const size_t qq = (size_t)win * a.nt_total + a.n0 + d;
        if (t == 0) {
          double b1 = 0, b2 = 0;
          for (int w = 0; w < 8; ++w) {
            b1 += dred[w];
            b2 += dred[8 + w];
          }
          atomicAdd(a.nn_sum + 2 * qq, b1);
          atomicAdd(a.nn_sum + 2 * qq + 1, b2);
        }
        for (int i = t; i < nch; i += 256) {
          unsigned long long best = 0;
          for (int w = 0; w < 8; ++w) best = red[i * 8 + w] > best ? red[i * 8 + w] : best;
          const float vb = key_float((uint32_t)(best >> 32));
          if (vb > 0.f) {
            const int chunk = Y0 * L / 256 + i;
            atomicMax(a.nn_key + qq, ((unsigned long long)float_key(vb) << 32) |
                                         ((unsigned long long)(0xFFFFFu - chunk) << 8) | (best & 0xffu));
          }
        }
      } else if constexpr (EPI == EPI_MAP) {
        float* out = a.map_out + (size_t)p * L2 + (size_t)Y0 * L;
        for (int q = t; q < npix; q += 256) {
          const int r = q / L, ox = q - r * L, x = ox + L / 2 - (ox + L / 2 >= L ? L : 0);
          const float2 w = f[(size_t)(r < hr ? r : r - hr) * ld + x];
          out[q] = (r < hr ? w.x : w.y) * inv;
        }
      }
      if constexpr (EPI == EPI_CHUNK || EPI == EPI_NONORM) __syncthreads();  // reduction slots reused next
    }
    __syncthreads();  // the transform buffers are rewritten next
  }

  if constexpr (EPI == EPI_SUM || EPI == EPI_TOPK) {
    for (int q = t; q < npix; q += 256) {
      atomicAdd(a.S1 + wpix + q, (double)s1[q]);
      atomicAdd(a.S2 + wpix + q, (double)s2[q]);
      if constexpr (EPI == EPI_TOPK) {
        if (barg[q] >= 0)
          atomicMax(a.peak + wpix + q,
                    ((unsigned long long)float_key(bst[q]) << 32) | (unsigned)(0xFFFFFFFFu - (unsigned)barg[q]));
      }
    }
  }
}

size_t gen_rows_smem(int L, int RB, int epi, int tb) {
  const size_t ld = (size_t)L + 1, npix = (size_t)RB * L, nch = npix / 256;
  size_t b = sizeof(float2) * tb * RB * ld + sizeof(unsigned long long) * nch * 8 + sizeof(double) * 16;
  if (epi == EPI_SUM || epi == EPI_TOPK) b += 16 * npix;
  if (epi == EPI_CHUNK) b += sizeof(float2) * npix;
  return b;
}

constexpr size_t kGenSmemMax = 200 * 1024;

// Templates per transform pass of gen_rows_kernel: up to kGenTB as the shared memory allows.
constexpr int kGenTB = 4;
int gen_rows_tb(int L, int RB, int epi) {
  int tb = kGenTB;
  while (tb > 1 && gen_rows_smem(L, RB, epi, tb) > kGenSmemMax) tb /= 2;
  return tb;
}

// The row kernels of one epilogue (compiled for L = 320, and for any L): raises their dynamic
// shared-memory limit to kGenSmemMax once per device, at the first launch that needs more
// than the default 48 KB (the first angle of a sweep runs before any graph capture), and
// returns the one for L.
template <auto K320, auto KANY>
auto gen_rows_pick(int L, size_t smem) {
  if (smem > 48 * 1024) {
    static PerDeviceOnce once;
    once([] {
      GISSPA_CUDA(cudaFuncSetAttribute(K320, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGenSmemMax));
      GISSPA_CUDA(cudaFuncSetAttribute(KANY, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGenSmemMax));
    });
  }
  return L == 320 ? K320 : KANY;
}

}  // namespace

bool generic_fused(int L, int epi) {
  if (L > kSmoothMax || smooth_plan(L).ns == 0) return false;
  const int rb = gen_rows_rb(L, epi);
  return rb > 0 && gen_rows_smem(L, rb, epi, 1) <= kGenSmemMax && (size_t)2 * sizeof(float2) * L <= kGenSmemMax;
}

bool correlate_fast(int L) { return L == 256 || L == 320 || L == 512 || L == 1024; }

size_t generic_z_elems(int L, int P) { return (size_t)P * (L / 2 + 1) * L; }
size_t generic_x_elems(int L, int P, int epi) { return generic_fused(L, epi) ? 0 : (size_t)P * L * L; }

void correlate_generic(const CorrLaunch& cl, const float2* I, const void* T, const CorrArgs& a, FftEngine& fft,
                       float2* z, float2* x, cudaStream_t s, cudaEvent_t* ev) {
  const int L = cl.L, P = cl.E * cl.D;
  const long long H = (long long)(L / 2 + 1) * L, L2 = (long long)L * L;
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[0], s));
  if (generic_fused(L, cl.epi)) {
    const SmoothPlan plan = smooth_plan(L);
    const float2* tw = fft.twiddles(L);
    const long long nrows = (long long)P * (L / 2 + 1);
    const int rpc = std::max(1, 2048 / L);
    const size_t smc = 2 * sizeof(float2) * (size_t)rpc * L;
    const unsigned gc = (unsigned)((nrows + rpc - 1) / rpc);
    // L = 320, the reference's default window size, runs kernels compiled for that length
    // at most 2048 points per CTA: 32 KB, within the default shared-memory limit
    auto cols = [&](auto k320, auto kany, const auto* t) {
      auto kernel = L == 320 ? k320 : kany;
      kernel<<<gc, 256, smc, s>>>(I, t, a.b0, a.n0, cl.D, L, nrows, rpc, plan, tw, z);
    };
    switch (cl.spec) {
      case GISSPA_SPEC_FP32:
        cols(gen_cols_kernel<320, SpecFp32>, gen_cols_kernel<0, SpecFp32>, static_cast<const float2*>(T));
        break;
      case GISSPA_SPEC_FP16:
        cols(gen_cols_kernel<320, SpecFp16>, gen_cols_kernel<0, SpecFp16>, static_cast<const __half2*>(T));
        break;
      case GISSPA_SPEC_BF16:
        cols(gen_cols_kernel<320, SpecBf16>, gen_cols_kernel<0, SpecBf16>, static_cast<const __nv_bfloat162*>(T));
        break;
      default: throw CudaError{cudaErrorInvalidValue, "unknown spectrum precision"};
    }
    GISSPA_LAUNCH_CHECK();
    if (ev) GISSPA_CUDA(cudaEventRecord(ev[1], s));
    const int rb = gen_rows_rb(L, cl.epi);
    const int tb = gen_rows_tb(L, rb, cl.epi);
    const size_t smr = gen_rows_smem(L, rb, cl.epi, tb);
    const dim3 gr((unsigned)(L / rb), (unsigned)cl.E);
    auto rows = [&](auto kernel) { kernel<<<gr, 256, smr, s>>>(z, a, L, rb, tb, plan, tw); };
    switch (cl.epi) {
      case EPI_SUM: rows(gen_rows_pick<gen_rows_kernel<320, EPI_SUM>, gen_rows_kernel<0, EPI_SUM>>(L, smr)); break;
      case EPI_TOPK:
        rows(gen_rows_pick<gen_rows_kernel<320, EPI_TOPK>, gen_rows_kernel<0, EPI_TOPK>>(L, smr));
        break;
      case EPI_CHUNK:
        rows(gen_rows_pick<gen_rows_kernel<320, EPI_CHUNK>, gen_rows_kernel<0, EPI_CHUNK>>(L, smr));
        break;
      case EPI_NONORM:
        rows(gen_rows_pick<gen_rows_kernel<320, EPI_NONORM>, gen_rows_kernel<0, EPI_NONORM>>(L, smr));
        break;
      case EPI_MAP: rows(gen_rows_pick<gen_rows_kernel<320, EPI_MAP>, gen_rows_kernel<0, EPI_MAP>>(L, smr)); break;
      default: throw CudaError{cudaErrorInvalidValue, "unknown epilogue"};
    }
    GISSPA_LAUNCH_CHECK();
    if (ev) GISSPA_CUDA(cudaEventRecord(ev[2], s));
    return;
  }
  const dim3 gp((unsigned)std::min(ceil_div(H, kT), 4096), (unsigned)P);
  switch (cl.spec) {
    case GISSPA_SPEC_FP32:
      gen_product_kernel<SpecFp32><<<gp, kT, 0, s>>>(I, static_cast<const float2*>(T), a.b0, a.n0, cl.D, H, z);
      break;
    case GISSPA_SPEC_FP16:
      gen_product_kernel<SpecFp16><<<gp, kT, 0, s>>>(I, static_cast<const __half2*>(T), a.b0, a.n0, cl.D, H, z);
      break;
    case GISSPA_SPEC_BF16:
      gen_product_kernel<SpecBf16><<<gp, kT, 0, s>>>(I, static_cast<const __nv_bfloat162*>(T), a.b0, a.n0, cl.D, H,
                                                     z);
      break;
    default: throw CudaError{cudaErrorInvalidValue, "unknown spectrum precision"};
  }
  GISSPA_LAUNCH_CHECK();
  fft.rows(z, (long long)P * (L / 2 + 1), L, +1, 1.f, s);  // columns over ky
  gen_hermitian_rows_kernel<<<dim3((unsigned)std::min(ceil_div(L2, kT), 4096), (unsigned)P), kT, 0, s>>>(z, L, x);
  GISSPA_LAUNCH_CHECK();
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[1], s));
  fft.rows(x, (long long)P * L, L, +1, 1.f, s);  // rows over kx: real maps
  const unsigned chunks = (unsigned)(L2 / 256);  // L % 16 == 0 makes L^2 a multiple of 256
  switch (cl.epi) {
    case EPI_SUM:
    case EPI_TOPK:
      gen_sum_kernel<<<dim3((unsigned)ceil_div(L2, kT), (unsigned)cl.E), kT, 0, s>>>(x, a, L, cl.epi == EPI_TOPK);
      break;
    case EPI_CHUNK: gen_chunk_kernel<<<dim3(chunks, (unsigned)P), kT, 0, s>>>(x, a, L); break;
    case EPI_NONORM: gen_nonorm_kernel<<<dim3(chunks, (unsigned)P), kT, 0, s>>>(x, a, L); break;
    case EPI_MAP: gen_map_kernel<<<dim3((unsigned)ceil_div(L2, kT), (unsigned)P), kT, 0, s>>>(x, a, L); break;
    default: throw CudaError{cudaErrorInvalidValue, "unknown epilogue"};
  }
  GISSPA_LAUNCH_CHECK();
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[2], s));
}

}  // namespace gisspa
