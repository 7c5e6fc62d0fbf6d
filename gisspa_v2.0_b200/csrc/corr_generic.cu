// corr_generic.cu — the correlation and its epilogues for window sizes without hand-tuned
// kernels.  Same results as pass A + pass B (correlate.cu) within FP32 rounding: the
// transforms run on the generic FFT engine (radix-2 / Bluestein), the epilogues reproduce
// pass B's per-pixel sums and maxima, chunk picks with the reference's tie order, norm_type=0
// peaks and sums, and maps.  The reference's chunks are 256 consecutive pixels of the window's
// linear index (norm.cu:583-597), so for L that is not a multiple of 256 they straddle rows:
// the chunk kernels work on linear indices.
#include "../../include/gisspa.h"
#include "corr_generic.cuh"

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
    const int tb = brev8(255 - (unsigned)(best & 0xffu));
    const unsigned long long g =
        ((unsigned long long)float_key(vb) << 32) | ((unsigned long long)(0xFFFFFu - chunk) << 8) | tb;
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

}  // namespace

bool correlate_fast(int L) { return L == 256 || L == 512 || L == 1024; }

size_t generic_z_elems(int L, int P) { return (size_t)P * (L / 2 + 1) * L; }
size_t generic_x_elems(int L, int P) { return (size_t)P * L * L; }

void correlate_generic(const CorrLaunch& cl, const float2* I, const void* T, const CorrArgs& a, FftEngine& fft,
                       float2* z, float2* x, cudaStream_t s) {
  const int L = cl.L, P = cl.E * cl.D;
  const long long H = (long long)(L / 2 + 1) * L, L2 = (long long)L * L;
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
}

}  // namespace gisspa
