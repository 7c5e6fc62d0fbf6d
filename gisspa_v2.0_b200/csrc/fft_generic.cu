// fft_generic.cu — batched FFTs outside the hot loop (see fft_generic.cuh).
#include <cmath>
#include <complex>

#include "fft.cuh"
#include "fft_smooth.cuh"

namespace gisspa {

bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

namespace {

// One or more rows of a power-of-two length per CTA, in shared memory:
// bit-reversed load, log2(n) in-place radix-2 stages, scaled store.
template <int SIGN>
__global__ void fft_pow2_rows_kernel(float2* __restrict__ data, long long nrows, int n, int logn, int rpc,
                                     const float2* __restrict__ tw, float scale) {
  extern __shared__ float2 sm[];
  const long long row0 = (long long)blockIdx.x * rpc;
  const int rows_here = (int)min((long long)rpc, nrows - row0);
  float2* base = data + row0 * n;
  const int total = rows_here * n;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int r = i >> logn, k = i & (n - 1);
    int rk = logn ? (int)(__brev((unsigned)k) >> (32 - logn)) : 0;
    sm[(r << logn) + rk] = base[i];
  }
  __syncthreads();
  const int hn = n >> 1;
  const int nb = rows_here * hn;
  for (int len = 2, lg = 1; len <= n; len <<= 1, ++lg) {
    const int half = len >> 1, step = n >> lg;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
      int r = t / hn, b = t - r * hn;
      int grp = b / half, j = b - grp * half;
      int i0 = (r << logn) + grp * len + j, i1 = i0 + half;
      float2 w = __ldg(tw + j * step);
      if (SIGN > 0) w.y = -w.y;
      float2 u = sm[i0], v = cmul(sm[i1], w);
      sm[i0] = cadd(u, v);
      sm[i1] = csub(u, v);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < total; i += blockDim.x) base[i] = cscale(sm[i], scale);
}

// Rows of 256, 320, 512 or 1024 points in registers with the correlation kernels' Stockham
// plans: one warp per row for 256 = 8·8·4 and 512 = 16·8·4 (two exchanges) and 1024 = 32·32 (one),
// a half warp per row for 320 = 20·4·4, through the team's slice of shared memory; the team's
// loads and stores of each register's points are coalesced.  Used for the template, window and
// micrograph transforms of those lengths (the per-angle template spectra above all), where the
// radix-2 and mixed-radix kernels spent a shared-memory round trip and a CTA barrier per stage.
template <int N>
struct RowPlan {
  static constexpr bool kTwoStage = N == 1024;
  static constexpr int kTeam = N == 320 ? 16 : 32;
  static constexpr int kRows = N == 1024 ? 4 : N == 320 ? 16 : 8;  // rows per CTA: <= 40 KiB of buffers
};
template <int N, int SIGN>
__global__ void __launch_bounds__(256) fft_reg_rows_kernel(float2* __restrict__ data, long long nrows,
                                                           const float2* __restrict__ tw, float scale) {
  constexpr int T = RowPlan<N>::kTeam, E = N / T, ROWS = RowPlan<N>::kRows;
  __shared__ __align__(16) float2 sm[ROWS][N];
  const int w = threadIdx.x / T, tid = threadIdx.x % T;
  const long long row = (long long)blockIdx.x * ROWS + w;
  // whole warps leave together (their exchanges use __syncwarp); a half-warp team past the
  // last row transforms zeros beside its partner and stores nothing
  if ((long long)blockIdx.x * ROWS + (w & ~(32 / T - 1)) >= nrows) return;
  const bool live = row < nrows;
  float2* p = data + (live ? row : 0) * N;
  float2 v[E];
  if constexpr (RowPlan<N>::kTwoStage) {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = p[fft2_in_index<N, T>(tid, e)];
    fft2s<N, T, SIGN>(v, sm[w], TwGlobal{tw}, tid, [] { __syncwarp(); });
#pragma unroll
    for (int e = 0; e < E; ++e) p[fft2_out_index<N, T>(tid, e)] = cscale(v[e], scale);
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = live ? p[fft3_in_index<N, T>(tid, e)] : make_float2(0.f, 0.f);
    fft3<N, T, SIGN>(v, sm[w], TwGlobal{tw}, tid, [] { __syncwarp(); });
    if (live)
#pragma unroll
      for (int e = 0; e < E; ++e) p[fft3_out_index<N, T>(tid, e)] = cscale(v[e], scale);
  }
}

template <int N>
void reg_rows(float2* data, long long nrows, int sign, float scale, const float2* tw, cudaStream_t s) {
  constexpr int R = RowPlan<N>::kRows, T = RowPlan<N>::kTeam;
  const long long grid = (nrows + R - 1) / R;
  if (sign < 0)
    fft_reg_rows_kernel<N, -1><<<(unsigned)grid, T * R, 0, s>>>(data, nrows, tw, scale);
  else
    fft_reg_rows_kernel<N, 1><<<(unsigned)grid, T * R, 0, s>>>(data, nrows, tw, scale);
  GISSPA_LAUNCH_CHECK();
}

// One or more rows of a length whose prime factors are 2, 3, 5 and 7 per CTA: load into
// shared memory, Stockham stages, scaled store.
template <int SIGN>
__global__ void fft_smooth_rows_kernel(float2* __restrict__ data, long long nrows, int n, int rpc, SmoothPlan plan,
                                       const float2* __restrict__ tw, float scale) {
  extern __shared__ float2 sm[];
  const long long row0 = (long long)blockIdx.x * rpc;
  const int rows_here = (int)min((long long)rpc, nrows - row0);
  float2* base = data + row0 * n;
  float2* a = sm;
  float2* b = sm + (size_t)rpc * n;
  const int total = rows_here * n;
  for (int i = threadIdx.x; i < total; i += blockDim.x) a[i] = base[i];
  __syncthreads();
  a = smooth_stages<SIGN>(a, b, rows_here, n, n, plan, tw);
  for (int i = threadIdx.x; i < total; i += blockDim.x) base[i] = cscale(a[i], scale);
}

__global__ void blue_pre_kernel(const float2* __restrict__ x, float2* __restrict__ a, long long rows, int n, int m,
                                const float2* __restrict__ chirp, int sign) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * m) return;
  long long r = i / m;
  int k = (int)(i - r * m);
  float2 v = make_float2(0.f, 0.f);
  if (k < n) {
    float2 c = chirp[k];
    if (sign > 0) c.y = -c.y;
    v = cmul(x[r * n + k], c);
  }
  a[i] = v;
}

__global__ void blue_mul_kernel(float2* __restrict__ a, long long rows, int m, const float2* __restrict__ bs) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * m) return;
  a[i] = cmul(a[i], bs[i % m]);
}

__global__ void blue_post_kernel(float2* __restrict__ x, const float2* __restrict__ a, long long rows, int n, int m,
                                 const float2* __restrict__ chirp, int sign, float scale) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * n) return;
  long long r = i / n;
  int k = (int)(i - r * n);
  float2 c = chirp[k];
  if (sign > 0) c.y = -c.y;
  x[i] = cscale(cmul(a[r * m + k], c), scale);
}

__global__ void transpose_kernel(const float2* __restrict__ in, float2* __restrict__ out, int rows, int cols,
                                 int out_rows) {
  __shared__ float2 tile[32][33];
  const size_t b = blockIdx.z;
  in += b * (size_t)rows * cols;
  out += b * (size_t)out_rows * rows;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    int r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    int c = c0 + i, r = r0 + threadIdx.x;
    if (c < out_rows && r < rows) out[(size_t)c * rows + r] = tile[threadIdx.x][i];
  }
}

// Host FP64 radix-2 transform used to build the Bluestein kernel spectra.
void host_fft_pow2(std::vector<std::complex<double>>& x, int sign) {
  const int n = (int)x.size();
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(x[i], x[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    double ang = sign * 2.0 * kPi / len;
    for (int i = 0; i < n; i += len)
      for (int j = 0; j < len / 2; ++j) {
        std::complex<double> w = std::polar(1.0, ang * j);
        auto u = x[i + j], v = x[i + j + len / 2] * w;
        x[i + j] = u + v;
        x[i + j + len / 2] = u - v;
      }
  }
}

}  // namespace

const float2* FftEngine::twiddles(int n) {
  auto it = tw_.find(n);
  if (it != tw_.end()) return it->second.as<float2>();
  std::vector<float2> h(n);
  for (int p = 0; p < n; ++p) {
    double a = -2.0 * kPi * (double)p / n;
    h[p] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  DevBuf b;
  b.ensure(sizeof(float2) * n);
  GISSPA_CUDA(cudaMemcpy(b.as<float2>(), h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  auto* p = b.as<float2>();
  tw_.emplace(n, std::move(b));
  return p;
}

FftEngine::Blue& FftEngine::bluestein(int n) {
  auto it = blue_.find(n);
  if (it != blue_.end()) return *it->second;
  auto bl = std::make_unique<Blue>();
  bl->n = n;
  bl->m = 1;
  while (bl->m < 2 * n - 1) bl->m <<= 1;
  const int m = bl->m;
  std::vector<std::complex<double>> c(n);
  for (long long k = 0; k < n; ++k) {
    long long q = (k * k) % (2LL * n);
    c[k] = std::polar(1.0, -kPi * (double)q / n);
  }
  std::vector<std::complex<double>> bf(m, 0.0), bi(m, 0.0);
  for (int t = 0; t < n; ++t) {
    bf[t] = std::conj(c[t]);
    bi[t] = c[t];
    if (t) {
      bf[m - t] = std::conj(c[t]);
      bi[m - t] = c[t];
    }
  }
  host_fft_pow2(bf, -1);
  host_fft_pow2(bi, -1);
  std::vector<float2> hc(n), hf(m), hi(m);
  for (int k = 0; k < n; ++k) hc[k] = make_float2((float)c[k].real(), (float)c[k].imag());
  for (int k = 0; k < m; ++k) {
    hf[k] = make_float2((float)bf[k].real(), (float)bf[k].imag());
    hi[k] = make_float2((float)bi[k].real(), (float)bi[k].imag());
  }
  bl->chirp.ensure(sizeof(float2) * n);
  bl->bfwd.ensure(sizeof(float2) * m);
  bl->binv.ensure(sizeof(float2) * m);
  GISSPA_CUDA(cudaMemcpy(bl->chirp.as<float2>(), hc.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  GISSPA_CUDA(cudaMemcpy(bl->bfwd.as<float2>(), hf.data(), sizeof(float2) * m, cudaMemcpyHostToDevice));
  GISSPA_CUDA(cudaMemcpy(bl->binv.as<float2>(), hi.data(), sizeof(float2) * m, cudaMemcpyHostToDevice));
  auto& ref = *bl;
  blue_.emplace(n, std::move(bl));
  return ref;
}

void FftEngine::rows(float2* data, long long nrows, int n, int sign, float scale, cudaStream_t s) {
  if (nrows <= 0 || n <= 0) return;
  if (n == 256 || n == 320 || n == 512 || n == 1024) {
    const float2* tw = twiddles(n);
    if (n == 256)
      reg_rows<256>(data, nrows, sign, scale, tw, s);
    else if (n == 320)
      reg_rows<320>(data, nrows, sign, scale, tw, s);
    else if (n == 512)
      reg_rows<512>(data, nrows, sign, scale, tw, s);
    else
      reg_rows<1024>(data, nrows, sign, scale, tw, s);
    return;
  }
  if (is_pow2(n)) {
    if (n > 16384) throw CudaError{cudaErrorInvalidValue, "fft length above 16384"};
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    const int rpc = n >= 2048 ? 1 : 2048 / n;
    const int threads = std::min(512, std::max(32, rpc * n / 2));
    const size_t smem = sizeof(float2) * (size_t)rpc * n;
    const float2* tw = twiddles(std::max(n, 2));
    const long long grid = (nrows + rpc - 1) / rpc;
    if (smem > 48 * 1024) {
      GISSPA_CUDA(cudaFuncSetAttribute(fft_pow2_rows_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      GISSPA_CUDA(cudaFuncSetAttribute(fft_pow2_rows_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (sign < 0)
      fft_pow2_rows_kernel<-1><<<(unsigned)grid, threads, smem, s>>>(data, nrows, n, logn, rpc, tw, scale);
    else
      fft_pow2_rows_kernel<1><<<(unsigned)grid, threads, smem, s>>>(data, nrows, n, logn, rpc, tw, scale);
    GISSPA_LAUNCH_CHECK();
    return;
  }
  const SmoothPlan sp = n <= kSmoothMax ? smooth_plan(n) : SmoothPlan{};
  if (sp.ns > 0) {
    const int rpc = n >= 2048 ? 1 : 2048 / n;
    const size_t smem = 2 * sizeof(float2) * (size_t)rpc * n;
    const float2* tw = twiddles(n);
    const long long grid = (nrows + rpc - 1) / rpc;
    if (smem > 48 * 1024) {
      GISSPA_CUDA(cudaFuncSetAttribute(fft_smooth_rows_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
      GISSPA_CUDA(cudaFuncSetAttribute(fft_smooth_rows_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    if (sign < 0)
      fft_smooth_rows_kernel<-1><<<(unsigned)grid, 256, smem, s>>>(data, nrows, n, rpc, sp, tw, scale);
    else
      fft_smooth_rows_kernel<1><<<(unsigned)grid, 256, smem, s>>>(data, nrows, n, rpc, sp, tw, scale);
    GISSPA_LAUNCH_CHECK();
    return;
  }
  Blue& bl = bluestein(n);
  const int m = bl.m;
  const float2* bs = sign < 0 ? bl.bfwd.as<float2>() : bl.binv.as<float2>();
  // bound the scratch to ~256 MB by processing rows in slices
  const long long slice = std::max(1LL, (256LL << 20) / ((long long)m * (long long)sizeof(float2)));
  for (long long r0 = 0; r0 < nrows; r0 += slice) {
    const long long nr = std::min(slice, nrows - r0);
    float2* a = static_cast<float2*>(scratch_.ensure(sizeof(float2) * (size_t)nr * m));
    const int T = 256;
    blue_pre_kernel<<<ceil_div(nr * m, T), T, 0, s>>>(data + r0 * n, a, nr, n, m, bl.chirp.as<float2>(), sign);
    GISSPA_LAUNCH_CHECK();
    rows(a, nr, m, -1, 1.f, s);
    blue_mul_kernel<<<ceil_div(nr * m, T), T, 0, s>>>(a, nr, m, bs);
    GISSPA_LAUNCH_CHECK();
    rows(a, nr, m, +1, 1.f, s);
    blue_post_kernel<<<ceil_div(nr * n, T), T, 0, s>>>(data + r0 * n, a, nr, n, m, bl.chirp.as<float2>(), sign,
                                                      scale / (float)m);
    GISSPA_LAUNCH_CHECK();
  }
}

void FftEngine::transpose(const float2* in, float2* out, int batch, int rows, int cols, cudaStream_t s,
                          int out_rows) {
  if (out_rows < 0) out_rows = cols;
  dim3 grid(ceil_div(out_rows, 32), ceil_div(rows, 32), batch);
  transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(in, out, rows, cols, out_rows);
  GISSPA_LAUNCH_CHECK();
}

void FftEngine::fft2(float2* data, float2* tmp, int batch, int ny, int nx, int sign, float scale, cudaStream_t s) {
  rows(data, (long long)batch * ny, nx, sign, 1.f, s);
  transpose(data, tmp, batch, ny, nx, s);
  rows(tmp, (long long)batch * nx, ny, sign, scale, s);
  transpose(tmp, data, batch, nx, ny, s);
}

}  // namespace gisspa
