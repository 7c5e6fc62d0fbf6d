// fft_generic.cuh — batched 1D/2D complex FFTs for every size outside the hot loop
// (template and image preparation, window spectra, per-angle template spectra).
//
// Power-of-two lengths up to 16384 run one shared-memory radix-2 transform per row; lengths
// up to 8192 whose prime factors are 2, 3, 5 and 7 run one shared-memory mixed-radix
// Stockham transform per row; other lengths use Bluestein's chirp-z algorithm on top of the
// power-of-two transform.  2D transforms are
// rows -> transpose -> rows (-> transpose).  All transforms are unnormalised.
#pragma once

#include <utility>

#include <atomic>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"

namespace gisspa {

// Incremented on every device buffer (re)allocation and release in the process: a captured
// CUDA graph holds raw buffer addresses and is rebuilt when this has moved since its capture.
inline std::atomic<unsigned long long>& alloc_generation() {
  static std::atomic<unsigned long long> g{0};
  return g;
}

// Grow-only device buffer.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  ~DevBuf() { release(); }
  void* ensure(size_t bytes) {
    if (bytes > n_) {
      release();
      ++alloc_generation();
      GISSPA_CUDA(cudaMalloc(&p_, bytes));
      n_ = bytes;
    }
    return p_;
  }
  void release() {
    if (p_) {
      ++alloc_generation();
      cudaFree(p_);
    }
    p_ = nullptr;
    n_ = 0;
  }
  template <typename T>
  T* as() const { return static_cast<T*>(p_); }
  size_t size() const { return n_; }
  void swap(DevBuf& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
  }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
};

// Radices (4 first, then 2, 3, 5, 7) whose product is n; ns = 0 when n has a prime factor
// above 7 (such lengths use Bluestein's algorithm).
struct SmoothPlan {
  static constexpr int kMax = 16;
  int ns = 0;
  int r[kMax] = {};
};
__host__ __device__ constexpr SmoothPlan smooth_plan_c(int n) {
  SmoothPlan p;
  if (n < 2) return p;
  const int fs[5] = {4, 2, 3, 5, 7};
  int rest = n;
  while (rest % 4 == 0 && rest > 4 && p.ns < SmoothPlan::kMax) {
    p.r[p.ns++] = 4;
    rest /= 4;
  }
  for (int i = 0; i < 5; ++i)
    while (rest % fs[i] == 0 && p.ns < SmoothPlan::kMax) {
      p.r[p.ns++] = fs[i];
      rest /= fs[i];
    }
  if (rest != 1) p.ns = 0;
  return p;
}
inline SmoothPlan smooth_plan(int n) { return smooth_plan_c(n); }
// Longest row the mixed-radix kernel takes (two shared-memory copies of 8192 complex = 128 KB).
constexpr int kSmoothMax = 8192;

class FftEngine {
 public:
  // Table of exp(-2 pi i p / n), p < n (device pointer, cached per n).
  const float2* twiddles(int n);
  // In-place transform of `rows` contiguous rows of length n (any n >= 1).
  void rows(float2* data, long long rows, int n, int sign, float scale, cudaStream_t s);
  // out[b][c][r] = in[b][r][c] for rows x cols matrices; optional row subset
  // [0, out_rows) of the transposed result (i.e. input columns [0, out_rows)).
  void transpose(const float2* in, float2* out, int batch, int rows, int cols, cudaStream_t s, int out_rows = -1);
  // In-place 2D transform of batch x ny x nx, using tmp (same size) as scratch.
  void fft2(float2* data, float2* tmp, int batch, int ny, int nx, int sign, float scale, cudaStream_t s);

 private:
  struct Blue {
    int n = 0, m = 0;
    DevBuf chirp, bfwd, binv;
  };
  Blue& bluestein(int n);
  std::map<int, DevBuf> tw_;
  std::map<int, std::unique_ptr<Blue>> blue_;
  DevBuf scratch_;
};

bool is_pow2(long long n);

}  // namespace gisspa
