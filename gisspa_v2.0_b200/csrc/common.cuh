// common.cuh — shared device/host helpers for the B200 search library.
#pragma once

#include <mutex>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <cstdio>
#include <string>

namespace gisspa {

// pi used where the reference uses its own PI constant (utils/constants.h:3)
constexpr double kRefPi = 3.1415926535;
constexpr double kPi = 3.14159265358979323846;

struct CudaError {
  cudaError_t code;
  std::string where;
};

#define GISSPA_CUDA(call)                                                               \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::gisspa::CudaError{e_, std::string(#call) + " @ " + __FILE__ + ":" +       \
                                        std::to_string(__LINE__)};                      \
  } while (0)

// Number of kernels this library has launched from the calling thread.
long long& launch_counter();

#define GISSPA_LAUNCH_CHECK()              \
  do {                                     \
    ++::gisspa::launch_counter();          \
    GISSPA_CUDA(cudaGetLastError());       \
  } while (0)

// Runs f once per device for one kernel instance (cudaFuncSetAttribute acts on the current
// device only, and one process may drive several GPUs from several threads).
struct PerDeviceOnce {
  std::mutex m;
  unsigned long long done = 0;  // bit per device ordinal
  template <typename F>
  void operator()(F&& f) {
    int dev = 0;
    GISSPA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(m);
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done & bit)) return;
    f();
    done |= bit;
  }
};

// ---- complex arithmetic on float2 / double2
// On sm_100 a complex add or subtract is one paired FP32 instruction ({add,sub}.f32x2 on the
// 64-bit register pair that holds the float2) instead of two.  The correlation kernels are
// bound by instruction issue and most of their arithmetic is butterfly additions; the
// rounding is that of two scalar additions.
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 d;
  asm("add.rn.f32x2 %0, %1, %2;"
      : "=l"(*reinterpret_cast<unsigned long long*>(&d))
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
  return d;
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 d;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(*reinterpret_cast<unsigned long long*>(&d))
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
  return d;
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// Element-wise product and fused multiply-add of two pairs ({mul,fma}.rn.f32x2 on sm_100; the
// rounding of two scalar operations).
__host__ __device__ __forceinline__ float2 pmul(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 d;
  asm("mul.rn.f32x2 %0, %1, %2;"
      : "=l"(*reinterpret_cast<unsigned long long*>(&d))
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
  return d;
#else
  return make_float2(a.x * b.x, a.y * b.y);
#endif
}
__host__ __device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(*reinterpret_cast<unsigned long long*>(&d))
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)),
        "l"(*reinterpret_cast<const unsigned long long*>(&c)));
  return d;
#else
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by +i (SIGN>0) or -i
template <int SIGN>
__host__ __device__ __forceinline__ float2 cmul_i(float2 a) {
  return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Angle of a sweep held in device memory: the rotation and the correlation epilogues read it
// when given, so one captured CUDA graph of an angle's launches serves every angle.
struct AngleState {
  int index;         // position in the float-stepped angle sequence
  float cose, sine;  // (float)cos / (float)sin of the angle in radians
  int pad;
};

// Programmatic dependent launch (sm_90+): a kernel launched with programmatic stream
// serialization may start before its predecessor finishes; griddep_wait blocks until the
// predecessor has completed and its memory is visible (a no-op for a normal launch), and
// griddep_launch_dependents lets the successor start as soon as every CTA has issued it.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

// Order-preserving map of a float onto uint32 (larger float -> larger key).
__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(b);
}

__device__ __forceinline__ unsigned brev8(unsigned v) { return __brev(v) >> 24; }

// Exact shell index floor(hypot(a, b) + 0.5) - 1 evaluated in integers:
// the k with k^2 - k < n <= k^2 + k, n = a^2 + b^2.
__host__ __device__ __forceinline__ int shell_index(int a, int b) {
  long long n = (long long)a * a + (long long)b * b;
#ifdef __CUDA_ARCH__
  long long k = (long long)floor(sqrt((double)n) + 0.5);
#else
  long long k = (long long)std::floor(std::sqrt((double)n) + 0.5);
#endif
  if (k > 0 && k * k - k >= n) --k;
  if (k * k + k < n) ++k;
  return (int)k - 1;
}
__host__ __device__ __forceinline__ int shell_xy(int x, int y, int nx, int ny) {
  int a = y < ny - y ? y : ny - y;
  int b = x < nx - x ? x : nx - x;
  return shell_index(a, b);
}

// Storage types for the template-spectrum stream.
struct SpecFp32 {
  using T = float2;
  __device__ __forceinline__ static float2 load(const T* p) { return *p; }
  __device__ __forceinline__ static T pack(float2 v) { return v; }
};
struct SpecFp16 {
  using T = __half2;
  __device__ __forceinline__ static float2 load(const T* p) { return __half22float2(*p); }
  __device__ __forceinline__ static T pack(float2 v) { return __float22half2_rn(v); }
};
struct SpecBf16 {
  using T = __nv_bfloat162;
  __device__ __forceinline__ static float2 load(const T* p) { return __bfloat1622float2(*p); }
  __device__ __forceinline__ static T pack(float2 v) { return __float22bfloat162_rn(v); }
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace gisspa

namespace gisspa {

// ---- asynchronous bulk copies (1D TMA) into shared memory, completed on an mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order earlier generic-proxy shared-memory accesses before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Bounded wait for the phase with the given parity: gives up after ~max_cycles SM
// clock cycles (or 2^24 polls) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long max_cycles) {
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  for (int i = 0; i < (1 << 24); ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
  return false;
}

}  // namespace gisspa
