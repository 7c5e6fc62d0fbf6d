// fft_smooth.cuh — device routine of the mixed-radix (2, 3, 4, 5, 7) Stockham transform in
// shared memory, shared by the generic FFT engine and the correlation of window sizes without
// hand-tuned kernels.
#pragma once

#include "fft_generic.cuh"

namespace gisspa {

// One butterfly of a Stockham stage of radix R for rows of length n, after stages whose
// radices multiply to Ns: butterfly j < m = n/R reads x_q = in[j + q m], applies the twiddles
// w^(q k), k = j mod Ns, w = e^(-+2 pi i/(Ns R)) (tw[p] = e^(-2 pi i p/n)), takes the R-point
// DFT and writes out[(j / Ns) Ns R + k + p Ns]: after the last stage the row is in natural order.
template <int R, int SIGN>
__device__ __forceinline__ void smooth_butterfly(const float2* __restrict__ in, float2* __restrict__ out, int n,
                                                 int m, int Ns, int j, const float2* __restrict__ tw) {
  const int k = j % Ns, tstep = n / (Ns * R);
  float2 x[R];
#pragma unroll
  for (int q = 0; q < R; ++q) x[q] = in[j + q * m];
#pragma unroll
  for (int q = 1; q < R; ++q) {
    float2 w = __ldg(tw + q * k * tstep);
    if (SIGN > 0) w.y = -w.y;
    x[q] = cmul(x[q], w);
  }
  float2 y[R];
  if constexpr (R == 2) {
    y[0] = cadd(x[0], x[1]);
    y[1] = csub(x[0], x[1]);
  } else if constexpr (R == 4) {
    // e^(-+2 pi i / 4) = -+i
    const float2 a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]), b0 = cadd(x[1], x[3]), b1 = csub(x[1], x[3]);
    const float2 jb = SIGN > 0 ? make_float2(-b1.y, b1.x) : make_float2(b1.y, -b1.x);
    y[0] = cadd(a0, b0);
    y[1] = cadd(a1, jb);
    y[2] = csub(a0, b0);
    y[3] = csub(a1, jb);
  } else {
    // direct R-point DFT with the roots e^(-+2 pi i p / R) = tw[p n / R]
    float2 root[R];
    root[0] = make_float2(1.f, 0.f);
#pragma unroll
    for (int p = 1; p < R; ++p) {
      root[p] = __ldg(tw + p * (n / R));
      if (SIGN > 0) root[p].y = -root[p].y;
    }
#pragma unroll
    for (int p = 0; p < R; ++p) {
      float2 acc = x[0];
#pragma unroll
      for (int q = 1; q < R; ++q) acc = cadd(acc, cmul(x[q], root[(p * q) % R]));
      y[p] = acc;
    }
  }
  const int base = (j / Ns) * Ns * R + k;
#pragma unroll
  for (int p = 0; p < R; ++p) out[base + p * Ns] = y[p];
}

// Runs every stage of `plan` on `rows` rows of length n (row stride ld) held in a, ping-
// ponging with b (same shape).  The caller has synchronised the block after filling a; returns
// the buffer holding the result, in natural order, after a final __syncthreads.
template <int SIGN>
__device__ __forceinline__ float2* smooth_stages(float2* a, float2* b, int rows, int n, int ld, const SmoothPlan& plan,
                                                 const float2* __restrict__ tw) {
  int Ns = 1;
#pragma unroll
  for (int s = 0; s < plan.ns; ++s) {
    const int R = plan.r[s], m = n / R, nb = rows * m;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
      const int r = t / m, j = t - r * m;
      const float2* in = a + (size_t)r * ld;
      float2* out = b + (size_t)r * ld;
      switch (R) {
        case 2: smooth_butterfly<2, SIGN>(in, out, n, m, Ns, j, tw); break;
        case 3: smooth_butterfly<3, SIGN>(in, out, n, m, Ns, j, tw); break;
        case 4: smooth_butterfly<4, SIGN>(in, out, n, m, Ns, j, tw); break;
        case 5: smooth_butterfly<5, SIGN>(in, out, n, m, Ns, j, tw); break;
        default: smooth_butterfly<7, SIGN>(in, out, n, m, Ns, j, tw); break;
      }
    }
    __syncthreads();
    float2* tmp = a;
    a = b;
    b = tmp;
    Ns *= R;
  }
  return a;
}

// smooth_stages with the length and plan fixed at compile time when LC != 0 (the stage loop
// unrolls and the index divisions become constant); LC = 0 takes n and plan at run time.
template <int LC, int SIGN>
__device__ __forceinline__ float2* smooth_stages_l(float2* a, float2* b, int rows, int n, int ld,
                                                   const SmoothPlan& plan, const float2* __restrict__ tw) {
  if constexpr (LC != 0) {
    constexpr SmoothPlan kp = smooth_plan_c(LC);
    static_assert(kp.ns > 0, "LC must factor into 2, 3, 5 and 7");
    return smooth_stages<SIGN>(a, b, rows, LC, ld, kp, tw);
  } else {
    return smooth_stages<SIGN>(a, b, rows, n, ld, plan, tw);
  }
}

}  // namespace gisspa
