// fft.cuh — register/shared-memory Stockham FFT building blocks (sm_100a).
//
// A transform of length N is spread over a team of T threads, each holding
// E = N/T complex points in registers.  Every stage of radix R runs E/R
// butterflies per thread; stage boundaries exchange data through a shared-memory
// buffer of N complex values addressed through an XOR swizzle of the low four
// index bits, swz(i) = (i & ~15) | ((i ^ (i >> S)) & 15) with S = log2(first radix):
// a replay of every store and load pattern of the plans below (16-lane phases,
// 8-byte accesses) shows it conflict-free, where no swizzle costs 3-5x and a
// one-in-sixteen pad 1.25x.  Stockham ordering needs no bit reversal: stage
// inputs are x[j + m N/R], outputs go to y[(j/Ns) Ns R + (j mod Ns) + r Ns],
// j = tid + T q.
//
// SIGN = -1 is the forward transform, +1 the inverse (unnormalised), matching the
// cuFFT convention the reference relies on.
#pragma once

#include "common.cuh"

namespace gisspa {

template <int S>
__host__ __device__ constexpr int fft_swz(int i) { return (i & ~15) | ((i ^ (i >> S)) & 15); }

// cos(2 pi k / 32) and sin(2 pi k / 32) for any integer k, from cos(j pi / 16), j = 0..8.
__host__ __device__ constexpr double cos32(int k) {
  constexpr double c[9] = {1.0,
                           0.98078528040323044913,
                           0.92387953251128675613,
                           0.83146961230254523708,
                           0.70710678118654752440,
                           0.55557023301960222474,
                           0.38268343236508977173,
                           0.19509032201612826785,
                           0.0};
  k &= 31;
  return k <= 8 ? c[k] : k <= 16 ? -c[16 - k] : k <= 24 ? -c[k - 16] : c[32 - k];
}
__host__ __device__ constexpr double sin32(int k) { return cos32(k - 8); }

// cos(2 pi k / 20) and sin(2 pi k / 20) for any integer k, from cos(j pi / 10), j = 0..5
// (cos 18 deg = sqrt(10 + 2 sqrt 5) / 4, cos 36 deg = (1 + sqrt 5) / 4, cos 54 deg =
// sqrt(10 - 2 sqrt 5) / 4, cos 72 deg = (sqrt 5 - 1) / 4).
__host__ __device__ constexpr double cos20(int k) {
  constexpr double c[6] = {1.0,
                           0.95105651629515357212,
                           0.80901699437494742410,
                           0.58778525229247312917,
                           0.30901699437494742410,
                           0.0};
  k %= 20;
  if (k < 0) k += 20;
  return k <= 5 ? c[k] : k <= 10 ? -c[10 - k] : k <= 15 ? -c[k - 10] : c[20 - k];
}
__host__ __device__ constexpr double sin20(int k) { return cos20(k - 5); }

// cos and sin of 2 pi K / R for a radix R dividing 32 or 20.
template <int R>
__host__ __device__ constexpr double root_cos(int k) {
  static_assert(32 % R == 0 || 20 % R == 0, "roots of unity for radices dividing 32 or 20");
  if constexpr (32 % R == 0)
    return cos32((32 / R) * k);
  else
    return cos20((20 / R) * k);
}
template <int R>
__host__ __device__ constexpr double root_sin(int k) {
  if constexpr (32 % R == 0)
    return sin32((32 / R) * k);
  else
    return sin20((20 / R) * k);
}

// Multiply v by W_R^K = exp(SIGN * 2 pi i K / R) (R dividing 32) with exact special cases.
template <int R, int K, int SIGN>
__device__ __forceinline__ float2 mul_wr(float2 v) {
  constexpr int KK = K % R;
  if constexpr (KK == 0) {
    return v;
  } else if constexpr (4 * KK == R) {
    return cmul_i<SIGN>(v);
  } else if constexpr (2 * KK == R) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (4 * KK == 3 * R) {
    return cmul_i<-SIGN>(v);
  } else if constexpr (8 * KK == R) {
    constexpr float h = 0.70710678118654752440f;
    return make_float2(h * (v.x - SIGN * v.y), h * (v.y + SIGN * v.x));
  } else if constexpr (8 * KK == 3 * R) {
    constexpr float h = 0.70710678118654752440f;
    return make_float2(h * (-v.x - SIGN * v.y), h * (-v.y + SIGN * v.x));
  } else {
    constexpr float c = (float)root_cos<R>(KK), s = (float)(SIGN * root_sin<R>(KK));
    return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
  }
}

template <int R, int SIGN>
struct Dft;

// 5-point DFT: X_k = sum_n x_n e^(SIGN 2 pi i n k / 5) from the symmetric pairs
// t1 = x1 + x4, t2 = x2 + x3, t3 = x1 - x4, t4 = x2 - x3:
//   X1, X4 = x0 + c1 t1 + c2 t2 +- SIGN i (s1 t3 + s2 t4)
//   X2, X3 = x0 + c2 t1 + c1 t2 +- SIGN i (s2 t3 - s1 t4)
// with c_k = cos(2 pi k / 5), s_k = sin(2 pi k / 5).
template <int SIGN>
struct Dft<5, SIGN> {
  __device__ __forceinline__ static void run(float2* a) {
    constexpr float c1 = (float)cos20(4), c2 = (float)cos20(8), s1 = (float)sin20(4), s2 = (float)sin20(8);
    const float2 t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]), t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
    const float2 x0 = a[0];
    const float2 p1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
    const float2 p2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
    // q = (s1 t3 + s2 t4), r = (s2 t3 - s1 t4); SIGN i q = SIGN (-q.y, q.x)
    const float2 q = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    const float2 r = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    const float2 iq = make_float2(-SIGN * q.y, SIGN * q.x), ir = make_float2(-SIGN * r.y, SIGN * r.x);
    a[0] = cadd(x0, cadd(t1, t2));
    a[1] = cadd(p1, iq);
    a[4] = csub(p1, iq);
    a[2] = cadd(p2, ir);
    a[3] = csub(p2, ir);
  }
};

// Composite DFT of length A B (A a power of two, B = 5) in registers: n = B n1 + n2,
// k = k1 + A k2:  X[k1 + A k2] = sum_n2 W_B^(n2 k2) W_AB^(n2 k1) (sum_n1 x[B n1 + n2] W_A^(n1 k1)).
template <int A, int B, int SIGN>
struct DftAB {
  template <int N2, int K1>
  __device__ __forceinline__ static void twiddle(float2 (&y)[B][A]) {
    if constexpr (N2 < B) {
      if constexpr (K1 < A) {
        y[N2][K1] = mul_wr<A * B, N2 * K1, SIGN>(y[N2][K1]);
        twiddle<N2, K1 + 1>(y);
      } else {
        twiddle<N2 + 1, 0>(y);
      }
    }
  }
  __device__ __forceinline__ static void run(float2* a) {
    float2 y[B][A];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) y[n2][n1] = a[B * n1 + n2];
      Dft<A, SIGN>::run(y[n2]);
    }
    twiddle<0, 0>(y);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      float2 z[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) z[n2] = y[n2][k1];
      Dft<B, SIGN>::run(z);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) a[k1 + A * k2] = z[k2];
    }
  }
};
template <int SIGN>
struct Dft<10, SIGN> : DftAB<2, 5, SIGN> {};
template <int SIGN>
struct Dft<20, SIGN> : DftAB<4, 5, SIGN> {};

// In-register DFT of length R (R in {1, 2, 4, 8, 16}), natural order in and out.
template <int R, int SIGN>
struct Dft {
  template <int K = 0>
  __device__ __forceinline__ static void combine(float2* a, const float2* e, const float2* o) {
    if constexpr (K < R / 2) {
      float2 t = mul_wr<R, K, SIGN>(o[K]);
      a[K] = cadd(e[K], t);
      a[K + R / 2] = csub(e[K], t);
      combine<K + 1>(a, e, o);
    }
  }
  __device__ __forceinline__ static void run(float2* a) {
    if constexpr (R == 1) {
      return;
    } else if constexpr (R == 2) {
      float2 t = a[1];
      a[1] = csub(a[0], t);
      a[0] = cadd(a[0], t);
    } else {
      float2 e[R / 2], o[R / 2];
#pragma unroll
      for (int m = 0; m < R / 2; ++m) {
        e[m] = a[2 * m];
        o[m] = a[2 * m + 1];
      }
      Dft<R / 2, SIGN>::run(e);
      Dft<R / 2, SIGN>::run(o);
      combine<0>(a, e, o);
    }
  }
};

// Twiddle tables exp(-2 pi i p / N), p < N, read through the read-only path (TwGlobal) or
// from a copy the CTA staged in shared memory (TwShared, for kernels that sweep the same
// table many times and would otherwise stall on L1 latency).
struct TwGlobal {
  const float2* __restrict__ p;
  __device__ __forceinline__ float2 operator()(int i) const { return __ldg(p + i); }
};
struct TwShared {  // staged with one pad entry per 16 (tw_pad_index): the strided reads of a
  const float2* p;  // Stockham stage (indices 4k, k < 8) fall in distinct banks
  __device__ __forceinline__ float2 operator()(int i) const { return p[i + (i >> 4)]; }
};
__host__ __device__ constexpr int tw_pad_index(int i) { return i + (i >> 4); }

// Twiddle W_N^p for the stage (conjugated for the inverse transform).
template <int SIGN, typename Tw>
__device__ __forceinline__ float2 table_tw(const Tw& tw, int p) {
  float2 w = tw(p);
  return SIGN > 0 ? make_float2(w.x, -w.y) : w;
}

// Powers w[m] = w1^m, 1 <= m < R, by products of powers of two: w[2^i] by squaring,
// w[m] = w[h] w[m - h] with h the highest power of two below m.  The deepest power (m = R - 1)
// is log2(R) products from w1, so each power carries a few ulp beyond the table entry.
template <int M, int R>
struct TwPow {
  static constexpr int H = M >= 16 ? 16 : M >= 8 ? 8 : M >= 4 ? 4 : M >= 2 ? 2 : 1;  // highest power of 2 <= M
  __device__ __forceinline__ static void run(float2* w) {
    if constexpr (M < R) {
      w[M] = (H == M) ? cmul(w[M / 2], w[M / 2]) : cmul(w[H], w[M - H]);
      TwPow<M + 1, R>::run(w);
    }
  }
};
template <int R>
__device__ __forceinline__ void tw_powers(float2 w1, float2* w) {
  static_assert(R <= 32, "powers up to 31");
  w[1] = w1;
  TwPow<2, R>::run(w);
}

// One Stockham stage: v holds this thread's inputs as v[q*R + m] = x[j_q + m N/R].
// Twiddles, butterflies, and (unless LAST) stores to shared memory.  Each butterfly reads one
// twiddle W_N^(k step) from the table and raises it to the powers m = 2..R-1 in registers: the
// table reads are gathers (k varies with the thread), R - 1 per butterfly they took most of the
// L1 load bandwidth of the correlation passes.
template <int N, int T, int R, int NS, int SIGN, bool LAST, int S, typename Tw>
__device__ __forceinline__ void stockham_stage(float2* v, float2* sm, const Tw& tw, int tid) {
  constexpr int E = N / T, B = E / R;
  static_assert(E % R == 0, "radix must divide the points per thread");
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const int j = tid + T * q;
    const int k = j % NS;
    float2* a = v + q * R;
    if constexpr (NS > 1) {
      constexpr int step = N / (NS * R);
      float2 w[R];
      tw_powers<R>(table_tw<SIGN>(tw, k * step), w);
#pragma unroll
      for (int m = 1; m < R; ++m) a[m] = cmul(a[m], w[m]);
    }
    Dft<R, SIGN>::run(a);
    if constexpr (!LAST) {
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) sm[fft_swz<S>(base + r * NS)] = a[r];
    }
  }
}

// Load the inputs of the next stage (radix R) from shared memory.
template <int N, int T, int R, int S>
__device__ __forceinline__ void stockham_load(float2* v, const float2* sm, int tid) {
  constexpr int E = N / T, B = E / R;
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const int j = tid + T * q;
#pragma unroll
    for (int m = 0; m < R; ++m) v[q * R + m] = sm[fft_swz<S>(j + m * (N / R))];
  }
}

// Radix plans: three stages for every length used by the correlation kernels.
//   first stage inputs of thread tid:  x[tid + T q + m N/R1]
//   last stage outputs of thread tid:  y[j + r N/R3], j = tid + T q
template <int N, int T>
struct Plan;
template <> struct Plan<256, 32> { static constexpr int R1 = 8, R2 = 8, R3 = 4, S = 3; };
template <> struct Plan<512, 64> { static constexpr int R1 = 8, R2 = 8, R3 = 8, S = 3; };
template <> struct Plan<512, 32> { static constexpr int R1 = 16, R2 = 8, R3 = 4, S = 4; };
template <> struct Plan<1024, 64> { static constexpr int R1 = 16, R2 = 16, R3 = 4, S = 4; };
template <> struct Plan<128, 16> { static constexpr int R1 = 8, R2 = 4, R3 = 4, S = 3; };
// window 320: columns of 320 points on 16 lanes (20 each, the first stage a 4 x 5 register DFT)
template <> struct Plan<320, 16> { static constexpr int R1 = 20, R2 = 4, R3 = 4, S = 2; };

// Full three-stage transform.  v: E inputs in first-stage order; on return v holds
// the outputs in last-stage order.  sm: this team's buffer of N values; SYNC() must be a
// barrier covering the team (warp or block).  The buffer is free again on return.
template <int N, int T, int SIGN, typename Sync, typename Tw>
__device__ __forceinline__ void fft3(float2* v, float2* sm, const Tw& tw, int tid, Sync sync) {
  using P = Plan<N, T>;
  constexpr int R1 = P::R1, R2 = P::R2, R3 = P::R3, S = P::S;
  static_assert(R1 * R2 * R3 == N, "plan must factor N");
  stockham_stage<N, T, R1, 1, SIGN, false, S>(v, sm, tw, tid);
  sync();
  stockham_load<N, T, R2, S>(v, sm, tid);
  sync();
  stockham_stage<N, T, R2, R1, SIGN, false, S>(v, sm, tw, tid);
  sync();
  stockham_load<N, T, R3, S>(v, sm, tid);
  sync();
  stockham_stage<N, T, R3, R1 * R2, SIGN, true, S>(v, sm, tw, tid);
}

// Index of output element e (0 <= e < E) held by thread tid after fft3.
template <int N, int T>
__device__ __forceinline__ int fft3_out_index(int tid, int e) {
  constexpr int R3 = Plan<N, T>::R3;
  const int q = e / R3, r = e % R3;
  return tid + T * q + r * (N / R3);
}
// Index of input element e held by thread tid before fft3.
template <int N, int T>
__device__ __forceinline__ int fft3_in_index(int tid, int e) {
  constexpr int R1 = Plan<N, T>::R1;
  const int q = e / R1, m = e % R1;
  return tid + T * q + m * (N / R1);
}

// Two-stage plans (radix R1 then R2, R1 * R2 = N) for teams of T <= 32 threads, E = N / T
// points per thread: one shared-memory exchange, one twiddle stage, and a team inside one warp
// (the exchange needs only __syncwarp).
template <int N, int T>
struct Plan2;
template <> struct Plan2<256, 16> { static constexpr int R1 = 16, R2 = 16, S = 4; };
template <> struct Plan2<512, 16> { static constexpr int R1 = 32, R2 = 16, S = 5; };
template <> struct Plan2<1024, 32> { static constexpr int R1 = 32, R2 = 32, S = 5; };

template <int N, int T, int SIGN, typename Sync, typename Tw>
__device__ __forceinline__ void fft2s(float2* v, float2* sm, const Tw& tw, int tid, Sync sync) {
  using P = Plan2<N, T>;
  static_assert(P::R1 * P::R2 == N, "plan must factor N");
  stockham_stage<N, T, P::R1, 1, SIGN, false, P::S>(v, sm, tw, tid);
  sync();
  stockham_load<N, T, P::R2, P::S>(v, sm, tid);
  stockham_stage<N, T, P::R2, P::R1, SIGN, true, P::S>(v, sm, tw, tid);
}
// Index of input element e held by thread tid before fft2s.
template <int N, int T>
__device__ __forceinline__ int fft2_in_index(int tid, int e) {
  constexpr int R1 = Plan2<N, T>::R1;
  return tid + T * (e / R1) + (e % R1) * (N / R1);
}
// Index of output element e held by thread tid after fft2s.
template <int N, int T>
__device__ __forceinline__ int fft2_out_index(int tid, int e) {
  constexpr int R2 = Plan2<N, T>::R2;
  return tid + T * (e / R2) + (e % R2) * (N / R2);
}

}  // namespace gisspa
