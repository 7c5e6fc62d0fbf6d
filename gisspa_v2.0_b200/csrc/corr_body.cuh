// corr_body.cuh — device building blocks of the correlation passes shared by the per-pass
// kernels (correlate.cu) and the pair engine (pair_engine.cu): the column transform of pass A
// with its fused conjugate multiply, the row transform of pass B, team reductions and the chunk
// pick emitter.
#pragma once

#include "correlate.cuh"
#include "fft.cuh"

namespace gisspa {
namespace {

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
// Barrier of one team of TEAM > 32 threads (whole warps): named barrier `id` (1..15; 0 is
// __syncthreads) counting TEAM threads.
template <int TEAM>
struct TeamSync {
  int id;
  __device__ __forceinline__ void operator()() const {
    if constexpr (TEAM <= 32)
      __syncwarp();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(TEAM) : "memory");
  }
};

// Pass A shapes: TT lanes per column, NC column slots per CTA, MINB CTAs per SM (the register
// cap).  Window 512 has two: 16 lanes with 32 points each (a two-stage 32 x 16 plan, one
// exchange, 128 registers) and 32 lanes with 16 points each (16 x 8 x 4, two exchanges, fewer
// registers and twice the warps per SM).
template <int L, int V = 0>
struct PassA;
template <> struct PassA<256, 0> { static constexpr int TT = 16, NC = 16, MINB = 2; };
template <> struct PassA<320, 0> { static constexpr int TT = 16, NC = 16, MINB = 2; };
template <> struct PassA<512, 0> { static constexpr int TT = 16, NC = 16, MINB = 2; };
template <> struct PassA<512, 1> { static constexpr int TT = 32, NC = 8, MINB = 4; };
template <> struct PassA<1024, 0> { static constexpr int TT = 32, NC = 8, MINB = 2; };

// The column transform of pass A: two Stockham stages (one exchange) for the powers of two,
// three (20 x 4 x 4, two exchanges) for 320, whose 20 points per lane allow no two-stage plan
// with every lane busy.
template <int L, int TT>
struct ColXform {
  __device__ __forceinline__ static int in_index(int tid, int e) { return fft2_in_index<L, TT>(tid, e); }
  __device__ __forceinline__ static int out_index(int tid, int e) { return fft2_out_index<L, TT>(tid, e); }
  __device__ __forceinline__ static void run(float2* v, float2* sm, const float2* tw, int tid) {
    fft2s<L, TT, +1>(v, sm, TwGlobal{tw}, tid, WarpSync{});
  }
};
template <>
struct ColXform<512, 32> {
  __device__ __forceinline__ static int in_index(int tid, int e) { return fft3_in_index<512, 32>(tid, e); }
  __device__ __forceinline__ static int out_index(int tid, int e) { return fft3_out_index<512, 32>(tid, e); }
  __device__ __forceinline__ static void run(float2* v, float2* sm, const float2* tw, int tid) {
    fft3<512, 32, +1>(v, sm, TwGlobal{tw}, tid, WarpSync{});
  }
};
template <>
struct ColXform<320, 16> {
  __device__ __forceinline__ static int in_index(int tid, int e) { return fft3_in_index<320, 16>(tid, e); }
  __device__ __forceinline__ static int out_index(int tid, int e) { return fft3_out_index<320, 16>(tid, e); }
  __device__ __forceinline__ static void run(float2* v, float2* sm, const float2* tw, int tid) {
    fft3<320, 16, +1>(v, sm, TwGlobal{tw}, tid, WarpSync{});
  }
};

// Pass A: one team of TT threads per column slot, NC slots per CTA, one pair per blockIdx.y.
// Each column is a two-stage Stockham transform (32 x 16 points at L = 512) with E = L / TT
// points per thread: one exchange through the team's slice of shared memory, inside a warp.
// The column transforms leave row-major, Q[pair][y][slot], through a shared tile: each team
// writes its column with the slot XOR-swizzled by the row (slot ^ (y mod NC)), and rows are
// read back as 16-byte pairs, so both sides are free of bank conflicts and every row segment
// of NC slots leaves as contiguous 16-byte stores.  The swizzle key is y >> SH with 16 / NC =
// 2^SH rows per 128-byte line, so 16 consecutive rows of one column fall in 16 distinct bank
// pairs.
template <int L, typename SPEC, int V = 0>
__device__ __forceinline__ void pass_a_body(float2* smem, const float2* __restrict__ I,
                                            const typename SPEC::T* __restrict__ T, float2* __restrict__ Q, int b0,
                                            int n0, int D, const float2* __restrict__ twL, int p, int cgroup,
                                            bool wait_before_store, const SkipMask& sk) {
  constexpr int TT = PassA<L, V>::TT, NC = PassA<L, V>::NC, E = L / TT, NZ = L / 2, HS = NZ + 1;
  using CX = ColXform<L, TT>;
  constexpr int SH = NC >= 16 ? 0 : NC == 8 ? 1 : 2;
  static_assert(NC == 4 || NC == 8 || NC == 16, "swizzle assumes 4, 8 or 16 slots per CTA");
  static_assert(TT <= 32 && 32 % TT == 0, "a team lies inside one warp");
  const int team = threadIdx.x / TT, tid = threadIdx.x - team * TT;
  const int c0 = cgroup * NC, c = c0 + team;
  const int e = p / D, d = p - e * D;
  if ((sk.windows && !sk.windows[b0 + e]) || !sk.pair_live(b0 + e, n0 + d)) {  // nothing needed (CTA-uniform)
    if (wait_before_store) griddep_wait();  // complete only after the kernel before, as when storing
    return;
  }
  const float2* Ib = I + (size_t)(b0 + e) * HS * L;
  const typename SPEC::T* Tn = T + (size_t)(n0 + d) * HS * L;
  float2 v[E];
  if (c == 0) {
    // columns kx = 0 and kx = L/2 have real inverse transforms: pack them as a + i b
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int ky = CX::in_index(tid, i);
      const float2 a = cmulc(Ib[ky], SPEC::load(Tn + ky));
      const float2 b = cmulc(Ib[(size_t)NZ * L + ky], SPEC::load(Tn + (size_t)NZ * L + ky));
      v[i] = make_float2(a.x - b.y, a.y + b.x);
    }
  } else {
    const float2* Ic = Ib + (size_t)c * L;
    const typename SPEC::T* Tc = Tn + (size_t)c * L;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int ky = CX::in_index(tid, i);
      v[i] = cmulc(__ldg(Ic + ky), SPEC::load(Tc + ky));
    }
  }
  CX::run(v, smem + team * L, twL, tid);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int y = CX::out_index(tid, i);
    smem[y * NC + (team ^ ((y >> SH) & (NC - 1)))] = v[i];
  }
  __syncthreads();
  if (wait_before_store) griddep_wait();  // Q is still being read by the previous pass B
  float2* Qp = Q + (size_t)p * L * NZ + c0;
  constexpr int HALF = NC / 2;  // 16-byte pairs per row segment
  // (a runtime loop: unrolled, with the swizzle at 16-byte granularity so that no pair needs
  // its halves swapped, the launch pair measured 75.0 against 69.9 us at window 512)
  const unsigned char* live = sk.rows ? sk.rows + (size_t)(b0 + e) * L : nullptr;
  for (int u = threadIdx.x; u < L * HALF; u += TT * NC) {
    const int y = u / HALF, k = (u - y * HALF) * 2, sw = (y >> SH) & (NC - 1);
    if (live && !live[y]) continue;  // a row the next pass skips
    const float4 q = *reinterpret_cast<const float4*>(smem + y * NC + ((k ^ sw) & ~1));
    *reinterpret_cast<float4*>(Qp + (size_t)y * NZ + k) =
        (sw & 1) ? make_float4(q.z, q.w, q.x, q.y) : q;
  }
}

template <int TEAM>
__device__ __forceinline__ unsigned long long team_max_u64(unsigned long long k) {
#pragma unroll
  for (int off = TEAM / 2; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(0xffffffffu, k, off, TEAM);
    k = o > k ? o : k;
  }
  return k;
}
// Maximum over each group of W lanes (a power of two up to 32) of the warp.
template <int W>
__device__ __forceinline__ float group_max(float x) {
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, off, W));
  return x;
}
template <int TEAM>
__device__ __forceinline__ double team_sum_f64(double x) {
#pragma unroll
  for (int off = TEAM / 2; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off, TEAM);
  return x;
}
template <int TEAM>
__device__ __forceinline__ bool team_any(bool pred) {
  unsigned b = __ballot_sync(0xffffffffu, pred);
  if constexpr (TEAM == 32) {
    return b != 0;
  } else {
    const int sh = (threadIdx.x & 31) & ~(TEAM - 1);
    return ((b >> sh) & ((1u << TEAM) - 1u)) != 0;
  }
}

// The row transform of pass B: the Hermitian half row (NZ + 1 values, the kx = 0 and kx = L/2
// terms packed in slot 0) becomes L real values through a length-NZ complex inverse transform
// of Z[k] = E[k] + i W_L^-k O[k] (E, O: the even / odd parts of the half row) and lane output j
// = (x[2j], x[2j + 1]).  EIN inputs and EOUT outputs per lane; the row's shared-memory slice is
// the exchange buffer once every lane of the team has read its inputs.
template <int L, int TEAM>
struct RowXform {
  static constexpr int NZ = L / 2, EIN = NZ / TEAM, EOUT = NZ / TEAM, EBUF = EIN;
  __device__ __forceinline__ static int out_index(int lt, int i) { return fft3_out_index<NZ, TEAM>(lt, i); }
  template <typename Sync>
  __device__ __forceinline__ static void run(float2* v, float2* row, const float2* tw_nz, const float2* tw_l, int lt,
                                             Sync tsync) {
    // only a lane's first input can be the row's slot 0 (lane 0)
    v[0] = row_unpack<NZ>(row, tw_l, fft3_in_index<NZ, TEAM>(lt, 0));
#pragma unroll
    for (int i = 1; i < EIN; ++i) v[i] = row_unpack<NZ, false>(row, tw_l, fft3_in_index<NZ, TEAM>(lt, i));
    tsync();  // every lane of the team has read the row before the transform overwrites it
    fft3<NZ, TEAM, +1>(v, row, TwShared{tw_nz}, lt, tsync);
  }
};
// Window 320: the 160-point row transform on 16 lanes as two Stockham stages, radix 16 then
// radix 10.  Stage 1 has 10 butterflies (lanes 0-9, 16 inputs x[j + 10 m] each); stage 2 has
// 16 (every lane, 10 inputs x[j + 16 m] with twiddles W_160^(j m)) and leaves lane j the outputs
// X[j + 16 r], r < 10: 20 pixels per lane, so the per-pixel accumulators of the epilogues stay
// in registers.  The exchange goes through the row's slice with the 16-slot XOR swizzle.
template <>
struct RowXform<320, 16> {
  static constexpr int NZ = 160, EIN = 16, EOUT = 10, EBUF = 16;
  __device__ __forceinline__ static int out_index(int lt, int i) { return lt + 16 * i; }
  template <typename Sync>
  __device__ __forceinline__ static void run(float2* v, float2* row, const float2* tw_nz, const float2* tw_l, int lt,
                                             Sync tsync) {
    if (lt < 10) {
      v[0] = row_unpack<NZ>(row, tw_l, lt);
#pragma unroll
      for (int m = 1; m < EIN; ++m) v[m] = row_unpack<NZ, false>(row, tw_l, lt + 10 * m);
    }
    tsync();
    if (lt < 10) {
      Dft<16, +1>::run(v);
#pragma unroll
      for (int r = 0; r < 16; ++r) row[fft_swz<4>(lt * 16 + r)] = v[r];
    }
    tsync();
#pragma unroll
    for (int m = 0; m < 10; ++m) v[m] = row[fft_swz<4>(lt + 16 * m)];
    float2 w[10];
    tw_powers<10>(table_tw<+1>(TwShared{tw_nz}, lt), w);
#pragma unroll
    for (int m = 1; m < 10; ++m) v[m] = cmul(v[m], w[m]);
    Dft<10, +1>::run(v);
  }
};

// A chunk pick: the chunk's best key (z, 255 - brev8(position in the chunk)) at or above the
// threshold whose pixel's centre passes the border test becomes a candidate (norm.cu:583-597).
template <int L>
__device__ __forceinline__ void emit_chunk(const CorrArgs& a, unsigned long long key, int chunk, int win, int templ,
                                           int angle) {
  const float zb = key_float((uint32_t)(key >> 32));
  if (!(zb >= a.thresh)) return;
  const int t = brev8(255 - (unsigned)(key & 0xffu));
  const int id = chunk * 256 + t;
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
  cd.templ = templ;
  cd.angle = angle;
  cd.chunk = chunk;
  cd.pad = 0;
  a.cand[slot] = cd;
}

}  // namespace
}  // namespace gisspa
