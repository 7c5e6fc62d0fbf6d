// correlate.cu — pass A (multiply + column IFFT) and pass B (row C2R + epilogue).
#include <mutex>
#include <utility>

#include "../../include/gisspa.h"
#include "corr_body.cuh"

namespace gisspa {
namespace {

// Pass A kernel: one pair per blockIdx.y, NC column slots per blockIdx.x (pass_a_body).
template <int L, typename SPEC, int V>
__global__ void __launch_bounds__(PassA<L, V>::TT * PassA<L, V>::NC, PassA<L, V>::MINB)
    pass_a_kernel(const float2* __restrict__ I, const typename SPEC::T* __restrict__ T, float2* __restrict__ Q,
                  int b0, int n0, int D, const float2* __restrict__ twL, int chained, SkipMask sk) {
  extern __shared__ __align__(16) float2 smem[];  // [NC * L]: FFT exchange buffers, then the output tile
  griddep_launch_dependents();
  if (!chained) griddep_wait();  // the spectra may come from the kernel just before
  pass_a_body<L, SPEC, V>(smem, I, T, Q, b0, n0, D, twL, blockIdx.y, blockIdx.x, chained != 0, sk);
}

// Pass A of a pruned second sweep: one CTA per pair looping over the column groups, so that the
// (almost all) dead pairs cost one CTA each instead of one per column group.
template <int L, typename SPEC, int V>
__global__ void __launch_bounds__(PassA<L, V>::TT * PassA<L, V>::NC, PassA<L, V>::MINB)
    pass_a_pair_kernel(const float2* __restrict__ I, const typename SPEC::T* __restrict__ T, float2* __restrict__ Q,
                       int b0, int n0, int D, const float2* __restrict__ twL, int chained, SkipMask sk) {
  extern __shared__ __align__(16) float2 smem[];
  constexpr int NZ = L / 2, NC = PassA<L, V>::NC;
  griddep_launch_dependents();
  if (!chained) griddep_wait();
  const int p = blockIdx.x, e = p / D, d = p - e * D;
  if ((sk.windows && !sk.windows[b0 + e]) || !sk.pair_live(b0 + e, n0 + d)) {
    if (chained) griddep_wait();  // complete only after the kernel before, as when storing
    return;
  }
  for (int cg = 0; cg < NZ / NC; ++cg) {
    if (cg) __syncthreads();  // the previous group's output tile has been read
    pass_a_body<L, SPEC, V>(smem, I, T, Q, b0, n0, D, twL, p, cg, chained != 0, sk);
  }
}

// Pass B: a team (TEAM lanes) per output row; RB rows per CTA, one window per blockIdx.y,
// looping over the launch's D templates.  The RB rows of each template are one
// contiguous block of Q: one bulk asynchronous copy per template into a
// double-buffered shared stage, completed on an mbarrier, so the next template's rows
// arrive while this one is transformed.  Every wait is bounded: on timeout the CTA
// sets *a.err and leaves.
template <int L, int TEAM, int RB, int NW, int EPI, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB)
    pass_b_kernel(CorrArgs a, const float2* __restrict__ twL, const float2* __restrict__ twNZ) {
  using RX = RowXform<L, TEAM>;
  constexpr int NZ = L / 2, E = RX::EOUT, NTEAM = NW * 32 / TEAM, RPT = RB / NTEAM;
  static_assert(TEAM <= 32 || (TEAM % 32 == 0 && NTEAM <= 15), "a wide team is whole warps with its own barrier");
  constexpr unsigned kStageBytes = RB * NZ * sizeof(float2);
  static_assert(RB % NTEAM == 0, "rows must split evenly over teams");
  extern __shared__ __align__(128) float2 stage[];  // [2][RB][NZ]
  __shared__ __align__(8) uint64_t bars[2];
  // the row transform's table (length NZ) and the first NZ entries of the length-L table
  // used by the even/odd unpack, staged once: every row of every template reads them
  __shared__ __align__(16) float2 tw_nz[NZ + NZ / 16], tw_l[NZ];
  for (int i = threadIdx.x; i < NZ; i += NW * 32) {
    tw_nz[tw_pad_index(i)] = __ldg(twNZ + i);
    tw_l[i] = __ldg(twL + i);
  }
  const int team = threadIdx.x / TEAM, lt = threadIdx.x - team * TEAM;
  const int e = blockIdx.y, y0 = blockIdx.x * RB, win = a.b0 + e;
  if constexpr (EPI == EPI_CHUNK) {
    // rows that cannot hold a pick are skipped; a CTA with none left leaves at once, after the
    // pass A before it has completed (so that this kernel completes after it, as when it reads Q)
    if (a.skip.rows) {
      bool any = false;
      for (int r = 0; r < RB; ++r) any = any || a.skip.rows[(size_t)win * L + y0 + r] != 0;
      if (!any) {
        griddep_wait();
        return;
      }
    }
  }
  const int angle = a.angle_state ? a.angle_state->index : a.angle;
  // L = 320: the CTA's output rows (L/2 + y0 ...) hold whole chunks (RB a multiple of 4 that
  // divides L/2: 4 rows = 5 chunks, and the rows never wrap inside one CTA); their maxima are
  // gathered per template in chunk_part
  static_assert(L % 256 == 0 || (L == 320 && RB % 4 == 0 && (L / 2) % RB == 0), "chunks must not leave the CTA");
  constexpr int kChunks = (L % 256 == 0 || EPI != EPI_CHUNK) ? 1 : RB * L / 256;
  __shared__ unsigned long long chunk_part[kChunks];
  const int cbase = (((y0 + L / 2) % L) * L) >> 8;
  if (L % 256 != 0 && EPI == EPI_CHUNK)
    for (int q = threadIdx.x; q < kChunks; q += NW * 32) chunk_part[q] = 0ull;
  // The correlation is the raw transform times 1/L^2, a power of two: scaling by it commutes
  // exactly with float rounding (no overflow or underflow at these magnitudes), so the sums,
  // the running maxima and the z-scores work on raw values and apply it once, bit for bit
  // as if every value had been scaled first.
  // (For L = 320 the factor is not a power of two; applying it once instead of to every value
  // then changes the results by FP32 rounding only.)
  const float inv = 1.0f / (float)(L * L);
  const size_t wbase = (size_t)win * L * L;
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  // the launch's templates this CTA transforms: all of them, or for a pruned second sweep those
  // whose pair with this window is live (pass A stored no Q for the others)
  __shared__ unsigned char live_d[EPI == EPI_CHUNK ? kMaxListedTemplates : 1];
  __shared__ int n_live;
  int nd = a.D;
  bool listed = false;
  if constexpr (EPI == EPI_CHUNK) {
    listed = a.skip.pairs != nullptr && a.D <= kMaxListedTemplates;
    if (listed) {
      for (int d = threadIdx.x; d < a.D; d += NW * 32) live_d[d] = a.skip.pair_live(win, a.n0 + d) ? 1 : 0;
      __syncthreads();
      if (threadIdx.x == 0) {
        int n = 0;
        for (int d = 0; d < a.D; ++d)
          if (live_d[d]) live_d[n++] = (unsigned char)d;
        n_live = n;
      }
    }
  }
  __syncthreads();
  if (listed) {
    nd = n_live;
    if (nd == 0) {  // (CTA-uniform) as for dead rows above
      griddep_wait();
      return;
    }
  }
  auto dof = [&](int k) { return listed ? (int)live_d[k] : k; };
  griddep_launch_dependents();
  griddep_wait();  // Q comes from the pass A just before
  auto issue = [&](int k) {
    const float2* src = a.Q + ((size_t)(e * a.D + dof(k)) * L + y0) * NZ;
    fence_proxy_async_smem();
    mbar_expect_tx(&bars[k & 1], kStageBytes);
    bulk_g2s(stage + (k & 1) * RB * NZ, src, kStageBytes, &bars[k & 1]);
  };
  if (threadIdx.x == 0) issue(0);

  // per-lane pixel coordinates: element i, half h -> (out_y of row s, out_x)
  int ox[E];
#pragma unroll
  for (int i = 0; i < E; ++i) ox[i] = (2 * RX::out_index(lt, i) + L / 2) % L;

  // per-pixel sums as pairs (pixels 2j, 2j + 1 of output element j): one paired FP32
  // instruction adds a row's two values, with the rounding of two scalar additions
  float2 acc1[RPT][E], acc2[RPT][E];
  constexpr bool SUMS = EPI == EPI_SUM || EPI == EPI_TOPK || EPI == EPI_SUMMAX;
  float best[(EPI == EPI_TOPK || EPI == EPI_SUMMAX) ? RPT : 1][E][2];
  int barg[(EPI == EPI_TOPK) ? RPT : 1][E][2];
  float2 mu[(EPI == EPI_CHUNK) ? RPT : 1][E], isg[(EPI == EPI_CHUNK) ? RPT : 1][E];
  if constexpr (SUMS) {
#pragma unroll
    for (int s = 0; s < RPT; ++s)
#pragma unroll
      for (int i = 0; i < E; ++i) {
        acc1[s][i] = make_float2(0.f, 0.f);
        acc2[s][i] = make_float2(0.f, 0.f);
        if constexpr (EPI == EPI_TOPK || EPI == EPI_SUMMAX) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            best[s][i][h] = -INFINITY;
            if constexpr (EPI == EPI_TOPK) barg[s][i][h] = -1;
          }
        }
      }
  }
  if constexpr (EPI == EPI_CHUNK) {
#pragma unroll
    for (int s = 0; s < RPT; ++s) {
      const int oy = (y0 + team + NTEAM * s + L / 2) % L;
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const float4 m = *reinterpret_cast<const float4*>(a.musig + wbase + (size_t)oy * L + ox[i]);
        // (mu L^2, (1/sigma) / L^2): z = (raw - mu L^2) (1/sigma) / L^2 = (c - mu) / sigma exactly
        mu[s][i] = make_float2(m.x * (float)(L * L), m.z * (float)(L * L));
        isg[s][i] = make_float2(m.y * inv, m.w * inv);
      }
    }
  }

  __shared__ unsigned pmax_s[2];  // EPI_SUMMAX: the pair maximum of templates k, k + 1
  if (EPI == EPI_SUMMAX && threadIdx.x < 2) pmax_s[threadIdx.x] = 0u;
  __syncthreads();
  int issued = 1;
  for (int k = 0; k < nd; ++k) {
    const int d = dof(k);
    const int p = e * a.D + d;
    if (threadIdx.x == 0 && k + 1 < nd) {
      issue(k + 1);
      ++issued;
    }
    const bool ok = mbar_wait(&bars[k & 1], (k >> 1) & 1, 4000000000LL);
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) {
        atomicOr(a.err, 1u);
        // let copies already in flight land before the CTA's shared memory goes away
        for (int j = k; j < issued; ++j) mbar_wait(&bars[j & 1], (j >> 1) & 1, 400000000LL);
      }
      __syncthreads();
      return;
    }
    float2* stg = stage + (k & 1) * RB * NZ;
    double nn_s1 = 0.0, nn_s2 = 0.0;
#pragma unroll
    for (int s = 0; s < RPT; ++s) {
      const int r = team + NTEAM * s;
      const int oy = (y0 + r + L / 2) % L;
      // a dead row (pass A did not store it) is skipped by its team; half-warp teams stay in
      // step (the chunk vote uses the whole warp): they transform it and discard its values
      const bool row_live = EPI != EPI_CHUNK || !a.skip.rows || a.skip.rows[(size_t)win * L + y0 + r];
      if constexpr (EPI == EPI_CHUNK && TEAM >= 32)
        if (!row_live) continue;
      float2* row = stg + r * NZ;
      float2 v[RX::EBUF];
      const TeamSync<TEAM> tsync{1 + team};
      RX::run(v, row, tw_nz, tw_l, lt, tsync);

      if constexpr (SUMS) {
#pragma unroll
        for (int i = 0; i < E; ++i) {
          // raw values: the 1/L^2 is applied when folding
          acc1[s][i] = cadd(acc1[s][i], v[i]);
          acc2[s][i] = pfma(v[i], v[i], acc2[s][i]);
          if constexpr (EPI == EPI_SUMMAX) {
            best[s][i][0] = fmaxf(best[s][i][0], v[i].x);
            best[s][i][1] = fmaxf(best[s][i][1], v[i].y);
          }
          if constexpr (EPI == EPI_TOPK) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const float c = h ? v[i].y : v[i].x;
              if (c > best[s][i][h]) {
                best[s][i][h] = c;
                barg[s][i][h] = angle * a.nt_total + a.n0 + d;
              }
            }
          }
        }
        if constexpr (EPI == EPI_SUMMAX) {
          // the pair's maximum over the window: this row's, reduced over the warp (the rows of
          // a warp's teams belong to the same pair) with one integer max on the float keys, then
          // over the CTA's warps in shared memory, and sent once per template (below)
          if (a.pair_max) {
            float m = -INFINITY;
#pragma unroll
            for (int i = 0; i < E; ++i) m = fmaxf(m, fmaxf(v[i].x, v[i].y));
            const unsigned km = __reduce_max_sync(0xffffffffu, float_key(m * inv));
            if ((threadIdx.x & 31) == 0) atomicMax(&pmax_s[k & 1], km);
          }
        }
      } else if constexpr (EPI == EPI_CHUNK) {
        // chunks (256 consecutive pixels of the window's linear index) touched by one row: whole
        // chunks for L a multiple of 256; at L = 320 a row starts 0, 64, 128 or 192 pixels into
        // a chunk and always touches two, each shared with a neighbouring row
        constexpr int CPR = L % 256 == 0 ? L / 256 : 2;
        const int c0 = (oy * L) >> 8;
        // a team wider than a warp (two warps per row) meets in shared memory: the warps'
        // votes and chunk maxima, behind the team's barrier (the next writes come after the
        // next row's barriers)
        constexpr int WT = TEAM > 32 ? TEAM / 32 : 1;
        __shared__ int chunk_vote[TEAM > 32 ? NTEAM : 1][WT];
        __shared__ unsigned long long chunk_key[TEAM > 32 ? NTEAM : 1][WT][CPR];
        const int wid = TEAM > 32 ? (lt >> 5) : 0;
        float z[E][2];
        float zmax = -INFINITY;
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const float2 zz = pmul(csub(v[i], mu[s][i]), isg[s][i]);
          z[i][0] = row_live ? zz.x : -INFINITY;
          z[i][1] = row_live ? zz.y : -INFINITY;
          zmax = fmaxf(zmax, fmaxf(z[i][0], z[i][1]));
        }
        // warp-uniform (and, for wide teams, team-uniform) branch: the shuffles below use the
        // full warp mask, so both half-warp teams (TEAM = 16) must enter together
        bool hit = __any_sync(0xffffffffu, zmax >= a.thresh);
        if constexpr (TEAM > 32) {
          if ((threadIdx.x & 31) == 0) chunk_vote[team][wid] = hit;
          tsync();
          hit = false;
#pragma unroll
          for (int w = 0; w < WT; ++w) hit = hit || chunk_vote[team][w];
        }
        if (hit) {
          unsigned long long keys[CPR];
#pragma unroll
          for (int ch = 0; ch < CPR; ++ch) {
            unsigned long long key = 0;
#pragma unroll
            for (int i = 0; i < E; ++i)
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const int x = ox[i] + h;
                if (((oy * L + x) >> 8) - c0 != ch) continue;
                const int t = (oy * L + x) & 255;
                const unsigned long long k2 =
                    ((unsigned long long)float_key(z[i][h]) << 32) | (unsigned)(255 - brev8(t));
                key = k2 > key ? k2 : key;
              }
            keys[ch] = team_max_u64<(TEAM > 32 ? 32 : TEAM)>(key);
          }
          if constexpr (L % 256 != 0) {
            // the row's part of each chunk meets the other row's in shared memory; the chunks
            // are complete once every team has done this template (see after the row loop)
            if (lt == 0)
#pragma unroll
              for (int ch = 0; ch < CPR; ++ch) atomicMax(&chunk_part[c0 + ch - cbase], keys[ch]);
          } else {
            if constexpr (TEAM > 32) {
              if ((threadIdx.x & 31) == 0)
#pragma unroll
                for (int ch = 0; ch < CPR; ++ch) chunk_key[team][wid][ch] = keys[ch];
              tsync();
              if (lt == 0)
#pragma unroll
                for (int ch = 0; ch < CPR; ++ch)
#pragma unroll
                  for (int w = 1; w < WT; ++w)
                    keys[ch] = keys[ch] > chunk_key[team][w][ch] ? keys[ch] : chunk_key[team][w][ch];
            }
            if (lt == 0)
#pragma unroll
              for (int ch = 0; ch < CPR; ++ch) emit_chunk<L>(a, keys[ch], c0 + ch, win, a.n0 + d, angle);
          }
        }
      } else if constexpr (EPI == EPI_NONORM) {
        static_assert(TEAM <= 32, "peak and sums reduce within a warp");
        constexpr int CPR = L % 256 == 0 ? L / 256 : 2;
        const int c0 = (oy * L) >> 8;
        // get_peak_and_SUM (kernels.cu:725-763): sums over every pixel, max with the
        // border (closer than diameter/4 to the window edge) forced to 0
#pragma unroll
        for (int i = 0; i < E; ++i) {
          nn_s1 += (double)v[i].x + (double)v[i].y;
          nn_s2 += (double)v[i].x * v[i].x + (double)v[i].y * v[i].y;
        }
#pragma unroll
        for (int ch = 0; ch < CPR; ++ch) {
          unsigned long long key = 0;
#pragma unroll
          for (int i = 0; i < E; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int x = ox[i] + h;
              if (((oy * L + x) >> 8) - c0 != ch) continue;
              float val = h ? v[i].y : v[i].x;
              if (x < a.border || x > L - a.border || oy < a.border || oy > L - a.border) val = 0.f;
              const int t = (oy * L + x) & 255;
              const unsigned long long k2 =
                  ((unsigned long long)float_key(val) << 32) | (unsigned)(255 - brev8(t));
              key = k2 > key ? k2 : key;
            }
          key = team_max_u64<TEAM>(key);
          if (lt == 0) {
            const float vb = key_float((uint32_t)(key >> 32));
            if (vb > 0.f) {
              // largest value, then the lowest chunk, then the reference's in-chunk order (the
              // byte 255 - brev8(t)): parts of one chunk from two rows combine correctly
              const int chunk = c0 + ch;
              const unsigned long long g = ((unsigned long long)float_key(vb) << 32) |
                                           ((unsigned long long)(0xFFFFFu - chunk) << 8) | (key & 0xffu);
              atomicMax(a.nn_key + (size_t)win * a.nt_total + a.n0 + d, g);
            }
          }
        }
      } else if constexpr (EPI == EPI_MAP) {
        float* out = a.map_out + (size_t)p * L * L + (size_t)oy * L;
#pragma unroll
        for (int i = 0; i < E; ++i)
          *reinterpret_cast<float2*>(out + ox[i]) = make_float2(v[i].x * inv, v[i].y * inv);
      }
    }
    if constexpr (EPI == EPI_CHUNK && L % 256 != 0) {
      __syncthreads();  // every row part of this template's chunks is in
      for (int q = threadIdx.x; q < kChunks; q += NW * 32) {
        const unsigned long long key = chunk_part[q];
        chunk_part[q] = 0ull;
        if (key) emit_chunk<L>(a, key, cbase + q, win, a.n0 + d, angle);
      }
    }
    if constexpr (EPI == EPI_NONORM) {
      nn_s1 = team_sum_f64<TEAM>(nn_s1);
      nn_s2 = team_sum_f64<TEAM>(nn_s2);
      if (lt == 0) {
        const size_t q = (size_t)win * a.nt_total + a.n0 + d;
        atomicAdd(a.nn_sum + 2 * q, nn_s1);
        atomicAdd(a.nn_sum + 2 * q + 1, nn_s2);
      }
    }
    __syncthreads();  // this stage buffer is refilled two templates later
    if constexpr (EPI == EPI_SUMMAX) {
      // every team's row maximum of template d is in (the next template uses the other slot)
      if (threadIdx.x == 0 && a.pair_max) {
        atomicMax(a.pair_max + pair_index(win, a.n0 + d, angle, a.n_windows, a.n_angles), pmax_s[k & 1]);
        pmax_s[k & 1] = 0u;
      }
    }
  }

  // Fold this launch's partial sums (and maxima) into the per-pixel state with reductions that
  // return nothing, so no warp waits on the state's memory latency.  Each pixel receives one
  // reduction per launch and launches are stream-ordered: the additions happen in the same
  // order, with the same rounding, as a read-modify-write.
  if constexpr (SUMS) {
#pragma unroll
    for (int s = 0; s < RPT; ++s) {
      const int oy = (y0 + team + NTEAM * s + L / 2) % L;
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const size_t pix = wbase + (size_t)oy * L + ox[i];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          atomicAdd(a.S1 + pix + h, (double)((h ? acc1[s][i].y : acc1[s][i].x) * inv));
          atomicAdd(a.S2 + pix + h, (double)((h ? acc2[s][i].y : acc2[s][i].x) * (inv * inv)));
          if constexpr (EPI == EPI_TOPK) {
            if (barg[s][i][h] >= 0)
              atomicMax(a.peak + pix + h, ((unsigned long long)float_key(best[s][i][h] * inv) << 32) |
                                              (unsigned)(0xFFFFFFFFu - (unsigned)barg[s][i][h]));
          }
          if constexpr (EPI == EPI_SUMMAX)
            atomicMax(a.peak + pix + h, (unsigned long long)float_key(best[s][i][h] * inv) << 32);
        }
      }
    }
  }
}

// Launch with programmatic stream serialization (the kernel's griddep_wait orders it after
// its predecessor).
template <typename... P, typename... A>
void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  GISSPA_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
  ++launch_counter();
}

// Pass A's mask: pairs only where pass B lists the live templates (D small enough).
SkipMask a_mask(const CorrLaunch& cl, const CorrArgs& args) {
  SkipMask m = args.skip;
  if (cl.D > kMaxListedTemplates) m.pairs = nullptr;
  return m;
}

template <int L, typename SPEC, int V>
void launch_a_cfg(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
                  const float2* twL, cudaStream_t s) {
  constexpr int NZ = L / 2;
  using P = PassA<L, V>;
  constexpr size_t smem = (size_t)P::NC * L * sizeof(float2);
  static PerDeviceOnce once;
  once([] {
    GISSPA_CUDA(
        cudaFuncSetAttribute(pass_a_kernel<L, SPEC, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
  const SkipMask sk = cl.epi == EPI_CHUNK ? a_mask(cl, args) : SkipMask{};
  if (sk.pairs) {
    static PerDeviceOnce once_pair;
    once_pair([] {
      GISSPA_CUDA(cudaFuncSetAttribute(pass_a_pair_kernel<L, SPEC, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    });
    launch_pdl(pass_a_pair_kernel<L, SPEC, V>, dim3(cl.E * cl.D), dim3(P::TT * P::NC), smem, s, I,
               static_cast<const typename SPEC::T*>(T), Q, args.b0, args.n0, cl.D, twL, cl.chained ? 1 : 0, sk);
    return;
  }
  dim3 grid(NZ / P::NC, cl.E * cl.D);
  launch_pdl(pass_a_kernel<L, SPEC, V>, grid, dim3(P::TT * P::NC), smem, s, I,
             static_cast<const typename SPEC::T*>(T), Q, args.b0, args.n0, cl.D, twL, cl.chained ? 1 : 0, sk);
}
template <int L, typename SPEC>
void launch_a(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
              const float2* twL, cudaStream_t s) {
  if constexpr (L == 512) {
    if (cl.a_variant == 1) {
      launch_a_cfg<L, SPEC, 1>(cl, I, T, Q, args, twL, s);
      return;
    }
  }
  launch_a_cfg<L, SPEC, 0>(cl, I, T, Q, args, twL, s);
}

template <int L, int TEAM, int RB, int NW, int EPI, int MINB>
void launch_b_cfg(const CorrLaunch& cl, const CorrArgs& args, const float2* twL, const float2* twNZ,
                  cudaStream_t s) {
  constexpr size_t smem = 2 * (size_t)RB * (L / 2) * sizeof(float2);
  static PerDeviceOnce once;
  once([] {
    GISSPA_CUDA(cudaFuncSetAttribute(pass_b_kernel<L, TEAM, RB, NW, EPI, MINB>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
  dim3 grid(L / RB, cl.E);
  launch_pdl(pass_b_kernel<L, TEAM, RB, NW, EPI, MINB>, grid, dim3(NW * 32), smem, s, args, twL, twNZ);
}

// Pass B shapes (rows per CTA RB, warps NW, min CTAs per SM) per window size and variant.
template <int L, int V>
struct PassB;
// A launch has L x E row chains (a window row over the launch's D templates).  Large CTAs
// share the bulk copies and tables; CTAs of one or two rows spread the chains evenly over the
// SMs when L x E is not much larger than the warps the GPU holds (e.g. 2048 chains at E = 4).
template <> struct PassB<256, 0> { static constexpr int TEAM = 16, RB = 16, NW = 8, MINB = 2; };
template <> struct PassB<256, 1> { static constexpr int TEAM = 16, RB = 4, NW = 2, MINB = 8; };
template <> struct PassB<512, 0> { static constexpr int TEAM = 32, RB = 16, NW = 16, MINB = 1; };
template <> struct PassB<512, 1> { static constexpr int TEAM = 32, RB = 8, NW = 8, MINB = 2; };
template <> struct PassB<512, 2> { static constexpr int TEAM = 32, RB = 2, NW = 2, MINB = 8; };
template <> struct PassB<512, 3> { static constexpr int TEAM = 32, RB = 1, NW = 1, MINB = 16; };
// window 320: 16-lane rows (the 16 x 10 row plan), RB a multiple of 4 dividing 160 so that the
// chunk picks stay inside the CTA
template <> struct PassB<320, 0> { static constexpr int TEAM = 16, RB = 16, NW = 8, MINB = 1; };
template <> struct PassB<320, 1> { static constexpr int TEAM = 16, RB = 8, NW = 4, MINB = 2; };
template <> struct PassB<320, 2> { static constexpr int TEAM = 16, RB = 4, NW = 2, MINB = 4; };
template <> struct PassB<1024, 0> { static constexpr int TEAM = 32, RB = 8, NW = 8, MINB = 1; };
template <> struct PassB<1024, 1> { static constexpr int TEAM = 32, RB = 2, NW = 2, MINB = 2; };
// the same, capped at 168 registers (6 CTAs per SM): no spills for the sum and chunk epilogues
template <> struct PassB<1024, 2> { static constexpr int TEAM = 32, RB = 2, NW = 2, MINB = 6; };
// 64-lane rows (8 points and 16 pixels per lane: half the accumulators); every epilogue but
// norm_type=0's
template <> struct PassB<1024, 3> { static constexpr int TEAM = 64, RB = 2, NW = 4, MINB = 4; };
template <> struct PassB<1024, 4> { static constexpr int TEAM = 64, RB = 1, NW = 2, MINB = 8; };

template <int L, int V>
void launch_b(const CorrLaunch& cl, const CorrArgs& args, const float2* twL, const float2* twNZ, cudaStream_t s) {
  using P = PassB<L, V>;
  if constexpr (P::TEAM > 32) {
    switch (cl.epi) {
      case EPI_SUM: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_SUM, P::MINB>(cl, args, twL, twNZ, s); break;
      case EPI_SUMMAX: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_SUMMAX, P::MINB>(cl, args, twL, twNZ, s); break;
      case EPI_TOPK: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_TOPK, P::MINB>(cl, args, twL, twNZ, s); break;
      case EPI_CHUNK: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_CHUNK, P::MINB>(cl, args, twL, twNZ, s); break;
      case EPI_MAP: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_MAP, P::MINB>(cl, args, twL, twNZ, s); break;
      default: throw CudaError{cudaErrorInvalidValue, "pass B shape without this epilogue"};
    }
    return;
  } else {
  switch (cl.epi) {
    case EPI_SUM: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_SUM, P::MINB>(cl, args, twL, twNZ, s); break;
    case EPI_SUMMAX: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_SUMMAX, P::MINB>(cl, args, twL, twNZ, s); break;
    case EPI_CHUNK: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_CHUNK, P::MINB>(cl, args, twL, twNZ, s); break;
    case EPI_TOPK: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_TOPK, P::MINB>(cl, args, twL, twNZ, s); break;
    case EPI_NONORM: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_NONORM, P::MINB>(cl, args, twL, twNZ, s); break;
    case EPI_MAP: launch_b_cfg<L, P::TEAM, P::RB, P::NW, EPI_MAP, P::MINB>(cl, args, twL, twNZ, s); break;
    default: throw CudaError{cudaErrorInvalidValue, "unknown epilogue"};
  }
  }
}

template <int L>
int launch_pair(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
                const float2* twL, const float2* twNZ, cudaStream_t s, cudaEvent_t* ev) {
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[0], s));
  switch (cl.spec) {
    case GISSPA_SPEC_FP32: launch_a<L, SpecFp32>(cl, I, T, Q, args, twL, s); break;
    case GISSPA_SPEC_FP16:
      if (L == 512 && cl.tc)
        launch_a_tc(cl, I, T, Q, args, twL, s);
      else
        launch_a<L, SpecFp16>(cl, I, T, Q, args, twL, s);
      break;
    case GISSPA_SPEC_BF16: launch_a<L, SpecBf16>(cl, I, T, Q, args, twL, s); break;
    default: throw CudaError{cudaErrorInvalidValue, "unknown spectrum precision"};
  }
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[1], s));
  if constexpr (L == 512) {
    if (cl.tc && cl.spec == GISSPA_SPEC_FP16 && cl.epi == EPI_TOPK) {
      launch_b_tc(cl, args, twL, twNZ, s);
      if (ev) GISSPA_CUDA(cudaEventRecord(ev[2], s));
      return 2;
    }
    switch (cl.variant) {
      case 1: launch_b<L, 1>(cl, args, twL, twNZ, s); break;
      case 2: launch_b<L, 2>(cl, args, twL, twNZ, s); break;
      case 3: launch_b<L, 3>(cl, args, twL, twNZ, s); break;
      case 0: launch_b<L, 0>(cl, args, twL, twNZ, s); break;
      default: throw CudaError{cudaErrorInvalidValue, "the pair engine runs through engine_launch"};
    }
  } else if constexpr (L == 320) {
    switch (cl.variant) {
      case 1: launch_b<L, 1>(cl, args, twL, twNZ, s); break;
      case 2: launch_b<L, 2>(cl, args, twL, twNZ, s); break;
      default: launch_b<L, 0>(cl, args, twL, twNZ, s); break;
    }
  } else if constexpr (L == 1024) {
    switch (cl.variant) {
      case 1: launch_b<L, 1>(cl, args, twL, twNZ, s); break;
      case 2: launch_b<L, 2>(cl, args, twL, twNZ, s); break;
      case 3: launch_b<L, 3>(cl, args, twL, twNZ, s); break;
      case 4: launch_b<L, 4>(cl, args, twL, twNZ, s); break;
      default: launch_b<L, 0>(cl, args, twL, twNZ, s); break;
    }
  } else {
    if (cl.variant == 1)
      launch_b<L, 1>(cl, args, twL, twNZ, s);
    else
      launch_b<L, 0>(cl, args, twL, twNZ, s);
  }
  if (ev) GISSPA_CUDA(cudaEventRecord(ev[2], s));
  return 2;
}

}  // namespace

int pass_a_variants(int L) { return L == 512 ? 2 : 1; }

bool correlate_supported(int L) { return L == 256 || L == 512 || L == 1024; }

// At window 512 shape 4 is the pair engine (pair_engine.cu), launched as a sequence by the caller.
int correlate_variants(int L) { return L == 512 ? 5 : L == 1024 ? 5 : L == 320 ? 3 : 2; }

int engine_variant(int L) { return L == 512 ? 4 : -1; }

bool correlate_variant_ok(int L, int variant, int epi) {
  if (variant < 0 || variant >= correlate_variants(L)) return false;
  if (variant == engine_variant(L)) return engine_supported(L, epi);
  const bool wide = L == 1024 && variant >= 3;  // 64-lane rows
  return !wide || epi == EPI_SUM || epi == EPI_SUMMAX || epi == EPI_TOPK || epi == EPI_CHUNK || epi == EPI_MAP;
}

int correlate_launch(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args_in,
                     const float2* twL, const float2* twNZ, cudaStream_t s, cudaEvent_t* ev) {
  CorrArgs args = args_in;
  args.skip.angle = args.angle;
  args.skip.angle_state = args.angle_state;
  switch (cl.L) {
    case 256: return launch_pair<256>(cl, I, T, Q, args, twL, twNZ, s, ev);
    case 320: return launch_pair<320>(cl, I, T, Q, args, twL, twNZ, s, ev);
    case 512: return launch_pair<512>(cl, I, T, Q, args, twL, twNZ, s, ev);
    case 1024: return launch_pair<1024>(cl, I, T, Q, args, twL, twNZ, s, ev);
    default: throw CudaError{cudaErrorInvalidValue, "window size without correlation kernels"};
  }
}

}  // namespace gisspa
