// pair_engine.cu — the two correlation passes of consecutive launch batches run side by side.
//
// Pass A (column transforms) waits mostly on global loads and pass B (row transforms and the
// epilogue) mostly on instruction issue; launched one after the other each has the SMs to itself
// and leaves about half of the issue slots idle.  Here one launch runs pass A of batch j and
// pass B of batch j - 1 (Q double-buffered, so the two are independent), in CTAs that take work
// items from two counters: the first CTA to arrive on an SM does pass A items first, the second
// pass B rows first, and each turns to the other pass when its own runs out.  Every SM then holds
// warps of both passes for most of the launch.  A sequence of nb batches takes nb + 1 launches
// (the first only pass A, the last only pass B); the outputs, their order and rounding are those
// of the per-pass kernels (correlate.cu): the same device code computes every value.
//
// Window 512 only, epilogues EPI_SUM, EPI_SUMMAX, EPI_TOPK and EPI_CHUNK.  Pass B runs one warp per row (the
// per-pass kernel's 32-lane team), each warp with its own double-buffered stage of Q rows filled
// by bulk copies, so B rows need no CTA-wide barrier.
#include "../../include/gisspa.h"
#include "corr_body.cuh"

namespace gisspa {
namespace {

constexpr int kL = 512, kNZ = 256;
constexpr int kThreads = 256, kWarps = kThreads / 32;
constexpr int kNC = PassA<kL>::NC;                 // column slots per pass-A item
constexpr int kGroups = kNZ / kNC;                 // pass-A items per pair
static_assert(PassA<kL>::TT * kNC == kThreads, "a pass-A item takes the whole CTA");
constexpr int kSmSlots = 256;                      // SM ids counted for the role split
constexpr size_t kTileBytes = (size_t)kNC * kL * sizeof(float2);          // pass A: 64 KiB
constexpr size_t kStageBytes = (size_t)kWarps * 2 * kNZ * sizeof(float2);  // pass B: 32 KiB
constexpr size_t kSmem = kTileBytes + kStageBytes;

struct EngineArgs {
  const float2* I;
  const void* T;
  const float2* twL;
  const float2* twNZ;
  EngineBatch A;  // pass A of this batch (valid = 0: none)
  EngineBatch B;  // pass B of this batch
  CorrArgs b;     // the epilogue's arguments for batch B (Q, b0, n0, D of B)
  int* ctr;       // [0] next pass-A item, [1] next pass-B row, [2 ..) CTAs seen per SM
  int chained;    // a launch of the same sequence precedes this one on the stream
};

// One row of one window of batch B over the batch's D templates: the per-pass kernel's row
// chain (pass_b_kernel with a 32-lane team and one row per team) run by one warp.  `ph` holds
// the parities of the warp's two stage barriers.  Returns false after a wait gave up (the
// warp's copies in flight have landed by then).
template <int EPI>
__device__ __forceinline__ bool engine_row(const CorrArgs& a, int e, int y, float2* stage, uint64_t* bars, unsigned& ph,
                                           const float2* tw_nz, const float2* tw_l, int lane) {
  using RX = RowXform<kL, 32>;
  constexpr int E = RX::EOUT;
  const int win = a.b0 + e;
  if constexpr (EPI == EPI_CHUNK)
    if (a.skip.rows && !a.skip.rows[(size_t)win * kL + y]) return true;  // a row that cannot hold a pick
  const int angle = a.angle_state ? a.angle_state->index : a.angle;
  const int oy = (y + kL / 2) % kL;
  const float inv = 1.0f / (float)(kL * kL);
  const size_t wbase = (size_t)win * kL * kL;
  int ox[E];
#pragma unroll
  for (int i = 0; i < E; ++i) ox[i] = (2 * RX::out_index(lane, i) + kL / 2) % kL;

  float2 acc1[E], acc2[E];  // pixels 2j, 2j + 1 of output element j as pairs
  constexpr bool SUMS = EPI == EPI_SUM || EPI == EPI_TOPK || EPI == EPI_SUMMAX;
  float best[(EPI == EPI_TOPK || EPI == EPI_SUMMAX) ? E : 1][2];
  int barg[(EPI == EPI_TOPK) ? E : 1][2];
  float2 mu[(EPI == EPI_CHUNK) ? E : 1], isg[(EPI == EPI_CHUNK) ? E : 1];
  if constexpr (SUMS) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      acc1[i] = make_float2(0.f, 0.f);
      acc2[i] = make_float2(0.f, 0.f);
      if constexpr (EPI == EPI_TOPK || EPI == EPI_SUMMAX) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          best[i][h] = -INFINITY;
          if constexpr (EPI == EPI_TOPK) barg[i][h] = -1;
        }
      }
    }
  }
  if constexpr (EPI == EPI_CHUNK) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const float4 m = *reinterpret_cast<const float4*>(a.musig + wbase + (size_t)oy * kL + ox[i]);
      mu[i] = make_float2(m.x * (float)(kL * kL), m.z * (float)(kL * kL));
      isg[i] = make_float2(m.y * inv, m.w * inv);
    }
  }

  auto issue = [&](int d) {
    const float2* src = a.Q + ((size_t)(e * a.D + d) * kL + y) * kNZ;
    fence_proxy_async_smem();
    mbar_expect_tx(&bars[d & 1], kNZ * sizeof(float2));
    bulk_g2s(stage + (d & 1) * kNZ, src, kNZ * sizeof(float2), &bars[d & 1]);
  };
  __syncwarp();  // every lane is done with both stage buffers (the previous row)
  if (lane == 0) issue(0);
  int issued = 1;
  for (int d = 0; d < a.D; ++d) {
    if (lane == 0 && d + 1 < a.D) {
      issue(d + 1);
      ++issued;
    }
    const unsigned par = (ph >> (d & 1)) & 1u;
    const bool ok = mbar_wait(&bars[d & 1], par, 4000000000LL);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) {
        atomicOr(a.err, 1u);
        // copies still in flight land before the shared memory goes away
        unsigned p2 = ph;
        for (int k = d; k < issued; ++k) {
          mbar_wait(&bars[k & 1], (p2 >> (k & 1)) & 1u, 400000000LL);
          p2 ^= 1u << (k & 1);
        }
      }
      __syncwarp();
      return false;
    }
    ph ^= 1u << (d & 1);
    float2 v[RX::EBUF];
    RX::run(v, stage + (d & 1) * kNZ, tw_nz, tw_l, lane, WarpSync{});

    if constexpr (SUMS) {
#pragma unroll
      for (int i = 0; i < E; ++i) {
        acc1[i] = cadd(acc1[i], v[i]);  // raw: the 1/L^2 is applied when folding
        acc2[i] = pfma(v[i], v[i], acc2[i]);
        if constexpr (EPI == EPI_SUMMAX) {
          best[i][0] = fmaxf(best[i][0], v[i].x);
          best[i][1] = fmaxf(best[i][1], v[i].y);
        }
        if constexpr (EPI == EPI_TOPK) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float c = h ? v[i].y : v[i].x;
            if (c > best[i][h]) {
              best[i][h] = c;
              barg[i][h] = angle * a.nt_total + a.n0 + d;
            }
          }
        }
      }
      if constexpr (EPI == EPI_SUMMAX) {
        if (a.pair_max) {  // the pair's maximum over the window, this row's part
          float m = -INFINITY;
#pragma unroll
          for (int i = 0; i < E; ++i) m = fmaxf(m, fmaxf(v[i].x, v[i].y));
          m = group_max<32>(m);
          if (lane == 0)
            atomicMax(a.pair_max + pair_index(win, a.n0 + d, angle, a.n_windows, a.n_angles), float_key(m * inv));
        }
      }
    } else if constexpr (EPI == EPI_CHUNK) {
      constexpr int CPR = kL / 256;
      const int c0 = (oy * kL) >> 8;
      float z[E][2];
      float zmax = -INFINITY;
#pragma unroll
      for (int i = 0; i < E; ++i) {
        const float2 zz = pmul(csub(v[i], mu[i]), isg[i]);
        z[i][0] = zz.x;
        z[i][1] = zz.y;
        zmax = fmaxf(zmax, fmaxf(zz.x, zz.y));
      }
      if (__any_sync(0xffffffffu, zmax >= a.thresh)) {
#pragma unroll
        for (int ch = 0; ch < CPR; ++ch) {
          unsigned long long key = 0;
#pragma unroll
          for (int i = 0; i < E; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int x = ox[i] + h;
              if (((oy * kL + x) >> 8) - c0 != ch) continue;
              const int t = (oy * kL + x) & 255;
              const unsigned long long k2 = ((unsigned long long)float_key(z[i][h]) << 32) | (unsigned)(255 - brev8(t));
              key = k2 > key ? k2 : key;
            }
          key = team_max_u64<32>(key);
          if (lane == 0) emit_chunk<kL>(a, key, c0 + ch, win, a.n0 + d, angle);
        }
      }
    }
    __syncwarp();  // this stage buffer is refilled two templates later
  }

  if constexpr (SUMS) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const size_t pix = wbase + (size_t)oy * kL + ox[i];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        atomicAdd(a.S1 + pix + h, (double)((h ? acc1[i].y : acc1[i].x) * inv));
        atomicAdd(a.S2 + pix + h, (double)((h ? acc2[i].y : acc2[i].x) * (inv * inv)));
        if constexpr (EPI == EPI_TOPK) {
          if (barg[i][h] >= 0)
            atomicMax(a.peak + pix + h, ((unsigned long long)float_key(best[i][h] * inv) << 32) |
                                            (unsigned)(0xFFFFFFFFu - (unsigned)barg[i][h]));
        }
        if constexpr (EPI == EPI_SUMMAX)
          atomicMax(a.peak + pix + h, (unsigned long long)float_key(best[i][h] * inv) << 32);
      }
    }
  }
  return true;
}

// The engine skips rows and windows of a pruned second sweep, not pairs: its pass B rows read
// every template of the batch.
template <int EPI>
__device__ __forceinline__ SkipMask engine_mask(const SkipMask& sk) {
  SkipMask m{};
  if constexpr (EPI == EPI_CHUNK) {
    m.rows = sk.rows;
    m.windows = sk.windows;
  }
  return m;
}

template <typename SPEC, int EPI>
__global__ void __launch_bounds__(kThreads, 2) pair_engine_kernel(EngineArgs g) {
  extern __shared__ __align__(128) float2 dsm[];  // pass-A tile [NC * L], then pass-B stages [warp][2][NZ]
  __shared__ __align__(8) uint64_t bars[kWarps][2];
  __shared__ __align__(16) float2 tw_nz[kNZ + kNZ / 16], tw_l[kNZ];
  __shared__ int s_item[2], s_role, s_abort;
  float2* tile = dsm;
  float2* stages = dsm + kNC * kL;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kNZ; i += kThreads) {
    tw_nz[tw_pad_index(i)] = __ldg(g.twNZ + i);
    tw_l[i] = __ldg(g.twL + i);
  }
  if (threadIdx.x == 0) {
    for (int w = 0; w < kWarps; ++w) {
      mbar_init(&bars[w][0], 1);
      mbar_init(&bars[w][1], 1);
    }
    fence_mbar_init();
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    s_role = atomicAdd(g.ctr + 2 + (smid % kSmSlots), 1) & 1;  // 0: pass A first, 1: pass B first
    s_abort = 0;
  }
  griddep_launch_dependents();
  if (!g.chained) griddep_wait();  // the template spectra may come from the kernel just before
  __syncthreads();
  const int role = s_role;
  unsigned ph = 0;
  for (int phase = 0; phase < 2; ++phase) {
    if ((phase == 0) == (role == 0) && g.A.valid) {
      // pass A items: (pair, group of NC column slots), the whole CTA per item
      const int nitems = kGroups * g.A.d * g.A.e;
      for (int k = 0;; ++k) {
        if (threadIdx.x == 0) s_item[k & 1] = s_abort ? nitems : atomicAdd(g.ctr, 1);
        __syncthreads();  // also: the previous item's output tile has been read
        const int it = s_item[k & 1];
        if (it >= nitems) break;
        pass_a_body<kL, SPEC>(tile, g.I, static_cast<const typename SPEC::T*>(g.T), g.A.Q, g.A.b0, g.A.n0, g.A.d,
                              g.twL, it / kGroups, it % kGroups, g.chained != 0,
                              engine_mask<EPI>(g.b.skip));
      }
    } else if ((phase == 0) != (role == 0) && g.B.valid) {
      // pass B rows: (window, row) of batch B, one warp per row
      if (g.chained) griddep_wait();  // Q of batch B comes from the launch just before
      const int nrows = kL * g.B.e;
      for (;;) {
        int r = 0;
        if (lane == 0) r = *reinterpret_cast<volatile int*>(&s_abort) ? nrows : atomicAdd(g.ctr + 1, 1);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= nrows) break;
        if (!engine_row<EPI>(g.b, r / kL, r % kL, stages + warp * 2 * kNZ, bars[warp], ph, tw_nz, tw_l, lane)) {
          if (lane == 0) s_abort = 1;
          break;
        }
      }
    }
    __syncthreads();
  }
}

template <typename SPEC, int EPI>
void launch_cfg(const EngineArgs& g, cudaStream_t s) {
  static PerDeviceOnce once;
  static int grid[64] = {};
  int dev = 0;
  GISSPA_CUDA(cudaGetDevice(&dev));
  once([dev] {
    GISSPA_CUDA(cudaFuncSetAttribute(pair_engine_kernel<SPEC, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSmem));
    GISSPA_CUDA(cudaFuncSetAttribute(pair_engine_kernel<SPEC, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     100));
    int sms = 0, per_sm = 0;
    GISSPA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    GISSPA_CUDA(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_engine_kernel<SPEC, EPI>, kThreads, kSmem));
    if (dev < 64) grid[dev] = sms * std::max(1, per_sm);
  });
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(dev < 64 && grid[dev] > 0 ? grid[dev] : 296);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  GISSPA_CUDA(cudaLaunchKernelEx(&cfg, pair_engine_kernel<SPEC, EPI>, g));
  ++launch_counter();
}

template <typename SPEC>
void launch_spec(int epi, const EngineArgs& g, cudaStream_t s) {
  switch (epi) {
    case EPI_SUM: launch_cfg<SPEC, EPI_SUM>(g, s); break;
    case EPI_SUMMAX: launch_cfg<SPEC, EPI_SUMMAX>(g, s); break;
    case EPI_TOPK: launch_cfg<SPEC, EPI_TOPK>(g, s); break;
    case EPI_CHUNK: launch_cfg<SPEC, EPI_CHUNK>(g, s); break;
    default: throw CudaError{cudaErrorInvalidValue, "pair engine without this epilogue"};
  }
}

}  // namespace

bool engine_supported(int L, int epi) {
  return L == kL && (epi == EPI_SUM || epi == EPI_SUMMAX || epi == EPI_TOPK || epi == EPI_CHUNK);
}

size_t engine_counter_ints() { return 2 + kSmSlots; }

void engine_launch(int spec, int epi, const float2* I, const void* T, const EngineBatch& A, const EngineBatch& B,
                   const CorrArgs& b_args, int* ctr, bool chained, const float2* twL, const float2* twNZ,
                   cudaStream_t s) {
  EngineArgs g;
  g.I = I;
  g.T = T;
  g.twL = twL;
  g.twNZ = twNZ;
  g.A = A;
  g.B = B;
  g.b = b_args;
  if (B.valid) {
    g.b.Q = B.Q;
    g.b.b0 = B.b0;
    g.b.n0 = B.n0;
    g.b.D = B.d;
  }
  g.ctr = ctr;
  g.chained = chained ? 1 : 0;
  switch (spec) {
    case GISSPA_SPEC_FP32: launch_spec<SpecFp32>(epi, g, s); break;
    case GISSPA_SPEC_FP16: launch_spec<SpecFp16>(epi, g, s); break;
    case GISSPA_SPEC_BF16: launch_spec<SpecBf16>(epi, g, s); break;
    default: throw CudaError{cudaErrorInvalidValue, "unknown spectrum precision"};
  }
}

}  // namespace gisspa
