// colmma.cu — pass A on the tensor cores: the column transforms of the correlation as two
// small DFT-matrix products per column on tcgen05, for FP16 template spectra at window 512 (the
// chosen form's precision).  Same inputs, outputs and launch grid as pass_a_kernel<512,
// SpecFp16> (correlate.cu); pass B is unchanged.
//
// A column Z[ky] (ky < 512; the kx = 0 and kx = 256 columns packed as a + i b in slot 0) is
// inverse-transformed as out[k1 + 16 k2] = sum_n2 e^(2 pi i n2 k2 / 32) e^(2 pi i n2 k1 / 512)
// sum_n1 e^(2 pi i n1 k1 / 16) Z[32 n1 + n2]:
//   stage 1  Y[n2][k1] = sum_n1 x[n1][n2] F16[n1][k1]     (MMA, M = (column, n2), K = n1, N = k1)
//   twiddle  Y[n2][k1] *= e^(2 pi i n2 k1 / 512)           (CUDA cores, FP32)
//   stage 2  out[k1 + 16 k2] = sum_n2 Y[n2][k1] F32[n2][k2] (MMA, M = (column, k1), K = n2, N = k2)
// Complex products are real GEMMs over (real, imaginary) halves of K and N.  Operands are FP16
// (the column data and the DFT matrices), accumulation FP32 in tensor memory, twiddles FP32.
// Peak scores stay within 3e-4 of FP64 (the chosen form's bar is 1e-3).
//
// One CTA (4 warps) owns 16 column slots of one (window, template) pair, in two groups of 8:
// per group, two stage-1 MMAs (4 columns x 32 rows each, M = 128, N = 32, K = 32) and one
// stage-2 MMA (8 columns x 16 rows, M = 128, N = 64, K = 64).  Every thread loads the 16 points
// of one column row (coalesced along n2), and after each MMA reads one tensor-memory lane.
#include "../../include/gisspa.h"
#include "correlate.cuh"
#include "fft.cuh"
#include "tcgen05.cuh"

namespace gisspa {
namespace {

constexpr int kL = 512, kNZ = 256, kHS = 257;
constexpr int kThreads = 128;
constexpr int kSlotsPerCta = 64;
constexpr uint32_t kTmemCols = 128;
// K-major tiles (tcgen05.cuh): stage-1 data 128 rows x 32 halves (two tiles), stage-2 data
// 128 rows x 64 halves (LBO padded to 144 bytes: the transposing 2-byte stores of a warp then
// fall in distinct banks), the DFT matrices 32 x 32 and 64 x 64
constexpr uint32_t kLbo1 = 128, kSbo1 = 512, kLbo2 = 144, kSbo2 = 8 * 144, kLboB = 128;
constexpr uint32_t kSboB1 = 512, kSboB2 = 1024;
constexpr uint32_t kOffA1 = 0, kA1Tile = 16 * kSbo1;              // 2 x 8192
constexpr uint32_t kOffA2 = kOffA1 + 2 * kA1Tile;                  // 16384
constexpr uint32_t kOffB1 = kOffA2 + 16 * kSbo2;                   // + 18432
constexpr uint32_t kOffB2 = kOffB1 + 4 * kSboB1;                   // + 2048
constexpr uint32_t kSmem = kOffB2 + 8 * kSboB2;                    // + 8192
static_assert(kOffA2 % 16 == 0 && kOffB1 % 16 == 0 && kOffB2 % 16 == 0, "16-byte tiles");

__device__ __forceinline__ void st_half(uint8_t* base, uint32_t off, float v) {
  *reinterpret_cast<__half*>(base + off) = __float2half_rn(v);
}

// The constant operands, built once per device by tc_tables_kernel and copied into every CTA's
// shared memory: the 16-point inverse DFT as a real 32 x 32 block (rows (q, k1), columns
// (p, n1)), the 32-point one as a real 64 x 64 block, both K-major FP16 tiles, and the FP32
// twiddles e^(+2 pi i p / 512).  F = e^(+i theta): rows q = 0 give the real output, q = 1 the
// imaginary; columns p = 0 multiply the real input, p = 1 the imaginary.
constexpr uint32_t kTabB16 = 0, kTabB32 = 32 * 64, kTabTw = kTabB32 + 64 * 128, kTabBytes = kTabTw + kL * 8;
static __device__ __align__(16) uint8_t g_tc_tables[kTabBytes];

__global__ void tc_tables_kernel() {
  for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) {
    const int nn = i >> 5, k = i & 31, q = nn >> 4, k1 = nn & 15, pp = k >> 4, n1 = k & 15;
    const int a = (2 * n1 * k1) & 31;  // angle in units of 2 pi / 32
    const float c = (float)cos32(a), s = (float)sin32(a);
    st_half(g_tc_tables + kTabB16, kmajor_off(nn, k, 128, 512), q == 0 ? (pp == 0 ? c : -s) : (pp == 0 ? s : c));
  }
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int nn = i >> 6, k = i & 63, q = nn >> 5, k2 = nn & 31, pp = k >> 5, n2 = k & 31;
    const int a = (n2 * k2) & 31;
    const float c = (float)cos32(a), s = (float)sin32(a);
    st_half(g_tc_tables + kTabB32, kmajor_off(nn, k, 128, 1024), q == 0 ? (pp == 0 ? c : -s) : (pp == 0 ? s : c));
  }
  float2* tw = reinterpret_cast<float2*>(g_tc_tables + kTabTw);
  for (int i = threadIdx.x; i < kL; i += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * i / kL, &sn, &cs);
    tw[i] = make_float2((float)cs, (float)sn);
  }
}

// Copies n bytes (a multiple of 16) of the constant tables into shared memory.
__device__ __forceinline__ void copy_table(uint8_t* dst, uint32_t src_off, uint32_t n) {
  const uint4* src = reinterpret_cast<const uint4*>(g_tc_tables + src_off);
  for (uint32_t i = threadIdx.x; i < n / 16; i += blockDim.x) reinterpret_cast<uint4*>(dst)[i] = src[i];
}

__global__ void __launch_bounds__(kThreads, 4)
    pass_a_tc_kernel(const float2* __restrict__ I, const __half2* __restrict__ T, float2* __restrict__ Q, int b0,
                     int n0, int D, const float2* __restrict__ twL, int chained, unsigned* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int p = blockIdx.y, e = p / D, d = p - e * D;
  const int c0 = blockIdx.x * kSlotsPerCta;

  // constant operands (g_tc_tables): B1[nn = (q, k1)][k = (p, n1)], B2[nn = (q, k2)][k = (p, n2)]
  copy_table(sm + kOffB1, kTabB16, 2048);
  copy_table(sm + kOffB2, kTabB32, 8192);
  // this thread's twiddles e^(2 pi i n2 k1 / 512), n2 = lane, for every group
  float2 twr[16];
  {
    const float2* tg = reinterpret_cast<const float2*>(g_tc_tables + kTabTw);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) twr[k1] = tg[lane * k1];
  }
  if (t == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  if (w == 0) tmem_alloc(&tmem_slot, kTmemCols);
  griddep_launch_dependents();
  if (!chained) griddep_wait();  // the spectra may come from the kernel just before
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = (uint32_t)(32 * w) << 16;

  const float2* Ib = I + (size_t)(b0 + e) * kHS * kL;
  const __half2* Tn = T + (size_t)(n0 + d) * kHS * kL;
  float2* Qp = Q + (size_t)p * kL * kNZ;
  unsigned parity = 0;
  bool ok = true;
  bool waited = chained == 0;
  for (int g = 0; g < kSlotsPerCta / 8 && ok; ++g) {
    // ---- load: thread (w, lane) fills row n2 = lane of columns c8 = w and w + 4
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = c0 + 8 * g + w + 4 * h;
      float re[16], im[16];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const int ky = 32 * n1 + lane;
        float2 v;
        if (c == 0) {
          const float2 a = cmulc(__ldg(Ib + ky), __half22float2(Tn[ky]));
          const float2 b = cmulc(__ldg(Ib + (size_t)kNZ * kL + ky), __half22float2(Tn[(size_t)kNZ * kL + ky]));
          v = make_float2(a.x - b.y, a.y + b.x);
        } else {
          v = cmulc(__ldg(Ib + (size_t)c * kL + ky), __half22float2(Tn[(size_t)c * kL + ky]));
        }
        re[n1] = v.x;
        im[n1] = v.y;
      }
      uint8_t* a1 = sm + kOffA1 + h * kA1Tile;
      const int m = 32 * w + lane;
#pragma unroll
      for (int kg = 0; kg < 4; ++kg) {
        uint32_t u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int i0 = 8 * (kg & 1) + 2 * j;
          const __half2 hh = kg < 2 ? __floats2half2_rn(re[i0], re[i0 + 1]) : __floats2half2_rn(im[i0], im[i0 + 1]);
          u[j] = *reinterpret_cast<const uint32_t*>(&hh);
        }
        *reinterpret_cast<uint4*>(a1 + kmajor_off(m, 8 * kg, kLbo1, kSbo1)) = make_uint4(u[0], u[1], u[2], u[3]);
      }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      const uint32_t idesc = idesc_f16(128, 32);
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int ks = 0; ks < 2; ++ks)
          tc_mma_f16(tmem + 32 * h,
                     smem_desc(smem_u32(sm + kOffA1 + h * kA1Tile) + ks * 2 * kLbo1, kLbo1, kSbo1),
                     smem_desc(smem_u32(sm + kOffB1) + ks * 2 * kLboB, kLboB, kSboB1), idesc, ks);
      tc_commit(&bar);
    }
    ok = __syncthreads_and(mbar_wait(&bar, parity, 4000000000LL));
    parity ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // ---- twiddles and the stage-2 operand: A2[(c8, k1)][(part, n2)]
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v[32];
      tmem_ld32(tmem + lane_base + 32 * h, v);  // row (c8 = w + 4h, n2 = lane): Yr[k1], Yi[k1]
      const int c8 = w + 4 * h;
#pragma unroll
      for (int k1 = 0; k1 < 16; ++k1) {
        const float2 z = cmul(make_float2(v[k1], v[16 + k1]), twr[k1]);
        st_half(sm + kOffA2, kmajor_off(16 * c8 + k1, lane, kLbo2, kSbo2), z.x);
        st_half(sm + kOffA2, kmajor_off(16 * c8 + k1, 32 + lane, kLbo2, kSbo2), z.y);
      }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      const uint32_t idesc = idesc_f16(128, 64);
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        tc_mma_f16(tmem + 64, smem_desc(smem_u32(sm + kOffA2) + ks * 2 * kLbo2, kLbo2, kSbo2),
                   smem_desc(smem_u32(sm + kOffB2) + ks * 2 * kLboB, kLboB, kSboB2), idesc, ks);
      tc_commit(&bar);
    }
    ok = __syncthreads_and(mbar_wait(&bar, parity, 4000000000LL));
    parity ^= 1u;
    if (!ok) break;
    tc_fence_after();
    // ---- outputs: row (c8, k1) = lane 32 w + lane holds out[k1 + 16 k2], k2 < 32
    float zr[32], zi[32];
    tmem_ld32(tmem + lane_base + 64, zr);
    tmem_ld32(tmem + lane_base + 96, zi);
    if (!waited) {
      griddep_wait();  // Q is still being read by the previous pass B
      waited = true;
    }
    // through a shared tile (the operand tiles are free now): rows y, 8 slots XOR-swizzled by
    // y mod 8, read back as 16-byte slot pairs so that each row segment leaves contiguous
    const int c8 = 2 * w + (lane >> 4), k1 = lane & 15;
    float2* tile = reinterpret_cast<float2*>(sm + kOffA1);
#pragma unroll
    for (int k2 = 0; k2 < 32; ++k2) {
      const int y = k1 + 16 * k2;
      tile[y * 8 + (c8 ^ (y & 7))] = make_float2(zr[k2], zi[k2]);
    }
    __syncthreads();
    float2* dst = Qp + c0 + 8 * g;
#pragma unroll
    for (int i = 0; i < kL * 4 / kThreads; ++i) {
      const int u = t + kThreads * i, y = u >> 2, k = (u & 3) * 2, sw = y & 7;
      const float4 q = *reinterpret_cast<const float4*>(tile + y * 8 + ((k ^ sw) & ~1));
      *reinterpret_cast<float4*>(dst + (size_t)y * kNZ + k) = (sw & 1) ? make_float4(q.z, q.w, q.x, q.y) : q;
    }
    tc_fence_before();
    __syncthreads();  // tensor memory and the operand tiles are reused by the next group
    tc_fence_after();
  }
  if (!ok) {
    if (t == 0) {
      atomicOr(err, 1u);
      // let an MMA still in flight finish before its tensor memory is released
      mbar_wait(&bar, parity ^ 1u, 400000000LL);
    }
    tc_fence_before();
    __syncthreads();
  }
  if (w == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---- pass B on the tensor cores (top-K epilogue)
//
// A row of the map (512 real pixels) comes from its half row Q[y][0..256) through the unpack
// Z[k] = E[k] + i W_512^-k O[k] (CUDA cores) and the 256-point inverse transform
// X[k1 + 16 k2] = sum_n2 e^(2 pi i n2 k2 / 16) e^(2 pi i n2 k1 / 256) sum_n1 e^(2 pi i n1 k1 / 16)
// Z[16 n1 + n2], pixels (2j, 2j + 1) = (Re, Im) X[j]:
//   stage 1  M = (row, n2) 8 x 16, K = (part, n1) 32, N = (part, k1) 32
//   twiddle  e^(2 pi i n2 k1 / 256), FP32
//   stage 2  M = (row, k1) 8 x 16, K = (part, n2) 32, N = (part, k2) 32
// against one 16-point DFT matrix as a real 32 x 32 block.  A CTA (4 warps) owns 8 rows of one
// window and loops over the launch's D templates; the rows of each template arrive by one bulk
// copy into a double-buffered stage, as in pass B.  Thread t reads tensor-memory lane t: after
// stage 2 that is (row t / 16, k1 = t % 16), the same 32 pixels for every template, whose sums,
// squares and maxima stay in registers and are folded into the state once per launch.
constexpr int kRowsB = 8;
constexpr uint32_t kTmemColsB = 64;
constexpr uint32_t kLboA = 128, kSboA = 512;           // stage-1 operand 128 x 32
// stage-2 operand 128 x 32: LBO 144 and SBO 592 bytes keep the transposing 2-byte stores of a
// warp (two rows 16 apart, 16 lanes each) in distinct banks
constexpr uint32_t kLboC = 144, kSboC = 592;
// stage rows padded by 16 bytes (one bulk copy per row): the unpack's reads of two rows by one
// warp then fall in distinct banks
constexpr uint32_t kRowPitch = kNZ * sizeof(float2) + 16;                  // 2064
constexpr uint32_t kStageB = kRowsB * kRowPitch;                           // 16512 per template
constexpr uint32_t kStageBytes = kRowsB * kNZ * sizeof(float2);            // 16384 copied
constexpr uint32_t kOffStage = 0;                                          // 2 x 16384
constexpr uint32_t kOffOpA = 2 * kStageB + 128 - (2 * kStageB) % 128;       // 128-aligned, 8192
constexpr uint32_t kOffOpC = kOffOpA + 16 * kSboA;                         // 40960, 9216
constexpr uint32_t kOffDft = kOffOpC + 16 * kSboC;                         // 50176, 2048
constexpr uint32_t kOffTwL = kOffDft + 4 * 512;                            // 52224, 2048
constexpr uint32_t kOffTwN = kOffTwL + kNZ * sizeof(float2);              // 54272, 2048
constexpr uint32_t kSmemB = kOffTwN + kNZ * sizeof(float2);               // 56320
static_assert(kOffOpA % 128 == 0 && kOffOpC % 16 == 0 && kOffDft % 16 == 0 && kOffTwL % 16 == 0, "aligned tiles");

__global__ void __launch_bounds__(kThreads, 2)
    pass_b_tc_kernel(CorrArgs a, const float2* __restrict__ twL, const float2* __restrict__ twNZ) {
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ __align__(8) uint64_t bars[3];  // two stage buffers, the MMAs
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, w = t >> 5;
  const int e = blockIdx.y, y0 = blockIdx.x * kRowsB, win = a.b0 + e;
  const int angle = a.angle_state ? a.angle_state->index : a.angle;
  float2* tw_l = reinterpret_cast<float2*>(sm + kOffTwL);
  float2* tw_n = reinterpret_cast<float2*>(sm + kOffTwN);
  for (int i = t; i < kNZ; i += kThreads) {
    tw_l[i] = __ldg(twL + i);
    const float2 v = __ldg(twNZ + i);
    tw_n[i] = make_float2(v.x, -v.y);  // e^(+2 pi i p / 256)
  }
  copy_table(sm + kOffDft, kTabB16, 2048);  // the 16-point inverse DFT as a real 32 x 32 block
  if (t == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
  }
  if (w == 0) tmem_alloc(&tmem_slot, kTmemColsB);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = (uint32_t)(32 * w) << 16;
  griddep_launch_dependents();
  griddep_wait();  // Q comes from the pass A just before
  auto issue = [&](int d) {
    const float2* src = a.Q + ((size_t)(e * a.D + d) * kL + y0) * kNZ;
    fence_proxy_async_smem();
    mbar_expect_tx(&bars[d & 1], kStageBytes);
#pragma unroll
    for (int r = 0; r < kRowsB; ++r)
      bulk_g2s(sm + kOffStage + (d & 1) * kStageB + r * kRowPitch, src + (size_t)r * kNZ, kNZ * sizeof(float2),
               &bars[d & 1]);
  };
  if (t == 0) issue(0);

  // this thread's 32 pixels after stage 2: row r, pixels 2 (k1 + 16 k2) + {0, 1}
  const int r2 = t >> 4, k1o = t & 15;
  float acc1[32], acc2[32], best[32];
  int barg[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    acc1[i] = 0.f;
    acc2[i] = 0.f;
    best[i] = -INFINITY;
    barg[i] = -1;
  }
  int issued = 1, dcur = 0;
  unsigned mma_parity = 0;
  bool ok = true;
  for (int d = 0; d < a.D; ++d) {
    dcur = d;
    if (t == 0 && d + 1 < a.D) {
      issue(d + 1);
      ++issued;
    }
    ok = __syncthreads_and(mbar_wait(&bars[d & 1], (d >> 1) & 1, 4000000000LL));
    if (!ok) break;
    const float2* stg = reinterpret_cast<const float2*>(sm + kOffStage + (d & 1) * kStageB);
    // unpack: thread t fills operand row (r = t / 16, n2 = t % 16) with Z[16 n1 + n2], n1 < 16
    {
      const int r = t >> 4, n2 = t & 15;
      const float2* row = reinterpret_cast<const float2*>(reinterpret_cast<const uint8_t*>(stg) + r * kRowPitch);
      uint32_t pk_re[8], pk_im[8];
#pragma unroll
      for (int n1 = 0; n1 < 16; n1 += 2) {
        const float2 z0 = row_unpack<kNZ>(row, tw_l, 16 * n1 + n2);
        const float2 z1 = row_unpack<kNZ>(row, tw_l, 16 * (n1 + 1) + n2);
        const __half2 hr = __floats2half2_rn(z0.x, z1.x), hi = __floats2half2_rn(z0.y, z1.y);
        pk_re[n1 >> 1] = *reinterpret_cast<const uint32_t*>(&hr);
        pk_im[n1 >> 1] = *reinterpret_cast<const uint32_t*>(&hi);
      }
      uint8_t* op = sm + kOffOpA;
      *reinterpret_cast<uint4*>(op + kmajor_off(t, 0, kLboA, kSboA)) = make_uint4(pk_re[0], pk_re[1], pk_re[2], pk_re[3]);
      *reinterpret_cast<uint4*>(op + kmajor_off(t, 8, kLboA, kSboA)) = make_uint4(pk_re[4], pk_re[5], pk_re[6], pk_re[7]);
      *reinterpret_cast<uint4*>(op + kmajor_off(t, 16, kLboA, kSboA)) = make_uint4(pk_im[0], pk_im[1], pk_im[2], pk_im[3]);
      *reinterpret_cast<uint4*>(op + kmajor_off(t, 24, kLboA, kSboA)) = make_uint4(pk_im[4], pk_im[5], pk_im[6], pk_im[7]);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();  // the stage buffer is free again: every row was unpacked
    if (t == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 2; ++ks)
        tc_mma_f16(tmem, smem_desc(smem_u32(sm + kOffOpA) + ks * 2 * kLboA, kLboA, kSboA),
                   smem_desc(smem_u32(sm + kOffDft) + ks * 2 * kLboB, kLboB, kSboB1), idesc_f16(128, 32), ks);
      tc_commit(&bars[2]);
    }
    ok = __syncthreads_and(mbar_wait(&bars[2], mma_parity, 4000000000LL));
    mma_parity ^= 1u;
    if (!ok) break;
    tc_fence_after();
    {
      float v[32];
      tmem_ld32(tmem + lane_base, v);  // lane t = (r, n2): Y[k1] re, im
      const int r = t >> 4, n2 = t & 15;
#pragma unroll
      for (int k1 = 0; k1 < 16; ++k1) {
        const float2 z = cmul(make_float2(v[k1], v[16 + k1]), tw_n[n2 * k1]);
        st_half(sm + kOffOpC, kmajor_off(16 * r + k1, n2, kLboC, kSboC), z.x);
        st_half(sm + kOffOpC, kmajor_off(16 * r + k1, 16 + n2, kLboC, kSboC), z.y);
      }
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < 2; ++ks)
        tc_mma_f16(tmem + 32, smem_desc(smem_u32(sm + kOffOpC) + ks * 2 * kLboC, kLboC, kSboC),
                   smem_desc(smem_u32(sm + kOffDft) + ks * 2 * kLboB, kLboB, kSboB1), idesc_f16(128, 32), ks);
      tc_commit(&bars[2]);
    }
    ok = __syncthreads_and(mbar_wait(&bars[2], mma_parity, 4000000000LL));
    mma_parity ^= 1u;
    if (!ok) break;
    tc_fence_after();
    {
      float x[32];
      tmem_ld32(tmem + lane_base + 32, x);  // lane t = (r, k1): X[k1 + 16 k2] re (k2 < 16), im
      const int kk = angle * a.nt_total + a.n0 + d;
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float c = x[16 * h + k2];  // raw: the 1/L^2 is applied when folding
          const int i = 2 * k2 + h;
          acc1[i] += c;
          acc2[i] = fmaf(c, c, acc2[i]);
          if (c > best[i]) {
            best[i] = c;
            barg[i] = kk;
          }
        }
    }
    tc_fence_before();
    __syncthreads();  // operand tiles and tensor memory are reused by the next template
    tc_fence_after();
  }
  if (!ok) {
    if (t == 0) {
      atomicOr(a.err, 1u);
      mbar_wait(&bars[2], mma_parity ^ 1u, 400000000LL);  // an MMA that may still be in flight
    }
  } else {
    const float inv = 1.0f / (float)(kL * kL);
    const size_t wbase = (size_t)win * kL * kL;
    const int oy = (y0 + r2 + kL / 2) & (kL - 1);
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = 2 * k2 + h;
        const int ox = (2 * (k1o + 16 * k2) + h + kL / 2) & (kL - 1);
        const size_t pix = wbase + (size_t)oy * kL + ox;
        atomicAdd(a.S1 + pix, (double)(acc1[i] * inv));
        atomicAdd(a.S2 + pix, (double)(acc2[i] * (inv * inv)));
        if (barg[i] >= 0)
          atomicMax(a.peak + pix, ((unsigned long long)float_key(best[i] * inv) << 32) |
                                      (unsigned)(0xFFFFFFFFu - (unsigned)barg[i]));
      }
  }
  // after a failed wait, let bulk copies still in flight land before the shared memory goes away
  if (!ok && t == 0)
    for (int k = dcur; k < issued; ++k) mbar_wait(&bars[k & 1], (k >> 1) & 1, 400000000LL);
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemColsB);
  }
}

// Builds the constant tables on the current device (idempotent; ordered before the first
// tensor-core pass by the stream).
void tc_tables(cudaStream_t s) {
  tc_tables_kernel<<<1, 256, 0, s>>>();
  GISSPA_LAUNCH_CHECK();
}

}  // namespace

void launch_b_tc(const CorrLaunch& cl, const CorrArgs& args, const float2* twL, const float2* twNZ, cudaStream_t s) {
  static PerDeviceOnce once;
  once([s] {
    GISSPA_CUDA(cudaFuncSetAttribute(pass_b_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemB));
    GISSPA_CUDA(cudaFuncSetAttribute(pass_b_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    tc_tables(s);
  });
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(kL / kRowsB, cl.E);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemB;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  GISSPA_CUDA(cudaLaunchKernelEx(&cfg, pass_b_tc_kernel, args, twL, twNZ));
  ++launch_counter();
}

void launch_a_tc(const CorrLaunch& cl, const float2* I, const void* T, float2* Q, const CorrArgs& args,
                 const float2* twL, cudaStream_t s) {
  static PerDeviceOnce once;
  once([s] {
    GISSPA_CUDA(cudaFuncSetAttribute(pass_a_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    GISSPA_CUDA(cudaFuncSetAttribute(pass_a_tc_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    tc_tables(s);
  });
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(kNZ / kSlotsPerCta, cl.E * cl.D);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  GISSPA_CUDA(cudaLaunchKernelEx(&cfg, pass_a_tc_kernel, I, static_cast<const __half2*>(T), Q, args.b0, args.n0, cl.D,
                                 twL, cl.chained ? 1 : 0, args.err));
  ++launch_counter();
}

}  // namespace gisspa
