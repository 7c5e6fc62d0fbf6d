// search.cu — per-micrograph orchestration of the search (SearchNorm::work,
// norm.cu:620-660; SearchNoNorm::work, nonorm.cu:559-589) on one stream.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <iterator>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "corr_generic.cuh"
#include "correlate.cuh"
#include "prep.cuh"
#include "project.cuh"
#include "search.cuh"

namespace gisspa {

std::vector<int> window_offsets(int len, int l, int ov) {
  std::vector<int> off{0};
  int o = 0;
  while (o + l < len) {
    o += l - ov;
    if (o + l >= len) o = len - l;
    off.push_back(o);
  }
  return off;
}

int window_count_nonorm(int len, int l, int ov) {
  int o = 0, n = 1;
  while (o + l < len) {
    o += l - ov;
    if (o + l >= len) o = len - l;
    ++n;
  }
  return n;
}

std::vector<float> angle_list(float step) {
  std::vector<float> a;
  for (float e = 0.0f; e < 360.0f; e += step) a.push_back(e);
  return a;
}

int validate_config(const gisspa_config& c, std::string& err) {
  const int l = c.window_size;
  if (l <= 0 || l % 16) {
    err = "window_size " + std::to_string(l) + " must be a positive multiple of 16";
    return GISSPA_ERR_SHAPE;
  }
  if (l < 32 || l > 2048) {
    err = "window_size " + std::to_string(l) + " outside [32, 2048]";
    return GISSPA_ERR_UNSUPPORTED;
  }
  if (c.overlap < 0 || c.overlap >= l) {
    err = "overlap must lie in [0, window_size)";
    return GISSPA_ERR_SHAPE;
  }
  if (!(c.phistep > 0) || c.phistep > 360) {
    err = "phistep must lie in (0, 360]";
    return GISSPA_ERR_ARG;
  }
  if (!(c.angpix > 0) || !(c.energy > 0) || !(c.highres > 0) || c.kk < 0 || c.diameter < 0) {
    err = "angpix, energy, Highres must be positive and kk, diameter non-negative";
    return GISSPA_ERR_ARG;
  }
  if (c.spectrum_precision < 0 || c.spectrum_precision > 2) {
    err = "unknown spectrum_precision";
    return GISSPA_ERR_ARG;
  }
  if (c.pick_mode != GISSPA_PICK_CHUNK && c.pick_mode != GISSPA_PICK_TOPK) {
    err = "unknown pick_mode";
    return GISSPA_ERR_ARG;
  }
  if (c.pick_mode == GISSPA_PICK_TOPK && (c.topk <= 0 || c.exclusion_radius < 0)) {
    err = "topk must be positive and exclusion_radius non-negative";
    return GISSPA_ERR_ARG;
  }
  if (c.norm_type == 0 && c.tile_size <= 0) {
    err = "tile_size must be positive";
    return GISSPA_ERR_ARG;
  }
  if (c.template_batch < 0 || c.window_batch < 0) {
    err = "template_batch and window_batch must be >= 0";
    return GISSPA_ERR_ARG;
  }
  if (c.pass_b_shape >= 0 && !correlate_fast(l)) {
    err = "pass_b_shape applies to window sizes with hand-tuned kernels (256, 512, 1024)";
    return GISSPA_ERR_ARG;
  }
  if (c.pass_b_shape < -1 || c.pass_b_shape >= correlate_variants(l)) {
    err = "pass_b_shape must be -1 or one of the " + std::to_string(correlate_variants(l)) +
          " shapes compiled for window_size " + std::to_string(l);
    return GISSPA_ERR_ARG;
  }
  if (c.pass_a_shape < -1 || c.pass_a_shape >= (correlate_fast(l) ? pass_a_variants(l) : 1)) {
    err = "pass_a_shape must be -1 or one of the shapes compiled for window_size " + std::to_string(l);
    return GISSPA_ERR_ARG;
  }
  if (c.pass_b_shape >= 0) {
    const int sweep1 = c.pick_mode == GISSPA_PICK_TOPK ? EPI_TOPK : c.prune_sweep2 ? EPI_SUMMAX : EPI_SUM;
    const int epis[3] = {c.norm_type == 0 ? EPI_NONORM : sweep1,
                         c.norm_type == 0 ? EPI_NONORM : EPI_CHUNK, EPI_MAP};
    for (int k = 0; k < (c.norm_type != 0 && c.pick_mode == GISSPA_PICK_CHUNK ? 2 : 1); ++k)
      if (!correlate_variant_ok(l, c.pass_b_shape, epis[k])) {
        err = "pass_b_shape " + std::to_string(c.pass_b_shape) + " has no epilogue for this search";
        return GISSPA_ERR_UNSUPPORTED;
      }
  }
  return GISSPA_OK;
}

int validate_image(const gisspa_config& c, int nx, int ny, std::string& err) {
  if (nx <= 0 || ny <= 0 || nx > 65536 || ny > 65536) {
    err = "image size " + std::to_string(nx) + "x" + std::to_string(ny) + " out of range";
    return GISSPA_ERR_SHAPE;
  }
  if (c.norm_type == 0 && (nx < c.tile_size || ny < c.tile_size)) {
    // TileImages copies tile_size rows of tile_size floats (tileimages.cpp:61-65)
    err = "norm_type=0 needs an image of at least tile_size x tile_size";
    return GISSPA_ERR_SHAPE;
  }
  if (std::max(nx, ny) / 2 > (1 << 15)) {
    err = "image too large for the radial shell tables";
    return GISSPA_ERR_SHAPE;
  }
  return GISSPA_OK;
}

namespace {

template <typename T>
T* buf(DevBuf& b, size_t count) {
  return static_cast<T*>(b.ensure(sizeof(T) * std::max<size_t>(count, 1)));
}

size_t spec_bytes(int spec) { return spec == GISSPA_SPEC_FP32 ? sizeof(float2) : sizeof(__half2); }

__global__ void musig_kernel(const double* __restrict__ S1, const double* __restrict__ S2, long long n, double N,
                             float2* __restrict__ ms) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // set_CCG_mean (kernels.cu:697-706) in FP64; update_CCG uses z = 0 when sigma <= 0 (kernels.cu:720)
  const double mu = S1[i] / N;
  const double sd = sqrt(S2[i] / N - mu * mu);
  ms[i] = make_float2((float)mu, sd > 0 ? (float)(1.0 / sd) : 0.f);
}

// Peak keys of the sharded search: the per-pixel key of the top-K sweep XOR 2^63, read as int64
// (a signed max then orders them as the unsigned max does; 0 = none becomes INT64_MIN).
__global__ void peak_flip_kernel(const unsigned long long* __restrict__ in, long long n,
                                 unsigned long long* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = in[i] ^ 0x8000000000000000ull;
}

// Rows that sweep 2 must transform.  Every pair's z at a pixel is at most the z of the pixel's
// best correlation over all pairs (fl((c - mu) s) does not decrease with c for s >= 0), so a row
// whose pixels all have a best z below the threshold holds no chunk pick for any template or
// angle: the chunk maximum that reaches the threshold lies on a pixel whose best z does.  The
// margin covers the rounding difference between this z (from the normalised best correlation)
// and pass B's (from the raw transform, possibly of another column-transform shape).  One warp
// per row; alive[w][y] by row y of Q (output row (y + l/2) mod l), alive_win[w] set when any row
// of window w is alive, *count += rows.  creq[w] (a float key, min-reduced) is the smallest
// correlation that reaches the threshold less the margin at any live pixel of the window: a
// pair whose maximum over the window stays below it holds no pick either.
constexpr float kAliveMargin = 1e-3f;
__global__ void row_alive_kernel(const unsigned long long* __restrict__ peak, const float2* __restrict__ ms, int l,
                                 long long rows, float thresh, unsigned char* __restrict__ alive,
                                 unsigned char* __restrict__ alive_win, unsigned* __restrict__ count,
                                 unsigned* __restrict__ creq) {
  const long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;  // whole warps
  const long long w = row / l;
  const int y = (int)(row % l), oy = (y + l / 2) % l;
  const size_t base = ((size_t)w * l + oy) * l;
  bool hit = false;
  unsigned req = 0xFFFFFFFFu;  // float_key of +inf and above: no bar yet
  const double t = (double)thresh - (double)kAliveMargin;
  for (int x = lane; x < l; x += 32) {
    const unsigned long long pk = peak[base + x];
    if (!pk) continue;
    const float2 m = ms[base + x];
    const float z = (key_float((uint32_t)(pk >> 32)) - m.x) * m.y;
    if (z >= thresh - kAliveMargin) {
      hit = true;
      // c reaches z = t where c = mu + t / (1 / sigma), rounded down; with 1 / sigma = 0 every c
      // gives z = 0, which reaches t here
      const float c = m.y > 0.f ? __double2float_rd((double)m.x + t / (double)m.y) : -INFINITY;
      req = min(req, float_key(c));
    }
  }
  hit = __any_sync(0xffffffffu, hit);
  req = __reduce_min_sync(0xffffffffu, req);
  if (lane == 0) {
    alive[row] = hit ? 1 : 0;
    if (hit) {
      alive_win[w] = 1;
      atomicAdd(count, 1u);
      atomicMin(creq + w, req);
    }
  }
}

// Pairs that sweep 2 must transform: those whose maximum correlation over the window (recorded
// by sweep 1) reaches the window's bar; alive by pair_index, *count += pairs.
__global__ void pair_alive_kernel(const unsigned* __restrict__ pair_max, const unsigned* __restrict__ creq,
                                  int n_windows, int n_angles, long long n, unsigned char* __restrict__ alive,
                                  unsigned* __restrict__ count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned pm = pair_max[i];
  const bool live = pm != 0 && pm >= creq[(i / n_angles) % n_windows];
  alive[i] = live ? 1 : 0;
  const unsigned b = __ballot_sync(__activemask(), live);
  if (b && (threadIdx.x & 31) == __ffs(b) - 1) atomicAdd(count, (unsigned)__popc(b));
}

// Top-K: image map of the max z over windows covering each pixel (ties: lowest window).
__global__ void zmap_kernel(const unsigned long long* __restrict__ peak, const float2* __restrict__ ms, int l,
                            const int* __restrict__ offx, const int* __restrict__ offy, int bx, int nx, int ny,
                            unsigned long long* __restrict__ zkey) {
  const int b = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= l * l) return;
  const size_t i = (size_t)b * l * l + k;
  const unsigned long long pk = peak[i];
  if (!pk) return;
  const float2 m = ms[i];
  const float z = (key_float((uint32_t)(pk >> 32)) - m.x) * m.y;
  const int cx = offx[b % bx] + k % l, cy = offy[b / bx] + k / l;
  if (cx >= nx || cy >= ny) return;
  const unsigned long long key = ((unsigned long long)float_key(z) << 32) | (unsigned)(0xFFFFFFFFu - (unsigned)b);
  atomicMax(zkey + (size_t)cy * nx + cx, key);
}

struct ZCand {
  float z;
  int q, win, arg;
};

// First node of a captured angle: the angle at the cursor becomes current, the cursor advances.
__global__ void angle_select_kernel(const AngleState* __restrict__ table, int* __restrict__ cursor,
                                    AngleState* __restrict__ cur) {
  *cur = table[*cursor];
  *cursor += 1;
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

// Copies of whole per-template blocks (n4 16-byte words each) by a list of template indices:
// dst[i] = src[list[i]] (gather) or dst[list[i]] = src[i] (scatter).
template <bool GATHER>
__global__ void template_copy_kernel(const uint4* __restrict__ src, const int* __restrict__ list, long long n4,
                                     uint4* __restrict__ dst) {
  const int i = blockIdx.y;
  const long long from = GATHER ? list[i] : i, to = GATHER ? i : list[i];
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n4; k += (long long)gridDim.x * blockDim.x)
    dst[to * n4 + k] = src[from * n4 + k];
}

// A bounded wait on an mbarrier phase that never completes (its single expected arrival is
// never made, and no asynchronous copy targets it): the wait gives up after max_cycles and the
// CTA raises the error flag, exactly as pass B does when its bulk copies do not land.
__global__ void wait_probe_kernel(unsigned* err, long long max_cycles) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0, max_cycles);
  if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicOr(err, 1u);
}

__global__ void zcompact_kernel(const unsigned long long* __restrict__ zkey, int nx, int ny, float thresh, float dmin,
                                const unsigned long long* __restrict__ peak, int l, const int* __restrict__ offx,
                                const int* __restrict__ offy, int bx, ZCand* __restrict__ out,
                                unsigned* __restrict__ count, unsigned cap) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nx * ny) return;
  const unsigned long long k = zkey[q];
  if (!k) return;
  const float z = key_float((uint32_t)(k >> 32));
  const int x = (int)(q % nx), y = (int)(q / nx);
  if (!(z >= thresh) || x < dmin || x >= nx - dmin || y < dmin || y >= ny - dmin) return;
  const int b = (int)(0xFFFFFFFFu - (unsigned)(k & 0xFFFFFFFFu));
  const int px = x - offx[b % bx], py = y - offy[b / bx];
  const unsigned s = atomicAdd(count, 1u);
  const unsigned long long pk = peak[(size_t)b * l * l + (size_t)py * l + px];
  if (s < cap) out[s] = ZCand{z, (int)q, b, (int)(0xFFFFFFFFu - (uint32_t)(pk & 0xFFFFFFFFu))};
}

struct Ctx {
  gisspa_handle* h;
  cudaStream_t s;
  int l;
  long long L2;
  DevParams p;
};

// ---- template preparation (PreprocessTemplate norm.cu:194-354 / nonorm.cu:178-344)
void prepare_templates(Ctx& c) {
  gisspa_handle* h = c.h;
  const int l = c.l, nt = h->nt;
  const bool nonorm = h->cfg.norm_type == 0;
  float2* tb = buf<float2>(h->tb, (size_t)nt * c.L2);
  float2* tmp = buf<float2>(h->tb_tmp, (size_t)nt * c.L2);
  tmpl_pad(h->d_stack.as<float>(), nt, h->tw, h->th, l, tb, c.s);
  tmpl_edge_normalise(tb, nt, l, nullptr, c.s);
  h->fft.fft2(tb, tmp, nt, l, l, -1, 1.0f / (float)c.L2, c.s);
  const int nb = l / 2;
  double* ra = buf<double>(h->ra, (size_t)nt * nb);
  unsigned* rb = buf<unsigned>(h->rb, nb);
  radial_power(tb, nt, l, l, ra, rb, nb, c.s);
  tmpl_whiten(tb, nt, l, ra, rb, nb, c.s);
  if (nonorm) {  // nonorm.cu:291-299: IFFT, real-space mask, FFT / l^2
    h->fft.fft2(tb, tmp, nt, l, l, +1, 1.f, c.s);
    mask_real(tb, nt, l, h->cfg.diameter, h->cfg.edge_half_width, c.s);
    h->fft.fft2(tb, tmp, nt, l, l, -1, 1.0f / (float)c.L2, c.s);
  }
  if (h->keep_whitened && !nonorm)  // the adjoint differentiates the weighting applied next
    GISSPA_CUDA(cudaMemcpyAsync(buf<float2>(h->tw_spec, (size_t)nt * c.L2), tb, sizeof(float2) * nt * c.L2,
                                cudaMemcpyDeviceToDevice, c.s));
  float* table = buf<float>(h->table, c.L2);
  tmpl_weight_table(table, l, c.p, c.s);
  apply_table(tb, nt, l, table, c.s);
  rms_normalise(tb, nt, l, buf<double>(h->tmpl_m, nt), c.s);
  if (!nonorm) {
    h->fft.fft2(tb, tmp, nt, l, l, +1, 1.f, c.s);  // norm.cu:350-351, unnormalised
    real_part(tb, buf<float>(h->prep_real, (size_t)nt * c.L2), (long long)nt * c.L2, 1.f, c.s);
  } else {
    h->fft.transpose(tb, tmp, nt, l, l, c.s, l / 2 + 1);
    void* ts = h->tspec.ensure(spec_bytes(h->cfg.spectrum_precision) * (size_t)nt * (l / 2 + 1) * l);
    finalize_spectra(tmp, nt, l, nullptr, h->cfg.spectrum_precision, ts, 1.0, c.s);
  }
}

// ---- micrograph preparation (LoadImage norm.cu:156-181 + PreprocessImage norm.cu:356-402)
void preprocess_full(Ctx& c, float2* G, int nx, int ny, bool zero_dc) {
  gisspa_handle* h = c.h;
  const long long N = (long long)nx * ny;
  float2* tmp = buf<float2>(h->img_tmp, N);
  h->fft.fft2(G, tmp, 1, ny, nx, -1, (float)(1.0 / (double)N), c.s);
  phase_flip(G, nx, ny, c.p, c.s);
  const int nb = std::max(nx, ny) / 2;
  double* ra = buf<double>(h->ra, std::max<size_t>((size_t)h->nt * (c.l / 2), nb));
  unsigned* rb = buf<unsigned>(h->rb, std::max(nb, c.l / 2));
  radial_power(G, 1, nx, ny, ra, rb, nb, c.s);
  image_filter(G, nx, ny, c.p, ra, rb, nb, zero_dc, c.s);
  h->fft.fft2(G, tmp, 1, ny, nx, +1, 1.f, c.s);
}

// SplitImage (norm.cu:404-477): windows -> FFT / l^2 -> radial RMS -> kx-major half spectra.
void window_spectra(Ctx& c, const float* img, int nx, int ny, const std::vector<int>& ox, const std::vector<int>& oy) {
  gisspa_handle* h = c.h;
  const int l = c.l, bx = (int)ox.size(), W = bx * (int)oy.size();
  int* dox = buf<int>(h->offx, ox.size());
  int* doy = buf<int>(h->offy, oy.size());
  GISSPA_CUDA(cudaMemcpyAsync(dox, ox.data(), sizeof(int) * ox.size(), cudaMemcpyHostToDevice, c.s));
  GISSPA_CUDA(cudaMemcpyAsync(doy, oy.data(), sizeof(int) * oy.size(), cudaMemcpyHostToDevice, c.s));
  float2* w = buf<float2>(h->win_c, (size_t)W * c.L2);
  float2* tmp = buf<float2>(h->win_tmp, (size_t)W * c.L2);
  gather_windows(img, nx, ny, dox, doy, bx, W, l, w, c.s);
  h->fft.fft2(w, tmp, W, l, l, -1, 1.0f / (float)c.L2, c.s);
  rms_normalise(w, W, l, buf<double>(h->win_m, W), c.s);
  h->fft.transpose(w, buf<float2>(h->ispec, (size_t)W * (l / 2 + 1) * l), W, l, l, c.s, l / 2 + 1);
}

// RotateTemplate (norm.cu:479-521): rotate, mask, (x - mean)/sqrt(var), FFT / l^2.
// st (optional): take the angle from device memory (graph replays); theta is then unused.
// Rotation by theta, forward transform and scaling of n prepared templates (src) into spectra
// (dst, in the storage type of the search's precision).
void spectra_of(Ctx& c, float theta, const float* src, int n, void* dst, const AngleState* st) {
  gisspa_handle* h = c.h;
  const int l = c.l, nt = h->nt, hs = l / 2 + 1;
  const double rad = (double)theta * kRefPi / 180.0;
  float2* rot = buf<float2>(h->rot, (size_t)nt * c.L2);
  float2* rtmp = buf<float2>(h->rot_tmp, (size_t)nt * hs * l);
  double* sums = buf<double>(h->rsums, 2 * (size_t)nt);
  rotate_batch(src, n, l, (float)std::cos(rad), (float)std::sin(rad), true, h->cfg.diameter, h->cfg.edge_half_width,
               rot, sums, c.s, st);
  h->fft.rows(rot, (long long)n * l, l, -1, 1.f, c.s);
  h->fft.transpose(rot, rtmp, n, l, l, c.s, hs);
  h->fft.rows(rtmp, (long long)n * hs, l, -1, 1.f, c.s);
  finalize_spectra(rtmp, n, l, sums, h->cfg.spectrum_precision, dst, 1.0 / (double)c.L2, c.s);
}

void template_spectra_at(Ctx& c, float theta, const AngleState* st = nullptr) {
  gisspa_handle* h = c.h;
  const int l = c.l, nt = h->nt, hs = l / 2 + 1;
  void* ts = h->tspec.ensure(spec_bytes(h->cfg.spectrum_precision) * (size_t)nt * hs * l);
  spectra_of(c, theta, h->prep_real.as<float>(), nt, ts, st);
}

// The spectra of the listed templates only, in their places among the template spectra (the
// others keep what an earlier angle left there: the pruned second sweep reads none of them).
// Each template's transform is independent of the others': the same values as for all.
void template_spectra_listed(Ctx& c, float theta, const std::vector<int>& list) {
  gisspa_handle* h = c.h;
  const int l = c.l, nt = h->nt, hs = l / 2 + 1, n = (int)list.size();
  if (2 * n > nt) {  // most templates: transforming all of them costs less than the copies
    template_spectra_at(c, theta);
    return;
  }
  const size_t tb = spec_bytes(h->cfg.spectrum_precision) * (size_t)hs * l;
  float* sub = buf<float>(h->prep_sub, (size_t)nt * c.L2 / 2);  // sized for half of them: allocated once
  char* ts_sub = static_cast<char*>(h->tspec_sub.ensure(tb * (nt / 2)));
  char* ts = static_cast<char*>(h->tspec.ensure(tb * nt));
  int* dlist = buf<int>(h->list_dev, (size_t)nt);
  GISSPA_CUDA(cudaMemcpyAsync(dlist, list.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c.s));
  static_assert(sizeof(float) * 4 == sizeof(uint4), "16-byte words");
  const long long w_in = (long long)c.L2 / 4, w_out = (long long)(tb / sizeof(uint4));
  template_copy_kernel<true><<<dim3(64, n), 256, 0, c.s>>>(reinterpret_cast<const uint4*>(h->prep_real.as<float>()),
                                                          dlist, w_in, reinterpret_cast<uint4*>(sub));
  GISSPA_LAUNCH_CHECK();
  spectra_of(c, theta, sub, n, ts_sub, nullptr);
  template_copy_kernel<false><<<dim3(64, n), 256, 0, c.s>>>(reinterpret_cast<const uint4*>(ts_sub), dlist, w_out,
                                                           reinterpret_cast<uint4*>(ts));
  GISSPA_LAUNCH_CHECK();
}

void choose_batches(const gisspa_config& cfg, int l, int W, int nt, int& D, int& E) {
  const long long per_pair = (long long)(l / 2) * l * (long long)sizeof(float2);
  const long long budget = 64LL << 20;
  // window sizes without hand-tuned kernels: 16 windows per launch give the generic row kernel
  // twice the CTAs of 8 (4096^2 at L = 320: 20.0 against 21.7 s per micrograph)
  E = cfg.window_batch > 0 ? cfg.window_batch : (!correlate_fast(l) ? 16 : (l >= 1024 ? 4 : 8));
  E = std::max(1, std::min(E, W));
  D = cfg.template_batch > 0 ? cfg.template_batch : (int)std::max(1LL, budget / per_pair / E);
  D = std::max(1, std::min(D, nt));
}

// The pair engine's launch sequence over `batches` (first window, first template, windows,
// templates): launch j runs pass A of batch j and pass B of batch j - 1, the batches' Q
// alternating between the two halves of the Q buffer.  Returns the number of launches.
struct Batch {
  int b0, n0, e, d;
};
int engine_sequence(Ctx& c, int epi, const float2* I, const void* T, const std::vector<Batch>& batches, int D, int E,
                    CorrArgs args) {
  gisspa_handle* h = c.h;
  const int l = c.l, nb = (int)batches.size();
  const size_t pairs_max = (size_t)D * E;
  float2* Q = buf<float2>(h->Q, 2 * pairs_max * (l / 2) * l);
  const size_t stride = engine_counter_ints();
  int* ctr = buf<int>(h->engine_ctr, (size_t)(nb + 1) * stride);
  GISSPA_CUDA(cudaMemsetAsync(ctr, 0, (size_t)(nb + 1) * stride * sizeof(int), c.s));
  const float2* twL = h->fft.twiddles(l);
  const float2* twNZ = h->fft.twiddles(l / 2);
  args.err = h->dev_err.as<unsigned>();
  for (int j = 0; j <= nb; ++j) {
    EngineBatch A{}, B{};
    if (j < nb) {
      const Batch& b = batches[j];
      A = EngineBatch{1, b.b0, b.n0, b.d, b.e, Q + (size_t)(j & 1) * pairs_max * (l / 2) * l};
    }
    if (j > 0) {
      const Batch& b = batches[j - 1];
      B = EngineBatch{1, b.b0, b.n0, b.d, b.e, Q + (size_t)((j - 1) & 1) * pairs_max * (l / 2) * l};
    }
    engine_launch(h->cfg.spectrum_precision, epi, I, T, A, B, args, ctr + (size_t)j * stride, j > 0, twL, twNZ, c.s);
  }
  return nb + 1;
}

// Whether a search runs the pair engine when its shape is chosen (the tensor-core passes are
// per-pass kernels).
bool engine_ok(const gisspa_config& cfg, int l, int epi) {
  return engine_supported(l, epi) && !(cfg.tensor_cores && cfg.spectrum_precision == GISSPA_SPEC_FP16);
}

constexpr bool kTuneEngine = false;

// Autotuner: times every candidate launch shape (pass B variant, template batch D, window
// batch E) on the sweep's own spectra, with the epilogue's outputs redirected to scratch,
// and keeps the fastest per (window size, epilogue, precision).
TuneChoice autotune(Ctx& c, int epi, const float2* I, int W, const void* T, int nt, CorrArgs args) {
  gisspa_handle* h = c.h;
  const int l = c.l;
  struct Cand { int D, E; };
  // (D, E): pass A runs L/2/NC x E CTAs, pass B L/RB x E; Q holds D x E pairs
  static const Cand c512[] = {{8, 8}, {12, 8}, {6, 12}, {8, 12}, {4, 16}, {6, 16}, {16, 6}, {24, 4}};
  static const Cand c1024[] = {{6, 4}, {4, 6}, {3, 8}, {2, 12}, {4, 8}, {8, 3}, {2, 16}};
  static const Cand c256[] = {{16, 8}, {32, 8}, {8, 16}, {16, 16}, {64, 4}};
  static const Cand c320[] = {{12, 8}, {16, 8}, {8, 16}, {24, 8}, {16, 16}, {32, 4}};
  const Cand* cb = l == 512 ? c512 : l == 1024 ? c1024 : l == 320 ? c320 : c256;
  const size_t nc = l == 512    ? std::size(c512)
                    : l == 1024 ? std::size(c1024)
                    : l == 320  ? std::size(c320)
                                : std::size(c256);
  std::vector<Cand> cands(cb, cb + nc);
  if (epi == EPI_CHUNK && args.skip.pairs) {
    // a pruned second sweep transforms a few pairs per angle and is launched from the host: its
    // launches are mostly CTAs that leave at once, and the fewer the better, so one batch shape,
    // the largest within 4 GiB of Q (only the row-transform shape is tuned)
    const long long per_pair = (long long)(l / 2) * l * (long long)sizeof(float2);
    const long long cap = std::max(1LL, (4LL << 30) / per_pair);  // pairs in 4 GiB: 16384 .. 1024
    const int dd = std::min(nt, kMaxListedTemplates);
    const int ee = (int)std::max(1LL, std::min<long long>(W, cap / dd));
    cands.assign(1, Cand{dd, ee});
  }
  int maxE = 1, maxDE = 1;
  for (auto& cd : cands) {
    cd.D = std::max(1, std::min(cd.D, nt));
    cd.E = std::max(1, std::min(cd.E, W));
    maxE = std::max(maxE, cd.E);
    maxDE = std::max(maxDE, cd.D * cd.E);
  }
  // scratch outputs: S1, S2 (double), peak keys (u64) for maxE windows; nn arrays; counter
  const size_t px = (size_t)maxE * c.L2;
  const size_t nn = (size_t)maxE * nt;
  char* base = static_cast<char*>(h->tune_scratch.ensure(px * 24 + nn * 24 + 256));
  args.S1 = reinterpret_cast<double*>(base);
  args.S2 = args.S1 + px;
  args.peak = reinterpret_cast<unsigned long long*>(args.S2 + px);
  args.nn_key = args.peak + px;
  args.nn_sum = reinterpret_cast<double*>(args.nn_key + nn);
  args.cand_count = reinterpret_cast<unsigned*>(args.nn_sum + 2 * nn);
  args.cand_cap = 0;
  args.cand = nullptr;
  args.pair_max = nullptr;
  args.nt_total = nt;
  args.err = h->dev_err.as<unsigned>();
  // (twice the largest batch when the pair engine, which alternates two Q slots, is tuned)
  float2* Q = buf<float2>(h->Q, (kTuneEngine ? 2 : 1) * (size_t)maxDE * (l / 2) * l);
  args.Q = Q;
  const float2* twL = h->fft.twiddles(l);
  const float2* twNZ = h->fft.twiddles(l / 2);
  TuneChoice best;
  best.us_per_pair = 1e30;
  const size_t tbytes = spec_bytes(h->cfg.spectrum_precision) * (size_t)(l / 2 + 1) * l;  // one template
  for (int v = 0; v < correlate_variants(l); ++v)
    for (const auto& cd : cands) {
      if (v == engine_variant(l)) {
        // measured slower than the per-pass kernels on B200 (83.6 against 70.0 us per batch of
        // 96 pairs at window 512): selectable with pass_b_shape, not tuned
        if (!kTuneEngine || !engine_ok(h->cfg, l, epi)) continue;
        // the engine runs whole sequences: kReps batches (kReps + 1 launches) of the same pairs
        constexpr int kReps = 4;
        const std::vector<Batch> seq(kReps, Batch{0, 0, cd.E, cd.D});
        args.Q = nullptr;
        engine_sequence(c, epi, I, T, std::vector<Batch>(1, Batch{0, 0, cd.E, cd.D}), cd.D, cd.E, args);
        GISSPA_CUDA(cudaEventRecord(h->ev[5], c.s));
        engine_sequence(c, epi, I, T, seq, cd.D, cd.E, args);
        GISSPA_CUDA(cudaEventRecord(h->ev[6], c.s));
        GISSPA_CUDA(cudaEventSynchronize(h->ev[6]));
        float ms = 0;
        GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]));
        const double us = 1000.0 * ms / (kReps * cd.D * cd.E);
        if (us < best.us_per_pair) best = TuneChoice{v, cd.D, cd.E, us};
        continue;
      }
      if (!correlate_variant_ok(l, v, epi)) continue;
      // (a pruned second sweep's few live pairs do not need the column shape tuned)
      const int n_av = (epi == EPI_CHUNK && args.skip.pairs) ? 1 : pass_a_variants(l);
      for (int av = 0; av < n_av; ++av) {
        CorrLaunch cl{l, cd.E, cd.D, h->cfg.spectrum_precision, epi, v};
        cl.tc = h->cfg.tensor_cores != 0;
        cl.a_variant = av;
        args.D = cd.D;
        // each timed launch on other windows and templates than the one before (where the
        // search has them), so that its spectra come from HBM as in a sweep, not from L2: the
        // spectra pointers move, the outputs stay on the scratch state of windows 0 .. E - 1
        args.b0 = 0;
        args.n0 = 0;
        auto at = [&](int r) {
          const int b0 = W > cd.E ? (r * cd.E) % (W - cd.E + 1) : 0;
          const int n0 = nt > cd.D ? (r * cd.D) % (nt - cd.D + 1) : 0;
          cl.chained = r > 0;
          correlate_launch(cl, I + (size_t)b0 * (l / 2 + 1) * l,
                           static_cast<const char*>(T) + (size_t)n0 * tbytes, Q, args, twL, twNZ, c.s);
        };
        at(0);
        GISSPA_CUDA(cudaEventRecord(h->ev[5], c.s));
        constexpr int kReps = 6;
        for (int r = 1; r <= kReps; ++r) at(r);
        GISSPA_CUDA(cudaEventRecord(h->ev[6], c.s));
        GISSPA_CUDA(cudaEventSynchronize(h->ev[6]));
        float ms = 0;
        GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]));
        const double us = 1000.0 * ms / (kReps * cd.D * cd.E);
        if (us < best.us_per_pair) best = TuneChoice{v, cd.D, cd.E, us, av};
      }
    }
  return best;
}

// One correlation sweep at one angle over every (window, template) pair.
long long correlate_all(Ctx& c, int epi, const float2* I, int W, const void* T, int nt, CorrArgs args, int D, int E) {
  gisspa_handle* h = c.h;
  const int l = c.l;
  int variant = 0, a_variant = 0;
  const bool generic = !correlate_fast(l);  // no hand-tuned kernels for this window size
  if (!generic && h->cfg.template_batch > 0 && h->cfg.window_batch > 0 && h->cfg.pass_b_shape >= 0) {
    if (!correlate_variant_ok(l, h->cfg.pass_b_shape, epi) ||
        (h->cfg.pass_b_shape == engine_variant(l) && !engine_ok(h->cfg, l, epi)))
      throw CudaError{cudaErrorInvalidValue, "pass_b_shape not compiled for this window size and epilogue"};
    variant = h->cfg.pass_b_shape;
  }
  if (!generic && h->cfg.template_batch > 0 && h->cfg.window_batch > 0 && h->cfg.pass_a_shape >= 0)
    a_variant = h->cfg.pass_a_shape;
  if (!generic && h->cfg.template_batch == 0 && h->cfg.window_batch == 0) {
    const long long key = (long long)l | ((long long)epi << 16) | ((long long)h->cfg.spectrum_precision << 24) |
                          ((long long)std::min(nt, 64) << 32) | ((long long)std::min(W, 64) << 40);
    auto it = h->tuned.find(key);
    if (it == h->tuned.end()) it = h->tuned.emplace(key, autotune(c, epi, I, W, T, nt, args)).first;
    D = it->second.D;
    E = it->second.E;
    variant = it->second.variant;
    a_variant = it->second.a_variant;
    h->st.pass_b_variant = variant;
    h->st.pass_a_variant = a_variant;
    h->st.tuned_us_per_pair = it->second.us_per_pair;
  }
  float2* Q = nullptr;
  const float2 *twL = nullptr, *twNZ = nullptr;
  float2 *gz = nullptr, *gx = nullptr;
  if (generic) {
    gz = buf<float2>(h->gen_z, generic_z_elems(l, D * E));
    const size_t xe = generic_x_elems(l, D * E, epi);
    gx = xe ? buf<float2>(h->gen_x, xe) : nullptr;
  } else {
    Q = buf<float2>(h->Q, (size_t)D * E * (l / 2) * l);
    twL = h->fft.twiddles(l);
    twNZ = h->fft.twiddles(l / 2);
  }
  args.err = h->dev_err.as<unsigned>();
  long long pairs = 0, launches = 0, dsum = 0;
  const int seq = (!h->capturing && h->n_seqs < gisspa_handle::kSeqs) ? h->n_seqs++ : -1;
  if (seq >= 0) GISSPA_CUDA(cudaEventRecord(h->qev[seq][0], c.s));
  const bool engine = !generic && variant == engine_variant(l);
  if (engine) {
    std::vector<Batch> batches;
    for (int n0 = 0; n0 < nt; n0 += D)
      for (int b0 = 0; b0 < W; b0 += E) {
        batches.push_back(Batch{b0, n0, std::min(E, W - b0), std::min(D, nt - n0)});
        pairs += (long long)batches.back().d * batches.back().e;
        dsum += batches.back().d;
      }
    engine_sequence(c, epi, I, T, batches, D, E, args);
    launches = (long long)batches.size();  // batches: the per-pass path's launch pairs
  }
  for (int n0 = 0; n0 < nt && !engine; n0 += D) {
    const int d = std::min(D, nt - n0);
    for (int b0 = 0; b0 < W; b0 += E) {
      const int e = std::min(E, W - b0);
      CorrLaunch cl{l, e, d, h->cfg.spectrum_precision, epi, variant};
      cl.tc = h->cfg.tensor_cores != 0;
      cl.a_variant = a_variant;
      cl.chained = pairs > 0;  // after this sequence's first pair of passes
      args.Q = Q;
      args.b0 = b0;
      args.n0 = n0;
      args.D = d;
      cudaEvent_t* ev = nullptr;
      if (h->cfg.cuda_graphs == 0 && (h->launch_index++ & 15) == 0 && h->n_samples < gisspa_handle::kSamples &&
          !h->capturing) {
        ev = h->sev[h->n_samples];
        h->sample_pairs[h->n_samples] = d * e;
        h->sample_d[h->n_samples] = d;
        ++h->n_samples;
      }
      if (generic)
        correlate_generic(cl, I, T, args, h->fft, gz, gx, c.s, ev);
      else
        correlate_launch(cl, I, T, Q, args, twL, twNZ, c.s, ev);
      pairs += (long long)d * e;
      dsum += d;
      ++launches;
    }
  }
  if (seq >= 0) {
    GISSPA_CUDA(cudaEventRecord(h->qev[seq][1], c.s));
    h->seq_launches[seq] = launches;
    h->seq_pairs[seq] = pairs;
    h->seq_d[seq] = dsum;
    h->seq_pruned[seq] = epi == EPI_CHUNK && args.skip.rows != nullptr;
  }
  return pairs;
}

// ---- norm_type = 1 (SearchNorm::work, norm.cu:620-660), in phases.

// Everything before the angle loop: LoadImage statistics, templates, micrograph, windows, the
// zeroed per-pixel state and the launch shape.
void norm_prepare(Ctx& c, const float* d_img, int nx, int ny, NormRun& r) {
  gisspa_handle* h = c.h;
  const gisspa_config& cfg = h->cfg;
  const int l = c.l, nt = h->nt;
  r = NormRun{};
  r.nx = nx;
  r.ny = ny;
  r.N = (long long)nx * ny;
  GISSPA_CUDA(cudaEventRecord(h->ev[0], c.s));
  // LoadImage statistics on the side stream (the serial FP32 form occupies one SM for
  // ~4 ns per pixel) while the templates are prepared on the main stream
  const bool prefetched = h->next_dev == d_img && h->next_nx == nx && h->next_ny == ny;
  h->next_dev = nullptr;
  if (prefetched) {
    // a batch started this micrograph's statistics during the previous one's sweeps
    h->stats.swap(h->stats_next);
    h->scratch.swap(h->scratch_next);
  } else {
    float* st0 = buf<float>(h->stats, 4);
    double* scr = buf<double>(h->scratch, 16);
    GISSPA_CUDA(cudaEventRecord(h->ev_in, c.s));
    GISSPA_CUDA(cudaStreamWaitEvent(h->side, h->ev_in, 0));
    image_stats(d_img, nx, ny, (cfg.quirks & GISSPA_QUIRK_OUTLIER_FP32_SERIAL) != 0, st0, scr, h->side);
    GISSPA_CUDA(cudaEventRecord(h->ev_stats, h->side));
  }
  float* stats = h->stats.as<float>();
  prepare_templates(c);
  GISSPA_CUDA(cudaStreamWaitEvent(c.s, prefetched ? h->ev_next : h->ev_stats, 0));
  // micrograph
  float2* G = buf<float2>(h->img_c, r.N);
  image_load(d_img, r.N, stats, true, cfg.invert != 0, G, c.s);
  preprocess_full(c, G, nx, ny, true);
  float* img = buf<float>(h->img_pre, r.N);
  real_part(G, img, r.N, 1.f, c.s);
  r.ox = window_offsets(nx, l, cfg.overlap);
  r.oy = window_offsets(ny, l, cfg.overlap);
  r.bx = (int)r.ox.size();
  r.W = r.bx * (int)r.oy.size();
  window_spectra(c, img, nx, ny, r.ox, r.oy);
  GISSPA_CUDA(cudaEventRecord(h->ev[1], c.s));
  h->last_nx = nx;
  h->last_ny = ny;
  h->last_W = r.W;
  h->last_bx = r.bx;
  h->last_offx = r.ox;
  h->last_offy = r.oy;

  r.angles = angle_list(cfg.phistep);
  h->last_angles = r.angles;
  const int n_euler =
      (cfg.quirks & GISSPA_QUIRK_NEULER_TRUNC) ? (int)(360.0f / cfg.phistep) : (int)r.angles.size();
  const int batch = (cfg.quirks & GISSPA_QUIRK_COUNT_PADDED_TEMPLATES) ? std::max(nt, r.W) : nt;
  r.Ntot = (double)batch * n_euler;
  r.topk = cfg.pick_mode == GISSPA_PICK_TOPK;
  r.npix = (size_t)r.W * c.L2;
  double* S1 = buf<double>(h->S1, r.npix);
  double* S2 = buf<double>(h->S2, r.npix);
  GISSPA_CUDA(cudaMemsetAsync(S1, 0, sizeof(double) * r.npix, c.s));
  GISSPA_CUDA(cudaMemsetAsync(S2, 0, sizeof(double) * r.npix, c.s));
  CorrArgs& args = r.args;
  args.S1 = S1;
  args.S2 = S2;
  args.nt_real = nt;
  args.nt_total = nt;
  args.offx = h->offx.as<int>();
  args.offy = h->offy.as<int>();
  args.bx = r.bx;
  args.nx = nx;
  args.ny = ny;
  args.dmin = cfg.diameter;
  args.thresh = cfg.threshold;
  if (r.topk) {
    args.peak = buf<unsigned long long>(h->peak, r.npix);
    GISSPA_CUDA(cudaMemsetAsync(args.peak, 0, sizeof(unsigned long long) * r.npix, c.s));
  }
  choose_batches(cfg, l, r.W, nt, r.D, r.E);
  r.phase = 1;
}

template <typename T>
void key_put(std::vector<unsigned char>& k, const T& v) {
  const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), p, p + sizeof(T));
}

// Everything one captured angle depends on besides the angle: shapes, buffer addresses, and the
// epilogue's arguments (device contents such as window offsets are read at replay time).
std::vector<unsigned char> angle_graph_key(Ctx& c, const NormRun& r, int epi) {
  gisspa_handle* h = c.h;
  const CorrArgs& a = r.args;
  std::vector<unsigned char> k;
  for (int v : {epi, c.l, r.W, h->nt, r.D, r.E, h->cfg.spectrum_precision, a.nt_real, a.nt_total, a.bx, a.nx, a.ny})
    key_put(k, v);
  for (float v : {a.thresh, a.dmin, h->cfg.diameter, h->cfg.edge_half_width}) key_put(k, v);
  key_put(k, a.cand_cap);
  for (const void* p : {(const void*)h->prep_real.as<void>(), (const void*)h->rot.as<void>(),
                        (const void*)h->rot_tmp.as<void>(), (const void*)h->rsums.as<void>(),
                        (const void*)h->tspec.as<void>(), (const void*)h->ispec.as<void>(),
                        (const void*)h->Q.as<void>(), (const void*)h->gen_z.as<void>(),
                        (const void*)h->gen_x.as<void>(), (const void*)a.S1, (const void*)a.S2, (const void*)a.peak,
                        (const void*)a.musig, (const void*)a.skip.rows, (const void*)a.skip.windows,
                        (const void*)a.skip.pairs, (const void*)a.pair_max,
                        (const void*)a.offx, (const void*)a.offy,
                        (const void*)a.cand, (const void*)a.cand_count, (const void*)h->dev_err.as<void>(),
                        (const void*)h->angle_table.as<void>(), (const void*)h->angle_cursor.as<void>(),
                        (const void*)h->angle_cur.as<void>()})
    key_put(k, p);
  return k;
}

// The captured graph of one angle of this sweep (captured on first use, and again whenever its
// key changes or any device buffer has been reallocated since).
AngleGraph& angle_graph(Ctx& c, NormRun& r, int epi) {
  gisspa_handle* h = c.h;
  std::vector<unsigned char> key = angle_graph_key(c, r, epi);
  const unsigned long long gen = alloc_generation().load();
  for (auto it = h->graphs.begin(); it != h->graphs.end();) {
    if (it->generation != gen) {  // stale addresses: never replay again
      cudaGraphExecDestroy(it->exec);
      it = h->graphs.erase(it);
    } else if (it->key == key) {
      return *it;
    } else {
      ++it;
    }
  }
  if (h->graphs.size() >= 8) {
    cudaGraphExecDestroy(h->graphs.front().exec);
    h->graphs.erase(h->graphs.begin());
  }
  AngleState* cur = h->angle_cur.as<AngleState>();
  r.args.angle_state = cur;
  const long long l0 = launch_counter();
  cudaGraph_t graph = nullptr;
  long long pairs = 0;
  h->capturing = true;
  GISSPA_CUDA(cudaStreamBeginCapture(c.s, cudaStreamCaptureModeThreadLocal));
  try {
    angle_select_kernel<<<1, 1, 0, c.s>>>(h->angle_table.as<AngleState>(), h->angle_cursor.as<int>(), cur);
    GISSPA_LAUNCH_CHECK();
    template_spectra_at(c, 0.f, cur);
    pairs = correlate_all(c, epi, h->ispec.as<float2>(), r.W, h->tspec.as<void>(), h->nt, r.args, r.D, r.E);
  } catch (...) {
    h->capturing = false;
    r.args.angle_state = nullptr;
    cudaStreamEndCapture(c.s, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  h->capturing = false;
  r.args.angle_state = nullptr;
  GISSPA_CUDA(cudaStreamEndCapture(c.s, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  GISSPA_CUDA(e);
  AngleGraph g;
  g.key = std::move(key);
  g.generation = gen;
  g.exec = exec;
  g.launches = launch_counter() - l0;
  g.pairs = pairs;
  launch_counter() = l0;  // the captured kernels run, and are counted, at each replay
  h->graphs.push_back(std::move(g));
  return h->graphs.back();
}

// Angles [a0, a1) of one sweep.  With cuda_graphs, the first angle runs from the host (it
// allocates, autotunes and samples the pass timings) and the rest replay one captured graph.
void run_angles(Ctx& c, NormRun& r, int epi, int a0, int a1) {
  gisspa_handle* h = c.h;
  const bool graphs = h->cfg.cuda_graphs != 0 && a1 - a0 >= 3;
  for (int a = a0; a < (graphs ? a0 + 1 : a1); ++a) {
    template_spectra_at(c, r.angles[a]);
    r.args.angle = a;
    r.args.angle_state = nullptr;
    r.pairs += correlate_all(c, epi, h->ispec.as<float2>(), r.W, h->tspec.as<void>(), h->nt, r.args, r.D, r.E);
  }
  if (!graphs) return;
  AngleState* table = buf<AngleState>(h->angle_table, r.angles.size());
  int* cursor = buf<int>(h->angle_cursor, 1);
  buf<AngleState>(h->angle_cur, 1);
  if (!r.angle_table_ready) {
    std::vector<AngleState>& t = r.angle_table;
    t.resize(r.angles.size());
    for (size_t a = 0; a < t.size(); ++a) {
      const double rad = (double)r.angles[a] * kRefPi / 180.0;  // as template_spectra_at
      t[a] = AngleState{(int)a, (float)std::cos(rad), (float)std::sin(rad), 0};
    }
    GISSPA_CUDA(cudaMemcpyAsync(table, t.data(), sizeof(AngleState) * t.size(), cudaMemcpyHostToDevice, c.s));
    r.angle_table_ready = true;
  }
  set_int_kernel<<<1, 1, 0, c.s>>>(cursor, a0 + 1);
  GISSPA_LAUNCH_CHECK();
  AngleGraph& g = angle_graph(c, r, epi);
  for (int a = a0 + 1; a < a1; ++a) GISSPA_CUDA(cudaGraphLaunch(g.exec, c.s));
  launch_counter() += g.launches * (a1 - a0 - 1);
  r.pairs += g.pairs * (a1 - a0 - 1);
  h->st.graph_replays += a1 - a0 - 1;
}

// Sweep 1 (ComputeCCGSum norm.cu:523-544) or the single top-K sweep over angles [a0, a1).
void norm_sweep1(Ctx& c, NormRun& r, int a0, int a1) {
  // with pruning the sums come with each pixel's best correlation (the same sums, added in the
  // same order)
  run_angles(c, r, r.topk ? EPI_TOPK : r.prune ? EPI_SUMMAX : EPI_SUM, a0, a1);
  r.phase = 2;
}

// set_CCG_mean (kernels.cu:697-706): mu and 1/sigma per window pixel from the complete sums.
void norm_stats(Ctx& c, NormRun& r) {
  float2* ms = buf<float2>(c.h->musig, r.npix);
  musig_kernel<<<ceil_div((long long)r.npix, 256), 256, 0, c.s>>>(r.args.S1, r.args.S2, (long long)r.npix, r.Ntot,
                                                                    ms);
  GISSPA_LAUNCH_CHECK();
  r.args.musig = ms;
  if (r.prune) {
    gisspa_handle* h = c.h;
    const long long rows = (long long)r.W * c.l, npairs = (long long)r.W * r.n_angles * h->nt;
    unsigned char* alive = buf<unsigned char>(h->alive, (size_t)rows + r.W + npairs);
    unsigned* cnt = buf<unsigned>(h->alive_count, 2 + r.W);  // rows, pairs, per-window bars
    GISSPA_CUDA(cudaMemsetAsync(alive + rows, 0, r.W, c.s));
    GISSPA_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), c.s));
    GISSPA_CUDA(cudaMemsetAsync(cnt + 2, 0xFF, sizeof(unsigned) * r.W, c.s));
    row_alive_kernel<<<ceil_div(rows * 32, 256), 256, 0, c.s>>>(r.args.peak, ms, c.l, rows, r.args.thresh, alive,
                                                               alive + rows, cnt, cnt + 2);
    GISSPA_LAUNCH_CHECK();
    pair_alive_kernel<<<ceil_div(npairs, 256), 256, 0, c.s>>>(r.args.pair_max, cnt + 2, r.W, r.n_angles, npairs,
                                                              alive + rows + r.W, cnt + 1);
    GISSPA_LAUNCH_CHECK();
    SkipMask& sk = r.args.skip;
    sk.rows = alive;
    sk.windows = alive + rows;
    sk.pairs = alive + rows + r.W;
    sk.nt_total = h->nt;
    sk.n_windows = r.W;
    sk.n_angles = r.n_angles;
  }
  r.phase = 3;
}

// A pruned second sweep over angles [a0, a1): from the host copy of the live pairs, each angle
// with any transforms the spectra of its live templates only and correlates (the launches skip
// the dead pairs); angles without a live pair are skipped.  Launched from the host (the
// templates differ from angle to angle).
void pruned_angles(Ctx& c, NormRun& r, int a0, int a1) {
  gisspa_handle* h = c.h;
  const int nt = h->nt, W = r.W, A = r.n_angles;
  if (r.live_templates.empty()) {
    std::vector<unsigned char> pa((size_t)W * A * nt);
    GISSPA_CUDA(cudaMemcpyAsync(pa.data(), r.args.skip.pairs, pa.size(), cudaMemcpyDeviceToHost, c.s));
    GISSPA_CUDA(cudaStreamSynchronize(c.s));
    r.live_templates.assign(A, {});
    for (int t = 0; t < nt; ++t)
      for (int a = 0; a < A; ++a)
        for (int w = 0; w < W; ++w)
          if (pa[pair_index(w, t, a, W, A)]) {
            r.live_templates[a].push_back(t);
            break;
          }
  }
  for (int a = a0; a < a1; ++a) {
    const std::vector<int>& list = r.live_templates[a];
    if (list.empty()) {
      r.pairs += (long long)W * nt;  // searched: every pair of this angle is known to hold no pick
      continue;
    }
    // every template's spectra where the launches read dead pairs too: the pair engine (a fixed
    // shape) and batches of more templates than pass B lists (a fixed template_batch)
    const bool fixed = h->cfg.template_batch > 0 && h->cfg.window_batch > 0;
    const bool all = (fixed && h->cfg.pass_b_shape == engine_variant(c.l)) ||
                     h->cfg.template_batch > kMaxListedTemplates;
    if (all)
      template_spectra_at(c, r.angles[a]);
    else
      template_spectra_listed(c, r.angles[a], list);
    r.args.angle = a;
    r.args.angle_state = nullptr;
    r.pairs += correlate_all(c, EPI_CHUNK, h->ispec.as<float2>(), W, h->tspec.as<void>(), nt, r.args, r.D, r.E);
  }
}

// Sweep 2 (PickParticles norm.cu:554-600) over angles [a0, a1): chunk candidates, grown and
// repeated once when the buffer overflows, left in r.cand in the reference's output order
// (angle, window with j outer and i inner, template, chunk; norm.cu:561-598).
void norm_sweep2(Ctx& c, NormRun& r, int a0, int a1) {
  gisspa_handle* h = c.h;
  unsigned cap = (unsigned)std::max<size_t>(h->cand.size() / sizeof(Cand), 1u << 16);
  r.cand.clear();
  for (int attempt = 0; attempt < 2; ++attempt) {
    Cand* cand = buf<Cand>(h->cand, cap);
    unsigned* cnt = buf<unsigned>(h->cand_count, 1);
    GISSPA_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned), c.s));
    r.args.cand = cand;
    r.args.cand_count = cnt;
    r.args.cand_cap = cap;
    if (r.args.skip.pairs)
      pruned_angles(c, r, a0, a1);
    else
      run_angles(c, r, EPI_CHUNK, a0, a1);
    GISSPA_CUDA(cudaEventRecord(h->ev[3], c.s));
    unsigned count = 0, alive_n[2] = {0, 0};
    GISSPA_CUDA(cudaMemcpyAsync(&count, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, c.s));
    if (r.args.skip.rows)
      GISSPA_CUDA(cudaMemcpyAsync(alive_n, h->alive_count.as<unsigned>(), 2 * sizeof(unsigned),
                                  cudaMemcpyDeviceToHost, c.s));
    GISSPA_CUDA(cudaStreamSynchronize(c.s));
    h->st.candidates = count;
    h->st.rows_alive = r.args.skip.rows ? (double)alive_n[0] / ((double)r.W * c.l) : 1.0;
    h->st.pairs_alive =
        r.args.skip.pairs ? (double)alive_n[1] / ((double)r.W * r.n_angles * h->nt) : 1.0;
    if (count > cap) {  // grow and repeat the second sweep only
      cap = count + count / 4 + 1024;
      continue;
    }
    r.cand.resize(count);
    if (count) GISSPA_CUDA(cudaMemcpyAsync(r.cand.data(), cand, sizeof(Cand) * count, cudaMemcpyDeviceToHost, c.s));
    GISSPA_CUDA(cudaStreamSynchronize(c.s));
    std::sort(r.cand.begin(), r.cand.end(), [](const Cand& u, const Cand& v) {
      if (u.angle != v.angle) return u.angle < v.angle;
      if (u.window != v.window) return u.window < v.window;
      if (u.templ != v.templ) return u.templ < v.templ;
      return u.chunk < v.chunk;
    });
    break;
  }
  r.phase = 4;
}

void chunk_picks(const NormRun& r, std::vector<gisspa_pick>& out) {
  out.reserve(out.size() + r.cand.size());
  for (const Cand& cd : r.cand) {
    gisspa_pick pk{};
    pk.score = cd.score;
    pk.x = (float)(r.ox[cd.window % r.bx] + cd.x);
    pk.y = (float)(r.oy[cd.window / r.bx] + cd.y);
    float cur_e = 360.0f - r.angles[cd.angle];  // norm.cu:700-701
    if (cur_e >= 360.0f) cur_e -= 360.0f;
    pk.angle = cur_e;
    pk.theta = r.angles[cd.angle];
    pk.template_id = cd.templ;
    pk.window = cd.window;
    pk.tile = 0;
    pk.angle_index = cd.angle;
    pk.chunk = cd.chunk;
    out.push_back(pk);
  }
}

// Top-K on the image map of the max z: threshold, centre rule, greedy exclusion in score order.
void topk_picks(Ctx& c, NormRun& r, std::vector<gisspa_pick>& out) {
  gisspa_handle* h = c.h;
  const gisspa_config& cfg = h->cfg;
  const int l = c.l, nt = h->nt, nx = r.nx, ny = r.ny, bx = r.bx;
  const long long N = r.N;
  unsigned long long* zk = buf<unsigned long long>(h->zkey, N);
  GISSPA_CUDA(cudaMemsetAsync(zk, 0, sizeof(unsigned long long) * N, c.s));
  zmap_kernel<<<dim3(ceil_div(c.L2, 256), r.W), 256, 0, c.s>>>(r.args.peak, r.args.musig, l, r.args.offx,
                                                                r.args.offy, bx, nx, ny, zk);
  GISSPA_LAUNCH_CHECK();
  unsigned cap = (unsigned)std::max<size_t>(h->zcand.size() / sizeof(ZCand), 1u << 16);
  std::vector<ZCand> hz;
  for (int attempt = 0; attempt < 2; ++attempt) {
    ZCand* zc = buf<ZCand>(h->zcand, cap);
    unsigned* cnt = buf<unsigned>(h->zcount, 1);
    GISSPA_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned), c.s));
    zcompact_kernel<<<ceil_div(N, 256), 256, 0, c.s>>>(zk, nx, ny, cfg.threshold, cfg.diameter, r.args.peak, l,
                                                        r.args.offx, r.args.offy, bx, zc, cnt, cap);
    GISSPA_LAUNCH_CHECK();
    unsigned count = 0;
    GISSPA_CUDA(cudaMemcpyAsync(&count, cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, c.s));
    GISSPA_CUDA(cudaStreamSynchronize(c.s));
    if (count > cap) {
      cap = count + 1024;
      continue;
    }
    hz.resize(count);
    if (count) GISSPA_CUDA(cudaMemcpy(hz.data(), zc, sizeof(ZCand) * count, cudaMemcpyDeviceToHost));
    break;
  }
  GISSPA_CUDA(cudaEventRecord(h->ev[3], c.s));
  h->st.candidates = (long long)hz.size();
  std::sort(hz.begin(), hz.end(), [](const ZCand& u, const ZCand& v) {
    if (u.z != v.z) return u.z > v.z;
    return u.q < v.q;
  });
  const double r2 = (double)cfg.exclusion_radius * cfg.exclusion_radius;
  std::vector<int> acc;
  for (const ZCand& zc : hz) {
    if ((int)acc.size() >= cfg.topk) break;
    const int x = zc.q % nx, y = zc.q / nx;
    bool ok = true;
    for (int q2 : acc) {
      const double dx = x - q2 % nx, dy = y - q2 / nx;
      if (dx * dx + dy * dy <= r2) {
        ok = false;
        break;
      }
    }
    if (!ok) continue;
    acc.push_back(zc.q);
    gisspa_pick pk{};
    pk.score = zc.z;
    pk.x = (float)x;
    pk.y = (float)y;
    const int a = zc.arg / nt, n = zc.arg % nt;
    float cur_e = 360.0f - r.angles[a];
    if (cur_e >= 360.0f) cur_e -= 360.0f;
    pk.angle = cur_e;
    pk.theta = r.angles[a];
    pk.template_id = n;
    pk.window = zc.win;
    pk.angle_index = a;
    pk.chunk = (int)acc.size() - 1;
    out.push_back(pk);
  }
}

void search_norm(Ctx& c, const float* d_img, int nx, int ny, std::vector<gisspa_pick>& out) {
  gisspa_handle* h = c.h;
  NormRun& r = h->run;
  norm_prepare(c, d_img, nx, ny, r);
  r.prune = h->cfg.prune_sweep2 != 0 && !r.topk && correlate_fast(c.l);
  if (r.prune) {  // sweep 1 keeps each pixel's best correlation and each pair's maximum
    r.args.peak = buf<unsigned long long>(h->peak, r.npix);
    GISSPA_CUDA(cudaMemsetAsync(r.args.peak, 0, sizeof(unsigned long long) * r.npix, c.s));
    r.n_angles = (int)r.angles.size();
    const size_t npairs = (size_t)r.W * r.n_angles * h->nt;
    r.args.pair_max = buf<unsigned>(h->pair_max, npairs);
    r.args.n_windows = r.W;
    r.args.n_angles = r.n_angles;
    GISSPA_CUDA(cudaMemsetAsync(r.args.pair_max, 0, sizeof(unsigned) * npairs, c.s));
  }
  const int A = (int)r.angles.size();
  norm_sweep1(c, r, 0, A);
  if (h->after_sweep1) {  // the sweep is queued: the host is free until the picks are read
    std::function<void()> f = std::move(h->after_sweep1);
    h->after_sweep1 = nullptr;
    f();
  }
  norm_stats(c, r);
  GISSPA_CUDA(cudaEventRecord(h->ev[2], c.s));
  if (!r.topk) {
    norm_sweep2(c, r, 0, A);
    chunk_picks(r, out);
  } else {
    topk_picks(c, r, out);
  }
  h->st.pairs = r.pairs;
  r.phase = 0;
}

// norm_type = 0 (SearchNoNorm, nonorm.cu): 720^2 tiles, rotate the windows, per-template best.
// One norm_type=0 peak: the best pixel of one (tile, angle, window, template) map (the
// reference's per-window peak, nonorm.cu:488-534), centre in micrograph coordinates.
struct NonormCand {
  double score;
  float x, y;
  int tile, angle, window;
};

// Per-template top-K with an exclusion radius over a template's norm_type=0 peaks (no
// counterpart in the reference, which keeps one window per template, angle and tile): peaks in
// descending score (ties in generation order: tile, angle, window), each taken unless it lies
// within exclusion_radius of a peak already taken for the same template; at most topk.
void nonorm_topk(std::vector<NonormCand>& cand, int n, const gisspa_config& cfg, const std::vector<float>& angles,
                 std::vector<gisspa_pick>& out) {
  std::stable_sort(cand.begin(), cand.end(),
                   [](const NonormCand& u, const NonormCand& v) { return u.score > v.score; });
  const double r2 = (double)cfg.exclusion_radius * cfg.exclusion_radius;
  std::vector<const NonormCand*> taken;
  for (const NonormCand& q : cand) {
    if ((int)taken.size() >= cfg.topk) break;
    bool ok = true;
    for (const NonormCand* u : taken) {
      const double dx = (double)q.x - u->x, dy = (double)q.y - u->y;
      if (dx * dx + dy * dy <= r2) {
        ok = false;
        break;
      }
    }
    if (!ok) continue;
    gisspa_pick pk{};
    pk.score = (float)q.score;
    pk.x = q.x;
    pk.y = q.y;
    pk.angle = angles[q.angle];
    pk.theta = angles[q.angle];
    pk.template_id = n;
    pk.window = q.window;
    pk.tile = q.tile;
    pk.angle_index = q.angle;
    pk.chunk = (int)taken.size();
    out.push_back(pk);
    taken.push_back(&q);
  }
}

void search_nonorm(Ctx& c, const float* d_img, int nx, int ny, std::vector<gisspa_pick>& out) {
  gisspa_handle* h = c.h;
  const gisspa_config& cfg = h->cfg;
  const int l = c.l, nt = h->nt, ts = cfg.tile_size, hs = l / 2 + 1;
  GISSPA_CUDA(cudaEventRecord(h->ev[0], c.s));
  prepare_templates(c);
  // tiles (TileImages, tileimages.cpp:18-70): column-major, centres clamped to the image
  const int cols = (int)std::ceil((double)nx / ts), rows = (int)std::ceil((double)ny / ts);
  const int x_step = nx / cols, y_step = ny / rows;
  std::vector<int> tx, ty;
  for (int j = 0; j < cols; ++j) {
    const int cxx = j == 0 ? ts / 2 : (j == cols - 1 ? nx - ts / 2 : x_step * (2 * j + 1) / 2);
    for (int i = 0; i < rows; ++i) {
      const int cyy = i == 0 ? ts / 2 : (i == rows - 1 ? ny - ts / 2 : y_step * (2 * i + 1) / 2);
      tx.push_back(std::max(cxx - ts / 2, 0));
      ty.push_back(std::max(cyy - ts / 2, 0));
    }
  }
  const int bx = window_count_nonorm(ts, l, cfg.overlap), W = bx * bx;
  std::vector<int> woff(bx);
  for (int k = 0; k < bx; ++k) woff[k] = k * (l - cfg.overlap);  // split_IMG unclamped (kernels.cu:605-624)
  const std::vector<float> angles = angle_list(cfg.phistep);
  int D, E;
  choose_batches(cfg, l, W, nt, D, E);
  const long long TS2 = (long long)ts * ts;
  int* dtx = buf<int>(h->offx, std::max<size_t>(woff.size(), 2));
  int* dty = buf<int>(h->offy, std::max<size_t>(woff.size(), 2));
  unsigned long long* nk = buf<unsigned long long>(h->nn_key, (size_t)W * nt);
  double* nsum = buf<double>(h->nn_sum, (size_t)W * nt * 2);
  std::vector<unsigned long long> hk((size_t)W * nt);
  std::vector<double> hsum((size_t)W * nt * 2);
  long long pairs = 0;
  // top-K: every (tile, angle, window) peak of each template that passes the reference's
  // centre test and the threshold, in that generation order
  const bool topk = cfg.pick_mode == GISSPA_PICK_TOPK;
  std::vector<std::vector<NonormCand>> cands(topk ? nt : 0);
  GISSPA_CUDA(cudaEventRecord(h->ev[1], c.s));
  for (size_t t = 0; t < tx.size(); ++t) {
    // LoadImage (nonorm.cu:157-165): the tile, inverted on request
    int tile_off[2] = {tx[t], ty[t]};
    GISSPA_CUDA(cudaMemcpyAsync(dtx, &tile_off[0], sizeof(int), cudaMemcpyHostToDevice, c.s));
    GISSPA_CUDA(cudaMemcpyAsync(dty, &tile_off[1], sizeof(int), cudaMemcpyHostToDevice, c.s));
    float2* G = buf<float2>(h->img_c, TS2);
    gather_windows(d_img, nx, ny, dtx, dty, 1, 1, ts, G, c.s);
    float* tile = buf<float>(h->tile_real, TS2);
    if (cfg.phase_flip == 1) {  // PreprocessImage (nonorm.cu:346-389), no DC zeroing
      if (cfg.invert) {
        real_part(G, tile, TS2, -1.f, c.s);
        to_complex(tile, G, TS2, c.s);
      }
      preprocess_full(c, G, ts, ts, false);
    }
    real_part(G, tile, TS2, (cfg.invert && cfg.phase_flip != 1) ? -1.f : 1.f, c.s);
    // SplitImage (nonorm.cu:391-450)
    GISSPA_CUDA(cudaMemcpyAsync(dtx, woff.data(), sizeof(int) * bx, cudaMemcpyHostToDevice, c.s));
    GISSPA_CUDA(cudaMemcpyAsync(dty, woff.data(), sizeof(int) * bx, cudaMemcpyHostToDevice, c.s));
    float2* w = buf<float2>(h->win_c, (size_t)W * c.L2);
    float2* wtmp = buf<float2>(h->win_tmp, (size_t)W * c.L2);
    gather_windows(tile, ts, ts, dtx, dty, bx, W, l, w, c.s);
    if (cfg.phase_flip == 1) {
      h->fft.fft2(w, wtmp, W, l, l, -1, 1.0f / (float)c.L2, c.s);
      rms_normalise(w, W, l, nullptr, c.s);
      h->fft.fft2(w, wtmp, W, l, l, +1, 1.f, c.s);
    }
    float* wr = buf<float>(h->win_real, (size_t)W * c.L2);
    real_part(w, wr, (long long)W * c.L2, 1.f, c.s);
    for (size_t a = 0; a < angles.size(); ++a) {
      const float e = angles[a];
      const double rad = (double)e * kRefPi / 180.0;
      // PickParticles (nonorm.cu:452-537): rotate the windows, transform, correlate
      float2* rot = buf<float2>(h->rot, (size_t)W * c.L2);
      float2* rtmp = buf<float2>(h->rot_tmp, (size_t)W * hs * l);
      rotate_batch(wr, W, l, (float)std::cos(rad), (float)std::sin(rad), false, 0.f, 0.f, rot, nullptr, c.s);
      h->fft.rows(rot, (long long)W * l, l, -1, 1.f, c.s);
      h->fft.transpose(rot, rtmp, W, l, l, c.s, hs);
      h->fft.rows(rtmp, (long long)W * hs, l, -1, 1.f, c.s);
      float2* I = buf<float2>(h->ispec, (size_t)W * hs * l);
      finalize_spectra(rtmp, W, l, nullptr, GISSPA_SPEC_FP32, I, 1.0 / (double)c.L2, c.s);
      GISSPA_CUDA(cudaMemsetAsync(nk, 0, sizeof(unsigned long long) * W * nt, c.s));
      GISSPA_CUDA(cudaMemsetAsync(nsum, 0, sizeof(double) * W * nt * 2, c.s));
      CorrArgs args{};
      args.nt_real = nt;
      args.nt_total = nt;
      args.angle = (int)a;
      args.nn_key = nk;
      args.nn_sum = nsum;
      args.border = cfg.diameter / 4;
      pairs += correlate_all(c, EPI_NONORM, I, W, h->tspec.as<void>(), nt, args, D, E);
      GISSPA_CUDA(cudaMemcpyAsync(hk.data(), nk, sizeof(unsigned long long) * W * nt, cudaMemcpyDeviceToHost, c.s));
      GISSPA_CUDA(cudaMemcpyAsync(hsum.data(), nsum, sizeof(double) * W * nt * 2, cudaMemcpyDeviceToHost, c.s));
      GISSPA_CUDA(cudaStreamSynchronize(c.s));
      // host merge (nonorm.cu:498-534): best window per template, centre rotated back
      std::vector<float> bs(nt, 0.f), bxp(nt, 0.f), byp(nt, 0.f);
      const double ce = std::cos(rad), se = std::sin(rad);
      for (int b = 0; b < W; ++b) {
        const int i = b % bx, j = b / bx;
        for (int n = 0; n < nt; ++n) {
          const unsigned long long k = hk[(size_t)b * nt + n];
          double peak = 0, pos = 0;
          if (k) {
            uint32_t hi = (uint32_t)(k >> 32);
            uint32_t bits = (hi & 0x80000000u) ? (hi & 0x7fffffffu) : ~hi;
            float pv;
            std::memcpy(&pv, &bits, 4);
            // low word: (0xFFFFF - chunk) << 8 | (255 - brev8(position in the chunk))
            const unsigned lo = (unsigned)(k & 0xFFFFFFFFu);
            const int chunk = (int)(0xFFFFFu - (lo >> 8));
            unsigned t = 255u - (lo & 0xFFu), tb = 0;
            for (int bit = 0; bit < 8; ++bit) tb |= ((t >> bit) & 1u) << (7 - bit);
            peak = pv;
            pos = (double)(chunk * 256 + (int)tb);
          }
          const double s1 = hsum[2 * ((size_t)b * nt + n)], s2 = hsum[2 * ((size_t)b * nt + n) + 1];
          const double rA = s1 - peak, rB = s2 - peak * peak, rC = (double)c.L2 - 1;
          const double sd = std::sqrt(rB / rC - (rA / rC) * (rA / rC));
          const double score = sd == 0 ? 0.0 : peak / sd;
          const int cx = (int)pos % l, cy = (int)pos / l;
          const double centerx = i * (l - cfg.overlap) + (cx - l / 2) * ce + (cy - l / 2) * se + l / 2;
          const double centery = j * (l - cfg.overlap) + (cy - l / 2) * ce - (cx - l / 2) * se + l / 2;
          const bool valid = centerx >= 0 && centerx < ts && centery >= 0 && centery < ts;
          if (topk) {
            if (valid && (float)score >= cfg.threshold)
              cands[n].push_back(NonormCand{score, (float)(tx[t] + centerx), (float)(ty[t] + centery), (int)t,
                                            (int)a, b});
            continue;
          }
          if (bs[n] < (float)score && valid) {
            bs[n] = (float)score;
            bxp[n] = (float)centerx;
            byp[n] = (float)centery;
          }
        }
      }
      if (topk) continue;
      for (int n = 0; n < nt; ++n)  // OutputScore (nonorm.cu:539-557)
        if (bs[n] >= cfg.threshold) {
          gisspa_pick pk{};
          pk.score = bs[n];
          pk.x = bxp[n];
          pk.y = byp[n];
          pk.angle = e;
          pk.theta = e;
          pk.template_id = n;
          pk.window = -1;
          pk.tile = (int)t;
          pk.angle_index = (int)a;
          pk.chunk = -1;
          out.push_back(pk);
        }
    }
  }
  GISSPA_CUDA(cudaEventRecord(h->ev[2], c.s));
  if (topk) {
    for (int n = 0; n < nt; ++n) nonorm_topk(cands[n], n, cfg, angles, out);
  }
  GISSPA_CUDA(cudaEventRecord(h->ev[3], c.s));
  h->st.pairs = pairs;
}

}  // namespace

void debug_stage(gisspa_handle* h, int what, const float* d_img, int nx, int ny, const gisspa_ctf& ctf, float theta,
                 void* out, size_t bytes) {
  Ctx c{h, h->stream, h->cfg.window_size, (long long)h->cfg.window_size * h->cfg.window_size,
        make_params(h->cfg, ctf)};
  const gisspa_config& cfg = h->cfg;
  const int l = c.l, hs = l / 2 + 1;
  auto fetch = [&](const void* src, size_t need) {
    if (bytes < need) throw CudaError{cudaErrorInvalidValue, "debug_stage: output buffer too small"};
    GISSPA_CUDA(cudaMemcpyAsync(out, src, need, cudaMemcpyDeviceToHost, c.s));
    GISSPA_CUDA(cudaStreamSynchronize(c.s));
  };
  if (what == GISSPA_STAGE_MUSIG) {
    if (!h->musig.size() || cfg.norm_type == 0)
      throw CudaError{cudaErrorInvalidValue, "debug_stage: no norm_type=1 search has run"};
    fetch(h->musig.as<void>(), std::min(bytes, h->musig.size()));
    return;
  }
  if (what == GISSPA_STAGE_TEMPLATE_SPECTRA && cfg.norm_type == 0)
    throw CudaError{cudaErrorInvalidValue, "debug_stage: per-angle template spectra exist for norm_type=1 only"};
  prepare_templates(c);
  if (what == GISSPA_STAGE_TEMPLATES) {
    if (cfg.norm_type != 0) {
      fetch(h->prep_real.as<void>(), sizeof(float) * (size_t)h->nt * c.L2);
    } else {
      float2* tmp = buf<float2>(h->tb_tmp, (size_t)h->nt * hs * l);
      h->fft.transpose(h->tb.as<float2>(), tmp, h->nt, l, l, c.s, hs);
      fetch(tmp, sizeof(float2) * (size_t)h->nt * hs * l);
    }
    return;
  }
  if (what == GISSPA_STAGE_TEMPLATE_SPECTRA) {
    template_spectra_at(c, theta);
    float2* tmp = buf<float2>(h->tb_tmp, (size_t)h->nt * hs * l);
    finalize_spectra(h->rot_tmp.as<float2>(), h->nt, l, h->rsums.as<double>(), GISSPA_SPEC_FP32, tmp,
                     1.0 / (double)c.L2, c.s);
    fetch(tmp, sizeof(float2) * (size_t)h->nt * hs * l);
    return;
  }
  if (!d_img) throw CudaError{cudaErrorInvalidValue, "debug_stage: image required"};
  const long long N = (long long)nx * ny;
  float* stats = buf<float>(h->stats, 4);
  double* scr = buf<double>(h->scratch, 16);
  image_stats(d_img, nx, ny, (cfg.quirks & GISSPA_QUIRK_OUTLIER_FP32_SERIAL) != 0, stats, scr, c.s);
  float2* G = buf<float2>(h->img_c, N);
  image_load(d_img, N, stats, true, cfg.invert != 0, G, c.s);
  preprocess_full(c, G, nx, ny, true);
  float* img = buf<float>(h->img_pre, N);
  real_part(G, img, N, 1.f, c.s);
  if (what == GISSPA_STAGE_IMAGE) {
    fetch(img, sizeof(float) * N);
    return;
  }
  const std::vector<int> ox = window_offsets(nx, l, cfg.overlap), oy = window_offsets(ny, l, cfg.overlap);
  window_spectra(c, img, nx, ny, ox, oy);
  if (what == GISSPA_STAGE_WINDOW_SPECTRA) {
    fetch(h->ispec.as<void>(), sizeof(float2) * ox.size() * oy.size() * hs * l);
    return;
  }
  throw CudaError{cudaErrorInvalidValue, "debug_stage: unknown stage"};
}

// ---- adjoint (a-Adj): score gradients and refinement of picks and of the micrograph CTF
namespace {

struct Psi {
  double dfu, dfv, dfang;
};
Psi psi_of(const gisspa_ctf& c) { return Psi{-c.defocus + c.dfdiff, -c.defocus - c.dfdiff, c.dfang}; }
gisspa_ctf ctf_of(const Psi& p) { return gisspa_ctf{-(p.dfu + p.dfv) / 2, (p.dfu - p.dfv) / 2, p.dfang}; }

// Prepared templates and their CTF derivatives at ctf; window sums of the last search.
void adjoint_prepare(gisspa_handle* h, const gisspa_ctf& ctf) {
  Ctx c{h, h->stream, h->cfg.window_size, (long long)h->cfg.window_size * h->cfg.window_size,
        make_params(h->cfg, ctf)};
  const int l = c.l, nt = h->nt;
  h->keep_whitened = true;
  prepare_templates(c);
  h->keep_whitened = false;
  float* dtab = buf<float>(h->dtab, 3 * (size_t)c.L2);
  ctf_dweight(dtab, l, c.p, c.s);
  float* dprep = buf<float>(h->dprep, 3 * (size_t)nt * c.L2);
  float2* tb = buf<float2>(h->tb, (size_t)nt * c.L2);
  float2* tmp = buf<float2>(h->tb_tmp, (size_t)nt * c.L2);
  for (int q = 0; q < 3; ++q) {
    scale_by_table(h->tw_spec.as<float2>(), dtab + (size_t)q * c.L2, h->tmpl_m.as<double>(), nt, l, tb, c.s);
    h->fft.fft2(tb, tmp, nt, l, l, +1, 1.f, c.s);  // same unnormalised IFFT as the prepared templates
    real_part(tb, dprep + (size_t)q * nt * c.L2, (long long)nt * c.L2, 1.f, c.s);
  }
  window_sums(h->img_pre.as<float>(), h->last_nx, h->last_ny, h->offx.as<int>(), h->offy.as<int>(), h->last_bx,
              h->last_W, l, h->win_m.as<double>(), buf<double>(h->win_sum, h->last_W), c.s);
  // the FP16 / BF16 template forms evaluate from templates stored at that precision
  const int prec = h->cfg.spectrum_precision;
  if (prec != GISSPA_SPEC_FP32)
    round_templates(h->prep_real.as<float>(), (long long)nt * c.L2, dprep, 3LL * nt * c.L2, prec,
                    buf<unsigned>(h->lp_scale, 1), buf<__half>(h->prep_lp, (size_t)nt * c.L2),
                    buf<__half>(h->dprep_lp, 3 * (size_t)nt * c.L2), c.s);
}

void eval_grads(gisspa_handle* h, const std::vector<GradPick>& gp, std::vector<float>& out) {
  const int n = (int)gp.size();
  GradArgs g{};
  g.prep = h->prep_real.as<float>();
  g.dprep = h->dprep.as<float>();
  g.precision = h->cfg.spectrum_precision;
  g.prep_lp = g.precision != GISSPA_SPEC_FP32 ? h->prep_lp.as<void>() : nullptr;
  g.dprep_lp = g.precision != GISSPA_SPEC_FP32 ? h->dprep_lp.as<void>() : nullptr;
  g.img = h->img_pre.as<float>();
  g.nx = h->last_nx;
  g.ny = h->last_ny;
  g.offx = h->offx.as<int>();
  g.offy = h->offy.as<int>();
  g.bx = h->last_bx;
  g.win_m = h->win_m.as<double>();
  g.win_sum = h->win_sum.as<double>();
  g.musig = h->musig.as<float2>();
  g.L = h->cfg.window_size;
  g.nt = h->nt;
  g.d_m = h->cfg.diameter;
  g.ehw = h->cfg.edge_half_width;
  GradPick* dp = buf<GradPick>(h->grad_in, n);
  float* dout = buf<float>(h->grad_out, (size_t)n * 7);
  GISSPA_CUDA(cudaMemcpyAsync(dp, gp.data(), sizeof(GradPick) * n, cudaMemcpyHostToDevice, h->stream));
  score_grads(g, dp, n, dout, h->stream);
  out.resize((size_t)n * 7);
  GISSPA_CUDA(cudaMemcpyAsync(out.data(), dout, sizeof(float) * n * 7, cudaMemcpyDeviceToHost, h->stream));
  GISSPA_CUDA(cudaStreamSynchronize(h->stream));
}

std::vector<GradPick> grad_picks(gisspa_handle* h, const gisspa_pick* picks, size_t n, const float* params) {
  std::vector<GradPick> gp(n);
  const int L = h->cfg.window_size;
  for (size_t i = 0; i < n; ++i) {
    const gisspa_pick& p = picks[i];
    if (p.window < 0 || p.window >= h->last_W || p.template_id < 0 || p.template_id >= h->nt)
      throw CudaError{cudaErrorInvalidValue, "pick " + std::to_string(i) + " does not belong to the last search"};
    GradPick g{};
    g.b = p.window;
    g.n = p.template_id;
    g.px = (int)p.x - h->last_offx[p.window % h->last_bx];
    g.py = (int)p.y - h->last_offy[p.window / h->last_bx];
    if (g.px < 0 || g.px >= L || g.py < 0 || g.py >= L)
      throw CudaError{cudaErrorInvalidValue, "pick " + std::to_string(i) + " lies outside its window"};
    g.dx = params ? params[3 * i] : 0.f;
    g.dy = params ? params[3 * i + 1] : 0.f;
    g.theta = params ? params[3 * i + 2] : p.theta;
    gp[i] = g;
  }
  return gp;
}

}  // namespace

void score_grad_run(gisspa_handle* h, const gisspa_pick* picks, size_t n, const float* params, const gisspa_ctf* ctf,
                    gisspa_grad* out) {
  if (h->last_W <= 0 || h->cfg.norm_type == 0)
    throw CudaError{cudaErrorInvalidValue, "score gradients need a preceding norm_type=1 search on this handle"};
  std::vector<GradPick> gp = grad_picks(h, picks, n, params);
  adjoint_prepare(h, ctf ? *ctf : h->last_ctf);
  std::vector<float> o;
  eval_grads(h, gp, o);
  for (size_t i = 0; i < n; ++i)
    out[i] = gisspa_grad{o[7 * i], o[7 * i + 1], o[7 * i + 2], o[7 * i + 3], o[7 * i + 4], o[7 * i + 5], o[7 * i + 6]};
}

// Batched local refinement: per pick, normalised gradient ascent on (dx, dy, theta) with an
// adaptive step (grown on success, halved on failure); per micrograph, the same on the CTF
// (dfu, dfv, dfang) driven by the summed pick gradients.  Each proposal is evaluated and kept
// only if it raises the score (mean score for the CTF).
void refine_run(gisspa_handle* h, gisspa_pick* picks, size_t n, int steps, gisspa_ctf* ctf, float* params_out) {
  if (h->last_W <= 0 || h->cfg.norm_type == 0)
    throw CudaError{cudaErrorInvalidValue, "refinement needs a preceding norm_type=1 search on this handle"};
  std::vector<GradPick> gp = grad_picks(h, picks, n, nullptr);
  Psi psi = psi_of(ctf ? *ctf : h->last_ctf);
  adjoint_prepare(h, ctf_of(psi));
  std::vector<float> cur, trial;
  eval_grads(h, gp, cur);
  std::vector<double> eps(n, 1.0);
  double eps_psi = 1.0;
  const double eta[3] = {1.0, 1.0, std::max(0.5, 0.5 * (double)h->cfg.phistep)};
  const double eta_psi[3] = {0.05, 0.05, 5.0};
  auto mean_score = [&](const std::vector<float>& v) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += v[7 * i];
    return n ? s / n : 0.0;
  };
  for (int it = 0; it < steps; ++it) {
    // picks
    std::vector<GradPick> prop = gp;
    for (size_t i = 0; i < n; ++i) {
      const double g[3] = {cur[7 * i + 1] * eta[0], cur[7 * i + 2] * eta[1], cur[7 * i + 3] * eta[2]};
      const double nrm = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
      if (!(nrm > 0)) continue;
      prop[i].dx = (float)(gp[i].dx + eps[i] * eta[0] * g[0] / nrm);
      prop[i].dy = (float)(gp[i].dy + eps[i] * eta[1] * g[1] / nrm);
      prop[i].theta = (float)(gp[i].theta + eps[i] * eta[2] * g[2] / nrm);
    }
    eval_grads(h, prop, trial);
    for (size_t i = 0; i < n; ++i) {
      if (trial[7 * i] > cur[7 * i]) {
        gp[i] = prop[i];
        for (int k = 0; k < 7; ++k) cur[7 * i + k] = trial[7 * i + k];
        eps[i] = std::min(eps[i] * 1.25, 4.0);
      } else {
        eps[i] *= 0.5;
      }
    }
    // micrograph CTF (only when the caller passes one to refine)
    if (!ctf) continue;
    double G[3] = {0, 0, 0};
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) G[k] += cur[7 * i + 4 + k] * eta_psi[k];
    const double nrm = std::sqrt(G[0] * G[0] + G[1] * G[1] + G[2] * G[2]);
    if (nrm > 0 && n) {
      Psi p2{psi.dfu + eps_psi * eta_psi[0] * G[0] / nrm, psi.dfv + eps_psi * eta_psi[1] * G[1] / nrm,
             psi.dfang + eps_psi * eta_psi[2] * G[2] / nrm};
      adjoint_prepare(h, ctf_of(p2));
      eval_grads(h, gp, trial);
      if (mean_score(trial) > mean_score(cur)) {
        psi = p2;
        cur = trial;
        eps_psi = std::min(eps_psi * 1.25, 4.0);
      } else {
        eps_psi *= 0.5;
        adjoint_prepare(h, ctf_of(psi));
      }
    }
  }
  const int L = h->cfg.window_size;
  (void)L;
  for (size_t i = 0; i < n; ++i) {
    picks[i].x += gp[i].dx;
    picks[i].y += gp[i].dy;
    picks[i].theta = gp[i].theta;
    float cur_e = 360.0f - gp[i].theta;
    while (cur_e >= 360.0f) cur_e -= 360.0f;
    while (cur_e < 0.0f) cur_e += 360.0f;
    picks[i].angle = cur_e;
    picks[i].score = cur[7 * i];
    if (params_out) {
      params_out[3 * i] = gp[i].dx;
      params_out[3 * i + 1] = gp[i].dy;
      params_out[3 * i + 2] = gp[i].theta;
    }
  }
  if (ctf) *ctf = ctf_of(psi);
}

void cc_maps(gisspa_handle* h, const void* d_win, int nw, const void* d_t, int ntm, int spec, float* d_out) {
  Ctx c{h, h->stream, h->cfg.window_size, (long long)h->cfg.window_size * h->cfg.window_size, DevParams{}};
  const int l = c.l;
  CorrArgs args{};
  args.map_out = d_out;
  args.nt_real = ntm;
  args.nt_total = ntm;
  args.err = buf<unsigned>(h->dev_err, 1);
  GISSPA_CUDA(cudaMemsetAsync(args.err, 0, sizeof(unsigned), c.s));
  const bool generic = !correlate_fast(l);
  float2* Q = generic ? nullptr : buf<float2>(h->Q, (size_t)ntm * (l / 2) * l);
  const float2* twL = generic ? nullptr : h->fft.twiddles(l);
  const float2* twNZ = generic ? nullptr : h->fft.twiddles(l / 2);
  float2* gz = generic ? buf<float2>(h->gen_z, generic_z_elems(l, ntm)) : nullptr;
  const size_t xe = generic ? generic_x_elems(l, ntm, EPI_MAP) : 0;
  float2* gx = xe ? buf<float2>(h->gen_x, xe) : nullptr;
  // one launch per window: pair p = d covers template d of window b, written at [b][d]
  for (int b = 0; b < nw; ++b) {
    CorrLaunch cl{l, 1, ntm, spec, EPI_MAP};
    args.Q = Q;
    args.b0 = b;
    args.n0 = 0;
    args.D = ntm;
    args.map_out = d_out + (size_t)b * ntm * c.L2;
    if (generic)
      correlate_generic(cl, static_cast<const float2*>(d_win), d_t, args, h->fft, gz, gx, c.s);
    else
      correlate_launch(cl, static_cast<const float2*>(d_win), d_t, Q, args, twL, twNZ, c.s);
  }
  GISSPA_CUDA(cudaStreamSynchronize(c.s));
  unsigned flag = 0;
  GISSPA_CUDA(cudaMemcpy(&flag, args.err, sizeof(flag), cudaMemcpyDeviceToHost));
  if (flag) throw TimeoutError{"cc_maps"};
}

void project_run(gisspa_handle* h, const float* volume, int nx, int ny, int nz, const float* angles, int n, int ri,
                 float* d_out) {
  const size_t nv = (size_t)nx * ny * nz;
  float* dv = buf<float>(h->proj_vol, nv);
  GISSPA_CUDA(cudaMemcpyAsync(dv, volume, sizeof(float) * nv, cudaMemcpyHostToDevice, h->stream));
  std::vector<float> mx;
  projection_matrices(angles, n, mx);
  float* dm = buf<float>(h->proj_mx, mx.size());
  GISSPA_CUDA(cudaMemcpyAsync(dm, mx.data(), sizeof(float) * mx.size(), cudaMemcpyHostToDevice, h->stream));
  project_volume(dv, projection_geometry(nx, ny, nz, ri), dm, n, d_out, h->stream);
  GISSPA_CUDA(cudaStreamSynchronize(h->stream));
}

void wait_probe(gisspa_handle* h, double seconds) {
  int khz = 0;
  GISSPA_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, h->device));
  unsigned* err = buf<unsigned>(h->dev_err, 1);
  GISSPA_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), h->stream));
  wait_probe_kernel<<<1, 32, 0, h->stream>>>(err, (long long)(seconds * 1e3 * (double)std::max(khz, 1)));
  GISSPA_LAUNCH_CHECK();
  GISSPA_CUDA(cudaStreamSynchronize(h->stream));
  unsigned flag = 0;
  GISSPA_CUDA(cudaMemcpy(&flag, err, sizeof(flag), cudaMemcpyDeviceToHost));
  if (flag) throw TimeoutError{"the wait probe"};
}

void run_search(gisspa_handle* h, const float* d_img, int nx, int ny, const gisspa_ctf& ctf,
                std::vector<gisspa_pick>& out) {
  Ctx c{h, h->stream, h->cfg.window_size, (long long)h->cfg.window_size * h->cfg.window_size,
        make_params(h->cfg, ctf)};
  h->last_ctf = ctf;
  h->last_W = 0;
  const long long l0 = launch_counter();
  h->st = gisspa_stats{};
  h->n_samples = 0;
  h->n_seqs = 0;
  h->launch_index = 0;
  unsigned* err = buf<unsigned>(h->dev_err, 1);
  GISSPA_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), c.s));
  if (h->cfg.norm_type != 0)
    search_norm(c, d_img, nx, ny, out);
  else
    search_nonorm(c, d_img, nx, ny, out);
  GISSPA_CUDA(cudaEventRecord(h->ev[4], c.s));
  GISSPA_CUDA(cudaStreamSynchronize(c.s));
  unsigned flag = 0;
  GISSPA_CUDA(cudaMemcpy(&flag, err, sizeof(flag), cudaMemcpyDeviceToHost));
  if (flag) throw TimeoutError{"the correlation kernels"};
  float ms = 0;
  GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[0], h->ev[4]));
  h->st.ms_total = ms;
  GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
  h->st.ms_prep = ms;
  GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]));
  h->st.ms_sweep1 = ms;
  GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[2], h->ev[3]));
  h->st.ms_sweep2 = ms;
  GISSPA_CUDA(cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]));
  h->st.ms_pick = ms;
  h->st.kernel_launches = launch_counter() - l0;
  h->st.window_size = c.l;
  double ta = 0, tb = 0, pp = 0, dd = 0;
  for (int i = 0; i < h->n_samples; ++i) {
    float a = 0, b = 0;
    GISSPA_CUDA(cudaEventElapsedTime(&a, h->sev[i][0], h->sev[i][1]));
    GISSPA_CUDA(cudaEventElapsedTime(&b, h->sev[i][1], h->sev[i][2]));
    ta += a;
    tb += b;
    pp += h->sample_pairs[i];
    dd += h->sample_d[i];
  }
  if (h->n_samples) {
    h->st.pass_a_us = 1000.0 * ta / h->n_samples;
    h->st.pass_b_us = 1000.0 * tb / h->n_samples;
    h->st.pairs_per_launch = pp / h->n_samples;
    h->st.templates_per_launch = dd / h->n_samples;
  }
  h->st.pass_samples = h->n_samples;
  double tq = 0;
  long long nl = 0, np = 0, nd = 0;
  for (int i = 0; i < h->n_seqs; ++i) {
    if (h->seq_pruned[i]) continue;  // the launch pair's time is that of full work
    float q = 0;
    GISSPA_CUDA(cudaEventElapsedTime(&q, h->qev[i][0], h->qev[i][1]));
    tq += q;
    nl += h->seq_launches[i];
    np += h->seq_pairs[i];
    nd += h->seq_d[i];
  }
  if (nl) {
    h->st.corr_pair_us = 1000.0 * tq / (double)nl;
    h->st.corr_timed_launches = nl;
    h->st.pairs_per_launch = (double)np / (double)nl;
    h->st.templates_per_launch = (double)nd / (double)nl;
  }
}

// ---- sharded norm_type=1 search: one contiguous angle range per rank, state merged by the
// caller's collective between the phases.
namespace {
Ctx shard_ctx(gisspa_handle* h) {
  return Ctx{h, h->stream, h->cfg.window_size, (long long)h->cfg.window_size * h->cfg.window_size,
             make_params(h->cfg, h->last_ctf)};
}

void shard_sync(gisspa_handle* h, const char* where) {
  GISSPA_CUDA(cudaStreamSynchronize(h->stream));
  unsigned flag = 0;
  GISSPA_CUDA(cudaMemcpy(&flag, h->dev_err.as<unsigned>(), sizeof(flag), cudaMemcpyDeviceToHost));
  if (flag) throw TimeoutError{where};
}
}  // namespace

void shard_begin(gisspa_handle* h, const float* d_img, int nx, int ny, const gisspa_ctf& ctf,
                 gisspa_shard_info* info) {
  h->last_ctf = ctf;
  h->last_W = 0;
  h->st = gisspa_stats{};
  h->n_samples = 0;
  h->n_seqs = 0;
  h->launch_index = 0;
  Ctx c = shard_ctx(h);
  unsigned* err = buf<unsigned>(h->dev_err, 1);
  GISSPA_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), c.s));
  norm_prepare(c, d_img, nx, ny, h->run);
  shard_sync(h, "shard_begin");
  info->n_pixels = h->run.npix;
  info->n_windows = h->run.W;
  info->n_angles = (int)h->run.angles.size();
  info->pick_mode = h->cfg.pick_mode;
}

void shard_sweep(gisspa_handle* h, int sweep, int a0, int a1) {
  Ctx c = shard_ctx(h);
  NormRun& r = h->run;
  if (sweep == 1)
    norm_sweep1(c, r, a0, a1);
  else
    norm_sweep2(c, r, a0, a1);
  h->st.pairs = r.pairs;
  shard_sync(h, "shard_sweep");
}

void shard_export(gisspa_handle* h, double* sum, double* sum_sq, long long* peak_key) {
  NormRun& r = h->run;
  cudaStream_t s = h->stream;
  GISSPA_CUDA(cudaMemcpyAsync(sum, r.args.S1, sizeof(double) * r.npix, cudaMemcpyDeviceToDevice, s));
  GISSPA_CUDA(cudaMemcpyAsync(sum_sq, r.args.S2, sizeof(double) * r.npix, cudaMemcpyDeviceToDevice, s));
  if (r.topk && peak_key) {
    peak_flip_kernel<<<ceil_div((long long)r.npix, 256), 256, 0, s>>>(
        r.args.peak, (long long)r.npix, reinterpret_cast<unsigned long long*>(peak_key));
    GISSPA_LAUNCH_CHECK();
  }
  shard_sync(h, "shard_export");
}

void shard_import(gisspa_handle* h, const double* sum, const double* sum_sq, const long long* peak_key) {
  Ctx c = shard_ctx(h);
  NormRun& r = h->run;
  GISSPA_CUDA(cudaMemcpyAsync(r.args.S1, sum, sizeof(double) * r.npix, cudaMemcpyDeviceToDevice, c.s));
  GISSPA_CUDA(cudaMemcpyAsync(r.args.S2, sum_sq, sizeof(double) * r.npix, cudaMemcpyDeviceToDevice, c.s));
  if (r.topk) {
    peak_flip_kernel<<<ceil_div((long long)r.npix, 256), 256, 0, c.s>>>(
        reinterpret_cast<const unsigned long long*>(peak_key), (long long)r.npix, r.args.peak);
    GISSPA_LAUNCH_CHECK();
  }
  norm_stats(c, r);
  shard_sync(h, "shard_import");
}

void shard_picks(gisspa_handle* h, std::vector<gisspa_pick>& out) {
  Ctx c = shard_ctx(h);
  NormRun& r = h->run;
  if (r.topk)
    topk_picks(c, r, out);
  else
    chunk_picks(r, out);
  shard_sync(h, "shard_picks");
}

int run_batch(gisspa_handle* h, int n, const float* const* images, const int* nx, const int* ny,
              const gisspa_ctf* ctfs, gisspa_pick* picks, size_t cap, size_t* offsets) {
  std::vector<gisspa_pick> all, one;
  offsets[0] = 0;
  gisspa_stats total{};
  h->next_dev = nullptr;
  // Micrographs alternate between two device buffers.  While micrograph i's first sweep runs
  // (norm_type=1), the host uploads micrograph i+1 into the other buffer on the side stream and
  // queues its LoadImage statistics (one thread, ~65 ms at 4096^2) there; search i+1 then starts
  // from them.  Buffer i+1 last held micrograph i-1, whose search has returned.
  gisspa::DevBuf* bufs[2] = {&h->img_in, &h->img_next};
  for (int i = 0; i < n; ++i) {
    one.clear();
    int st = guarded(h, [&] {
      GISSPA_CUDA(cudaSetDevice(h->device));
      gisspa::DevBuf& cur = *bufs[i & 1];
      const size_t bytes = sizeof(float) * (size_t)nx[i] * ny[i];
      if (h->next_dev == nullptr || h->next_dev != cur.as<float>()) {
        h->next_dev = nullptr;
        cur.ensure(bytes);
        GISSPA_CUDA(cudaMemcpyAsync(cur.as<float>(), images[i], bytes, cudaMemcpyHostToDevice, h->stream));
      }
      if (i + 1 < n && h->cfg.norm_type != 0) {
        h->after_sweep1 = [h, &bufs, i, images, nx, ny] {
          gisspa::DevBuf& nb = *bufs[(i + 1) & 1];
          const size_t b2 = sizeof(float) * (size_t)nx[i + 1] * ny[i + 1];
          float* dst = static_cast<float*>(nb.ensure(b2));
          float* st1 = buf<float>(h->stats_next, 4);
          double* scr = buf<double>(h->scratch_next, 16);
          GISSPA_CUDA(cudaMemcpyAsync(dst, images[i + 1], b2, cudaMemcpyHostToDevice, h->side));
          image_stats(dst, nx[i + 1], ny[i + 1], (h->cfg.quirks & GISSPA_QUIRK_OUTLIER_FP32_SERIAL) != 0, st1, scr,
                      h->side);
          GISSPA_CUDA(cudaEventRecord(h->ev_next, h->side));  // the next search waits on it
          h->next_dev = dst;
          h->next_nx = nx[i + 1];
          h->next_ny = ny[i + 1];
        };
      }
      run_search(h, cur.as<float>(), nx[i], ny[i], ctfs[i], one);
      h->after_sweep1 = nullptr;
    });
    if (st) {
      h->after_sweep1 = nullptr;
      h->next_dev = nullptr;
      return st;
    }
    total.ms_total += h->st.ms_total;
    total.ms_prep += h->st.ms_prep;
    total.ms_sweep1 += h->st.ms_sweep1;
    total.ms_sweep2 += h->st.ms_sweep2;
    total.ms_pick += h->st.ms_pick;
    total.pairs += h->st.pairs;
    total.kernel_launches += h->st.kernel_launches;
    total.candidates += h->st.candidates;
    total.pass_a_us += h->st.pass_a_us / n;
    total.pass_b_us += h->st.pass_b_us / n;
    total.pairs_per_launch += h->st.pairs_per_launch / n;
    total.templates_per_launch += h->st.templates_per_launch / n;
    total.pass_samples += h->st.pass_samples;
    total.graph_replays += h->st.graph_replays;
    total.window_size = h->st.window_size;
    total.rows_alive += h->st.rows_alive / n;
    total.pairs_alive += h->st.pairs_alive / n;
    total.pass_a_variant = h->st.pass_a_variant;
    total.pass_b_variant = h->st.pass_b_variant;
    all.insert(all.end(), one.begin(), one.end());
    offsets[i + 1] = all.size();
  }
  h->st = total;
  if (all.size() > cap) {
    h->err = "search_batch: " + std::to_string(all.size()) + " picks exceed capacity " + std::to_string(cap);
    return GISSPA_ERR_CAPACITY;
  }
  if (!all.empty()) std::memcpy(picks, all.data(), sizeof(gisspa_pick) * all.size());
  return GISSPA_OK;
}

}  // namespace gisspa
