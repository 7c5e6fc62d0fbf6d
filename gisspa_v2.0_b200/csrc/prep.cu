// prep.cu — template / micrograph / window preparation and per-angle rotation.
//
// Every step restates the reference kernel it replaces (cited per function).  The
// reference's amplitude/phase (AP) round trips are replaced by real scaling of
// the complex value, which keeps the phase; reductions are FP64; the CTF phase is
// evaluated in FP64.
#include <cmath>

#include "prep.cuh"

namespace gisspa {

DevParams make_params(const gisspa_config& c, const gisspa_ctf& ctf) {
  DevParams p{};
  p.apix = c.angpix; p.kk = c.kk; p.cs = c.cs; p.highres = c.highres; p.lowres = c.lowres;
  p.d_m = c.diameter; p.thresh = c.threshold; p.ehw = c.edge_half_width; p.ampconst = c.ampconst;
  p.a = c.a; p.b = c.b; p.b2 = c.b2; p.bf = c.bfactor; p.bf2 = c.bfactor2; p.bf3 = c.bfactor3;
  const double E = c.energy;
  p.lambda = 12.2639 / std::sqrt(E * 1000.0 + 0.97845 * E * E);
  p.dfu = -ctf.defocus + ctf.dfdiff;
  p.dfv = -ctf.defocus - ctf.dfdiff;
  p.dfdiff = ctf.dfdiff;
  p.dfang = ctf.dfang;
  return p;
}

namespace {

constexpr int kT = 256;

// CTF_AST (kernels.cu:290-317) in FP64.  mode 0: sign, 2: |v|, else v.
__device__ double ctf_ast(int x1, int y1, int nx, int ny, const DevParams& p, int mode) {
  y1 = x1 > nx / 2 ? ny - y1 : y1;
  x1 = min(x1, nx - x1);
  const double dx = x1;
  const double dy = y1 - ny / 2;
  const double ss = (dx * dx / ((double)nx * nx) + dy * dy / ((double)ny * ny)) / (p.apix * p.apix);
  const double ag = atan2((double)(y1 - ny / 2), (double)x1);
  const double df_ast = 0.5 * (p.dfu + p.dfv + 2.0 * p.dfdiff * cos(2.0 * (p.dfang * kRefPi / 180.0 - ag)));
  const double l3 = p.lambda * p.lambda * p.lambda;
  const double gamma = -2.0 * kRefPi * (p.cs * 2.5e6 * l3 * ss * ss + df_ast * 5000.0 * p.lambda * ss);
  double sg, cg;
  sincos(gamma, &sg, &cg);
  const double v = sqrt(1.0 - p.ampconst * p.ampconst) * sg + p.ampconst * cg;
  if (mode == 0) return v > 0 ? 1.0 : -1.0;
  if (mode == 2) return fabs(v);
  return v;
}

// Band-pass branch structure of apply_weighting_function (kernels.cu:262-275) and
// whiten_filter_weight_Img (kernels.cu:182-189); r is the integer shell index.
__device__ double band_factor(double r, double hi, double lo) {
  if (r < hi && r >= 0) return 1.0;
  if (r >= hi && r < hi + 8) return 0.5 * cos(kRefPi * (r - hi) / 16.0) + 0.5;
  if (r >= lo - 8 && r < lo && r >= 0) return 0.5 * cos(kRefPi * (lo - r) / 16.0) + 0.5;
  return 0.0;
}

template <typename Tv>
__device__ Tv warp_sum(Tv v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sum over the block; the result is valid in every thread.
template <typename Tv>
__device__ Tv block_sum(Tv v, Tv* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (ln == 0) sh[w] = v;
  __syncthreads();
  Tv r = 0;
  if (w == 0) {
    r = ln < (int)(blockDim.x >> 5) ? sh[ln] : Tv(0);
    r = warp_sum(r);
    if (ln == 0) sh[0] = r;
  }
  __syncthreads();
  return sh[0];
}

__global__ void tmpl_pad_kernel(const float* __restrict__ st, int nt, int tw, int th, int l, float2* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long L2 = (long long)l * l;
  if (i >= L2 * nt) return;
  const int n = (int)(i / L2);
  const int k = (int)(i - (long long)n * L2);
  const int x = k % l, y = k / l;
  const int sx = (l - tw) / 2, sy = (l - th) / 2;  // LoadTemplate (norm.cu:137-149)
  float v = 0.f;
  if (x >= sx && x < sx + tw && y >= sy && y < sy + th) v = st[(size_t)n * tw * th + (size_t)(y - sy) * tw + (x - sx)];
  out[i] = make_float2(v, 0.f);
}

// generate_mask + multiCount_dot + UpdateSigma + scale_each (kernels.cu:4-90, host norm.cu:194-280)
__global__ void tmpl_edge_normalise_kernel(float2* __restrict__ tb, int l) {
  __shared__ double sh[32];
  float2* t = tb + (size_t)blockIdx.x * l * l;
  const float rf = l / 2.f - 2.f;
  float up = 0.f, low = 0.f;
  if (rf > 1) {
    up = (rf + 1) * (rf + 1);
    low = (rf - 1) * (rf - 1);
  }
  double cnt = 0, dot = 0, s1 = 0, s2 = 0;
  const int L2 = l * l;
  for (int k = threadIdx.x; k < L2; k += blockDim.x) {
    const int x = k % l, y = k / l;
    const float rr = (float)((x - l / 2) * (x - l / 2) + (y - l / 2) * (y - l / 2));
    const double v = t[k].x;
    if (rr >= low && rr <= up) {
      cnt += 1;
      dot += v;
    }
    s1 += v;
    s2 += v * v;
  }
  cnt = block_sum(cnt, sh);
  dot = block_sum(dot, sh);
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  const double em = cnt != 0 ? dot / cnt : dot;
  const double mean = s1 / (double)L2;
  double sigma = sqrt(s2 / (double)L2 - mean * mean);
  if (sigma < 0 || !isfinite(sigma)) sigma = 0;
  if (sigma < 1e-8 && sigma > -1e-8) return;
  for (int k = threadIdx.x; k < L2; k += blockDim.x) t[k].x = (float)((t[k].x - em) / sigma);
}

// SQRSum_by_circle (kernels.cu:94-126): shared-memory histogram, one global merge per block.
__global__ void radial_power_kernel(const float2* __restrict__ F, int nx, int ny, double* __restrict__ ra,
                                    unsigned* __restrict__ rb, int nbins) {
  extern __shared__ unsigned char smraw[];
  double* hra = reinterpret_cast<double*>(smraw);
  unsigned* hrb = reinterpret_cast<unsigned*>(hra + nbins);
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
    hra[i] = 0.0;
    hrb[i] = 0u;
  }
  __syncthreads();
  const int b = blockIdx.y;
  const float2* G = F + (size_t)b * nx * ny;
  const int hx = nx / 2 + 1;
  const long long npix = (long long)hx * ny;
  const int L = max(nx, ny);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / hx), x = (int)(i - (long long)y * hx);
    const int r = shell_xy(x, y, nx, ny);
    if (r < L / 2 && r >= 0 && r < nbins) {
      const float2 g = G[(size_t)y * nx + x];
      atomicAdd(hra + r, (double)g.x * g.x + (double)g.y * g.y);
      if (b == 0) atomicAdd(hrb + r, 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
    if (hra[i] != 0.0) atomicAdd(ra + (size_t)b * nbins + i, hra[i]);
    if (b == 0 && hrb[i]) atomicAdd(rb + i, hrb[i]);
  }
}

__global__ void tmpl_whiten_kernel(float2* __restrict__ F, int batch, int l, const double* __restrict__ ra,
                                   const unsigned* __restrict__ rb, int nbins) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long L2 = (long long)l * l;
  if (i >= L2 * batch) return;
  const int b = (int)(i / L2);
  const int k = (int)(i - (long long)b * L2);
  const int x = k % l, y = k / l;
  const int r = shell_xy(x, y, l, l);
  if (r < l / 2 && r >= 0) {
    const double f = sqrt(ra[(size_t)b * nbins + r] / (double)rb[r]);
    const float2 v = F[i];
    F[i] = make_float2((float)(v.x / f), (float)(v.y / f));
  }
}

__global__ void mask_real_kernel(float2* __restrict__ d, int batch, int l, float d_m, float ehw) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long L2 = (long long)l * l;
  if (i >= L2 * batch) return;
  const int k = (int)(i % L2);
  const int x = k % l, y = k / l;
  const float dm = 1.5f * d_m;
  const float r = hypotf((float)(x - l / 2), (float)(y - l / 2));
  float v = d[i].x;
  if (r > dm / 2 + 2 * ehw) v = 0.f;
  else if (r >= dm / 2) v *= (float)(0.5 * cos(kRefPi * (r - dm / 2) / (2.0 * ehw)) + 0.5);
  d[i] = make_float2(v, 0.f);
}

__global__ void tmpl_weight_table_kernel(float* __restrict__ table, int l, DevParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= l * l) return;
  const int x = i % l, y = i / l;
  const double rf = hypot((double)min(y, l - y), (double)min(x, l - x));
  const int rr = shell_xy(x, y, l, l);
  const double hi = (double)l * p.apix / p.highres, lo = (double)l * p.apix / p.lowres;
  double w = band_factor(rr, hi, lo);
  const double ss = rf / (p.apix * l);
  if (rr < l / 2 && rr >= 0) {
    const double v = ctf_ast(x, (y + l / 2) % l, l, l, p, 2);
    const double signal = exp(p.bf * ss * ss + p.bf2 * ss + p.bf3) / (p.kk + 1);
    const double ncurve = exp(p.a * ss * ss + p.b * ss + p.b2) / signal;
    w *= v * sqrt(1.0 / (ncurve + p.kk * v * v));
  }
  table[i] = (float)w;
}

__global__ void apply_table_kernel(float2* __restrict__ F, int batch, int l, const float* __restrict__ table) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long L2 = (long long)l * l;
  if (i >= L2 * batch) return;
  const float w = table[i % L2];
  const float2 v = F[i];
  F[i] = make_float2(v.x * w, v.y * w);
}

__global__ void rms_normalise_kernel(float2* __restrict__ F, int l, double* __restrict__ factors) {
  __shared__ double sh[32];
  float2* G = F + (size_t)blockIdx.x * l * l;
  double s = 0, cnt = 0;
  const int hx = l / 2 + 1;
  for (int i = threadIdx.x; i < hx * l; i += blockDim.x) {
    const int y = i / hx, x = i - y * hx;
    const int r = shell_xy(x, y, l, l);
    if (r < l / 2 && r >= 0) {
      const float2 g = G[(size_t)y * l + x];
      s += (double)g.x * g.x + (double)g.y * g.y;
      cnt += 1;
    }
  }
  s = block_sum(s, sh);
  cnt = block_sum(cnt, sh);
  const double m = sqrt(s / (cnt * cnt));
  if (factors && threadIdx.x == 0) factors[blockIdx.x] = m;
  if (m == 0) return;
  const double inv = 1.0 / m;
  for (int i = threadIdx.x; i < l * l; i += blockDim.x) {
    const float2 g = G[i];
    G[i] = make_float2((float)(g.x * inv), (float)(g.y * inv));
  }
}

__global__ void real_part_kernel(const float2* __restrict__ in, float* __restrict__ out, long long n, float scale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i].x * scale;
}
__global__ void to_complex_kernel(const float* __restrict__ in, float2* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float2(in[i], 0.f);
}

// LoadImage mean/sigma exactly as the reference's serial FP32 loop (norm.cu:157-167):
// warps 1.. compute the per-element terms of the next tile while lane 0 of warp 0
// accumulates the current tile in the original order.  IEEE intrinsics keep the
// compiler from contracting or reordering.
constexpr int kStatTile = 2048;
__global__ void __launch_bounds__(1024) stats_serial_kernel(const float* __restrict__ img, long long n, float fnx,
                                                            float fny, float* __restrict__ stats) {
  __shared__ float t1[2][kStatTile], t2[2][kStatTile];
  float sum = 0.f, sum_s2 = 0.f;
  const long long ntiles = (n + kStatTile - 1) / kStatTile;
  const int w = threadIdx.x >> 5;
  // prologue: fill tile 0
  for (int i = threadIdx.x; i < kStatTile; i += blockDim.x) {
    if (i < n) {
      const float cur = img[i];
      t1[0][i] = __fdiv_rn(__fdiv_rn(cur, fnx), fny);
      t2[0][i] = __fdiv_rn(__fdiv_rn(__fmul_rn(cur, cur), fnx), fny);
    }
  }
  __syncthreads();
  for (long long tI = 0; tI < ntiles; ++tI) {
    const int cb = (int)(tI & 1);
    if (w == 0) {
      if (threadIdx.x == 0) {
        const long long base = tI * kStatTile;
        const int cnt = (int)min((long long)kStatTile, n - base);
        for (int i = 0; i < cnt; ++i) {
          sum = __fadd_rn(sum, t1[cb][i]);
          sum_s2 = __fadd_rn(sum_s2, t2[cb][i]);
        }
      }
    } else if (tI + 1 < ntiles) {
      const long long base = (tI + 1) * kStatTile;
      for (int i = threadIdx.x - 32; i < kStatTile; i += blockDim.x - 32) {
        if (base + i < n) {
          const float cur = img[base + i];
          t1[cb ^ 1][i] = __fdiv_rn(__fdiv_rn(cur, fnx), fny);
          t2[cb ^ 1][i] = __fdiv_rn(__fdiv_rn(__fmul_rn(cur, cur), fnx), fny);
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const float avg = sum;
    const float var = __fsqrt_rn(__fsub_rn(sum_s2, __fmul_rn(avg, avg)));
    const float up = __fadd_rn(avg, __fmul_rn(6.f, var));
    const float lo = __fsub_rn(avg, __fmul_rn(6.f, var));
    stats[0] = avg;
    stats[1] = (float)(int)up;  // int truncation (norm.cu:166-167)
    stats[2] = (float)(int)lo;
    stats[3] = (sum_s2 > __fmul_rn(avg, avg)) ? 1.f : 0.f;
    if (!(up == up) || !(lo == lo)) stats[3] = 0.f;
  }
}

__global__ void stats_fp64_kernel(const float* __restrict__ img, long long n, double* __restrict__ acc) {
  __shared__ double sh[32];
  double s = 0, s2 = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = img[i];
    s += v;
    s2 += v * v;
  }
  s = block_sum(s, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    atomicAdd(acc, s);
    atomicAdd(acc + 1, s2);
  }
}
__global__ void stats_fp64_finish(const double* __restrict__ acc, long long n, float* __restrict__ stats) {
  const double avg = acc[0] / n, var = sqrt(acc[1] / n - avg * avg);
  stats[0] = (float)avg;
  stats[1] = (float)(int)(avg + 6 * var);
  stats[2] = (float)(int)(avg - 6 * var);
  stats[3] = (acc[1] / n > avg * avg) ? 1.f : 0.f;
}

__global__ void image_load_kernel(const float* __restrict__ img, long long n, const float* __restrict__ stats,
                                  int clamp, int invert, float2* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v = img[i];
  if (clamp && stats[3] != 0.f && (v > stats[1] || v < stats[2])) v = stats[0];
  if (invert) v = -v;
  out[i] = make_float2(v, 0.f);
}

__global__ void phase_flip_kernel(float2* __restrict__ G, int nx, int ny, DevParams p) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = (int)(i % nx), y = (int)(i / nx);
  const float s = (float)ctf_ast(x, (y + ny / 2) % ny, nx, ny, p, 0);
  const float2 g = G[i];
  G[i] = make_float2(g.x * s, g.y * s);
}

__global__ void image_filter_kernel(float2* __restrict__ G, int nx, int ny, DevParams p, const double* __restrict__ ra,
                                    const unsigned* __restrict__ rb, int nbins, int zero_dc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nx * ny) return;
  const int x = (int)(i % nx), y = (int)(i / nx);
  const double dx = min(x, nx - x), dy = min(y, ny - y);
  const int r = shell_xy(x, y, nx, ny);
  const double ss = sqrt((dx * dx / ((double)nx * nx) + dy * dy / ((double)ny * ny)) / (p.apix * p.apix));
  const int L = max(nx, ny);
  double f = 1.0, v = 0.0, signal = 0.0, ncurve = 0.0;
  if (r < L / 2 && r >= 0) {
    v = ctf_ast(x, (y + ny / 2) % ny, nx, ny, p, 2);
    signal = exp(p.bf * ss * ss + p.bf2 * ss + p.bf3);
    ncurve = exp(p.a * ss * ss + p.b * ss + p.b2);
    f *= sqrt((signal * v * v + ncurve) / signal) / sqrt(ra[r] / (double)rb[r]);
    if (r > L * p.apix / 6) f *= exp(-100 * ss * ss);
  }
  f *= band_factor(r, (double)L * p.apix / p.highres, (double)L * p.apix / p.lowres);
  if (r < L / 2 && r >= 0) {
    signal /= (p.kk + 1);
    ncurve /= signal;
    f *= sqrt(1.0 / (ncurve + p.kk * v * v));
  }
  if (zero_dc && i == 0) f = 0.0;
  const float2 g = G[i];
  G[i] = make_float2((float)(g.x * f), (float)(g.y * f));
}

__global__ void gather_windows_kernel(const float* __restrict__ img, int nx, int ny, const int* __restrict__ offx,
                                      const int* __restrict__ offy, int bx, int l, float2* __restrict__ out) {
  const int b = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= l * l) return;
  const int x = k % l, y = k / l;
  const int ox = offx[b % bx] + x, oy = offy[b / bx] + y;
  float v = 0.f;
  if (ox < nx && oy < ny) v = img[(size_t)oy * nx + ox];
  out[(size_t)b * l * l + k] = make_float2(v, 0.f);
}

__global__ void rotate_kernel(const float* __restrict__ in, int l, float cose, float sine, int mask, float d_m,
                              float ehw, float2* __restrict__ out, double* __restrict__ sums,
                              const AngleState* __restrict__ st) {
  __shared__ double sh[32];
  if (st) {
    cose = st->cose;
    sine = st->sine;
  }
  const int n = blockIdx.y;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const float* src = in + (size_t)n * l * l;
  float res = 0.f;
  if (id < l * l) {
    const int i = id % l, j = id / l;
    const float x = (float)(i - l / 2), y = (float)(j - l / 2);
    // same float expression as rotate_subIMG (kernels.cu:554-555)
    const float x2 = (cose * x + sine * y) + l / 2;
    const float y2 = (-sine * x + cose * y) + l / 2;
    if (!(x2 < 0 || x2 > l - 1.0f || y2 < 0 || y2 > l - 1.0f)) {
      const int ii = (int)floorf(x2), jj = (int)floorf(y2);
      int k0 = ii + jj * l, k1 = k0 + 1, k2 = k0 + l + 1, k3 = k0 + l;
      if (ii == l - 1) { k1 -= 1; k2 -= 1; }
      if (jj == l - 1) { k2 -= l; k3 -= l; }
      const float t = x2 - ii, u = y2 - jj, tt = 1.0f - t, uu = 1.0f - u;
      res = src[k0] * tt * uu + src[k1] * t * uu + src[k2] * t * u + src[k3] * tt * u;
    }
    if (mask) {
      const float dm = 1.5f * d_m;
      const float r = hypotf((float)(i - l / 2), (float)(j - l / 2));
      if (r > dm / 2 + 2 * ehw) res = 0.f;
      else if (r >= dm / 2) res *= (float)(0.5 * cos(kRefPi * (r - dm / 2) / (2.0 * ehw)) + 0.5);
    }
    out[(size_t)n * l * l + id] = make_float2(res, 0.f);
  }
  if (sums) {
    const double s1 = block_sum((double)res, sh);
    const double s2 = block_sum((double)res * res, sh);
    if (threadIdx.x == 0) {
      atomicAdd(sums + 2 * n, s1);
      atomicAdd(sums + 2 * n + 1, s2);
    }
  }
}

template <typename SPEC>
__global__ void finalize_spectra_kernel(const float2* __restrict__ X, int l, const double* __restrict__ sums,
                                        typename SPEC::T* __restrict__ out, double base) {
  const int n = blockIdx.y;
  const long long per = (long long)(l / 2 + 1) * l;
  const double L2 = (double)l * l;
  double sc = base;
  if (sums) {
    const double mean = sums[2 * n] / L2;
    const double var = sums[2 * n + 1] / L2 - mean * mean;
    if (var != 0) sc = base / sqrt(var);
  }
  const float fs = (float)sc;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < per; k += (long long)gridDim.x * blockDim.x) {
    float2 v = X[(size_t)n * per + k];
    v = make_float2(v.x * fs, v.y * fs);
    if (sums && k == 0) v = make_float2(0.f, 0.f);  // mean subtracted: DC is exactly zero
    out[(size_t)n * per + k] = SPEC::pack(v);
  }
}

__global__ void scale_batch_kernel(float2* __restrict__ F, long long per, const double* __restrict__ f) {
  const int b = blockIdx.y;
  const float s = (float)f[b];
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < per; k += (long long)gridDim.x * blockDim.x) {
    float2 v = F[(size_t)b * per + k];
    F[(size_t)b * per + k] = make_float2(v.x * s, v.y * s);
  }
}

}  // namespace

void tmpl_pad(const float* stack, int nt, int tw, int th, int l, float2* out, cudaStream_t s) {
  const long long n = (long long)l * l * nt;
  tmpl_pad_kernel<<<ceil_div(n, kT), kT, 0, s>>>(stack, nt, tw, th, l, out);
  GISSPA_LAUNCH_CHECK();
}

void tmpl_edge_normalise(float2* tb, int nt, int l, double*, cudaStream_t s) {
  tmpl_edge_normalise_kernel<<<nt, 512, 0, s>>>(tb, l);
  GISSPA_LAUNCH_CHECK();
}

void radial_power(const float2* F, int batch, int nx, int ny, double* ra, unsigned* rb, int nbins, cudaStream_t s) {
  GISSPA_CUDA(cudaMemsetAsync(ra, 0, sizeof(double) * (size_t)batch * nbins, s));
  GISSPA_CUDA(cudaMemsetAsync(rb, 0, sizeof(unsigned) * (size_t)nbins, s));
  const long long npix = (long long)(nx / 2 + 1) * ny;
  const int gx = std::max(1, std::min(ceil_div(npix, kT * 16), 2048));
  const size_t smem = (sizeof(double) + sizeof(unsigned)) * (size_t)nbins;
  if (smem > 48 * 1024)
    GISSPA_CUDA(cudaFuncSetAttribute(radial_power_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  radial_power_kernel<<<dim3(gx, batch), kT, smem, s>>>(F, nx, ny, ra, rb, nbins);
  GISSPA_LAUNCH_CHECK();
}

void tmpl_whiten(float2* F, int batch, int l, const double* ra, const unsigned* rb, int nbins, cudaStream_t s) {
  const long long n = (long long)l * l * batch;
  tmpl_whiten_kernel<<<ceil_div(n, kT), kT, 0, s>>>(F, batch, l, ra, rb, nbins);
  GISSPA_LAUNCH_CHECK();
}

void mask_real(float2* data, int batch, int l, float d_m, float ehw, cudaStream_t s) {
  const long long n = (long long)l * l * batch;
  mask_real_kernel<<<ceil_div(n, kT), kT, 0, s>>>(data, batch, l, d_m, ehw);
  GISSPA_LAUNCH_CHECK();
}

void tmpl_weight_table(float* table, int l, const DevParams& p, cudaStream_t s) {
  tmpl_weight_table_kernel<<<ceil_div((long long)l * l, kT), kT, 0, s>>>(table, l, p);
  GISSPA_LAUNCH_CHECK();
}

void apply_table(float2* F, int batch, int l, const float* table, cudaStream_t s) {
  const long long n = (long long)l * l * batch;
  apply_table_kernel<<<ceil_div(n, kT), kT, 0, s>>>(F, batch, l, table);
  GISSPA_LAUNCH_CHECK();
}

void rms_normalise(float2* F, int batch, int l, double* factors, cudaStream_t s) {
  rms_normalise_kernel<<<batch, 512, 0, s>>>(F, l, factors);
  GISSPA_LAUNCH_CHECK();
}

void real_part(const float2* in, float* out, long long n, float scale, cudaStream_t s) {
  real_part_kernel<<<ceil_div(n, kT), kT, 0, s>>>(in, out, n, scale);
  GISSPA_LAUNCH_CHECK();
}

void to_complex(const float* in, float2* out, long long n, cudaStream_t s) {
  to_complex_kernel<<<ceil_div(n, kT), kT, 0, s>>>(in, out, n);
  GISSPA_LAUNCH_CHECK();
}

void image_stats(const float* img, int nx, int ny, bool fp32_serial, float* stats, double* scratch, cudaStream_t s) {
  const long long n = (long long)nx * ny;
  if (fp32_serial) {
    stats_serial_kernel<<<1, 1024, 0, s>>>(img, n, (float)nx, (float)ny, stats);
    GISSPA_LAUNCH_CHECK();
  } else {
    GISSPA_CUDA(cudaMemsetAsync(scratch, 0, 2 * sizeof(double), s));
    stats_fp64_kernel<<<std::min(ceil_div(n, kT), 1184), kT, 0, s>>>(img, n, scratch);
    GISSPA_LAUNCH_CHECK();
    stats_fp64_finish<<<1, 1, 0, s>>>(scratch, n, stats);
    GISSPA_LAUNCH_CHECK();
  }
}

void image_load(const float* img, long long n, const float* stats, bool clamp, bool invert, float2* out, cudaStream_t s) {
  image_load_kernel<<<ceil_div(n, kT), kT, 0, s>>>(img, n, stats, clamp ? 1 : 0, invert ? 1 : 0, out);
  GISSPA_LAUNCH_CHECK();
}

void phase_flip(float2* G, int nx, int ny, const DevParams& p, cudaStream_t s) {
  phase_flip_kernel<<<ceil_div((long long)nx * ny, kT), kT, 0, s>>>(G, nx, ny, p);
  GISSPA_LAUNCH_CHECK();
}

void image_filter(float2* G, int nx, int ny, const DevParams& p, const double* ra, const unsigned* rb, int nbins,
                  bool zero_dc, cudaStream_t s) {
  image_filter_kernel<<<ceil_div((long long)nx * ny, kT), kT, 0, s>>>(G, nx, ny, p, ra, rb, nbins, zero_dc ? 1 : 0);
  GISSPA_LAUNCH_CHECK();
}

void gather_windows(const float* img, int nx, int ny, const int* offx, const int* offy, int bx, int nwin, int l,
                    float2* out, cudaStream_t s) {
  gather_windows_kernel<<<dim3(ceil_div((long long)l * l, kT), nwin), kT, 0, s>>>(img, nx, ny, offx, offy, bx, l, out);
  GISSPA_LAUNCH_CHECK();
}

void rotate_batch(const float* in, int n, int l, float cose, float sine, bool mask, float d_m, float ehw, float2* out,
                  double* sums, cudaStream_t s, const AngleState* st) {
  if (sums) GISSPA_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * 2 * n, s));
  rotate_kernel<<<dim3(ceil_div((long long)l * l, kT), n), kT, 0, s>>>(in, l, cose, sine, mask ? 1 : 0, d_m, ehw, out,
                                                                       sums, st);
  GISSPA_LAUNCH_CHECK();
}

void finalize_spectra(const float2* X, int n, int l, const double* sums, int spec, void* out, double base,
                      cudaStream_t s) {
  const long long per = (long long)(l / 2 + 1) * l;
  dim3 grid(std::min(ceil_div(per, kT), 512), n);
  switch (spec) {
    case GISSPA_SPEC_FP32:
      finalize_spectra_kernel<SpecFp32><<<grid, kT, 0, s>>>(X, l, sums, static_cast<float2*>(out), base);
      break;
    case GISSPA_SPEC_FP16:
      finalize_spectra_kernel<SpecFp16><<<grid, kT, 0, s>>>(X, l, sums, static_cast<__half2*>(out), base);
      break;
    default:
      finalize_spectra_kernel<SpecBf16><<<grid, kT, 0, s>>>(X, l, sums, static_cast<__nv_bfloat162*>(out), base);
      break;
  }
  GISSPA_LAUNCH_CHECK();
}

void scale_batch(float2* F, int batch, long long per, const double* factors, cudaStream_t s) {
  scale_batch_kernel<<<dim3(std::min(ceil_div(per, kT), 512), batch), kT, 0, s>>>(F, per, factors);
  GISSPA_LAUNCH_CHECK();
}

}  // namespace gisspa
