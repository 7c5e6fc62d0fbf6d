// adjoint.cu — gradient of a pick's normalised correlation score.
//
// For a pick (window b, template t, pixel p, search angle theta) the search's score is
//   z = (c - mu) / sigma,   c = (1/L^2) sum_y W_b(y + p + L/2) n(y)
// with W_b the filtered window (IFFT of its normalised spectrum) and n the rotated, masked,
// mean/variance-normalised template (RotateTemplate, norm.cu:479-521; compute_corner_CCG +
// IFFT, kernels.cu:645-678).  The continuous extension differentiated here:
//   * sub-pixel shift (dx, dy): the template is sampled at y - d (on the periodic grid this is
//     the Fourier shift of the window by +d); mask and normalisation follow the shifted samples;
//   * theta: through the bilinear rotation's sampling coordinates (piecewise linear, defined
//     almost everywhere);
//   * dfu, dfv, dfang: through the template-side |CTF| x SSNR weight (apply_weighting_function,
//     kernels.cu:243-288).  The RMS normalisation that follows it only scales the template, to
//     which n (and so z) is invariant, so it drops out.  The micrograph's preprocessing (phase
//     flip, whitening) is held at the search's CTF: the sign flip has zero derivative almost
//     everywhere.
//   mu and sigma (the per-pixel statistics over all templates and angles) are held fixed at the
//   pick pixel.  Everything is recomputed from the prepared templates and the preprocessed
//   micrograph; no spectrum of the search is stored.
#include <cmath>
#include <type_traits>

#include "../../include/gisspa.h"
#include "adjoint.cuh"

namespace gisspa {
namespace {

constexpr int kGT = 256;
constexpr int kSums = 21;

__device__ double ctf_value_dgamma(int x1, int y1, int nx, int ny, const DevParams& p, double* v_out,
                                   double* dgamma_dfast, double* dfast) {
  // CTF_AST (kernels.cu:290-317) with its derivative pieces
  y1 = x1 > nx / 2 ? ny - y1 : y1;
  x1 = min(x1, nx - x1);
  const double dx = x1, dy = y1 - ny / 2;
  const double ss = (dx * dx / ((double)nx * nx) + dy * dy / ((double)ny * ny)) / (p.apix * p.apix);
  const double ag = atan2((double)(y1 - ny / 2), (double)x1);
  const double phi = p.dfang * kRefPi / 180.0 - ag;
  const double df_ast = 0.5 * (p.dfu + p.dfv + 2.0 * p.dfdiff * cos(2.0 * phi));
  const double l3 = p.lambda * p.lambda * p.lambda;
  const double gamma = -2.0 * kRefPi * (p.cs * 2.5e6 * l3 * ss * ss + df_ast * 5000.0 * p.lambda * ss);
  double sg, cg;
  sincos(gamma, &sg, &cg);
  const double A = p.ampconst, B = sqrt(1.0 - A * A);
  *v_out = B * sg + A * cg;
  *dgamma_dfast = -2.0 * kRefPi * 5000.0 * p.lambda * ss;
  // d df_ast / d(dfu, dfv, dfang), with dfdiff = (dfu - dfv) / 2
  const double c2 = cos(2.0 * phi), s2 = sin(2.0 * phi);
  dfast[0] = 0.5 + 0.5 * c2;
  dfast[1] = 0.5 - 0.5 * c2;
  dfast[2] = -(p.dfu - p.dfv) * s2 * (kRefPi / 180.0);
  return B * cg - A * sg;  // dv / dgamma
}

__device__ double band_factor_d(double r, double hi, double lo) {
  if (r < hi && r >= 0) return 1.0;
  if (r >= hi && r < hi + 8) return 0.5 * cos(kRefPi * (r - hi) / 16.0) + 0.5;
  if (r >= lo - 8 && r < lo && r >= 0) return 0.5 * cos(kRefPi * (lo - r) / 16.0) + 0.5;
  return 0.0;
}

// dW/dpsi for the template weight W = band x |v| / sqrt(N + kk v^2) on valid shells.
__global__ void ctf_dweight_kernel(float* __restrict__ dtab, int l, DevParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= l * l) return;
  const int x = i % l, y = i / l;
  const double rf = hypot((double)min(y, l - y), (double)min(x, l - x));
  const int rr = shell_xy(x, y, l, l);
  double d[3] = {0, 0, 0};
  if (rr < l / 2 && rr >= 0) {
    const double band = band_factor_d(rr, (double)l * p.apix / p.highres, (double)l * p.apix / p.lowres);
    if (band != 0.0) {
      double v, dg, dfa[3];
      const double dvdg = ctf_value_dgamma(x, (y + l / 2) % l, l, l, p, &v, &dg, dfa);
      const double ss = rf / (p.apix * l);
      const double signal = exp(p.bf * ss * ss + p.bf2 * ss + p.bf3) / (p.kk + 1);
      const double ncurve = exp(p.a * ss * ss + p.b * ss + p.b2) / signal;
      const double den = ncurve + p.kk * v * v;
      // d/dv [ |v| (N + kk v^2)^-1/2 ] = sign(v) N (N + kk v^2)^-3/2
      const double dfdv = (v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0)) * ncurve / (den * sqrt(den));
      for (int k = 0; k < 3; ++k) d[k] = band * dfdv * dvdg * dg * dfa[k];
    }
  }
  for (int k = 0; k < 3; ++k) dtab[(size_t)k * l * l + i] = (float)d[k];
}

__global__ void scale_by_table_kernel(const float2* __restrict__ F, const float* __restrict__ tab,
                                      const double* __restrict__ m, int nt, int l, float2* __restrict__ out) {
  const long long L2 = (long long)l * l;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L2 * nt) return;
  const int t = (int)(i / L2);
  const double mt = m[t];
  const float s = (float)(mt != 0 ? (double)tab[i % L2] / mt : (double)tab[i % L2]);
  const float2 v = F[i];
  out[i] = make_float2(v.x * s, v.y * s);
}

__global__ void window_sum_kernel(const float* __restrict__ img, int nx, int ny, const int* __restrict__ offx,
                                  const int* __restrict__ offy, int bx, int l, const double* __restrict__ win_m,
                                  double* __restrict__ out) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  double s = 0;
  for (int k = threadIdx.x; k < l * l; k += blockDim.x) {
    const int x = offx[b % bx] + k % l, y = offy[b / bx] + k / l;
    if (x < nx && y < ny) s += img[(size_t)y * nx + x];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    const double m = win_m[b];
    out[b] = t / ((double)l * l * (m != 0 ? m : 1.0));
  }
}

// Bilinear sample with the reference's boundary rules (rotate_subIMG kernels.cu:557-579) and
// its derivative in the sampling coordinates.
__device__ __forceinline__ void bilinear(int l, double x2, double y2, int& k0, int& k1,
                                         int& k2, int& k3, double& t, double& u, bool& inside) {
  inside = !(x2 < 0 || x2 > l - 1.0 || y2 < 0 || y2 > l - 1.0);
  if (!inside) return;
  const int ii = (int)floor(x2), jj = (int)floor(y2);
  k0 = ii + jj * l;
  k1 = k0 + 1;
  k2 = k0 + l + 1;
  k3 = k0 + l;
  if (ii == l - 1) {
    k1 -= 1;
    k2 -= 1;
  }
  if (jj == l - 1) {
    k2 -= l;
    k3 -= l;
  }
  t = x2 - ii;
  u = y2 - jj;
}

__device__ __forceinline__ double to_d(float v) { return (double)v; }
__device__ __forceinline__ double to_d(__half v) { return (double)__half2float(v); }
__device__ __forceinline__ double to_d(__nv_bfloat16 v) { return (double)__bfloat162float(v); }

// Largest |value| of in[0, n), as the bits of a non-negative float (ordered like the value),
// folded into *out.
__global__ void abs_max_kernel(const float* __restrict__ in, long long n, unsigned* __restrict__ out) {
  unsigned m = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fabsf(in[i])));
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Rounds to V.  FP16 has five exponent bits: the unnormalised real-space templates and their CTF
// derivatives exceed its range, so every value is first scaled by one power of two that brings
// the largest (*absmax, over both arrays) to [2^13, 2^14).  A common factor leaves the
// normalised score and all its derivatives unchanged (the score is invariant to the template's
// scale), and a power of two adds no rounding.  BF16 keeps FP32's exponent range (absmax null).
template <typename V>
__global__ void round_kernel(const float* __restrict__ in, long long n, const unsigned* __restrict__ absmax,
                             V* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float scale = 1.f;
  if (absmax) {
    const float m = __uint_as_float(*absmax);
    if (m > 0.f && isfinite(m)) scale = ldexpf(1.f, max(-120, min(120, 13 - ilogbf(m))));
  }
  if constexpr (std::is_same<V, __half>::value)
    out[i] = __float2half_rn(in[i] * scale);
  else
    out[i] = __float2bfloat16_rn(in[i] * scale);
}

// V: storage type of the prepared templates and their CTF derivatives (float, __half or
// __nv_bfloat16); every sum is FP64 whatever the storage.
template <typename V>
__global__ void __launch_bounds__(kGT) score_grad_kernel(GradArgs g, const V* __restrict__ prep,
                                                         const V* __restrict__ dprep,
                                                         const GradPick* __restrict__ picks, float* __restrict__ out) {
  __shared__ double sh[kSums][kGT / 32];
  const GradPick pk = picks[blockIdx.x];
  const int L = g.L;
  const double L2 = (double)L * L;
  const double th = (double)pk.theta * kRefPi / 180.0;
  const double cs = cos(th), sn = sin(th);
  const double dm = 1.5 * g.d_m, r_in = dm / 2, r_out = dm / 2 + 2 * g.ehw;
  const V* P = prep + (size_t)pk.n * L * L;
  const V* D0 = dprep + (size_t)pk.n * L * L;
  const size_t dstride = (size_t)g.nt * L * L;
  const int wx0 = g.offx[pk.b % g.bx], wy0 = g.offy[pk.b / g.bx];
  const double wscale = 1.0 / (L2 * (g.win_m[pk.b] != 0 ? g.win_m[pk.b] : 1.0));
  const double cx = L / 2 + (double)pk.dx, cy = L / 2 + (double)pk.dy;
  const int x_lo = max(0, (int)floor(cx - r_out) - 1), x_hi = min(L - 1, (int)ceil(cx + r_out) + 1);
  const int y_lo = max(0, (int)floor(cy - r_out) - 1), y_hi = min(L - 1, (int)ceil(cy + r_out) + 1);
  const int bw = x_hi - x_lo + 1, bh = y_hi - y_lo + 1;
  double acc[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k) acc[k] = 0.0;
  for (int idx = threadIdx.x; idx < bw * bh; idx += blockDim.x) {
    const int X = x_lo + idx % bw, Y = y_lo + idx / bw;
    const double ux = X - cx, uy = Y - cy;
    const double r = sqrt(ux * ux + uy * uy);
    if (r > r_out) continue;
    double m = 1.0, dmdr = 0.0;
    if (r >= r_in) {
      const double arg = kRefPi * (r - r_in) / (2.0 * g.ehw);
      m = 0.5 * cos(arg) + 0.5;
      dmdr = -0.5 * sin(arg) * kRefPi / (2.0 * g.ehw);
    }
    const double x2 = cs * ux + sn * uy + L / 2, y2 = -sn * ux + cs * uy + L / 2;
    int k0 = 0, k1 = 0, k2 = 0, k3 = 0;
    double t = 0, u = 0;
    bool inside;
    bilinear(L, x2, y2, k0, k1, k2, k3, t, u, inside);
    double R = 0, Rx = 0, Ry = 0, Dv[3] = {0, 0, 0};
    if (inside) {
      const double p0 = to_d(P[k0]), p1 = to_d(P[k1]), p2 = to_d(P[k2]), p3 = to_d(P[k3]);
      R = p0 * (1 - t) * (1 - u) + p1 * t * (1 - u) + p2 * t * u + p3 * (1 - t) * u;
      Rx = (1 - u) * (p1 - p0) + u * (p2 - p3);
      Ry = (1 - t) * (p3 - p0) + t * (p2 - p1);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const V* Dq = D0 + q * dstride;
        Dv[q] = to_d(Dq[k0]) * (1 - t) * (1 - u) + to_d(Dq[k1]) * t * (1 - u) + to_d(Dq[k2]) * t * u +
                to_d(Dq[k3]) * (1 - t) * u;
      }
    }
    const double a = m * R;
    const double drx = r > 0 ? -ux / r : 0.0, dry = r > 0 ? -uy / r : 0.0;
    double da[6];
    da[0] = dmdr * drx * R + m * (Rx * (-cs) + Ry * sn);
    da[1] = dmdr * dry * R + m * (Rx * (-sn) + Ry * (-cs));
    da[2] = m * (Rx * (-sn * ux + cs * uy) + Ry * (-cs * ux - sn * uy)) * (kRefPi / 180.0);
    da[3] = m * Dv[0];
    da[4] = m * Dv[1];
    da[5] = m * Dv[2];
    // window sample at the circularly shifted position (zero lag at L/2)
    const int wxl = (X + pk.px + L / 2) & (L - 1), wyl = (Y + pk.py + L / 2) & (L - 1);
    const int ix = wx0 + wxl, iy = wy0 + wyl;
    const double w = (ix < g.nx && iy < g.ny) ? (double)g.img[(size_t)iy * g.nx + ix] * wscale : 0.0;
    acc[0] += a;
    acc[1] += a * a;
    acc[2] += w * a;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      acc[3 + q] += da[q];
      acc[9 + q] += a * da[q];
      acc[15 + q] += w * da[q];
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kSums; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double S[kSums];
    for (int k = 0; k < kSums; ++k) {
      S[k] = 0;
      for (int w = 0; w < kGT / 32; ++w) S[k] += sh[k][w];
    }
    const double Sw = g.win_sum[pk.b];
    const double mean = S[0] / L2, var = S[1] / L2 - mean * mean, sd = sqrt(var);
    const double num = S[2] - mean * Sw;
    const double c = num / (L2 * sd);
    const float2 ms = g.musig[(size_t)pk.b * L * L + (size_t)pk.py * L + pk.px];
    float* o = out + (size_t)blockIdx.x * 7;
    o[0] = (float)((c - ms.x) * ms.y);
    for (int q = 0; q < 6; ++q) {
      const double dmean = S[3 + q] / L2;
      const double dvar = 2.0 * S[9 + q] / L2 - 2.0 * mean * dmean;
      const double dsd = dvar / (2.0 * sd);
      const double dnum = S[15 + q] - dmean * Sw;
      const double dc = (dnum * sd - num * dsd) / (L2 * sd * sd);
      o[1 + q] = (float)(dc * ms.y);
    }
  }
}

}  // namespace

void ctf_dweight(float* dtab, int l, const DevParams& p, cudaStream_t s) {
  ctf_dweight_kernel<<<ceil_div((long long)l * l, 256), 256, 0, s>>>(dtab, l, p);
  GISSPA_LAUNCH_CHECK();
}

void scale_by_table(const float2* F, const float* tab, const double* m, int nt, int l, float2* out, cudaStream_t s) {
  scale_by_table_kernel<<<ceil_div((long long)l * l * nt, 256), 256, 0, s>>>(F, tab, m, nt, l, out);
  GISSPA_LAUNCH_CHECK();
}

void window_sums(const float* img, int nx, int ny, const int* offx, const int* offy, int bx, int nwin, int l,
                 const double* win_m, double* out, cudaStream_t s) {
  window_sum_kernel<<<nwin, 256, 0, s>>>(img, nx, ny, offx, offy, bx, l, win_m, out);
  GISSPA_LAUNCH_CHECK();
}

void round_templates(const float* prep, long long n1, const float* dprep, long long n2, int precision,
                     unsigned* absmax, void* out1, void* out2, cudaStream_t s) {
  if (precision == GISSPA_SPEC_FP16) {
    GISSPA_CUDA(cudaMemsetAsync(absmax, 0, sizeof(unsigned), s));
    abs_max_kernel<<<4 * 148, 256, 0, s>>>(prep, n1, absmax);
    GISSPA_LAUNCH_CHECK();
    abs_max_kernel<<<4 * 148, 256, 0, s>>>(dprep, n2, absmax);
    GISSPA_LAUNCH_CHECK();
    round_kernel<__half><<<ceil_div(n1, 256), 256, 0, s>>>(prep, n1, absmax, static_cast<__half*>(out1));
    GISSPA_LAUNCH_CHECK();
    round_kernel<__half><<<ceil_div(n2, 256), 256, 0, s>>>(dprep, n2, absmax, static_cast<__half*>(out2));
  } else {
    round_kernel<__nv_bfloat16><<<ceil_div(n1, 256), 256, 0, s>>>(prep, n1, nullptr,
                                                                  static_cast<__nv_bfloat16*>(out1));
    GISSPA_LAUNCH_CHECK();
    round_kernel<__nv_bfloat16><<<ceil_div(n2, 256), 256, 0, s>>>(dprep, n2, nullptr,
                                                                  static_cast<__nv_bfloat16*>(out2));
  }
  GISSPA_LAUNCH_CHECK();
}

void score_grads(const GradArgs& g, const GradPick* picks, int n, float* out, cudaStream_t s) {
  if (n <= 0) return;
  if (g.precision == GISSPA_SPEC_FP16)
    score_grad_kernel<__half><<<n, kGT, 0, s>>>(g, static_cast<const __half*>(g.prep_lp),
                                                 static_cast<const __half*>(g.dprep_lp), picks, out);
  else if (g.precision == GISSPA_SPEC_BF16)
    score_grad_kernel<__nv_bfloat16><<<n, kGT, 0, s>>>(g, static_cast<const __nv_bfloat16*>(g.prep_lp),
                                                        static_cast<const __nv_bfloat16*>(g.dprep_lp), picks, out);
  else
    score_grad_kernel<float><<<n, kGT, 0, s>>>(g, g.prep, g.dprep, picks, out);
  GISSPA_LAUNCH_CHECK();
}

}  // namespace gisspa
