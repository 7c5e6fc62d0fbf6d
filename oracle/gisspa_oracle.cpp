// gisspa_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement of the GisSPA_v2.0 template-matching search path, used as
// the checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
// Nothing in the product library links or calls this file.
//
// Each stage cites the reference lines it restates (paths relative to the
// GisSPA_v2.0 tree).  The reference's FFTs are cuFFT C2C FP32 transforms; here
// every transform is an FP64 C2C transform of our own (radix-2, or Bluestein for
// other lengths), validated against numpy.fft by the tests.  The AP<->RI
// (amplitude/phase) round trips of the reference are replaced by the equivalent
// real scaling of the complex value (scaling an amplitude by a non-negative real
// factor keeps the phase).
//
// Deliberate differences from the reference, all below 1e-6 relative:
//  * shell index floor(hypot+0.5)-1 is evaluated exactly in integers instead of
//    through float hypotf (they differ only where a^2+b^2 = k^2+k at large k);
//  * every reduction is an exact-order FP64 sum (the reference's warp-synchronous
//    tails at kernels.cu:362-375, 423-436 have no defined result).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <map>
#include <vector>

#include "../include/gisspa.h"

namespace {

using cd = std::complex<double>;
constexpr double REF_PI = 3.1415926535;  // utils/constants.h:3 (used where the reference uses PI)
constexpr double TRUE_PI = 3.14159265358979323846;

// ------------------------------------------------------------------ FFT
struct Fft {
  int n = 0, m = 0;
  bool pow2 = true;
  std::vector<cd> tw;         // e^{-2 pi i k / n}, k < n/2 (radix-2)
  std::vector<int> rev;       // bit reversal
  std::vector<cd> chirp;      // Bluestein: e^{-i pi k^2 / n}
  std::vector<cd> bspec;      // FFT_m of the conjugate chirp kernel
  std::unique_ptr<Fft> inner; // power-of-two FFT of length m

  explicit Fft(int n_) : n(n_) {
    pow2 = n > 0 && (n & (n - 1)) == 0;
    if (pow2) {
      tw.resize(std::max(1, n / 2));
      for (int k = 0; k < n / 2; ++k) tw[k] = std::polar(1.0, -2.0 * TRUE_PI * k / n);
      rev.resize(n);
      int lg = 0;
      while ((1 << lg) < n) ++lg;
      for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < lg; ++b) r |= ((i >> b) & 1) << (lg - 1 - b);
        rev[i] = r;
      }
    } else {
      m = 1;
      while (m < 2 * n - 1) m <<= 1;
      inner = std::make_unique<Fft>(m);
      chirp.resize(n);
      for (long long k = 0; k < n; ++k) {
        long long q = (k * k) % (2LL * n);  // exact phase reduction
        chirp[k] = std::polar(1.0, -TRUE_PI * (double)q / n);
      }
      std::vector<cd> b(m, cd(0, 0));
      for (int k = 0; k < n; ++k) {
        b[k] = std::conj(chirp[k]);
        if (k) b[m - k] = std::conj(chirp[k]);
      }
      inner->exec(b.data(), -1);
      bspec = b;
    }
  }
  // sign -1: forward, +1: inverse; unnormalised (cuFFT convention)
  void exec(cd* x, int sign) const {
    if (pow2) {
      for (int i = 0; i < n; ++i)
        if (i < rev[i]) std::swap(x[i], x[rev[i]]);
      for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int i = 0; i < n; i += len)
          for (int j = 0; j < half; ++j) {
            cd w = tw[j * step];
            if (sign > 0) w = std::conj(w);
            cd u = x[i + j], v = x[i + j + half] * w;
            x[i + j] = u + v;
            x[i + j + half] = u - v;
          }
      }
      return;
    }
    std::vector<cd> a(m, cd(0, 0));
    for (int k = 0; k < n; ++k) a[k] = x[k] * (sign < 0 ? chirp[k] : std::conj(chirp[k]));
    inner->exec(a.data(), -1);
    if (sign < 0) {
      for (int k = 0; k < m; ++k) a[k] *= bspec[k];
    } else {
      // inverse chirp kernel is the conjugate of the forward one: FFT(conj b)[k] = conj(FFT(b)[-k])
      for (int k = 0; k < m; ++k) a[k] *= std::conj(bspec[(m - k) % m]);
    }
    inner->exec(a.data(), +1);
    for (int k = 0; k < n; ++k)
      x[k] = a[k] / (double)m * (sign < 0 ? chirp[k] : std::conj(chirp[k]));
  }
};

// Plans are cached per thread and length (building one costs as much as a few transforms).
const Fft& plan(int n) {
  thread_local std::map<int, std::unique_ptr<Fft>> cache;
  std::unique_ptr<Fft>& p = cache[n];
  if (!p) p = std::make_unique<Fft>(n);
  return *p;
}

// 2D transform of ny rows x nx columns (row-major), unnormalised.  Columns are gathered in
// groups of 16 (each row segment one contiguous read) and transformed one by one.
void fft2(cd* d, int ny, int nx, int sign, bool parallel = true) {
  const Fft& fr = plan(nx);
  const Fft& fc = plan(ny);
  constexpr int G = 16;
#pragma omp parallel for schedule(static) if (parallel)
  for (int y = 0; y < ny; ++y) fr.exec(d + (size_t)y * nx, sign);
#pragma omp parallel if (parallel)
  {
    std::vector<cd> cols((size_t)G * ny);
#pragma omp for schedule(static)
    for (int x0 = 0; x0 < nx; x0 += G) {
      const int g = std::min(G, nx - x0);
      for (int y = 0; y < ny; ++y)
        for (int q = 0; q < g; ++q) cols[(size_t)q * ny + y] = d[(size_t)y * nx + x0 + q];
      for (int q = 0; q < g; ++q) fc.exec(cols.data() + (size_t)q * ny, sign);
      for (int y = 0; y < ny; ++y)
        for (int q = 0; q < g; ++q) d[(size_t)y * nx + x0 + q] = cols[(size_t)q * ny + y];
    }
  }
}

// ------------------------------------------------------------------ parameters
struct Params {  // DataReader2.h:73-83 + SetParams (norm.cu:183-192), in FP64
  double apix, kk, energy, cs, highres, lowres, d_m, thresh;
  double ehw, ampconst, a, b, b2, bf, bf2, bf3;
  double lambda, dfu, dfv, ds, defocus, dfdiff, dfang;
};

Params make_params(const gisspa_config& c, const gisspa_ctf& ctf, int l) {
  Params p{};
  p.apix = c.angpix; p.kk = c.kk; p.energy = c.energy; p.cs = c.cs;
  p.highres = c.highres; p.lowres = c.lowres; p.d_m = c.diameter; p.thresh = c.threshold;
  p.ehw = c.edge_half_width; p.ampconst = c.ampconst;
  p.a = c.a; p.b = c.b; p.b2 = c.b2; p.bf = c.bfactor; p.bf2 = c.bfactor2; p.bf3 = c.bfactor3;
  p.defocus = -ctf.defocus;
  p.dfang = ctf.dfang;
  p.dfdiff = ctf.dfdiff;
  p.dfu = -ctf.defocus + ctf.dfdiff;
  p.dfv = -ctf.defocus - ctf.dfdiff;
  p.lambda = 12.2639 / std::sqrt(p.energy * 1000.0 + 0.97845 * p.energy * p.energy);
  p.ds = 1.0 / (p.apix * l);
  return p;
}

// CTF_AST (kernels.cu:290-317): Hermitian fold, astigmatic defocus, amplitude contrast.
double ctf_ast(int x1, int y1, int nx, int ny, const Params& p, int mode) {
#ifdef ORC_CTF_REFERENCE_FP32
  // The reference's own arithmetic (kernels.cu:290-317): float parameters and float sinf /
  // cosf / atan2, with the double literals promoting the middle of the expressions.
  {
    const float apix = (float)p.apix, dfu = (float)p.dfu, dfv = (float)p.dfv, dfdiff = (float)p.dfdiff;
    const float dfang = (float)p.dfang, lambda = (float)p.lambda, cs = (float)p.cs, ac = (float)p.ampconst;
    y1 = x1 > nx / 2 ? ny - y1 : y1;
    x1 = std::min(x1, nx - x1);
    const float dx = (float)std::min(x1, nx - x1), dy = (float)(y1 - ny / 2);
    const float ss = (dx * dx / (float)(nx * nx) + dy * dy / (float)(ny * ny)) / (apix * apix);
    const float ag = std::atan2((float)(y1 - ny / 2), (float)x1);
    const float df_ast = (float)(0.5 * (dfu + dfv + 2 * dfdiff * cosf((float)(2 * (dfang * REF_PI / 180 - ag)))));
    const float gamma = (float)(-2 * REF_PI *
                                (cs * 2.5e6 * lambda * lambda * lambda * ss * ss + df_ast * 5000.0 * lambda * ss));
    const float v = sqrtf((float)(1.0 - ac * ac)) * sinf(gamma) + ac * cosf(gamma);
    if (mode == 0) return v > 0 ? 1.0 : -1.0;
    if (mode == 2) return std::fabs(v);
    return v;
  }
#endif
  y1 = x1 > nx / 2 ? ny - y1 : y1;
  x1 = std::min(x1, nx - x1);
  double dx = std::min(x1, nx - x1);
  double dy = y1 - ny / 2;
  double ss = (dx * dx / ((double)nx * nx) + dy * dy / ((double)ny * ny)) / (p.apix * p.apix);
  double ag = std::atan2((double)(y1 - ny / 2), (double)x1);
  double df_ast = 0.5 * (p.dfu + p.dfv + 2 * p.dfdiff * std::cos(2 * (p.dfang * REF_PI / 180 - ag)));
  double l3 = p.lambda * p.lambda * p.lambda;
  double gamma = -2 * REF_PI * (p.cs * 2.5e6 * l3 * ss * ss + df_ast * 5000.0 * p.lambda * ss);
  double v = std::sqrt(1.0 - p.ampconst * p.ampconst) * std::sin(gamma) + p.ampconst * std::cos(gamma);
  if (mode == 0) return v > 0 ? 1.0 : -1.0;
  if (mode == 2) return std::fabs(v);
  return v;
}

// floor(hypot(a,b) + 0.5) - 1 evaluated exactly: k with k^2-k < n <= k^2+k.
inline int shell_index(long long a, long long b) {
  long long n = a * a + b * b;
  long long k = (long long)std::floor(std::sqrt((double)n) + 0.5);
  while (k > 0 && k * k - k >= n) --k;
  while (k * k + k < n) ++k;
  return (int)k - 1;
}
inline int shell_xy(int x, int y, int nx, int ny) {
  return shell_index(std::min(y, ny - y), std::min(x, nx - x));
}

// band-pass branch structure shared by apply_weighting_function (kernels.cu:262-275)
// and whiten_filter_weight_Img (kernels.cu:182-189); r is the integer shell index.
double band_factor(double r, double hi, double lo) {
  if (r < hi && r >= 0) return 1.0;
  if (r >= hi && r < hi + 8) return 0.5 * std::cos(REF_PI * (r - hi) / (2 * 8)) + 0.5;
  if (r >= lo - 8 && r < lo && r >= 0) return 0.5 * std::cos(REF_PI * (lo - r) / (2 * 8)) + 0.5;
  return 0.0;
}

// Soft circular mask (apply_mask, kernels.cu:225-241) on an l x l real image.
void apply_mask(double* img, int l, const Params& p) {
  double dm = 1.5 * p.d_m;
  for (int y = 0; y < l; ++y)
    for (int x = 0; x < l; ++x) {
      double r = std::hypot((double)(x - l / 2), (double)(y - l / 2));
      double& v = img[(size_t)y * l + x];
      if (r > dm / 2 + 2 * p.ehw) v = 0;
      else if (r >= dm / 2) v *= 0.5 * std::cos(REF_PI * (r - dm / 2) / (2 * p.ehw)) + 0.5;
    }
}

// Radial RMS normalisation used for templates and windows: m = sqrt(sum|F|^2 / count^2)
// over x <= l/2 and valid shells (compute_area_sum_ofSQR kernels.cu:319-382; host
// finish norm.cu:334-348 / 452-466).
void rms_normalise(cd* F, int l) {
  double s = 0, cnt = 0;
  for (int y = 0; y < l; ++y)
    for (int x = 0; x <= l / 2; ++x) {
      int r = shell_xy(x, y, l, l);
      if (r < l / 2 && r >= 0) { s += std::norm(F[(size_t)y * l + x]); cnt += 1; }
    }
  double m = std::sqrt(s / (cnt * cnt));
  if (m != 0)
    for (size_t i = 0; i < (size_t)l * l; ++i) F[i] /= m;
}

std::vector<int> window_offsets(int len, int l, int ov) {  // blocks_one_axis, norm.cu:68-81
  std::vector<int> off{0};
  int o = 0;
  while (o + l < len) {
    o += l - ov;
    if (o + l >= len) o = len - l;
    off.push_back(o);
  }
  return off;
}
int window_count_nonorm(int len, int l, int ov) {  // nonorm.cu:71-81
  int o = 0, n = 1;
  while (o + l < len) {
    o += l - ov;
    if (o + l >= len) o = len - l;
    ++n;
  }
  return n;
}

std::vector<float> angle_list(float phistep) {  // for (float e = 0; e < 360; e += step), norm.cu:684
  std::vector<float> a;
  for (float e = 0.0f; e < 360.0f; e += phistep) a.push_back(e);
  return a;
}

// ------------------------------------------------------------------ template preparation
// PreprocessTemplate (norm.cu:194-354; nonorm.cu:178-344).  Output: norm_type=1 the
// real-space preprocessed template (real part of the unnormalised IFFT), norm_type=0
// the preprocessed spectrum.  out holds l*l complex values per template.
void prep_templates(const gisspa_config& c, const Params& p, const float* stack, int nt, int tw,
                    int th, cd* out) {
  const int l = c.window_size;
  const size_t L2 = (size_t)l * l;
  const int sx = (l - tw) / 2, sy = (l - th) / 2;  // LoadTemplate, norm.cu:137-149
  // ring mask for the edge mean (generate_mask kernels.cu:28-55, bounds norm.cu:198-203)
  float rf = l / 2.f - 2.f;
  double up = 0, low = 0;
  if (rf > 1) { up = (rf + 1.0) * (rf + 1.0); low = (rf - 1.0) * (rf - 1.0); }
  const double hi = (double)l * p.apix / p.highres, lo = (double)l * p.apix / p.lowres;
#pragma omp parallel for schedule(dynamic)
  for (int n = 0; n < nt; ++n) {
    std::vector<double> P(L2, 0.0);
    for (int j = 0; j < th; ++j)
      for (int i = 0; i < tw; ++i) P[(size_t)(sy + j) * l + (sx + i)] = stack[(size_t)n * tw * th + (size_t)j * tw + i];
    // edge mean em over the ring (multiCount_dot kernels.cu:57-80)
    double cnt = 0, dot = 0;
    for (int y = 0; y < l; ++y)
      for (int x = 0; x < l; ++x) {
        double rr = (double)(x - l / 2) * (x - l / 2) + (double)(y - l / 2) * (y - l / 2);
        if (rr >= low && rr <= up) { cnt += 1; dot += P[(size_t)y * l + x]; }
      }
    double em = cnt != 0 ? dot / cnt : dot;
    // sigma over the padded window (UpdateSigma kernels.cu:4-26, host norm.cu:268-273)
    double s1 = 0, s2 = 0;
    for (size_t i = 0; i < L2; ++i) { s1 += P[i]; s2 += P[i] * P[i]; }
    double mean = s1 / (double)L2;
    double sigma = std::sqrt(s2 / (double)L2 - mean * mean);
    if (sigma < 0 || !std::isfinite(sigma)) sigma = 0;
    std::vector<cd> F(L2);
    bool scale = !(sigma < 1e-8 && sigma > -1e-8);  // scale_each kernels.cu:82-90
    for (size_t i = 0; i < L2; ++i) F[i] = cd(scale ? (P[i] - em) / sigma : P[i], 0);
    fft2(F.data(), l, l, -1, false);
    for (auto& v : F) v /= (double)L2;
    // whitening by the template's own radial power (SQRSum_by_circle kernels.cu:94-126,
    // whiten_Tmp kernels.cu:128-149)
    std::vector<double> ra(l, 0.0), rb(l, 0.0);
    for (int y = 0; y < l; ++y)
      for (int x = 0; x <= l / 2; ++x) {
        int r = shell_xy(x, y, l, l);
        if (r < l / 2 && r >= 0) { ra[r] += std::norm(F[(size_t)y * l + x]); rb[r] += 1; }
      }
    for (int y = 0; y < l; ++y)
      for (int x = 0; x < l; ++x) {
        int r = shell_xy(x, y, l, l);
        if (r < l / 2 && r >= 0) F[(size_t)y * l + x] /= std::sqrt(ra[r] / rb[r]);
      }
    if (c.norm_type == 0) {
      // nonorm.cu:291-299: IFFT -> real-space soft mask -> FFT / l^2
      fft2(F.data(), l, l, +1, false);
      std::vector<double> R(L2);
      for (size_t i = 0; i < L2; ++i) R[i] = F[i].real();
      apply_mask(R.data(), l, p);
      for (size_t i = 0; i < L2; ++i) F[i] = cd(R[i], 0);
      fft2(F.data(), l, l, -1, false);
      for (auto& v : F) v /= (double)L2;
    }
    // band-pass + CTF/SSNR weighting (apply_weighting_function kernels.cu:243-288)
    for (int y = 0; y < l; ++y)
      for (int x = 0; x < l; ++x) {
        double r = std::hypot((double)std::min(y, l - y), (double)std::min(x, l - x));
        int rr = shell_xy(x, y, l, l);
        cd& v = F[(size_t)y * l + x];
        v *= band_factor(rr, hi, lo);
        double ss = r * p.ds;
        if (rr < l / 2 && rr >= 0) {
          double ct = ctf_ast(x, (y + l / 2) % l, l, l, p, 2);
          double signal = std::exp(p.bf * ss * ss + p.bf2 * ss + p.bf3) / (p.kk + 1);
          double ncurve = std::exp(p.a * ss * ss + p.b * ss + p.b2) / signal;
          v *= ct * std::sqrt(1 / (ncurve + p.kk * ct * ct));
        }
      }
    rms_normalise(F.data(), l);
    cd* o = out + (size_t)n * L2;
    if (c.norm_type != 0) {
      fft2(F.data(), l, l, +1, false);  // norm.cu:350-351 (unnormalised IFFT)
      for (size_t i = 0; i < L2; ++i) o[i] = cd(F[i].real(), 0);
    } else {
      for (size_t i = 0; i < L2; ++i) o[i] = F[i];
    }
  }
}

// ------------------------------------------------------------------ image preparation
// LoadImage (norm.cu:156-181): outlier clamp + optional invert.  With the quirk bit the
// statistics are the reference's serial FP32 sums and int-truncated bounds.
void load_image(const gisspa_config& c, std::vector<double>& img, const float* src, int nx, int ny) {
  size_t N = (size_t)nx * ny;
  img.assign(src, src + N);
  double avg_d, var_d;
  bool clamp;
  int up_bound, low_bound;
  if (c.quirks & GISSPA_QUIRK_OUTLIER_FP32_SERIAL) {
    volatile float sum = 0, sum_s2 = 0;  // volatile: keep the serial float order
    for (size_t i = 0; i < N; ++i) {
      float cur = src[i];
      sum = sum + cur / (float)nx / (float)ny;
      sum_s2 = sum_s2 + (cur * cur / (float)nx / (float)ny);
    }
    float avg = sum;
    float var = std::sqrt((float)(sum_s2 - avg * avg));
    float t_up = avg + 6.0f * var, t_lo = avg - 6.0f * var;
    up_bound = (int)t_up;
    low_bound = (int)t_lo;
    clamp = sum_s2 > avg * avg;
    avg_d = avg;
    var_d = var;
    if (clamp)
      for (size_t i = 0; i < N; ++i)
        if (src[i] > (float)up_bound || src[i] < (float)low_bound) img[i] = (double)avg;
  } else {
    double s = 0, s2 = 0;
    for (size_t i = 0; i < N; ++i) { s += src[i]; s2 += (double)src[i] * src[i]; }
    avg_d = s / N;
    var_d = std::sqrt(s2 / N - avg_d * avg_d);
    up_bound = (int)(avg_d + 6 * var_d);
    low_bound = (int)(avg_d - 6 * var_d);
    clamp = s2 / N > avg_d * avg_d;
    if (clamp)
      for (size_t i = 0; i < N; ++i)
        if (src[i] > up_bound || src[i] < low_bound) img[i] = avg_d;
  }
  (void)var_d;
  if (c.invert)
    for (auto& v : img) v = -v;
}

// PreprocessImage (norm.cu:356-402; nonorm.cu:346-389 when phase_flip=1): FFT/(nx ny),
// phase flip, radial whitening + SSNR weighting + band-pass (whiten_filter_weight_Img
// kernels.cu:151-202), DC = 0 (norm only), unnormalised IFFT, real part.
void preprocess_image(const Params& p, std::vector<double>& img, int nx, int ny, bool zero_dc) {
  size_t N = (size_t)nx * ny;
  std::vector<cd> G(N);
  for (size_t i = 0; i < N; ++i) G[i] = cd(img[i], 0);
  fft2(G.data(), ny, nx, -1);
  for (auto& v : G) v /= (double)N;
#pragma omp parallel for
  for (int y = 0; y < ny; ++y)  // do_phase_flip kernels.cu:828-839
    for (int x = 0; x < nx; ++x) G[(size_t)y * nx + x] *= ctf_ast(x, (y + ny / 2) % ny, nx, ny, p, 0);
  const int L = std::max(nx, ny);
  std::vector<double> ra(L, 0.0), rb(L, 0.0);  // SQRSum_by_circle mode 1
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x <= nx / 2; ++x) {
      int r = shell_xy(x, y, nx, ny);
      if (r < L / 2 && r >= 0) { ra[r] += std::norm(G[(size_t)y * nx + x]); rb[r] += 1; }
    }
  const double hi = (double)L * p.apix / p.highres, lo = (double)L * p.apix / p.lowres;
#pragma omp parallel for
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      double dx = std::min(x, nx - x), dy = std::min(y, ny - y);
      int r = shell_xy(x, y, nx, ny);
      double ss = std::sqrt((dx * dx / ((double)nx * nx) + dy * dy / ((double)ny * ny)) / (p.apix * p.apix));
      cd& g = G[(size_t)y * nx + x];
      double v = 0, signal = 0, ncurve = 0;
      if (r < L / 2 && r >= 0) {
        v = ctf_ast(x, (y + ny / 2) % ny, nx, ny, p, 2);
        signal = std::exp(p.bf * ss * ss + p.bf2 * ss + p.bf3);
        ncurve = std::exp(p.a * ss * ss + p.b * ss + p.b2);
        g *= std::sqrt((signal * v * v + ncurve) / signal) / std::sqrt(ra[r] / rb[r]);
        if (r > L * p.apix / 6) g *= std::exp(-100 * ss * ss);
      }
      g *= band_factor(r, hi, lo);
      if (r < L / 2 && r >= 0) {
        signal /= (p.kk + 1);
        ncurve /= signal;
        g *= std::sqrt(1 / (ncurve + p.kk * v * v));
      }
    }
  if (zero_dc) G[0] = 0;  // set_0Hz_to_0_at_RI kernels.cu:204-223
  fft2(G.data(), ny, nx, +1);
  for (size_t i = 0; i < N; ++i) img[i] = G[i].real();
}

// ------------------------------------------------------------------ rotation
// rotate_subIMG (kernels.cu:534-603) of a real l x l image by theta degrees about (l/2, l/2).
// The sampling coordinates are computed in float as the reference does (cos/sin in double,
// rounded to float; x2 = (cose x + sine y) + l/2 in float): whether a border pixel is
// interpolated or zeroed (x2 > l - 1) depends on that rounding at 90/180/270 degrees.
// The interpolation itself is FP64.
void rotate(const double* in, double* out, int l, float theta) {
  const float cose = (float)std::cos((double)theta * REF_PI / 180), sine = (float)std::sin((double)theta * REF_PI / 180);
  for (int j = 0; j < l; ++j)
    for (int i = 0; i < l; ++i) {
      const float x = (float)(i - l / 2), y = (float)(j - l / 2);
      volatile float a1 = cose * x, a2 = sine * y, b1 = -sine * x, b2 = cose * y;
      volatile float s1 = a1 + a2, s2 = b1 + b2;
      const float fx2 = s1 + (float)(l / 2), fy2 = s2 + (float)(l / 2);
      double x2 = fx2, y2 = fy2;
      double res = 0;
      if (!(x2 < 0 || x2 > l - 1.0 || y2 < 0 || y2 > l - 1.0)) {
        int ii = (int)std::floor(x2), jj = (int)std::floor(y2);
        int k0 = ii + jj * l, k1 = k0 + 1, k2 = k0 + l + 1, k3 = k0 + l;
        if (ii == l - 1) { k1 -= 1; k2 -= 1; }
        if (jj == l - 1) { k2 -= l; k3 -= l; }
        double t = x2 - ii, u = y2 - jj, tt = 1 - t, uu = 1 - u;
        res = in[k0] * tt * uu + in[k1] * t * uu + in[k2] * t * u + in[k3] * tt * u;
      }
      out[(size_t)j * l + i] = res;
    }
}

// RotateTemplate (norm.cu:479-521): rotate -> mask -> (x - mean)/sqrt(var) -> FFT / l^2.
void rotated_template_spectrum(const Params& p, const cd* prep, int l, float theta, cd* T) {
  const size_t L2 = (size_t)l * l;
  std::vector<double> in(L2), R(L2);
  for (size_t i = 0; i < L2; ++i) in[i] = prep[i].real();
  rotate(in.data(), R.data(), l, theta);
  apply_mask(R.data(), l, p);
  double s1 = 0, s2 = 0;
  for (size_t i = 0; i < L2; ++i) { s1 += R[i]; s2 += R[i] * R[i]; }
  double mean = s1 / L2, var = s2 / L2 - mean * mean;
  for (size_t i = 0; i < L2; ++i) {
    double v = R[i];
    if (mean != 0) v -= mean;
    if (var != 0) v /= std::sqrt(var);
    T[i] = cd(v, 0);
  }
  fft2(T, l, l, -1, false);
  for (size_t i = 0; i < L2; ++i) T[i] /= (double)L2;
}

// Correlation map (compute_corner_CCG kernels.cu:645-678 + inverse FFT): returns the
// real part of IFFT(I conj(T) (-1)^(kx+ky)) (unnormalised), zero lag at (l/2, l/2).
void correlate(const cd* I, const cd* T, int l, double* out, std::vector<cd>& buf) {
  const size_t L2 = (size_t)l * l;
  buf.resize(L2);
  for (int y = 0; y < l; ++y)
    for (int x = 0; x < l; ++x) {
      size_t k = (size_t)y * l + x;
      cd v = I[k] * std::conj(T[k]);
      buf[k] = ((x + y) & 1) ? -v : v;
    }
  fft2(buf.data(), l, l, +1, false);
  for (size_t i = 0; i < L2; ++i) out[i] = buf[i].real();
}

// Two correlation maps with one transform.  Z1 = I conj(T1) (-1)^(kx+ky) and Z2 likewise are
// Hermitian (spectra of real images; the checkerboard is even for even l), so their inverse
// transforms c1, c2 are real and IFFT(Z1 + i Z2) = c1 + i c2.  T2 = nullptr: c1 only.
void correlate2(const cd* I, const cd* T1, const cd* T2, int l, double* out1, double* out2,
                std::vector<cd>& buf) {
  if (!T2) {
    correlate(I, T1, l, out1, buf);
    return;
  }
  const size_t L2 = (size_t)l * l;
  buf.resize(L2);
  const cd j(0, 1);
  for (int y = 0; y < l; ++y)
    for (int x = 0; x < l; ++x) {
      size_t k = (size_t)y * l + x;
      cd v = I[k] * std::conj(T1[k]) + j * (I[k] * std::conj(T2[k]));
      buf[k] = ((x + y) & 1) ? -v : v;
    }
  fft2(buf.data(), l, l, +1, false);
  for (size_t i = 0; i < L2; ++i) {
    out1[i] = buf[i].real();
    out2[i] = buf[i].imag();
  }
}

inline unsigned brev8(unsigned v) {
  unsigned r = 0;
  for (int b = 0; b < 8; ++b) r |= ((v >> b) & 1u) << (7 - b);
  return r;
}
// Winner of the reference's 256-wide shared-memory max tree (get_peak_pos kernels.cu:766-793):
// strict '>' keeps the left operand, so among equal maxima the lane with the smallest
// bit-reversed index survives.
inline bool chunk_better(double v, unsigned lane, double bv, unsigned blane) {
  if (v > bv) return true;
  if (v < bv) return false;
  return brev8(lane) < brev8(blane);
}

struct Workspace {
  int l = 0, nx = 0, ny = 0, bx = 0, by = 0, W = 0, nt = 0, batch = 0;
  std::vector<int> offx, offy;
  std::vector<cd> windows;  // W * l * l spectra
  std::vector<cd> prep;     // nt * l * l
};

// SplitImage (norm.cu:404-477): windows at clamped offsets, FFT/l^2, radial RMS normalisation.
void split_windows(const gisspa_config& c, const std::vector<double>& img, Workspace& ws) {
  const int l = c.window_size;
  const size_t L2 = (size_t)l * l;
  ws.windows.assign((size_t)ws.W * L2, cd(0, 0));
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < ws.W; ++b) {
    int i = b % ws.bx, j = b / ws.bx;
    cd* w = ws.windows.data() + (size_t)b * L2;
    for (int y = 0; y < l; ++y)
      for (int x = 0; x < l; ++x) {
        int ox = ws.offx[i] + x, oy = ws.offy[j] + y;
        if (ox < ws.nx && oy < ws.ny) w[(size_t)y * l + x] = cd(img[(size_t)oy * ws.nx + ox], 0);
      }
    fft2(w, l, l, -1, false);
    for (size_t k = 0; k < L2; ++k) w[k] /= (double)L2;
    rms_normalise(w, l);
  }
}

int validate(const gisspa_config* c, int nx, int ny, int nt, int tw, int th) {
  if (!c || nx <= 0 || ny <= 0 || nt <= 0 || tw <= 0 || th <= 0) return GISSPA_ERR_ARG;
  int l = c->window_size;
  if (l <= 0 || l % 16) return GISSPA_ERR_SHAPE;
  if (tw > l || th > l) return GISSPA_ERR_SHAPE;
  if (!(c->phistep > 0)) return GISSPA_ERR_ARG;
  return GISSPA_OK;
}

int n_euler_count(const gisspa_config& c, size_t n_angles) {
  if (c.quirks & GISSPA_QUIRK_NEULER_TRUNC) return (int)(360.0f / c.phistep);
  return (int)n_angles;
}

}  // namespace

extern "C" {

// 1D/2D transforms exposed for validation against numpy.fft (interleaved re/im doubles).
int orc_fft2d(double* data, int ny, int nx, int sign) {
  fft2(reinterpret_cast<cd*>(data), ny, nx, sign);
  return 0;
}

// Stage outputs for stage-by-stage parity tests (all complex arrays interleaved re/im).
int orc_prep_templates(const gisspa_config* c, const gisspa_ctf* ctf, const float* stack, int nt,
                       int tw, int th, double* out) {
  int st = validate(c, c->window_size, c->window_size, nt, tw, th);
  if (st) return st;
  Params p = make_params(*c, *ctf, c->window_size);
  prep_templates(*c, p, stack, nt, tw, th, reinterpret_cast<cd*>(out));
  return 0;
}

int orc_prep_image(const gisspa_config* c, const gisspa_ctf* ctf, const float* img, int nx, int ny,
                   double* out) {
  Params p = make_params(*c, *ctf, c->window_size);
  std::vector<double> v;
  load_image(*c, v, img, nx, ny);
  preprocess_image(p, v, nx, ny, true);
  std::memcpy(out, v.data(), sizeof(double) * v.size());
  return 0;
}

int orc_window_offsets(int len, int l, int ov, int* out, int cap) {
  auto o = window_offsets(len, l, ov);
  for (int i = 0; i < (int)o.size() && i < cap; ++i) out[i] = o[i];
  return (int)o.size();
}

int orc_window_spectra(const gisspa_config* c, const double* img_pre, int nx, int ny, double* out) {
  Workspace ws;
  const int l = c->window_size;
  ws.l = l; ws.nx = nx; ws.ny = ny;
  ws.offx = window_offsets(nx, l, c->overlap);
  ws.offy = window_offsets(ny, l, c->overlap);
  ws.bx = ws.offx.size(); ws.by = ws.offy.size(); ws.W = ws.bx * ws.by;
  std::vector<double> img(img_pre, img_pre + (size_t)nx * ny);
  split_windows(*c, img, ws);
  std::memcpy(out, ws.windows.data(), sizeof(cd) * ws.windows.size());
  return ws.W;
}

int orc_rotated_spectrum(const gisspa_config* c, const gisspa_ctf* ctf, const double* prep, float theta,
                         double* out) {
  Params p = make_params(*c, *ctf, c->window_size);
  rotated_template_spectrum(p, reinterpret_cast<const cd*>(prep), c->window_size, theta,
                            reinterpret_cast<cd*>(out));
  return 0;
}

// Full norm_type=1 search (SearchNorm::work, norm.cu:620-660).
//  picks/cap/n_out: reference chunk picks (GISSPA_PICK_CHUNK) or top-K picks.
//  stats_out (optional): W*l*l*2 doubles, per-window-pixel (mu, sigma).
//  max_templates / max_angles (optional, > 0): restrict the search to a sample (timing only).
//  margin_out (optional, cap doubles): for each pick, how far (in z) its outcome stands from the
//    nearest alternative outcome; a pick whose margin is below twice a comparison tolerance may
//    legitimately come out differently in FP32.  Chunk picks: best z of the chunk minus the
//    next best pixel's.  Top-K picks: the smallest of (best z at the pixel minus the best z of
//    any other (template, angle) there), (z minus the best z of the other candidate pixels within
//    the exclusion radius that no earlier pick excluded) and, for the last pick, (z minus the
//    next pick a larger K would take).
//  near_out / near_margin (optional, chunk picks): chunks that gave no pick only because their
//    best pixel's centre failed the border test although another pixel within 1 % of the best z
//    passes it; each record is the pick that pixel would give (score = its z) and near_margin
//    the z distance to the chunk's best.
int orc_search_norm(const gisspa_config* cin, const gisspa_ctf* ctf, const float* image, int nx, int ny,
                    const float* stack, int nt, int tw, int th, gisspa_pick* picks, size_t cap,
                    size_t* n_out, double* stats_out, int max_templates, int max_angles, double* margin_out,
                    gisspa_pick* near_out, double* near_margin, size_t near_cap, size_t* n_near) {
  int st = validate(cin, nx, ny, nt, tw, th);
  if (st) return st;
  gisspa_config c = *cin;
  const int l = c.window_size;
  const size_t L2 = (size_t)l * l;
  Params p = make_params(c, *ctf, l);
  Workspace ws;
  ws.l = l; ws.nx = nx; ws.ny = ny;
  ws.offx = window_offsets(nx, l, c.overlap);
  ws.offy = window_offsets(ny, l, c.overlap);
  ws.bx = ws.offx.size(); ws.by = ws.offy.size(); ws.W = ws.bx * ws.by;
  int nts = nt;
  if (max_templates > 0) nts = std::min(nt, max_templates);
  ws.nt = nts;
  ws.batch = (c.quirks & GISSPA_QUIRK_COUNT_PADDED_TEMPLATES) ? std::max(nt, ws.W) : nt;
  ws.prep.assign((size_t)nts * L2, cd(0, 0));
  prep_templates(c, p, stack, nts, tw, th, ws.prep.data());
  std::vector<double> img;
  load_image(c, img, image, nx, ny);
  preprocess_image(p, img, nx, ny, true);
  split_windows(c, img, ws);

  std::vector<float> angles = angle_list(c.phistep);
  const int n_angles_run = max_angles > 0 ? std::min<int>(max_angles, angles.size()) : (int)angles.size();
  const double Ntot = (double)ws.batch * n_euler_count(c, angles.size());
  const bool topk = c.pick_mode == GISSPA_PICK_TOPK;

  // sweep 1 (ComputeCCGSum norm.cu:523-544): per window pixel sum and sum of squares of CC/l^2
  std::vector<double> S1((size_t)ws.W * L2, 0.0), S2((size_t)ws.W * L2, 0.0);
  std::vector<float> cmax;
  std::vector<int> carg;
  std::vector<double> cmax2;  // second-largest correlation at the pixel (margins only)
  if (topk) {
    cmax.assign((size_t)ws.W * L2, -INFINITY);
    carg.assign((size_t)ws.W * L2, -1);
    cmax2.assign((size_t)ws.W * L2, -INFINITY);
  }
  std::vector<cd> T((size_t)nts * L2);
  for (int a = 0; a < n_angles_run; ++a) {
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < nts; ++n)
      rotated_template_spectrum(p, ws.prep.data() + (size_t)n * L2, l, angles[a], T.data() + (size_t)n * L2);
#pragma omp parallel
    {
      std::vector<cd> buf;
      std::vector<double> ccs(2 * L2);
#pragma omp for schedule(dynamic)
      for (int b = 0; b < ws.W; ++b) {
        double* s1 = S1.data() + (size_t)b * L2;
        double* s2 = S2.data() + (size_t)b * L2;
        for (int n = 0; n < nts; ++n) {
          if ((n & 1) == 0)
            correlate2(ws.windows.data() + (size_t)b * L2, T.data() + (size_t)n * L2,
                       n + 1 < nts ? T.data() + (size_t)(n + 1) * L2 : nullptr, l, ccs.data(), ccs.data() + L2, buf);
          const double* cc = ccs.data() + (n & 1) * L2;
          for (size_t k = 0; k < L2; ++k) {
            double v = cc[k] / (double)L2;
            s1[k] += v;
            s2[k] += v * v;
            if (topk) {
              if (v > cmax[(size_t)b * L2 + k]) {
                cmax2[(size_t)b * L2 + k] = std::max<double>(cmax2[(size_t)b * L2 + k], cmax[(size_t)b * L2 + k]);
                cmax[(size_t)b * L2 + k] = (float)v;
                carg[(size_t)b * L2 + k] = a * nt + n;
              } else if (v > cmax2[(size_t)b * L2 + k]) {
                cmax2[(size_t)b * L2 + k] = v;
              }
            }
          }
        }
      }
    }
  }
  // ComputeCCGMean (set_CCG_mean kernels.cu:697-706)
  std::vector<double> mu((size_t)ws.W * L2), sd((size_t)ws.W * L2);
  for (size_t k = 0; k < mu.size(); ++k) {
    double m = S1[k] / Ntot;
    mu[k] = m;
    sd[k] = std::sqrt(S2[k] / Ntot - m * m);
  }
  if (stats_out)
    for (size_t k = 0; k < mu.size(); ++k) { stats_out[2 * k] = mu[k]; stats_out[2 * k + 1] = sd[k]; }

  std::vector<gisspa_pick> out, near;
  std::vector<double> margins, near_m;
  if (!topk) {
    // sweep 2 (PickParticles norm.cu:554-600): z-score, 256-pixel chunk max, threshold,
    // centre inside [d, n-d)
    const size_t chunks = L2 / 256;
    for (int a = 0; a < n_angles_run; ++a) {
#pragma omp parallel for schedule(dynamic)
      for (int n = 0; n < nts; ++n)
        rotated_template_spectrum(p, ws.prep.data() + (size_t)n * L2, l, angles[a], T.data() + (size_t)n * L2);
      std::vector<std::vector<gisspa_pick>> per_b(ws.W), near_b(ws.W);
      std::vector<std::vector<double>> per_m(ws.W), near_mb(ws.W);
#pragma omp parallel
      {
        std::vector<cd> buf;
        std::vector<double> ccs(2 * L2);
#pragma omp for schedule(dynamic)
        for (int b = 0; b < ws.W; ++b) {
          int i = b % ws.bx, j = b / ws.bx;
          for (int n = 0; n < nts; ++n) {
            if ((n & 1) == 0)
              correlate2(ws.windows.data() + (size_t)b * L2, T.data() + (size_t)n * L2,
                         n + 1 < nts ? T.data() + (size_t)(n + 1) * L2 : nullptr, l, ccs.data(), ccs.data() + L2,
                         buf);
            const double* cc = ccs.data() + (n & 1) * L2;
            for (size_t ch = 0; ch < chunks; ++ch) {
              double best = 0, zs[256];
              unsigned blane = 0;
              for (unsigned t = 0; t < 256; ++t) {
                size_t k = ch * 256 + t;
                double s = sd[(size_t)b * L2 + k];
                double z = s > 0 ? (cc[k] / (double)L2 - mu[(size_t)b * L2 + k]) / s : 0.0;
                zs[t] = z;
                if (t == 0 || chunk_better(z, t, best, blane)) { best = z; blane = t; }
              }
              auto inside = [&](unsigned t) {
                size_t idx = ch * 256 + t;
                int cx = ws.offx[i] + (int)(idx % l), cy = ws.offy[j] + (int)(idx / l);
                return cx >= p.d_m && cx < nx - p.d_m && cy >= p.d_m && cy < ny - p.d_m;
              };
              auto make = [&](unsigned t, double z) {
                size_t idx = ch * 256 + t;
                gisspa_pick pk{};
                pk.score = (float)z;
                pk.x = (float)(ws.offx[i] + (int)(idx % l)); pk.y = (float)(ws.offy[j] + (int)(idx / l));
                float cur_e = 360.0f - angles[a];
                if (cur_e >= 360.0f) cur_e -= 360.0f;
                pk.angle = cur_e;
                pk.theta = angles[a];
                pk.template_id = n; pk.window = b; pk.tile = 0; pk.angle_index = a; pk.chunk = (int)ch;
                return pk;
              };
              if (best >= p.thresh && inside(blane)) {
                per_b[b].push_back(make(blane, best));
                if (margin_out) {
                  double second = -INFINITY;
                  for (unsigned t = 0; t < 256; ++t)
                    if (t != blane) second = std::max(second, zs[t]);
                  per_m[b].push_back(best - second);
                }
              } else if (near_out && best >= p.thresh - 0.01 * std::fabs(best)) {
                // the best pixel's centre failed the border test: the best pixel that passes it
                double bz = -INFINITY;
                unsigned bt = 0;
                for (unsigned t = 0; t < 256; ++t)
                  if (t != blane && inside(t) && zs[t] > bz) { bz = zs[t]; bt = t; }
                if (bz >= p.thresh - 0.01 * std::fabs(best) && best - bz <= 0.01 * std::fabs(best)) {
                  near_b[b].push_back(make(bt, bz));
                  near_mb[b].push_back(best - bz);
                }
              }
            }
          }
        }
      }
      // output order: angle, window (j outer, i inner == b ascending), template, chunk
      for (int b = 0; b < ws.W; ++b) {
        out.insert(out.end(), per_b[b].begin(), per_b[b].end());
        margins.insert(margins.end(), per_m[b].begin(), per_m[b].end());
        near.insert(near.end(), near_b[b].begin(), near_b[b].end());
        near_m.insert(near_m.end(), near_mb[b].begin(), near_mb[b].end());
      }
    }
  } else {
    // one-sweep top-K: image map of max z over windows, then greedy exclusion
    std::vector<float> Z((size_t)nx * ny, -INFINITY);
    std::vector<int> Zarg((size_t)nx * ny, -1), Zwin((size_t)nx * ny, -1);
    // per image pixel, for the margins: the best z of each window covering it with its
    // (template, angle), and the best z of a second (template, angle) within any window
    std::vector<double> Zalt;
    if (margin_out) Zalt.assign((size_t)nx * ny, -INFINITY);
    for (int b = 0; b < ws.W; ++b) {
      int i = b % ws.bx, j = b / ws.bx;
      for (size_t k = 0; k < L2; ++k) {
        if (carg[(size_t)b * L2 + k] < 0) continue;
        double s = sd[(size_t)b * L2 + k];
        double z = s > 0 ? (cmax[(size_t)b * L2 + k] - mu[(size_t)b * L2 + k]) / s : 0.0;
        int cx = ws.offx[i] + (int)(k % l), cy = ws.offy[j] + (int)(k / l);
        if (cx >= nx || cy >= ny) continue;
        size_t q = (size_t)cy * nx + cx;
        if (margin_out && s > 0 && cmax2[(size_t)b * L2 + k] > -INFINITY)
          Zalt[q] = std::max(Zalt[q], (cmax2[(size_t)b * L2 + k] - mu[(size_t)b * L2 + k]) / s);
        if ((float)z > Z[q]) { Z[q] = (float)z; Zarg[q] = carg[(size_t)b * L2 + k]; Zwin[q] = b; }
      }
    }
    if (margin_out)  // a window whose best is another (template, angle) than the pixel's winner
      for (int b = 0; b < ws.W; ++b) {
        int i = b % ws.bx, j = b / ws.bx;
        for (size_t k = 0; k < L2; ++k) {
          if (carg[(size_t)b * L2 + k] < 0) continue;
          double s = sd[(size_t)b * L2 + k];
          int cx = ws.offx[i] + (int)(k % l), cy = ws.offy[j] + (int)(k / l);
          if (cx >= nx || cy >= ny || s <= 0) continue;
          size_t q = (size_t)cy * nx + cx;
          if (carg[(size_t)b * L2 + k] != Zarg[q])
            Zalt[q] = std::max(Zalt[q], (cmax[(size_t)b * L2 + k] - mu[(size_t)b * L2 + k]) / s);
        }
      }
    std::vector<size_t> cand;
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        size_t q = (size_t)y * nx + x;
        if (Zarg[q] >= 0 && Z[q] >= p.thresh && x >= p.d_m && x < nx - p.d_m && y >= p.d_m && y < ny - p.d_m)
          cand.push_back(q);
      }
    std::stable_sort(cand.begin(), cand.end(), [&](size_t u, size_t v) { return Z[u] > Z[v]; });
    const double r2 = (double)c.exclusion_radius * c.exclusion_radius;
    std::vector<size_t> acc;
    auto excluded = [&](size_t q, size_t upto) {
      int x = q % nx, y = q / nx;
      for (size_t u = 0; u < upto; ++u) {
        double dx = x - (int)(acc[u] % nx), dy = y - (int)(acc[u] / nx);
        if (dx * dx + dy * dy <= r2) return true;
      }
      return false;
    };
    size_t next_rank = cand.size();  // rank of the first candidate a (K+1)-th pick would take
    for (size_t rk = 0; rk < cand.size(); ++rk) {
      size_t q = cand[rk];
      if (excluded(q, acc.size())) continue;
      if ((int)acc.size() >= c.topk) { next_rank = rk; break; }
      int x = q % nx, y = q / nx;
      acc.push_back(q);
      gisspa_pick pk{};
      pk.score = Z[q];
      pk.x = (float)x; pk.y = (float)y;
      int a = Zarg[q] / nt, n = Zarg[q] % nt;
      float cur_e = 360.0f - angles[a];
      if (cur_e >= 360.0f) cur_e -= 360.0f;
      pk.angle = cur_e; pk.theta = angles[a];
      pk.template_id = n; pk.window = Zwin[q]; pk.angle_index = a; pk.chunk = (int)acc.size() - 1;
      out.push_back(pk);
    }
    if (margin_out) {
      // position competitors: candidates within the radius of a pick that no earlier pick excluded
      std::vector<double> pos_m(acc.size(), INFINITY);
      const int rr = (int)std::ceil(c.exclusion_radius);
      for (size_t u = 0; u < acc.size(); ++u) {
        const int x = acc[u] % nx, y = acc[u] / nx;
        for (int yy = std::max(0, y - rr); yy <= std::min(ny - 1, y + rr); ++yy)
          for (int xx = std::max(0, x - rr); xx <= std::min(nx - 1, x + rr); ++xx) {
            const size_t q = (size_t)yy * nx + xx;
            double dx = xx - x, dy = yy - y;
            if (q == acc[u] || dx * dx + dy * dy > r2) continue;
            if (Zarg[q] < 0 || Z[q] < p.thresh || xx < p.d_m || xx >= nx - p.d_m || yy < p.d_m || yy >= ny - p.d_m)
              continue;
            if (excluded(q, u)) continue;
            pos_m[u] = std::min(pos_m[u], (double)Z[acc[u]] - (double)Z[q]);
          }
      }
      for (size_t u = 0; u < acc.size(); ++u) {
        double m = std::min(pos_m[u], (double)Z[acc[u]] - Zalt[acc[u]]);
        if (u + 1 == acc.size() && next_rank < cand.size()) m = std::min(m, (double)Z[acc[u]] - Z[cand[next_rank]]);
        margins.push_back(m);
      }
    }
  }
  if (margin_out && !margins.empty()) std::memcpy(margin_out, margins.data(), sizeof(double) * std::min(cap, margins.size()));
  if (n_near) {
    *n_near = near.size();
    if (near_out && near.size() <= near_cap && !near.empty()) {
      std::memcpy(near_out, near.data(), sizeof(gisspa_pick) * near.size());
      std::memcpy(near_margin, near_m.data(), sizeof(double) * near.size());
    }
  }
  *n_out = out.size();
  if (out.size() > cap) return GISSPA_ERR_CAPACITY;
  if (!out.empty()) std::memcpy(picks, out.data(), sizeof(gisspa_pick) * out.size());
  return GISSPA_OK;
}

// Tile centres and upper-left corners (TileImages, tileimages.cpp:5-71); returns the count.
int orc_tiles(int width, int height, int tile, int* ulx, int* uly, int cap) {
  int cols = (int)std::ceil((double)width / tile), rows = (int)std::ceil((double)height / tile);
  int x_step = width / cols, y_step = height / rows, n = 0;
  for (int j = 0; j < cols; ++j) {
    int cxx = (j == 0) ? j * tile + tile / 2 : (j == cols - 1 ? width - tile / 2 : x_step * (2 * j + 1) / 2);
    for (int i = 0; i < rows; ++i) {
      int cyy = (i == 0) ? i * tile + tile / 2 : (i == rows - 1 ? height - tile / 2 : y_step * (2 * i + 1) / 2);
      if (n < cap) { ulx[n] = std::max(cxx - tile / 2, 0); uly[n] = std::max(cyy - tile / 2, 0); }
      ++n;
    }
  }
  return n;
}

// Full norm_type=0 search (SearchNoNorm::work, nonorm.cu:559-589) over the tiles of one
// micrograph.  max_angles > 0 restricts the angle loop (timing samples only).
//  margin_out (optional, cap doubles): per pick, the smaller of (its score minus the best score
//  of another window with a valid centre) and (its score minus the score its window's next best
//  pixel would give, (peak - second peak) / sd); below twice a comparison tolerance the pick may
//  legitimately land on the other window or pixel in FP32.
int orc_search_nonorm(const gisspa_config* cin, const gisspa_ctf* ctf, const float* image, int nx, int ny,
                      const float* stack, int nt, int tw, int th, gisspa_pick* picks, size_t cap,
                      size_t* n_out, int max_angles, double* margin_out) {
  int st = validate(cin, nx, ny, nt, tw, th);
  if (st) return st;
  gisspa_config c = *cin;
  const int l = c.window_size, ts = c.tile_size > 0 ? c.tile_size : 720;
  if (nx < ts || ny < ts) return GISSPA_ERR_SHAPE;  // tileimages.cpp:61-65 reads ts x ts
  const size_t L2 = (size_t)l * l;
  Params p = make_params(c, *ctf, l);
  const int bx = window_count_nonorm(ts, l, c.overlap), by = bx, W = bx * by;
  std::vector<cd> Tsp((size_t)nt * L2);
  prep_templates(c, p, stack, nt, tw, th, Tsp.data());
  std::vector<int> ulx(4096), uly(4096);
  int ntiles = orc_tiles(nx, ny, ts, ulx.data(), uly.data(), 4096);
  std::vector<float> angles = angle_list(c.phistep);
  int n_ang = max_angles > 0 ? std::min<int>(max_angles, angles.size()) : (int)angles.size();
  std::vector<gisspa_pick> out;
  std::vector<double> margins;
  // top-K per template (no counterpart in the reference): every (tile, angle, window) peak with a
  // valid centre and score >= threshold, centre in micrograph coordinates, then greedy selection
  struct Cand { double score; float x, y; int tile, angle, window; double pos_margin; };
  const bool topk = c.pick_mode == GISSPA_PICK_TOPK;
  std::vector<std::vector<Cand>> cands(topk ? nt : 0);
  for (int tI = 0; tI < ntiles && tI < 4096; ++tI) {
    std::vector<double> tile((size_t)ts * ts);
    for (int r = 0; r < ts; ++r)
      for (int q = 0; q < ts; ++q) tile[(size_t)r * ts + q] = image[(size_t)(uly[tI] + r) * nx + ulx[tI] + q];
    if (c.invert) for (auto& v : tile) v = -v;  // nonorm.cu:157-165
    if (c.phase_flip == 1) preprocess_image(p, tile, ts, ts, false);
    // SplitImage (nonorm.cu:391-450): unclamped offsets k*(l-ov), zero outside the tile
    std::vector<double> win((size_t)W * L2, 0.0);
    for (int b = 0; b < W; ++b) {
      int ax = b % bx, ay = b / bx;
      for (int y = 0; y < l; ++y)
        for (int x = 0; x < l; ++x) {
          int ox = ax * (l - c.overlap) + x, oy = ay * (l - c.overlap) + y;
          if (ox < ts && oy < ts) win[(size_t)b * L2 + (size_t)y * l + x] = tile[(size_t)oy * ts + ox];
        }
      if (c.phase_flip == 1) {
        std::vector<cd> F(L2);
        for (size_t k = 0; k < L2; ++k) F[k] = cd(win[(size_t)b * L2 + k], 0);
        fft2(F.data(), l, l, -1, false);
        for (auto& v : F) v /= (double)L2;
        rms_normalise(F.data(), l);
        fft2(F.data(), l, l, +1, false);
        for (size_t k = 0; k < L2; ++k) win[(size_t)b * L2 + k] = F[k].real();
      }
    }
    for (int a = 0; a < n_ang; ++a) {
      float e = angles[a];
      // rotate the windows (not the templates) and transform them (nonorm.cu:457-467)
      std::vector<cd> I((size_t)W * L2);
#pragma omp parallel
      {
        std::vector<double> R(L2);
#pragma omp for
        for (int b = 0; b < W; ++b) {
          rotate(win.data() + (size_t)b * L2, R.data(), l, e);
          for (size_t k = 0; k < L2; ++k) I[(size_t)b * L2 + k] = cd(R[k], 0);
          fft2(I.data() + (size_t)b * L2, l, l, -1, false);
          for (size_t k = 0; k < L2; ++k) I[(size_t)b * L2 + k] /= (double)L2;
        }
      }
      std::vector<float> best_s(nt, 0.f), best_x(nt, 0.f), best_y(nt, 0.f);
      std::vector<double> second_s(nt, 0.0), best_pm(nt, INFINITY);  // margins only
      for (int b = 0; b < W; ++b) {
        int i = b % bx, j = b / bx;
        std::vector<double> peaks(nt), pos(nt), sums(nt), sum2s(nt), peak2(nt);
#pragma omp parallel
        {
          std::vector<cd> buf;
          std::vector<double> cc(L2);
#pragma omp for schedule(dynamic)
          for (int n = 0; n < nt; ++n) {
            correlate(I.data() + (size_t)b * L2, Tsp.data() + (size_t)n * L2, l, cc.data(), buf);
            // get_peak_and_SUM (kernels.cu:725-763) + host merge (nonorm.cu:498-506)
            double pk = 0, ps = 0, s = 0, s2 = 0, v1 = -INFINITY, v2 = -INFINITY;
            for (size_t ch = 0; ch < L2 / 256; ++ch) {
              double cb = 0;
              unsigned cl = 0;
              for (unsigned t = 0; t < 256; ++t) {
                size_t k = ch * 256 + t;
                int x = k % l, y = k / l;
                double v = cc[k];
                s += v; s2 += v * v;
                if (x < p.d_m / 4 || x > l - p.d_m / 4 || y < p.d_m / 4 || y > l - p.d_m / 4) v = 0;
                if (t == 0 || chunk_better(v, t, cb, cl)) { cb = v; cl = t; }
                if (v > v1) { v2 = v1; v1 = v; } else if (v > v2) { v2 = v; }
              }
              if (pk < cb) { pk = cb; ps = (double)(ch * 256 + cl); }
            }
            peaks[n] = pk; pos[n] = ps; sums[n] = s; sum2s[n] = s2; peak2[n] = v2;
          }
        }
        // score = peak / sd of the map without the peak (nonorm.cu:509-533)
        for (int n = 0; n < nt; ++n) {
          double ra = sums[n] - peaks[n], rb = sum2s[n] - peaks[n] * peaks[n], rc = (double)L2 - 1;
          double var = rb / rc - (ra / rc) * (ra / rc);
          double sdv = std::sqrt(var);
          double score = (sdv == 0) ? 0 : peaks[n] / sdv;
          int cx = (int)pos[n] % l, cy = (int)pos[n] / l;
          double centerx = i * (l - c.overlap) + (cx - l / 2) * std::cos(e * REF_PI / 180) +
                           (cy - l / 2) * std::sin(e * REF_PI / 180) + l / 2;
          double centery = j * (l - c.overlap) + (cy - l / 2) * std::cos(e * REF_PI / 180) -
                           (cx - l / 2) * std::sin(e * REF_PI / 180) + l / 2;
          const bool valid = centerx >= 0 && centerx < ts && centery >= 0 && centery < ts;
          if (topk) {
            if (valid && (float)score >= p.thresh)
              cands[n].push_back(Cand{score, (float)(ulx[tI] + centerx), (float)(uly[tI] + centery), tI, a, b,
                                      sdv == 0 ? 0.0 : (peaks[n] - peak2[n]) / sdv});
            continue;
          }
          if (best_s[n] < (float)score && valid) {
            second_s[n] = best_s[n];
            best_s[n] = (float)score; best_x[n] = (float)centerx; best_y[n] = (float)centery;
            best_pm[n] = sdv == 0 ? 0.0 : (peaks[n] - peak2[n]) / sdv;
          } else if (valid) {
            second_s[n] = std::max(second_s[n], score);
          }
        }
      }
      if (topk) continue;
      // OutputScore (nonorm.cu:539-557): one line per template with score >= threshold
      for (int n = 0; n < nt; ++n)
        if (best_s[n] >= p.thresh) {
          gisspa_pick pk{};
          pk.score = best_s[n]; pk.x = best_x[n]; pk.y = best_y[n];
          pk.angle = e; pk.theta = e; pk.template_id = n; pk.window = -1; pk.tile = tI;
          pk.angle_index = a; pk.chunk = -1;
          out.push_back(pk);
          margins.push_back(std::min((double)best_s[n] - second_s[n], best_pm[n]));
        }
    }
  }
  for (int n = 0; topk && n < nt; ++n) {
    std::vector<Cand>& cd_ = cands[n];
    std::stable_sort(cd_.begin(), cd_.end(), [](const Cand& u, const Cand& v) { return u.score > v.score; });
    const double r2 = (double)c.exclusion_radius * c.exclusion_radius;
    std::vector<size_t> taken;
    auto near_taken = [&](const Cand& q, size_t upto) {
      for (size_t u = 0; u < upto; ++u) {
        const double dx = (double)q.x - cd_[taken[u]].x, dy = (double)q.y - cd_[taken[u]].y;
        if (dx * dx + dy * dy <= r2) return true;
      }
      return false;
    };
    size_t next = cd_.size();
    for (size_t k = 0; k < cd_.size(); ++k) {
      if (near_taken(cd_[k], taken.size())) continue;
      if ((int)taken.size() >= c.topk) { next = k; break; }
      taken.push_back(k);
    }
    for (size_t u = 0; u < taken.size(); ++u) {
      const Cand& q = cd_[taken[u]];
      gisspa_pick pk{};
      pk.score = (float)q.score; pk.x = q.x; pk.y = q.y;
      pk.angle = angles[q.angle]; pk.theta = angles[q.angle]; pk.template_id = n; pk.window = q.window;
      pk.tile = q.tile; pk.angle_index = q.angle; pk.chunk = (int)u;
      out.push_back(pk);
      // margin: the peak's own pixel competitor, the other not-yet-excluded peaks within the
      // radius, and for the last pick the peak a larger K would take next
      double m = q.pos_margin;
      for (size_t k = 0; k < cd_.size(); ++k) {
        if (k == taken[u]) continue;
        const double dx = (double)cd_[k].x - q.x, dy = (double)cd_[k].y - q.y;
        if (dx * dx + dy * dy > r2 || near_taken(cd_[k], u)) continue;
        m = std::min(m, std::fabs(q.score - cd_[k].score));
      }
      if (u + 1 == taken.size() && next < cd_.size()) m = std::min(m, q.score - cd_[next].score);
      margins.push_back(m);
    }
  }
  if (margin_out && !margins.empty())
    std::memcpy(margin_out, margins.data(), sizeof(double) * std::min(cap, margins.size()));
  *n_out = out.size();
  if (out.size() > cap) return GISSPA_ERR_CAPACITY;
  if (!out.empty()) std::memcpy(picks, out.data(), sizeof(gisspa_pick) * out.size());
  return GISSPA_OK;
}

int orc_num_threads(void) { return omp_get_max_threads(); }

// Projection of a volume [nz][ny][nx] along Euler angles (alt, az, phi; radians) as the
// reference's emdata::project3d (EMReader/emdata.cpp:891-996) computes it, with its
// translation (dx, dy) zero and its depth the volume's (the members it reads; see the
// projection harness oracle/ref_project_main.cpp):
//  * the rotation matrix in double from C's double cos/sin, stored as float (emdata.cpp:913-921);
//  * mask radius rmax = ri (nx/2 when ri <= 0), sphere r^2 >= i^2 + j^2 + k^2 in float, i and j
//    over [-rmax + 0.5, rmax + 0.5) truncated and clamped to [-n/2, n/2] (emdata.cpp:934-939);
//  * the in-plane source coordinates are truncated to int (x2, y2 are int at emdata.cpp:899),
//    so of the trilinear weights only the one along z survives: (1 - v) p(z) + v p(z + 1)
//    in double (emdata.h:173-179), added in float to the output pixel, k ascending.
int orc_project3d(const float* vol, int nx, int ny, int nz, const float* angles, int n, int ri, float* out) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || n < 0) return GISSPA_ERR_ARG;
  int rmax = int((float)ri * 1.0f + 0.5);
  if (rmax <= 0) rmax = nx / 2;
  const float r2 = (float)(rmax * rmax);
  int jmin = int(-rmax + 0.0f + 0.5), jmax = int(rmax + 0.0f + 0.5);
  int imin = int(-rmax + 0.0f + 0.5), imax = int(rmax + 0.0f + 0.5);
  jmin = std::max(jmin, -ny / 2);
  jmax = std::min(jmax, ny / 2);
  imin = std::max(imin, -nx / 2);
  imax = std::min(imax, nx / 2);
  const long long xy = (long long)nx * ny;
#pragma omp parallel for schedule(dynamic)
  for (int q = 0; q < n; ++q) {
    const float alt = angles[3 * q], az = angles[3 * q + 1], phi = angles[3 * q + 2];
    float m[9];
    m[0] = (float)(cos((double)phi) * cos((double)az) - cos((double)alt) * sin((double)az) * sin((double)phi));
    m[1] = (float)(-(sin((double)phi) * cos((double)az) + cos((double)alt) * sin((double)az) * cos((double)phi)));
    m[2] = (float)(sin((double)alt) * sin((double)az));
    m[3] = (float)(cos((double)phi) * sin((double)az) + cos((double)alt) * cos((double)az) * sin((double)phi));
    m[4] = (float)(-sin((double)phi) * sin((double)az) + cos((double)alt) * cos((double)az) * cos((double)phi));
    m[5] = (float)(-sin((double)alt) * cos((double)az));
    m[6] = (float)(sin((double)alt) * sin((double)phi));
    m[7] = (float)(sin((double)alt) * cos((double)phi));
    m[8] = (float)cos((double)alt);
    float* o = out + (size_t)q * xy;
    std::fill(o, o + xy, 0.0f);
    for (int k = -rmax; k < rmax; ++k) {
      const float kz = (float)k;
      for (int j = jmin; j < jmax; ++j) {
        const float jy = (float)j;
        for (int i = imin; i < imax; ++i) {
          const float ix = (float)i;
          if (r2 < ix * ix + jy * jy + kz * kz) continue;
          const int x2 = (int)(m[0] * ix + m[1] * jy + m[2] * kz + (float)(nx / 2));
          const int y2 = (int)(m[3] * ix + m[4] * jy + m[5] * kz + (float)(ny / 2));
          const float z2 = m[6] * ix + m[7] * jy + m[8] * kz + (float)(nz / 2);
          if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= nx - 1 || y2 >= ny - 1 || z2 >= nz - 1) continue;
          const int z = (int)z2;
          const float v = z2 - (float)z;
          const long long ii = x2 + (long long)y2 * nx + (long long)z * xy;
          const double s = (1.0 - (double)v) * (double)vol[ii] + (double)v * (double)vol[ii + xy];
          o[(size_t)(j + ny / 2) * nx + i + nx / 2] += (float)s;
        }
      }
    }
  }
  return GISSPA_OK;
}

}  // extern "C"
