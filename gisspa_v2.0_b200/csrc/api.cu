// api.cu — the C-ABI (include/gisspa.h) and the per-micrograph orchestration.
//
// One handle owns one CUDA stream and every device buffer; buffers grow on demand
// and are reused across micrographs (the reference rebuilds its search object and
// cuFFT plans for every micrograph, main.cu:42).  Nothing here falls back to the
// CPU: every numeric stage runs in this library's kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/gisspa.h"
#include "common.cuh"
#include "correlate.cuh"
#include "fft_generic.cuh"
#include "prep.cuh"
#include "search.cuh"

namespace {
thread_local std::string g_create_error;
const char* kVersion = "gisspa-b200 0.1 (sm_100a)";
}  // namespace

namespace gisspa {
long long& launch_counter() {
  static thread_local long long c = 0;
  return c;
}
void set_handleless_error(const std::string& msg) { g_create_error = msg; }
}  // namespace gisspa

using namespace gisspa;

extern "C" {

void gisspa_config_default(gisspa_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  // EMReader/DataReader2.h:19-44
  c->angpix = -1.f; c->phistep = -1.f; c->kk = -1.f; c->energy = -1.f; c->cs = -1.f;
  c->highres = -1.f; c->lowres = 0.f; c->diameter = -1.f; c->threshold = 7.f;
  c->window_size = 320; c->overlap = 0; c->norm_type = 0; c->invert = 0; c->phase_flip = 0;
  // DataReader2.h:73-77
  c->edge_half_width = 4.f; c->ampconst = 0.07f;
  c->a = -10.81f; c->b = 1.f; c->b2 = 0.32f; c->bfactor = -18.17f; c->bfactor2 = -15.22f; c->bfactor3 = 1.72f;
  c->pick_mode = GISSPA_PICK_CHUNK; c->topk = 1000; c->exclusion_radius = 64.f;
  c->spectrum_precision = GISSPA_SPEC_FP32; c->template_batch = 0; c->window_batch = 0;
  c->quirks = GISSPA_QUIRKS_REFERENCE; c->tile_size = 720;
  c->cuda_graphs = 1;
  c->pass_b_shape = -1;
  c->tensor_cores = 0;
  c->pass_a_shape = -1;
  c->prune_sweep2 = 1;
}

int gisspa_create(const gisspa_config* cfg, int device, gisspa_handle** out) {
  if (!cfg || !out) {
    g_create_error = "null argument";
    return GISSPA_ERR_ARG;
  }
  *out = nullptr;
  auto* h = new (std::nothrow) gisspa_handle();
  if (!h) {
    g_create_error = "out of host memory";
    return GISSPA_ERR_NOMEM;
  }
  h->cfg = *cfg;
  h->device = device;
  int st = validate_config(h->cfg, h->err);
  if (st) {
    g_create_error = h->err;
    delete h;
    return st;
  }
  try {
    int n = 0;
    GISSPA_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) {
      g_create_error = "device " + std::to_string(device) + " not present (" + std::to_string(n) + " devices)";
      delete h;
      return GISSPA_ERR_ARG;
    }
    GISSPA_CUDA(cudaSetDevice(device));
    GISSPA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    GISSPA_CUDA(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    GISSPA_CUDA(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
    GISSPA_CUDA(cudaEventCreateWithFlags(&h->ev_stats, cudaEventDisableTiming));
    GISSPA_CUDA(cudaEventCreateWithFlags(&h->ev_next, cudaEventDisableTiming));
    for (auto& e : h->ev) GISSPA_CUDA(cudaEventCreate(&e));
    for (auto& r : h->sev)
      for (auto& e : r) GISSPA_CUDA(cudaEventCreate(&e));
    for (auto& r : h->qev)
      for (auto& e : r) GISSPA_CUDA(cudaEventCreate(&e));
  } catch (const CudaError& e) {
    g_create_error = std::string(cudaGetErrorString(e.code)) + " at " + e.where;
    delete h;
    return GISSPA_ERR_CUDA;
  }
  *out = h;
  return GISSPA_OK;
}

void gisspa_destroy(gisspa_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h;
}

const char* gisspa_last_error(const gisspa_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

const char* gisspa_version(void) { return kVersion; }

int gisspa_get_stats(const gisspa_handle* h, gisspa_stats* out) {
  if (!h || !out) return GISSPA_ERR_ARG;
  *out = h->st;
  return GISSPA_OK;
}

int gisspa_set_templates(gisspa_handle* h, const float* stack, int n, int width, int height) {
  if (!h) return GISSPA_ERR_ARG;
  if (!stack || n <= 0 || width <= 0 || height <= 0) {
    h->err = "set_templates: empty template stack";
    return GISSPA_ERR_ARG;
  }
  if (width > h->cfg.window_size || height > h->cfg.window_size) {
    h->err = "set_templates: template " + std::to_string(width) + "x" + std::to_string(height) +
             " larger than window_size " + std::to_string(h->cfg.window_size);
    return GISSPA_ERR_SHAPE;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(float) * (size_t)n * width * height;
    h->d_stack.ensure(bytes);
    GISSPA_CUDA(cudaMemcpy(h->d_stack.as<float>(), stack, bytes, cudaMemcpyHostToDevice));
    h->nt = n;
    h->tw = width;
    h->th = height;
    h->templates_ready = true;
  });
}

int gisspa_search_device(gisspa_handle* h, const float* d_image, int nx, int ny, const gisspa_ctf* ctf,
                         gisspa_pick* picks, size_t cap, size_t* n_out) {
  if (!h) return GISSPA_ERR_ARG;
  if (!d_image || !ctf || !n_out || (cap && !picks)) {
    h->err = "search: null argument";
    return GISSPA_ERR_ARG;
  }
  if (!h->templates_ready) {
    h->err = "search: gisspa_set_templates has not been called";
    return GISSPA_ERR_STATE;
  }
  int st = validate_image(h->cfg, nx, ny, h->err);
  if (st) return st;
  std::vector<gisspa_pick> out;
  st = guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    run_search(h, d_image, nx, ny, *ctf, out);
  });
  if (st) return st;
  *n_out = out.size();
  if (out.size() > cap) {
    h->err = "search: " + std::to_string(out.size()) + " picks exceed capacity " + std::to_string(cap);
    return GISSPA_ERR_CAPACITY;
  }
  if (!out.empty()) std::memcpy(picks, out.data(), sizeof(gisspa_pick) * out.size());
  return GISSPA_OK;
}

int gisspa_search(gisspa_handle* h, const float* image, int nx, int ny, const gisspa_ctf* ctf, gisspa_pick* picks,
                  size_t cap, size_t* n_out) {
  if (!h) return GISSPA_ERR_ARG;
  if (!image) {
    h->err = "search: null image";
    return GISSPA_ERR_ARG;
  }
  int st = validate_image(h->cfg, nx, ny, h->err);
  if (st) return st;
  st = guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(float) * (size_t)nx * ny;
    h->img_in.ensure(bytes);
    GISSPA_CUDA(cudaMemcpyAsync(h->img_in.as<float>(), image, bytes, cudaMemcpyHostToDevice, h->stream));
  });
  if (st) return st;
  return gisspa_search_device(h, h->img_in.as<float>(), nx, ny, ctf, picks, cap, n_out);
}

// ---- sharded search (one micrograph across ranks)
namespace {
int shard_check(gisspa_handle* h, const char* what, int need_min, int need_max) {
  if (!h) return GISSPA_ERR_ARG;
  if (h->cfg.norm_type == 0) {
    h->err = std::string(what) + ": the sharded search is defined for norm_type=1";
    return GISSPA_ERR_UNSUPPORTED;
  }
  if (h->run.phase < need_min || h->run.phase > need_max) {
    h->err = std::string(what) + ": called out of order (phase " + std::to_string(h->run.phase) + ")";
    return GISSPA_ERR_STATE;
  }
  return GISSPA_OK;
}
}  // namespace

int gisspa_shard_begin(gisspa_handle* h, const float* image, int nx, int ny, const gisspa_ctf* ctf,
                       gisspa_shard_info* info) {
  int st = shard_check(h, "shard_begin", 0, 4);
  if (st) return st;
  if (!image || !ctf || !info) {
    h->err = "shard_begin: null argument";
    return GISSPA_ERR_ARG;
  }
  if (!h->templates_ready) {
    h->err = "shard_begin: gisspa_set_templates has not been called";
    return GISSPA_ERR_STATE;
  }
  st = validate_image(h->cfg, nx, ny, h->err);
  if (st) return st;
  h->run.phase = 0;
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    const size_t bytes = sizeof(float) * (size_t)nx * ny;
    h->img_in.ensure(bytes);
    GISSPA_CUDA(cudaMemcpyAsync(h->img_in.as<float>(), image, bytes, cudaMemcpyHostToDevice, h->stream));
    shard_begin(h, h->img_in.as<float>(), nx, ny, *ctf, info);
  });
}

int gisspa_shard_sweep(gisspa_handle* h, int sweep, int angle_begin, int angle_end) {
  if (!h) return GISSPA_ERR_ARG;
  if (sweep != 1 && sweep != 2) {
    h->err = "shard_sweep: sweep must be 1 or 2";
    return GISSPA_ERR_ARG;
  }
  int st = sweep == 1 ? shard_check(h, "shard_sweep", 1, 2) : shard_check(h, "shard_sweep", 3, 4);
  if (st) return st;
  if (sweep == 2 && h->run.topk) {
    h->err = "shard_sweep: top-K picking has no second sweep";
    return GISSPA_ERR_STATE;
  }
  const int A = (int)h->run.angles.size();
  if (angle_begin < 0 || angle_end > A || angle_begin > angle_end) {
    h->err = "shard_sweep: angle range [" + std::to_string(angle_begin) + ", " + std::to_string(angle_end) +
             ") outside [0, " + std::to_string(A) + ")";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    shard_sweep(h, sweep, angle_begin, angle_end);
  });
}

int gisspa_shard_export(gisspa_handle* h, double* sum, double* sum_sq, long long* peak_key) {
  int st = shard_check(h, "shard_export", 1, 2);
  if (st) return st;
  if (!sum || !sum_sq || (h->run.topk && !peak_key)) {
    h->err = "shard_export: null argument";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    shard_export(h, sum, sum_sq, peak_key);
  });
}

int gisspa_shard_import(gisspa_handle* h, const double* sum, const double* sum_sq, const long long* peak_key) {
  int st = shard_check(h, "shard_import", 1, 2);
  if (st) return st;
  if (!sum || !sum_sq || (h->run.topk && !peak_key)) {
    h->err = "shard_import: null argument";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    shard_import(h, sum, sum_sq, peak_key);
  });
}

int gisspa_shard_picks(gisspa_handle* h, gisspa_pick* picks, size_t cap, size_t* n_out) {
  if (!h) return GISSPA_ERR_ARG;
  int st = h->run.topk ? shard_check(h, "shard_picks", 3, 3) : shard_check(h, "shard_picks", 4, 4);
  if (st) return st;
  if (!n_out || (cap && !picks)) {
    h->err = "shard_picks: null argument";
    return GISSPA_ERR_ARG;
  }
  std::vector<gisspa_pick> out;
  st = guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    shard_picks(h, out);
  });
  if (st) return st;
  *n_out = out.size();
  if (out.size() > cap) {
    h->err = "shard_picks: " + std::to_string(out.size()) + " picks exceed capacity " + std::to_string(cap);
    return GISSPA_ERR_CAPACITY;
  }
  if (!out.empty()) std::memcpy(picks, out.data(), sizeof(gisspa_pick) * out.size());
  return GISSPA_OK;
}

int gisspa_search_batch(gisspa_handle* h, int n, const float* const* images, const int* nx, const int* ny,
                        const gisspa_ctf* ctfs, gisspa_pick* picks, size_t cap, size_t* offsets) {
  if (!h) return GISSPA_ERR_ARG;
  if (n < 0 || (n && (!images || !nx || !ny || !ctfs)) || !offsets) {
    h->err = "search_batch: null argument";
    return GISSPA_ERR_ARG;
  }
  for (int i = 0; i < n; ++i) {
    if (!images[i]) {
      h->err = "search_batch: null image " + std::to_string(i);
      return GISSPA_ERR_ARG;
    }
    int st = validate_image(h->cfg, nx[i], ny[i], h->err);
    if (st) return st;
  }
  return run_batch(h, n, images, nx, ny, ctfs, picks, cap, offsets);
}

int gisspa_score_grad(gisspa_handle* h, const gisspa_pick* picks, size_t n, const float* params,
                      const gisspa_ctf* ctf, gisspa_grad* out) {
  if (!h) return GISSPA_ERR_ARG;
  if ((n && (!picks || !out))) {
    h->err = "score_grad: null argument";
    return GISSPA_ERR_ARG;
  }
  if (n == 0) return GISSPA_OK;
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    score_grad_run(h, picks, n, params, ctf, out);
  });
}

int gisspa_refine(gisspa_handle* h, gisspa_pick* picks, size_t n, int steps, gisspa_ctf* ctf, float* params_out) {
  if (!h) return GISSPA_ERR_ARG;
  if ((n && !picks) || steps < 0) {
    h->err = "refine: bad argument";
    return GISSPA_ERR_ARG;
  }
  if (n == 0) return GISSPA_OK;
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    refine_run(h, picks, n, steps, ctf, params_out);
  });
}

int gisspa_cc_maps(gisspa_handle* h, const void* d_windows, int n_windows, const void* d_templates, int n_templates,
                   int spec, float* d_out) {
  if (!h) return GISSPA_ERR_ARG;
  if (!d_windows || !d_templates || !d_out || n_windows <= 0 || n_templates <= 0 || spec < 0 || spec > 2) {
    h->err = "cc_maps: bad argument";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    cc_maps(h, d_windows, n_windows, d_templates, n_templates, spec, d_out);
  });
}

int gisspa_debug_stage(gisspa_handle* h, int what, const float* image, int nx, int ny, const gisspa_ctf* ctf,
                       float theta, void* out, size_t bytes) {
  if (!h) return GISSPA_ERR_ARG;
  if (!out || !ctf) {
    h->err = "debug_stage: null argument";
    return GISSPA_ERR_ARG;
  }
  if (what != GISSPA_STAGE_MUSIG && !h->templates_ready) {
    h->err = "debug_stage: gisspa_set_templates has not been called";
    return GISSPA_ERR_STATE;
  }
  if (image) {
    int st = validate_image(h->cfg, nx, ny, h->err);
    if (st) return st;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    const float* d_img = nullptr;
    if (image) {
      const size_t b = sizeof(float) * (size_t)nx * ny;
      h->img_in.ensure(b);
      GISSPA_CUDA(cudaMemcpyAsync(h->img_in.as<float>(), image, b, cudaMemcpyHostToDevice, h->stream));
      d_img = h->img_in.as<float>();
    }
    debug_stage(h, what, d_img, nx, ny, *ctf, theta, out, bytes);
  });
}

int gisspa_format_pick(const gisspa_pick* p, int lst_index, const char* path, const gisspa_ctf* ctf, float euler1,
                       float euler2, char* buf, size_t cap) {
  if (!p || !buf || !ctf) return -1;
  // OutputScore (norm.cu:610-614): defocus printed with its original sign
  int n = std::snprintf(buf, cap,
                        "%d\t%s\tdefocus=%f\tdfdiff=%f\tdfang=%f\teuler=%f,%f,%f\tcenter=%f,%f\tscore=%f\n",
                        lst_index, path ? path : "", (float)ctf->defocus, (float)ctf->dfdiff, (float)ctf->dfang,
                        euler1, euler2, p->angle, p->x, p->y, p->score);
  if (n < 0 || (size_t)n >= cap) return -1;
  return n;
}

namespace {
int check_projection(gisspa_handle* h, const char* what, const float* volume, int nx, int ny, int nz,
                     const float* angles, int n, int ri) {
  if (!volume || !angles || n <= 0 || nx < 2 || ny < 2 || nz < 2 || ri < 0) {
    h->err = std::string(what) + ": need a volume of at least 2^3, n > 0 angles and ri >= 0";
    return GISSPA_ERR_ARG;
  }
  if ((long long)nx * ny * nz > (1LL << 31) || (long long)n * nx * ny > (1LL << 31)) {
    h->err = std::string(what) + ": volume or projection stack above 2^31 floats";
    return GISSPA_ERR_SHAPE;
  }
  return GISSPA_OK;
}
}  // namespace

int gisspa_project(gisspa_handle* h, const float* volume, int nx, int ny, int nz, const float* angles, int n,
                   int ri, float* out) {
  if (!h) return GISSPA_ERR_ARG;
  int st = check_projection(h, "project", volume, nx, ny, nz, angles, n, ri);
  if (st) return st;
  if (!out) {
    h->err = "project: null output";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    const size_t np = (size_t)n * nx * ny;
    float* d = static_cast<float*>(h->proj_out.ensure(sizeof(float) * np));
    project_run(h, volume, nx, ny, nz, angles, n, ri, d);
    GISSPA_CUDA(cudaMemcpy(out, d, sizeof(float) * np, cudaMemcpyDeviceToHost));
  });
}

int gisspa_set_templates_from_volume(gisspa_handle* h, const float* volume, int nx, int ny, int nz,
                                     const float* angles, int n, int ri) {
  if (!h) return GISSPA_ERR_ARG;
  int st = check_projection(h, "set_templates_from_volume", volume, nx, ny, nz, angles, n, ri);
  if (st) return st;
  if (nx > h->cfg.window_size || ny > h->cfg.window_size) {
    h->err = "set_templates_from_volume: projection " + std::to_string(nx) + "x" + std::to_string(ny) +
             " larger than window_size " + std::to_string(h->cfg.window_size);
    return GISSPA_ERR_SHAPE;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    float* d = static_cast<float*>(h->d_stack.ensure(sizeof(float) * (size_t)n * nx * ny));
    project_run(h, volume, nx, ny, nz, angles, n, ri, d);
    h->nt = n;
    h->tw = nx;
    h->th = ny;
    h->templates_ready = true;
  });
}

int gisspa_debug_wait_probe(gisspa_handle* h, double seconds) {
  if (!h) return GISSPA_ERR_ARG;
  if (!(seconds > 0.0) || seconds > 10.0) {
    h->err = "wait_probe: seconds must lie in (0, 10]";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    wait_probe(h, seconds);
  });
}

int gisspa_debug_fft(gisspa_handle* h, void* data, long long rows, int n, int sign) {
  if (!h) return GISSPA_ERR_ARG;
  if (!data || rows < 0 || n < 1 || n > 16384 || (sign != -1 && sign != 1)) {
    h->err = "debug_fft: data non-null, rows >= 0, 1 <= n <= 16384, sign -1 or +1";
    return GISSPA_ERR_ARG;
  }
  return guarded(h, [&] {
    GISSPA_CUDA(cudaSetDevice(h->device));
    h->fft.rows(static_cast<float2*>(data), rows, n, sign, 1.f, h->stream);
    GISSPA_CUDA(cudaStreamSynchronize(h->stream));
  });
}

}  // extern "C"
