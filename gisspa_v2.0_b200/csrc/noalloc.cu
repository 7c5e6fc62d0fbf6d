// noalloc.cu — correlation maps without any device allocation.
//
// gisspa_cc_maps (api.cu) keeps its correlation intermediate and twiddle tables in
// memory the handle allocates with cudaMalloc.  Some callers cannot allocate
// device memory at all: code running under a memory pool or budget that another
// framework owns, a process whose allocator is locked down, or a caller that must
// not add allocations to a stream it captures.  This entry point serves them: the
// intermediate and the twiddle tables live in fixed file-scope __device__ arrays
// that every GPU loading the library holds until the process exits, and the call
// makes no cudaMalloc, cudaFree or other allocating call.
#include <cmath>
#include <exception>
#include <mutex>
#include <string>

#include "../../include/gisspa.h"
#include "common.cuh"
#include "correlate.cuh"

namespace gisspa {
namespace {

// Intermediate of the column pass: 16 MiB (every (window, template) pair of one call).
constexpr size_t kNoAllocScratchBytes = 16u << 20;
static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocScratchBytes / sizeof(float2)];
// Twiddle tables exp(-2 pi i p / n) for n = 1024, 512, 256, 128, back to back.
constexpr int kTwTotal = 1024 + 512 + 256 + 128;
static __device__ __align__(256) float2 g_noalloc_twiddles[kTwTotal];
// Set by a kernel whose bounded wait gave up.  Every call zeroes it on its stream before
// its launches and reads it back after them.
static __device__ unsigned g_noalloc_flag;

int tw_offset(int n) { return n == 1024 ? 0 : n == 512 ? 1024 : n == 256 ? 1536 : 1792; }

struct DeviceSlot {
  bool ready = false;
  float2* scratch = nullptr;
  float2* twiddles = nullptr;
  unsigned* flag = nullptr;
};
std::mutex g_mu;
DeviceSlot g_slots[64];

// Per-device set-up, run by the first call on each device with that device current:
// resolve the arrays' device addresses (their host-side names are only stand-ins) and
// fill the twiddle tables.
int setup(int dev, std::string& err) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceSlot& s = g_slots[dev];
  if (s.ready) return GISSPA_OK;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
    return GISSPA_ERR_CUDA;
  }
  s.scratch = static_cast<float2*>(p);
  e = cudaGetSymbolAddress(&p, g_noalloc_twiddles);
  if (e != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress(twiddles): ") + cudaGetErrorString(e);
    return GISSPA_ERR_CUDA;
  }
  s.twiddles = static_cast<float2*>(p);
  e = cudaGetSymbolAddress(&p, g_noalloc_flag);
  if (e != cudaSuccess) {
    err = std::string("cudaGetSymbolAddress(flag): ") + cudaGetErrorString(e);
    return GISSPA_ERR_CUDA;
  }
  s.flag = static_cast<unsigned*>(p);
  float2 h[kTwTotal];
  for (int n : {1024, 512, 256, 128})
    for (int k = 0; k < n; ++k) {
      const double a = -2.0 * kPi * (double)k / n;
      h[tw_offset(n) + k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  e = cudaMemcpy(s.twiddles, h, sizeof(h), cudaMemcpyHostToDevice);
  // A copy from pageable memory may return before its DMA lands; a kernel on a caller's
  // non-blocking stream would not be ordered after it, so wait for the device here (once).
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    err = std::string("twiddle upload: ") + cudaGetErrorString(e);
    return GISSPA_ERR_CUDA;
  }
  s.ready = true;
  return GISSPA_OK;
}

}  // namespace

// Error text readable through gisspa_last_error(NULL) (api.cu).
void set_handleless_error(const std::string& msg);

}  // namespace gisspa

using namespace gisspa;

static int cc_maps_noalloc(const void* d_windows, int n_windows, const void* d_templates, int n_templates,
                           int window_size, int spec, float* d_out, void* stream, std::string& err) {
  if (!d_windows || !d_templates || !d_out || n_windows <= 0 || n_templates <= 0 || spec < 0 || spec > 2) {
    err = "cc_maps_noalloc: bad argument";
    return GISSPA_ERR_ARG;
  }
  const int L = window_size;
  if (!correlate_supported(L)) {
    err = "cc_maps_noalloc: window_size must be 256, 512 or 1024";
    return GISSPA_ERR_SHAPE;
  }
  const size_t need = (size_t)n_windows * n_templates * (L / 2) * L * sizeof(float2);
  if (need > kNoAllocScratchBytes) {
    err = "cc_maps_noalloc: " + std::to_string(n_windows) + " x " + std::to_string(n_templates) +
          " pairs of window_size " + std::to_string(L) + " need " + std::to_string(need >> 10) +
          " KiB of scratch; the fixed scratch holds " + std::to_string(kNoAllocScratchBytes >> 10) +
          " KiB (split the call)";
    return GISSPA_ERR_CAPACITY;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    err = "cc_maps_noalloc: no current device";
    return GISSPA_ERR_CUDA;
  }
  int st = setup(dev, err);
  if (st) return st;
  const DeviceSlot& ds = g_slots[dev];
  CorrArgs args{};
  args.Q = ds.scratch;
  args.b0 = 0;
  args.n0 = 0;
  args.D = n_templates;
  args.nt_real = n_templates;
  args.nt_total = n_templates;
  args.map_out = d_out;
  args.err = ds.flag;
  CorrLaunch cl{L, n_windows, n_templates, spec, EPI_MAP, 0};
  const cudaStream_t cs = static_cast<cudaStream_t>(stream);
  try {
    // The flag keeps the previous call's value: clear it on this call's stream first.
    GISSPA_CUDA(cudaMemsetAsync(ds.flag, 0, sizeof(unsigned), cs));
    correlate_launch(cl, static_cast<const float2*>(d_windows), d_templates, ds.scratch, args,
                     ds.twiddles + tw_offset(L), ds.twiddles + tw_offset(L / 2), cs);
    // A row kernel whose bounded wait for its slice of the intermediate gave up leaves its
    // maps partly unwritten: wait for the launches and report that as a timeout.
    GISSPA_CUDA(cudaStreamSynchronize(cs));
    unsigned flag = 0;
    GISSPA_CUDA(cudaMemcpy(&flag, ds.flag, sizeof(flag), cudaMemcpyDeviceToHost));
    if (flag) {
      err = "cc_maps_noalloc: a bounded wait inside the correlation kernels gave up (GPU overloaded or "
            "stalled); the maps are incomplete";
      return GISSPA_ERR_TIMEOUT;
    }
  } catch (const CudaError& ce) {
    err = std::string(cudaGetErrorString(ce.code)) + " at " + ce.where;
    return GISSPA_ERR_CUDA;
  } catch (const std::exception& ex) {
    err = std::string("cc_maps_noalloc: ") + ex.what();
    return GISSPA_ERR_CUDA;
  }
  return GISSPA_OK;
}

extern "C" int gisspa_cc_maps_noalloc(const void* d_windows, int n_windows, const void* d_templates, int n_templates,
                                      int window_size, int spec, float* d_out, void* stream) {
  std::string err;
  int st;
  try {
    st = cc_maps_noalloc(d_windows, n_windows, d_templates, n_templates, window_size, spec, d_out, stream, err);
  } catch (...) {  // nothing may unwind through the C ABI
    err = "cc_maps_noalloc: unexpected exception";
    st = GISSPA_ERR_CUDA;
  }
  if (st) set_handleless_error(err);
  return st;
}
