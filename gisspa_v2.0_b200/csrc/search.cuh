// search.cuh — the search handle and the per-micrograph orchestration.
#pragma once

#include <functional>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/gisspa.h"
#include "common.cuh"
#include "correlate.cuh"
#include "fft_generic.cuh"

namespace gisspa {
// Correlation launch shape chosen by the autotuner for one (window size, epilogue, precision).
struct TuneChoice {
  int variant = 0, D = 1, E = 1;
  double us_per_pair = 0;
  int a_variant = 0;  // pass A shape
};

// One norm_type=1 search between its phases: preparation, sweeps over angle ranges, the
// normalisation statistics, picks.  Kept in the handle so that the sharded entry points
// (one angle range per rank, state merged by the caller's collective) can resume it.
struct NormRun {
  int phase = 0;  // 0 none, 1 prepared, 2 sweep 1 done (this rank's range), 3 statistics in place,
                  // 4 sweep 2 done
  int nx = 0, ny = 0, W = 0, bx = 0;
  long long N = 0;
  size_t npix = 0;
  std::vector<int> ox, oy;
  std::vector<float> angles;
  double Ntot = 0;
  bool topk = false;
  bool prune = false;  // sweep 2 skips the rows and pairs that cannot hold a pick (search_norm only)
  int n_angles = 0;
  std::vector<std::vector<int>> live_templates;  // pruned second sweep: per angle, host copy
  int D = 1, E = 1;
  CorrArgs args{};
  long long pairs = 0;
  std::vector<Cand> cand;  // sweep 2 candidates of the last range, reference order
  bool angle_table_ready = false;
  std::vector<AngleState> angle_table;  // host copy, alive while its upload is in flight
};

// One angle's launches of a sweep captured as a CUDA graph: the angle comes from a device
// cursor advanced by the graph's first node, so replaying it walks the angle sequence.
struct AngleGraph {
  std::vector<unsigned char> key;   // shapes, buffer addresses and epilogue arguments captured
  unsigned long long generation = 0;  // alloc_generation() at capture
  cudaGraphExec_t exec = nullptr;
  long long launches = 0, pairs = 0;  // kernels and (window, template) pairs per replay
};
}  // namespace gisspa

struct gisspa_handle {
  gisspa_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // the serial LoadImage statistics overlap template preparation here
  cudaEvent_t ev[8] = {};
  cudaEvent_t ev_in = nullptr, ev_stats = nullptr;
  std::string err;
  gisspa::FftEngine fft;

  // template stack (device copy of the caller's array)
  gisspa::DevBuf d_stack;
  int nt = 0, tw = 0, th = 0;
  bool templates_ready = false;

  // template preparation
  gisspa::DevBuf tb, tb_tmp, prep_real, table, tspec;
  // per-angle rotation
  gisspa::DevBuf rot, rot_tmp, rsums;
  // micrograph and windows
  gisspa::DevBuf img_in, img_c, img_tmp, img_pre, tile_real;
  gisspa::DevBuf win_c, win_tmp, win_real, ispec;
  gisspa::DevBuf offx, offy;
  // shells, statistics
  gisspa::DevBuf ra, rb, stats, scratch;
  // per-window-pixel state
  gisspa::DevBuf S1, S2, peak, musig;
  // correlation intermediate and outputs
  gisspa::DevBuf Q, cand, cand_count, nn_key, nn_sum, zkey, zcand, zcount;
  gisspa::DevBuf alive, alive_count, pair_max;  // rows and pairs sweep 2 transforms (prune_sweep2)
  gisspa::DevBuf prep_sub, tspec_sub, list_dev;  // the live templates of an angle of that sweep
  gisspa::DevBuf engine_ctr;  // work counters of the pair engine, one block per launch of a sequence
  gisspa::DevBuf gen_z, gen_x;  // workspace of the generic correlation (window sizes without tuned kernels)
  gisspa::DevBuf dev_err;  // set by kernels whose bounded waits gave up
  // adjoint: whitened template spectra before weighting, RMS factors, dW/dpsi tables,
  // d(prepared template)/dpsi, window RMS factors and sums
  gisspa::DevBuf tw_spec, tmpl_m, dtab, dprep, win_m, win_sum, grad_in, grad_out;
  gisspa::DevBuf prep_lp, dprep_lp, lp_scale;  // adjoint templates at the FP16 / BF16 precision
  // batches: the next micrograph's upload and LoadImage statistics run while the current one's
  // first sweep is on the GPU (gisspa_search_batch)
  gisspa::DevBuf img_next, stats_next, scratch_next;
  cudaEvent_t ev_next = nullptr;
  const float* next_dev = nullptr;  // device image whose statistics wait in stats_next
  int next_nx = 0, next_ny = 0;
  std::function<void()> after_sweep1;
  bool keep_whitened = false;
  int last_nx = 0, last_ny = 0, last_W = 0, last_bx = 0;
  gisspa_ctf last_ctf{};
  std::vector<int> last_offx, last_offy;
  std::vector<float> last_angles;
  gisspa::NormRun run;  // the norm_type=1 search in progress (sharded entry points)
  gisspa::DevBuf proj_vol, proj_mx, proj_out;  // template generation
  // CUDA-graph replay of the sweeps' angles
  std::vector<gisspa::AngleGraph> graphs;
  gisspa::DevBuf angle_table, angle_cursor, angle_cur;
  bool capturing = false;

  gisspa_stats st{};
  std::map<long long, gisspa::TuneChoice> tuned;
  gisspa::DevBuf tune_scratch;
  // sampled per-launch timing of the correlation kernels
  static constexpr int kSamples = 64;
  cudaEvent_t sev[kSamples][3] = {};
  int sample_pairs[kSamples] = {}, sample_d[kSamples] = {};
  int n_samples = 0;
  long long launch_index = 0;
  // events around whole runs of correlation launches (no event between the two passes)
  static constexpr int kSeqs = 16;
  cudaEvent_t qev[kSeqs][2] = {};
  long long seq_launches[kSeqs] = {}, seq_pairs[kSeqs] = {}, seq_d[kSeqs] = {};
  bool seq_pruned[kSeqs] = {};  // a sweep-2 run that skipped rows: not the full work per pair
  int n_seqs = 0;

  ~gisspa_handle() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& r : sev)
      for (auto& e : r)
        if (e) cudaEventDestroy(e);
    for (auto& r : qev)
      for (auto& e : r)
        if (e) cudaEventDestroy(e);
    if (ev_next) cudaEventDestroy(ev_next);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_stats) cudaEventDestroy(ev_stats);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace gisspa {

// Shape / parameter checks (the reference has none; norm.cu:222-224 needs l^2 % 256 == 0).
int validate_config(const gisspa_config& c, std::string& err);
int validate_image(const gisspa_config& c, int nx, int ny, std::string& err);

struct TimeoutError {
  std::string where;
};

// Runs fn, turning CUDA and allocation failures into status codes + h->err.
template <typename F>
int guarded(gisspa_handle* h, F&& fn) {
  try {
    fn();
    return GISSPA_OK;
  } catch (const TimeoutError& e) {
    h->err = "a bounded device wait gave up in " + e.where;
    return GISSPA_ERR_TIMEOUT;
  } catch (const CudaError& e) {
    h->err = std::string(cudaGetErrorString(e.code)) + " at " + e.where;
    cudaGetLastError();
    return e.code == cudaErrorMemoryAllocation ? GISSPA_ERR_NOMEM : GISSPA_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    h->err = "out of host memory";
    return GISSPA_ERR_NOMEM;
  }
}

void run_search(gisspa_handle* h, const float* d_img, int nx, int ny, const gisspa_ctf& ctf,
                std::vector<gisspa_pick>& out);
// Sharded norm_type=1 search (see gisspa_shard_* in gisspa.h).
void shard_begin(gisspa_handle* h, const float* d_img, int nx, int ny, const gisspa_ctf& ctf,
                 gisspa_shard_info* info);
void shard_sweep(gisspa_handle* h, int sweep, int a0, int a1);
void shard_export(gisspa_handle* h, double* sum, double* sum_sq, long long* peak_key);
void shard_import(gisspa_handle* h, const double* sum, const double* sum_sq, const long long* peak_key);
void shard_picks(gisspa_handle* h, std::vector<gisspa_pick>& out);
// Projections of a host volume at host angles into device memory d_out (n x ny x nx).
void project_run(gisspa_handle* h, const float* volume, int nx, int ny, int nz, const float* angles, int n, int ri,
                 float* d_out);
// Bounded device wait that is made to run out (gisspa_debug_wait_probe); throws TimeoutError.
void wait_probe(gisspa_handle* h, double seconds);
int run_batch(gisspa_handle* h, int n, const float* const* images, const int* nx, const int* ny,
              const gisspa_ctf* ctfs, gisspa_pick* picks, size_t cap, size_t* offsets);

void debug_stage(gisspa_handle* h, int what, const float* d_img, int nx, int ny, const gisspa_ctf& ctf, float theta,
                 void* out, size_t bytes);
void cc_maps(gisspa_handle* h, const void* d_win, int nw, const void* d_t, int ntm, int spec, float* d_out);
void score_grad_run(gisspa_handle* h, const gisspa_pick* picks, size_t n, const float* params, const gisspa_ctf* ctf,
                    gisspa_grad* out);
void refine_run(gisspa_handle* h, gisspa_pick* picks, size_t n, int steps, gisspa_ctf* ctf, float* params_out);

// Window offsets along one axis (blocks_one_axis, norm.cu:68-81).
std::vector<int> window_offsets(int len, int l, int ov);
// Window count along one axis for norm_type=0 (nonorm.cu:71-81).
int window_count_nonorm(int len, int l, int ov);
// Float-stepped angle sequence: for (float e = 0; e < 360; e += step) (norm.cu:684).
std::vector<float> angle_list(float step);

}  // namespace gisspa
