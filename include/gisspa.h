/*
 * gisspa.h — C-ABI of the B200 template-matching search library (libgisspa.so).
 *
 * This is the drop-in boundary for GisSPA's per-micrograph search loop.  Each
 * entry point names the reference interface it replaces (paths are relative to
 * the GisSPA_v2.0 source tree).  All pointers are plain host pointers unless the
 * name says "device"; no CUDA or C++ types cross the boundary.  Every call
 * returns an int status (GISSPA_OK == 0) and never exits the process; the text
 * of the last error is available from gisspa_last_error().
 *
 * Threading: one handle per device.  Calls on one handle are not thread-safe;
 * separate handles are independent.  Each call makes the handle's device
 * current itself (the reference relies on cudaSetDevice in the constructor,
 * norm.cu:64).
 */
#ifndef GISSPA_H
#define GISSPA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference has none: it calls exit(-1), utils.h:24-38) ---- */
enum {
  GISSPA_OK = 0,
  GISSPA_ERR_ARG = 1,         /* null pointer or out-of-range argument */
  GISSPA_ERR_SHAPE = 2,       /* window_size % 16 != 0, window larger than image, ... */
  GISSPA_ERR_UNSUPPORTED = 3, /* accepted by the reference but not by this build */
  GISSPA_ERR_CUDA = 4,        /* CUDA runtime error (text in gisspa_last_error) */
  GISSPA_ERR_NOMEM = 5,       /* device or host allocation failed */
  GISSPA_ERR_CAPACITY = 6,    /* pick buffer too small: *n_out holds the count needed */
  GISSPA_ERR_STATE = 7,       /* call order (search before set_templates, ...) */
  GISSPA_ERR_TIMEOUT = 8,     /* a bounded device wait gave up */
  GISSPA_ERR_IO = 9           /* file could not be read or parsed */
};

/* ---- pick modes ---- */
enum {
  GISSPA_PICK_CHUNK = 0, /* reference picks: two sweeps, one pick per 256-pixel chunk
                            with z >= threshold (norm.cu:554-600) */
  GISSPA_PICK_TOPK = 1   /* norm_type=1: one sweep, per-pixel max z over templates x angles,
                            then greedy top-K with an exclusion radius.  norm_type=0: per
                            template, every (tile, angle, window) peak with a valid centre and
                            score >= threshold, then greedy top-K per template with the
                            exclusion radius; centres in micrograph coordinates (tile
                            offset added), pick.chunk = rank within the template */
};

/* ---- template-spectrum storage precision (FFT arithmetic is FP32 in all cases) ---- */
enum { GISSPA_SPEC_FP32 = 0, GISSPA_SPEC_FP16 = 1, GISSPA_SPEC_BF16 = 2 };

/* ---- reference quirks (bit set = reproduce the reference's behaviour) ---- */
/* LoadImage: mean/sigma by a serial FP32 sum, bounds truncated to int (norm.cu:157-171). */
#define GISSPA_QUIRK_OUTLIER_FP32_SERIAL 0x1
/* Templates beyond N_T (when windows outnumber templates) count in N (norm.cu:91, 550).
   The reference reads past the template array there; this build uses all-zero maps. */
#define GISSPA_QUIRK_COUNT_PADDED_TEMPLATES 0x2
/* N_euler = (int)(360 / phistep) instead of the float-stepped loop count (norm.cu:550, 684). */
#define GISSPA_QUIRK_NEULER_TRUNC 0x4
#define GISSPA_QUIRKS_REFERENCE 0x7

/* Search configuration.  The first block mirrors the reference Config keys
 * (EMReader/DataReader2.h:19-44) and Parameters constants (DataReader2.h:73-77). */
typedef struct gisspa_config {
  float angpix, phistep, kk, energy, cs, highres, lowres, diameter, threshold;
  int window_size, overlap, norm_type, invert, phase_flip;
  float edge_half_width, ampconst, a, b, b2, bfactor, bfactor2, bfactor3;
  /* additions (no counterpart in the reference) */
  int pick_mode;          /* GISSPA_PICK_* */
  int topk;               /* K for GISSPA_PICK_TOPK */
  float exclusion_radius; /* pixels, GISSPA_PICK_TOPK */
  int spectrum_precision; /* GISSPA_SPEC_* */
  int template_batch;     /* templates per correlation pass (0 = automatic) */
  int window_batch;       /* windows per correlation pass (0 = automatic) */
  int quirks;             /* GISSPA_QUIRK_* bits */
  int tile_size;          /* norm_type=0 tile edge; reference constant 720 (utils/constants.h:5) */
  int cuda_graphs;        /* norm_type=1 sweeps: 1 = capture one angle's launches in a CUDA graph and
                             replay it for the other angles, 0 = launch every kernel from the host */
  int pass_b_shape;       /* with template_batch and window_batch set: row-transform kernel shape
                             (0.. compiled shapes - 1; -1 = the first); ignored when autotuning */
  int tensor_cores;       /* 1: with FP16 template spectra at window_size 512 the column transforms
                             of the correlation, and with top-K picking also the row transforms,
                             run on the tensor cores (tcgen05, FP16 operands, FP32 accumulation;
                             same picks, scores within 1.1e-4 of the FP32 form) -- measured 1.7x
                             slower per launch pair than 0 on B200; 0 (default): CUDA cores */
  int pass_a_shape;       /* with template_batch and window_batch set: column-transform kernel shape
                             (0 .. compiled shapes - 1: two at window 512, one elsewhere; -1 = the
                             first); ignored when autotuning */
  int prune_sweep2;       /* norm_type=1 chunk picks at window sizes with hand-tuned kernels: 1
                             (default) = sweep 1 also keeps each pixel's best correlation, and
                             sweep 2 skips the window rows whose best z is below the threshold
                             (they cannot hold a pick for any template or angle: same picks);
                             0 = sweep 2 transforms every row */
} gisspa_config;

/* Per-micrograph CTF, as in an LST line "defocus= dfdiff= dfang=" (DataReader2.h:93-103).
   defocus and dfdiff in micrometres, dfang in degrees. */
typedef struct gisspa_ctf {
  double defocus, dfdiff, dfang;
} gisspa_ctf;

/* One pick.  x, y, angle and score are the values the reference prints in its
 * pick-list line (norm.cu:602-618, nonorm.cu:539-557). */
typedef struct gisspa_pick {
  float score;
  float x, y;      /* centre; tile-local for norm_type=0, as the reference prints it */
  float angle;     /* printed in-plane angle: 360-theta for norm_type=1, theta for 0 */
  int template_id; /* index into the template stack */
  int window;      /* window index i + j*block_x */
  int tile;        /* norm_type=0 tile index (column-major, tileimages.cpp:27-70), else 0 */
  int angle_index; /* index of theta in the float-stepped angle sequence */
  int chunk;       /* chunk pick: 256-pixel chunk within the window; top-K: rank */
  float theta;     /* search angle theta in degrees (before the printed convention) */
} gisspa_pick;

/* Paths and run range of a reference config file (DataReader2.h:19-44). */
typedef struct gisspa_run_paths {
  char input[1024];
  char template_path[1024];
  char eulerfile[1024];
  char output[1024];
  int first, last, gpu_id;
  /* addition: a 3D map (MRC) to project into the templates on the GPU at the Euler file's
     angles (alt, az, phi in degrees), instead of reading a projected stack from `template` */
  char template_volume[1024];
} gisspa_run_paths;

/* Per-call timing and counters. */
typedef struct gisspa_stats {
  double ms_total, ms_prep, ms_sweep1, ms_sweep2, ms_pick;
  long long pairs;            /* window x template x angle correlations evaluated */
  long long kernel_launches;  /* launches of this library's kernels in the last search */
  long long candidates;       /* picks found before the capacity check */
  /* CUDA-event timing of a sample of correlation launches (every 16th launch pair), taken
   * only with cuda_graphs = 0: an event between the two passes breaks their programmatic
   * dependent launch overlap, so these split times are for profiling runs */
  double pass_a_us, pass_b_us; /* mean duration of one pass A / pass B launch */
  double pairs_per_launch;     /* mean (window, template) pairs per launch of the search */
  double templates_per_launch; /* mean template batch depth D per launch of the search */
  int pass_samples;
  int window_size;
  int pass_b_variant;          /* pass B shape picked by the autotuner (last sweep); at window 512
                                  shape 4 is the pair engine (both passes in one launch) */
  double tuned_us_per_pair;    /* autotuner's measured time per pair of that shape */
  long long graph_replays;     /* angles run as replays of a captured CUDA graph */
  /* CUDA events around whole runs of correlation launches (every host-launched angle: the
   * first of each sweep when graphs are on, except a pruned second sweep), nothing recorded
   * between them */
  double corr_pair_us;         /* mean duration of one pass A + pass B launch pair */
  long long corr_timed_launches; /* launch pairs inside those runs */
  int pass_a_variant;          /* pass A shape picked by the autotuner (last sweep) */
  double rows_alive;           /* fraction of window rows sweep 2 transformed (below 1 with
                                  prune_sweep2; 0 when the search has no second sweep; a batch
                                  reports the mean over its micrographs) */
  double pairs_alive;          /* fraction of (window, template, angle) pairs sweep 2 transformed
                                  (same conventions) */
} gisspa_stats;

typedef struct gisspa_handle gisspa_handle;

/* Fill *cfg with the reference defaults (DataReader2.h:19-44, 73-77) plus the
 * defaults of the additions. */
void gisspa_config_default(gisspa_config* cfg);

/* Parse a reference config file ("key = value" tokens, unknown keys ignored;
 * DataReader2.cpp:6-28).  Replaces Config::Config(path).  paths may be NULL. */
int gisspa_config_load(const char* path, gisspa_config* cfg, gisspa_run_paths* paths);

/* Replaces SearchNorm::SearchNorm / SearchNoNorm::SearchNoNorm (norm.cu:48-123,
 * nonorm.cu:50-122).  Buffers are sized lazily and reused across micrographs. */
int gisspa_create(const gisspa_config* cfg, int device, gisspa_handle** out);

/* Replaces Templates(path, count) + LoadTemplate (templates.cpp:11-31, norm.cu:132-154).
 * stack: n images of width x height floats, row-major, copied by the call. */
int gisspa_set_templates(gisspa_handle* h, const float* stack, int n, int width, int height);

/* Replaces SearchNorm::work / SearchNoNorm::work (norm.cu:620-660, nonorm.cu:559-589)
 * for one micrograph held in host memory (ny rows of nx floats; not modified).
 * Picks are written in the reference's output order.  If more than cap picks
 * are found, GISSPA_ERR_CAPACITY is returned and *n_out holds the count. */
int gisspa_search(gisspa_handle* h, const float* image, int nx, int ny, const gisspa_ctf* ctf,
                  gisspa_pick* picks, size_t cap, size_t* n_out);

/* As gisspa_search, with the micrograph already in this handle's device memory. */
int gisspa_search_device(gisspa_handle* h, const float* d_image, int nx, int ny,
                         const gisspa_ctf* ctf, gisspa_pick* picks, size_t cap, size_t* n_out);

/* Replaces the per-micrograph loop of main.cu:36-50: n micrographs of uneven size,
 * each with its own CTF, searched in one call.  picks of micrograph i are
 * picks[offsets[i] .. offsets[i+1]) (offsets has n+1 entries). */
int gisspa_search_batch(gisspa_handle* h, int n, const float* const* images, const int* nx,
                        const int* ny, const gisspa_ctf* ctfs, gisspa_pick* picks, size_t cap,
                        size_t* offsets);

/* Format one pick as the reference's pick-list line (norm.cu:610-614), including
 * the trailing newline.  Returns the number of characters written (excluding NUL)
 * or -1 when cap is too small. */
int gisspa_format_pick(const gisspa_pick* p, int lst_index, const char* micrograph_path,
                       const gisspa_ctf* ctf, float euler1, float euler2, char* buf, size_t cap);

/* Timing and counters of the last search on this handle. */
int gisspa_get_stats(const gisspa_handle* h, gisspa_stats* out);

/* Text of the last error on this handle (or of the last failed create when h is NULL). */
const char* gisspa_last_error(const gisspa_handle* h);

/* Replaces ~SearchNorm / ~SearchNoNorm (norm.cu:125-130). */
void gisspa_destroy(gisspa_handle* h);

/* Library version string. */
const char* gisspa_version(void);

/* Gradient of a pick's normalised score z = (c - mu)/sigma (no counterpart in the
 * reference).  mu and sigma are held at the pick pixel; the shift moves the template's
 * sampling (a Fourier shift on the periodic window), theta acts through the bilinear
 * rotation, and the CTF through the template-side |CTF| x SSNR weight (the micrograph's
 * preprocessing keeps the search's CTF).  With spectrum_precision FP16 or BF16 the prepared
 * templates and their CTF derivatives are read as stored at that precision (half the bytes
 * per pick); sums are FP64 in every form. */
typedef struct gisspa_grad {
  float score;          /* z at the evaluated parameters */
  float d_dx, d_dy;     /* per pixel of shift of the pick centre */
  float d_theta;        /* per degree of the search angle theta (the printed angle is 360 - theta) */
  float d_dfu, d_dfv;   /* per micrometre of the SetParams defocus_u / defocus_v (norm.cu:188-189) */
  float d_dfang;        /* per degree of the astigmatism angle */
} gisspa_grad;

/* Scores and gradients of picks returned by the last norm_type=1 search on this handle.
 * params: n x (dx, dy, theta) floats, or NULL for (0, 0, pick.theta); ctf: the CTF to
 * evaluate the template weight at, or NULL for the search's. */
int gisspa_score_grad(gisspa_handle* h, const gisspa_pick* picks, size_t n, const float* params,
                      const gisspa_ctf* ctf, gisspa_grad* out);

/* Batched local refinement of those picks (centre, theta) and of the micrograph CTF by
 * gradient ascent for `steps` steps; picks (x, y, theta, angle, score) and *ctf are updated
 * in place (ctf NULL: keep the search's CTF fixed and refine the picks only).  params_out
 * (optional): n x (dx, dy, theta) relative to the input picks' centres. */
int gisspa_refine(gisspa_handle* h, gisspa_pick* picks, size_t n, int steps, gisspa_ctf* ctf, float* params_out);

/* Correlation maps of every (window, template) pair of device-resident half spectra
 * (compute_corner_CCG kernels.cu:645-678 + cufftExecC2C norm.cu:532-537, real part / L^2).
 * d_windows: n_windows x (L/2+1) x L complex FP32, kx-major (S[kx][ky]);
 * d_templates: n_templates x (L/2+1) x L complex in `spec` precision, same layout;
 * d_out: n_windows x n_templates x L x L floats, zero lag at (L/2, L/2).
 * L is the handle's window_size.  Uses handle-owned scratch memory (allocated on
 * first use). */
int gisspa_cc_maps(gisspa_handle* h, const void* d_windows, int n_windows, const void* d_templates, int n_templates,
                   int spec, float* d_out);

/* Correlation maps as gisspa_cc_maps, for callers that cannot allocate device memory
 * (a framework that owns the device memory pool or budget, a locked-down allocator):
 * this call makes no cudaMalloc/cudaFree or other allocating call.  No counterpart in
 * the reference.  Its intermediate lives in a fixed 16 MiB __device__ array (plus a
 * 15 KiB twiddle table) that every GPU loading the library holds until exit, so one
 * call takes at most 16 MiB / (window_size^2 * 4 bytes) (window, template) pairs:
 * 64 pairs at window_size 256, 16 at 512, 4 at 1024; larger calls return
 * GISSPA_ERR_CAPACITY with the reason in gisspa_last_error(NULL).  d_windows,
 * d_templates, d_out and window_size as for gisspa_cc_maps; runs on `stream`
 * (a cudaStream_t, NULL = default stream) of the current device and returns once the
 * maps are written (it waits for `stream`).  GISSPA_ERR_TIMEOUT: a bounded wait inside
 * the kernels gave up and the maps are incomplete (the next call starts clean).  The
 * first call on each device sets up that device's copy of the arrays (make that first
 * call before any stream capture).  Every call shares the one intermediate and error
 * flag, which keep the last call's contents; the intermediate is fully overwritten
 * before it is read and the flag is cleared at the start of each call, so calls that
 * overlap on the GPU (other streams or threads) race on them and must be serialised by
 * the caller. */
int gisspa_cc_maps_noalloc(const void* d_windows, int n_windows, const void* d_templates, int n_templates,
                           int window_size, int spec, float* d_out, void* stream);

/* ---- template generation on the device ----
 * The reference searches a template stack made beforehand, by projecting a 3D map with EMAN's
 * project3d (EMReader/emdata.cpp:891-996).  These calls make that stack on the GPU, bit for
 * bit as project3d does with zero translation (its dx, dy members, which no constructor or
 * reader of the reference sets) and the volume's own depth.  The volume is [nz][ny][nx] floats
 * in host memory, angles are n (alt, az, phi) triples in radians (project3d's units), ri is
 * the mask radius in pixels (0: nx/2). */
/* Projections into host memory out: n x ny x nx floats. */
int gisspa_project(gisspa_handle* h, const float* volume, int nx, int ny, int nz, const float* angles, int n,
                   int ri, float* out);
/* The projections become this handle's template stack (as gisspa_set_templates, without the
 * host round trip). */
int gisspa_set_templates_from_volume(gisspa_handle* h, const float* volume, int nx, int ny, int nz,
                                     const float* angles, int n, int ri);

/* ---- one micrograph across several GPUs (no counterpart in the reference, whose GPUs
 * only split the micrograph list, main.cu:51-90) ----
 * norm_type=1 only.  Every rank holds a handle on its own GPU with the same config and
 * templates, and takes a contiguous range of the angle sequence
 * (for (float e = 0; e < 360; e += phistep), norm.cu:684).  The ranks' per-window-pixel
 * state is merged by the caller's collective (sum of the two FP64 sums, max of the
 * signed 64-bit peak keys), then:
 *   top-K:  begin -> sweep(1, a0, a1) -> export -> [all-reduce] -> import -> picks
 *           (every rank returns the same picks);
 *   chunk:  begin -> sweep(1, a0, a1) -> export -> [all-reduce] -> import
 *           -> sweep(2, a0, a1) -> picks (this rank's angles only; concatenating the
 *           ranks' lists in angle order gives the single-GPU list).
 * A peak key packs the largest correlation of a window pixel over this rank's
 * template-rotations with its index k = angle * n_templates + template:
 * ((order-preserving bits of the FP32 value) << 32 | (0xFFFFFFFF - k)) XOR 2^63, read as
 * int64, so a signed max picks the larger value and, on ties, the lower k (as one GPU
 * does); 0x8000000000000000 (INT64_MIN) marks a pixel with none. */
typedef struct gisspa_shard_info {
  size_t n_pixels;  /* window pixels W x window_size^2: length of each exported array */
  int n_windows;    /* W */
  int n_angles;     /* length of the angle sequence */
  int pick_mode;    /* GISSPA_PICK_* of the handle */
} gisspa_shard_info;

/* Preparation of one micrograph (host image, as gisspa_search) and zeroed state. */
int gisspa_shard_begin(gisspa_handle* h, const float* image, int nx, int ny, const gisspa_ctf* ctf,
                       gisspa_shard_info* info);
/* Sweep 1 (or 2, chunk mode, after import) over angles [angle_begin, angle_end). */
int gisspa_shard_sweep(gisspa_handle* h, int sweep, int angle_begin, int angle_end);
/* Copies this rank's state to caller-owned device memory on the handle's GPU, n_pixels
 * entries each: sum and sum_sq of the correlation (FP64), and (top-K mode) the peak keys;
 * peak_key may be NULL in chunk mode. */
int gisspa_shard_export(gisspa_handle* h, double* sum, double* sum_sq, long long* peak_key);
/* Loads the merged state (same layout) and computes the normalisation statistics. */
int gisspa_shard_import(gisspa_handle* h, const double* sum, const double* sum_sq, const long long* peak_key);
/* Picks after import (top-K) or after sweep 2 (chunk); capacity as gisspa_search. */
int gisspa_shard_picks(gisspa_handle* h, gisspa_pick* picks, size_t cap, size_t* n_out);

/* ---- diagnostics: stage outputs for parity tests (no counterpart in the reference) ---- */
enum {
  GISSPA_STAGE_TEMPLATES = 1,        /* norm_type=1: float [nt][L][L] real-space prepared templates;
                                        norm_type=0: float2 [nt][L/2+1][L] prepared spectra (kx-major) */
  GISSPA_STAGE_IMAGE = 2,            /* float [ny][nx] preprocessed micrograph (norm_type=1) */
  GISSPA_STAGE_WINDOW_SPECTRA = 3,   /* float2 [W][L/2+1][L] normalised window spectra (kx-major) */
  GISSPA_STAGE_TEMPLATE_SPECTRA = 4, /* float2 [nt][L/2+1][L] rotated template spectra at theta */
  GISSPA_STAGE_MUSIG = 5             /* float2 [W][L][L] (mu, 1/sigma) of the last norm_type=1 search */
};
/* Runs the preparation stages for `image` (host, may be NULL for stages 1 and 5) and
 * copies the requested stage output to host memory `out` of `bytes` bytes. */
int gisspa_debug_stage(gisspa_handle* h, int what, const float* image, int nx, int ny, const gisspa_ctf* ctf,
                       float theta, void* out, size_t bytes);

/* Failure-path check (no counterpart in the reference, which has no device waits): one
 * kernel waits, through the same bounded mbarrier wait the correlation kernels use, for an
 * arrival that never comes, gives up after `seconds` (0 < seconds <= 10) and raises the
 * handle's device error flag.  Returns GISSPA_ERR_TIMEOUT, as a search whose bulk copies
 * never landed would; the handle stays usable. */
int gisspa_debug_wait_probe(gisspa_handle* h, double seconds);

/* In-place unnormalised 1D transform (sign -1 forward, +1 inverse) of `rows` contiguous
 * complex rows of length n (1 <= n <= 16384) in DEVICE memory, through the library's generic
 * FFT engine (the transforms of the preparation stages: radix 2, mixed radix 2/3/4/5/7 or
 * Bluestein by length).  No counterpart in the reference, which calls cuFFT. */
int gisspa_debug_fft(gisspa_handle* h, void* data, long long rows, int n, int sign);

#ifdef __cplusplus
}
#endif
#endif /* GISSPA_H */
