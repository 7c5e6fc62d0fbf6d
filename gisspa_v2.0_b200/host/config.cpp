// config.cpp — reference config-file parser (Config::Config, EMReader/DataReader2.cpp:6-28).
//
// Same syntax: a stream of "key = value" tokens; unknown keys are ignored; keys
// have the reference's types and defaults (DataReader2.h:19-44).  Extension keys
// (pick_mode, topk, exclusion_radius, spectrum_precision, template_batch,
// window_batch, quirks, tile_size, cuda_graphs, pass_b_shape, tensor_cores, pass_a_shape,
// prune_sweep2) configure the additions of
// this library.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "../../include/gisspa.h"

namespace {

void copy_str(char* dst, const std::string& v) {
  std::strncpy(dst, v.c_str(), 1023);
  dst[1023] = 0;
}

bool parse_int(const std::string& v, int& out) {
  try {
    size_t pos = 0;
    out = std::stoi(v, &pos);
    return true;
  } catch (...) {
    return false;
  }
}
bool parse_float(const std::string& v, float& out) {
  try {
    size_t pos = 0;
    out = std::stof(v, &pos);
    return true;
  } catch (...) {
    return false;
  }
}

}  // namespace

extern "C" int gisspa_config_load(const char* path, gisspa_config* cfg, gisspa_run_paths* paths) {
  if (!path || !cfg) return GISSPA_ERR_ARG;
  gisspa_config_default(cfg);
  gisspa_run_paths local{};
  gisspa_run_paths* rp = paths ? paths : &local;
  std::memset(rp, 0, sizeof(*rp));
  rp->first = 0;
  rp->last = 0;
  rp->gpu_id = -1;
  std::ifstream in(path);
  if (!in) return GISSPA_ERR_IO;
  std::string key, eq, val;
  while (in >> key >> eq >> val) {
    if (eq != "=") return GISSPA_ERR_IO;
    bool ok = true;
    // reference keys
    if (key == "input") copy_str(rp->input, val);
    else if (key == "template") copy_str(rp->template_path, val);
    else if (key == "template_volume") copy_str(rp->template_volume, val);
    else if (key == "eulerfile") copy_str(rp->eulerfile, val);
    else if (key == "output") copy_str(rp->output, val);
    else if (key == "first") ok = parse_int(val, rp->first);
    else if (key == "last") ok = parse_int(val, rp->last);
    else if (key == "GPU_ID") ok = parse_int(val, rp->gpu_id);
    else if (key == "template_dims") { int d; ok = parse_int(val, d); }
    else if (key == "angpix") ok = parse_float(val, cfg->angpix);
    else if (key == "phistep") ok = parse_float(val, cfg->phistep);
    else if (key == "kk") ok = parse_float(val, cfg->kk);
    else if (key == "energy") ok = parse_float(val, cfg->energy);
    else if (key == "cs") ok = parse_float(val, cfg->cs);
    else if (key == "Highres") ok = parse_float(val, cfg->highres);
    else if (key == "Lowres") ok = parse_float(val, cfg->lowres);
    else if (key == "diameter") ok = parse_float(val, cfg->diameter);
    else if (key == "threshold") ok = parse_float(val, cfg->threshold);
    else if (key == "window_size") ok = parse_int(val, cfg->window_size);
    else if (key == "phase_flip") ok = parse_int(val, cfg->phase_flip);
    else if (key == "overlap") ok = parse_int(val, cfg->overlap);
    else if (key == "norm_type") ok = parse_int(val, cfg->norm_type);
    else if (key == "invert") ok = parse_int(val, cfg->invert);
    // additions
    else if (key == "pick_mode") {
      if (val == "chunk") cfg->pick_mode = GISSPA_PICK_CHUNK;
      else if (val == "topk") cfg->pick_mode = GISSPA_PICK_TOPK;
      else ok = parse_int(val, cfg->pick_mode);
    } else if (key == "topk") ok = parse_int(val, cfg->topk);
    else if (key == "exclusion_radius") ok = parse_float(val, cfg->exclusion_radius);
    else if (key == "spectrum_precision") {
      if (val == "fp32") cfg->spectrum_precision = GISSPA_SPEC_FP32;
      else if (val == "fp16") cfg->spectrum_precision = GISSPA_SPEC_FP16;
      else if (val == "bf16") cfg->spectrum_precision = GISSPA_SPEC_BF16;
      else ok = parse_int(val, cfg->spectrum_precision);
    } else if (key == "template_batch") ok = parse_int(val, cfg->template_batch);
    else if (key == "window_batch") ok = parse_int(val, cfg->window_batch);
    else if (key == "quirks") ok = parse_int(val, cfg->quirks);
    else if (key == "tile_size") ok = parse_int(val, cfg->tile_size);
    else if (key == "cuda_graphs") ok = parse_int(val, cfg->cuda_graphs);
    else if (key == "pass_b_shape") ok = parse_int(val, cfg->pass_b_shape);
    else if (key == "tensor_cores") ok = parse_int(val, cfg->tensor_cores);
    else if (key == "pass_a_shape") ok = parse_int(val, cfg->pass_a_shape);
    else if (key == "prune_sweep2") ok = parse_int(val, cfg->prune_sweep2);
    // unknown keys are ignored (DataReader2.cpp:17-18)
    if (!ok) return GISSPA_ERR_IO;
  }
  return GISSPA_OK;
}
