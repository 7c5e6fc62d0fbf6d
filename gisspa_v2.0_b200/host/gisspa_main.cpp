// gisspa_main.cpp — command-line driver with the reference's interface (main.cu:14-97):
//   gisspa_main <config>
// reads the LST micrograph list, the Euler file and the template stack named in the
// config, searches micrographs [first, last) and writes the reference pick-list lines.
// GPU_ID = -1 fans micrographs out over all devices in contiguous intervals
// (work_intervals, helper.cu:23-33) with one host thread and one handle per device;
// the per-device outputs are concatenated in device order (main.cu:51-90).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gisspa.h"

namespace {

struct LstEntry {  // LST::Entry (DataReader2.h:93-103)
  int unused = 0;
  std::string rpath;
  double defocus = 0, dfdiff = 0, dfang = 0;
};

std::vector<LstEntry> load_lst(const std::string& path) {  // LST::load (DataReader2.cpp:80-107)
  std::vector<LstEntry> out;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    if (!line.empty() && line[0] == '#') continue;
    LstEntry e;
    char buf[1024] = {0};
    std::sscanf(line.c_str(), "%d %1023s defocus=%lf dfdiff=%lf dfang=%lf", &e.unused, buf, &e.defocus, &e.dfdiff,
                &e.dfang);
    e.rpath = buf;
    out.push_back(e);
  }
  return out;
}

struct Euler {
  std::vector<float> e1, e2, e3;
};
Euler load_euler(const std::string& path) {  // EulerData (DataReader2.cpp:55-78): three line forms
  Euler e;
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    float a, b, c;
    if (std::sscanf(line.c_str(), "%*f %f %f %f", &a, &b, &c) == 3 || std::sscanf(line.c_str(), "%f %f %f", &a, &b, &c) == 3 ||
        std::sscanf(line.c_str(), "%*d %*s %f %f %f", &a, &b, &c) == 3) {
      e.e1.push_back(a);
      e.e2.push_back(b);
      e.e3.push_back(c);
    }
  }
  return e;
}

// MRC section reader (little-endian modes 0, 1, 2, 6); section n if 0 <= n < nz, else the whole map
// (emdata::readMRC, emdata.cpp:412-677).
bool read_mrc(const std::string& path, int n, std::vector<float>& data, int& nx, int& ny, int& nz_out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  int32_t hdr[256];
  if (!in.read(reinterpret_cast<char*>(hdr), 1024)) return false;
  nx = hdr[0];
  ny = hdr[1];
  const int nz = hdr[2], mode = hdr[3], next = hdr[23];
  nz_out = nz;
  if (nx <= 0 || ny <= 0 || nz <= 0) return false;
  int bpp = mode == 0 ? 1 : (mode == 1 || mode == 6) ? 2 : mode == 2 ? 4 : 0;
  if (!bpp) return false;
  int z0 = 0, cnt = nz;
  if (n >= 0 && n < nz) {
    z0 = n;
    cnt = 1;
  }
  const size_t sec = (size_t)nx * ny;
  in.seekg(1024 + (std::streamoff)next + (std::streamoff)z0 * sec * bpp);
  std::vector<char> raw(sec * cnt * bpp);
  if (!in.read(raw.data(), raw.size())) return false;
  data.resize(sec * cnt);
  for (size_t i = 0; i < data.size(); ++i) {
    switch (mode) {
      case 0: data[i] = (float)reinterpret_cast<int8_t*>(raw.data())[i]; break;
      case 1: data[i] = (float)reinterpret_cast<int16_t*>(raw.data())[i]; break;
      case 6: data[i] = (float)reinterpret_cast<uint16_t*>(raw.data())[i]; break;
      default: std::memcpy(&data[i], raw.data() + 4 * i, 4); break;
    }
  }
  if (cnt > 1) ny *= cnt;
  return true;
}

std::vector<std::pair<int, int>> work_intervals(int first, int last, int procs) {  // helper.cu:23-33
  std::vector<std::pair<int, int>> r;
  const float total = (float)(last - first);
  const int per = std::max((int)std::round(total / procs), 1);
  for (int i = 0; i < procs && first < last; ++i) {
    r.push_back({first, std::min(first + per, last)});
    first += per;
  }
  if (!r.empty()) r.back().second = last;
  return r;
}

// Templates: a projected stack (tw x th x nt), or a 3D map (tw x th x td) projected on the
// device at the angles in `angles` (nt triples, radians) when td > 0.
struct TemplateSource {
  std::vector<float> data;
  int tw = 0, th = 0, td = 0;
  std::vector<float> angles;
};

int run_device(int dev, const gisspa_config& cfg, const TemplateSource& ts, int nt, const Euler& eu,
               const std::vector<LstEntry>& lst, int first, int last, std::string& out) {
  gisspa_handle* h = nullptr;
  int st = gisspa_create(&cfg, dev, &h);
  if (st) {
    std::fprintf(stderr, "device %d: %s\n", dev, gisspa_last_error(nullptr));
    return st;
  }
  st = ts.td > 0 ? gisspa_set_templates_from_volume(h, ts.data.data(), ts.tw, ts.th, ts.td, ts.angles.data(), nt, 0)
                 : gisspa_set_templates(h, ts.data.data(), nt, ts.tw, ts.th);
  if (st) std::fprintf(stderr, "device %d: %s\n", dev, gisspa_last_error(h));
  std::vector<gisspa_pick> picks(1 << 16);
  // Read-ahead: micrograph i + 1 is read and decoded on a host thread while micrograph i is
  // searched on the GPU.
  struct Mic {
    bool ok = false;
    std::vector<float> img;
    int nx = 0, ny = 0, nz = 0;
  };
  auto read_one = [&lst](int i) {
    Mic m;
    m.ok = read_mrc(lst[i].rpath, lst[i].unused, m.img, m.nx, m.ny, m.nz);
    return m;
  };
  std::future<Mic> next;
  if (first < last && !st) next = std::async(std::launch::async, read_one, first);
  for (int i = first; i < last && !st; ++i) {
    const LstEntry& e = lst[i];
    Mic cur = next.get();
    if (i + 1 < last) next = std::async(std::launch::async, read_one, i + 1);
    std::vector<float>& img = cur.img;
    const int nx = cur.nx, ny = cur.ny;
    if (!cur.ok) {
      std::fprintf(stderr, "cannot read micrograph %s\n", e.rpath.c_str());
      st = GISSPA_ERR_IO;
      break;
    }
    gisspa_ctf ctf{e.defocus, e.dfdiff, e.dfang};
    size_t n = 0;
    st = gisspa_search(h, img.data(), nx, ny, &ctf, picks.data(), picks.size(), &n);
    if (st == GISSPA_ERR_CAPACITY) {
      picks.resize(n);
      st = gisspa_search(h, img.data(), nx, ny, &ctf, picks.data(), picks.size(), &n);
    }
    if (st) {
      std::fprintf(stderr, "device %d: %s\n", dev, gisspa_last_error(h));
      break;
    }
    char buf[2048];
    for (size_t k = 0; k < n; ++k) {
      const int j = picks[k].template_id;
      if (gisspa_format_pick(&picks[k], e.unused, e.rpath.c_str(), &ctf, eu.e1[j], eu.e2[j], buf, sizeof buf) > 0)
        out += buf;
    }
    gisspa_stats s{};
    gisspa_get_stats(h, &s);
    std::printf("Device %d: %s: %zu picks in %.1f ms\n", dev, e.rpath.c_str(), n, s.ms_total);
  }
  gisspa_destroy(h);
  return st;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <config>\n", argv[0]);
    return 2;
  }
  gisspa_config cfg;
  gisspa_run_paths rp;
  if (gisspa_config_load(argv[1], &cfg, &rp)) {
    std::fprintf(stderr, "cannot parse config %s\n", argv[1]);
    return 1;
  }
  const auto lst = load_lst(rp.input);
  const Euler eu = load_euler(rp.eulerfile);
  const int nt = (int)eu.e1.size();
  if (lst.empty() || nt == 0) {
    std::fprintf(stderr, "empty micrograph list or Euler file\n");
    return 1;
  }
  TemplateSource ts;
  if (rp.template_volume[0]) {
    // a 3D map projected on the device at the Euler file's angles (degrees -> radians with the
    // reference's pi, utils/constants.h:3)
    int x, y, z;
    if (!read_mrc(rp.template_volume, -1, ts.data, x, y, z) || z < 2) {
      std::fprintf(stderr, "cannot read the 3D map %s\n", rp.template_volume);
      return 1;
    }
    ts.tw = x;
    ts.th = y / z;  // read_mrc stacks the sections: y holds ny * nz
    ts.td = z;
    for (int i = 0; i < nt; ++i)
      for (float e : {eu.e1[i], eu.e2[i], eu.e3[i]}) ts.angles.push_back((float)((double)e * 3.1415926535 / 180.0));
  } else {
    // Templates(path, count) (templates.cpp:11-31): count = number of Euler lines
    for (int i = 0; i < nt; ++i) {
      std::vector<float> one;
      int x, y, z;
      if (!read_mrc(rp.template_path, i, one, x, y, z)) {
        std::fprintf(stderr, "cannot read template %d of %s\n", i, rp.template_path);
        return 1;
      }
      ts.tw = x;
      ts.th = y;
      ts.data.insert(ts.data.end(), one.begin(), one.end());
    }
  }
  const int first = std::max(0, std::min(rp.first, (int)lst.size() - 1));
  const int last = std::min(rp.last, std::max(0, (int)lst.size()));
  std::ofstream output(rp.output, std::ios::out | std::ios::trunc);
  int st = 0;
  if (rp.gpu_id != -1) {
    std::string out;
    st = run_device(rp.gpu_id, cfg, ts, nt, eu, lst, first, last, out);
    output << out;
  } else {
    int ndev = 0;
    cudaGetDeviceCount(&ndev);
    if (ndev <= 0) return 1;
    const auto iv = work_intervals(first, last, ndev);
    std::vector<std::string> outs(iv.size());
    std::vector<int> sts(iv.size(), 0);
    std::vector<std::thread> workers;
    for (size_t d = 0; d < iv.size(); ++d)
      workers.emplace_back([&, d] {
        sts[d] = run_device((int)d, cfg, ts, nt, eu, lst, iv[d].first, iv[d].second, outs[d]);
      });
    for (auto& t : workers) t.join();
    for (size_t d = 0; d < iv.size(); ++d) {
      output << outs[d];
      if (sts[d]) st = sts[d];
    }
  }
  return st ? 1 : 0;
}
