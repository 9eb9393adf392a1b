// libvti_wave.so: the reference's C++ entry points (include/vti_wave.h) on top
// of the C ABI. Side channels are read the way the reference's myio layer
// does (lib/io/myio.cpp:29-90, myio.h:131-405): key=value words of the argv
// recorded by myio_init(), a par= file, SEP headers whose in= names the
// binary, datapath= for new binaries.
//
// Shots are spread over the listed GPUs (one context and one resident plan
// per device, cached across calls); results are summed on the host. Time
// levels and recorded samples follow the reference pipeline of the same GPU
// count (VTI_OPT_REF_GPUS), so numbers match the reference run on those GPUs.
// Errors are printed to stderr and, like the reference, do not throw; misfits
// are then NaN.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "vti_b200.h"
#include "vti_hessian_op.h"
#include "vti_modeling_op3d.h"
#include "vti_wave.h"

// Recorded by the caller's myio_init(); weak so the shim also links without it.
extern int gargc __attribute__((weak));
extern char** gargv __attribute__((weak));

namespace {

// ---------------------------------------------------------------- argv / SEP
std::string value_in_line_set(const std::vector<std::string>& lines, const std::string& key) {
  const std::string k = key + "=";
  std::string out;
  for (const std::string& line : lines) {
    size_t pos = line.find(k);
    while (pos != std::string::npos) {
      size_t next = pos + k.size();
      if (pos == 0 || !std::isalnum((unsigned char)line[pos - 1])) {
        if (next < line.size() && line[next] == '"') {
          size_t e = line.find('"', next + 1);
          out = line.substr(next + 1, e == std::string::npos ? std::string::npos : e - next - 1);
        } else {
          size_t e = line.find(' ', next);
          out = line.substr(next, e == std::string::npos ? std::string::npos : e - next);
        }
      }
      pos = line.find(k, next);
    }
  }
  return out;
}

std::string file_value(const std::string& file, const std::string& key) {
  std::ifstream in(file);
  if (!in) return "";
  std::vector<std::string> lines;
  for (std::string l; std::getline(in, l);) lines.push_back(l);
  return value_in_line_set(lines, key);
}

std::string arg(const std::string& key) {
  if (&gargc && &gargv && gargv) {
    const std::string k = key + "=";
    for (int i = 0; i < gargc; ++i)
      if (gargv[i] && std::strncmp(gargv[i], k.c_str(), k.size()) == 0)
        return std::string(gargv[i] + k.size());
  }
  std::string par;  // myio.h:155-160: fall back to the par= file
  if (&gargc && &gargv && gargv)
    for (int i = 0; i < gargc; ++i)
      if (gargv[i] && std::strncmp(gargv[i], "par=", 4) == 0) par = gargv[i] + 4;
  return par.empty() ? "" : file_value(par, key);
}

std::vector<int> gpus_from_argv() {
  std::vector<int> g;
  std::stringstream ss(arg("gpu"));
  for (std::string t; std::getline(ss, t, ',');)
    if (!t.empty()) g.push_back(std::atoi(t.c_str()));
  if (g.empty()) g.push_back(0);
  return g;
}

float float_arg(const std::string& key, float dflt) {
  std::string v = arg(key);
  return v.empty() ? dflt : (float)std::atof(v.c_str());
}

void bswap4(float* p, size_t n) {
  for (size_t i = 0; i < n; ++i) {
    unsigned char* b = (unsigned char*)(p + i);
    std::swap(b[0], b[3]);
    std::swap(b[1], b[2]);
  }
}

// read(tag, buff, n, pos) of myio.h:396
bool sep_read(const std::string& tag, float* buf, size_t n, size_t pos) {
  std::string hdr = arg(tag);
  if (hdr.empty()) {
    std::fprintf(stderr, "vti: cannot find header %s\n", tag.c_str());
    return false;
  }
  std::string bin = file_value(hdr, "in");
  std::ifstream in(bin, std::ios::binary);
  if (!in) {
    std::fprintf(stderr, "vti: cannot read binary file %s of header %s\n", bin.c_str(), hdr.c_str());
    return false;
  }
  in.seekg((std::streamoff)(pos * sizeof(float)));
  in.read((char*)buf, (std::streamsize)(n * sizeof(float)));
  std::string fmt = file_value(hdr, "data_format");
  if (fmt != "native_float" && fmt != "native_double") bswap4(buf, n);
  return (size_t)in.gcount() == n * sizeof(float);
}

std::string datapath() {
  std::string p = arg("datapath");
  if (p.empty()) {
    const char* home = std::getenv("HOME");
    if (home) p = file_value(std::string(home) + "/.datapath", "datapath");
  }
  return p;
}

// write(tag, buff, n[, mode]) of myio.h:273-320
bool sep_write(const std::string& tag, const float* buf, size_t n, bool append) {
  std::string hdr = arg(tag);
  if (hdr.empty()) {
    std::fprintf(stderr, "vti: cannot find header %s\n", tag.c_str());
    return false;
  }
  std::string name = hdr.substr(hdr.rfind('/') == std::string::npos ? 0 : hdr.rfind('/') + 1);
  std::string dp = datapath();
  if (dp.empty()) {
    std::fprintf(stderr, "vti: cannot find datapath\n");
    return false;
  }
  std::string bin = dp + name + "@";
  std::ofstream out(bin, std::ios::binary | (append ? std::ios::app : std::ios::trunc));
  if (!out) return false;
  out.write((const char*)buf, (std::streamsize)(n * sizeof(float)));
  out.close();
  std::ofstream h(hdr, std::ios::app);
  if (&gargc && &gargv && gargv)
    for (int i = 0; i < gargc; ++i) h << gargv[i] << " ";
  h << "\n\nin=" << bin << "\ndata_format=native_float\n";
  return true;
}

template <typename T>
void to_header(const std::string& tag, const std::string& key, T value) {
  std::string hdr = arg(tag);
  if (hdr.empty()) return;
  std::ofstream h(hdr, std::ios::app);
  h << "\n" << key << "=" << value << "\n";
}

// ---------------------------------------------------------- device cache
struct Device {
  vti_ctx* ctx = nullptr;
  std::map<std::tuple<int, int, int, int, int, unsigned>, vti3d_plan*> plans;
  std::mutex mu;
};

std::mutex g_mu;
std::map<int, std::unique_ptr<Device>>& devices() {
  static std::map<int, std::unique_ptr<Device>> d;
  return d;
}

Device* device(int id) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto& m = devices();
  auto it = m.find(id);
  if (it != m.end()) return it->second.get();
  auto d = std::make_unique<Device>();
  if (vti_ctx_create(id, &d->ctx) != VTI_OK) {
    std::fprintf(stderr, "vti: cannot open CUDA device %d\n", id);
    return nullptr;
  }
  Device* p = d.get();
  m[id] = std::move(d);
  return p;
}

bool report(vti_ctx* ctx, int st, const char* what) {
  if (st == VTI_OK) return true;
  std::fprintf(stderr, "vti: %s: %s (%s)\n", what, vti_status_string(st), vti_ctx_last_error(ctx));
  return false;
}

vti3d_plan* plan_for(Device* dev, const vti3d_geom& g, unsigned flags) {
  auto key = std::make_tuple(g.nx, g.ny, g.nz, g.nt, g.npad, flags);
  auto it = dev->plans.find(key);
  if (it != dev->plans.end()) return it->second;
  vti3d_plan* p = nullptr;
  if (!report(dev->ctx, vti3d_plan_create(dev->ctx, &g, flags, &p), "plan")) return nullptr;
  dev->plans[key] = p;
  return p;
}

vti3d_geom geom3(int nx, int ny, int nz, int nt, int npad, float ox, float oy, float oz, float ot,
                 float dx, float dy, float dz, float dt, float rate) {
  vti3d_geom g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.nt = nt; g.npad = npad;
  g.ox = ox; g.oy = oy; g.oz = oz; g.ot = ot;
  g.dx = dx; g.dy = dy; g.dz = dz; g.dt = dt;
  g.sampling_rate = rate;
  return g;
}

int nnt_of(const vti3d_geom& g) {
  return (g.nt - 1) / (int)std::round(g.sampling_rate / g.dt) + 1;
}

int total_receivers(const float* souloc, const std::vector<int>& shots) {
  int n = 0;
  for (int s : shots) n = std::max(n, (int)souloc[5 * s + 3] + (int)souloc[5 * s + 4]);
  return n;
}

// Run `fn(device, shots)` for a round-robin split of the shots over GPUs.
template <typename F>
bool over_gpus(const std::vector<int>& gpus, const std::vector<int>& shots, F fn) {
  std::vector<std::vector<int>> part(gpus.size());
  for (size_t i = 0; i < shots.size(); ++i) part[i % gpus.size()].push_back(shots[i]);
  std::vector<int> ok(gpus.size(), 1);
  std::vector<std::thread> th;
  for (size_t i = 0; i < gpus.size(); ++i) {
    if (part[i].empty()) continue;
    th.emplace_back([&, i]() { ok[i] = fn(gpus[i], part[i]) ? 1 : 0; });
  }
  for (auto& t : th) t.join();
  for (int v : ok)
    if (!v) return false;
  return true;
}

// get_param("tpow"/"objtype"/"halfwidth") of objFuncGradient3d_f.cu:743-773
struct MisfitParams {
  float tpow = 0.f;
  int objtype = 0;
  int halfwidth = 20;
};
MisfitParams misfit_params() {
  MisfitParams m;
  m.tpow = float_arg("tpow", 0.f);
  m.objtype = (int)float_arg("objtype", 0.f);
  m.halfwidth = (int)float_arg("halfwidth", 20.f);
  return m;
}

unsigned ref_flags(size_t ngpu) { return VTI_OPT_REF_GPUS((unsigned)(ngpu ? ngpu : 1)); }

// gradient (or misfit) of `shots` on the GPUs of one pipeline group
bool gradient_group(float* fgcij, double* misfit, const float* souloc, const std::vector<int>& shots,
                    const float* recloc, const float* wavelet, const float* cij, const float* padb,
                    const float* randb, const vti3d_geom& g, const std::vector<int>& gpus,
                    bool misfit_only, const float* dobs, int nrec) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  std::vector<std::vector<float>> parts(gpus.size());
  std::vector<double> mis(gpus.size(), 0.0);
  std::map<int, size_t> slot;
  for (size_t i = 0; i < gpus.size(); ++i) slot[gpus[i]] = i;
  const unsigned flags = ref_flags(gpus.size());
  bool ok = over_gpus(gpus, shots, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    vti3d_plan* p = plan_for(dev, g, flags);
    if (!p) return false;
    size_t k = slot[id];
    if (!report(dev->ctx, vti3d_plan_set_model(p, cij, cij + n, cij + 2 * n, padb, randb,
                                               VTI_MEM_HOST), "model") ||
        !report(dev->ctx, vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST), "wavelet") ||
        !report(dev->ctx, vti3d_plan_set_receivers(p, recloc, nrec), "receivers"))
      return false;
    if (misfit_only)
      return report(dev->ctx, vti3d_plan_objfunc(p, souloc, sub.data(), (int)sub.size(), dobs,
                                                 VTI_MEM_HOST, &mis[k]), "misfit");
    const MisfitParams mp = misfit_params();
    if (!report(dev->ctx, vti3d_plan_set_misfit(p, mp.tpow, mp.objtype, mp.halfwidth),
                "misfit options"))
      return false;
    parts[k].assign(1 + 3 * n, 0.f);
    return report(dev->ctx, vti3d_plan_gradient(p, souloc, sub.data(), (int)sub.size(), dobs,
                                                VTI_MEM_HOST, parts[k].data(), VTI_MEM_HOST,
                                                &mis[k]), "gradient");
  });
  double total = 0;
  for (double m : mis) total += m;
  *misfit = ok ? total : NAN;
  if (!misfit_only && fgcij) {
    std::memset(fgcij, 0, (1 + 3 * n) * sizeof(float));
    for (auto& pz : parts)
      if (!pz.empty())
        for (size_t i = 1; i < 1 + 3 * n; ++i) fgcij[i] += pz[i];
    fgcij[0] = (float)*misfit;
  }
  return ok;
}

bool read_observed(const float* souloc, const std::vector<int>& shots, const vti3d_geom& g,
                   std::vector<float>* dobs, int* nrec) {
  *nrec = total_receivers(souloc, shots);
  const int nnt = nnt_of(g);
  dobs->assign((size_t)nnt * *nrec, 0.f);
  // per shot, as objFuncGradient3d_f.cu:759-760 reads it
  for (int s : shots) {
    const int nr = (int)souloc[5 * s + 3], irb = (int)souloc[5 * s + 4];
    if (!sep_read("data", dobs->data() + (size_t)nnt * irb, (size_t)nnt * nr, (size_t)nnt * irb))
      return false;
  }
  return true;
}


}  // namespace

// ---------------------------------------------------------------- 3D
void objFuncGradientCij3d_f(float* fgcij, float* souloc, int ns, std::vector<int>& shotid,
                            float* recloc, float* wavelet, float* cij, float* padboundaryCij,
                            float* randboundaryCij, int nx, int ny, int nz, int nt, int npad,
                            float ox, float oy, float oz, float ot, float dx, float dy, float dz,
                            float dt, float samplingRate, std::vector<int>& GPUs) {
  (void)ns;
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  const size_t n = (size_t)nx * ny * nz;
  std::memset(fgcij, 0, (1 + 3 * n) * sizeof(float));
  std::vector<float> dobs;
  int nrec = 0;
  double mis = NAN;
  if (read_observed(souloc, shotid, g, &dobs, &nrec))
    gradient_group(fgcij, &mis, souloc, shotid, recloc, wavelet, cij, padboundaryCij,
                   randboundaryCij, g, GPUs, false, dobs.data(), nrec);
  fgcij[0] = (float)mis;
  // the reference leaves the random boundary in the caller's cij
  // (objFuncGradient3d_f.cu:786-788)
  const size_t nb = n - (size_t)(nx - 2 * npad) * (ny - 2 * npad) * (nz - 2 * npad);
  for (int k = 0; k < 3; ++k)
    vti3d_put_boundary(randboundaryCij + k * nb, cij + k * n, nx, ny, nz, npad);
}

void objFuncGradientCij3d(float* fgcij, float* souloc, int ns, std::vector<int>& shotid,
                          float* recloc, float* wavelet, float* cij, float* padboundaryCij,
                          float* randboundaryCij, int nx, int ny, int nz, int nt, int npad,
                          float ox, float oy, float oz, float ot, float dx, float dy, float dz,
                          float dt, float samplingRate, std::vector<int>& GPUs, int ngpugroup) {
  if (ngpugroup <= 1) {
    objFuncGradientCij3d_f(fgcij, souloc, ns, shotid, recloc, wavelet, cij, padboundaryCij,
                           randboundaryCij, nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt,
                           samplingRate, GPUs);
    return;
  }
  // objFuncGradient3d_f.cu:307-359: contiguous shot groups, one per GPU group
  const size_t n = (size_t)nx * ny * nz;
  const int ngpu1 = (int)GPUs.size() / ngpugroup;
  const int nshot1 = (int)shotid.size() / ngpugroup, r = (int)shotid.size() % ngpugroup;
  std::vector<std::vector<float>> fg(ngpugroup, std::vector<float>(1 + 3 * n));
  std::vector<std::vector<float>> tc(ngpugroup, std::vector<float>(cij, cij + 3 * n));
  std::vector<std::thread> th;
  for (int i = 0; i < ngpugroup; ++i) {
    th.emplace_back([&, i]() {
      std::vector<int> gpus(GPUs.begin() + i * ngpu1, GPUs.begin() + (i + 1) * ngpu1);
      int b = i < r ? i * (nshot1 + 1) : r * (nshot1 + 1) + (i - r) * nshot1;
      int e = b + (i < r ? nshot1 + 1 : nshot1);
      std::vector<int> sh(shotid.begin() + b, shotid.begin() + e);
      objFuncGradientCij3d_f(fg[i].data(), souloc, ns, sh, recloc, wavelet, tc[i].data(),
                             padboundaryCij, randboundaryCij, nx, ny, nz, nt, npad, ox, oy, oz,
                             ot, dx, dy, dz, dt, samplingRate, gpus);
    });
  }
  for (auto& t : th) t.join();
  std::memset(fgcij, 0, (1 + 3 * n) * sizeof(float));
  for (int i = ngpugroup - 1; i >= 0; --i)
    for (size_t j = 0; j < 1 + 3 * n; ++j) fgcij[j] += fg[i][j];
}

void objFuncCij3d_f(float* f, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                    float* wavelet, float* cij, float* padboundaryCij, int nx, int ny, int nz,
                    int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                    float dz, float dt, float samplingRate, std::vector<int>& GPUs) {
  (void)ns;
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  std::vector<float> dobs;
  int nrec = 0;
  double mis = NAN;
  if (read_observed(souloc, shotid, g, &dobs, &nrec))
    gradient_group(nullptr, &mis, souloc, shotid, recloc, wavelet, cij, padboundaryCij, nullptr,
                   g, GPUs, true, dobs.data(), nrec);
  *f = (float)mis;
}

void objFuncCij3d(float* f, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                  float* wavelet, float* cij, float* padboundaryCij, int nx, int ny, int nz,
                  int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                  float dz, float dt, float samplingRate, std::vector<int>& GPUs, int ngpugroup) {
  if (ngpugroup <= 1) {
    objFuncCij3d_f(f, souloc, ns, shotid, recloc, wavelet, cij, padboundaryCij, nx, ny, nz, nt,
                   npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate, GPUs);
    return;
  }
  const int ngpu1 = (int)GPUs.size() / ngpugroup;
  const int nshot1 = (int)shotid.size() / ngpugroup, r = (int)shotid.size() % ngpugroup;
  std::vector<float> part(ngpugroup, 0.f);
  std::vector<std::thread> th;
  for (int i = 0; i < ngpugroup; ++i) {
    th.emplace_back([&, i]() {
      std::vector<int> gpus(GPUs.begin() + i * ngpu1, GPUs.begin() + (i + 1) * ngpu1);
      int b = i < r ? i * (nshot1 + 1) : r * (nshot1 + 1) + (i - r) * nshot1;
      int e = b + (i < r ? nshot1 + 1 : nshot1);
      std::vector<int> sh(shotid.begin() + b, shotid.begin() + e);
      objFuncCij3d_f(&part[i], souloc, ns, sh, recloc, wavelet, cij, padboundaryCij, nx, ny, nz,
                     nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate, gpus);
    });
  }
  for (auto& t : th) t.join();
  *f = 0.f;
  for (float v : part) *f += v;
}

double objFuncGradientVEpsDel(float* gv, float* geps, float* gdel, float* souloc, int ns,
                              std::vector<int>& shotid, float* recloc, float* wavelet, float* v,
                              float* eps, float* del, float* padboundaryV, float* randboundaryV,
                              int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                              float oz, float ot, float dx, float dy, float dz, float dt,
                              float samplingRate, float v0, float eps0, float wbottom,
                              std::vector<int>& GPUs, int ngpugroup) {
  // objFuncGradient3d_f.cu:249-305, multi-GPU through objFuncGradientCij3d
  const size_t nxy = (size_t)nx * ny, n = nxy * nz;
  const size_t nb = n - (size_t)(nx - 2 * npad) * (ny - 2 * npad) * (nz - 2 * npad);
  std::vector<float> cij(3 * n), fg(1 + 3 * n), be(nb), bd(nb), padb(3 * nb), randb(3 * nb);
  vti_vepsdel_to_cij(cij.data(), cij.data() + n, cij.data() + 2 * n, v, eps, del, v0, eps0, 1.f,
                     n);
  vti3d_get_boundary(be.data(), eps, nx, ny, nz, npad);
  vti3d_get_boundary(bd.data(), del, nx, ny, nz, npad);
  vti_vepsdel_to_cij(padb.data(), padb.data() + nb, padb.data() + 2 * nb, padboundaryV, be.data(),
                     bd.data(), v0, eps0, 1.f, nb);
  vti_vepsdel_to_cij(randb.data(), randb.data() + nb, randb.data() + 2 * nb, randboundaryV,
                     be.data(), bd.data(), v0, eps0, 1.f, nb);
  objFuncGradientCij3d(fg.data(), souloc, ns, shotid, recloc, wavelet, cij.data(), padb.data(),
                       randb.data(), nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt,
                       samplingRate, GPUs, ngpugroup);
  double objfunc = fg[0];
  float* gc[3] = {fg.data() + 1, fg.data() + 1 + n, fg.data() + 1 + 2 * n};
  int nwbottom = (wbottom - oz) / dz + 1 - npad;
  for (int k = 0; k < 3; ++k) {
    vti3d_zero_boundary(gc[k], nx, ny, nz, npad);
    if (nwbottom > 0)
      std::memset(gc[k] + (size_t)npad * nxy, 0,
                  std::min<size_t>(nwbottom, nz - npad) * nxy * sizeof(float));
  }
  vti_grad_cij_to_vepsdel(gv, geps, gdel, gc[0], gc[1], gc[2], v, eps, del, v0, eps0, 1.f, n);
  return objfunc;
}

void modelDataCij3d_f(float* ddata, float* souloc, int ns, std::vector<int>& shotid,
                      float* recloc, const float* wavelet, float* c11, float* c13, float* c33,
                      int nx, int ny, int nz, int nt, int npad, float ox, float oy, float oz,
                      float ot, float dx, float dy, float dz, float dt, float samplingRate,
                      std::vector<int>& GPUs) {
  (void)ns;
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  const int nrec = total_receivers(souloc, shotid);
  const unsigned flags = ref_flags(GPUs.size());
  over_gpus(GPUs, shotid, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    vti3d_plan* p = plan_for(dev, g, flags);
    return p &&
           report(dev->ctx, vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr, VTI_MEM_HOST),
                  "model") &&
           report(dev->ctx, vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST), "wavelet") &&
           report(dev->ctx, vti3d_plan_set_receivers(p, recloc, nrec), "receivers") &&
           report(dev->ctx, vti3d_plan_model_data(p, souloc, sub.data(), (int)sub.size(), ddata,
                                                  VTI_MEM_HOST), "modeling");
  });
}

void modelData3d_f(float* ddata, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                   const float* wavelet, float* c11, float* c13, float* c33, int nx, int ny,
                   int nz, int nt, int npad, float ox, float oy, float oz, float ot, float dx,
                   float dy, float dz, float dt, float samplingRate, std::vector<int>& GPUs,
                   int ngpugroup) {
  // modelData3d_f.cu:395-425: the groups' shot ranges are disjoint in ddata
  const int ng = ngpugroup < 1 ? 1 : ngpugroup;
  const int ngpu1 = (int)GPUs.size() / ng;
  const int nshot1 = (int)shotid.size() / ng, r = (int)shotid.size() % ng;
  std::vector<std::thread> th;
  for (int i = 0; i < ng; ++i) {
    th.emplace_back([&, i]() {
      std::vector<int> gpus(GPUs.begin() + i * ngpu1, GPUs.begin() + (i + 1) * ngpu1);
      int b = i < r ? i * (nshot1 + 1) : r * (nshot1 + 1) + (i - r) * nshot1;
      int e = b + (i < r ? nshot1 + 1 : nshot1);
      std::vector<int> sh(shotid.begin() + b, shotid.begin() + e);
      modelDataCij3d_f(ddata, souloc, ns, sh, recloc, wavelet, c11, c13, c33, nx, ny, nz, nt, npad,
                       ox, oy, oz, ot, dx, dy, dz, dt, samplingRate, gpus);
    });
  }
  for (auto& t : th) t.join();
}

namespace {
// forward modeling of `shots` on one device, then the last sigma_x level
bool model_and_wavefield(const vti3d_geom& g, unsigned flags, int dev_id, const float* souloc,
                         const std::vector<int>& shots, const float* recloc, int nrec,
                         const float* wavelet, const float* c11, const float* c13,
                         const float* c33, float* ddata, float* wavefield) {
  Device* dev = device(dev_id);
  if (!dev) return false;
  std::lock_guard<std::mutex> lk(dev->mu);
  vti3d_plan* p = plan_for(dev, g, flags);
  return p &&
         report(dev->ctx, vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr, VTI_MEM_HOST),
                "model") &&
         report(dev->ctx, vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST), "wavelet") &&
         report(dev->ctx, vti3d_plan_set_receivers(p, recloc, nrec), "receivers") &&
         report(dev->ctx, vti3d_plan_model_data(p, souloc, shots.data(), (int)shots.size(),
                                                ddata, VTI_MEM_HOST), "modeling") &&
         report(dev->ctx, vti3d_plan_get_wavefield(p, wavefield, VTI_MEM_HOST), "wavefield");
}
}  // namespace

void modelData3d_f(float* souloc, int ns, float* recloc, float* wavelet, float* c11, float* c13,
                   float* c33, int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                   float oz, float ot, float dx, float dy, float dz, float dt, float samplingRate) {
  // modelData3d_f.cu:15-330: all shots, traces appended to data=, last
  // level of the last shot to wavefield=
  std::vector<int> gpus = gpus_from_argv();
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  std::vector<int> shots(ns);
  for (int i = 0; i < ns; ++i) shots[i] = i;
  const int nrec = total_receivers(souloc, shots);
  const int nnt = nnt_of(g);
  std::vector<float> ddata((size_t)nnt * nrec, 0.f), wf((size_t)nx * ny * nz, 0.f);
  const unsigned flags = ref_flags(gpus.size());
  if (!model_and_wavefield(g, flags, gpus[0], souloc, shots, recloc, nrec, wavelet, c11, c13,
                           c33, ddata.data(), wf.data()))
    return;
  for (int is = 0; is < ns; ++is) {
    const int nr = (int)souloc[5 * is + 3], irb = (int)souloc[5 * is + 4];
    sep_write("data", ddata.data() + (size_t)nnt * irb, (size_t)nnt * nr, true);
  }
  const int nrtotal = (int)souloc[5 * (ns - 1) + 3] + (int)souloc[5 * (ns - 1) + 4];
  to_header("data", "n1", nnt);
  to_header("data", "o1", ot);
  to_header("data", "d1", samplingRate);
  to_header("data", "n2", nrtotal);
  to_header("data", "o2", 0.);
  to_header("data", "d2", 1);
  sep_write("wavefield", wf.data(), wf.size(), false);
  to_header("wavefield", "n1", nx); to_header("wavefield", "o1", ox); to_header("wavefield", "d1", dx);
  to_header("wavefield", "n2", ny); to_header("wavefield", "o2", oy); to_header("wavefield", "d2", dy);
  to_header("wavefield", "n3", nz); to_header("wavefield", "o3", oz); to_header("wavefield", "d3", dz);
}

void modeling3d_f(float soulocX, float soulocY, float soulocZ, float* wavelet, float* c11,
                  float* c13, float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
                  float oy, float oz, float ot, float dx, float dy, float dz, float dt) {
  // modeling3d_f.cu:15-270: one shot, last sigma_x level to wavefield=
  std::vector<int> gpus = gpus_from_argv();
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, dt);
  float souloc[5] = {soulocX, soulocY, soulocZ, 0.f, 0.f};
  std::vector<int> shots{0};
  std::vector<float> wf((size_t)nx * ny * nz, 0.f);
  float dummy = 0.f;
  if (!model_and_wavefield(g, ref_flags(gpus.size()), gpus[0], souloc, shots, nullptr, 0, wavelet,
                           c11, c13, c33, &dummy, wf.data()))
    return;
  sep_write("wavefield", wf.data(), wf.size(), false);
  to_header("wavefield", "n1", nx); to_header("wavefield", "o1", ox); to_header("wavefield", "d1", dx);
  to_header("wavefield", "n2", ny); to_header("wavefield", "o2", oy); to_header("wavefield", "d2", dy);
  to_header("wavefield", "n3", nz); to_header("wavefield", "o3", oz); to_header("wavefield", "d3", dz);
}

// ---------------------------------------------------------------- 2D
void synthetic_f(float* d, const float* c11, const float* c13, const float* c33,
                 const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                 const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot) {
  // synthetic_f.cu:58-124: shots over the gpu= devices
  std::vector<int> gpus = gpus_from_argv();
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  std::vector<int> shots(ns);
  for (int i = 0; i < ns; ++i) shots[i] = i;
  over_gpus(gpus, shots, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    for (int is : sub)
      if (!report(dev->ctx, vti2d_synthetic(dev->ctx, &g, c11, c13, c33, wavelet, sloc + 4 * is,
                                             1, rloc, nr, taper, d), "synthetic"))
        return false;
    return true;
  });
}

void modeling_f(float* d, const float* c11, const float* c13, const float* c33,
                const float* wavelet, int slocxz, const float* taper, int nx, int nz, int nt,
                int npad, float dx, float dz, float dt, float rate, float ot) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  Device* dev = device(0);
  if (dev) {
    std::lock_guard<std::mutex> lk(dev->mu);
    report(dev->ctx, vti2d_modeling(dev->ctx, &g, c11, c13, c33, wavelet, slocxz, taper, d),
           "modeling");
  }
}

namespace {
// Shots of pass p on GPU i are is = p*nGPUs + i (objFuncGradient_f.cu:138-147,
// hessian_f.cu the same); each GPU keeps its own checkpoint buffers across its
// shots, so every device processes exactly that subsequence, in order.
std::vector<std::vector<int>> shots_per_gpu(int ns, size_t ngpu) {
  std::vector<std::vector<int>> part(ngpu);
  for (int is = 0; is < ns; ++is) part[is % ngpu].push_back(is);
  return part;
}

// Runs the 2D gradient (dc == nullptr) or GN product on the gpu= devices and
// sums the per-device results.
double grad2d_over_gpus(float* gc11, float* gc13, float* gc33, const float* data,
                        const float* c11, const float* c13, const float* c33, const float* dc11,
                        const float* dc13, const float* dc33, const float* wavelet,
                        const int* sloc, int ns, const int* rloc, int nr, const float* taper,
                        const vti2d_geom& g) {
  const std::vector<int> gpus = gpus_from_argv();
  const size_t n = (size_t)(g.nx + 2 * g.npad) * (g.nz + 2 * g.npad);
  auto parts = shots_per_gpu(ns, gpus.size());
  std::vector<std::vector<float>> out(gpus.size());
  std::vector<double> mis(gpus.size(), 0.0);
  std::vector<int> ok(gpus.size(), 1);
  std::vector<std::thread> th;
  for (size_t k = 0; k < gpus.size(); ++k) {
    if (parts[k].empty()) continue;
    th.emplace_back([&, k]() {
      Device* dev = device(gpus[k]);
      if (!dev) {
        ok[k] = 0;
        return;
      }
      std::lock_guard<std::mutex> lk(dev->mu);
      std::vector<int> sl;
      for (int is : parts[k]) sl.insert(sl.end(), sloc + 4 * is, sloc + 4 * is + 4);
      out[k].assign(3 * n, 0.f);
      int st = dc11 ? vti2d_gn_hessian(dev->ctx, &g, out[k].data(), out[k].data() + n,
                                       out[k].data() + 2 * n, c11, c13, c33, dc11, dc13, dc33,
                                       wavelet, sl.data(), (int)parts[k].size(), rloc, nr, taper)
                    : vti2d_gradient(dev->ctx, &g, out[k].data(), out[k].data() + n,
                                     out[k].data() + 2 * n, data, c11, c13, c33, wavelet,
                                     sl.data(), (int)parts[k].size(), rloc, nr, taper, &mis[k]);
      ok[k] = report(dev->ctx, st, dc11 ? "GNhessian" : "gradient") ? 1 : 0;
    });
  }
  for (auto& t : th) t.join();
  // objFuncGradient_f.cu:25-27: outputs zeroed, per-GPU sums added
  std::memset(gc11, 0, n * sizeof(float));
  std::memset(gc13, 0, n * sizeof(float));
  std::memset(gc33, 0, n * sizeof(float));
  double total = 0;
  for (size_t k = 0; k < gpus.size(); ++k) {
    if (out[k].empty()) continue;
    total += mis[k];
    for (size_t i = 0; i < n; ++i) {
      gc11[i] += out[k][i];
      gc13[i] += out[k][n + i];
      gc33[i] += out[k][2 * n + i];
    }
  }
  for (int v : ok)
    if (!v) return NAN;
  return total;
}
}  // namespace

float objFuncGradient_f(float* gc11, float* gc13, float* gc33, const float* data,
                        const float* c11, const float* c13, const float* c33, const float* wavelet,
                        const int* sloc, int ns, const int* rloc, int nr, const float* taper,
                        int nx, int nz, int nt, int npad, float dx, float dz, float dt, float rate,
                        float ot) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  return (float)grad2d_over_gpus(gc11, gc13, gc33, data, c11, c13, c33, nullptr, nullptr, nullptr,
                                 wavelet, sloc, ns, rloc, nr, taper, g);
}

void GNhessian_f(float* gc11, float* gc13, float* gc33, const float* data, const float* c11,
                 const float* c13, const float* c33, const float* dc11, const float* dc13,
                 const float* dc33, const float* wavelet, const int* sloc, int ns, const int* rloc,
                 int nr, const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  grad2d_over_gpus(gc11, gc13, gc33, data, c11, c13, c33, dc11, dc13, dc33, wavelet, sloc, ns,
                   rloc, nr, taper, g);
}

float objFuncGradientVEpsDel(float* gv, float* geps, float* gdel, const float* data, float* v,
                             float* eps, float* del, float v0, float eps0, float del0,
                             const float* wavelet, const int* sloc, int ns, const int* rloc,
                             int nr, const float* taper, int nx, int nz, int nt, int npad,
                             float dx, float dz, float dt, float rate, float ot, float wbottom,
                             float* m) {
  // objFuncGradient.cu:28-54
  const int nnx = nx + 2 * npad, nnz = nz + 2 * npad;
  const size_t n = (size_t)nnx * nnz;
  vti_check_eps_del(eps, del, eps0, del0, n, m);
  std::vector<float> c(3 * n), gc(3 * n);
  vti_vepsdel_to_cij(c.data(), c.data() + n, c.data() + 2 * n, v, eps, del, v0, eps0, del0, n);
  double val = objFuncGradient_f(gc.data(), gc.data() + n, gc.data() + 2 * n, data, c.data(),
                                 c.data() + n, c.data() + 2 * n, wavelet, sloc, ns, rloc, nr,
                                 taper, nx, nz, nt, npad, dx, dz, dt, rate, ot);
  vti_grad_cij_to_vepsdel(gv, geps, gdel, gc.data(), gc.data() + n, gc.data() + 2 * n, v, eps,
                          del, v0, eps0, del0, n);
  int nwbottom = wbottom / dz + 1;
  size_t rows = std::min<size_t>((size_t)(npad + nwbottom), (size_t)nnz);
  std::memset(gv, 0, rows * nnx * sizeof(float));
  std::memset(geps, 0, rows * nnx * sizeof(float));
  std::memset(gdel, 0, rows * nnx * sizeof(float));
  return (float)val;
}

void GNhessianVEpsDel(float* gv, float* geps, float* gdel, const float* d0, float* v, float* eps,
                      float* del, const float* dv, const float* deps, const float* ddel, float v0,
                      float eps0, float del0, const float* wavelet, const int* sloc, int ns,
                      const int* rloc, int nr, const float* taper, int nx, int nz, int nt,
                      int npad, float dx, float dz, float dt, float rate, float ot, float wbottom,
                      float* m) {
  // hessians.cu:72-95
  const int nnx = nx + 2 * npad, nnz = nz + 2 * npad;
  const size_t n = (size_t)nnx * nnz;
  vti_check_eps_del(eps, del, eps0, del0, n, m);
  std::vector<float> c(3 * n), dc(3 * n), gc(3 * n);
  vti_dvepsdel_to_dcij(c.data(), c.data() + n, c.data() + 2 * n, dc.data(), dc.data() + n,
                       dc.data() + 2 * n, v, eps, del, dv, deps, ddel, v0, eps0, del0, n);
  GNhessian_f(gc.data(), gc.data() + n, gc.data() + 2 * n, d0, c.data(), c.data() + n,
              c.data() + 2 * n, dc.data(), dc.data() + n, dc.data() + 2 * n, wavelet, sloc, ns,
              rloc, nr, taper, nx, nz, nt, npad, dx, dz, dt, rate, ot);
  vti_grad_cij_to_vepsdel(gv, geps, gdel, gc.data(), gc.data() + n, gc.data() + 2 * n, v, eps,
                          del, v0, eps0, del0, n);
  size_t rows = std::min<size_t>((size_t)(npad + wbottom / dz + 1), (size_t)nnz);
  std::memset(gv, 0, rows * nnx * sizeof(float));
  std::memset(geps, 0, rows * nnx * sizeof(float));
  std::memset(gdel, 0, rows * nnx * sizeof(float));
}

// hessians.cu:28-45 and checkCij (check.cpp:6-20).
void GNhessianCij(float* gc11, float* gc13, float* gc33, const float* d0, float* c11, float* c13,
                  float* c33, const float* dc11, const float* dc13, const float* dc33, float c110,
                  float c130, float c330, const float* wavelet, const int* sloc, int ns,
                  const int* rloc, int nr, const float* taper, int nx, int nz, int nt, int npad,
                  float dx, float dz, float dt, float rate, float ot, float wbottom, float* m) {
  const int nnx = nx + 2 * npad, nnz = nz + 2 * npad;
  const size_t n = (size_t)nnx * nnz;
  int count = 0;
  std::memset(m, 0, n * sizeof(float));
  for (size_t i = 0; i < n; ++i) {
    const float bound = std::sqrt(c110 * c11[i] * c330 * c33[i]) / c130;
    if (c13[i] > bound) {
      c13[i] = (float)(0.99 * bound);
      ++count;
      m[i] = 1.f;
    }
  }
  std::fprintf(stderr, "Modified models at %d points\n", count);
  std::vector<float> c(3 * n), dc(3 * n);
  for (size_t i = 0; i < n; ++i) {
    c[i] = c11[i] * c110;
    c[n + i] = c13[i] * c130;
    c[2 * n + i] = c33[i] * c330;
    dc[i] = dc11[i] * c110;
    dc[n + i] = dc13[i] * c130;
    dc[2 * n + i] = dc33[i] * c330;
  }
  GNhessian_f(gc11, gc13, gc33, d0, c.data(), c.data() + n, c.data() + 2 * n, dc.data(),
              dc.data() + n, dc.data() + 2 * n, wavelet, sloc, ns, rloc, nr, taper, nx, nz, nt,
              npad, dx, dz, dt, rate, ot);
  const size_t rows = std::min<size_t>((size_t)(int)(npad + wbottom / dz + 1), (size_t)nnz);
  float* gs[3] = {gc11, gc13, gc33};
  const float sc[3] = {c110, c130, c330};
  for (int k = 0; k < 3; ++k) {
    std::memset(gs[k], 0, rows * nnx * sizeof(float));
    for (size_t i = 0; i < n; ++i) gs[k][i] *= sc[k];
  }
}

// Operator interface of the GN Hessian (HessianOp.cu:29-51, 77-99): the
// product is symmetric, so forward and adjoint are the same call; add = true
// accumulates into the output.
namespace {
template <typename F>
void apply_op(bool add, long long size, float* out, F&& product) {
  if (!add) {
    product(out);
    return;
  }
  std::vector<float> t((size_t)size, 0.f);
  product(t.data());
  for (long long i = 0; i < size; ++i) out[i] += t[i];
}
}  // namespace

void GNHessianOpCij::forward(bool add, const float* model, float* data) {
  const long long n = (long long)(_nx + 2 * _npad) * (_nz + 2 * _npad);
  apply_op(add, _dataSize, data, [&](float* o) {
    GNhessianCij(o, o + n, o + 2 * n, _d0, _c11, _c13, _c33, model, model + n, model + 2 * n,
                 _c110, _c130, _c330, _wavelet, _sloc, _ns, _rloc, _nr, _taper, _nx, _nz, _nt,
                 _npad, _dx, _dz, _dt, _rate, _ot, _wbottom, _m);
  });
}

void GNHessianOpCij::adjoint(bool add, float* model, const float* data) {
  const long long n = (long long)(_nx + 2 * _npad) * (_nz + 2 * _npad);
  apply_op(add, _modelSize, model, [&](float* o) {
    GNhessianCij(o, o + n, o + 2 * n, _d0, _c11, _c13, _c33, data, data + n, data + 2 * n,
                 _c110, _c130, _c330, _wavelet, _sloc, _ns, _rloc, _nr, _taper, _nx, _nz, _nt,
                 _npad, _dx, _dz, _dt, _rate, _ot, _wbottom, _m);
  });
}

void GNHessianOpVEpsDel::forward(bool add, const float* model, float* data) {
  const long long n = (long long)(_nx + 2 * _npad) * (_nz + 2 * _npad);
  apply_op(add, _dataSize, data, [&](float* o) {
    GNhessianVEpsDel(o, o + n, o + 2 * n, _d0, _v, _eps, _del, model, model + n, model + 2 * n,
                     _v0, _eps0, _del0, _wavelet, _sloc, _ns, _rloc, _nr, _taper, _nx, _nz, _nt,
                     _npad, _dx, _dz, _dt, _rate, _ot, _wbottom, _m);
  });
}

void GNHessianOpVEpsDel::adjoint(bool add, float* model, const float* data) {
  const long long n = (long long)(_nx + 2 * _npad) * (_nz + 2 * _npad);
  apply_op(add, _modelSize, model, [&](float* o) {
    GNhessianVEpsDel(o, o + n, o + 2 * n, _d0, _v, _eps, _del, data, data + n, data + 2 * n,
                     _v0, _eps0, _del0, _wavelet, _sloc, _ns, _rloc, _nr, _taper, _nx, _nz, _nt,
                     _npad, _dx, _dz, _dt, _rate, _ot, _wbottom, _m);
  });
}

// ---------------------------------------------------------------- RTM
// rtmCij3d_f (rtm3d_f.cu:161-620): devices from gpu=, three floats (x, y, z)
// per receiver, each shot's traces read from data= (rtm3d_f.cu:505); the
// model is used as passed (the caller puts the random boundary in). Images of
// the devices' shots are summed.
void rtmCij3d_f(float* image, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                float* wavelet, float* c11, float* c13, float* c33, int nx, int ny, int nz,
                int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                float dz, float dt, float samplingRate) {
  (void)ns;
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  const size_t n = (size_t)nx * ny * nz;
  std::memset(image, 0, n * sizeof(float));
  const std::vector<int> gpus = gpus_from_argv();
  const int nrec = total_receivers(souloc, shotid);
  std::vector<float> rec4(4 * (size_t)nrec);
  for (int ir = 0; ir < nrec; ++ir) {
    for (int k = 0; k < 3; ++k) rec4[4 * (size_t)ir + k] = recloc[3 * (size_t)ir + k];
    rec4[4 * (size_t)ir + 3] = 1.f;
  }
  std::vector<float> data;
  int nr_read = 0;
  if (!read_observed(souloc, shotid, g, &data, &nr_read)) return;
  const unsigned flags = ref_flags(gpus.size());
  std::vector<std::vector<float>> parts(gpus.size());
  std::map<int, size_t> slot;
  for (size_t i = 0; i < gpus.size(); ++i) slot[gpus[i]] = i;
  over_gpus(gpus, shotid, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    vti3d_plan* p = plan_for(dev, g, flags);
    if (!p) return false;
    std::vector<float>& img = parts[slot[id]];
    img.assign(n, 0.f);
    return report(dev->ctx, vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr,
                                                 VTI_MEM_HOST), "model") &&
           report(dev->ctx, vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST), "wavelet") &&
           report(dev->ctx, vti3d_plan_set_receivers(p, rec4.data(), nrec), "receivers") &&
           report(dev->ctx, vti3d_plan_rtm(p, souloc, sub.data(), (int)sub.size(), data.data(),
                                           VTI_MEM_HOST, img.data(), VTI_MEM_HOST), "rtm");
  });
  for (auto& img : parts)
    if (!img.empty())
      for (size_t i = 0; i < n; ++i) image[i] += img[i];
}

// rtmVEpsDel (rtm3d_f.cu:139-159): v, eps, del -> c_ij with unit scales,
// migration, then the pad region and the water layer of the image zeroed.
void rtmVEpsDel(float* image, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                float* wavelet, float* v, float* eps, float* del, float* randboundaryV, int nx,
                int ny, int nz, int nt, int npad, float ox, float oy, float oz, float ot,
                float dx, float dy, float dz, float dt, float samplingRate, float wbottom) {
  (void)randboundaryV;  // the reference leaves its putBoundary call commented out
  const size_t nxy = (size_t)nx * ny, n = nxy * nz;
  std::vector<float> c(3 * n);
  vti_vepsdel_to_cij(c.data(), c.data() + n, c.data() + 2 * n, v, eps, del, 1.f, 1.f, 1.f, n);
  rtmCij3d_f(image, souloc, ns, shotid, recloc, wavelet, c.data(), c.data() + n,
             c.data() + 2 * n, nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt,
             samplingRate);
  vti3d_zero_boundary(image, nx, ny, nz, npad);
  const int nwbottom = (int)((wbottom - oz) / dz + 1 - npad);
  if (nwbottom > 0)
    std::memset(image + (size_t)npad * nxy, 0,
                std::min<size_t>((size_t)nwbottom, (size_t)nz - npad) * nxy * sizeof(float));
}

// odcig3d_f (odcig3d_f.cu:15-543): all ns shots, v/eps/del converted with
// unit scales (the c13 = c33 sqrt(1 + 2 del) of wave3d.cu:86), the migration
// of rtmCij3d_f with the x-offset gathers of extendedImagingKernel
// (wave3d.cu:1299-1313) for |lag| <= 32 (NLAG, wave3d.h:19). Images of the
// devices' shots are summed.
void odcig3d_f(float* image, float* souloc, int ns, float* recloc, float* wavelet, float* v,
               float* eps, float* del, int nx, int ny, int nz, int nt, int npad, float ox,
               float oy, float oz, float ot, float dx, float dy, float dz, float dt,
               float samplingRate) {
  constexpr int kNlag = 32;
  const size_t n = (size_t)nx * ny * nz, nimg = (2 * kNlag + 1) * n;
  std::memset(image, 0, nimg * sizeof(float));
  std::vector<float> c(3 * n);
  vti_vepsdel_to_cij(c.data(), c.data() + n, c.data() + 2 * n, v, eps, del, 1.f, 1.f, 1.f, n);
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  std::vector<int> shotid(ns);
  for (int i = 0; i < ns; ++i) shotid[i] = i;
  const std::vector<int> gpus = gpus_from_argv();
  const int nrec = total_receivers(souloc, shotid);
  std::vector<float> rec4(4 * (size_t)nrec);
  for (int ir = 0; ir < nrec; ++ir) {
    for (int k = 0; k < 3; ++k) rec4[4 * (size_t)ir + k] = recloc[3 * (size_t)ir + k];
    rec4[4 * (size_t)ir + 3] = 1.f;
  }
  std::vector<float> data;
  int nr_read = 0;
  if (!read_observed(souloc, shotid, g, &data, &nr_read)) return;
  const unsigned flags = ref_flags(gpus.size());
  std::vector<std::vector<float>> parts(gpus.size());
  std::map<int, size_t> slot;
  for (size_t i = 0; i < gpus.size(); ++i) slot[gpus[i]] = i;
  over_gpus(gpus, shotid, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    vti3d_plan* p = plan_for(dev, g, flags);
    if (!p) return false;
    std::vector<float>& img = parts[slot[id]];
    img.assign(nimg, 0.f);
    return report(dev->ctx, vti3d_plan_set_model(p, c.data(), c.data() + n, c.data() + 2 * n,
                                                 nullptr, nullptr, VTI_MEM_HOST), "model") &&
           report(dev->ctx, vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST), "wavelet") &&
           report(dev->ctx, vti3d_plan_set_receivers(p, rec4.data(), nrec), "receivers") &&
           report(dev->ctx, vti3d_plan_odcig(p, souloc, sub.data(), (int)sub.size(),
                                             data.data(), VTI_MEM_HOST, kNlag, img.data(),
                                             VTI_MEM_HOST), "odcig");
  });
  for (auto& img : parts)
    if (!img.empty())
      for (size_t i = 0; i < nimg; ++i) image[i] += img[i];
}

// rtm_f (rtm_f.cu:13-267): shots round-robin over the gpu= devices
// (is = pass*nGPUs + i), per-device images summed.
void rtm_f(float* image, const float* data, const float* c11, const float* c13, const float* c33,
           const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
           const float* taper, int nx, int nz, int nt, int npad, float dx, float dz, float dt,
           float rate, float ot) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  const size_t n = (size_t)(nx + 2 * npad) * (nz + 2 * npad);
  std::memset(image, 0, n * sizeof(float));
  const std::vector<int> gpus = gpus_from_argv();
  auto parts = shots_per_gpu(ns, gpus.size());
  std::vector<std::vector<float>> img(gpus.size());
  std::vector<std::thread> th;
  for (size_t k = 0; k < gpus.size(); ++k) {
    if (parts[k].empty()) continue;
    th.emplace_back([&, k]() {
      Device* dev = device(gpus[k]);
      if (!dev) return;
      std::lock_guard<std::mutex> lk(dev->mu);
      std::vector<int> sl;
      for (int is : parts[k]) sl.insert(sl.end(), sloc + 4 * is, sloc + 4 * is + 4);
      img[k].assign(n, 0.f);
      if (!report(dev->ctx, vti2d_rtm(dev->ctx, &g, img[k].data(), data, c11, c13, c33, wavelet,
                                      sl.data(), (int)parts[k].size(), rloc, nr, taper), "rtm"))
        img[k].clear();
    });
  }
  for (auto& t : th) t.join();
  for (auto& v : img)
    if (!v.empty())
      for (size_t i = 0; i < n; ++i) image[i] += v[i];
}

// ---------------------------------------------------------- wavelet gradient
// waveletGradientCij3d_f (modelData3d_f.cu:858-1294): the traces come in ddata
// (nnt per receiver, shot ranges at nnt*irbegin); shots round-robin over the
// GPUs, per-device results summed. The level count follows the pipeline of
// GPUs.size() devices.
void waveletGradientCij3d_f(float* gwavelet, const float* ddata, float* souloc, int ns,
                            std::vector<int>& shotid, float* recloc, float* c11, float* c13,
                            float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
                            float oy, float oz, float ot, float dx, float dy, float dz, float dt,
                            float samplingRate, std::vector<int>& GPUs) {
  (void)ns;
  vti3d_geom g = geom3(nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate);
  std::memset(gwavelet, 0, nt * sizeof(float));
  const int nrec = total_receivers(souloc, shotid);
  const unsigned flags = ref_flags(GPUs.size());
  std::vector<std::vector<float>> parts(GPUs.size());
  std::map<int, size_t> slot;
  for (size_t i = 0; i < GPUs.size(); ++i) slot[GPUs[i]] = i;
  over_gpus(GPUs, shotid, [&](int id, const std::vector<int>& sub) {
    Device* dev = device(id);
    if (!dev) return false;
    std::lock_guard<std::mutex> lk(dev->mu);
    vti3d_plan* p = plan_for(dev, g, flags);
    if (!p) return false;
    std::vector<float>& gw = parts[slot[id]];
    gw.assign(nt, 0.f);
    return report(dev->ctx, vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr,
                                                 VTI_MEM_HOST), "model") &&
           report(dev->ctx, vti3d_plan_set_receivers(p, recloc, nrec), "receivers") &&
           report(dev->ctx, vti3d_plan_wavelet_gradient(p, souloc, sub.data(), (int)sub.size(),
                                                        ddata, VTI_MEM_HOST, gw.data(),
                                                        VTI_MEM_HOST), "wavelet gradient");
  });
  for (auto& gw : parts)
    if (!gw.empty())
      for (int i = 0; i < nt; ++i) gwavelet[i] += gw[i];
}

// waveletGradient3d_f (modelData3d_f.cu:810-856): contiguous shot groups, one
// per GPU group, summed.
void waveletGradient3d_f(float* gwavelet, const float* ddata, float* souloc, int ns,
                         std::vector<int>& shotid, float* recloc, float* c11, float* c13,
                         float* c33, int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                         float oz, float ot, float dx, float dy, float dz, float dt,
                         float samplingRate, std::vector<int>& GPUs, int ngpugroup) {
  if (ngpugroup <= 1) {
    waveletGradientCij3d_f(gwavelet, ddata, souloc, ns, shotid, recloc, c11, c13, c33, nx, ny,
                           nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate, GPUs);
    return;
  }
  const int ngpu1 = (int)GPUs.size() / ngpugroup;
  const int nshot1 = (int)shotid.size() / ngpugroup, r = (int)shotid.size() % ngpugroup;
  std::vector<std::vector<float>> gw(ngpugroup, std::vector<float>(nt));
  std::vector<std::thread> th;
  for (int i = 0; i < ngpugroup; ++i) {
    th.emplace_back([&, i]() {
      std::vector<int> gpus(GPUs.begin() + i * ngpu1, GPUs.begin() + (i + 1) * ngpu1);
      int b = i < r ? i * (nshot1 + 1) : r * (nshot1 + 1) + (i - r) * nshot1;
      int e = b + (i < r ? nshot1 + 1 : nshot1);
      std::vector<int> sh(shotid.begin() + b, shotid.begin() + e);
      waveletGradientCij3d_f(gw[i].data(), ddata, souloc, ns, sh, recloc, c11, c13, c33, nx, ny,
                             nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, samplingRate, gpus);
    });
  }
  for (auto& t : th) t.join();
  std::memset(gwavelet, 0, nt * sizeof(float));
  for (int i = ngpugroup - 1; i >= 0; --i)  // the reference's summation order
    for (int j = 0; j < nt; ++j) gwavelet[j] += gw[i][j];
}

// Source-inversion operator (ModelingOp3d.cu:12-33): traces of the wavelet
// `model`, and the wavelet gradient of the traces `data`; add = true
// accumulates.
void ModelingOp3d::forward(bool add, const float* model, float* data) {
  apply_op(add, _dataSize, data, [&](float* o) {
    modelData3d_f(o, _souloc, _ns, _shotid, _recloc, model, _c11, _c13, _c33, _nx, _ny, _nz, _nt,
                  _npad, _ox, _oy, _oz, _ot, _dx, _dy, _dz, _dt, _samplingRate, _GPUs,
                  _ngpugroup);
  });
}

void ModelingOp3d::adjoint(bool add, float* model, const float* data) {
  apply_op(add, _modelSize, model, [&](float* o) {
    waveletGradient3d_f(o, data, _souloc, _ns, _shotid, _recloc, _c11, _c13, _c33, _nx, _ny, _nz,
                        _nt, _npad, _ox, _oy, _oz, _ot, _dx, _dy, _dz, _dt, _samplingRate, _GPUs,
                        _ngpugroup);
  });
}

// waveletGradient_f (objFuncGradient_f.cu:373-530): shots round-robin over the
// gpu= devices (the reference uses every visible device; the result does not
// depend on the device count), per-device sums added.
void waveletGradient_f(float* gwavelet, const float* d0, const float* c11, const float* c13,
                       const float* c33, const int* sloc, int ns, const int* rloc, int nr,
                       const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                       float dt, float rate) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, 0.f};
  std::memset(gwavelet, 0, nt * sizeof(float));
  const std::vector<int> gpus = gpus_from_argv();
  auto parts = shots_per_gpu(ns, gpus.size());
  std::vector<std::vector<float>> gw(gpus.size());
  std::vector<std::thread> th;
  for (size_t k = 0; k < gpus.size(); ++k) {
    if (parts[k].empty()) continue;
    th.emplace_back([&, k]() {
      Device* dev = device(gpus[k]);
      if (!dev) return;
      std::lock_guard<std::mutex> lk(dev->mu);
      std::vector<int> sl;
      for (int is : parts[k]) sl.insert(sl.end(), sloc + 4 * is, sloc + 4 * is + 4);
      gw[k].assign(nt, 0.f);
      if (!report(dev->ctx, vti2d_wavelet_gradient(dev->ctx, &g, gw[k].data(), d0, c11, c13, c33,
                                                   sl.data(), (int)parts[k].size(), rloc, nr,
                                                   taper), "wavelet gradient"))
        gw[k].clear();
    });
  }
  for (auto& t : th) t.join();
  for (auto& v : gw)
    if (!v.empty())
      for (int i = 0; i < nt; ++i) gwavelet[i] += v[i];
}

// odcig_f (odcig_f.cu:12-232): shots round-robin over the gpu= devices,
// per-device gathers summed.
void odcig_f(float* image, const float* data, const float* c11, const float* c13,
             const float* c33, const float* wavelet, const int* sloc, int ns, const int* rloc,
             int nr, const float* taper, int nx, int nz, int nhx, int nt, int npad, float dx,
             float dz, float dt, float rate, float ot) {
  vti2d_geom g{nx, nz, nt, npad, dx, dz, dt, rate, ot};
  const size_t n = (size_t)(nx + 2 * npad) * (nz + 2 * npad) * (2 * (size_t)std::max(nhx, 0) + 1);
  std::memset(image, 0, n * sizeof(float));
  const std::vector<int> gpus = gpus_from_argv();
  auto parts = shots_per_gpu(ns, gpus.size());
  std::vector<std::vector<float>> img(gpus.size());
  std::vector<std::thread> th;
  for (size_t k = 0; k < gpus.size(); ++k) {
    if (parts[k].empty()) continue;
    th.emplace_back([&, k]() {
      Device* dev = device(gpus[k]);
      if (!dev) return;
      std::lock_guard<std::mutex> lk(dev->mu);
      std::vector<int> sl;
      for (int is : parts[k]) sl.insert(sl.end(), sloc + 4 * is, sloc + 4 * is + 4);
      img[k].assign(n, 0.f);
      if (!report(dev->ctx, vti2d_odcig(dev->ctx, &g, nhx, img[k].data(), data, c11, c13, c33,
                                        wavelet, sl.data(), (int)parts[k].size(), rloc, nr,
                                        taper), "odcig"))
        img[k].clear();
    });
  }
  for (auto& t : th) t.join();
  for (auto& v : img)
    if (!v.empty())
      for (size_t i = 0; i < n; ++i) image[i] += v[i];
}
