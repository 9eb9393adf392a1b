// Harness that runs the REFERENCE's own 3D GPU path (compiled from its
// sources by oracle/build_ref.sh into oracle/_ref/ref3d) on inputs written by
// tests/golden/make_golden.py. TEST INFRASTRUCTURE ONLY: it produces golden
// traces and gradients that pin the oracle; nothing in the library uses it.
//
// usage: ref3d <dir> model|grad|rtm|wgrad|modop|odcig [key=value ...] (modop,
//   odcig: built with -DVTI_SHIM against libvti_wave.so, which provides
//   ModelingOp3d and a linkable odcig3d_f)
//   <dir>/params.txt : nx ny nz nt npad ox oy oz ot dx dy dz dt rate ns nrec
//   <dir>/{souloc,recloc,wavelet,cij,padb,randb,dobs}.bin (float32)
//   writes <dir>/ref_ddata.bin (model), <dir>/ref_fgcij.bin (grad) or
//   <dir>/ref_image.bin (rtm: the traces in dobs.bin migrated with cij) or
//   <dir>/ref_wgrad.bin (wgrad: wavelet gradient driven by dobs.bin)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#ifdef VTI_SHIM
// built against libvti_wave.so: the source-inversion operator class
// (ModelingOp3d.h) and odcig3d_f (wave3d.h:116; the reference's own target
// does not link) are available as well (modes modop, odcig)
#include "vti_modeling_op3d.h"
void odcig3d_f(float* image, float* souloc, int ns, float* recloc, float* wavelet, float* v,
               float* eps, float* del, int nx, int ny, int nz, int nt, int npad, float ox,
               float oy, float oz, float ot, float dx, float dy, float dz, float dt,
               float samplingRate);
#endif

// Entry points of lib/vti-fwi-3d/gpu (wave3d.h:84-122) and lib/io/myio.cpp:15.
void myio_init(int argc, char** argv);
void modelDataCij3d_f(float* ddata, float* souloc, int ns, std::vector<int>& shotid,
                      float* recloc, const float* wavelet, float* c11, float* c13, float* c33,
                      int nx, int ny, int nz, int nt, int npad, float ox, float oy, float oz,
                      float ot, float dx, float dy, float dz, float dt, float samplingRate,
                      std::vector<int>& GPUs);
void objFuncGradientCij3d_f(float* fgcij, float* souloc, int ns, std::vector<int>& shotid,
                            float* recloc, float* wavelet, float* cij, float* padboundaryCij,
                            float* randboundaryCij, int nx, int ny, int nz, int nt, int npad,
                            float ox, float oy, float oz, float ot, float dx, float dy, float dz,
                            float dt, float samplingRate, std::vector<int>& GPUs);
void waveletGradientCij3d_f(float* gwavelet, const float* ddata, float* souloc, int ns,
                            std::vector<int>& shotid, float* recloc, float* c11, float* c13,
                            float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
                            float oy, float oz, float ot, float dx, float dy, float dz, float dt,
                            float samplingRate, std::vector<int>& GPUs);
void rtmCij3d_f(float* image, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                float* wavelet, float* c11, float* c13, float* c33, int nx, int ny, int nz,
                int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                float dz, float dt, float samplingRate);

static std::vector<float> load(const std::string& path, size_t n) {
  std::vector<float> v(n);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot read %s (%zu floats)\n", path.c_str(), n);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

static void save(const std::string& path, const float* p, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(p, sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <dir> model|grad|rtm|wgrad\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1], mode = argv[2];
  std::ifstream pf(dir + "/params.txt");
  int nx, ny, nz, nt, npad, ns, nrec;
  float ox, oy, oz, ot, dx, dy, dz, dt, rate;
  if (!(pf >> nx >> ny >> nz >> nt >> npad >> ox >> oy >> oz >> ot >> dx >> dy >> dz >> dt >>
        rate >> ns >> nrec)) {
    std::fprintf(stderr, "bad params.txt\n");
    return 2;
  }
  const size_t n = (size_t)nx * ny * nz;
  const size_t nb = n - (size_t)(nx - 2 * npad) * (ny - 2 * npad) * (nz - 2 * npad);
  const int st = (int)(rate / dt + 0.5f);
  const int nnt = (nt - 1) / st + 1;
  auto souloc = load(dir + "/souloc.bin", 5 * (size_t)ns);
  auto recloc = load(dir + "/recloc.bin", 4 * (size_t)nrec);
  auto wavelet = load(dir + "/wavelet.bin", nt);
  auto cij = load(dir + "/cij.bin", 3 * n);
  std::vector<int> shotid(ns), gpus{0};
  for (int i = 0; i < ns; ++i) shotid[i] = i;
  // side channel read by the reference: data=<header> (objFuncGradient3d_f.cu:760)
  const std::string hdr = dir + "/dobs.H";
  {
    std::ofstream h(hdr);
    h << "in=" << dir << "/dobs.bin\ndata_format=native_float\n";
  }
  // gpu= is read by rtmCij3d_f (rtm3d_f.cu:164); further key=value words on
  // the command line (tpow=, objtype=, halfwidth=) go to the reference's argv
  std::vector<std::string> words = {"ref3d", "data=" + hdr, "gpu=0"};
  for (int i = 3; i < argc; ++i) words.push_back(argv[i]);
  std::vector<char*> av;
  for (auto& w : words) av.push_back(&w[0]);
  av.push_back(nullptr);
  myio_init((int)words.size(), av.data());
  if (mode == "model") {
    std::vector<float> ddata((size_t)nnt * nrec, 0.f);
    modelDataCij3d_f(ddata.data(), souloc.data(), ns, shotid, recloc.data(), wavelet.data(),
                     cij.data(), cij.data() + n, cij.data() + 2 * n, nx, ny, nz, nt, npad, ox,
                     oy, oz, ot, dx, dy, dz, dt, rate, gpus);
    save(dir + "/ref_ddata.bin", ddata.data(), ddata.size());
  } else if (mode == "grad") {
    auto padb = load(dir + "/padb.bin", 3 * nb);
    auto randb = load(dir + "/randb.bin", 3 * nb);
    std::vector<float> fg(1 + 3 * n, 0.f);
    objFuncGradientCij3d_f(fg.data(), souloc.data(), ns, shotid, recloc.data(), wavelet.data(),
                           cij.data(), padb.data(), randb.data(), nx, ny, nz, nt, npad, ox, oy,
                           oz, ot, dx, dy, dz, dt, rate, gpus);
    save(dir + "/ref_fgcij.bin", fg.data(), fg.size());
  } else if (mode == "rtm") {
    // rtmCij3d_f reads three floats (x, y, z) per receiver (rtm3d_f.cu:347-350)
    std::vector<float> rec3(3 * (size_t)nrec);
    for (int ir = 0; ir < nrec; ++ir)
      for (int k = 0; k < 3; ++k) rec3[3 * ir + k] = recloc[4 * ir + k];
    std::vector<float> image(n, 0.f);
    rtmCij3d_f(image.data(), souloc.data(), ns, shotid, rec3.data(), wavelet.data(), cij.data(),
               cij.data() + n, cij.data() + 2 * n, nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy,
               dz, dt, rate);
    save(dir + "/ref_image.bin", image.data(), image.size());
  } else if (mode == "wgrad") {
    auto data = load(dir + "/dobs.bin", (size_t)nnt * nrec);
    std::vector<float> gw(nt, 0.f);
    waveletGradientCij3d_f(gw.data(), data.data(), souloc.data(), ns, shotid, recloc.data(),
                           cij.data(), cij.data() + n, cij.data() + 2 * n, nx, ny, nz, nt, npad,
                           ox, oy, oz, ot, dx, dy, dz, dt, rate, gpus);
    save(dir + "/ref_wgrad.bin", gw.data(), gw.size());
#ifdef VTI_SHIM
  } else if (mode == "modop") {
    // ModelingOp3d (ModelingOp3d.cu:12-33) with and without add: forward of
    // the wavelet -> ref_modop_fwd.bin, forward added onto ones ->
    // ref_modop_fwd_add.bin, adjoint of dobs.bin -> ref_modop_adj.bin,
    // adjoint added onto ones -> ref_modop_adj_add.bin
    ModelingOp3d op(souloc.data(), ns, shotid, recloc.data(), cij.data(), cij.data() + n,
                    cij.data() + 2 * n, nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt,
                    rate, gpus, 1);
    auto data = load(dir + "/dobs.bin", (size_t)nnt * nrec);
    std::vector<float> d0((size_t)op._dataSize, 0.f), d1((size_t)op._dataSize, 1.f);
    std::vector<float> m0((size_t)op._modelSize, 0.f), m1((size_t)op._modelSize, 1.f);
    op.forward(false, wavelet.data(), d0.data());
    op.forward(true, wavelet.data(), d1.data());
    op.adjoint(false, m0.data(), data.data());
    op.adjoint(true, m1.data(), data.data());
    save(dir + "/ref_modop_fwd.bin", d0.data(), d0.size());
    save(dir + "/ref_modop_fwd_add.bin", d1.data(), d1.size());
    save(dir + "/ref_modop_adj.bin", m0.data(), m0.size());
    save(dir + "/ref_modop_adj_add.bin", m1.data(), m1.size());
  } else if (mode == "odcig") {
    // odcig3d_f of the traces in dobs.bin with v, eps, del derived from cij
    // (c33 = v^2, c11 = c33 (1 + 2 eps), c13 = c33 sqrt(1 + 2 del)) ->
    // ref_odcig.bin (65 lags x nxyz)
    std::vector<float> v(n), eps(n), del(n);
    for (size_t i = 0; i < n; ++i) {
      const double c11 = cij[i], c13 = cij[n + i], c33 = cij[2 * n + i];
      v[i] = (float)std::sqrt(c33);
      eps[i] = (float)((c11 / c33 - 1.) / 2.);
      del[i] = (float)(((c13 / c33) * (c13 / c33) - 1.) / 2.);
    }
    std::vector<float> rec3(3 * (size_t)nrec);
    for (int ir = 0; ir < nrec; ++ir)
      for (int k = 0; k < 3; ++k) rec3[3 * ir + k] = recloc[4 * ir + k];
    std::vector<float> image(65 * n, 0.f);
    odcig3d_f(image.data(), souloc.data(), ns, rec3.data(), wavelet.data(), v.data(), eps.data(),
              del.data(), nx, ny, nz, nt, npad, ox, oy, oz, ot, dx, dy, dz, dt, rate);
    save(dir + "/ref_odcig.bin", image.data(), image.size());
#endif
  } else {
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
  }
  return 0;
}
