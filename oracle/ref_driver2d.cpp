// Harness that runs the REFERENCE's own 2D GPU path (compiled from its
// sources by oracle/build_ref.sh into oracle/_ref/ref2d) on inputs written by
// tests/golden/make_golden.py. TEST INFRASTRUCTURE ONLY.
//
// usage: ref2d <dir> synthetic|modeling|grad|gnhess|rtm|wgrad|odcig [nhx]
//   <dir>/params.txt : nx nz nt npad dx dz dt rate ot ns nr
//   <dir>/{c11,c13,c33,taper,wavelet}.bin (float32), sloc.bin / rloc.bin (int32)
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

// lib/vti-fwi-2d/wave.h:4,16 and lib/io/myio.cpp:15.
void myio_init(int argc, char** argv);
void synthetic_f(float* d, const float* c11, const float* c13, const float* c33,
                 const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                 const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot);
void modeling_f(float* d, const float* c11, const float* c13, const float* c33,
                const float* wavelet, int slocxz, const float* taper, int nx, int nz, int nt,
                int npad, float dx, float dz, float dt, float rate, float ot);
// wave.h:12 and wave.h:38
float objFuncGradient_f(float* gc11, float* gc13, float* gc33, const float* data,
                        const float* c11, const float* c13, const float* c33, const float* wavelet,
                        const int* sloc, int ns, const int* rloc, int nr, const float* taper,
                        int nx, int nz, int nt, int npad, float dx, float dz, float dt, float rate,
                        float ot);
void GNhessian_f(float* gc11, float* gc13, float* gc33, const float* data, const float* c11,
                 const float* c13, const float* c33, const float* dc11, const float* dc13,
                 const float* dc33, const float* wavelet, const int* sloc, int ns, const int* rloc,
                 int nr, const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot);

void rtm_f(float* image, const float* data, const float* c11, const float* c13, const float* c33,
           const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
           const float* taper, int nx, int nz, int nt, int npad, float dx, float dz, float dt,
           float rate, float ot);

void odcig_f(float* image, const float* data, const float* c11, const float* c13,
             const float* c33, const float* wavelet, const int* sloc, int ns, const int* rloc,
             int nr, const float* taper, int nx, int nz, int nhx, int nt, int npad, float dx,
             float dz, float dt, float rate, float ot);
void waveletGradient_f(float* gwavelet, const float* d0, const float* c11, const float* c13,
                       const float* c33, const int* sloc, int ns, const int* rloc, int nr,
                       const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                       float dt, float rate);

#ifdef VTI_SHIM
// Built against libvti_wave.so only: the Gauss-Newton operator classes of
// lib/vti-fwi-2d/HessianOp.h (declared with the same layout).
#include "vti_hessian_op.h"
#endif

template <typename T>
static std::vector<T> load(const std::string& path, size_t n) {
  std::vector<T> v(n);
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f || std::fread(v.data(), sizeof(T), n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", path.c_str());
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

static void save(const std::string& path, const float* p, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(p, sizeof(float), n, f) != n) std::exit(2);
  std::fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string dir = argv[1], mode = argv[2];
  std::ifstream pf(dir + "/params.txt");
  int nx, nz, nt, npad, ns, nr;
  float dx, dz, dt, rate, ot;
  if (!(pf >> nx >> nz >> nt >> npad >> dx >> dz >> dt >> rate >> ot >> ns >> nr)) return 2;
  const size_t nnx = nx + 2 * npad, nnz = nz + 2 * npad, nnxz = nnx * nnz;
  auto c11 = load<float>(dir + "/c11.bin", nnxz);
  auto c13 = load<float>(dir + "/c13.bin", nnxz);
  auto c33 = load<float>(dir + "/c33.bin", nnxz);
  auto taper = load<float>(dir + "/taper.bin", nnxz);
  auto wavelet = load<float>(dir + "/wavelet.bin", nt);
  auto sloc = load<int>(dir + "/sloc.bin", 4 * (size_t)ns);
  // the 2D drivers read the device list from argv (synthetic_f.cu:20-21)
  std::string a0 = "ref2d", a1 = "gpu=0";
  char* av[] = {&a0[0], &a1[0], nullptr};
  myio_init(2, av);
  if (mode == "synthetic") {
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    const int ratio = (int)(rate / dt + 0.5f);
    const int ntneg = (int)(ot < 0 ? (-ot / dt + 0.5f) : 0);
    const size_t rows = (nt - ntneg - 1) / ratio + 1;
    std::vector<float> data(rows * nr, 0.f);
    synthetic_f(data.data(), c11.data(), c13.data(), c33.data(), wavelet.data(), sloc.data(), ns,
                rloc.data(), nr, taper.data(), nx, nz, nt, npad, dx, dz, dt, rate, ot);
    save(dir + "/ref_data.bin", data.data(), data.size());
  } else if (mode == "modeling") {
    const int ratio = (int)(rate / dt + 0.5f);
    size_t rows = (nt - 1) / ratio + 1;
    if (rows < 2) rows = 2;
    std::vector<float> w(rows * nnxz, 0.f);
    int slocxz = sloc[0] + sloc[1] * (int)nnx;
    modeling_f(w.data(), c11.data(), c13.data(), c33.data(), wavelet.data(), slocxz, taper.data(),
               nx, nz, nt, npad, dx, dz, dt, rate, ot);
    save(dir + "/ref_wavefield.bin", w.data(), w.size());
  } else if (mode == "grad" || mode == "gnhess") {
    // <dir>/data.bin: observed traces (grad); <dir>/dc{11,13,33}.bin (gnhess)
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    const int ratio = (int)(rate / dt + 0.5f);
    const int ntneg = (int)(ot < 0 ? (-ot / dt + 0.5f) : 0);
    const size_t rows = (nt - ntneg - 1) / ratio + 1;
    std::vector<float> g(3 * nnxz + 1, 0.f);
    if (mode == "grad") {
      auto data = load<float>(dir + "/data.bin", rows * nr);
      g[3 * nnxz] = objFuncGradient_f(g.data(), g.data() + nnxz, g.data() + 2 * nnxz,
                                      data.data(), c11.data(), c13.data(), c33.data(),
                                      wavelet.data(), sloc.data(), ns, rloc.data(), nr,
                                      taper.data(), nx, nz, nt, npad, dx, dz, dt, rate, ot);
    } else {
      auto d11 = load<float>(dir + "/dc11.bin", nnxz);
      auto d13 = load<float>(dir + "/dc13.bin", nnxz);
      auto d33 = load<float>(dir + "/dc33.bin", nnxz);
      std::vector<float> unused(rows * nr, 0.f);
      GNhessian_f(g.data(), g.data() + nnxz, g.data() + 2 * nnxz, unused.data(), c11.data(),
                  c13.data(), c33.data(), d11.data(), d13.data(), d33.data(), wavelet.data(),
                  sloc.data(), ns, rloc.data(), nr, taper.data(), nx, nz, nt, npad, dx, dz, dt,
                  rate, ot);
    }
    save(dir + "/ref_" + mode + ".bin", g.data(), g.size());
#ifdef VTI_SHIM
  } else if (mode == "gnhessop") {
    // GNHessianOpCij (c110 = c130 = c330 = 1, no water-bottom rows beyond the
    // pad): forward without and adjoint with accumulation
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    std::vector<float> dc(3 * nnxz);
    const char* names[3] = {"/dc11.bin", "/dc13.bin", "/dc33.bin"};
    for (int k = 0; k < 3; ++k) {
      auto part = load<float>(dir + names[k], nnxz);
      std::copy(part.begin(), part.end(), dc.begin() + k * nnxz);
    }
    std::vector<float> mask(nnxz), out(6 * nnxz, 0.f), d0(1, 0.f);
    GNHessianOpCij op(d0.data(), c11.data(), c13.data(), c33.data(), 1.f, 1.f, 1.f,
                      wavelet.data(), sloc.data(), ns, rloc.data(), nr, taper.data(), nx, nz, nt,
                      npad, dx, dz, dt, rate, ot, 0.f, mask.data());
    op.forward(false, dc.data(), out.data());
    std::copy(out.begin(), out.begin() + 3 * nnxz, out.begin() + 3 * nnxz);
    op.adjoint(true, out.data() + 3 * nnxz, dc.data());
    save(dir + "/ref_gnhessop.bin", out.data(), out.size());
#endif
  } else if (mode == "rtm") {
    // <dir>/data.bin: the traces to migrate (receiver-fastest rows)
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    const int ratio = (int)(rate / dt + 0.5f);
    const int ntneg = (int)(ot < 0 ? (-ot / dt + 0.5f) : 0);
    const size_t rows = (nt - ntneg - 1) / ratio + 1;
    auto data = load<float>(dir + "/data.bin", rows * nr);
    std::vector<float> image(nnxz, 0.f);
    rtm_f(image.data(), data.data(), c11.data(), c13.data(), c33.data(), wavelet.data(),
          sloc.data(), ns, rloc.data(), nr, taper.data(), nx, nz, nt, npad, dx, dz, dt, rate, ot);
    save(dir + "/ref_rtm.bin", image.data(), image.size());
  } else if (mode == "odcig") {
    const int nhx = argc > 3 ? std::atoi(argv[3]) : 4;
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    const int ratio = (int)(rate / dt + 0.5f);
    const int ntneg = (int)(ot < 0 ? (-ot / dt + 0.5f) : 0);
    const size_t rows = (nt - ntneg - 1) / ratio + 1;
    auto data = load<float>(dir + "/data.bin", rows * nr);
    std::vector<float> image((2 * nhx + 1) * nnxz, 0.f);
    odcig_f(image.data(), data.data(), c11.data(), c13.data(), c33.data(), wavelet.data(),
            sloc.data(), ns, rloc.data(), nr, taper.data(), nx, nz, nhx, nt, npad, dx, dz, dt,
            rate, ot);
    save(dir + "/ref_odcig.bin", image.data(), image.size());
  } else if (mode == "wgrad") {
    // <dir>/data.bin: the traces driving the adjoint (nnt = (nt-1)/ratio+1 rows)
    auto rloc = load<int>(dir + "/rloc.bin", 2 * (size_t)nr);
    const int ratio = (int)(rate / dt + 0.5);
    const size_t rows = (nt - 1) / ratio + 1;
    auto data = load<float>(dir + "/data.bin", rows * nr);
    std::vector<float> gw(nt, 0.f);
    waveletGradient_f(gw.data(), data.data(), c11.data(), c13.data(), c33.data(), sloc.data(), ns,
                      rloc.data(), nr, taper.data(), nx, nz, nt, npad, dx, dz, dt, rate);
    save(dir + "/ref_wgrad.bin", gw.data(), gw.size());
  } else {
    return 2;
  }
  return 0;
}
