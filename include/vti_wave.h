// vti_wave.h — drop-in C++ entry points with the reference's signatures,
// implemented by libvti_wave.so on top of the C ABI (vti_b200.h).
//
// Callers of the reference (the lib/lbfgs FWI drivers, the 3D executables,
// the 2D drivers) link libvti_wave.so instead of the reference objects
// (objFuncGradient3d_f.o, modelData3d_f.o, kernel3d.o, injectRecord3d.o,
// abc3d.o, memcpy3d.o, synthetic_f.o, modeling_f.o, kernels.o). They keep
// linking their own myio.o: the shim reads the same argv side channels that
// myio_init() records (data=, gpu=, tpow=, objtype=, par=, datapath=).
//
// Each declaration names the reference declaration it replaces.
#ifndef VTI_WAVE_H
#define VTI_WAVE_H

#include <vector>

// ---- 3D (lib/vti-fwi-3d/gpu/wave3d.h)

// wave3d.h:84 — forward modeling of ns shots with the sponge; traces are
// appended to the SEP file named by data= (n1=nnt, n2=receivers) and the last
// sigma_x level is written to wavefield=. Devices from gpu=.
void modelData3d_f(float* souloc, int ns, float* recloc, float* wavelet, float* c11, float* c13,
                   float* c33, int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                   float oz, float ot, float dx, float dy, float dz, float dt, float samplingRate);

// wave3d.h:86 — one shot at (soulocX, soulocY, soulocZ), no receivers; the
// last sigma_x level goes to wavefield=.
void modeling3d_f(float soulocX, float soulocY, float soulocZ, float* wavelet, float* c11,
                  float* c13, float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
                  float oy, float oz, float ot, float dx, float dy, float dz, float dt);

// wave3d.h:94 — gradient over GPU groups (ngpugroup groups of GPUs).
void objFuncGradientCij3d(float* fgcij, float* souloc, int ns, std::vector<int>& shotid,
                          float* recloc, float* wavelet, float* cij, float* padboundaryCij,
                          float* randboundaryCij, int nx, int ny, int nz, int nt, int npad,
                          float ox, float oy, float oz, float ot, float dx, float dy, float dz,
                          float dt, float samplingRate, std::vector<int>& GPUs, int ngpugroup);

// wave3d.h:96 — gradient of the L2 misfit w.r.t. c11, c13, c33;
// fgcij = [misfit/2, gc11, gc13, gc33]; observed traces from data=.
// Like the reference, cij holds the random boundary in its pad on return.
void objFuncGradientCij3d_f(float* fgcij, float* souloc, int ns, std::vector<int>& shotid,
                            float* recloc, float* wavelet, float* cij, float* padboundaryCij,
                            float* randboundaryCij, int nx, int ny, int nz, int nt, int npad,
                            float ox, float oy, float oz, float ot, float dx, float dy, float dz,
                            float dt, float samplingRate, std::vector<int>& GPUs);

// wave3d.h:98 / :100 — misfit only (*f = misfit/2).
void objFuncCij3d(float* f, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                  float* wavelet, float* cij, float* padboundaryCij, int nx, int ny, int nz,
                  int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                  float dz, float dt, float samplingRate, std::vector<int>& GPUs, int ngpugroup);
void objFuncCij3d_f(float* f, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                    float* wavelet, float* cij, float* padboundaryCij, int nx, int ny, int nz,
                    int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                    float dz, float dt, float samplingRate, std::vector<int>& GPUs);

// wave3d.h:102 — gradient w.r.t. v, eps, del; returns misfit/2.
double objFuncGradientVEpsDel(float* gv, float* geps, float* gdel, float* souloc, int ns,
                              std::vector<int>& shotid, float* recloc, float* wavelet, float* v,
                              float* eps, float* del, float* padboundaryV, float* randboundaryV,
                              int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                              float oz, float ot, float dx, float dy, float dz, float dt,
                              float samplingRate, float v0, float eps0, float wbottom,
                              std::vector<int>& GPUs, int ngpugroup);

// wave3d.h:88 — reverse-time migration of the traces in data= with the model
// as given; recloc holds three floats (x, y, z) per receiver. Devices from gpu=.
void rtmCij3d_f(float* image, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                float* wavelet, float* c11, float* c13, float* c33, int nx, int ny, int nz,
                int nt, int npad, float ox, float oy, float oz, float ot, float dx, float dy,
                float dz, float dt, float samplingRate);

// wave3d.h:90 — the same from v, eps, del; pad region and water layer zeroed.
void rtmVEpsDel(float* image, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                float* wavelet, float* v, float* eps, float* del, float* randboundaryV, int nx,
                int ny, int nz, int nt, int npad, float ox, float oy, float oz, float ot,
                float dx, float dy, float dz, float dt, float samplingRate, float wbottom);

// wave3d.h:116 — offset-domain common-image gathers of all ns shots: the
// migration of rtmCij3d_f (traces from data=, three floats per receiver,
// devices from gpu=) from v, eps, del (c33 = v^2, c11 = c33 (1 + 2 eps),
// c13 = c33 sqrt(1 + 2 del)), with x-offset lags |lag| <= 32 (NLAG,
// wave3d.h:19); image holds 65 * nx*ny*nz floats, lag -32 first.
void odcig3d_f(float* image, float* souloc, int ns, float* recloc, float* wavelet, float* v,
               float* eps, float* del, int nx, int ny, int nz, int nt, int npad, float ox,
               float oy, float oz, float ot, float dx, float dy, float dz, float dt,
               float samplingRate);

// wave3d.h:112 / :114 — gradient of the misfit w.r.t. the source wavelet (nt
// floats), the adjoint driven by the traces in ddata (nnt*irbegin layout).
void waveletGradient3d_f(float* gwavelet, const float* ddata, float* souloc, int ns,
                         std::vector<int>& shotid, float* recloc, float* c11, float* c13,
                         float* c33, int nx, int ny, int nz, int nt, int npad, float ox, float oy,
                         float oz, float ot, float dx, float dy, float dz, float dt,
                         float samplingRate, std::vector<int>& GPUs, int ngpugroup);
void waveletGradientCij3d_f(float* gwavelet, const float* ddata, float* souloc, int ns,
                            std::vector<int>& shotid, float* recloc, float* c11, float* c13,
                            float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
                            float oy, float oz, float ot, float dx, float dy, float dz, float dt,
                            float samplingRate, std::vector<int>& GPUs);

// wave3d.h:108 / :110 — forward modeling into memory, ddata[nnt*irbegin ...].
void modelData3d_f(float* ddata, float* souloc, int ns, std::vector<int>& shotid, float* recloc,
                   const float* wavelet, float* c11, float* c13, float* c33, int nx, int ny,
                   int nz, int nt, int npad, float ox, float oy, float oz, float ot, float dx,
                   float dy, float dz, float dt, float samplingRate, std::vector<int>& GPUs,
                   int ngpugroup);
void modelDataCij3d_f(float* ddata, float* souloc, int ns, std::vector<int>& shotid,
                      float* recloc, const float* wavelet, float* c11, float* c13, float* c33,
                      int nx, int ny, int nz, int nt, int npad, float ox, float oy, float oz,
                      float ot, float dx, float dy, float dz, float dt, float samplingRate,
                      std::vector<int>& GPUs);

// ---- 2D (lib/vti-fwi-2d/wave.h)

// wave.h:4 — traces data[(it/ratio)*nr + ir] of ns shots; devices from gpu=.
void synthetic_f(float* d, const float* c11, const float* c13, const float* c33,
                 const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                 const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot = 0.);

// wave.h:16 — sigma_h snapshots of one shot.
void modeling_f(float* d, const float* c11, const float* c13, const float* c33,
                const float* wavelet, int slocxz, const float* taper, int nx, int nz, int nt,
                int npad, float dx, float dz, float dt, float rate, float ot = 0.);

// wave.h:12 — gradient of the L2 misfit w.r.t. c11, c13, c33; returns
// misfit/2. Devices from gpu=.
float objFuncGradient_f(float* gc11, float* gc13, float* gc33, const float* data,
                        const float* c11, const float* c13, const float* c33, const float* wavelet,
                        const int* sloc, int ns, const int* rloc, int nr, const float* taper,
                        int nx, int nz, int nt, int npad, float dx, float dz, float dt, float rate,
                        float ot = 0.);

// wave.h:10 (objFuncGradient.cu:28) — same w.r.t. v, eps, del; eps/del are
// projected so that del0*del <= eps0*eps (mask m), gradient zero down to the
// water bottom.
float objFuncGradientVEpsDel(float* gv, float* geps, float* gdel, const float* data, float* v,
                             float* eps, float* del, float v0, float eps0, float del0,
                             const float* wavelet, const int* sloc, int ns, const int* rloc,
                             int nr, const float* taper, int nx, int nz, int nt, int npad,
                             float dx, float dz, float dt, float rate, float ot, float wbottom,
                             float* m);

// wave.h:40 — Gauss-Newton Hessian times (dc11, dc13, dc33).
void GNhessian_f(float* gc11, float* gc13, float* gc33, const float* data, const float* c11,
                 const float* c13, const float* c33, const float* dc11, const float* dc13,
                 const float* dc33, const float* wavelet, const int* sloc, int ns, const int* rloc,
                 int nr, const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                 float dt, float rate, float ot);

// wave.h:38 (hessians.cu:28) — GN H*v w.r.t. c11, c13, c33 scaled by c110, c130,
// c330: the bound check of checkCij (check.cpp:6-20, c13 lowered to 0.99 of
// sqrt(c110 c11 c330 c33)/c130 where above it, mask m), scaled model and
// perturbation, GNhessian_f, water-bottom rows zeroed, result scaled back.
void GNhessianCij(float* gc11, float* gc13, float* gc33, const float* d0, float* c11, float* c13,
                  float* c33, const float* dc11, const float* dc13, const float* dc33, float c110,
                  float c130, float c330, const float* wavelet, const int* sloc, int ns,
                  const int* rloc, int nr, const float* taper, int nx, int nz, int nt, int npad,
                  float dx, float dz, float dt, float rate, float ot, float wbottom, float* m);

// wave.h:46 (hessians.cu:72) — same w.r.t. v, eps, del.
void GNhessianVEpsDel(float* gv, float* geps, float* gdel, const float* d0, float* v, float* eps,
                      float* del, const float* dv, const float* deps, const float* ddel, float v0,
                      float eps0, float del0, const float* wavelet, const int* sloc, int ns,
                      const int* rloc, int nr, const float* taper, int nx, int nz, int nt,
                      int npad, float dx, float dz, float dt, float rate, float ot, float wbottom,
                      float* m);

// wave.h:6 — reverse-time migration of data[(it/ratio)*nr + ir].
void rtm_f(float* image, const float* data, const float* c11, const float* c13, const float* c33,
           const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
           const float* taper, int nx, int nz, int nt, int npad, float dx, float dz, float dt,
           float rate, float ot = 0.);

// wave.h:16 — offset-domain common-image gathers, (2nhx+1) * nnxz floats.
void odcig_f(float* image, const float* data, const float* c11, const float* c13,
             const float* c33, const float* wavelet, const int* sloc, int ns, const int* rloc,
             int nr, const float* taper, int nx, int nz, int nhx, int nt, int npad, float dx,
             float dz, float dt, float rate, float ot = 0.);

// wave.h:18 — gradient w.r.t. the source wavelet (nt floats).
void waveletGradient_f(float* gwavelet, const float* d0, const float* c11, const float* c13,
                       const float* c33, const int* sloc, int ns, const int* rloc, int nr,
                       const float* taper, int nx, int nz, int nt, int npad, float dx, float dz,
                       float dt, float rate);

#endif  // VTI_WAVE_H
