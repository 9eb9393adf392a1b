// CPU ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A plain C++/OpenMP restatement of the reference's VTI pseudo-acoustic
// modeling / gradient path (huyleq/thesis-source-code, lib/vti-fwi-3d/gpu and
// lib/vti-fwi-2d). It is the checker for the CUDA path and, in its FP32
// instance, the timed CPU baseline. Nothing in the product library links,
// loads or calls this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it (through ctypes).
//
// Every function is templated on the arithmetic type T:
//   T = double : the FP64 error oracle
//   T = float  : the FP32 CPU baseline
// Model arrays, damping tables and the scale factors dt^2/dx^2 are float
// values in the reference, so they enter here as float and are promoted to T.
//
// Semantics restated (all file:line refer to the reference tree):
//  * 3D step: lib/vti-fwi-3d/gpu/kernel3d.cu:3-74 (forward form, scale folded
//    as dt2/dx2) and kernel3d.cu:222-298 (gradient form, dt2*(c*L/dx2)).
//    x/y updates cover [4,n-4) (kernel3d.cu:7-10); z covers [0,nz) with zero
//    planes outside (TopBlock/BottomBlock, kernel3d.cu:92,409).
//  * Sponge: abc3d.cu:23-50 (profile), abc3d.cu:82-126 (applied per 4-plane
//    z-block to next AND cur after each block's update,
//    objFuncGradient3d_f.cu:661-662). Because blocks are processed in z
//    order, the z-stencil of block b reads already-damped cur planes of block
//    b-1 and undamped planes of blocks >= b. Stored values here are "once
//    damped" (v_t); prev is read as d*v_{t-2} and the planes of the block
//    above as d*v_{t-1}, which reproduces the reference bit-for-bit in the
//    sequence of multiplications while writing each array once.
//  * Time loop / source / recording: objFuncGradient3d_f.cu:605-706,
//    modelData3d_f.cu:174-302 (source dt2*w[it-1] into next before the
//    sponge; record 2/3 sx + 1/3 sz at it == s*j, j>=1, trace-major
//    data[j + ir*nnt]); number of updates 64*floor((nt-2)/64)
//    (objFuncGradient3d_f.cu:538-542, NUPDATE=64 wave3d.h:17).
//  * Gradient: objFuncGradient3d_f.cu:361-1111 (pass 1 pad boundary + sponge
//    + record; L2 misfit :759-771; pass 2 random boundary, no sponge;
//    pass 3 time-reversed sigma (gradientKernel) + adjoint lambda with the
//    FORWARD operator and the sponge + zero-lag imaging; residual injected
//    2/3,1/3 * dt2 * linearly interpolated residual, injectRecord3d.cu:38-78).
//  * 2D forward: lib/vti-fwi-2d/kernels.cu:452-498 (forwardCD),
//    synthetic_f.cu:81-119, modeling_f.cu:43-82, taper kernels.cu:293-315.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <map>
#include <omp.h>

namespace {

// 8th-order second-derivative coefficients as the 3D reference writes them
// (lib/vti-fwi-3d/gpu/wave3d.h:8-12, double literals).
const double k3C0 = -2.84722222222, k3C1 = 1.6, k3C2 = -0.2, k3C3 = 0.02539682539,
             k3C4 = -0.00178571428;
// The 2D reference writes the same values as float literals
// (lib/vti-fwi-2d/kernels.h:4-8).
const float k2C0 = -2.84722222222f, k2C1 = 1.6f, k2C2 = -0.2f, k2C3 = 0.02539682539f,
            k2C4 = -0.00178571428f;
const double kTwoThird = 0.6666666666, kOneThird = 0.3333333333;  // wave3d.h:5-6
const double kDamper = 0.95, kPi = 3.14159265359;                 // wave3d.h:4,14
const int kNUpdate = 64;                                           // wave3d.h:17
const int kHalf = 4;                                               // wave3d.h:19

struct Geo3 {
  int nx, ny, nz, nt, npad, ref_steps, ref_gpus;
  float ox, oy, oz, ot, dx, dy, dz, dt, rate;
  long nxy() const { return (long)nx * ny; }
  long nxyz() const { return (long)nx * ny * nz; }
};

Geo3 unpack3(const int* ip, const float* fp) {
  Geo3 g;
  g.nx = ip[0]; g.ny = ip[1]; g.nz = ip[2]; g.nt = ip[3]; g.npad = ip[4]; g.ref_steps = ip[5];
  g.ref_gpus = ip[6] < 1 ? 1 : ip[6];
  g.ox = fp[0]; g.oy = fp[1]; g.oz = fp[2]; g.ot = fp[3];
  g.dx = fp[4]; g.dy = fp[5]; g.dz = fp[6]; g.dt = fp[7]; g.rate = fp[8];
  return g;
}

// Last time level computed by the reference pipeline on ref_gpus GPUs
// (objFuncGradient3d_f.cu:538-542: it runs 2..1+NGPU*64*nround).
int last_level(const Geo3& g) {
  if (g.ref_steps) return 1 + kNUpdate * g.ref_gpus * ((g.nt - 2) / (kNUpdate * g.ref_gpus));
  return g.nt - 1;
}

int sampling_step(float rate, float dt) { return (int)std::round(rate / dt); }

// Trace samples the reference actually records: its host loop
// (modelData3d_f.cu:179-296) records level it of the receiver block into
// sample itdata only if it == s*itdata at the tick that block is updated,
// and advances itdata two ticks later (:263-275). Replayed tick by tick.
std::vector<int> record_schedule(const Geo3& g, int rec_block, int st, int nnt) {
  std::vector<int> at(std::max(g.nt, 2), -1);
  if (!g.ref_steps) {
    for (int it = 2; it <= last_level(g); ++it)
      if (it % st == 0 && it / st >= 1 && it / st < nnt) at[it] = it / st;
    return at;
  }
  const int NG = g.ref_gpus, nb = g.nz / kHalf;
  const int pipelen = NG * (kNUpdate + 3) + 3;
  const int nround = (g.nt - 2) / (NG * kNUpdate);
  const int roundlen = std::max(pipelen, nb);
  const int nroundlen = nround * roundlen;
  const int nk = (nround - 1) * roundlen + pipelen + nb - 1;
  int itdata = 1, krecord = -2, ktransf = -2, rec_it = -1;
  for (int k = 0; k < nk; k++) {
    for (int gpu = 0; gpu < NG; gpu++) {
      int kgpu = k - gpu * (kNUpdate + 3);
      if (!(kgpu > 2 && kgpu <= kNUpdate + 1 + nroundlen)) continue;
      for (int i = 0; i < kNUpdate; i++) {
        int ib = (kgpu - 3 - i) % roundlen, iround = (kgpu - 3 - i) / roundlen;
        if (ib >= 0 && ib < nb && iround >= 0 && iround < nround) {
          int it = iround * NG * kNUpdate + gpu * kNUpdate + 2 + i;
          if (ib == rec_block && it == st * itdata && itdata < nnt) {
            krecord = k;
            rec_it = it;
          }
        }
      }
    }
    if (k - 1 == krecord && itdata < nnt) { krecord = -2; ktransf = k; }
    if (k - 1 == ktransf && itdata < nnt) {
      at[rec_it] = itdata;
      itdata++;
      ktransf = -2;
    }
  }
  return at;
}

// abc3d.cu:23-50: one-dimensional sponge profile in float.
float damp_profile(int i, int n, int npad) {
  float dist;
  if (i < npad) dist = npad - i;
  else if (i > n - npad) dist = i - n + npad;
  else dist = 0.f;
  return (float)(kDamper + (1. - kDamper) * std::cos(kPi * dist / npad));
}

struct Damp3 {
  std::vector<float> xy, z;
  Damp3(const Geo3& g) : xy(g.nxy()), z(g.nz) {
    for (int iy = 0; iy < g.ny; ++iy) {
      float dy = damp_profile(iy, g.ny, g.npad);
      for (int ix = 0; ix < g.nx; ++ix) xy[ix + (long)iy * g.nx] = damp_profile(ix, g.nx, g.npad) * dy;
    }
    for (int iz = 0; iz < g.nz; ++iz) z[iz] = damp_profile(iz, g.nz, g.npad);
  }
  // abc3d.cu:93 (the abcXY variant multiplies by xy only, identical since
  // the z profile is exactly 1.0f outside the pad).
  float at(long ixy, int iz) const { return xy[ixy] * z[iz]; }
};

// One update of a (sigma_x, sigma_z) pair over the reference's update region.
//   cur  : v_{t-1}            prev_next : in v_{t-2}, out v_t
// kForwardForm: kernel3d.cu:54-69 (scale dt2/dx2 folded into the Laplacian)
// otherwise    : kernel3d.cu:273-288 (dt2 * (c * L/dx2)).
// damp != nullptr selects the sponge with the block-order reading rule.
// Optional imaging (kernel3d.cu:291-293) uses lam_x/lam_z at time t-1.
template <typename T, bool kForwardForm>
void step3d(const Geo3& g, const float* c11, const float* c13, const float* c33,
            const T* __restrict cx, const T* __restrict cz, T* __restrict px, T* __restrict pz,
            const Damp3* damp, const T* __restrict lamx, const T* __restrict lamz,
            T* __restrict g11, T* __restrict g13, T* __restrict g33) {
  const long nx = g.nx, ny = g.ny, nz = g.nz, nxy = g.nxy();
  const float dx2 = g.dx * g.dx, dy2 = g.dy * g.dy, dz2 = g.dz * g.dz, dt2 = g.dt * g.dt;
  const float sx = dt2 / dx2, sy = dt2 / dy2, sz = dt2 / dz2;
  const T C[5] = {(T)k3C0, (T)k3C1, (T)k3C2, (T)k3C3, (T)k3C4};
  // Rows used in place of planes outside [0, nz) (zeros) and of the damping
  // factors of undamped planes (ones): multiplying by (T)(1.0f * 1.0f) keeps
  // the value exact, so every point evaluates the same expressions as the
  // plain per-point form while the x loop stays free of branches.
  const std::vector<T> zeros(nx, (T)0);
  const std::vector<float> ones(nx, 1.f);
#pragma omp parallel for collapse(2) schedule(static)
  for (long iz = 0; iz < nz; ++iz) {
    for (long iy = kHalf; iy < ny - kHalf; ++iy) {
      const long blk = iz / kHalf;
      const long row = iy * nx;
      const T* zr[9];
      const float* dr[9];
      float zf[9];
      for (int k = -4; k <= 4; ++k) {
        const long z2 = iz + k;
        const bool in = z2 >= 0 && z2 < nz;
        // the block-order rule: planes of the blocks above were damped as cur
        const bool dm = in && damp && z2 / kHalf < blk;
        zr[k + 4] = in ? cz + row + z2 * nxy : zeros.data();
        dr[k + 4] = dm ? damp->xy.data() + row : ones.data();
        zf[k + 4] = dm ? damp->z[z2] : 1.f;
      }
      const float* dc = damp ? damp->xy.data() + row : ones.data();
      const float zc = damp ? damp->z[iz] : 1.f;
      const long base = row + iz * nxy;
#pragma omp simd
      for (long ix = kHalf; ix < nx - kHalf; ++ix) {
        const long i = base + ix;
        T lxx = C[0] * cx[i], lyy = C[0] * cx[i];
        for (int k = 1; k <= 4; ++k) {
          lxx += C[k] * (cx[i - k] + cx[i + k]);
          lyy += C[k] * (cx[i - k * nx] + cx[i + k * nx]);
        }
        T zv[9];
        for (int k = 0; k < 9; ++k) zv[k] = zr[k][ix] * (T)(dr[k][ix] * zf[k]);
        T lzz = C[0] * zv[4];
        for (int k = 1; k <= 4; ++k) lzz += C[k] * (zv[4 - k] + zv[4 + k]);
        const T d = (T)(dc[ix] * zc);
        T nxv, nzv, lxy_u = 0, lz_u = 0;
        if (kForwardForm) {
          const T lxy = lxx * (T)sx + lyy * (T)sy, lz = lzz * (T)sz;
          nxv = (T)c11[i] * lxy + (T)c13[i] * lz + 2 * cx[i] - d * px[i];
          nzv = (T)c13[i] * lxy + (T)c33[i] * lz + 2 * cz[i] - d * pz[i];
        } else {
          lxy_u = lxx / (T)dx2 + lyy / (T)dy2;
          lz_u = lzz / (T)dz2;
          nxv = (T)dt2 * ((T)c11[i] * lxy_u + (T)c13[i] * lz_u) + 2 * cx[i] - d * px[i];
          nzv = (T)dt2 * ((T)c13[i] * lxy_u + (T)c33[i] * lz_u) + 2 * cz[i] - d * pz[i];
        }
        px[i] = d * nxv;
        pz[i] = d * nzv;
        if (g11) {
          g11[i] += lamx[i] * lxy_u;
          g33[i] += lamz[i] * lz_u;
          g13[i] += lamx[i] * lz_u + lamz[i] * lxy_u;
        }
      }
    }
  }
}

struct Shot3 {
  long sidx;                 // source flat index
  std::vector<long> ridx;    // receiver read / residual-injection points
  std::vector<long> seed;    // adjoint seeding points
  std::vector<char> inner;   // receiver inside the x/y update region
  std::vector<char> live;    // receiver flag != 0
  std::vector<int> rec_at;   // level -> recorded sample (-1: none)
  int irbegin, nr;
};

// objFuncGradient3d_f.cu:545-575: float arithmetic, truncation toward zero.
// Traces are read and residuals injected in the 4-plane block of the first
// receiver of the survey (recBlock, recIndexBlock); the adjoint is seeded at
// each receiver's own depth (recIndex, :922-927). Cells of the 4-wide x/y
// frame are never updated by the scheme; no residual is injected there.
Shot3 make_shot3(const Geo3& g, const float* souloc, const float* recloc, int is) {
  Shot3 s;
  s.nr = (int)souloc[5 * is + 3];
  s.irbegin = (int)souloc[5 * is + 4];
  int sx = (int)((souloc[5 * is] - g.ox) / g.dx);
  int sy = (int)((souloc[5 * is + 1] - g.oy) / g.dy);
  int sz = (int)((souloc[5 * is + 2] - g.oz) / g.dz);
  s.sidx = sx + (long)sy * g.nx + (long)sz * g.nxy();
  const int rec_block = (int)((recloc[2] - g.oz) / g.dz / kHalf);
  s.ridx.resize(s.nr);
  s.seed.resize(s.nr);
  s.inner.resize(s.nr);
  s.live.resize(s.nr);
  for (int ir = 0; ir < s.nr; ++ir) {
    int r = ir + s.irbegin;
    int ix = (int)((recloc[4 * r] - g.ox) / g.dx);
    int iy = (int)((recloc[4 * r + 1] - g.oy) / g.dy);
    int iz = (int)((recloc[4 * r + 2] - g.oz) / g.dz);
    int izr = g.ref_steps ? rec_block * kHalf + iz % kHalf : iz;
    s.ridx[ir] = ix + (long)iy * g.nx + (long)izr * g.nxy();
    s.seed[ir] = ix + (long)iy * g.nx + (long)iz * g.nxy();
    s.inner[ir] = ix >= kHalf && ix < g.nx - kHalf && iy >= kHalf && iy < g.ny - kHalf;
    s.live[ir] = recloc[4 * r + 3] != 0.f;
  }
  const int st = sampling_step(g.rate, g.dt);
  s.rec_at = record_schedule(g, rec_block, st, (g.nt - 1) / st + 1);
  return s;
}

// Forward propagation from the source. With damp: pass 1 of the gradient /
// modelDataCij3d_f (records traces). Without: pass 2 (random boundary).
// On return (cx,cz) = v_M and (px,pz) = v_{M-1}.
template <typename T>
void forward3d(const Geo3& g, const float* c11, const float* c13, const float* c33,
               const float* wavelet, const Shot3& s, const Damp3* damp, T* trace /*nnt*nr or null*/,
               std::vector<T>& cx, std::vector<T>& cz, std::vector<T>& px, std::vector<T>& pz) {
  const long n = g.nxyz();
  const float dt2 = g.dt * g.dt;
  const int st = sampling_step(g.rate, g.dt);
  const int nnt = (g.nt - 1) / st + 1;
  const int M = last_level(g);
  cx.assign(n, 0); cz.assign(n, 0); px.assign(n, 0); pz.assign(n, 0);
  // "injecting source at time 0 to wavefields at time 1"
  // (objFuncGradient3d_f.cu:605-608): assignment, no sponge.
  const float s0 = dt2 * wavelet[0];
  cx[s.sidx] = s0;
  cz[s.sidx] = s0;
  if (trace) std::fill(trace, trace + (long)nnt * s.nr, (T)0);
  for (int it = 2; it <= M; ++it) {
    step3d<T, true>(g, c11, c13, c33, cx.data(), cz.data(), px.data(), pz.data(), damp, nullptr,
                    nullptr, nullptr, nullptr, nullptr);
    // source before the sponge (objFuncGradient3d_f.cu:655-662): d*(raw+src)
    const float src = dt2 * wavelet[it - 1];
    const T d = damp ? (T)damp->at(s.sidx % g.nxy(), (int)(s.sidx / g.nxy())) : (T)1;
    px[s.sidx] += d * (T)src;
    pz[s.sidx] += d * (T)src;
    std::swap(cx, px);
    std::swap(cz, pz);
    // recordData (injectRecord3d.cu:22-28) into the sample the reference's
    // bookkeeping assigns to this level
    if (trace && s.rec_at[it] >= 0) {
      const int j = s.rec_at[it];
      for (int ir = 0; ir < s.nr; ++ir)
        trace[j + (long)ir * nnt] = (T)kTwoThird * cx[s.ridx[ir]] + (T)kOneThird * cz[s.ridx[ir]];
    }
  }
  if (trace)
    for (int ir = 0; ir < s.nr; ++ir)
      if (!s.live[ir]) std::fill(trace + (long)ir * nnt, trace + (long)(ir + 1) * nnt, (T)0);
}

// boundary.cpp:48-84 putBoundary: scatter the pad-region list into a full array.
void put_boundary(const float* b, float* v, int nx, int ny, int nz, int npad) {
  size_t cb = 0, cv = 0, n = (size_t)nx * ny * npad;
  std::memcpy(v + cv, b + cb, n * 4); cb += n; cv += n;
  for (int iz = 0; iz < nz - 2 * npad; iz++) {
    for (int iy = 0; iy < npad; iy++) { std::memcpy(v + cv, b + cb, nx * 4); cb += nx; cv += nx; }
    for (int iy = 0; iy < ny - 2 * npad; iy++) {
      std::memcpy(v + cv, b + cb, npad * 4); cb += npad; cv += nx - npad;
      std::memcpy(v + cv, b + cb, npad * 4); cb += npad; cv += npad;
    }
    for (int iy = 0; iy < npad; iy++) { std::memcpy(v + cv, b + cb, nx * 4); cb += nx; cv += nx; }
  }
  n = (size_t)nx * ny * npad;
  std::memcpy(v + cv, b + cb, n * 4);
}

template <typename T>
T interp_residual(const T* res_trace, int time_index, int nnt, int st) {
  // injectRecord3d.cu:60-78 (float f, double weights)
  float f = float(time_index) / float(st);
  int i = (int)f;
  if (i >= nnt - 1) return res_trace[nnt - 1];
  f = f - i;
  return (T)((1. - f) * res_trace[i] + f * res_trace[i + 1]);
}

// runsum (agc.cpp:14-25): windowed sum over i-hw..i+hw, indices wrapping.
template <typename T>
void runsum(int nt, int hw, const T* w, T* s) {
  for (int i = 0; i < nt; ++i) {
    T v = 0;
    for (int j = i - hw; j <= i + hw; ++j) v += w[j < 0 ? j + nt : (j >= nt ? j - nt : j)];
    s[i] = v;
  }
}

// residualAGC (agc.cpp:62-99) for one trace: d (modeled) becomes the adjoint
// source; returns the trace's squared AGC residual.
template <typename T>
double agc_adjoint(int nt, int hw, T* d, const float* d0) {
  const T eps = (T)1e-6f;
  std::vector<T> e(nt), e0(nt), sd(nt), sd0(nt), rs(nt), drss(nt), acc(nt);
  for (int i = 0; i < nt; ++i) {
    e[i] = d[i] * d[i];
    e0[i] = (T)d0[i] * (T)d0[i];
  }
  runsum(nt, hw, e.data(), sd.data());
  runsum(nt, hw, e0.data(), sd0.data());
  double fi = 0;
  for (int i = 0; i < nt; ++i) {
    T res = d[i] / std::sqrt(std::max(eps, sd[i])) - (T)d0[i] / std::sqrt(std::max(eps, sd0[i]));
    fi += (double)(res * res);
    T t1 = std::max(eps, sd[i]);
    T t2 = res / std::sqrt(t1);
    drss[i] = d[i] * t2 / t1;
    rs[i] = t2;
  }
  runsum(nt, hw, drss.data(), acc.data());
  for (int i = 0; i < nt; ++i) d[i] = rs[i] - d[i] * acc[i];
  return fi;
}

// objFuncGradientCij3d_f (objFuncGradient3d_f.cu:361-1111) for the shots in
// shotid. fgcij[0] = misfit/2, then gc11, gc13, gc33 (nxyz each).
// misfit_only: objFuncCij3d_f (pass 1 + misfit).
template <typename T>
void gradient3d(const Geo3& g, const float* cij_in, const float* padb, const float* randb,
                const float* wavelet, const float* souloc, const int* shotid, int nshot,
                const float* recloc, const float* dobs, T* fgcij, bool misfit_only,
                T* modeled /*optional: nnt*nrtotal modeled traces*/, float tpow = 0.f,
                int objtype = 0, int halfwidth = 20) {
  const long n = g.nxyz(), nxy = g.nxy();
  const float dt2 = g.dt * g.dt;
  const int st = sampling_step(g.rate, g.dt);
  const int nnt = (g.nt - 1) / st + 1;
  const int M = last_level(g);
  std::vector<float> cij(cij_in, cij_in + 3 * n);
  float *c11 = cij.data(), *c13 = c11 + n, *c33 = c13 + n;
  const long nb = n - (long)(g.nx - 2 * g.npad) * (g.ny - 2 * g.npad) * (g.nz - 2 * g.npad);
  if (!misfit_only) std::fill(fgcij, fgcij + 1 + 3 * n, (T)0);
  T *g11 = fgcij + 1, *g13 = g11 + n, *g33 = g13 + n;
  Damp3 damp(g);
  double objfunc = 0;
  std::vector<T> cx, cz, px, pz, lcx, lcz, lpx, lpz;
  for (int k = 0; k < nshot; ++k) {
    const int is = shotid[k];
    Shot3 s = make_shot3(g, souloc, recloc, is);
    // pass 1: pad boundary + sponge + record (objFuncGradient3d_f.cu:594-727)
    put_boundary(padb, c11, g.nx, g.ny, g.nz, g.npad);
    put_boundary(padb + nb, c13, g.nx, g.ny, g.nz, g.npad);
    put_boundary(padb + 2 * nb, c33, g.nx, g.ny, g.nz, g.npad);
    std::vector<T> res((long)nnt * s.nr);
    forward3d<T>(g, c11, c13, c33, wavelet, s, &damp, res.data(), cx, cz, px, pz);
    if (modeled)
      std::copy(res.begin(), res.end(), modeled + (long)nnt * s.irbegin);
    // L2 misfit (objFuncGradient3d_f.cu:759-771): residual = modeled - observed;
    // the gradient (not the misfit-only entry, :1579-1590) first applies the
    // t^p gain (tpower, agc.cpp:104-116) and may use the AGC misfit instead
    const float* ob = dobs + (long)nnt * s.irbegin;
    if (!misfit_only && tpow != 0.f)
      for (int ir = 0; ir < s.nr; ++ir)
        for (int it = 0; it < nnt; ++it) {
          float t = g.ot + it * g.rate;
          res[it + (long)ir * nnt] *= (T)std::pow((double)t, (double)tpow);
        }
    if (!misfit_only && objtype != 0) {
      for (int ir = 0; ir < s.nr; ++ir)
        objfunc += agc_adjoint<T>(nnt, halfwidth, res.data() + (long)ir * nnt,
                                  ob + (long)ir * nnt);
    } else {
      for (long i = 0; i < (long)nnt * s.nr; ++i) {
        res[i] = res[i] - (T)ob[i];
        objfunc += (double)(res[i] * res[i]);
      }
    }
    if (misfit_only) continue;
    // pass 2: random boundary, no sponge (objFuncGradient3d_f.cu:786-895)
    put_boundary(randb, c11, g.nx, g.ny, g.nz, g.npad);
    put_boundary(randb + nb, c13, g.nx, g.ny, g.nz, g.npad);
    put_boundary(randb + 2 * nb, c33, g.nx, g.ny, g.nz, g.npad);
    forward3d<T>(g, c11, c13, c33, wavelet, s, nullptr, nullptr, cx, cz, px, pz);
    // flip (objFuncGradient3d_f.cu:912-914): cur = v_{M-1}, prev = v_M
    std::swap(cx, px);
    std::swap(cz, pz);
    lcx.assign(n, 0); lcz.assign(n, 0); lpx.assign(n, 0); lpz.assign(n, 0);
    // objFuncGradient3d_f.cu:922-927: adjoint seeded by assignment
    for (int ir = 0; ir < s.nr; ++ir) {
      if (!s.inner[ir]) continue;
      T temp = (T)dt2 * res[(nnt - 1) + (long)ir * nnt];
      lcx[s.seed[ir]] = (T)kTwoThird * temp;
      lcz[s.seed[ir]] = (T)kOneThird * temp;
    }
    const long sxy = s.sidx % nxy;
    const int sz = (int)(s.sidx / nxy);
    (void)sz;
    std::vector<T> rfine(s.nr);
    for (int i = 0; i < M - 1; ++i) {
      const int it = g.nt - 3 - i;  // objFuncGradient3d_f.cu:996-997
      // sigma back one step + imaging with the current adjoint
      step3d<T, false>(g, c11, c13, c33, cx.data(), cz.data(), px.data(), pz.data(), nullptr,
                       lcx.data(), lcz.data(), g11, g13, g33);
      // adjoint with the forward operator and the sponge
      step3d<T, true>(g, c11, c13, c33, lcx.data(), lcz.data(), lpx.data(), lpz.data(), &damp,
                      nullptr, nullptr, nullptr, nullptr, nullptr);
      const float src = dt2 * wavelet[it + 1];  // objFuncGradient3d_f.cu:1014
      px[s.sidx] += (T)src;
      pz[s.sidx] += (T)src;
      // residual injection before the sponge (injectRecord3d.cu:38-46)
      for (int ir = 0; ir < s.nr; ++ir) {
        if (!s.inner[ir]) continue;
        T r = interp_residual<T>(res.data() + (long)ir * nnt, it + 1, nnt, st);
        T inj = (T)dt2 * r;
        long ri = s.ridx[ir];
        T d = (T)damp.at(ri % nxy, (int)(ri / nxy));
        lpx[ri] += d * ((T)kTwoThird * inj);
        lpz[ri] += d * ((T)kOneThird * inj);
      }
      (void)sxy;
      std::swap(cx, px); std::swap(cz, pz);
      std::swap(lcx, lpx); std::swap(lcz, lpz);
    }
  }
  fgcij[0] = (T)(objfunc / 2);
}

// rtmCij3d_f (lib/vti-fwi-3d/gpu/rtm3d_f.cu:161-620) for the shots in shotid:
// pass 1 propagates the source wavefield with the model as given and no
// sponge (:378-468); after the flip (:495-497) the source wavefield steps back
// (forward form, source re-injected with w[it+1], :585-600) while the
// receiver wavefield is seeded with the last data sample (:509-514), stepped
// with the forward operator, fed the data interpolated at it+1 and damped by
// the sponge (:586-608); imagingKernel (kernel3d.cu:456-469) then adds
// (2/3 sx + 1/3 sz)(2/3 lx + 1/3 lz) with both fields at the step's current
// level, the receiver wavefield already damped by this step's sponge.
// image is zeroed first and accumulates over shots (rtm3d_f.cu:175).
// nlag >= 0: offset-domain gathers with the extended imaging condition of
// extendedImagingKernel (lib/vti-fwi-3d/gpu/wave3d.cu:1299-1313): for
// |lag| <= nlag, image[j + (lag+nlag)*n] += S[j] * R[j+lag] (x offsets) with
// S = 2/3 sx + 1/3 sz and R the damped receiver term of the zero-lag image,
// for x in [max(4,nlag), min(nx-4, nx-nlag)), y in [4, ny-4), all z. The 3D
// reference driver (odcig3d_f.cu) does not link (its forwardKernel calls do
// not match the declared kernel), so this restatement follows the kernel.
template <typename T>
void rtm3d(const Geo3& g, const float* c11, const float* c13, const float* c33,
           const float* wavelet, const float* souloc, const int* shotid, int nshot,
           const float* recloc, const float* data, T* image, int nlag = -1) {
  const long n = g.nxyz(), nxy = g.nxy();
  const long nimg = nlag >= 0 ? (2L * nlag + 1) * n : n;
  const float dt2 = g.dt * g.dt;
  const int st = sampling_step(g.rate, g.dt);
  const int nnt = (g.nt - 1) / st + 1;
  const int M = last_level(g);
  std::fill(image, image + nimg, (T)0);
  Damp3 damp(g);
  const long xlo = std::max<long>(kHalf, nlag), xhi = std::min<long>(g.nx - kHalf, g.nx - nlag);
  std::vector<T> cx, cz, px, pz, lcx, lcz, lpx, lpz;
  for (int k = 0; k < nshot; ++k) {
    Shot3 s = make_shot3(g, souloc, recloc, shotid[k]);
    const float* dat = data + (long)nnt * s.irbegin;
    forward3d<T>(g, c11, c13, c33, wavelet, s, nullptr, nullptr, cx, cz, px, pz);
    std::swap(cx, px);
    std::swap(cz, pz);
    lcx.assign(n, 0); lcz.assign(n, 0); lpx.assign(n, 0); lpz.assign(n, 0);
    for (int ir = 0; ir < s.nr; ++ir) {
      if (!s.inner[ir]) continue;
      T temp = (T)dt2 * (T)dat[(nnt - 1) + (long)ir * nnt];
      lcx[s.seed[ir]] = (T)kTwoThird * temp;
      lcz[s.seed[ir]] = (T)kOneThird * temp;
    }
    for (int i = 0; i < M - 1; ++i) {
      const int it = g.nt - 3 - i;
      step3d<T, true>(g, c11, c13, c33, cx.data(), cz.data(), px.data(), pz.data(), nullptr,
                      nullptr, nullptr, nullptr, nullptr, nullptr);
      const float src = dt2 * wavelet[it + 1];
      px[s.sidx] += (T)src;
      pz[s.sidx] += (T)src;
      step3d<T, true>(g, c11, c13, c33, lcx.data(), lcz.data(), lpx.data(), lpz.data(), &damp,
                      nullptr, nullptr, nullptr, nullptr, nullptr);
      for (int ir = 0; ir < s.nr; ++ir) {
        if (!s.inner[ir]) continue;
        std::vector<T> tr(dat + (long)ir * nnt, dat + (long)(ir + 1) * nnt);
        T inj = (T)dt2 * interp_residual<T>(tr.data(), it + 1, nnt, st);
        long ri = s.ridx[ir];
        T d = (T)damp.at(ri % nxy, (int)(ri / nxy));
        lpx[ri] += d * ((T)kTwoThird * inj);
        lpz[ri] += d * ((T)kOneThird * inj);
      }
      if (nlag < 0) {
#pragma omp parallel for collapse(2) schedule(static)
        for (long iz = 0; iz < g.nz; ++iz)
          for (long iy = kHalf; iy < g.ny - kHalf; ++iy)
            for (long ix = kHalf; ix < g.nx - kHalf; ++ix) {
              const long ixy = ix + iy * g.nx, j = ixy + iz * nxy;
              const T d = (T)damp.at(ixy, (int)iz);
              image[j] += ((T)kTwoThird * cx[j] + (T)kOneThird * cz[j]) *
                          (d * ((T)kTwoThird * lcx[j] + (T)kOneThird * lcz[j]));
            }
      } else {
#pragma omp parallel for collapse(2) schedule(static)
        for (long iz = 0; iz < g.nz; ++iz)
          for (long iy = kHalf; iy < g.ny - kHalf; ++iy)
            for (long ix = xlo; ix < xhi; ++ix) {
              const long ixy = ix + iy * g.nx, j = ixy + iz * nxy;
              const T sv = (T)kTwoThird * cx[j] + (T)kOneThird * cz[j];
              for (int lag = -nlag; lag <= nlag; ++lag) {
                const T d = (T)damp.at(ixy + lag, (int)iz);
                image[j + (lag + nlag) * n] +=
                    sv * (d * ((T)kTwoThird * lcx[j + lag] + (T)kOneThird * lcz[j + lag]));
              }
            }
      }
      std::swap(cx, px); std::swap(cz, pz);
      std::swap(lcx, lpx); std::swap(lcz, lpz);
    }
  }
}

// waveletGradientCij3d_f (lib/vti-fwi-3d/gpu/modelData3d_f.cu:858-1294): the
// adjoint wavefield alone, seeded with the last data sample (:1048-1053),
// stepped with the forward operator, fed the data interpolated at it+1 and
// damped by the sponge; extractAdjWfldAtSouLoc (injectRecord3d.cu:9-12) adds
// lambda_x + lambda_z of the new level at the source, as the step computed
// it (before the residual injection and the sponge), into g[it]; finally
// g *= dt2 (:1293). Here the undamped value is the stored one over the sponge
// factor d at the source.
template <typename T>
void wavelet_grad3d(const Geo3& g, const float* c11, const float* c13, const float* c33,
                    const float* souloc, const int* shotid, int nshot, const float* recloc,
                    const float* data, T* gw) {
  const long n = g.nxyz(), nxy = g.nxy();
  const float dt2 = g.dt * g.dt;
  const int st = sampling_step(g.rate, g.dt);
  const int nnt = (g.nt - 1) / st + 1;
  const int M = last_level(g);
  std::fill(gw, gw + g.nt, (T)0);
  Damp3 damp(g);
  std::vector<T> lcx, lcz, lpx, lpz;
  for (int k = 0; k < nshot; ++k) {
    Shot3 s = make_shot3(g, souloc, recloc, shotid[k]);
    const float* dat = data + (long)nnt * s.irbegin;
    lcx.assign(n, 0); lcz.assign(n, 0); lpx.assign(n, 0); lpz.assign(n, 0);
    for (int ir = 0; ir < s.nr; ++ir) {
      if (!s.inner[ir]) continue;
      T temp = (T)dt2 * (T)dat[(nnt - 1) + (long)ir * nnt];
      lcx[s.seed[ir]] = (T)kTwoThird * temp;
      lcz[s.seed[ir]] = (T)kOneThird * temp;
    }
    const T ds = (T)damp.at(s.sidx % nxy, (int)(s.sidx / nxy));
    for (int i = 0; i < M - 1; ++i) {
      const int it = g.nt - 3 - i;
      step3d<T, true>(g, c11, c13, c33, lcx.data(), lcz.data(), lpx.data(), lpz.data(), &damp,
                      nullptr, nullptr, nullptr, nullptr, nullptr);
      gw[it] += (lpx[s.sidx] + lpz[s.sidx]) / ds;
      for (int ir = 0; ir < s.nr; ++ir) {
        if (!s.inner[ir]) continue;
        std::vector<T> tr(dat + (long)ir * nnt, dat + (long)(ir + 1) * nnt);
        T inj = (T)dt2 * interp_residual<T>(tr.data(), it + 1, nnt, st);
        long ri = s.ridx[ir];
        T d = (T)damp.at(ri % nxy, (int)(ri / nxy));
        lpx[ri] += d * ((T)kTwoThird * inj);
        lpz[ri] += d * ((T)kOneThird * inj);
      }
      std::swap(lcx, lpx); std::swap(lcz, lpz);
    }
  }
  for (int it = 0; it < g.nt; ++it) gw[it] *= (T)dt2;
}

// ----------------------------------------------------------------- 2D ------
struct Geo2 {
  int nx, nz, nt, npad;
  float dx, dz, dt, rate, ot;
  int nnx() const { return nx + 2 * npad; }
  int nnz() const { return nz + 2 * npad; }
};

Geo2 unpack2(const int* ip, const float* fp) {
  Geo2 g;
  g.nx = ip[0]; g.nz = ip[1]; g.nt = ip[2]; g.npad = ip[3];
  g.dx = fp[0]; g.dz = fp[1]; g.dt = fp[2]; g.rate = fp[3]; g.ot = fp[4];
  return g;
}

// forwardCD (kernels.cu:452-498): p0 <- 2p1 + dt2(c11 Dxx p1 + c13 Dzz q1) - p0.
template <typename T>
void step2d(const Geo2& g, const float* c11, const float* c13, const float* c33, const T* p1,
            const T* q1, T* p0, T* q0) {
  const long nnx = g.nnx(), nnz = g.nnz();
  const float dx2 = g.dx * g.dx, dz2 = g.dz * g.dz, dt2 = g.dt * g.dt;
  const T C[5] = {(T)k2C0, (T)k2C1, (T)k2C2, (T)k2C3, (T)k2C4};
#pragma omp parallel for schedule(static)
  for (long iz = kHalf; iz < nnz - kHalf; ++iz)
    for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
      long i = ix + iz * nnx;
      T tp = C[0] * p1[i], tq = C[0] * q1[i];
      for (int k = 1; k <= 4; ++k) {
        tp += C[k] * (p1[i - k] + p1[i + k]);
        tq += C[k] * (q1[i - k * nnx] + q1[i + k * nnx]);
      }
      tp /= (T)dx2;
      tq /= (T)dz2;
      p0[i] = 2 * p1[i] + (T)dt2 * ((T)c11[i] * tp + (T)c13[i] * tq) - p0[i];
      q0[i] = 2 * q1[i] + (T)dt2 * ((T)c13[i] * tp + (T)c33[i] * tq) - q0[i];
    }
}

template <typename T>
void taper2d(const Geo2& g, const float* taper, T* a) {
  const long nnx = g.nnx(), nnz = g.nnz();
  for (long iz = kHalf; iz < nnz - kHalf; ++iz)
    for (long ix = kHalf; ix < nnx - kHalf; ++ix) a[ix + iz * nnx] *= (T)taper[ix + iz * nnx];
}

// injectDipoleSource / injectDipoleData (kernels.cu:232-256): +a at i, -a one
// row below.
template <typename T>
void dipole2d(const Geo2& g, T* p, T* q, long i, T a) {
  p[i] += a;
  q[i] += a;
  p[i + g.nnx()] -= a;
  q[i + g.nnx()] -= a;
}

// rtm_f (lib/vti-fwi-2d/rtm_f.cu:13-267): dipole source; source wavefield
// slices 0.5(p+q) of the interior at it % ratio == 0 (and level 1 when
// ratio == 1, recordWavefieldSlice kernels.cu:335-343) kept for the whole
// shot; the receiver wavefield (forwardCD, data as dipoles interpolated in
// time, taper) is imaged with imagingCrossCor (kernels.cu:414-423):
// image += 0.5(p+q) * ((1-f) S0 + f S1). Slices never written are zero (the
// host array is zero-initialised once, rtm_f.cu:55; the index one past the
// last slice, read with weight 0 at the first imaging, is taken as zero).
// nhx >= 0: odcig_f (lib/vti-fwi-2d/odcig_f.cu:12-232), the same migration
// with extendedImagingCrossCor (kernels.cu:425-436): image[i + (h+nhx)*nnxz]
// += 0.5(p+q)[i-h] * S[i+h] for |h| <= nhx over the reference kernel's threads
// (16x16 blocks from (4,4): x in [max(4,nhx), min(nnx-nhx, 4+16*gx)), z in
// [4, min(nnz, 4+16*gz))); its source pass injects w[it-1] without the dt2
// factor after level 1 (odcig_f.cu:124).
template <typename T>
void rtm2d(const Geo2& g, const float* c11, const float* c13, const float* c33,
           const float* wavelet, const float* data, const int* sloc, int ns, const int* rloc,
           int nr_total, const float* taper, T* image, int nhx = -1) {
  const long nnx = g.nnx(), nnz = g.nnz(), nnxz = nnx * nnz;
  const float dt = g.dt, dt2 = dt * dt;
  const int ratio = (int)(g.rate / dt + 0.5f);
  const int ntNeg = (int)std::round(std::fabs(g.ot) / dt);
  const int nnt = (g.nt - 1) / ratio + 1;
  const int nnt_data = (g.nt - ntNeg - 1) / ratio + 1;
  const long nimg = nhx < 0 ? 1 : 2 * nhx + 1;
  std::fill(image, image + nnxz * nimg, (T)0);
  std::vector<T> sw((size_t)(nnt + 1) * nnxz, 0);
  auto slice = [&](int j, const T* p, const T* q) {
    for (long iz = kHalf; iz < nnz - kHalf; ++iz)
      for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
        long i = ix + iz * nnx;
        sw[(size_t)j * nnxz + i] = (T)0.5f * (p[i] + q[i]);
      }
  };
  const long gx = (nnx - 8 + 15) / 16, gz = (nnz - 8 + 15) / 16;
  auto img = [&](const T* p, const T* q, int s0, int s1, float f) {
    const T* A = sw.data() + (size_t)s0 * nnxz;
    const T* B = sw.data() + (size_t)s1 * nnxz;
    if (nhx >= 0) {
      for (long iz = kHalf; iz < std::min(nnz, 4 + 16 * gz); ++iz)
        for (long ix = std::max<long>(kHalf, nhx); ix < std::min<long>(nnx - nhx, 4 + 16 * gx);
             ++ix) {
          long i = ix + iz * nnx;
          for (int h = -nhx; h <= nhx; ++h) {
            T d = (1 - (T)f) * A[i + h] + (T)f * B[i + h];
            image[i + (h + nhx) * nnxz] += (T)0.5f * (p[i - h] + q[i - h]) * d;
          }
        }
      return;
    }
    for (long iz = kHalf; iz < nnz - kHalf; ++iz)
      for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
        long i = ix + iz * nnx;
        T d = (1 - (T)f) * A[i] + (T)f * B[i];
        image[i] += (T)0.5f * (p[i] + q[i]) * d;
      }
  };
  for (int is = 0; is < ns; ++is) {
    const long sxz = sloc[4 * is] + (long)sloc[4 * is + 1] * nnx;
    const int nri = sloc[4 * is + 2], ir0 = sloc[4 * is + 3];
    std::vector<T> p0(nnxz, 0), q0(nnxz, 0), p1(nnxz, 0), q1(nnxz, 0);
    dipole2d<T>(g, p1.data(), q1.data(), sxz, (T)(dt2 * wavelet[0]));
    taper2d(g, taper, p1.data());
    taper2d(g, taper, q1.data());
    if (ratio == 1) slice(1, p1.data(), q1.data());
    for (int it = 2; it < g.nt; ++it) {
      step2d<T>(g, c11, c13, c33, p1.data(), q1.data(), p0.data(), q0.data());
      dipole2d<T>(g, p0.data(), q0.data(), sxz,
                  (T)(nhx < 0 ? dt2 * wavelet[it - 1] : wavelet[it - 1]));
      taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
      taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
      if (it % ratio == 0) slice(it / ratio, p0.data(), q0.data());
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
    std::fill(p0.begin(), p0.end(), (T)0); std::fill(q0.begin(), q0.end(), (T)0);
    std::fill(p1.begin(), p1.end(), (T)0); std::fill(q1.begin(), q1.end(), (T)0);
    std::vector<float> d0(nri, 0.f), d1(nri, 0.f);
    for (int ir = 0; ir < nri; ++ir) d0[ir] = data[(long)(nnt_data - 1) * nr_total + ir0 + ir];
    auto inject = [&](T* p, T* q, float f) {
      for (int ir = 0; ir < nri; ++ir) {
        long i = rloc[2 * (ir0 + ir)] + (long)rloc[2 * (ir0 + ir) + 1] * nnx;
        float s = 0.5f * ((1.f - f) * d0[ir] + f * d1[ir]);
        dipole2d<T>(g, p, q, i, (T)(dt2 * s));
      }
    };
    inject(p0.data(), q0.data(), 0.f);
    taper2d(g, taper, p0.data());
    taper2d(g, taper, q0.data());
    float f = (g.nt - 2.) / ratio;
    int s0 = (int)f, s1 = s0 + 1;
    if (s1 > nnt) s1 = nnt;
    f = f - s0;
    img(p0.data(), q0.data(), s0, s1, f);
    for (int it = g.nt - 3; it >= 0; --it) {
      step2d<T>(g, c11, c13, c33, p0.data(), q0.data(), p1.data(), q1.data());
      if (it >= ntNeg) {
        f = (it - ntNeg + 1.) / ratio;
        int i1 = (int)f;
        if ((it - ntNeg + 2) % ratio == 0) {
          for (int ir = 0; ir < nri; ++ir) d1[ir] = data[(long)i1 * nr_total + ir0 + ir];
          std::swap(d0, d1);
        }
        f = f - i1;
        inject(p1.data(), q1.data(), f);
      }
      taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
      taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
      f = (float)it / ratio;
      int i1 = (int)f;
      if ((it + 1) % ratio == 0) {
        s1 = i1;
        std::swap(s0, s1);
      }
      f = f - i1;
      img(p1.data(), q1.data(), s0, s1, f);
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
  }
}

// waveletGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:373-530): per shot
// the adjoint wavefield (forwardCD, point injection of the data interpolated
// at it+1, taper), g[it] = dt2 (p + q) at the source after the taper
// (extractWavelet, kernels.cu:258-261; an assignment), g[nt-2] from the
// seeded level; shots summed. ratio uses a double 0.5 here (:375). The second
// data row of the first step is weighted 0 (the reference leaves that buffer
// uninitialised; it is taken as zero).
template <typename T>
void wavelet_grad2d(const Geo2& g, const float* c11, const float* c13, const float* c33,
                    const float* data, const int* sloc, int ns, const int* rloc, int nr_total,
                    const float* taper, T* gw) {
  const long nnx = g.nnx(), nnxz = nnx * g.nnz();
  const float dt = g.dt, dt2 = dt * dt;
  const int ratio = (int)(g.rate / dt + 0.5);
  const int nnt = (g.nt - 1) / ratio + 1;
  std::fill(gw, gw + g.nt, (T)0);
  for (int is = 0; is < ns; ++is) {
    const long sxz = sloc[4 * is] + (long)sloc[4 * is + 1] * nnx;
    const int nri = sloc[4 * is + 2], ir0 = sloc[4 * is + 3];
    std::vector<T> gs(g.nt, 0);
    std::vector<T> p0(nnxz, 0), q0(nnxz, 0), p1(nnxz, 0), q1(nnxz, 0);
    std::vector<float> d0(nri, 0.f), d1(nri, 0.f);
    for (int ir = 0; ir < nri; ++ir) d0[ir] = data[(long)(nnt - 1) * nr_total + ir0 + ir];
    auto inject = [&](T* p, T* q, float f) {  // injectData (kernels.cu:208-217)
      for (int ir = 0; ir < nri; ++ir) {
        long i = rloc[2 * (ir0 + ir)] + (long)rloc[2 * (ir0 + ir) + 1] * nnx;
        float s = 0.5f * ((1.f - f) * d0[ir] + f * d1[ir]);
        p[i] += (T)(dt2 * s);
        q[i] += (T)(dt2 * s);
      }
    };
    inject(p0.data(), q0.data(), 0.f);
    taper2d(g, taper, p0.data());
    taper2d(g, taper, q0.data());
    gs[g.nt - 2] = (T)dt2 * (p0[sxz] + q0[sxz]);
    for (int it = g.nt - 3; it >= 0; --it) {
      step2d<T>(g, c11, c13, c33, p0.data(), q0.data(), p1.data(), q1.data());
      float f = (it + 1.) / ratio;
      int i1 = (int)f;
      if ((it + 2) % ratio == 0) {
        for (int ir = 0; ir < nri; ++ir) d1[ir] = data[(long)i1 * nr_total + ir0 + ir];
        std::swap(d0, d1);
      }
      f = f - i1;
      inject(p1.data(), q1.data(), f);
      taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
      taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
      gs[it] = (T)dt2 * (p1[sxz] + q1[sxz]);
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
    for (int it = 0; it < g.nt; ++it) gw[it] += gs[it];
  }
}

// synthetic_f (synthetic_f.cu:13-124) and modeling_f (modeling_f.cu:10-82).
// mode 0: traces, data[t*nr + ir_global] = 0.5(p+q) at receivers.
// mode 1: snapshots of p (modeling_f), out[t*nnxz + i]; the source term of
//         modeling_f's time loop is wavelet[it-1] without dt2
//         (modeling_f.cu:66).
template <typename T>
void forward2d(const Geo2& g, const float* c11, const float* c13, const float* c33,
               const float* wavelet, const int* sloc, int is, const int* rloc, int nr_total,
               const float* taper, T* out, int mode) {
  const long nnx = g.nnx(), nnxz = nnx * g.nnz();
  const float dt = g.dt, dt2 = dt * dt;
  const int ratio = mode == 0 ? (int)(g.rate / dt + 0.5f) : (int)std::round(g.rate / dt);
  const int ntNeg = (int)std::round(std::fabs(g.ot) / dt);
  std::vector<T> p0(nnxz, 0), q0(nnxz, 0), p1(nnxz, 0), q1(nnxz, 0);
  long slocxz = mode == 0 ? sloc[4 * is] + (long)sloc[4 * is + 1] * nnx : sloc[0];
  const int nri = mode == 0 ? sloc[4 * is + 2] : 0;
  const int ir0 = mode == 0 ? sloc[4 * is + 3] : 0;
  auto record = [&](long row, const T* p, const T* q) {
    if (mode == 0) {
      for (int ir = 0; ir < nri; ++ir) {
        long i = rloc[2 * (ir0 + ir)] + (long)rloc[2 * (ir0 + ir) + 1] * nnx;
        out[row * nr_total + ir0 + ir] = (T)0.5f * (p[i] + q[i]);
      }
    } else {
      std::copy(p, p + nnxz, out + row * nnxz);
    }
  };
  p1[slocxz] += (T)(dt2 * wavelet[0]);
  q1[slocxz] += (T)(dt2 * wavelet[0]);
  taper2d(g, taper, p1.data());
  taper2d(g, taper, q1.data());
  if (ratio == 1 && g.ot == 0.f) record(1, p1.data(), q1.data());
  for (int it = 2; it < g.nt; ++it) {
    float t = it * dt + g.ot;
    step2d<T>(g, c11, c13, c33, p1.data(), q1.data(), p0.data(), q0.data());
    float src = mode == 0 ? dt2 * wavelet[it - 1] : wavelet[it - 1];
    p0[slocxz] += (T)src;
    q0[slocxz] += (T)src;
    taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
    taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
    if (t >= 0.f && (it - ntNeg) % ratio == 0) record((it - ntNeg) / ratio, p0.data(), q0.data());
    std::swap(p0, p1);
    std::swap(q0, q1);
  }
}

// --------------------------------------------- 2D gradient and GN H*v ------
// D kernel (kernels.cu:345-387): tp = Dxx p / dx2, tq = Dzz q / dz2 on the
// interior, zero elsewhere.
template <typename T>
void dop2d(const Geo2& g, const T* p, const T* q, T* tp, T* tq) {
  const long nnx = g.nnx(), nnz = g.nnz();
  const float dx2 = g.dx * g.dx, dz2 = g.dz * g.dz;
  const T C[5] = {(T)k2C0, (T)k2C1, (T)k2C2, (T)k2C3, (T)k2C4};
  std::fill(tp, tp + nnx * nnz, (T)0);
  std::fill(tq, tq + nnx * nnz, (T)0);
#pragma omp parallel for schedule(static)
  for (long iz = kHalf; iz < nnz - kHalf; ++iz)
    for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
      long i = ix + iz * nnx;
      T a = C[0] * p[i], b = C[0] * q[i];
      for (int k = 1; k <= 4; ++k) {
        a += C[k] * (p[i - k] + p[i + k]);
        b += C[k] * (q[i - k * nnx] + q[i + k * nnx]);
      }
      tp[i] = a / (T)dx2;
      tq[i] = b / (T)dz2;
    }
}

// One adjoint level on the interior. exact: backwardDC (kernels.cu:104-148),
// p1 <- 2p0 + dt2 * D(C p0) - p1; otherwise forwardCD (kernels.cu:452-498).
template <typename T>
void adj2d(const Geo2& g, const float* c11, const float* c13, const float* c33, const T* p0,
           const T* q0, T* p1, T* q1, bool exact) {
  const long nnx = g.nnx(), nnz = g.nnz(), n = nnx * nnz;
  const float dx2 = g.dx * g.dx, dz2 = g.dz * g.dz, dt2 = g.dt * g.dt;
  const T C[5] = {(T)k2C0, (T)k2C1, (T)k2C2, (T)k2C3, (T)k2C4};
  std::vector<T> a(n), b(n);
  if (exact) {
    for (long i = 0; i < n; ++i) {
      a[i] = (T)c11[i] * p0[i] + (T)c13[i] * q0[i];
      b[i] = (T)c13[i] * p0[i] + (T)c33[i] * q0[i];
    }
  }
#pragma omp parallel for schedule(static)
  for (long iz = kHalf; iz < nnz - kHalf; ++iz)
    for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
      long i = ix + iz * nnx;
      const T* u = exact ? a.data() : p0;
      const T* w = exact ? b.data() : q0;
      T tp = C[0] * u[i], tq = C[0] * w[i];
      for (int k = 1; k <= 4; ++k) {
        tp += C[k] * (u[i - k] + u[i + k]);
        tq += C[k] * (w[i - k * nnx] + w[i + k * nnx]);
      }
      tp /= (T)dx2;
      tq /= (T)dz2;
      if (exact) {
        p1[i] = 2 * p0[i] + (T)dt2 * tp - p1[i];
        q1[i] = 2 * q0[i] + (T)dt2 * tq - q1[i];
      } else {
        p1[i] = 2 * p0[i] + (T)dt2 * ((T)c11[i] * tp + (T)c13[i] * tq) - p1[i];
        q1[i] = 2 * q0[i] + (T)dt2 * ((T)c13[i] * tp + (T)c33[i] * tq) - q1[i];
      }
    }
}

// Which stored D(sigma) levels each backward imaging step of the 2D gradient
// and Gauss-Newton product reads. The reference moves checkpoints through
// three device buffers (Dpq, Dpqa, Dpqb), two pinned host buffers and a host
// array Dp[] (objFuncGradient_f.cu:168-202 forward, :240-292 backward;
// hessian_f.cu mirrors it). This replays those copies with labels: label t
// means D(v_t), -1 a zero buffer. Entry 0 is the imaging of lambda(nt-1)
// before the loop; entry 1+j the step it = nt-3-j.
// None of these buffers is cleared between shots (only at allocation), so a
// shot can image against checkpoints left by the previous shot on the same
// GPU: labels therefore carry the shot, label = shot*(nt+1) + t.
struct Pair {
  long a, b;  // labels of Dp0 (d_Dpqa) and Dp1 (d_Dpq)
  float f;    // weight of b
};
struct CkState {
  long dq = -1, da = -1, db = -1, ha = -1, hb = -1;
  std::vector<long> Dp;
};
std::vector<Pair> checkpoint_shot(CkState& S, int shot, int nt, int r) {
  const int nnt = (nt - 1) / r + 1;
  auto L = [&](int t) { return (long)shot * (nt + 1) + t; };
  if (S.Dp.empty()) S.Dp.assign(std::max(nnt, 1), -1);
  S.dq = L(1);  // D(v_1) computed at the start of every shot
  for (int it = 2; it < nt; ++it) {
    S.dq = L(it);
    if (it % r == 0) {
      if (it != nt - 1) S.da = S.dq;
      if (it > r && it / r - 1 < nnt) S.Dp[it / r - 1] = S.ha;
    }
    if (it % r == 1 && it != nt - r) S.ha = S.da;
  }
  std::vector<Pair> out;
  if (nnt - 3 >= 0) S.hb = S.Dp[nnt - 3];
  {
    float f = (nt - 2.) / r;
    int i1 = (int)f;
    out.push_back({S.da, S.dq, f - i1});
  }
  for (int it = nt - 3; it >= 0; --it) {
    if (it % r == 0) {
      std::swap(S.ha, S.hb);
      S.db = S.ha;
      if (it >= 2 * r) S.hb = S.Dp[it / r - 2];
    }
    if ((it + 1) % r == 0) {
      long t = S.db;
      S.db = S.dq;
      S.dq = S.da;
      S.da = t;
    }
    float f = (float)it / r;
    int i1 = (int)f;
    out.push_back({S.da, S.dq, f - i1});
  }
  return out;
}
std::vector<Pair> checkpoint_schedule(int nt, int r) {
  CkState S;
  return checkpoint_shot(S, 0, nt, r);
}

// gradientCrossCor (kernels.cu:438-450)
template <typename T>
void image2d(const Geo2& g, const T* ap, const T* aq, const T* Dp0, const T* Dq0, const T* Dp1,
             const T* Dq1, float f, T* g11, T* g13, T* g33) {
  const long nnx = g.nnx(), nnz = g.nnz();
  for (long iz = kHalf; iz < nnz - kHalf; ++iz)
    for (long ix = kHalf; ix < nnx - kHalf; ++ix) {
      long i = ix + iz * nnx;
      T Dp = (1 - (T)f) * (Dp0 ? Dp0[i] : 0) + (T)f * (Dp1 ? Dp1[i] : 0);
      T Dq = (1 - (T)f) * (Dq0 ? Dq0[i] : 0) + (T)f * (Dq1 ? Dq1[i] : 0);
      g11[i] += ap[i] * Dp;
      g13[i] += ap[i] * Dq + aq[i] * Dp;
      g33[i] += aq[i] * Dq;
    }
}

// objFuncGradient_f (objFuncGradient_f.cu:15-371) when born == false;
// GNhessian_f (hessian_f.cu:575-1010) when born == true (dc = model
// perturbation, the Born data replace the residual, the adjoint uses the
// forward operator). Returns 0.5 * sum of squared residuals (gradient).
template <typename T>
double grad2d(const Geo2& g, const float* c11, const float* c13, const float* c33,
              const float* dc11, const float* dc13, const float* dc33, const float* wavelet,
              const int* sloc, int ns, const int* rloc, int nr_total, const float* taper,
              const float* data, T* g11, T* g13, T* g33, bool born) {
  const long nnx = g.nnx(), nnxz = nnx * g.nnz();
  const float dt = g.dt, dt2 = dt * dt;
  const int ratio = (int)(g.rate / dt + 0.5f);
  const int ntNeg = (int)std::round(std::fabs(g.ot) / dt);
  const int nnt_data = (g.nt - ntNeg - 1) / ratio + 1;
  std::fill(g11, g11 + nnxz, (T)0);
  std::fill(g13, g13 + nnxz, (T)0);
  std::fill(g33, g33 + nnxz, (T)0);
  // checkpoint pairing of every shot (state carried from shot to shot)
  std::vector<std::vector<Pair>> sched(ns);
  {
    CkState S;
    for (int is = 0; is < ns; ++is) sched[is] = checkpoint_shot(S, is, g.nt, ratio);
  }
  std::map<long, std::pair<std::vector<T>, std::vector<T>>> ck;  // label -> (Dp, Dq)
  for (const auto& v : sched)
    for (const Pair& p : v) {
      if (p.a >= 0) ck[p.a];
      if (p.b >= 0) ck[p.b];
    }
  auto keep = [&](int is, int t, const std::vector<T>& a, const std::vector<T>& b) {
    auto it = ck.find((long)is * (g.nt + 1) + t);
    if (it != ck.end()) it->second = {a, b};
  };
  double objfunc = 0;
  // the Born D buffer (d_Ddpq) is zeroed once, not per shot (hessian_f.cu:647-648)
  std::vector<T> dtp(nnxz, 0), dtq(nnxz, 0);
  for (int is = 0; is < ns; ++is) {
    const long sxz = sloc[4 * is] + (long)sloc[4 * is + 1] * nnx;
    const int nri = sloc[4 * is + 2], ir0 = sloc[4 * is + 3];
    std::vector<long> ridx(nri);
    for (int ir = 0; ir < nri; ++ir)
      ridx[ir] = rloc[2 * (ir0 + ir)] + (long)rloc[2 * (ir0 + ir) + 1] * nnx;
    std::vector<T> p0(nnxz, 0), q0(nnxz, 0), p1(nnxz, 0), q1(nnxz, 0);
    std::vector<T> dp0(nnxz, 0), dq0(nnxz, 0), dp1(nnxz, 0), dq1(nnxz, 0);
    std::vector<T> tp(nnxz), tq(nnxz);
    std::vector<T> rec((long)nnt_data * nri, 0);
    p1[sxz] = (T)(dt2 * wavelet[0]);
    q1[sxz] = (T)(dt2 * wavelet[0]);
    dop2d(g, p1.data(), q1.data(), tp.data(), tq.data());
    keep(is, 1, tp, tq);
    for (int it = 2; it < g.nt; ++it) {
      const float t = it * dt + g.ot;
      // forwardC with the stored D of the previous level (kernels.cu:546-556)
      for (long i = 0; i < nnxz; ++i) {
        long ix = i % nnx, iz = i / nnx;
        if (ix < kHalf || ix >= nnx - kHalf || iz < kHalf || iz >= g.nnz() - kHalf) continue;
        p0[i] = 2 * p1[i] + (T)dt2 * ((T)c11[i] * tp[i] + (T)c13[i] * tq[i]) - p0[i];
        q0[i] = 2 * q1[i] + (T)dt2 * ((T)c13[i] * tp[i] + (T)c33[i] * tq[i]) - q0[i];
        if (born) {
          dp0[i] = 2 * dp1[i] + (T)dt2 * ((T)c11[i] * dtp[i] + (T)c13[i] * dtq[i]) - dp0[i];
          dq0[i] = 2 * dq1[i] + (T)dt2 * ((T)c13[i] * dtp[i] + (T)c33[i] * dtq[i]) - dq0[i];
          // scattering (kernels.cu:282-291) with the background D of it-1
          dp0[i] += (T)dt2 * ((T)dc11[i] * tp[i] + (T)dc13[i] * tq[i]);
          dq0[i] += (T)dt2 * ((T)dc13[i] * tp[i] + (T)dc33[i] * tq[i]);
        }
      }
      p0[sxz] += (T)(dt2 * wavelet[it - 1]);
      q0[sxz] += (T)(dt2 * wavelet[it - 1]);
      taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
      taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
      if (born) {
        taper2d(g, taper, dp1.data()); taper2d(g, taper, dq1.data());
        taper2d(g, taper, dp0.data()); taper2d(g, taper, dq0.data());
        dop2d(g, dp0.data(), dq0.data(), dtp.data(), dtq.data());
      }
      dop2d(g, p0.data(), q0.data(), tp.data(), tq.data());
      keep(is, it, tp, tq);
      if (t >= 0.f && (it - ntNeg) % ratio == 0) {
        const T* a = born ? dp0.data() : p0.data();
        const T* b = born ? dq0.data() : q0.data();
        for (int ir = 0; ir < nri; ++ir)
          rec[(long)((it - ntNeg) / ratio) * nri + ir] = (T)0.5f * (a[ridx[ir]] + b[ridx[ir]]);
      }
      std::swap(p0, p1); std::swap(q0, q1);
      std::swap(dp0, dp1); std::swap(dq0, dq1);
    }
    // adjoint source: residual (gradient) or Born data (GN product)
    if (!born) {
      for (int t = 0; t < nnt_data; ++t)
        for (int ir = 0; ir < nri; ++ir) {
          T& r = rec[(long)t * nri + ir];
          r = r - (T)data[(long)t * nr_total + ir0 + ir];
          objfunc += (double)(r * r);
        }
    }
    std::fill(p0.begin(), p0.end(), (T)0); std::fill(q0.begin(), q0.end(), (T)0);
    std::fill(p1.begin(), p1.end(), (T)0); std::fill(q1.begin(), q1.end(), (T)0);
    std::vector<T> b0(nri, 0), b1(nri, 0);
    for (int ir = 0; ir < nri; ++ir) b0[ir] = rec[(long)(nnt_data - 1) * nri + ir];
    auto inject = [&](T* p, T* q, float f) {  // injectData (kernels.cu:208-217)
      for (int ir = 0; ir < nri; ++ir) {
        T s = (T)0.5f * ((1 - (T)f) * b0[ir] + (T)f * b1[ir]);
        p[ridx[ir]] += (T)dt2 * s;
        q[ridx[ir]] += (T)dt2 * s;
      }
    };
    auto img = [&](const Pair& pr, const T* ap, const T* aq) {
      const std::vector<T>* A = pr.a >= 0 ? &ck[pr.a].first : nullptr;
      const std::vector<T>* Aq = pr.a >= 0 ? &ck[pr.a].second : nullptr;
      const std::vector<T>* B = pr.b >= 0 ? &ck[pr.b].first : nullptr;
      const std::vector<T>* Bq = pr.b >= 0 ? &ck[pr.b].second : nullptr;
      auto ptr = [](const std::vector<T>* v) { return v && !v->empty() ? v->data() : nullptr; };
      image2d<T>(g, ap, aq, ptr(A), ptr(Aq), ptr(B), ptr(Bq), pr.f, g11, g13, g33);
    };
    inject(p0.data(), q0.data(), 0.f);
    img(sched[is][0], p0.data(), q0.data());
    int step = 1;
    for (int it = g.nt - 3; it >= 0; --it, ++step) {
      adj2d<T>(g, c11, c13, c33, p0.data(), q0.data(), p1.data(), q1.data(), !born);
      if (it >= ntNeg) {
        float f = (it - ntNeg + 1.) / ratio;
        int i1 = (int)f;
        if ((it - ntNeg + 2) % ratio == 0) {
          for (int ir = 0; ir < nri; ++ir) b1[ir] = rec[(long)i1 * nri + ir];
          std::swap(b0, b1);
        }
        inject(p1.data(), q1.data(), f - i1);
      }
      taper2d(g, taper, p1.data()); taper2d(g, taper, q1.data());
      taper2d(g, taper, p0.data()); taper2d(g, taper, q0.data());
      img(sched[is][step], p1.data(), q1.data());
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
  }
  return 0.5 * objfunc;
}

}  // namespace

// ------------------------------------------------- EXACT adjoint mode ------
// Self-check operators. The reference's 3D gradient is not the derivative of
// its own misfit: it propagates the adjoint with the forward operator C.L
// (objFuncGradient3d_f.cu:1002-1010) rather than its transpose L.C (the form
// of adjointCij, laplacian3d.ispc:166-190), rebuilds the source field through
// a random boundary and injects time-interpolated residuals
// (injectRecord3d.cu:60-78). EXACT mode fixes one discrete forward operator
// and differentiates it exactly, so a dot-product test and centred finite
// differences can check the adjoint-state machinery itself:
//   a_0 = 0, a_1 = dt2 w[0] e_s,
//   a_t = P [ D ((2 + C L) a_{t-1} + dt2 w[t-1] e_s) - (2D - 1) a_{t-2} ],  t = 2..M
// with P the x/y update region, D the sponge profile (abc3d.cu:23-50) as a
// diagonal, C L the forward-form VTI operator of step3d. The damping is the
// centred form u'' + g u' = C L u with D = 1/(1 + g dt/2), which is
// energy-stable for any D <= 1 (the reference's form, D applied to next and
// again to cur, subtracts D^2 a_{t-2}; equal to first order in 1 - D, and
// without the block-order reading it grew without bound over 4000 steps of a
// 600x600x300 grid). Traces d_j = 2/3 a_x + 1/3 a_z at each receiver's own
// cell and level j*st; J = 1/2 sum over live receivers of (d - dobs)^2. Its
// adjoint:
//   mu_t = P [ D (R^T r_t + 2 mu_{t+1} + (C L)^T mu_{t+1}) - (2D - 1) mu_{t+2} ],
//   (C L)^T mu = ( L_xy(c11 mu_x + c13 mu_z), L_z(c13 mu_x + c33 mu_z) ),
//   dJ/dc11 = sum_t mu_t,x L_xy a_{t-1,x},  dJ/dc33 = sum_t mu_t,z L_z a_{t-1,z},
//   dJ/dc13 = sum_t mu_t,x L_z a_{t-1,z} + mu_t,z L_xy a_{t-1,x}.
// The Born operator (dJ/dc applied to a model perturbation) is the
// linearisation of the same recursion: source term dC L a_{t-1}.

// lxy <- L_xy ux, lz <- L_z uz (forward-form scaling dt2/dx2 as step3d) on
// the update region, zero elsewhere; z reads outside [0,nz) are zero.
template <typename T>
void lap3d(const Geo3& g, const T* ux, const T* uz, T* lxy, T* lz) {
  const long nx = g.nx, ny = g.ny, nz = g.nz, nxy = g.nxy();
  const float dt2 = g.dt * g.dt;
  const float sx = dt2 / (g.dx * g.dx), sy = dt2 / (g.dy * g.dy), sz = dt2 / (g.dz * g.dz);
  const T C[5] = {(T)k3C0, (T)k3C1, (T)k3C2, (T)k3C3, (T)k3C4};
  std::fill(lxy, lxy + g.nxyz(), (T)0);
  std::fill(lz, lz + g.nxyz(), (T)0);
#pragma omp parallel for collapse(2) schedule(static)
  for (long iz = 0; iz < nz; ++iz)
    for (long iy = kHalf; iy < ny - kHalf; ++iy)
      for (long ix = kHalf; ix < nx - kHalf; ++ix) {
        const long i = ix + iy * nx + iz * nxy;
        T lxx = C[0] * ux[i], lyy = C[0] * ux[i], lzz = C[0] * uz[i];
        for (int k = 1; k <= 4; ++k) {
          lxx += C[k] * (ux[i - k] + ux[i + k]);
          lyy += C[k] * (ux[i - k * nx] + ux[i + k * nx]);
          lzz += C[k] * ((iz - k >= 0 ? uz[i - k * nxy] : (T)0) +
                         (iz + k < nz ? uz[i + k * nxy] : (T)0));
        }
        lxy[i] = lxx * (T)sx + lyy * (T)sy;
        lz[i] = lzz * (T)sz;
      }
}

struct ExactShot {
  long sidx;
  std::vector<long> ridx;
  std::vector<char> live;
  int irbegin, nr;
};

ExactShot exact_shot(const Geo3& g, const float* souloc, const float* recloc, int is) {
  Shot3 s = make_shot3(g, souloc, recloc, is);
  return ExactShot{s.sidx, s.seed, s.live, s.irbegin, s.nr};
}

// Level recorded into sample j (0: none).
inline int exact_level(int j, int st, int M) { return j >= 1 && j * st <= M ? j * st : 0; }

template <typename T>
struct ExactHistory {
  std::vector<std::vector<T>> a;  // level t: x then z components (2n)
};

// Forward recursion; a.a[t] for t = 0..M. dc != nullptr: the Born field of
// the perturbation (dc11,dc13,dc33) around the background history `bg`.
template <typename T>
void exact_forward3d(const Geo3& g, const T* c11, const T* c13, const T* c33,
                     const float* wavelet, const ExactShot& s, const Damp3& damp,
                     ExactHistory<T>& h, const ExactHistory<T>* bg = nullptr,
                     const T* dc = nullptr) {
  const long n = g.nxyz(), nxy = g.nxy();
  const int M = last_level(g);
  const float dt2 = g.dt * g.dt;
  h.a.assign(M + 1, std::vector<T>(2 * n, (T)0));
  if (!dc) {
    h.a[1][s.sidx] = (T)(dt2 * wavelet[0]);
    h.a[1][n + s.sidx] = (T)(dt2 * wavelet[0]);
  }
  std::vector<T> lxy(n), lz(n), bxy(n), bz(n);
  for (int t = 2; t <= M; ++t) {
    const T* u1 = h.a[t - 1].data();
    const T* u2 = h.a[t - 2].data();
    T* u = h.a[t].data();
    lap3d<T>(g, u1, u1 + n, lxy.data(), lz.data());
    if (dc) lap3d<T>(g, bg->a[t - 1].data(), bg->a[t - 1].data() + n, bxy.data(), bz.data());
#pragma omp parallel for collapse(2) schedule(static)
    for (long iz = 0; iz < g.nz; ++iz)
      for (long iy = kHalf; iy < g.ny - kHalf; ++iy)
        for (long ix = kHalf; ix < g.nx - kHalf; ++ix) {
          const long ixy = ix + iy * g.nx, i = ixy + iz * nxy;
          const T d = (T)damp.at(ixy, (int)iz);
          T vx = c11[i] * lxy[i] + c13[i] * lz[i] + 2 * u1[i];
          T vz = c13[i] * lxy[i] + c33[i] * lz[i] + 2 * u1[n + i];
          if (dc) {
            vx += dc[i] * bxy[i] + dc[n + i] * bz[i];
            vz += dc[n + i] * bxy[i] + dc[2 * n + i] * bz[i];
          }
          u[i] = d * vx - (2 * d - 1) * u2[i];
          u[n + i] = d * vz - (2 * d - 1) * u2[n + i];
        }
    if (!dc) {
      const T d = (T)damp.at(s.sidx % nxy, (int)(s.sidx / nxy));
      u[s.sidx] += d * (T)(dt2 * wavelet[t - 1]);
      u[n + s.sidx] += d * (T)(dt2 * wavelet[t - 1]);
    }
  }
}

template <typename T>
void exact_record3d(const Geo3& g, const ExactShot& s, const ExactHistory<T>& h, T* trace) {
  const long n = g.nxyz();
  const int st = sampling_step(g.rate, g.dt), nnt = (g.nt - 1) / st + 1, M = last_level(g);
  std::fill(trace, trace + (long)nnt * s.nr, (T)0);
  for (int j = 1; j < nnt; ++j) {
    const int t = exact_level(j, st, M);
    if (!t) continue;
    for (int ir = 0; ir < s.nr; ++ir)
      if (s.live[ir])
        trace[j + (long)ir * nnt] = (T)kTwoThird * h.a[t][s.ridx[ir]] +
                                    (T)kOneThird * h.a[t][n + s.ridx[ir]];
  }
}

// Adds the adjoint-state gradient of sum_j <res_j, d_j> to grad (3n).
template <typename T>
void exact_adjoint3d(const Geo3& g, const T* c11, const T* c13, const T* c33,
                     const ExactShot& s, const Damp3& damp, const ExactHistory<T>& h,
                     const T* res, T* grad) {
  const long n = g.nxyz(), nxy = g.nxy();
  const int st = sampling_step(g.rate, g.dt), nnt = (g.nt - 1) / st + 1, M = last_level(g);
  std::vector<T> mu1(2 * n, 0), mu2(2 * n, 0), mu(2 * n, 0), w(2 * n, 0);
  std::vector<T> lxy(n), lz(n), axy(n), az(n);
  std::vector<T> src(2 * n, 0);
  for (int t = M; t >= 2; --t) {
    // w = C mu_{t+1}; (lxy, lz) = (L_xy w_x, L_z w_z)
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      w[i] = c11[i] * mu1[i] + c13[i] * mu1[n + i];
      w[n + i] = c13[i] * mu1[i] + c33[i] * mu1[n + i];
    }
    lap3d<T>(g, w.data(), w.data() + n, lxy.data(), lz.data());
    std::fill(src.begin(), src.end(), (T)0);
    if (t % st == 0 && t / st < nnt && exact_level(t / st, st, M) == t)
      for (int ir = 0; ir < s.nr; ++ir)
        if (s.live[ir]) {
          const T r = res[t / st + (long)ir * nnt];
          src[s.ridx[ir]] += (T)kTwoThird * r;
          src[n + s.ridx[ir]] += (T)kOneThird * r;
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (long iz = 0; iz < g.nz; ++iz)
      for (long iy = kHalf; iy < g.ny - kHalf; ++iy)
        for (long ix = kHalf; ix < g.nx - kHalf; ++ix) {
          const long ixy = ix + iy * g.nx, i = ixy + iz * nxy;
          const T d = (T)damp.at(ixy, (int)iz);
          mu[i] = d * (src[i] + 2 * mu1[i] + lxy[i]) - (2 * d - 1) * mu2[i];
          mu[n + i] = d * (src[n + i] + 2 * mu1[n + i] + lz[i]) - (2 * d - 1) * mu2[n + i];
        }
    const T* a1 = h.a[t - 1].data();
    lap3d<T>(g, a1, a1 + n, axy.data(), az.data());
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      grad[i] += mu[i] * axy[i];
      grad[n + i] += mu[i] * az[i] + mu[n + i] * axy[i];
      grad[2 * n + i] += mu[n + i] * az[i];
    }
    std::swap(mu2, mu1);
    std::swap(mu1, mu);
  }
}

extern "C" {

// Damping tables of abc3d.cu:23-50 (nx*ny then nz floats).
void orc3d_damping(int nx, int ny, int nz, int npad, float* out) {
  Geo3 g{};
  g.nx = nx; g.ny = ny; g.nz = nz; g.npad = npad;
  Damp3 d(g);
  std::copy(d.xy.begin(), d.xy.end(), out);
  std::copy(d.z.begin(), d.z.end(), out + d.xy.size());
}

int orc3d_last_level(const int* ip, const float* fp) { return last_level(unpack3(ip, fp)); }

#define ORC3D_MODEL(T, SUF)                                                                    \
  int orc3d_model_data_##SUF(const int* ip, const float* fp, const float* c11, const float* c13, \
                             const float* c33, const float* wavelet, const float* souloc,       \
                             const int* shotid, int nshot, const float* recloc, T* ddata,       \
                             T* final_x) {                                                      \
    Geo3 g = unpack3(ip, fp);                                                                   \
    Damp3 damp(g);                                                                              \
    const int nnt = (g.nt - 1) / sampling_step(g.rate, g.dt) + 1;                               \
    std::vector<T> cx, cz, px, pz;                                                              \
    for (int k = 0; k < nshot; ++k) {                                                           \
      Shot3 s = make_shot3(g, souloc, recloc, shotid[k]);                                       \
      forward3d<T>(g, c11, c13, c33, wavelet, s, &damp, ddata + (long)nnt * s.irbegin, cx, cz,  \
                   px, pz);                                                                     \
      if (final_x) std::copy(cx.begin(), cx.end(), final_x);                                    \
    }                                                                                           \
    return 0;                                                                                   \
  }
ORC3D_MODEL(double, f64)
ORC3D_MODEL(float, f32)

#define ORC3D_GRAD(T, SUF)                                                                      \
  int orc3d_gradient_cij_##SUF(const int* ip, const float* fp, const float* cij,                \
                               const float* padb, const float* randb, const float* wavelet,     \
                               const float* souloc, const int* shotid, int nshot,               \
                               const float* recloc, const float* dobs, T* fgcij, int misfit_only, \
                               T* modeled, float tpow, int objtype, int halfwidth) {             \
    Geo3 g = unpack3(ip, fp);                                                                   \
    gradient3d<T>(g, cij, padb, randb, wavelet, souloc, shotid, nshot, recloc, dobs, fgcij,     \
                  misfit_only != 0, modeled, tpow, objtype, halfwidth);                         \
    return 0;                                                                                   \
  }
ORC3D_GRAD(double, f64)
ORC3D_GRAD(float, f32)

#define ORC3D_RTM(T, SUF)                                                                      \
  int orc3d_rtm_##SUF(const int* ip, const float* fp, const float* c11, const float* c13,       \
                      const float* c33, const float* wavelet, const float* souloc,              \
                      const int* shotid, int nshot, const float* recloc, const float* data,     \
                      T* image) {                                                               \
    Geo3 g = unpack3(ip, fp);                                                                   \
    rtm3d<T>(g, c11, c13, c33, wavelet, souloc, shotid, nshot, recloc, data, image);           \
    return 0;                                                                                   \
  }
ORC3D_RTM(double, f64)
ORC3D_RTM(float, f32)

#define ORC3D_ODCIG(T, SUF)                                                                    \
  int orc3d_odcig_##SUF(const int* ip, const float* fp, const float* c11, const float* c13,     \
                        const float* c33, const float* wavelet, const float* souloc,            \
                        const int* shotid, int nshot, const float* recloc, const float* data,   \
                        int nlag, T* image) {                                                   \
    if (nlag < 0) return 1;                                                                     \
    Geo3 g = unpack3(ip, fp);                                                                   \
    rtm3d<T>(g, c11, c13, c33, wavelet, souloc, shotid, nshot, recloc, data, image, nlag);     \
    return 0;                                                                                   \
  }
ORC3D_ODCIG(double, f64)
ORC3D_ODCIG(float, f32)

#define ORC3D_WGRAD(T, SUF)                                                                    \
  int orc3d_wavelet_gradient_##SUF(const int* ip, const float* fp, const float* c11,            \
                                   const float* c13, const float* c33, const float* souloc,     \
                                   const int* shotid, int nshot, const float* recloc,           \
                                   const float* data, T* gw) {                                  \
    Geo3 g = unpack3(ip, fp);                                                                   \
    wavelet_grad3d<T>(g, c11, c13, c33, souloc, shotid, nshot, recloc, data, gw);               \
    return 0;                                                                                   \
  }
ORC3D_WGRAD(double, f64)
ORC3D_WGRAD(float, f32)

// EXACT mode (self-checks, FP64). Traces of the EXACT forward operator.
int orc3d_exact_forward(const int* ip, const float* fp, const double* c11, const double* c13,
                        const double* c33, const float* wavelet, const float* souloc,
                        const int* shotid, int nshot, const float* recloc, double* ddata) {
  Geo3 g = unpack3(ip, fp);
  Damp3 damp(g);
  const int nnt = (g.nt - 1) / sampling_step(g.rate, g.dt) + 1;
  ExactHistory<double> h;
  for (int k = 0; k < nshot; ++k) {
    ExactShot s = exact_shot(g, souloc, recloc, shotid[k]);
    exact_forward3d<double>(g, c11, c13, c33, wavelet, s, damp, h);
    exact_record3d<double>(g, s, h, ddata + (long)nnt * s.irbegin);
  }
  return 0;
}

// Born traces: the derivative of the EXACT traces along dc (3n: dc11,dc13,dc33).
int orc3d_exact_born(const int* ip, const float* fp, const double* c11, const double* c13,
                     const double* c33, const float* wavelet, const float* souloc,
                     const int* shotid, int nshot, const float* recloc, const double* dc,
                     double* ddata) {
  Geo3 g = unpack3(ip, fp);
  Damp3 damp(g);
  const int nnt = (g.nt - 1) / sampling_step(g.rate, g.dt) + 1;
  ExactHistory<double> bg, h;
  for (int k = 0; k < nshot; ++k) {
    ExactShot s = exact_shot(g, souloc, recloc, shotid[k]);
    exact_forward3d<double>(g, c11, c13, c33, wavelet, s, damp, bg);
    exact_forward3d<double>(g, c11, c13, c33, wavelet, s, damp, h, &bg, dc);
    exact_record3d<double>(g, s, h, ddata + (long)nnt * s.irbegin);
  }
  return 0;
}

// Adjoint of the Born operator applied to traces `res` (grad: 3n, overwritten).
// With res = modeled - observed it is the gradient of the EXACT misfit.
int orc3d_exact_adjoint(const int* ip, const float* fp, const double* c11, const double* c13,
                        const double* c33, const float* wavelet, const float* souloc,
                        const int* shotid, int nshot, const float* recloc, const double* res,
                        double* grad) {
  Geo3 g = unpack3(ip, fp);
  Damp3 damp(g);
  const int nnt = (g.nt - 1) / sampling_step(g.rate, g.dt) + 1;
  std::fill(grad, grad + 3 * g.nxyz(), 0.0);
  ExactHistory<double> h;
  for (int k = 0; k < nshot; ++k) {
    ExactShot s = exact_shot(g, souloc, recloc, shotid[k]);
    exact_forward3d<double>(g, c11, c13, c33, wavelet, s, damp, h);
    exact_adjoint3d<double>(g, c11, c13, c33, s, damp, h, res + (long)nnt * s.irbegin, grad);
  }
  return 0;
}

// Time `nsteps` forward steps (forward form, sponge) of a zero-initialised
// grid with a point source: the FP32 instance is the CPU baseline's unit of
// work. Returns the number of threads used.
int orc3d_time_forward_f32(const int* ip, const float* fp, const float* c11, const float* c13,
                           const float* c33, int nsteps, float* scratch4) {
  Geo3 g = unpack3(ip, fp);
  Damp3 damp(g);
  const long n = g.nxyz();
  float *cx = scratch4, *cz = cx + n, *px = cz + n, *pz = px + n;
  for (int it = 0; it < nsteps; ++it) {
    step3d<float, true>(g, c11, c13, c33, cx, cz, px, pz, &damp, nullptr, nullptr, nullptr,
                        nullptr, nullptr);
    std::swap(cx, px);
    std::swap(cz, pz);
  }
  return omp_get_max_threads();
}

// Time `nsteps` of the fused backward work (sigma back-step + imaging +
// adjoint step with sponge), FP32.
int orc3d_time_backward_f32(const int* ip, const float* fp, const float* c11, const float* c13,
                            const float* c33, int nsteps, float* scratch11) {
  Geo3 g = unpack3(ip, fp);
  Damp3 damp(g);
  const long n = g.nxyz();
  float *cx = scratch11, *cz = cx + n, *px = cz + n, *pz = px + n;
  float *lx = pz + n, *lz = lx + n, *lpx = lz + n, *lpz = lpx + n;
  float *g11 = lpz + n, *g13 = g11 + n, *g33 = g13 + n;
  for (int it = 0; it < nsteps; ++it) {
    step3d<float, false>(g, c11, c13, c33, cx, cz, px, pz, nullptr, lx, lz, g11, g13, g33);
    step3d<float, true>(g, c11, c13, c33, lx, lz, lpx, lpz, &damp, nullptr, nullptr, nullptr,
                        nullptr, nullptr);
    std::swap(cx, px); std::swap(cz, pz);
    std::swap(lx, lpx); std::swap(lz, lpz);
  }
  return omp_get_max_threads();
}

// OpenMP threads the oracle's parallel loops use.
int orc_max_threads() { return omp_get_max_threads(); }

#define ORC2D_FWD(T, SUF)                                                                      \
  int orc2d_forward_##SUF(const int* ip, const float* fp, const float* c11, const float* c13,   \
                          const float* c33, const float* wavelet, const int* sloc, int ns,      \
                          const int* rloc, int nr, const float* taper, T* out, int mode) {      \
    Geo2 g = unpack2(ip, fp);                                                                   \
    for (int is = 0; is < (mode == 0 ? ns : 1); ++is)                                           \
      forward2d<T>(g, c11, c13, c33, wavelet, sloc, is, rloc, nr, taper, out, mode);            \
    return 0;                                                                                   \
  }
ORC2D_FWD(double, f64)
ORC2D_FWD(float, f32)

// objFuncGradient_f (born = 0, dc = NULL) / GNhessian_f (born = 1).
#define ORC2D_GRAD(T, SUF)                                                                      \
  double orc2d_gradient_##SUF(const int* ip, const float* fp, const float* c11, const float* c13, \
                              const float* c33, const float* dc11, const float* dc13,           \
                              const float* dc33, const float* wavelet, const int* sloc, int ns,  \
                              const int* rloc, int nr, const float* taper, const float* data,    \
                              T* g11, T* g13, T* g33, int born) {                                \
    Geo2 g = unpack2(ip, fp);                                                                   \
    return grad2d<T>(g, c11, c13, c33, dc11, dc13, dc33, wavelet, sloc, ns, rloc, nr, taper,    \
                     data, g11, g13, g33, born != 0);                                           \
  }
ORC2D_GRAD(double, f64)
ORC2D_GRAD(float, f32)

#define ORC2D_RTM(T, SUF)                                                                       \
  int orc2d_rtm_##SUF(const int* ip, const float* fp, const float* c11, const float* c13,        \
                      const float* c33, const float* wavelet, const float* data,                 \
                      const int* sloc, int ns, const int* rloc, int nr, const float* taper,      \
                      T* image) {                                                                \
    Geo2 g = unpack2(ip, fp);                                                                    \
    rtm2d<T>(g, c11, c13, c33, wavelet, data, sloc, ns, rloc, nr, taper, image);                 \
    return 0;                                                                                    \
  }
ORC2D_RTM(double, f64)
ORC2D_RTM(float, f32)

#define ORC2D_ODCIG(T, SUF)                                                                     \
  int orc2d_odcig_##SUF(const int* ip, const float* fp, int nhx, const float* c11,               \
                        const float* c13, const float* c33, const float* wavelet,                \
                        const float* data, const int* sloc, int ns, const int* rloc, int nr,     \
                        const float* taper, T* image) {                                          \
    Geo2 g = unpack2(ip, fp);                                                                    \
    rtm2d<T>(g, c11, c13, c33, wavelet, data, sloc, ns, rloc, nr, taper, image, nhx);            \
    return 0;                                                                                    \
  }
ORC2D_ODCIG(double, f64)
ORC2D_ODCIG(float, f32)

#define ORC2D_WGRAD(T, SUF)                                                                     \
  int orc2d_wavelet_gradient_##SUF(const int* ip, const float* fp, const float* c11,             \
                                   const float* c13, const float* c33, const float* data,        \
                                   const int* sloc, int ns, const int* rloc, int nr,             \
                                   const float* taper, T* gw) {                                  \
    Geo2 g = unpack2(ip, fp);                                                                    \
    wavelet_grad2d<T>(g, c11, c13, c33, data, sloc, ns, rloc, nr, taper, gw);                    \
    return 0;                                                                                    \
  }
ORC2D_WGRAD(double, f64)
ORC2D_WGRAD(float, f32)

// The checkpoint pairing of the 2D gradient: 3 values (a, b, f) per imaging
// step, nt-1 steps. Returns the number of steps.
int orc2d_checkpoint_schedule(int nt, int ratio, float* out) {
  std::vector<Pair> s = checkpoint_schedule(nt, ratio);  // first shot
  for (size_t k = 0; k < s.size(); ++k) {
    out[3 * k] = (float)s[k].a;
    out[3 * k + 1] = (float)s[k].b;
    out[3 * k + 2] = s[k].f;
  }
  return (int)s.size();
}

}  // extern "C"
