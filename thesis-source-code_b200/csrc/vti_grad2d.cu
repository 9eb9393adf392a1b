// 2D adjoint gradient (objFuncGradient_f, lib/vti-fwi-2d/objFuncGradient_f.cu:15-371)
// and Gauss-Newton Hessian-vector product (GNhessian_f, hessian_f.cu:575-1010)
// for sm_100a.
//
// Forward: one fused kernel per level (background; with the Born field and
// its scattering source for the GN product), checkpoints D(sigma) = (Dxx p,
// Dzz q) of the levels the backward pass reads, kept on the device.
// Backward: one fused kernel per level: adjoint step (backwardDC, the exact
// adjoint D(C lambda), for the gradient; forwardCD for the GN product), taper,
// and the zero-lag imaging of the current adjoint against the interpolated
// checkpoint pair. Which checkpoint pair each level is imaged with follows the
// reference's buffer rotation, replayed on the host (checkpoint_schedule).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

#include "vti_internal.h"

namespace vti {
namespace {

constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;
constexpr int BX = 32, BZ = 8;

__device__ __forceinline__ float lap9(const float* r, int s) {
  float v = kC0 * r[0];
  v = fmaf(kC1, r[-s] + r[s], v);
  v = fmaf(kC2, r[-2 * s] + r[2 * s], v);
  v = fmaf(kC3, r[-3 * s] + r[3 * s], v);
  v = fmaf(kC4, r[-4 * s] + r[4 * s], v);
  return v;
}

struct Grid2 {
  int nnx, nnz;
};

// Forward level of the background (and Born) field, forwardC semantics
// (kernels.cu:546-556, scattering :282-291), taper of cur and next
// (kernels.cu:304-315) folded as in the forward-modeling kernel.
struct Fwd2 {
  Grid2 g;
  const float *p1, *q1;
  float *p0, *q0;
  const float *dp1, *dq1;  // Born (null: background only)
  float *dp0, *dq0;
  const float *c11, *c13, *c33, *dc11, *dc13, *dc33, *taper;
  float idx2, idz2, dt2;
  int src;
  float amp;
  // when set, the Born stencil reads these D values instead of D(dp1): the
  // reference never clears its Born D buffer between shots (hessian_f.cu)
  const float *bdp, *bdq;
  // non-null: store D of the current level (k_dop2d's checkpoint of level
  // it-1, the same expressions as tp / tq below)
  float *ckp, *ckq;
  // receiver of each cell (-1: none); with rec_row >= 0 the new level
  // (Born field for the Gauss-Newton product) is recorded into that row
  const int* rmap;
  float* rec;
  int rec_row, nri;
};

// injectData value of one receiver (kernels.cu:208-217): dt2 times half
// the residual interpolated between rows b0 and b1.
__device__ __forceinline__ float inject_value(const float* b0, const float* b1, int ir, float f,
                                              float dt2) {
  const float s = 0.5f * __fadd_rn(__fmul_rn(1.f - f, b0[ir]), __fmul_rn(f, b1[ir]));
  return __fmul_rn(dt2, s);
}

__global__ void __launch_bounds__(BX* BZ) k_fwd2d(Fwd2 a) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  __shared__ float sp[BZ][BX + 8], sq[BZ + 8][BX];
  __shared__ float sdp[BZ][BX + 8], sdq[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx, iz = kHalo + blockIdx.y * BZ + tz;
  const int nnx = a.g.nnx, nnz = a.g.nnz;
  const bool born = a.dp1 != nullptr;
  auto ld = [&](const float* f, int x, int z) {
    return (x < nnx && z < nnz) ? f[x + z * nnx] : 0.f;
  };
  sp[tz][tx + 4] = ld(a.p1, ix, iz);
  sq[tz + 4][tx] = ld(a.q1, ix, iz);
  if (tx < 4) {
    sp[tz][tx] = ld(a.p1, ix - 4, iz);
    sp[tz][tx + BX + 4] = ld(a.p1, ix + BX, iz);
  }
  if (tz < 4) {
    sq[tz][tx] = ld(a.q1, ix, iz - 4);
    sq[tz + BZ + 4][tx] = ld(a.q1, ix, iz + BZ);
  }
  if (born) {
    sdp[tz][tx + 4] = ld(a.dp1, ix, iz);
    sdq[tz + 4][tx] = ld(a.dq1, ix, iz);
    if (tx < 4) {
      sdp[tz][tx] = ld(a.dp1, ix - 4, iz);
      sdp[tz][tx + BX + 4] = ld(a.dp1, ix + BX, iz);
    }
    if (tz < 4) {
      sdq[tz][tx] = ld(a.dq1, ix, iz - 4);
      sdq[tz + BZ + 4][tx] = ld(a.dq1, ix, iz + BZ);
    }
  }
  __syncthreads();
  if (!(ix < nnx - kHalo && iz < nnz - kHalo)) return;
  const int i = ix + iz * nnx;
  const float tp = lap9(&sp[tz][tx + 4], 1) * a.idx2;
  const float tq = lap9(&sq[tz + 4][tx], BX) * a.idz2;
  if (a.ckp) {
    a.ckp[i] = tp;
    a.ckq[i] = tq;
  }
  const float t = a.taper[i];
  const float c11 = a.c11[i], c13 = a.c13[i], c33 = a.c33[i];
  float pn = fmaf(a.dt2, fmaf(c11, tp, c13 * tq), 2.f * sp[tz][tx + 4] - t * a.p0[i]);
  float qn = fmaf(a.dt2, fmaf(c13, tp, c33 * tq), 2.f * sq[tz + 4][tx] - t * a.q0[i]);
  if (i == a.src) {
    pn += a.amp;
    qn += a.amp;
  }
  // the stored products, rounded before they are recorded (no contraction)
  const float pv = __fmul_rn(t, pn), qv = __fmul_rn(t, qn);
  a.p0[i] = pv;
  a.q0[i] = qv;
  const int ir = (a.rec_row >= 0 && !born) ? a.rmap[i] : -1;
  if (ir >= 0) a.rec[(long long)a.rec_row * a.nri + ir] = 0.5f * (pv + qv);
  if (born) {
    const float dtp = a.bdp ? a.bdp[i] : lap9(&sdp[tz][tx + 4], 1) * a.idx2;
    const float dtq = a.bdq ? a.bdq[i] : lap9(&sdq[tz + 4][tx], BX) * a.idz2;
    float dpn = fmaf(a.dt2, fmaf(c11, dtp, c13 * dtq), 2.f * sdp[tz][tx + 4] - t * a.dp0[i]);
    float dqn = fmaf(a.dt2, fmaf(c13, dtp, c33 * dtq), 2.f * sdq[tz + 4][tx] - t * a.dq0[i]);
    dpn = fmaf(a.dt2, fmaf(a.dc11[i], tp, a.dc13[i] * tq), dpn);
    dqn = fmaf(a.dt2, fmaf(a.dc13[i], tp, a.dc33[i] * tq), dqn);
    const float dpv = __fmul_rn(t, dpn), dqv = __fmul_rn(t, dqn);
    a.dp0[i] = dpv;
    a.dq0[i] = dqv;
    const int irb = a.rec_row >= 0 ? a.rmap[i] : -1;
    if (irb >= 0) a.rec[(long long)a.rec_row * a.nri + irb] = 0.5f * (dpv + dqv);
  }
}

// D kernel (kernels.cu:345-387): checkpoint of (Dxx p / dx2, Dzz q / dz2).
__global__ void __launch_bounds__(BX* BZ) k_dop2d(Grid2 g, const float* p, const float* q,
                                                  float* tp, float* tq, float idx2, float idz2) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  __shared__ float sp[BZ][BX + 8], sq[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx, iz = kHalo + blockIdx.y * BZ + tz;
  auto ld = [&](const float* f, int x, int z) {
    return (x < g.nnx && z < g.nnz) ? f[x + z * g.nnx] : 0.f;
  };
  sp[tz][tx + 4] = ld(p, ix, iz);
  sq[tz + 4][tx] = ld(q, ix, iz);
  if (tx < 4) {
    sp[tz][tx] = ld(p, ix - 4, iz);
    sp[tz][tx + BX + 4] = ld(p, ix + BX, iz);
  }
  if (tz < 4) {
    sq[tz][tx] = ld(q, ix, iz - 4);
    sq[tz + BZ + 4][tx] = ld(q, ix, iz + BZ);
  }
  __syncthreads();
  if (!(ix < g.nnx - kHalo && iz < g.nnz - kHalo)) return;
  const int i = ix + iz * g.nnx;
  tp[i] = lap9(&sp[tz][tx + 4], 1) * idx2;
  tq[i] = lap9(&sq[tz + 4][tx], BX) * idz2;
}

// Backward level: adjoint step, taper, imaging of the current adjoint.
struct Adj2 {
  Grid2 g;
  const float *p0, *q0;  // current adjoint (lambda at it+2)
  float *p1, *q1;        // prev in / next out
  const float *c11, *c13, *c33, *taper;
  float idx2, idz2, dt2;
  int exact;             // 1: backwardDC (D C lambda); 0: forwardCD (C D lambda)
  // imaging of p0,q0 against (1-f) D_a + f D_b (null pointer: zero buffer)
  const float *ap, *aq, *bp, *bq;
  float f;
  int image;
  float *g11, *g13, *g33;
  // receiver of each cell (-1: none); with inject, the residual rows b0/b1
  // interpolated at fi are injected into the new level (k_inject2d, scaled)
  const int* rmap;
  const float *b0, *b1;
  float fi;
  int inject;
};

__global__ void __launch_bounds__(BX* BZ) k_adj2d(Adj2 a) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  __shared__ float su[BZ][BX + 8], sw[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx, iz = kHalo + blockIdx.y * BZ + tz;
  const int nnx = a.g.nnx, nnz = a.g.nnz;
  // u = c11 p + c13 q along x, w = c13 p + c33 q along z (exact adjoint);
  // the plain fields for forwardCD
  auto U = [&](int x, int z) -> float {
    if (!(x < nnx && z < nnz)) return 0.f;
    int k = x + z * nnx;
    return a.exact ? a.c11[k] * a.p0[k] + a.c13[k] * a.q0[k] : a.p0[k];
  };
  auto W = [&](int x, int z) -> float {
    if (!(x < nnx && z < nnz)) return 0.f;
    int k = x + z * nnx;
    return a.exact ? a.c13[k] * a.p0[k] + a.c33[k] * a.q0[k] : a.q0[k];
  };
  su[tz][tx + 4] = U(ix, iz);
  sw[tz + 4][tx] = W(ix, iz);
  if (tx < 4) {
    su[tz][tx] = U(ix - 4, iz);
    su[tz][tx + BX + 4] = U(ix + BX, iz);
  }
  if (tz < 4) {
    sw[tz][tx] = W(ix, iz - 4);
    sw[tz + BZ + 4][tx] = W(ix, iz + BZ);
  }
  __syncthreads();
  if (!(ix < nnx - kHalo && iz < nnz - kHalo)) return;
  const int i = ix + iz * nnx;
  const float p = a.p0[i], q = a.q0[i];
  if (a.image) {  // gradientCrossCor (kernels.cu:438-450)
    const float f = a.f;
    const float Dp = (1.f - f) * (a.ap ? a.ap[i] : 0.f) + f * (a.bp ? a.bp[i] : 0.f);
    const float Dq = (1.f - f) * (a.aq ? a.aq[i] : 0.f) + f * (a.bq ? a.bq[i] : 0.f);
    a.g11[i] += p * Dp;
    a.g13[i] += p * Dq + q * Dp;
    a.g33[i] += q * Dq;
  }
  if (!a.p1) return;  // imaging only
  const float tp = lap9(&su[tz][tx + 4], 1) * a.idx2;
  const float tq = lap9(&sw[tz + 4][tx], BX) * a.idz2;
  const float t = a.taper[i];
  float pn, qn;
  if (a.exact) {
    pn = fmaf(a.dt2, tp, 2.f * p - t * a.p1[i]);
    qn = fmaf(a.dt2, tq, 2.f * q - t * a.q1[i]);
  } else {
    pn = fmaf(a.dt2, fmaf(a.c11[i], tp, a.c13[i] * tq), 2.f * p - t * a.p1[i]);
    qn = fmaf(a.dt2, fmaf(a.c13[i], tp, a.c33[i] * tq), 2.f * q - t * a.q1[i]);
  }
  // the stored products, rounded before the injection adds to them (the
  // arithmetic of a store followed by k_inject2d)
  float pv = __fmul_rn(t, pn), qv = __fmul_rn(t, qn);
  const int ir = a.inject ? a.rmap[i] : -1;
  if (ir >= 0) {
    const float v = __fmul_rn(inject_value(a.b0, a.b1, ir, a.fi, a.dt2), t);
    pv += v;
    qv += v;
  }
  a.p1[i] = pv;
  a.q1[i] = qv;
}

// injectData (kernels.cu:208-217) into a tapered level: taper factor applied.
__global__ void k_inject2d(float* p, float* q, const float* b0, const float* b1, float f,
                           const int* ridx, const float* taper, int nr, float dt2, int scale) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    const int i = ridx[ir];
    float v = inject_value(b0, b1, ir, f, dt2);
    if (scale) v = __fmul_rn(v, taper[i]);
    p[i] += v;
    q[i] += v;
  }
}

__global__ void k_record_rows(float* rec, int row, const float* p, const float* q,
                              const int* ridx, int nr) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    int i = ridx[ir];
    rec[(long long)row * nr + ir] = 0.5f * (p[i] + q[i]);
  }
}

__global__ void k_set2(float* a, float* b, int i, float v) {
  // launched as programmatic dependents (launch_pdl): wait for the previous
  // kernel of the stream before touching anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  a[i] = v;
  b[i] = v;
}

struct Pair {
  long a, b;  // checkpoint labels, shot*(nt+1)+t; -1: zero buffer
  float f;
};

// Replays the reference's checkpoint copies (forward objFuncGradient_f.cu:182-202,
// backward :240-292; hessian_f.cu the same). The device buffers Dpq/Dpqa/Dpqb,
// the pinned host pair and the host array Dp[] are cleared once, not per
// shot, so the state carries from shot to shot on the same GPU.
struct CkState {
  long dq = -1, da = -1, db = -1, ha = -1, hb = -1;
  std::vector<long> Dp;
};
std::vector<Pair> checkpoint_shot(CkState& S, int shot, int nt, int r) {
  const int nnt = (nt - 1) / r + 1;
  auto L = [&](int t) { return (long)shot * (nt + 1) + t; };
  if (S.Dp.empty()) S.Dp.assign(std::max(nnt, 1), -1);
  S.dq = L(1);
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

struct Buf {
  float* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
};

int run_grad2d(vti_ctx* ctx, const vti2d_geom* g, float* gc11, float* gc13, float* gc33,
               const float* data, const float* c11, const float* c13, const float* c33,
               const float* dc11, const float* dc13, const float* dc33, const float* wavelet,
               const int* sloc, int ns, const int* rloc, int nr, const float* taper,
               double* misfit, bool born) {
  if (!ctx || !g || !gc11 || !gc13 || !gc33 || !c11 || !c13 || !c33 || !wavelet || !sloc ||
      !taper || (!born && !data) || (born && (!dc11 || !dc13 || !dc33)))
    return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5f);
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  if (nnx < 9 || nnz < 9 || ratio < 1 || g->nt < 3 || (g->nt - 1) / ratio + 1 < 3)
    return fail(ctx, VTI_ERR_ARG, "2D gradient needs nt >= 2*ratio+1 and a grid of 9x9 or more");
  const int nnt_data = (g->nt - ntNeg - 1) / ratio + 1;
  if (nnt_data < 1)
    return fail(ctx, VTI_ERR_ARG, "the whole record lies before time zero (|ot| too large)");
  {
    const int cst = check_cfl2d(ctx, g, c11, c13, c33);
    if (cst != VTI_OK) return cst;
  }
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<std::vector<Pair>> sched(ns);
  {
    CkState S;
    for (int is = 0; is < ns; ++is) sched[is] = checkpoint_shot(S, is, g->nt, ratio);
  }
  std::map<long, int> slot;  // checkpoint label -> device slot
  for (const auto& v : sched)
    for (const Pair& p : v) {
      if (p.a >= 0 && !slot.count(p.a)) slot[p.a] = (int)slot.size();
      if (p.b >= 0 && !slot.count(p.b)) slot[p.b] = (int)slot.size();
    }
  const int nslot = (int)slot.size();
  // device memory: model 3 (+3 dc) + taper + 4 fields (+4 Born) + 3 gradients
  // + 2 D buffers per checkpoint
  const size_t nfield = 3 + (born ? 3 : 0) + 1 + 4 + (born ? 4 : 0) + 3 + 2 + (born ? 2 : 0);
  Buf all;
  VTI_CUDA(ctx, cudaMalloc((void**)&all.p, (nfield + 2 * (size_t)nslot) * nnxz * sizeof(float)));
  float* cur = all.p;
  auto take = [&]() {
    float* r = cur;
    cur += nnxz;
    return r;
  };
  float *d11 = take(), *d13 = take(), *d33 = take();
  float *e11 = born ? take() : nullptr, *e13 = born ? take() : nullptr,
        *e33 = born ? take() : nullptr;
  float* tap = take();
  float *p0 = take(), *q0 = take(), *p1 = take(), *q1 = take();
  float *dp0 = born ? take() : nullptr, *dq0 = born ? take() : nullptr;
  float *dp1 = born ? take() : nullptr, *dq1 = born ? take() : nullptr;
  float *g11 = take(), *g13 = take(), *g33 = take();
  float *tmpp = take(), *tmpq = take();
  // D of the last Born level of the previous shot (hessian_f.cu never
  // re-zeroes d_Ddpq)
  float *stale_p = born ? take() : nullptr, *stale_q = born ? take() : nullptr;
  float* ck = cur;
  auto ckp = [&](long label) {
    return label < 0 ? nullptr : ck + (size_t)(2 * slot[label]) * nnxz;
  };
  auto ckq = [&](long label) {
    return label < 0 ? nullptr : ck + (size_t)(2 * slot[label] + 1) * nnxz;
  };
  cudaStream_t s = ctx->stream;
  VTI_CUDA(ctx, cudaMemcpyAsync(d11, c11, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(d13, c13, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(d33, c33, nnxz * 4, cudaMemcpyHostToDevice, s));
  if (born) {
    VTI_CUDA(ctx, cudaMemcpyAsync(e11, dc11, nnxz * 4, cudaMemcpyHostToDevice, s));
    VTI_CUDA(ctx, cudaMemcpyAsync(e13, dc13, nnxz * 4, cudaMemcpyHostToDevice, s));
    VTI_CUDA(ctx, cudaMemcpyAsync(e33, dc33, nnxz * 4, cudaMemcpyHostToDevice, s));
  }
  VTI_CUDA(ctx, cudaMemcpyAsync(tap, taper, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemsetAsync(g11, 0, 3 * nnxz * 4, s));
  VTI_CUDA(ctx, cudaMemsetAsync(ck, 0, 2 * (size_t)nslot * nnxz * 4, s));
  const Grid2 G{nnx, nnz};
  const dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  const float idx2 = 1.f / (g->dx * g->dx), idz2 = 1.f / (g->dz * g->dz);
  double* d_acc = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&d_acc, (1 + residual_blocks(ctx)) * sizeof(double)));
  Buf accbuf;
  accbuf.p = (float*)d_acc;
  VTI_CUDA(ctx, cudaMemsetAsync(d_acc, 0, sizeof(double), s));
  for (int is = 0; is < ns; ++is) {
    const int* sl = sloc + 4 * is;
    const int sxz = sl[0] + sl[1] * nnx, nri = sl[2], ir0 = sl[3];
    if (sxz < 0 || sxz >= nnxz || nri < 0 || ir0 < 0 || ir0 + nri > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot outside the grid or receiver range");
    std::vector<int> ridx(std::max(nri, 1));
    for (int ir = 0; ir < nri; ++ir) {
      int x = rloc[2 * (ir0 + ir)], z = rloc[2 * (ir0 + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz)
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
      ridx[ir] = x + z * nnx;
    }
    Buf rb, recb, obsb, live, b01, rmapb;
    VTI_CUDA(ctx, cudaMalloc((void**)&rb.p, ridx.size() * sizeof(int)));
    VTI_CUDA(ctx, cudaMemcpyAsync(rb.p, ridx.data(), ridx.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, s));
    // receiver of each cell: the step kernels record and inject themselves
    // (one launch per level instead of two); a cell holding two receivers
    // keeps the separate receiver kernels
    std::vector<int> rmh;
    bool fuse = nri > 0;
    if (fuse) {
      rmh.assign(nnxz, -1);
      for (int ir = 0; ir < nri && fuse; ++ir) {
        if (rmh[ridx[ir]] >= 0) fuse = false;
        rmh[ridx[ir]] = ir;
      }
    }
    if (fuse) {
      VTI_CUDA(ctx, cudaMalloc((void**)&rmapb.p, nnxz * sizeof(int)));
      VTI_CUDA(ctx, cudaMemcpyAsync(rmapb.p, rmh.data(), nnxz * sizeof(int),
                                    cudaMemcpyHostToDevice, s));
    }
    const int* d_rmap = fuse ? (const int*)rmapb.p : nullptr;
    const size_t nrec = (size_t)nnt_data * std::max(nri, 1);
    VTI_CUDA(ctx, cudaMalloc((void**)&recb.p, nrec * sizeof(float)));
    VTI_CUDA(ctx, cudaMemsetAsync(recb.p, 0, nrec * sizeof(float), s));
    VTI_CUDA(ctx, cudaMalloc((void**)&b01.p, 2 * std::max(nri, 1) * sizeof(float)));
    const int* d_ridx = (const int*)rb.p;
    // ---- forward
    VTI_CUDA(ctx, cudaMemsetAsync(p0, 0, 4 * nnxz * 4, s));
    if (born) VTI_CUDA(ctx, cudaMemsetAsync(dp0, 0, 4 * nnxz * 4, s));
    float *P0 = p0, *Q0 = q0, *P1 = p1, *Q1 = q1;
    float *DP0 = dp0, *DQ0 = dq0, *DP1 = dp1, *DQ1 = dq1;
    VTI_CUDA(ctx, launch_pdl(k_set2, dim3(1), dim3(1), s, P1, Q1, sxz,
                             dt2 * wavelet[0]));  // no taper at level 1
    ctx->launches++;
    auto checkpoint = [&](int t, const float* p, const float* q) -> cudaError_t {
      const long label = (long)is * (g->nt + 1) + t;
      if (!slot.count(label)) return cudaSuccess;
      ctx->launches++;
      return launch_pdl(k_dop2d, grid, block, s, G, p, q, ckp(label), ckq(label), idx2, idz2);
    };
    for (int it = 2; it < g->nt; ++it) {
      const float t = it * dt + g->ot;
      Fwd2 a{G,   P1,  Q1,  P0,  Q0,   DP1,  DQ1, DP0, DQ0, d11, d13, d33, e11,
             e13, e33, tap, idx2, idz2, dt2, sxz, dt2 * wavelet[it - 1], nullptr, nullptr};
      if (!born) a.dp1 = a.dq1 = a.dp0 = a.dq0 = nullptr;
      if (born && it == 2 && is > 0) {
        a.bdp = stale_p;
        a.bdq = stale_q;
      }
      // the checkpoint of the current level it-1 (k_dop2d's D of P1, Q1)
      {
        const long label = (long)is * (g->nt + 1) + (it - 1);
        a.ckp = slot.count(label) ? ckp(label) : nullptr;
        a.ckq = slot.count(label) ? ckq(label) : nullptr;
      }
      const bool record = t >= 0.f && (it - ntNeg) % ratio == 0 && nri > 0;
      a.rmap = d_rmap;
      a.rec = recb.p;
      a.rec_row = (fuse && record) ? (it - ntNeg) / ratio : -1;
      a.nri = nri;
      VTI_CUDA(ctx, launch_pdl(k_fwd2d, grid, block, s, a));
      ctx->launches++;
      if (record && !fuse) {
        VTI_CUDA(ctx, launch_pdl(k_record_rows, dim3((nri + 127) / 128), dim3(128), s, recb.p,
                                 (it - ntNeg) / ratio, (const float*)(born ? DP0 : P0),
                                 (const float*)(born ? DQ0 : Q0), d_ridx, nri));
        ctx->launches++;
      }
      std::swap(P0, P1);
      std::swap(Q0, Q1);
      std::swap(DP0, DP1);
      std::swap(DQ0, DQ1);
    }
    // the last level has no next step to carry its checkpoint
    VTI_CUDA(ctx, checkpoint(g->nt - 1, P1, Q1));
    if (born) {  // D of the last Born level, read by the next shot's first step
      VTI_CUDA(ctx, launch_pdl(k_dop2d, grid, block, s, G, (const float*)DP1,
                               (const float*)DQ1, stale_p, stale_q, idx2, idz2));
      ctx->launches++;
    }
    if (!born && nri > 0) {
      // residual and FP64 misfit (objFuncGradient_f.cu:214-219)
      VTI_CUDA(ctx, cudaMalloc((void**)&obsb.p, nrec * sizeof(float)));
      VTI_CUDA(ctx, cudaMemcpy2DAsync(obsb.p, nri * sizeof(float), data + ir0,
                                      (size_t)nr * sizeof(float), nri * sizeof(float), nnt_data,
                                      cudaMemcpyHostToDevice, s));
      // launch_residual walks [row][receiver] with one "live" flag per row
      VTI_CUDA(ctx, cudaMalloc((void**)&live.p, nnt_data));
      VTI_CUDA(ctx, cudaMemsetAsync(live.p, 1, nnt_data, s));
      int st = launch_residual(ctx, recb.p, obsb.p, (const unsigned char*)live.p, nri, nnt_data,
                               d_acc);
      if (st != VTI_OK) return st;
    }
    // ---- backward
    VTI_CUDA(ctx, cudaMemsetAsync(p0, 0, 4 * nnxz * 4, s));
    P0 = p0; Q0 = q0; P1 = p1; Q1 = q1;
    // the two trace rows interpolated between (injectData): pointers into the
    // recorded rows, starting with the last row and a row of zeros
    VTI_CUDA(ctx, cudaMemsetAsync(b01.p, 0, std::max(nri, 1) * sizeof(float), s));
    const float* b0 = recb.p + (size_t)(nnt_data - 1) * std::max(nri, 1);
    const float* b1 = b01.p;
    if (nri > 0) {
      VTI_CUDA(ctx, launch_pdl(k_inject2d, dim3((nri + 127) / 128), dim3(128), s, P0, Q0, b0,
                               b1, 0.f, d_ridx, (const float*)tap, nri, dt2, 0));
      ctx->launches++;
    }
    int step = 0;  // sched[step] images the current adjoint
    for (int it = g->nt - 3; it >= 0; --it, ++step) {
      const Pair& pr = sched[is][step];
      // the residual rows injected into the new level (injectData), chosen
      // before the step
      const bool inject = it >= ntNeg && nri > 0;
      float fi = 0.f;
      if (inject) {
        float f = (it - ntNeg + 1.) / ratio;
        int i1 = (int)f;
        if ((it - ntNeg + 2) % ratio == 0) {  // row i1 enters, the older row leaves
          b1 = recb.p + (size_t)i1 * nri;
          std::swap(b0, b1);
        }
        fi = f - i1;
      }
      Adj2 a{G,      P0,  Q0,  P1,  Q1,  d11, d13, d33, tap,  idx2, idz2, dt2, born ? 0 : 1,
             ckp(pr.a), ckq(pr.a), ckp(pr.b), ckq(pr.b), pr.f, 1, g11, g13, g33};
      a.rmap = d_rmap;
      a.b0 = b0;
      a.b1 = b1;
      a.fi = fi;
      a.inject = (inject && fuse) ? 1 : 0;
      VTI_CUDA(ctx, launch_pdl(k_adj2d, grid, block, s, a));
      ctx->launches++;
      if (inject && !fuse) {
        VTI_CUDA(ctx, launch_pdl(k_inject2d, dim3((nri + 127) / 128), dim3(128), s, P1, Q1, b0,
                                 b1, fi, d_ridx, (const float*)tap, nri, dt2, 1));
        ctx->launches++;
      }
      std::swap(P0, P1);
      std::swap(Q0, Q1);
    }
    {  // imaging of the last adjoint level
      const Pair& pr = sched[is][step];
      Adj2 a{G,      P0,  Q0,  nullptr, nullptr, d11, d13, d33, tap,  idx2, idz2, dt2, 1,
             ckp(pr.a), ckq(pr.a), ckp(pr.b), ckq(pr.b), pr.f, 1, g11, g13, g33};
      VTI_CUDA(ctx, launch_pdl(k_adj2d, grid, block, s, a));
      ctx->launches++;
    }
    VTI_CUDA(ctx, cudaGetLastError());
    VTI_CUDA(ctx, cudaStreamSynchronize(s));  // per-shot host vectors
  }
  (void)tmpp;
  (void)tmpq;
  VTI_CUDA(ctx, cudaMemcpyAsync(gc11, g11, nnxz * 4, cudaMemcpyDeviceToHost, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(gc13, g13, nnxz * 4, cudaMemcpyDeviceToHost, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(gc33, g33, nnxz * 4, cudaMemcpyDeviceToHost, s));
  double acc = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&acc, d_acc, sizeof(double), cudaMemcpyDeviceToHost, s));
  VTI_CUDA(ctx, cudaStreamSynchronize(s));
  if (misfit) *misfit = 0.5 * acc;
  return VTI_OK;
}

}  // namespace
}  // namespace vti

extern "C" {

int vti2d_gradient(vti_ctx* ctx, const vti2d_geom* g, float* gc11, float* gc13, float* gc33,
                   const float* data, const float* c11, const float* c13, const float* c33,
                   const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                   const float* taper, double* misfit) {
  return vti::run_grad2d(ctx, g, gc11, gc13, gc33, data, c11, c13, c33, nullptr, nullptr, nullptr,
                         wavelet, sloc, ns, rloc, nr, taper, misfit, false);
}

int vti2d_gn_hessian(vti_ctx* ctx, const vti2d_geom* g, float* gc11, float* gc13, float* gc33,
                     const float* c11, const float* c13, const float* c33, const float* dc11,
                     const float* dc13, const float* dc33, const float* wavelet, const int* sloc,
                     int ns, const int* rloc, int nr, const float* taper) {
  return vti::run_grad2d(ctx, g, gc11, gc13, gc33, nullptr, c11, c13, c33, dc11, dc13, dc33,
                         wavelet, sloc, ns, rloc, nr, taper, nullptr, true);
}

}  // extern "C"
