// 2D reverse-time migration (rtm_f, lib/vti-fwi-2d/rtm_f.cu:13-267) for
// sm_100a.
//
// One step kernel serves both wavefields; both are forwardCD levels
// (kernels.cu:452-498) with the taper of cur and next folded in as in the
// forward-modeling kernel (stored levels are once-tapered, prev is read as
// taper * prev):
//   * source pass: dipole source (injectDipoleSource, kernels.cu:251-256:
//     +a at the source, -a one row below) and, every `ratio` steps, the slice
//     0.5(p+q) of the new level (recordWavefieldSlice, kernels.cu:335-343) into
//     a device array holding all slices of the shot;
//   * receiver pass: the kernel first images the current level,
//     image += 0.5(p+q) * ((1-f) S0 + f S1) (imagingCrossCor,
//     kernels.cu:414-423), then steps; the traces enter as dipoles
//     interpolated in time (injectDipoleData, kernels.cu:232-244), scaled by
//     the taper the reference applies right after the injection.
// The slice pair and weight each level is imaged with, and the data rows
// each injection interpolates, follow rtm_f's bookkeeping on the host.
#include <algorithm>
#include <cmath>
#include <vector>

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

struct RtmStep {
  int nnx, nnz;
  const float *p1, *q1;  // current level
  float *p0, *q0;        // prev in / next out; null: imaging only
  const float *c11, *c13, *c33, *taper;
  float idx2, idz2, dt2;
  int src;    // dipole source at src (+amp) and src + nnx (-amp); -1: none
  float amp;
  float* slice;  // set: 0.5(p+q) of the new level
  float* image;  // set: image the current level against (1-f) s0 + f s1
  const float *s0, *s1;
  float f;
  float* probe_out;  // set: *probe_out = dt2 (p + q) of the current level at probe
  int probe;
};

__global__ void __launch_bounds__(BX* BZ) k_rtm2d_step(RtmStep a) {
  __shared__ float sp[BZ][BX + 8], sq[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx, iz = kHalo + blockIdx.y * BZ + tz;
  const int nnx = a.nnx, nnz = a.nnz;
  auto ld = [&](const float* v, int x, int z) {
    return (x < nnx && z < nnz) ? v[x + z * nnx] : 0.f;
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
  __syncthreads();
  if (!(ix < nnx - kHalo && iz < nnz - kHalo)) return;
  const int i = ix + iz * nnx;
  const float p = sp[tz][tx + 4], q = sq[tz + 4][tx];
  if (a.image) {
    const float d = (1.f - a.f) * a.s0[i] + a.f * a.s1[i];
    a.image[i] += 0.5f * (p + q) * d;
  }
  if (a.probe_out && i == a.probe) *a.probe_out = a.dt2 * (p + q);  // extractWavelet
  if (!a.p0) return;
  const float tp = lap9(&sp[tz][tx + 4], 1) * a.idx2;
  const float tq = lap9(&sq[tz + 4][tx], BX) * a.idz2;
  const float t = a.taper[i];
  float pn = fmaf(a.dt2, fmaf(a.c11[i], tp, a.c13[i] * tq), 2.f * p - t * a.p0[i]);
  float qn = fmaf(a.dt2, fmaf(a.c13[i], tp, a.c33[i] * tq), 2.f * q - t * a.q0[i]);
  if (i == a.src) {
    pn += a.amp;
    qn += a.amp;
  } else if (a.src >= 0 && i == a.src + nnx) {
    pn -= a.amp;
    qn -= a.amp;
  }
  pn *= t;
  qn *= t;
  a.p0[i] = pn;
  a.q0[i] = qn;
  if (a.slice) a.slice[i] = 0.5f * (pn + qn);
}

// injectDipoleData (dipole != 0) or injectData (kernels.cu:208-217) into a
// level that has already been tapered: the taper factor of each point (1 in
// the never-updated 4-cell frame) is applied to the injected value. Receivers
// may share points, hence the atomics.
__global__ void k_rtm2d_inject(float* p, float* q, const float* d0, const float* d1, float f,
                               const int* ridx, const float* taper, int nr, float dt2, int nnx,
                               int nnz, int dipole) {
  const int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir >= nr) return;
  const float v = dt2 * (0.5f * ((1.f - f) * (d0 ? d0[ir] : 0.f) + f * (d1 ? d1[ir] : 0.f)));
  auto add = [&](int k, float w) {
    const int x = k % nnx, z = k / nnx;
    const bool in = x >= kHalo && x < nnx - kHalo && z >= kHalo && z < nnz - kHalo;
    const float s = in ? taper[k] * w : w;
    atomicAdd(p + k, s);
    atomicAdd(q + k, s);
  };
  add(ridx[ir], v);
  if (dipole) add(ridx[ir] + nnx, -v);
}

// extendedImagingCrossCor (kernels.cu:425-436) over the reference kernel's
// threads: image[i + (h+nhx)*nnxz] += 0.5(p+q)[i-h] * ((1-f) S0 + f S1)[i+h],
// x in [x_lo, x_hi), z in [4, z_hi).
__global__ void k_odcig_image(float* image, const float* p, const float* q, const float* s0,
                              const float* s1, float f, int nnx, int nnz, int nhx, int x_lo,
                              int x_hi, int z_hi) {
  const int ix = x_lo + blockIdx.x * blockDim.x + threadIdx.x;
  const int iz = kHalo + blockIdx.y * blockDim.y + threadIdx.y;
  if (ix >= x_hi || iz >= z_hi) return;
  const long long nnxz = (long long)nnx * nnz;
  const int i = ix + iz * nnx;
  for (int h = -nhx; h <= nhx; ++h) {
    const float d = (1.f - f) * s0[i + h] + f * s1[i + h];
    image[i + (h + nhx) * nnxz] += 0.5f * (p[i - h] + q[i - h]) * d;
  }
}

}  // namespace
}  // namespace vti

using namespace vti;

namespace {

// rtm_f (nhx < 0) and odcig_f (nhx >= 0, lib/vti-fwi-2d/odcig_f.cu:12-232):
// the same passes; odcig_f images with subsurface x offsets |h| <= nhx and its
// source pass injects w[it-1] without the dt2 factor after level 1
// (odcig_f.cu:124).
int rtm2d_impl(vti_ctx* ctx, const vti2d_geom* g, int nhx, float* image, const float* data,
               const float* c11, const float* c13, const float* c33, const float* wavelet,
               const int* sloc, int ns, const int* rloc, int nr, const float* taper) {
  if (!ctx || !g || !image || !data || !c11 || !c13 || !c33 || !wavelet || !sloc || !taper ||
      (nr > 0 && !rloc) || ns < 0)
    return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 10 || g->nt < 3 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5f);  // rtm_f.cu:16
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  const int nnt = (g->nt - 1) / ratio + 1;
  const int nnt_data = (g->nt - ntNeg - 1) / ratio + 1;
  // the dipole source needs both of its points inside the updated region;
  // receivers only need theirs inside the grid
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[0] < kHalo || s[0] >= nnx - kHalo || s[1] < kHalo || s[1] + 1 >= nnz - kHalo)
      return fail(ctx, VTI_ERR_ARG, "2D RTM source (and the point below it) must lie in the "
                                    "updated region");
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
    for (int ir = 0; ir < s[2]; ++ir) {
      const int x = rloc[2 * (s[3] + ir)], z = rloc[2 * (s[3] + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z + 1 >= nnz)
        return fail(ctx, VTI_ERR_ARG, "2D receiver (and the point below it) outside the grid");
    }
  }
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t sm = ctx->stream;
  // device buffers: model, taper, 4 wavefields, image, slices, traces, receivers
  const size_t nslices = (size_t)nnt + 1;  // one past the last slice reads zeros
  const size_t nimg = nhx < 0 ? 1 : 2 * (size_t)nhx + 1;
  if (nhx >= 0 && 2 * nhx + 1 > nnx)
    return fail(ctx, VTI_ERR_ARG, "ODCIG: 2*nhx+1 exceeds the grid width");
  const size_t nfloat = (8 + nimg) * (size_t)nnxz + nslices * nnxz + (size_t)nnt_data * nr;
  float* buf = nullptr;
  int* d_ridx = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&buf, nfloat * sizeof(float)));
  int st = VTI_OK;
  if (cudaMalloc((void**)&d_ridx, std::max(nr, 1) * sizeof(int)) != cudaSuccess) {
    cudaFree(buf);
    return fail(ctx, VTI_ERR_OOM, "cannot allocate the receiver table");
  }
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float *p0 = dtap + nnxz, *q0 = p0 + nnxz, *p1 = q0 + nnxz, *q1 = p1 + nnxz;
  float* dimg = q1 + nnxz;
  float* slices = dimg + nimg * nnxz;
  float* ddata = slices + nslices * nnxz;
  auto done = [&](int status) {
    cudaStreamSynchronize(sm);
    cudaFree(buf);
    cudaFree(d_ridx);
    return status;
  };
#define RTM_CK(call)                                               \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return done(cuda_check(ctx, e_, #call)); \
  } while (0)
  RTM_CK(cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, sm));
  RTM_CK(cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, sm));
  RTM_CK(cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, sm));
  RTM_CK(cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, sm));
  if (nr > 0)
    RTM_CK(cudaMemcpyAsync(ddata, data, (size_t)nnt_data * nr * 4, cudaMemcpyHostToDevice, sm));
  // image and every slice start at zero (rtm_f.cu:24,55)
  RTM_CK(cudaMemsetAsync(dimg, 0, (nimg * nnxz + nslices * nnxz) * 4, sm));
  std::vector<int> ridx(std::max(nr, 1));
  for (int ir = 0; ir < nr; ++ir) ridx[ir] = rloc[2 * ir] + rloc[2 * ir + 1] * nnx;
  RTM_CK(cudaMemcpyAsync(d_ridx, ridx.data(), std::max(nr, 1) * sizeof(int),
                         cudaMemcpyHostToDevice, sm));
  const dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  RtmStep a{};
  a.nnx = nnx;
  a.nnz = nnz;
  a.c11 = dc11;
  a.c13 = dc13;
  a.c33 = dc33;
  a.taper = dtap;
  a.idx2 = 1.f / (g->dx * g->dx);
  a.idz2 = 1.f / (g->dz * g->dz);
  a.dt2 = dt2;
  auto step = [&](const float* cp, const float* cq, float* np, float* nq) -> int {
    a.p1 = cp;
    a.q1 = cq;
    a.p0 = np;
    a.q0 = nq;
    k_rtm2d_step<<<grid, block, 0, sm>>>(a);
    ctx->launches++;
    return cuda_check(ctx, cudaGetLastError(), "k_rtm2d_step");
  };
  auto slice_at = [&](int j) { return slices + (size_t)j * nnxz; };
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    const int sxz = s[0] + s[1] * nnx, nri = s[2], ir0 = s[3];
    RTM_CK(cudaMemsetAsync(p0, 0, 4 * nnxz * 4, sm));
    // level 1 (rtm_f.cu:113-120): the dipole source, then the taper, so
    // t * (dt2 w0) at the source and -t * (dt2 w0) below it; with ratio 1 its
    // slice 0.5(p+q) holds the same two values (p = q there)
    {
      const float a0 = dt2 * wavelet[0];
      const float v[2] = {taper[sxz] * a0, -(taper[sxz + nnx] * a0)};
      for (float* f : {p1, q1}) {
        RTM_CK(cudaMemcpyAsync(f + sxz, &v[0], 4, cudaMemcpyHostToDevice, sm));
        RTM_CK(cudaMemcpyAsync(f + sxz + nnx, &v[1], 4, cudaMemcpyHostToDevice, sm));
      }
      if (ratio == 1) {  // a whole new slice: clear the previous shot's points
        RTM_CK(cudaMemsetAsync(slice_at(1), 0, nnxz * 4, sm));
        RTM_CK(cudaMemcpyAsync(slice_at(1) + sxz, &v[0], 4, cudaMemcpyHostToDevice, sm));
        RTM_CK(cudaMemcpyAsync(slice_at(1) + sxz + nnx, &v[1], 4, cudaMemcpyHostToDevice, sm));
      }
      RTM_CK(cudaStreamSynchronize(sm));  // v goes out of scope
    }
    float *cp = p1, *cq = q1, *np = p0, *nq = q0;
    a.image = nullptr;
    for (int it = 2; it < g->nt; ++it) {
      a.src = sxz;
      a.amp = nhx < 0 ? dt2 * wavelet[it - 1] : wavelet[it - 1];
      a.slice = (it % ratio == 0) ? slice_at(it / ratio) : nullptr;
      st = step(cp, cq, np, nq);
      if (st != VTI_OK) return done(st);
      std::swap(cp, np);
      std::swap(cq, nq);
    }
    // receiver pass (rtm_f.cu:152-225)
    a.src = -1;
    a.slice = nullptr;
    RTM_CK(cudaMemsetAsync(p0, 0, 4 * nnxz * 4, sm));
    cp = p0;
    cq = q0;
    np = p1;
    nq = q1;
    const float* row_base = ddata + ir0;
    const float* d0 = row_base + (size_t)(nnt_data - 1) * nr;
    const float* d1 = nullptr;  // zeros
    auto inject = [&](float* p, float* q, float f) -> int {
      if (nri <= 0) return VTI_OK;
      k_rtm2d_inject<<<(nri + 127) / 128, 128, 0, sm>>>(p, q, d0, d1, f, d_ridx + ir0, dtap, nri,
                                                         dt2, nnx, nnz, 1);
      ctx->launches++;
      return cuda_check(ctx, cudaGetLastError(), "k_rtm2d_inject");
    };
    st = inject(cp, cq, 0.f);  // into the zero level, then its taper (rtm_f.cu:162-164)
    if (st != VTI_OK) return done(st);
    float f = (g->nt - 2.) / ratio;
    int s0 = (int)f, s1 = std::min(s0 + 1, nnt);
    f -= s0;
    // extended imaging of a finished level, right after its injection
    const int x_lo = std::max(kHalo, nhx);
    const int x_hi = std::min(nnx - nhx, kHalo + 16 * ((nnx - 8 + 15) / 16));
    const int z_hi = std::min(nnz, kHalo + 16 * ((nnz - 8 + 15) / 16));
    auto odcig = [&](const float* p, const float* q, float fw) -> int {
      if (x_hi <= x_lo) return VTI_OK;
      const dim3 b2(32, 8), g2((x_hi - x_lo + 31) / 32, (z_hi - kHalo + 7) / 8);
      k_odcig_image<<<g2, b2, 0, sm>>>(dimg, p, q, slice_at(s0), slice_at(s1), fw, nnx, nnz, nhx,
                                       x_lo, x_hi, z_hi);
      ctx->launches++;
      return cuda_check(ctx, cudaGetLastError(), "k_odcig_image");
    };
    if (nhx >= 0) {
      st = odcig(cp, cq, f);
      if (st != VTI_OK) return done(st);
    }
    // RTM: the level just made is imaged by the next kernel, which reads it as cur
    a.image = nhx < 0 ? dimg : nullptr;
    a.s0 = slice_at(s0);
    a.s1 = slice_at(s1);
    a.f = f;
    for (int it = g->nt - 3; it >= 0; --it) {
      st = step(cp, cq, np, nq);  // images cur (level it+1), makes level it
      if (st != VTI_OK) return done(st);
      if (it >= ntNeg) {
        float fd = (it - ntNeg + 1.) / ratio;
        const int i1 = (int)fd;
        if ((it - ntNeg + 2) % ratio == 0) {
          d1 = row_base + (size_t)i1 * nr;
          std::swap(d0, d1);
        }
        fd -= i1;
        st = inject(np, nq, fd);
        if (st != VTI_OK) return done(st);
      }
      float fs = (float)it / ratio;
      const int i1 = (int)fs;
      if ((it + 1) % ratio == 0) {
        s1 = i1;
        std::swap(s0, s1);
      }
      fs -= i1;
      a.s0 = slice_at(s0);
      a.s1 = slice_at(s1);
      a.f = fs;
      if (nhx >= 0) {
        st = odcig(np, nq, fs);
        if (st != VTI_OK) return done(st);
      }
      std::swap(cp, np);
      std::swap(cq, nq);
    }
    if (nhx < 0) {  // image the last level (it = 0)
      st = step(cp, cq, nullptr, nullptr);
      if (st != VTI_OK) return done(st);
    }
    a.image = nullptr;
  }
  RTM_CK(cudaMemcpyAsync(image, dimg, nimg * nnxz * 4, cudaMemcpyDeviceToHost, sm));
  RTM_CK(cudaStreamSynchronize(sm));
#undef RTM_CK
  return done(VTI_OK);
}

}  // namespace

extern "C" int vti2d_rtm(vti_ctx* ctx, const vti2d_geom* g, float* image, const float* data,
                         const float* c11, const float* c13, const float* c33,
                         const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                         const float* taper) {
  return rtm2d_impl(ctx, g, -1, image, data, c11, c13, c33, wavelet, sloc, ns, rloc, nr, taper);
}

extern "C" int vti2d_odcig(vti_ctx* ctx, const vti2d_geom* g, int nhx, float* image,
                           const float* data, const float* c11, const float* c13,
                           const float* c33, const float* wavelet, const int* sloc, int ns,
                           const int* rloc, int nr, const float* taper) {
  if (nhx < 0) return fail(ctx, VTI_ERR_ARG, "ODCIG: nhx must be >= 0");
  return rtm2d_impl(ctx, g, nhx, image, data, c11, c13, c33, wavelet, sloc, ns, rloc, nr, taper);
}

// waveletGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:373-530): per shot the
// adjoint wavefield driven by the traces as points (injectData), forwardCD and
// the taper; g[it] = dt2 (p + q) at the source for every level (extractWavelet,
// an assignment per shot, kernels.cu:258-261), g[nt-2] from the seeded level;
// shots summed on the host in float. The step kernel reads the extracted value
// from the finished level when it steps from it.
extern "C" int vti2d_wavelet_gradient(vti_ctx* ctx, const vti2d_geom* g, float* gwavelet,
                                      const float* data, const float* c11, const float* c13,
                                      const float* c33, const int* sloc, int ns, const int* rloc,
                                      int nr, const float* taper) {
  if (!ctx || !g || !gwavelet || !data || !c11 || !c13 || !c33 || !sloc || !taper ||
      (nr > 0 && !rloc) || ns < 0)
    return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 3 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  {
    const int cst = check_cfl2d(ctx, g, c11, c13, c33);
    if (cst != VTI_OK) return cst;
  }
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5);  // objFuncGradient_f.cu:375 (double 0.5)
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int nnt = (g->nt - 1) / ratio + 1;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[0] < kHalo || s[0] >= nnx - kHalo || s[1] < kHalo || s[1] >= nnz - kHalo)
      return fail(ctx, VTI_ERR_ARG, "2D source must lie in the updated region");
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
    for (int ir = 0; ir < s[2]; ++ir) {
      const int x = rloc[2 * (s[3] + ir)], z = rloc[2 * (s[3] + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz)
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
    }
  }
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t sm = ctx->stream;
  const size_t nfloat = 8 * (size_t)nnxz + (size_t)nnt * nr + g->nt;
  float* buf = nullptr;
  int* d_ridx = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&buf, nfloat * sizeof(float)));
  if (cudaMalloc((void**)&d_ridx, std::max(nr, 1) * sizeof(int)) != cudaSuccess) {
    cudaFree(buf);
    return fail(ctx, VTI_ERR_OOM, "cannot allocate the receiver table");
  }
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float *p0 = dtap + nnxz, *q0 = p0 + nnxz, *p1 = q0 + nnxz, *q1 = p1 + nnxz;
  float* ddata = q1 + nnxz;
  float* gs = ddata + (size_t)nnt * nr;
  auto done = [&](int status) {
    cudaStreamSynchronize(sm);
    cudaFree(buf);
    cudaFree(d_ridx);
    return status;
  };
#define WG_CK(call)                                                 \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) return done(cuda_check(ctx, e_, #call)); \
  } while (0)
  WG_CK(cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, sm));
  WG_CK(cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, sm));
  WG_CK(cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, sm));
  WG_CK(cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, sm));
  if (nr > 0)
    WG_CK(cudaMemcpyAsync(ddata, data, (size_t)nnt * nr * 4, cudaMemcpyHostToDevice, sm));
  std::vector<int> ridx(std::max(nr, 1));
  for (int ir = 0; ir < nr; ++ir) ridx[ir] = rloc[2 * ir] + rloc[2 * ir + 1] * nnx;
  WG_CK(cudaMemcpyAsync(d_ridx, ridx.data(), std::max(nr, 1) * sizeof(int),
                        cudaMemcpyHostToDevice, sm));
  const dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  RtmStep a{};
  a.nnx = nnx;
  a.nnz = nnz;
  a.c11 = dc11;
  a.c13 = dc13;
  a.c33 = dc33;
  a.taper = dtap;
  a.idx2 = 1.f / (g->dx * g->dx);
  a.idz2 = 1.f / (g->dz * g->dz);
  a.dt2 = dt2;
  a.src = -1;
  std::vector<float> acc(g->nt, 0.f), hs(g->nt);
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    const int nri = s[2], ir0 = s[3];
    WG_CK(cudaMemsetAsync(p0, 0, 4 * nnxz * 4, sm));
    WG_CK(cudaMemsetAsync(gs, 0, g->nt * 4, sm));
    const float* row_base = ddata + ir0;
    const float* d0 = row_base + (size_t)(nnt - 1) * nr;
    const float* d1 = nullptr;  // zeros
    auto inject = [&](float* p, float* q, float f) -> int {
      if (nri <= 0) return VTI_OK;
      k_rtm2d_inject<<<(nri + 127) / 128, 128, 0, sm>>>(p, q, d0, d1, f, d_ridx + ir0, dtap, nri,
                                                         dt2, nnx, nnz, 0);
      ctx->launches++;
      return cuda_check(ctx, cudaGetLastError(), "k_rtm2d_inject");
    };
    float *cp = p0, *cq = q0, *np = p1, *nq = q1;
    int st = inject(cp, cq, 0.f);
    if (st != VTI_OK) return done(st);
    a.probe = s[0] + s[1] * nnx;
    a.probe_out = gs + (g->nt - 2);
    for (int it = g->nt - 3; it >= 0; --it) {
      a.p1 = cp;
      a.q1 = cq;
      a.p0 = np;
      a.q0 = nq;
      k_rtm2d_step<<<grid, block, 0, sm>>>(a);  // extracts cur, makes level it
      ctx->launches++;
      WG_CK(cudaGetLastError());
      float f = (it + 1.) / ratio;
      const int i1 = (int)f;
      if ((it + 2) % ratio == 0) {
        d1 = row_base + (size_t)i1 * nr;
        std::swap(d0, d1);
      }
      f -= i1;
      st = inject(np, nq, f);
      if (st != VTI_OK) return done(st);
      a.probe_out = gs + it;
      std::swap(cp, np);
      std::swap(cq, nq);
    }
    a.p1 = cp;  // extract the last level
    a.q1 = cq;
    a.p0 = a.q0 = nullptr;
    k_rtm2d_step<<<grid, block, 0, sm>>>(a);
    ctx->launches++;
    WG_CK(cudaGetLastError());
    WG_CK(cudaMemcpyAsync(hs.data(), gs, g->nt * 4, cudaMemcpyDeviceToHost, sm));
    WG_CK(cudaStreamSynchronize(sm));
    for (int it = 0; it < g->nt; ++it) acc[it] += hs[it];
  }
  std::copy(acc.begin(), acc.end(), gwavelet);
#undef WG_CK
  return done(VTI_OK);
}
