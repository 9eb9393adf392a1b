// 2D VTI pseudo-acoustic forward modeling for sm_100a
// (lib/vti-fwi-2d: forwardCD kernels.cu:452-498, synthetic_f.cu:13-124,
// modeling_f.cu:10-82).
//
// Arrays are (nx+2npad) x (nz+2npad), x fastest, updated on [4, n-4) in both
// directions. p (sigma_h) carries the x stencil, q (sigma_v) the z stencil.
// The taper multiplies cur and next after every step (kernels.cu:304-315);
// stored values here are the once-tapered levels, prev is read as taper*prev.
//
// One fused kernel per time step: stencil + source + taper; receivers are
// recorded by a small gather kernel. The source amplitudes of all steps are
// uploaded once, so every step's launch differs only in its buffer pointers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "vti_internal.h"

namespace vti {
namespace {

// lib/vti-fwi-2d/kernels.h:4-8 (float literals)
constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;

constexpr int BX = 32, BZ = 8;

struct Step2d {
  int nnx, nnz;
  const float* p1;
  const float* q1;
  float* p0;
  float* q0;
  const float* c11;
  const float* c13;
  const float* c33;
  const float* taper;
  float idx2, idz2, dt2;
  int src;        // flat index of the source
  const float* amp;  // device pointer to the source amplitude of this step
};

__global__ void __launch_bounds__(BX* BZ) k_step2d(Step2d a) {
  __shared__ float sp[BZ][BX + 8];
  __shared__ float sq[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx;
  const int iz = kHalo + blockIdx.y * BZ + tz;
  const bool valid = ix < a.nnx - kHalo && iz < a.nnz - kHalo;
  const int i = ix + iz * a.nnx;
  // stage p rows (x halo) and q columns (z halo); out-of-range lanes load 0
  auto ldp = [&](int x) { return (x < a.nnx && iz < a.nnz) ? a.p1[x + iz * a.nnx] : 0.f; };
  auto ldq = [&](int z) { return (ix < a.nnx && z < a.nnz) ? a.q1[ix + z * a.nnx] : 0.f; };
  sp[tz][tx + 4] = ldp(ix);
  if (tx < 4) {
    sp[tz][tx] = ldp(ix - 4);
    sp[tz][tx + BX + 4] = ldp(ix + BX);
  }
  sq[tz + 4][tx] = ldq(iz);
  if (tz < 4) {
    sq[tz][tx] = ldq(iz - 4);
    sq[tz + BZ + 4][tx] = ldq(iz + BZ);
  }
  __syncthreads();
  if (!valid) return;
  const float* r = &sp[tz][tx + 4];
  float tp = kC0 * r[0];
  tp = fmaf(kC1, r[-1] + r[1], tp);
  tp = fmaf(kC2, r[-2] + r[2], tp);
  tp = fmaf(kC3, r[-3] + r[3], tp);
  tp = fmaf(kC4, r[-4] + r[4], tp);
  float tq = kC0 * sq[tz + 4][tx];
  tq = fmaf(kC1, sq[tz + 3][tx] + sq[tz + 5][tx], tq);
  tq = fmaf(kC2, sq[tz + 2][tx] + sq[tz + 6][tx], tq);
  tq = fmaf(kC3, sq[tz + 1][tx] + sq[tz + 7][tx], tq);
  tq = fmaf(kC4, sq[tz][tx] + sq[tz + 8][tx], tq);
  tp *= a.idx2;
  tq *= a.idz2;
  const float t = a.taper[i];
  float pn = fmaf(a.dt2, fmaf(a.c11[i], tp, a.c13[i] * tq), 2.f * r[0] - t * a.p0[i]);
  float qn = fmaf(a.dt2, fmaf(a.c13[i], tp, a.c33[i] * tq), 2.f * sq[tz + 4][tx] - t * a.q0[i]);
  if (i == a.src) {
    const float s = *a.amp;
    pn += s;
    qn += s;
  }
  a.p0[i] = t * pn;
  a.q0[i] = t * qn;
}

// recordData (kernels.cu:317-324): 0.5(p+q) at receivers into row `row`.
__global__ void k_record2d(float* data, long long row_off, const float* p, const float* q,
                           const int* ridx, int nr) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    int i = ridx[ir];
    data[row_off + ir] = 0.5f * (p[i] + q[i]);
  }
}

// injectSource + abc(p1,q1) at t=1 (synthetic_f.cu:86-89).
__global__ void k_init2d(float* p, float* q, int src, float value, float taper_at_src) {
  p[src] = value * taper_at_src;
  q[src] = value * taper_at_src;
}

struct Dev2d {
  float* buf = nullptr;  // c11 c13 c33 taper p0 q0 p1 q1 amps
  size_t n = 0;
};

}  // namespace
}  // namespace vti

using namespace vti;

namespace {

int run2d(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13, const float* c33,
          const float* wavelet, const float* taper, int slocxz, const int* rloc, int nri,
          int nr_total, int ir0, float* out, int mode) {
  if (!ctx || !g || !c11 || !c13 || !c33 || !wavelet || !taper || !out) return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 2 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  if (slocxz < 0 || slocxz >= nnxz) return fail(ctx, VTI_ERR_ARG, "2D source outside the grid");
  const float dt = g->dt, dt2 = dt * dt;
  const float dx2 = g->dx * g->dx, dz2 = g->dz * g->dz;
  const int ratio = mode == 0 ? (int)(g->rate / dt + 0.5f) : (int)std::round(g->rate / dt);
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  // device buffers: 4 model/taper + 4 wavefields + nt amplitudes + receivers + output rows
  const long long nrows_out = mode == 0 ? (g->nt - ntNeg - 1) / ratio + 1 : 0;
  float* buf = nullptr;
  size_t nbuf = 8 * (size_t)nnxz + g->nt;
  VTI_CUDA(ctx, cudaMalloc((void**)&buf, nbuf * sizeof(float)));
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float* w[4] = {dtap + nnxz, dtap + 2 * nnxz, dtap + 3 * nnxz, dtap + 4 * nnxz};
  float* amps = dtap + 5 * nnxz;
  int* d_ridx = nullptr;
  float* d_data = nullptr;
  int st = VTI_OK;
  auto cleanup = [&]() {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(buf);
    if (d_ridx) cudaFree(d_ridx);
    if (d_data) cudaFree(d_data);
  };
#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) {                      \
      st = cuda_check(ctx, e_, #call);            \
      cleanup();                                  \
      return st;                                  \
    }                                             \
  } while (0)
  CK(cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(w[0], 0, 4 * nnxz * 4, ctx->stream));
  std::vector<float> h_amp(g->nt, 0.f);
  for (int it = 2; it < g->nt; ++it)
    h_amp[it] = mode == 0 ? dt2 * wavelet[it - 1] : wavelet[it - 1];  // modeling_f.cu:66
  CK(cudaMemcpyAsync(amps, h_amp.data(), g->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
  std::vector<int> ridx;
  if (mode == 0 && nri > 0) {
    ridx.resize(nri);
    for (int ir = 0; ir < nri; ++ir) {
      int x = rloc[2 * (ir0 + ir)], z = rloc[2 * (ir0 + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz) {
        cleanup();
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
      }
      ridx[ir] = x + z * nnx;
    }
    CK(cudaMalloc((void**)&d_ridx, nri * sizeof(int)));
    CK(cudaMemcpyAsync(d_ridx, ridx.data(), nri * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMalloc((void**)&d_data, (size_t)nrows_out * nri * sizeof(float)));
    CK(cudaMemsetAsync(d_data, 0, (size_t)nrows_out * nri * sizeof(float), ctx->stream));
  }
  // time level 1: source then taper (synthetic_f.cu:86-89)
  k_init2d<<<1, 1, 0, ctx->stream>>>(w[2], w[3], slocxz, dt2 * wavelet[0], taper[slocxz]);
  ctx->launches++;
  float *p1 = w[2], *q1 = w[3], *p0 = w[0], *q0 = w[1];
  auto snapshot = [&](long long row, const float* p, const float* q) -> int {
    if (mode == 0) {
      if (nri > 0) {
        k_record2d<<<(nri + 127) / 128, 128, 0, ctx->stream>>>(d_data, row * nri, p, q, d_ridx,
                                                                nri);
        ctx->launches++;
      }
    } else {
      cudaError_t e = cudaMemcpyAsync(out + row * nnxz, p, nnxz * 4, cudaMemcpyDeviceToHost,
                                      ctx->stream);
      if (e != cudaSuccess) return cuda_check(ctx, e, "snapshot copy");
    }
    return VTI_OK;
  };
  if (ratio == 1 && g->ot == 0.f) {
    st = snapshot(1, p1, q1);
    if (st != VTI_OK) {
      cleanup();
      return st;
    }
  }
  dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  // The trace-recording time loop (every node a kernel) is captured as one
  // CUDA graph: a 2D step is a few microseconds of work, so per-launch
  // overhead is most of its cost. With per-kernel timing on, or snapshots
  // copied to the host (modeling), the launches are issued directly.
  const bool use_graph = mode == 0 && !ctx->timing;
  cudaGraph_t graph = nullptr;
  if (use_graph) CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  for (int it = 2; it < g->nt; ++it) {
    float t = it * dt + g->ot;
    Step2d a{nnx, nnz, p1, q1, p0, q0, dc11, dc13, dc33, dtap, 1.f / dx2, 1.f / dz2, dt2,
             slocxz, amps + it};
    {
      LaunchTimer tm(ctx, kTimedStep2d);
      k_step2d<<<grid, block, 0, ctx->stream>>>(a);
    }
    ctx->launches++;
    if (t >= 0.f && (it - ntNeg) % ratio == 0) {
      st = snapshot((it - ntNeg) / ratio, p0, q0);
      if (st != VTI_OK) {
        if (use_graph) {
          cudaStreamEndCapture(ctx->stream, &graph);
          if (graph) cudaGraphDestroy(graph);
        }
        cleanup();
        return st;
      }
    }
    std::swap(p0, p1);
    std::swap(q0, q1);
  }
  if (use_graph) {
    CK(cudaStreamEndCapture(ctx->stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ei);
    const cudaError_t el = cudaGraphLaunch(exec, ctx->stream);
    cudaGraphExecDestroy(exec);  // released once the launch completes
    CK(el);
  }
  CK(cudaGetLastError());
  if (mode == 0 && nri > 0) {
    // scatter rows into the caller's receiver-fastest layout
    CK(cudaMemcpy2DAsync(out + ir0, (size_t)nr_total * 4, d_data, (size_t)nri * 4,
                         (size_t)nri * 4, nrows_out, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  cleanup();
#undef CK
  return VTI_OK;
}

}  // namespace

extern "C" {

int vti2d_synthetic(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                    const float* c33, const float* wavelet, const int* sloc, int ns,
                    const int* rloc, int nr, const float* taper, float* data) {
  if (!ctx || !g || !sloc || (nr > 0 && !rloc)) return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
    int st = run2d(ctx, g, c11, c13, c33, wavelet, taper, s[0] + s[1] * nnx, rloc, s[2], nr, s[3],
                   data, 0);
    if (st != VTI_OK) return st;
  }
  return VTI_OK;
}

int vti2d_modeling(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                   const float* c33, const float* wavelet, int slocxz, const float* taper,
                   float* wavefield) {
  return run2d(ctx, g, c11, c13, c33, wavelet, taper, slocxz, nullptr, 0, 0, 0, wavefield, 1);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free synthetic traces.
//
// vti2d_synthetic_noalloc() computes what vti2d_synthetic() computes (same
// kernels, same launch order, same host arithmetic) but never allocates
// device memory: the model, the four wavefields, the source amplitudes, the
// receiver indices and the trace rows of one shot all live in one file-scope
// static device array of kNoAllocFloats floats (40 MiB), reserved once when
// this module is loaded.
//
// Who needs it: callers that must not allocate inside a call. cudaMalloc and
// cudaFree synchronise the whole device, so a caller that keeps other streams
// busy (a 3D gradient running beside 2D modeling, say) would see them stall
// at every call; a long-running job that shares the GPU can find cudaMalloc
// failing for lack of memory hours after start-up, while a static
// reservation either exists from the first call on or never; and hosts that
// give the library a fixed memory budget forbid allocations inside calls.
//
// Limits and rules:
//  * need = 8*nnx*nnz + nt + nri + rows*nri floats (rows =
//    (nt-ntNeg-1)/ratio + 1, nri the largest shot's receiver count); a call
//    that needs more than kNoAllocFloats is rejected with VTI_ERR_ARG before
//    any work is queued. A 1000 x 1000 padded grid with nt = 4000 and 1000
//    receivers per shot sampled every 4 steps fits.
//  * The first call on a device (that device current) looks up the array's
//    address with cudaGetSymbolAddress and caches it; make that first call
//    before any stream capture begins.
//  * The wavefields and the trace rows must start at zero for every shot;
//    they are cleared with cudaMemsetAsync on the context stream (the model,
//    amplitudes and receiver indices are overwritten by copies).
//  * There is one array per device and process: calls that overlap in time on
//    the same device (two threads, two contexts, two streams) race on it and
//    corrupt each other's results. Serialise them.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocFloats = (size_t)10 << 20;  // 40 MiB
__device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

// Address of this device's scratch array; looked up once per device.
int noalloc_scratch(vti_ctx* ctx, float** out) {
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return fail(ctx, VTI_ERR_ARG, "device index beyond the allocation-free table");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[ctx->device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_check(ctx, e, "cudaGetSymbolAddress(static scratch)");
    g_noalloc_ptr[ctx->device] = (float*)p;
  }
  *out = g_noalloc_ptr[ctx->device];
  return VTI_OK;
}

}  // namespace

extern "C" int vti2d_synthetic_noalloc(vti_ctx* ctx, const vti2d_geom* g, const float* c11,
                                       const float* c13, const float* c33, const float* wavelet,
                                       const int* sloc, int ns, const int* rloc, int nr,
                                       const float* taper, float* data) {
  if (!ctx || !g || !sloc || (nr > 0 && !rloc) || !c11 || !c13 || !c33 || !wavelet || !taper ||
      !data)
    return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 2 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5f);  // as vti2d_synthetic
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  const long long rows = (g->nt - ntNeg - 1) / ratio + 1;
  // validate every shot and size the largest before queuing anything
  long long max_nri = 0;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
    const long long src = s[0] + (long long)s[1] * nnx;
    if (src < 0 || src >= nnxz) return fail(ctx, VTI_ERR_ARG, "2D source outside the grid");
    for (int ir = 0; ir < s[2]; ++ir) {
      const int x = rloc[2 * (s[3] + ir)], z = rloc[2 * (s[3] + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz)
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
    }
    max_nri = std::max<long long>(max_nri, s[2]);
  }
  const long long need = 8 * nnxz + g->nt + max_nri + rows * max_nri;
  if (need > (long long)kNoAllocFloats) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "allocation-free modeling needs %lld floats of static scratch, capacity %zu",
                  need, kNoAllocFloats);
    return fail(ctx, VTI_ERR_ARG, msg);
  }
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  float* buf = nullptr;
  int st = noalloc_scratch(ctx, &buf);
  if (st != VTI_OK) return st;
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float* w[4] = {dtap + nnxz, dtap + 2 * nnxz, dtap + 3 * nnxz, dtap + 4 * nnxz};
  float* amps = dtap + 5 * nnxz;
  int* d_ridx = reinterpret_cast<int*>(amps + g->nt);
  float* d_rows = amps + g->nt + max_nri;
  cudaStream_t sm = ctx->stream;
  VTI_CUDA(ctx, cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, sm));
  VTI_CUDA(ctx, cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, sm));
  VTI_CUDA(ctx, cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, sm));
  VTI_CUDA(ctx, cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, sm));
  std::vector<float> h_amp(g->nt, 0.f);
  for (int it = 2; it < g->nt; ++it) h_amp[it] = dt2 * wavelet[it - 1];
  VTI_CUDA(ctx, cudaMemcpyAsync(amps, h_amp.data(), g->nt * 4, cudaMemcpyHostToDevice, sm));
  const float idx2 = 1.f / (g->dx * g->dx), idz2 = 1.f / (g->dz * g->dz);
  const dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  std::vector<int> ridx;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    const int slocxz = s[0] + s[1] * nnx, nri = s[2], ir0 = s[3];
    VTI_CUDA(ctx, cudaMemsetAsync(w[0], 0, 4 * nnxz * 4, sm));  // wavefields start at zero
    if (nri > 0) {
      ridx.resize(nri);
      for (int ir = 0; ir < nri; ++ir)
        ridx[ir] = rloc[2 * (ir0 + ir)] + rloc[2 * (ir0 + ir) + 1] * nnx;
      VTI_CUDA(ctx, cudaMemcpyAsync(d_ridx, ridx.data(), nri * sizeof(int),
                                    cudaMemcpyHostToDevice, sm));
      VTI_CUDA(ctx, cudaMemsetAsync(d_rows, 0, (size_t)rows * nri * 4, sm));  // row 0 stays 0
    }
    // time level 1: source then taper (synthetic_f.cu:86-89)
    k_init2d<<<1, 1, 0, sm>>>(w[2], w[3], slocxz, dt2 * wavelet[0], taper[slocxz]);
    ctx->launches++;
    float *p1 = w[2], *q1 = w[3], *p0 = w[0], *q0 = w[1];
    auto record = [&](long long row, const float* p, const float* q) {
      if (nri > 0) {
        k_record2d<<<(nri + 127) / 128, 128, 0, sm>>>(d_rows, row * nri, p, q, d_ridx, nri);
        ctx->launches++;
      }
    };
    if (ratio == 1 && g->ot == 0.f) record(1, p1, q1);
    for (int it = 2; it < g->nt; ++it) {
      const float t = it * dt + g->ot;
      Step2d a{nnx, nnz, p1, q1, p0, q0, dc11, dc13, dc33, dtap, idx2, idz2, dt2, slocxz,
               amps + it};
      k_step2d<<<grid, block, 0, sm>>>(a);
      ctx->launches++;
      if (t >= 0.f && (it - ntNeg) % ratio == 0) record((it - ntNeg) / ratio, p0, q0);
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
    VTI_CUDA(ctx, cudaGetLastError());
    if (nri > 0)  // the caller's receiver-fastest layout, as vti2d_synthetic
      VTI_CUDA(ctx, cudaMemcpy2DAsync(data + ir0, (size_t)nr * 4, d_rows, (size_t)nri * 4,
                                      (size_t)nri * 4, rows, cudaMemcpyDeviceToHost, sm));
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(sm));
  return VTI_OK;
}
