// Context, status strings and pitched device volumes.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "vti_internal.h"

namespace vti {

int fail(vti_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int cuda_check(vti_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return VTI_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  int st = (e == cudaErrorMemoryAllocation) ? VTI_ERR_OOM : VTI_ERR_DEVICE;
  return fail(ctx, st, m);
}

double nyquist_factor(double h) {
  // lib/vti-fwi-3d/gpu/wave3d.h:8-12 coefficients
  const double C[5] = {-2.84722222222, 1.6, -0.2, 0.02539682539, -0.00178571428};
  double s = C[0];
  for (int k = 1; k <= 4; ++k) s += 2.0 * C[k] * ((k & 1) ? -1.0 : 1.0);
  return std::fabs(s) / (h * h);
}

int cfl3d_device(vti_ctx* ctx, const vti3d_geom& g, const Dims3& d, const float* c11,
                 const float* c13, const float* c33, double* number) {
  const double s = nyquist_factor(1.0);
  const double kh = s / ((double)g.dx * g.dx) + (g.ny > 1 ? s / ((double)g.dy * g.dy) : 0.0);
  const double kz = s / ((double)g.dz * g.dz);
  VTI_CUDA(ctx, cudaMemsetAsync(ctx->d_cfl, 0, sizeof(unsigned long long), ctx->stream));
  const int st = launch_cfl_max(ctx, d, c11, c13, c33, kh, kz, ctx->d_cfl);
  if (st != VTI_OK) return st;
  unsigned long long bits = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&bits, ctx->d_cfl, sizeof bits, cudaMemcpyDeviceToHost,
                                ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double lam;
  std::memcpy(&lam, &bits, sizeof lam);
  *number = lam * (double)g.dt * g.dt;
  return VTI_OK;
}

int check_cfl2d(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                const float* c33) {
  return cfl_verdict(ctx, vti2d_cfl_number(g, c11, c13, c33), "2D model");
}

int cfl_verdict(vti_ctx* ctx, double number, const char* what) {
  if (number < 4.0) return VTI_OK;  // false for NaN as well
  char msg[256];
  std::snprintf(msg, sizeof msg,
                "%s: dt^2 * lambda_max = %.4g is not below 4, the leapfrog stability bound of "
                "the 8th-order scheme (reduce dt or the stiffnesses)",
                what, number);
  return fail(ctx, VTI_ERR_CFL, msg);
}

Dims3 make_dims(int nx, int ny, int nz) {
  Dims3 d;
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.pitch = (nx + 31) & ~31;
  d.plane = (long long)d.pitch * ny;
  return d;
}

int vol_alloc(vti_ctx* ctx, const Dims3& d, Vol* v) {
  v->bytes = (size_t)d.plane * (d.nz + 2 * kZPad) * sizeof(float);
  cudaError_t e = cudaMalloc((void**)&v->alloc, v->bytes);
  if (e != cudaSuccess) {
    v->alloc = nullptr;
    return cuda_check(ctx, e, "cudaMalloc(volume)");
  }
  v->origin = v->alloc + (size_t)kZPad * d.plane;
  return vol_zero(ctx, d, v);
}

void vol_free(Vol* v) {
  if (v->alloc) cudaFree(v->alloc);
  v->alloc = v->origin = nullptr;
  v->bytes = 0;
}

int vol_zero(vti_ctx* ctx, const Dims3& d, Vol* v) {
  (void)d;
  VTI_CUDA(ctx, cudaMemsetAsync(v->alloc, 0, v->bytes, ctx->stream));
  return VTI_OK;
}

int vol_upload(vti_ctx* ctx, const Dims3& d, Vol* v, const float* src, int mem) {
  cudaMemcpyKind k = mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  VTI_CUDA(ctx, cudaMemcpy2DAsync(v->origin, d.pitch * sizeof(float), src, d.nx * sizeof(float),
                                  d.nx * sizeof(float), (size_t)d.ny * d.nz, k, ctx->stream));
  return VTI_OK;
}

int vol_download(vti_ctx* ctx, const Dims3& d, const Vol* v, float* dst, int mem) {
  cudaMemcpyKind k = mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  VTI_CUDA(ctx, cudaMemcpy2DAsync(dst, d.nx * sizeof(float), v->origin, d.pitch * sizeof(float),
                                  d.nx * sizeof(float), (size_t)d.ny * d.nz, k, ctx->stream));
  return VTI_OK;
}

int check_device_status(vti_ctx* ctx) {
  int h = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                                ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h == 0) return VTI_OK;
  VTI_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  if (h & (1 << VTI_ERR_TIMEOUT))
    return fail(ctx, VTI_ERR_TIMEOUT, "a device-side pipeline wait timed out");
  if (h & (1 << VTI_ERR_NONFINITE))
    return fail(ctx, VTI_ERR_NONFINITE, "a wavefield, trace or gradient holds NaN or Inf");
  return fail(ctx, VTI_ERR_DEVICE, "device status word " + std::to_string(h));
}

static cudaEvent_t pool_get(vti_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

LaunchTimer::LaunchTimer(vti_ctx* c, int k) : ctx(c), kind(k) {
  if (!ctx->timing) return;
  cudaEvent_t start = pool_get(ctx);
  stop = pool_get(ctx);
  cudaEventRecord(start, ctx->stream);
  ctx->events[kind].push_back({start, stop});
}

LaunchTimer::~LaunchTimer() {
  if (stop) cudaEventRecord(stop, ctx->stream);
}

static void release_events(vti_ctx* ctx) {
  for (auto& v : ctx->events) {
    for (auto& p : v) {
      ctx->event_pool.push_back(p.first);
      ctx->event_pool.push_back(p.second);
    }
    v.clear();
  }
}

}  // namespace vti

using namespace vti;

extern "C" {

int vti_ctx_set_timing(vti_ctx* ctx, int enable) {
  if (!ctx) return VTI_ERR_ARG;
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  release_events(ctx);
  ctx->timing = enable != 0;
  return VTI_OK;
}

int vti_ctx_kernel_time(vti_ctx* ctx, const char* kernel, double* total_ms, uint64_t* count) {
  if (!ctx || !kernel) return VTI_ERR_ARG;
  int k = -1;
  if (!strcmp(kernel, "fwd3d")) k = kTimedFwd3d;
  else if (!strcmp(kernel, "bwd3d")) k = kTimedBwd3d;
  else if (!strcmp(kernel, "step2d")) k = kTimedStep2d;
  if (k < 0) return fail(ctx, VTI_ERR_ARG, std::string("unknown kernel ") + kernel);
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double ms = 0;
  for (auto& p : ctx->events[k]) {
    float t = 0;
    VTI_CUDA(ctx, cudaEventElapsedTime(&t, p.first, p.second));
    ms += t;
  }
  if (total_ms) *total_ms = ms;
  if (count) *count = ctx->events[k].size();
  return VTI_OK;
}

int vti_ctx_create(int device, vti_ctx** out) {
  if (!out) return VTI_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return VTI_ERR_DEVICE;
  vti_ctx* c = new vti_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) !=
          cudaSuccess ||
      cudaMalloc((void**)&c->d_status, 16) != cudaSuccess ||
      cudaMemset(c->d_status, 0, 16) != cudaSuccess) {
    delete c;
    return VTI_ERR_DEVICE;
  }
  c->d_cfl = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(c->d_status) + 8);
  *out = c;
  return VTI_OK;
}

int vti_ctx_destroy(vti_ctx* ctx) {
  if (!ctx) return VTI_OK;
  cudaSetDevice(ctx->device);
  vti_ctx_set_plan_cache(ctx, 0);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    release_events(ctx);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->stream);
  }
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->scratch2d) cudaFree(ctx->scratch2d);
  delete ctx;
  return VTI_OK;
}

int vti_ctx_check_bounded_wait(vti_ctx* ctx, unsigned polls) {
  if (!ctx) return VTI_ERR_ARG;
  return wait_selftest(ctx, polls);
}

int vti_ctx_set_2d_resident(vti_ctx* ctx, int enable) {
  if (!ctx) return VTI_ERR_ARG;
  ctx->resident2d = enable != 0;
  return VTI_OK;
}

const char* vti_status_string(int status) {
  switch (status) {
    case VTI_OK: return "ok";
    case VTI_ERR_ARG: return "invalid argument";
    case VTI_ERR_CFL: return "time step violates the stability bound";
    case VTI_ERR_OOM: return "device out of memory";
    case VTI_ERR_DEVICE: return "CUDA error";
    case VTI_ERR_TIMEOUT: return "device-side wait timed out";
    case VTI_ERR_NONFINITE: return "non-finite wavefield or misfit";
    case VTI_ERR_UNSUPPORTED: return "unsupported request";
    case VTI_ERR_BUSY: return "busy (memory budget full or job not finished)";
    default: return "unknown status";
  }
}

const char* vti_ctx_last_error(const vti_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

void* vti_ctx_stream(vti_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

uint64_t vti_ctx_kernel_launches(const vti_ctx* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"
