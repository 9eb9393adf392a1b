// 3D VTI pseudo-acoustic kernels for sm_100a.
//
// Data layout: every volume is x-fastest with a row pitch that is a multiple
// of 32 floats and kZPad zero planes above and below (vti_internal.h).
//
// Update region and arithmetic follow the reference:
//   * x,y in [4, n-4), z in [0, nz) with zero planes outside
//     (lib/vti-fwi-3d/gpu/kernel3d.cu:7-10, 92, 409);
//   * sigma_x carries the horizontal stencil, sigma_z the vertical one;
//     next = c11*Lxy + c13*Lz + 2cur - prev,  next_z = c13*Lxy + c33*Lz + ...
//     (kernel3d.cu:54-69), and the gradient form dt2*(c*L/dx2)
//     (kernel3d.cu:273-293) for the time-reversed source wavefield;
//   * the sponge (abc3d.cu:82-126) damps next and cur of each 4-plane block
//     after that block is updated, in z order. Stored values here are the
//     once-damped levels v_t; prev is read as d*v_{t-2} and the z stencil
//     multiplies the four planes of the block above by d (they have already
//     been damped as "cur" when the reference reaches this block).
//
// The step kernels themselves (TMA-staged 2.5D blocking) are in
// vti_tma3d.cu; this file holds the sparse per-receiver kernels and the
// device side of the boundary merge and the misfit.
#include <cuda_fp16.h>

#include "vti_internal.h"

namespace vti {
namespace {

// ------------------------------------------------------ sparse kernels
// recordData (injectRecord3d.cu:22-28) into trace-major traces.
__global__ void k_record(float* trace, int nnt, int j, const float* cx, const float* cz,
                         const long long* rec, int nr) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    long long o = rec[ir];
    trace[(long long)ir * nnt + j] = (float)(kTwoThird * cx[o] + kOneThird * cz[o]);
  }
}

// injectResidual with the interpolation of interpolateResidual
// (injectRecord3d.cu:38-46,60-78); the sponge factor of the receiver point is
// applied because the step kernel has already damped next.
__global__ void k_inject_residual(float* lx, float* lz, const float* res, int nnt, int i0,
                                  float f, int clamp_last, const long long* rec,
                                  const float* rec_damp, int nr, float dt2) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    const float* t = res + (long long)ir * nnt;
    float r = clamp_last ? t[nnt - 1] : (float)((1. - f) * t[i0] + f * t[i0 + 1]);
    float s = dt2 * r;
    long long o = rec[ir];
    float d = rec_damp[ir];
    lx[o] += d * (float)(kTwoThird * s);
    lz[o] += d * (float)(kOneThird * s);
  }
}

// objFuncGradient3d_f.cu:922-927: adjoint seeded by assignment.
__global__ void k_seed_adjoint(float* lx, float* lz, const float* res, int nnt,
                               const long long* rec, const float* rec_damp, int nr, float dt2) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr && rec_damp[ir] != 0.f) {
    float temp = dt2 * res[(long long)ir * nnt + nnt - 1];
    long long o = rec[ir];
    lx[o] = (float)(kTwoThird * temp);
    lz[o] = (float)(kOneThird * temp);
  }
}

__global__ void k_set_point(float* a, float* b, long long off, float value) {
  a[off] = value;
  b[off] = value;
}

// Residual + FP64 misfit (objFuncGradient3d_f.cu:735-771). Each block writes
// its partial sum; k_sum_partials adds them in a fixed order, so the misfit is
// bitwise reproducible run to run.
__global__ void k_residual(float* trace, const float* obs, const unsigned char* live, int nnt,
                           int nr, double* partial) {
  long long n = (long long)nnt * nr;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int ir = (int)(i / nnt);
    float m = live[ir] ? trace[i] : 0.f;
    if (!obs) {
      trace[i] = m;
      continue;
    }
    float r = m - obs[i];
    trace[i] = r;
    s += (double)(r * r);
  }
  if (!partial) return;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// acc[0] += sum(partial[0..n)) in a fixed order (one warp).
__global__ void k_sum_partials(const double* partial, int n, double* acc) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) v += partial[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) acc[0] += v;
}

// tpower (lib/vti-fwi-3d/gpu/agc.cpp:104-116): trace[it + ir*nnt] *= (ot + it*dt)^p,
// the time in float as the reference computes it.
__global__ void k_tpower(float* trace, int nnt, int nr, float ot, float dt, float p) {
  const long long n = (long long)nnt * nr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int it = (int)(i % nnt);
    const float t = ot + it * dt;
    trace[i] *= powf(t, p);
  }
}

// residualAGC (agc.cpp:62-99), one block per trace: AGC of the modeled and the
// observed trace (windowed energy over it-hw..it+hw, indices wrapping around
// the trace, runsum :14-25), residual of the two, its misfit into part[ir]
// (float squares summed in double, fixed order), and the adjoint source
// rs - d * runsum(d * rs / max(EPS, s)) written over the modeled trace.
// Shared memory: 5 * nnt floats.
constexpr float kAgcEps = 1e-6f;  // agc.cpp:10

__device__ __forceinline__ float runsum_at(const float* w, int nnt, int hw, int i) {
  float s = 0.f;
  for (int j = i - hw; j <= i + hw; ++j) s += w[j < 0 ? j + nnt : (j >= nnt ? j - nnt : j)];
  return s;
}

__global__ void k_agc_adjoint(float* trace, const float* obs, int nnt, int hw, double* part) {
  extern __shared__ float sm[];
  float* d = sm;              // modeled trace
  float* e = d + nnt;         // d^2
  float* e0 = e + nnt;        // d0^2
  float* drss = e0 + nnt;     // d * rs / max(EPS, s)
  float* rs = drss + nnt;     // res / sqrt(max(EPS, s))
  __shared__ double red[32];
  float* tr = trace + (long long)blockIdx.x * nnt;
  const float* ob = obs + (long long)blockIdx.x * nnt;
  for (int i = threadIdx.x; i < nnt; i += blockDim.x) {
    const float v = tr[i], v0 = ob[i];
    d[i] = v;
    e[i] = v * v;
    e0[i] = v0 * v0;
  }
  __syncthreads();
  double fi = 0.0;
  for (int i = threadIdx.x; i < nnt; i += blockDim.x) {
    const float sd = runsum_at(e, nnt, hw, i), sd0 = runsum_at(e0, nnt, hw, i);
    const float hd = d[i] / sqrtf(fmaxf(kAgcEps, sd));
    const float hd0 = ob[i] / sqrtf(fmaxf(kAgcEps, sd0));
    const float res = hd - hd0;
    fi += (double)(res * res);
    const float t1 = fmaxf(kAgcEps, sd);
    const float t2 = res / sqrtf(t1);
    drss[i] = d[i] * t2 / t1;
    rs[i] = t2;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nnt; i += blockDim.x)
    tr[i] = rs[i] - d[i] * runsum_at(drss, nnt, hw, i);
  // block reduction of the misfit in a fixed order
  for (int o = 16; o > 0; o >>= 1) fi += __shfl_down_sync(0xffffffffu, fi, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = fi;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += red[w];
    part[blockIdx.x] = s;
  }
}

// putBoundary applied on the device: out = full, with the pad region replaced
// by the boundary list (order of boundary.cpp:10-46).
__global__ void k_boundary_merge(Dims3 d, int npad, const float* full, const float* blist,
                                 float* out) {
  long long n = d.npoints();
  const long long nxy = (long long)d.nx * d.ny;
  const long long top = nxy * npad;
  const long long mid_plane = 2LL * npad * d.nx + (long long)(d.ny - 2 * npad) * 2 * npad;
  const long long mid_total = (long long)(d.nz - 2 * npad) * mid_plane;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int x = (int)(t % d.nx);
    int y = (int)((t / d.nx) % d.ny);
    int z = (int)(t / nxy);
    long long k = -1;
    if (z < npad) {
      k = x + (long long)y * d.nx + (long long)z * nxy;
    } else if (z >= d.nz - npad) {
      k = top + mid_total + x + (long long)y * d.nx + (long long)(z - (d.nz - npad)) * nxy;
    } else {
      long long base = top + (long long)(z - npad) * mid_plane;
      if (y < npad) {
        k = base + x + (long long)y * d.nx;
      } else if (y >= d.ny - npad) {
        k = base + (long long)npad * d.nx + (long long)(d.ny - 2 * npad) * 2 * npad + x +
            (long long)(y - (d.ny - npad)) * d.nx;
      } else {
        long long rb = base + (long long)npad * d.nx + (long long)(y - npad) * 2 * npad;
        if (x < npad) k = rb + x;
        else if (x >= d.nx - npad) k = rb + npad + (x - (d.nx - npad));
      }
    }
    long long o = d.off(x, y, z);
    out[o] = k >= 0 ? blist[k] : full[o];
  }
}

// Offset-domain image gathers of one backward level (extendedImagingKernel,
// lib/vti-fwi-3d/gpu/wave3d.cu:1299-1313, on this library's RTM pair): with
// S(p) = 2/3 sx + 1/3 sz and R(p) = sponge(p) (2/3 lx + 1/3 lz) at the step's
// current level, evaluated with the operations of the zero-lag image of the
// fused backward kernel, image[lag][p] = fma(S(p), R(p + lag), image[lag][p])
// for |lag| <= nlag (x offsets) and x in [xlo, xhi). One block: 128 points
// of one row; R of the row segment and its nlag-wide margins staged in
// shared memory.
constexpr int kOdcigTX = 128;
constexpr float kTwoThirdF = (float)kTwoThird, kOneThirdF = (float)kOneThird;

__global__ void __launch_bounds__(kOdcigTX)
    k_odcig3d(Dims3 d, const float* sx, const float* sz, const float* lx, const float* lz,
              const float* dampx, const float* dampy, const float* dampz, int nlag, int xlo,
              int xhi, float* image, long long lag_stride) {
  extern __shared__ float rs[];  // R at x0 - nlag .. x0 + kOdcigTX + nlag - 1
  const int x0 = blockIdx.x * kOdcigTX;
  const int y = kHalo + blockIdx.y;
  const int z = blockIdx.z;
  const float dz = dampz[z], dy = dampy[y];
  const long long row = (long long)z * d.plane + (long long)y * d.pitch;
  for (int t = threadIdx.x; t < kOdcigTX + 2 * nlag; t += kOdcigTX) {
    const int xr = x0 - nlag + t;
    float r = 0.f;
    if (xr >= 0 && xr < d.nx) {
      const float dd = (dampx[xr] * dy) * dz;
      r = dd * fmaf(kTwoThirdF, lx[row + xr], kOneThirdF * lz[row + xr]);
    }
    rs[t] = r;
  }
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x < xlo || x >= xhi) return;
  const float sv = fmaf(kTwoThirdF, sx[row + x], kOneThirdF * sz[row + x]);
  float* img = image + row + x;
  for (int lag = -nlag; lag <= nlag; ++lag) {
    float* q = img + (long long)(lag + nlag) * lag_stride;
    *q = fmaf(sv, rs[threadIdx.x + nlag + lag], *q);
  }
}

}  // namespace

int launch_odcig3d(vti_ctx* ctx, const Dims3& d, const float* sx, const float* sz,
                   const float* lx, const float* lz, const Damping& damp, int nlag,
                   float* image) {
  const int xlo = nlag > kHalo ? nlag : kHalo;
  const int xhi = d.nx - xlo;
  if (xhi <= xlo || d.ny <= 2 * kHalo || d.nz < 1) return VTI_OK;
  dim3 grid((d.nx + kOdcigTX - 1) / kOdcigTX, d.ny - 2 * kHalo, d.nz);
  const size_t smem = (kOdcigTX + 2 * (size_t)nlag) * sizeof(float);
  k_odcig3d<<<grid, kOdcigTX, smem, ctx->stream>>>(d, sx, sz, lx, lz, damp.x, damp.y, damp.z,
                                                   nlag, xlo, xhi, image,
                                                   d.plane * (long long)d.nz);
  VTI_LAUNCHED(ctx, "k_odcig3d");
  return VTI_OK;
}

int launch_record(vti_ctx* ctx, float* trace, int nnt, int j, const float* cx, const float* cz,
                  const long long* rec, int nr) {
  if (nr <= 0) return VTI_OK;
  k_record<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(trace, nnt, j, cx, cz, rec, nr);
  VTI_LAUNCHED(ctx, "k_record");
  return VTI_OK;
}

int launch_inject_residual(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                           int i0, float f, int clamp_last, const long long* rec,
                           const float* rec_damp, int nr, float dt2) {
  if (nr <= 0) return VTI_OK;
  k_inject_residual<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(lx, lz, res, nnt, i0, f,
                                                               clamp_last, rec, rec_damp, nr, dt2);
  VTI_LAUNCHED(ctx, "k_inject_residual");
  return VTI_OK;
}

int launch_seed_adjoint(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                        const long long* rec, const float* rec_damp, int nr, float dt2) {
  if (nr <= 0) return VTI_OK;
  k_seed_adjoint<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(lx, lz, res, nnt, rec, rec_damp, nr,
                                                            dt2);
  VTI_LAUNCHED(ctx, "k_seed_adjoint");
  return VTI_OK;
}

int launch_set_point(vti_ctx* ctx, float* a, float* b, long long off, float value) {
  k_set_point<<<1, 1, 0, ctx->stream>>>(a, b, off, value);
  VTI_LAUNCHED(ctx, "k_set_point");
  return VTI_OK;
}

int residual_blocks(vti_ctx* ctx) { return ctx->sm_count * 8; }

int launch_residual(vti_ctx* ctx, float* trace, const float* obs, const unsigned char* live,
                    int nnt, int nr, double* acc) {
  long long n = (long long)nnt * nr;
  if (n <= 0) return VTI_OK;
  int blocks = (int)std::min<long long>((n + 255) / 256, (long long)residual_blocks(ctx));
  // acc[0] is the running sum, acc[1 .. 1+residual_blocks) the partials
  k_residual<<<blocks, 256, 0, ctx->stream>>>(trace, obs, live, nnt, nr, acc ? acc + 1 : nullptr);
  VTI_LAUNCHED(ctx, "k_residual");
  if (acc) {
    k_sum_partials<<<1, 32, 0, ctx->stream>>>(acc + 1, blocks, acc);
    VTI_LAUNCHED(ctx, "k_sum_partials");
  }
  return VTI_OK;
}

int launch_tpower(vti_ctx* ctx, float* trace, int nnt, int nr, float ot, float dt, float p) {
  const long long n = (long long)nnt * nr;
  if (n <= 0) return VTI_OK;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 8);
  k_tpower<<<blocks, 256, 0, ctx->stream>>>(trace, nnt, nr, ot, dt, p);
  VTI_LAUNCHED(ctx, "k_tpower");
  return VTI_OK;
}

int launch_agc_adjoint(vti_ctx* ctx, float* trace, const float* obs, int nnt, int nr, int hw,
                       double* part, double* acc) {
  if (nnt <= 0 || nr <= 0) return VTI_OK;
  const size_t smem = 5 * (size_t)nnt * sizeof(float);
  if (smem > 200 * 1024)
    return fail(ctx, VTI_ERR_UNSUPPORTED, "AGC misfit: trace longer than 10240 samples");
  if (hw < 0 || 2 * hw + 1 > nnt)
    return fail(ctx, VTI_ERR_ARG, "AGC half width must satisfy 0 <= 2*halfwidth+1 <= nnt");
  VTI_CUDA(ctx, cudaFuncSetAttribute(k_agc_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  k_agc_adjoint<<<nr, 256, smem, ctx->stream>>>(trace, obs, nnt, hw, part);
  VTI_LAUNCHED(ctx, "k_agc_adjoint");
  k_sum_partials<<<1, 32, 0, ctx->stream>>>(part, nr, acc);
  VTI_LAUNCHED(ctx, "k_sum_partials");
  return VTI_OK;
}

namespace {
// dt^2-free stability number of every point: the largest eigenvalue of
// [[c11 kh, c13 kz], [c13 kh, c33 kz]] (the symbol of the scheme at the
// Nyquist wavenumber, as vti3d_cfl_number evaluates it), in double; the
// maximum is reduced with an atomic max on the bit pattern (non-negative
// doubles order like their bits; a NaN model value wins and is rejected).
__global__ void k_cfl_max(Dims3 d, const float* c11, const float* c13, const float* c33,
                          double kh, double kz, unsigned long long* out) {
  const long long n = (long long)d.nx * d.ny * d.nz;
  double worst = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % d.nx);
    const long long yz = t / d.nx;
    const long long o = (yz / d.ny) * d.plane + (yz % d.ny) * d.pitch + x;
    const double a = c11[o] * kh, b = c13[o] * kz, c = c13[o] * kh, e = c33[o] * kz;
    const double tr = a + e, det = a * e - b * c;
    const double disc = tr * tr * 0.25 - det;
    const double lam = tr * 0.5 + sqrt(disc > 0 ? disc : 0.0);
    if (!(lam <= worst)) worst = lam;
  }
  unsigned long long bits = __double_as_longlong(worst);
  for (int k = 16; k > 0; k >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, k);
    bits = other > bits ? other : bits;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}
}  // namespace

namespace {
// Sets the VTI_ERR_NONFINITE bit of the status word if any of a[0, n) is NaN
// or infinite.
__global__ void k_check_finite(const float* a, long long n, int* status) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(a[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0)
    atomicOr(status, 1 << VTI_ERR_NONFINITE);
}
}  // namespace

int launch_check_finite(vti_ctx* ctx, const float* a, long long n) {
  if (n <= 0) return VTI_OK;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 8);
  k_check_finite<<<blocks, 256, 0, ctx->stream>>>(a, n, ctx->d_status);
  VTI_LAUNCHED(ctx, "k_check_finite");
  return VTI_OK;
}

namespace {
// 16-bit traces in flight: sample t of every trace is h * scale[t], h an
// IEEE half. One block per trace, threads along time (contiguous).
__global__ void k_unpack_traces_f16(const __half* src, const float* scale, int nnt,
                                    float* dst) {
  const long long row = (long long)blockIdx.x * nnt;
  for (int t = threadIdx.x; t < nnt; t += blockDim.x)
    dst[row + t] = __half2float(src[row + t]) * scale[t];
}
}  // namespace

int launch_unpack_traces_f16(vti_ctx* ctx, const uint16_t* src, const float* scale, int nnt,
                             int nr, float* dst) {
  if (nr <= 0) return VTI_OK;
  k_unpack_traces_f16<<<nr, 256, 0, ctx->stream>>>(reinterpret_cast<const __half*>(src), scale,
                                                  nnt, dst);
  VTI_LAUNCHED(ctx, "k_unpack_traces_f16");
  return VTI_OK;
}

int launch_cfl_max(vti_ctx* ctx, const Dims3& d, const float* c11, const float* c13,
                   const float* c33, double kh, double kz, unsigned long long* out) {
  const long long n = (long long)d.nx * d.ny * d.nz;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 8);
  k_cfl_max<<<blocks, 256, 0, ctx->stream>>>(d, c11, c13, c33, kh, kz, out);
  VTI_LAUNCHED(ctx, "k_cfl_max");
  return VTI_OK;
}

int launch_boundary_merge(vti_ctx* ctx, const Dims3& d, int npad, const float* full,
                          const float* blist, float* out) {
  long long n = d.npoints();
  int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 16);
  k_boundary_merge<<<blocks, 256, 0, ctx->stream>>>(d, npad, full, blist, out);
  VTI_LAUNCHED(ctx, "k_boundary_merge");
  return VTI_OK;
}

}  // namespace vti
