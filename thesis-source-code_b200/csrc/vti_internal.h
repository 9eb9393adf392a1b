// Internal declarations shared by the libvti_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "vti_b200.h"

namespace vti {

// Half width of the 8th-order stencil (lib/vti-fwi-3d/gpu/wave3d.h:19).
constexpr int kHalo = 4;
// z planes of zeros kept above and below every device volume so the z
// stencil never needs a bounds test (the reference pads with zero planes in
// its top/bottom kernels, kernel3d.cu:92,409).
constexpr int kZPad = kHalo;
// The reference pipeline advances 64 steps per block visit
// (wave3d.h:17) and therefore runs 2 + 64*floor((nt-2)/64) time levels.
constexpr int kRefUpdate = 64;

// Recording / injection weights (wave3d.h:5-6).
constexpr double kTwoThird = 0.6666666666;
constexpr double kOneThird = 0.3333333333;

// A device volume: x-fastest rows of `pitch` floats, ny rows per plane,
// nz planes plus kZPad zero planes on each side. `origin` points at
// element (0,0,0).
struct Vol {
  float* alloc = nullptr;
  float* origin = nullptr;
  size_t bytes = 0;
};

struct Dims3 {
  int nx, ny, nz;
  int pitch;          // floats per row (multiple of 32)
  long long plane;    // floats per plane = pitch * ny
  __host__ __device__ long long npoints() const { return (long long)nx * ny * nz; }
  __host__ __device__ long long off(int x, int y, int z) const {
    return (long long)z * plane + (long long)y * pitch + x;
  }
};

}  // namespace vti

namespace vti {
// Kernels whose launches can be timed with CUDA events (vti_ctx_set_timing).
enum TimedKernel { kTimedFwd3d = 0, kTimedBwd3d = 1, kTimedStep2d = 2, kNumTimed = 3 };
}  // namespace vti

struct vti_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  uint64_t launches = 0;
  int sm_count = 0;
  // device status word written by kernels (0 = ok); the same allocation holds
  // the stability-number reduction slot at byte 8
  int* d_status = nullptr;
  unsigned long long* d_cfl = nullptr;
  // optional per-kernel timing: event pairs recorded around timed launches
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events[vti::kNumTimed];
  std::vector<cudaEvent_t> event_pool;
  // 2D traces of grids that fit one thread-block cluster run shared-memory resident
  bool resident2d = true;
  // device scratch of the 2D forward forms, kept between calls
  float* scratch2d = nullptr;
  size_t scratch2d_bytes = 0;
  // plan kept by the one-call 3D forms while their geometry and flags repeat
  bool plan_cache = true;
  vti3d_plan* cached_plan = nullptr;
  vti3d_geom cached_geom{};
  unsigned cached_flags = 0;
};

namespace vti {
// NVTX range for the lifetime of the object (header-only NVTX v3: a no-op
// unless a profiler is attached). Names the passes and calls of the path in
// timeline tools.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
// Launch with programmatic stream serialization: the kernel may start while
// the previous kernel of the stream runs; it must execute griddepcontrol.wait
// before it touches anything the previous kernels write (launched normally,
// the wait returns at once).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}
// Brackets one launch with events on ctx->stream when timing is enabled.
struct LaunchTimer {
  vti_ctx* ctx;
  int kind;
  cudaEvent_t stop = nullptr;
  LaunchTimer(vti_ctx* c, int k);
  ~LaunchTimer();
};
}  // namespace vti

namespace vti {

// Sets ctx->last_error and returns the status.
int fail(vti_ctx* ctx, int status, const std::string& msg);
// Converts a CUDA error to a status (and message) if any.
int cuda_check(vti_ctx* ctx, cudaError_t e, const char* what);

#define VTI_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::vti::cuda_check(ctx, e_, #call); \
  } while (0)

#define VTI_LAUNCHED(ctx, what)                                              \
  do {                                                                       \
    (ctx)->launches++;                                                       \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess) return ::vti::cuda_check(ctx, e_, what);          \
  } while (0)

int vol_alloc(vti_ctx* ctx, const Dims3& d, Vol* v);
void vol_free(Vol* v);
// Zero the whole allocation (data and pad planes).
int vol_zero(vti_ctx* ctx, const Dims3& d, Vol* v);
// Contiguous x-fastest host/device array <-> pitched volume.
int vol_upload(vti_ctx* ctx, const Dims3& d, Vol* v, const float* src, int mem);
int vol_download(vti_ctx* ctx, const Dims3& d, const Vol* v, float* dst, int mem);

Dims3 make_dims(int nx, int ny, int nz);

// -------------------------------------------------------------- kernels
struct Damping {
  const float* x;  // nx
  const float* y;  // ny
  const float* z;  // nz
};

struct PointSource {
  int x = -1, y = -1, z = -1;  // grid indices; x < 0 disables
  float amp = 0.f;             // added to next before the sponge
};

// One grid point of the new level read out by the step kernel:
// *out += next_x + next_z as the stencil computed it (before the source and
// the sponge). x < 0 disables.
struct Probe {
  int x = -1, y = -1, z = -1;
  float* out = nullptr;
};

// TMA descriptors (CUtensorMap, 128 bytes each) of one volume: 32 x 16 tiles
// and 40 x 24 tiles (with the 4-cell halo). Plain storage keeps cuda.h out
// of this header.
struct TileMaps {
  alignas(64) unsigned char plain[128];
  alignas(64) unsigned char halo[128];
  const float* origin = nullptr;  // plane 0 of the volume (FP32 volumes; kernels that read it directly)
};
int make_tile_maps(vti_ctx* ctx, const Dims3& d, const Vol& v, TileMaps* out);
// Single-grid step schedule of d with ctas_per_sm resident CTAs: returns its
// modelled duration in CTA-slot plane-steps (waves x (segment + restart) x
// slots); *work = the plane-steps of useful work (columns x planes).
long long step_sched_cost(vti_ctx* ctx, const Dims3& d, int ctas_per_sm, long long* work);
// The same over a volume of `elem_bytes` (4: float, 2: bfloat16) elements
// with the layout of Vol (alloc = start of the pad planes).
int make_tile_maps_typed(vti_ctx* ctx, const Dims3& d, void* alloc, int elem_bytes,
                         TileMaps* out);

// One forward-form leapfrog step over the update region (x,y in [4,n-4),
// all z): next written through px_ptr/pz_ptr (prev is read through the px/pz
// maps; the same volume for an in-place step); damp == nullptr: no sponge
// (random-boundary pass); exact: the sponge as a plain diagonal (exact-mode
// operator). TMA-pipelined, see vti_tma3d.cu.
int launch_fwd3d_tma(vti_ctx* ctx, const Dims3& d, const TileMaps& cx, const TileMaps& cz,
                     const TileMaps& px, const TileMaps& pz, const TileMaps& c11,
                     const TileMaps& c13, const TileMaps& c33, const float* cz_ptr,
                     float* px_ptr, float* pz_ptr, const Damping* damp, float sx, float sy,
                     float sz, PointSource src, Probe probe = Probe(), bool exact = false);
// Fused backward step: sigma back one level (gradient form, no sponge, +src),
// adjoint lambda one level (forward form, sponge), zero-lag imaging into g
// (rtm: the RTM image in g11 instead).
int launch_bwd3d_tma(vti_ctx* ctx, const Dims3& d, const TileMaps& scx, const TileMaps& scz,
                     const TileMaps& spx, const TileMaps& spz, const TileMaps& lcx,
                     const TileMaps& lcz, const TileMaps& lpx, const TileMaps& lpz,
                     const TileMaps& c11, const TileMaps& c13, const TileMaps& c33,
                     const TileMaps& g11, const TileMaps& g13, const TileMaps& g33,
                     const float* scz_ptr, const float* lcz_ptr, float* spx_ptr, float* spz_ptr,
                     float* lpx_ptr, float* lpz_ptr, float* g11_ptr, float* g13_ptr,
                     float* g33_ptr, const Damping& damp, float dt2, float idx2, float idy2,
                     float idz2, float sx, float sy, float sz, PointSource src, bool rtm);

// One job of a batched forward launch (k_fwd3d_tma over the items of many
// volumes). Step s = tick - t0 of the job uses parity p = s & 1:
// cur = cx[p]/cz[p], prev in and next out = px[p]/pz[p]; the source gets
// amp[s] (device array).
struct FwdJobSpec {
  Dims3 d;
  const TileMaps* cx[2];
  const TileMaps* cz[2];
  const TileMaps* px[2];
  const TileMaps* pz[2];
  const TileMaps* c[3];
  const float* cz_ptr[2];
  float* px_ptr[2];
  float* pz_ptr[2];
  const Damping* damp;  // null: no sponge
  float sx, sy, sz;
  int src_x, src_y, src_z;
  const float* amp;
  int t0;
  int seg;  // planes per z-segment; 0: the single-launch schedule
};
// One job of a batched backward launch (roles as launch_bwd3d_tma, by parity).
struct BwdJobSpec {
  Dims3 d;
  const TileMaps* scx[2];
  const TileMaps* scz[2];
  const TileMaps* spx[2];
  const TileMaps* spz[2];
  const TileMaps* lcx[2];
  const TileMaps* lcz[2];
  const TileMaps* lpx[2];
  const TileMaps* lpz[2];
  const TileMaps* c[3];
  const TileMaps* g[3];
  const float* scz_ptr[2];
  const float* lcz_ptr[2];
  float* spx_ptr[2];
  float* spz_ptr[2];
  float* lpx_ptr[2];
  float* lpz_ptr[2];
  float* g_ptr[3];
  Damping damp;
  float dt2, idx2, idy2, idz2, sx, sy, sz;
  int src_x, src_y, src_z;
  const float* amp;
  int t0;
  int seg;
};
// A batched step launch plan: the jobs' arguments as kernel parameter blocks
// (chunks of at most 128 forward / 96 backward jobs, one launch each) and
// their TMA descriptors on the device.
struct StepBatch;
int fwd_batch_build(vti_ctx* ctx, const FwdJobSpec* spec, int njobs, StepBatch** out);
int bwd_batch_build(vti_ctx* ctx, const BwdJobSpec* spec, int njobs, StepBatch** out);
// Launches every chunk for step `tick` on the context stream.
int step_batch_launch(vti_ctx* ctx, StepBatch* b, int tick);
// Kernel launches per step_batch_launch.
int step_batch_launches(const StepBatch* b);
void step_batch_free(StepBatch* b);
// Sets the batched kernels' launch attributes (before any stream capture).
int prepare_batch_kernels(vti_ctx* ctx);

// k_wait_selftest with `polls` polls; returns the status it leaves.
int wait_selftest(vti_ctx* ctx, unsigned polls);
// Reads (and clears) the device status word; VTI_ERR_TIMEOUT if a bounded
// device-side wait gave up since the last check.
int check_device_status(vti_ctx* ctx);

// Sparse receiver kernels. rec: device offsets (Dims3::off) per receiver.
int launch_record(vti_ctx* ctx, float* trace, int nnt, int j, const float* cx, const float* cz,
                  const long long* rec, int nr);
int launch_inject_residual(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                           int i0, float f, int clamp_last, const long long* rec,
                           const float* rec_damp, int nr, float dt2);
int launch_seed_adjoint(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                        const long long* rec, const float* rec_damp, int nr, float dt2);
int launch_set_point(vti_ctx* ctx, float* a, float* b, long long off, float value);
// Offset-domain gathers of one backward level: image holds 2*nlag+1 volumes
// of d.plane*d.nz floats (pitched rows, no z pad planes), lag -nlag first;
// sx, sz, lx, lz are the level's current source and receiver wavefields.
int launch_odcig3d(vti_ctx* ctx, const Dims3& d, const float* sx, const float* sz,
                   const float* lx, const float* lz, const Damping& damp, int nlag,
                   float* image);
// res <- modeled - observed (dead receivers: modeled zeroed first);
// acc[0] += sum(res^2) in FP64, reproducibly; acc must hold
// 1 + residual_blocks(ctx) doubles. obs == nullptr: only zero dead traces.
int launch_residual(vti_ctx* ctx, float* trace, const float* obs, const unsigned char* live,
                    int nnt, int nr, double* acc);
int residual_blocks(vti_ctx* ctx);
// trace[it + ir*nnt] *= (ot + it*dt)^p (the reference's tpow gain).
int launch_tpower(vti_ctx* ctx, float* trace, int nnt, int nr, float ot, float dt, float p);
// AGC misfit: trace (modeled, dead traces already zeroed) becomes the AGC
// adjoint source; part (nr doubles) gets the per-trace misfits and acc[0]
// their fixed-order sum.
int launch_agc_adjoint(vti_ctx* ctx, float* trace, const float* obs, int nnt, int nr, int hw,
                       double* part, double* acc);
int launch_boundary_merge(vti_ctx* ctx, const Dims3& d, int npad, const float* full,
                          const float* blist, float* out);
// VTI_ERR_NONFINITE bit of the status word if a[0, n) holds a NaN or Inf.
int launch_check_finite(vti_ctx* ctx, const float* a, long long n);
// nr traces of nnt FP16 samples (trace-major) times the per-sample scales
// into FP32 traces.
int launch_unpack_traces_f16(vti_ctx* ctx, const uint16_t* src, const float* scale, int nnt,
                             int nr, float* dst);
// *out (zeroed by the caller) <- bits of max over the volume of the largest
// eigenvalue of [[c11 kh, c13 kz], [c13 kh, c33 kz]]; dt^2 times it is the
// number vti3d_cfl_number returns.
int launch_cfl_max(vti_ctx* ctx, const Dims3& d, const float* c11, const float* c13,
                   const float* c33, double kh, double kz, unsigned long long* out);
// Nyquist symbol factors of the 8th-order second derivative per axis:
// |C0 + 2 sum (-1)^k C_k| / h^2 (0 for an absent axis).
double nyquist_factor(double h);
// Stability number of a device-resident pitched model (three volumes at
// their origin planes) of geometry g: dt^2 * max lambda over the grid.
int cfl3d_device(vti_ctx* ctx, const vti3d_geom& g, const Dims3& d, const float* c11,
                 const float* c13, const float* c33, double* number);
// cfl_verdict of vti2d_cfl_number for a 2D model (non-null arrays).
int check_cfl2d(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                const float* c33);
// VTI_ERR_CFL (with the number in the context's message) when
// dt^2 lambda_max >= 4, the leapfrog bound; VTI_OK otherwise.
int cfl_verdict(vti_ctx* ctx, double number, const char* what);

}  // namespace vti
