/*
 * vti_b200.h — C ABI of the B200-native VTI pseudo-acoustic modeling and
 * gradient library (libvti_b200.so).
 *
 * Plain C types only: pointers, sizes, status codes. No CUDA or torch types
 * appear in any signature; device pointers are passed as `void*`/`float*`
 * together with a VTI_MEM_* tag.
 *
 * Array conventions follow the reference (huyleq/thesis-source-code):
 *  - 3D arrays are x-fastest, i = ix + iy*nx + iz*nx*ny, the absorbing pad
 *    inside nx, ny, nz (lib/vti-fwi-3d/gpu/boundary.cpp:10-46).
 *  - 3D traces are time-fastest, data[it + ir*nnt], nnt = (nt-1)/s + 1,
 *    s = round(sampling_rate/dt) (lib/vti-fwi-3d/gpu/modelData3d_f.cu:29-30,272).
 *  - souloc holds 5 floats per shot (x, y, z, nr, irbegin), recloc 4 floats
 *    per receiver (x, y, z, live flag) (objFuncGradient3d_f.cu:551-575).
 *  - "boundary" arrays are the pad-region lists produced by getBoundary
 *    (boundary.cpp:10-46), nb = nx*ny*nz - (nx-2npad)(ny-2npad)(nz-2npad).
 *  - 2D arrays are i = ix + iz*nnx with nnx = nx + 2*npad
 *    (lib/vti-fwi-2d/init.cpp:11-18); 2D traces are receiver-fastest,
 *    data[it*nr + ir] (synthetic_f.cu:110).
 *
 * Every entry point returns a vti_status. On a non-OK status the context's
 * last-error string (vti_ctx_last_error) holds a one-line reason.
 */
#ifndef VTI_B200_H
#define VTI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  VTI_OK = 0,
  VTI_ERR_ARG = 1,        /* invalid argument (sizes, indices, null pointers) */
  VTI_ERR_CFL = 2,        /* dt violates the scheme's stability bound */
  VTI_ERR_OOM = 3,        /* device allocation failed */
  VTI_ERR_DEVICE = 4,     /* a CUDA call failed; see vti_ctx_last_error */
  VTI_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up */
  VTI_ERR_NONFINITE = 6,  /* a wavefield or misfit became NaN/Inf */
  VTI_ERR_UNSUPPORTED = 7, /* valid request this build does not implement */
  VTI_ERR_BUSY = 8         /* not now: engine memory full / job not finished */
} vti_status;

/* where a pointer lives */
#define VTI_MEM_HOST 0
#define VTI_MEM_DEVICE 1

/* option flags (bitwise OR) */
/* Run every time level 0..nt-1. Without it the 3D propagators run the
 * reference pipeline's 2 + 64*floor((nt-2)/64) levels
 * (objFuncGradient3d_f.cu:538-542), so results match it for every nt. */
#define VTI_OPT_FULL_STEPS 1u
/* 3D plans: after each pass the wavefields of its last two levels (a NaN or
 * Inf propagates into every later level), the traces of pass 1 and the
 * gradients of pass 3 are scanned for NaN/Inf, and so is the misfit; the
 * call then returns VTI_ERR_NONFINITE. Costs one read of those volumes per
 * pass. */
#define VTI_OPT_CHECK_FINITE 2u
/* Without VTI_OPT_FULL_STEPS the 3D time levels and the recorded trace
 * samples follow the reference pipeline run on G GPUs (G = its GPUs.size(),
 * default 1): 1 + 64*G*floor((nt-2)/(64*G)) levels, and the samples its
 * record/transfer bookkeeping captures (modelData3d_f.cu:233-275; with a
 * sampling step of 1 or 2 time steps it records only part of the trace). */
#define VTI_OPT_REF_GPUS(g) ((((unsigned)(g)) & 0xffu) << 8)

typedef struct vti_ctx vti_ctx;
typedef struct vti3d_plan vti3d_plan;
typedef struct vti3d_batch vti3d_batch;

typedef struct {
  int nx, ny, nz; /* grid including the absorbing pad; x fastest */
  int nt;         /* time samples of the wavelet / simulation */
  int npad;       /* pad width (sponge and random-boundary region) */
  float ox, oy, oz, ot;
  float dx, dy, dz, dt;
  float sampling_rate; /* trace sampling interval (seconds) */
} vti3d_geom;

typedef struct {
  int nx, nz; /* interior size; arrays are (nx+2npad) x (nz+2npad) */
  int nt, npad;
  float dx, dz, dt;
  float rate; /* trace/snapshot sampling interval */
  float ot;   /* time of sample 0 (<= 0) */
} vti2d_geom;

/* ---------------------------------------------------------------- context */
/* One context per CUDA device; owns the streams and a device error word. */
int vti_ctx_create(int device, vti_ctx** out);
int vti_ctx_destroy(vti_ctx* ctx);
const char* vti_status_string(int status);
const char* vti_ctx_last_error(const vti_ctx* ctx);
/* The CUDA stream (cudaStream_t) all work of this context is ordered on. */
void* vti_ctx_stream(vti_ctx* ctx);
/* Number of library kernels launched on this context so far. */
uint64_t vti_ctx_kernel_launches(const vti_ctx* ctx);
/* Per-kernel device timing with CUDA events on the context stream.
 * enable != 0 starts (and clears) recording; kernel is "fwd3d", "bwd3d" or
 * "step2d". vti_ctx_kernel_time synchronizes the stream and returns the summed
 * device time (ms) and the number of timed launches. */
int vti_ctx_set_timing(vti_ctx* ctx, int enable);
/* 2D traces (vti2d_synthetic) of a grid whose state fits the shared memory of
 * one thread-block cluster (up to 16 CTAs; (nnx-8) <= 1024 columns, e.g.
 * 461 x 261) run with the wavefields resident on chip, one cluster per shot
 * (shots with disjoint receiver ranges in one launch); results are those of
 * the per-step path. enable = 0 forces the per-step path (default 1). */
int vti_ctx_set_2d_resident(vti_ctx* ctx, int enable);
int vti_ctx_kernel_time(vti_ctx* ctx, const char* kernel, double* total_ms, uint64_t* count);
/* Diagnostic (no counterpart in the reference): one CTA waits on a shared-
 * memory mbarrier that nothing arrives at, through the bounded wait of the
 * TMA pipeline kernels but with at most `polls` polls (1..65536). The wait
 * gives up, the kernel sets the context's status word and returns, and this
 * call reports VTI_ERR_TIMEOUT: the path every pipeline stall takes, shown
 * without stalling a real kernel. */
int vti_ctx_check_bounded_wait(vti_ctx* ctx, unsigned polls);

/* ------------------------------------------------------------- host glue */
/* Stability bound of the leapfrog scheme: largest dt^2 * lambda_max(M) over
 * the model, M = [[c11 Kh, c13 Kz],[c13 Kh, c33 Kz]]. Stable iff < 4 (NaN if
 * the model holds a NaN). Every entry point that takes a model refuses one
 * whose number is not below 4 with VTI_ERR_CFL before it computes anything
 * (the reference runs such a model and returns growing garbage). */
double vti3d_cfl_number(const vti3d_geom* g, const float* c11, const float* c13,
                        const float* c33);
/* The same number for a 2D model on its padded (nx+2npad) x (nz+2npad) grid
 * (lib/vti-fwi-2d/kernels.h:4-8 stencil). New entry point, no counterpart in
 * the reference. */
double vti2d_cfl_number(const vti2d_geom* g, const float* c11, const float* c13,
                        const float* c33);
/* getBoundary / putBoundary / zeroBoundary (boundary.cpp:10-117). */
void vti3d_get_boundary(float* boundary, const float* v, int nx, int ny, int nz, int npad);
void vti3d_put_boundary(const float* boundary, float* v, int nx, int ny, int nz, int npad);
void vti3d_zero_boundary(float* v, int nx, int ny, int nz, int npad);
/* VEpsDel2Cij, GradCij2GradVEpsDel, dVEpsDel2dCij, checkEpsDel
 * (lib/vti-fwi-2d/conversions.cpp:42-81, check.cpp:22-40). */
void vti_vepsdel_to_cij(float* c11, float* c13, float* c33, const float* v, const float* eps,
                        const float* del, float v0, float eps0, float del0, size_t n);
void vti_grad_cij_to_vepsdel(float* gv, float* geps, float* gdel, const float* gc11,
                             const float* gc13, const float* gc33, const float* v,
                             const float* eps, const float* del, float v0, float eps0, float del0,
                             size_t n);
void vti_dvepsdel_to_dcij(float* c11, float* c13, float* c33, float* dc11, float* dc13,
                          float* dc33, const float* v, const float* eps, const float* del,
                          const float* dv, const float* deps, const float* ddel, float v0,
                          float eps0, float del0, size_t n);
int vti_check_eps_del(float* eps, float* del, float eps0, float del0, size_t n, float* mask);

/* ------------------------------------------------------------ 3D plans */
/* A plan owns the device-resident state of one 3D geometry: model (pad and
 * random-boundary versions), wavefields, gradient accumulators, traces. */
int vti3d_plan_create(vti_ctx* ctx, const vti3d_geom* g, unsigned flags, vti3d_plan** out);
int vti3d_plan_destroy(vti3d_plan* plan);
/* Model c11,c13,c33 (nxyz each, mem = VTI_MEM_*). padb / randb are the
 * 3*nb boundary lists (c11 list, c13 list, c33 list) swapped into the pad for
 * the sponge pass and the random-boundary passes (objFuncGradient3d_f.cu:594,786);
 * NULL leaves the model's own pad in place. */
int vti3d_plan_set_model(vti3d_plan* plan, const float* c11, const float* c13, const float* c33,
                         const float* padb, const float* randb, int mem);
/* wavelet: nt floats. */
int vti3d_plan_set_wavelet(vti3d_plan* plan, const float* wavelet, int mem);
/* Receivers (host): 4 floats each, the whole survey. */
int vti3d_plan_set_receivers(vti3d_plan* plan, const float* recloc, int nrec_total);
/* Forward modeling with the sponge (modelDataCij3d_f, modelData3d_f.cu:427):
 * ddata gets nnt*nr traces per shot at offset nnt*irbegin. */
int vti3d_plan_model_data(vti3d_plan* plan, const float* souloc, const int* shotid, int nshot,
                          float* ddata, int mem);
/* L2 misfit gradient (objFuncGradientCij3d_f, objFuncGradient3d_f.cu:361):
 * dobs as ddata; fgcij = [misfit/2 (float), gc11, gc13, gc33] (1+3*nxyz).
 * misfit (optional) receives the FP64 sum of squared residuals / 2. */
int vti3d_plan_gradient(vti3d_plan* plan, const float* souloc, const int* shotid, int nshot,
                        const float* dobs, int dobs_mem, float* fgcij, int fgcij_mem,
                        double* misfit);
/* Misfit options of vti3d_plan_gradient (objFuncGradient3d_f.cu:743-775, the
 * tpow= / objtype= / halfwidth= parameters of the reference): the modeled
 * traces are multiplied by (ot + it*sampling_rate)^tpow when tpow != 0 (no
 * chain-rule factor on the adjoint source, as in the reference); objtype 0 is
 * the L2 misfit, any other value the AGC misfit (residualAGC, agc.cpp:62-99,
 * energy window of 2*halfwidth+1 samples wrapping around the trace). The
 * misfit-only entry (vti3d_plan_objfunc) stays plain L2, as objFuncCij3d_f.
 * Defaults: 0, 0, 20. */
int vti3d_plan_set_misfit(vti3d_plan* plan, float tpow, int objtype, int halfwidth);
/* Observed traces in flight as 16 bits. VTI_TRACES_F32 (default): dobs /
 * data arguments are FP32 traces as the reference passes them. VTI_TRACES_F16:
 * they point to a packed block of vti_traces_f16_bytes(nr_total, nnt)
 * bytes made by vti_traces_pack_f16 (host or device memory, per the call's
 * mem argument), which moves half the bytes; each shot's traces are expanded
 * to FP32 on the device before the misfit; the results are bitwise those of
 * the FP32 traces the block stands for (vti_traces_unpack_f16). Plane scales
 * keep every sample at FP16's full relative precision (2^-11). The gradient
 * is linear in the residual, so against the gradient of the original FP32
 * traces it moves by about |dq - d| / |residual| (relative L2, dq the
 * unpacked data): measured 4e-6 with a residual of 91 % of the data and 1e-3
 * with 13 % — a format for early FWI iterations, not for late ones. BF16
 * values move it 12x more and are not offered. */
#define VTI_TRACES_F32 0
#define VTI_TRACES_F16 1
int vti3d_plan_set_trace_format(vti3d_plan* plan, int format);
/* Bytes of a packed block of nr traces of nnt samples: nnt FP32 scales (one
 * per time sample, the maximum |value| over all nr traces at that sample, 1
 * where it is 0) followed by nr*nnt IEEE half values, trace-major. */
size_t vti_traces_f16_bytes(int nr, int nnt);
/* Packs nr FP32 traces of nnt samples (trace-major, host) into a block
 * (host): value / scale rounded to the nearest half (ties to even). Returns
 * VTI_ERR_NONFINITE if a sample is NaN or Inf. */
int vti_traces_pack_f16(const float* traces, int nr, int nnt, void* block);
/* The FP32 traces a block stands for (host). */
int vti_traces_unpack_f16(const void* block, int nr, int nnt, float* traces);
/* Misfit only (objFuncCij3d_f, objFuncGradient3d_f.cu:1272). */
int vti3d_plan_objfunc(vti3d_plan* plan, const float* souloc, const int* shotid, int nshot,
                       const float* dobs, int dobs_mem, double* misfit);
/* Reverse-time migration (rtmCij3d_f, lib/vti-fwi-3d/gpu/rtm3d_f.cu:161-620):
 * image (nxyz, zeroed first) = sum over shots of the zero-lag product
 * (2/3 sx + 1/3 sz)(2/3 lx + 1/3 lz) of the back-propagated source wavefield
 * and the receiver wavefield driven by the traces `data` (nnt x nrec_total,
 * trace-major). Uses the random-boundary model if one was set, else the
 * model; no sponge on the source wavefield. */
int vti3d_plan_rtm(vti3d_plan* plan, const float* souloc, const int* shotid, int nshot,
                   const float* data, int data_mem, float* image, int image_mem);
/* Offset-domain common-image gathers (odcig3d_f, lib/vti-fwi-3d/gpu/odcig3d_f.cu:15,
 * with the imaging condition of extendedImagingKernel, wave3d.cu:1299-1313):
 * the migration of vti3d_plan_rtm with, for every level, image[lag][p] +=
 * (2/3 sx + 1/3 sz)(p) * sponge(p+lag) (2/3 lx + 1/3 lz)(p+lag) for
 * |lag| <= nlag (x offsets; the reference fixes nlag = 32, wave3d.h:19), at
 * x in [max(4,nlag), nx-max(4,nlag)), y in [4, ny-4), all z; zero elsewhere.
 * image: (2*nlag+1) * nxyz floats, lag -nlag first; its lag-0 volume equals
 * the vti3d_plan_rtm image on those x (bit for bit). 0 <= nlag <= 1024. */
int vti3d_plan_odcig(vti3d_plan* plan, const float* souloc, const int* shotid, int nshot,
                     const float* data, int data_mem, int nlag, float* image, int image_mem);
/* Wavelet gradient (waveletGradientCij3d_f, lib/vti-fwi-3d/gpu/modelData3d_f.cu:858):
 * gwavelet (nt) = dt2 * sum over shots and levels of lambda_x + lambda_z at the
 * source, the adjoint wavefield driven by the traces `data` (nnt x nrec_total)
 * with the sponge and the model's pad (the random boundary is not used). */
int vti3d_plan_wavelet_gradient(vti3d_plan* plan, const float* souloc, const int* shotid,
                                int nshot, const float* data, int data_mem, float* gwavelet,
                                int mem);
/* Device pointer of the last forward wavefield sigma_x (pitched volume). */
const float* vti3d_plan_wavefield(vti3d_plan* plan);
/* Copies the last forward level of sigma_x (the "wavefield" output of
 * modelData3d_f.cu:324 / modeling3d_f.cu:266) into nxyz contiguous floats. */
int vti3d_plan_get_wavefield(vti3d_plan* plan, float* out, int mem);

/* One-call host-buffer forms (what the drop-in shim calls). The context keeps
 * the plan of the last 3D one-call form (device volumes, tensor maps) and
 * reuses it while the next call has the same geometry and flags: every call
 * rewrites the model, wavelet and receivers and zeroes the wavefields and
 * accumulators, so results do not depend on the calls before. A call that
 * fails drops the kept plan. vti_ctx_set_plan_cache(ctx, 0) frees the kept
 * plan and makes each call create and free its own (the reference's
 * behaviour); 1 (the default) turns keeping back on. */
int vti_ctx_set_plan_cache(vti_ctx* ctx, int enable);
int vti3d_model_data_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                         const float* c33, const float* wavelet, const float* souloc,
                         const int* shotid, int nshot, const float* recloc, int nrec_total,
                         float* ddata, unsigned flags);
int vti3d_gradient_cij(vti_ctx* ctx, const vti3d_geom* g, const float* cij, const float* padb,
                       const float* randb, const float* wavelet, const float* souloc,
                       const int* shotid, int nshot, const float* recloc, int nrec_total,
                       const float* dobs, float* fgcij, double* misfit, unsigned flags);
/* waveletGradientCij3d_f with host buffers (modelData3d_f.cu:858). */
int vti3d_wavelet_gradient_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11,
                               const float* c13, const float* c33, const float* souloc,
                               const int* shotid, int nshot, const float* recloc, int nrec_total,
                               const float* data, float* gwavelet, unsigned flags);
/* rtmCij3d_f with host buffers: the model as given (rtm3d_f.cu:161). */
int vti3d_rtm_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                  const float* c33, const float* wavelet, const float* souloc, const int* shotid,
                  int nshot, const float* recloc, int nrec_total, const float* data,
                  float* image, unsigned flags);

/* objFuncGradientVEpsDel (objFuncGradient3d_f.cu:249-305): gradient of the
 * L2 misfit with respect to v, eps, del (nxyz each). padboundary_v /
 * randboundary_v are the velocity pad-region lists (nb each); the boundary
 * lists of eps/del are taken from the model. The gradient is zero in the pad
 * and in the nwbottom = (wbottom-oz)/dz+1-npad planes below it; *misfit gets
 * the float misfit/2 as a double (the reference returns fgcij[0]). */
int vti3d_gradient_vepsdel(vti_ctx* ctx, const vti3d_geom* g, const float* v, const float* eps,
                           const float* del, const float* padboundary_v,
                           const float* randboundary_v, float v0, float eps0, float wbottom,
                           const float* wavelet, const float* souloc, const int* shotid,
                           int nshot, const float* recloc, int nrec_total, const float* dobs,
                           float* gv, float* geps, float* gdel, double* misfit, unsigned flags);

/* ------------------------------------------------------------------- 2D */
/* synthetic_f (lib/vti-fwi-2d/synthetic_f.cu:13): data[(it/ratio)*nr + ir]. */
int vti2d_synthetic(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                    const float* c33, const float* wavelet, const int* sloc, int ns,
                    const int* rloc, int nr, const float* taper, float* data);
/* Same arguments and results as vti2d_synthetic, without any device
 * allocation: all device data of a call sits in one static 40 MiB array per
 * device (need = 8*nnx*nnz + nt + nri + rows*nri floats; larger calls return
 * VTI_ERR_ARG). For callers that may not allocate inside a call. The first
 * call on a device does the set-up (looks up the array's address) and should
 * come before any stream capture. Overlapping calls on one device race on the
 * shared array: serialise them. No counterpart in the reference. */
int vti2d_synthetic_noalloc(vti_ctx* ctx, const vti2d_geom* g, const float* c11,
                            const float* c13, const float* c33, const float* wavelet,
                            const int* sloc, int ns, const int* rloc, int nr,
                            const float* taper, float* data);
/* modeling_f (modeling_f.cu:10): sigma_h snapshots wavefield[(it/ratio)*nnxz + i]. */
int vti2d_modeling(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                   const float* c33, const float* wavelet, int slocxz, const float* taper,
                   float* wavefield);
/* objFuncGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:15): gradient of the
 * L2 misfit w.r.t. c11, c13, c33 (arrays (nx+2npad)*(nz+2npad)) for ns shots;
 * observed data as synthetic_f writes them; *misfit = 0.5 * sum(res^2). */
int vti2d_gradient(vti_ctx* ctx, const vti2d_geom* g, float* gc11, float* gc13, float* gc33,
                   const float* data, const float* c11, const float* c13, const float* c33,
                   const float* wavelet, const int* sloc, int ns, const int* rloc, int nr,
                   const float* taper, double* misfit);
/* GNhessian_f (lib/vti-fwi-2d/hessian_f.cu:575): Gauss-Newton Hessian times
 * the model perturbation (dc11, dc13, dc33). */
int vti2d_gn_hessian(vti_ctx* ctx, const vti2d_geom* g, float* gc11, float* gc13, float* gc33,
                     const float* c11, const float* c13, const float* c33, const float* dc11,
                     const float* dc13, const float* dc33, const float* wavelet, const int* sloc,
                     int ns, const int* rloc, int nr, const float* taper);
/* rtm_f (lib/vti-fwi-2d/rtm_f.cu:13): reverse-time migration of the traces
 * data[(it/ratio)*nr + ir] (the layout vti2d_synthetic writes) into image
 * ((nx+2npad)*(nz+2npad) floats, zeroed first, summed over shots). Dipole
 * source and data injection; the source and the point below it must lie in
 * the updated region. */
int vti2d_rtm(vti_ctx* ctx, const vti2d_geom* g, float* image, const float* data,
              const float* c11, const float* c13, const float* c33, const float* wavelet,
              const int* sloc, int ns, const int* rloc, int nr, const float* taper);
/* odcig_f (lib/vti-fwi-2d/odcig_f.cu:12): offset-domain common-image gathers,
 * image[(h+nhx)*nnxz + i] for subsurface x offsets |h| <= nhx ((2nhx+1)*nnxz
 * floats), the migration of vti2d_rtm with the extended imaging condition. */
int vti2d_odcig(vti_ctx* ctx, const vti2d_geom* g, int nhx, float* image, const float* data,
                const float* c11, const float* c13, const float* c33, const float* wavelet,
                const int* sloc, int ns, const int* rloc, int nr, const float* taper);
/* waveletGradient_f (lib/vti-fwi-2d/objFuncGradient_f.cu:373): gradient of the
 * misfit with respect to the source wavelet (nt floats): dt2 (p + q) of the
 * adjoint wavefield at the source for every level, the adjoint driven by the
 * traces data[(it/ratio)*nr + ir] (injected as points). */
int vti2d_wavelet_gradient(vti_ctx* ctx, const vti2d_geom* g, float* gwavelet, const float* data,
                           const float* c11, const float* c13, const float* c33,
                           const int* sloc, int ns, const int* rloc, int nr, const float* taper);
/* 2D taper of lib/vti-fwi-2d/init.cpp:70-89 ((nx+2npad)*(nz+2npad) floats). */
void vti2d_init_taper(float* taper, int nx, int nz, int npad);
/* Random boundary (lib/random-boundary/randomBound.h:48, RandomMY; randomB.x
 * calls it with bval = 1, eval = 0.2): field (n1 fastest, n3 = 1 for 2D) is
 * multiplied, inside the pad of width `pad`, by per-cluster random factors;
 * clusters grow by a random walk continued with probability pct_g; random
 * numbers from the C library's rand() after srand(seed), in the reference's
 * order (host code). */
int vti_random_boundary(float* field, int n1, int n2, int n3, int pad, float pct_g, int seed,
                        float bval, float eval);

/* ------------------------------------------------- 3D batched multi-shot */
/* A window of the model for one shot: cells [x0, x0+nx) x [y0, y0+ny) and the
 * full z range; the window's outer npad cells are its sponge and random
 * boundary. */
typedef struct {
  int x0, y0, nx, ny;
} vti3d_window;
/* Many shots, each on its own window, advanced together: one forward launch
 * per time step for passes 1 and 2 of every shot, one backward launch per
 * step for pass 3 (reference mode of vti3d_plan_gradient per shot). g is the
 * full model grid. */
int vti3d_batch_create(vti_ctx* ctx, const vti3d_geom* g, unsigned flags, vti3d_batch** out);
int vti3d_batch_destroy(vti3d_batch* b);
/* Full model c11, c13, c33 (nxyz each); kept on the device. */
int vti3d_batch_set_model(vti3d_batch* b, const float* c11, const float* c13, const float* c33,
                          int mem);
int vti3d_batch_set_wavelet(vti3d_batch* b, const float* wavelet, int mem);
/* Receiver list as vti3d_plan_set_receivers (x, y, z, flag per receiver). */
int vti3d_batch_set_receivers(vti3d_batch* b, const float* recloc, int nrec_total);
/* Shots: souloc 5 floats per shot (x, y, z, nrec, first receiver) in model
 * coordinates, win one window per shot, seed of the random boundaries
 * (generated on the device per shot). Allocates every shot's state. */
int vti3d_batch_set_shots(vti3d_batch* b, int nshot, const float* souloc,
                          const vti3d_window* win, unsigned seed);
/* use_graph != 0: the time loops are captured once as CUDA graphs and
 * replayed. seg_fwd/seg_bwd: z planes per work item (0: default schedule). */
int vti3d_batch_set_options(vti3d_batch* b, int use_graph, int seg_fwd, int seg_bwd);
/* Schedules of vti3d_batch_gradient. Side by side: every level is one
 * forward launch over passes 1 and 2 of all shots and one backward launch
 * over pass 3 of all shots. Per shot: the shots run one after another, each
 * with the single-grid launches of vti3d_plan_gradient (windows that fill the
 * GPU alone lose nothing to this and keep the single-grid kernels' higher
 * bandwidth). Auto: per shot when every window alone fills every SM with at
 * least kBatchPerShotWaves waves of full-depth columns (vti3d_batch_autotune
 * replaces this rule by timing both). The gradient is the same under every
 * schedule. */
#define VTI_BATCH_AUTO 0
#define VTI_BATCH_SIDE_BY_SIDE 1
#define VTI_BATCH_PER_SHOT 2
int vti3d_batch_set_schedule(vti3d_batch* b, int schedule);
/* Observed traces of vti3d_batch_gradient as FP32 (default) or as a
 * VTI_TRACES_F16 block over all nr_total receivers (see
 * vti3d_plan_set_trace_format). */
int vti3d_batch_set_trace_format(vti3d_batch* b, int format);
/* The schedule the next gradient runs (VTI_BATCH_SIDE_BY_SIDE or
 * VTI_BATCH_PER_SHOT): the one set, or what auto resolves to. */
int vti3d_batch_get_schedule(vti3d_batch* b, int* schedule);
/* Times candidate segment lengths on the current shots and keeps the
 * fastest; under VTI_BATCH_AUTO also times one level of each schedule and
 * keeps the faster. */
int vti3d_batch_autotune(vti3d_batch* b, int* seg_fwd, int* seg_bwd);
/* Gradient of all shots: dobs as vti3d_plan_gradient (trace-major, global
 * receiver order); fgcij = [misfit/2, gc11, gc13, gc33] over the full model,
 * each window's gradient added without its npad x/y frame (unless that frame
 * is the model's edge). */
int vti3d_batch_gradient(vti3d_batch* b, const float* dobs, int dobs_mem, float* fgcij,
                         int fgcij_mem, double* misfit);
/* Window models of shot k (pad-boundary and random-boundary, 3 * nx*ny*nz
 * each, host; either may be NULL). */
int vti3d_batch_get_shot_models(vti3d_batch* b, int k, float* cpad, float* crand);

/* ---------------------------------------------------- 3D serving engine */
/* Continuous batching of 3D modeling and gradient jobs of different grids:
 * jobs are admitted between time steps while their device footprint fits the
 * engine's byte budget (VTI_ERR_BUSY otherwise); every engine tick advances
 * every admitted job by one time level, all jobs sharing one forward and one
 * backward launch. A job's state stays resident until its result is
 * collected. Per job the result is that of vti3d_plan_model_data /
 * vti3d_plan_gradient with VTI_OPT_FULL_STEPS on the job's grid. */
typedef struct vti3d_engine vti3d_engine;
#define VTI_JOB_MODEL 0    /* traces of one shot */
#define VTI_JOB_GRADIENT 1 /* misfit and c11/c13/c33 gradient of one shot */
typedef struct {
  int kind;
  vti3d_geom g;                   /* the job's own grid */
  const float *c11, *c13, *c33;   /* host, nxyz each */
  const float* wavelet;           /* host, nt */
  const float* souloc;            /* host, 5 floats: x, y, z, nrec, 0 */
  const float* recloc;            /* host, 4 floats per receiver */
  int nrec;
  const float* dobs;              /* gradient: host, nnt * nrec observed traces */
  const float* randb;             /* gradient: host, 3*nb random-boundary lists, or NULL */
  unsigned seed;                  /* gradient without randb: device random boundary seed */
} vti3d_job;
/* Device bytes a job holds while admitted. */
size_t vti3d_engine_job_bytes(const vti3d_job* job);
int vti3d_engine_create(vti_ctx* ctx, size_t max_bytes, vti3d_engine** out);
int vti3d_engine_destroy(vti3d_engine* e);
/* Admits a job (copies its inputs to the device) or returns VTI_ERR_BUSY. */
int vti3d_engine_submit(vti3d_engine* e, const vti3d_job* job, int* id);
/* Enqueues up to `ticks` time levels of every admitted job; *active = jobs
 * still running. */
int vti3d_engine_step(vti3d_engine* e, int ticks, int* active);
/* Drops an admitted job (running or finished, result not collected): waits
 * for the launches already queued, then releases its device state and its
 * share of the byte budget; the jobs beside it continue unchanged. For
 * request loops that cancel requests; no counterpart in the reference. */
int vti3d_engine_cancel(vti3d_engine* e, int id);
/* Ids of finished jobs whose results are ready (non-blocking). */
int vti3d_engine_poll(vti3d_engine* e, int* ids, int max_ids, int* n_done);
/* Result of a finished job, then its device state is released: modeling:
 * nnt*nrec traces; gradient: [misfit/2, gc11, gc13, gc33] (1 + 3 nxyz). */
int vti3d_engine_result(vti3d_engine* e, int id, float* out, double* misfit);
int vti3d_engine_stats(vti3d_engine* e, size_t* used_bytes, int* jobs, int* tick);

/* ------------------------------------------- 3D Gauss-Newton product */
/* Exact-mode 3D Gauss-Newton Hessian-vector product and gradient of one shot
 * (no counterpart on the reference's GPU; its CPU twin has bornCij /
 * adjointCij, lib/vti-fwi-3d/cpu/laplacian3d.ispc:132-190). Forward operator:
 * the 3D VTI step with the sponge as a plain diagonal, every level up to
 * nt-1, receivers at their own cells; its Born linearisation along dc and its
 * exact discrete adjoint. Background checkpoints every `checkpoint_every`
 * levels (0: 64), recomputed per block in the backward pass; with
 * VTI_GNHV_BF16 the recomputed levels the imaging reads are kept as BF16
 * with one FP32 scale per z plane (half the segment memory; checkpoints
 * stay FP32, so the recomputation is exact), rounded to nearest, or
 * stochastically with VTI_GNHV_BF16_SR (each stored value unbiased,
 * independent errors from level to level).
 * Outputs (host, each may be NULL): hv = H dc (3*nxyz), grad = dJ/dc of
 * J = 1/2|d - dobs|^2 (3*nxyz; needs dobs), misfit = J, traces d and Born
 * traces (nnt*nrec each). souloc: 5 floats (x, y, z, nrec, 0). */
#define VTI_GNHV_BF16 1u /* background levels of the imaging stored as BF16 + plane scales */
#define VTI_GNHV_BF16_SR 2u /* with VTI_GNHV_BF16: stochastic instead of nearest rounding */
int vti3d_gnhv_exact(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                     const float* c33, const float* dc, const float* wavelet, const float* souloc,
                     const float* recloc, int nrec, const float* dobs, int checkpoint_every,
                     unsigned flags, float* hv, float* grad, double* misfit, float* traces,
                     float* born);

#ifdef __cplusplus
}
#endif
#endif /* VTI_B200_H */
