// 3D plan: device-resident state of one grid and the three-pass gradient
// (objFuncGradientCij3d_f, lib/vti-fwi-3d/gpu/objFuncGradient3d_f.cu:361-1111),
// forward modeling (modelDataCij3d_f, modelData3d_f.cu:427) and the misfit
// (objFuncCij3d_f, objFuncGradient3d_f.cu:1272).
//
// The reference streams 4-plane z-blocks between host and GPUs through a
// 64-step temporal pipeline because its GPUs could not hold a shot. Here the
// whole shot is resident in HBM; each time step is one fused kernel over the
// volume, and the pipeline's observable conventions are kept:
//   * number of levels: 2 + 64*floor((nt-2)/64) unless VTI_OPT_FULL_STEPS;
//   * source dt2*w[it-1] into level it before the sponge; recording of level
//     it at it == s*j, j >= 1 (objFuncGradient3d_f.cu:655-668);
//   * pass 3: level it = nt-3-i of the source wavefield gets dt2*w[it+1],
//     the adjoint gets the residual interpolated at it+1 (:958-1024).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>

#include "vti_plan3d.h"

using namespace vti;
using namespace vti::p3d;

namespace vti {
namespace p3d {

int sampling_step(const vti3d_geom& g) { return (int)std::round(g.sampling_rate / g.dt); }
int nnt_of(const vti3d_geom& g) { return (g.nt - 1) / sampling_step(g) + 1; }
int ref_gpus(unsigned flags) {
  int gpus = (int)((flags >> 8) & 0xffu);
  return gpus < 1 ? 1 : gpus;
}
// objFuncGradient3d_f.cu:538-542: the pipeline runs nround rounds of
// NGPU*64 updates starting at level 2.
int last_level(const vti3d_geom& g, unsigned flags) {
  if (flags & VTI_OPT_FULL_STEPS) return g.nt - 1;
  const int per_round = kRefUpdate * ref_gpus(flags);
  return 1 + per_round * ((g.nt - 2) / per_round);
}

// Which level is recorded into which trace sample. The reference records
// level it into sample itdata only when, at the pipeline tick that updates
// the receiver block at level it, it == s*itdata; itdata advances two ticks
// after each record (device->host copy, then host store). This replays that
// bookkeeping (modelData3d_f.cu:123-296, recording at :233-275) for a
// pipeline of `ngpu` GPUs and returns rec_at[it] = sample index or -1.
std::vector<int> reference_record_schedule(int nt, int nz, int rec_block, int st, int nnt,
                                           int ngpu) {
  const int NU = kRefUpdate;
  const int nb = nz / kHalo;
  const int pipelen = ngpu * (NU + 3) + 3;
  const int nround = (nt - 2) / (ngpu * NU);
  const int roundlen = std::max(pipelen, nb);
  const int nroundlen = nround * roundlen;
  const int nk = (nround - 1) * roundlen + pipelen + nb - 1;
  std::vector<int> rec_at(std::max(nt, 2), -1);
  int itdata = 1, krecord = -2, ktransf = -2, pending_it = -1;
  for (int k = 0; k < nk; ++k) {
    for (int gpu = 0; gpu < ngpu; ++gpu) {
      const int kgpu = k - gpu * (NU + 3);
      if (kgpu > 2 && kgpu <= NU + 1 + nroundlen) {
        for (int i = 0; i < NU; ++i) {
          const int ib = (kgpu - 3 - i) % roundlen;  // C++ truncating division,
          const int iround = (kgpu - 3 - i) / roundlen;  // as in the reference
          if (ib >= 0 && ib < nb && iround >= 0 && iround < nround) {
            const int it = iround * ngpu * NU + gpu * NU + 2 + i;
            if (ib == rec_block && it == st * itdata && itdata < nnt) {
              krecord = k;
              pending_it = it;
            }
          }
        }
      }
    }
    if (k - 1 == krecord && itdata < nnt) {
      krecord = -2;
      ktransf = k;
    }
    if (k - 1 == ktransf && itdata < nnt) {
      if (pending_it >= 0 && pending_it < (int)rec_at.size()) rec_at[pending_it] = itdata;
      itdata++;
      ktransf = -2;
    }
  }
  return rec_at;
}
long long boundary_count(const vti3d_geom& g) {
  return (long long)g.nx * g.ny * g.nz -
         (long long)(g.nx - 2 * g.npad) * (g.ny - 2 * g.npad) * (g.nz - 2 * g.npad);
}

// abc3d.cu:23-50, evaluated in the same float/double mix.
float damp_profile(int i, int n, int npad) {
  float dist;
  if (i < npad) dist = npad - i;
  else if (i > n - npad) dist = i - n + npad;
  else dist = 0.f;
  return (float)(0.95 + (1. - 0.95) * std::cos(3.14159265359 * dist / npad));
}

// Index arithmetic of objFuncGradient3d_f.cu:551-575 (float, truncation).
// In reference mode the receivers are read and injected inside the 4-plane
// block of the first receiver of the survey (recBlock, :545, recIndexBlock
// :568) and seeded at their own depth (recIndex, :567, :922-927).
int shot_geom(vti3d_plan* p, const float* souloc, int is, ShotGeom* s) {
  const vti3d_geom& g = p->g;
  const float* hx = p->h_damp.data();
  const float* hy = hx + g.nx;
  const float* hz = hy + g.ny;
  s->nr = (int)souloc[5 * is + 3];
  s->irbegin = (int)souloc[5 * is + 4];
  s->sx = (int)((souloc[5 * is] - g.ox) / g.dx);
  s->sy = (int)((souloc[5 * is + 1] - g.oy) / g.dy);
  s->sz = (int)((souloc[5 * is + 2] - g.oz) / g.dz);
  if (s->sx < kHalo || s->sx >= g.nx - kHalo || s->sy < kHalo || s->sy >= g.ny - kHalo ||
      s->sz < 0 || s->sz >= g.nz)
    return fail(p->ctx, VTI_ERR_ARG,
                "source of shot " + std::to_string(is) +
                    " lies outside the update region (x,y in [4,n-4), z in [0,nz))");
  if (s->nr < 0 || s->irbegin < 0 || s->irbegin + s->nr > p->nrec_total)
    return fail(p->ctx, VTI_ERR_ARG,
                "receiver range of shot " + std::to_string(is) + " exceeds the receiver list");
  const bool ref_mode = !(p->flags & VTI_OPT_FULL_STEPS);
  const int st = sampling_step(g), nnt = nnt_of(g);
  int rec_block = -1;
  if (p->nrec_total > 0) rec_block = (int)((p->recloc[2] - g.oz) / g.dz / kHalo);
  s->rec.resize(s->nr);
  s->seed.resize(s->nr);
  s->rec_damp.resize(s->nr);
  s->live.resize(s->nr);
  for (int ir = 0; ir < s->nr; ++ir) {
    const float* r = p->recloc.data() + 4 * (size_t)(ir + s->irbegin);
    int ix = (int)((r[0] - g.ox) / g.dx);
    int iy = (int)((r[1] - g.oy) / g.dy);
    int iz = (int)((r[2] - g.oz) / g.dz);
    int izr = ref_mode ? rec_block * kHalo + iz % kHalo : iz;
    if (ix < 0 || ix >= g.nx || iy < 0 || iy >= g.ny || iz < 0 || iz >= g.nz || izr < 0 ||
        izr >= g.nz)
      return fail(p->ctx, VTI_ERR_ARG,
                  "receiver " + std::to_string(ir + s->irbegin) + " lies outside the grid");
    s->rec[ir] = p->d.off(ix, iy, izr);
    s->seed[ir] = p->d.off(ix, iy, iz);
    // The step kernel has already applied the sponge to next, so injected
    // residuals are scaled by the same factor. Cells of the 4-wide x/y frame
    // are never updated by the scheme; nothing is injected there.
    bool inner = ix >= kHalo && ix < g.nx - kHalo && iy >= kHalo && iy < g.ny - kHalo;
    s->rec_damp[ir] = inner ? (hx[ix] * hy[iy]) * hz[izr] : 0.f;
    s->live[ir] = r[3] != 0.f;
  }
  const int M = last_level(g, p->flags);
  if (ref_mode) {
    s->rec_at = reference_record_schedule(g.nt, g.nz, rec_block, st, nnt, ref_gpus(p->flags));
  } else {
    s->rec_at.assign(std::max(g.nt, 2), -1);
    for (int it = 2; it <= M; ++it)
      if (it % st == 0 && it / st >= 1 && it / st < nnt) s->rec_at[it] = it / st;
  }
  return VTI_OK;
}

int upload_shot(vti3d_plan* p, const ShotGeom& s) {
  vti_ctx* ctx = p->ctx;
  size_t nr = std::max(s.nr, 1);
  if (p->rec_cap < nr) {
    if (p->d_rec) cudaFree(p->d_rec);
    if (p->d_rec_damp) cudaFree(p->d_rec_damp);
    if (p->d_live) cudaFree(p->d_live);
    p->d_rec = nullptr;
    p->d_rec_damp = nullptr;
    p->d_live = nullptr;
    p->rec_cap = 0;
    // recording offsets [0, nr), seeding offsets [nr, 2nr)
    VTI_CUDA(ctx, cudaMalloc((void**)&p->d_rec, 2 * nr * sizeof(long long)));
    VTI_CUDA(ctx, cudaMalloc((void**)&p->d_rec_damp, nr * sizeof(float)));
    VTI_CUDA(ctx, cudaMalloc((void**)&p->d_live, nr));
    p->rec_cap = nr;
  }
  if (s.nr > 0) {
    VTI_CUDA(ctx, cudaMemcpyAsync(p->d_rec, s.rec.data(), s.nr * sizeof(long long),
                                  cudaMemcpyHostToDevice, ctx->stream));
    VTI_CUDA(ctx, cudaMemcpyAsync(p->d_rec + p->rec_cap, s.seed.data(),
                                  s.nr * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream));
    VTI_CUDA(ctx, cudaMemcpyAsync(p->d_rec_damp, s.rec_damp.data(), s.nr * sizeof(float),
                                  cudaMemcpyHostToDevice, ctx->stream));
    VTI_CUDA(ctx, cudaMemcpyAsync(p->d_live, s.live.data(), s.nr, cudaMemcpyHostToDevice,
                                  ctx->stream));
  }
  VTI_TRY(ensure(ctx, &p->d_trace, &p->trace_cap, (size_t)nnt_of(p->g) * nr));
  // the host vectors are released when the caller's ShotGeom goes away
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VTI_OK;
}

// VTI_OPT_CHECK_FINITE: the volumes (whole allocations, zero padding
// included) are scanned for NaN / Inf; a hit sets the status word's
// VTI_ERR_NONFINITE bit, which the call's final status check reports. A
// non-finite value propagates through every later level, so checking the
// last two levels of each pass catches one that arose anywhere in it.
int check_finite(vti3d_plan* p, std::initializer_list<const Vol*> vols) {
  if (!(p->flags & VTI_OPT_CHECK_FINITE)) return VTI_OK;
  for (const Vol* v : vols)
    VTI_TRY(launch_check_finite(p->ctx, v->alloc, (long long)(v->bytes / sizeof(float))));
  return VTI_OK;
}

// One forward level (objFuncGradient3d_f.cu:610-700): level `it` from
// sx[A] (level it-1) and sx[B] (level it-2) into sx[B], then, for pass 1, the
// traces of the new level. Pass 1 (sponge) runs on the pad-boundary model,
// pass 2 on the random-boundary model when the plan has one.
int fwd_level(vti3d_plan* p, const ShotGeom& s, bool sponge, int A, int B, int it) {
  vti_ctx* ctx = p->ctx;
  const vti3d_geom& g = p->g;
  const float dt2 = g.dt * g.dt;
  const TileMaps* cm = (sponge || !p->have_rand) ? p->m_cpad : p->m_crand;
  Damping dmp{p->dampx, p->dampy, p->dampz};
  PointSource src;
  src.x = s.sx;
  src.y = s.sy;
  src.z = s.sz;
  src.amp = dt2 * p->wavelet[it - 1];
  VTI_TRY(launch_fwd3d_tma(ctx, p->d, p->m_sx[A], p->m_sz[A], p->m_sx[B], p->m_sz[B], cm[0],
                           cm[1], cm[2], p->sz[A].origin, p->sx[B].origin, p->sz[B].origin,
                           sponge ? &dmp : nullptr, dt2 / (g.dx * g.dx), dt2 / (g.dy * g.dy),
                           dt2 / (g.dz * g.dz), src));
  if (sponge && it < (int)s.rec_at.size() && s.rec_at[it] >= 0)
    VTI_TRY(launch_record(ctx, p->d_trace, nnt_of(g), s.rec_at[it], p->sx[B].origin,
                          p->sz[B].origin, p->d_rec, s.nr));
  return VTI_OK;
}

// Forward propagation of one shot. sponge: pass 1 (pad-boundary model, sponge,
// traces recorded into d_trace). Otherwise pass 2 (random-boundary model, no
// sponge). On return sx[last_cur] holds level M and the other buffer M-1.
int forward_pass(vti3d_plan* p, const ShotGeom& s, bool sponge) {
  NvtxRange nv(sponge ? "vti3d pass 1 (sponge, traces)" : "vti3d pass 2 (random boundary)");
  vti_ctx* ctx = p->ctx;
  const vti3d_geom& g = p->g;
  const Dims3& d = p->d;
  const float dt2 = g.dt * g.dt;
  const int nnt = nnt_of(g), M = last_level(g, p->flags);
  for (int k = 0; k < 2; ++k) {
    VTI_TRY(vol_zero(ctx, d, &p->sx[k]));
    VTI_TRY(vol_zero(ctx, d, &p->sz[k]));
  }
  int A = 0, B = 1;
  // "injecting source at time 0 to wavefields at time 1"
  // (objFuncGradient3d_f.cu:605-608): assignment, no sponge.
  VTI_TRY(launch_set_point(ctx, p->sx[A].origin, p->sz[A].origin, d.off(s.sx, s.sy, s.sz),
                           dt2 * p->wavelet[0]));
  if (sponge && s.nr > 0)
    VTI_CUDA(ctx,
             cudaMemsetAsync(p->d_trace, 0, (size_t)nnt * s.nr * sizeof(float), ctx->stream));
  for (int it = 2; it <= M; ++it) {
    VTI_TRY(fwd_level(p, s, sponge, A, B, it));
    std::swap(A, B);
  }
  p->last_cur = A;
  if (sponge && s.nr > 0 && (p->flags & VTI_OPT_CHECK_FINITE))
    VTI_TRY(launch_check_finite(ctx, p->d_trace, (long long)nnt * s.nr));
  return check_finite(p, {&p->sx[0], &p->sx[1], &p->sz[0], &p->sz[1]});
}

// Backward step i of pass 3 (objFuncGradient3d_f.cu:920-1060): the source
// field reconstructed from sx[SA] (current) and sx[SB] (next, overwritten),
// the adjoint from lx[LA] and lx[LB] (overwritten) and the imaging terms
// added into g11/g13/g33 (the RTM image into g11), then the residual of time
// nt-2-i injected into the new adjoint level (injectRecord3d.cu:60-78).
int bwd_level(vti3d_plan* p, const ShotGeom& s, bool rtm, int SA, int SB, int LA, int LB,
              int i) {
  vti_ctx* ctx = p->ctx;
  const vti3d_geom& g = p->g;
  const float dx2 = g.dx * g.dx, dy2 = g.dy * g.dy, dz2 = g.dz * g.dz, dt2 = g.dt * g.dt;
  const int st = sampling_step(g), nnt = nnt_of(g);
  const TileMaps* cm = p->have_rand ? p->m_crand : p->m_cpad;
  Damping dmp{p->dampx, p->dampy, p->dampz};
  const int it = g.nt - 3 - i;
  PointSource src;
  src.x = s.sx;
  src.y = s.sy;
  src.z = s.sz;
  src.amp = dt2 * p->wavelet[it + 1];
  VTI_TRY(launch_bwd3d_tma(
      ctx, p->d, p->m_sx[SA], p->m_sz[SA], p->m_sx[SB], p->m_sz[SB], p->m_lx[LA], p->m_lz[LA],
      p->m_lx[LB], p->m_lz[LB], cm[0], cm[1], cm[2], p->m_g[0], p->m_g[1], p->m_g[2],
      p->sz[SA].origin, p->lz[LA].origin, p->sx[SB].origin, p->sz[SB].origin,
      p->lx[LB].origin, p->lz[LB].origin, p->g11.origin, p->g13.origin, p->g33.origin, dmp,
      dt2, 1.f / dx2, 1.f / dy2, 1.f / dz2, dt2 / dx2, dt2 / dy2, dt2 / dz2, src, rtm));
  // residual interpolated at it+1 (injectRecord3d.cu:60-78)
  const int ti = it + 1;
  float f = float(ti) / float(st);
  int i0 = (int)f;
  int clamp = i0 >= nnt - 1;
  f = f - i0;
  return launch_inject_residual(ctx, p->lx[LB].origin, p->lz[LB].origin, p->d_trace, nnt,
                                clamp ? 0 : i0, f, clamp, p->d_rec, p->d_rec_damp, s.nr, dt2);
}

// Time-reversed source wavefield + adjoint + imaging (pass 3,
// objFuncGradient3d_f.cu:910-1078). Expects sx[last_cur] = level M,
// sx[other] = level M-1 from pass 2, and the residual in d_trace.
// rtm: the observed traces are in d_trace and the RTM image accumulates in
// g11 (rtm3d_f.cu:470-620, same schedule).
// ext (nlag >= 0, RTM only): offset-domain gathers of each level added after
// its fused step, from the same current wavefields.
int backward_pass(vti3d_plan* p, const ShotGeom& s, bool rtm, float* ext, int nlag) {
  NvtxRange nv(rtm ? "vti3d RTM back-propagation" : "vti3d pass 3 (reconstruction, adjoint, imaging)");
  vti_ctx* ctx = p->ctx;
  const vti3d_geom& g = p->g;
  const Dims3& d = p->d;
  const float dt2 = g.dt * g.dt;
  const int nnt = nnt_of(g), M = last_level(g, p->flags);
  Damping dmp{p->dampx, p->dampy, p->dampz};
  // flip (objFuncGradient3d_f.cu:912-914): cur = level M-1, prev = level M
  int SA = 1 - p->last_cur, SB = p->last_cur;
  for (int k = 0; k < 2; ++k) {
    VTI_TRY(vol_zero(ctx, d, &p->lx[k]));
    VTI_TRY(vol_zero(ctx, d, &p->lz[k]));
  }
  int LA = 0, LB = 1;
  VTI_TRY(launch_seed_adjoint(ctx, p->lx[LA].origin, p->lz[LA].origin, p->d_trace, nnt,
                              p->d_rec + p->rec_cap, p->d_rec_damp, s.nr, dt2));
  for (int i = 0; i < M - 1; ++i) {
    VTI_TRY(bwd_level(p, s, rtm, SA, SB, LA, LB, i));
    // the gathers read the current levels sx[SA], lx[LA]; the step and the
    // injection write only sx[SB], lx[LB]
    if (ext)
      VTI_TRY(launch_odcig3d(ctx, d, p->sx[SA].origin, p->sz[SA].origin, p->lx[LA].origin,
                             p->lz[LA].origin, dmp, nlag, ext));
    std::swap(SA, SB);
    std::swap(LA, LB);
  }
  return check_finite(p, {&p->sx[0], &p->sx[1], &p->sz[0], &p->sz[1], &p->lx[0], &p->lx[1],
                          &p->lz[0], &p->lz[1], &p->g11, &p->g13, &p->g33});
}

int check_geom(vti_ctx* ctx, const vti3d_geom* g) {
  if (!g) return fail(ctx, VTI_ERR_ARG, "null geometry");
  if (g->nx < 2 * kHalo + 1 || g->ny < 2 * kHalo + 1 || g->nz < 1 || g->nt < 3)
    return fail(ctx, VTI_ERR_ARG, "grid too small (need nx,ny >= 9, nz >= 1, nt >= 3)");
  if (g->npad < 1 || 2 * g->npad > g->nx || 2 * g->npad > g->ny || 2 * g->npad > g->nz)
    return fail(ctx, VTI_ERR_ARG, "npad out of range (1 <= npad <= n/2)");
  if (!(g->dx > 0 && g->dy > 0 && g->dz > 0 && g->dt > 0 && g->sampling_rate > 0))
    return fail(ctx, VTI_ERR_ARG, "non-positive spacing, dt or sampling rate");
  if ((int)std::round(g->sampling_rate / g->dt) < 1)
    return fail(ctx, VTI_ERR_ARG, "sampling_rate < dt");
  if ((long long)((g->nx + 31) & ~31) * g->ny >= (1LL << 31))
    return fail(ctx, VTI_ERR_ARG, "plane too large");
  return VTI_OK;
}

int get_obs(vti3d_plan* p, const ShotGeom& s, const float* dobs, int mem, const float** out) {
  const int nnt = nnt_of(p->g);
  const size_t n = (size_t)nnt * s.nr;
  if (p->trace_format == VTI_TRACES_F16) {
    // block: nnt plane scales, then the halves of every trace
    vti_ctx* ctx = p->ctx;
    const float* scale = dobs;
    const uint16_t* h = reinterpret_cast<const uint16_t*>(dobs + nnt) + (size_t)nnt * s.irbegin;
    VTI_TRY(ensure(ctx, &p->d_obs, &p->obs_cap, n));
    if (mem != VTI_MEM_DEVICE) {
      VTI_TRY(ensure(ctx, &p->d_obs16, &p->obs16_cap, n));
      VTI_TRY(ensure(ctx, &p->d_obs_scale, &p->obs_scale_cap, (size_t)nnt));
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_obs16, h, n * sizeof(uint16_t),
                                    cudaMemcpyHostToDevice, ctx->stream));
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_obs_scale, scale, (size_t)nnt * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream));
      h = p->d_obs16;
      scale = p->d_obs_scale;
    }
    VTI_TRY(launch_unpack_traces_f16(ctx, h, scale, nnt, s.nr, p->d_obs));
    *out = p->d_obs;
    return VTI_OK;
  }
  const float* src = dobs + (size_t)nnt * s.irbegin;
  if (mem == VTI_MEM_DEVICE) {
    *out = src;
    return VTI_OK;
  }
  VTI_TRY(ensure(p->ctx, &p->d_obs, &p->obs_cap, n));
  VTI_CUDA(p->ctx, cudaMemcpyAsync(p->d_obs, src, n * sizeof(float), cudaMemcpyHostToDevice,
                                   p->ctx->stream));
  *out = p->d_obs;
  return VTI_OK;
}

int run_gradient(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                 const float* dobs, int dobs_mem, float* fgcij, int fgcij_mem, double* misfit,
                 bool misfit_only) {
  NvtxRange nv(misfit_only ? "vti3d misfit" : "vti3d gradient");
  vti_ctx* ctx = p->ctx;
  if (!p->have_model) return fail(ctx, VTI_ERR_ARG, "model not set");
  if ((int)p->wavelet.size() != p->g.nt) return fail(ctx, VTI_ERR_ARG, "wavelet not set");
  if (!souloc || (nshot > 0 && !shotid) || !dobs || nshot < 0)
    return fail(ctx, VTI_ERR_ARG, "null pointer or negative shot count");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const Dims3& d = p->d;
  const int nnt = nnt_of(p->g);
  if (!p->d_acc)
    VTI_CUDA(ctx, cudaMalloc((void**)&p->d_acc, (1 + residual_blocks(ctx)) * sizeof(double)));
  VTI_CUDA(ctx, cudaMemsetAsync(p->d_acc, 0, sizeof(double), ctx->stream));
  if (!misfit_only) {
    VTI_TRY(vol_zero(ctx, d, &p->g11));
    VTI_TRY(vol_zero(ctx, d, &p->g13));
    VTI_TRY(vol_zero(ctx, d, &p->g33));
  }
  for (int k = 0; k < nshot; ++k) {
    ShotGeom s;
    VTI_TRY(shot_geom(p, souloc, shotid[k], &s));
    VTI_TRY(upload_shot(p, s));
    VTI_TRY(forward_pass(p, s, true));
    const float* obs = nullptr;
    VTI_TRY(get_obs(p, s, dobs, dobs_mem, &obs));
    if (misfit_only || (p->tpow == 0.f && p->objtype == 0)) {
      VTI_TRY(launch_residual(ctx, p->d_trace, obs, p->d_live, nnt, s.nr, p->d_acc));
    } else {
      // objFuncGradient3d_f.cu:733-773: dead traces zeroed, t^p gain on the
      // modeled traces, then the L2 residual or the AGC adjoint source
      VTI_TRY(launch_residual(ctx, p->d_trace, nullptr, p->d_live, nnt, s.nr, nullptr));
      if (p->tpow != 0.f)
        VTI_TRY(launch_tpower(ctx, p->d_trace, nnt, s.nr, p->g.ot, p->g.sampling_rate, p->tpow));
      if (p->objtype == 0) {
        VTI_TRY(launch_residual(ctx, p->d_trace, obs, p->d_live, nnt, s.nr, p->d_acc));
      } else {
        VTI_TRY(ensure(ctx, &p->d_part, &p->part_cap, (size_t)std::max(s.nr, 1)));
        VTI_TRY(launch_agc_adjoint(ctx, p->d_trace, obs, nnt, s.nr, p->halfwidth, p->d_part,
                                   p->d_acc));
      }
    }
    if (misfit_only) continue;
    VTI_TRY(forward_pass(p, s, false));
    VTI_TRY(backward_pass(p, s, false));
    // keep host vectors alive until this shot's uploads are consumed
    VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  double acc = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&acc, p->d_acc, sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
  if (!misfit_only && fgcij) {
    const size_t n = (size_t)d.npoints();
    VTI_TRY(vol_download(ctx, d, &p->g11, fgcij + 1, fgcij_mem));
    VTI_TRY(vol_download(ctx, d, &p->g13, fgcij + 1 + n, fgcij_mem));
    VTI_TRY(vol_download(ctx, d, &p->g33, fgcij + 1 + 2 * n, fgcij_mem));
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  VTI_TRY(check_device_status(ctx));
  if ((p->flags & VTI_OPT_CHECK_FINITE) && !std::isfinite(acc))
    return fail(ctx, VTI_ERR_NONFINITE, "misfit is not finite");
  if (misfit) *misfit = acc / 2;
  if (!misfit_only && fgcij) {
    float f0 = (float)(acc / 2);
    if (fgcij_mem == VTI_MEM_DEVICE)
      VTI_CUDA(ctx, cudaMemcpy(fgcij, &f0, sizeof(float), cudaMemcpyHostToDevice));
    else
      fgcij[0] = f0;
  }
  return VTI_OK;
}

// Plan of a one-call form: the context's kept plan when geometry and flags
// match it, else a new one (kept in its place when keeping is on).
int one_call_plan(vti_ctx* ctx, const vti3d_geom* g, unsigned flags, vti3d_plan** out) {
  if (!ctx || !g || !out) return VTI_ERR_ARG;
  if (ctx->plan_cache && ctx->cached_plan && ctx->cached_flags == flags &&
      std::memcmp(&ctx->cached_geom, g, sizeof(vti3d_geom)) == 0) {
    *out = ctx->cached_plan;
    return VTI_OK;
  }
  if (ctx->cached_plan) {
    vti3d_plan_destroy(ctx->cached_plan);
    ctx->cached_plan = nullptr;
  }
  VTI_TRY(vti3d_plan_create(ctx, g, flags, out));
  if (ctx->plan_cache) {
    ctx->cached_plan = *out;
    ctx->cached_geom = *g;
    ctx->cached_flags = flags;
  }
  return VTI_OK;
}

// End of a one-call form: a plan that is not kept, or that saw an error, is
// freed.
int one_call_done(vti_ctx* ctx, vti3d_plan* p, int st) {
  if (p == ctx->cached_plan && st == VTI_OK) return st;
  if (p == ctx->cached_plan) ctx->cached_plan = nullptr;
  vti3d_plan_destroy(p);
  return st;
}

}  // namespace p3d
}  // namespace vti

extern "C" {

int vti_ctx_set_plan_cache(vti_ctx* ctx, int enable) {
  if (!ctx) return VTI_ERR_ARG;
  ctx->plan_cache = enable != 0;
  if (!ctx->plan_cache && ctx->cached_plan) {
    vti3d_plan_destroy(ctx->cached_plan);
    ctx->cached_plan = nullptr;
  }
  return VTI_OK;
}

int vti3d_plan_create(vti_ctx* ctx, const vti3d_geom* g, unsigned flags, vti3d_plan** out) {
  if (!ctx || !out) return VTI_ERR_ARG;
  *out = nullptr;
  VTI_TRY(check_geom(ctx, g));
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  vti3d_plan* p = new vti3d_plan();
  p->ctx = ctx;
  p->g = *g;
  p->flags = flags;
  p->d = make_dims(g->nx, g->ny, g->nz);
  int st = VTI_OK;
  Vol* vols[] = {&p->cpad[0], &p->cpad[1], &p->cpad[2], &p->sx[0], &p->sx[1], &p->sz[0],
                 &p->sz[1],   &p->lx[0],   &p->lx[1],   &p->lz[0], &p->lz[1], &p->g11,
                 &p->g13,     &p->g33};
  for (Vol* v : vols)
    if (st == VTI_OK) st = vol_alloc(ctx, p->d, v);
  if (st == VTI_OK) {
    for (int k = 0; k < 2 && st == VTI_OK; ++k) {
      st = make_tile_maps(ctx, p->d, p->sx[k], &p->m_sx[k]);
      if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->sz[k], &p->m_sz[k]);
      if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->lx[k], &p->m_lx[k]);
      if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->lz[k], &p->m_lz[k]);
    }
    for (int k = 0; k < 3 && st == VTI_OK; ++k) st = make_tile_maps(ctx, p->d, p->cpad[k], &p->m_cpad[k]);
    if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->g11, &p->m_g[0]);
    if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->g13, &p->m_g[1]);
    if (st == VTI_OK) st = make_tile_maps(ctx, p->d, p->g33, &p->m_g[2]);
  }
  if (st == VTI_OK) {
    p->h_damp.resize((size_t)g->nx + g->ny + g->nz);
    for (int i = 0; i < g->nx; ++i) p->h_damp[i] = damp_profile(i, g->nx, g->npad);
    for (int i = 0; i < g->ny; ++i) p->h_damp[g->nx + i] = damp_profile(i, g->ny, g->npad);
    for (int i = 0; i < g->nz; ++i) p->h_damp[g->nx + g->ny + i] = damp_profile(i, g->nz, g->npad);
    cudaError_t e = cudaMalloc((void**)&p->dampx, p->h_damp.size() * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->dampx, p->h_damp.data(), p->h_damp.size() * sizeof(float),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_check(ctx, e, "damping tables");
    p->dampy = p->dampx + g->nx;
    p->dampz = p->dampy + g->ny;
  }
  if (st != VTI_OK) {
    vti3d_plan_destroy(p);
    return st;
  }
  *out = p;
  return VTI_OK;
}

int vti3d_plan_destroy(vti3d_plan* p) {
  if (!p) return VTI_OK;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  for (int k = 0; k < 3; ++k) {
    vol_free(&p->cpad[k]);
    vol_free(&p->crand[k]);
  }
  for (int k = 0; k < 2; ++k) {
    vol_free(&p->sx[k]);
    vol_free(&p->sz[k]);
    vol_free(&p->lx[k]);
    vol_free(&p->lz[k]);
  }
  vol_free(&p->g11);
  vol_free(&p->g13);
  vol_free(&p->g33);
  void* ptrs[] = {p->dampx, p->d_rec, p->d_rec_damp, p->d_live, p->d_trace,
                  p->d_obs, p->d_blist, p->d_acc, p->d_gw, p->d_part, p->d_ext,
                  p->d_obs16, p->d_obs_scale};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete p;
  return VTI_OK;
}

int vti3d_plan_set_model(vti3d_plan* p, const float* c11, const float* c13, const float* c33,
                         const float* padb, const float* randb, int mem) {
  if (!p) return VTI_ERR_ARG;
  vti_ctx* ctx = p->ctx;
  if (!c11 || !c13 || !c33) return fail(ctx, VTI_ERR_ARG, "null model array");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const Dims3& d = p->d;
  const float* cs[3] = {c11, c13, c33};
  const long long nb = boundary_count(p->g);
  if (randb) {
    for (int k = 0; k < 3; ++k)
      if (!p->crand[k].alloc) {
        VTI_TRY(vol_alloc(ctx, d, &p->crand[k]));
        VTI_TRY(make_tile_maps(ctx, d, p->crand[k], &p->m_crand[k]));
      }
  }
  if (padb || randb) VTI_TRY(ensure(ctx, &p->d_blist, &p->blist_cap, (size_t)nb));
  for (int k = 0; k < 3; ++k) {
    VTI_TRY(vol_upload(ctx, d, &p->cpad[k], cs[k], mem));
    if (randb) {
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_blist, randb + (size_t)k * nb, nb * sizeof(float),
                                    mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                          : cudaMemcpyHostToDevice,
                                    ctx->stream));
      VTI_TRY(launch_boundary_merge(ctx, d, p->g.npad, p->cpad[k].origin, p->d_blist,
                                    p->crand[k].origin));
    }
    if (padb) {
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_blist, padb + (size_t)k * nb, nb * sizeof(float),
                                    mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                          : cudaMemcpyHostToDevice,
                                    ctx->stream));
      VTI_TRY(launch_boundary_merge(ctx, d, p->g.npad, p->cpad[k].origin, p->d_blist,
                                    p->cpad[k].origin));
    }
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  p->have_model = false;
  // refuse a model the scheme cannot step stably (the random boundary only
  // lowers velocities, but a caller's list may not)
  double num = 0;
  VTI_TRY(cfl3d_device(ctx, p->g, d, p->cpad[0].origin, p->cpad[1].origin, p->cpad[2].origin,
                       &num));
  VTI_TRY(cfl_verdict(ctx, num, "model"));
  if (randb) {
    VTI_TRY(cfl3d_device(ctx, p->g, d, p->crand[0].origin, p->crand[1].origin,
                         p->crand[2].origin, &num));
    VTI_TRY(cfl_verdict(ctx, num, "model with the random boundary"));
  }
  p->have_rand = randb != nullptr;
  p->have_model = true;
  return VTI_OK;
}

int vti3d_plan_set_wavelet(vti3d_plan* p, const float* wavelet, int mem) {
  if (!p || !wavelet) return VTI_ERR_ARG;
  p->wavelet.resize(p->g.nt);
  if (mem == VTI_MEM_DEVICE) {
    VTI_CUDA(p->ctx, cudaMemcpy(p->wavelet.data(), wavelet, p->g.nt * sizeof(float),
                                cudaMemcpyDeviceToHost));
  } else {
    std::memcpy(p->wavelet.data(), wavelet, p->g.nt * sizeof(float));
  }
  return VTI_OK;
}

int vti3d_plan_set_receivers(vti3d_plan* p, const float* recloc, int nrec_total) {
  if (!p || (!recloc && nrec_total > 0) || nrec_total < 0) return VTI_ERR_ARG;
  p->recloc.assign(recloc, recloc + 4 * (size_t)nrec_total);
  p->nrec_total = nrec_total;
  return VTI_OK;
}

int vti3d_plan_model_data(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                          float* ddata, int mem) {
  if (!p) return VTI_ERR_ARG;
  vti_ctx* ctx = p->ctx;
  if (!p->have_model) return fail(ctx, VTI_ERR_ARG, "model not set");
  if ((int)p->wavelet.size() != p->g.nt) return fail(ctx, VTI_ERR_ARG, "wavelet not set");
  if (!souloc || !ddata || (nshot > 0 && !shotid)) return fail(ctx, VTI_ERR_ARG, "null pointer");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nnt = nnt_of(p->g);
  for (int k = 0; k < nshot; ++k) {
    ShotGeom s;
    VTI_TRY(shot_geom(p, souloc, shotid[k], &s));
    VTI_TRY(upload_shot(p, s));
    VTI_TRY(forward_pass(p, s, true));
    // modelData3d_f.cu:298-302: dead receivers give zero traces
    VTI_TRY(launch_residual(ctx, p->d_trace, nullptr, p->d_live, nnt, s.nr, nullptr));
    float* dst = ddata + (size_t)nnt * s.irbegin;
    VTI_CUDA(ctx, cudaMemcpyAsync(dst, p->d_trace, (size_t)nnt * s.nr * sizeof(float),
                                  mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                        : cudaMemcpyDeviceToHost,
                                  ctx->stream));
    VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return check_device_status(ctx);
}

int vti3d_plan_set_misfit(vti3d_plan* p, float tpow, int objtype, int halfwidth) {
  if (!p) return VTI_ERR_ARG;
  if (objtype != 0 && halfwidth < 0)
    return fail(p->ctx, VTI_ERR_ARG, "AGC half width must be >= 0");
  p->tpow = tpow;
  p->objtype = objtype;
  p->halfwidth = halfwidth;
  return VTI_OK;
}

int vti3d_plan_set_trace_format(vti3d_plan* p, int format) {
  if (!p) return VTI_ERR_ARG;
  if (format != VTI_TRACES_F32 && format != VTI_TRACES_F16)
    return fail(p->ctx, VTI_ERR_ARG, "unknown trace format");
  p->trace_format = format;
  return VTI_OK;
}

int vti3d_plan_gradient(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                        const float* dobs, int dobs_mem, float* fgcij, int fgcij_mem,
                        double* misfit) {
  if (!p) return VTI_ERR_ARG;
  return run_gradient(p, souloc, shotid, nshot, dobs, dobs_mem, fgcij, fgcij_mem, misfit, false);
}

int vti3d_plan_objfunc(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                       const float* dobs, int dobs_mem, double* misfit) {
  if (!p) return VTI_ERR_ARG;
  return run_gradient(p, souloc, shotid, nshot, dobs, dobs_mem, nullptr, VTI_MEM_HOST, misfit,
                      true);
}

const float* vti3d_plan_wavefield(vti3d_plan* p) {
  return p ? p->sx[p->last_cur].origin : nullptr;
}

int vti3d_plan_get_wavefield(vti3d_plan* p, float* out, int mem) {
  if (!p || !out) return VTI_ERR_ARG;
  VTI_CUDA(p->ctx, cudaSetDevice(p->ctx->device));
  VTI_TRY(vol_download(p->ctx, p->d, &p->sx[p->last_cur], out, mem));
  VTI_CUDA(p->ctx, cudaStreamSynchronize(p->ctx->stream));
  return VTI_OK;
}

int vti3d_model_data_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                         const float* c33, const float* wavelet, const float* souloc,
                         const int* shotid, int nshot, const float* recloc, int nrec_total,
                         float* ddata, unsigned flags) {
  vti3d_plan* p = nullptr;
  VTI_TRY(one_call_plan(ctx, g, flags, &p));
  int st = vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_receivers(p, recloc, nrec_total);
  if (st == VTI_OK) st = vti3d_plan_model_data(p, souloc, shotid, nshot, ddata, VTI_MEM_HOST);
  return one_call_done(ctx, p, st);
}

int vti3d_plan_rtm(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                   const float* data, int data_mem, float* image, int image_mem) {
  if (!p) return VTI_ERR_ARG;
  vti_ctx* ctx = p->ctx;
  if (!p->have_model) return fail(ctx, VTI_ERR_ARG, "model not set");
  if ((int)p->wavelet.size() != p->g.nt) return fail(ctx, VTI_ERR_ARG, "wavelet not set");
  if (!souloc || (nshot > 0 && !shotid) || !data || !image || nshot < 0)
    return fail(ctx, VTI_ERR_ARG, "null pointer or negative shot count");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nnt = nnt_of(p->g);
  // rtm3d_f.cu:175: the image is zeroed, then summed over the shots
  VTI_TRY(vol_zero(ctx, p->d, &p->g11));
  for (int k = 0; k < nshot; ++k) {
    ShotGeom s;
    VTI_TRY(shot_geom(p, souloc, shotid[k], &s));
    VTI_TRY(upload_shot(p, s));
    // the recorded traces drive the receiver wavefield as they are
    // (rtm3d_f.cu:505-514, 547-566): no residual, no dead-trace masking
    const float* obs = nullptr;
    VTI_TRY(get_obs(p, s, data, data_mem, &obs));
    if (s.nr > 0)
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_trace, obs, (size_t)nnt * s.nr * sizeof(float),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    VTI_TRY(forward_pass(p, s, false));
    VTI_TRY(backward_pass(p, s, true));
    VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  VTI_TRY(vol_download(ctx, p->d, &p->g11, image, image_mem));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return check_device_status(ctx);
}

int vti3d_plan_odcig(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                     const float* data, int data_mem, int nlag, float* image, int image_mem) {
  if (!p) return VTI_ERR_ARG;
  vti_ctx* ctx = p->ctx;
  if (!p->have_model) return fail(ctx, VTI_ERR_ARG, "model not set");
  if ((int)p->wavelet.size() != p->g.nt) return fail(ctx, VTI_ERR_ARG, "wavelet not set");
  if (!souloc || (nshot > 0 && !shotid) || !data || !image || nshot < 0)
    return fail(ctx, VTI_ERR_ARG, "null pointer or negative shot count");
  if (nlag < 0 || nlag > 1024) return fail(ctx, VTI_ERR_ARG, "nlag out of range (0..1024)");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const Dims3& d = p->d;
  const int nnt = nnt_of(p->g);
  const int nl = 2 * nlag + 1;
  const size_t vol = (size_t)d.plane * d.nz;  // one lag: pitched rows, no pad planes
  VTI_TRY(ensure(ctx, &p->d_ext, &p->ext_cap, nl * vol));
  VTI_CUDA(ctx, cudaMemsetAsync(p->d_ext, 0, nl * vol * sizeof(float), ctx->stream));
  // the zero-lag image of the same passes accumulates in g11 (unused here)
  VTI_TRY(vol_zero(ctx, d, &p->g11));
  for (int k = 0; k < nshot; ++k) {
    ShotGeom s;
    VTI_TRY(shot_geom(p, souloc, shotid[k], &s));
    VTI_TRY(upload_shot(p, s));
    const float* obs = nullptr;
    VTI_TRY(get_obs(p, s, data, data_mem, &obs));
    if (s.nr > 0)
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_trace, obs, (size_t)nnt * s.nr * sizeof(float),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    VTI_TRY(forward_pass(p, s, false));
    VTI_TRY(backward_pass(p, s, true, p->d_ext, nlag));
    VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  const cudaMemcpyKind kind =
      image_mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t nxyz = (size_t)d.nx * d.ny * d.nz;
  for (int l = 0; l < nl; ++l)
    VTI_CUDA(ctx, cudaMemcpy2DAsync(image + l * nxyz, d.nx * sizeof(float), p->d_ext + l * vol,
                                    d.pitch * sizeof(float), d.nx * sizeof(float),
                                    (size_t)d.ny * d.nz, kind, ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return check_device_status(ctx);
}

int vti3d_plan_wavelet_gradient(vti3d_plan* p, const float* souloc, const int* shotid, int nshot,
                                const float* data, int data_mem, float* gwavelet, int mem) {
  if (!p) return VTI_ERR_ARG;
  vti_ctx* ctx = p->ctx;
  if (!p->have_model) return fail(ctx, VTI_ERR_ARG, "model not set");
  if (!souloc || (nshot > 0 && !shotid) || !data || !gwavelet || nshot < 0)
    return fail(ctx, VTI_ERR_ARG, "null pointer or negative shot count");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const vti3d_geom& g = p->g;
  const Dims3& d = p->d;
  const float dx2 = g.dx * g.dx, dy2 = g.dy * g.dy, dz2 = g.dz * g.dz, dt2 = g.dt * g.dt;
  const float sxs = dt2 / dx2, sys = dt2 / dy2, szs = dt2 / dz2;
  const int st = sampling_step(g), nnt = nnt_of(g), M = last_level(g, p->flags);
  VTI_TRY(ensure(ctx, &p->d_gw, &p->gw_cap, (size_t)g.nt));
  VTI_CUDA(ctx, cudaMemsetAsync(p->d_gw, 0, g.nt * sizeof(float), ctx->stream));
  Damping dmp{p->dampx, p->dampy, p->dampz};
  for (int k = 0; k < nshot; ++k) {
    ShotGeom s;
    VTI_TRY(shot_geom(p, souloc, shotid[k], &s));
    VTI_TRY(upload_shot(p, s));
    const float* obs = nullptr;
    VTI_TRY(get_obs(p, s, data, data_mem, &obs));
    if (s.nr > 0)
      VTI_CUDA(ctx, cudaMemcpyAsync(p->d_trace, obs, (size_t)nnt * s.nr * sizeof(float),
                                    cudaMemcpyDeviceToDevice, ctx->stream));
    for (int j = 0; j < 2; ++j) {
      VTI_TRY(vol_zero(ctx, d, &p->lx[j]));
      VTI_TRY(vol_zero(ctx, d, &p->lz[j]));
    }
    int LA = 0, LB = 1;
    VTI_TRY(launch_seed_adjoint(ctx, p->lx[LA].origin, p->lz[LA].origin, p->d_trace, nnt,
                                p->d_rec + p->rec_cap, p->d_rec_damp, s.nr, dt2));
    Probe probe;
    probe.x = s.sx;
    probe.y = s.sy;
    probe.z = s.sz;
    for (int i = 0; i < M - 1; ++i) {
      const int it = g.nt - 3 - i;  // modelData3d_f.cu:1103-1104
      probe.out = p->d_gw + it;
      VTI_TRY(launch_fwd3d_tma(ctx, d, p->m_lx[LA], p->m_lz[LA], p->m_lx[LB], p->m_lz[LB],
                               p->m_cpad[0], p->m_cpad[1], p->m_cpad[2], p->lz[LA].origin,
                               p->lx[LB].origin, p->lz[LB].origin, &dmp, sxs, sys, szs,
                               PointSource(), probe));
      const int ti = it + 1;
      float f = float(ti) / float(st);
      int i0 = (int)f;
      const int clamp = i0 >= nnt - 1;
      f = f - i0;
      VTI_TRY(launch_inject_residual(ctx, p->lx[LB].origin, p->lz[LB].origin, p->d_trace, nnt,
                                     clamp ? 0 : i0, f, clamp, p->d_rec, p->d_rec_damp, s.nr,
                                     dt2));
      std::swap(LA, LB);
    }
    VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  std::vector<float> h(g.nt);
  VTI_CUDA(ctx, cudaMemcpyAsync(h.data(), p->d_gw, g.nt * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  VTI_TRY(check_device_status(ctx));
  for (float& v : h) v *= dt2;  // modelData3d_f.cu:1293
  VTI_CUDA(ctx, cudaMemcpy(gwavelet, h.data(), g.nt * sizeof(float),
                           mem == VTI_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost));
  return VTI_OK;
}

int vti3d_wavelet_gradient_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11,
                               const float* c13, const float* c33, const float* souloc,
                               const int* shotid, int nshot, const float* recloc, int nrec_total,
                               const float* data, float* gwavelet, unsigned flags) {
  vti3d_plan* p = nullptr;
  VTI_TRY(one_call_plan(ctx, g, flags, &p));
  int st = vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_receivers(p, recloc, nrec_total);
  if (st == VTI_OK)
    st = vti3d_plan_wavelet_gradient(p, souloc, shotid, nshot, data, VTI_MEM_HOST, gwavelet,
                                     VTI_MEM_HOST);
  return one_call_done(ctx, p, st);
}

int vti3d_rtm_cij(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                  const float* c33, const float* wavelet, const float* souloc, const int* shotid,
                  int nshot, const float* recloc, int nrec_total, const float* data,
                  float* image, unsigned flags) {
  vti3d_plan* p = nullptr;
  VTI_TRY(one_call_plan(ctx, g, flags, &p));
  int st = vti3d_plan_set_model(p, c11, c13, c33, nullptr, nullptr, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_receivers(p, recloc, nrec_total);
  if (st == VTI_OK)
    st = vti3d_plan_rtm(p, souloc, shotid, nshot, data, VTI_MEM_HOST, image, VTI_MEM_HOST);
  return one_call_done(ctx, p, st);
}

int vti3d_gradient_cij(vti_ctx* ctx, const vti3d_geom* g, const float* cij, const float* padb,
                       const float* randb, const float* wavelet, const float* souloc,
                       const int* shotid, int nshot, const float* recloc, int nrec_total,
                       const float* dobs, float* fgcij, double* misfit, unsigned flags) {
  if (!cij) return fail(ctx, VTI_ERR_ARG, "null cij");
  vti3d_plan* p = nullptr;
  VTI_TRY(one_call_plan(ctx, g, flags, &p));
  const size_t n = (size_t)g->nx * g->ny * g->nz;
  int st = vti3d_plan_set_model(p, cij, cij + n, cij + 2 * n, padb, randb, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_wavelet(p, wavelet, VTI_MEM_HOST);
  if (st == VTI_OK) st = vti3d_plan_set_receivers(p, recloc, nrec_total);
  if (st == VTI_OK)
    st = vti3d_plan_gradient(p, souloc, shotid, nshot, dobs, VTI_MEM_HOST, fgcij, VTI_MEM_HOST,
                             misfit);
  return one_call_done(ctx, p, st);
}

}  // extern "C"
