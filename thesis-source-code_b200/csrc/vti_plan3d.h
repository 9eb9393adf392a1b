// Device-resident state of one 3D grid (vti3d_plan) and the per-shot
// helpers shared by the single-shot plan (vti_plan3d.cu) and the batched
// multi-shot executor (vti_batch3d.cu).
#pragma once

#include <cmath>
#include <vector>

#include "vti_internal.h"

#define VTI_TRY(x)                 \
  do {                             \
    int st_ = (x);                 \
    if (st_ != VTI_OK) return st_; \
  } while (0)

struct vti3d_plan {
  using Dims3 = vti::Dims3;
  using Vol = vti::Vol;
  using TileMaps = vti::TileMaps;
  vti_ctx* ctx = nullptr;
  vti3d_geom g{};
  unsigned flags = 0;
  Dims3 d{};
  Vol cpad[3], crand[3];
  bool have_rand = false;
  Vol sx[2], sz[2], lx[2], lz[2];
  Vol g11, g13, g33;
  // TMA descriptors of every volume
  TileMaps m_sx[2], m_sz[2], m_lx[2], m_lz[2], m_cpad[3], m_crand[3], m_g[3];
  float* dampx = nullptr;  // nx + ny + nz floats, one allocation
  float* dampy = nullptr;
  float* dampz = nullptr;
  std::vector<float> h_damp;  // host copy: x | y | z
  std::vector<float> wavelet;
  std::vector<float> recloc;
  int nrec_total = 0;
  // per-shot device scratch
  long long* d_rec = nullptr;
  float* d_rec_damp = nullptr;
  unsigned char* d_live = nullptr;
  size_t rec_cap = 0;
  float* d_trace = nullptr;
  size_t trace_cap = 0;
  float* d_obs = nullptr;
  size_t obs_cap = 0;
  int trace_format = VTI_TRACES_F32;  // observed traces as passed by the caller
  uint16_t* d_obs16 = nullptr;        // FP16 traces of one shot (host blocks)
  size_t obs16_cap = 0;
  float* d_obs_scale = nullptr;       // their plane scales
  size_t obs_scale_cap = 0;
  float* d_blist = nullptr;
  size_t blist_cap = 0;
  double* d_acc = nullptr;
  float* d_gw = nullptr;  // wavelet gradient accumulator (nt)
  size_t gw_cap = 0;
  float* d_ext = nullptr;  // offset-domain gathers ((2 nlag + 1) pitched volumes)
  size_t ext_cap = 0;
  double* d_part = nullptr;  // per-trace AGC misfits
  size_t part_cap = 0;
  // misfit options of the gradient (objFuncGradient3d_f.cu:743-775)
  float tpow = 0.f;
  int objtype = 0;
  int halfwidth = 20;
  int last_cur = 0;  // index into sx[] of the last forward level
  bool have_model = false;
};

namespace vti {
namespace p3d {

struct ShotGeom {
  int sx, sy, sz;
  int nr, irbegin;
  std::vector<long long> rec;   // recording / residual-injection points
  std::vector<long long> seed;  // adjoint seeding points
  std::vector<float> rec_damp;  // sponge factor at rec (0: frame cell, skipped)
  std::vector<unsigned char> live;
  std::vector<int> rec_at;      // level -> trace sample (-1: not recorded)
};


int sampling_step(const vti3d_geom& g);
int nnt_of(const vti3d_geom& g);
// Levels run: 1 + 64*G*floor((nt-2)/(64G)), or nt-1 with VTI_OPT_FULL_STEPS.
int last_level(const vti3d_geom& g, unsigned flags);
long long boundary_count(const vti3d_geom& g);
float damp_profile(int i, int n, int npad);
int check_geom(vti_ctx* ctx, const vti3d_geom* g);
// Source, receivers and record schedule of shot `is` of souloc (5 floats per
// shot) in the plan's grid.
int shot_geom(vti3d_plan* p, const float* souloc, int is, ShotGeom* s);
// Receiver tables of s into the plan's device scratch; trace buffer sized.
int upload_shot(vti3d_plan* p, const ShotGeom& s);
// Device pointer to the shot's observed traces as FP32 (copied from the host
// if needed; a VTI_TRACES_F16 block is expanded on the device).
int get_obs(vti3d_plan* p, const ShotGeom& s, const float* dobs, int mem, const float** out);
// One forward level `it` of pass 1 (sponge: pad model, traces) or pass 2
// (random-boundary model): sx[A] = level it-1, sx[B] = level it-2 in, level
// it out in sx[B].
int fwd_level(vti3d_plan* p, const ShotGeom& s, bool sponge, int A, int B, int it);
// Backward step i of pass 3 with its residual injection: source fields
// sx[SA] (current) / sx[SB] (overwritten), adjoint lx[LA] / lx[LB]
// (overwritten), imaging into g11/g13/g33.
int bwd_level(vti3d_plan* p, const ShotGeom& s, bool rtm, int SA, int SB, int LA, int LB,
              int i);
// Whole passes: forward_pass leaves level M in sx[last_cur] and M-1 in the
// other buffer; backward_pass runs the M-1 backward steps from there (nlag
// offset-domain gathers into ext when ext is given).
int forward_pass(vti3d_plan* p, const ShotGeom& s, bool sponge);
int backward_pass(vti3d_plan* p, const ShotGeom& s, bool rtm, float* ext = nullptr,
                  int nlag = 0);

template <typename T>
int ensure(vti_ctx* ctx, T** ptr, size_t* cap, size_t n) {
  if (*ptr && *cap >= n) return VTI_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *cap = 0;
  VTI_CUDA(ctx, cudaMalloc((void**)ptr, std::max<size_t>(n, 1) * sizeof(T)));
  *cap = n;
  return VTI_OK;
}

}  // namespace p3d
}  // namespace vti
