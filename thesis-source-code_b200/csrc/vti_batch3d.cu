// Batched multi-shot 3D gradient.
//
// Many shots, each on its own window (subgrid) of the model, advance
// together: every time step is ONE forward launch over the items of all
// shots' pass 1 (pad model, sponge, recording) and pass 2 (random boundary,
// no sponge) - the two passes are independent, so they run side by side -
// and, after the residuals, ONE backward launch per step over all shots'
// pass 3 (time-reversed source field, adjoint, imaging). Receiver work is one
// launch per step over the receivers of all shots. The time loops can be
// captured once as CUDA graphs and replayed on every later call.
//
// Under the per-shot schedule the shots instead run one after another, each
// with the plan's own single-grid passes (fwd_level / bwd_level), which is the
// better order when every window alone fills the GPU: the single-grid step
// kernels keep their parameters in the constant bank and their neighbouring
// columns in step, and reach a higher fraction of HBM bandwidth than the
// side-by-side launches.
//
// Per shot the arithmetic is exactly that of vti3d_plan_gradient on a plan
// whose grid is the window (the same kernels' item bodies, the same source,
// recording and injection schedule), so a shot's gradient is the plan's; the
// window gradients are then added into the full model, each without the
// npad-wide x/y frame of its window (sponge and random boundary there), except
// where that frame is the model's own edge.
//
// Random boundaries are generated on the device per shot from a seed: inside
// the window's pad, c <- c * r^2 (velocity times r) with
// r = 1 - min(dist/npad, 1) * (1 - 0.7) * u, u uniform in [0,1) from a hash of
// (seed, model cell); velocity is only lowered, as in the reference's
// generator (lib/random-boundary/randomBound.h:233-248), so the random pass
// stays within the CFL bound of the model.
#include <algorithm>
#include <cstring>

#include "vti_plan3d.h"

using namespace vti;
using namespace vti::p3d;

namespace {

constexpr float kRandLow = 0.7f;

struct RecJob {
  const float* rx[2];  // pass-1 sigma written at a step of parity p
  const float* rz[2];
  float* lx[2];        // adjoint written at a backward step of parity p
  float* lz[2];
  float* trace;        // residual / traces of the shot (nnt * nr)
  const int* rec_at;   // level -> sample (-1: not recorded)
  int nnt, st, nt, t0;
  float dt2;
};

struct RecEntry {
  long long off;  // recording / injection cell
  int job, ir;
  float damp;     // sponge factor at the cell (0: frame cell)
  int pad_;
};

// recordData (injectRecord3d.cu:22-28) for every receiver of every shot
// after forward step `tick`; the arithmetic of k_record.
__global__ void k_record_batch(const RecJob* jobs, const RecEntry* e, int n, int tick) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RecEntry r = e[i];
  const RecJob& J = jobs[r.job];
  const int s = tick - J.t0;
  const int j = J.rec_at[s + 2];
  if (j < 0) return;
  const int p = s & 1;
  J.trace[(long long)r.ir * J.nnt + j] =
      (float)(kTwoThird * J.rx[p][r.off] + kOneThird * J.rz[p][r.off]);
}

// Residual injection after backward step `tick` (level it = nt-3-s, residual
// interpolated at it+1, injectRecord3d.cu:38-78); the arithmetic of
// k_inject_residual with the interpolation weights of the plan's host loop.
__global__ void k_inject_batch(const RecJob* jobs, const RecEntry* e, int n, int tick) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RecEntry r = e[i];
  const RecJob& J = jobs[r.job];
  const int s = tick - J.t0;
  const int ti = J.nt - 3 - s + 1;
  float f = float(ti) / float(J.st);
  int i0 = (int)f;
  const bool clamp = i0 >= J.nnt - 1;
  f = f - i0;
  const float* t = J.trace + (long long)r.ir * J.nnt;
  const float res = clamp ? t[J.nnt - 1] : (float)((1. - f) * t[i0] + f * t[i0 + 1]);
  const float sv = J.dt2 * res;
  const int p = 1 - (s & 1);
  J.lx[p][r.off] += r.damp * (float)(kTwoThird * sv);
  J.lz[p][r.off] += r.damp * (float)(kOneThird * sv);
}

// Window [x0, x0+nx) x [y0, y0+ny) x [0, nz) of a contiguous full model into a
// pitched volume.
__global__ void k_cut_window(const float* full, int fnx, int fny, int x0, int y0, Dims3 d,
                             float* vol) {
  const long long n = d.npoints();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long r = i / d.nx;
    const int y = (int)(r % d.ny);
    const int z = (int)(r / d.ny);
    vol[d.off(x, y, z)] = full[((long long)z * fny + (y0 + y)) * fnx + (x0 + x)];
  }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long h) {
  h ^= h >> 30;
  h *= 0xbf58476d1ce4e5b9ULL;
  h ^= h >> 27;
  h *= 0x94d049bb133111ebULL;
  h ^= h >> 31;
  return h;
}

__device__ __forceinline__ int pad_depth(int i, int n, int npad) {
  return max(max(npad - i, i - (n - 1 - npad)), 0);
}

// Random-boundary copy of the three stiffness volumes of one window.
__global__ void k_random_boundary(const float* c11, const float* c13, const float* c33,
                                  float* r11, float* r13, float* r33, Dims3 d, int npad,
                                  unsigned seed, int x0, int y0, int fnx, int fny) {
  const long long n = d.npoints();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long rr = i / d.nx;
    const int y = (int)(rr % d.ny);
    const int z = (int)(rr / d.ny);
    const long long o = d.off(x, y, z);
    const int dist = max(max(pad_depth(x, d.nx, npad), pad_depth(y, d.ny, npad)),
                         pad_depth(z, d.nz, npad));
    float m = 1.f;
    if (dist > 0) {
      const unsigned long long cell = ((unsigned long long)z * fny + (y0 + y)) * fnx + (x0 + x);
      const unsigned long long h = mix64(cell * 0x9e3779b97f4a7c15ULL + mix64(seed + 1ULL));
      const float u = (float)(h >> 40) * (1.f / 16777216.f);
      const float pct = fminf((float)dist / (float)npad, 1.f);
      const float r = 1.f - pct * (1.f - kRandLow) * u;
      m = r * r;
    }
    r11[o] = c11[o] * m;
    r13[o] = c13[o] * m;
    r33[o] = c33[o] * m;
  }
}

// full[window] += g over the window's cells that are not in its npad-wide x/y
// frame, unless that frame is the model's own edge.
__global__ void k_add_window(const float* g, Dims3 d, int npad, int x0, int y0, int fnx,
                             int fny, float* full) {
  const long long n = d.npoints();
  const int xlo = x0 == 0 ? 0 : npad, xhi = x0 + d.nx == fnx ? d.nx : d.nx - npad;
  const int ylo = y0 == 0 ? 0 : npad, yhi = y0 + d.ny == fny ? d.ny : d.ny - npad;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % d.nx);
    const long long r = i / d.nx;
    const int y = (int)(r % d.ny);
    const int z = (int)(r / d.ny);
    if (x < xlo || x >= xhi || y < ylo || y >= yhi) continue;
    full[((long long)z * fny + (y0 + y)) * fnx + (x0 + x)] += g[d.off(x, y, z)];
  }
}

int grid_for(vti_ctx* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, ctx->sm_count * 8LL));
}

}  // namespace

struct vti3d_batch {
  vti_ctx* ctx = nullptr;
  vti3d_geom g{};
  unsigned flags = 0;
  float* d_model = nullptr;  // c11 | c13 | c33, contiguous, nxyz each
  long long model_version = 0;
  std::vector<float> wavelet;
  std::vector<float> recloc;
  int nrec_total = 0;
  // shots
  std::vector<vti3d_window> win;
  std::vector<float> souloc;
  unsigned seed = 0;
  std::vector<vti3d_plan*> plans;
  std::vector<ShotGeom> geo;
  std::vector<int*> d_rec_at;
  long long cut_version = -1;  // model version cut into the windows
  // batched step launch plans
  StepBatch* fwd = nullptr;         // passes 1 and 2 of every shot
  StepBatch* bwd = nullptr;         // pass 3 of every shot
  float* d_amp = nullptr;           // forward (M-1) | backward (M-1) amplitudes
  RecJob* d_recjobs = nullptr;
  RecEntry* d_entries = nullptr;
  int nentries = 0;
  bool tables_ok = false;
  int seg_fwd = 0, seg_bwd = 0;
  bool use_graph = false;
  cudaGraphExec_t graph_fwd = nullptr, graph_bwd = nullptr;
  double* d_acc = nullptr;
  float* d_full = nullptr;  // stacked gradient, 3 * nxyz
  int schedule = VTI_BATCH_AUTO;
  int tuned = 0;  // schedule measured by vti3d_batch_autotune (0: none yet)
  int trace_format = VTI_TRACES_F32;
};

namespace {

int free_graphs(vti3d_batch* b) {
  if (b->graph_fwd) cudaGraphExecDestroy(b->graph_fwd);
  if (b->graph_bwd) cudaGraphExecDestroy(b->graph_bwd);
  b->graph_fwd = b->graph_bwd = nullptr;
  return VTI_OK;
}

void free_shots(vti3d_batch* b) {
  free_graphs(b);
  for (auto* p : b->plans) vti3d_plan_destroy(p);
  for (int* q : b->d_rec_at)
    if (q) cudaFree(q);
  b->plans.clear();
  b->geo.clear();
  b->d_rec_at.clear();
  step_batch_free(b->fwd);
  step_batch_free(b->bwd);
  b->fwd = b->bwd = nullptr;
  void* ptrs[] = {b->d_amp, b->d_recjobs, b->d_entries};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  b->d_amp = nullptr;
  b->d_recjobs = nullptr;
  b->d_entries = nullptr;
  b->tables_ok = false;
  b->cut_version = -1;
  b->tuned = 0;
}

int levels(const vti3d_batch* b) { return last_level(b->g, b->flags); }

// Batched launch plans, amplitudes and receiver tables of the current shots
// and segment lengths.
int build_tables(vti3d_batch* b) {
  vti_ctx* ctx = b->ctx;
  free_graphs(b);
  step_batch_free(b->fwd);
  step_batch_free(b->bwd);
  b->fwd = b->bwd = nullptr;
  b->tables_ok = false;
  const int S = (int)b->plans.size();
  const int M = levels(b);
  const float dt2 = b->g.dt * b->g.dt;
  const float sxs = dt2 / (b->g.dx * b->g.dx), sys = dt2 / (b->g.dy * b->g.dy),
              szs = dt2 / (b->g.dz * b->g.dz);
  const float idx2 = 1.f / (b->g.dx * b->g.dx), idy2 = 1.f / (b->g.dy * b->g.dy),
              idz2 = 1.f / (b->g.dz * b->g.dz);
  // amplitudes: forward step s -> dt2 w[s+1]; backward step s -> dt2 w[nt-2-s]
  std::vector<float> amp(2 * (size_t)std::max(M - 1, 1), 0.f);
  for (int s = 0; s < M - 1; ++s) {
    amp[s] = dt2 * b->wavelet[s + 1];
    amp[(M - 1) + s] = dt2 * b->wavelet[b->g.nt - 2 - s];
  }
  if (b->d_amp) cudaFree(b->d_amp);
  b->d_amp = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&b->d_amp, amp.size() * sizeof(float)));
  VTI_CUDA(ctx, cudaMemcpy(b->d_amp, amp.data(), amp.size() * sizeof(float),
                           cudaMemcpyHostToDevice));
  const float* ampf = b->d_amp;
  const float* ampb = b->d_amp + (M - 1);
  // after the forward loop, level M is in buffer 1 - ((M-2) & 1)
  const int last_cur = 1 - ((M - 2) & 1);
  std::vector<FwdJobSpec> fspec;
  std::vector<BwdJobSpec> bspec;
  std::vector<Damping> damps(S);
  for (int k = 0; k < S; ++k) {
    vti3d_plan* p = b->plans[k];
    const ShotGeom& sg = b->geo[k];
    damps[k] = Damping{p->dampx, p->dampy, p->dampz};
    for (int pass = 0; pass < 2; ++pass) {
      // pass 1 runs in the adjoint volumes (free until pass 3), pass 2 in sigma
      Vol* vx = pass == 0 ? p->lx : p->sx;
      Vol* vz = pass == 0 ? p->lz : p->sz;
      TileMaps* mx = pass == 0 ? p->m_lx : p->m_sx;
      TileMaps* mz = pass == 0 ? p->m_lz : p->m_sz;
      FwdJobSpec sp{};
      sp.d = p->d;
      for (int par = 0; par < 2; ++par) {
        sp.cx[par] = &mx[par];
        sp.cz[par] = &mz[par];
        sp.px[par] = &mx[1 - par];
        sp.pz[par] = &mz[1 - par];
        sp.cz_ptr[par] = vz[par].origin;
        sp.px_ptr[par] = vx[1 - par].origin;
        sp.pz_ptr[par] = vz[1 - par].origin;
      }
      const TileMaps* cm = pass == 0 ? p->m_cpad : p->m_crand;
      for (int c = 0; c < 3; ++c) sp.c[c] = &cm[c];
      sp.damp = pass == 0 ? &damps[k] : nullptr;
      sp.sx = sxs;
      sp.sy = sys;
      sp.sz = szs;
      sp.src_x = sg.sx;
      sp.src_y = sg.sy;
      sp.src_z = sg.sz;
      sp.amp = ampf;
      sp.t0 = 0;
      sp.seg = b->seg_fwd;
      fspec.push_back(sp);
    }
    BwdJobSpec sp{};
    sp.d = p->d;
    for (int par = 0; par < 2; ++par) {
      const int sa = last_cur ^ 1 ^ par, sb = 1 - sa;  // sigma cur / prev
      const int la = par, lb = 1 - par;                // lambda cur / prev
      sp.scx[par] = &p->m_sx[sa];
      sp.scz[par] = &p->m_sz[sa];
      sp.spx[par] = &p->m_sx[sb];
      sp.spz[par] = &p->m_sz[sb];
      sp.lcx[par] = &p->m_lx[la];
      sp.lcz[par] = &p->m_lz[la];
      sp.lpx[par] = &p->m_lx[lb];
      sp.lpz[par] = &p->m_lz[lb];
      sp.scz_ptr[par] = p->sz[sa].origin;
      sp.lcz_ptr[par] = p->lz[la].origin;
      sp.spx_ptr[par] = p->sx[sb].origin;
      sp.spz_ptr[par] = p->sz[sb].origin;
      sp.lpx_ptr[par] = p->lx[lb].origin;
      sp.lpz_ptr[par] = p->lz[lb].origin;
    }
    for (int c = 0; c < 3; ++c) {
      sp.c[c] = &p->m_crand[c];
      sp.g[c] = &p->m_g[c];
    }
    sp.g_ptr[0] = p->g11.origin;
    sp.g_ptr[1] = p->g13.origin;
    sp.g_ptr[2] = p->g33.origin;
    sp.damp = damps[k];
    sp.dt2 = dt2;
    sp.idx2 = idx2;
    sp.idy2 = idy2;
    sp.idz2 = idz2;
    sp.sx = sxs;
    sp.sy = sys;
    sp.sz = szs;
    sp.src_x = sg.sx;
    sp.src_y = sg.sy;
    sp.src_z = sg.sz;
    sp.amp = ampb;
    sp.t0 = 0;
    sp.seg = b->seg_bwd;
    bspec.push_back(sp);
  }
  VTI_TRY(fwd_batch_build(ctx, fspec.data(), (int)fspec.size(), &b->fwd));
  VTI_TRY(bwd_batch_build(ctx, bspec.data(), (int)bspec.size(), &b->bwd));
  // receiver tables
  std::vector<RecJob> rj(S);
  std::vector<RecEntry> ent;
  for (int k = 0; k < S; ++k) {
    vti3d_plan* p = b->plans[k];
    const ShotGeom& sg = b->geo[k];
    RecJob& J = rj[k];
    for (int par = 0; par < 2; ++par) {
      J.rx[par] = p->lx[1 - par].origin;  // pass 1 writes next = buffer 1 - parity
      J.rz[par] = p->lz[1 - par].origin;
      J.lx[par] = p->lx[par].origin;      // indexed by 1 - parity in the kernel
      J.lz[par] = p->lz[par].origin;
    }
    J.trace = p->d_trace;
    J.rec_at = b->d_rec_at[k];
    J.nnt = nnt_of(b->g);
    J.st = sampling_step(b->g);
    J.nt = b->g.nt;
    J.t0 = 0;
    J.dt2 = dt2;
    for (int ir = 0; ir < sg.nr; ++ir) {
      RecEntry e{};
      e.off = sg.rec[ir];
      e.job = k;
      e.ir = ir;
      e.damp = sg.rec_damp[ir];
      ent.push_back(e);
    }
  }
  b->nentries = (int)ent.size();
  if (b->d_recjobs) cudaFree(b->d_recjobs);
  if (b->d_entries) cudaFree(b->d_entries);
  b->d_recjobs = nullptr;
  b->d_entries = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&b->d_recjobs, std::max<size_t>(rj.size(), 1) * sizeof(RecJob)));
  VTI_CUDA(ctx, cudaMalloc((void**)&b->d_entries,
                           std::max<size_t>(ent.size(), 1) * sizeof(RecEntry)));
  if (!rj.empty())
    VTI_CUDA(ctx, cudaMemcpy(b->d_recjobs, rj.data(), rj.size() * sizeof(RecJob),
                             cudaMemcpyHostToDevice));
  if (!ent.empty())
    VTI_CUDA(ctx, cudaMemcpy(b->d_entries, ent.data(), ent.size() * sizeof(RecEntry),
                             cudaMemcpyHostToDevice));
  b->tables_ok = true;
  return VTI_OK;
}

}  // namespace

namespace {

// Window models of every shot: the model window (pad-boundary model) and its
// random-boundary copy.
int cut_windows(vti3d_batch* b) {
  if (b->cut_version == b->model_version) return VTI_OK;
  vti_ctx* ctx = b->ctx;
  const long long n = (long long)b->g.nx * b->g.ny * b->g.nz;
  for (size_t k = 0; k < b->plans.size(); ++k) {
    vti3d_plan* p = b->plans[k];
    const vti3d_window& w = b->win[k];
    const int grid = grid_for(ctx, p->d.npoints());
    for (int c = 0; c < 3; ++c) {
      k_cut_window<<<grid, 256, 0, ctx->stream>>>(b->d_model + c * n, b->g.nx, b->g.ny, w.x0,
                                                  w.y0, p->d, p->cpad[c].origin);
      VTI_LAUNCHED(ctx, "k_cut_window");
    }
    k_random_boundary<<<grid, 256, 0, ctx->stream>>>(
        p->cpad[0].origin, p->cpad[1].origin, p->cpad[2].origin, p->crand[0].origin,
        p->crand[1].origin, p->crand[2].origin, p->d, p->g.npad, b->seed + 7919u * (unsigned)k,
        w.x0, w.y0, b->g.nx, b->g.ny);
    VTI_LAUNCHED(ctx, "k_random_boundary");
  }
  b->cut_version = b->model_version;
  return VTI_OK;
}

// One side-by-side forward level (passes 1 and 2 of every shot) and its
// recording.
int fwd_tick(vti3d_batch* b, int tick) {
  vti_ctx* ctx = b->ctx;
  VTI_TRY(step_batch_launch(ctx, b->fwd, tick));
  if (b->nentries > 0) {
    k_record_batch<<<(b->nentries + 255) / 256, 256, 0, ctx->stream>>>(
        b->d_recjobs, b->d_entries, b->nentries, tick);
    VTI_LAUNCHED(ctx, "k_record_batch");
  }
  return VTI_OK;
}

// One side-by-side backward level (pass 3 of every shot) and its injection.
int bwd_tick(vti3d_batch* b, int tick) {
  vti_ctx* ctx = b->ctx;
  VTI_TRY(step_batch_launch(ctx, b->bwd, tick));
  if (b->nentries > 0) {
    k_inject_batch<<<(b->nentries + 255) / 256, 256, 0, ctx->stream>>>(
        b->d_recjobs, b->d_entries, b->nentries, tick);
    VTI_LAUNCHED(ctx, "k_inject_batch");
  }
  return VTI_OK;
}

int forward_loop(vti3d_batch* b) {
  const int M = levels(b);
  for (int tick = 0; tick < M - 1; ++tick) VTI_TRY(fwd_tick(b, tick));
  return VTI_OK;
}

int backward_loop(vti3d_batch* b) {
  const int M = levels(b);
  for (int tick = 0; tick < M - 1; ++tick) VTI_TRY(bwd_tick(b, tick));
  return VTI_OK;
}

// Ratio of the side-by-side step kernels' HBM bandwidth to the single-grid
// kernels' (measured on windows of 160..400 x 160..400 x 200 cells: 0.64 and
// 0.81 of the copy bandwidth for the backward step), and the gap between two
// single-grid launches in CTA-slot plane-steps (about 3 us; one plane-step
// of a 32 x 16 column is about 2 us).
constexpr double kSideBySideRel = 0.79;
constexpr long long kLaunchGap = 2;

// The schedule of the next gradient: the one set; under auto the one
// vti3d_batch_autotune measured faster, else per shot when the single-grid
// schedules of the windows (backward step, two CTAs per SM, launch gaps
// included) keep the SMs busy at least kSideBySideRel of the time.
int resolve_schedule(vti3d_batch* b) {
  if (b->schedule != VTI_BATCH_AUTO) return b->schedule;
  if (b->tuned) return b->tuned;
  vti_ctx* ctx = b->ctx;
  long long work = 0, cost = 0;
  for (vti3d_plan* p : b->plans) {
    long long w = 0;
    cost += step_sched_cost(ctx, p->d, 2, &w) + kLaunchGap * ctx->sm_count * 2;
    work += w;
  }
  return cost > 0 && (double)work >= kSideBySideRel * (double)cost ? VTI_BATCH_PER_SHOT
                                                                   : VTI_BATCH_SIDE_BY_SIDE;
}

// Shot k's window gradient added into the full-model gradient.
int add_window(vti3d_batch* b, int k) {
  vti_ctx* ctx = b->ctx;
  const size_t n = (size_t)b->g.nx * b->g.ny * b->g.nz;
  vti3d_plan* p = b->plans[k];
  const vti3d_window& w = b->win[k];
  const Vol* gv[3] = {&p->g11, &p->g13, &p->g33};
  const int grid = grid_for(ctx, p->d.npoints());
  for (int c = 0; c < 3; ++c) {
    k_add_window<<<grid, 256, 0, ctx->stream>>>(gv[c]->origin, p->d, p->g.npad, w.x0, w.y0,
                                                b->g.nx, b->g.ny, b->d_full + c * n);
    VTI_LAUNCHED(ctx, "k_add_window");
  }
  return VTI_OK;
}

// Runs a time loop directly, or through a CUDA graph captured on first use.
int run_loop(vti3d_batch* b, int (*loop)(vti3d_batch*), cudaGraphExec_t* exec) {
  vti_ctx* ctx = b->ctx;
  if (!b->use_graph) return loop(b);
  if (!*exec) {
    const bool timing = ctx->timing;
    ctx->timing = false;  // no event records inside the graph
    VTI_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int st = loop(b);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    ctx->timing = timing;
    if (st != VTI_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    VTI_CUDA(ctx, e);
    const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    VTI_CUDA(ctx, ei);
  }
  VTI_CUDA(ctx, cudaGraphLaunch(*exec, ctx->stream));
  // kernels inside the graph: the step launches and the receiver kernel per tick
  const StepBatch* sb = exec == &b->graph_fwd ? b->fwd : b->bwd;
  ctx->launches += (uint64_t)(step_batch_launches(sb) + (b->nentries > 0)) * (levels(b) - 1);
  return VTI_OK;
}

int zero_shot_fields(vti3d_plan* p, bool sigma, bool lambda, bool grad) {
  vti_ctx* ctx = p->ctx;
  for (int k = 0; k < 2; ++k) {
    if (sigma) {
      VTI_TRY(vol_zero(ctx, p->d, &p->sx[k]));
      VTI_TRY(vol_zero(ctx, p->d, &p->sz[k]));
    }
    if (lambda) {
      VTI_TRY(vol_zero(ctx, p->d, &p->lx[k]));
      VTI_TRY(vol_zero(ctx, p->d, &p->lz[k]));
    }
  }
  if (grad) {
    VTI_TRY(vol_zero(ctx, p->d, &p->g11));
    VTI_TRY(vol_zero(ctx, p->d, &p->g13));
    VTI_TRY(vol_zero(ctx, p->d, &p->g33));
  }
  return VTI_OK;
}

int check_ready(vti3d_batch* b) {
  if (!b->d_model) return fail(b->ctx, VTI_ERR_ARG, "model not set");
  if ((int)b->wavelet.size() != b->g.nt) return fail(b->ctx, VTI_ERR_ARG, "wavelet not set");
  if (b->plans.empty()) return fail(b->ctx, VTI_ERR_ARG, "no shots set");
  return VTI_OK;
}

}  // namespace

extern "C" {

int vti3d_batch_create(vti_ctx* ctx, const vti3d_geom* g, unsigned flags, vti3d_batch** out) {
  if (!ctx || !out) return VTI_ERR_ARG;
  *out = nullptr;
  VTI_TRY(check_geom(ctx, g));
  vti3d_batch* b = new vti3d_batch();
  b->ctx = ctx;
  b->g = *g;
  b->flags = flags;
  *out = b;
  return VTI_OK;
}

int vti3d_batch_destroy(vti3d_batch* b) {
  if (!b) return VTI_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  free_shots(b);
  void* ptrs[] = {b->d_model, b->d_acc, b->d_full};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete b;
  return VTI_OK;
}

int vti3d_batch_set_model(vti3d_batch* b, const float* c11, const float* c13, const float* c33,
                          int mem) {
  if (!b) return VTI_ERR_ARG;
  vti_ctx* ctx = b->ctx;
  if (!c11 || !c13 || !c33) return fail(ctx, VTI_ERR_ARG, "null model array");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t n = (size_t)b->g.nx * b->g.ny * b->g.nz;
  if (!b->d_model) VTI_CUDA(ctx, cudaMalloc((void**)&b->d_model, 3 * n * sizeof(float)));
  const float* cs[3] = {c11, c13, c33};
  const cudaMemcpyKind kind =
      mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  for (int c = 0; c < 3; ++c)
    VTI_CUDA(ctx, cudaMemcpyAsync(b->d_model + c * n, cs[c], n * sizeof(float), kind,
                                  ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  b->model_version++;
  // the model as stored: x-fastest rows of nx floats, no z pad planes
  Dims3 flat = make_dims(b->g.nx, b->g.ny, b->g.nz);
  flat.pitch = b->g.nx;
  flat.plane = (long long)b->g.nx * b->g.ny;
  double num = 0;
  VTI_TRY(cfl3d_device(ctx, b->g, flat, b->d_model, b->d_model + n, b->d_model + 2 * n, &num));
  return cfl_verdict(ctx, num, "batch model");
}

int vti3d_batch_set_wavelet(vti3d_batch* b, const float* wavelet, int mem) {
  if (!b || !wavelet) return VTI_ERR_ARG;
  b->wavelet.resize(b->g.nt);
  VTI_CUDA(b->ctx, cudaMemcpy(b->wavelet.data(), wavelet, b->g.nt * sizeof(float),
                              mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToHost
                                                    : cudaMemcpyHostToHost));
  for (auto* p : b->plans) p->wavelet = b->wavelet;
  b->tables_ok = false;  // amplitudes
  return VTI_OK;
}

int vti3d_batch_set_receivers(vti3d_batch* b, const float* recloc, int nrec_total) {
  if (!b || (nrec_total > 0 && !recloc) || nrec_total < 0) return VTI_ERR_ARG;
  b->recloc.assign(recloc, recloc + 4 * (size_t)nrec_total);
  b->nrec_total = nrec_total;
  return VTI_OK;
}

int vti3d_batch_set_shots(vti3d_batch* b, int nshot, const float* souloc,
                          const vti3d_window* win, unsigned seed) {
  if (!b) return VTI_ERR_ARG;
  vti_ctx* ctx = b->ctx;
  if (nshot < 1 || !souloc || !win) return fail(ctx, VTI_ERR_ARG, "no shots");
  if ((int)b->wavelet.size() != b->g.nt)
    return fail(ctx, VTI_ERR_ARG, "set the wavelet before the shots");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const vti3d_geom& G = b->g;
  for (int k = 0; k < nshot; ++k) {
    const vti3d_window& w = win[k];
    if (w.x0 < 0 || w.y0 < 0 || w.x0 + w.nx > G.nx || w.y0 + w.ny > G.ny)
      return fail(ctx, VTI_ERR_ARG, "window of shot " + std::to_string(k) +
                                        " exceeds the model");
  }
  free_shots(b);
  b->win.assign(win, win + nshot);
  b->souloc.assign(souloc, souloc + 5 * (size_t)nshot);
  b->seed = seed;
  for (int k = 0; k < nshot; ++k) {
    const vti3d_window& w = win[k];
    vti3d_geom gs = G;
    gs.nx = w.nx;
    gs.ny = w.ny;
    gs.ox = G.ox + w.x0 * G.dx;
    gs.oy = G.oy + w.y0 * G.dy;
    vti3d_plan* p = nullptr;
    int st = vti3d_plan_create(ctx, &gs, b->flags, &p);
    if (st != VTI_OK) {
      free_shots(b);
      return st;
    }
    b->plans.push_back(p);
    p->trace_format = b->trace_format;
    p->wavelet = b->wavelet;
    p->recloc = b->recloc;
    p->nrec_total = b->nrec_total;
    for (int c = 0; c < 3; ++c) {
      VTI_TRY(vol_alloc(ctx, p->d, &p->crand[c]));
      VTI_TRY(make_tile_maps(ctx, p->d, p->crand[c], &p->m_crand[c]));
    }
    p->have_rand = true;
    p->have_model = true;
    ShotGeom sg;
    VTI_TRY(shot_geom(p, b->souloc.data() + 5 * (size_t)k, 0, &sg));
    VTI_TRY(upload_shot(p, sg));
    int* d = nullptr;
    VTI_CUDA(ctx, cudaMalloc((void**)&d, sg.rec_at.size() * sizeof(int)));
    b->d_rec_at.push_back(d);
    VTI_CUDA(ctx, cudaMemcpy(d, sg.rec_at.data(), sg.rec_at.size() * sizeof(int),
                             cudaMemcpyHostToDevice));
    b->geo.push_back(std::move(sg));
  }
  return VTI_OK;
}

int vti3d_batch_set_options(vti3d_batch* b, int use_graph, int seg_fwd, int seg_bwd) {
  if (!b || seg_fwd < 0 || seg_bwd < 0) return VTI_ERR_ARG;
  if (seg_fwd != b->seg_fwd || seg_bwd != b->seg_bwd) b->tables_ok = false;
  if (!use_graph) free_graphs(b);
  b->use_graph = use_graph != 0;
  b->seg_fwd = seg_fwd;
  b->seg_bwd = seg_bwd;
  return VTI_OK;
}

int vti3d_batch_set_trace_format(vti3d_batch* b, int format) {
  if (!b) return VTI_ERR_ARG;
  if (format != VTI_TRACES_F32 && format != VTI_TRACES_F16)
    return fail(b->ctx, VTI_ERR_ARG, "unknown trace format");
  b->trace_format = format;
  for (vti3d_plan* p : b->plans) p->trace_format = format;
  return VTI_OK;
}

int vti3d_batch_set_schedule(vti3d_batch* b, int schedule) {
  if (!b) return VTI_ERR_ARG;
  if (schedule != VTI_BATCH_AUTO && schedule != VTI_BATCH_SIDE_BY_SIDE &&
      schedule != VTI_BATCH_PER_SHOT)
    return fail(b->ctx, VTI_ERR_ARG, "unknown batch schedule");
  b->schedule = schedule;
  return VTI_OK;
}

int vti3d_batch_get_schedule(vti3d_batch* b, int* schedule) {
  if (!b || !schedule) return VTI_ERR_ARG;
  *schedule = resolve_schedule(b);
  return VTI_OK;
}

int vti3d_batch_gradient(vti3d_batch* b, const float* dobs, int dobs_mem, float* fgcij,
                         int fgcij_mem, double* misfit) {
  if (!b) return VTI_ERR_ARG;
  NvtxRange nv("vti3d batched gradient");
  vti_ctx* ctx = b->ctx;
  VTI_TRY(check_ready(b));
  if (!dobs) return fail(ctx, VTI_ERR_ARG, "null observed data");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const int S = (int)b->plans.size();
  const int nnt = nnt_of(b->g);
  const float dt2 = b->g.dt * b->g.dt;
  VTI_TRY(cut_windows(b));
  if (!b->d_acc) VTI_CUDA(ctx, cudaMalloc((void**)&b->d_acc, (1 + residual_blocks(ctx)) * sizeof(double)));
  const size_t n = (size_t)b->g.nx * b->g.ny * b->g.nz;
  if (!b->d_full) VTI_CUDA(ctx, cudaMalloc((void**)&b->d_full, 3 * n * sizeof(float)));
  VTI_CUDA(ctx, cudaMemsetAsync(b->d_full, 0, 3 * n * sizeof(float), ctx->stream));
  VTI_CUDA(ctx, cudaMemsetAsync(b->d_acc, 0, sizeof(double), ctx->stream));
  if (resolve_schedule(b) == VTI_BATCH_PER_SHOT) {
    // one shot after another, the plan's passes on its window
    // (objFuncGradient3d_f.cu:600-1078 per shot)
    for (int k = 0; k < S; ++k) {
      vti3d_plan* p = b->plans[k];
      const ShotGeom& sg = b->geo[k];
      VTI_TRY(zero_shot_fields(p, false, false, true));
      VTI_TRY(forward_pass(p, sg, true));
      const float* obs = nullptr;
      VTI_TRY(get_obs(p, sg, dobs, dobs_mem, &obs));
      VTI_TRY(launch_residual(ctx, p->d_trace, obs, p->d_live, nnt, sg.nr, b->d_acc));
      VTI_TRY(forward_pass(p, sg, false));
      VTI_TRY(backward_pass(p, sg, false));
      VTI_TRY(add_window(b, k));
    }
  } else {
    if (!b->tables_ok) VTI_TRY(build_tables(b));
    // passes 1 and 2 of every shot, side by side
    for (int k = 0; k < S; ++k) {
      vti3d_plan* p = b->plans[k];
      const ShotGeom& sg = b->geo[k];
      VTI_TRY(zero_shot_fields(p, true, true, true));
      const long long o = p->d.off(sg.sx, sg.sy, sg.sz);
      // "injecting source at time 0 to wavefields at time 1" (objFuncGradient3d_f.cu:605-608)
      VTI_TRY(launch_set_point(ctx, p->lx[0].origin, p->lz[0].origin, o, dt2 * b->wavelet[0]));
      VTI_TRY(launch_set_point(ctx, p->sx[0].origin, p->sz[0].origin, o, dt2 * b->wavelet[0]));
      if (sg.nr > 0)
        VTI_CUDA(ctx, cudaMemsetAsync(p->d_trace, 0, (size_t)nnt * sg.nr * sizeof(float),
                                      ctx->stream));
    }
    VTI_TRY(run_loop(b, forward_loop, &b->graph_fwd));
    // residuals and misfit (objFuncGradient3d_f.cu:735-771), shots in order
    for (int k = 0; k < S; ++k) {
      vti3d_plan* p = b->plans[k];
      const ShotGeom& sg = b->geo[k];
      const float* obs = nullptr;
      VTI_TRY(get_obs(p, sg, dobs, dobs_mem, &obs));
      VTI_TRY(launch_residual(ctx, p->d_trace, obs, p->d_live, nnt, sg.nr, b->d_acc));
      VTI_TRY(zero_shot_fields(p, false, true, false));
      VTI_TRY(launch_seed_adjoint(ctx, p->lx[0].origin, p->lz[0].origin, p->d_trace, nnt,
                                  p->d_rec + p->rec_cap, p->d_rec_damp, sg.nr, dt2));
    }
    VTI_TRY(run_loop(b, backward_loop, &b->graph_bwd));
    // stack the window gradients
    for (int k = 0; k < S; ++k) VTI_TRY(add_window(b, k));
  }
  double acc = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&acc, b->d_acc, sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
  if (fgcij)
    VTI_CUDA(ctx, cudaMemcpyAsync(fgcij + 1, b->d_full, 3 * n * sizeof(float),
                                  fgcij_mem == VTI_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                              : cudaMemcpyDeviceToHost,
                                  ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  VTI_TRY(check_device_status(ctx));
  if (misfit) *misfit = acc / 2;
  if (fgcij) {
    const float f0 = (float)(acc / 2);
    if (fgcij_mem == VTI_MEM_DEVICE)
      VTI_CUDA(ctx, cudaMemcpy(fgcij, &f0, sizeof(float), cudaMemcpyHostToDevice));
    else
      fgcij[0] = f0;
  }
  return VTI_OK;
}

int vti3d_batch_get_shot_models(vti3d_batch* b, int k, float* cpad, float* crand) {
  if (!b) return VTI_ERR_ARG;
  vti_ctx* ctx = b->ctx;
  if (k < 0 || k >= (int)b->plans.size()) return fail(ctx, VTI_ERR_ARG, "shot index");
  VTI_TRY(check_ready(b));
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  VTI_TRY(cut_windows(b));
  vti3d_plan* p = b->plans[k];
  const size_t n = (size_t)p->d.npoints();
  for (int c = 0; c < 3; ++c) {
    if (cpad) VTI_TRY(vol_download(ctx, p->d, &p->cpad[c], cpad + c * n, VTI_MEM_HOST));
    if (crand) VTI_TRY(vol_download(ctx, p->d, &p->crand[c], crand + c * n, VTI_MEM_HOST));
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VTI_OK;
}

// Segment lengths (z planes per item) of the forward and backward batched
// launches: each candidate is timed over a few steps of the current shots
// (CUDA events), the fastest kept. The wavefields are left arbitrary; the
// next gradient starts from zero.
int vti3d_batch_autotune(vti3d_batch* b, int* seg_fwd, int* seg_bwd) {
  if (!b) return VTI_ERR_ARG;
  vti_ctx* ctx = b->ctx;
  VTI_TRY(check_ready(b));
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  VTI_TRY(cut_windows(b));
  const int M = levels(b);
  const int reps = std::min(3, M - 1);
  const int nz = b->g.nz;
  std::vector<int> cand = {0, 8, 12, 16, 24, 32, 48, 64, 96, nz};
  cudaEvent_t e0, e1;
  VTI_CUDA(ctx, cudaEventCreate(&e0));
  VTI_CUDA(ctx, cudaEventCreate(&e1));
  int best[2] = {0, 0};
  for (int which = 0; which < 2; ++which) {
    float tbest = -1.f;
    for (int c : cand) {
      if (c > nz) continue;
      if (which == 0) b->seg_fwd = c;
      else b->seg_bwd = c;
      int st = build_tables(b);
      if (st != VTI_OK) break;
      auto one = [&](int tick) {
        return step_batch_launch(ctx, which == 0 ? b->fwd : b->bwd, tick);
      };
      VTI_TRY(one(0));  // warm-up
      VTI_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
      for (int t = 0; t < reps; ++t) VTI_TRY(one(t));
      VTI_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
      VTI_CUDA(ctx, cudaEventSynchronize(e1));
      float ms = 0.f;
      VTI_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
      if (tbest < 0.f || ms < tbest) {
        tbest = ms;
        best[which] = c;
      }
    }
    if (which == 0) b->seg_fwd = best[0];
    else b->seg_bwd = best[1];
  }
  VTI_TRY(build_tables(b));
  if (b->schedule == VTI_BATCH_AUTO) {
    // one level of each schedule (both forward passes, the backward pass and
    // the receiver work of every shot), timed over `reps` levels after one
    // untimed level
    auto side = [&](int t) -> int {
      VTI_TRY(fwd_tick(b, t));
      return bwd_tick(b, t);
    };
    auto per_shot = [&](int) -> int {
      for (size_t k = 0; k < b->plans.size(); ++k) {
        vti3d_plan* p = b->plans[k];
        const ShotGeom& sg = b->geo[k];
        VTI_TRY(fwd_level(p, sg, true, 0, 1, 2));
        VTI_TRY(fwd_level(p, sg, false, 0, 1, 2));
        VTI_TRY(bwd_level(p, sg, false, 0, 1, 0, 1, 0));
      }
      return VTI_OK;
    };
    float t[2] = {0.f, 0.f};
    for (int which = 0; which < 2; ++which) {
      auto one = [&](int tick) { return which == 0 ? side(tick) : per_shot(tick); };
      VTI_TRY(one(0));
      VTI_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
      for (int r = 0; r < reps; ++r) VTI_TRY(one(r));
      VTI_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
      VTI_CUDA(ctx, cudaEventSynchronize(e1));
      VTI_CUDA(ctx, cudaEventElapsedTime(&t[which], e0, e1));
    }
    b->tuned = t[1] < t[0] ? VTI_BATCH_PER_SHOT : VTI_BATCH_SIDE_BY_SIDE;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  VTI_TRY(check_device_status(ctx));
  if (seg_fwd) *seg_fwd = b->seg_fwd;
  if (seg_bwd) *seg_bwd = b->seg_bwd;
  return VTI_OK;
}

}  // extern "C"

// ------------------------------------------------------------ serving engine
//
// Continuous batching of 3D modeling and gradient jobs of different grids.
// Jobs are admitted at tick boundaries while their device footprint fits the
// engine's byte budget; every tick is one forward launch over all jobs in a
// forward phase (modeling, or passes 1 and 2 of a gradient) and one backward
// launch over all jobs in pass 3, so jobs that arrive while others run share
// the launches. A job's state (model, random-boundary model, wavefields,
// traces) stays resident until its result is collected. Per job the
// arithmetic is that of a plan on the job's grid (vti3d_plan_model_data /
// vti3d_plan_gradient with VTI_OPT_FULL_STEPS), whatever else runs beside it.

namespace {

struct EngineJob {
  int id = 0;
  int kind = VTI_JOB_MODEL;
  vti3d_plan* p = nullptr;
  ShotGeom sg;
  int* d_rec_at = nullptr;
  float* d_amp = nullptr;  // forward (M-1) | backward (M-1)
  double* d_acc = nullptr;
  cudaEvent_t done = nullptr;
  int M = 0;
  int phase = 0;  // 0 forward, 1 backward, 2 done
  int t0 = 0;     // tick of the current phase's step 0
  size_t bytes = 0;
};

size_t vol_bytes(const vti3d_geom& g) {
  const Dims3 d = make_dims(g.nx, g.ny, g.nz);
  return (size_t)d.plane * (d.nz + 2 * kZPad) * sizeof(float);
}

}  // namespace

struct vti3d_engine {
  vti_ctx* ctx = nullptr;
  size_t max_bytes = 0, used = 0;
  int tick = 0, next_id = 1;
  std::vector<EngineJob*> jobs;
  bool dirty = true;
  StepBatch* fwd = nullptr;
  StepBatch* bwd = nullptr;
  RecJob* d_recjobs = nullptr;
  RecEntry* d_rec = nullptr;  // recording entries of jobs in a forward phase
  RecEntry* d_inj = nullptr;  // injection entries of jobs in pass 3
  size_t cap_jobs = 0, cap_rec = 0, cap_inj = 0;
  int n_rec = 0, n_inj = 0;
  cudaStream_t copy = nullptr;
};

namespace {

void engine_free_job(vti3d_engine* e, EngineJob* j) {
  if (j->p) vti3d_plan_destroy(j->p);
  if (j->d_rec_at) cudaFree(j->d_rec_at);
  if (j->d_amp) cudaFree(j->d_amp);
  if (j->d_acc) cudaFree(j->d_acc);
  if (j->done) cudaEventDestroy(j->done);
  e->used -= std::min(e->used, j->bytes);
  delete j;
}

template <typename T>
int grow(vti_ctx* ctx, T** p, size_t* cap, size_t n) {
  if (*cap >= n && *p) return VTI_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t m = std::max<size_t>(n, 1) * 2;
  VTI_CUDA(ctx, cudaMalloc((void**)p, m * sizeof(T)));
  *cap = m;
  return VTI_OK;
}

// Launch plans and receiver tables of the jobs in a forward or backward phase.
int engine_rebuild(vti3d_engine* e) {
  vti_ctx* ctx = e->ctx;
  step_batch_free(e->fwd);
  step_batch_free(e->bwd);
  e->fwd = e->bwd = nullptr;
  std::vector<FwdJobSpec> fspec;
  std::vector<BwdJobSpec> bspec;
  std::vector<Damping> damps(e->jobs.size());
  std::vector<RecJob> rj(e->jobs.size());
  std::vector<RecEntry> rec, inj;
  for (size_t k = 0; k < e->jobs.size(); ++k) {
    EngineJob* j = e->jobs[k];
    if (j->phase > 1) continue;
    vti3d_plan* p = j->p;
    const vti3d_geom& g = p->g;
    const float dt2 = g.dt * g.dt;
    const float sxs = dt2 / (g.dx * g.dx), sys = dt2 / (g.dy * g.dy), szs = dt2 / (g.dz * g.dz);
    damps[k] = Damping{p->dampx, p->dampy, p->dampz};
    if (j->phase == 0) {
      const int passes = j->kind == VTI_JOB_GRADIENT ? 2 : 1;
      for (int pass = 0; pass < passes; ++pass) {
        Vol* vx = pass == 0 ? p->lx : p->sx;
        Vol* vz = pass == 0 ? p->lz : p->sz;
        TileMaps* mx = pass == 0 ? p->m_lx : p->m_sx;
        TileMaps* mz = pass == 0 ? p->m_lz : p->m_sz;
        FwdJobSpec sp{};
        sp.d = p->d;
        for (int par = 0; par < 2; ++par) {
          sp.cx[par] = &mx[par];
          sp.cz[par] = &mz[par];
          sp.px[par] = &mx[1 - par];
          sp.pz[par] = &mz[1 - par];
          sp.cz_ptr[par] = vz[par].origin;
          sp.px_ptr[par] = vx[1 - par].origin;
          sp.pz_ptr[par] = vz[1 - par].origin;
        }
        const TileMaps* cm = pass == 0 ? p->m_cpad : p->m_crand;
        for (int c = 0; c < 3; ++c) sp.c[c] = &cm[c];
        sp.damp = pass == 0 ? &damps[k] : nullptr;
        sp.sx = sxs;
        sp.sy = sys;
        sp.sz = szs;
        sp.src_x = j->sg.sx;
        sp.src_y = j->sg.sy;
        sp.src_z = j->sg.sz;
        sp.amp = j->d_amp;
        sp.t0 = j->t0;
        sp.seg = 0;
        fspec.push_back(sp);
      }
    } else {
      const int last_cur = 1 - ((j->M - 2) & 1);
      BwdJobSpec sp{};
      sp.d = p->d;
      for (int par = 0; par < 2; ++par) {
        const int sa = last_cur ^ 1 ^ par, sb = 1 - sa;
        const int la = par, lb = 1 - par;
        sp.scx[par] = &p->m_sx[sa];
        sp.scz[par] = &p->m_sz[sa];
        sp.spx[par] = &p->m_sx[sb];
        sp.spz[par] = &p->m_sz[sb];
        sp.lcx[par] = &p->m_lx[la];
        sp.lcz[par] = &p->m_lz[la];
        sp.lpx[par] = &p->m_lx[lb];
        sp.lpz[par] = &p->m_lz[lb];
        sp.scz_ptr[par] = p->sz[sa].origin;
        sp.lcz_ptr[par] = p->lz[la].origin;
        sp.spx_ptr[par] = p->sx[sb].origin;
        sp.spz_ptr[par] = p->sz[sb].origin;
        sp.lpx_ptr[par] = p->lx[lb].origin;
        sp.lpz_ptr[par] = p->lz[lb].origin;
      }
      for (int c = 0; c < 3; ++c) {
        sp.c[c] = &p->m_crand[c];
        sp.g[c] = &p->m_g[c];
      }
      sp.g_ptr[0] = p->g11.origin;
      sp.g_ptr[1] = p->g13.origin;
      sp.g_ptr[2] = p->g33.origin;
      sp.damp = damps[k];
      sp.dt2 = dt2;
      sp.idx2 = 1.f / (g.dx * g.dx);
      sp.idy2 = 1.f / (g.dy * g.dy);
      sp.idz2 = 1.f / (g.dz * g.dz);
      sp.sx = sxs;
      sp.sy = sys;
      sp.sz = szs;
      sp.src_x = j->sg.sx;
      sp.src_y = j->sg.sy;
      sp.src_z = j->sg.sz;
      sp.amp = j->d_amp + (j->M - 1);
      sp.t0 = j->t0;
      sp.seg = 0;
      bspec.push_back(sp);
    }
    RecJob& J = rj[k];
    for (int par = 0; par < 2; ++par) {
      J.rx[par] = p->lx[1 - par].origin;
      J.rz[par] = p->lz[1 - par].origin;
      J.lx[par] = p->lx[par].origin;
      J.lz[par] = p->lz[par].origin;
    }
    J.trace = p->d_trace;
    J.rec_at = j->d_rec_at;
    J.nnt = nnt_of(g);
    J.st = sampling_step(g);
    J.nt = g.nt;
    J.t0 = j->t0;
    J.dt2 = dt2;
    for (int ir = 0; ir < j->sg.nr; ++ir) {
      RecEntry en{};
      en.off = j->sg.rec[ir];
      en.job = (int)k;
      en.ir = ir;
      en.damp = j->sg.rec_damp[ir];
      (j->phase == 0 ? rec : inj).push_back(en);
    }
  }
  if (!fspec.empty()) VTI_TRY(fwd_batch_build(ctx, fspec.data(), (int)fspec.size(), &e->fwd));
  if (!bspec.empty()) VTI_TRY(bwd_batch_build(ctx, bspec.data(), (int)bspec.size(), &e->bwd));
  VTI_TRY(grow(ctx, &e->d_recjobs, &e->cap_jobs, rj.size()));
  VTI_TRY(grow(ctx, &e->d_rec, &e->cap_rec, rec.size()));
  VTI_TRY(grow(ctx, &e->d_inj, &e->cap_inj, inj.size()));
  if (!rj.empty())
    VTI_CUDA(ctx, cudaMemcpyAsync(e->d_recjobs, rj.data(), rj.size() * sizeof(RecJob),
                                  cudaMemcpyHostToDevice, ctx->stream));
  if (!rec.empty())
    VTI_CUDA(ctx, cudaMemcpyAsync(e->d_rec, rec.data(), rec.size() * sizeof(RecEntry),
                                  cudaMemcpyHostToDevice, ctx->stream));
  if (!inj.empty())
    VTI_CUDA(ctx, cudaMemcpyAsync(e->d_inj, inj.data(), inj.size() * sizeof(RecEntry),
                                  cudaMemcpyHostToDevice, ctx->stream));
  // the host tables are released on return
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  e->n_rec = (int)rec.size();
  e->n_inj = (int)inj.size();
  e->dirty = false;
  return VTI_OK;
}

// After the tick: phase changes of jobs whose phase ran all M-1 steps.
int engine_transitions(vti3d_engine* e) {
  vti_ctx* ctx = e->ctx;
  for (EngineJob* j : e->jobs) {
    if (j->phase > 1 || e->tick - j->t0 < j->M - 1) continue;
    vti3d_plan* p = j->p;
    const int nnt = nnt_of(p->g);
    const float dt2 = p->g.dt * p->g.dt;
    if (j->phase == 0 && j->kind == VTI_JOB_GRADIENT) {
      // residual and misfit (objFuncGradient3d_f.cu:735-771), adjoint seeded
      VTI_TRY(launch_residual(ctx, p->d_trace, p->d_obs, p->d_live, nnt, j->sg.nr, j->d_acc));
      for (int k = 0; k < 2; ++k) {
        VTI_TRY(vol_zero(ctx, p->d, &p->lx[k]));
        VTI_TRY(vol_zero(ctx, p->d, &p->lz[k]));
      }
      VTI_TRY(launch_seed_adjoint(ctx, p->lx[0].origin, p->lz[0].origin, p->d_trace, nnt,
                                  p->d_rec + p->rec_cap, p->d_rec_damp, j->sg.nr, dt2));
      j->phase = 1;
      j->t0 = e->tick;
    } else {
      if (j->kind == VTI_JOB_MODEL)  // dead receivers give zero traces
        VTI_TRY(launch_residual(ctx, p->d_trace, nullptr, p->d_live, nnt, j->sg.nr, nullptr));
      j->phase = 2;
      VTI_CUDA(ctx, cudaEventRecord(j->done, ctx->stream));
    }
    e->dirty = true;
  }
  return VTI_OK;
}

EngineJob* engine_find(vti3d_engine* e, int id) {
  for (EngineJob* j : e->jobs)
    if (j->id == id) return j;
  return nullptr;
}

}  // namespace

extern "C" {

size_t vti3d_engine_job_bytes(const vti3d_job* job) {
  if (!job) return 0;
  const size_t v = vol_bytes(job->g);
  const int nvol = job->kind == VTI_JOB_GRADIENT ? 17 : 14;
  const int st = (int)std::round(job->g.sampling_rate / job->g.dt);
  const size_t nnt = st > 0 ? (size_t)(job->g.nt - 1) / st + 1 : 0;
  const size_t nr = (size_t)std::max(job->nrec, 1);
  return nvol * v + 2 * nnt * nr * sizeof(float) + nr * 32 + 2 * (size_t)job->g.nt * 8 +
         (size_t)(job->g.nx + job->g.ny + job->g.nz) * 4;
}

int vti3d_engine_create(vti_ctx* ctx, size_t max_bytes, vti3d_engine** out) {
  if (!ctx || !out) return VTI_ERR_ARG;
  *out = nullptr;
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  vti3d_engine* e = new vti3d_engine();
  e->ctx = ctx;
  e->max_bytes = max_bytes;
  if (cudaStreamCreateWithFlags(&e->copy, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return fail(ctx, VTI_ERR_DEVICE, "copy stream");
  }
  *out = e;
  return VTI_OK;
}

int vti3d_engine_destroy(vti3d_engine* e) {
  if (!e) return VTI_OK;
  cudaSetDevice(e->ctx->device);
  cudaStreamSynchronize(e->ctx->stream);
  cudaStreamSynchronize(e->copy);
  for (EngineJob* j : e->jobs) engine_free_job(e, j);
  step_batch_free(e->fwd);
  step_batch_free(e->bwd);
  void* ptrs[] = {e->d_recjobs, e->d_rec, e->d_inj};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  cudaStreamDestroy(e->copy);
  delete e;
  return VTI_OK;
}

int vti3d_engine_submit(vti3d_engine* e, const vti3d_job* job, int* id) {
  if (!e || !job || !id) return VTI_ERR_ARG;
  vti_ctx* ctx = e->ctx;
  *id = 0;
  if (job->kind != VTI_JOB_MODEL && job->kind != VTI_JOB_GRADIENT)
    return fail(ctx, VTI_ERR_ARG, "unknown job kind");
  if (!job->c11 || !job->c13 || !job->c33 || !job->wavelet || !job->souloc ||
      (job->nrec > 0 && !job->recloc) || (job->kind == VTI_JOB_GRADIENT && !job->dobs))
    return fail(ctx, VTI_ERR_ARG, "null job array");
  VTI_TRY(check_geom(ctx, &job->g));
  VTI_TRY(cfl_verdict(ctx, vti3d_cfl_number(&job->g, job->c11, job->c13, job->c33), "job model"));
  const size_t bytes = vti3d_engine_job_bytes(job);
  if (e->used + bytes > e->max_bytes)
    return fail(ctx, VTI_ERR_BUSY, "engine memory budget full; submit again later");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  EngineJob* j = new EngineJob();
  j->kind = job->kind;
  j->bytes = bytes;
  e->used += bytes;
  int st = VTI_OK;
  auto fail_job = [&](int s) {
    engine_free_job(e, j);
    return s;
  };
  const unsigned flags = VTI_OPT_FULL_STEPS;
  st = vti3d_plan_create(ctx, &job->g, flags, &j->p);
  if (st != VTI_OK) return fail_job(st);
  vti3d_plan* p = j->p;
  p->wavelet.assign(job->wavelet, job->wavelet + job->g.nt);
  p->recloc.assign(job->recloc, job->recloc + 4 * (size_t)job->nrec);
  p->nrec_total = job->nrec;
  const Dims3& d = p->d;
  const float* cs[3] = {job->c11, job->c13, job->c33};
  for (int c = 0; c < 3 && st == VTI_OK; ++c) st = vol_upload(ctx, d, &p->cpad[c], cs[c], VTI_MEM_HOST);
  if (st != VTI_OK) return fail_job(st);
  p->have_model = true;
  if (job->kind == VTI_JOB_GRADIENT) {
    for (int c = 0; c < 3 && st == VTI_OK; ++c) {
      st = vol_alloc(ctx, d, &p->crand[c]);
      if (st == VTI_OK) st = make_tile_maps(ctx, d, p->crand[c], &p->m_crand[c]);
    }
    if (st != VTI_OK) return fail_job(st);
    p->have_rand = true;
    if (job->randb) {
      const long long nb = boundary_count(job->g);
      st = ensure(ctx, &p->d_blist, &p->blist_cap, (size_t)nb);
      for (int c = 0; c < 3 && st == VTI_OK; ++c) {
        const cudaError_t ce =
            cudaMemcpyAsync(p->d_blist, job->randb + (size_t)c * nb, nb * sizeof(float),
                            cudaMemcpyHostToDevice, ctx->stream);
        st = ce == cudaSuccess ? launch_boundary_merge(ctx, d, job->g.npad, p->cpad[c].origin,
                                                       p->d_blist, p->crand[c].origin)
                               : cuda_check(ctx, ce, "random boundary upload");
        if (st == VTI_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
          st = fail(ctx, VTI_ERR_DEVICE, "random boundary upload");
      }
    } else {
      k_random_boundary<<<grid_for(ctx, d.npoints()), 256, 0, ctx->stream>>>(
          p->cpad[0].origin, p->cpad[1].origin, p->cpad[2].origin, p->crand[0].origin,
          p->crand[1].origin, p->crand[2].origin, d, job->g.npad, job->seed, 0, 0, job->g.nx,
          job->g.ny);
      ctx->launches++;
      if (cudaGetLastError() != cudaSuccess) st = fail(ctx, VTI_ERR_DEVICE, "k_random_boundary");
    }
    if (st != VTI_OK) return fail_job(st);
  }
  st = shot_geom(p, job->souloc, 0, &j->sg);
  if (st == VTI_OK) st = upload_shot(p, j->sg);
  if (st != VTI_OK) return fail_job(st);
  j->M = last_level(job->g, flags);
  if (j->M < 2) return fail_job(fail(ctx, VTI_ERR_ARG, "fewer than 3 time samples"));
  const int nnt = nnt_of(job->g);
  const float dt2 = job->g.dt * job->g.dt;
  std::vector<float> amp(2 * (size_t)(j->M - 1));
  for (int s = 0; s < j->M - 1; ++s) {
    amp[s] = dt2 * p->wavelet[s + 1];
    amp[(j->M - 1) + s] = dt2 * p->wavelet[job->g.nt - 2 - s];
  }
  if (cudaMalloc((void**)&j->d_amp, amp.size() * sizeof(float)) != cudaSuccess ||
      cudaMalloc((void**)&j->d_rec_at, j->sg.rec_at.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&j->d_acc, (1 + residual_blocks(ctx)) * sizeof(double)) != cudaSuccess ||
      cudaEventCreateWithFlags(&j->done, cudaEventDisableTiming) != cudaSuccess)
    return fail_job(fail(ctx, VTI_ERR_OOM, "job tables"));
  if (cudaMemcpy(j->d_amp, amp.data(), amp.size() * sizeof(float), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(j->d_rec_at, j->sg.rec_at.data(), j->sg.rec_at.size() * sizeof(int),
                 cudaMemcpyHostToDevice) != cudaSuccess)
    return fail_job(fail(ctx, VTI_ERR_DEVICE, "job tables"));
  if (job->kind == VTI_JOB_GRADIENT) {
    const float* obs = nullptr;
    st = get_obs(p, j->sg, job->dobs, VTI_MEM_HOST, &obs);
    if (st != VTI_OK) return fail_job(st);
  }
  // fields of step 0: level 1 holds the source (objFuncGradient3d_f.cu:605-608)
  for (int k = 0; k < 2 && st == VTI_OK; ++k) {
    st = vol_zero(ctx, d, &p->sx[k]);
    if (st == VTI_OK) st = vol_zero(ctx, d, &p->sz[k]);
    if (st == VTI_OK) st = vol_zero(ctx, d, &p->lx[k]);
    if (st == VTI_OK) st = vol_zero(ctx, d, &p->lz[k]);
  }
  if (st == VTI_OK && job->kind == VTI_JOB_GRADIENT) {
    st = vol_zero(ctx, d, &p->g11);
    if (st == VTI_OK) st = vol_zero(ctx, d, &p->g13);
    if (st == VTI_OK) st = vol_zero(ctx, d, &p->g33);
  }
  const long long o = d.off(j->sg.sx, j->sg.sy, j->sg.sz);
  if (st == VTI_OK) st = launch_set_point(ctx, p->lx[0].origin, p->lz[0].origin, o, dt2 * p->wavelet[0]);
  if (st == VTI_OK && job->kind == VTI_JOB_GRADIENT)
    st = launch_set_point(ctx, p->sx[0].origin, p->sz[0].origin, o, dt2 * p->wavelet[0]);
  if (st == VTI_OK && j->sg.nr > 0 &&
      cudaMemsetAsync(p->d_trace, 0, (size_t)nnt * j->sg.nr * sizeof(float), ctx->stream) !=
          cudaSuccess)
    st = fail(ctx, VTI_ERR_DEVICE, "trace reset");
  if (st == VTI_OK && cudaMemsetAsync(j->d_acc, 0, sizeof(double), ctx->stream) != cudaSuccess)
    st = fail(ctx, VTI_ERR_DEVICE, "misfit reset");
  if (st == VTI_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    st = fail(ctx, VTI_ERR_DEVICE, "job set-up");
  if (st != VTI_OK) return fail_job(st);
  j->phase = 0;
  j->t0 = e->tick;
  j->id = e->next_id++;
  e->jobs.push_back(j);
  e->dirty = true;
  *id = j->id;
  return VTI_OK;
}

int vti3d_engine_step(vti3d_engine* e, int ticks, int* active) {
  if (!e || ticks < 0) return VTI_ERR_ARG;
  NvtxRange nv("vti3d engine ticks");
  vti_ctx* ctx = e->ctx;
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  for (int i = 0; i < ticks; ++i) {
    bool any = false;
    for (EngineJob* j : e->jobs) any |= j->phase <= 1;
    if (!any) break;
    if (e->dirty) VTI_TRY(engine_rebuild(e));
    if (e->fwd) VTI_TRY(step_batch_launch(ctx, e->fwd, e->tick));
    if (e->n_rec > 0) {
      k_record_batch<<<(e->n_rec + 255) / 256, 256, 0, ctx->stream>>>(e->d_recjobs, e->d_rec,
                                                                       e->n_rec, e->tick);
      VTI_LAUNCHED(ctx, "k_record_batch");
    }
    if (e->bwd) VTI_TRY(step_batch_launch(ctx, e->bwd, e->tick));
    if (e->n_inj > 0) {
      k_inject_batch<<<(e->n_inj + 255) / 256, 256, 0, ctx->stream>>>(e->d_recjobs, e->d_inj,
                                                                       e->n_inj, e->tick);
      VTI_LAUNCHED(ctx, "k_inject_batch");
    }
    e->tick++;
    VTI_TRY(engine_transitions(e));
  }
  if (active) {
    int n = 0;
    for (EngineJob* j : e->jobs) n += j->phase <= 1;
    *active = n;
  }
  return VTI_OK;
}

int vti3d_engine_poll(vti3d_engine* e, int* ids, int max_ids, int* n_done) {
  if (!e || !n_done || (max_ids > 0 && !ids)) return VTI_ERR_ARG;
  int n = 0;
  for (EngineJob* j : e->jobs) {
    if (j->phase != 2 || n >= max_ids) continue;
    const cudaError_t q = cudaEventQuery(j->done);
    if (q == cudaSuccess) ids[n++] = j->id;
    else if (q != cudaErrorNotReady) return cuda_check(e->ctx, q, "job completion");
  }
  *n_done = n;
  return VTI_OK;
}

int vti3d_engine_result(vti3d_engine* e, int id, float* out, double* misfit) {
  if (!e) return VTI_ERR_ARG;
  vti_ctx* ctx = e->ctx;
  EngineJob* j = engine_find(e, id);
  if (!j) return fail(ctx, VTI_ERR_ARG, "unknown job id");
  if (j->phase != 2) return fail(ctx, VTI_ERR_BUSY, "job not finished");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  vti3d_plan* p = j->p;
  // copies on the engine's copy stream, after the job's last step only
  VTI_CUDA(ctx, cudaStreamWaitEvent(e->copy, j->done, 0));
  double acc = 0;
  const int nnt = nnt_of(p->g);
  if (j->kind == VTI_JOB_MODEL) {
    if (out && j->sg.nr > 0)
      VTI_CUDA(ctx, cudaMemcpyAsync(out, p->d_trace, (size_t)nnt * j->sg.nr * sizeof(float),
                                    cudaMemcpyDeviceToHost, e->copy));
  } else {
    VTI_CUDA(ctx, cudaMemcpyAsync(&acc, j->d_acc, sizeof(double), cudaMemcpyDeviceToHost,
                                  e->copy));
    if (out) {
      const size_t n = (size_t)p->d.npoints();
      const Vol* gv[3] = {&p->g11, &p->g13, &p->g33};
      for (int c = 0; c < 3; ++c)
        VTI_CUDA(ctx, cudaMemcpy2DAsync(out + 1 + c * n, p->d.nx * sizeof(float),
                                        gv[c]->origin, p->d.pitch * sizeof(float),
                                        p->d.nx * sizeof(float), (size_t)p->d.ny * p->d.nz,
                                        cudaMemcpyDeviceToHost, e->copy));
    }
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(e->copy));
  if (j->kind == VTI_JOB_GRADIENT) {
    if (misfit) *misfit = acc / 2;
    if (out) out[0] = (float)(acc / 2);
  }
  // release the job's device state
  e->jobs.erase(std::find(e->jobs.begin(), e->jobs.end(), j));
  engine_free_job(e, j);
  e->dirty = true;
  return check_device_status(ctx);
}

int vti3d_engine_cancel(vti3d_engine* e, int id) {
  if (!e) return VTI_ERR_ARG;
  vti_ctx* ctx = e->ctx;
  EngineJob* j = engine_find(e, id);
  if (!j) return fail(ctx, VTI_ERR_ARG, "unknown job id");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  // nothing of the job may be in flight when its memory goes: the launches
  // that advanced it are on the context stream, its result copies on the
  // copy stream
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(e->copy));
  e->jobs.erase(std::find(e->jobs.begin(), e->jobs.end(), j));
  engine_free_job(e, j);
  e->dirty = true;
  return VTI_OK;
}

int vti3d_engine_stats(vti3d_engine* e, size_t* used_bytes, int* jobs, int* tick) {
  if (!e) return VTI_ERR_ARG;
  if (used_bytes) *used_bytes = e->used;
  if (jobs) *jobs = (int)e->jobs.size();
  if (tick) *tick = e->tick;
  return VTI_OK;
}

}  // extern "C"
