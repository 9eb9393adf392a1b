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

int forward_loop(vti3d_batch* b) {
  vti_ctx* ctx = b->ctx;
  const int M = levels(b);
  const int rgrid = (b->nentries + 255) / 256;
  for (int tick = 0; tick < M - 1; ++tick) {
    VTI_TRY(step_batch_launch(ctx, b->fwd, tick));
    if (b->nentries > 0) {
      k_record_batch<<<rgrid, 256, 0, ctx->stream>>>(b->d_recjobs, b->d_entries, b->nentries,
                                                     tick);
      VTI_LAUNCHED(ctx, "k_record_batch");
    }
  }
  return VTI_OK;
}

int backward_loop(vti3d_batch* b) {
  vti_ctx* ctx = b->ctx;
  const int M = levels(b);
  const int rgrid = (b->nentries + 255) / 256;
  for (int tick = 0; tick < M - 1; ++tick) {
    VTI_TRY(step_batch_launch(ctx, b->bwd, tick));
    if (b->nentries > 0) {
      k_inject_batch<<<rgrid, 256, 0, ctx->stream>>>(b->d_recjobs, b->d_entries, b->nentries,
                                                     tick);
      VTI_LAUNCHED(ctx, "k_inject_batch");
    }
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
  return VTI_OK;
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

int vti3d_batch_gradient(vti3d_batch* b, const float* dobs, int dobs_mem, float* fgcij,
                         int fgcij_mem, double* misfit) {
  if (!b) return VTI_ERR_ARG;
  vti_ctx* ctx = b->ctx;
  VTI_TRY(check_ready(b));
  if (!dobs) return fail(ctx, VTI_ERR_ARG, "null observed data");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const int S = (int)b->plans.size();
  const int nnt = nnt_of(b->g);
  const float dt2 = b->g.dt * b->g.dt;
  VTI_TRY(cut_windows(b));
  if (!b->tables_ok) VTI_TRY(build_tables(b));
  if (!b->d_acc) VTI_CUDA(ctx, cudaMalloc((void**)&b->d_acc, (1 + residual_blocks(ctx)) * sizeof(double)));
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
  VTI_CUDA(ctx, cudaMemsetAsync(b->d_acc, 0, sizeof(double), ctx->stream));
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
  const size_t n = (size_t)b->g.nx * b->g.ny * b->g.nz;
  if (!b->d_full) VTI_CUDA(ctx, cudaMalloc((void**)&b->d_full, 3 * n * sizeof(float)));
  VTI_CUDA(ctx, cudaMemsetAsync(b->d_full, 0, 3 * n * sizeof(float), ctx->stream));
  for (int k = 0; k < S; ++k) {
    vti3d_plan* p = b->plans[k];
    const vti3d_window& w = b->win[k];
    const Vol* gv[3] = {&p->g11, &p->g13, &p->g33};
    const int grid = grid_for(ctx, p->d.npoints());
    for (int c = 0; c < 3; ++c) {
      k_add_window<<<grid, 256, 0, ctx->stream>>>(gv[c]->origin, p->d, p->g.npad, w.x0, w.y0,
                                                  b->g.nx, b->g.ny, b->d_full + c * n);
      VTI_LAUNCHED(ctx, "k_add_window");
    }
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
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  VTI_TRY(check_device_status(ctx));
  VTI_TRY(build_tables(b));
  if (seg_fwd) *seg_fwd = b->seg_fwd;
  if (seg_bwd) *seg_bwd = b->seg_bwd;
  return VTI_OK;
}

}  // extern "C"
