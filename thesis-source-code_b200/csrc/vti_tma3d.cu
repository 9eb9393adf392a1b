// 3D VTI step kernels, sm_100a: TMA-staged 2.5D blocking.
//
// Work decomposition. The grid is cut into 32 x 16 columns whose x origin is
// a multiple of 32 (so every 128-byte TMA row is one L2 line; cells x < 4 and
// x >= nx-4 are loaded as halo but not updated), y from 4. Each column is cut
// into equal z-segments; an item is one (column, segment) pair, numbered
// segment-major. Persistent CTAs (resident slots = SMs x CTAs per SM) take
// items cyclically, so the CTAs of one wave start their segments together
// and neighbouring columns walk down z in step: the halo and the 128-byte
// lines two columns share are read from DRAM once and hit in L2 for the
// other. The segment length is chosen on the host to balance whole waves
// against the cost of restarting the z register queue.
//
// Pipeline. Warp 8 (producer) issues, for every plane of its range, TMA tile
// loads (cp.async.bulk.tensor.3d, no multicast) of all input planes into a
// ring of shared-memory stages: the current sigma_x (and lambda_x) plane with
// a 4-cell halo, the sigma_z (lambda_z) plane 4 below for the register queue,
// prev, c11/c13/c33 and, in the backward kernel, the gradient tiles. Each
// stage completes on an mbarrier with a transaction count; consumers (warps
// 0-7, two rows each) release a stage with one arrive per warp. Out-of-range
// tiles at the far x/y edges are zero-filled by the TMA unit.
//
// All waits are bounded: a wait that runs out sets VTI_ERR_TIMEOUT in the
// context's status word and the CTA stops.
//
// Arithmetic and the sponge rule are those of vti_kernels3d.cu (see there);
// the reference is lib/vti-fwi-3d/gpu/kernel3d.cu:3-74,222-298 and
// abc3d.cu:82-126.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "vti_tma_common.cuh"

namespace vti {

#define VTI_TRY_ST(x)              \
  do {                             \
    int st_ = (x);                 \
    if (st_ != VTI_OK) return st_; \
  } while (0)

namespace {

// ------------------------------------------------------------ forward
// Forward step arguments: the part every step of a job shares and the part
// that alternates with the step parity (which buffer is cur / prev).
struct FwdCommon {
  Dims3 d;
  Sched sc;
  const float* dampx;  // null: no sponge
  const float* dampy;
  const float* dampz;
  float sx, sy, sz;
  PointSource src;     // amp: single launches only
  const float* amp;    // batched: source amplitude per step
  int t0;              // batched: tick of the job's step 0
  const float* c11;    // the model, read per point with read-only loads
  const float* c13;
  const float* c33;
};
struct FwdPar {
  const float* cz;  // cur sigma_z (queue initialisation)
  float* px;        // prev in / next out
  float* pz;
};
struct FwdArgs {
  FwdCommon c;
  FwdPar p;
  Probe probe;
  int* status;
};

constexpr int F_STAGES = 6;
// stage layout: [halo x][z+4][prev x][prev z]. The model (c11, c13, c33) is
// not staged: each consumer thread reads its own pair with read-only loads
// issued before it waits for the plane's stage, so a stage is 10 KB and six
// of them per CTA fit three CTAs per SM (five stages in flight per CTA).
constexpr int F_OFF_H = 0;
constexpr int F_OFF_Z = HALO_BYTES;
constexpr int F_OFF_PX = F_OFF_Z + PLAIN_BYTES;
constexpr int F_OFF_PZ = F_OFF_PX + PLAIN_BYTES;
constexpr int F_STAGE_BYTES = F_OFF_PZ + PLAIN_BYTES;  // 9984
constexpr int F_SMEM = F_STAGES * F_STAGE_BYTES + 1024 + 2 * F_STAGES * 8;
static_assert(3 * F_SMEM <= 228 * 1024, "three forward CTAs per SM");

struct FwdMaps {
  CUtensorMap cx, cz, px, pz;
};

// The model pair of one thread at plane z (zeros where neither point is in
// the update region; x + 1 < pitch always).
__device__ __forceinline__ void model_pair(const float* c11, const float* c13, const float* c33,
                                           long long i, bool any, float2& a11, float2& a13,
                                           float2& a33) {
  const float2 zero = make_float2(0.f, 0.f);
  a11 = any ? __ldg(reinterpret_cast<const float2*>(c11 + i)) : zero;
  a13 = any ? __ldg(reinterpret_cast<const float2*>(c13 + i)) : zero;
  a33 = any ? __ldg(reinterpret_cast<const float2*>(c33 + i)) : zero;
}

// Producer side of one item: TMA loads of every plane of the item's range.
__device__ __forceinline__ bool fwd_produce(const FwdCommon& a, const FwdMaps& m, int* status,
                                            int li, unsigned char* smem, uint64_t* full,
                                            uint64_t* empty, long long& k) {
  int bx, by, z0, z1;
  item(a.sc, li, bx, by, z0, z1);
  const int x0 = bx * TX, y0 = kHalo + by * TY;
  for (int z = z0; z < z1; ++z, ++k) {
    const int s = (int)(k % F_STAGES);
    if (k >= F_STAGES && !mbar_wait(&empty[s], (uint32_t)(((k / F_STAGES) & 1) ^ 1), status))
      return false;
    const int zp = z + kZPad;
    unsigned char* st = smem + s * F_STAGE_BYTES;
    mbar_arrive_expect_tx(&full[s], F_STAGE_BYTES);
    tma_load(st + F_OFF_H, &m.cx, &full[s], x0 - kHalo, y0 - kHalo, zp);
    tma_load(st + F_OFF_Z, &m.cz, &full[s], x0, y0, zp + kHalo);
    tma_load(st + F_OFF_PX, &m.px, &full[s], x0, y0, zp);
    tma_load(st + F_OFF_PZ, &m.pz, &full[s], x0, y0, zp);
  }
  return true;
}

// Consumer side of one item. Thread (lane, warp) owns the x pair
// x0 + 2*(lane%16) + {0,1} of tile row 2*warp + lane/16; shared-memory reads
// and global stores are float2.
// kExact: the exact-mode forward operator whose discrete adjoint the
// Gauss-Newton product uses: centred damping next = D (C L cur + 2 cur + src)
// - (2D - 1) prev (energy-stable for D <= 1), no block-order reading of the
// z stencil.
template <bool kProbe, bool kExact = false>
__device__ __forceinline__ bool fwd_consume(const FwdCommon& a, const FwdPar& bp,
                                            const Probe& probe, int* status, int li, float amp,
                                            const unsigned char* smem, uint64_t* full,
                                            uint64_t* empty, long long& k, int warp, int lane) {
  const bool damp = a.dampz != nullptr;
  const int ry = warp * 2 + (lane >> 4);
  const int xo = 2 * (lane & 15);
  const int sr = (ry + kHalo) * HX + xo + kHalo;  // centre in the halo tile
  const int pi = ry * TX + xo;                    // centre in a plain tile
  float2 q[9];  // z queue of the pair: planes z-4 .. z+4
  float dxy[2];
  int bx, by, z0, z1;
  item(a.sc, li, bx, by, z0, z1);
  const int x = bx * TX + xo;
  const int y = kHalo + by * TY + ry;
  const bool vy = y < a.d.ny - kHalo;
  const bool v0 = vy && x >= kHalo && x < a.d.nx - kHalo;
  const bool v1 = vy && x + 1 >= kHalo && x + 1 < a.d.nx - kHalo;
  const int off = y * a.d.pitch + x;  // x + 1 < pitch: 32 * gx <= pitch
  // which of this thread's two points (0, 1; else -1) holds the source / probe
  const int src_e = (y == a.src.y && a.src.x >= 0) ? a.src.x - x : -1;
  const int prb_e = (kProbe && y == probe.y && probe.x >= 0) ? probe.x - x : -1;
  dxy[0] = (damp && v0) ? a.dampx[x] * a.dampy[y] : 1.f;
  dxy[1] = (damp && v1) ? a.dampx[x + 1] * a.dampy[y] : 1.f;
  // start the queue: planes z0-4 .. z0+3 from global
  q[0] = make_float2(0.f, 0.f);
#pragma unroll
  for (int kk = 1; kk < 9; ++kk) {
    const int zz = z0 - 5 + kk;
    float2 v = (v0 || v1)
                   ? __ldg(reinterpret_cast<const float2*>(bp.cz + (long long)zz * a.d.plane + off))
                   : make_float2(0.f, 0.f);
    // planes of the block above z0 were already damped as "cur"
    if (!kExact && damp && zz >= 0 && (zz >> 2) < (z0 >> 2)) {
      v.x *= dxy[0] * a.dampz[zz];
      v.y *= dxy[1] * a.dampz[zz];
    }
    q[kk] = v;
  }
  // z damping factors in registers: dzr holds planes z-3..z once plane z
  // is entered (the block transition rescales those four queue entries);
  // the next plane's factor is fetched one plane ahead
  float dzr[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) dzr[j] = (damp && z0 - 4 + j >= 0) ? a.dampz[z0 - 4 + j] : 1.f;
  float dz_next = damp ? a.dampz[z0] : 1.f;
  for (int z = z0; z < z1; ++z, ++k) {
    const float dz = dz_next;
    if (damp && z + 1 < z1) dz_next = a.dampz[z + 1];
#pragma unroll
    for (int j = 0; j < 3; ++j) dzr[j] = dzr[j + 1];
    dzr[3] = dz;
    // the model pair: loads issued before the stage wait
    float2 c11, c13, c33;
    model_pair(a.c11, a.c13, a.c33, (long long)z * a.d.plane + off, v0 || v1, c11, c13, c33);
    const int s = (int)(k % F_STAGES);
    if (!mbar_wait(&full[s], (uint32_t)((k / F_STAGES) & 1), status)) return false;
    const unsigned char* st = smem + s * F_STAGE_BYTES;
    const float* sh = (const float*)(st + F_OFF_H) + sr;
    const float* pl = (const float*)(st + F_OFF_Z) + pi;  // [z+4][prev x][prev z]
    constexpr int T = TX * TY;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) q[kk] = q[kk + 1];
    q[8] = ld2(pl);
    // the row x-4 .. x+5 and the column pairs y +- 1..4
    float r[10];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const float2 t = ld2(sh - 4 + 2 * j);
      r[2 * j] = t.x;
      r[2 * j + 1] = t.y;
    }
    float2 ym[4], yp[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      ym[j] = ld2(sh - (j + 1) * HX);
      yp[j] = ld2(sh + (j + 1) * HX);
    }
    const float2 px = ld2(pl + T), pz = ld2(pl + 2 * T);
    stage_release(&empty[s], lane);
    float nxv[2], nzv[2];
    if (kExact) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        auto pick = [e](float2 v) { return e ? v.y : v.x; };
        const float c = r[4 + e];
        const float lxx = lap9(c, r[3 + e], r[5 + e], r[2 + e], r[6 + e], r[1 + e], r[7 + e],
                               r[e], r[8 + e]);
        const float lyy = lap9(c, pick(ym[0]), pick(yp[0]), pick(ym[1]), pick(yp[1]),
                               pick(ym[2]), pick(yp[2]), pick(ym[3]), pick(yp[3]));
        const float lzz = lap9(pick(q[4]), pick(q[3]), pick(q[5]), pick(q[2]), pick(q[6]),
                               pick(q[1]), pick(q[7]), pick(q[0]), pick(q[8]));
        const float lxy = fmaf(lyy, a.sy, lxx * a.sx);
        const float lz = lzz * a.sz;
        const float dd = dxy[e] * dz;
        const float a11 = pick(c11), a13 = pick(c13), a33 = pick(c33);
        // centred damping: D (C L cur + 2 cur + src) - (2D - 1) prev
        nxv[e] = fmaf(a11, lxy, fmaf(a13, lz, 2.f * c));
        nzv[e] = fmaf(a13, lxy, fmaf(a33, lz, 2.f * pick(q[4])));
        if (src_e == e && z == a.src.z) {
          nxv[e] += amp;
          nzv[e] += amp;
        }
        nxv[e] = fmaf(dd, nxv[e], -(2.f * dd - 1.f) * pick(px));
        nzv[e] = fmaf(dd, nzv[e], -(2.f * dd - 1.f) * pick(pz));
      }
    } else {
      // the y and z stencils and the update of both points as packed FP32
      // pairs (each lane rounded as the scalar operation); the x stencil per
      // point, its neighbour pairs straddling the loaded float2s
      const float2 c2 = make_float2(r[4], r[5]);
      float2 lxx;
      lxx.x = lap9(r[4], r[3], r[5], r[2], r[6], r[1], r[7], r[0], r[8]);
      lxx.y = lap9(r[5], r[4], r[6], r[3], r[7], r[2], r[8], r[1], r[9]);
      const float2 lyy = lap9_2(c2, ym[0], yp[0], ym[1], yp[1], ym[2], yp[2], ym[3], yp[3]);
      const float2 lzz = lap9_2(q[4], q[3], q[5], q[2], q[6], q[1], q[7], q[0], q[8]);
      const float2 lxy = fma2(lyy, splat(a.sy), mul2(lxx, splat(a.sx)));
      const float2 lz = mul2(lzz, splat(a.sz));
      const float2 dd = mul2(make_float2(dxy[0], dxy[1]), splat(dz));
      const float2 ndd = mul2(dd, splat(-1.f));
      // 2 cur - dd prev, rounded once
      float2 nx = fma2(c11, lxy, fma2(c13, lz, fma2(ndd, px, mul2(splat(2.f), c2))));
      float2 nz = fma2(c13, lxy, fma2(c33, lz, fma2(ndd, pz, mul2(splat(2.f), q[4]))));
      if (kProbe && z == probe.z) {
        if (prb_e == 0) *probe.out += nx.x + nz.x;
        if (prb_e == 1) *probe.out += nx.y + nz.y;
      }
      if (z == a.src.z) {
        if (src_e == 0) {
          nx.x += amp;
          nz.x += amp;
        }
        if (src_e == 1) {
          nx.y += amp;
          nz.y += amp;
        }
      }
      nx = mul2(nx, dd);
      nz = mul2(nz, dd);
      nxv[0] = nx.x;
      nxv[1] = nx.y;
      nzv[0] = nz.x;
      nzv[1] = nz.y;
    }
    const long long i = (long long)z * a.d.plane + off;
    if (v0 && v1) {
      *reinterpret_cast<float2*>(bp.px + i) = make_float2(nxv[0], nxv[1]);
      *reinterpret_cast<float2*>(bp.pz + i) = make_float2(nzv[0], nzv[1]);
    } else {
      if (v0) {
        bp.px[i] = nxv[0];
        bp.pz[i] = nzv[0];
      }
      if (v1) {
        bp.px[i + 1] = nxv[1];
        bp.pz[i + 1] = nzv[1];
      }
    }
    // entering the next plane: if it starts a new 4-plane block of the same
    // column, the four planes of the block just finished become "damped cur"
    if (!kExact && damp && ((z + 1) & 3) == 0 && z + 1 < a.d.nz) {
      // after the shift at z+1, entries 0..3 hold planes z-3..z; they are
      // entries 1..4 now
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        q[kk + 1] = mul2(q[kk + 1], make_float2(dxy[0] * dzr[kk], dxy[1] * dzr[kk]));
    }
  }
  return true;
}

// kProbe: the probe point of FwdArgs is read out (wavelet gradient); the
// propagation kernels are instantiated without it.
template <bool kProbe, bool kExact>
__global__ void __launch_bounds__(NTHREADS, 3)
    k_fwd3d_tma(const __grid_constant__ FwdMaps m0, const __grid_constant__ FwdArgs a0) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<F_STAGES, F_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;  // planes issued / consumed by this CTA
  if (warp == NCW) {  // ---------------- producer
    if (lane == 0)
      for (int it = blockIdx.x; it < a0.c.sc.items; it += gridDim.x)
        if (!fwd_produce(a0.c, m0, a0.status, it, smem, full, empty, k)) break;
    return;
  }
  for (int it = blockIdx.x; it < a0.c.sc.items; it += gridDim.x)
    if (!fwd_consume<kProbe, kExact>(a0.c, a0.p, a0.probe, a0.status, it, a0.c.src.amp, smem,
                                     full, empty, k, warp, lane))
      break;
}

// Batched launches: the arguments of up to kMaxFwdJobs jobs travel as kernel
// parameters (constant bank), indexed by a job number that is uniform over
// the CTA, so the item bodies read them as they read a single launch's
// parameters. Job j's items are [base[j], base[j+1]); its step is
// tick - t0, whose parity selects the buffer roles. The TMA descriptors
// (2 per job) are in global memory.
constexpr int kMaxFwdJobs = 128;
constexpr int kMaxBwdJobs = 96;

struct FwdBatch {
  const FwdMaps* maps;  // [2 * job + parity]
  int* status;
  int njobs, items, tick;
  int base[kMaxFwdJobs + 1];
  FwdCommon c[kMaxFwdJobs];
  FwdPar p[kMaxFwdJobs][2];
};

template <typename Batch>
__device__ __forceinline__ int find_job(const Batch& b, int item) {
  int lo = 0, hi = b.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.base[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(NTHREADS, 3) k_fwd3d_batch(const __grid_constant__ FwdBatch B) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<F_STAGES, F_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0)
      for (int it = blockIdx.x; it < B.items; it += gridDim.x) {
        const int j = find_job(B, it);
        const int par = (B.tick - B.c[j].t0) & 1;
        if (!fwd_produce(B.c[j], B.maps[2 * j + par], B.status, it - B.base[j], smem, full,
                         empty, k))
          break;
      }
    return;
  }
  const Probe none;
  for (int it = blockIdx.x; it < B.items; it += gridDim.x) {
    const int j = find_job(B, it);
    const int step = B.tick - B.c[j].t0;
    if (!fwd_consume<false>(B.c[j], B.p[j][step & 1], none, B.status, it - B.base[j],
                            __ldg(B.c[j].amp + step), smem, full, empty, k, warp, lane))
      break;
  }
}

// ------------------------------------------------------------ backward
struct BwdCommon {
  Dims3 d;
  Sched sc;
  float* g11;
  float* g13;
  float* g33;
  const float* dampx;
  const float* dampy;
  const float* dampz;
  float dt2, idx2, idy2, idz2;
  float sx, sy, sz;
  PointSource src;
  const float* amp;
  int t0;
  const float* c11;  // the model, read per point with read-only loads
  const float* c13;
  const float* c33;
};
struct BwdPar {
  const float* scz;  // cur sigma_z, lambda_z (queue initialisation)
  const float* lcz;
  float* spx;        // prev in / next out
  float* spz;
  float* lpx;
  float* lpz;
};
struct BwdArgs {
  BwdCommon c;
  BwdPar p;
  int* status;
};

constexpr int B_STAGES = 5;
// stage: [sigma_x halo][lambda_x halo][sz+4][lz+4][spx][spz][lpx][lpz]
// The model and gradient tiles are not staged: each consumer thread reads
// its own c11/c13/c33 and g11/g13/g33 pairs with plain loads issued before
// it waits for the plane's stage (it alone writes those gradient cells),
// which keeps a stage at 20 KB so that five stages of two CTAs fit one SM
// (four stages in flight per CTA).
constexpr int B_OFF_SH = 0;
constexpr int B_OFF_LH = HALO_BYTES;
constexpr int B_OFF_P = 2 * HALO_BYTES;  // 6 plain tiles from here
constexpr int B_STAGE_BYTES = B_OFF_P + 6 * PLAIN_BYTES;  // 19968
constexpr int B_SMEM = B_STAGES * B_STAGE_BYTES + 1024 + 2 * B_STAGES * 8;
static_assert(2 * B_SMEM <= 228 * 1024, "two backward CTAs per SM");

struct BwdMaps {
  CUtensorMap scx, scz, spx, spz, lcx, lcz, lpx, lpz;
};

// wave3d.h:5-6 recording / imaging weights, as float
constexpr float kTwoThirdF = (float)kTwoThird, kOneThirdF = (float)kOneThird;

template <bool kRtm>
__device__ __forceinline__ bool bwd_produce(const BwdCommon& a, const BwdMaps& m, int* status,
                                            int li, unsigned char* smem, uint64_t* full,
                                            uint64_t* empty, long long& k) {
  int bx, by, z0, z1;
  item(a.sc, li, bx, by, z0, z1);
  const int x0 = bx * TX, y0 = kHalo + by * TY;
  for (int z = z0; z < z1; ++z, ++k) {
    const int s = (int)(k % B_STAGES);
    if (k >= B_STAGES && !mbar_wait(&empty[s], (uint32_t)(((k / B_STAGES) & 1) ^ 1), status))
      return false;
    const int zp = z + kZPad;
    unsigned char* st = smem + s * B_STAGE_BYTES;
    unsigned char* pl = st + B_OFF_P;
    mbar_arrive_expect_tx(&full[s], B_STAGE_BYTES);
    tma_load(st + B_OFF_SH, &m.scx, &full[s], x0 - kHalo, y0 - kHalo, zp);
    tma_load(st + B_OFF_LH, &m.lcx, &full[s], x0 - kHalo, y0 - kHalo, zp);
    tma_load(pl + 0 * PLAIN_BYTES, &m.scz, &full[s], x0, y0, zp + kHalo);
    tma_load(pl + 1 * PLAIN_BYTES, &m.lcz, &full[s], x0, y0, zp + kHalo);
    tma_load(pl + 2 * PLAIN_BYTES, &m.spx, &full[s], x0, y0, zp);
    tma_load(pl + 3 * PLAIN_BYTES, &m.spz, &full[s], x0, y0, zp);
    tma_load(pl + 4 * PLAIN_BYTES, &m.lpx, &full[s], x0, y0, zp);
    tma_load(pl + 5 * PLAIN_BYTES, &m.lpz, &full[s], x0, y0, zp);
  }
  return true;
}

// Consumers: the x pair x0 + 2*(lane%16) + {0,1} of tile row 2*warp + lane/16.
template <bool kRtm>
__device__ __forceinline__ bool bwd_consume(const BwdCommon& a, const BwdPar& bp, int* status,
                                            int li, float amp, const unsigned char* smem,
                                            uint64_t* full, uint64_t* empty, long long& k,
                                            int warp, int lane) {
  const int ry = warp * 2 + (lane >> 4);
  const int xo = 2 * (lane & 15);
  const int sr = (ry + kHalo) * HX + xo + kHalo;
  const int pi = ry * TX + xo;
  float2 sq[9], lq[9];  // z queues of the pair (source, adjoint): planes z-4 .. z+4
  float dxy[2];
  int bx, by, z0, z1;
  item(a.sc, li, bx, by, z0, z1);
  const int x = bx * TX + xo;
  const int y = kHalo + by * TY + ry;
  const bool vy = y < a.d.ny - kHalo;
  const bool v0 = vy && x >= kHalo && x < a.d.nx - kHalo;
  const bool v1 = vy && x + 1 >= kHalo && x + 1 < a.d.nx - kHalo;
  const int off = y * a.d.pitch + x;  // x + 1 < pitch: 32 * gx <= pitch
  dxy[0] = v0 ? a.dampx[x] * a.dampy[y] : 1.f;
  dxy[1] = v1 ? a.dampx[x + 1] * a.dampy[y] : 1.f;
  // start the queues: planes z0-4 .. z0+3 from global
  sq[0] = lq[0] = make_float2(0.f, 0.f);
#pragma unroll
  for (int kk = 1; kk < 9; ++kk) {
    const int zz = z0 - 5 + kk;
    const long long i = (long long)zz * a.d.plane + off;
    const bool any = v0 || v1;
    const float2 sv =
        any ? __ldg(reinterpret_cast<const float2*>(bp.scz + i)) : make_float2(0.f, 0.f);
    float2 lv = any ? __ldg(reinterpret_cast<const float2*>(bp.lcz + i)) : make_float2(0.f, 0.f);
    if (zz >= 0 && (zz >> 2) < (z0 >> 2)) {
      lv.x *= dxy[0] * a.dampz[zz];
      lv.y *= dxy[1] * a.dampz[zz];
    }
    sq[kk] = sv;
    lq[kk] = lv;
  }
  // z damping factors in registers (see the forward kernel)
  float dzr[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) dzr[j] = z0 - 4 + j >= 0 ? a.dampz[z0 - 4 + j] : 1.f;
  float dz_next = a.dampz[z0];
  // this thread's gradient pair of a plane (read with plain loads)
  const bool anyv = v0 || v1;
  auto gload = [&](int zz, float2& r11, float2& r13, float2& r33) {
    const long long i = (long long)zz * a.d.plane + off;
    const float2 zero = make_float2(0.f, 0.f);
    r11 = anyv ? __ldg(reinterpret_cast<const float2*>(a.g11 + i)) : zero;
    r13 = (anyv && !kRtm) ? __ldg(reinterpret_cast<const float2*>(a.g13 + i)) : zero;
    r33 = (anyv && !kRtm) ? __ldg(reinterpret_cast<const float2*>(a.g33 + i)) : zero;
  };
  for (int z = z0; z < z1; ++z, ++k) {
    const float dz = dz_next;
    if (z + 1 < z1) dz_next = a.dampz[z + 1];
    // issued before the stage wait: the loads complete while the stage
    // arrives and the stencils are evaluated
    float2 g11o, g13o, g33o, c11, c13, c33;
    gload(z, g11o, g13o, g33o);
    model_pair(a.c11, a.c13, a.c33, (long long)z * a.d.plane + off, anyv, c11, c13, c33);
#pragma unroll
    for (int j = 0; j < 3; ++j) dzr[j] = dzr[j + 1];
    dzr[3] = dz;
    const int s = (int)(k % B_STAGES);
    if (!mbar_wait(&full[s], (uint32_t)((k / B_STAGES) & 1), status)) return false;
    const unsigned char* st = smem + s * B_STAGE_BYTES;
    const float* sh = (const float*)(st + B_OFF_SH) + sr;
    const float* lh = (const float*)(st + B_OFF_LH) + sr;
    const float* pl = (const float*)(st + B_OFF_P) + pi;
    constexpr int T = TX * TY;
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      sq[kk] = sq[kk + 1];
      lq[kk] = lq[kk + 1];
    }
    sq[8] = ld2(pl);
    lq[8] = ld2(pl + T);
    // x rows (x-4 .. x+5) and y column pairs of both halo fields
    float rs[10], rl[10];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const float2 t = ld2(sh - 4 + 2 * j), u = ld2(lh - 4 + 2 * j);
      rs[2 * j] = t.x;
      rs[2 * j + 1] = t.y;
      rl[2 * j] = u.x;
      rl[2 * j + 1] = u.y;
    }
    float2 sym[4], syp[4], lym[4], lyp[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      sym[j] = ld2(sh - (j + 1) * HX);
      syp[j] = ld2(sh + (j + 1) * HX);
      lym[j] = ld2(lh - (j + 1) * HX);
      lyp[j] = ld2(lh + (j + 1) * HX);
    }
    const float2 spx = ld2(pl + 2 * T), spz = ld2(pl + 3 * T);
    const float2 lpx = ld2(pl + 4 * T), lpz = ld2(pl + 5 * T);
    stage_release(&empty[s], lane);
    // the y and z stencils, the updates and the imaging of both points as
    // packed FP32 pairs (each lane rounded as the scalar operation); the x
    // stencils per point, their neighbour pairs straddling the loaded float2s
    const float2 two = splat(2.f);
    // source wavefield back one level (gradient form)
    // every stencil first (the y columns and x rows die as they are used)
    const float2 sc = make_float2(rs[4], rs[5]);
    const float2 lc = make_float2(rl[4], rl[5]);
    const float2 syy = lap9_2(sc, sym[0], syp[0], sym[1], syp[1], sym[2], syp[2], sym[3], syp[3]);
    const float2 lyy = lap9_2(lc, lym[0], lyp[0], lym[1], lyp[1], lym[2], lyp[2], lym[3], lyp[3]);
    float2 sxx, lxx;
    sxx.x = lap9(rs[4], rs[3], rs[5], rs[2], rs[6], rs[1], rs[7], rs[0], rs[8]);
    sxx.y = lap9(rs[5], rs[4], rs[6], rs[3], rs[7], rs[2], rs[8], rs[1], rs[9]);
    lxx.x = lap9(rl[4], rl[3], rl[5], rl[2], rl[6], rl[1], rl[7], rl[0], rl[8]);
    lxx.y = lap9(rl[5], rl[4], rl[6], rl[3], rl[7], rl[2], rl[8], rl[1], rl[9]);
    const float2 szz = lap9_2(sq[4], sq[3], sq[5], sq[2], sq[6], sq[1], sq[7], sq[0], sq[8]);
    const float2 lzz = lap9_2(lq[4], lq[3], lq[5], lq[2], lq[6], lq[1], lq[7], lq[0], lq[8]);
    const float2 sxy_u = fma2(syy, splat(a.idy2), mul2(sxx, splat(a.idx2)));
    const float2 sz_u = mul2(szz, splat(a.idz2));
    const long long i = (long long)z * a.d.plane + off;
    // each result pair is stored as soon as it is complete (shorter live
    // ranges: the whole step fits the 96 registers of two CTAs per SM)
    auto store2 = [&](float* f, float2 v) {
      if (v0 && v1) {
        *reinterpret_cast<float2*>(f + i) = v;
      } else {
        if (v0) f[i] = v.x;
        if (v1) f[i + 1] = v.y;
      }
    };
    const float2 dt2 = splat(a.dt2);
    float2 snx = fma2(dt2, fma2(c11, sxy_u, mul2(c13, sz_u)), sub2(mul2(two, sc), spx));
    float2 snz = fma2(dt2, fma2(c13, sxy_u, mul2(c33, sz_u)), sub2(mul2(two, sq[4]), spz));
    if (y == a.src.y && z == a.src.z) {
      if (x == a.src.x) {
        snx.x += amp;
        snz.x += amp;
      }
      if (x + 1 == a.src.x) {
        snx.y += amp;
        snz.y += amp;
      }
    }
    store2(bp.spx, snx);
    store2(bp.spz, snz);
    // imaging with the current adjoint
    const float2 lz0 = lq[4];
    const float2 dd = mul2(make_float2(dxy[0], dxy[1]), splat(dz));
    if (kRtm) {
      store2(a.g11, fma2(fma2(splat(kTwoThirdF), sc, mul2(splat(kOneThirdF), sq[4])),
                         mul2(dd, fma2(splat(kTwoThirdF), lc, mul2(splat(kOneThirdF), lz0))),
                         g11o));
    } else {
      store2(a.g11, fma2(lc, sxy_u, g11o));
      store2(a.g33, fma2(lz0, sz_u, g33o));
      store2(a.g13, fma2(lz0, sxy_u, fma2(lc, sz_u, g13o)));
    }
    // adjoint, forward form with the sponge
    const float2 lxy = fma2(lyy, splat(a.sy), mul2(lxx, splat(a.sx)));
    const float2 lzs = mul2(lzz, splat(a.sz));
    const float2 ndd = mul2(dd, splat(-1.f));
    // 2 cur - dd prev, rounded once
    store2(bp.lpx, mul2(dd, fma2(c11, lxy, fma2(c13, lzs, fma2(ndd, lpx, mul2(two, lc))))));
    store2(bp.lpz, mul2(dd, fma2(c13, lxy, fma2(c33, lzs, fma2(ndd, lpz, mul2(two, lz0))))));
    if (((z + 1) & 3) == 0 && z + 1 < a.d.nz) {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        lq[kk + 1] = mul2(lq[kk + 1], make_float2(dxy[0] * dzr[kk], dxy[1] * dzr[kk]));
    }
  }
  return true;
}

// kRtm selects the imaging condition of rtmCij3d_f (kernel3d.cu:456-469,
// rtm3d_f.cu:607-610): one image volume, kept in the g11 slot, gains
// (2/3 sx + 1/3 sz)(2/3 lx + 1/3 lz) with both fields at the current level and
// the adjoint already multiplied by this step's sponge; g13/g33 are neither
// loaded nor written.
template <bool kRtm>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_bwd3d_tma(const __grid_constant__ BwdMaps m0, const __grid_constant__ BwdArgs a0) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<B_STAGES, B_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0)
      for (int it = blockIdx.x; it < a0.c.sc.items; it += gridDim.x)
        if (!bwd_produce<kRtm>(a0.c, m0, a0.status, it, smem, full, empty, k)) break;
    return;
  }
  for (int it = blockIdx.x; it < a0.c.sc.items; it += gridDim.x)
    if (!bwd_consume<kRtm>(a0.c, a0.p, a0.status, it, a0.c.src.amp, smem, full, empty, k, warp,
                           lane))
      break;
}

struct BwdBatch {
  const BwdMaps* maps;  // [2 * job + parity]
  int* status;
  int njobs, items, tick;
  int base[kMaxBwdJobs + 1];
  BwdCommon c[kMaxBwdJobs];
  BwdPar p[kMaxBwdJobs][2];
};

__global__ void __launch_bounds__(NTHREADS, 2) k_bwd3d_batch(const __grid_constant__ BwdBatch B) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<B_STAGES, B_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0)
      for (int it = blockIdx.x; it < B.items; it += gridDim.x) {
        const int j = find_job(B, it);
        const int par = (B.tick - B.c[j].t0) & 1;
        if (!bwd_produce<false>(B.c[j], B.maps[2 * j + par], B.status, it - B.base[j], smem,
                                full, empty, k))
          break;
      }
    return;
  }
  for (int it = blockIdx.x; it < B.items; it += gridDim.x) {
    const int j = find_job(B, it);
    const int step = B.tick - B.c[j].t0;
    if (!bwd_consume<false>(B.c[j], B.p[j][step & 1], B.status, it - B.base[j],
                            __ldg(B.c[j].amp + step), smem, full, empty, k, warp, lane))
      break;
  }
}

static_assert(sizeof(FwdBatch) <= 32000 && sizeof(BwdBatch) <= 32000, "kernel parameter size");

// vti_ctx_check_bounded_wait: thread 0 waits on an mbarrier (expected count
// 1) that no thread arrives at and no copy completes, with a poll limit; the
// wait gives up and sets the status word. Nothing is in flight, so the CTA
// simply returns.
__global__ void k_wait_selftest(int* status, unsigned polls) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait(&bar, 0, status, polls);
}

}  // namespace

// ------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// Segment length: the smallest modelled time, counted in plane-steps of one
// CTA, waves * (seg + restart), where a wave is one item per resident slot
// and a restart (8 queue planes read with plain loads, pipeline refill) costs
// about kRestart plane-steps.
constexpr long long kRestart = 4;

Sched make_sched(vti_ctx* ctx, const Dims3& d, int ctas_per_sm) {
  Sched s;
  s.gx = (d.nx - kHalo + TX - 1) / TX;  // x origins 0, 32, ...; updated x < nx-4
  s.gy = (d.ny - 2 * kHalo + TY - 1) / TY;
  s.nz = d.nz;
  const long long cols = (long long)s.gx * s.gy;
  const long long slots = (long long)ctx->sm_count * ctas_per_sm;
  long long best = -1;
  for (int nseg = 1; nseg <= d.nz; ++nseg) {
    const int seg = (d.nz + nseg - 1) / nseg;
    if (nseg > 1 && seg < 8) break;  // at least 8 planes per queue start
    if (nseg > 1 && seg == (d.nz + nseg - 2) / (nseg - 1)) continue;  // same seg
    const long long items = cols * ((d.nz + seg - 1) / seg);
    if (items > (1LL << 30)) break;
    const long long waves = (items + slots - 1) / slots;
    const long long cost = waves * (seg + kRestart);
    if (best < 0 || cost < best) {
      best = cost;
      s.seg = seg;
      s.items = (int)items;
    }
  }
  s.grid = (int)std::min<long long>(s.items, slots);
  return s;
}

long long step_sched_cost(vti_ctx* ctx, const Dims3& d, int ctas_per_sm, long long* work) {
  const Sched s = make_sched(ctx, d, ctas_per_sm);
  const long long slots = (long long)ctx->sm_count * ctas_per_sm;
  const long long waves = (s.items + slots - 1) / slots;
  if (work) *work = (long long)s.gx * s.gy * s.nz;
  return waves * (s.seg + kRestart) * slots;
}

int make_tile_maps(vti_ctx* ctx, const Dims3& d, const Vol& v, TileMaps* out) {
  const int st = make_tile_maps_typed(ctx, d, v.alloc, 4, out);
  out->origin = v.origin;
  return st;
}

int make_tile_maps_typed(vti_ctx* ctx, const Dims3& d, void* alloc, int elem_bytes,
                         TileMaps* out) {
  auto fn = encode_fn();
  if (!fn) return fail(ctx, VTI_ERR_DEVICE, "cuTensorMapEncodeTiled unavailable");
  if (elem_bytes != 4 && elem_bytes != 2) return fail(ctx, VTI_ERR_ARG, "element size");
  const CUtensorMapDataType ty =
      elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  cuuint64_t dims[3] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)(d.nz + 2 * kZPad)};
  cuuint64_t strides[2] = {(cuuint64_t)d.pitch * elem_bytes, (cuuint64_t)d.plane * elem_bytes};
  cuuint32_t estr[3] = {1, 1, 1};
  cuuint32_t box_plain[3] = {TX, TY, 1};
  // TMA x coordinates must be multiples of 16 bytes: a BF16 halo tile starts
  // 8 cells (16 bytes) left of the column and is 16 cells wider (HXB)
  cuuint32_t box_halo[3] = {elem_bytes == 4 ? (cuuint32_t)HX : (cuuint32_t)HXB, HY, 1};
  CUresult r1 = fn((CUtensorMap*)out->plain, ty, 3, alloc, dims,
                   strides, box_plain, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = fn((CUtensorMap*)out->halo, ty, 3, alloc, dims,
                   strides, box_halo, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS)
    return fail(ctx, VTI_ERR_DEVICE, "cuTensorMapEncodeTiled failed");
  return VTI_OK;
}

static const CUtensorMap* P(const TileMaps& m) { return (const CUtensorMap*)m.plain; }
static const CUtensorMap* H(const TileMaps& m) { return (const CUtensorMap*)m.halo; }

namespace {

// Segment schedule with a fixed segment length (batched jobs, autotuned).
Sched sched_with_seg(const Dims3& d, int seg) {
  Sched s;
  s.gx = (d.nx - kHalo + TX - 1) / TX;
  s.gy = (d.ny - 2 * kHalo + TY - 1) / TY;
  s.nz = d.nz;
  s.seg = std::max(1, std::min(seg, d.nz));
  s.items = s.gx * s.gy * ((d.nz + s.seg - 1) / s.seg);
  s.grid = s.items;
  return s;
}

// Once per device and kernel; the flags are atomic because first calls may
// come from several host threads (setting the attribute twice is harmless).
template <typename K>
int set_smem_attr(vti_ctx* ctx, K kern, int bytes, std::atomic<bool>* done) {
  if (ctx->device < 64 && done[ctx->device].load(std::memory_order_acquire)) return VTI_OK;
  VTI_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (ctx->device < 64) done[ctx->device].store(true, std::memory_order_release);
  return VTI_OK;
}

FwdCommon fwd_common(const Dims3& d, const Sched& sc, const Damping* damp, float sx, float sy,
                     float sz, PointSource src, const TileMaps& c11, const TileMaps& c13,
                     const TileMaps& c33) {
  FwdCommon c{};
  c.c11 = c11.origin;
  c.c13 = c13.origin;
  c.c33 = c33.origin;
  c.d = d;
  c.sc = sc;
  c.dampx = damp ? damp->x : nullptr;
  c.dampy = damp ? damp->y : nullptr;
  c.dampz = damp ? damp->z : nullptr;
  c.sx = sx;
  c.sy = sy;
  c.sz = sz;
  c.src = src;
  return c;
}

std::atomic<bool> attr_fwd[3][64], attr_bwd[2][64], attr_fwd_batch[64], attr_bwd_batch[64];

}  // namespace

int launch_fwd3d_tma(vti_ctx* ctx, const Dims3& d, const TileMaps& cx, const TileMaps& cz,
                     const TileMaps& px, const TileMaps& pz, const TileMaps& c11,
                     const TileMaps& c13, const TileMaps& c33, const float* cz_ptr,
                     float* px_ptr, float* pz_ptr, const Damping* damp, float sx, float sy,
                     float sz, PointSource src, Probe probe, bool exact) {
  const bool pr = probe.x >= 0 && probe.out;
  if (pr && exact) return fail(ctx, VTI_ERR_UNSUPPORTED, "probe with the exact-mode step");
  auto kern = pr ? k_fwd3d_tma<true, false>
                 : (exact ? k_fwd3d_tma<false, true> : k_fwd3d_tma<false, false>);
  const int variant = pr ? 1 : (exact ? 2 : 0);
  VTI_TRY_ST(set_smem_attr(ctx, kern, F_SMEM, attr_fwd[variant]));
  FwdMaps m;
  m.cx = *H(cx); m.cz = *P(cz); m.px = *P(px); m.pz = *P(pz);
  FwdArgs a{};
  a.c = fwd_common(d, make_sched(ctx, d, 3), damp, sx, sy, sz, src, c11, c13, c33);
  a.p = FwdPar{cz_ptr, px_ptr, pz_ptr};
  a.probe = probe;
  a.status = ctx->d_status;
  const int grid = a.c.sc.grid;
  {
    LaunchTimer tm(ctx, kTimedFwd3d);
    kern<<<grid, NTHREADS, F_SMEM, ctx->stream>>>(m, a);
  }
  VTI_LAUNCHED(ctx, "k_fwd3d_tma");
  return VTI_OK;
}

int launch_bwd3d_tma(vti_ctx* ctx, const Dims3& d, const TileMaps& scx, const TileMaps& scz,
                     const TileMaps& spx, const TileMaps& spz, const TileMaps& lcx,
                     const TileMaps& lcz, const TileMaps& lpx, const TileMaps& lpz,
                     const TileMaps& c11, const TileMaps& c13, const TileMaps& c33,
                     const TileMaps& g11, const TileMaps& g13, const TileMaps& g33,
                     const float* scz_ptr, const float* lcz_ptr, float* spx_ptr, float* spz_ptr,
                     float* lpx_ptr, float* lpz_ptr, float* g11_ptr, float* g13_ptr,
                     float* g33_ptr, const Damping& damp, float dt2, float idx2, float idy2,
                     float idz2, float sx, float sy, float sz, PointSource src, bool rtm) {
  VTI_TRY_ST(set_smem_attr(ctx, rtm ? k_bwd3d_tma<true> : k_bwd3d_tma<false>, B_SMEM,
                           attr_bwd[rtm]));
  BwdMaps m;
  m.scx = *H(scx); m.scz = *P(scz); m.spx = *P(spx); m.spz = *P(spz);
  m.lcx = *H(lcx); m.lcz = *P(lcz); m.lpx = *P(lpx); m.lpz = *P(lpz);
  BwdArgs a{};
  BwdCommon& c = a.c;
  c.d = d;
  c.sc = make_sched(ctx, d, 2);
  c.g11 = g11_ptr; c.g13 = g13_ptr; c.g33 = g33_ptr;
  c.c11 = c11.origin; c.c13 = c13.origin; c.c33 = c33.origin;
  c.dampx = damp.x; c.dampy = damp.y; c.dampz = damp.z;
  c.dt2 = dt2; c.idx2 = idx2; c.idy2 = idy2; c.idz2 = idz2;
  c.sx = sx; c.sy = sy; c.sz = sz;
  c.src = src;
  a.p = BwdPar{scz_ptr, lcz_ptr, spx_ptr, spz_ptr, lpx_ptr, lpz_ptr};
  a.status = ctx->d_status;
  const int grid = c.sc.grid;
  {
    LaunchTimer tm(ctx, kTimedBwd3d);
    if (rtm)
      k_bwd3d_tma<true><<<grid, NTHREADS, B_SMEM, ctx->stream>>>(m, a);
    else
      k_bwd3d_tma<false><<<grid, NTHREADS, B_SMEM, ctx->stream>>>(m, a);
  }
  VTI_LAUNCHED(ctx, "k_bwd3d_tma");
  return VTI_OK;
}

// ------------------------------------------------------------ batched steps
// A batched step: its jobs in chunks of at most kMax*Jobs, one launch each.
struct StepBatch {
  bool fwd = true;
  std::vector<FwdBatch> fb;  // host parameter blocks, one per chunk
  std::vector<BwdBatch> bb;
  std::vector<void*> d_maps;  // device TMA descriptors of each chunk
  int items = 0;
};

int prepare_batch_kernels(vti_ctx* ctx) {
  VTI_TRY_ST(set_smem_attr(ctx, k_fwd3d_batch, F_SMEM, attr_fwd_batch));
  VTI_TRY_ST(set_smem_attr(ctx, k_bwd3d_batch, B_SMEM, attr_bwd_batch));
  return VTI_OK;
}

void step_batch_free(StepBatch* b) {
  if (!b) return;
  for (void* p : b->d_maps)
    if (p) cudaFree(p);
  delete b;
}

int fwd_batch_build(vti_ctx* ctx, const FwdJobSpec* spec, int njobs, StepBatch** out) {
  *out = nullptr;
  VTI_TRY_ST(prepare_batch_kernels(ctx));
  StepBatch* b = new StepBatch();
  b->fwd = true;
  for (int j0 = 0; j0 < njobs; j0 += kMaxFwdJobs) {
    const int nj = std::min(kMaxFwdJobs, njobs - j0);
    b->fb.emplace_back();
    FwdBatch& B = b->fb.back();
    std::memset(&B, 0, sizeof(B));
    std::vector<FwdMaps> maps(2 * nj);
    int items = 0;
    for (int j = 0; j < nj; ++j) {
      const FwdJobSpec& sp = spec[j0 + j];
      const Sched sc = sp.seg > 0 ? sched_with_seg(sp.d, sp.seg) : make_sched(ctx, sp.d, 3);
      PointSource src;
      src.x = sp.src_x; src.y = sp.src_y; src.z = sp.src_z;
      B.c[j] = fwd_common(sp.d, sc, sp.damp, sp.sx, sp.sy, sp.sz, src, *sp.c[0], *sp.c[1],
                          *sp.c[2]);
      B.c[j].amp = sp.amp;
      B.c[j].t0 = sp.t0;
      for (int par = 0; par < 2; ++par) {
        B.p[j][par] = FwdPar{sp.cz_ptr[par], sp.px_ptr[par], sp.pz_ptr[par]};
        FwdMaps& m = maps[2 * j + par];
        m.cx = *H(*sp.cx[par]); m.cz = *P(*sp.cz[par]); m.px = *P(*sp.px[par]);
        m.pz = *P(*sp.pz[par]);
      }
      B.base[j] = items;
      items += sc.items;
    }
    B.base[nj] = items;
    B.njobs = nj;
    B.items = items;
    B.status = ctx->d_status;
    b->items += items;
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, maps.size() * sizeof(FwdMaps));
    if (e == cudaSuccess)
      e = cudaMemcpy(d, maps.data(), maps.size() * sizeof(FwdMaps), cudaMemcpyHostToDevice);
    b->d_maps.push_back(d);
    if (e != cudaSuccess) {
      step_batch_free(b);
      return cuda_check(ctx, e, "batched forward descriptors");
    }
    B.maps = (const FwdMaps*)d;
  }
  *out = b;
  return VTI_OK;
}

int bwd_batch_build(vti_ctx* ctx, const BwdJobSpec* spec, int njobs, StepBatch** out) {
  *out = nullptr;
  VTI_TRY_ST(prepare_batch_kernels(ctx));
  StepBatch* b = new StepBatch();
  b->fwd = false;
  for (int j0 = 0; j0 < njobs; j0 += kMaxBwdJobs) {
    const int nj = std::min(kMaxBwdJobs, njobs - j0);
    b->bb.emplace_back();
    BwdBatch& B = b->bb.back();
    std::memset(&B, 0, sizeof(B));
    std::vector<BwdMaps> maps(2 * nj);
    int items = 0;
    for (int j = 0; j < nj; ++j) {
      const BwdJobSpec& sp = spec[j0 + j];
      const Sched sc = sp.seg > 0 ? sched_with_seg(sp.d, sp.seg) : make_sched(ctx, sp.d, 2);
      BwdCommon& c = B.c[j];
      c.d = sp.d;
      c.sc = sc;
      c.g11 = sp.g_ptr[0]; c.g13 = sp.g_ptr[1]; c.g33 = sp.g_ptr[2];
      c.c11 = sp.c[0]->origin; c.c13 = sp.c[1]->origin; c.c33 = sp.c[2]->origin;
      c.dampx = sp.damp.x; c.dampy = sp.damp.y; c.dampz = sp.damp.z;
      c.dt2 = sp.dt2; c.idx2 = sp.idx2; c.idy2 = sp.idy2; c.idz2 = sp.idz2;
      c.sx = sp.sx; c.sy = sp.sy; c.sz = sp.sz;
      c.src.x = sp.src_x; c.src.y = sp.src_y; c.src.z = sp.src_z; c.src.amp = 0.f;
      c.amp = sp.amp;
      c.t0 = sp.t0;
      for (int par = 0; par < 2; ++par) {
        B.p[j][par] = BwdPar{sp.scz_ptr[par], sp.lcz_ptr[par], sp.spx_ptr[par], sp.spz_ptr[par],
                             sp.lpx_ptr[par], sp.lpz_ptr[par]};
        BwdMaps& m = maps[2 * j + par];
        m.scx = *H(*sp.scx[par]); m.scz = *P(*sp.scz[par]); m.spx = *P(*sp.spx[par]);
        m.spz = *P(*sp.spz[par]);
        m.lcx = *H(*sp.lcx[par]); m.lcz = *P(*sp.lcz[par]); m.lpx = *P(*sp.lpx[par]);
        m.lpz = *P(*sp.lpz[par]);
      }
      B.base[j] = items;
      items += sc.items;
    }
    B.base[nj] = items;
    B.njobs = nj;
    B.items = items;
    B.status = ctx->d_status;
    b->items += items;
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, maps.size() * sizeof(BwdMaps));
    if (e == cudaSuccess)
      e = cudaMemcpy(d, maps.data(), maps.size() * sizeof(BwdMaps), cudaMemcpyHostToDevice);
    b->d_maps.push_back(d);
    if (e != cudaSuccess) {
      step_batch_free(b);
      return cuda_check(ctx, e, "batched backward descriptors");
    }
    B.maps = (const BwdMaps*)d;
  }
  *out = b;
  return VTI_OK;
}

int step_batch_launch(vti_ctx* ctx, StepBatch* b, int tick) {
  if (b->fwd) {
    for (FwdBatch& B : b->fb) {
      if (B.items <= 0) continue;
      B.tick = tick;
      const int grid = std::min(B.items, ctx->sm_count * 3);
      {
        LaunchTimer tm(ctx, kTimedFwd3d);
        k_fwd3d_batch<<<grid, NTHREADS, F_SMEM, ctx->stream>>>(B);
      }
      VTI_LAUNCHED(ctx, "k_fwd3d_batch");
    }
  } else {
    for (BwdBatch& B : b->bb) {
      if (B.items <= 0) continue;
      B.tick = tick;
      const int grid = std::min(B.items, ctx->sm_count * 2);
      {
        LaunchTimer tm(ctx, kTimedBwd3d);
        k_bwd3d_batch<<<grid, NTHREADS, B_SMEM, ctx->stream>>>(B);
      }
      VTI_LAUNCHED(ctx, "k_bwd3d_batch");
    }
  }
  return VTI_OK;
}

int wait_selftest(vti_ctx* ctx, unsigned polls) {
  if (polls < 1 || polls > 65536) return fail(ctx, VTI_ERR_ARG, "polls must be in [1, 65536]");
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  k_wait_selftest<<<1, 32, 0, ctx->stream>>>(ctx->d_status, polls);
  VTI_LAUNCHED(ctx, "k_wait_selftest");
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return check_device_status(ctx);
}

int step_batch_launches(const StepBatch* b) {
  return (int)(b->fwd ? b->fb.size() : b->bb.size());
}

}  // namespace vti
