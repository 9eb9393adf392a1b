// 3D Gauss-Newton Hessian-vector product and gradient in exact mode.
//
// The reference has no 3D Gauss-Newton product on the GPU (its CPU twin has
// the Born step bornCij and the transposed operator adjointCij,
// lib/vti-fwi-3d/cpu/laplacian3d.ispc:132-190). This file builds one from the
// exact-mode operators, whose discrete adjoint is exact (the checks are the
// dot-product and finite-difference tests of the oracle's EXACT mode):
//   a_0 = 0, a_1 = dt2 w[0] e_s,
//   a_t = P [ D ((2 + C L) a_{t-1} + dt2 w[t-1] e_s) - (2D - 1) a_{t-2} ],  t = 2..M
//   da_t = P [ D ((2 + C L) da_{t-1} + dC L a_{t-1}) - (2D - 1) da_{t-2} ]  (Born)
//   (centred damping, energy-stable for D <= 1)
//   traces d_j = 2/3 a_x + 1/3 a_z at the receivers' cells, level j*st;
//   mu_t = P [ D (R^T r_t + 2 mu_{t+1} + (C L)^T mu_{t+1}) - (2D - 1) mu_{t+2} ],
//   (C L)^T mu = (L_xy w_x, L_z w_z), w = C mu,
//   image += (mu_x L_xy a_{t-1}, mu_x L_z a_{t-1} + mu_z L_xy a_{t-1}, mu_z L_z a_{t-1}).
// With r = d - d_obs the image is the gradient of J = 1/2 |d - d_obs|^2; with
// r = the Born traces of dc it is H dc, H = J^T J the Gauss-Newton Hessian.
//
// Passes. Forward: one fused kernel advances the background and the Born
// field (reading C and dC once; 72 B per point), the traces of both are
// recorded, and the background pair (a_{k-1}, a_k) is kept at every K-th
// level (checkpoints). Backward: level blocks from the last to the first;
// each block recomputes its background levels from its checkpoint with the
// exact forward step into a segment buffer, then the adjoint step (w = C mu
// carried as its own field, so the transposed operator is a plain stencil
// of w) images against a_{t-1} from the segment. Both adjoints (gradient and
// H dc) share the recomputation. The images are summed blockwise: FP32 within
// a checkpoint block, Kahan-compensated FP32 across blocks (one compensated
// read-modify-write per point per block instead of a compensation term per
// step).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "vti_plan3d.h"
#include "vti_tma_common.cuh"

namespace vti {
namespace {

// ------------------------------------------------------------ Born step
struct BornArgs {
  Dims3 d;
  Sched sc;
  const float* az;  // cur background sigma_z (queue start)
  const float* bz;  // cur Born sigma_z
  float* apx;       // prev in / next out
  float* apz;
  float* bpx;
  float* bpz;
  const float* dampx;
  const float* dampy;
  const float* dampz;
  float sx, sy, sz;
  PointSource src;
  int* status;
};
struct BornMaps {
  CUtensorMap ax, bx, az, bz, apx, apz, bpx, bpz, c11, c13, c33, d11, d13, d33;
};
// Born step stage: two halo tiles (x fields) and 12 plain tiles (the two z
// fields 4 planes below, the four previous-level tiles, the model and the
// perturbation), three stages. Reading the model and the perturbation with
// read-only loads instead (as the adjoint does) measured 4 % slower here:
// the kernel already spills at 96 registers and the six pairs held across
// the stage wait add to it.
constexpr int GB_STAGES = 3;
constexpr int G_OFF_P = 2 * HALO_BYTES;
constexpr int GB_STAGE_BYTES = G_OFF_P + 12 * PLAIN_BYTES;  // 32256
constexpr int GB_SMEM = GB_STAGES * GB_STAGE_BYTES + 1024 + 2 * GB_STAGES * 8;
static_assert(2 * GB_SMEM <= 228 * 1024, "two Born CTAs per SM");
// Adjoint step stage: two halo tiles and 6 plain tiles (the two z fields 4
// planes below, the four previous-level tiles). The model and the images are
// not staged: each consumer thread reads its own float2 pairs with read-only
// loads issued before it waits for the plane's stage, which keeps a stage at
// 20 KB and five stages of two CTAs on one SM (0.583 -> 0.514 ms per
// 400x400x200 launch).
constexpr int G_STAGES = 5;
constexpr int G_STAGE_BYTES = G_OFF_P + 6 * PLAIN_BYTES;  // 19968
constexpr int G_SMEM = G_STAGES * G_STAGE_BYTES + 1024 + 2 * G_STAGES * 8;
static_assert(2 * G_SMEM <= 228 * 1024, "two Gauss-Newton CTAs per SM");

// Three float2 pairs of one thread at plane offset i (zeros where neither
// point is updated).
__device__ __forceinline__ void ldg3(const float* p0, const float* p1, const float* p2,
                                     long long i, bool any, float2& r0, float2& r1, float2& r2) {
  const float2 zero = make_float2(0.f, 0.f);
  r0 = any ? __ldg(reinterpret_cast<const float2*>(p0 + i)) : zero;
  r1 = any ? __ldg(reinterpret_cast<const float2*>(p1 + i)) : zero;
  r2 = any ? __ldg(reinterpret_cast<const float2*>(p2 + i)) : zero;
}

// Loads of one item: two halo tiles (x fields) and kNumPlain plain tiles per
// plane, into a ring of kStages stages of kStageBytes.
template <typename Maps, int kNumPlain, int kStages, int kStageBytes>
__device__ __forceinline__ bool produce14(const Sched& sc, const Maps& m, int* status, int li,
                                          unsigned char* smem, uint64_t* full, uint64_t* empty,
                                          long long& k) {
  static_assert(sizeof(Maps) == (2 + kNumPlain) * sizeof(CUtensorMap), "map layout");
  static_assert(2 * HALO_BYTES + kNumPlain * PLAIN_BYTES <= kStageBytes, "stage size");
  const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(&m);
  int bx, by, z0, z1;
  item(sc, li, bx, by, z0, z1);
  const int x0 = bx * TX, y0 = kHalo + by * TY;
  for (int z = z0; z < z1; ++z, ++k) {
    const int s = (int)(k % kStages);
    if (k >= kStages && !mbar_wait(&empty[s], (uint32_t)(((k / kStages) & 1) ^ 1), status))
      return false;
    const int zp = z + kZPad;
    unsigned char* st = smem + s * kStageBytes;
    mbar_arrive_expect_tx(&full[s], 2 * HALO_BYTES + kNumPlain * PLAIN_BYTES);
    tma_load(st, &maps[0], &full[s], x0 - kHalo, y0 - kHalo, zp);
    tma_load(st + HALO_BYTES, &maps[1], &full[s], x0 - kHalo, y0 - kHalo, zp);
    // plain tiles 0, 1: the z fields 4 planes below (register queues)
    tma_load(st + G_OFF_P, &maps[2], &full[s], x0, y0, zp + kHalo);
    tma_load(st + G_OFF_P + PLAIN_BYTES, &maps[3], &full[s], x0, y0, zp + kHalo);
#pragma unroll
    for (int j = 2; j < kNumPlain; ++j)
      tma_load(st + G_OFF_P + j * PLAIN_BYTES, &maps[2 + j], &full[s], x0, y0, zp);
  }
  return true;
}

struct Stencil2 {  // the x-row, y-column and z-queue stencil of one x pair
  float r[10];
  float2 ym[4], yp[4];
  __device__ __forceinline__ void load(const float* h) {
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const float2 t = ld2(h - 4 + 2 * j);
      r[2 * j] = t.x;
      r[2 * j + 1] = t.y;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      ym[j] = ld2(h - (j + 1) * HX);
      yp[j] = ld2(h + (j + 1) * HX);
    }
  }
  // L_xy (forward-form scaled) of element e
  __device__ __forceinline__ float lxy(int e, float sx, float sy) const {
    auto pick = [e](float2 v) { return e ? v.y : v.x; };
    const float c = r[4 + e];
    const float lxx = lap9(c, r[3 + e], r[5 + e], r[2 + e], r[6 + e], r[1 + e], r[7 + e], r[e],
                           r[8 + e]);
    const float lyy = lap9(c, pick(ym[0]), pick(yp[0]), pick(ym[1]), pick(yp[1]), pick(ym[2]),
                           pick(yp[2]), pick(ym[3]), pick(yp[3]));
    return fmaf(lyy, sy, lxx * sx);
  }
};

__device__ __forceinline__ float lz_of(const float* q, float sz) {
  return lap9(q[4], q[3], q[5], q[2], q[6], q[1], q[7], q[0], q[8]) * sz;
}

// Queue start: planes z0-4 .. z0+3 of a z field from global memory.
__device__ __forceinline__ void queue_init(float (&q)[2][9], const float* f, const Dims3& d,
                                           int off, int z0, bool any) {
  q[0][0] = q[1][0] = 0.f;
#pragma unroll
  for (int kk = 1; kk < 9; ++kk) {
    const int zz = z0 - 5 + kk;
    const float2 v = any ? __ldg(reinterpret_cast<const float2*>(f + (long long)zz * d.plane + off))
                         : make_float2(0.f, 0.f);
    q[0][kk] = v.x;
    q[1][kk] = v.y;
  }
}

__device__ __forceinline__ void queue_push(float (&q)[2][9], float2 v) {
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    q[0][kk] = q[0][kk + 1];
    q[1][kk] = q[1][kk + 1];
  }
  q[0][8] = v.x;
  q[1][8] = v.y;
}

__global__ void __launch_bounds__(NTHREADS, 2)
    k_born3d_tma(const __grid_constant__ BornMaps m, const __grid_constant__ BornArgs a) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<GB_STAGES, GB_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0)
      for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x)
        if (!produce14<BornMaps, 12, GB_STAGES, GB_STAGE_BYTES>(a.sc, m, a.status, it, smem,
                                                               full, empty, k))
          break;
    return;
  }
  const int ry = warp * 2 + (lane >> 4);
  const int xo = 2 * (lane & 15);
  const int sr = (ry + kHalo) * HX + xo + kHalo;
  const int pi = ry * TX + xo;
  for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x) {
    int bx, by, z0, z1;
    item(a.sc, it, bx, by, z0, z1);
    const int x = bx * TX + xo;
    const int y = kHalo + by * TY + ry;
    const bool vy = y < a.d.ny - kHalo;
    const bool v0 = vy && x >= kHalo && x < a.d.nx - kHalo;
    const bool v1 = vy && x + 1 >= kHalo && x + 1 < a.d.nx - kHalo;
    const int off = y * a.d.pitch + x;
    float aq[2][9], bq[2][9], dxy[2];
    queue_init(aq, a.az, a.d, off, z0, v0 || v1);
    queue_init(bq, a.bz, a.d, off, z0, v0 || v1);
    dxy[0] = v0 ? a.dampx[x] * a.dampy[y] : 1.f;
    dxy[1] = v1 ? a.dampx[x + 1] * a.dampy[y] : 1.f;
    bool ok = true;
    for (int z = z0; z < z1; ++z, ++k) {
      const float dz = a.dampz[z];
      const int s = (int)(k % GB_STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((k / GB_STAGES) & 1), a.status)) {
        ok = false;
        break;
      }
      const unsigned char* st = smem + s * GB_STAGE_BYTES;
      const float* pl = (const float*)(st + G_OFF_P) + pi;
      constexpr int T = TX * TY;
      queue_push(aq, ld2(pl));
      queue_push(bq, ld2(pl + T));
      Stencil2 sa, sb;
      sa.load((const float*)st + sr);
      sb.load((const float*)(st + HALO_BYTES) + sr);
      const float2 apx = ld2(pl + 2 * T), apz = ld2(pl + 3 * T);
      const float2 bpx = ld2(pl + 4 * T), bpz = ld2(pl + 5 * T);
      const float2 c11 = ld2(pl + 6 * T), c13 = ld2(pl + 7 * T), c33 = ld2(pl + 8 * T);
      const float2 d11 = ld2(pl + 9 * T), d13 = ld2(pl + 10 * T), d33 = ld2(pl + 11 * T);
      stage_release(&empty[s], lane);
      float anx[2], anz[2], bnx[2], bnz[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        auto pick = [e](float2 v) { return e ? v.y : v.x; };
        const float dd = dxy[e] * dz;
        const float a11 = pick(c11), a13 = pick(c13), a33 = pick(c33);
        // background: the exact forward step (same expression as k_fwd3d_tma)
        const float lxy = sa.lxy(e, a.sx, a.sy);
        const float lz = lz_of(aq[e], a.sz);
        const float pc = 2.f * dd - 1.f;  // centred damping: - (2D - 1) prev
        anx[e] = fmaf(a11, lxy, fmaf(a13, lz, 2.f * sa.r[4 + e]));
        anz[e] = fmaf(a13, lxy, fmaf(a33, lz, 2.f * aq[e][4]));
        if (x + e == a.src.x && y == a.src.y && z == a.src.z) {
          anx[e] += a.src.amp;
          anz[e] += a.src.amp;
        }
        anx[e] = fmaf(dd, anx[e], -pc * pick(apx));
        anz[e] = fmaf(dd, anz[e], -pc * pick(apz));
        // Born field: same operator plus the scattering source dC L a_{t-1}
        const float blxy = sb.lxy(e, a.sx, a.sy);
        const float blz = lz_of(bq[e], a.sz);
        const float sx_ = fmaf(pick(d11), lxy, pick(d13) * lz);
        const float sz_ = fmaf(pick(d13), lxy, pick(d33) * lz);
        bnx[e] = fmaf(dd, fmaf(a11, blxy, fmaf(a13, blz, 2.f * sb.r[4 + e])) + sx_,
                      -pc * pick(bpx));
        bnz[e] = fmaf(dd, fmaf(a13, blxy, fmaf(a33, blz, 2.f * bq[e][4])) + sz_,
                      -pc * pick(bpz));
      }
      const long long i = (long long)z * a.d.plane + off;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (e ? v1 : v0) {
          a.apx[i + e] = anx[e];
          a.apz[i + e] = anz[e];
          a.bpx[i + e] = bnx[e];
          a.bpz[i + e] = bnz[e];
        }
      }
    }
    if (!ok) break;
  }
}

// ------------------------------------------------------------ exact adjoint
struct AdjArgs {
  Dims3 d;
  Sched sc;
  const float* wz;   // w_{t+1} z (queue start)
  const float* az;   // a_{t-1} z (queue start)
  float* mpx;        // mu_{t+2} in, mu_t out
  float* mpz;
  float* wox;        // w_t out
  float* woz;
  float* g11;
  float* g13;
  float* g33;
  const float* dampx;
  const float* dampy;
  const float* dampz;
  float sx, sy, sz;
  int* status;
  const float* c11;  // the model, read per point with read-only loads
  const float* c13;
  const float* c33;
};
struct AdjMaps {
  CUtensorMap wx, ax, wz, az, m1x, m1z, mpx, mpz;
};

__global__ void __launch_bounds__(NTHREADS, 2)
    k_adj3d_tma(const __grid_constant__ AdjMaps m, const __grid_constant__ AdjArgs a) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<G_STAGES, G_STAGE_BYTES>(smem_raw, full, empty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0)
      for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x)
        if (!produce14<AdjMaps, 6, G_STAGES, G_STAGE_BYTES>(a.sc, m, a.status, it, smem, full,
                                                            empty, k))
          break;
    return;
  }
  const int ry = warp * 2 + (lane >> 4);
  const int xo = 2 * (lane & 15);
  const int sr = (ry + kHalo) * HX + xo + kHalo;
  const int pi = ry * TX + xo;
  for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x) {
    int bx, by, z0, z1;
    item(a.sc, it, bx, by, z0, z1);
    const int x = bx * TX + xo;
    const int y = kHalo + by * TY + ry;
    const bool vy = y < a.d.ny - kHalo;
    const bool v0 = vy && x >= kHalo && x < a.d.nx - kHalo;
    const bool v1 = vy && x + 1 >= kHalo && x + 1 < a.d.nx - kHalo;
    const int off = y * a.d.pitch + x;
    float wq[2][9], aq[2][9], dxy[2];
    queue_init(wq, a.wz, a.d, off, z0, v0 || v1);
    queue_init(aq, a.az, a.d, off, z0, v0 || v1);
    dxy[0] = v0 ? a.dampx[x] * a.dampy[y] : 1.f;
    dxy[1] = v1 ? a.dampx[x + 1] * a.dampy[y] : 1.f;
    bool ok = true;
    const bool any = v0 || v1;
    for (int z = z0; z < z1; ++z, ++k) {
      const float dz = a.dampz[z];
      // issued before the stage wait; this thread alone writes its image cells
      float2 c11, c13, c33, g11o, g13o, g33o;
      const long long gi = (long long)z * a.d.plane + off;
      ldg3(a.c11, a.c13, a.c33, gi, any, c11, c13, c33);
      ldg3(a.g11, a.g13, a.g33, gi, any, g11o, g13o, g33o);
      const int s = (int)(k % G_STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((k / G_STAGES) & 1), a.status)) {
        ok = false;
        break;
      }
      const unsigned char* st = smem + s * G_STAGE_BYTES;
      const float* pl = (const float*)(st + G_OFF_P) + pi;
      constexpr int T = TX * TY;
      queue_push(wq, ld2(pl));
      queue_push(aq, ld2(pl + T));
      Stencil2 sw, sa;
      sw.load((const float*)st + sr);
      sa.load((const float*)(st + HALO_BYTES) + sr);
      const float2 m1x = ld2(pl + 2 * T), m1z = ld2(pl + 3 * T);
      const float2 m2x = ld2(pl + 4 * T), m2z = ld2(pl + 5 * T);
      stage_release(&empty[s], lane);
      float mx[2], mz[2], wx[2], wzv[2], g11[2], g13[2], g33[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        auto pick = [e](float2 v) { return e ? v.y : v.x; };
        const float dd = dxy[e] * dz;
        const float lxy = sw.lxy(e, a.sx, a.sy);   // L_xy w_x
        const float lz = lz_of(wq[e], a.sz);         // L_z w_z
        mx[e] = fmaf(dd, 2.f * pick(m1x) + lxy, -(2.f * dd - 1.f) * pick(m2x));
        mz[e] = fmaf(dd, 2.f * pick(m1z) + lz, -(2.f * dd - 1.f) * pick(m2z));
        wx[e] = fmaf(pick(c11), mx[e], pick(c13) * mz[e]);
        wzv[e] = fmaf(pick(c13), mx[e], pick(c33) * mz[e]);
        const float axy = sa.lxy(e, a.sx, a.sy);   // L_xy a_{t-1,x}
        const float az = lz_of(aq[e], a.sz);         // L_z a_{t-1,z}
        g11[e] = fmaf(mx[e], axy, pick(g11o));
        g13[e] = fmaf(mx[e], az, fmaf(mz[e], axy, pick(g13o)));
        g33[e] = fmaf(mz[e], az, pick(g33o));
      }
      const long long i = (long long)z * a.d.plane + off;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (e ? v1 : v0) {
          a.mpx[i + e] = mx[e];
          a.mpz[i + e] = mz[e];
          a.wox[i + e] = wx[e];
          a.woz[i + e] = wzv[e];
          a.g11[i + e] = g11[e];
          a.g13[i + e] = g13[e];
          a.g33[i + e] = g33[e];
        }
      }
    }
    if (!ok) break;
  }
}

// ------------------------------------------------ BF16 background storage
// The background levels the adjoint images against are stored as bfloat16
// with one FP32 scale per z plane (value = bf16 * scale[z + kZPad]; the
// scale is the plane's largest magnitude, pad planes hold 0).
//
// Rounding: nearest by default. Stochastic rounding (VTI_GNHV_BF16_SR;
// Connolly, Higham & Mary, "Stochastic rounding and its probabilistic
// backward error analysis", SIAM J. Sci. Comput. 43(1), 2021) rounds x up to
// the next BF16 value with probability (x - lower) / ulp, so each stored
// value is unbiased and the errors of different levels are independent. It
// pays when round-to-nearest errors add coherently over the imaging sum; on
// the reduced config-4 case they do not, and stochastic rounding's larger
// per-value variance (ulp^2/6 against ulp^2/12) gives about twice the image
// error, so nearest stays the default. Implemented on the bits: the
// FP32 pattern plus 16 random low bits, truncated to its upper 16 bits
// (carries into the exponent round the magnitude up across a binade, as
// they should). The random bits are a counter hash of (level, plane, cell),
// so a run is reproducible.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  // xorshift-multiply integer hash (constants of a published low-bias
  // 32-bit mixer)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float x, uint32_t r) {
  const uint32_t b = __float_as_uint(x) + (r & 0xffffu);
  __nv_bfloat16_raw raw;
  raw.x = (unsigned short)(b >> 16);
  return __nv_bfloat16(raw);
}

__global__ void k_pack_bf16(const float* src, Dims3 d, __nv_bfloat16* dst, float* scale,
                            uint32_t seed, int stochastic) {
  const int z = blockIdx.x;
  const float* s = src + (long long)z * d.plane;
  __nv_bfloat16* o = dst + (long long)z * d.plane;
  const int n = d.ny * d.pitch;
  float m = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (i % d.pitch < d.nx) m = fmaxf(m, fabsf(s[i]));
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  __shared__ float wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : 0.f;
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (threadIdx.x == 0) wm[0] = v;
  }
  __syncthreads();
  const float sc = wm[0] > 0.f ? wm[0] : 1.f;
  const float inv = 1.f / sc;
  if (threadIdx.x == 0) scale[z + kZPad] = sc;
  const uint32_t zs = mix32(seed ^ (0x9e3779b9u * (uint32_t)(z + 1)));
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = i % d.pitch < d.nx ? s[i] * inv : 0.f;
    o[i] = stochastic ? bf16_stochastic(x, mix32(zs + (uint32_t)i)) : __float2bfloat16_rn(x);
  }
}

__device__ __forceinline__ float2 ldb2(const __nv_bfloat16* p) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}

// Adjoint step imaging against a BF16 background (stage: w halo FP32, a halo
// BF16, w_z FP32, a_z BF16, then mu_{t+1} and mu_{t+2}; the model and the
// image by read-only loads as in the FP32 step).
constexpr int A_OFF_AH = HALO_BYTES;
constexpr int A_OFF_P = A_OFF_AH + HXB * HY * 2;  // BF16 halo tile, HXB x HY
constexpr int A_OFF_AZ = A_OFF_P + PLAIN_BYTES;
constexpr int A_OFF_R = A_OFF_AZ + PLAIN_BYTES / 2;
constexpr int A_STAGE_BYTES = A_OFF_R + 4 * PLAIN_BYTES;  // 17408
constexpr int A_SMEM = G_STAGES * A_STAGE_BYTES + 1024 + 2 * G_STAGES * 8;
static_assert(2 * A_SMEM <= 228 * 1024, "two BF16 adjoint CTAs per SM");
static_assert(A_OFF_AH % 128 == 0 && A_OFF_P % 128 == 0 && A_OFF_AZ % 128 == 0 &&
                  A_OFF_R % 128 == 0 && A_STAGE_BYTES % 128 == 0,
              "TMA destinations on 128-byte boundaries");

struct AdjArgsB {
  AdjArgs f;              // as the FP32 step; az unused
  const __nv_bfloat16* az;  // a_{t-1} z (queue start)
  const float* sxs;       // per-plane scales of a_{t-1} x and z
  const float* szs;
};

__global__ void __launch_bounds__(NTHREADS, 2)
    k_adj3d_b16(const __grid_constant__ AdjMaps m, const __grid_constant__ AdjArgsB b) {
  extern __shared__ unsigned char smem_raw[];
  uint64_t *full, *empty;
  unsigned char* smem = ring_init<G_STAGES, A_STAGE_BYTES>(smem_raw, full, empty);
  const AdjArgs& a = b.f;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  long long k = 0;
  if (warp == NCW) {
    if (lane == 0) {
      const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(&m);
      for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x) {
        int bx, by, z0, z1;
        item(a.sc, it, bx, by, z0, z1);
        const int x0 = bx * TX, y0 = kHalo + by * TY;
        bool ok = true;
        for (int z = z0; z < z1; ++z, ++k) {
          const int s = (int)(k % G_STAGES);
          if (k >= G_STAGES &&
              !mbar_wait(&empty[s], (uint32_t)(((k / G_STAGES) & 1) ^ 1), a.status)) {
            ok = false;
            break;
          }
          const int zp = z + kZPad;
          unsigned char* st = smem + s * A_STAGE_BYTES;
          mbar_arrive_expect_tx(&full[s], A_STAGE_BYTES);
          tma_load(st, &maps[0], &full[s], x0 - kHalo, y0 - kHalo, zp);
          tma_load(st + A_OFF_AH, &maps[1], &full[s], x0 - 8, y0 - kHalo, zp);
          tma_load(st + A_OFF_P, &maps[2], &full[s], x0, y0, zp + kHalo);
          tma_load(st + A_OFF_AZ, &maps[3], &full[s], x0, y0, zp + kHalo);
#pragma unroll
          for (int j = 0; j < 4; ++j)
            tma_load(st + A_OFF_R + j * PLAIN_BYTES, &maps[4 + j], &full[s], x0, y0, zp);
        }
        if (!ok) break;
      }
    }
    return;
  }
  const int ry = warp * 2 + (lane >> 4);
  const int xo = 2 * (lane & 15);
  const int sr = (ry + kHalo) * HX + xo + kHalo;
  const int srb = (ry + kHalo) * HXB + xo + 8;  // centre in the BF16 halo tile
  const int pi = ry * TX + xo;
  for (int it = blockIdx.x; it < a.sc.items; it += gridDim.x) {
    int bx, by, z0, z1;
    item(a.sc, it, bx, by, z0, z1);
    const int x = bx * TX + xo;
    const int y = kHalo + by * TY + ry;
    const bool vy = y < a.d.ny - kHalo;
    const bool v0 = vy && x >= kHalo && x < a.d.nx - kHalo;
    const bool v1 = vy && x + 1 >= kHalo && x + 1 < a.d.nx - kHalo;
    const int off = y * a.d.pitch + x;
    float wq[2][9], aq[2][9], dxy[2];
    queue_init(wq, a.wz, a.d, off, z0, v0 || v1);
    aq[0][0] = aq[1][0] = 0.f;
#pragma unroll
    for (int kk = 1; kk < 9; ++kk) {
      const int zz = z0 - 5 + kk;
      const float2 v = (v0 || v1) ? ldb2(b.az + (long long)zz * a.d.plane + off)
                                  : make_float2(0.f, 0.f);
      const float sc = b.szs[zz + kZPad];
      aq[0][kk] = v.x * sc;
      aq[1][kk] = v.y * sc;
    }
    dxy[0] = v0 ? a.dampx[x] * a.dampy[y] : 1.f;
    dxy[1] = v1 ? a.dampx[x + 1] * a.dampy[y] : 1.f;
    bool ok = true;
    const bool any = v0 || v1;
    for (int z = z0; z < z1; ++z, ++k) {
      const float dz = a.dampz[z];
      const float scx = b.sxs[z + kZPad];
      const float scz = b.szs[z + kHalo + kZPad];
      // issued before the stage wait; this thread alone writes its image cells
      float2 c11, c13, c33, g11o, g13o, g33o;
      const long long gi = (long long)z * a.d.plane + off;
      ldg3(a.c11, a.c13, a.c33, gi, any, c11, c13, c33);
      ldg3(a.g11, a.g13, a.g33, gi, any, g11o, g13o, g33o);
      const int s = (int)(k % G_STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((k / G_STAGES) & 1), a.status)) {
        ok = false;
        break;
      }
      const unsigned char* st = smem + s * A_STAGE_BYTES;
      const float* pw = (const float*)(st + A_OFF_P) + pi;
      const __nv_bfloat16* paz = (const __nv_bfloat16*)(st + A_OFF_AZ) + pi;
      const float* pr = (const float*)(st + A_OFF_R) + pi;
      constexpr int T = TX * TY;
      queue_push(wq, ld2(pw));
      {
        const float2 v = ldb2(paz);
        queue_push(aq, make_float2(v.x * scz, v.y * scz));
      }
      Stencil2 sw;
      sw.load((const float*)st + sr);
      // a halo in BF16: the same stencil on the unscaled values, times the
      // plane's scale (linear)
      float ra[10];
      float2 yam[4], yap[4];
      {
        const __nv_bfloat16* h = (const __nv_bfloat16*)(st + A_OFF_AH) + srb;
#pragma unroll
        for (int j = 0; j < 5; ++j) {
          const float2 t = ldb2(h - 4 + 2 * j);
          ra[2 * j] = t.x;
          ra[2 * j + 1] = t.y;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          yam[j] = ldb2(h - (j + 1) * HXB);
          yap[j] = ldb2(h + (j + 1) * HXB);
        }
      }
      const float2 m1x = ld2(pr), m1z = ld2(pr + T);
      const float2 m2x = ld2(pr + 2 * T), m2z = ld2(pr + 3 * T);
      stage_release(&empty[s], lane);
      float mx[2], mz[2], wx[2], wzv[2], g11[2], g13[2], g33[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        auto pick = [e](float2 v) { return e ? v.y : v.x; };
        const float dd = dxy[e] * dz;
        const float lxy = sw.lxy(e, a.sx, a.sy);
        const float lz = lz_of(wq[e], a.sz);
        mx[e] = fmaf(dd, 2.f * pick(m1x) + lxy, -(2.f * dd - 1.f) * pick(m2x));
        mz[e] = fmaf(dd, 2.f * pick(m1z) + lz, -(2.f * dd - 1.f) * pick(m2z));
        wx[e] = fmaf(pick(c11), mx[e], pick(c13) * mz[e]);
        wzv[e] = fmaf(pick(c13), mx[e], pick(c33) * mz[e]);
        const float c = ra[4 + e];
        const float lxx = lap9(c, ra[3 + e], ra[5 + e], ra[2 + e], ra[6 + e], ra[1 + e],
                               ra[7 + e], ra[e], ra[8 + e]);
        const float lyy = lap9(c, pick(yam[0]), pick(yap[0]), pick(yam[1]), pick(yap[1]),
                               pick(yam[2]), pick(yap[2]), pick(yam[3]), pick(yap[3]));
        const float axy = fmaf(lyy, a.sy, lxx * a.sx) * scx;
        const float az = lz_of(aq[e], a.sz);
        g11[e] = fmaf(mx[e], axy, pick(g11o));
        g13[e] = fmaf(mx[e], az, fmaf(mz[e], axy, pick(g13o)));
        g33[e] = fmaf(mz[e], az, pick(g33o));
      }
      const long long i = (long long)z * a.d.plane + off;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (e ? v1 : v0) {
          a.mpx[i + e] = mx[e];
          a.mpz[i + e] = mz[e];
          a.wox[i + e] = wx[e];
          a.woz[i + e] = wzv[e];
          a.g11[i + e] = g11[e];
          a.g13[i + e] = g13[e];
          a.g33[i + e] = g33[e];
        }
      }
    }
    if (!ok) break;
  }
}

__device__ __forceinline__ float lap_b16(const __nv_bfloat16* f, long long o, long long stride,
                                         const float* sc, int z, int zstep) {
  auto v = [&](int k) { return __bfloat162float(f[o + k * stride]) * sc[z + k * zstep + kZPad]; };
  return lap9(v(0), v(-1), v(1), v(-2), v(2), v(-3), v(3), v(-4), v(4));
}

// k_inject_exact with the background a_{t-1} in BF16.
__global__ void k_inject_exact_b16(float* mx, float* mz, float* wx, float* wz, float* g11,
                                   float* g13, float* g33, const float* c11, const float* c13,
                                   const float* c33, const __nv_bfloat16* ax,
                                   const __nv_bfloat16* az, const float* sxs, const float* szs,
                                   const float* res, int nnt, int j, const long long* rec,
                                   const float* rec_damp, const unsigned char* live, int nr,
                                   Dims3 d, float sx, float sy, float sz) {
  const int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir >= nr || !live[ir] || rec_damp[ir] == 0.f) return;
  const float r = res[(long long)ir * nnt + j];
  const float dd = rec_damp[ir];
  const float dx_ = dd * (float)(kTwoThird * r);
  const float dz_ = dd * (float)(kOneThird * r);
  const long long o = rec[ir];
  const int z = (int)(o / d.plane);
  const float axy = fmaf(lap_b16(ax, o, d.pitch, sxs, z, 0), sy, lap_b16(ax, o, 1, sxs, z, 0) * sx);
  const float azz = lap_b16(az, o, d.plane, szs, z, 1) * sz;
  atomicAdd(mx + o, dx_);
  atomicAdd(mz + o, dz_);
  atomicAdd(wx + o, fmaf(c11[o], dx_, c13[o] * dz_));
  atomicAdd(wz + o, fmaf(c13[o], dx_, c33[o] * dz_));
  atomicAdd(g11 + o, dx_ * axy);
  atomicAdd(g13 + o, fmaf(dx_, azz, dz_ * axy));
  atomicAdd(g33 + o, dz_ * azz);
}

__device__ __forceinline__ float lap_at(const float* f, long long o, long long stride) {
  return lap9(f[o], f[o - stride], f[o + stride], f[o - 2 * stride], f[o + 2 * stride],
              f[o - 3 * stride], f[o + 3 * stride], f[o - 4 * stride], f[o + 4 * stride]);
}

// The residual term R^T r_t of the adjoint step at level t: for every live
// receiver cell inside the update region, mu += D (2/3 r, 1/3 r), w += C of
// that, and the image gets that increment times L a_{t-1} (the step kernel
// imaged mu without it). atomicAdd: receivers may share a cell.
__global__ void k_inject_exact(float* mx, float* mz, float* wx, float* wz, float* g11,
                               float* g13, float* g33, const float* c11, const float* c13,
                               const float* c33, const float* ax, const float* az,
                               const float* res, int nnt, int j, const long long* rec,
                               const float* rec_damp, const unsigned char* live, int nr, Dims3 d,
                               float sx, float sy, float sz) {
  const int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir >= nr || !live[ir] || rec_damp[ir] == 0.f) return;
  const float r = res[(long long)ir * nnt + j];
  const float dd = rec_damp[ir];
  const float dx_ = dd * (float)(kTwoThird * r);
  const float dz_ = dd * (float)(kOneThird * r);
  const long long o = rec[ir];
  const float axy = fmaf(lap_at(ax, o, d.pitch), sy, lap_at(ax, o, 1) * sx);
  const float azz = lap_at(az, o, d.plane) * sz;
  atomicAdd(mx + o, dx_);
  atomicAdd(mz + o, dz_);
  atomicAdd(wx + o, fmaf(c11[o], dx_, c13[o] * dz_));
  atomicAdd(wz + o, fmaf(c13[o], dx_, c33[o] * dz_));
  atomicAdd(g11 + o, dx_ * axy);
  atomicAdd(g13 + o, fmaf(dx_, azz, dz_ * axy));
  atomicAdd(g33 + o, dz_ * azz);
}

// Blocked, compensated summation of the images: the FP32 sums of one
// checkpoint block are added into an FP32 master with a Kahan compensation
// term (k_fold) and cleared; the master is the result (k_unfold copies it
// back). n = the volume's planes x plane floats from origin.
__global__ void k_fold(float* master, float* comp, float* img, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float y = img[i] - comp[i];
    const float t = master[i] + y;
    comp[i] = __fsub_rn(__fsub_rn(t, master[i]), y);
    master[i] = t;
    img[i] = 0.f;
  }
}

__global__ void k_unfold(const float* master, float* img, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    img[i] = master[i];
}

const CUtensorMap& PM(const TileMaps& m) { return *(const CUtensorMap*)m.plain; }
const CUtensorMap& HM(const TileMaps& m) { return *(const CUtensorMap*)m.halo; }

struct VolM {
  Vol v;
  TileMaps m;
};

// A BF16 volume (layout of Vol, 2-byte elements) with its per-plane scales.
struct VolB {
  void* alloc = nullptr;
  __nv_bfloat16* origin = nullptr;
  float* scale = nullptr;  // nz + 2 kZPad
  TileMaps m;
};

// once per device and kernel (atomic flags: first calls may come from
// several host threads)
std::atomic<bool> attr_born[64], attr_adj[64];

int smem_attr(vti_ctx* ctx, const void* kern, std::atomic<bool>* done, int bytes = G_SMEM) {
  if (ctx->device < 64 && done[ctx->device].load(std::memory_order_acquire)) return VTI_OK;
  VTI_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if (ctx->device < 64) done[ctx->device].store(true, std::memory_order_release);
  return VTI_OK;
}

// Exact-mode state of one shot: model, perturbation, fields, checkpoints,
// the segment buffer and the adjoint fields of the two images.
struct GnState {
  vti_ctx* ctx = nullptr;
  vti3d_geom g{};
  Dims3 d{};
  int M = 0, K = 0;
  bool stochastic = false;  // BF16 packing: stochastic rounding (else nearest)
  VolM c[3], dc[3];
  VolM a[2][2], b[2][2];       // [buffer][x, z]
  std::vector<VolM> ck;        // checkpoint k: levels k*K (x, z), k*K+1 (x, z)
  std::vector<VolM> seg;       // (K+1) levels x (x, z)
  VolM mu[2][2][2], w[2][2][2];  // [image][buffer][x, z]
  VolM img[2][3];
  float* master[2][3] = {};   // compensated FP32 sums of the images: master
  float* comp[2][3] = {};     // and Kahan compensation
  VolM ring[3][2];            // BF16 mode: FP32 levels of the recomputation
  std::vector<VolB> segb;     // BF16 mode: (K+1) levels x (x, z)
  float* damp = nullptr;
  ~GnState() {
    for (auto& x : segb) {
      if (x.alloc) cudaFree(x.alloc);
      if (x.scale) cudaFree(x.scale);
    }
    for (auto& r : ring) for (auto& x : r) vol_free(&x.v);
    for (auto& i : master)
      for (float* q : i)
        if (q) cudaFree(q);
    for (auto& i : comp)
      for (float* q : i)
        if (q) cudaFree(q);
    auto fr = [](VolM& x) { vol_free(&x.v); };
    for (auto& x : c) fr(x);
    for (auto& x : dc) fr(x);
    for (auto& r : a) for (auto& x : r) fr(x);
    for (auto& r : b) for (auto& x : r) fr(x);
    for (auto& x : ck) fr(x);
    for (auto& x : seg) fr(x);
    for (auto& i : mu) for (auto& r : i) for (auto& x : r) fr(x);
    for (auto& i : w) for (auto& r : i) for (auto& x : r) fr(x);
    for (auto& i : img) for (auto& x : i) fr(x);
    if (damp) cudaFree(damp);
  }
  int alloc(VolM* x) {
    VTI_TRY(vol_alloc(ctx, d, &x->v));
    VTI_TRY(vol_zero(ctx, d, &x->v));
    return make_tile_maps(ctx, d, x->v, &x->m);
  }
  int alloc(VolB* x) {
    const size_t n = (size_t)d.plane * (d.nz + 2 * kZPad);
    if (cudaMalloc(&x->alloc, n * 2) != cudaSuccess ||
        cudaMalloc((void**)&x->scale, (d.nz + 2 * kZPad) * sizeof(float)) != cudaSuccess)
      return fail(ctx, VTI_ERR_OOM, "BF16 segment");
    VTI_CUDA(ctx, cudaMemsetAsync(x->alloc, 0, n * 2, ctx->stream));
    VTI_CUDA(ctx, cudaMemsetAsync(x->scale, 0, (d.nz + 2 * kZPad) * sizeof(float), ctx->stream));
    x->origin = (__nv_bfloat16*)x->alloc + (size_t)kZPad * d.plane;
    return make_tile_maps_typed(ctx, d, x->alloc, 2, &x->m);
  }
};

int launch_born(GnState& S, int cur, const p3d::ShotGeom& sg, float amp) {
  vti_ctx* ctx = S.ctx;
  VTI_TRY(smem_attr(ctx, (const void*)k_born3d_tma, attr_born, GB_SMEM));
  const int nxt = 1 - cur;
  BornMaps m;
  m.ax = HM(S.a[cur][0].m);
  m.bx = HM(S.b[cur][0].m);
  m.az = PM(S.a[cur][1].m);
  m.bz = PM(S.b[cur][1].m);
  m.apx = PM(S.a[nxt][0].m);
  m.apz = PM(S.a[nxt][1].m);
  m.bpx = PM(S.b[nxt][0].m);
  m.bpz = PM(S.b[nxt][1].m);
  m.c11 = PM(S.c[0].m); m.c13 = PM(S.c[1].m); m.c33 = PM(S.c[2].m);
  m.d11 = PM(S.dc[0].m); m.d13 = PM(S.dc[1].m); m.d33 = PM(S.dc[2].m);
  const float dt2 = S.g.dt * S.g.dt;
  BornArgs x{};
  x.d = S.d;
  x.sc = make_sched(ctx, S.d, 2);
  x.az = S.a[cur][1].v.origin;
  x.bz = S.b[cur][1].v.origin;
  x.apx = S.a[nxt][0].v.origin;
  x.apz = S.a[nxt][1].v.origin;
  x.bpx = S.b[nxt][0].v.origin;
  x.bpz = S.b[nxt][1].v.origin;
  x.dampx = S.damp;
  x.dampy = S.damp + S.g.nx;
  x.dampz = S.damp + S.g.nx + S.g.ny;
  x.sx = dt2 / (S.g.dx * S.g.dx);
  x.sy = dt2 / (S.g.dy * S.g.dy);
  x.sz = dt2 / (S.g.dz * S.g.dz);
  x.src.x = sg.sx; x.src.y = sg.sy; x.src.z = sg.sz; x.src.amp = amp;
  x.status = ctx->d_status;
  {
    LaunchTimer tm(ctx, kTimedFwd3d);
    k_born3d_tma<<<x.sc.grid, NTHREADS, GB_SMEM, ctx->stream>>>(m, x);
  }
  VTI_LAUNCHED(ctx, "k_born3d_tma");
  return VTI_OK;
}

// Adjoint step of image `im` at level t: mu_{t+1} in mu[im][cur], mu_{t+2}
// (overwritten by mu_t) in mu[im][1-cur], w_{t+1} in w[im][cur] (w_t into
// w[im][1-cur]), a_{t-1} in segment slot `slot`.
int launch_adj(GnState& S, int im, int cur, int slot) {
  vti_ctx* ctx = S.ctx;
  VTI_TRY(smem_attr(ctx, (const void*)k_adj3d_tma, attr_adj));
  const int nx_ = 1 - cur;
  const VolM* ax = &S.seg[2 * slot];
  const VolM* az = &S.seg[2 * slot + 1];
  AdjMaps m;
  m.wx = HM(S.w[im][cur][0].m);
  m.ax = HM(ax->m);
  m.wz = PM(S.w[im][cur][1].m);
  m.az = PM(az->m);
  m.m1x = PM(S.mu[im][cur][0].m);
  m.m1z = PM(S.mu[im][cur][1].m);
  m.mpx = PM(S.mu[im][nx_][0].m);
  m.mpz = PM(S.mu[im][nx_][1].m);
  const float dt2 = S.g.dt * S.g.dt;
  AdjArgs x{};
  x.c11 = S.c[0].v.origin; x.c13 = S.c[1].v.origin; x.c33 = S.c[2].v.origin;
  x.d = S.d;
  x.sc = make_sched(ctx, S.d, 2);
  x.wz = S.w[im][cur][1].v.origin;
  x.az = az->v.origin;
  x.mpx = S.mu[im][nx_][0].v.origin;
  x.mpz = S.mu[im][nx_][1].v.origin;
  x.wox = S.w[im][nx_][0].v.origin;
  x.woz = S.w[im][nx_][1].v.origin;
  x.g11 = S.img[im][0].v.origin;
  x.g13 = S.img[im][1].v.origin;
  x.g33 = S.img[im][2].v.origin;
  x.dampx = S.damp;
  x.dampy = S.damp + S.g.nx;
  x.dampz = S.damp + S.g.nx + S.g.ny;
  x.sx = dt2 / (S.g.dx * S.g.dx);
  x.sy = dt2 / (S.g.dy * S.g.dy);
  x.sz = dt2 / (S.g.dz * S.g.dz);
  x.status = ctx->d_status;
  {
    LaunchTimer tm(ctx, kTimedBwd3d);
    k_adj3d_tma<<<x.sc.grid, NTHREADS, G_SMEM, ctx->stream>>>(m, x);
  }
  VTI_LAUNCHED(ctx, "k_adj3d_tma");
  return VTI_OK;
}

std::atomic<bool> attr_adjb[64];

int launch_adj_b16(GnState& S, int im, int cur, int slot) {
  vti_ctx* ctx = S.ctx;
  {
    const int st = smem_attr(ctx, (const void*)k_adj3d_b16, attr_adjb, A_SMEM);
    if (st != VTI_OK) return st;
  }
  const int nx_ = 1 - cur;
  const VolB& ax = S.segb[2 * slot];
  const VolB& az = S.segb[2 * slot + 1];
  AdjMaps m;
  m.wx = HM(S.w[im][cur][0].m);
  m.ax = HM(ax.m);
  m.wz = PM(S.w[im][cur][1].m);
  m.az = PM(az.m);
  m.m1x = PM(S.mu[im][cur][0].m);
  m.m1z = PM(S.mu[im][cur][1].m);
  m.mpx = PM(S.mu[im][nx_][0].m);
  m.mpz = PM(S.mu[im][nx_][1].m);
  const float dt2 = S.g.dt * S.g.dt;
  AdjArgsB b{};
  AdjArgs& x = b.f;
  x.c11 = S.c[0].v.origin; x.c13 = S.c[1].v.origin; x.c33 = S.c[2].v.origin;
  x.d = S.d;
  x.sc = make_sched(ctx, S.d, 2);
  x.wz = S.w[im][cur][1].v.origin;
  x.az = nullptr;
  x.mpx = S.mu[im][nx_][0].v.origin;
  x.mpz = S.mu[im][nx_][1].v.origin;
  x.wox = S.w[im][nx_][0].v.origin;
  x.woz = S.w[im][nx_][1].v.origin;
  x.g11 = S.img[im][0].v.origin;
  x.g13 = S.img[im][1].v.origin;
  x.g33 = S.img[im][2].v.origin;
  x.dampx = S.damp;
  x.dampy = S.damp + S.g.nx;
  x.dampz = S.damp + S.g.nx + S.g.ny;
  x.sx = dt2 / (S.g.dx * S.g.dx);
  x.sy = dt2 / (S.g.dy * S.g.dy);
  x.sz = dt2 / (S.g.dz * S.g.dz);
  x.status = ctx->d_status;
  b.az = az.origin;
  b.sxs = ax.scale;
  b.szs = az.scale;
  {
    LaunchTimer tm(ctx, kTimedBwd3d);
    k_adj3d_b16<<<x.sc.grid, NTHREADS, A_SMEM, ctx->stream>>>(m, b);
  }
  VTI_LAUNCHED(ctx, "k_adj3d_b16");
  return VTI_OK;
}

// level: time level of the packed field, component: 0 x, 1 z (random bits)
int pack(GnState& S, const VolM& src, VolB& dst, int level, int component) {
  const uint32_t seed = (uint32_t)level * 2u + (uint32_t)component;
  k_pack_bf16<<<S.d.nz, 256, 0, S.ctx->stream>>>(src.v.origin, S.d, dst.origin, dst.scale, seed,
                                                 S.stochastic ? 1 : 0);
  VTI_LAUNCHED(S.ctx, "k_pack_bf16");
  return VTI_OK;
}

int copy_vol(vti_ctx* ctx, const Vol& src, Vol* dst) {
  VTI_CUDA(ctx, cudaMemcpyAsync(dst->alloc, src.alloc, src.bytes, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  return VTI_OK;
}

}  // namespace
}  // namespace vti

using namespace vti;

extern "C" {

int vti3d_gnhv_exact(vti_ctx* ctx, const vti3d_geom* g, const float* c11, const float* c13,
                     const float* c33, const float* dc, const float* wavelet, const float* souloc,
                     const float* recloc, int nrec, const float* dobs, int checkpoint_every,
                     unsigned gn_flags, float* hv, float* grad, double* misfit, float* traces,
                     float* born) {
  if (!ctx || !g) return VTI_ERR_ARG;
  const bool b16 = (gn_flags & VTI_GNHV_BF16) != 0;
  if ((gn_flags & VTI_GNHV_BF16_SR) && !b16)
    return fail(ctx, VTI_ERR_ARG, "VTI_GNHV_BF16_SR needs VTI_GNHV_BF16");
  VTI_TRY(p3d::check_geom(ctx, g));
  if (!c11 || !c13 || !c33 || !wavelet || !souloc || (nrec > 0 && !recloc))
    return fail(ctx, VTI_ERR_ARG, "null input");
  if ((hv || born) && !dc) return fail(ctx, VTI_ERR_ARG, "H dc / Born traces need dc");
  if ((grad || misfit) && !dobs) return fail(ctx, VTI_ERR_ARG, "the gradient needs dobs");
  VTI_TRY(cfl_verdict(ctx, vti3d_cfl_number(g, c11, c13, c33), "model"));
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  const unsigned flags = VTI_OPT_FULL_STEPS;
  // the per-shot helpers of the plan: receivers, schedule, damping tables
  vti3d_plan* p = nullptr;
  VTI_TRY(vti3d_plan_create(ctx, g, flags, &p));
  struct PlanGuard {
    vti3d_plan* p;
    ~PlanGuard() { vti3d_plan_destroy(p); }
  } guard{p};
  p->wavelet.assign(wavelet, wavelet + g->nt);
  p->recloc.assign(recloc, recloc + 4 * (size_t)nrec);
  p->nrec_total = nrec;
  p3d::ShotGeom sg;
  VTI_TRY(p3d::shot_geom(p, souloc, 0, &sg));
  VTI_TRY(p3d::upload_shot(p, sg));
  GnState S;
  S.ctx = ctx;
  S.stochastic = (gn_flags & VTI_GNHV_BF16_SR) != 0;
  S.g = *g;
  S.d = p->d;
  S.M = p3d::last_level(*g, flags);
  S.K = checkpoint_every > 0 ? checkpoint_every : 64;
  const int M = S.M, K = S.K;
  const int nnt = p3d::nnt_of(*g);
  const float dt2 = g->dt * g->dt;
  const bool want_born = hv || born;
  const bool want_grad = grad || misfit;
  S.damp = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&S.damp, p->h_damp.size() * sizeof(float)));
  VTI_CUDA(ctx, cudaMemcpy(S.damp, p->h_damp.data(), p->h_damp.size() * sizeof(float),
                           cudaMemcpyHostToDevice));
  const float* cs[3] = {c11, c13, c33};
  for (int k = 0; k < 3; ++k) {
    VTI_TRY(S.alloc(&S.c[k]));
    VTI_TRY(vol_upload(ctx, S.d, &S.c[k].v, cs[k], VTI_MEM_HOST));
    VTI_TRY(S.alloc(&S.dc[k]));
    if (dc) VTI_TRY(vol_upload(ctx, S.d, &S.dc[k].v, dc + (size_t)k * S.d.npoints(), VTI_MEM_HOST));
  }
  for (int bf = 0; bf < 2; ++bf)
    for (int f = 0; f < 2; ++f) {
      VTI_TRY(S.alloc(&S.a[bf][f]));
      VTI_TRY(S.alloc(&S.b[bf][f]));
    }
  // checkpoints: blocks of K levels a_{1+iK} ... ; block i needs a_{iK}, a_{1+iK}
  const int nblk = (M - 1 + K - 1) / K;
  S.ck.resize(4 * (size_t)nblk);
  for (auto& x : S.ck) VTI_TRY(vol_alloc(ctx, S.d, &x.v));
  if (b16) {
    for (auto& r : S.ring)
      for (auto& x : r) VTI_TRY(S.alloc(&x));
    S.segb.resize(2 * (size_t)(K + 1));
    for (auto& x : S.segb) VTI_TRY(S.alloc(&x));
  } else {
    S.seg.resize(2 * (size_t)(K + 1));
    for (auto& x : S.seg) VTI_TRY(S.alloc(&x));
  }
  // traces: background, Born
  float* d_tr = p->d_trace;  // nnt * nr (the plan's buffer)
  float* d_born = nullptr;
  const size_t ntr = (size_t)nnt * std::max(sg.nr, 1);
  VTI_CUDA(ctx, cudaMalloc((void**)&d_born, ntr * sizeof(float)));
  struct Free {
    void* q;
    ~Free() { if (q) cudaFree(q); }
  } free_born{d_born};
  VTI_CUDA(ctx, cudaMemsetAsync(d_tr, 0, ntr * sizeof(float), ctx->stream));
  VTI_CUDA(ctx, cudaMemsetAsync(d_born, 0, ntr * sizeof(float), ctx->stream));
  // ---- forward: background + Born, traces, checkpoints
  const long long so = S.d.off(sg.sx, sg.sy, sg.sz);
  VTI_TRY(launch_set_point(ctx, S.a[0][0].v.origin, S.a[0][1].v.origin, so, dt2 * wavelet[0]));
  auto store_ck = [&](int blk, int cur) -> int {
    // a_{level-1} is in buffer 1-cur, a_level in cur
    VTI_TRY(copy_vol(ctx, S.a[1 - cur][0].v, &S.ck[4 * blk + 0].v));
    VTI_TRY(copy_vol(ctx, S.a[1 - cur][1].v, &S.ck[4 * blk + 1].v));
    VTI_TRY(copy_vol(ctx, S.a[cur][0].v, &S.ck[4 * blk + 2].v));
    VTI_TRY(copy_vol(ctx, S.a[cur][1].v, &S.ck[4 * blk + 3].v));
    return VTI_OK;
  };
  VTI_TRY(store_ck(0, 0));  // a_0 = 0 (buffer 1), a_1 (buffer 0)
  int cur = 0;
  for (int t = 2; t <= M; ++t) {
    VTI_TRY(launch_born(S, cur, sg, dt2 * wavelet[t - 1]));
    cur = 1 - cur;  // level t now in `cur`
    if (t < (int)sg.rec_at.size() && sg.rec_at[t] >= 0) {
      VTI_TRY(launch_record(ctx, d_tr, nnt, sg.rec_at[t], S.a[cur][0].v.origin,
                            S.a[cur][1].v.origin, p->d_rec, sg.nr));
      if (want_born)
        VTI_TRY(launch_record(ctx, d_born, nnt, sg.rec_at[t], S.b[cur][0].v.origin,
                              S.b[cur][1].v.origin, p->d_rec, sg.nr));
    }
    if ((t - 1) % K == 0 && (t - 1) / K < nblk) VTI_TRY(store_ck((t - 1) / K, cur));
  }
  // dead receivers record zero; residual and FP64 misfit
  VTI_TRY(launch_residual(ctx, d_born, nullptr, p->d_live, nnt, sg.nr, nullptr));
  double* d_acc = nullptr;
  VTI_CUDA(ctx, cudaMalloc((void**)&d_acc, (1 + residual_blocks(ctx)) * sizeof(double)));
  struct FreeD {
    void* q;
    ~FreeD() { if (q) cudaFree(q); }
  } free_acc{d_acc};
  VTI_CUDA(ctx, cudaMemsetAsync(d_acc, 0, sizeof(double), ctx->stream));
  std::vector<float> h_tr;
  if (traces) {
    VTI_TRY(launch_residual(ctx, d_tr, nullptr, p->d_live, nnt, sg.nr, nullptr));
    VTI_CUDA(ctx, cudaMemcpyAsync(traces, d_tr, (size_t)nnt * sg.nr * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (born)
    VTI_CUDA(ctx, cudaMemcpyAsync(born, d_born, (size_t)nnt * sg.nr * sizeof(float),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  if (want_grad) {
    const float* obs = nullptr;
    VTI_TRY(p3d::get_obs(p, sg, dobs, VTI_MEM_HOST, &obs));
    VTI_TRY(launch_residual(ctx, d_tr, obs, p->d_live, nnt, sg.nr, d_acc));
  }
  // ---- backward: images 0 (gradient, residual d_tr) and 1 (H dc, Born d_born)
  const bool want[2] = {grad != nullptr, hv != nullptr};
  const float* src[2] = {d_tr, d_born};
  for (int im = 0; im < 2; ++im) {
    if (!want[im]) continue;
    for (int bf = 0; bf < 2; ++bf)
      for (int f = 0; f < 2; ++f) {
        VTI_TRY(S.alloc(&S.mu[im][bf][f]));
        VTI_TRY(S.alloc(&S.w[im][bf][f]));
      }
    for (int k = 0; k < 3; ++k) {
      VTI_TRY(S.alloc(&S.img[im][k]));
      const size_t nb = (size_t)S.d.plane * S.d.nz * sizeof(float);
      VTI_CUDA(ctx, cudaMalloc((void**)&S.master[im][k], nb));
      VTI_CUDA(ctx, cudaMalloc((void**)&S.comp[im][k], nb));
      VTI_CUDA(ctx, cudaMemsetAsync(S.master[im][k], 0, nb, ctx->stream));
      VTI_CUDA(ctx, cudaMemsetAsync(S.comp[im][k], 0, nb, ctx->stream));
    }
  }
  const long long nimg = S.d.plane * S.d.nz;
  const int fgrid = (int)std::min<long long>((nimg + 255) / 256, ctx->sm_count * 8LL);
  int mcur = 0;  // mu_{t+1} / w_{t+1} buffer (both images step together)
  const float sxs = dt2 / (g->dx * g->dx), sys = dt2 / (g->dy * g->dy), szs = dt2 / (g->dz * g->dz);
  for (int blk = nblk - 1; blk >= 0; --blk) {
    const int k0 = 1 + blk * K;             // first level a_{t-1} of the block
    const int k1 = std::min(k0 + K - 1, M - 1);  // last
    // slots: s holds level k0 - 1 + s (FP32 segment, or BF16 segment fed
    // from a 3-level FP32 ring, level L in ring slot L % 3)
    auto lvl = [&](int L) -> VolM* { return b16 ? S.ring[L % 3] : &S.seg[2 * (L - (k0 - 1))]; };
    for (int f = 0; f < 2; ++f) {
      VTI_TRY(copy_vol(ctx, S.ck[4 * blk + f].v, &lvl(k0 - 1)[f].v));
      VTI_TRY(copy_vol(ctx, S.ck[4 * blk + 2 + f].v, &lvl(k0)[f].v));
    }
    if (b16)
      for (int f = 0; f < 2; ++f) {
        VTI_TRY(pack(S, lvl(k0 - 1)[f], S.segb[f], k0 - 1, f));
        VTI_TRY(pack(S, lvl(k0)[f], S.segb[2 + f], k0, f));
      }
    Damping dmp{S.damp, S.damp + g->nx, S.damp + g->nx + g->ny};
    for (int t = k0 + 1; t <= k1; ++t) {
      PointSource ps;
      ps.x = sg.sx; ps.y = sg.sy; ps.z = sg.sz; ps.amp = dt2 * wavelet[t - 1];
      const VolM* cx = lvl(t - 1);
      const VolM* px = lvl(t - 2);
      VolM* nx_ = lvl(t);
      VTI_TRY(launch_fwd3d_tma(ctx, S.d, cx[0].m, cx[1].m, px[0].m, px[1].m, S.c[0].m, S.c[1].m,
                               S.c[2].m, cx[1].v.origin, nx_[0].v.origin, nx_[1].v.origin, &dmp,
                               sxs, sys, szs, ps, Probe(), true));
      if (b16) {
        const int sl = t - (k0 - 1);
        VTI_TRY(pack(S, nx_[0], S.segb[2 * sl], t, 0));
        VTI_TRY(pack(S, nx_[1], S.segb[2 * sl + 1], t, 1));
      }
    }
    for (int tm1 = k1; tm1 >= k0; --tm1) {
      const int t = tm1 + 1;
      const int slot = tm1 - (k0 - 1);
      for (int im = 0; im < 2; ++im) {
        if (!want[im]) continue;
        VTI_TRY(b16 ? launch_adj_b16(S, im, mcur, slot) : launch_adj(S, im, mcur, slot));
        const int nb = 1 - mcur;  // mu_t / w_t were written there
        if (b16 && t < (int)sg.rec_at.size() && sg.rec_at[t] >= 0 && sg.nr > 0) {
          k_inject_exact_b16<<<(sg.nr + 127) / 128, 128, 0, ctx->stream>>>(
              S.mu[im][nb][0].v.origin, S.mu[im][nb][1].v.origin, S.w[im][nb][0].v.origin,
              S.w[im][nb][1].v.origin, S.img[im][0].v.origin, S.img[im][1].v.origin,
              S.img[im][2].v.origin, S.c[0].v.origin, S.c[1].v.origin, S.c[2].v.origin,
              S.segb[2 * slot].origin, S.segb[2 * slot + 1].origin, S.segb[2 * slot].scale,
              S.segb[2 * slot + 1].scale, src[im], nnt, sg.rec_at[t], p->d_rec, p->d_rec_damp,
              p->d_live, sg.nr, S.d, sxs, sys, szs);
          VTI_LAUNCHED(ctx, "k_inject_exact_b16");
        } else if (t < (int)sg.rec_at.size() && sg.rec_at[t] >= 0 && sg.nr > 0) {
          k_inject_exact<<<(sg.nr + 127) / 128, 128, 0, ctx->stream>>>(
              S.mu[im][nb][0].v.origin, S.mu[im][nb][1].v.origin, S.w[im][nb][0].v.origin,
              S.w[im][nb][1].v.origin, S.img[im][0].v.origin, S.img[im][1].v.origin,
              S.img[im][2].v.origin, S.c[0].v.origin, S.c[1].v.origin, S.c[2].v.origin,
              S.seg[2 * slot].v.origin, S.seg[2 * slot + 1].v.origin, src[im], nnt,
              sg.rec_at[t], p->d_rec, p->d_rec_damp, p->d_live, sg.nr, S.d, sxs, sys, szs);
          VTI_LAUNCHED(ctx, "k_inject_exact");
        }
      }
      mcur = 1 - mcur;
    }
    // this block's FP32 image sums into the compensated masters
    for (int im = 0; im < 2; ++im)
      if (want[im])
        for (int k = 0; k < 3; ++k) {
          k_fold<<<fgrid, 256, 0, ctx->stream>>>(S.master[im][k], S.comp[im][k],
                                                 S.img[im][k].v.origin, nimg);
          VTI_LAUNCHED(ctx, "k_fold");
        }
  }
  for (int im = 0; im < 2; ++im)
    if (want[im])
      for (int k = 0; k < 3; ++k) {
        k_unfold<<<fgrid, 256, 0, ctx->stream>>>(S.master[im][k], S.img[im][k].v.origin, nimg);
        VTI_LAUNCHED(ctx, "k_unfold");
      }
  const size_t n = (size_t)S.d.npoints();
  float* outs[2] = {grad, hv};
  for (int im = 0; im < 2; ++im)
    if (want[im] && outs[im])
      for (int k = 0; k < 3; ++k)
        VTI_TRY(vol_download(ctx, S.d, &S.img[im][k].v, outs[im] + k * n, VTI_MEM_HOST));
  double acc = 0;
  VTI_CUDA(ctx, cudaMemcpyAsync(&acc, d_acc, sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
  VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  VTI_TRY(check_device_status(ctx));
  if (misfit) *misfit = acc / 2;
  return VTI_OK;
}

}  // extern "C"
