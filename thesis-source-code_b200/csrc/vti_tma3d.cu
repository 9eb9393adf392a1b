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

#include <cuda.h>
#include <cudaTypedefs.h>

#include "vti_internal.h"

namespace vti {
namespace {

constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;

constexpr int TX = 32, TY = 16, RY = 2, NCW = TY / RY;  // consumer warps
constexpr int NTHREADS = (NCW + 1) * 32;
constexpr int HX = TX + 2 * kHalo, HY = TY + 2 * kHalo;
constexpr int PLAIN_BYTES = TX * TY * 4;  // 2048
constexpr int HALO_BYTES = HX * HY * 4;   // 3840
constexpr unsigned kSpinLimit = 1u << 26;

__device__ __forceinline__ float lap9(float c, float m1, float p1, float m2, float p2, float m3,
                                      float p3, float m4, float p4) {
  float s = kC0 * c;
  s = fmaf(kC1, m1 + p1, s);
  s = fmaf(kC2, m2 + p2, s);
  s = fmaf(kC3, m3 + p3, s);
  s = fmaf(kC4, m4 + p4, s);
  return s;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false (and the status word set) if the phase never completes.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
  for (unsigned i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(status, 1 << VTI_ERR_TIMEOUT);
  return false;
}
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                         int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

struct Sched {
  int gx, gy;  // columns in x, y
  int nz;
  int seg;     // planes per segment
  int items;   // gx * gy * ceil(nz / seg)
  int grid;    // persistent CTAs, min(items, resident slots)
};

// Item i: segment i / (gx*gy) of column i % (gx*gy), planes [z0, z1).
__device__ __forceinline__ void item(const Sched& s, int i, int& bx, int& by, int& z0,
                                     int& z1) {
  const int cols = s.gx * s.gy;
  const int sg = i / cols, col = i - sg * cols;
  bx = col % s.gx;
  by = col / s.gx;
  z0 = sg * s.seg;
  z1 = min(s.nz, z0 + s.seg);
}

// ------------------------------------------------------------ forward
struct FwdArgs {
  Dims3 d;
  Sched sc;
  const float* cz;  // cur sigma_z (queue initialisation)
  float* px;        // prev in / next out
  float* pz;
  const float* dampx;  // null: no sponge
  const float* dampy;
  const float* dampz;
  float sx, sy, sz;
  PointSource src;
  int* status;
};

constexpr int F_STAGES = 4;
// stage layout: [halo x][z+4][prev x][prev z][c11][c13][c33]
constexpr int F_OFF_H = 0;
constexpr int F_OFF_Z = HALO_BYTES;
constexpr int F_OFF_PX = F_OFF_Z + PLAIN_BYTES;
constexpr int F_OFF_PZ = F_OFF_PX + PLAIN_BYTES;
constexpr int F_OFF_C = F_OFF_PZ + PLAIN_BYTES;
constexpr int F_STAGE_BYTES = F_OFF_C + 3 * PLAIN_BYTES;  // 15872
constexpr int F_SMEM = F_STAGES * F_STAGE_BYTES + 1024 + 2 * F_STAGES * 8;

__global__ void __launch_bounds__(NTHREADS, 3)
    k_fwd3d_tma(const __grid_constant__ CUtensorMap m_cx, const __grid_constant__ CUtensorMap m_cz,
                const __grid_constant__ CUtensorMap m_px, const __grid_constant__ CUtensorMap m_pz,
                const __grid_constant__ CUtensorMap m_c11,
                const __grid_constant__ CUtensorMap m_c13,
                const __grid_constant__ CUtensorMap m_c33, const FwdArgs a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + F_STAGES * F_STAGE_BYTES);
  uint64_t* empty = full + F_STAGES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < F_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const Dims3 d = a.d;

  if (warp == NCW) {  // ---------------- producer
    if (lane == 0) {
      long long k = 0;  // planes issued by this CTA
      bool ok = true;
      for (int it = blockIdx.x; ok && it < a.sc.items; it += gridDim.x) {
        int bx, by, z0, z1;
        item(a.sc, it, bx, by, z0, z1);
        const int x0 = bx * TX, y0 = kHalo + by * TY;
        for (int z = z0; z < z1; ++z, ++k) {
          const int s = (int)(k % F_STAGES);
          if (k >= F_STAGES &&
              !mbar_wait(&empty[s], (uint32_t)(((k / F_STAGES) & 1) ^ 1), a.status)) {
            ok = false;
            break;
          }
          const int zp = z + kZPad;
          unsigned char* st = smem + s * F_STAGE_BYTES;
          mbar_arrive_expect_tx(&full[s], F_STAGE_BYTES);
          tma_load(st + F_OFF_H, &m_cx, &full[s], x0 - kHalo, y0 - kHalo, zp);
          tma_load(st + F_OFF_Z, &m_cz, &full[s], x0, y0, zp + kHalo);
          tma_load(st + F_OFF_PX, &m_px, &full[s], x0, y0, zp);
          tma_load(st + F_OFF_PZ, &m_pz, &full[s], x0, y0, zp);
          tma_load(st + F_OFF_C, &m_c11, &full[s], x0, y0, zp);
          tma_load(st + F_OFF_C + PLAIN_BYTES, &m_c13, &full[s], x0, y0, zp);
          tma_load(st + F_OFF_C + 2 * PLAIN_BYTES, &m_c33, &full[s], x0, y0, zp);
        }
      }
    }
    return;
  }

  // ---------------- consumers: thread (lane, warp) owns x = x0+lane, rows 2w, 2w+1
  const bool damp = a.dampz != nullptr;
  float q[RY][9];
  float dxy[RY];
  int off[RY];
  bool valid[RY];
  long long k = 0;  // planes consumed by this CTA
  bool ok = true;
  for (int it = blockIdx.x; ok && it < a.sc.items; it += gridDim.x) {
    int bx, by, z0, z1;
    item(a.sc, it, bx, by, z0, z1);
    const int x = bx * TX + lane;
    const int y0 = kHalo + by * TY;
    // start the queue: planes z0-4 .. z0+3 from global
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int y = y0 + warp * RY + r;
      valid[r] = x >= kHalo && x < d.nx - kHalo && y < d.ny - kHalo;
      off[r] = y * d.pitch + x;
      dxy[r] = (damp && valid[r]) ? a.dampx[x] * a.dampy[y] : 1.f;
      q[r][0] = 0.f;
#pragma unroll
      for (int kk = 1; kk < 9; ++kk) {
        const int zz = z0 - 5 + kk;
        float v = valid[r] ? __ldg(a.cz + (long long)zz * d.plane + off[r]) : 0.f;
        // planes of the block above z0 were already damped as "cur"
        if (damp && zz >= 0 && (zz >> 2) < (z0 >> 2)) v *= dxy[r] * a.dampz[zz];
        q[r][kk] = v;
      }
    }
    for (int z = z0; z < z1; ++z, ++k) {
      const int s = (int)(k % F_STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((k / F_STAGES) & 1), a.status)) {
        ok = false;
        break;
      }
      const float* sh = (const float*)(smem + s * F_STAGE_BYTES + F_OFF_H);
      const float* sq = (const float*)(smem + s * F_STAGE_BYTES + F_OFF_Z);
      const float* spx = (const float*)(smem + s * F_STAGE_BYTES + F_OFF_PX);
      const float* spz = (const float*)(smem + s * F_STAGE_BYTES + F_OFF_PZ);
      const float* s11 = (const float*)(smem + s * F_STAGE_BYTES + F_OFF_C);
      const float* s13 = s11 + TX * TY;
      const float* s33 = s13 + TX * TY;
      const float dz = damp ? a.dampz[z] : 1.f;
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int ry = warp * RY + r;
        const int pi = ry * TX + lane;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) q[r][kk] = q[r][kk + 1];
        q[r][8] = sq[pi];
        const int sr = (ry + kHalo) * HX + lane + kHalo;
        const float c = sh[sr];
        const float lxx = lap9(c, sh[sr - 1], sh[sr + 1], sh[sr - 2], sh[sr + 2], sh[sr - 3],
                               sh[sr + 3], sh[sr - 4], sh[sr + 4]);
        const float lyy = lap9(c, sh[sr - HX], sh[sr + HX], sh[sr - 2 * HX], sh[sr + 2 * HX],
                               sh[sr - 3 * HX], sh[sr + 3 * HX], sh[sr - 4 * HX], sh[sr + 4 * HX]);
        const float lzz =
            lap9(q[r][4], q[r][3], q[r][5], q[r][2], q[r][6], q[r][1], q[r][7], q[r][0], q[r][8]);
        const float lxy = fmaf(lyy, a.sy, lxx * a.sx);
        const float lz = lzz * a.sz;
        const float dd = dxy[r] * dz;
        float nxv = fmaf(s11[pi], lxy, fmaf(s13[pi], lz, 2.f * c - dd * spx[pi]));
        float nzv = fmaf(s13[pi], lxy, fmaf(s33[pi], lz, 2.f * q[r][4] - dd * spz[pi]));
        const int y = y0 + ry;
        if (x == a.src.x && y == a.src.y && z == a.src.z) {
          nxv += a.src.amp;
          nzv += a.src.amp;
        }
        if (valid[r]) {
          const long long i = (long long)z * d.plane + off[r];
          a.px[i] = dd * nxv;
          a.pz[i] = dd * nzv;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      // entering the next plane: if it starts a new 4-plane block of the same
      // column, the four planes of the block just finished become "damped cur"
      if (damp && ((z + 1) & 3) == 0 && z + 1 < d.nz) {
#pragma unroll
        for (int r = 0; r < RY; ++r) {
          // after the shift at z+1, entries 0..3 hold planes z-3..z; they are
          // entries 1..4 now
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) q[r][kk + 1] *= dxy[r] * a.dampz[z - 3 + kk];
        }
      }
    }
  }
}

// ------------------------------------------------------------ backward
struct BwdArgs {
  Dims3 d;
  Sched sc;
  const float* scz;  // cur sigma_z, lambda_z (queue initialisation)
  const float* lcz;
  float* spx;        // prev in / next out
  float* spz;
  float* lpx;
  float* lpz;
  float* g11;
  float* g13;
  float* g33;
  const float* dampx;
  const float* dampy;
  const float* dampz;
  float dt2, idx2, idy2, idz2;
  float sx, sy, sz;
  PointSource src;
  int* status;
};

constexpr int B_STAGES = 3;
// stage: [sigma_x halo][lambda_x halo][sz+4][lz+4][spx][spz][lpx][lpz][c11 c13 c33][g11 g13 g33]
constexpr int B_OFF_SH = 0;
constexpr int B_OFF_LH = HALO_BYTES;
constexpr int B_OFF_P = 2 * HALO_BYTES;  // 10 plain tiles from here
constexpr int B_STAGE_BYTES = B_OFF_P + 12 * PLAIN_BYTES;  // 32256
constexpr int B_SMEM = B_STAGES * B_STAGE_BYTES + 1024 + 2 * B_STAGES * 8;

struct BwdMaps {
  CUtensorMap scx, scz, spx, spz, lcx, lcz, lpx, lpz, c11, c13, c33, g11, g13, g33;
};

__global__ void __launch_bounds__(NTHREADS, 2)
    k_bwd3d_tma(const __grid_constant__ BwdMaps m, const BwdArgs a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem =
      (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + B_STAGES * B_STAGE_BYTES);
  uint64_t* empty = full + B_STAGES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < B_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const Dims3 d = a.d;

  if (warp == NCW) {  // ---------------- producer
    if (lane == 0) {
      long long k = 0;
      bool ok = true;
      for (int it = blockIdx.x; ok && it < a.sc.items; it += gridDim.x) {
        int bx, by, z0, z1;
        item(a.sc, it, bx, by, z0, z1);
        const int x0 = bx * TX, y0 = kHalo + by * TY;
        for (int z = z0; z < z1; ++z, ++k) {
          const int s = (int)(k % B_STAGES);
          if (k >= B_STAGES &&
              !mbar_wait(&empty[s], (uint32_t)(((k / B_STAGES) & 1) ^ 1), a.status)) {
            ok = false;
            break;
          }
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
          tma_load(pl + 6 * PLAIN_BYTES, &m.c11, &full[s], x0, y0, zp);
          tma_load(pl + 7 * PLAIN_BYTES, &m.c13, &full[s], x0, y0, zp);
          tma_load(pl + 8 * PLAIN_BYTES, &m.c33, &full[s], x0, y0, zp);
          tma_load(pl + 9 * PLAIN_BYTES, &m.g11, &full[s], x0, y0, zp);
          tma_load(pl + 10 * PLAIN_BYTES, &m.g13, &full[s], x0, y0, zp);
          tma_load(pl + 11 * PLAIN_BYTES, &m.g33, &full[s], x0, y0, zp);
        }
      }
    }
    return;
  }

  float sq[RY][9], lq[RY][9];
  float dxy[RY];
  int off[RY];
  bool valid[RY];
  long long k = 0;
  bool ok = true;
  for (int it = blockIdx.x; ok && it < a.sc.items; it += gridDim.x) {
    int bx, by, z0, z1;
    item(a.sc, it, bx, by, z0, z1);
    const int x = bx * TX + lane;
    const int y0 = kHalo + by * TY;
    // start the queues: planes z0-4 .. z0+3 from global
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const int y = y0 + warp * RY + r;
      valid[r] = x >= kHalo && x < d.nx - kHalo && y < d.ny - kHalo;
      off[r] = y * d.pitch + x;
      dxy[r] = valid[r] ? a.dampx[x] * a.dampy[y] : 1.f;
      sq[r][0] = lq[r][0] = 0.f;
#pragma unroll
      for (int kk = 1; kk < 9; ++kk) {
        const int zz = z0 - 5 + kk;
        const long long i = (long long)zz * d.plane + off[r];
        sq[r][kk] = valid[r] ? __ldg(a.scz + i) : 0.f;
        float v = valid[r] ? __ldg(a.lcz + i) : 0.f;
        if (zz >= 0 && (zz >> 2) < (z0 >> 2)) v *= dxy[r] * a.dampz[zz];
        lq[r][kk] = v;
      }
    }
    for (int z = z0; z < z1; ++z, ++k) {
      const int s = (int)(k % B_STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((k / B_STAGES) & 1), a.status)) {
        ok = false;
        break;
      }
      const unsigned char* st = smem + s * B_STAGE_BYTES;
      const float* sh = (const float*)(st + B_OFF_SH);
      const float* lh = (const float*)(st + B_OFF_LH);
      const float* pl = (const float*)(st + B_OFF_P);
      constexpr int T = TX * TY;
      const float dz = a.dampz[z];
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const int ry = warp * RY + r;
        const int pi = ry * TX + lane;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          sq[r][kk] = sq[r][kk + 1];
          lq[r][kk] = lq[r][kk + 1];
        }
        sq[r][8] = pl[0 * T + pi];
        lq[r][8] = pl[1 * T + pi];
        const float a11 = pl[6 * T + pi], a13 = pl[7 * T + pi], a33 = pl[8 * T + pi];
        const int sr = (ry + kHalo) * HX + lane + kHalo;
        const int y = y0 + ry;
        // source wavefield back one level (gradient form)
        const float sc = sh[sr];
        const float sxx = lap9(sc, sh[sr - 1], sh[sr + 1], sh[sr - 2], sh[sr + 2], sh[sr - 3],
                               sh[sr + 3], sh[sr - 4], sh[sr + 4]);
        const float syy = lap9(sc, sh[sr - HX], sh[sr + HX], sh[sr - 2 * HX], sh[sr + 2 * HX],
                               sh[sr - 3 * HX], sh[sr + 3 * HX], sh[sr - 4 * HX], sh[sr + 4 * HX]);
        const float szz = lap9(sq[r][4], sq[r][3], sq[r][5], sq[r][2], sq[r][6], sq[r][1],
                               sq[r][7], sq[r][0], sq[r][8]);
        const float sxy_u = fmaf(syy, a.idy2, sxx * a.idx2);
        const float sz_u = szz * a.idz2;
        float snx = fmaf(a.dt2, fmaf(a11, sxy_u, a13 * sz_u), 2.f * sc - pl[2 * T + pi]);
        float snz = fmaf(a.dt2, fmaf(a13, sxy_u, a33 * sz_u), 2.f * sq[r][4] - pl[3 * T + pi]);
        if (x == a.src.x && y == a.src.y && z == a.src.z) {
          snx += a.src.amp;
          snz += a.src.amp;
        }
        // imaging with the current adjoint
        const float lc = lh[sr];
        const float lz0 = lq[r][4];
        const float g11 = fmaf(lc, sxy_u, pl[9 * T + pi]);
        const float g33 = fmaf(lz0, sz_u, pl[11 * T + pi]);
        const float g13 = fmaf(lz0, sxy_u, fmaf(lc, sz_u, pl[10 * T + pi]));
        // adjoint, forward form with the sponge
        const float lxx = lap9(lc, lh[sr - 1], lh[sr + 1], lh[sr - 2], lh[sr + 2], lh[sr - 3],
                               lh[sr + 3], lh[sr - 4], lh[sr + 4]);
        const float lyy = lap9(lc, lh[sr - HX], lh[sr + HX], lh[sr - 2 * HX], lh[sr + 2 * HX],
                               lh[sr - 3 * HX], lh[sr + 3 * HX], lh[sr - 4 * HX], lh[sr + 4 * HX]);
        const float lzz = lap9(lz0, lq[r][3], lq[r][5], lq[r][2], lq[r][6], lq[r][1], lq[r][7],
                               lq[r][0], lq[r][8]);
        const float lxy = fmaf(lyy, a.sy, lxx * a.sx);
        const float lzs = lzz * a.sz;
        const float dd = dxy[r] * dz;
        const float lnx = fmaf(a11, lxy, fmaf(a13, lzs, 2.f * lc - dd * pl[4 * T + pi]));
        const float lnz = fmaf(a13, lxy, fmaf(a33, lzs, 2.f * lz0 - dd * pl[5 * T + pi]));
        if (valid[r]) {
          const long long i = (long long)z * d.plane + off[r];
          a.spx[i] = snx;
          a.spz[i] = snz;
          a.lpx[i] = dd * lnx;
          a.lpz[i] = dd * lnz;
          a.g11[i] = g11;
          a.g13[i] = g13;
          a.g33[i] = g33;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (((z + 1) & 3) == 0 && z + 1 < d.nz) {
#pragma unroll
        for (int r = 0; r < RY; ++r) {
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) lq[r][kk + 1] *= dxy[r] * a.dampz[z - 3 + kk];
        }
      }
    }
  }
}

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
Sched make_sched(vti_ctx* ctx, const Dims3& d, int ctas_per_sm) {
  constexpr long long kRestart = 4;
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

}  // namespace

int make_tile_maps(vti_ctx* ctx, const Dims3& d, const Vol& v, TileMaps* out) {
  auto fn = encode_fn();
  if (!fn) return fail(ctx, VTI_ERR_DEVICE, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)(d.nz + 2 * kZPad)};
  cuuint64_t strides[2] = {(cuuint64_t)d.pitch * 4, (cuuint64_t)d.plane * 4};
  cuuint32_t estr[3] = {1, 1, 1};
  cuuint32_t box_plain[3] = {TX, TY, 1};
  cuuint32_t box_halo[3] = {HX, HY, 1};
  CUresult r1 = fn((CUtensorMap*)out->plain, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, v.alloc, dims,
                   strides, box_plain, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = fn((CUtensorMap*)out->halo, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, v.alloc, dims,
                   strides, box_halo, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS)
    return fail(ctx, VTI_ERR_DEVICE, "cuTensorMapEncodeTiled failed");
  return VTI_OK;
}

static const CUtensorMap* P(const TileMaps& m) { return (const CUtensorMap*)m.plain; }
static const CUtensorMap* H(const TileMaps& m) { return (const CUtensorMap*)m.halo; }

int launch_fwd3d_tma(vti_ctx* ctx, const Dims3& d, const TileMaps& cx, const TileMaps& cz,
                     const TileMaps& px, const TileMaps& pz, const TileMaps& c11,
                     const TileMaps& c13, const TileMaps& c33, const float* cz_ptr,
                     float* px_ptr, float* pz_ptr, const Damping* damp, float sx, float sy,
                     float sz, PointSource src) {
  static bool attr[64] = {};  // the attribute is per device
  if (ctx->device >= 64 || !attr[ctx->device]) {
    VTI_CUDA(ctx, cudaFuncSetAttribute(k_fwd3d_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       F_SMEM));
    if (ctx->device < 64) attr[ctx->device] = true;
  }
  FwdArgs a;
  a.d = d;
  a.sc = make_sched(ctx, d, 3);
  a.cz = cz_ptr;
  a.px = px_ptr;
  a.pz = pz_ptr;
  a.dampx = damp ? damp->x : nullptr;
  a.dampy = damp ? damp->y : nullptr;
  a.dampz = damp ? damp->z : nullptr;
  a.sx = sx;
  a.sy = sy;
  a.sz = sz;
  a.src = src;
  a.status = ctx->d_status;
  const int grid = a.sc.grid;
  {
    LaunchTimer tm(ctx, kTimedFwd3d);
    k_fwd3d_tma<<<grid, NTHREADS, F_SMEM, ctx->stream>>>(*H(cx), *P(cz), *P(px), *P(pz), *P(c11),
                                                         *P(c13), *P(c33), a);
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
                     float idz2, float sx, float sy, float sz, PointSource src) {
  static bool attr[64] = {};
  if (ctx->device >= 64 || !attr[ctx->device]) {
    VTI_CUDA(ctx, cudaFuncSetAttribute(k_bwd3d_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       B_SMEM));
    if (ctx->device < 64) attr[ctx->device] = true;
  }
  BwdMaps m;
  m.scx = *H(scx); m.scz = *P(scz); m.spx = *P(spx); m.spz = *P(spz);
  m.lcx = *H(lcx); m.lcz = *P(lcz); m.lpx = *P(lpx); m.lpz = *P(lpz);
  m.c11 = *P(c11); m.c13 = *P(c13); m.c33 = *P(c33);
  m.g11 = *P(g11); m.g13 = *P(g13); m.g33 = *P(g33);
  BwdArgs a;
  a.d = d;
  a.sc = make_sched(ctx, d, 2);
  a.scz = scz_ptr; a.lcz = lcz_ptr;
  a.spx = spx_ptr; a.spz = spz_ptr; a.lpx = lpx_ptr; a.lpz = lpz_ptr;
  a.g11 = g11_ptr; a.g13 = g13_ptr; a.g33 = g33_ptr;
  a.dampx = damp.x; a.dampy = damp.y; a.dampz = damp.z;
  a.dt2 = dt2; a.idx2 = idx2; a.idy2 = idy2; a.idz2 = idz2;
  a.sx = sx; a.sy = sy; a.sz = sz;
  a.src = src;
  a.status = ctx->d_status;
  const int grid = a.sc.grid;
  {
    LaunchTimer tm(ctx, kTimedBwd3d);
    k_bwd3d_tma<<<grid, NTHREADS, B_SMEM, ctx->stream>>>(m, a);
  }
  VTI_LAUNCHED(ctx, "k_bwd3d_tma");
  return VTI_OK;
}

}  // namespace vti
