// TMA-pipeline building blocks shared by the 3D step kernels
// (vti_tma3d.cu: modeling / gradient steps, vti_gnhv3d.cu: Born and exact
// adjoint steps): tile geometry, the 8th-order stencil, mbarrier / TMA
// wrappers with bounded waits, the (column, z-segment) item schedule and the
// stage-ring prologue. Internal linkage: every including file gets its own
// copy.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "vti_internal.h"
#include "vti_pair.cuh"

namespace vti {

struct Sched {
  int gx, gy;  // columns in x, y
  int nz;
  int seg;     // planes per segment
  int items;   // gx * gy * ceil(nz / seg)
  int grid;    // persistent CTAs, min(items, resident slots)
};

namespace {

constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;

constexpr int TX = 32, TY = 16, RY = 2, NCW = TY / RY;  // consumer warps
constexpr int NTHREADS = (NCW + 1) * 32;
constexpr int HX = TX + 2 * kHalo, HY = TY + 2 * kHalo;
// BF16 halo tiles: x from x0-8 so the TMA x coordinate is 16-byte aligned
constexpr int HXB = TX + 16;
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

// lap9 of two adjacent points as packed FP32 pairs: each lane is rounded as
// the scalar lap9 (the same operation sequence).
__device__ __forceinline__ float2 lap9_2(float2 c, float2 m1, float2 p1, float2 m2, float2 p2,
                                         float2 m3, float2 p3, float2 m4, float2 p4) {
  float2 s = mul2(splat(kC0), c);
  s = fma2(splat(kC1), add2(m1, p1), s);
  s = fma2(splat(kC2), add2(m2, p2), s);
  s = fma2(splat(kC3), add2(m3, p3), s);
  s = fma2(splat(kC4), add2(m4, p4), s);
  return s;
}

// Two adjacent floats (8-byte aligned: x offsets are even, rows even-sized).
__device__ __forceinline__ float2 ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
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
// Release of a consumed stage by one consumer warp. The stage was read with
// ordinary shared-memory loads (generic proxy) and is refilled by TMA (async
// proxy) once the producer sees the release: each lane's proxy fence orders
// its reads before those writes, so no lane can read a row of the next
// plane's tile. Without the fence an unlucky half-warp read was observed to
// see the refill (about once per thousand backward launches of a 400^2 x 200
// grid).
__device__ __forceinline__ void stage_release(uint64_t* bar, int lane) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncwarp();
  if (lane == 0) mbar_arrive(bar);
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
// Bounded wait; false (and the status word set) if the phase never completes
// within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status,
                                          unsigned limit = kSpinLimit) {
  for (unsigned i = 0; i < limit; ++i)
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

// Kernel prologue shared by the step kernels: 1024-aligned stage ring and
// its full/empty mbarriers.
template <int kStages, int kStageBytes>
__device__ __forceinline__ unsigned char* ring_init(unsigned char* smem_raw, uint64_t*& full,
                                                    uint64_t*& empty) {
  unsigned char* smem =
      (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  full = (uint64_t*)(smem + kStages * kStageBytes);
  empty = full + kStages;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  return smem;
}

}  // namespace

// Segment schedule of one launch over d with `ctas_per_sm` resident CTAs per SM.
Sched make_sched(vti_ctx* ctx, const Dims3& d, int ctas_per_sm);
// cuTensorMapEncodeTiled from the driver (null if unavailable).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn();

}  // namespace vti
