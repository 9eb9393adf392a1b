// 2D VTI pseudo-acoustic forward modeling for sm_100a
// (lib/vti-fwi-2d: forwardCD kernels.cu:452-498, synthetic_f.cu:13-124,
// modeling_f.cu:10-82).
//
// Arrays are (nx+2npad) x (nz+2npad), x fastest, updated on [4, n-4) in both
// directions. p (sigma_h) carries the x stencil, q (sigma_v) the z stencil.
// The taper multiplies cur and next after every step (kernels.cu:304-315);
// stored values here are the once-tapered levels, prev is read as taper*prev.
//
// One fused kernel per time step: stencil + source + taper; receivers are
// recorded by a small gather kernel. The source amplitudes of all steps are
// uploaded once, so every step's launch differs only in its buffer pointers.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <utility>

#include <cooperative_groups.h>

#include "vti_internal.h"
#include "vti_pair.cuh"

namespace vti {
namespace {

// lib/vti-fwi-2d/kernels.h:4-8 (float literals)
constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;

constexpr int BX = 32, BZ = 8;

struct Step2d {
  int nnx, nnz;
  const float* p1;
  const float* q1;
  float* p0;
  float* q0;
  const float* c11;
  const float* c13;
  const float* c33;
  const float* taper;
  float idx2, idz2, dt2;
  int src;        // flat index of the source
  const float* amp;  // device pointer to the source amplitude of this step
};

// The operation sequence of one 2D update, written with explicit rounding
// (no contraction by the compiler), so that the per-level kernel and the
// resident kernel (scalar or packed pairs) compute bitwise the same values:
// lap = C0 c + C1 (m1 + p1) + ... (forwardCD, kernels.cu:452-498),
// next = dt2 (ca * lap_h * idx2 + cb * lap_v * idz2) + (2 cur - taper prev).
__device__ __forceinline__ float lap2d(float c, float m1, float p1, float m2, float p2, float m3,
                                       float p3, float m4, float p4) {
  float s = __fmul_rn(kC0, c);
  s = __fmaf_rn(kC1, __fadd_rn(m1, p1), s);
  s = __fmaf_rn(kC2, __fadd_rn(m2, p2), s);
  s = __fmaf_rn(kC3, __fadd_rn(m3, p3), s);
  s = __fmaf_rn(kC4, __fadd_rn(m4, p4), s);
  return s;
}
__device__ __forceinline__ float update2d(float dt2, float ca, float cb, float tp, float tq,
                                          float cur, float t, float prev) {
  return __fmaf_rn(dt2, __fmaf_rn(ca, tp, __fmul_rn(cb, tq)),
                   __fsub_rn(__fmul_rn(2.f, cur), __fmul_rn(t, prev)));
}

// Launched as a programmatic dependent launch: the model and taper (fixed for
// the whole run) are read before griddepcontrol.wait, which returns once the
// previous kernel of the stream (the step that wrote cur, or a recording) has
// completed and its writes are visible; prev, which that step read as its cur,
// is read and overwritten only after it. Launched normally, the wait returns
// at once.
__global__ void __launch_bounds__(BX* BZ) k_step2d(Step2d a) {
  __shared__ float sp[BZ][BX + 8];
  __shared__ float sq[BZ + 8][BX];
  const int tx = threadIdx.x, tz = threadIdx.y;
  const int ix = kHalo + blockIdx.x * BX + tx;
  const int iz = kHalo + blockIdx.y * BZ + tz;
  const bool valid = ix < a.nnx - kHalo && iz < a.nnz - kHalo;
  const int i = ix + iz * a.nnx;
  float t = 0.f, c11 = 0.f, c13 = 0.f, c33 = 0.f;
  if (valid) {
    t = __ldg(a.taper + i);
    c11 = __ldg(a.c11 + i);
    c13 = __ldg(a.c13 + i);
    c33 = __ldg(a.c33 + i);
  }
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  float p0 = 0.f, q0 = 0.f;
  if (valid) {
    p0 = a.p0[i];
    q0 = a.q0[i];
  }
  // stage p rows (x halo) and q columns (z halo); out-of-range lanes load 0
  auto ldp = [&](int x) { return (x < a.nnx && iz < a.nnz) ? a.p1[x + iz * a.nnx] : 0.f; };
  auto ldq = [&](int z) { return (ix < a.nnx && z < a.nnz) ? a.q1[ix + z * a.nnx] : 0.f; };
  sp[tz][tx + 4] = ldp(ix);
  if (tx < 4) {
    sp[tz][tx] = ldp(ix - 4);
    sp[tz][tx + BX + 4] = ldp(ix + BX);
  }
  sq[tz + 4][tx] = ldq(iz);
  if (tz < 4) {
    sq[tz][tx] = ldq(iz - 4);
    sq[tz + BZ + 4][tx] = ldq(iz + BZ);
  }
  __syncthreads();
  if (!valid) return;
  const float* r = &sp[tz][tx + 4];
  const float tp = __fmul_rn(lap2d(r[0], r[-1], r[1], r[-2], r[2], r[-3], r[3], r[-4], r[4]),
                             a.idx2);
  const float tq = __fmul_rn(lap2d(sq[tz + 4][tx], sq[tz + 3][tx], sq[tz + 5][tx],
                                   sq[tz + 2][tx], sq[tz + 6][tx], sq[tz + 1][tx],
                                   sq[tz + 7][tx], sq[tz][tx], sq[tz + 8][tx]),
                             a.idz2);
  float pn = update2d(a.dt2, c11, c13, tp, tq, r[0], t, p0);
  float qn = update2d(a.dt2, c13, c33, tp, tq, sq[tz + 4][tx], t, q0);
  if (i == a.src) {
    const float s = *a.amp;
    pn = __fadd_rn(pn, s);
    qn = __fadd_rn(qn, s);
  }
  a.p0[i] = __fmul_rn(t, pn);
  a.q0[i] = __fmul_rn(t, qn);
}

// recordData (kernels.cu:317-324): 0.5(p+q) at receivers into row `row`.
__global__ void k_record2d(float* data, long long row_off, const float* p, const float* q,
                           const int* ridx, int nr) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    int i = ridx[ir];
    data[row_off + ir] = 0.5f * (p[i] + q[i]);
  }
}

// injectSource + abc(p1,q1) at t=1 (synthetic_f.cu:86-89).
__global__ void k_init2d(float* p, float* q, int src, float value, float taper_at_src) {
  p[src] = value * taper_at_src;
  q[src] = value * taper_at_src;
}

// ---------------------------------------------------------------- resident
// The whole 2D state of one shot held in the shared memory of one thread-block
// cluster for all time steps (one cluster per shot, blockIdx.x / cluster size
// picks the shot; any number of shots per launch). CTA r of the cluster owns
// update rows z in [4 + r*R, 4 + r*R + nr) and keeps, in rows of W floats
// (W = nnx rounded up to even), p at two levels (R rows each), q at two
// levels with 4 halo rows above and below (R + 8 rows each), and the taper
// and c13 of its rows. Every step each point is updated exactly as in
// k_step2d (same operations in the same order), the new q of the first and
// last 4 owned rows is also stored into the neighbours' halo rows (distributed
// shared memory), and one cluster barrier closes the step. Thread t < S*NP
// (NP = ceil(X/2) column pairs of the X = nnx - 8 update columns, S =
// blockDim / NP segments) owns the columns x0 = 4 + 2*(t % NP) and x0 + 1
// (when x0 + 1 < nnx - 4) over up to kResRows consecutive rows of its CTA:
// 64-bit shared loads serve both columns, c11 and c33 stay in registers, q's z
// stencil runs as a register queue, and the arithmetic of the two columns
// runs on packed FP32 pairs (except the x stencil, whose neighbour pairs
// straddle the loaded float2s).
constexpr int kResThreads = 512, kResRows = 8, kResMaxCluster = 16;

struct Res2d {
  int nnx, nnz, nt;
  int W;             // shared-memory row stride (floats, even)
  int rows_per_cta;  // R
  int seg_rows;      // rows per thread segment
  int segs;          // S
  const float* c11;
  const float* c13;
  const float* c33;
  const float* taper;
  float idx2, idz2, dt2;
  float init_value;     // dt2 * wavelet[0], level 1 at the source before the taper
  const float* amp;     // amp[it]: source term of level it
  const int* rec_row;   // trace row recorded at level it, -1 none
  const int* shots;     // per shot (cluster): source x, source z, first receiver, receivers
  const int* rx;        // receiver columns and rows (all receivers of the survey)
  const int* rz;
  int nr_total;
  float* data;          // rows x nr_total, receiver-fastest
};

// 32-bit shared::cluster address of `p` (this CTA's shared memory) in the
// shared memory of cluster CTA `rank`, and stores there.
__device__ __forceinline__ uint32_t cluster_addr(const float* p, int rank) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster2(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y)
               : "memory");
}

// Receivers of this shot in the CTA's rows: 0.5 (p + q) into trace row
// `row` (recordData, kernels.cu:317-324); the CTA owning row 4 also writes 0
// for receivers outside the update region (never updated, so 0 there), so
// every receiver of the shot is written in every recorded row.
__device__ __forceinline__ void res_record(const Res2d& a, int row, const float* p, const float* q,
                                           int zr0, int nr, int ir0, int nri) {
  for (int ir = threadIdx.x; ir < nri; ir += blockDim.x) {
    const int x = __ldg(a.rx + ir0 + ir), z = __ldg(a.rz + ir0 + ir), lz = z - zr0;
    const bool inside = x >= kHalo && x < a.nnx - kHalo && z >= kHalo && z < a.nnz - kHalo;
    float* d = a.data + (long long)row * a.nr_total + ir0 + ir;
    if (inside && lz >= 0 && lz < nr)
      *d = 0.5f * (p[lz * a.W + x] + q[(lz + 4) * a.W + x]);
    else if (!inside && zr0 == kHalo)
      *d = 0.f;
  }
}

// One thread's rows of one level (k_synth2d_resident).
struct ResRows {
  const float* Pc;  // cur p, q (q rows -4 .. nr+3), next p, q, taper, c13: at column x
  const float* Qc;
  float* Pn;
  float* Qn;
  const float* Tr;
  const float* Cr;
  uint32_t up, dn;  // the neighbours' next-q slots at column x (shared::cluster)
  int W, r0, cnt, nr, R;
  bool to_up, to_dn, two;
  int src_row, src_e;
  float amp;
};

template <bool kFull>
__device__ __forceinline__ void res_rows(const Res2d& a, const ResRows& rr,
                                         const float2 (&m11)[kResRows],
                                         const float2 (&m33)[kResRows]) {
  const int W = rr.W;
  float2 qz[9];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    qz[k + 1] = *reinterpret_cast<const float2*>(rr.Qc + (rr.r0 - 4 + k) * W);
#pragma unroll
  for (int j = 0; j < kResRows; ++j) {
    if (kFull || j < rr.cnt) {
      const int lr = rr.r0 + j;
#pragma unroll
      for (int k = 0; k < 8; ++k) qz[k] = qz[k + 1];
      qz[8] = *reinterpret_cast<const float2*>(rr.Qc + (lr + 4) * W);
      const float* pr = rr.Pc + lr * W;
      float v[10];
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const float2 u = *reinterpret_cast<const float2*>(pr - 4 + 2 * k);
        v[2 * k] = u.x;
        v[2 * k + 1] = u.y;
      }
      const int o = lr * W;
      const float2 pp = *reinterpret_cast<const float2*>(rr.Pn + o);
      const float2 qp = *reinterpret_cast<const float2*>(rr.Qn + o);
      const float2 tt = *reinterpret_cast<const float2*>(rr.Tr + o);
      const float2 cc = *reinterpret_cast<const float2*>(rr.Cr + o);
      // the sequence of lap2d / update2d on packed pairs; the x stencil per
      // lane (its neighbour pairs straddle the loaded float2s)
      float2 tp2 = make_float2(lap2d(v[4], v[3], v[5], v[2], v[6], v[1], v[7], v[0], v[8]),
                               lap2d(v[5], v[4], v[6], v[3], v[7], v[2], v[8], v[1], v[9]));
      float2 tq2 = mul2(splat(kC0), qz[4]);
      tq2 = fma2(splat(kC1), add2(qz[3], qz[5]), tq2);
      tq2 = fma2(splat(kC2), add2(qz[2], qz[6]), tq2);
      tq2 = fma2(splat(kC3), add2(qz[1], qz[7]), tq2);
      tq2 = fma2(splat(kC4), add2(qz[0], qz[8]), tq2);
      tp2 = mul2(tp2, splat(a.idx2));
      tq2 = mul2(tq2, splat(a.idz2));
      const float2 dt2 = splat(a.dt2), two = splat(2.f);
      float2 a2 = fma2(dt2, fma2(m11[j], tp2, mul2(cc, tq2)),
                       sub2(mul2(two, make_float2(v[4], v[5])), mul2(tt, pp)));
      float2 b2 = fma2(dt2, fma2(cc, tp2, mul2(m33[j], tq2)), sub2(mul2(two, qz[4]), mul2(tt, qp)));
      if (lr == rr.src_row) {
        if (rr.src_e == 0) {
          a2.x = __fadd_rn(a2.x, rr.amp);
          b2.x = __fadd_rn(b2.x, rr.amp);
        } else {
          a2.y = __fadd_rn(a2.y, rr.amp);
          b2.y = __fadd_rn(b2.y, rr.amp);
        }
      }
      const float2 p2 = mul2(tt, a2);
      const float2 q2 = mul2(tt, b2);
      const float pn[2] = {p2.x, p2.y}, qn[2] = {q2.x, q2.y};
      // halo rows of the neighbours: my first 4 rows are the bottom halo of
      // rank - 1 (which owns R rows), my last 4 the top halo of rank + 1
      const bool to_up = rr.to_up && lr < 4;
      const bool to_dn = rr.to_dn && lr >= rr.nr - 4;
      const uint32_t ua = rr.up + 4u * (uint32_t)((rr.R + 4 + lr) * W);
      const uint32_t da = rr.dn + 4u * (uint32_t)((lr - rr.nr + 4) * W);
      if (rr.two) {
        *reinterpret_cast<float2*>(rr.Pn + o) = make_float2(pn[0], pn[1]);
        *reinterpret_cast<float2*>(rr.Qn + o) = q2;
        if (to_up) st_cluster2(ua, q2);
        if (to_dn) st_cluster2(da, q2);
      } else {
        rr.Pn[o] = pn[0];
        rr.Qn[o] = qn[0];
        if (to_up) st_cluster(ua, qn[0]);
        if (to_dn) st_cluster(da, qn[0]);
      }
    }
  }
}

__global__ void __launch_bounds__(kResThreads, 1)
    k_synth2d_resident(const __grid_constant__ Res2d a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) float sm[];
  const int rank = (int)cl.block_rank();
  const int ncta = (int)cl.num_blocks();
  const int nnx = a.nnx, W = a.W;
  // this cluster's shot
  const int shot = blockIdx.x / ncta;
  const int src_x = __ldg(a.shots + 4 * shot), src_z = __ldg(a.shots + 4 * shot + 1);
  const int ir0 = __ldg(a.shots + 4 * shot + 2), nri = __ldg(a.shots + 4 * shot + 3);
  const int R = a.rows_per_cta;
  const int zr0 = kHalo + rank * R;
  const int nr = min(R, a.nnz - 2 * kHalo - rank * R);
  // float offsets of the slots in sm
  const int oP0 = 0, oP1 = R * W, oQ0 = 2 * R * W, oQ1 = oQ0 + (R + 8) * W;
  const int oT = oQ1 + (R + 8) * W, oM13 = oT + R * W;
  for (int i = threadIdx.x; i < oT; i += blockDim.x) sm[i] = 0.f;
  for (int i = threadIdx.x; i < nr * nnx; i += blockDim.x) {
    const int row = i / nnx, col = i - row * nnx;
    sm[oT + row * W + col] = __ldg(a.taper + zr0 * nnx + i);
    sm[oM13 + row * W + col] = __ldg(a.c13 + zr0 * nnx + i);
  }
  __syncthreads();
  // level 1 (slot 1): the source after the taper (synthetic_f.cu:86-89); every
  // CTA writes its own copy, halo rows included
  if (threadIdx.x == 0) {
    const float v = a.init_value * __ldg(a.taper + src_x + src_z * nnx);
    const int lz = src_z - zr0;
    if (lz >= 0 && lz < nr) sm[oP1 + lz * W + src_x] = v;
    if (lz >= -4 && lz < nr + 4) sm[oQ1 + (lz + 4) * W + src_x] = v;
  }
  // this thread's column pair and rows
  const int NP = (nnx - 2 * kHalo + 1) / 2;
  const int t = threadIdx.x;
  const bool active = t < a.segs * NP;
  const int seg = active ? t / NP : 0;
  const int x = kHalo + 2 * (active ? t % NP : 0);
  const bool two = x + 1 < nnx - kHalo;  // the second column is updated
  const int r0 = seg * a.seg_rows;
  const int cnt = active ? max(0, min(a.seg_rows, nr - r0)) : 0;
  const int src_e = src_x - x;  // 0 or 1 when the source is in this thread's columns
  const bool src_mine = cnt > 0 && (src_e == 0 || (src_e == 1 && two)) &&
                        src_z >= zr0 + r0 && src_z < zr0 + r0 + cnt;
  const int src_row = src_mine ? src_z - zr0 : -1;  // owned row of the source
  // c11 and c33 of the thread's rows
  float2 m11[kResRows], m33[kResRows];
#pragma unroll
  for (int j = 0; j < kResRows; ++j) {
    const int i = x + (zr0 + r0 + j) * nnx;
    const bool v = j < cnt;
    m11[j] = make_float2(v ? __ldg(a.c11 + i) : 0.f, v && two ? __ldg(a.c11 + i + 1) : 0.f);
    m33[j] = make_float2(v ? __ldg(a.c33 + i) : 0.f, v && two ? __ldg(a.c33 + i + 1) : 0.f);
  }
  // Q slot 0 of the CTA above (rank - 1) and below (rank + 1); slot 1 lies
  // qslot bytes further
  const uint32_t up0 = rank > 0 ? cluster_addr(sm + oQ0, rank - 1) : 0u;
  const uint32_t dn0 = rank + 1 < ncta ? cluster_addr(sm + oQ0, rank + 1) : 0u;
  const uint32_t qslot = (uint32_t)((oQ1 - oQ0) * sizeof(float));
  // every CTA of the cluster is running and initialised before any remote store
  cl.sync();
  if (a.nt > 1 && __ldg(a.rec_row + 1) >= 0)
    res_record(a, __ldg(a.rec_row + 1), sm + oP1, sm + oQ1, zr0, nr, ir0, nri);
  int cur = 1;
  float amp_next = a.nt > 2 ? __ldg(a.amp + 2) : 0.f;
  for (int it = 2; it < a.nt; ++it) {
    const int nxt = cur ^ 1;
    const float amp = amp_next;
    if (it + 1 < a.nt) amp_next = __ldg(a.amp + it + 1);
    if (cnt > 0) {
      ResRows rr;
      rr.Pc = sm + (cur ? oP1 : oP0) + x;
      rr.Qc = sm + (cur ? oQ1 : oQ0) + 4 * W + x;  // row = owned row, -4 .. nr+3
      rr.Pn = sm + (nxt ? oP1 : oP0) + x;
      rr.Qn = sm + (nxt ? oQ1 : oQ0) + 4 * W + x;
      rr.Tr = sm + oT + x;
      rr.Cr = sm + oM13 + x;
      rr.up = up0 + (nxt ? qslot : 0u) + 4u * (uint32_t)x;
      rr.dn = dn0 + (nxt ? qslot : 0u) + 4u * (uint32_t)x;
      rr.W = W;
      rr.r0 = r0;
      rr.cnt = cnt;
      rr.nr = nr;
      rr.R = R;
      rr.to_up = rank > 0;
      rr.to_dn = rank + 1 < ncta;
      rr.two = two;
      rr.src_row = src_row;
      rr.src_e = src_e;
      rr.amp = amp;
      // threads with a full segment run the rows without per-row guards
      if (cnt == kResRows)
        res_rows<true>(a, rr, m11, m33);
      else
        res_rows<false>(a, rr, m11, m33);
    }
    cl.sync();
    const int row = __ldg(a.rec_row + it);
    if (row >= 0)
      res_record(a, row, sm + (nxt ? oP1 : oP0), sm + (nxt ? oQ1 : oQ0), zr0, nr, ir0, nri);
    cur = nxt;
  }
  // no CTA leaves while a neighbour may still read its memory
  cl.sync();
}

struct Dev2d {
  float* buf = nullptr;  // c11 c13 c33 taper p0 q0 p1 q1 amps
  size_t n = 0;
};

// Cluster shape of the resident path for an nnx x nnz grid: the largest
// cluster (most SMs) whose CTAs each own >= 4 rows, whose threads each own
// <= kResRows rows of one column pair, whose shared memory fits one CTA and
// which the device can schedule. false: the grid does not fit one cluster.
struct ResShape {
  int ctas = 0, rows = 0, segs = 0, seg_rows = 0, W = 0;
  size_t smem = 0;
};
bool attr_res[64] = {};
std::mutex attr_res_mu;  // first calls from several threads set the attributes once

bool resident_shape(vti_ctx* ctx, int nnx, int nnz, ResShape* out) {
  constexpr size_t kMaxSmem = 227 * 1024;
  const int NP = (nnx - 2 * kHalo + 1) / 2, rows = nnz - 2 * kHalo;
  const int W = (nnx + 1) & ~1;
  if (NP < 1 || rows < 4 || NP > kResThreads) return false;
  if (ctx->device < 0 || ctx->device >= 64) return false;
  std::lock_guard<std::mutex> lk(attr_res_mu);
  if (!attr_res[ctx->device]) {
    if (cudaFuncSetAttribute(k_synth2d_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMaxSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_synth2d_resident,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    attr_res[ctx->device] = true;
  }
  const int S = kResThreads / NP;
  for (int C = kResMaxCluster; C >= 1; --C) {
    const int R = (rows + C - 1) / C;
    const int last = rows - (C - 1) * R;
    if (R < 4 || last < 4) continue;
    const int RS = (R + S - 1) / S;
    const size_t smem = (size_t)(6 * R + 16) * W * sizeof(float);
    if (RS > kResRows || smem > kMaxSmem) return false;  // fewer CTAs only need more
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kResThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_synth2d_resident, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (nclusters < 1) continue;
    *out = ResShape{C, R, S, RS, W, smem};
    return true;
  }
  return false;
}

// One cluster of sh.ctas CTAs per shot; clusters that do not fit at once run
// as earlier ones finish (no cluster waits for another).
cudaError_t launch_resident(const ResShape& sh, const Res2d& a, int nshots,
                            cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sh.ctas * nshots);
  cfg.blockDim = dim3(kResThreads);
  cfg.dynamicSmemBytes = sh.smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = sh.ctas;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_synth2d_resident, a);
}

}  // namespace
}  // namespace vti

using namespace vti;

namespace {

#define VTI_TRY_RES(call)            \
  do {                               \
    const int st_ = (call);          \
    if (st_ != VTI_OK) return st_;   \
  } while (0)

// The context's 2D scratch, grown (never shrunk) to `bytes`; freed with the
// context.
int scratch2d(vti_ctx* ctx, size_t bytes, float** out) {
  if (ctx->scratch2d_bytes < bytes) {
    if (ctx->scratch2d) {
      VTI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      cudaFree(ctx->scratch2d);
      ctx->scratch2d = nullptr;
      ctx->scratch2d_bytes = 0;
    }
    VTI_CUDA(ctx, cudaMalloc((void**)&ctx->scratch2d, bytes));
    ctx->scratch2d_bytes = bytes;
  }
  *out = ctx->scratch2d;
  return VTI_OK;
}

int run2d(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13, const float* c33,
          const float* wavelet, const float* taper, int slocxz, const int* rloc, int nri,
          int nr_total, int ir0, float* out, int mode) {
  if (!ctx || !g || !c11 || !c13 || !c33 || !wavelet || !taper || !out) return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 2 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  if (slocxz < 0 || slocxz >= nnxz) return fail(ctx, VTI_ERR_ARG, "2D source outside the grid");
  const float dt = g->dt, dt2 = dt * dt;
  const float dx2 = g->dx * g->dx, dz2 = g->dz * g->dz;
  const int ratio = mode == 0 ? (int)(g->rate / dt + 0.5f) : (int)std::round(g->rate / dt);
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  // trace row (or snapshot) taken at each level, -1 none (synthetic_f.cu:95-110)
  std::vector<int> rec_row(g->nt, -1);
  if (ratio == 1 && g->ot == 0.f) rec_row[1] = 1;
  for (int it = 2; it < g->nt; ++it) {
    float t = it * dt + g->ot;
    if (t >= 0.f && (it - ntNeg) % ratio == 0) rec_row[it] = (it - ntNeg) / ratio;
  }
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  // device buffers (the context's 2D scratch, kept between calls): 4
  // model/taper + 4 wavefields + nt amplitudes, then the flat receiver
  // indices, then the output rows
  const long long nrows_out = mode == 0 ? (g->nt - ntNeg - 1) / ratio + 1 : 0;
  if (mode == 0 && nrows_out < 1)
    return fail(ctx, VTI_ERR_ARG, "the whole record lies before time zero (|ot| too large)");
  const int nrec = mode == 0 ? std::max(nri, 0) : 0;
  const size_t nbuf = 8 * (size_t)nnxz + g->nt;
  const size_t n_ints = (size_t)nrec;
  const size_t n_data = (size_t)nrows_out * nrec;
  float* buf = nullptr;
  {
    const int sst = scratch2d(ctx, (nbuf + n_ints + n_data) * sizeof(float), &buf);
    if (sst != VTI_OK) return sst;
  }
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float* w[4] = {dtap + nnxz, dtap + 2 * nnxz, dtap + 3 * nnxz, dtap + 4 * nnxz};
  float* amps = dtap + 5 * nnxz;
  int* d_ridx = reinterpret_cast<int*>(buf + nbuf);
  float* d_data = nrec > 0 ? buf + nbuf + n_ints : nullptr;
  int st = VTI_OK;
  auto cleanup = [&]() { cudaStreamSynchronize(ctx->stream); };
#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) {                      \
      st = cuda_check(ctx, e_, #call);            \
      cleanup();                                  \
      return st;                                  \
    }                                             \
  } while (0)
  CK(cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(w[0], 0, 4 * nnxz * 4, ctx->stream));
  std::vector<float> h_amp(g->nt, 0.f);
  for (int it = 2; it < g->nt; ++it)
    h_amp[it] = mode == 0 ? dt2 * wavelet[it - 1] : wavelet[it - 1];  // modeling_f.cu:66
  CK(cudaMemcpyAsync(amps, h_amp.data(), g->nt * 4, cudaMemcpyHostToDevice, ctx->stream));
  std::vector<int> ridx;
  if (mode == 0 && nri > 0) {
    ridx.resize(nri);
    for (int ir = 0; ir < nri; ++ir) {
      int x = rloc[2 * (ir0 + ir)], z = rloc[2 * (ir0 + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz) {
        cleanup();
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
      }
      ridx[ir] = x + z * nnx;
    }
    CK(cudaMemsetAsync(d_data, 0, (size_t)nrows_out * nri * sizeof(float), ctx->stream));
  }
  if (nrec > 0)
    CK(cudaMemcpyAsync(d_ridx, ridx.data(), nri * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream));
  // time level 1: source then taper (synthetic_f.cu:86-89)
  k_init2d<<<1, 1, 0, ctx->stream>>>(w[2], w[3], slocxz, dt2 * wavelet[0], taper[slocxz]);
  ctx->launches++;
  float *p1 = w[2], *q1 = w[3], *p0 = w[0], *q0 = w[1];
  auto snapshot = [&](long long row, const float* p, const float* q) -> int {
    if (mode == 0) {
      if (nri > 0) {
        cudaError_t e = launch_pdl(k_record2d, dim3((nri + 127) / 128), dim3(128), ctx->stream,
                                   d_data, row * nri, p, q, (const int*)d_ridx, nri);
        if (e != cudaSuccess) return cuda_check(ctx, e, "k_record2d launch");
        ctx->launches++;
      }
    } else {
      cudaError_t e = cudaMemcpyAsync(out + row * nnxz, p, nnxz * 4, cudaMemcpyDeviceToHost,
                                      ctx->stream);
      if (e != cudaSuccess) return cuda_check(ctx, e, "snapshot copy");
    }
    return VTI_OK;
  };
  if (rec_row[1] >= 0) {
    st = snapshot(rec_row[1], p1, q1);
    if (st != VTI_OK) {
      cleanup();
      return st;
    }
  }
  dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  // The trace-recording time loop (every node a kernel) is captured as one
  // CUDA graph: a 2D step is a few microseconds of work, so per-launch
  // overhead is most of its cost. With per-kernel timing on, or snapshots
  // copied to the host (modeling), the launches are issued directly.
  const bool use_graph = mode == 0 && !ctx->timing;
  cudaGraph_t graph = nullptr;
  if (use_graph) CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  for (int it = 2; it < g->nt; ++it) {
    Step2d a{nnx, nnz, p1, q1, p0, q0, dc11, dc13, dc33, dtap, 1.f / dx2, 1.f / dz2, dt2,
             slocxz, amps + it};
    {
      LaunchTimer tm(ctx, kTimedStep2d);
      const cudaError_t e = launch_pdl(k_step2d, grid, block, ctx->stream, a);
      st = e == cudaSuccess ? VTI_OK : cuda_check(ctx, e, "k_step2d launch");
    }
    ctx->launches++;
    if (st == VTI_OK && rec_row[it] >= 0) st = snapshot(rec_row[it], p0, q0);
    if (st != VTI_OK) {
      if (use_graph) {
        cudaStreamEndCapture(ctx->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
      }
      cleanup();
      return st;
    }
    std::swap(p0, p1);
    std::swap(q0, q1);
  }
  if (use_graph) {
    CK(cudaStreamEndCapture(ctx->stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(ei);
    const cudaError_t el = cudaGraphLaunch(exec, ctx->stream);
    cudaGraphExecDestroy(exec);  // released once the launch completes
    CK(el);
  }
  CK(cudaGetLastError());
  if (mode == 0 && nri > 0) {
    // scatter rows into the caller's receiver-fastest layout
    CK(cudaMemcpy2DAsync(out + ir0, (size_t)nr_total * 4, d_data, (size_t)nri * 4,
                         (size_t)nri * 4, nrows_out, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  cleanup();
#undef CK
  return VTI_OK;
}

// Traces of all shots of a grid that fits one thread-block cluster
// (resident_shape) with every source in the update region: the model is
// uploaded once and each shot runs in its own cluster of k_synth2d_resident
// (all levels in shared memory). Shots whose receiver ranges are disjoint
// share one launch; otherwise one launch per shot, in shot order, so a later
// shot overwrites the receivers it shares with an earlier one (the per-shot
// order of synthetic_f.cu:31-124). VTI_ERR_UNSUPPORTED: not eligible, the
// caller runs the per-level path (nothing was computed).
int synth2d_resident(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                     const float* c33, const float* wavelet, const int* sloc, int ns,
                     const int* rloc, int nr_total, const float* taper, float* out) {
  if (!ctx->resident2d || ns < 1) return VTI_ERR_UNSUPPORTED;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 2 || !(g->dt > 0) || !(g->rate > 0))
    return VTI_ERR_UNSUPPORTED;
  for (int is = 0; is < ns; ++is) {
    const int* sh = sloc + 4 * is;
    if (sh[0] < kHalo || sh[0] >= nnx - kHalo || sh[1] < kHalo || sh[1] >= nnz - kHalo)
      return VTI_ERR_UNSUPPORTED;
  }
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5f);
  if (ratio < 1) return VTI_ERR_UNSUPPORTED;
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  ResShape shape;
  if (!resident_shape(ctx, nnx, nnz, &shape)) return VTI_ERR_UNSUPPORTED;
  for (int ir = 0; ir < nr_total; ++ir) {
    const int x = rloc[2 * ir], z = rloc[2 * ir + 1];
    if (x < 0 || x >= nnx || z < 0 || z >= nnz)
      return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
  }
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  // trace row taken at each level, -1 none (the arithmetic of run2d)
  std::vector<int> hi(g->nt, -1);
  if (ratio == 1 && g->ot == 0.f) hi[1] = 1;
  for (int it = 2; it < g->nt; ++it) {
    float t = it * dt + g->ot;
    if (t >= 0.f && (it - ntNeg) % ratio == 0) hi[it] = (it - ntNeg) / ratio;
  }
  const long long nrows = (g->nt - ntNeg - 1) / ratio + 1;
  if (nrows < 1)
    return fail(ctx, VTI_ERR_ARG, "the whole record lies before time zero (|ot| too large)");
  // ints: trace rows, per-shot table, receiver columns, receiver rows
  for (int is = 0; is < ns; ++is) {
    const int* sh = sloc + 4 * is;
    hi.push_back(sh[0]);
    hi.push_back(sh[1]);
    hi.push_back(sh[3]);
    hi.push_back(sh[2]);
  }
  for (int ir = 0; ir < nr_total; ++ir) hi.push_back(rloc[2 * ir]);
  for (int ir = 0; ir < nr_total; ++ir) hi.push_back(rloc[2 * ir + 1]);
  const size_t nf = 4 * (size_t)nnxz + g->nt;
  const size_t n_data = (size_t)nrows * nr_total;
  float* buf = nullptr;
  VTI_TRY_RES(scratch2d(ctx, (nf + hi.size() + n_data) * sizeof(float), &buf));
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float* amps = dtap + nnxz;
  int* d_ints = reinterpret_cast<int*>(buf + nf);
  float* d_data = buf + nf + hi.size();
  cudaStream_t s = ctx->stream;
  VTI_CUDA(ctx, cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, s));
  std::vector<float> h_amp(g->nt, 0.f);
  for (int it = 2; it < g->nt; ++it) h_amp[it] = dt2 * wavelet[it - 1];
  VTI_CUDA(ctx, cudaMemcpyAsync(amps, h_amp.data(), g->nt * 4, cudaMemcpyHostToDevice, s));
  VTI_CUDA(ctx, cudaMemcpyAsync(d_ints, hi.data(), hi.size() * sizeof(int),
                                cudaMemcpyHostToDevice, s));
  if (n_data) VTI_CUDA(ctx, cudaMemsetAsync(d_data, 0, n_data * sizeof(float), s));
  // receiver ranges pairwise disjoint?
  std::vector<std::pair<int, int>> rng;
  for (int is = 0; is < ns; ++is)
    if (sloc[4 * is + 2] > 0) rng.push_back({sloc[4 * is + 3], sloc[4 * is + 3] + sloc[4 * is + 2]});
  std::sort(rng.begin(), rng.end());
  bool disjoint = true;
  for (size_t k = 1; k < rng.size(); ++k)
    if (rng[k].first < rng[k - 1].second) disjoint = false;
  const float dx2 = g->dx * g->dx, dz2 = g->dz * g->dz;
  Res2d a{nnx, nnz, g->nt, shape.W, shape.rows, shape.seg_rows, shape.segs, dc11, dc13, dc33,
          dtap, 1.f / dx2, 1.f / dz2, dt2, dt2 * wavelet[0], amps, d_ints, d_ints + g->nt,
          d_ints + g->nt + 4 * ns, d_ints + g->nt + 4 * ns + nr_total, nr_total, d_data};
  {
    LaunchTimer tm(ctx, kTimedStep2d);
    if (disjoint) {
      VTI_CUDA(ctx, launch_resident(shape, a, ns, s));
      ctx->launches++;
    } else {
      for (int is = 0; is < ns; ++is) {
        Res2d b = a;
        b.shots = a.shots + 4 * is;
        VTI_CUDA(ctx, launch_resident(shape, b, 1, s));
        ctx->launches++;
      }
    }
  }
  VTI_CUDA(ctx, cudaGetLastError());
  // each shot's receiver columns into the caller's receiver-fastest rows
  for (int is = 0; is < ns; ++is) {
    const int nri = sloc[4 * is + 2], ir0 = sloc[4 * is + 3];
    if (nri > 0)
      VTI_CUDA(ctx, cudaMemcpy2DAsync(out + ir0, (size_t)nr_total * 4, d_data + ir0,
                                      (size_t)nr_total * 4, (size_t)nri * 4, nrows,
                                      cudaMemcpyDeviceToHost, s));
  }
  VTI_CUDA(ctx, cudaStreamSynchronize(s));
  return VTI_OK;
}

}  // namespace

extern "C" {

int vti2d_synthetic(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                    const float* c33, const float* wavelet, const int* sloc, int ns,
                    const int* rloc, int nr, const float* taper, float* data) {
  if (!ctx || !g || !sloc || (nr > 0 && !rloc)) return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
  }
  if (!c11 || !c13 || !c33 || !wavelet || !taper || !data) return VTI_ERR_ARG;
  VTI_TRY_RES(check_cfl2d(ctx, g, c11, c13, c33));
  const int rst = synth2d_resident(ctx, g, c11, c13, c33, wavelet, sloc, ns, rloc, nr, taper,
                                   data);
  if (rst != VTI_ERR_UNSUPPORTED) return rst;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    int st = run2d(ctx, g, c11, c13, c33, wavelet, taper, s[0] + s[1] * nnx, rloc, s[2], nr, s[3],
                   data, 0);
    if (st != VTI_OK) return st;
  }
  return VTI_OK;
}

int vti2d_modeling(vti_ctx* ctx, const vti2d_geom* g, const float* c11, const float* c13,
                   const float* c33, const float* wavelet, int slocxz, const float* taper,
                   float* wavefield) {
  if (ctx && g && c11 && c13 && c33) VTI_TRY_RES(check_cfl2d(ctx, g, c11, c13, c33));
  return run2d(ctx, g, c11, c13, c33, wavelet, taper, slocxz, nullptr, 0, 0, 0, wavefield, 1);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free synthetic traces.
//
// vti2d_synthetic_noalloc() computes what vti2d_synthetic() computes (same
// kernels, same launch order, same host arithmetic) but never allocates
// device memory: the model, the four wavefields, the source amplitudes, the
// receiver indices and the trace rows of one shot all live in one file-scope
// static device array of kNoAllocFloats floats (40 MiB), reserved once when
// this module is loaded.
//
// Who needs it: callers that must not allocate inside a call. cudaMalloc and
// cudaFree synchronise the whole device, so a caller that keeps other streams
// busy (a 3D gradient running beside 2D modeling, say) would see them stall
// at every call; a long-running job that shares the GPU can find cudaMalloc
// failing for lack of memory hours after start-up, while a static
// reservation either exists from the first call on or never; and hosts that
// give the library a fixed memory budget forbid allocations inside calls.
//
// Limits and rules:
//  * need = 8*nnx*nnz + nt + nri + rows*nri floats (rows =
//    (nt-ntNeg-1)/ratio + 1, nri the largest shot's receiver count); a call
//    that needs more than kNoAllocFloats is rejected with VTI_ERR_ARG before
//    any work is queued. A 1000 x 1000 padded grid with nt = 4000 and 1000
//    receivers per shot sampled every 4 steps fits.
//  * The first call on a device (that device current) looks up the array's
//    address with cudaGetSymbolAddress and caches it; make that first call
//    before any stream capture begins.
//  * The wavefields and the trace rows must start at zero for every shot;
//    they are cleared with cudaMemsetAsync on the context stream (the model,
//    amplitudes and receiver indices are overwritten by copies).
//  * There is one array per device and process: calls that overlap in time on
//    the same device (two threads, two contexts, two streams) race on it and
//    corrupt each other's results. Serialise them.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocFloats = (size_t)10 << 20;  // 40 MiB
__device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

// Address of this device's scratch array; looked up once per device.
int noalloc_scratch(vti_ctx* ctx, float** out) {
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return fail(ctx, VTI_ERR_ARG, "device index beyond the allocation-free table");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[ctx->device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_check(ctx, e, "cudaGetSymbolAddress(static scratch)");
    g_noalloc_ptr[ctx->device] = (float*)p;
  }
  *out = g_noalloc_ptr[ctx->device];
  return VTI_OK;
}

}  // namespace

extern "C" int vti2d_synthetic_noalloc(vti_ctx* ctx, const vti2d_geom* g, const float* c11,
                                       const float* c13, const float* c33, const float* wavelet,
                                       const int* sloc, int ns, const int* rloc, int nr,
                                       const float* taper, float* data) {
  if (!ctx || !g || !sloc || (nr > 0 && !rloc) || !c11 || !c13 || !c33 || !wavelet || !taper ||
      !data)
    return VTI_ERR_ARG;
  const int nnx = g->nx + 2 * g->npad, nnz = g->nz + 2 * g->npad;
  const long long nnxz = (long long)nnx * nnz;
  if (nnx < 9 || nnz < 9 || g->nt < 2 || !(g->dt > 0) || !(g->rate > 0))
    return fail(ctx, VTI_ERR_ARG, "2D geometry out of range");
  const float dt = g->dt, dt2 = dt * dt;
  const int ratio = (int)(g->rate / dt + 0.5f);  // as vti2d_synthetic
  if (ratio < 1) return fail(ctx, VTI_ERR_ARG, "rate < dt");
  const int ntNeg = (int)std::round(std::fabs(g->ot) / dt);
  const long long rows = (g->nt - ntNeg - 1) / ratio + 1;
  if (rows < 1)
    return fail(ctx, VTI_ERR_ARG, "the whole record lies before time zero (|ot| too large)");
  // validate every shot and size the largest before queuing anything
  long long max_nri = 0;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    if (s[2] < 0 || s[3] < 0 || s[3] + s[2] > nr)
      return fail(ctx, VTI_ERR_ARG, "2D shot receiver range exceeds rloc");
    const long long src = s[0] + (long long)s[1] * nnx;
    if (src < 0 || src >= nnxz) return fail(ctx, VTI_ERR_ARG, "2D source outside the grid");
    for (int ir = 0; ir < s[2]; ++ir) {
      const int x = rloc[2 * (s[3] + ir)], z = rloc[2 * (s[3] + ir) + 1];
      if (x < 0 || x >= nnx || z < 0 || z >= nnz)
        return fail(ctx, VTI_ERR_ARG, "2D receiver outside the grid");
    }
    max_nri = std::max<long long>(max_nri, s[2]);
  }
  {
    const int cst = check_cfl2d(ctx, g, c11, c13, c33);
    if (cst != VTI_OK) return cst;
  }
  const long long need = 8 * nnxz + g->nt + max_nri + rows * max_nri;
  if (need > (long long)kNoAllocFloats) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "allocation-free modeling needs %lld floats of static scratch, capacity %zu",
                  need, kNoAllocFloats);
    return fail(ctx, VTI_ERR_ARG, msg);
  }
  // the caller's current device is restored on every return
  int caller_dev = -1;
  VTI_CUDA(ctx, cudaGetDevice(&caller_dev));
  struct DeviceRestore {
    int dev;
    ~DeviceRestore() {
      if (dev >= 0) cudaSetDevice(dev);
    }
  } restore{caller_dev};
  VTI_CUDA(ctx, cudaSetDevice(ctx->device));
  float* buf = nullptr;
  int st = noalloc_scratch(ctx, &buf);
  if (st != VTI_OK) return st;
  cudaStream_t sm = ctx->stream;
  // From the first queued operation on, an error return first waits for the
  // work already queued on the shared array, so no call returns while its
  // copies or kernels can still touch it.
#define NK(call)                                \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) {                    \
      st = cuda_check(ctx, e_, #call);          \
      cudaStreamSynchronize(sm);                \
      return st;                                \
    }                                           \
  } while (0)
  float *dc11 = buf, *dc13 = dc11 + nnxz, *dc33 = dc13 + nnxz, *dtap = dc33 + nnxz;
  float* w[4] = {dtap + nnxz, dtap + 2 * nnxz, dtap + 3 * nnxz, dtap + 4 * nnxz};
  float* amps = dtap + 5 * nnxz;
  int* d_ridx = reinterpret_cast<int*>(amps + g->nt);
  float* d_rows = amps + g->nt + max_nri;
  NK(cudaMemcpyAsync(dc11, c11, nnxz * 4, cudaMemcpyHostToDevice, sm));
  NK(cudaMemcpyAsync(dc13, c13, nnxz * 4, cudaMemcpyHostToDevice, sm));
  NK(cudaMemcpyAsync(dc33, c33, nnxz * 4, cudaMemcpyHostToDevice, sm));
  NK(cudaMemcpyAsync(dtap, taper, nnxz * 4, cudaMemcpyHostToDevice, sm));
  std::vector<float> h_amp(g->nt, 0.f);
  for (int it = 2; it < g->nt; ++it) h_amp[it] = dt2 * wavelet[it - 1];
  NK(cudaMemcpyAsync(amps, h_amp.data(), g->nt * 4, cudaMemcpyHostToDevice, sm));
  const float idx2 = 1.f / (g->dx * g->dx), idz2 = 1.f / (g->dz * g->dz);
  const dim3 block(BX, BZ), grid((nnx - 8 + BX - 1) / BX, (nnz - 8 + BZ - 1) / BZ);
  std::vector<int> ridx;
  for (int is = 0; is < ns; ++is) {
    const int* s = sloc + 4 * is;
    const int slocxz = s[0] + s[1] * nnx, nri = s[2], ir0 = s[3];
    NK(cudaMemsetAsync(w[0], 0, 4 * nnxz * 4, sm));  // wavefields start at zero
    if (nri > 0) {
      ridx.resize(nri);
      for (int ir = 0; ir < nri; ++ir)
        ridx[ir] = rloc[2 * (ir0 + ir)] + rloc[2 * (ir0 + ir) + 1] * nnx;
      NK(cudaMemcpyAsync(d_ridx, ridx.data(), nri * sizeof(int), cudaMemcpyHostToDevice, sm));
      NK(cudaMemsetAsync(d_rows, 0, (size_t)rows * nri * 4, sm));  // row 0 stays 0
    }
    // time level 1: source then taper (synthetic_f.cu:86-89)
    k_init2d<<<1, 1, 0, sm>>>(w[2], w[3], slocxz, dt2 * wavelet[0], taper[slocxz]);
    ctx->launches++;
    float *p1 = w[2], *q1 = w[3], *p0 = w[0], *q0 = w[1];
    auto record = [&](long long row, const float* p, const float* q) {
      if (nri > 0) {
        k_record2d<<<(nri + 127) / 128, 128, 0, sm>>>(d_rows, row * nri, p, q, d_ridx, nri);
        ctx->launches++;
      }
    };
    if (ratio == 1 && g->ot == 0.f) record(1, p1, q1);
    for (int it = 2; it < g->nt; ++it) {
      const float t = it * dt + g->ot;
      Step2d a{nnx, nnz, p1, q1, p0, q0, dc11, dc13, dc33, dtap, idx2, idz2, dt2, slocxz,
               amps + it};
      k_step2d<<<grid, block, 0, sm>>>(a);
      ctx->launches++;
      if (t >= 0.f && (it - ntNeg) % ratio == 0) record((it - ntNeg) / ratio, p0, q0);
      std::swap(p0, p1);
      std::swap(q0, q1);
    }
    NK(cudaGetLastError());
    if (nri > 0)  // the caller's receiver-fastest layout, as vti2d_synthetic
      NK(cudaMemcpy2DAsync(data + ir0, (size_t)nr * 4, d_rows, (size_t)nri * 4,
                           (size_t)nri * 4, rows, cudaMemcpyDeviceToHost, sm));
  }
  NK(cudaStreamSynchronize(sm));
#undef NK
  return VTI_OK;
}
