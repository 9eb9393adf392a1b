// 3D VTI pseudo-acoustic kernels for sm_100a.
//
// Data layout: every volume is x-fastest with a row pitch that is a multiple
// of 32 floats and kZPad zero planes above and below (vti_internal.h).
//
// Update region and arithmetic follow the reference:
//   * x,y in [4, n-4), z in [0, nz) with zero planes outside
//     (lib/vti-fwi-3d/gpu/kernel3d.cu:7-10, 92, 409);
//   * sigma_x carries the horizontal stencil, sigma_z the vertical one;
//     next = c11*Lxy + c13*Lz + 2cur - prev,  next_z = c13*Lxy + c33*Lz + ...
//     (kernel3d.cu:54-69), and the gradient form dt2*(c*L/dx2)
//     (kernel3d.cu:273-293) for the time-reversed source wavefield;
//   * the sponge (abc3d.cu:82-126) damps next and cur of each 4-plane block
//     after that block is updated, in z order. Stored values here are the
//     once-damped levels v_t; prev is read as d*v_{t-2} and the z stencil
//     multiplies the four planes of the block above by d (they have already
//     been damped as "cur" when the reference reaches this block).
//
// Design (2.5D blocking): a CTA owns a TX x TY column of the grid for a slab
// of z and marches down it. The current sigma_x plane (tile + 4-cell halo)
// is staged in shared memory for the horizontal stencil; sigma_z lives in a
// 9-deep register queue per output point for the vertical stencil. All loads
// for plane z+1 are issued before plane z is computed, so two planes per CTA
// are in flight.
#include "vti_internal.h"

namespace vti {
namespace {

// 8th-order coefficients (lib/vti-fwi-3d/gpu/wave3d.h:8-12).
constexpr float kC0 = -2.84722222222f, kC1 = 1.6f, kC2 = -0.2f, kC3 = 0.02539682539f,
                kC4 = -0.00178571428f;

__device__ __forceinline__ float lap9(float c, float m1, float p1, float m2, float p2, float m3,
                                      float p3, float m4, float p4) {
  float s = kC0 * c;
  s = fmaf(kC1, m1 + p1, s);
  s = fmaf(kC2, m2 + p2, s);
  s = fmaf(kC3, m3 + p3, s);
  s = fmaf(kC4, m4 + p4, s);
  return s;
}

constexpr int TX = 32;   // tile width (one warp)
constexpr int NTY = 8;   // warps per CTA
constexpr int RY = 2;    // rows per thread
constexpr int TY = NTY * RY;
constexpr int SW = TX + 2 * kHalo;
constexpr int SH = TY + 2 * kHalo;
constexpr int NTH = TX * NTY;
constexpr int NLD = (SW * SH + NTH - 1) / NTH;

struct FwdParams {
  Dims3 d;
  const float* cx;
  const float* cz;
  float* px;
  float* pz;
  const float* c11;
  const float* c13;
  const float* c33;
  const float* dampx;  // null: no sponge
  const float* dampy;
  const float* dampz;
  float sx, sy, sz;
  int zslab;
  PointSource src;
};

// Per-thread loader for the (TY+8) x (TX+8) halo tile of one plane.
struct TileLoader {
  int off[NLD];
  int sidx[NLD];
  bool ok[NLD];
  __device__ void init(const Dims3& d, int x0, int y0, int tid) {
#pragma unroll
    for (int k = 0; k < NLD; ++k) {
      int e = tid + k * NTH;
      int r = e / SW, c = e % SW;
      int gx = x0 - kHalo + c, gy = y0 - kHalo + r;
      ok[k] = e < SW * SH && gx < d.nx && gy < d.ny;
      off[k] = gy * d.pitch + gx;
      sidx[k] = e < SW * SH ? e : 0;
    }
  }
  __device__ __forceinline__ void load(const float* plane, float (&v)[NLD]) const {
#pragma unroll
    for (int k = 0; k < NLD; ++k) v[k] = ok[k] ? __ldg(plane + off[k]) : 0.f;
  }
  __device__ __forceinline__ void store(float* tile, const float (&v)[NLD], int tid) const {
#pragma unroll
    for (int k = 0; k < NLD; ++k)
      if (tid + k * NTH < SW * SH) tile[sidx[k]] = v[k];
  }
};

__global__ void __launch_bounds__(NTH, 2) k_fwd3d(const FwdParams p) {
  __shared__ float tile[SH * SW];
  const Dims3 d = p.d;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * TX;
  const int x0 = kHalo + blockIdx.x * TX, y0 = kHalo + blockIdx.y * TY;
  const int x = x0 + tx;
  const int zb = blockIdx.z * p.zslab;
  const int ze = min(d.nz, zb + p.zslab);
  const bool damp = p.dampz != nullptr;

  TileLoader tl;
  tl.init(d, x0, y0, tid);

  int off[RY];
  bool valid[RY];
  float dxy[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    int y = y0 + ty * RY + r;
    valid[r] = x < d.nx - kHalo && y < d.ny - kHalo;
    off[r] = y * d.pitch + x;
    dxy[r] = (damp && valid[r]) ? p.dampx[x] * p.dampy[y] : 1.f;
  }

  // register queue for sigma_z: q[k] holds plane z-4+k during plane z
  float q[RY][9];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    q[r][0] = 0.f;
#pragma unroll
    for (int k = 1; k < 9; ++k)
      q[r][k] = valid[r] ? __ldg(p.cz + (long long)(zb - 5 + k) * d.plane + off[r]) : 0.f;
  }
  float qn[RY], pxr[RY], pzr[RY], a11[RY], a13[RY], a33[RY];
  float tv[NLD];
  {
    const long long pb = (long long)zb * d.plane;
    tl.load(p.cx + pb, tv);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const long long i = pb + off[r];
      qn[r] = valid[r] ? __ldg(p.cz + i + 4 * d.plane) : 0.f;
      pxr[r] = valid[r] ? p.px[i] : 0.f;
      pzr[r] = valid[r] ? p.pz[i] : 0.f;
      a11[r] = valid[r] ? __ldg(p.c11 + i) : 0.f;
      a13[r] = valid[r] ? __ldg(p.c13 + i) : 0.f;
      a33[r] = valid[r] ? __ldg(p.c33 + i) : 0.f;
    }
    tl.store(tile, tv, tid);
  }

  for (int z = zb; z < ze; ++z) {
    // prefetch plane z+1
    float tvn[NLD], qnn[RY], pxn[RY], pzn[RY], b11[RY], b13[RY], b33[RY];
    const bool more = z + 1 < ze;
    if (more) {
      const long long pb = (long long)(z + 1) * d.plane;
      tl.load(p.cx + pb, tvn);
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const long long i = pb + off[r];
        qnn[r] = valid[r] ? __ldg(p.cz + i + 4 * d.plane) : 0.f;
        pxn[r] = valid[r] ? p.px[i] : 0.f;
        pzn[r] = valid[r] ? p.pz[i] : 0.f;
        b11[r] = valid[r] ? __ldg(p.c11 + i) : 0.f;
        b13[r] = valid[r] ? __ldg(p.c13 + i) : 0.f;
        b33[r] = valid[r] ? __ldg(p.c33 + i) : 0.f;
      }
    }
    __syncthreads();
    const float dz = damp ? p.dampz[z] : 1.f;
    const bool new_block = damp && (z & 3) == 0 && z > 0;
    float dzq[4];
    if (new_block) {
#pragma unroll
      for (int k = 0; k < 4; ++k) dzq[k] = p.dampz[z - 4 + k];
    }
#pragma unroll
    for (int r = 0; r < RY; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) q[r][k] = q[r][k + 1];
      q[r][8] = qn[r];
      if (new_block) {
#pragma unroll
        for (int k = 0; k < 4; ++k) q[r][k] *= dxy[r] * dzq[k];
      }
      const int sr = (ty * RY + r + kHalo) * SW + tx + kHalo;
      const float c = tile[sr];
      const float lxx = lap9(c, tile[sr - 1], tile[sr + 1], tile[sr - 2], tile[sr + 2],
                             tile[sr - 3], tile[sr + 3], tile[sr - 4], tile[sr + 4]);
      const float lyy = lap9(c, tile[sr - SW], tile[sr + SW], tile[sr - 2 * SW],
                             tile[sr + 2 * SW], tile[sr - 3 * SW], tile[sr + 3 * SW],
                             tile[sr - 4 * SW], tile[sr + 4 * SW]);
      const float lzz = lap9(q[r][4], q[r][3], q[r][5], q[r][2], q[r][6], q[r][1], q[r][7],
                             q[r][0], q[r][8]);
      const float lxy = fmaf(lyy, p.sy, lxx * p.sx);
      const float lz = lzz * p.sz;
      const float dd = dxy[r] * dz;
      float nxv = fmaf(a11[r], lxy, fmaf(a13[r], lz, 2.f * c - dd * pxr[r]));
      float nzv = fmaf(a13[r], lxy, fmaf(a33[r], lz, 2.f * q[r][4] - dd * pzr[r]));
      const int y = y0 + ty * RY + r;
      if (x == p.src.x && y == p.src.y && z == p.src.z) {
        nxv += p.src.amp;
        nzv += p.src.amp;
      }
      if (valid[r]) {
        const long long i = (long long)z * d.plane + off[r];
        p.px[i] = dd * nxv;
        p.pz[i] = dd * nzv;
      }
    }
    __syncthreads();
    if (more) {
      tl.store(tile, tvn, tid);
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        qn[r] = qnn[r];
        pxr[r] = pxn[r];
        pzr[r] = pzn[r];
        a11[r] = b11[r];
        a13[r] = b13[r];
        a33[r] = b33[r];
      }
    }
  }
}

struct BwdParams {
  Dims3 d;
  const float* scx;
  const float* scz;
  float* spx;
  float* spz;
  const float* lcx;
  const float* lcz;
  float* lpx;
  float* lpz;
  const float* c11;
  const float* c13;
  const float* c33;
  float* g11;
  float* g13;
  float* g33;
  const float* dampx;
  const float* dampy;
  const float* dampz;
  float dt2, idx2, idy2, idz2;
  float sx, sy, sz;
  int zslab;
  PointSource src;
};

__global__ void __launch_bounds__(NTH, 1) k_bwd3d(const BwdParams p) {
  __shared__ float st[SH * SW];  // sigma_x plane
  __shared__ float lt[SH * SW];  // lambda_x plane
  const Dims3 d = p.d;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * TX;
  const int x0 = kHalo + blockIdx.x * TX, y0 = kHalo + blockIdx.y * TY;
  const int x = x0 + tx;
  const int zb = blockIdx.z * p.zslab;
  const int ze = min(d.nz, zb + p.zslab);

  TileLoader tl;
  tl.init(d, x0, y0, tid);

  int off[RY];
  bool valid[RY];
  float dxy[RY];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    int y = y0 + ty * RY + r;
    valid[r] = x < d.nx - kHalo && y < d.ny - kHalo;
    off[r] = y * d.pitch + x;
    dxy[r] = valid[r] ? p.dampx[x] * p.dampy[y] : 1.f;
  }

  float sq[RY][9], lq[RY][9];
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    sq[r][0] = 0.f;
    lq[r][0] = 0.f;
#pragma unroll
    for (int k = 1; k < 9; ++k) {
      const long long i = (long long)(zb - 5 + k) * d.plane + off[r];
      sq[r][k] = valid[r] ? __ldg(p.scz + i) : 0.f;
      lq[r][k] = valid[r] ? __ldg(p.lcz + i) : 0.f;
    }
  }
  // per-point stream for the current plane
  float sqn[RY], lqn[RY], spx[RY], spz[RY], lpx[RY], lpz[RY], a11[RY], a13[RY], a33[RY];
  float gr11[RY], gr13[RY], gr33[RY];
  float tvs[NLD], tvl[NLD];
  {
    const long long pb = (long long)zb * d.plane;
    tl.load(p.scx + pb, tvs);
    tl.load(p.lcx + pb, tvl);
#pragma unroll
    for (int r = 0; r < RY; ++r) {
      const long long i = pb + off[r];
      const bool v = valid[r];
      sqn[r] = v ? __ldg(p.scz + i + 4 * d.plane) : 0.f;
      lqn[r] = v ? __ldg(p.lcz + i + 4 * d.plane) : 0.f;
      spx[r] = v ? p.spx[i] : 0.f;
      spz[r] = v ? p.spz[i] : 0.f;
      lpx[r] = v ? p.lpx[i] : 0.f;
      lpz[r] = v ? p.lpz[i] : 0.f;
      a11[r] = v ? __ldg(p.c11 + i) : 0.f;
      a13[r] = v ? __ldg(p.c13 + i) : 0.f;
      a33[r] = v ? __ldg(p.c33 + i) : 0.f;
      gr11[r] = v ? p.g11[i] : 0.f;
      gr13[r] = v ? p.g13[i] : 0.f;
      gr33[r] = v ? p.g33[i] : 0.f;
    }
    tl.store(st, tvs, tid);
    tl.store(lt, tvl, tid);
  }

  for (int z = zb; z < ze; ++z) {
    float tvsn[NLD], tvln[NLD];
    float sqnn[RY], lqnn[RY], spxn[RY], spzn[RY], lpxn[RY], lpzn[RY], b11[RY], b13[RY], b33[RY];
    float h11[RY], h13[RY], h33[RY];
    const bool more = z + 1 < ze;
    const long long pbz = (long long)z * d.plane;
    if (more) {
      const long long pb = (long long)(z + 1) * d.plane;
      tl.load(p.scx + pb, tvsn);
      tl.load(p.lcx + pb, tvln);
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        const long long i = pb + off[r];
        const bool v = valid[r];
        sqnn[r] = v ? __ldg(p.scz + i + 4 * d.plane) : 0.f;
        lqnn[r] = v ? __ldg(p.lcz + i + 4 * d.plane) : 0.f;
        spxn[r] = v ? p.spx[i] : 0.f;
        spzn[r] = v ? p.spz[i] : 0.f;
        lpxn[r] = v ? p.lpx[i] : 0.f;
        lpzn[r] = v ? p.lpz[i] : 0.f;
        b11[r] = v ? __ldg(p.c11 + i) : 0.f;
        b13[r] = v ? __ldg(p.c13 + i) : 0.f;
        b33[r] = v ? __ldg(p.c33 + i) : 0.f;
        h11[r] = v ? p.g11[i] : 0.f;
        h13[r] = v ? p.g13[i] : 0.f;
        h33[r] = v ? p.g33[i] : 0.f;
      }
    }
    __syncthreads();
    const float dz = p.dampz[z];
    const bool new_block = (z & 3) == 0 && z > 0;
    float dzq[4];
    if (new_block) {
#pragma unroll
      for (int k = 0; k < 4; ++k) dzq[k] = p.dampz[z - 4 + k];
    }
#pragma unroll
    for (int r = 0; r < RY; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        sq[r][k] = sq[r][k + 1];
        lq[r][k] = lq[r][k + 1];
      }
      sq[r][8] = sqn[r];
      lq[r][8] = lqn[r];
      if (new_block) {
#pragma unroll
        for (int k = 0; k < 4; ++k) lq[r][k] *= dxy[r] * dzq[k];
      }
      const int sr = (ty * RY + r + kHalo) * SW + tx + kHalo;
      const int y = y0 + ty * RY + r;
      // ---- source wavefield, gradient form (kernel3d.cu:273-288)
      const float sc = st[sr];
      const float sxx = lap9(sc, st[sr - 1], st[sr + 1], st[sr - 2], st[sr + 2], st[sr - 3],
                             st[sr + 3], st[sr - 4], st[sr + 4]);
      const float syy = lap9(sc, st[sr - SW], st[sr + SW], st[sr - 2 * SW], st[sr + 2 * SW],
                             st[sr - 3 * SW], st[sr + 3 * SW], st[sr - 4 * SW], st[sr + 4 * SW]);
      const float szz = lap9(sq[r][4], sq[r][3], sq[r][5], sq[r][2], sq[r][6], sq[r][1],
                             sq[r][7], sq[r][0], sq[r][8]);
      const float sxy_u = fmaf(syy, p.idy2, sxx * p.idx2);
      const float sz_u = szz * p.idz2;
      float snx = fmaf(p.dt2, fmaf(a11[r], sxy_u, a13[r] * sz_u), 2.f * sc - spx[r]);
      float snz = fmaf(p.dt2, fmaf(a13[r], sxy_u, a33[r] * sz_u), 2.f * sq[r][4] - spz[r]);
      if (x == p.src.x && y == p.src.y && z == p.src.z) {
        snx += p.src.amp;
        snz += p.src.amp;
      }
      // ---- zero-lag imaging with the current adjoint (kernel3d.cu:291-293)
      const float lc = lt[sr];
      const float lzc0 = lq[r][4];
      gr11[r] = fmaf(lc, sxy_u, gr11[r]);
      gr33[r] = fmaf(lzc0, sz_u, gr33[r]);
      gr13[r] = fmaf(lzc0, sxy_u, fmaf(lc, sz_u, gr13[r]));
      // ---- adjoint wavefield, forward form with the sponge
      const float lxx = lap9(lc, lt[sr - 1], lt[sr + 1], lt[sr - 2], lt[sr + 2], lt[sr - 3],
                             lt[sr + 3], lt[sr - 4], lt[sr + 4]);
      const float lyy = lap9(lc, lt[sr - SW], lt[sr + SW], lt[sr - 2 * SW], lt[sr + 2 * SW],
                             lt[sr - 3 * SW], lt[sr + 3 * SW], lt[sr - 4 * SW], lt[sr + 4 * SW]);
      const float lzz = lap9(lzc0, lq[r][3], lq[r][5], lq[r][2], lq[r][6], lq[r][1], lq[r][7],
                             lq[r][0], lq[r][8]);
      const float lxy = fmaf(lyy, p.sy, lxx * p.sx);
      const float lz = lzz * p.sz;
      const float dd = dxy[r] * dz;
      const float lnx = fmaf(a11[r], lxy, fmaf(a13[r], lz, 2.f * lc - dd * lpx[r]));
      const float lnz = fmaf(a13[r], lxy, fmaf(a33[r], lz, 2.f * lzc0 - dd * lpz[r]));
      if (valid[r]) {
        const long long i = pbz + off[r];
        p.spx[i] = snx;
        p.spz[i] = snz;
        p.lpx[i] = dd * lnx;
        p.lpz[i] = dd * lnz;
        p.g11[i] = gr11[r];
        p.g13[i] = gr13[r];
        p.g33[i] = gr33[r];
      }
    }
    __syncthreads();
    if (more) {
      tl.store(st, tvsn, tid);
      tl.store(lt, tvln, tid);
#pragma unroll
      for (int r = 0; r < RY; ++r) {
        sqn[r] = sqnn[r];
        lqn[r] = lqnn[r];
        spx[r] = spxn[r];
        spz[r] = spzn[r];
        lpx[r] = lpxn[r];
        lpz[r] = lpzn[r];
        a11[r] = b11[r];
        a13[r] = b13[r];
        a33[r] = b33[r];
        gr11[r] = h11[r];
        gr13[r] = h13[r];
        gr33[r] = h33[r];
      }
    }
  }
}

// ------------------------------------------------------ sparse kernels
// recordData (injectRecord3d.cu:22-28) into trace-major traces.
__global__ void k_record(float* trace, int nnt, int j, const float* cx, const float* cz,
                         const long long* rec, int nr) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    long long o = rec[ir];
    trace[(long long)ir * nnt + j] = (float)(kTwoThird * cx[o] + kOneThird * cz[o]);
  }
}

// injectResidual with the interpolation of interpolateResidual
// (injectRecord3d.cu:38-46,60-78); the sponge factor of the receiver point is
// applied because the step kernel has already damped next.
__global__ void k_inject_residual(float* lx, float* lz, const float* res, int nnt, int i0,
                                  float f, int clamp_last, const long long* rec,
                                  const float* rec_damp, int nr, float dt2) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr) {
    const float* t = res + (long long)ir * nnt;
    float r = clamp_last ? t[nnt - 1] : (float)((1. - f) * t[i0] + f * t[i0 + 1]);
    float s = dt2 * r;
    long long o = rec[ir];
    float d = rec_damp[ir];
    lx[o] += d * (float)(kTwoThird * s);
    lz[o] += d * (float)(kOneThird * s);
  }
}

// objFuncGradient3d_f.cu:922-927: adjoint seeded by assignment.
__global__ void k_seed_adjoint(float* lx, float* lz, const float* res, int nnt,
                               const long long* rec, const float* rec_damp, int nr, float dt2) {
  int ir = blockIdx.x * blockDim.x + threadIdx.x;
  if (ir < nr && rec_damp[ir] != 0.f) {
    float temp = dt2 * res[(long long)ir * nnt + nnt - 1];
    long long o = rec[ir];
    lx[o] = (float)(kTwoThird * temp);
    lz[o] = (float)(kOneThird * temp);
  }
}

__global__ void k_set_point(float* a, float* b, long long off, float value) {
  a[off] = value;
  b[off] = value;
}

// Residual + FP64 misfit (objFuncGradient3d_f.cu:735-771). Each block writes
// its partial sum; k_sum_partials adds them in a fixed order, so the misfit is
// bitwise reproducible run to run.
__global__ void k_residual(float* trace, const float* obs, const unsigned char* live, int nnt,
                           int nr, double* partial) {
  long long n = (long long)nnt * nr;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int ir = (int)(i / nnt);
    float m = live[ir] ? trace[i] : 0.f;
    if (!obs) {
      trace[i] = m;
      continue;
    }
    float r = m - obs[i];
    trace[i] = r;
    s += (double)(r * r);
  }
  if (!partial) return;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// acc[0] += sum(partial[0..n)) in a fixed order (one warp).
__global__ void k_sum_partials(const double* partial, int n, double* acc) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) v += partial[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) acc[0] += v;
}

// putBoundary applied on the device: out = full, with the pad region replaced
// by the boundary list (order of boundary.cpp:10-46).
__global__ void k_boundary_merge(Dims3 d, int npad, const float* full, const float* blist,
                                 float* out) {
  long long n = d.npoints();
  const long long nxy = (long long)d.nx * d.ny;
  const long long top = nxy * npad;
  const long long mid_plane = 2LL * npad * d.nx + (long long)(d.ny - 2 * npad) * 2 * npad;
  const long long mid_total = (long long)(d.nz - 2 * npad) * mid_plane;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int x = (int)(t % d.nx);
    int y = (int)((t / d.nx) % d.ny);
    int z = (int)(t / nxy);
    long long k = -1;
    if (z < npad) {
      k = x + (long long)y * d.nx + (long long)z * nxy;
    } else if (z >= d.nz - npad) {
      k = top + mid_total + x + (long long)y * d.nx + (long long)(z - (d.nz - npad)) * nxy;
    } else {
      long long base = top + (long long)(z - npad) * mid_plane;
      if (y < npad) {
        k = base + x + (long long)y * d.nx;
      } else if (y >= d.ny - npad) {
        k = base + (long long)npad * d.nx + (long long)(d.ny - 2 * npad) * 2 * npad + x +
            (long long)(y - (d.ny - npad)) * d.nx;
      } else {
        long long rb = base + (long long)npad * d.nx + (long long)(y - npad) * 2 * npad;
        if (x < npad) k = rb + x;
        else if (x >= d.nx - npad) k = rb + npad + (x - (d.nx - npad));
      }
    }
    long long o = d.off(x, y, z);
    out[o] = k >= 0 ? blist[k] : full[o];
  }
}

int zslab_for(vti_ctx* ctx, const Dims3& d, int tiles, int ctas_per_sm) {
  // choose the number of z slabs so the grid fills the GPU a few times over
  int target = ctx->sm_count * ctas_per_sm * 4;
  int nslab = (target + tiles - 1) / tiles;
  int maxslab = (d.nz + 3) / 4;
  if (nslab > maxslab) nslab = maxslab;
  if (nslab < 1) nslab = 1;
  int zs = (d.nz + nslab - 1) / nslab;
  zs = (zs + 3) & ~3;
  return zs;
}

}  // namespace

int launch_fwd3d(vti_ctx* ctx, const Dims3& d, const float* cx, const float* cz, float* px,
                 float* pz, const float* c11, const float* c13, const float* c33,
                 const Damping* damp, float sx, float sy, float sz, PointSource src) {
  FwdParams p;
  p.d = d;
  p.cx = cx; p.cz = cz; p.px = px; p.pz = pz;
  p.c11 = c11; p.c13 = c13; p.c33 = c33;
  p.dampx = damp ? damp->x : nullptr;
  p.dampy = damp ? damp->y : nullptr;
  p.dampz = damp ? damp->z : nullptr;
  p.sx = sx; p.sy = sy; p.sz = sz;
  p.src = src;
  dim3 block(TX, NTY);
  int gx = (d.nx - 2 * kHalo + TX - 1) / TX, gy = (d.ny - 2 * kHalo + TY - 1) / TY;
  p.zslab = zslab_for(ctx, d, gx * gy, 3);
  dim3 grid(gx, gy, (d.nz + p.zslab - 1) / p.zslab);
  {
    LaunchTimer tm(ctx, kTimedFwd3d);
    k_fwd3d<<<grid, block, 0, ctx->stream>>>(p);
  }
  VTI_LAUNCHED(ctx, "k_fwd3d");
  return VTI_OK;
}

int launch_bwd3d(vti_ctx* ctx, const Dims3& d, const float* scx, const float* scz, float* spx,
                 float* spz, const float* lcx, const float* lcz, float* lpx, float* lpz,
                 const float* c11, const float* c13, const float* c33, float* g11, float* g13,
                 float* g33, const Damping& damp, float dt2, float idx2, float idy2, float idz2,
                 float sx, float sy, float sz, PointSource src) {
  BwdParams p;
  p.d = d;
  p.scx = scx; p.scz = scz; p.spx = spx; p.spz = spz;
  p.lcx = lcx; p.lcz = lcz; p.lpx = lpx; p.lpz = lpz;
  p.c11 = c11; p.c13 = c13; p.c33 = c33;
  p.g11 = g11; p.g13 = g13; p.g33 = g33;
  p.dampx = damp.x; p.dampy = damp.y; p.dampz = damp.z;
  p.dt2 = dt2; p.idx2 = idx2; p.idy2 = idy2; p.idz2 = idz2;
  p.sx = sx; p.sy = sy; p.sz = sz;
  p.src = src;
  dim3 block(TX, NTY);
  int gx = (d.nx - 2 * kHalo + TX - 1) / TX, gy = (d.ny - 2 * kHalo + TY - 1) / TY;
  p.zslab = zslab_for(ctx, d, gx * gy, 2);
  dim3 grid(gx, gy, (d.nz + p.zslab - 1) / p.zslab);
  {
    LaunchTimer tm(ctx, kTimedBwd3d);
    k_bwd3d<<<grid, block, 0, ctx->stream>>>(p);
  }
  VTI_LAUNCHED(ctx, "k_bwd3d");
  return VTI_OK;
}

int launch_record(vti_ctx* ctx, float* trace, int nnt, int j, const float* cx, const float* cz,
                  const long long* rec, int nr) {
  if (nr <= 0) return VTI_OK;
  k_record<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(trace, nnt, j, cx, cz, rec, nr);
  VTI_LAUNCHED(ctx, "k_record");
  return VTI_OK;
}

int launch_inject_residual(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                           int i0, float f, int clamp_last, const long long* rec,
                           const float* rec_damp, int nr, float dt2) {
  if (nr <= 0) return VTI_OK;
  k_inject_residual<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(lx, lz, res, nnt, i0, f,
                                                               clamp_last, rec, rec_damp, nr, dt2);
  VTI_LAUNCHED(ctx, "k_inject_residual");
  return VTI_OK;
}

int launch_seed_adjoint(vti_ctx* ctx, float* lx, float* lz, const float* res, int nnt,
                        const long long* rec, const float* rec_damp, int nr, float dt2) {
  if (nr <= 0) return VTI_OK;
  k_seed_adjoint<<<(nr + 255) / 256, 256, 0, ctx->stream>>>(lx, lz, res, nnt, rec, rec_damp, nr,
                                                            dt2);
  VTI_LAUNCHED(ctx, "k_seed_adjoint");
  return VTI_OK;
}

int launch_set_point(vti_ctx* ctx, float* a, float* b, long long off, float value) {
  k_set_point<<<1, 1, 0, ctx->stream>>>(a, b, off, value);
  VTI_LAUNCHED(ctx, "k_set_point");
  return VTI_OK;
}

int residual_blocks(vti_ctx* ctx) { return ctx->sm_count * 8; }

int launch_residual(vti_ctx* ctx, float* trace, const float* obs, const unsigned char* live,
                    int nnt, int nr, double* acc) {
  long long n = (long long)nnt * nr;
  if (n <= 0) return VTI_OK;
  int blocks = (int)std::min<long long>((n + 255) / 256, (long long)residual_blocks(ctx));
  // acc[0] is the running sum, acc[1 .. 1+residual_blocks) the partials
  k_residual<<<blocks, 256, 0, ctx->stream>>>(trace, obs, live, nnt, nr, acc ? acc + 1 : nullptr);
  VTI_LAUNCHED(ctx, "k_residual");
  if (acc) {
    k_sum_partials<<<1, 32, 0, ctx->stream>>>(acc + 1, blocks, acc);
    VTI_LAUNCHED(ctx, "k_sum_partials");
  }
  return VTI_OK;
}

int launch_boundary_merge(vti_ctx* ctx, const Dims3& d, int npad, const float* full,
                          const float* blist, float* out) {
  long long n = d.npoints();
  int blocks = (int)std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 16);
  k_boundary_merge<<<blocks, 256, 0, ctx->stream>>>(d, npad, full, blist, out);
  VTI_LAUNCHED(ctx, "k_boundary_merge");
  return VTI_OK;
}

}  // namespace vti
