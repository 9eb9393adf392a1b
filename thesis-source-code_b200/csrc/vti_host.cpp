// Host-side glue of the VTI path: pad-region boundary lists, parameter
// conversions, bound projection, the 2D taper and the stability bound.
// These are O(n) host operations around the device time loops; their
// arithmetic (including the float/double mix) is kept as the reference
// writes it so that drop-in callers see identical numbers.
#include <immintrin.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "vti_b200.h"

namespace {

// Copy helper walking the getBoundary order (boundary.cpp:10-46):
// top npad planes, then per middle plane: npad full rows, npad-wide strips at
// both ends of each middle row, npad full rows; then the bottom npad planes.
template <typename F>
void walk_boundary(int nx, int ny, int nz, int npad, F&& run) {
  size_t cb = 0, cv = 0, n = (size_t)nx * ny * npad;
  run(cb, cv, n);
  cb += n;
  cv += n;
  for (int iz = 0; iz < nz - 2 * npad; iz++) {
    for (int iy = 0; iy < npad; iy++) {
      run(cb, cv, (size_t)nx);
      cb += nx;
      cv += nx;
    }
    for (int iy = 0; iy < ny - 2 * npad; iy++) {
      run(cb, cv, (size_t)npad);
      cb += npad;
      cv += nx - npad;
      run(cb, cv, (size_t)npad);
      cb += npad;
      cv += npad;
    }
    for (int iy = 0; iy < npad; iy++) {
      run(cb, cv, (size_t)nx);
      cb += nx;
      cv += nx;
    }
  }
  run(cb, cv, (size_t)nx * ny * npad);
}

const float kDamper2d = 0.95f;  // lib/vti-fwi-2d/init.h:11

// |C0 + 2 sum (-1)^k C_k| of the 8th-order second derivative
// (lib/vti-fwi-3d/gpu/wave3d.h:8-12): its symbol at the Nyquist wavenumber
// times h^2.
double nyq() {
  const double C[5] = {-2.84722222222, 1.6, -0.2, 0.02539682539, -0.00178571428};
  double s = C[0];
  for (int k = 1; k <= 4; ++k) s += 2.0 * C[k] * ((k & 1) ? -1.0 : 1.0);
  return std::fabs(s);
}

// max over the points of the largest eigenvalue of
// [[c11 kh, c13 kz], [c13 kh, c33 kz]]; a NaN value makes the result NaN.
double max_symbol(const float* c11, const float* c13, const float* c33, size_t n, double kh,
                  double kz) {
  double worst = 0.0;
  int bad = 0;
#pragma omp parallel for reduction(max : worst) reduction(| : bad)
  for (size_t i = 0; i < n; ++i) {
    double a = c11[i] * kh, b = c13[i] * kz, c = c13[i] * kh, d = c33[i] * kz;
    double tr = a + d, det = a * d - b * c;
    double disc = tr * tr * 0.25 - det;
    double lam = tr * 0.5 + std::sqrt(disc > 0 ? disc : 0.0);
    if (std::isnan(lam)) bad = 1;
    else if (lam > worst) worst = lam;
  }
  return bad ? std::nan("") : worst;
}

}  // namespace

extern "C" {

void vti3d_get_boundary(float* boundary, const float* v, int nx, int ny, int nz, int npad) {
  walk_boundary(nx, ny, nz, npad, [&](size_t cb, size_t cv, size_t n) {
    std::memcpy(boundary + cb, v + cv, n * sizeof(float));
  });
}

void vti3d_put_boundary(const float* boundary, float* v, int nx, int ny, int nz, int npad) {
  walk_boundary(nx, ny, nz, npad, [&](size_t cb, size_t cv, size_t n) {
    std::memcpy(v + cv, boundary + cb, n * sizeof(float));
  });
}

void vti3d_zero_boundary(float* v, int nx, int ny, int nz, int npad) {
  walk_boundary(nx, ny, nz, npad,
                [&](size_t, size_t cv, size_t n) { std::memset(v + cv, 0, n * sizeof(float)); });
}

// conversions.cpp:42-50
void vti_vepsdel_to_cij(float* c11, float* c13, float* c33, const float* v, const float* eps,
                        const float* del, float v0, float eps0, float del0, size_t n) {
#pragma omp parallel for
  for (size_t i = 0; i < n; ++i) {
    c33[i] = v0 * v0 * v[i] * v[i];
    c11[i] = c33[i] * (1. + 2 * eps0 * eps[i]);
    c13[i] = c33[i] * std::sqrt(1. + 2 * del0 * del[i]);
  }
}

// conversions.cpp:69-81
void vti_grad_cij_to_vepsdel(float* gv, float* geps, float* gdel, const float* gc11,
                             const float* gc13, const float* gc33, const float* v,
                             const float* eps, const float* del, float v0, float eps0, float del0,
                             size_t n) {
#pragma omp parallel for
  for (size_t i = 0; i < n; ++i) {
    float tv = v0 * v[i];
    float teps = 1. + 2 * eps0 * eps[i];
    float tdel = std::sqrt(1. + 2 * del0 * del[i]);
    gv[i] = 2 * tv * (gc11[i] * teps + gc13[i] * tdel + gc33[i]) * v0;
    tv = tv * tv;
    geps[i] = 2 * tv * gc11[i] * eps0;
    gdel[i] = tv / tdel * gc13[i] * del0;
  }
}

// conversions.cpp:52-67
void vti_dvepsdel_to_dcij(float* c11, float* c13, float* c33, float* dc11, float* dc13,
                          float* dc33, const float* v, const float* eps, const float* del,
                          const float* dv, const float* deps, const float* ddel, float v0,
                          float eps0, float del0, size_t n) {
#pragma omp parallel for
  for (size_t i = 0; i < n; ++i) {
    float vv = v0 * v[i], ee = eps0 * eps[i], dd = del0 * del[i];
    float vv2 = vv * vv;
    ee = 1. + 2 * ee;
    dd = std::sqrt(1. + 2 * dd);
    c11[i] = vv2 * ee;
    c13[i] = vv2 * dd;
    c33[i] = vv2;
    dc33[i] = 2 * vv * dv[i] * v0;
    dc11[i] = dc33[i] * ee + 2 * vv2 * deps[i] * eps0;
    dc13[i] = dc33[i] * dd + vv2 / dd * ddel[i] * del0;
  }
}

// check.cpp:22-40: project (eps, del) so that del0*del <= eps0*eps.
int vti_check_eps_del(float* eps, float* del, float eps0, float del0, size_t n, float* mask) {
  int count = 0;
  if (mask) std::memset(mask, 0, n * sizeof(float));
#pragma omp parallel for reduction(+ : count)
  for (size_t i = 0; i < n; ++i) {
    if (del0 * del[i] == eps0 * eps[i]) {
      if (mask) mask[i] = 1;
    } else if (del0 * del[i] > eps0 * eps[i]) {
      float temp = (eps0 * del[i] + del0 * eps[i]) / (eps0 * eps0 + del0 * del0);
      eps[i] = temp * del0;
      del[i] = temp * eps0;
      if (mask) mask[i] = 2;
      count += 1;
    }
  }
  return count;
}

// lib/vti-fwi-2d/init.cpp:70-89
void vti2d_init_taper(float* taper, int nx, int nz, int npad) {
  const double pi = 4.f * std::atan(1.f);  // init.h:9 (float-precision pi)
  float* t0 = new float[npad > 0 ? npad : 1];
  for (int i = 0; i < npad; ++i)
    t0[i] = kDamper2d + (1. - kDamper2d) * std::cos(pi * (float)(npad - 1 - i) / npad);
  const int nnx = nx + 2 * npad, nnz = nz + 2 * npad;
  for (long i = 0; i < (long)nnx * nnz; ++i) taper[i] = 1.f;
  for (int i = 0; i < nnz; ++i) {
    float* row = taper + (long)i * nnx;
    for (int j = 0; j < npad; ++j) row[j] = row[j] * t0[j];
    float* tail = row + npad + nx;
    for (int j = 0; j < npad; ++j) tail[j] = tail[j] * t0[npad - 1 - j];
  }
  for (int i = 0; i < npad; ++i) {
    float* r0 = taper + (long)i * nnx;
    float* r1 = taper + (long)(i + npad + nz) * nnx;
    for (int j = 0; j < nnx; ++j) r0[j] = r0[j] * t0[i];
    for (int j = 0; j < nnx; ++j) r1[j] = r1[j] * t0[npad - 1 - i];
  }
  delete[] t0;
}

// dt^2 * lambda_max of [[c11 Kh, c13 Kz],[c13 Kh, c33 Kz]] at the Nyquist
// wavenumber, where K = |C0 + 2 sum (-1)^k C_k| / h^2 for each axis
// (coefficients of lib/vti-fwi-3d/gpu/wave3d.h:8-12).
double vti3d_cfl_number(const vti3d_geom* g, const float* c11, const float* c13,
                        const float* c33) {
  const double s = nyq();
  const double kh = s / ((double)g->dx * g->dx) + (g->ny > 1 ? s / ((double)g->dy * g->dy) : 0.0);
  const double kz = s / ((double)g->dz * g->dz);
  const size_t n = (size_t)g->nx * g->ny * g->nz;
  return max_symbol(c11, c13, c33, n, kh, kz) * (double)g->dt * g->dt;
}

// The same bound for the 2D scheme (x and z second derivatives of the same
// 8th-order stencil, lib/vti-fwi-2d/kernels.h:4-8) on the padded grid.
double vti2d_cfl_number(const vti2d_geom* g, const float* c11, const float* c13,
                        const float* c33) {
  const double s = nyq();
  const double kh = s / ((double)g->dx * g->dx), kz = s / ((double)g->dz * g->dz);
  const size_t n = (size_t)(g->nx + 2 * g->npad) * (g->nz + 2 * g->npad);
  return max_symbol(c11, c13, c33, n, kh, kz) * (double)g->dt * g->dt;
}

}  // extern "C"

// ------------------------------------------------ 16-bit traces in flight
// Block layout: nnt FP32 plane scales, then nr * nnt IEEE halves
// (trace-major). The scale of time sample t is the largest |value| of any
// trace at t, so every sample is packed at the half's full relative
// precision (F16C conversions, round to nearest even).
extern "C" {

size_t vti_traces_f16_bytes(int nr, int nnt) {
  if (nr < 0 || nnt < 0) return 0;
  return (size_t)nnt * sizeof(float) + (size_t)nr * nnt * sizeof(uint16_t);
}

int vti_traces_pack_f16(const float* traces, int nr, int nnt, void* block) {
  if ((!traces && nr > 0) || !block || nr < 0 || nnt < 1) return VTI_ERR_ARG;
  float* scale = static_cast<float*>(block);
  uint16_t* h = reinterpret_cast<uint16_t*>(scale + nnt);
  std::vector<float> mx((size_t)nnt, 0.f);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<float> local((size_t)nnt, 0.f);
    int lbad = 0;
#pragma omp for nowait
    for (int r = 0; r < nr; ++r) {
      const float* t = traces + (size_t)r * nnt;
      for (int i = 0; i < nnt; ++i) {
        const float a = std::fabs(t[i]);
        if (!std::isfinite(a)) lbad = 1;
        local[i] = std::max(local[i], a);
      }
    }
#pragma omp critical
    {
      bad |= lbad;
      for (int i = 0; i < nnt; ++i) mx[i] = std::max(mx[i], local[i]);
    }
  }
  if (bad) return VTI_ERR_NONFINITE;
  for (int i = 0; i < nnt; ++i) scale[i] = mx[i] > 0.f ? mx[i] : 1.f;
  std::vector<float> inv((size_t)nnt);
  for (int i = 0; i < nnt; ++i) inv[i] = 1.f / scale[i];
#pragma omp parallel for
  for (int r = 0; r < nr; ++r) {
    const float* t = traces + (size_t)r * nnt;
    uint16_t* o = h + (size_t)r * nnt;
    int i = 0;
    for (; i + 8 <= nnt; i += 8) {
      const __m256 v = _mm256_mul_ps(_mm256_loadu_ps(t + i), _mm256_loadu_ps(inv.data() + i));
      _mm_storeu_si128(reinterpret_cast<__m128i*>(o + i),
                       _mm256_cvtps_ph(v, _MM_FROUND_TO_NEAREST_INT));
    }
    for (; i < nnt; ++i) o[i] = _cvtss_sh(t[i] * inv[i], _MM_FROUND_TO_NEAREST_INT);
  }
  return VTI_OK;
}

int vti_traces_unpack_f16(const void* block, int nr, int nnt, float* traces) {
  if (!block || (!traces && nr > 0) || nr < 0 || nnt < 1) return VTI_ERR_ARG;
  const float* scale = static_cast<const float*>(block);
  const uint16_t* h = reinterpret_cast<const uint16_t*>(scale + nnt);
#pragma omp parallel for
  for (int r = 0; r < nr; ++r)
    for (int i = 0; i < nnt; ++i)
      traces[(size_t)r * nnt + i] = _cvtsh_ss(h[(size_t)r * nnt + i]) * scale[i];
  return VTI_OK;
}

}  // extern "C"
