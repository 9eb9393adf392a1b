// v/eps/del parameterisation around the c_ij gradient
// (objFuncGradientVEpsDel, lib/vti-fwi-3d/gpu/objFuncGradient3d_f.cu:249-305).
#include <cstring>
#include <vector>

#include "vti_b200.h"

extern "C" int vti3d_gradient_vepsdel(vti_ctx* ctx, const vti3d_geom* g, const float* v,
                                      const float* eps, const float* del,
                                      const float* padboundary_v, const float* randboundary_v,
                                      float v0, float eps0, float wbottom, const float* wavelet,
                                      const float* souloc, const int* shotid, int nshot,
                                      const float* recloc, int nrec_total, const float* dobs,
                                      float* gv, float* geps, float* gdel, double* misfit,
                                      unsigned flags) {
  if (!ctx || !g || !v || !eps || !del || !padboundary_v || !randboundary_v || !gv || !geps ||
      !gdel)
    return VTI_ERR_ARG;
  const int nx = g->nx, ny = g->ny, nz = g->nz, npad = g->npad;
  const size_t nxy = (size_t)nx * ny, n = nxy * nz;
  const size_t nb = n - (size_t)(nx - 2 * npad) * (ny - 2 * npad) * (nz - 2 * npad);
  // :254-269 model and both boundary sets in c_ij (delta scale del0 = 1)
  std::vector<float> cij(3 * n), fgcij(1 + 3 * n), be(nb), bd(nb), padb(3 * nb), randb(3 * nb);
  vti_vepsdel_to_cij(cij.data(), cij.data() + n, cij.data() + 2 * n, v, eps, del, v0, eps0, 1.f,
                     n);
  vti3d_get_boundary(be.data(), eps, nx, ny, nz, npad);
  vti3d_get_boundary(bd.data(), del, nx, ny, nz, npad);
  vti_vepsdel_to_cij(padb.data(), padb.data() + nb, padb.data() + 2 * nb, padboundary_v,
                     be.data(), bd.data(), v0, eps0, 1.f, nb);
  vti_vepsdel_to_cij(randb.data(), randb.data() + nb, randb.data() + 2 * nb, randboundary_v,
                     be.data(), bd.data(), v0, eps0, 1.f, nb);
  int st = vti3d_gradient_cij(ctx, g, cij.data(), padb.data(), randb.data(), wavelet, souloc,
                              shotid, nshot, recloc, nrec_total, dobs, fgcij.data(), nullptr,
                              flags);
  if (st != VTI_OK) return st;
  // :274 the misfit travels through the float fgcij[0]
  if (misfit) *misfit = (double)fgcij[0];
  float* gc[3] = {fgcij.data() + 1, fgcij.data() + 1 + n, fgcij.data() + 1 + 2 * n};
  // :276-282 no update in the pad nor above the water bottom
  int nwbottom = (wbottom - g->oz) / g->dz + 1 - npad;
  for (int k = 0; k < 3; ++k) {
    vti3d_zero_boundary(gc[k], nx, ny, nz, npad);
    if (nwbottom > 0) {
      size_t nrow = (size_t)nwbottom;
      if (npad + nrow > (size_t)nz) nrow = nz - npad;
      std::memset(gc[k] + (size_t)npad * nxy, 0, nrow * nxy * sizeof(float));
    }
  }
  // :284 chain rule
  vti_grad_cij_to_vepsdel(gv, geps, gdel, gc[0], gc[1], gc[2], v, eps, del, v0, eps0, 1.f, n);
  return VTI_OK;
}
