/* Source-inversion operator of the 3D library (lib/vti-fwi-3d/gpu/ModelingOp3d.h,
 * ModelingOp3d.cu:12-33), declared with the same class layout so that a
 * driver compiled against the reference header (sourceInv-cg.cu, which hands
 * it to simpleSolver) links to libvti_wave.so. The model is the wavelet (nt
 * samples); the data are the traces of all shots (nnt x nrtotal, nrtotal =
 * irbegin + nr of the last shot in souloc). forward = modelData3d_f with the
 * model as the wavelet, adjoint = waveletGradient3d_f; add = true
 * accumulates into the output. */
#ifndef VTI_MODELING_OP3D_H
#define VTI_MODELING_OP3D_H

#include <cmath>
#include <vector>

#include "vti_operator.h"

class ModelingOp3d : public Operator {
 public:
  ModelingOp3d(float* souloc, int ns, std::vector<int> shotid, float* recloc, float* c11,
               float* c13, float* c33, int nx, int ny, int nz, int nt, int npad, float ox,
               float oy, float oz, float ot, float dx, float dy, float dz, float dt,
               float samplingRate, std::vector<int> GPUs, int ngpugroup)
      : Operator(nt, (long long)((nt - 1) / std::round(samplingRate / dt) + 1) *
                         (long long)(souloc[5 * ns - 1] + souloc[5 * ns - 2])),
        _souloc(souloc), _recloc(recloc), _c11(c11), _c13(c13), _c33(c33), _ns(ns), _nx(nx),
        _ny(ny), _nz(nz), _nt(nt), _npad(npad), _ngpugroup(ngpugroup), _ox(ox), _oy(oy),
        _oz(oz), _ot(ot), _dx(dx), _dy(dy), _dz(dz), _dt(dt), _samplingRate(samplingRate),
        _shotid(shotid), _GPUs(GPUs) {}
  void forward(bool add, const float* model, float* data);
  void adjoint(bool add, float* model, const float* data);
  float *_souloc, *_recloc, *_c11, *_c13, *_c33;
  int _ns, _nx, _ny, _nz, _nt, _npad, _ngpugroup;
  float _ox, _oy, _oz, _ot, _dx, _dy, _dz, _dt, _samplingRate;
  std::vector<int> _shotid, _GPUs;
};

#endif /* VTI_MODELING_OP3D_H */
