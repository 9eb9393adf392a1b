/* The reference's linear-operator interface (lib/LinearSolver/LinearSolver.h:6-12),
 * declared with the same class layout so that solvers compiled against the
 * reference headers (CG, LSQR, simpleSolver of LinearSolver.cpp) drive the
 * operator classes of libvti_wave.so unchanged. */
#ifndef VTI_OPERATOR_H
#define VTI_OPERATOR_H

class Operator {
 public:
  Operator(long long modelSize, long long dataSize) : _modelSize(modelSize), _dataSize(dataSize) {}
  virtual void forward(bool add, const float* model, float* data) = 0;
  virtual void adjoint(bool add, float* model, const float* data) = 0;
  long long _modelSize, _dataSize;
};

#endif /* VTI_OPERATOR_H */
