// Function table of the per-degree cell-kernel launchers.
#pragma once

#include <cuda_runtime.h>

namespace mpdg {

template <typename T> struct CellArgs;

struct DegreeTable {
  int n = 0;
  void (*upload)(const double *tab, const float *tabf, const double *w, const float *wf) = nullptr;
  cudaError_t (*vmult_d)(const CellArgs<double> &, int geo, int law, cudaStream_t, int sm) = nullptr;
  cudaError_t (*vmult_f)(const CellArgs<float> &, int geo, int law, cudaStream_t, int sm) = nullptr;
  cudaError_t (*rhs)(const CellArgs<double> &, int geo, int law, cudaStream_t, int sm) = nullptr;
  cudaError_t (*diag)(const CellArgs<double> &, int geo, int law, cudaStream_t, int sm) = nullptr;
  cudaError_t (*norm)(const CellArgs<double> &, int geo, int law, cudaStream_t, int sm) = nullptr;
  // kq[cell][q] = k(T_lin) in FP32; nullptr where the degree has no register-resident kernel
  cudaError_t (*conductivity_q)(const CellArgs<double> &, float *kq, int law, cudaStream_t,
                                int sm) = nullptr;
  // tangent coefficient fields of the LAW 5 operator at a.Tl (8 per point, FP64)
  cudaError_t (*coef_tangent)(const CellArgs<double> &, double *out, int geo, cudaStream_t,
                              int sm) = nullptr;
  // heaviside and velocity values at the quadrature points into the coefficient array's
  // slots 0 and 2..4 ([cell][5][npt])
  cudaError_t (*field_values)(const CellArgs<double> &, const double *H, const double *vel,
                              int64_t n_dofs, double *cf, cudaStream_t, int sm) = nullptr;
  // linear-k tangent fields at a.Tl (4 per point, FP64)
  cudaError_t (*coef_lineark)(const CellArgs<double> &, double *out, int geo, cudaStream_t,
                              int sm) = nullptr;
  // the register-resident operator kernel exists for this degree (FP64 / FP32)
  bool v2_d = false, v2_f = false;
  // a.dst += diagonal of the FP32 Picard operator (conductivity field a.kq); same degrees
  cudaError_t (*diag_picard)(const CellArgs<float> &, int geo, cudaStream_t, int sm) = nullptr;
  // a.dst += the FP32 Picard operator on the tensor cores (uniform box, FE_Q(3) only; gmat:
  // the 128 KB of optc::build_gmat in device memory, err: raised on a timed-out wait)
  cudaError_t (*vmult_picard_tc)(const CellArgs<float> &, const float *gmat, int *err,
                                 cudaStream_t, int sm) = nullptr;
  // a.dst += the FP32 Picard operator with a.src in the cell-row layout (FE_Q(3) only)
  cudaError_t (*vmult_picard_rows)(const CellArgs<float> &, int geo, cudaStream_t,
                                   int sm) = nullptr;
};

DegreeTable degree_table_2();
DegreeTable degree_table_3();
DegreeTable degree_table_4();
DegreeTable degree_table_5();
DegreeTable degree_table_6();
DegreeTable degree_table_7();

}  // namespace mpdg
