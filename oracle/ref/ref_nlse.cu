// Runs the reference's own NLSE device code, compiled from its sources
// (device/include/nlse_dev.hpp: NLSESolverDevice with step = Strang SS2,
// step_sewi = SEWI, apply_bc, store_snapshot_online; matfunc_complex.hpp and
// lanczos_complex.hpp: the complex Lanczos matrix functions with cuBLAS and
// cuSOLVER Zheevd; boundaries.cuh: the ghost copies). Test infrastructure: the
// tests compare the oracle and the engine with it.
//
// The solver class takes its operator as an Eigen sparse matrix; Eigen is not
// installed here, so oracle/ref/eigen_stub/Eigen/Sparse supplies the five
// members the class reads, over the caller's CSR arrays (L itself, positive,
// nlse_cubic_driver_2d.cpp:94-97). The driver loop is restated from
// nlse_cubic_driver_2d.cpp:103-110 (and its SEWI / 3-D siblings), whose files
// need Eigen for their host vectors: snapshot 0 stored before the loop, then
// for i = 1..nt-1 the step (which stores a snapshot when i % freq == 0, SEWI
// only for i > 1) followed by the boundary copy, with dt_i = (0, T/nt).
// Square and cubic grids only, as the class (nlse_dev.hpp:133-140).
#include <complex>
#include <cstdint>
#include <vector>

#include <Eigen/Sparse>

#include "nlse_dev.hpp"

extern "C" int ref_nlse_run(int32_t dim, int32_t sewi, int32_t nx, const int32_t *row_ptr, const int32_t *col_ind,
                            const double *vals_c, int32_t nnz, int32_t k, const double *u0_c, const double *m,
                            double dt, int32_t nt, int32_t ns, double *traj_c, double *loop_ms) {
  if ((dim != 2 && dim != 3) || nx < 3 || k < 2 || nt < 1 || ns < 1 || nt < ns) return -3;
  const uint32_t n = (uint32_t)nx * (uint32_t)nx * (dim == 3 ? (uint32_t)nx : 1u);
  if (row_ptr[0] != 0 || row_ptr[n] != nnz) return -3;
  const Eigen::SparseMatrix<std::complex<double>> L((long)n, (long)nnz, row_ptr, col_ind,
                                                    reinterpret_cast<const std::complex<double> *>(vals_c));
  std::complex<double> *out = reinterpret_cast<std::complex<double> *>(traj_c);
  const std::complex<double> dti(0, dt);
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  int rc = 0;
  try {
    device::NLSESolverDevice::Parameters params((uint32_t)ns, (uint32_t)(nt / ns), (uint32_t)k);
    device::NLSESolverDevice solver(L, reinterpret_cast<const std::complex<double> *>(u0_c), m, dim == 3, params);
    solver.store_snapshot_online(out);
    cudaDeviceSynchronize();
    cudaEventRecord(ev[0], 0);
    for (uint32_t i = 1; i < (uint32_t)nt; ++i) {
      if (sewi)
        solver.step_sewi(dti, i, out);
      else
        solver.step(dti, i, out);
      solver.apply_bc();
    }
    cudaEventRecord(ev[1], 0);
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = -1;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    if (loop_ms) *loop_ms = ms;
  } catch (...) {  // the reference's error checks throw (pragmas.hpp, nlse_dev.hpp:199-202)
    rc = -2;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return rc;
}
