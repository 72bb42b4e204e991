// Test infrastructure only: C-linkage entry to the reference's own GPU flux kernels, compiled
// from the reference's CUDA_KERNELS/*.cu sources by oracle/Makefile (target refcuda) into
// oracle/_ref/librefcuda.so.  Used by a GPU test as the checker of the HLLC face flux.
#include "Advanced_Flux_Schemes_Cuda.h"

extern "C" int refcu_hllc_flux(const double *U, const double *P, const int *nbr, const double *normals,
                               const double *areas, double *flux, int num_cells) {
  cudaError_t e = launch_hllc_flux(U, P, nbr, normals, areas, flux, num_cells, 1.4, 256);
  if (e != cudaSuccess) return (int)e;
  return (int)cudaDeviceSynchronize();
}
