// Test infrastructure only: C-linkage entries to the reference's own GPU kernels, compiled from
// the reference's CUDA_KERNELS/*.cu sources by oracle/Makefile (target refcuda) into
// oracle/_ref/librefcuda.so.  GPU tests use them as the checkers of the HLLC face flux, the phi
// limiters, the AUSM face flux, the far-field boundary state and the TVD-RK3 / RK4 stage updates,
// and time the reference's Roe and HLLC flux kernels beside this library's on the same GPU.
#include <vector>

#include "Advanced_Flux_Schemes_Cuda.h"

extern "C" int refcu_hllc_flux(const double *U, const double *P, const int *nbr, const double *normals,
                               const double *areas, double *flux, int num_cells) {
  cudaError_t e = launch_hllc_flux(U, P, nbr, normals, areas, flux, num_cells, 1.4, 256);
  if (e != cudaSuccess) return (int)e;
  return (int)cudaDeviceSynchronize();
}

// Launch only (no synchronisation), on the legacy default stream as the reference's wrappers
// launch: the same-box timing comparison brackets these with CUDA events.
extern "C" int refcu_hllc_flux_launch(const double *U, const double *P, const int *nbr, const double *normals,
                                      const double *areas, double *flux, int num_cells) {
  return (int)launch_hllc_flux(U, P, nbr, normals, areas, flux, num_cells, 1.4, 256);
}
extern "C" int refcu_roe_flux_launch(const double *U, const double *P, const int *nbr, const double *normals,
                                     const double *areas, double *flux, int num_cells) {
  return (int)launch_roe_flux(U, P, nbr, normals, areas, flux, num_cells, 1.4, 256);
}

// ---- Further checkers: host arrays in and out; the shim copies them to and from the device and
// runs the reference's own device functions / kernels on them (their sources compiled with
// --fmad=false, separate compilation, so the symbols below are the reference's).
#include "Boundary_Conditions_Cuda_Kernels.h"

extern __device__ double vanleer_limiter_device(double a, double b);     // Limiter_Cuda_Kernels.cu:116
extern __device__ double superbee_limiter_device(double a, double b);    // :130
extern __device__ double vanalbada_limiter_device(double a, double b);   // :146
__global__ void ausm_flux_kernel(const double *U_left, const double *U_right, const double *face_normals,
                                 const double *face_areas, double *fluxes, int num_faces);  // Flux_Calculations_Cuda_Kernels.cu:37
__global__ void tvd_rk3_kernel(double *U_cells, double *U_temp1, double *U_temp2, double *Net_Flux,
                               double *Viscous_Flux, double *Cell_Volumes, double dt, int num_cells,
                               int stage);  // Time_Integration_Cuda_Kernels.cu:94
__global__ void rk4_complete_kernel(double *U_cells, double *U_cells_temp, double *Net_Flux, double *Viscous_Flux,
                                    double *Cell_Volumes, double *Del2_Q, double *Del4_Q, double *Cell_Diagonal,
                                    double dt, double lambda, int num_cells, int stage);  // :11

namespace {
struct Dev {
  void *p[16];
  int n = 0;
  ~Dev() {
    for (int i = 0; i < n; i++) cudaFree(p[i]);
  }
  template <typename T>
  T *put(const T *h, size_t count) {
    void *d = nullptr;
    if (cudaMalloc(&d, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
    p[n++] = d;
    if (h) cudaMemcpy(d, h, count * sizeof(T), cudaMemcpyHostToDevice);
    else cudaMemset(d, 0, count * sizeof(T));
    return static_cast<T *>(d);
  }
};

__global__ void k_ref_limiter(int kind, const double *a, const double *b, int n, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (kind == 2) out[i] = vanleer_limiter_device(a[i], b[i]);
  else if (kind == 3) out[i] = superbee_limiter_device(a[i], b[i]);
  else out[i] = vanalbada_limiter_device(a[i], b[i]);
}
}  // namespace

// phi(a, b) of the reference's Van Leer (kind 2), Superbee (3) and Van Albada (4) device functions.
extern "C" int refcu_limiter(int kind, const double *a, const double *b, int n, double *out) {
  Dev d;
  double *da = d.put(a, n), *db = d.put(b, n), *dout = d.put<double>(nullptr, n);
  k_ref_limiter<<<(n + 255) / 256, 256>>>(kind, da, db, n, dout);
  cudaError_t e = cudaMemcpy(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost);
  return (int)(e != cudaSuccess ? e : cudaGetLastError());
}

// ausm_flux_kernel on n faces: UL, UR [n*5] (rho, rho u, rho v, rho w, E), normals [n*3], areas
// [n] -> fluxes [n*5].
extern "C" int refcu_ausm_flux(const double *UL, const double *UR, const double *normals, const double *areas,
                               int n, double *fluxes) {
  Dev d;
  double *dl = d.put(UL, 5 * (size_t)n), *dr = d.put(UR, 5 * (size_t)n), *dn = d.put(normals, 3 * (size_t)n),
         *da = d.put(areas, n), *df = d.put<double>(nullptr, 5 * (size_t)n);
  ausm_flux_kernel<<<(n + 255) / 256, 256>>>(dl, dr, dn, da, df, n);
  cudaError_t e = cudaMemcpy(fluxes, df, 5 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  return (int)(e != cudaSuccess ? e : cudaGetLastError());
}

// farfield_bc_kernel on n cells: U [n*4] is replaced by the boundary state computed from it, with
// face 0 of normals [n*8] as the boundary normal, free stream (rho, u, v, p).
extern "C" int refcu_farfield(double *U, const double *normals, int n, double rho_inf, double u_inf, double v_inf,
                              double p_inf) {
  Dev d;
  std::vector<int> list(n);
  for (int i = 0; i < n; i++) list[i] = i;
  double *dU = d.put(U, 4 * (size_t)n), *dn = d.put(normals, 8 * (size_t)n);
  int *dlist = d.put(list.data(), n);
  FarfieldCondition_GPU bc{rho_inf, u_inf, v_inf, p_inf, 0.0};
  farfield_bc_kernel<<<(n + 255) / 256, 256>>>(dU, dlist, dn, bc, n, 1.4);
  cudaError_t e = cudaMemcpy(U, dU, 4 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  return (int)(e != cudaSuccess ? e : cudaGetLastError());
}

// One stage of tvd_rk3_kernel (which = 3) or rk4_complete_kernel (which = 4; zero dissipation
// arrays and lambda) on n cells with 5-component rows; U, T1, T2 are updated in place as the
// kernel does (T2 unused by RK4).
extern "C" int refcu_rk_stage(int which, int stage, double *U, double *T1, double *T2, const double *net_flux,
                              const double *volumes, double dt, int n) {
  Dev d;
  const size_t n5 = 5 * (size_t)n;
  double *dU = d.put(U, n5), *d1 = d.put(T1, n5), *d2 = d.put(T2, n5), *dF = d.put(net_flux, n5);
  double *dV = d.put<double>(nullptr, n5), *dvol = d.put(volumes, n);
  if (which == 3) {
    tvd_rk3_kernel<<<(n + 255) / 256, 256>>>(dU, d1, d2, dF, dV, dvol, dt, n, stage);
  } else {
    double *z5a = d.put<double>(nullptr, n5), *z5b = d.put<double>(nullptr, n5), *z3 = d.put<double>(nullptr, 3 * (size_t)n);
    rk4_complete_kernel<<<(n + 255) / 256, 256>>>(dU, d1, dF, dV, dvol, z5a, z5b, z3, dt, 0.0, n, stage);
  }
  cudaError_t e = cudaMemcpy(U, dU, n5 * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(T1, d1, n5 * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(T2, d2, n5 * sizeof(double), cudaMemcpyDeviceToHost);
  return (int)(e != cudaSuccess ? e : cudaGetLastError());
}
