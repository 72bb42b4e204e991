// Device-side arithmetic of the explicit FV residual path.
//
// Every function follows the reference's CPU code operation by operation (same association
// order, same constants as the reference's macros expand them), so that, compiled with
// --fmad=false, each result is bit-identical to the reference built with -ffp-contract=off.
// IEEE double +, -, *, /, sqrt are correctly rounded on both sides.
//
// Macro constants of include/definitions.h:63-65 as the preprocessor expands them:
//   gamma_M_1 -> (1.4 - 1.0)            gamma1 * x -> 1.4 / (1.4 - 1.0) * x
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace cfdb {

constexpr double kGamma = 1.4;
constexpr double kGM1 = 1.4 - 1.0;               // gamma_M_1 and (gamma - 1.0)
constexpr double kGamma1 = 1.4 / (1.4 - 1.0);    // gamma1 (left operand of a product)

struct Prim {  // the five primitive slots the fluxes read: Primitive_Cells[c][0,1,2,4,5]
  double rho, u, v, p, a;
};

// Calculate_Primitive_Variables, src/Basic_Functions.cpp:100-156 (slots 0,1,2,4,5).
// Returns false when the sound speed is NaN (the reference exits there, :151-155).
__host__ __device__ inline bool eos_prim(double U0, double U1, double U2, double U3, Prim &q) {
  double Rho = U0;
  double inv = 1.0 / Rho;
  double v1 = U1 * inv;
  double v2 = U2 * inv;
  if (fabs(v1) <= 1e-10) v1 = 0.0;
  if (fabs(v2) <= 1e-10) v2 = 0.0;
  double vmag = (v1 * v1 + v2 * v2);
  double P = kGM1 * (U3 - 0.5 * Rho * vmag);
  double C = sqrt(kGamma * P * inv);
  q.rho = Rho;
  q.u = v1;
  q.v = v2;
  q.p = P;
  q.a = C;
  return !(C != C);
}

// Calculate_Face_Average_Flux, src/Average_Interface_Flux.cpp:20-82 (wall flag is never set on
// the reference path, src/Initialize.cpp:100).
template <typename T>
__device__ __forceinline__ void average_flux(const T rL, const T uL, const T vL, const T pL, const T rR, const T uR,
                                             const T vR, const T pR, const T nx, const T ny, const T dl, T F[4]) {
  const T g1 = T(kGamma1);
  T VnL = (uL * nx + vL * ny);
  T VnR = (uR * nx + vR * ny);
  T VmL = T(0.5) * (uL * uL + vL * vL);
  T VmR = T(0.5) * (uR * uR + vR * vR);
  T VnLdl = VnL * dl;
  T VnRdl = VnR * dl;
  T FL0 = rL * VnLdl, FL1 = rL * uL * VnLdl + pL * nx * dl, FL2 = rL * vL * VnLdl + pL * ny * dl,
    FL3 = (g1 * pL + rL * VmL) * VnLdl;
  T FR0 = rR * VnRdl, FR1 = rR * uR * VnRdl + pR * nx * dl, FR2 = rR * vR * VnRdl + pR * ny * dl,
    FR3 = (g1 * pR + rR * VmR) * VnRdl;
  F[0] = T(0.5) * (FL0 + FR0);
  F[1] = T(0.5) * (FL1 + FR1);
  F[2] = T(0.5) * (FL2 + FR2);
  F[3] = T(0.5) * (FL3 + FR3);
}

// The wave-decomposition tail shared by ROE and ROE_2O (src/Roe_Scheme.cpp:193-228, :376-423):
// eigenvalues with Harten's fix delta = 0.1*a_Roe on the acoustic waves, right eigenvectors,
// D = 0.5*sum|l|a r*dl.  eflin > 0 (no reference counterpart; the gradient-MUSCL form's option
// against the carbuncle) also fixes the two linear waves, |Un| below eflin*a_Roe.
template <typename T>
__device__ __forceinline__ void roe_tail(const T Ru, const T Rv, const T RH, const T RVm, const T Ra, const T RoeRho,
                                         const T Un, const T Ut, const T dP, const T dRho, const T dUn, const T dUt,
                                         const T nx, const T ny, const T dl, T D[4], const T eflin = T(0.0)) {
  T R11 = T(1.0), R12 = Ru - nx * Ra, R13 = Rv - ny * Ra, R14 = RH - Ra * Un;
  T R21 = T(1.0), R22 = Ru, R23 = Rv, R24 = RVm;
  T R31 = T(0.0), R32 = -ny, R33 = nx, R34 = Ut;
  T R41 = T(1.0), R42 = Ru + nx * Ra, R43 = Rv + ny * Ra, R44 = RH + Ra * Un;
  T Term2 = T(1.0) / (Ra * Ra);
  T a1 = T(0.5) * Term2 * (dP - RoeRho * Ra * dUn);
  T a2 = dRho - Term2 * dP;
  T a3 = RoeRho * dUt;
  T a4 = T(0.5) * Term2 * (dP + RoeRho * Ra * dUn);
  T L1 = fabs(Un - Ra), L2 = fabs(Un), L3 = fabs(Un), L4 = fabs(Un + Ra);
  T ef = T(0.1) * Ra;
  if (L1 < ef) L1 = T(0.5) * (L1 * L1 / ef + ef);
  if (L4 < ef) L4 = T(0.5) * (L4 * L4 / ef + ef);
  if (eflin > T(0.0)) {
    const T el = eflin * Ra;
    if (L2 < el) {
      L2 = T(0.5) * (L2 * L2 / el + el);
      L3 = L2;
    }
  }
  D[0] = T(0.5) * (L1 * a1 * R11 + L2 * a2 * R21 + L3 * a3 * R31 + L4 * a4 * R41) * dl;
  D[1] = T(0.5) * (L1 * a1 * R12 + L2 * a2 * R22 + L3 * a3 * R32 + L4 * a4 * R42) * dl;
  D[2] = T(0.5) * (L1 * a1 * R13 + L2 * a2 * R23 + L3 * a3 * R33 + L4 * a4 * R43) * dl;
  D[3] = T(0.5) * (L1 * a1 * R14 + L2 * a2 * R24 + L3 * a3 * R34 + L4 * a4 * R44) * dl;
}

// ROE, src/Roe_Scheme.cpp:6-256.  `degenerate` is the precomputed |n| < 1e-12 test (:71-76);
// a ghost neighbour has already been replaced by the cell itself (:79-84) by the caller.
template <typename T>
__device__ __forceinline__ void roe_1o(const T rL, const T uL, const T vL, const T pL, const T cL, const T rR,
                                       const T uR, const T vR, const T pR, const T cR, const T nx, const T ny,
                                       const T dl, bool degenerate, T D[4], const T eflin = T(0.0)) {
  D[0] = D[1] = D[2] = D[3] = T(0.0);
  if (degenerate) return;
  if (rL <= T(0.0) || pL <= T(0.0) || cL <= T(0.0)) return;
  T VmL = T(0.5) * (uL * uL + vL * vL);
  T HL = ((cL * cL) / T(kGM1)) + VmL;
  if (rR <= T(0.0) || pR <= T(0.0) || cR <= T(0.0)) return;
  T VmR = T(0.5) * (uR * uR + vR * vR);
  T HR = ((cR * cR) / T(kGM1)) + VmR;
  T sL = sqrt(rL), sR = sqrt(rR);
  T Term1 = T(1.0) / (sL + sR);
  T RoeRho = sqrt(rL * rR);
  T Ru = Term1 * (uR * sR + uL * sL);
  T Rv = Term1 * (vR * sR + vL * sL);
  T RH = Term1 * (HR * sR + HL * sL);
  T RVm = T(0.5) * (Ru * Ru + Rv * Rv);
  T Ra = sqrt(T(kGM1) * (RH - RVm));
  if (Ra <= T(0.0)) {
    Ra = T(0.5) * (cL + cR);
    if (Ra <= T(0.0)) return;
  }
  T Un = nx * Ru + ny * Rv;
  T Ut = -ny * Ru + nx * Rv;
  T du = (uR - uL), dv = (vR - vL), dP = (pR - pL), dRho = (rR - rL);
  T dUn = nx * du + ny * dv;
  T dUt = -ny * du + nx * dv;
  roe_tail<T>(Ru, Rv, RH, RVm, Ra, RoeRho, Un, Ut, dP, dRho, dUn, dUt, nx, ny, dl, D, eflin);
}

// ROE_2O, src/Roe_Scheme.cpp:257-447: Roe averages of the unreconstructed cell states, wave
// strengths from the limited conserved jump dU (Second_Order_Limiter).
template <typename T>
__device__ __forceinline__ void roe_2o(const T rL, const T uL, const T vL, const T pL, const T cL, const T rR,
                                       const T uR, const T vR, const T pR, const T cR, const T nx, const T ny,
                                       const T dl, const T dU[4], T D[4]) {
  T VmL = T(0.5) * (uL * uL + vL * vL);
  T HL = ((cL * cL) / T(kGM1)) + VmL;
  T VmR = T(0.5) * (uR * uR + vR * vR);
  T HR = ((cR * cR) / T(kGM1)) + VmR;
  T sR = sqrt(rR), sL = sqrt(rL);
  T Term1 = T(1.0) / (sL + sR);
  T RoeRho = sqrt(rL * rR);
  T Ru = Term1 * (uR * sR + uL * sL);
  T Rv = Term1 * (vR * sR + vL * sL);
  T RH = Term1 * (HR * sR + HL * sL);
  T RVm = T(0.5) * (Ru * Ru + Rv * Rv);
  T Un = nx * Ru + ny * Rv;
  T Ut = -ny * Ru + nx * Rv;
  T Ra = sqrt(T(kGM1) * (RH - RVm));
  T du = dU[1] / RoeRho - dU[0] * Ru / (RoeRho * RoeRho);
  T dv = dU[2] / RoeRho - dU[0] * Rv / (RoeRho * RoeRho);
  T dE = dU[3] - T(0.5) * RoeRho * (T(2.0) * (Ru * du + Rv * dv) + du * du + dv * dv) - T(0.5) * dU[0] * RVm;
  T dP = T(kGM1) * dE;
  T dRho = dU[0];
  T dUn = nx * du + ny * dv;
  T dUt = -ny * du + nx * dv;
  roe_tail<T>(Ru, Rv, RH, RVm, Ra, RoeRho, Un, Ut, dP, dRho, dUn, dUt, nx, ny, dl, D);
}

// Maximum(a,b,c) / Maximum(a,b), src/Utility_Files.cpp:5-31.
template <typename T>
__device__ __forceinline__ T max3_ref(T a, T b, T c) {
  if ((a >= b) && (a >= c)) return a;
  if ((b >= a) && (b >= c)) return b;
  return c;
}
template <typename T>
__device__ __forceinline__ T max2_ref(T a, T b) {
  return (a >= b) ? a : b;
}

// LLF, src/LLF.cpp:8-83: 0.5 * max|lambda|*dl * (U_R - U_L) with U from U_Cells.
template <typename T>
__device__ __forceinline__ void llf_1o(const T uL, const T vL, const T cL, const T uR, const T vR, const T cR,
                                       const T UL[4], const T UR[4], const T nx, const T ny, const T dl, T D[4]) {
  T VnL = (uL * nx + vL * ny);
  T VnR = (uR * nx + vR * ny);
  T S0 = fabs(VnL - cL) * dl, S1 = fabs(VnL + cL) * dl, S2 = fabs(VnL) * dl;
  T S3 = fabs(VnR - cR) * dl, S4 = fabs(VnR + cR) * dl, S5 = fabs(VnR) * dl;
  T M1 = max3_ref<T>(S0, S1, S2);
  T M2 = max3_ref<T>(S3, S4, S5);
  T mev = max2_ref<T>(M1, M2);
  for (int k = 0; k < 4; k++) D[k] = T(0.5) * mev * (UR[k] - UL[k]);
}

// Sign(a), include/definitions.h:76.
template <typename T>
__device__ __forceinline__ int sign_ref(T a) {
  return (a > T(0.0)) - (a < T(0.0));
}

// Minimum(a,b,c), src/Utility_Files.cpp:15-23.
template <typename T>
__device__ __forceinline__ T min3_ref(T a, T b, T c) {
  if ((a <= b) && (a <= c)) return a;
  if ((b <= a) && (b <= c)) return b;
  return c;
}

// Jump of the interface flux F(q_R).n dl - F(q_L).n dl of the MOVERS family
// (src/MOVERS.cpp:114-117, src/RICCA.cpp:103-108, src/MOVERS_NWSC.cpp:80-83), in the reference's
// association order.  `plus_pl` is the sign the reference gives the left pressure term of the two
// momentum components: + in MOVERS, MOVERS_2O, RICCA, RICCA_2O and MOVERS_NWSC, - in
// MOVERS_NWSC_2O (src/MOVERS_NWSC.cpp:183-184).
template <typename T>
__device__ __forceinline__ void movers_flux_jump(const T rL, const T uL, const T vL, const T pL, const T rR,
                                                 const T uR, const T vR, const T pR, const T nx, const T ny,
                                                 const T dl, const T VnL, const T VnR, bool plus_pl, T dF[4]) {
  const T VmL = T(0.5) * (uL * uL + vL * vL);
  const T VmR = T(0.5) * (uR * uR + vR * vR);
  dF[0] = (rR * VnR - rL * VnL) * dl;
  if (plus_pl) {
    dF[1] = (rR * uR * VnR + pR * nx - rL * uL * VnL + pL * nx) * dl;
    dF[2] = (rR * vR * VnR + pR * ny - rL * vL * VnL + pL * ny) * dl;
  } else {
    dF[1] = (rR * uR * VnR + pR * nx - rL * uL * VnL - pL * nx) * dl;
    dF[2] = (rR * vR * VnR + pR * ny - rL * vL * VnL - pL * ny) * dl;
  }
  dF[3] = ((((pR / T(kGM1)) + rR * VmR) + pR) * VnR - (((pL / T(kGM1)) + rL * VmL) + pL) * VnL) * dl;
}

// Conserved jump rebuilt from the two cells' primitives (src/MOVERS.cpp:208-211, src/RICCA.cpp:96-100).
template <typename T>
__device__ __forceinline__ void prim_jump(const T rL, const T uL, const T vL, const T pL, const T rR, const T uR,
                                          const T vR, const T pR, T dU[4]) {
  dU[0] = rR - rL;
  dU[1] = rR * uR - rL * uL;
  dU[2] = rR * vR - rL * vL;
  dU[3] = ((pR / T(kGM1)) + T(0.5) * rR * (uR * uR + vR * vR)) - ((pL / T(kGM1)) + T(0.5) * rL * (uL * uL + vL * vL));
}

// Condition_For_MOVERS, src/MOVERS.cpp:19-43 (epsilon 1e-10).
template <typename T>
__device__ __forceinline__ T movers_alpha(const T dU, const T dF, const T Lmax, const T Lmin) {
  const T eps = T(1e-10);
  if (fabs(dF) < eps && fabs(dU) > eps) return T(0.0);
  if (fabs(dF) < eps && fabs(dU) < eps) return Lmin;
  if (fabs(dF) > eps && fabs(dU) > eps) {
    T A = fabs(dF / dU);
    if (A >= Lmax) A = T(sign_ref<T>(A)) * Lmax;
    else if (A <= Lmin) A = T(sign_ref<T>(A)) * Lmin;
    return A;
  }
  return Lmin;
}

// Entropy_Fix, src/MOVERS.cpp:7-17 (delta = 1.0 * L_Max).
template <typename T>
__device__ __forceinline__ T movers_entropy_fix(const T A, const T Lmax) {
  const T delta = T(1.0) * Lmax;
  if (fabs(A) < delta) return (A * A + delta * delta) / (T(2.0) * delta);
  return Lmax;
}

// MOVERS (src/MOVERS.cpp:45-167) and MOVERS_2O (:169-276): wave speeds |V.n -+ a| dl of both
// cells bound alpha = |dF/dU| between max-of-max and max-of-min; `single` (Is_MOVERS_1) uses the
// energy component's alpha for all four; `efix` (Enable_Entropy_Fix) smooths alpha below L_Max
// (all four components at first order, the energy one at second order).  At second order the
// reference keeps the unreconstructed primitive jump and zero sound speeds (its MOVERS_2O never
// sets C_L, C_R).  D = 0.5 alpha dU.
template <typename T, int ORDER>
__device__ __forceinline__ void movers_diss(const T rL, const T uL, const T vL, const T pL, const T cL0, const T rR,
                                            const T uR, const T vR, const T pR, const T cR0, const T UL[4],
                                            const T UR[4], const T nx, const T ny, const T dl, bool single, bool efix,
                                            T D[4]) {
  T dU[4];
  if (ORDER == 1) {
#pragma unroll
    for (int k = 0; k < 4; k++) dU[k] = UR[k] - UL[k];
  } else {
    prim_jump<T>(rL, uL, vL, pL, rR, uR, vR, pR, dU);
  }
  const T cL = ORDER == 1 ? cL0 : T(0.0), cR = ORDER == 1 ? cR0 : T(0.0);
  const T VnL = (uL * nx + vL * ny);
  const T VnR = (uR * nx + vR * ny);
  T dF[4];
  movers_flux_jump<T>(rL, uL, vL, pL, rR, uR, vR, pR, nx, ny, dl, VnL, VnR, true, dF);
  const T S0 = fabs(VnL - cL) * dl, S1 = fabs(VnL + cL) * dl, S2 = fabs(VnL) * dl;
  const T S3 = fabs(VnR - cR) * dl, S4 = fabs(VnR + cR) * dl, S5 = fabs(VnR) * dl;
  const T Lmax = max2_ref<T>(max3_ref<T>(S0, S1, S2), max3_ref<T>(S3, S4, S5));
  const T Lmin = max2_ref<T>(min3_ref<T>(S0, S1, S2), min3_ref<T>(S3, S4, S5));
  T A[4];
  A[3] = movers_alpha<T>(dU[3], dF[3], Lmax, Lmin);
  A[0] = A[1] = A[2] = A[3];
  if (!single) {
#pragma unroll
    for (int k = 0; k < 3; k++) A[k] = movers_alpha<T>(dU[k], dF[k], Lmax, Lmin);
  }
  if (efix) {
    if (ORDER == 1) {
#pragma unroll
      for (int k = 0; k < 3; k++) A[k] = movers_entropy_fix<T>(A[k], Lmax);
    }
    A[3] = movers_entropy_fix<T>(A[3], Lmax);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) D[k] = T(0.5) * A[k] * dU[k];
}

// RICCA (src/RICCA.cpp:61-116) and RICCA_2O (:129-199) with Condition_For_RICCA (:31-48):
// alpha = max|V.n| + sign(dP) sqrt(gamma p_I / rho_I), or the mean |V.n| where both jumps are
// below 1e-8; dP = |p_L - p_R| is zeroed below 1e-8 (the reference zeroes its variable in
// place, so it stays zero for the later components).  dU is the primitive-rebuilt jump at first
// order and the limited conserved jump `dU2` (Second_Order_Limiter) at second order.
// D = 0.5 alpha dl dU.
template <typename T, int ORDER>
__device__ __forceinline__ void ricca_diss(const T rL, const T uL, const T vL, const T pL, const T rR, const T uR,
                                           const T vR, const T pR, const T nx, const T ny, const T dl, const T dU2[4],
                                           T D[4]) {
  const T VnL = uL * nx + vL * ny;
  const T VnR = uR * nx + vR * ny;
  T dU[4];
  if (ORDER == 1) prim_jump<T>(rL, uL, vL, pL, rR, uR, vR, pR, dU);
  else {
#pragma unroll
    for (int k = 0; k < 4; k++) dU[k] = dU2[k];
  }
  T dF[4];
  movers_flux_jump<T>(rL, uL, vL, pL, rR, uR, vR, pR, nx, ny, dl, VnL, VnR, true, dF);
  T dP = fabs(pL - pR);
  const T PI = T(0.5) * (pL + pR);
  const T RI = T(0.5) * (rL + rR);
  if (dP < T(1e-8)) dP = T(0.0);
  const T aL = fabs(VnL), aR = fabs(VnR);
  const T Mx = (aL < aR) ? aR : aL;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    T A;
    if (fabs(dF[k]) < T(1e-8) && fabs(dU[k]) < T(1e-8)) A = T(0.5) * (aL + aR);
    else A = Mx + T(1.0) * T(sign_ref<T>(dP)) * sqrt(T(kGamma) * PI / RI);
    D[k] = T(0.5) * A * dl * dU[k];
  }
}

// MOVERS_NWSC (src/MOVERS_NWSC.cpp:23-107) and MOVERS_NWSC_2O (:109-202) with
// Condition_For_MOVERS_NWSC (:6-21): alpha_k = sign(dU_k) |dF_k| (0 across a discontinuity),
// pressure sensor 0.21 |dp / (2 p_I)|, D = 0.5 (sensor alpha + 0.5(|V_R.n dl| + |V_L.n dl|) dU).
// dU: conserved jump U_R - U_L at first order, the limited jump `dU2` at second order.
template <typename T, int ORDER>
__device__ __forceinline__ void nwsc_diss(const T rL, const T uL, const T vL, const T pL, const T rR, const T uR,
                                          const T vR, const T pR, const T UL[4], const T UR[4], const T nx, const T ny,
                                          const T dl, const T dU2[4], T D[4]) {
  const T VnL = (uL * nx + vL * ny);
  const T VnR = (uR * nx + vR * ny);
  T dU[4];
#pragma unroll
  for (int k = 0; k < 4; k++) dU[k] = ORDER == 1 ? UR[k] - UL[k] : dU2[k];
  T dF[4];
  movers_flux_jump<T>(rL, uL, vL, pL, rR, uR, vR, pR, nx, ny, dl, VnL, VnR, ORDER == 1, dF);
  T A[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (fabs(dF[k]) <= T(1e-8) && fabs(dU[k]) >= T(1e-8)) A[k] = T(0.0);
    else A[k] = T(sign_ref<T>(dU[k])) * fabs(dF[k]);
  }
  const T dP = pR - pL;
  const T PI = T(0.5) * (pR + pL);
  const T AP = T(0.5) * (fabs(VnR * dl) + fabs(VnL * dl));
  const T Sensor = T(0.21) * fabs(dP / (T(2.0) * PI));
#pragma unroll
  for (int k = 0; k < 4; k++) D[k] = T(0.5) * (Sensor * A[k] + AP * dU[k]);
}

// Limiter functions phi(a, b), r = a / b, as the reference's GPU limiter family defines them
// (CUDA_KERNELS/Limiter_Cuda_Kernels.cu:89-154): phi = 0 when |b| < 1e-12 or r <= 0, else
//   minmod min(r, 1); Van Leer 2r/(1+r); superbee max(min(2r,1), min(r,2)); Van Albada (r^2+r)/(r^2+1).
enum LimiterKind : int { LIM_REF_MINMOD = 0, LIM_MINMOD = 1, LIM_VANLEER = 2, LIM_SUPERBEE = 3, LIM_VANALBADA = 4 };

template <typename T>
__device__ __forceinline__ T phi_ab(int kind, T a, T b) {
  if (fabs(b) < T(1e-12)) return T(0.0);
  T r = a / b;
  if (r <= T(0.0)) return T(0.0);
  switch (kind) {
    case LIM_MINMOD: return fmin(r, T(1.0));
    case LIM_VANLEER: return T(2.0) * r / (T(1.0) + r);
    case LIM_SUPERBEE: return fmax(fmin(T(2.0) * r, T(1.0)), fmin(r, T(2.0)));
    case LIM_VANALBADA: {
      T r_sq = r * r;
      return (r_sq + r) / (r_sq + T(1.0));
    }
    default: return T(0.0);
  }
}

// The limited slope phi(a / b) * b of the gradient-MUSCL reconstruction (no reference
// counterpart), algebraically the phi forms above times b but with at most one division:
//   minmod  |a| < |b| ? a : b;   Van Leer 2ab / (a + b);
//   superbee sign(b) max(min(2|a|, |b|), min(|a|, 2|b|));   Van Albada b (a^2 + ab) / (a^2 + b^2);
// 0 when |b| < 1e-12 or ab <= 0 (r <= 0).  The face kernel evaluates eight of these per face, and
// FP64 division chains bound it.
template <typename T>
__device__ __forceinline__ T muscl_slope(int kind, T a, T b) {
  if (fabs(b) < T(1e-12)) return T(0.0);
  const T ab = a * b;
  if (ab <= T(0.0)) return T(0.0);
  switch (kind) {
    case LIM_MINMOD: return fabs(a) < fabs(b) ? a : b;
    case LIM_VANLEER: return T(2.0) * ab / (a + b);
    case LIM_SUPERBEE: {
      const T aa = fabs(a), bb = fabs(b);
      const T m = fmax(fmin(T(2.0) * aa, bb), fmin(aa, T(2.0) * bb));
      return b > T(0.0) ? m : -m;
    }
    case LIM_VANALBADA: {
      const T a2 = a * a;
      return b * (a2 + ab) / (a2 + b * b);
    }
    default: return T(0.0);
  }
}

// Limited slope of one variable on the reference's directional stencil (src/Limiters.cpp:109-134):
//   S1 = zeta*(q_c - q_N1)/d1 (across the face), S2 = zeta1*(q_N1 - q_N2)/d2 (beyond N1)
// Reference minmod (src/Limiters.cpp:58-63): 0.5*(sgn S1 + sgn S2)*min(|S1|,|S2|).
// phi forms: phi(S2, S1) * S1.
template <typename T>
__device__ __forceinline__ T limited_slope(int kind, T qc, T q1, T q2, T d1, T d2, T zeta, T zeta1) {
  T S1 = zeta * (qc - q1) / d1;
  T S2 = zeta1 * (q1 - q2) / d2;
  if (kind == LIM_REF_MINMOD) {
    T a1 = fabs(S1), b1 = fabs(S2);
    T m = (b1 < a1) ? b1 : a1;
    return T(0.5) * T(sign_ref<T>(S1) + sign_ref<T>(S2)) * m;
  }
  return phi_ab<T>(kind, S2, S1) * S1;
}

}  // namespace cfdb

namespace cfdb {

// AUSM face flux of Ausm_Flux (src/Ausm_Flux.cpp:36-160) from the two conserved states:
// velocities and pressure from U, Roe-averaged interface sound speed, M+/- and P+/- splittings,
// upwinded mass flux; F already multiplied by the face length.
template <typename T>
__device__ __forceinline__ void ausm_face(const T UL[4], const T UR[4], const T nx, const T ny, const T area, T F[4]) {
  const T rho_L = UL[0], rhou_L = UL[1], rhov_L = UL[2], rhoE_L = UL[3];
  const T u_L = rhou_L / rho_L, v_L = rhov_L / rho_L;
  const T p_L = T(kGM1) * (rhoE_L - T(0.5) * rho_L * (u_L * u_L + v_L * v_L));
  const T H_L = (rhoE_L + p_L) / rho_L;
  const T rho_R = UR[0], rhou_R = UR[1], rhov_R = UR[2], rhoE_R = UR[3];
  const T u_R = rhou_R / rho_R, v_R = rhov_R / rho_R;
  const T p_R = T(kGM1) * (rhoE_R - T(0.5) * rho_R * (u_R * u_R + v_R * v_R));
  const T H_R = (rhoE_R + p_R) / rho_R;
  const T Vn_L = u_L * nx + v_L * ny, Vn_R = u_R * nx + v_R * ny;
  const T sqrt_rho_L = sqrt(rho_L), sqrt_rho_R = sqrt(rho_R);
  const T inv_sqrt_sum = T(1.0) / (sqrt_rho_L + sqrt_rho_R);
  const T u_roe = (sqrt_rho_L * u_L + sqrt_rho_R * u_R) * inv_sqrt_sum;
  const T v_roe = (sqrt_rho_L * v_L + sqrt_rho_R * v_R) * inv_sqrt_sum;
  const T H_roe = (sqrt_rho_L * H_L + sqrt_rho_R * H_R) * inv_sqrt_sum;
  const T a_roe = sqrt(T(kGM1) * (H_roe - T(0.5) * (u_roe * u_roe + v_roe * v_roe)));
  const T M_L = Vn_L / a_roe, M_R = Vn_R / a_roe;
  T M_plus, M_minus, P_plus, P_minus;
  if (fabs(M_L) >= T(1.0)) M_plus = (M_L > T(0.0)) ? M_L : T(0.0);
  else M_plus = T(0.25) * (M_L + T(1.0)) * (M_L + T(1.0));
  if (fabs(M_R) >= T(1.0)) M_minus = (M_R < T(0.0)) ? M_R : T(0.0);
  else M_minus = T(-0.25) * (M_R - T(1.0)) * (M_R - T(1.0));
  const T M_interface = M_plus + M_minus;
  if (fabs(M_L) >= T(1.0)) P_plus = (M_L > T(0.0)) ? T(1.0) : T(0.0);
  else P_plus = T(0.25) * (M_L + T(1.0)) * (M_L + T(1.0)) * (T(2.0) - M_L);
  if (fabs(M_R) >= T(1.0)) P_minus = (M_R < T(0.0)) ? T(1.0) : T(0.0);
  else P_minus = T(0.25) * (M_R - T(1.0)) * (M_R - T(1.0)) * (T(2.0) + M_R);
  const T p_interface = P_plus * p_L + P_minus * p_R;
  if (M_interface >= T(0.0)) {
    const T mass_flux = M_interface * a_roe * rho_L;
    F[0] = mass_flux * area;
    F[1] = (mass_flux * u_L + p_interface * nx) * area;
    F[2] = (mass_flux * v_L + p_interface * ny) * area;
    F[3] = mass_flux * H_L * area;
  } else {
    const T mass_flux = M_interface * a_roe * rho_R;
    F[0] = mass_flux * area;
    F[1] = (mass_flux * u_R + p_interface * nx) * area;
    F[2] = (mass_flux * v_R + p_interface * ny) * area;
    F[3] = mass_flux * H_R * area;
  }
}

// HLLC face flux of the reference's GPU kernel (CUDA_KERNELS/HLLC_LLF_Flux_Cuda_Kernels.cu:25-204):
// normal renormalised, Davis/Roe wave-speed bounds, contact speed S*, star states; zero flux for
// a degenerate normal or a non-physical state; F multiplied by the face length.  q = (rho, u, v,
// p, a) with the conserved U of the same cell.
template <typename T>
__device__ __forceinline__ void hllc_face(const T qL[5], const T UL[4], const T qR[5], const T UR[4], T nx, T ny,
                                          const T area, T F[4]) {
  F[0] = F[1] = F[2] = F[3] = T(0.0);
  const T normal_mag = sqrt(nx * nx + ny * ny);
  if (normal_mag < T(1e-14)) return;
  nx /= normal_mag;
  ny /= normal_mag;
  const T rho_L = qL[0], u_L = qL[1], v_L = qL[2], P_L = qL[3], a_L = qL[4];
  if (rho_L <= T(0.0) || P_L <= T(0.0) || a_L <= T(0.0)) return;
  const T rho_R = qR[0], u_R = qR[1], v_R = qR[2], P_R = qR[3], a_R = qR[4];
  if (rho_R <= T(0.0) || P_R <= T(0.0) || a_R <= T(0.0)) return;
  const T un_L = nx * u_L + ny * v_L, un_R = nx * u_R + ny * v_R;
  const T sqrt_rho_L = sqrt(rho_L), sqrt_rho_R = sqrt(rho_R);
  const T a_roe = (a_L * sqrt_rho_L + a_R * sqrt_rho_R) / (sqrt_rho_L + sqrt_rho_R);
  const T u_roe = (u_L * sqrt_rho_L + u_R * sqrt_rho_R) / (sqrt_rho_L + sqrt_rho_R);
  const T v_roe = (v_L * sqrt_rho_L + v_R * sqrt_rho_R) / (sqrt_rho_L + sqrt_rho_R);
  const T un_roe = nx * u_roe + ny * v_roe;
  const T S_L = fmin(un_L - a_L, un_roe - a_roe);
  const T S_R = fmax(un_R + a_R, un_roe + a_roe);
  const T numer = P_R - P_L + rho_L * un_L * (S_L - un_L) - rho_R * un_R * (S_R - un_R);
  const T denom = rho_L * (S_L - un_L) - rho_R * (S_R - un_R);
  T S_star;
  if (fabs(denom) > T(1e-14)) S_star = numer / denom;
  else S_star = T(0.5) * (un_L + un_R);
  T flux[4];
  if (S_L >= T(0.0)) {
    flux[0] = rho_L * un_L;
    flux[1] = rho_L * u_L * un_L + P_L * nx;
    flux[2] = rho_L * v_L * un_L + P_L * ny;
    flux[3] = (UL[3] + P_L) * un_L;
  } else if (S_R <= T(0.0)) {
    flux[0] = rho_R * un_R;
    flux[1] = rho_R * u_R * un_R + P_R * nx;
    flux[2] = rho_R * v_R * un_R + P_R * ny;
    flux[3] = (UR[3] + P_R) * un_R;
  } else {
    const bool left = S_star >= T(0.0);
    const T rho = left ? rho_L : rho_R, u = left ? u_L : u_R, v = left ? v_L : v_R, P = left ? P_L : P_R;
    const T *U = left ? UL : UR;
    const T S_K = left ? S_L : S_R;
    const T un = nx * u + ny * v;
    const T FK[4] = {rho * un, rho * u * un + P * nx, rho * v * un + P * ny, (U[3] + P) * un};
    const T factor = rho * (S_K - un) / (S_K - S_star);
    const T Us[4] = {factor, factor * (u + (S_star - un) * nx), factor * (v + (S_star - un) * ny),
                     factor * (U[3] / rho + (S_star - un) * (S_star + P / (rho * (S_K - un))))};
#pragma unroll
    for (int i = 0; i < 4; i++) flux[i] = FK[i] + S_K * (Us[i] - U[i]);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) F[i] = flux[i] * area;
}


// AUSM face flux of the reference's GPU kernel ausm_flux_kernel
// (CUDA_KERNELS/Flux_Calculations_Cuda_Kernels.cu:11-113), 2-D: its third velocity and normal
// components are zero and kept in the expressions, so the arithmetic is the kernel's own.  Its
// macros expand to gamma 1.4 and R 287.5; T = P/(rho R), a = sqrt(gamma R T); the interface Mach
// number upwinds the convected part, the split pressures are added.
template <typename T>
__device__ __forceinline__ T ausm_gpu_mplus(T M) {
  if (M >= T(1.0)) return M;
  else if (M > T(-1.0) && M < T(1.0)) return T(0.25) * (M + T(1.0)) * (M + T(1.0));
  else return T(0.0);
}
template <typename T>
__device__ __forceinline__ T ausm_gpu_mminus(T M) {
  if (M >= T(1.0)) return T(0.0);
  else if (M > T(-1.0) && M < T(1.0)) return T(-0.25) * (M - T(1.0)) * (M - T(1.0));
  else return M;
}
template <typename T>
__device__ __forceinline__ T ausm_gpu_pplus(T P, T M) {
  if (M >= T(1.0)) return P;
  else if (M > T(-1.0) && M < T(1.0)) return (P * T(0.25)) * (M + T(1.0)) * (M + T(1.0)) * (T(2.0) - M);
  else return T(0.0);
}
template <typename T>
__device__ __forceinline__ T ausm_gpu_pminus(T P, T M) {
  if (M >= T(1.0)) return T(0.0);
  else if (M > T(-1.0) && M < T(1.0)) return (P * T(0.25)) * (M - T(1.0)) * (M - T(1.0)) * (T(2.0) + M);
  else return P;
}

template <typename T>
__device__ __forceinline__ void ausm_gpu_face(const T UL[4], const T UR[4], const T nx, const T ny, const T area,
                                              T F[4]) {
  const T g = T(1.4), Rg = T(287.5), gm1 = T(1.4 - 1.0), gR = T(1.4 * 287.5), zero = T(0.0);
  const T rho_L = UL[0];
  const T u_L = UL[1] / rho_L, v_L = UL[2] / rho_L, w_L = zero / rho_L;
  const T E_L = UL[3];
  const T P_L = gm1 * (E_L - T(0.5) * rho_L * (u_L * u_L + v_L * v_L + w_L * w_L));
  const T T_L = P_L / (rho_L * Rg);
  const T a_L = sqrt(gR * T_L);
  const T rho_R = UR[0];
  const T u_R = UR[1] / rho_R, v_R = UR[2] / rho_R, w_R = zero / rho_R;
  const T E_R = UR[3];
  const T P_R = gm1 * (E_R - T(0.5) * rho_R * (u_R * u_R + v_R * v_R + w_R * w_R));
  const T T_R = P_R / (rho_R * Rg);
  const T a_R = sqrt(gR * T_R);
  (void)g;
  const T nz = zero;
  const T V_L = u_L * nx + v_L * ny + w_L * nz;
  const T V_R = u_R * nx + v_R * ny + w_R * nz;
  const T M_L = V_L / a_L, M_R = V_R / a_R;
  const T Mi = ausm_gpu_mplus(M_L) + ausm_gpu_mminus(M_R);
  const T Pi = ausm_gpu_pplus(P_L, M_L) + ausm_gpu_pminus(P_R, M_R);
  const T H_L = (E_L + P_L) / rho_L, H_R = (E_R + P_R) / rho_R;
  if (Mi > T(0)) {
    F[0] = area * rho_L * a_L * Mi;
    F[1] = area * (rho_L * a_L * Mi * u_L + Pi * nx);
    F[2] = area * (rho_L * a_L * Mi * v_L + Pi * ny);
    F[3] = area * rho_L * a_L * Mi * H_L;
  } else {
    F[0] = area * rho_R * a_R * Mi;
    F[1] = area * (rho_R * a_R * Mi * u_R + Pi * nx);
    F[2] = area * (rho_R * a_R * Mi * v_R + Pi * ny);
    F[3] = area * rho_R * a_R * Mi * H_R;
  }
}

// Far-field (Riemann-invariant) boundary state of the reference's GPU kernel farfield_bc_kernel
// (CUDA_KERNELS/Boundary_Conditions_Cuda_Kernels.cu:257-325, with calculate_primitive_device
// :28-49 and its GAMMA_VAL 1.4, GAMMA_M1 0.4): the interior conserved state Ui, the outward unit
// normal (nx, ny) and the free stream give the conserved boundary state G, written to the ghost.
__device__ __forceinline__ void farfield_state(const double Ui[4], double nx, double ny, double rho_inf,
                                               double u_inf, double v_inf, double p_inf, double G[4]) {
  const double GV = 1.4, GM = 0.4;
  double rho = Ui[0];
  if (rho < 1e-12) rho = 1e-12;
  const double u = Ui[1] / rho, v = Ui[2] / rho, E = Ui[3];
  const double kinetic_energy = 0.5 * rho * (u * u + v * v);
  double p = GM * (E - kinetic_energy);
  if (p < 1e-12) p = 1e-12;
  const double rho_i = rho, u_i = u, v_i = v, p_i = p;
  const double a_i = sqrt(GV * p_i / rho_i);
  const double a_inf = sqrt(GV * p_inf / rho_inf);
  const double v_n_i = u_i * nx + v_i * ny;
  const double v_n_inf = u_inf * nx + v_inf * ny;
  const double R_plus = v_n_i + 2.0 * a_i / GM;
  const double R_minus = v_n_inf - 2.0 * a_inf / GM;
  const double v_n_b = 0.5 * (R_plus + R_minus);
  double a_b = 0.25 * GM * (R_plus - R_minus);
  if (a_b < 1e-12) a_b = 1e-12;
  double rho_b, u_b, v_b, p_b;
  if (v_n_b >= 0.0) {
    const double s_i = p_i / pow(rho_i, GV);
    rho_b = pow(a_b * a_b / (GV * s_i), 1.0 / GM);
    u_b = u_i + (v_n_b - v_n_i) * nx;
    v_b = v_i + (v_n_b - v_n_i) * ny;
    p_b = rho_b * a_b * a_b / GV;
  } else {
    const double s_inf = p_inf / pow(rho_inf, GV);
    rho_b = pow(a_b * a_b / (GV * s_inf), 1.0 / GM);
    u_b = u_inf + (v_n_b - v_n_inf) * nx;
    v_b = v_inf + (v_n_b - v_n_inf) * ny;
    p_b = rho_b * a_b * a_b / GV;
  }
  const double v_mag_sq = u_b * u_b + v_b * v_b;
  G[0] = rho_b;
  G[1] = rho_b * u_b;
  G[2] = rho_b * v_b;
  G[3] = p_b / GM + 0.5 * rho_b * v_mag_sq;
}

// Fixed-pressure exit of the reference (Subsonic_Exit_Boundary_Condition,
// src/Exit_Boundary_Conditions.cpp:8-66; present in the reference but not called by its
// Apply_Boundary_Conditions): linearised characteristic face state with the prescribed pressure
// P_f and reference density and sound speed 1, mirrored into the ghost.  Inputs: the interior
// cell's primitives (rho, u, v, p), its rho*E (primitive slot 6 = conserved energy of the state
// the primitives were computed from) and the face's outward normal.
__device__ __forceinline__ void fixed_p_exit_state(double Rho, double v1, double v2, double P, double rho_Et,
                                                   double n1, double n2, double P_f, double G[4]) {
  const double Rho_o = 1.0, C_o = 1.0;
  const double temp = (P - P_f) / (Rho_o * C_o * C_o);
  const double rho_f = Rho - temp * Rho_o;
  const double u_f = v1 + n1 * temp * C_o;
  const double v_f = v2 + n2 * temp * C_o;
  const double v_mag_f = 0.5 * (u_f * u_f + v_f * v_f);
  const double F0 = rho_f, F1 = rho_f * u_f, F2 = rho_f * v_f, F3 = ((P_f / (1.4 - 1.0)) + rho_f * v_mag_f);
  G[0] = 2.0 * F0 - Rho;
  G[1] = 2.0 * F1 - Rho * v1;
  G[2] = 2.0 * F2 - Rho * v2;
  G[3] = 2.0 * F3 - rho_Et;
}


// ---- WENO path (src/WENO2D.cpp), double precision, the reference's association order ----

// WENO_Reconstruction, src/WENO2D.cpp:9-85: fifth-order WENO value at a face from five cell
// values, shift 0 for the left and 1 for the right state.  The reference's pow(x, 2) calls are
// x*x here (its libm returns exactly that, checked on 2e8 samples); non-finite inputs or result
// fall back to the central value.
__device__ __forceinline__ double weno5(double a, double b, double c, double d, double e, int shift) {
  if (!isfinite(a) || !isfinite(b) || !isfinite(c) || !isfinite(d) || !isfinite(e)) return c;
  const double epsilon = 1e-6;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0;
  if (shift == 0) {
    d0 = 3.0 / 10.0;
    d1 = 6.0 / 10.0;
    d2 = 1.0 / 10.0;
    v2 = (2.0 * a - 7.0 * b + 11.0 * c) / 6.0;
    v1 = (-1.0 * b + 5.0 * c + 2.0 * d) / 6.0;
    v0 = (2.0 * c + 5.0 * d - 1.0 * e) / 6.0;
  } else if (shift == 1) {
    d0 = 1.0 / 10.0;
    d1 = 6.0 / 10.0;
    d2 = 3.0 / 10.0;
    v2 = (-1.0 * a + 5.0 * b + 2.0 * c) / 6.0;
    v1 = (2.0 * b + 5.0 * c - 1.0 * d) / 6.0;
    v0 = (11.0 * c - 7.0 * d + 2.0 * e) / 6.0;
  }
  const double s2a = a - 2.0 * b + c, s2b = a - 4.0 * b + 3.0 * c;
  const double s1a = b - 2.0 * c + d, s1b = b - d;
  const double s0a = c - 2.0 * d + e, s0b = 3.0 * c - 4.0 * d + e;
  const double b2 = (13.0 / 12.0) * (s2a * s2a) + (1.0 / 4.0) * (s2b * s2b);
  const double b1 = (13.0 / 12.0) * (s1a * s1a) + (1.0 / 4.0) * (s1b * s1b);
  const double b0 = (13.0 / 12.0) * (s0a * s0a) + (1.0 / 4.0) * (s0b * s0b);
  const double q0 = epsilon + b0, q1 = epsilon + b1, q2 = epsilon + b2;
  const double a0 = d0 / (q0 * q0);
  const double a1 = d1 / (q1 * q1);
  const double a2 = d2 / (q2 * q2);
  const double sum = a0 + a1 + a2;
  double U;
  if (sum < epsilon) {
    U = (v0 + v1 + v2) / 3.0;
  } else {
    const double w0 = a0 / sum, w1 = a1 / sum, w2 = a2 / sum;
    U = w0 * v0 + w1 * v1 + w2 * v2;
  }
  if (!isfinite(U)) U = c;
  return U;
}

// Get_LR, src/WENO2D.cpp:87-199: conserved-to-characteristic matrix L and its inverse IL (column
// major, [i + 4 j]) from the Roe-type average of the two face cells' (rho, u, v, a).  Returns
// false where the reference would stop on a NaN entry.
__device__ __forceinline__ bool weno_lr(double dL, double uL, double vL, double aL, double dR, double uR, double vR,
                                        double aR, double nx, double ny, double L[16], double IL[16]) {
  const double sqrt_dL = sqrt(fmax(dL, 1e-14)), sqrt_dR = sqrt(fmax(dR, 1e-14));
  const double denom = sqrt_dL + sqrt_dR;
  double u_RL, v_RL, a_RL;
  if (denom < 1e-14) {
    u_RL = 0.5 * (uL + uR);
    v_RL = 0.5 * (vL + vR);
    a_RL = 0.5 * (aL + aR);
  } else {
    u_RL = (uL * sqrt_dL + uR * sqrt_dR) / denom;
    v_RL = (vL * sqrt_dL + vR * sqrt_dR) / denom;
    a_RL = (aL * sqrt_dL + aR * sqrt_dR) / denom;
  }
  const double vn = (u_RL * nx + v_RL * ny);
  const double ek = 0.5 * (u_RL * u_RL + v_RL * v_RL);
  const double h = (a_RL * a_RL / kGM1) + ek;
  if (a_RL < 1e-14) a_RL = 1e-14;
  const double t1 = 0.5 / (a_RL * a_RL);
  const double t2 = kGM1 * t1;
  L[0] = 1.0 - 2.0 * t2 * ek;
  L[4] = 2.0 * t2 * u_RL;
  L[8] = 2.0 * t2 * v_RL;
  L[12] = -2.0 * t2;
  L[1] = v_RL * nx - u_RL * ny;
  L[5] = ny;
  L[9] = -nx;
  L[13] = 0.0;
  L[2] = t2 * ek - a_RL * vn * t1;
  L[6] = -t2 * u_RL + a_RL * t1 * nx;
  L[10] = -t2 * v_RL + a_RL * t1 * ny;
  L[14] = t2;
  L[3] = t2 * ek + a_RL * vn * t1;
  L[7] = -t2 * u_RL - a_RL * t1 * nx;
  L[11] = -t2 * v_RL - a_RL * t1 * ny;
  L[15] = t2;
  IL[0] = 1.0;
  IL[4] = 0.0;
  IL[8] = 1.0;
  IL[12] = 1.0;
  IL[1] = u_RL;
  IL[5] = ny;
  IL[9] = u_RL + a_RL * nx;
  IL[13] = u_RL - a_RL * nx;
  IL[2] = v_RL;
  IL[6] = -nx;
  IL[10] = v_RL + a_RL * ny;
  IL[14] = v_RL - a_RL * ny;
  IL[3] = ek;
  IL[7] = u_RL * ny - v_RL * nx;
  IL[11] = h + a_RL * vn;
  IL[15] = h - a_RL * vn;
  bool ok = true;
#pragma unroll
  for (int i = 0; i < 16; i++) ok = ok && !(L[i] != L[i]) && !(IL[i] != IL[i]);
  return ok;
}

// MatVecMul, src/WENO2D.cpp:201-214: B = A x with A column major, each row summed from 0.0.
__device__ __forceinline__ void weno_matvec(const double A[16], const double x[4], double B[4]) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++) s += A[i + 4 * j] * x[j];
    B[i] = s;
  }
}

// Calculate_Face_WENO_Flux, src/WENO2D.cpp:458-562 (the wall-face flag is never set on the
// reference path): average of the two face states' fluxes minus 0.5 * max|lambda| dl (UR - UL).
// F receives Average - Dissipative; returns false when a face state has a NaN sound speed.
__device__ __forceinline__ bool weno_face_flux(const double UL[4], const double UR[4], double nx, double ny, double dl,
                                               double F[4]) {
  Prim L, R;
  const bool okL = eos_prim(UL[0], UL[1], UL[2], UL[3], L);
  const bool okR = eos_prim(UR[0], UR[1], UR[2], UR[3], R);
  const double Vdotn_L = (L.u * nx + L.v * ny), Vdotn_R = (R.u * nx + R.v * ny);
  const double Vmag_L = 0.5 * (L.u * L.u + L.v * L.v), Vmag_R = 0.5 * (R.u * R.u + R.v * R.v);
  double FL[4], FR[4];
  FL[0] = L.rho * Vdotn_L * dl;
  FL[1] = L.rho * L.u * Vdotn_L * dl + L.p * nx * dl;
  FL[2] = L.rho * L.v * Vdotn_L * dl + L.p * ny * dl;
  FL[3] = (kGamma1 * L.p + L.rho * Vmag_L) * Vdotn_L * dl;
  FR[0] = R.rho * Vdotn_R * dl;
  FR[1] = R.rho * R.u * Vdotn_R * dl + R.p * nx * dl;
  FR[2] = R.rho * R.v * Vdotn_R * dl + R.p * ny * dl;
  FR[3] = (kGamma1 * R.p + R.rho * Vmag_R) * Vdotn_R * dl;
  double C_L = L.a, C_R = R.a;
  if (C_L < 1e-14) C_L = 1e-14;
  if (C_R < 1e-14) C_R = 1e-14;
  const double S0 = fabs(Vdotn_L - C_L) * dl, S1 = fabs(Vdotn_L + C_L) * dl, S2 = fabs(Vdotn_L) * dl;
  const double S3 = fabs(Vdotn_R - C_R) * dl, S4 = fabs(Vdotn_R + C_R) * dl, S5 = fabs(Vdotn_R) * dl;
  const double mx = max2_ref<double>(max3_ref<double>(S0, S1, S2), max3_ref<double>(S3, S4, S5));
#pragma unroll
  for (int i = 0; i < 4; i++) F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * mx * (UR[i] - UL[i]);
  return okL && okR;
}

}  // namespace cfdb
