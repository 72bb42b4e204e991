/* Test infrastructure only: plain-C restatement of the reference's explicit FV residual/update
 * path (rameshkolluru43/CFD_Solver_withCUDA).  It is the checker for the CUDA library and is
 * never linked into it.  Each function names the reference file:line it restates; the
 * arithmetic keeps the reference's association order, and this file is compiled without FMA
 * contraction, so results are bit-identical to the reference built the same way. */
#include "cfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define GM1 (1.4 - 1.0)          /* gamma_M_1, include/definitions.h:64 */
#define G1 (1.4 / (1.4 - 1.0))   /* gamma1 as it expands in a product, include/definitions.h:65 */
#define RGC 287.0                /* R_GC, include/definitions.h:66 */

struct orc_state {
  int NP, NG, NT, NB;
  const int *nf, *nbr, *bnd;
  const double *nrm, *len, *ccd, *cvec, *area, *inva;
  orc_config c;
  double *U, *P, *R, *dt, *dU, *S1, *S2, *Racc, *dtk, *Urd, *G, *Ff;
  int *slot;
  double err[4], min_dt, dt_step, total_time;
  int iterations, bad_cell;
  int stage;   /* 0: flux of U^n, >0: a later stage of the current step */
};

/* Calculate_Primitive_Variables, src/Basic_Functions.cpp:162-219 (inviscid: mu = K = 0). */
static void eos(orc_state *s, int cell, const double *Uv, double *G) {
  double Rho = Uv[0];
  double inv = 1.0 / Rho;
  double v1 = Uv[1] * inv, v2 = Uv[2] * inv;
  if (fabs(v1) <= 1e-10) v1 = 0.0;
  if (fabs(v2) <= 1e-10) v2 = 0.0;
  double vmag = (v1 * v1 + v2 * v2);
  double Pr = GM1 * (Uv[3] - 0.5 * Rho * vmag);
  double T = (Pr * inv / RGC);
  double C = sqrt(1.4 * Pr * inv);
  double M = sqrt(vmag) / C;
  G[0] = Rho;
  G[1] = v1;
  G[2] = v2;
  G[3] = T;
  G[4] = Pr;
  G[5] = C;
  G[6] = Uv[3];
  G[7] = M;
  G[8] = 0.0;
  G[9] = 0.0;
  G[10] = Pr * pow((1.0 + 0.5 * GM1 * M * M), G1);
  if (isnan(C) && (s->bad_cell < 0 || cell < s->bad_cell)) s->bad_cell = cell;
}

orc_state *orc_create(int NP, int NG, const int *nf, const int *nbr, const double *normals, const double *lengths,
                      const double *ccd, const double *cvec, const double *area, const double *inv_area, int NB,
                      const int *bnd, const orc_config *cfg) {
  orc_state *s = (orc_state *)calloc(1, sizeof(orc_state));
  s->NP = NP;
  s->NG = NG;
  s->NT = NP + NG;
  s->NB = NB;
  s->nf = nf;
  s->nbr = nbr;
  s->nrm = normals;
  s->len = lengths;
  s->ccd = ccd;
  s->cvec = cvec;
  s->area = area;
  s->inva = inv_area;
  s->bnd = bnd;
  s->c = *cfg;
  size_t NT = (size_t)s->NT;
  s->U = (double *)calloc(4 * NT, sizeof(double));
  s->Urd = (double *)calloc(4 * NT, sizeof(double));
  s->P = (double *)calloc(11 * NT, sizeof(double));
  s->R = (double *)calloc(4 * (size_t)NP, sizeof(double));
  s->dt = (double *)calloc(NT, sizeof(double));
  s->dU = (double *)calloc(4 * (size_t)NP, sizeof(double));
  s->S1 = (double *)calloc(4 * (size_t)NP, sizeof(double));
  s->S2 = (double *)calloc(4 * (size_t)NP, sizeof(double));
  s->Racc = (double *)calloc(4 * (size_t)NP, sizeof(double));
  s->dtk = (double *)calloc((size_t)NP, sizeof(double));
  s->G = (double *)calloc(8 * (size_t)NP, sizeof(double));
  s->Ff = (double *)calloc(16 * (size_t)NP, sizeof(double));
  s->slot = (int *)calloc(4 * (size_t)NP, sizeof(int));
  for (size_t g = (size_t)NP; g < NT; g++) s->dt[g] = 1e300; /* ghost del_t never written (harness fix) */
  s->bad_cell = -1;
  return s;
}

void orc_destroy(orc_state *s) {
  if (!s) return;
  free(s->U);
  free(s->Urd);
  free(s->P);
  free(s->R);
  free(s->dt);
  free(s->dU);
  free(s->S1);
  free(s->S2);
  free(s->Racc);
  free(s->dtk);
  free(s->G);
  free(s->Ff);
  free(s->slot);
  free(s);
}

/* Initialize_TestCase, src/Initialize_TestCase.cpp:36-58: U given, primitives from the EOS.
 * With n == NP the ghost rows copy their owner cell. */
void orc_set_state(orc_state *s, const double *U, int n) {
  for (int c = 0; c < n; c++) memcpy(s->U + 4 * (size_t)c, U + 4 * (size_t)c, 4 * sizeof(double));
  if (n == s->NP)
    for (int e = 0; e < s->NB; e++) memcpy(s->U + 4 * (size_t)s->bnd[4 * e + 3], U + 4 * (size_t)s->bnd[4 * e + 1], 4 * sizeof(double));
  for (int c = 0; c < s->NT; c++) eos(s, c, s->U + 4 * (size_t)c, s->P + 11 * (size_t)c);
  s->stage = 0;
}

/* The conserved state the limiter, LLF and the exit BC read: U_Cells (U^n on physical rows,
 * boundary values on ghost rows) for the reference integrator; the current stage state for the
 * stage-consistent integrators. */
/* The stage state of the current stage (> 0): RK4 forms keep it in S1, three-stage forms in
 * S1 then S2. */
static const double *stage_state(const orc_state *s) {
  const int integ = s->c.integrator;
  return (integ == 1 || integ == 4) ? s->S1 : (s->stage == 1 ? s->S1 : s->S2);
}

static const double *uread(orc_state *s) {
  if (s->c.integrator == 0 || s->stage == 0) return s->U;
  memcpy(s->Urd, s->U, 4 * (size_t)s->NT * sizeof(double));
  memcpy(s->Urd, stage_state(s), 4 * (size_t)s->NP * sizeof(double));
  return s->Urd;
}

/* Conserved state of cell c that the primitives were last computed from (U^n at stage 0, the
 * stage state after). */
static const double *ucur(const orc_state *s, int c) {
  return (s->stage == 0 ? s->U : stage_state(s)) + 4 * (size_t)c;
}

/* farfield_bc_kernel, CUDA_KERNELS/Boundary_Conditions_Cuda_Kernels.cu:257-325, with
 * calculate_primitive_device :28-49 (GAMMA_VAL 1.4, GAMMA_M1 0.4).  libm pow, so the result
 * is compared with the device's within a relative tolerance. */
static void farfield_state(const double *Ui, double nx, double ny, double rho_inf, double u_inf, double v_inf,
                           double p_inf, double *G) {
  const double GV = 1.4, GM = 0.4;
  double rho = Ui[0];
  if (rho < 1e-12) rho = 1e-12;
  double u = Ui[1] / rho, v = Ui[2] / rho, E = Ui[3];
  double kinetic_energy = 0.5 * rho * (u * u + v * v);
  double p = GM * (E - kinetic_energy);
  if (p < 1e-12) p = 1e-12;
  double a_i = sqrt(GV * p / rho), a_inf = sqrt(GV * p_inf / rho_inf);
  double v_n_i = u * nx + v * ny, v_n_inf = u_inf * nx + v_inf * ny;
  double R_plus = v_n_i + 2.0 * a_i / GM, R_minus = v_n_inf - 2.0 * a_inf / GM;
  double v_n_b = 0.5 * (R_plus + R_minus);
  double a_b = 0.25 * GM * (R_plus - R_minus);
  if (a_b < 1e-12) a_b = 1e-12;
  double rho_b, u_b, v_b, p_b;
  if (v_n_b >= 0.0) {
    double s_i = p / pow(rho, GV);
    rho_b = pow(a_b * a_b / (GV * s_i), 1.0 / GM);
    u_b = u + (v_n_b - v_n_i) * nx;
    v_b = v + (v_n_b - v_n_i) * ny;
  } else {
    double s_inf = p_inf / pow(rho_inf, GV);
    rho_b = pow(a_b * a_b / (GV * s_inf), 1.0 / GM);
    u_b = u_inf + (v_n_b - v_n_inf) * nx;
    v_b = v_inf + (v_n_b - v_n_inf) * ny;
  }
  p_b = rho_b * a_b * a_b / GV;
  G[0] = rho_b;
  G[1] = rho_b * u_b;
  G[2] = rho_b * v_b;
  G[3] = p_b / GM + 0.5 * rho_b * (u_b * u_b + v_b * v_b);
}

/* Apply_Boundary_Conditions, src/Boundary_Conditions.cpp:12-61 and the per-kind functions:
 * wall/symmetry src/Wall_Boundary_Conditions.cpp:8-53,79-124; supersonic inlet
 * src/Inlet_Boundary_Conditions.cpp:41-74; subsonic inlet :7-39; supersonic exit
 * src/Exit_Boundary_Conditions.cpp:68-94; subsonic exit :83-85 (empty).  Additive: total-(p,T)
 * inflow and static-pressure outflow. */
void orc_apply_bc(orc_state *s) {
  const double *Ur = uread(s);
  for (int e = 0; e < s->NB; e++) {
    const int kind = s->bnd[4 * e], c = s->bnd[4 * e + 1], f = s->bnd[4 * e + 2], g = s->bnd[4 * e + 3];
    const double *Pc = s->P + 11 * (size_t)c;
    double G[4];
    if (kind == 2 || kind == 3) {
      double v1 = Pc[1], v2 = Pc[2];
      double n1 = s->nrm[8 * c + 2 * f], n2 = s->nrm[8 * c + 2 * f + 1];
      double vdotn = (v1 * n1 + v2 * n2);
      double v1g = v1 - 2.0 * vdotn * n1;
      double v2g = v2 - 2.0 * vdotn * n2;
      double vmag = 0.5 * (v1g * v1g + v2g * v2g);
      G[0] = Pc[0];
      G[1] = Pc[0] * v1g;
      G[2] = Pc[0] * v2g;
      G[3] = ((Pc[4] / GM1) + Pc[0] * vmag);
    } else if (kind == 0) {
      double u = Pc[1], v = Pc[2];
      if (s->c.inlet_bc == 4) {
        farfield_state(ucur(s, c), s->nrm[8 * c + 2 * f], s->nrm[8 * c + 2 * f + 1], s->c.inlet_rho, s->c.inlet_u,
                       s->c.inlet_v, s->c.inlet_p, G);
      } else if (s->c.inlet_bc == 3) {
        /* Fully prescribed inflow (rho, u, v, p) (no reference counterpart). */
        const double r = s->c.inlet_rho, ui = s->c.inlet_u, vi = s->c.inlet_v;
        G[0] = r;
        G[1] = r * ui;
        G[2] = r * vi;
        G[3] = s->c.inlet_p / GM1 + 0.5 * r * (ui * ui + vi * vi);
      } else if (s->c.inlet_bc == 0) {
        double vmag = (u * u + v * v) * 0.5;
        G[0] = s->c.inlet_rho;
        G[1] = s->c.inlet_rho * u;
        G[2] = s->c.inlet_rho * v;
        G[3] = (s->c.inlet_p / GM1) + s->c.inlet_rho * vmag;
      } else if (s->c.inlet_bc == 1) {
        double Vm = 0.5 * (u * u + v * v);
        G[0] = s->c.inlet_rho;
        G[1] = s->c.inlet_rho * u;
        G[2] = s->c.inlet_rho * v;
        G[3] = (s->c.inlet_p / GM1) + s->c.inlet_rho * Vm * Vm;
      } else {
        /* Characteristic total-(p, T) inflow (no reference counterpart): R+ = Vn + 2a/(g-1)
         * from the interior, H0 = a0^2/(g-1) fixed, flow along the inward normal. */
        double n1 = s->nrm[8 * c + 2 * f], n2 = s->nrm[8 * c + 2 * f + 1];
        double Rp = (u * n1 + v * n2) + 2.0 * Pc[5] / GM1;
        double a0sq = 1.4 * s->c.r_gas * s->c.inlet_t0;
        double qa = (1.4 + 1.0) / GM1, qb = -2.0 * Rp, qc = 0.5 * GM1 * Rp * Rp - a0sq;
        double disc = qb * qb - 4.0 * qa * qc;
        double ab = (-qb + sqrt(disc > 0.0 ? disc : 0.0)) / (2.0 * qa);
        double vn = Rp - 2.0 * ab / GM1;
        if (vn > 0.0) vn = 0.0;
        double Tb = ab * ab / (1.4 * s->c.r_gas);
        double pb = s->c.inlet_p0 * pow(Tb / s->c.inlet_t0, 1.4 / GM1);
        double rb = pb / (s->c.r_gas * Tb);
        double ub = vn * n1, vb = vn * n2;
        G[0] = rb;
        G[1] = rb * ub;
        G[2] = rb * vb;
        G[3] = pb / GM1 + 0.5 * rb * (ub * ub + vb * vb);
      }
    } else {
      if (s->c.exit_bc == 1) continue;
      if (s->c.exit_bc == 0) {
        for (int k = 0; k < 4; k++) G[k] = Ur[4 * (size_t)c + k];
      } else if (s->c.exit_bc == 3) {
        /* Subsonic_Exit_Boundary_Condition, src/Exit_Boundary_Conditions.cpp:8-66, P_f = exit_p. */
        double Rho = Pc[0], v1 = Pc[1], v2 = Pc[2], P = Pc[4], rho_Et = Pc[6];
        double n1 = s->nrm[8 * c + 2 * f], n2 = s->nrm[8 * c + 2 * f + 1];
        double Rho_o = 1.0, C_o = 1.0, P_f = s->c.exit_p;
        double temp = (P - P_f) / (Rho_o * C_o * C_o);
        double rho_f = Rho - temp * Rho_o;
        double u_f = v1 + n1 * temp * C_o;
        double v_f = v2 + n2 * temp * C_o;
        double v_mag_f = 0.5 * (u_f * u_f + v_f * v_f);
        double UF[4] = {rho_f, rho_f * u_f, rho_f * v_f, ((P_f / GM1) + rho_f * v_mag_f)};
        G[0] = 2.0 * UF[0] - Rho;
        G[1] = 2.0 * UF[1] - Rho * v1;
        G[2] = 2.0 * UF[2] - Rho * v2;
        G[3] = 2.0 * UF[3] - rho_Et;
      } else {
        double n1 = s->nrm[8 * c + 2 * f], n2 = s->nrm[8 * c + 2 * f + 1];
        double vn = Pc[1] * n1 + Pc[2] * n2;
        double pb = (vn < Pc[5]) ? s->c.exit_p : Pc[4];
        G[0] = Pc[0];
        G[1] = Pc[0] * Pc[1];
        G[2] = Pc[0] * Pc[2];
        G[3] = pb / GM1 + 0.5 * Pc[0] * (Pc[1] * Pc[1] + Pc[2] * Pc[2]);
      }
    }
    memcpy(s->U + 4 * (size_t)g, G, sizeof(G));
    eos(s, g, G, s->P + 11 * (size_t)g);
  }
}

/* Calculate_Face_Average_Flux, src/Average_Interface_Flux.cpp:20-82. */
static void avg_flux(const double *PL, const double *PR, double nx, double ny, double dl, double *F) {
  double Rho_L = PL[0], u_L = PL[1], v_L = PL[2], P_L = PL[4];
  double Rho_R = PR[0], u_R = PR[1], v_R = PR[2], P_R = PR[4];
  double Vdotn_L = (u_L * nx + v_L * ny), Vdotn_R = (u_R * nx + v_R * ny);
  double Vmag_L = 0.5 * (u_L * u_L + v_L * v_L), Vmag_R = 0.5 * (u_R * u_R + v_R * v_R);
  double a = Vdotn_L * dl, b = Vdotn_R * dl;
  double FL[4] = {Rho_L * a, Rho_L * u_L * a + P_L * nx * dl, Rho_L * v_L * a + P_L * ny * dl, (G1 * P_L + Rho_L * Vmag_L) * a};
  double FR[4] = {Rho_R * b, Rho_R * u_R * b + P_R * nx * dl, Rho_R * v_R * b + P_R * ny * dl, (G1 * P_R + Rho_R * Vmag_R) * b};
  for (int i = 0; i < 4; i++) F[i] = 0.5 * (FL[i] + FR[i]);
}

/* Eigen-decomposition tail of ROE / ROE_2O, src/Roe_Scheme.cpp:164-228 and :376-423. */
static void roe_tail(double Roe_u, double Roe_v, double Roe_H, double Roe_Vmag, double Roe_a, double Roe_Rho,
                     double Un, double Ut, double dP, double dRho, double dUn, double dUt, double nx, double ny,
                     double dl, double *D) {
  double R1[4] = {1.0, Roe_u - nx * Roe_a, Roe_v - ny * Roe_a, Roe_H - Roe_a * Un};
  double R2[4] = {1.0, Roe_u, Roe_v, Roe_Vmag};
  double R3[4] = {0.0, -ny, nx, Ut};
  double R4[4] = {1.0, Roe_u + nx * Roe_a, Roe_v + ny * Roe_a, Roe_H + Roe_a * Un};
  double Term2 = 1.0 / (Roe_a * Roe_a);
  double a1 = 0.5 * Term2 * (dP - Roe_Rho * Roe_a * dUn);
  double a2 = dRho - Term2 * dP;
  double a3 = Roe_Rho * dUt;
  double a4 = 0.5 * Term2 * (dP + Roe_Rho * Roe_a * dUn);
  double L1 = fabs(Un - Roe_a), L2 = fabs(Un), L3 = fabs(Un), L4 = fabs(Un + Roe_a);
  double ef = 0.1 * Roe_a;
  if (L1 < ef) L1 = 0.5 * (L1 * L1 / ef + ef);
  if (L4 < ef) L4 = 0.5 * (L4 * L4 / ef + ef);
  for (int k = 0; k < 4; k++) D[k] = 0.5 * (L1 * a1 * R1[k] + L2 * a2 * R2[k] + L3 * a3 * R3[k] + L4 * a4 * R4[k]) * dl;
}

/* ROE, src/Roe_Scheme.cpp:6-256. */
static void roe_1o(orc_state *s, int c, int N, int f, double *D) {
  D[0] = D[1] = D[2] = D[3] = 0.0;
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  if (sqrt(nx * nx + ny * ny) < 1e-12) return;
  if (N < 0 || N >= s->NP) N = c;
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double Rho_L = L[0], u_L = L[1], v_L = L[2], P_L = L[4], C_L = L[5];
  if (Rho_L <= 0.0 || P_L <= 0.0 || C_L <= 0.0) return;
  double Vmag_L = 0.5 * (u_L * u_L + v_L * v_L);
  double H_L = ((C_L * C_L) / (1.4 - 1.0)) + Vmag_L;
  double Rho_R = R[0], u_R = R[1], v_R = R[2], P_R = R[4], C_R = R[5];
  if (Rho_R <= 0.0 || P_R <= 0.0 || C_R <= 0.0) return;
  double Vmag_R = 0.5 * (u_R * u_R + v_R * v_R);
  double H_R = ((C_R * C_R) / (1.4 - 1.0)) + Vmag_R;
  double sL = sqrt(Rho_L), sR = sqrt(Rho_R);
  double Term1 = 1.0 / (sL + sR);
  double Roe_Rho = sqrt(Rho_L * Rho_R);
  double Roe_u = Term1 * (u_R * sR + u_L * sL);
  double Roe_v = Term1 * (v_R * sR + v_L * sL);
  double Roe_H = Term1 * (H_R * sR + H_L * sL);
  double Roe_Vmag = 0.5 * (Roe_u * Roe_u + Roe_v * Roe_v);
  double Roe_a = sqrt((1.4 - 1.0) * (Roe_H - Roe_Vmag));
  if (Roe_a <= 0.0) {
    Roe_a = 0.5 * (C_L + C_R);
    if (Roe_a <= 0.0) return;
  }
  double Un = nx * Roe_u + ny * Roe_v, Ut = -ny * Roe_u + nx * Roe_v;
  double du = (u_R - u_L), dv = (v_R - v_L), dP = (P_R - P_L), dRho = (Rho_R - Rho_L);
  double dUn = nx * du + ny * dv, dUt = -ny * du + nx * dv;
  roe_tail(Roe_u, Roe_v, Roe_H, Roe_Vmag, Roe_a, Roe_Rho, Un, Ut, dP, dRho, dUn, dUt, nx, ny, dl, D);
}

static int sgn(double a) { return (a > 0.0) - (a < 0.0); }

/* phi(a, b), r = a/b: the reference GPU limiter family, CUDA_KERNELS/Limiter_Cuda_Kernels.cu:89-154. */
static double phi_ab(int kind, double a, double b) {
  if (fabs(b) < 1e-12) return 0.0;
  double r = a / b;
  if (r <= 0.0) return 0.0;
  switch (kind) {
    case 1: return fmin(r, 1.0);
    case 2: return 2.0 * r / (1.0 + r);
    case 3: return fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0));
    case 4: {
      double r_sq = r * r;
      return (r_sq + r) / (r_sq + 1.0);
    }
    default: return 0.0;
  }
}

/* Slope limiting of Second_Order_Limiter, src/Limiters.cpp:58-63,109-134 (kind 0: the
 * reference 2-argument MinMod; kinds 1-4: phi(S2, S1) * S1). */
static double slope(int kind, double qc, double q1, double q2, double d1, double d2, double z, double z1) {
  double S1 = z * (qc - q1) / d1;
  double S2 = z1 * (q1 - q2) / d2;
  if (kind == 0) {
    double a1 = fabs(S1), b1 = fabs(S2);
    return 0.5 * (sgn(S1) + sgn(S2)) * ((b1 < a1) ? b1 : a1);
  }
  return phi_ab(kind, S2, S1) * S1;
}

/* Directional stencil of Second_Order_Limiter, src/Limiters.cpp:136-191. */
static void stencil(const orc_state *s, int c, int f, int *N1, int *N2, double *d1, double *d2) {
  const int NP = s->NP;
  if (s->nf[c] != 4) {
    *N1 = s->nbr[4 * c + f];
    *d1 = s->ccd[4 * c + f];
    if (*d1 <= 0.0) *d1 = 1.0;
    *N2 = *N1;
    *d2 = *d1;
    return;
  }
  *N1 = s->nbr[4 * c + f];
  *d1 = s->ccd[4 * c + f];
  if (f < 2) {
    *N2 = (*N1 >= NP) ? *N1 : s->nbr[4 * *N1 + f];
    *d2 = (*N1 >= NP) ? *d1 : s->ccd[4 * *N1 + f];
  } else {
    *N2 = s->nbr[4 * c + f - 2];
    *d2 = s->ccd[4 * c + f - 2];
  }
}

/* Second_Order_Limiter (src/Limiters.cpp:97-200) on conserved variables, or the same stencil on
 * (rho, u, v, p) of the stage primitives (additive), giving the conserved jump d_U. */
static void limited_jump(orc_state *s, const double *Ur, int c, int f, double *dU) {
  int N1, N2;
  double d1, d2;
  stencil(s, c, f, &N1, &N2, &d1, &d2);
  if (!s->c.reconstruct_primitive) {
    for (int k = 0; k < 4; k++) {
      double q1 = Ur[4 * (size_t)N1 + k], q2 = Ur[4 * (size_t)N2 + k], qc = Ur[4 * (size_t)c + k];
      double phi = slope(s->c.limiter, qc, q1, q2, d1, d2, s->c.zeta, s->c.zeta1);
      double VR = q1 + 0.5 * phi * d1;
      double VL = qc - 0.5 * phi * d1;
      dU[k] = VR - VL;
    }
  } else {
    static const int slot[4] = {0, 1, 2, 4};
    double qR[4], qL[4];
    for (int k = 0; k < 4; k++) {
      double qc = s->P[11 * (size_t)c + slot[k]], q1 = s->P[11 * (size_t)N1 + slot[k]], q2 = s->P[11 * (size_t)N2 + slot[k]];
      double phi = slope(s->c.limiter, qc, q1, q2, d1, d2, s->c.zeta, s->c.zeta1);
      qR[k] = q1 + 0.5 * phi * d1;
      qL[k] = qc - 0.5 * phi * d1;
    }
    dU[0] = qR[0] - qL[0];
    dU[1] = qR[0] * qR[1] - qL[0] * qL[1];
    dU[2] = qR[0] * qR[2] - qL[0] * qL[2];
    dU[3] = (qR[3] / GM1 + 0.5 * qR[0] * (qR[1] * qR[1] + qR[2] * qR[2])) -
            (qL[3] / GM1 + 0.5 * qL[0] * (qL[1] * qL[1] + qL[2] * qL[2]));
  }
}

/* ROE_2O, src/Roe_Scheme.cpp:257-447. */
static void roe_2o(orc_state *s, const double *Ur, int c, int N, int f, double *D) {
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double Rho_L = L[0], u_L = L[1], v_L = L[2], C_L = L[5];
  double Vmag_L = 0.5 * (u_L * u_L + v_L * v_L), H_L = ((C_L * C_L) / (1.4 - 1.0)) + Vmag_L;
  double Rho_R = R[0], u_R = R[1], v_R = R[2], C_R = R[5];
  double Vmag_R = 0.5 * (u_R * u_R + v_R * v_R), H_R = ((C_R * C_R) / (1.4 - 1.0)) + Vmag_R;
  double sR = sqrt(Rho_R), sL = sqrt(Rho_L);
  double Term1 = 1.0 / (sL + sR);
  double Roe_Rho = sqrt(Rho_L * Rho_R);
  double Roe_u = Term1 * (u_R * sR + u_L * sL);
  double Roe_v = Term1 * (v_R * sR + v_L * sL);
  double Roe_H = Term1 * (H_R * sR + H_L * sL);
  double Roe_Vmag = 0.5 * (Roe_u * Roe_u + Roe_v * Roe_v);
  double Un = nx * Roe_u + ny * Roe_v, Ut = -ny * Roe_u + nx * Roe_v;
  double Roe_a = sqrt((1.4 - 1.0) * (Roe_H - Roe_Vmag));
  double d_U[4];
  limited_jump(s, Ur, c, f, d_U);
  double du = d_U[1] / Roe_Rho - d_U[0] * Roe_u / (Roe_Rho * Roe_Rho);
  double dv = d_U[2] / Roe_Rho - d_U[0] * Roe_v / (Roe_Rho * Roe_Rho);
  double dE = d_U[3] - 0.5 * Roe_Rho * (2.0 * (Roe_u * du + Roe_v * dv) + du * du + dv * dv) - 0.5 * d_U[0] * Roe_Vmag;
  double dP = (1.4 - 1.0) * dE, dRho = d_U[0];
  double dUn = nx * du + ny * dv, dUt = -ny * du + nx * dv;
  roe_tail(Roe_u, Roe_v, Roe_H, Roe_Vmag, Roe_a, Roe_Rho, Un, Ut, dP, dRho, dUn, dUt, nx, ny, dl, D);
}

static double max3(double a, double b, double c) {
  if ((a >= b) && (a >= c)) return a;
  if ((b >= a) && (b >= c)) return b;
  return c;
}

/* LLF, src/LLF.cpp:8-83. */
static void llf_1o(orc_state *s, const double *Ur, int c, int N, int f, double *D) {
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  double Vdotn_L = (L[1] * nx + L[2] * ny), Vdotn_R = (R[1] * nx + R[2] * ny);
  double S[6] = {fabs(Vdotn_L - L[5]) * dl, fabs(Vdotn_L + L[5]) * dl, fabs(Vdotn_L) * dl,
                 fabs(Vdotn_R - R[5]) * dl, fabs(Vdotn_R + R[5]) * dl, fabs(Vdotn_R) * dl};
  double M1 = max3(S[0], S[1], S[2]), M2 = max3(S[3], S[4], S[5]);
  double mev = (M1 >= M2) ? M1 : M2;
  for (int k = 0; k < 4; k++) D[k] = 0.5 * mev * (Ur[4 * (size_t)N + k] - Ur[4 * (size_t)c + k]);
}

static double min3(double a, double b, double c) {
  if ((a <= b) && (a <= c)) return a;
  if ((b <= a) && (b <= c)) return b;
  return c;
}

/* Interface flux jump of the MOVERS family, src/MOVERS.cpp:114-117 (plus_pl = 1: the reference's
 * "+ P_L * nx" / "+ P_L * ny" momentum terms of MOVERS, MOVERS_2O, RICCA, RICCA_2O, MOVERS_NWSC;
 * 0: the "- P_L" terms of MOVERS_NWSC_2O, src/MOVERS_NWSC.cpp:183-184). */
static void flux_jump(const double *L, const double *R, double nx, double ny, double dl, int plus_pl, double *dF) {
  double Rho_L = L[0], P_L = L[4], u_L = L[1], v_L = L[2];
  double Rho_R = R[0], P_R = R[4], u_R = R[1], v_R = R[2];
  double Vdotn_L = (u_L * nx + v_L * ny), Vdotn_R = (u_R * nx + v_R * ny);
  double Vmag_L = 0.5 * (u_L * u_L + v_L * v_L), Vmag_R = 0.5 * (u_R * u_R + v_R * v_R);
  dF[0] = (Rho_R * Vdotn_R - Rho_L * Vdotn_L) * dl;
  if (plus_pl) {
    dF[1] = (Rho_R * u_R * Vdotn_R + P_R * nx - Rho_L * u_L * Vdotn_L + P_L * nx) * dl;
    dF[2] = (Rho_R * v_R * Vdotn_R + P_R * ny - Rho_L * v_L * Vdotn_L + P_L * ny) * dl;
  } else {
    dF[1] = (Rho_R * u_R * Vdotn_R + P_R * nx - Rho_L * u_L * Vdotn_L - P_L * nx) * dl;
    dF[2] = (Rho_R * v_R * Vdotn_R + P_R * ny - Rho_L * v_L * Vdotn_L - P_L * ny) * dl;
  }
  dF[3] = ((((P_R / (1.4 - 1.0)) + Rho_R * Vmag_R) + P_R) * Vdotn_R -
           (((P_L / (1.4 - 1.0)) + Rho_L * Vmag_L) + P_L) * Vdotn_L) * dl;
}

/* Conserved jump from the two primitive states, src/MOVERS.cpp:208-211 / src/RICCA.cpp:96-100. */
static void prim_jump(const double *L, const double *R, double *dU) {
  double Rho_L = L[0], P_L = L[4], u_L = L[1], v_L = L[2];
  double Rho_R = R[0], P_R = R[4], u_R = R[1], v_R = R[2];
  dU[0] = Rho_R - Rho_L;
  dU[1] = Rho_R * u_R - Rho_L * u_L;
  dU[2] = Rho_R * v_R - Rho_L * v_L;
  dU[3] = ((P_R / (1.4 - 1.0)) + 0.5 * Rho_R * (u_R * u_R + v_R * v_R)) -
          ((P_L / (1.4 - 1.0)) + 0.5 * Rho_L * (u_L * u_L + v_L * v_L));
}

/* Condition_For_MOVERS, src/MOVERS.cpp:19-43. */
static void movers_condition(double d_U, double d_F, double L_Max, double L_Min, double *Alpha) {
  double epsilon = 1e-10;
  if (fabs(d_F) < epsilon && fabs(d_U) > epsilon) {
    *Alpha = 0.0;
  } else if (fabs(d_F) < epsilon && fabs(d_U) < epsilon) {
    *Alpha = L_Min;
  } else if (fabs(d_F) > epsilon && fabs(d_U) > epsilon) {
    *Alpha = fabs(d_F / d_U);
    if (*Alpha >= L_Max) *Alpha = sgn(*Alpha) * L_Max;
    else if (*Alpha <= L_Min) *Alpha = sgn(*Alpha) * L_Min;
  } else {
    *Alpha = L_Min;
  }
}

/* Entropy_Fix, src/MOVERS.cpp:7-17. */
static void movers_entropy_fix(double *Alpha, double L_Max) {
  double k = 1.0, delta = k * L_Max;
  if (fabs(*Alpha) < delta) *Alpha = (*Alpha * *Alpha + delta * delta) / (2.0 * delta);
  else *Alpha = L_Max;
}

/* MOVERS, src/MOVERS.cpp:45-167, and MOVERS_2O, :169-276 (primitive jump, sound speeds left at
 * the zero its globals were reset to, entropy fix on the energy component only). */
static void movers(orc_state *s, const double *Ur, int c, int N, int f, double *D) {
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  int second = s->c.is_second_order;
  double C_L = second ? 0.0 : L[5], C_R = second ? 0.0 : R[5];
  double d_U[4], d_F[4], A[4];
  if (!second)
    for (int k = 0; k < 4; k++) d_U[k] = Ur[4 * (size_t)N + k] - Ur[4 * (size_t)c + k];
  else
    prim_jump(L, R, d_U);
  flux_jump(L, R, nx, ny, dl, 1, d_F);
  double Vdotn_L = (L[1] * nx + L[2] * ny), Vdotn_R = (R[1] * nx + R[2] * ny);
  double S[6] = {fabs(Vdotn_L - C_L) * dl, fabs(Vdotn_L + C_L) * dl, fabs(Vdotn_L) * dl,
                 fabs(Vdotn_R - C_R) * dl, fabs(Vdotn_R + C_R) * dl, fabs(Vdotn_R) * dl};
  double Max1 = max3(S[0], S[1], S[2]), Max2 = max3(S[3], S[4], S[5]);
  double Lambda_Max = (Max1 >= Max2) ? Max1 : Max2;
  double Min1 = min3(S[0], S[1], S[2]), Min2 = min3(S[3], S[4], S[5]);
  double Lambda_Min = (Min1 >= Min2) ? Min1 : Min2;
  movers_condition(d_U[3], d_F[3], Lambda_Max, Lambda_Min, &A[3]);
  A[0] = A[1] = A[2] = A[3];
  if (!s->c.movers_single)
    for (int k = 0; k < 3; k++) movers_condition(d_U[k], d_F[k], Lambda_Max, Lambda_Min, &A[k]);
  if (s->c.movers_efix) {
    if (!second)
      for (int k = 0; k < 3; k++) movers_entropy_fix(&A[k], Lambda_Max);
    movers_entropy_fix(&A[3], Lambda_Max);
  }
  for (int k = 0; k < 4; k++) D[k] = 0.5 * A[k] * d_U[k];
}

/* RICCA, src/RICCA.cpp:61-116, and RICCA_2O, :129-199, with Condition_For_RICCA (:31-48); the
 * reference zeroes its dP in place, so a small dP stays zero for the later components. */
static void ricca(orc_state *s, const double *Ur, int c, int N, int f, double *D) {
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  double Vdotn_L = L[1] * nx + L[2] * ny, Vdotn_R = R[1] * nx + R[2] * ny;
  double d_U[4], d_F[4];
  prim_jump(L, R, d_U);
  flux_jump(L, R, nx, ny, dl, 1, d_F);
  double dP = fabs(L[4] - R[4]);
  double P_I = 0.5 * (L[4] + R[4]);
  double Rho_I = 0.5 * (L[0] + R[0]);
  if (s->c.is_second_order) limited_jump(s, Ur, c, f, d_U);
  for (int i = 0; i < 4; i++) {
    double epsilon = 1e-8, ita = 1.0, Alpha;
    if (dP < epsilon) dP = 0.0;
    double a = fabs(Vdotn_L), b = fabs(Vdotn_R);
    double Max = (a < b) ? b : a; /* std::max */
    if (fabs(d_F[i]) < epsilon && fabs(d_U[i]) < epsilon) Alpha = 0.5 * (fabs(Vdotn_L) + fabs(Vdotn_R));
    else Alpha = Max + ita * sgn(dP) * sqrt(1.4 * P_I / Rho_I);
    D[i] = 0.5 * Alpha * dl * d_U[i];
  }
}

/* MOVERS_NWSC, src/MOVERS_NWSC.cpp:23-107, and MOVERS_NWSC_2O, :109-202, with
 * Condition_For_MOVERS_NWSC (:6-21). */
static void movers_nwsc(orc_state *s, const double *Ur, int c, int N, int f, double *D) {
  const double *L = s->P + 11 * (size_t)c, *R = s->P + 11 * (size_t)N;
  double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
  int second = s->c.is_second_order;
  double Vdotn_L = (L[1] * nx + L[2] * ny), Vdotn_R = (R[1] * nx + R[2] * ny);
  double d_U[4], d_F[4], A[4];
  if (!second)
    for (int i = 0; i < 4; i++) d_U[i] = Ur[4 * (size_t)N + i] - Ur[4 * (size_t)c + i];
  flux_jump(L, R, nx, ny, dl, !second, d_F);
  if (second) limited_jump(s, Ur, c, f, d_U);
  for (int i = 0; i < 4; i++) {
    double epsilon = 1e-8;
    if (fabs(d_F[i]) <= epsilon && fabs(d_U[i]) >= epsilon) A[i] = 0.0;
    else A[i] = sgn(d_U[i]) * fabs(d_F[i]);
  }
  double d_P = R[4] - L[4];
  double P_I = 0.5 * (R[4] + L[4]);
  double Alpha_P = 0.5 * (fabs(Vdotn_R * dl) + fabs(Vdotn_L * dl));
  double Sensor = 0.21 * fabs(d_P / (2.0 * P_I));
  for (int i = 0; i < 4; i++) D[i] = 0.5 * (Sensor * A[i] + Alpha_P * d_U[i]);
}

/* Green-Gauss gradients of (rho, u, v, p) with ghost values on boundary faces (gradient MUSCL
 * form; no reference counterpart). */
static void muscl_gradients(orc_state *s) {
  static const int slot[4] = {0, 1, 2, 4};
  for (int c = 0; c < s->NP; c++) {
    double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int f = 0; f < s->nf[c]; f++) {
      int N = s->nbr[4 * c + f];
      double wx = s->nrm[8 * c + 2 * f] * s->len[4 * c + f], wy = s->nrm[8 * c + 2 * f + 1] * s->len[4 * c + f];
      for (int k = 0; k < 4; k++) {
        double qf = 0.5 * (s->P[11 * (size_t)c + slot[k]] + s->P[11 * (size_t)N + slot[k]]);
        g[2 * k] += qf * wx;
        g[2 * k + 1] += qf * wy;
      }
    }
    for (int k = 0; k < 8; k++) s->G[8 * (size_t)c + k] = g[k] * s->inva[c];
  }
}

#define REAL double
#define FN(x) x##_d
#define K(x) ((double)(x))
#define FABS fabs
#define SQRT sqrt
#define FMIN fmin
#define FMAX fmax
#include "face_flux.inc"
#undef REAL
#undef FN
#undef K
#undef FABS
#undef SQRT
#undef FMIN
#undef FMAX
#define REAL float
#define FN(x) x##_f
#define K(x) ((float)(x))
#define FABS fabsf
#define SQRT sqrtf
#define FMIN fminf
#define FMAX fmaxf
#include "face_flux.inc"
#undef REAL
#undef FN
#undef K
#undef FABS
#undef SQRT
#undef FMIN
#undef FMAX

/* Face-based gradient-MUSCL net flux: faces numbered in reference order (a face belongs to the
 * lower-numbered cell, a boundary face to its cell), each flux computed once from the owner's
 * side; every cell sums its faces in face order, +F as owner, -F as neighbour. */
static void muscl_net_flux(orc_state *s) {
  const int NP = s->NP;
  int nfaces = 0;
  for (int c = 0; c < NP; c++)
    for (int f = 0; f < s->nf[c]; f++) {
      int N = s->nbr[4 * c + f];
      if (N < NP && N < c) continue;
      double *F = s->Ff + 4 * (size_t)nfaces;
      if (s->c.precision == 1) face_flux_f(s, c, N, f, F);
      else face_flux_d(s, c, N, f, F);
      s->slot[4 * c + f] = nfaces;
      if (N < NP)
        for (int k = 0; k < s->nf[N]; k++)
          if (s->nbr[4 * N + k] == c) s->slot[4 * N + k] = -(nfaces + 1);
      nfaces++;
    }
  for (int c = 0; c < NP; c++) {
    double net[4] = {0.0, 0.0, 0.0, 0.0};
    for (int f = 0; f < s->nf[c]; f++) {
      int e = s->slot[4 * c + f];
      const double *F = s->Ff + 4 * (size_t)(e < 0 ? -e - 1 : e);
      for (int v = 0; v < 4; v++) net[v] += (e < 0) ? -F[v] : F[v];
    }
    memcpy(s->R + 4 * (size_t)c, net, sizeof(net));
  }
}

/* ---- WENO path, src/WENO2D.cpp ---- */

/* WENO_Reconstruction, src/WENO2D.cpp:9-85 (pow(x, 2) written x*x, which libm returns). */
static double weno5(double a, double b, double c, double d, double e, int shift) {
  if (!isfinite(a) || !isfinite(b) || !isfinite(c) || !isfinite(d) || !isfinite(e)) return c;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0, epsilon = 1e-6;
  if (shift == 0) {
    d0 = 3.0 / 10.0; d1 = 6.0 / 10.0; d2 = 1.0 / 10.0;
    v2 = (2.0 * a - 7.0 * b + 11.0 * c) / 6.0;
    v1 = (-1.0 * b + 5.0 * c + 2.0 * d) / 6.0;
    v0 = (2.0 * c + 5.0 * d - 1.0 * e) / 6.0;
  } else if (shift == 1) {
    d0 = 1.0 / 10.0; d1 = 6.0 / 10.0; d2 = 3.0 / 10.0;
    v2 = (-1.0 * a + 5.0 * b + 2.0 * c) / 6.0;
    v1 = (2.0 * b + 5.0 * c - 1.0 * d) / 6.0;
    v0 = (11.0 * c - 7.0 * d + 2.0 * e) / 6.0;
  }
  double s2a = a - 2.0 * b + c, s2b = a - 4.0 * b + 3.0 * c;
  double s1a = b - 2.0 * c + d, s1b = b - d;
  double s0a = c - 2.0 * d + e, s0b = 3.0 * c - 4.0 * d + e;
  double b2 = (13.0 / 12.0) * (s2a * s2a) + (1.0 / 4.0) * (s2b * s2b);
  double b1 = (13.0 / 12.0) * (s1a * s1a) + (1.0 / 4.0) * (s1b * s1b);
  double b0 = (13.0 / 12.0) * (s0a * s0a) + (1.0 / 4.0) * (s0b * s0b);
  double q0 = epsilon + b0, q1 = epsilon + b1, q2 = epsilon + b2;
  double a0 = d0 / (q0 * q0), a1 = d1 / (q1 * q1), a2 = d2 / (q2 * q2);
  double sum = a0 + a1 + a2, U;
  if (sum < epsilon) U = (v0 + v1 + v2) / 3.0;
  else U = (a0 / sum) * v0 + (a1 / sum) * v1 + (a2 / sum) * v2;
  if (!isfinite(U)) U = c;
  return U;
}

/* Get_LR, src/WENO2D.cpp:87-199 (column-major L and its inverse). */
static void weno_lr(const double *PL, const double *PR, double nx, double ny, double *L, double *IL) {
  double dL = PL[0], uL = PL[1], vL = PL[2], aL = PL[5], dR = PR[0], uR = PR[1], vR = PR[2], aR = PR[5];
  double sqrt_dL = sqrt(fmax(dL, 1e-14)), sqrt_dR = sqrt(fmax(dR, 1e-14)), denom = sqrt_dL + sqrt_dR;
  double u_RL, v_RL, a_RL;
  if (denom < 1e-14) {
    u_RL = 0.5 * (uL + uR); v_RL = 0.5 * (vL + vR); a_RL = 0.5 * (aL + aR);
  } else {
    u_RL = (uL * sqrt_dL + uR * sqrt_dR) / denom;
    v_RL = (vL * sqrt_dL + vR * sqrt_dR) / denom;
    a_RL = (aL * sqrt_dL + aR * sqrt_dR) / denom;
  }
  double vn = (u_RL * nx + v_RL * ny), ek = 0.5 * (u_RL * u_RL + v_RL * v_RL), h = (a_RL * a_RL / GM1) + ek;
  if (a_RL < 1e-14) a_RL = 1e-14;
  double t1 = 0.5 / (a_RL * a_RL), t2 = GM1 * t1;
  L[0] = 1.0 - 2.0 * t2 * ek; L[4] = 2.0 * t2 * u_RL; L[8] = 2.0 * t2 * v_RL; L[12] = -2.0 * t2;
  L[1] = v_RL * nx - u_RL * ny; L[5] = ny; L[9] = -nx; L[13] = 0.0;
  L[2] = t2 * ek - a_RL * vn * t1; L[6] = -t2 * u_RL + a_RL * t1 * nx; L[10] = -t2 * v_RL + a_RL * t1 * ny; L[14] = t2;
  L[3] = t2 * ek + a_RL * vn * t1; L[7] = -t2 * u_RL - a_RL * t1 * nx; L[11] = -t2 * v_RL - a_RL * t1 * ny; L[15] = t2;
  IL[0] = 1.0; IL[4] = 0.0; IL[8] = 1.0; IL[12] = 1.0;
  IL[1] = u_RL; IL[5] = ny; IL[9] = u_RL + a_RL * nx; IL[13] = u_RL - a_RL * nx;
  IL[2] = v_RL; IL[6] = -nx; IL[10] = v_RL + a_RL * ny; IL[14] = v_RL - a_RL * ny;
  IL[3] = ek; IL[7] = u_RL * ny - v_RL * nx; IL[11] = h + a_RL * vn; IL[15] = h - a_RL * vn;
}

static void weno_matvec(const double *A, const double *x, double *B) {
  for (int i = 0; i < 4; i++) {
    B[i] = 0.0;
    for (int j = 0; j < 4; j++) B[i] += A[i + 4 * j] * x[j];
  }
}

/* Calculate_Computational_Variables(cell, U), src/Basic_Functions.cpp:156-163. */
static void weno_cons(const orc_state *s, int i, double *U) {
  const double *P = s->P + 11 * (size_t)i;
  U[0] = P[0];
  U[1] = P[0] * P[1];
  U[2] = P[0] * P[2];
  U[3] = P[6];
}

/* Get_Reconstructed_U, src/WENO2D.cpp:216-243. */
static void weno_recon(const orc_state *s, int chr, const double *L, const double *IL, const int *ix, int lr,
                       double *U) {
  double v[5][4];
  for (int k = 0; k < 5; k++) weno_cons(s, ix[k], v[k]);
  if (chr) {
    double w[5][4], W[4];
    for (int k = 0; k < 5; k++) weno_matvec(L, v[k], w[k]);
    for (int i = 0; i < 4; i++) W[i] = weno5(w[0][i], w[1][i], w[2][i], w[3][i], w[4][i], lr);
    weno_matvec(IL, W, U);
  } else {
    for (int i = 0; i < 4; i++) U[i] = weno5(v[0][i], v[1][i], v[2][i], v[3][i], v[4][i], lr);
  }
}

/* Calculate_Face_WENO_Flux, src/WENO2D.cpp:458-562; F = Average - Dissipative. */
static void weno_face_flux(orc_state *s, int c, int N, const double *UL, const double *UR, double nx, double ny,
                           double dl, double *F) {
  double GL[11], GR[11];
  eos(s, c, UL, GL);
  eos(s, N, UR, GR);
  double Rho_L = GL[0], P_L = GL[4], u_L = GL[1], v_L = GL[2], C_L = GL[5];
  double Rho_R = GR[0], P_R = GR[4], u_R = GR[1], v_R = GR[2], C_R = GR[5];
  double Vdotn_L = (u_L * nx + v_L * ny), Vdotn_R = (u_R * nx + v_R * ny);
  double Vmag_L = 0.5 * (u_L * u_L + v_L * v_L), Vmag_R = 0.5 * (u_R * u_R + v_R * v_R);
  double FL[4], FR[4];
  FL[0] = Rho_L * Vdotn_L * dl;
  FL[1] = Rho_L * u_L * Vdotn_L * dl + P_L * nx * dl;
  FL[2] = Rho_L * v_L * Vdotn_L * dl + P_L * ny * dl;
  FL[3] = (G1 * P_L + Rho_L * Vmag_L) * Vdotn_L * dl;
  FR[0] = Rho_R * Vdotn_R * dl;
  FR[1] = Rho_R * u_R * Vdotn_R * dl + P_R * nx * dl;
  FR[2] = Rho_R * v_R * Vdotn_R * dl + P_R * ny * dl;
  FR[3] = (G1 * P_R + Rho_R * Vmag_R) * Vdotn_R * dl;
  if (C_L < 1e-14) C_L = 1e-14;
  if (C_R < 1e-14) C_R = 1e-14;
  double S0 = fabs(Vdotn_L - C_L) * dl, S1 = fabs(Vdotn_L + C_L) * dl, S2 = fabs(Vdotn_L) * dl;
  double S3 = fabs(Vdotn_R - C_R) * dl, S4 = fabs(Vdotn_R + C_R) * dl, S5 = fabs(Vdotn_R) * dl;
  double mx = max3(S0, S1, S2), m2 = max3(S3, S4, S5);
  if (!(mx >= m2)) mx = m2;
  for (int i = 0; i < 4; i++) F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * mx * (UR[i] - UL[i]);
}

/* Evaluate_Cell_Net_Flux_WENO, src/WENO2D.cpp:395-456 with the stencils of
 * WENO_Reconstruction_X (:245-393). */
static void weno_net_flux(orc_state *s, int c, double *net) {
  const int NP = s->NP, *nb = s->nbr + 4 * c;
  for (int k = 0; k < 4; k++) net[k] = 0.0;
  if (s->nf[c] != 4) return;
  int im1 = nb[0], ip1 = nb[1], jm1 = nb[2], jp1 = nb[3], im2, im3, ip2, ip3, jm2, jm3, jp2, jp3;
  if (im1 >= NP) { im2 = im1; im3 = im1; }
  else {
    im2 = s->nbr[4 * im1 + 0];
    if (im2 >= NP || im2 < 0) im3 = im2;
    else { im3 = s->nbr[4 * im2 + 0]; if (im3 < 0) im3 = im2; }
  }
  if (ip1 >= NP) { ip2 = ip1; ip3 = ip1; }
  else {
    ip2 = s->nbr[4 * ip1 + 1];
    if (ip2 >= NP || ip2 < 0) ip3 = ip2;
    else { ip3 = s->nbr[4 * ip2 + 1]; if (ip3 < 0) ip3 = ip2; }
  }
  if (jm1 >= NP) { jm2 = jm1; jm3 = jm1; }
  else { jm2 = s->nbr[4 * jm1 + 2]; jm3 = (jm2 >= NP) ? jm2 : s->nbr[4 * jm2 + 2]; }
  if (jp1 >= NP) { jp2 = jp1; jp3 = jp1; }
  else { jp2 = s->nbr[4 * jp1 + 3]; jp3 = (jp2 >= NP) ? jp2 : s->nbr[4 * jp2 + 3]; }
  const int st[4][2][5] = {{{im3, im2, im1, c, ip1}, {im2, im1, c, ip1, ip2}},
                           {{jm3, jm2, jm1, c, jp1}, {jm2, jm1, c, jp1, jp2}},
                           {{im2, im1, c, ip1, ip2}, {im1, c, ip1, ip2, ip3}},
                           {{jm2, jm1, c, jp1, jp2}, {jm1, c, jp1, jp2, jp3}}};
  const int N4[4] = {im1, ip1, jm1, jp1};
  for (int f = 0; f < 4; f++) {
    double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f];
    double L[16], IL[16], UL[4], UR[4], F[4];
    if (s->c.weno_char) weno_lr(s->P + 11 * (size_t)c, s->P + 11 * (size_t)N4[f], nx, ny, L, IL);
    weno_recon(s, s->c.weno_char, L, IL, st[f][0], 0, UL);
    weno_recon(s, s->c.weno_char, L, IL, st[f][1], 1, UR);
    weno_face_flux(s, c, N4[f], UL, UR, nx, ny, dl, F);
    for (int k = 0; k < 4; k++) net[k] += F[k];
  }
}

/* Evaluate_Cell_Net_Flux_1O/2O + Calculate_Flux_For_All_Faces, src/Net_Flux.cpp:7-129;
 * Inviscid_Time_Step, src/Time_Step.cpp:293-329. */
void orc_net_flux(orc_state *s) {
  const double *Ur = uread(s);
  int all_quads = 1;
  for (int c = 0; c < s->NP; c++) all_quads = all_quads && s->nf[c] == 4;
  /* Explicit_Method falls back to the 1O/2O residual on meshes with non-quad cells
   * (src/Numerical_Method.cpp:31-55); Runge_Kutta_Method does not. */
  const int weno = s->c.weno && (all_quads || s->c.time_accurate || s->c.integrator != 0);
  const int gmuscl = s->c.muscl && s->c.is_second_order && !weno;
  if (gmuscl) {
    muscl_gradients(s);
    muscl_net_flux(s);
  }
  for (int c = 0; c < s->NP; c++) {
    double net[4] = {0.0, 0.0, 0.0, 0.0};
    if (weno) weno_net_flux(s, c, net);
    for (int f = 0; f < s->nf[c] && !gmuscl && !weno; f++) {
      int N = s->nbr[4 * c + f];
      if (N < 0) continue;
      double A[4], D[4];
      if (s->c.dissipation_type == 6 || s->c.dissipation_type == 7) {
        /* Reference forms: Ausm_Flux (src/Ausm_Flux.cpp:26-169) from U_Cells, and the GPU HLLC
         * (CUDA_KERNELS/HLLC_LLF_Flux_Cuda_Kernels.cu:93-205); faces to ghost cells skipped. */
        if (N >= s->NP) continue;
        double nx = s->nrm[8 * c + 2 * f], ny = s->nrm[8 * c + 2 * f + 1], dl = s->len[4 * c + f], F[4];
        const double *UL = Ur + 4 * (size_t)c, *UR = Ur + 4 * (size_t)N;
        if (s->c.dissipation_type == 6) {
          ausm_face_d(UL, UR, nx, ny, dl, F);
        } else {
          const double *PL = s->P + 11 * (size_t)c, *PR = s->P + 11 * (size_t)N;
          double qL[5] = {PL[0], PL[1], PL[2], PL[4], PL[5]}, qR[5] = {PR[0], PR[1], PR[2], PR[4], PR[5]};
          hllc_face_d(qL, UL, qR, UR, nx, ny, dl, F);
        }
        for (int v = 0; v < 4; v++) net[v] += F[v];
        continue;
      }
      avg_flux(s->P + 11 * (size_t)c, s->P + 11 * (size_t)N, s->nrm[8 * c + 2 * f], s->nrm[8 * c + 2 * f + 1],
               s->len[4 * c + f], A);
      if (s->c.dissipation_type == 3 && !s->c.is_second_order) roe_1o(s, c, N, f, D);
      else if (s->c.dissipation_type == 3) roe_2o(s, Ur, c, N, f, D);
      else if (s->c.dissipation_type == 2) movers(s, Ur, c, N, f, D);
      else if (s->c.dissipation_type == 4) ricca(s, Ur, c, N, f, D);
      else if (s->c.dissipation_type == 5) movers_nwsc(s, Ur, c, N, f, D);
      else llf_1o(s, Ur, c, N, f, D);
      for (int v = 0; v < 4; v++) net[v] += A[v] - D[v];
    }
    if (!gmuscl) memcpy(s->R + 4 * (size_t)c, net, sizeof(net));
    const double u0 = s->P[11 * (size_t)c + 1], v0 = s->P[11 * (size_t)c + 2], a0 = s->P[11 * (size_t)c + 5];
    double denom = 0.0;
    for (int f = 0; f < s->nf[c]; f++) {
      double vn = u0 * s->nrm[8 * c + 2 * f] + v0 * s->nrm[8 * c + 2 * f + 1];
      denom += (fabs(vn) + a0) * s->len[4 * c + f];
    }
    s->dt[c] = (denom <= 0.0 || !isfinite(denom)) ? 0.0 : s->c.cfl * s->area[c] / denom;
  }
  /* get_Min_dt, src/Numerical_Method.cpp:322-330 (ghost del_t = 1e300). */
  double m = s->dt[0];
  for (int c = 1; c < s->NT; c++)
    if (s->dt[c] < m) m = s->dt[c];
  s->min_dt = m;
}

/* Lax_Fedrichs, src/Numerical_Method.cpp:459-481: the sequential in-place sweep over the cells
 * (get_Min_dt is the minimum of the last net-flux evaluation).  Returns -1 on a non-quad cell. */
int orc_lax_friedrichs(orc_state *s) {
  for (int c = 0; c < s->NP; c++)
    if (s->nf[c] != 4) return -1;
  double Dt = s->min_dt;
  for (int c = 0; c < s->NP; c++) {
    int N1 = s->nbr[4 * c], N2 = s->nbr[4 * c + 1], N3 = s->nbr[4 * c + 2], N4 = s->nbr[4 * c + 3];
    double inv_Area = s->inva[c];
    for (int k = 0; k < 4; k++)
      s->U[4 * (size_t)c + k] = 0.25 * (s->U[4 * (size_t)N1 + k] + s->U[4 * (size_t)N2 + k] + s->U[4 * (size_t)N3 + k] +
                                        s->U[4 * (size_t)N4 + k]) -
                                Dt * inv_Area * s->R[4 * (size_t)c + k];
  }
  return 0;
}

/* Explicit_Method, src/Numerical_Method.cpp:26-103.  Returns -1 when Min_dt <= 0. */
int orc_explicit(orc_state *s) {
  s->stage = 0;
  orc_net_flux(s);
  if (!(s->min_dt > 0.0)) return -1;
  for (int c = 0; c < s->NP; c++)
    for (int k = 0; k < 4; k++) s->dU[4 * c + k] = -s->min_dt * s->inva[c] * s->R[4 * c + k];
  return 0;
}

static void refresh_prims(orc_state *s, const double *src) {
  for (int c = 0; c < s->NP; c++) eos(s, c, src + 4 * (size_t)c, s->P + 11 * (size_t)c);
}

/* Runge_Kutta_Method, src/Numerical_Method.cpp:342-457 (integrator 0); stage-consistent SSP-RK3
 * with dt frozen per step (integrator 2); classical RK4 (integrator 1). */
void orc_rk(orc_state *s) {
  const int NP = s->NP, integ = s->c.integrator, lts = s->c.local_time_stepping;
  if (integ == 3 || integ == 4) {
    /* The reference's GPU kernels tvd_rk3_kernel (integrator 3) and rk4_complete_kernel
     * (integrator 4), CUDA_KERNELS/Time_Integration_Cuda_Kernels.cu:94-131 and :11-73 (its
     * dissipation terms are zero for the inviscid path), dt taken at the first stage.  The last
     * stage produces U^{n+1}; dU = U^{n+1} - U^n, and U^{n+1} is kept for orc_update. */
    const int ns = integ == 3 ? 3 : 4;
    for (int st = 0; st < ns; st++) {
      s->stage = st;
      if (st > 0) orc_apply_bc(s);
      orc_net_flux(s);
      if (st == 0) {
        s->dt_step = s->min_dt;
        memcpy(s->dtk, s->dt, (size_t)NP * sizeof(double));
      }
      for (int c = 0; c < NP; c++) {
        double dt = lts ? s->dtk[c] : s->dt_step, invA = s->inva[c];
        for (int k = 0; k < 4; k++) {
          size_t i = 4 * (size_t)c + k;
          double Un = s->U[i], Rk = s->R[i], nu;
          if (integ == 3) {
            if (st == 0) { s->S1[i] = Un - dt * invA * Rk; continue; }
            if (st == 1) { s->S2[i] = 0.25 * (3.0 * Un + s->S1[i] - dt * invA * Rk); continue; }
            nu = (1.0 / 3.0) * (Un + 2.0 * s->S2[i] - 2.0 * dt * invA * Rk);
          } else {
            if (st < 2) { s->S1[i] = Un - 0.5 * dt * invA * Rk; continue; }
            if (st == 2) { s->S1[i] = Un - dt * invA * Rk; continue; }
            nu = Un - (dt * invA / 6.0) * Rk;
          }
          s->Racc[i] = nu;
          s->dU[i] = nu - Un;
        }
      }
      if (st < ns - 1) refresh_prims(s, (integ == 3 && st == 1) ? s->S2 : s->S1);
    }
    s->min_dt = s->dt_step;
    s->stage = 0;
    return;
  }
  if (integ == 1) {
    const double w[3] = {0.5, 0.5, 1.0};
    for (int st = 0; st < 4; st++) {
      s->stage = st;
      if (st > 0) orc_apply_bc(s);
      orc_net_flux(s);
      if (st == 0) {
        s->dt_step = s->min_dt;
        memcpy(s->dtk, s->dt, (size_t)NP * sizeof(double));
      }
      for (int c = 0; c < NP; c++) {
        double dt = lts ? s->dtk[c] : s->dt_step, invA = s->inva[c];
        for (int k = 0; k < 4; k++) {
          size_t i = 4 * (size_t)c + k;
          double Rk = s->R[i];
          if (st == 0) {
            s->Racc[i] = Rk;
            s->S1[i] = s->U[i] - w[0] * (dt * invA) * Rk;
          } else if (st < 3) {
            s->Racc[i] = s->Racc[i] + 2.0 * Rk;
            s->S1[i] = s->U[i] - w[st] * (dt * invA) * Rk;
          } else {
            double acc = s->Racc[i] + Rk;
            s->dU[i] = -((dt * invA) * acc) / 6.0;
          }
        }
      }
      if (st < 3) refresh_prims(s, s->S1);
    }
    s->min_dt = s->dt_step;
    s->stage = 0;
    return;
  }
  const int ssp = integ == 2;
  for (int st = 0; st < 3; st++) {
    s->stage = st;
    if (st > 0) orc_apply_bc(s);
    orc_net_flux(s);
    if (st == 0) {
      s->dt_step = s->min_dt;
      memcpy(s->dtk, s->dt, (size_t)NP * sizeof(double));
    }
    for (int c = 0; c < NP; c++) {
      double dt;
      if (ssp) dt = lts ? s->dtk[c] : s->dt_step;
      else dt = (st == 0 && lts) ? s->dt[c] : s->min_dt;
      double invA = s->inva[c];
      for (int k = 0; k < 4; k++) {
        size_t i = 4 * (size_t)c + k;
        double RV = s->R[i] - 0.0; /* Cells_Net_Flux - Cells_Viscous_Flux (zero when inviscid) */
        if (st == 0) s->S1[i] = s->U[i] - dt * invA * RV;
        else if (st == 1) s->S2[i] = 0.25 * (s->S1[i] + 3.0 * s->U[i] - dt * invA * RV);
        else s->dU[i] = (2.0 / 3.0) * (s->S2[i] - s->U[i] - dt * invA * RV);
      }
    }
    if (st == 0) refresh_prims(s, s->S1);
    else if (st == 1) refresh_prims(s, s->S2);
  }
  if (ssp) s->min_dt = s->dt_step;
  s->stage = 0;
}

/* Estimate_Error, src/Error_Estimate_Update.cpp:10-28. */
void orc_estimate_error(orc_state *s) {
  double e[4] = {0, 0, 0, 0};
  for (int c = 0; c < s->NP; c++)
    for (int i = 0; i < 4; i++) {
      double d = s->dU[4 * c + i], t;
      if (d < 1e-9) t = fabs(d);
      else t = (fabs(d) / s->U[4 * c + i]);
      e[i] += t * t;
    }
  for (int i = 0; i < 4; i++) s->err[i] = sqrt(e[i]);
}

/* Update(), src/Error_Estimate_Update.cpp:31-43 (the reference GPU integrators: U = U^{n+1}). */
void orc_update(orc_state *s) {
  const int direct = s->c.integrator == 3 || s->c.integrator == 4;
  for (int c = 0; c < s->NP; c++) {
    for (int k = 0; k < 4; k++) {
      if (direct) s->U[4 * c + k] = s->Racc[4 * c + k];
      else s->U[4 * c + k] += s->dU[4 * c + k];
    }
    eos(s, c, s->U + 4 * (size_t)c, s->P + 11 * (size_t)c);
  }
}

/* Loop body of Inviscid_Solver, src/Solver.cpp:94-125; stops at t_end (> 0) like the harness. */
int orc_iterate(orc_state *s, int n, double t_end) {
  int done = 0;
  for (int it = 0; it < n; it++) {
    s->stage = 0;
    orc_apply_bc(s);
    if (s->c.time_accurate || s->c.integrator != 0) orc_rk(s);
    else if (orc_explicit(s) != 0) return -1 - done;
    s->total_time += s->min_dt;
    s->iterations++;
    orc_estimate_error(s);
    orc_update(s);
    done++;
    if (t_end > 0.0 && s->total_time >= t_end) break;
  }
  return done;
}

void orc_get(const orc_state *s, double *U, double *prim11, double *dt, double *net, double *delu) {
  if (U) memcpy(U, s->U, 4 * (size_t)s->NT * sizeof(double));
  if (prim11) memcpy(prim11, s->P, 11 * (size_t)s->NT * sizeof(double));
  if (dt) memcpy(dt, s->dt, (size_t)s->NP * sizeof(double));
  if (net) memcpy(net, s->R, 4 * (size_t)s->NP * sizeof(double));
  if (delu) memcpy(delu, s->dU, 4 * (size_t)s->NP * sizeof(double));
}

void orc_get_stage(const orc_state *s, double *S) { memcpy(S, s->S2, 4 * (size_t)s->NP * sizeof(double)); }
double orc_min_dt(const orc_state *s) { return s->min_dt; }
double orc_total_time(const orc_state *s) { return s->total_time; }
void orc_error(const orc_state *s, double *err) { memcpy(err, s->err, sizeof(s->err)); }
int orc_bad_cell(const orc_state *s) { return s->bad_cell; }

/* Calculate_Gradient_At_Cell_Center, src/Grid_Refine_Functions.cpp:221-246. */
void orc_gradient(orc_state *s, int slot, double *grad) {
  for (int c = 0; c < s->NP; c++) {
    double g0 = 0.0, g1 = 0.0;
    if (s->nf[c] > 0 && s->area[c] > 0.0) {
      double pc = s->P[11 * (size_t)c + slot];
      for (int f = 0; f < s->nf[c]; f++) {
        int N = s->nbr[4 * c + f];
        double pn = pc;
        if (N >= 0 && N < s->NP) pn = s->P[11 * (size_t)N + slot];
        double pf = 0.5 * (pc + pn);
        g0 += pf * s->nrm[8 * c + 2 * f] * s->len[4 * c + f];
        g1 += pf * s->nrm[8 * c + 2 * f + 1] * s->len[4 * c + f];
      }
      g0 *= s->inva[c];
      g1 *= s->inva[c];
    }
    grad[2 * c] = g0;
    grad[2 * c + 1] = g1;
  }
}

static const double *g_sort_key;
static int cmp_desc(const void *a, const void *b) {
  int i = *(const int *)a, j = *(const int *)b;
  double x = g_sort_key[i], y = g_sort_key[j];
  if (x > y) return -1;
  if (x < y) return 1;
  return (i > j) - (i < j);
}

/* Compute_Gradient_Refinement_Indicator + TagRefinableCells, src/Grid_Refine_Functions.cpp:8-63
 * (ties at the cut are broken by lower cell index; the reference's std::sort leaves them
 * implementation-defined). */
void orc_amr(orc_state *s, double threshold, double max_fraction, double *indicator, unsigned char *tags) {
  const int NP = s->NP;
  double *gr = (double *)malloc(2 * (size_t)NP * sizeof(double));
  double *gp = (double *)malloc(2 * (size_t)NP * sizeof(double));
  orc_gradient(s, 0, gr);
  orc_gradient(s, 4, gp);
  for (int i = 0; i < NP; i++) {
    double ind = 0.0, h = sqrt(s->area[i]);
    ind += sqrt(gr[2 * i] * gr[2 * i] + gr[2 * i + 1] * gr[2 * i + 1]) * h;
    double P = s->P[11 * (size_t)i + 4];
    if (P > 1e-14) ind += (sqrt(gp[2 * i] * gp[2 * i] + gp[2 * i + 1] * gp[2 * i + 1]) / P) * h;
    indicator[i] = ind;
    tags[i] = 0;
  }
  if (max_fraction > 0.0 && max_fraction < 1.0) {
    int *order = (int *)malloc((size_t)NP * sizeof(int));
    for (int i = 0; i < NP; i++) order[i] = i;
    g_sort_key = indicator;
    qsort(order, NP, sizeof(int), cmp_desc);
    int nRefine = (int)(max_fraction * NP);
    if (nRefine < 1) nRefine = 1;
    for (int k = 0; k < nRefine && k < NP; k++)
      if (indicator[order[k]] >= threshold) tags[order[k]] = 1;
    free(order);
  } else {
    for (int i = 0; i < NP; i++)
      if (indicator[i] > threshold) tags[i] = 1;
  }
  free(gr);
  free(gp);
}
