/*
 * CPU oracle for the matrix-free heat path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of MeltPoolDG's implicit heat-transfer hot
 * path, used as the correctness checker for the CUDA implementation and as
 * the timed CPU baseline. It is never linked into, loaded by, or called from
 * the product library; only the tests, the smoke check and the CPU-baseline
 * leg of bench.py use it.
 *
 * Reference behaviour it restates (paths inside the MeltPoolDG tree):
 *   operator  source/heat/heat_diffuse_operator.cpp:179-284 (vmult, inverse
 *             diagonal), :393-529 (rhs_cell_loop), :955-1086 (local tangent
 *             operation), :1167-1210 (material parameters + derivatives)
 *   material  include/meltpooldg/core/material.templates.hpp:296-375,543-597,
 *             745-780; include/meltpooldg/level_set/level_set_tools.hpp:72-89
 *   solvers   include/meltpooldg/linear_algebra/linear_solver.hpp:36-38,106-111;
 *             preconditioner_jacobi.hpp:51-69; newton_raphson_solver.cpp:22-152
 *   predictor include/meltpooldg/linear_algebra/predictor.hpp:118-160,
 *             source/linear_algebra/predictor_linear.cpp:74-96
 *   FE setup  FE_Q(p) on Gauss-Lobatto support points, QGauss(p+1)
 *             (source/utilities/fe_util.cpp:40-55, finite_element_data.cpp:62-65)
 * The sum-factorised arithmetic itself lives in deal.II's FEEvaluation
 * (third party, not vendored); it is restated here from the published
 * sum-factorisation / even-odd algorithm.
 *
 * Parity pins: the application regression norms of
 *   applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/
 *     unidirectional_heat_transfer.mpirun=4.output  (2D, Q1)
 *   applications/mp-heat-transfer/cases/solidification_slab/tests/
 *     solidification_slab.mpirun=1.output            (1D, Q1, liquid-solid law)
 * are reproduced on 3D meshes that are one cell thick in the extra
 * directions (the solution is constant across them, so the norms agree).
 */
#ifndef MPDG_ORACLE_H
#define MPDG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Structured hexahedral box mesh, FE_Q(degree), QGauss(degree+1). */
typedef struct {
  int      degree;             /* 1..6 */
  int      cells[3];           /* cells per direction */
  double   lo[3], hi[3];       /* box corners */
  double   perturb;            /* interior-vertex perturbation, fraction of h */
  uint64_t seed;               /* perturbation seed */
  int      dirichlet_mask;     /* bit f: face f Dirichlet (0 x-,1 x+,2 y-,3 y+,4 z-,5 z+) */
  double   dirichlet_value[6]; /* constant Dirichlet value per face */
} orc_mesh_desc;

enum {
  ORC_LAW_CONSTANT = 0,
  ORC_LAW_LINEAR_K = 1,
  ORC_LAW_LIQUID_SOLID = 2,
  ORC_LAW_GAS_LIQUID = 3,
  ORC_LAW_GAS_LIQUID_SOLID = 4
};

typedef struct {
  int    law;             /* ORC_LAW_* */
  int    sharp;           /* liquid-solid transition: 0 mushy zone, 1 sharp */
  int    volume_specific; /* interpolate rho*cp directly (heat "diffuse" option) */
  double rho_l, cp_l, k_l;  /* liquid (or the single constant phase) */
  double rho_s, cp_s, k_s;  /* solid */
  double T_solidus, T_liquidus;
  double k1;              /* linear law: k(T) = k_l + k1*T */
  int    sharp_gas_liquid;  /* gas-liquid transition: 0 smooth (w = H), 1 sharp (w = H > 0.5) */
  double rho_g, cp_g, k_g;  /* gas */
  double latent_heat;       /* latent heat of fusion (> 0: apparent capacity in the mushy zone) */
  int    apparent_capacity; /* ORC_APPARENT_* profile of that capacity */
} orc_material;

/* apparent-capacity profiles (ApparentCapacityType, material_data.hpp:43; qlq the default) */
enum { ORC_APPARENT_QLQ = 0, ORC_APPARENT_CONSTANT = 1, ORC_APPARENT_POLY4_BELL = 2 };

typedef struct orc_heat orc_heat;

orc_heat *orc_create(const orc_mesh_desc *desc);
void      orc_destroy(orc_heat *h);
int64_t   orc_n_dofs(const orc_heat *h);
int64_t   orc_n_cells(const orc_heat *h);
void      orc_dof_dims(const orc_heat *h, int dims[3]);
void      orc_constraint_mask(const orc_heat *h, uint8_t *mask);
void      orc_support_points(const orc_heat *h, double *xyz); /* n_dofs x 3 */
void      orc_distribute(const orc_heat *h, double *u);       /* set Dirichlet values */
void      orc_set_threads(int n);

/* Boundary terms of one box face (face 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+):
 * type bit 1 convection  h (T - T_inf_c)       (tangent h)
 *      bit 2 radiation   eps sigma (T^4 - T_inf_r^4)  (tangent 4 eps sigma T^3)
 *      bit 4 Neumann     prescribed normal flux q_n (rhs only)
 * (heat_diffuse_operator.cpp:243-269 tangent, :719-781 rhs, :1088-1129 local op). */
int orc_set_boundary(orc_heat *h, int face, int type, double h_conv, double T_inf_conv,
                     double emissivity, double T_inf_rad, double q_n);

/* The material law at temperature T and heaviside H: out = {rho*cp, k, d(rho*cp)/dT, dk/dT}
 * (the values the operator uses at a quadrature point). */
void orc_material_eval(const orc_material *m, double T, double H, double out[4]);

/* Operator coefficients: material law and time step (reset_time_increment).  Returns -1
 * if a velocity field is set and the law is the linear-k law. */
int orc_set_material(orc_heat *h, const orc_material *m, double dt);

/* Two-phase and transport fields (HeatDiffuseMultiPhaseOperator's level_set_as_heaviside and
 * velocity, heat_diffuse_operator.cpp:51-67), nodal on the temperature space: heaviside (n_dofs)
 * weights the gas-liquid law, velocity ([3][n_dofs], component-major) adds the convective term
 * rho_cp v.grad(T) to the residual and rho_cp v.grad(u) to the tangent (:499-500, :1038-1042).
 * With a temperature-dependent law the tangent also gets d(rho_cp)/dT (v.grad T_lin) u
 * (:1044-1049).  Either may be NULL (no heaviside: weight 1, the liquid or liquid-solid
 * properties).  Returns -1 if a velocity is combined with the linear-k law. */
int orc_set_fields(orc_heat *h, const double *heaviside, const double *velocity);
/* Dirichlet values per face from now on (time-dependent boundary data) */
void orc_set_dirichlet_values(orc_heat *h, const double values[6]);

/* dst = J(T_lin, T_old) src.  form 0: sum-factorised, 1: direct quadrature,
 * 2: sum-factorised Picard operator (the tangent without its dk/dT grad(T_lin) u
 * term: conductivity k(T_lin) frozen at the quadrature points). */
void orc_vmult(const orc_heat *h, double *dst, const double *src, const double *T_lin,
               const double *T_old, int form);
/* inverse diagonal of J with the |d| > 1e-10 ? 1/d : 1 rule; form as above (2: of the
 * Picard operator). */
void orc_inverse_diagonal(const orc_heat *h, double *inv_diag, const double *T_lin,
                          const double *T_old, int form);
/* dst += -R(T) (rhs_cell_loop); T_old plain, heat_source nodal vector. */
void orc_create_rhs(const orc_heat *h, double *dst, const double *T, const double *T_old,
                    const double *heat_source);
/* FE L2 norm with QGauss(p+1) (VectorTools::compute_norm). */
double orc_l2_norm(const orc_heat *h, const double *u);

/* Linear solvers.  precond: 0 identity, 1 Jacobi (inv_diag), 2 Chebyshev-Jacobi. */
typedef struct {
  int    max_iterations;
  double rel_tolerance;
  double abs_tolerance;
  int    precond;
  int    cheb_degree;      /* Chebyshev: operator applications per preconditioner call */
  double cheb_lambda_min;  /* interval of D^-1 J covered by the polynomial */
  double cheb_lambda_max;
} orc_solver_params;

/* PCG on J(T_lin,T_old) x = b, deal.II SolverCG + ReductionControl semantics.
 * Returns the iteration count, or -1 if max_iterations was hit. */
int orc_cg(const orc_heat *h, const orc_solver_params *prm, double *x, const double *b,
           const double *inv_diag, const double *T_lin, const double *T_old, double *res_norm);

/* Restarted right-preconditioned GMRES (deal.II SolverGMRES semantics). */
int orc_gmres(const orc_heat *h, const orc_solver_params *prm, int restart, double *x,
              const double *b, const double *inv_diag, const double *T_lin, const double *T_old,
              double *res_norm);

/* Lanczos estimate of the extreme eigenvalues of D^-1 J from n_it CG steps. */
void orc_estimate_eigenvalues(const orc_heat *h, const double *inv_diag, const double *T_lin,
                              const double *T_old, int n_it, double *lmin, double *lmax);

/* Chebyshev-Jacobi preconditioner application dst = P(r). */
void orc_chebyshev_apply(const orc_heat *h, const orc_solver_params *prm, double *dst,
                         const double *r, const double *inv_diag, const double *T_lin,
                         const double *T_old);

/* Linear extrapolation predictor (compute_linear_predictor). */
void orc_linear_predictor(const orc_heat *h, const double *T_cur, const double *T_oldv,
                          double *pred, double dt, double dt_old);

typedef struct {
  int    max_iterations;
  double residual_tolerance;
  double correction_tolerance;
} orc_newton_params;

typedef struct {
  int    newton_iterations;
  int    linear_iterations;
  int    converged;
} orc_step_stats;

/* One implicit Euler step with MeltPoolDG's HeatDiffuseOperation::solve
 * semantics: predictor, history commit, Jacobi update at the predictor,
 * Newton-Raphson with increment solves. T_cur/T_old are updated in place.
 * predictor: 0 none (copy), 1 linear extrapolation; solver_type: 0 CG, 1 GMRES(28). */
int orc_time_step_newton(orc_heat *h, double *T_cur, double *T_old, const double *heat_source,
                         double dt, double dt_old, int predictor, int solver_type,
                         const orc_solver_params *lin, const orc_newton_params *nl,
                         orc_step_stats *stats);

/* Nodal interpolation of a volumetric Gaussian source
 * q(x) = amp * exp(-|x - c|^2 / r^2) at the DoF support points. */
void orc_gaussian_source(const orc_heat *h, double *q, double amp, const double c[3], double r);
/* volumetric laser intensity at the support points; profile 0 uniform, 1 Gauss
 * volumetric, 2 Gauss projection (unit dir), 3 Gusarov (rho, beta, L); planar != 0: the
 * two-dimensional profile of a 2D problem (points (x, z), the y coordinate of a one-cell-
 * thick mesh ignored; laser_intensity_profiles.hpp with dim = 2) */
void orc_laser_source(const orc_heat *h, double *q, int profile, double power, const double c[3],
                      const double dir[3], double radius, double rho, double beta, double L,
                      int planar);

#ifdef __cplusplus
}
#endif
#endif
