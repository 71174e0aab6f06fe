/*
 * mpdg_heat.h - C ABI of the B200-native matrix-free heat operator and solve.
 *
 * This is the drop-in boundary for MeltPoolDG's implicit heat-transfer hot
 * path. Every entry point is `extern "C"`, takes plain pointers and sizes,
 * returns an int status (MPDG_OK = 0) and never throws. Vectors passed as
 * `double *` / `float *` are DEVICE pointers of length n_dofs (locally owned
 * DoFs, no ghosts: one GPU owns the whole mesh) unless the name ends in
 * `_host`. Work is enqueued on the handle's stream (mpdg_heat_set_stream);
 * entry points that return host scalars synchronise that stream.
 *
 * Reference interfaces replaced (paths inside the MeltPoolDG tree):
 *   OperatorBase<number>            include/meltpooldg/core/operator_base.hpp:21-84
 *   OperatorMatrixFree<dim,number>  include/meltpooldg/core/operator_base.hpp:188-282
 *   HeatDiffuseMultiPhaseOperator   source/heat/heat_diffuse_operator.cpp
 *   JacobiPreconditioner            include/meltpooldg/linear_algebra/preconditioner_jacobi.hpp
 *   LinearSolver::solve             include/meltpooldg/linear_algebra/linear_solver.hpp:22-134
 *   NewtonRaphsonSolver             source/linear_algebra/newton_raphson_solver.cpp:22-152
 *   Predictor (linear)              include/meltpooldg/linear_algebra/predictor.hpp:118-160
 *   HeatDiffuseOperation::solve     source/heat/heat_diffuse_operation.cpp:213-289
 *
 * Mesh: a structured hexahedral box, FE_Q(degree) on Gauss-Lobatto support
 * points, QGauss(degree+1), DoFs numbered lexicographically on the
 * (degree*cells+1)^3 nodal grid (x fastest). The geometry is either the
 * affine box or a trilinear map of vertices perturbed inside the box, with
 * per-quadrature-point geometric factors resident on the device.
 */
#ifndef MPDG_HEAT_H
#define MPDG_HEAT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
  MPDG_OK = 0,
  MPDG_ERR_INVALID_ARGUMENT = 1,   /* deal.II Assert/AssertThrow on arguments      */
  MPDG_ERR_OUT_OF_MEMORY = 2,
  MPDG_ERR_NOT_CONVERGED = 3,      /* SolverControl::NoConvergence                 */
  MPDG_ERR_NAN = 4,                /* residual became NaN/Inf                      */
  MPDG_ERR_BREAKDOWN = 5,          /* CG p.Ap <= 0 or GMRES breakdown              */
  MPDG_ERR_CUDA = 6,               /* a CUDA runtime call failed                   */
  MPDG_ERR_ZERO_TIME_INCREMENT = 7,/* AssertThrowZeroTimeIncrement (exceptions.hpp:6) */
  MPDG_ERR_NEWTON_NOT_CONVERGED = 8,/* ExcNewtonDidNotConverge -> ExcHeatTransferNoConvergence */
  MPDG_ERR_NOT_SUPPORTED = 9
};

/* ---- mesh, material, parameters -------------------------------------- */
typedef struct {
  int      degree;             /* FE_Q degree, 1..6 (fe_util.hpp:30)                 */
  int      cells[3];           /* cells per direction                                */
  double   lo[3], hi[3];       /* box corners                                        */
  double   perturb;            /* interior vertex perturbation, fraction of h (0 = affine) */
  uint64_t seed;               /* perturbation seed (splitmix64 counter hash)        */
  int      dirichlet_mask;     /* bit f: face f Dirichlet (0 x-,1 x+,2 y-,3 y+,4 z-,5 z+) */
  double   dirichlet_value[6]; /* constant Dirichlet value per face                  */
} mpdg_mesh_desc;

enum { MPDG_LAW_CONSTANT = 0, MPDG_LAW_LINEAR_K = 1, MPDG_LAW_LIQUID_SOLID = 2,
       MPDG_LAW_GAS_LIQUID = 3, MPDG_LAW_GAS_LIQUID_SOLID = 4 };

/* Material law (Material::compute_parameters, material.templates.hpp:104-137,226-375):
 *   CONSTANT      rho*cp and k constant (material type gas / liquid)
 *   LINEAR_K      k(T) = k_l + k1*T, rho*cp constant (new law, no reference counterpart)
 *   LIQUID_SOLID  cubic smoothstep in the solid fraction between liquid and solid values,
 *                 mushy zone or sharp transition (material.templates.hpp:296-375,745-780)
 *   GAS_LIQUID    (1 - w) gas + w liquid with w = H (smooth) or H > 0.5 (sharp), H the
 *                 level-set heaviside field of mpdg_heat_set_fields
 *                 (material.templates.hpp:240-295,515-524)
 *   GAS_LIQUID_SOLID  (1 - w) gas + w liquid_solid(T), temperature derivatives w d/dT
 *                 liquid_solid (material.templates.hpp:376-500,620-740) */
typedef struct {
  int    law;
  int    sharp;            /* liquid-solid transition: 0 mushy zone, 1 sharp         */
  int    volume_specific;  /* interpolate rho*cp directly (heat_data diffuse option) */
  double rho_l, cp_l, k_l; /* liquid, or the single constant phase                   */
  double rho_s, cp_s, k_s; /* solid                                                  */
  double T_solidus, T_liquidus;
  double k1;
  int    sharp_gas_liquid; /* gas-liquid transition: 0 smooth (w = H), 1 sharp        */
  double rho_g, cp_g, k_g; /* gas (GAS_LIQUID, GAS_LIQUID_SOLID)                      */
} mpdg_material;

/* Apparent-capacity profiles of the latent heat of fusion (ApparentCapacityType,
 * include/meltpooldg/core/material_data.hpp:43; qlq the reference's default). */
enum { MPDG_APPARENT_QLQ = 0, MPDG_APPARENT_CONSTANT = 1, MPDG_APPARENT_POLY4_BELL = 2 };

enum { MPDG_SOLVER_CG = 0, MPDG_SOLVER_GMRES = 1 };           /* LinearSolverType  */
enum { MPDG_PRECOND_IDENTITY = 0, MPDG_PRECOND_JACOBI = 1,    /* PreconditionerType */
       MPDG_PRECOND_CHEBYSHEV_JACOBI_F32 = 2,
       /* FP32 p-multigrid V-cycle (no reference counterpart; the reference's GMG
        * pattern is unit_tests/gmg.cc): FE_Q(p) -> FE_Q(1) on the same mesh, then
        * FE_Q(1) on meshes coarsened by 2 per direction while the cell counts stay
        * even and >= mg_min_cells; Chebyshev-Jacobi smoothing on every level */
       MPDG_PRECOND_MG_F32 = 3 };

typedef struct {
  int    solver;              /* MPDG_SOLVER_*                                      */
  int    preconditioner;      /* MPDG_PRECOND_*                                     */
  int    max_iterations;      /* linear_solver_data.hpp:44 default 10000            */
  double rel_tolerance;       /* default 1e-12                                      */
  double abs_tolerance;       /* default 1e-20                                      */
  int    gmres_restart;       /* GMRES basis size before restart (default 28)       */
  int    cheb_degree;         /* Chebyshev: FP32 operator applications per call      */
  int    cheb_eig_iterations; /* Lanczos steps for the eigenvalue estimate          */
  double cheb_max_factor;     /* upper bound = factor * estimated lambda_max        */
  double cheb_min_fraction;   /* lower bound = max(lambda_min estimate, fraction*upper) */
  double tol_reference_norm;  /* > 0: stop when |r| <= rel_tolerance * this value   */
  int    cheb_picard;         /* 1: the FP32 Chebyshev applies the Picard operator
                                 (conductivity k(T_lin) at the q-points, no dk/dT term);
                                 the outer FP64 CG keeps the exact tangent          */
  int    cheb_eig_reuse;      /* 1: keep the Chebyshev interval across solves and
                                 time steps until the material or the mesh changes  */
  int    mg_smoothing_degree; /* multigrid: Chebyshev steps of pre- and post-smoothing */
  int    mg_coarse_degree;    /* multigrid: Chebyshev steps on the coarsest level    */
  double mg_smoothing_range;  /* multigrid: smoothing interval [upper / range, upper] */
  int    mg_min_cells;        /* multigrid: coarsen while every cell count / 2 >= this */
  int    mg_fine_pre_steps;   /* multigrid, finest level: pre-smoothing steps (< 0: as above) */
  int    mg_fine_post_steps;  /* multigrid, finest level: post-smoothing steps after the
                                 restart step (< 0: as mg_smoothing_degree)             */
} mpdg_solver_params;

typedef struct {
  int    iterations;          /* SolverControl::last_step()                         */
  int    status;              /* MPDG_OK or an error code                           */
  double initial_residual;
  double final_residual;      /* recursive residual at exit                         */
  double true_residual;       /* |b - A x| recomputed in FP64 (mixed precision)     */
  double lambda_min, lambda_max; /* Chebyshev interval used                         */
} mpdg_solve_stats;

typedef struct mpdg_heat mpdg_heat;

/* Default parameters (MeltPoolDG defaults, linear_solver_data.hpp:40-47). */
void mpdg_solver_params_default(mpdg_solver_params *prm);

/* ---- lifetime (ScratchData::build + operator construction) ----------- */
int mpdg_heat_create(const mpdg_mesh_desc *desc, int device, mpdg_heat **out);
/* One rank's part of a z-slab decomposition of the box `global` (the partitioning of the
 * reference's distributed triangulation, replaced by a structured split): the cells with
 * z index in [z_begin, z_end), same vertices as the global mesh (its perturbation
 * included), Dirichlet faces of the global mesh only (the slab's interior z faces carry
 * none). DoF planes K = p z_begin .. p z_end of the global grid are local planes
 * 0 .. p (z_end - z_begin); the two end planes are shared with the neighbouring slabs,
 * whose partial sums the caller adds after each assembly (vmult, diagonal, rhs). */
int mpdg_heat_create_slab(const mpdg_mesh_desc *global, int z_begin, int z_end, int device,
                          mpdg_heat **out);
int mpdg_heat_destroy(mpdg_heat *h);
/* Enqueue all work of this handle on `stream` (a cudaStream_t; NULL = legacy default). */
int mpdg_heat_set_stream(mpdg_heat *h, void *stream);
int mpdg_heat_n_dofs(const mpdg_heat *h, int64_t *n_dofs);
int mpdg_heat_n_cells(const mpdg_heat *h, int64_t *n_cells);
int mpdg_heat_dof_dims(const mpdg_heat *h, int dims[3]);
/* Device memory the handle holds (geometry, FP32 copies, solver workspace), bytes. */
int mpdg_heat_device_bytes(const mpdg_heat *h, int64_t *bytes);

/* ---- operator coefficients ------------------------------------------ */
/* Material law (Material ctor + HeatDiffuseMultiPhaseOperator ctor, do_solidification =
 * law != CONSTANT). */
int mpdg_heat_set_material(mpdg_heat *h, const mpdg_material *m);
/* Two-phase and transport fields of HeatDiffuseMultiPhaseOperator (its level_set_as_heaviside
 * and velocity vectors, heat_diffuse_operator.cpp:47-72): device vectors on this handle's
 * DoFs, caller-owned, read when the per-quadrature-point coefficients are built.
 *   heaviside  n_dofs values, weights the GAS_LIQUID and GAS_LIQUID_SOLID laws (required
 *              by them)
 *   velocity   3 x n_dofs, component-major (x block, y block, z block) or NULL; adds
 *              rho_cp v.grad(T) to the residual and rho_cp v.grad(u) to the tangent and its
 *              diagonal (:499-500, :1038-1042), with a temperature-dependent law also
 *              d(rho_cp)/dT (v.grad T_lin) u (:1044-1049); not allowed with LINEAR_K
 * The coefficients are rebuilt at the next operator call after set_fields or set_material:
 * call set_fields again after changing the vectors' contents.  With a velocity the operator
 * is nonsymmetric (use MPDG_SOLVER_GMRES); the multigrid preconditioner is not available
 * with either field.  A field that was interpolated from another finite element space is
 * passed after its interpolation to this one. */
int mpdg_heat_set_fields(mpdg_heat *h, const double *heaviside, const double *velocity);
/* Latent heat of fusion as an apparent heat capacity in the mushy zone: with latent_heat > 0
 * the liquid-solid specific heat capacity (LIQUID_SOLID, GAS_LIQUID_SOLID) gains the profile's
 * capacity and its temperature derivative enters the tangent (MaterialData::
 * latent_heat_of_fusion and apparent_capacity_type, material.hpp:655-656,
 * material.templates.hpp:562-616, source/heat/apparent_capacity.cpp). 0 switches it off.
 * MPDG_ERR_NOT_SUPPORTED with volume_specific (the reference throws there). */
int mpdg_heat_set_latent_heat(mpdg_heat *h, double latent_heat, int profile);
/* Dirichlet values per face (x-, x+, y-, y+, z-, z+; the faces of the mesh description's mask)
 * for the following steps and distribute calls: boundary data that change in time
 * (HeatData::enable_time_dependent_bc, whose constraints init_time_advance rebuilds every step,
 * heat_diffuse_operation.cpp:219-226), constant per face. The first flagged face in that order
 * owns an edge or corner DoF. */
int mpdg_heat_set_dirichlet_values(mpdg_heat *h, const double values[6]);
/* Host evaluation of a law as the cell kernels evaluate it, at temperature T and heaviside H:
 * out = {rho*cp, k, d(rho*cp)/dT, dk/dT} (Material::compute_parameters with the temperature
 * derivatives of get_material_parameters_and_derivatives, heat_diffuse_operator.cpp:1167-1210).
 * Laws CONSTANT, LINEAR_K, LIQUID_SOLID and GAS_LIQUID_SOLID; needs no GPU. */
int mpdg_material_eval(const mpdg_material *m, double latent_heat, int profile, double T,
                       double H, double out[4]);
/* Boundary terms on one box face (0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+), replacing the
 * heat BoundaryConditionManager's "convection" / "radiation" / "neumann" entries
 * (heat_diffuse_operator.cpp:243-269 tangent, :690-781 rhs, :1088-1129 local op):
 *   MPDG_BC_CONVECTION  rhs -h (T - T_inf_conv), tangent h
 *   MPDG_BC_RADIATION   rhs -eps sigma (T^4 - T_inf_rad^4), tangent 4 eps sigma T^3
 *   MPDG_BC_NEUMANN     rhs -q_n (prescribed normal flux)
 * Neumann cannot be combined with the others on a face (:708-712); type 0 clears. */
enum { MPDG_BC_CONVECTION = 1, MPDG_BC_RADIATION = 2, MPDG_BC_NEUMANN = 4 };
int mpdg_heat_set_boundary(mpdg_heat *h, int face, int type, double h_conv, double T_inf_conv,
                           double emissivity, double T_inf_rad, double q_n);
/* OperatorBase::reset_time_increment (operator_base.hpp:41-46). */
int mpdg_heat_reset_time_increment(mpdg_heat *h, double dt);
/* The operator's references to `temperature` (linearisation point) and
 * `temperature_old` (heat_diffuse_operator.hpp:128-135). Device pointers that must
 * stay valid while the operator is used; FP32 copies for the FP32 operator are
 * refreshed by this call. */
int mpdg_heat_set_linearization(mpdg_heat *h, const double *temperature,
                                const double *temperature_old);

/* ---- OperatorMatrixFree verbs --------------------------------------- */
/* dst = J src (vmult, heat_diffuse_operator.cpp:179-197): dst zeroed first, Dirichlet
 * entries of src read as zero, constrained rows of dst left zero. */
int mpdg_heat_vmult(mpdg_heat *h, double *dst, const double *src);
/* Same operator in FP32 (geometry, linearisation point and coefficients in FP32). */
int mpdg_heat_vmult_f32(mpdg_heat *h, float *dst, const float *src);
/* FP32 Picard operator of the mixed-precision preconditioner (no reference
 * counterpart; the FP32 Chebyshev smoother applies it): the tangent of the
 * linear-k law without its dk/dT grad(T_lin) u term, i.e. the conductivity
 * k(T_lin) frozen at the quadrature points. Boundary-face terms as in
 * mpdg_heat_vmult_f32. MPDG_ERR_INVALID_ARGUMENT for the other laws. */
int mpdg_heat_vmult_f32_picard(mpdg_heat *h, float *dst, const float *src);
/* The cell-row layout of an FP32 nodal vector on an FE_Q(3) mesh, in which the multigrid's fine
 * level keeps its Chebyshev iterate so that the FP32 Picard operator gathers a cell's x-row of
 * 4 nodes with one aligned 16-byte load (no reference counterpart): x-row r = j + nd1 k of the
 * nodal grid holds 4 slots per cell column c, slot s = node 3c + s, so the node shared by
 * columns c - 1 and c is stored in both. *n_floats = 4 m0 nd1 nd2 (m0 cells and nd0 = 3 m0 + 1
 * nodes per x-row). MPDG_ERR_NOT_SUPPORTED for the other degrees. */
int mpdg_heat_cell_rows_size(const mpdg_heat *h, int64_t *n_floats);
/* rows = the cell-row copy of the lexicographic FP32 vector lex (device pointers). */
int mpdg_heat_to_cell_rows_f32(mpdg_heat *h, float *rows, const float *lex);
/* dst = the FP32 Picard operator of mpdg_heat_vmult_f32_picard applied to an operand given in
 * cell rows: the CUDA-core kernel of the multigrid's fine level. FE_Q(3) without Robin/Neumann
 * faces; not with the tensor-core or nodal-conductivity forms (MPDG_ERR_INVALID_ARGUMENT). */
int mpdg_heat_vmult_f32_picard_rows(mpdg_heat *h, float *dst, const float *src_rows);
/* 1 when the handle's last FP64 CG with the FP32 Chebyshev or multigrid preconditioner kept the
 * fine level's Chebyshev iterate in cell rows (opt-in: the environment sets MPDG_PICARD_ROWS=1;
 * FE_Q(3), Picard operator on the CUDA cores, no Robin/Neumann faces), else 0. */
int mpdg_heat_picard_cell_rows(const mpdg_heat *h);
/* The FP32 Picard operator (mpdg_heat_vmult_f32_picard and the multigrid fine level) on the
 * tensor cores: tcgen05 TF32 GEMMs over bricks of 128 cells, operands rounded to TF32
 * (relative error ~5e-4 against the oracle), FP32 accumulation. Exists for uniform box meshes
 * and FE_Q(3); on = 1 uses it where it exists, on = 0 keeps the CUDA-core kernel (the default
 * unless the environment sets MPDG_PICARD_TC=1: the CUDA-core kernel measured faster). The
 * second call returns 1 when the handle applies the operator on the tensor cores. */
int mpdg_heat_set_picard_tensor_cores(mpdg_heat *h, int on);
int mpdg_heat_picard_tensor_cores(const mpdg_heat *h);
/* The two 256 x 64 matrices that kernel keeps in shared memory (2 x 16384 floats, host memory,
 * no device needed): G^T then G, rows j = c * 64 + q (c = 0..2 the reference-gradient
 * components, 3 the values, q = qx + 4 (qy + 4 qz) the Gauss point), columns i = ix + 4 (iy +
 * 4 iz) the cell's DoF, entries rounded to TF32, in the no-swizzle K-major UMMA layout:
 * G^T (j, i) at (j / 8) * 512 + (i / 4) * 32 + (j % 8) * 4 + i % 4, G (i, j) at 16384 +
 * (i / 8) * 2048 + (j / 4) * 32 + (i % 8) * 4 + j % 4. */
int mpdg_picard_tc_matrices(float *out);
/* Inverse diagonal of that FP32 Picard operator (|d| > 1e-10 ? 1/d : 1), the Jacobi
 * scaling of the multigrid smoothers. Same restrictions. */
int mpdg_heat_inverse_diagonal_f32_picard(mpdg_heat *h, float *inv_diag);
/* compute_inverse_diagonal_from_matrixfree (heat_diffuse_operator.cpp:271-284):
 * diag(J) inverted with |d| > 1e-10 ? 1/d : 1. */
int mpdg_heat_compute_inverse_diagonal(mpdg_heat *h, double *inv_diag);
/* diag(J) itself (constrained rows 0): the partial diagonal of a slab, summed over the
 * shared planes before it is inverted. */
int mpdg_heat_compute_diagonal(mpdg_heat *h, double *diag);
/* create_rhs(dst, src) (heat_diffuse_operator.cpp:783-806): dst += -R(T) with T the
 * linearisation point, src = temperature_old, heat_source the nodal source vector
 * (may be NULL for zero); dst is not zeroed. */
int mpdg_heat_create_rhs(mpdg_heat *h, double *dst, const double *src,
                         const double *heat_source);
/* ---- OperatorMatrixFree verbs on HOST vectors ------------------------------------------
 * OperatorMatrixFree<dim, double>::VectorType is the host vector
 * dealii::LinearAlgebra::distributed::Vector<double> (operator_base.hpp:192); on one rank its
 * local array holds every DoF. These verbs take such arrays (length n_dofs, host memory, in
 * the caller's DoF numbering), copy them into device mirrors the handle keeps, run the device
 * verb and copy the result back before returning (the stream is synchronised).
 * set_dof_permutation gives the caller's numbering: lex_of_dof[i] is the lexicographic index
 * (I + nx (J + ny K) on the nodal grid) of the caller's DoF i; it must be a permutation of
 * 0 .. n_dofs-1 (MPDG_ERR_INVALID_ARGUMENT otherwise); NULL restores the identity. deal.II
 * numbers DoFs cell by cell, so a MeltPoolDG adapter passes the map built from its
 * DoFHandler. The device verbs above keep taking lexicographic vectors. */
int mpdg_heat_set_dof_permutation(mpdg_heat *h, const int64_t *lex_of_dof);
/* HeatDiffuseMultiPhaseOperator::pre() with the operator's references to temperature and
 * temperature_old (heat_diffuse_operator.hpp:128-135): copies both to the device mirrors and
 * linearises there (T_old may be NULL). */
int mpdg_heat_set_linearization_host(mpdg_heat *h, const double *T, const double *T_old);
/* vmult(dst, src) (heat_diffuse_operator.cpp:179-197) on host vectors. */
int mpdg_heat_vmult_host(mpdg_heat *h, double *dst, const double *src);
/* compute_inverse_diagonal_from_matrixfree(diag) (heat_diffuse_operator.cpp:271-284). */
int mpdg_heat_compute_inverse_diagonal_host(mpdg_heat *h, double *inv_diag);
/* create_rhs(dst, src) (heat_diffuse_operator.cpp:783-806): dst += -R(T), src = T_old,
 * heat_source the nodal source (may be NULL). */
int mpdg_heat_create_rhs_host(mpdg_heat *h, double *dst, const double *src,
                              const double *heat_source);

/* AffineConstraints::distribute: set Dirichlet DoFs of u to their values. */
int mpdg_heat_distribute_constraints(mpdg_heat *h, double *u);
/* VectorTools::compute_norm(u, L2) with QGauss(p+1) (vector_tools.cpp:188-200). */
int mpdg_heat_l2_norm(mpdg_heat *h, const double *u, double *norm);
/* FE L2 norm for callers that cannot allocate device memory (code inside a foreign
 * memory pool whose accounting a raw allocation would break, loops that must not
 * synchronise on a first-use allocation). No counterpart in the reference. Writes
 * |u|_L2 to the caller's device scalar `norm` on the handle's stream; the reduction
 * scratch is a fixed 128 KiB array in the library (at most 16384 partial sums;
 * larger reductions are rejected with MPDG_ERR_INVALID_ARGUMENT), so the call calls
 * no cudaMalloc/cudaFree. The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) and caches it: make that first call before any
 * stream capture. The cached address is not valid after cudaDeviceReset. Calls
 * share the array: calls that overlap on the GPU race. */
int mpdg_heat_l2_norm_noalloc(mpdg_heat *h, const double *u, double *norm);
/* DoF support point coordinates, xyz[3*i + d] (device pointer, 3*n_dofs doubles). */
int mpdg_heat_support_points(mpdg_heat *h, double *xyz);
/* Nodal interpolation of the volumetric Gaussian source
 * q(x) = amplitude * exp(-|x - center|^2 / radius^2) (cf. laser_heat_source_volumetric.cpp). */
int mpdg_heat_gaussian_source(mpdg_heat *h, double *q, double amplitude, const double center[3],
                              double radius);

/* Volumetric laser heat source: LaserHeatSourceVolumetric::compute_volumetric_heat_source
 * (laser_heat_source_volumetric.cpp:20-58) with the intensity profiles of
 * laser_intensity_profiles.hpp, q[i] = I(x_i) at the DoF support points:
 *   UNIFORM           I = power                                          (:62-90)
 *   GAUSS_VOLUMETRIC  I = power / (r sqrt(pi/2))^3 exp(-2 |x - c|^2 / r^2) (:175-235)
 *   GAUSS_PROJECTION  I = power / (r^2 pi/2) exp(-2 d^2 / r^2), d = distance of x to
 *                     the beam line through c along the unit direction   (:36-60, :98-170)
 *   GUSAROV           powder-layer absorption, reflectivity rho, extinction beta, layer
 *                     thickness L                                        (:243-340)
 * A zero or negative radius (Gauss, Gusarov) or a non-unit direction (projection) is
 * MPDG_ERR_INVALID_ARGUMENT. */
enum { MPDG_LASER_UNIFORM = 0, MPDG_LASER_GAUSS_VOLUMETRIC = 1, MPDG_LASER_GAUSS_PROJECTION = 2,
       MPDG_LASER_GUSAROV = 3 };
typedef struct {
  int    profile;                 /* MPDG_LASER_*                                        */
  double power;                   /* current power (LaserOperation::get_laser_power)     */
  double position[3];             /* beam centre (LaserOperation::get_laser_position)    */
  double direction[3];            /* unit beam direction (Gauss projection)              */
  double radius;                  /* beam radius                                         */
  double reflectivity;            /* Gusarov: rho                                        */
  double extinction_coefficient;  /* Gusarov: beta                                       */
  double layer_thickness;         /* Gusarov: L                                          */
  int    planar;                  /* 1: the profile of a 2D problem (laser_intensity_profiles
                                     with dim = 2) on a mesh one cell thick in y: distances
                                     in the x-z plane, z the depth direction; 0: 3D         */
} mpdg_laser;
int mpdg_heat_laser_source(mpdg_heat *h, double *q, const mpdg_laser *laser);
/* The same laser as the source of the residual, evaluated at the support points inside the
 * create_rhs cell kernels (no nodal source vector is written or read): create_rhs and the time
 * steps use it wherever their heat_source is NULL, with the same values as
 * mpdg_heat_laser_source followed by create_rhs on that vector (the reference integrates the
 * nodal interpolant, heat_diffuse_operator.cpp:445-447). NULL switches it off; call again when
 * the power or the position change (every step of a moving laser). */
int mpdg_heat_set_laser(mpdg_heat *h, const mpdg_laser *laser);

/* ---- preconditioner + linear solver ---------------------------------- */
/* JacobiPreconditioner::update (preconditioner_jacobi.hpp:65-69): stores the inverse
 * diagonal at the current linearisation point inside the handle. */
int mpdg_heat_preconditioner_update(mpdg_heat *h);
/* JacobiPreconditioner::vmult: dst = src .* inv_diag. */
int mpdg_heat_preconditioner_vmult(mpdg_heat *h, double *dst, const double *src);
/* LinearSolver::solve(op, x, b, data, precond) (linear_solver.hpp:22-134): solve J x = b
 * from the initial guess in x, ReductionControl(max_it, abs_tol, rel_tol); the
 * preconditioner must have been updated.
 *   CG:    identity, Jacobi (FP64); FP32 Chebyshev-Jacobi or FP32 p-multigrid inside FP64
 *          flexible CG
 *   GMRES: identity, Jacobi (FP64, right preconditioning); FP32 Chebyshev-Jacobi as a
 *          flexible GMRES (the preconditioned directions kept in FP32, the FP64 operator
 *          applied to their exact widening); not the multigrid preconditioner */
int mpdg_heat_linear_solve(mpdg_heat *h, const mpdg_solver_params *prm, double *x,
                           const double *b, mpdg_solve_stats *stats);

/* ---- Jacobi-CG across ranks (z-slab decomposition; no reference counterpart beyond the
 *      MPI_Allreduce'd dot products of SolverCG and the ghost exchange of MatrixFree::loop,
 *      scratch_data.cpp:149-188) ----------------------------------------------------------
 * The caller owns the collectives. Each stage reduces over this rank's owned DoFs (the first
 * n_owned entries of the slab vector; a shared plane is owned by the upper slab) into
 * `partial` (device doubles), which the caller all-reduces before the next stage; alpha and
 * beta are device scalars, so an iteration needs no host round trip except the convergence
 * test. One iteration: Ap = J p (mpdg_heat_vmult, shared planes summed by the caller),
 * dcg_dot(p, Ap) -> all-reduce -> alpha = rz / pAp, dcg_update -> all-reduce ->
 * (rz', rr) -> beta = rz' / rz, dcg_direction.
 *   dcg_start      r = b - Ax (Ax may be NULL: x = 0), z = D r, p = z; partial = (r.z, r.r)
 *   dcg_dot        partial[0] = a.b
 *   dcg_update     x += alpha p, r -= alpha Ap, z = D r; partial = (r.z, r.r)
 *   dcg_direction  p = z + beta p
 *   invert_diagonal  d <- |d| > 1e-10 ? 1/d : 1 (after the shared planes of the diagonal
 *                  of mpdg_heat_compute_diagonal were summed) */
int mpdg_heat_dcg_start(mpdg_heat *h, int64_t n_owned, const double *b, const double *Ax,
                        const double *inv_diag, double *r, double *z, double *p, double *partial);
int mpdg_heat_dcg_dot(mpdg_heat *h, int64_t n_owned, const double *a, const double *b,
                      double *partial);
int mpdg_heat_dcg_update(mpdg_heat *h, int64_t n_owned, double *x, double *r, double *z,
                         const double *p, const double *Ap, const double *inv_diag,
                         const double *alpha, double *partial);
int mpdg_heat_dcg_direction(mpdg_heat *h, double *p, const double *z, const double *beta);
int mpdg_heat_invert_diagonal(mpdg_heat *h, double *d);

/* ---- time step --------------------------------------------------------- */
/* LINEAR_DIRECTION (no reference counterpart; single_linearization only): the linear
 * extrapolation is the linearisation point, and the increment solve starts from alpha d instead
 * of 0, d the direction of mpdg_heat_set_direction (e.g. mpdg_heat_learned_direction) and
 * alpha = argmin |r - alpha J d| (one operator application, handed to the solver as its
 * initial A x); the converged T is that of LINEAR to the solver tolerance. */
enum { MPDG_PREDICTOR_NONE = 0, MPDG_PREDICTOR_LINEAR = 1, MPDG_PREDICTOR_GIVEN = 2,
       MPDG_PREDICTOR_LINEAR_DIRECTION = 3 };

typedef struct {
  int    newton_max_iterations;   /* nonlinear_solver_data.hpp:13 default 10 */
  double newton_residual_tolerance;   /* default 1e-9  */
  double newton_correction_tolerance; /* default 1e-10 */
  int    predictor;               /* MPDG_PREDICTOR_*                         */
  int    single_linearization;    /* 1: one linearisation per step, stop at
                                     |b - J T| <= rel_tolerance |b|, b = J T_g - R(T_g) */
  mpdg_solver_params linear;
} mpdg_step_params;

typedef struct {
  int    newton_iterations;
  int    linear_iterations;
  int    converged;
  double initial_relative_residual; /* |R(T_g)| / |b| for single_linearization      */
  double step_ms;                   /* device time of the step (CUDA events)        */
} mpdg_step_stats;

void mpdg_step_params_default(mpdg_step_params *prm);

/* Initial guess used by MPDG_PREDICTOR_GIVEN (e.g. a learned predictor's output);
 * a device pointer that must stay valid until the step has run. */
int mpdg_heat_set_guess(mpdg_heat *h, const double *guess);
/* Increment direction used by MPDG_PREDICTOR_LINEAR_DIRECTION (zero at Dirichlet DoFs); a
 * device pointer that must stay valid until the step has run. */
int mpdg_heat_set_direction(mpdg_heat *h, const double *direction);

/* HeatDiffuseOperation::solve (heat_diffuse_operation.cpp:213-289) on device vectors:
 * predictor (none / linear extrapolation / the guess already in T_cur), history
 * commit (T_old <- T_cur), Dirichlet values, preconditioner update at the predicted
 * state, Newton-Raphson with increment solves (or one linearisation, see above).
 * T_cur and T_old are updated in place; heat_source may be NULL. */
int mpdg_heat_time_step(mpdg_heat *h, const mpdg_step_params *prm, double dt, double dt_old,
                        double *T_cur, double *T_old, const double *heat_source,
                        mpdg_step_stats *stats);

/* Same with HOST vectors: copies T_cur, T_old, heat_source to the device, runs the
 * step, copies T_cur and T_old back (the reference operation's own data location). The
 * host vectors of the time-step entry points (here and in the resident ones below) are in
 * the lexicographic numbering; mpdg_heat_set_dof_permutation applies to the *_host verbs
 * above only. */
int mpdg_heat_time_step_host(mpdg_heat *h, const mpdg_step_params *prm, double dt,
                             double dt_old, double *T_cur, double *T_old,
                             const double *heat_source, mpdg_step_stats *stats);

/* Host-buffer steps with the solution history resident on the device, as
 * HeatDiffuseOperation owns its SolutionHistory (heat_diffuse_operation.hpp:63):
 * load_history copies a host T and T_old into the handle's device history; each
 * time_step_resident uploads the step's host heat source (NULL: none) while the step
 * starts, advances the history and copies the new T to T_out (NULL: no copy);
 * store_history copies T and T_old back (either may be NULL). */
int mpdg_heat_load_history(mpdg_heat *h, const double *T_host, const double *T_old_host);
int mpdg_heat_store_history(mpdg_heat *h, double *T_host, double *T_old_host);
int mpdg_heat_time_step_resident(mpdg_heat *h, const mpdg_step_params *prm, double dt,
                                 double dt_old, const double *heat_source, double *T_out,
                                 mpdg_step_stats *stats);

/* ---- learned initial guess (no counterpart in the reference; the hook is the
 *      Predictor's type switch, predictor.hpp:122-154) ---------------------- */
/* A 3D U-Net (4 levels, 16/32/48/64 channels, 3x3x3 convolutions, BF16 weights and
 * activations, FP32 accumulation) on an nx x ny x nz nodal grid; input 3 channels,
 * output 1 channel, the tensors of these calls planar [C][z][y][x] FP32 on the device (the
 * activations inside are BF16 and channel-chunked). */
typedef struct mpdg_unet mpdg_unet;
int mpdg_unet_create(int nx, int ny, int nz, uint64_t seed, mpdg_unet **out);
int mpdg_unet_destroy(mpdg_unet *u);
int mpdg_unet_set_stream(mpdg_unet *u, void *stream);
int mpdg_unet_n_params(const mpdg_unet *u, int64_t *n);
int mpdg_unet_dims(const mpdg_unet *u, int dims[3]);
/* FP32 master parameters (device, n_params): get / set (set refreshes the BF16 copy). */
int mpdg_unet_get_params(mpdg_unet *u, float *dst);
int mpdg_unet_set_params(mpdg_unet *u, const float *src);
/* Enqueued on the network's stream without a host synchronisation; an expired wait of a
 * tensor-core convolution (a hardware fault path, with bounded waits) is reported as
 * MPDG_ERR_CUDA by the next mpdg_unet_forward or by mpdg_unet_train_step. */
int mpdg_unet_forward(mpdg_unet *u, const float *input, float *output);
/* Gradient of sum(grad_output * output) w.r.t. the parameters after a forward. */
int mpdg_unet_backward(mpdg_unet *u, const float *grad_output, float *grad_params);
/* One Adam step (beta 0.9/0.999) on the mean squared error; loss returned on the host. */
int mpdg_unet_train_step(mpdg_unet *u, const float *input, const float *target, float lr,
                         double *loss);
int mpdg_unet_loss(mpdg_unet *u, const float *target, double *loss);
const char *mpdg_unet_last_error(void);

/* Network input from the solution history on the nodal grid sampled every `stride`
 * DoFs per direction ((n_d - 1) % stride == 0): channels (T - T_old)/s[0],
 * dt*q/s[1], T/s[2] (q may be NULL). */
int mpdg_heat_learned_input(mpdg_heat *h, int stride, const double *T, const double *T_old,
                            const double *heat_source, double dt, const double scales[3],
                            float *input);
/* Learned guess for the next step: guess = LE + alpha d with LE = 2 T - T_old the
 * linear extrapolation, d = a P(y) the network correction (a = RMS of T - T_old, the
 * inputs scaled by a, a and T_scale, P the trilinear prolongation from the sampled
 * grid) and, with line_search, alpha = argmin |r(LE) - alpha J d| (J linearised at
 * LE), so the guess's residual never exceeds the extrapolation's; else alpha = 1.
 * Dirichlet values applied; alpha returned in *alpha_out (may be NULL). The network's
 * grid must equal the sampled grid (else MPDG_ERR_INVALID_ARGUMENT). */
int mpdg_heat_learned_guess(mpdg_heat *h, mpdg_unet *u, int stride, const double *T,
                            const double *T_old, const double *heat_source, double dt,
                            double T_scale, int line_search, double *guess, double *alpha_out);

/* The network's correction as an increment direction for MPDG_PREDICTOR_LINEAR_DIRECTION:
 * direction = a P(y) with the inputs and the scale a of mpdg_heat_learned_guess, zero at the
 * Dirichlet DoFs (and everywhere when T == T_old). Unlike learned_guess it linearises nothing:
 * the step applies J to the direction once, at the point it linearises at anyway. */
int mpdg_heat_learned_direction(mpdg_heat *h, mpdg_unet *u, int stride, const double *T,
                                const double *T_old, const double *heat_source, double dt,
                                double T_scale, double *direction);

/* ---- instrumentation -------------------------------------------------- */
typedef struct {
  int64_t launches;        /* kernels this handle launched since the last reset      */
  int64_t vmult64_calls, vmult32_calls;
  double  vmult64_ms, vmult32_ms; /* summed device time of the operator applications
                                     (CUDA events on the handle's stream; only while
                                     timing is enabled)                                */
} mpdg_counters;

/* Enable/disable per-launch CUDA-event timing of the operator applications. */
int mpdg_heat_set_timing(mpdg_heat *h, int enable);
/* Read (synchronises the stream) and optionally reset the counters. */
int mpdg_heat_get_counters(mpdg_heat *h, mpdg_counters *c, int reset);

/* ---- meshes with hanging nodes (adaptive refinement) ---------------------------------
 * A box of coarse cells, each refined uniformly `refine[c]` times (mz*my*mx bytes, x fastest;
 * 0 = unrefined, 1 = split into 8 children, up to 6), neighbouring coarse cells across faces,
 * edges and vertices differing by one level at most: the 2:1-balanced meshes refine_grid
 * produces (source/utilities/amr.cpp:18-41). A node hangs when the coarsest cells holding it do
 * not have it as a node: it is constrained to such a cell's interpolant (DoFTools::
 * make_hanging_node_constraints merged into the Dirichlet constraints,
 * include/meltpooldg/utilities/constraints.hpp:111-132). The DoFs are the other nodes,
 * numbered by position (z, then y, then x). Affine boxes only (perturb = 0), degree 1..4,
 * levels 0..6 (each coarse cell's 8^level cells), Dirichlet values zero. device < 0 builds the
 * host description only (no CUDA call; the operator verbs then fail). */
typedef struct mpdg_amr mpdg_amr;
int mpdg_amr_create(const mpdg_mesh_desc *desc, const uint8_t *refine, int device,
                    mpdg_amr **out);
int mpdg_amr_destroy(mpdg_amr *h);
int64_t mpdg_amr_n_dofs(const mpdg_amr *h);
int64_t mpdg_amr_n_cells(const mpdg_amr *h);
/* Host arrays: support points (n_dofs x 3), Dirichlet mask (n_dofs bytes). */
int mpdg_amr_support_points(const mpdg_amr *h, double *xyz);
int mpdg_amr_constraint_mask(const mpdg_amr *h, uint8_t *mask);
/* Host arrays per active cell (coarse cells in z, y, x order, a refined one as its 8 children
 * in the same order): the (p+1)^3 gathered DoF indices, where the nodes of a hanging face or
 * edge name the unrefined neighbour's face or edge DoFs of the same local indices, and the
 * hanging code: bits 0-2 the child position in the parent, bit 3+d a hanging face normal to
 * direction d, bit 6+d a hanging edge parallel to d whose faces do not hang (bits 0-8 zero
 * without hanging nodes), bit 9 a refined cell, bits 10-12 its level. Coarse cells are
 * listed in z, y, x order, each as its 8^level cells in z, y, x order of its own lattice. */
int mpdg_amr_cell_data(const mpdg_amr *h, int64_t *dofs, uint16_t *codes);
/* Constant or LINEAR_K material and the time increment (mpdg_heat_set_material,
 * mpdg_heat_reset_time_increment). */
int mpdg_amr_set_material(mpdg_amr *h, const mpdg_material *m, double dt);
/* dst = J src (HeatDiffuseMultiPhaseOperator::vmult, heat_diffuse_operator.cpp:179-197) on
 * device vectors of n_dofs: Dirichlet DoFs read as zero, their rows zero; the hanging nodes
 * interpolated inside each refined cell from its gathered coarse DoFs and the transpose
 * applied in the scatter. T_lin: the linearisation point for LINEAR_K (NULL otherwise).
 * The mpdg_amr_* verbs run on the legacy default stream and return once the result is
 * complete. */
int mpdg_amr_vmult(mpdg_amr *h, double *dst, const double *src, const double *T_lin);
/* compute_inverse_diagonal_from_matrixfree (heat_diffuse_operator.cpp:271-284) on the refined
 * mesh: diag(F^T A_e F) accumulated cell by cell (F the cell's hanging-node interpolation),
 * inverted with |d| > 1e-10 ? 1/d : 1. */
int mpdg_amr_inverse_diagonal(mpdg_amr *h, double *inv_diag, const double *T_lin);
/* create_rhs (heat_diffuse_operator.cpp:783-806): dst += -R(T) with T, T_old and the nodal
 * source (nullable) interpolated by the hanging rule inside each cell; Dirichlet rows
 * untouched. */
int mpdg_amr_create_rhs(mpdg_amr *h, double *dst, const double *T, const double *T_old,
                        const double *heat_source);
/* LinearSolver::solve with CG and Jacobi (linear_solver.hpp:22-134) from x = 0:
 * |r| <= max(abs_tol, rel_tol |b|); MPDG_ERR_NOT_CONVERGED after max_iterations. */
int mpdg_amr_linear_solve(mpdg_amr *h, double *x, const double *b, const double *T_lin,
                          double rel_tolerance, double abs_tolerance, int max_iterations,
                          int *iterations);
/* HeatDiffuseOperation::solve (heat_diffuse_operation.cpp:213-289) on the refined mesh:
 * linear predictor (or a copy, prm->predictor), history commit, Dirichlet DoFs zero, Jacobi at
 * the predicted state, Newton-Raphson with Jacobi-CG increment solves (prm->linear's
 * tolerances) and the reference's convergence test. T_cur and T_old are updated in place. */
int mpdg_amr_time_step(mpdg_amr *h, double dt, double dt_old, double *T_cur, double *T_old,
                       const double *heat_source, const mpdg_step_params *prm,
                       mpdg_step_stats *stats);

/* Last error message of this thread (static storage). */
const char *mpdg_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
