/*
 * lpg_oracle.h -- CPU oracle for the litepgo volumetric neo-Hookean hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain C++17 restatement of the reference
 * CPU algorithm (annajcy/litepgo, Eigen/TBB based), used as the parity checker
 * for the CUDA path and as the timed CPU baseline. Nothing in the product
 * (litepgo_b200/) links, loads or calls it; only tests/, the smoke check and
 * the cpu_baseline / reference legs of bench.py do.
 *
 * Conventions (identical to the reference):
 *   - 3x3 matrices are column-major arrays: m[i + 3*j] is row i, column j
 *     (Eigen default storage, src/core/common/types.hpp:18-22).
 *   - theta = [lambda, mu] (src/core/fem/material/volumetric/neo_hookean.hpp:9).
 *   - DOF layout is vertex-major xyz, DOF = 3*v + c
 *     (src/core/dof/vertex_dof_map.hpp:43-50).
 *   - The Hessian is scalar CSC with both triangles, int32 indices
 *     (src/core/common/types.hpp:18-22).
 *
 * Parity status: pinned by the reference's own known-answer tests (closed
 * forms, finite differences, feasible-step constants) reproduced in
 * tests/test_oracle_known_answers.py. The reference itself cannot be built in
 * this container (Eigen 5, oneTBB, nanobind and GoogleTest are fetched at
 * configure time and there is no network), so no reference binary exists.
 */
#ifndef LPG_ORACLE_H
#define LPG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, mirroring the reference's exception classes. */
enum {
    ORC_OK = 0,
    ORC_EINVAL = 1,  /* std::invalid_argument */
    ORC_EDOMAIN = 2, /* std::domain_error     */
    ORC_ELOGIC = 6   /* std::logic_error      */
};

const char* orc_last_error(void);
void orc_set_threads(int threads);
int orc_get_threads(void);

/* ---- NeoHookean pointwise (neo_hookean.cpp) ---- */
int orc_nh_W(const double F[9], const double Fp[9], const double theta[2], double* W);
int orc_nh_dW_dF(const double F[9], const double Fp[9], const double theta[2], double P[9]);
int orc_nh_d2W_dF2(const double F[9], const double Fp[9], const double theta[2], double A[81]);
int orc_nh_d2W_dF_dtheta(const double F[9], const double Fp[9], const double theta[2], double out[18]);
int orc_nh_d2W_dF_dFp(const double F[9], const double Fp[9], const double theta[2], double out[81]);
int orc_nh_feasible_step(const double F[9], const double Fp[9], const double theta[2], const double dF[9],
                         const double dFp[9], const double dtheta[2], double* alpha);

/* ---- positive_det_feasible_step.cpp ---- */
int orc_positive_det_step(const double A[9], const double dA[9], double* alpha);

/* ---- symmetric PSD projection of a dense n x n matrix (mesh_energy.cpp:16-27) ---- */
int orc_project_psd(int n, const double* H_colmajor, double* out_colmajor);

/* ---- mesh energy: VolumetricFemEnergy<NeoHookean, TetP1Basis, TetCentroidQuadrature> ---- */
typedef struct orc_mesh orc_mesh;

/* rest: either per-vertex X (V*3, with Xe == NULL) or per-element corners Xe (T*12).
 * theta: per element (T*2) when theta_per_element != 0, else one shared [lambda, mu].
 * Fp: per element column-major (T*9) or NULL for identity. */
int orc_mesh_create(int num_vertices, const double* X, int num_tets, const int* tets, const double* Xe,
                    const double* theta, int theta_per_element, const double* Fp, orc_mesh** out);
void orc_mesh_destroy(orc_mesh* m);
int orc_mesh_num_dofs(const orc_mesh* m);
long long orc_mesh_nnz(const orc_mesh* m);
/* CSC pattern: outer[num_dofs+1], inner[nnz]. */
int orc_mesh_pattern(const orc_mesh* m, int* outer, int* inner);

/* hessian: 0 none, 1 exact, 2 projected (12x12 eigen clamp). Outputs may be NULL.
 * elem_E (T), elem_g (T*12), elem_H (T*144, column-major) give per-element results. */
int orc_mesh_eval(orc_mesh* m, const double* u, double* E, double* grad, int hessian, double* csc_values,
                  double* elem_E, double* elem_g, double* elem_H);
int orc_mesh_feasible_step(orc_mesh* m, const double* u, const double* du, double* alpha);

/* VolumetricFemForceMaterialResponse VJP at displacement u with weights w (num_dofs):
 * per-element [d/dlambda, d/dmu] of w . g (T*2). The reference returns the positive
 * displacement gradient (force response) products; the equilibrium VJP negates it. */
int orc_mesh_force_vjp_theta(orc_mesh* m, const double* u, const double* w, double* out);
/* (d g / d X)^T w for the vertex rest positions X (3V), no plastic field; restated from the
 * shape derivative of the element force (the reference has no such derivative). */
int orc_mesh_force_vjp_rest(orc_mesh* m, const double* u, const double* w, double* out);
/* (d g / d vec Fp)^T w per element: 9 values each (column-major Fp index). */
int orc_mesh_force_vjp_fp(orc_mesh* m, const double* u, const double* w, double* out);

/* ---- Newton (newton.cpp) over E(u) = elastic(u) - f_ext . u ---- */
typedef struct {
    double gradient_tolerance; /* reference rule: max-norm of the free gradient; rel rule: relative 2-norm */
    int max_iterations;
    int hessian;               /* 1 exact, 2 projected */
    int max_line_search_steps;
    double line_search_shrink;
    int stop_rule;             /* 0 reference (abs max-norm), 1 relative 2-norm */
    int accept_rule;           /* 0 reference (decrease within 16 eps noise), 1 Armijo c=1e-4 (+ noise) */
    int linear_solver;         /* 0 envelope LDL^T (direct), 1 block-Jacobi PCG */
    double cg_tolerance;       /* PCG: forcing-term cap (relative residual) */
    int cg_max_iterations;
} orc_newton_options;

typedef struct {
    int status; /* 0 Converged, 1 MaxIterations, 2 StepTooSmall, 3 NoDescentDirection */
    int iterations;
    double energy;
    double gradient_norm;
    double gradient_norm0;
    long long cg_iterations;
    int line_search_evaluations;
} orc_newton_result;

int orc_newton_solve(orc_mesh* m, const int* fixed_dofs, int num_fixed, const double* f_ext, const double* x0,
                     const orc_newton_options* options, double* x_out, orc_newton_result* result);

/* A weighted-sum potential around the elastic energy (weighted_sum_energy.hpp:16-47 with
 * QuadraticEnergy terms, quadratic_energy.hpp:10-20): E = w elastic + 1/2 x^T A x - f_ext . x + c,
 * A a symmetric scalar CSR matrix inside the elastic pattern (a_indptr NULL: none). */
typedef struct {
    double elastic_weight;
    const int* a_indptr;
    const int* a_indices;
    const double* a_values;
    double constant;
} orc_terms;

/* orc_newton_solve over terms (NULL: elastic and load only) with the reference's NewtonStep trace
 * (newton.hpp:34-44, reported where newton.cpp:123-181 reports it): 7 doubles per step
 * {iteration, energy, max|g_free|, diagonal_shifts, feasible_step, step, line_search_evaluations},
 * at most trace_cap steps; *trace_len receives the count (trace may be NULL). */
int orc_newton_solve_ex(orc_mesh* m, const orc_terms* terms, const int* fixed_dofs, int num_fixed, const double* f_ext,
                        const double* x0, const orc_newton_options* options, double* x_out, orc_newton_result* result,
                        double* trace, int trace_cap, int* trace_len);

/* Adjoint of the static equilibrium (static_equilibrium_response.cpp:43-88, transpose branch):
 * solves K_ff lambda = dLdu_free with the exact Hessian at u_star and returns
 * dtheta = -(d g / d theta)^T expand(lambda) per element (T*2). linear_solver as above. */
int orc_adjoint_theta(orc_mesh* m, const double* u_star, const double* dLdu, const int* fixed_dofs, int num_fixed,
                      int linear_solver, double cg_tolerance, double* dtheta, double* lambda_out);

#ifdef __cplusplus
}
#endif
#endif
