/*
 * litepgo_b200.h -- C ABI of the B200 (sm_100a) volumetric neo-Hookean hot path.
 *
 * This is the drop-in boundary for litepgo's
 *   VolumetricFemEnergy<NeoHookean, TetP1Basis, TetCentroidQuadrature>
 * energy / gradient / Hessian interface, its Newton solve and the adjoint
 * equilibrium sensitivity. Every entry point cites the reference interface it
 * replaces (paths inside annajcy/litepgo).
 *
 * Conventions kept from the reference:
 *   - unknowns are displacements u, F = I + B u_e
 *     (src/core/fem/assembly/volumetric_fem_energy.hpp:186-192);
 *   - DOF = 3 * vertex + component (src/core/dof/vertex_dof_map.hpp:43-50);
 *   - theta = [lambda, mu] (src/core/fem/material/volumetric/neo_hookean.hpp:9);
 *   - 3x3 matrices (Fp) are column-major, index i + 3 j;
 *   - the Hessian is the full symmetric matrix; its pattern is exported both as
 *     3x3 block-CSR (row_ptr, col_idx) and as the reference's scalar CSC with
 *     both triangles and int32 indices (src/core/common/types.hpp:18-22).
 *
 * Errors: every call returns an int status; no exception crosses the ABI. The
 * message of the last failure on the calling thread is lpg_last_error().
 *   LPG_EINVAL  <- std::invalid_argument (bad sizes, indices, theta)
 *   LPG_EDOMAIN <- std::domain_error     (det F <= 0, non-finite values)
 *   LPG_EBUSY   <- BusyScope's std::logic_error on overlapping calls
 *                  (src/core/common/busy_scope.hpp:11-26)
 *   LPG_ENOCONV <- a solve that did not converge
 *   LPG_ECUDA   <- a CUDA runtime failure
 *   LPG_ELOGIC  <- a broken contract (std::logic_error)
 *   LPG_EIO     <- std::runtime_error of the mesh-file readers (missing file, bad format)
 *   LPG_ESTOPPED <- an exception raised by a caller's per-iteration callback (the solve stops)
 *
 * Memory: the library owns its device buffers. Array arguments carry an
 * explicit LPG_MEM_HOST / LPG_MEM_DEVICE flag. Device pointers must be device
 * memory of the handle's GPU. A handle owns one CUDA stream (or the stream set
 * with lpg_fem_set_stream); calls on one handle must not overlap.
 */
#ifndef LITEPGO_B200_H
#define LITEPGO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LPG_ABI_VERSION 1

enum lpg_status {
    LPG_OK = 0,
    LPG_EINVAL = 1,
    LPG_EDOMAIN = 2,
    LPG_EBUSY = 3,
    LPG_ENOCONV = 4,
    LPG_ECUDA = 5,
    LPG_ELOGIC = 6,
    LPG_EIO = 7,
    LPG_ESTOPPED = 8 /* a caller's per-iteration callback asked the solve to stop */
};

/* HessianKind (src/core/energy/scalar/energy.hpp:6-13); NONE = no Hessian. */
enum lpg_hessian_kind {
    LPG_HESSIAN_NONE = 0,
    LPG_HESSIAN_EXACT = 1,
    LPG_HESSIAN_PROJECTED = 2 /* 12x12 eigenvalue clamp, mesh_energy.cpp:16-27 */
};

enum lpg_precision {
    LPG_PRECISION_F64 = 0,  /* all element arithmetic and outputs in FP64 */
    LPG_PRECISION_MIXED = 1 /* element arithmetic + Hessian in FP32; energy/gradient sums in FP64 */
};

enum lpg_memory { LPG_MEM_HOST = 0, LPG_MEM_DEVICE = 1 };

enum lpg_layout {
    LPG_LAYOUT_BSR = 0, /* nnzb blocks of 9 values, row-major 3x3 */
    LPG_LAYOUT_CSC = 1  /* the reference's scalar CSC value order (9 * nnzb values) */
};

typedef struct lpg_fem* lpg_fem_t;

/* Message of the last failed call on this thread ("" if none). */
const char* lpg_last_error(void);
int lpg_abi_version(void);
/* Writes a short build description (CUDA version, arch, and the number of device allocations
 * the library has made in this process so far) into buf. */
int lpg_build_info(char* buf, size_t size);

/*
 * Host-only (no GPU needed): block-CSR pattern of a tet mesh, the same pattern that
 * lpg_fem_pattern_bsr returns. Validates the connectivity like MeshTopology
 * (src/core/mesh/mesh_topology.hpp:25-44). Call with col_idx == NULL to get *nnzb first.
 */
int lpg_mesh_pattern_bsr(int num_vertices, int num_tets, const int32_t* tets, int64_t* nnzb, int32_t* row_ptr,
                         int32_t* col_idx);

/*
 * Host-only summary of the vertex clusters of the element-once assembly (no reference
 * counterpart; it replaces the per-column contribution lists of EnergyAssembler,
 * src/core/dof/energy_assembler.cpp:49-68, for the Exact Hessian): out[0] clusters,
 * out[1] most rows in one cluster, out[2] most elements in one cluster, out[3] element
 * evaluations per pass (sum over clusters), out[4] block contributor entries (16 per tet).
 * The plan's invariants are checked (LPG_ELOGIC if one fails): every referenced vertex is
 * owned by one cluster, every element's energy is counted once, and every block of every
 * owned row lists exactly the elements that share its two vertices, in ascending order. The
 * solvers' upper-triangle sliced-ELL layout (lpg_fem_solver_layout) is checked too: every row
 * once, its blocks with column >= row stored (diagonal first), and every block left of the
 * diagonal referencing the stored block of its transpose.
 */
int lpg_mesh_cluster_summary(int num_vertices, int num_tets, const int32_t* tets, int64_t out[5]);
/* The same for cells of cell_width vertices: 4 (tets, as above) or 8 (hexes; out[4] counts
 * 64 contributor entries per hex). */
int lpg_mesh_cluster_summary_cells(int num_vertices, int num_cells, const int32_t* cells, int cell_width,
                                   int64_t out[5]);

/*
 * Creates the element data and assembly plan of one tet mesh on `device`.
 * Replaces the constructor
 *   VolumetricFemEnergy(const VertexDofMap&, rest_positions, Fp, theta, int batch_size)
 *   (src/core/fem/assembly/volumetric_fem_energy.hpp:29-65)
 * together with MeshEnergy / EnergyAssembler set-up
 *   (src/core/energy/scalar/mesh_energy.cpp:29-42, src/core/dof/energy_assembler.cpp:22-68).
 *   X      : num_vertices * 3 rest positions (host), used when Xe == NULL
 *   tets   : num_tets * 4 vertex indices (host)
 *   Xe     : optional num_tets * 12 per-element rest corners (the reference's one
 *            rest-position Response per element); NULL uses X[tets]
 *   theta  : num_tets * 2 when theta_per_element != 0, else 2 shared values
 *   Fp     : num_tets * 9 column-major plastic gradients, or NULL for identity
 * Fails with LPG_EINVAL for out-of-range or repeated cell indices and for
 * degenerate or inverted rest tets (volumetric_element.hpp:35-36).
 */
int lpg_fem_create(int num_vertices, const double* X, int num_tets, const int32_t* tets, const double* Xe,
                   const double* theta, int theta_per_element, const double* Fp, int device, lpg_fem_t* out);
int lpg_fem_destroy(lpg_fem_t h);

/*
 * Hex Q1 mesh: VolumetricFemEnergy<NeoHookean, HexQ1Basis, GaussLegendre3D<n>>
 * (src/core/fem/assembly/volumetric_fem_energy.hpp:29-65 with fem/basis/3d/hex_q1_basis.hpp,
 * fem/quadrature/3d/gauss_legendre_3d.hpp). cells: 8 per element in HexQ1Basis corner order
 * ((0,0,0), (1,0,0), (1,1,0), (0,1,0), (0,0,1), (1,0,1), (1,1,1), (0,1,1) of [0,1]^3); X: rest
 * positions (3 per vertex); theta: [lambda, mu] (2, or 2 per element); points_per_axis: 2 or
 * 4. Every quadrature point must have det J > 0 (LPG_EINVAL otherwise, as
 * VolumetricElement3D). The handle answers lpg_fem_eval (Exact, and Projected: each element's
 * 24x24 Hessian projected to PSD), lpg_fem_feasible_step, lpg_fem_element_energies, the
 * patterns, lpg_newton_solve, lpg_fem_set_theta, lpg_fem_force_vjp_theta, lpg_adjoint_theta,
 * lpg_fem_deformation_gradients and lpg_fem_eval_material (one material row per quadrature
 * point); the rest-position, plastic-field and batch entry points are for tet meshes only
 * (LPG_EINVAL). No plastic field (Fp = I).
 */
int lpg_fem_create_hex(int num_vertices, const double* X, int num_cells, const int32_t* cells, const double* theta,
                       int theta_per_element, int points_per_axis, int device, lpg_fem_t* out);

/*
 * Tricubic Hermite hex mesh: VolumetricFemEnergy<NeoHookean, HexHermiteBasis, GaussLegendre3D<n>>
 * with BasisDofTransform<HexHermiteBasis> (fem/basis/3d/hex_hermite_basis.hpp,
 * fem/assembly/basis_dof_transform.hpp:59-148). Arguments as lpg_fem_create_hex; every cell must
 * be a positive axis-aligned box in corner order (LPG_EINVAL otherwise). The unknowns are 24
 * physical DOFs per vertex (num_dofs = 24 num_vertices): slots u, u_X, u_Y, u_Z, u_XY, u_XZ,
 * u_YZ, u_XYZ of 3 components each, DOF 24 v + 3 slot + c. Block patterns and Hessians are over
 * 3x3 blocks of (vertex, slot) rows, 8 per vertex (lpg_fem_sizes reports 8 num_vertices block
 * rows). The handle answers lpg_fem_eval (Exact Hessian; Projected is LPG_EINVAL),
 * lpg_fem_feasible_step, lpg_fem_element_energies, lpg_fem_set_theta, the patterns,
 * lpg_newton_solve with the Exact Hessian, lpg_fem_force_vjp_theta and lpg_adjoint_theta (over
 * the physical DOFs); the rest-position, plastic-field, material and batch entry points are
 * LPG_EINVAL. No plastic field (Fp = I).
 */
int lpg_fem_create_hex_hermite(int num_vertices, const double* X, int num_cells, const int32_t* cells,
                               const double* theta, int theta_per_element, int points_per_axis, int device,
                               lpg_fem_t* out);

/* Uses `stream` (a cudaStream_t) for all later work of this handle; NULL = the handle's own stream. */
int lpg_fem_set_stream(lpg_fem_t h, void* stream);

/* Sizes: vertices, tets, DOFs (3V), nnzb (3x3 blocks) and nnz (= 9 nnzb). Any pointer may be NULL. */
int lpg_fem_sizes(lpg_fem_t h, int* num_vertices, int* num_tets, int* num_dofs, int64_t* nnzb, int64_t* nnz);

/* Block-CSR pattern of the Hessian: row_ptr[V+1], col_idx[nnzb] (host). */
int lpg_fem_pattern_bsr(lpg_fem_t h, int32_t* row_ptr, int32_t* col_idx);

/* Scalar CSC pattern identical to EnergyAssembler::hessian_pattern()
 * (energy_assembler.cpp:38-47): outer[3V+1], inner[nnz] (host). */
int lpg_fem_pattern_csc(lpg_fem_t h, int32_t* outer, int32_t* inner);

/*
 * Energy, gradient and Hessian in one assembly. Replaces
 *   Energy::eval(x, gradient, optional<HessianKind>)  (src/core/energy/scalar/energy.hpp:29-30)
 * as implemented by MeshEnergy::eval_values + EnergyAssembler::assemble
 *   (src/core/energy/scalar/mesh_energy.cpp:48-87, src/core/dof/energy_assembler.cpp:123-170).
 *   u       : num_dofs displacements (io_mem)
 *   energy  : host double (may be NULL)
 *   grad    : num_dofs doubles (io_mem) or NULL
 *   hessian : lpg_hessian_kind; values written to hess (hess_mem) in `layout`
 *             as doubles (LPG_PRECISION_F64) or floats (LPG_PRECISION_MIXED)
 * Sums are deterministic and atomic-free: each block is accumulated in element
 * order, as the reference's per-column contribution lists do.
 */
int lpg_fem_eval(lpg_fem_t h, const double* u, int io_mem, double* energy, double* grad, int hessian, int precision,
                 int layout, void* hess, int hess_mem);

/*
 * Profiling helper (no reference counterpart): enqueues `launches` evaluations of device
 * arrays on the handle's stream and reports, from CUDA events recorded on that stream, the
 * mean duration of the assembly kernel alone (ms_assemble) and of one whole evaluation
 * including projection and the energy reduction (ms_eval). With flush_l2 != 0 a 512 MB
 * buffer is written before each launch, outside the measured intervals. Besides
 * LPG_LAYOUT_BSR and LPG_LAYOUT_CSC, layout 2 selects the solvers' upper-triangle sliced-ELL
 * layout of lpg_fem_solver_layout (hess then holds 9 * num_slots values; padding entries are
 * not written).
 */
int lpg_fem_time_eval(lpg_fem_t h, const double* u, double* grad, int hessian, int precision, int layout, void* hess,
                      int launches, int flush_l2, double* ms_assemble, double* ms_eval);

/*
 * The block layout the Newton and adjoint solvers keep the Hessian in (no reference
 * counterpart): the upper triangle of the symmetric block matrix (the blocks of row v with
 * column >= v, the diagonal first) in sliced ELL with chunks of 32 rows, rows sorted by their
 * BSR block count (descending, stable) within windows of 128 rows. Chunk c holds rows
 * sell_row[32 c + l] (l = 0..31, -1 past the last row) and slots [sell_ptr[c], sell_ptr[c + 1]),
 * 32 per stored block of its row with the most; stored block q of the row in lane l is slot
 * sell_ptr[c] + 32 q + l, and entry t (row-major) of that block is value
 * 9 sell_ptr[c] + 32 (9 q + t) + l. Blocks left of the diagonal are not stored (the solvers
 * read them as transposes). Any output may be NULL; sell_ptr has num_chunks + 1 entries,
 * sell_row 32 * num_chunks.
 */
int lpg_fem_solver_layout(lpg_fem_t h, int64_t* num_slots, int* num_chunks, int32_t* sell_ptr, int32_t* sell_row);

/* Per-element energies vol * W (num_tets doubles, io_mem). */
int lpg_fem_element_energies(lpg_fem_t h, const double* u, int io_mem, double* elem_energy);

/*
 * Largest safe step along du: Energy::max_feasible_step(x, dx)
 *   (src/core/energy/scalar/energy.cpp:35-46) via MeshEnergy::feasible_step
 *   (mesh_energy.cpp:88-107) and eval_positive_det_feasible_step
 *   (src/core/fem/kinematics/positive_det_feasible_step.cpp:13-84).
 */
int lpg_fem_feasible_step(lpg_fem_t h, const double* u, const double* du, int io_mem, double* alpha);

/*
 * The feasible step of lpg_fem_feasible_step, for callers that must not allocate device
 * memory when they call it: a solver embedded in a framework that owns the device memory pool
 * (a training loop on a caching allocator, an application with a fixed memory budget), where
 * a library cudaMalloc mid-step fragments or exceeds that budget. This entry point has no
 * counterpart in the reference: it is the same computation on tet, hex and Hermite handles,
 * with its scratch in a fixed ~512 KB array inside the library image instead of a
 * cudaMalloc'd buffer, so it calls no cudaMalloc / cudaFree. It is synchronous: it returns
 * once the step is on the host. u and du are DEVICE arrays (device or managed memory on the
 * handle's GPU) of num_dofs doubles; other pointers fail with LPG_EINVAL. *alpha is written on
 * the host. Limits and rules:
 *   - meshes of at most 16,777,216 elements; larger ones fail with LPG_EINVAL;
 *   - the array is shared by every call on a device and keeps the last call's contents
 *     (each call clears what it needs), so calls that overlap on the GPU race: order them;
 *   - the first call on a device looks the array's device address up (cudaGetSymbolAddress
 *     with that device current); make that first call before any stream capture begins.
 */
int lpg_fem_feasible_step_noalloc(lpg_fem_t h, const double* u, const double* du, double* alpha);

/*
 * Parameter VJP of the force response: per element [d/dlambda, d/dmu] of w . g(u).
 * Replaces VolumetricFemForceMaterialResponse::eval_vjp
 *   (src/core/fem/assembly/detail/volumetric_fem_force_response.hpp:155-179 through
 *   src/core/energy/response/mesh_response.cpp:70-98) with an ElementDofMap
 *   (per-element output, num_tets * 2) or ConstantDofMap (summed in element order, 2).
 */
int lpg_fem_force_vjp_theta(lpg_fem_t h, const double* u, const double* w, int io_mem, int per_element,
                            double* out);

/* Options of newton_solve (src/core/solver/newton.hpp:13-20) plus the GPU linear solve. */
typedef struct {
    double gradient_tolerance;  /* required; see stop_rule */
    int max_iterations;         /* default 50 */
    int hessian;                /* lpg_hessian_kind, default LPG_HESSIAN_PROJECTED */
    int max_line_search_steps;  /* default 30 */
    double line_search_shrink;  /* default 0.5 */
    int stop_rule;              /* 0: max|g_free| <= tol (newton.cpp:34-36); 1: ||g_free||_2 <= tol ||g_free(x0)||_2 */
    int accept_rule;            /* 0: E(trial) <= E + 16 eps max(1,|E|) (newton.cpp:83-86); 1: Armijo c=1e-4 plus that noise */
    int precision;              /* lpg_precision of the Hessian and PCG; residual and energy stay FP64 */
    double cg_tolerance;        /* forcing-term cap: relative PCG residual min(cg_tolerance, sqrt(||g||/||g0||)) */
    int cg_max_iterations;      /* per Newton iteration */
    double exact_below;         /* not in the reference; default 0 (off): once ||g_free||_2 <= exact_below
                                   ||g_free(x0)||_2, use the Exact Hessian instead of `hessian` (near a stable
                                   equilibrium it is positive definite, and Newton converges quadratically) */
} lpg_newton_options;

typedef struct {
    int status;                  /* 0 Converged, 1 MaxIterations, 2 StepTooSmall, 3 NoDescentDirection (newton.hpp:22-31) */
    int iterations;              /* accepted steps */
    double energy;
    double gradient_norm;        /* of the chosen stop rule */
    double gradient_norm0;       /* ||g_free(x0)||_2 */
    int64_t cg_iterations;       /* total PCG iterations */
    int line_search_evaluations;
    double seconds;              /* device time of the solve */
} lpg_newton_result;

void lpg_newton_default_options(lpg_newton_options* options);

/*
 * Minimises E(u) = elastic(u) - f_ext . u over the free DOFs from x0; fixed DOFs keep
 * their x0 values. Replaces
 *   newton_solve(Energy&, const DofReduction&, x0, const NewtonOptions&, SparseSolver&, on_iteration)
 *   (src/core/solver/newton.hpp:67-69, newton.cpp:112-183)
 * where the load is the reference's QuadraticEnergy with b = -f_ext in a WeightedSumEnergy
 * (quadratic_energy.hpp:10-20, weighted_sum_energy.hpp:16-47), and the direct
 * SparseSolver is replaced by block-Jacobi PCG on the 3x3 block-CSR Hessian.
 *   fixed_dofs : num_fixed unique DOF indices (host)
 *   f_ext      : num_dofs or NULL (io_mem)
 *   x0, x_out  : num_dofs (io_mem)
 */
int lpg_newton_solve(lpg_fem_t h, const int32_t* fixed_dofs, int num_fixed, const double* f_ext, const double* x0,
                     int io_mem, const lpg_newton_options* options, double* x_out, lpg_newton_result* result);

/*
 * What one Newton iteration did: the reference's NewtonStep (src/core/solver/newton.hpp:34-44),
 * reported at the same points (after each accepted step, and once for the iteration that ends
 * the solve; newton.cpp:123-181), plus two fields it does not have.
 */
typedef struct {
    int iteration;
    double energy;
    double gradient_norm;        /* max |g| over the free DOFs (the reference's norm) */
    int pattern_changed;         /* 1 on the first evaluation (the Hessian pattern is fixed after it) */
    int diagonal_shifts;         /* diagonal shifts of the descent-direction search (10 when none worked) */
    double feasible_step;        /* max_feasible_step's bound on the step; 0 when no search ran */
    double step;                 /* the accepted step length; 0 when none was */
    int line_search_evaluations;
    double gradient_norm_2;      /* ||g_free||_2 (not in the reference) */
    int64_t cg_iterations;       /* PCG iterations of this iteration (not in the reference) */
} lpg_newton_step;

/* Per-iteration callback: return 0 to continue; any other value stops the solve, which then
 * returns LPG_ESTOPPED (for a binding's callback that raised). */
typedef int (*lpg_newton_callback)(const lpg_newton_step* step, void* user);

/*
 * A caller's volumetric material (the reference's PyVolumetricMaterial / TorchVolumetricMaterial
 * in the Material slot of VolumetricFemEnergy, src/python/fem.py:59-109, src/python/torch.py:72-94):
 * given F at every material row (rows 3x3 row-major matrices on the device: one row per tet,
 * or per quadrature point of a hex, element-major), it writes W (rows), and with want >= 1
 * P = dW/dF (9 rows, row-major 3x3), with want = 2 A = d2W/dF2 (81 rows, A[9 (3 i + j) + 3 k + l]
 * = d2W / dF_ij dF_kl) into the library's device buffers, on the handle's stream. Returns 0, or
 * non-zero to stop the solve (LPG_ESTOPPED).
 */
typedef int (*lpg_material_fn)(const double* F, int rows, int want, double* W, double* P, double* A, void* user);

/* A caller's material bound on the step from x along dx (PyVolumetricMaterial.eval_feasible_step):
 * F = I + grad x and G = I + grad dx at every material row (device, as for lpg_material_fn; the
 * increment is dF = G - I); writes a value in [0, 1] to *alpha and returns 0, or non-zero to
 * stop the solve (LPG_ESTOPPED). */
typedef int (*lpg_feasible_fn)(const double* F, const double* G, int rows, double* alpha, void* user);

/*
 * The terms of a weighted-sum potential around the handle's elastic energy, for
 * lpg_newton_solve_terms (the reference's WeightedSumEnergy, weighted_sum_energy.hpp:16-47, of
 * one VolumetricFemEnergy and QuadraticEnergy terms, quadratic_energy.hpp:10-20, summed
 * beforehand into one A; f_ext carries the linear part):
 *   E(x) = elastic_weight elastic(x) + 1/2 x^T A x - f_ext . x + constant.
 * A is a scalar CSR matrix on the host (num_dofs rows, a_indptr[num_dofs + 1], a_indices and
 * a_values of a_indptr[num_dofs] entries; duplicates are summed) or a_indptr = NULL for none. It
 * must be symmetric and lie inside the elastic Hessian's pattern (vertex pairs sharing an
 * element), else LPG_EINVAL. on_iteration (may be NULL) is called with user at every step.
 * With material set, every evaluation of the elastic term exports F, calls material and
 * integrates its W, P and A (as lpg_fem_eval_material); feasible, if set, bounds each line search.
 */
typedef struct {
    double elastic_weight; /* finite and non-zero; 1 for the elastic energy alone */
    const int32_t* a_indptr;
    const int32_t* a_indices;
    const double* a_values;
    double constant;
    lpg_newton_callback on_iteration;
    void* user;
    lpg_material_fn material;   /* NULL: the handle's neo-Hookean records; else the caller's material
                                   (the handle then carries rest geometry only) */
    lpg_feasible_fn feasible;   /* NULL: the positive-determinant step of lpg_fem_feasible_step */
    void* material_user;
} lpg_newton_terms;

/*
 * lpg_newton_solve over the weighted-sum potential of terms (NULL: the elastic energy and the
 * load alone, as lpg_newton_solve). Replaces newton_solve(energy, fixed, x0, options, solver,
 * on_iteration) (src/core/solver/newton.hpp:67-69; binding src/binding/solver/newton.cpp:62-82)
 * for such an energy, with its on_iteration callback.
 */
int lpg_newton_solve_terms(lpg_fem_t h, const lpg_newton_terms* terms, const int32_t* fixed_dofs, int num_fixed,
                           const double* f_ext, const double* x0, int io_mem, const lpg_newton_options* options,
                           double* x_out, lpg_newton_result* result);

/*
 * The adjoint solve of StaticEquilibriumResponse over a weighted-sum potential
 * (static_equilibrium_response.cpp:43-68): lambda (num_dofs, io_mem; fixed entries zero) of
 * K_ff lambda = dLdu_free, K the Exact Hessian of the potential of terms (NULL: the handle's
 * elastic energy) at u_star, by PCG with FP64 refinement and the reference's residual check. A
 * caller then forms the parameter gradient -(dg/dtheta)^T lambda with its own force response
 * (for a Python material, through the material's d2W/dF dtheta).
 */
int lpg_adjoint_solve_terms(lpg_fem_t h, const lpg_newton_terms* terms, const double* u_star, const double* dLdu,
                            const int32_t* fixed_dofs, int num_fixed, int io_mem, int precision, double cg_tolerance,
                            double* lambda_out);

/* Per-mesh outcome of lpg_batch_newton_solve (status as lpg_newton_result.status). */
typedef struct {
    int status;
    int iterations;
    double energy;
    double gradient_norm;
    double gradient_norm0;
    double seconds; /* from the start of the call to the iteration that ended this mesh */
} lpg_batch_mesh_result;

/*
 * Batched newton_solve (no reference counterpart; the reference solves one energy per call):
 * num_meshes independent tet meshes (a tet handle; others fail with LPG_EINVAL) stored in one
 * handle as contiguous vertex ranges
 * [vertex_offsets[m], vertex_offsets[m+1]) and element ranges [element_offsets[m],
 * element_offsets[m+1]) (every element inside its mesh's vertices). Assembly and SpMV run once
 * over all meshes; every mesh has its own stop test, PCG scalars (one block-Jacobi PCG per mesh,
 * in lockstep), feasible step and line search, as lpg_newton_solve has for one mesh. Where a
 * mesh's PCG direction is not a descent direction, that iteration takes -g for the mesh instead
 * of lpg_newton_solve's diagonal shifts. With exact_below the Exact Hessian is used once every
 * unfinished mesh meets the threshold. fixed_dofs, f_ext, x0 and x_out are over the whole
 * handle. per_mesh[num_meshes] receives the per-mesh outcomes; result (may be NULL) the totals
 * (status = the worst mesh's, iterations = Newton iterations run, cg_iterations = lockstep PCG
 * iterations, energy = the sum). A finished mesh is skipped by the later iterations' assembly,
 * projection, feasible step and PCG.
 */
int lpg_batch_newton_solve(lpg_fem_t h, int num_meshes, const int32_t* vertex_offsets, const int32_t* element_offsets,
                           const int32_t* fixed_dofs, int num_fixed, const double* f_ext, const double* x0, int io_mem,
                           const lpg_newton_options* options, double* x_out, lpg_batch_mesh_result* per_mesh,
                           lpg_newton_result* result);

/*
 * Adjoint of the static equilibrium: solves K_ff lambda = dLdu_free with the EXACT
 * Hessian at u_star and returns dtheta = -(dg/dtheta)^T lambda, per element
 * (num_tets * 2) or summed (2). Replaces the transpose branch of
 *   StaticEquilibriumResponse::evaluate (src/core/solver/static_equilibrium_response.cpp:43-88)
 * with its residual check ||K lambda - rhs|| <= 1e-8 (1 + ||rhs||) (:61-68).
 * lambda_out (num_dofs, io_mem) may be NULL.
 */
int lpg_adjoint_theta(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed_dofs,
                      int num_fixed, int io_mem, int precision, double cg_tolerance, int per_element, double* dtheta,
                      double* lambda_out);

/*
 * Rest-position sensitivity of the elastic force (no reference counterpart: the reference
 * differentiates its force response in theta and Fp only). out = (dg/dX)^T w, where g is
 * the gradient of the elastic energy in u and X the vertex rest positions (num_dofs values,
 * io_mem). Needs a handle created from vertex positions (Xe == NULL) without a plastic field
 * (LPG_EINVAL otherwise). Per element d(w . g_e)/dX, summed per vertex in element order.
 */
int lpg_fem_force_vjp_rest(lpg_fem_t h, const double* u, const double* w, int io_mem, double* out);

/*
 * Adjoint rest-position sensitivity: the adjoint solve of lpg_adjoint_theta, then
 * dX = -(dg/dX)^T lambda (num_dofs values, io_mem). Same requirements as
 * lpg_fem_force_vjp_rest. lambda_out (num_dofs, io_mem) may be NULL.
 */
int lpg_adjoint_rest(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed_dofs, int num_fixed,
                     int io_mem, int precision, double cg_tolerance, double* dX, double* lambda_out);

/*
 * Replaces the Lame parameters [lambda, mu] (num_tets * 2 when theta_per_element, else 2;
 * host) of an existing handle, keeping its plan and rest geometry (no reference
 * counterpart; the reference builds a new energy for new parameters). Values are checked at
 * evaluation like the constructor's (lambda >= 0, mu > 0).
 */
int lpg_fem_set_theta(lpg_fem_t h, const double* theta, int theta_per_element);

/*
 * Plastic field of an existing handle: VolumetricFemForceFpResponse's input
 * (src/core/fem/assembly/volumetric_fem_force_fp_response.hpp:8-10; the reference builds the
 * response with a new Fp per evaluation). Fp: 9 column-major values per element
 * (fp_per_element) or 9 shared ones, host; NULL removes the plastic field (Fp = I). Checked as
 * MultiplicativeKinematics does (finite: LPG_EINVAL; det Fp > 0: LPG_EDOMAIN). The plan, rest
 * geometry and [lambda, mu] are kept.
 */
int lpg_fem_set_fp(lpg_fem_t h, const double* Fp, int fp_per_element);

/*
 * (d g / d vec Fp)^T w of VolumetricFemForceFpResponse::eval_vjp (MeshResponse::product,
 * mesh_response.cpp:70-98, with NeoHookean::eval_d2W_dF_dFp, neo_hookean.cpp:103-128) at
 * displacement u: per element 9 values (column-major Fp index) when per_element, else their
 * sum over elements (9). u, w: num_dofs values (io_mem); out likewise.
 */
int lpg_fem_force_vjp_fp(lpg_fem_t h, const double* u, const double* w, int io_mem, int per_element, double* out);

/*
 * StaticEquilibriumResponse VJP in the plastic field (static_equilibrium_response.cpp:43-88
 * with the Fp force response): K lambda = dL/du on the free DOFs with the Exact FP64 Hessian
 * at u_star (as lpg_adjoint_theta), then dFp = -(dg/dFp)^T lambda, 9 per element or 9 summed.
 */
int lpg_adjoint_fp(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed_dofs, int num_fixed,
                   int io_mem, int precision, double cg_tolerance, int per_element, double* dFp, double* lambda_out);

/*
 * Materials evaluated by the caller (the reference's PyVolumetricMaterial and
 * TorchVolumetricMaterial, src/python/fem.py:59-109, src/python/torch.py:72-94, bound through
 * src/binding/fem/material/py_material.cpp), on a handle created without a plastic field (the
 * caller's material receives Fp itself; LPG_EINVAL otherwise):
 *   lpg_fem_deformation_gradients: F = I + grad u of every element at u (num_dofs values,
 *     io_mem), 9 values per element, row-major F_ij at 3 i + j, into F (io_mem);
 *   lpg_fem_eval_material: with the caller's W (num_tets, the density per reference volume),
 *     P = dW/dF (9 per element, row-major) and, for a Hessian, A = d2W/dF2 (81 per element,
 *     [3 i + j][3 k + l]) — host or device (in_mem) — writes E = sum vol W, the gradient
 *     (sum vol P grad N_a per vertex; may be NULL) and the Hessian sum vol B^T A B (LPG_HESSIAN_
 *     EXACT) or its per-element eigenvalue clamp (LPG_HESSIAN_PROJECTED) in BSR or CSC order, as
 *     lpg_fem_eval does (grad and hess in out_mem). Each element's A is symmetrised,
 *     (A + A^T) / 2, before use; non-finite material outputs give LPG_EDOMAIN. P may be NULL
 *     when grad is NULL, A when hessian is LPG_HESSIAN_NONE.
 * On a hex handle (lpg_fem_create_hex with n points per axis) a material row is a quadrature
 * point instead of an element: F, W, P and A have num_cells * n^3 rows, the points of an element
 * consecutive in the quadrature order, and the sums run over the points with weight
 * w_q = weight_q det J_q (E = sum w_q W, g_a = sum w_q P grad N_a, H = sum w_q B_q^T A_q B_q).
 * LPG_HESSIAN_PROJECTED then projects each hex's 24x24 Hessian as lpg_fem_eval does.
 */
int lpg_fem_deformation_gradients(lpg_fem_t h, const double* u, int io_mem, double* F);
int lpg_fem_eval_material(lpg_fem_t h, const double* W, const double* P, const double* A, int in_mem, double* energy,
                          double* grad, int hessian, int precision, int layout, void* hess, int out_mem);

/*
 * Autotuner (no reference counterpart). Three kernels come in launch variants that differ in
 * register budget and loop unrolling only, so every variant computes bitwise the same
 * results: the Exact-Hessian assembly (3 variants per precision), the PCG SpMV of the
 * Newton and adjoint solvers (3 per precision) and the projected Hessian's eigenvalue clamp
 * (2 in FP32, 1 in FP64). lpg_fem_create times every variant on the new handle's mesh (rest
 * state; seeded 9x9 matrices for the clamp; mean of 3 launches after a warm-up) and keeps the
 * fastest per precision, unless the environment variable LPG_AUTOTUNE is "0" (then variant 0
 * everywhere). lpg_fem_autotune runs the timing again.
 * lpg_fem_get_tuning: choice[6] = {assembly FP64, assembly FP32, SpMV FP64, SpMV FP32,
 *   clamp FP64, clamp FP32}; ms[18] = mean ms per launch, ms[6 f + 3 p + v] for family f
 *   (assembly, SpMV, clamp), precision p (FP64, FP32) and variant v; NaN where not timed
 *   (variants a family does not have, and the FP64 clamp, which has one).
 *   Either output may be NULL.
 * lpg_fem_set_tuning: forces choices (same order; -1 keeps the current one); LPG_EINVAL
 *   for an index outside the family's variants.
 */
int lpg_fem_autotune(lpg_fem_t h);

/*
 * VEG volume-mesh files: read_veg / write_veg (src/core/mesh/io/veg.cpp; Python
 * mesh.read_veg / mesh.write_veg, src/binding/mesh/io/veg.cpp). lpg_read_veg parses the file
 * (*VERTICES, one *ELEMENTS section of TET or CUBIC cells, *INCLUDE, '#' comments, 0- or
 * 1-based ids) and reports num_vertices, num_cells and cell_width (4 or 8); positions (3 per
 * vertex) and cells (cell_width per cell, 0-based) are filled when not NULL, so a caller
 * asks for the sizes first (that call keeps the parsed mesh for the next call on the same
 * thread with the same, unchanged file, which then does not parse it again). File and format
 * errors are LPG_EIO, an invalid mesh LPG_EINVAL.
 * lpg_write_veg writes 1-based ids and 17 significant digits (exact round trip).
 */
int lpg_read_veg(const char* path, int* num_vertices, int* num_cells, int* cell_width, double* positions,
                 int32_t* cells);
int lpg_write_veg(const char* path, int num_vertices, const double* positions, int num_cells, int cell_width,
                  const int32_t* cells);
int lpg_fem_get_tuning(lpg_fem_t h, int32_t choice[6], double ms[18]);
int lpg_fem_set_tuning(lpg_fem_t h, const int32_t choice[6]);

#ifdef __cplusplus
}
#endif
#endif
