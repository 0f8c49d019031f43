// lpg_solver.h -- the handle behind lpg_fem_t and the solver entry points.
#pragma once

#include <atomic>
#include <cstddef>
#include <vector>

#include "lpg_internal.h"

namespace lpg {

// Owned device allocation that only grows.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer();
    void* ensure(size_t n);
    template <class T> T* as(size_t count) { return static_cast<T*>(ensure(count * sizeof(T))); }
};

void raise_status(unsigned st);

} // namespace lpg

struct lpg_fem {
    int device = 0;
    bool from_vertices = true; // rest geometry given as vertex positions (no per-element corners)
    cudaStream_t own_stream = nullptr, stream = nullptr;
    lpg::HostPlan plan;
    lpg::DevMesh dm;
    std::atomic<bool> busy{false};
    // Plan and element data.
    lpg::DeviceBuffer b_row_ptr, b_col_idx, b_inc_ptr, b_tets, b_rec64, b_rec32, b_fpinv64, b_fpinv32, b_diag_slot,
        b_unused;
    lpg::DeviceBuffer b_hex[4]; // hex meshes: rest positions, cells, [lambda, mu], quadrature table
    lpg::DeviceBuffer b_herm;   // Hermite hex meshes: box edge lengths per element
    lpg::DeviceBuffer d_herm_q; // Hermite projected Hessian: eigenvector scratch, 192^2 doubles per CTA
    lpg::DeviceBuffer b_cl[11]; // assembly clusters
    lpg::DeviceBuffer b_tc[13]; // tet assembly clusters
    lpg::DeviceBuffer b_sell[6]; // sliced-ELL pattern of the solvers
    lpg::DeviceBuffer bt_int[8], bt_dbl[4], bt_skip[2]; // batched Newton (bt_skip: per-cluster skip flags)
    // Scratch of the evaluation entry points.
    lpg::DeviceBuffer d_plist, d_pcount; // elements listed for the projection's eigenvalue clamp
    lpg::DeviceBuffer d_mat[6];          // material outputs (W, P, A), per-element energies, F and G
    lpg::DeviceBuffer d_status, d_cluster_energy, d_energy, d_block, d_alpha, d_u, d_u2, d_grad, d_hess, d_proj, d_vjp;
    // Solver state (Newton / PCG / adjoint).
    lpg::DeviceBuffer s_x, s_g, s_f, s_d, s_trial, s_mask, s_hess, s_hess64, s_dinv, s_r, s_z, s_p, s_ap, s_xcg, s_r64,
        s_b64, s_scal, s_part, s_flag, d_flush, s_p2, s_mask4;
    lpg::DeviceBuffer s_q[6]; // quadratic term of a weighted-sum potential (CSR, solver-layout entries, A x)
    std::vector<double> geo_base; // per element: G = rows of Dm^-1 (9) and w_dV, before any Fp
    lpg::Tuning tune; // autotuned launch variants (lpg::autotune)
    // CUDA graph of a chunk of PCG iterations, reused while its pointers stay the same.
    cudaGraphExec_t pcg_graph = nullptr;
    const void* pcg_graph_key[12] = {};
    cudaGraphExec_t batch_graph = nullptr; // the batched (per-mesh) PCG iterations
    const void* batch_graph_key[12] = {};
    ~lpg_fem();
    void sync();
    unsigned take_status();
    const double* stage_in(const double* p, int mem, lpg::DeviceBuffer& buf, size_t n);
    // Enqueues one evaluation on the handle's stream (no synchronisation).
    void eval_async(const double* du, double* dgrad, int hessian, int precision, int layout, void* dhess,
                    double* delem, cudaEvent_t ev_begin = nullptr, cudaEvent_t ev_end = nullptr,
                    const int* emesh = nullptr, const int* mesh_exact = nullptr,
                    const unsigned char* tc_skip = nullptr, const unsigned char* cl_skip = nullptr);
};

namespace lpg {
// terms (may be null): elastic weight, quadratic term, constant and per-iteration callback.
void newton_solve(lpg_fem& h, const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                  const lpg_newton_options& o, double* x_out, lpg_newton_result* res,
                  const lpg_newton_terms* terms = nullptr);
// The adjoint solve alone over a weighted-sum potential (terms may be null): lambda of
// K_ff lambda = dL/du_free with the potential's Exact Hessian at u*.
void adjoint_lambda(lpg_fem& h, const lpg_newton_terms* terms, const double* u_star, const double* dLdu,
                    const int32_t* fixed, int nfixed, int io_mem, int precision, double cg_tolerance, double* lambda_out);
void adjoint_theta(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                   int precision, double cg_tolerance, int per_element, double* dtheta, double* lambda_out);
void batch_newton_solve(lpg_fem& h, int num_meshes, const int32_t* vertex_offsets, const int32_t* element_offsets,
                        const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                        const lpg_newton_options& o, double* x_out, lpg_batch_mesh_result* per_mesh,
                        lpg_newton_result* total);
void adjoint_fp(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                int precision, double cg_tolerance, int per_element, double* dFp, double* lambda_out);
// Times every launch variant of the tuned kernels on this handle's mesh (rest state, seeded
// clamp inputs) and keeps the fastest per precision in h.tune.
void autotune(lpg_fem& h);
void adjoint_rest(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                  int precision, double cg_tolerance, double* dX, double* lambda_out);
} // namespace lpg
