// lpg_assemble.cu -- sm_100a kernels of the neo-Hookean element pass.
//
// Element arithmetic follows the reference NeoHookean (src/core/fem/material/volumetric/
// neo_hookean.cpp:14-60) on a TetP1 element with centroid quadrature
// (src/core/fem/assembly/volumetric_fem_energy.hpp:78-123, dof_derivatives.cpp:22-51),
// written in closed form: with grad N_a the P1 shape gradients, h_a = F^-T grad N_a and
// p = lambda log J - mu,
//   E_e   = vol * psi,   psi = mu/2 (|F|^2 - 3) - mu log J + lambda/2 (log J)^2
//   g_a   = vol * P grad N_a,   P = mu F + p F^-T
//   H_ab  = vol * [ mu (grad N_a . grad N_b) I + lambda h_a h_b^T - p h_b h_a^T ]
// which equals vol * B^T (d2W/dF2) B for B = kron(grad N^T, I3).
//
// Assembly (replacing EnergyAssembler::assemble, src/core/dof/energy_assembler.cpp:123-170)
// is atomic-free over vertex clusters: a thread block evaluates the elements incident to its
// cluster of rows once, then sums every block slot of those rows over the slot's contributor
// list, in ascending element order (the reference's per-column order,
// energy_assembler.cpp:49-54). An off-diagonal block is summed in the orientation of its
// lower-numbered vertex and stored transposed for the other, so the assembled matrix is
// bitwise symmetric. The projected Hessian goes through per-element blocks (project_kernel,
// clamp_kernel) gathered by the same cluster plan (block_gather_kernel).

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include <cuda_pipeline.h>

#include "lpg_internal.h"
#include "lpg_clamp9.h"
#include "lpg_psd.h"

namespace lpg {
namespace {

template <typename R> struct M;
template <> struct M<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double log1p_(double x) { return log1p(x); }
    static __device__ __forceinline__ double log_(double x) { return log(x); }
    static __device__ __forceinline__ bool finite(double x) { return isfinite(x); }
};
template <> struct M<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float log1p_(float x) { return log1pf(x); }
    static __device__ __forceinline__ float log_(float x) { return logf(x); }
    static __device__ __forceinline__ bool finite(float x) { return isfinite(x); }
};

template <typename R> __device__ __forceinline__ const R* rec_ptr(const DevMesh& m);
template <> __device__ __forceinline__ const double* rec_ptr<double>(const DevMesh& m) { return m.rec64; }
template <> __device__ __forceinline__ const float* rec_ptr<float>(const DevMesh& m) { return m.rec32; }
template <typename R> __device__ __forceinline__ const R* fpinv_ptr(const DevMesh& m);
template <> __device__ __forceinline__ const double* fpinv_ptr<double>(const DevMesh& m) { return m.fpinv64; }
template <> __device__ __forceinline__ const float* fpinv_ptr<float>(const DevMesh& m) { return m.fpinv32; }

// 12-value element record, loaded with 16-byte vector loads.
template <typename R> __device__ __forceinline__ void load_rec(const R* rec, int e, R* r);
template <> __device__ __forceinline__ void load_rec<double>(const double* rec, int e, double* r) {
    const double2* p = reinterpret_cast<const double2*>(rec + 12 * static_cast<size_t>(e));
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double2 v = __ldg(p + k);
        r[2 * k] = v.x;
        r[2 * k + 1] = v.y;
    }
}
template <> __device__ __forceinline__ void load_rec<float>(const float* rec, int e, float* r) {
    const float4* p = reinterpret_cast<const float4*>(rec + 12 * static_cast<size_t>(e));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 v = __ldg(p + k);
        r[4 * k] = v.x;
        r[4 * k + 1] = v.y;
        r[4 * k + 2] = v.z;
        r[4 * k + 3] = v.w;
    }
}

// Kinematics of one element: shape gradients n[a], F, F^-T, log J, psi.
template <typename R> struct Kin {
    R n[4][3];
    R F[9];   // row-major
    R FiT[9]; // row-major
    R logJ, psi, vol, lam, mu;
};

// Returns status bits. u is FP64; edge differences are formed in FP64 and rounded once.
// FP64: det F and log det F as the reference computes them (neo_hookean.cpp:14-23). FP32:
// det F - 1 from the invariants of the displacement gradient and log1p, which keeps log J
// accurate near the rest state. Validity is checked once on J; the rare failure path then
// tells a non-finite input from a non-finite F and from det F <= 0.
template <typename R>
__device__ __forceinline__ unsigned kinematics_of(const DevMesh& m, int e, const R (&rec)[12], const double (&uu)[4][3],
                                                  Kin<R>& k);

template <typename R>
__device__ __forceinline__ unsigned kinematics(const DevMesh& m, int e, const int4 tv, const double* __restrict__ u,
                                               Kin<R>& k) {
    R rec[12];
    load_rec<R>(rec_ptr<R>(m), e, rec);
    const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
    double uu[4][3];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) uu[c][i] = __ldg(u + 3 * static_cast<size_t>(vs[c]) + i);
    return kinematics_of<R>(m, e, rec, uu, k);
}

// Edge differences of the displacements, formed in FP64 and rounded once: Ds[i][c] =
// u_{c+1,i} - u_{0,i}; returns whether every displacement is finite.
template <typename R> __device__ __forceinline__ bool edge_differences(const double (&uu)[4][3], R (&Ds)[3][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) Ds[i][c] = static_cast<R>(uu[c + 1][i] - uu[0][i]);
    bool in_ok = true;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) in_ok = in_ok && isfinite(uu[c][i]);
    return in_ok;
}

template <typename R>
__device__ __forceinline__ unsigned kinematics_ds(const DevMesh& m, int e, const R (&rec)[12], const R (&Ds)[3][3],
                                                  bool in_ok, Kin<R>& k);

// The element's kinematics from its record (rec) and its vertices' displacements (uu).
template <typename R>
__device__ __forceinline__ unsigned kinematics_of(const DevMesh& m, int e, const R (&rec)[12], const double (&uu)[4][3],
                                                  Kin<R>& k) {
    R Ds[3][3];
    const bool in_ok = edge_differences<R>(uu, Ds);
    return kinematics_ds<R>(m, e, rec, Ds, in_ok, k);
}

// The element's kinematics from its record and its displacement edge differences (in_ok: every
// displacement was finite).
template <typename R>
__device__ __forceinline__ unsigned kinematics_ds(const DevMesh& m, int e, const R (&rec)[12], const R (&Ds)[3][3],
                                                  bool in_ok, Kin<R>& k) {
    using X = M<R>;
    unsigned st = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < 3; ++j) k.n[c + 1][j] = rec[3 * c + j];
#pragma unroll
    for (int j = 0; j < 3; ++j) k.n[0][j] = -(k.n[1][j] + k.n[2][j] + k.n[3][j]);
    k.vol = rec[9];
    k.lam = rec[10];
    k.mu = rec[11];
    if (!(k.lam >= R(0) && k.mu > R(0) && k.lam < R(INFINITY) && k.mu < R(INFINITY))) st |= ST_BAD_THETA;
    R H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            H[3 * i + j] = X::fma(Ds[i][2], rec[6 + j], X::fma(Ds[i][1], rec[3 + j], X::mul(Ds[i][0], rec[j])));
    const R* fpi = fpinv_ptr<R>(m);
    if (fpi == nullptr) {
#pragma unroll
        for (int t = 0; t < 9; ++t) k.F[t] = H[t];
        k.F[0] += R(1);
        k.F[4] += R(1);
        k.F[8] += R(1);
    } else {
        const R* o = fpi + 9 * static_cast<size_t>(e);
#pragma unroll
        for (int t = 0; t < 9; ++t) k.F[t] = __ldg(o + t) + H[t];
    }
    const R* F = k.F;
    R C[9]; // cofactors: F^-T = C / det F
    C[0] = F[4] * F[8] - F[5] * F[7];
    C[1] = F[5] * F[6] - F[3] * F[8];
    C[2] = F[3] * F[7] - F[4] * F[6];
    C[3] = F[2] * F[7] - F[1] * F[8];
    C[4] = F[0] * F[8] - F[2] * F[6];
    C[5] = F[1] * F[6] - F[0] * F[7];
    C[6] = F[1] * F[5] - F[2] * F[4];
    C[7] = F[2] * F[3] - F[0] * F[5];
    C[8] = F[0] * F[4] - F[1] * F[3];
    R J, sqm3;
    if (sizeof(R) == 8 || fpi != nullptr) {
        J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
        k.logJ = X::log_(J);
        R ff = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) ff = X::fma(F[t], F[t], ff);
        sqm3 = ff - R(3);
    } else {
        const R c1 = H[0] + H[4] + H[8];
        const R c2 = (H[0] * H[4] - H[1] * H[3]) + (H[0] * H[8] - H[2] * H[6]) + (H[4] * H[8] - H[5] * H[7]);
        const R c3 = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
                     H[2] * (H[3] * H[7] - H[4] * H[6]);
        const R Jm1 = c1 + c2 + c3;
        J = R(1) + Jm1;
        k.logJ = X::log1p_(Jm1);
        R hh = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) hh = X::fma(H[t], H[t], hh);
        sqm3 = R(2) * c1 + hh;
    }
    const R iJ = R(1) / J;
#pragma unroll
    for (int t = 0; t < 9; ++t) k.FiT[t] = C[t] * iJ;
    k.psi = R(0.5) * k.mu * sqm3 - k.mu * k.logJ + R(0.5) * k.lam * k.logJ * k.logJ;
    if (!(J > R(0) && J < R(INFINITY) && k.psi == k.psi && k.psi < R(INFINITY) && k.psi > R(-INFINITY))) {
        bool f_ok = true;
#pragma unroll
        for (int t = 0; t < 9; ++t) f_ok = f_ok && X::finite(F[t]);
        st |= !in_ok ? ST_BAD_INPUT : !f_ok ? ST_NONFINITE_F : !(J > R(0)) || !X::finite(J) ? ST_BAD_DET
                                                                                          : ST_NONFINITE_OUT;
    }
    return st;
}

template <typename R> struct HOut;
template <> struct HOut<double> { using T = double; };
template <> struct HOut<float> { using T = float; };


// Orthonormal basis of {x in R^4 : sum x = 0}: q = 1/2 [[1,1,1],[1,-1,-1],[-1,1,-1],[-1,-1,1]].
// P1 shape gradients satisfy grad N = q (q^T grad N), so the element Hessian is
// kron(q, I3) M kron(q, I3)^T for the 9x9 matrix M below, and clamping M's eigenvalues
// clamps the element Hessian's (its remaining three eigenvalues are the zero translations).
template <typename R> __device__ __forceinline__ R qbasis(int a, int j) {
    const int sgn = (a == 0) ? 1 : ((a == j + 1) ? 1 : -1);
    return sgn > 0 ? R(0.5) : R(-0.5);
}

// Gradient rows of vertices that no element references are zero.
__global__ void zero_rows_kernel(double* __restrict__ grad, const int* __restrict__ rows, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const size_t r = rows[i];
        grad[3 * r] = 0;
        grad[3 * r + 1] = 0;
        grad[3 * r + 2] = 0;
    }
}

// Deterministic sum of n doubles: kSumBlocks blocks sum fixed contiguous chunks (fixed thread ->
// index map and tree), then one block sums the partials in order.
constexpr int kSumBlocks = 256;
__global__ void __launch_bounds__(256) sum_partial_kernel(const double* __restrict__ x, int n, double* part) {
    __shared__ double s[8];
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    double v = 0;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) v += x[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) t += s[w];
        part[blockIdx.x] = t;
    }
}
__global__ void __launch_bounds__(256) sum_final_kernel(const double* __restrict__ part, int nb, double* out) {
    __shared__ double s[8];
    double v = threadIdx.x < nb ? part[threadIdx.x] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) t += s[w];
        *out = t;
    }
}

// ---------------------------------------------------------------------------
// Feasible step: eval_positive_det_feasible_step (positive_det_feasible_step.cpp:13-84)
// on F = I + Ds G and dF = dDs G, per element, then the minimum (mesh_energy.cpp:88-107).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double det3r(const double* a) { // row-major
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// Column j of a row-major 3x3 is (a[j], a[3+j], a[6+j]).
__device__ double positive_det_step(const double* A, const double* dA, unsigned& st) {
    const double detA = det3r(A);
    if (!isfinite(detA) || detA <= 0) {
        st |= ST_BAD_DET;
        return 0;
    }
    double a[9], d[9];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double s = 0, t = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            s = fmax(s, fabs(A[3 * i + j]));
            t = fmax(t, fabs(dA[3 * i + j]));
        }
        const double scale = fmax(s, t);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            a[3 * i + j] = A[3 * i + j] / scale;
            d[3 * i + j] = dA[3 * i + j] / scale;
        }
    }
    // Columns x_j = (m[j], m[3+j], m[6+j]); triple product x . (y cross z).
    auto triple = [](const double* x, int jx, const double* y, int jy, const double* z, int jz) {
        const double x0 = x[jx], x1 = x[3 + jx], x2 = x[6 + jx];
        const double y0 = y[jy], y1 = y[3 + jy], y2 = y[6 + jy];
        const double z0 = z[jz], z1 = z[3 + jz], z2 = z[6 + jz];
        return x0 * (y1 * z2 - y2 * z1) + x1 * (y2 * z0 - y0 * z2) + x2 * (y0 * z1 - y1 * z0);
    };
    const double c0 = det3r(a);
    const double c1 = triple(d, 0, a, 1, a, 2) + triple(a, 0, d, 1, a, 2) + triple(a, 0, a, 1, d, 2);
    const double c2 = triple(d, 0, d, 1, a, 2) + triple(d, 0, a, 1, d, 2) + triple(a, 0, d, 1, d, 2);
    const double c3 = det3r(d);
    if (!(c0 > 0)) return 0;
    const double eps = 2.220446049250313e-16;
    auto value = [&](double t) { return fma(fma(fma(c3, t, c2), t, c1), t, c0); };
    auto tol = [&](double t) { return 64 * eps * (((fabs(c3) * t + fabs(c2)) * t + fabs(c1)) * t + c0); };
    double knots[4] = {0, 1, 0, 0};
    int count = 2;
    auto add_knot = [&](double t) {
        if (t > 0 && t < 1) knots[count++] = t;
    };
    const double qa = 3 * c3, qb = 2 * c2, qc = c1;
    if (qa == 0) {
        if (qb != 0) add_knot(-qc / qb);
    } else {
        double disc = fma(qb, qb, -4 * qa * qc);
        const double err = 8 * eps * (qb * qb + fabs(4 * qa * qc));
        if (disc >= -err) {
            disc = fmax(0.0, disc);
            const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
            if (q == 0)
                add_knot(-qb / (2 * qa));
            else {
                add_knot(q / qa);
                add_knot(qc / q);
            }
        }
    }
    for (int i = 1; i < count; ++i)
        for (int j = i; j > 0 && knots[j - 1] > knots[j]; --j) {
            const double t = knots[j - 1];
            knots[j - 1] = knots[j];
            knots[j] = t;
        }
    for (int i = 1; i < count; ++i) {
        double lo = knots[i - 1], hi = knots[i];
        if (value(hi) > tol(hi)) continue;
        // Bisection ends when the midpoint equals an end; 1100 halvings cover any bracket in [0, 1].
        for (int it = 0; it < 1100; ++it) {
            const double mid = lo + (hi - lo) / 2;
            if (mid == lo || mid == hi) break;
            if (value(mid) > tol(mid))
                lo = mid;
            else
                hi = mid;
        }
        return 0.9 * lo;
    }
    return 1;
}

__global__ void __launch_bounds__(256) feasible_kernel(const DevMesh m, const double* __restrict__ u,
                                                       const double* __restrict__ du, double* block_min,
                                                       unsigned* status, double* per_elem,
                                                       const int* __restrict__ emesh, const int* __restrict__ mstate) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double alpha = 1.0;
    unsigned st = 0;
    // Batched solves: an element of a finished mesh (state 2) is skipped (step 1, no constraint).
    if (e < m.T && !(emesh != nullptr && mstate[emesh[e]] == 2)) {
        const int4 tv = __ldg(m.tets + e);
        const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
        double rec[12];
        load_rec<double>(m.rec64, e, rec);
        double Ds[9], dDs[9];
        bool ok = true, dok = true;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double a0 = u[3 * static_cast<size_t>(vs[0]) + i], ac = u[3 * static_cast<size_t>(vs[c + 1]) + i];
                const double b0 = du[3 * static_cast<size_t>(vs[0]) + i], bc = du[3 * static_cast<size_t>(vs[c + 1]) + i];
                ok = ok && isfinite(a0) && isfinite(ac);
                dok = dok && isfinite(b0) && isfinite(bc);
                Ds[3 * i + c] = ac - a0;
                dDs[3 * i + c] = bc - b0;
            }
        if (!ok || !dok) st |= ST_BAD_INPUT;
        const double lam = rec[10], mu = rec[11];
        if (!(isfinite(lam) && isfinite(mu) && lam >= 0 && mu > 0)) st |= ST_BAD_THETA;
        double F[9], dF[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                F[3 * i + j] = Ds[3 * i] * rec[j] + Ds[3 * i + 1] * rec[3 + j] + Ds[3 * i + 2] * rec[6 + j];
                dF[3 * i + j] = dDs[3 * i] * rec[j] + dDs[3 * i + 1] * rec[3 + j] + dDs[3 * i + 2] * rec[6 + j];
            }
        if (m.fpinv64) {
#pragma unroll
            for (int t = 0; t < 9; ++t) F[t] += m.fpinv64[9 * static_cast<size_t>(e) + t];
        } else {
            F[0] += 1;
            F[4] += 1;
            F[8] += 1;
        }
        bool fin = true;
#pragma unroll
        for (int t = 0; t < 9; ++t) fin = fin && isfinite(F[t]) && isfinite(dF[t]);
        if (!fin)
            st |= ST_NONFINITE_F;
        else if (st == 0)
            alpha = positive_det_step(F, dF, st);
        if (per_elem) per_elem[e] = alpha;
    }
    // Block minimum (order-independent, hence deterministic).
    __shared__ double s[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) alpha = fmin(alpha, __shfl_xor_sync(0xffffffffu, alpha, off));
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = alpha;
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = s[0];
        for (int w = 1; w < (blockDim.x >> 5); ++w) v = fmin(v, s[w]);
        block_min[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(1024) min_kernel(const double* __restrict__ x, int n, double* out) {
    __shared__ double s[32];
    double v = 1.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v = fmin(v, x[i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 1.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (threadIdx.x == 0) *out = v;
    }
}

// ---------------------------------------------------------------------------
// Force-response parameter VJP (detail/volumetric_fem_force_response.hpp:155-179 with
// NeoHookean::eval_d2W_dF_dtheta, neo_hookean.cpp:88-101): per element
//   d/dlambda = vol log J  sum_a w_a . (F^-T grad N_a)
//   d/dmu     = vol        sum_a w_a . ((F - F^-T) grad N_a)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) force_vjp_kernel(const DevMesh m, const double* __restrict__ u,
                                                        const double* __restrict__ w, double* out, unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const int4 tv = __ldg(m.tets + e);
        Kin<double> k;
        st |= kinematics<double>(m, e, tv, u, k);
        const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
        double sl = 0, sm = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double wi = w[3 * static_cast<size_t>(vs[b]) + i];
                double hf = 0, ff = 0;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    hf += k.FiT[3 * i + j] * k.n[b][j];
                    ff += k.F[3 * i + j] * k.n[b][j];
                }
                sl += wi * hf;
                sm += wi * (ff - hf);
            }
        }
        // With a plastic field the record's G and vol already carry Fp^-1 and det Fp.
        double dl = k.vol * k.logJ * sl, dm = k.vol * sm;
        if (!isfinite(dl) || !isfinite(dm)) st |= ST_NONFINITE_OUT;
        out[2 * static_cast<size_t>(e)] = dl;
        out[2 * static_cast<size_t>(e) + 1] = dm;
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// ---------------------------------------------------------------------------
// Plastic sensitivity of the elastic force (VolumetricFemForceFpResponse,
// volumetric_fem_force_fp_response.hpp:8-10, with NeoHookean::eval_d2W_dF_dFp,
// neo_hookean.cpp:103-128): per element the VJP out_c = w_dV <dP/dFp_c, grad w>, c = i + 3 j the
// column-major index of Fp. With Fe = F Fp^-1, sigma = dpsi/dFe = mu Fe + p Fe^-T, the record's
// rows n_a = grad N_a^T Fp^-1 (so H = grad w Fp^-1 = sum_a w_a n_a^T), Q = A : H (the
// neo-Hookean tangent: mu H + lambda (Fe^-T : H) Fe^-T - p Fe^-T H^T Fe^-T) and the record's
// vol = w_dV det Fp, the three terms of dP = tr(Fp^-1 dFp) P + det Fp (A : dFe) Fp^-T -
// P dFp^T Fp^-T (dFe = -Fe dFp Fp^-1) contract with grad w to
//   out_{i+3j} = vol [ (sigma : H) Fp^-1_{ji} - (Fe^T Q Fp^-T)_{ij} - (Fp^-1 sigma^T H)_{ji} ].
// 9 values per element; FP64.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) fp_vjp_kernel(const DevMesh m, const double* __restrict__ u,
                                                     const double* __restrict__ w, double* out, unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const int4 tv = __ldg(m.tets + e);
        Kin<double> k;
        st |= kinematics<double>(m, e, tv, u, k);
        const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
        double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; // row-major
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double wi = __ldg(w + 3 * static_cast<size_t>(vs[a]) + i);
#pragma unroll
                for (int j = 0; j < 3; ++j) H[3 * i + j] = fma(wi, k.n[a][j], H[3 * i + j]);
            }
        double Pi[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}; // Fp^-1, row-major
        if (m.fpinv64)
#pragma unroll
            for (int t = 0; t < 9; ++t) Pi[t] = __ldg(m.fpinv64 + 9 * static_cast<size_t>(e) + t);
        const double p = k.lam * k.logJ - k.mu;
        const double* Fe = k.F;
        const double* G = k.FiT;
        double sig[9], Q[9], fh = 0, sH = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            sig[t] = k.mu * Fe[t] + p * G[t];
            fh += G[t] * H[t];
            sH += sig[t] * H[t];
        }
        // Q = mu H + lambda (G : H) G - p G H^T G.
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double ghg = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) ghg += G[3 * i + a] * H[3 * b + a] * G[3 * b + j];
                Q[3 * i + j] = k.mu * H[3 * i + j] + k.lam * fh * G[3 * i + j] - p * ghg;
            }
        // A1 = Fe^T Q Fp^-T, A2 = Fp^-1 sigma^T H.
        double A1[9], A2[9], T1[9], T2[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double a = 0, b = 0;
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    a += Fe[3 * t + i] * Q[3 * t + j]; // (Fe^T Q)_ij
                    b += Pi[3 * i + t] * sig[3 * j + t]; // (Fp^-1 sigma^T)_ij
                }
                T1[3 * i + j] = a;
                T2[3 * i + j] = b;
            }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double a = 0, b = 0;
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    a += T1[3 * i + t] * Pi[3 * j + t]; // (Fe^T Q Fp^-T)_ij
                    b += T2[3 * i + t] * H[3 * t + j];  // (Fp^-1 sigma^T H)_ij
                }
                A1[3 * i + j] = a;
                A2[3 * i + j] = b;
            }
        double* o = out + 9 * static_cast<size_t>(e);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double v = k.vol * (sH * Pi[3 * j + i] - A1[3 * i + j] - A2[3 * j + i]);
                if (!isfinite(v)) st |= ST_NONFINITE_OUT;
                o[i + 3 * j] = v;
            }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Deterministic column sums of an (n x K) row-major array: fixed contiguous chunks per block,
// a fixed warp tree, then one thread sums the partials in order.
template <int K>
__global__ void __launch_bounds__(256) sum_cols_partial(const double* __restrict__ x, int n, double* partial) {
    __shared__ double s[K][8];
    double a[K];
#pragma unroll
    for (int c = 0; c < K; ++c) a[c] = 0;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per, hi = min(n, lo + per);
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x)
#pragma unroll
        for (int c = 0; c < K; ++c) a[c] += x[K * static_cast<size_t>(i) + c];
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a[c] += __shfl_xor_sync(0xffffffffu, a[c], off);
        if ((threadIdx.x & 31) == 0) s[c][threadIdx.x >> 5] = a[c];
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double t = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) t += s[threadIdx.x][w];
        partial[K * blockIdx.x + threadIdx.x] = t;
    }
}
template <int K> __global__ void sum_cols_final(const double* __restrict__ partial, int nb, double* out) {
    if (threadIdx.x < K) {
        double t = 0;
        for (int i = 0; i < nb; ++i) t += partial[K * i + threadIdx.x];
        out[threadIdx.x] = t;
    }
}

// Writes new geometry (G, vol: the first 10 values of each record) into both precisions'
// records, keeping each element's [lambda, mu].
__global__ void set_geometry_kernel(const DevMesh m, const double* __restrict__ geo) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
#pragma unroll
    for (int t = 0; t < 10; ++t) {
        const double v = geo[10 * static_cast<size_t>(e) + t];
        m.rec64[12 * static_cast<size_t>(e) + t] = v;
        m.rec32[12 * static_cast<size_t>(e) + t] = static_cast<float>(v);
    }
}

// Deterministic column sums of an (n x 2) array: partial sums per block, then one block.
__global__ void __launch_bounds__(256) sum_pairs_partial(const double* __restrict__ x, int n, double* partial) {
    __shared__ double s0[8], s1[8];
    double a = 0, b = 0;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per, hi = min(n, lo + per);
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        a += x[2 * static_cast<size_t>(i)];
        b += x[2 * static_cast<size_t>(i) + 1];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
        s0[threadIdx.x >> 5] = a;
        s1[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x0 = 0, x1 = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) {
            x0 += s0[w];
            x1 += s1[w];
        }
        partial[2 * blockIdx.x] = x0;
        partial[2 * blockIdx.x + 1] = x1;
    }
}
__global__ void sum_pairs_final(const double* __restrict__ partial, int nb, double* out) {
    if (threadIdx.x == 0) {
        double x0 = 0, x1 = 0;
        for (int i = 0; i < nb; ++i) {
            x0 += partial[2 * i];
            x1 += partial[2 * i + 1];
        }
        out[0] = x0;
        out[1] = x1;
    }
}

// ---------------------------------------------------------------------------
// Projected Hessian (HessianKind::Projected, mesh_energy.cpp:16-27): per element the 9x9
// matrix M with H_e = kron(q, I3) M kron(q, I3)^T,
//   M(3j'+i, 3l'+k) = vol [mu d_ik S_j'l' + lambda f_ij' f_kl' - p f_il' f_kj'],
//   Rq = q^T grad N (3x3), S = Rq Rq^T, f = F^-T Rq^T,
// is clamped to its non-negative eigenvalues: kept as is when an LDL^T test shows it
// positive definite, else by cyclic Jacobi (Golub & Van Loan, Alg. 8.5.3). The result is
// stored packed (45 values per element) for the assembly kernel.
// ---------------------------------------------------------------------------
// Index of the unordered vertex pair (a, b) of a tet among its 10.
__host__ __device__ constexpr int pair10(int a, int b) {
    return (a < b ? a : b) * 4 - ((a < b ? a : b) * ((a < b ? a : b) - 1)) / 2 + ((a < b ? b : a) - (a < b ? a : b));
}

// The element's ten 3x3 blocks H_ab (a <= b, pair10 order, row-major) from its 9x9 tangent M in
// the orthonormal basis q (packed upper triangle, index 3 j' + i):
//   H_ab(i, k) = sum_{j', l'} q_a(j') q_b(l') M(3 j' + i, 3 l' + k),
// as Y_a(i, c) = sum_j' q_a(j') M(3 j' + i, c), then H_ab(i, k) = sum_l' q_b(l') Y_a(i, 3 l' + k).
// MA is any array-like of 45 values (registers or shared memory); out receives 90 values.
template <typename R, typename MA> __device__ __forceinline__ void blocks_from_q(const MA& Mq, R* __restrict__ out) {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        R Y[3][9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                R y = 0;
#pragma unroll
                for (int jp = 0; jp < 3; ++jp) y = fma(qbasis<R>(a, jp), static_cast<R>(Mq[sym9(3 * jp + i, c)]), y);
                Y[i][c] = y;
            }
#pragma unroll
        for (int b = a; b < 4; ++b) {
            R* o = out + 9 * pair10(a, b);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    R h = 0;
#pragma unroll
                    for (int lp = 0; lp < 3; ++lp) h = fma(qbasis<R>(b, lp), Y[i][3 * lp + kk], h);
                    o[3 * i + kk] = h;
                }
        }
    }
}

constexpr int kProjThreads = 64;
constexpr int kProjStride = 127; // 45 (M) + 81 (V) + 1: odd stride, conflict-free 8-byte lanes


// Tangent sources of the projection pass: each forms the element's 9x9 tangent M in the q basis
// (packed upper triangle into A; V is 81 values of per-thread scratch) and returns status bits.
// NhTangent: the neo-Hookean closed form at displacement u.
struct NhTangent {
    const double* u;
};
__device__ __forceinline__ bool keeps_exact(const NhTangent&) { return false; }
// MatTangent: a material's d2W/dF2 per element (81 FP64 values, [3 i + j][3 k + l] =
// d2W / dF_ij dF_kl), M(3 j' + i, 3 l' + k) = vol sum_{j,l} Rq[j'][j] A[(i,j),(k,l)] Rq[l'][l],
// symmetrised as (M + M^T) / 2; with exact set the tangent is kept as it is (the Exact Hessian).
struct MatTangent {
    const double* A;
    bool exact;
};
__device__ __forceinline__ bool keeps_exact(const MatTangent& s) { return s.exact; }

template <typename R>
__device__ __forceinline__ void rq_basis(const R (&n)[4][3], R (&Rq)[3][3]) {
#pragma unroll
    for (int jp = 0; jp < 3; ++jp)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R s = 0;
#pragma unroll
            for (int a = 0; a < 4; ++a) s += qbasis<R>(a, jp) * n[a][j];
            Rq[jp][j] = s;
        }
}

template <typename R>
__device__ __forceinline__ unsigned form_tangent(const NhTangent& src, const DevMesh& m, int e, R* A, R* /*V*/) {
    const int4 tv = __ldg(m.tets + e);
    Kin<R> k;
    const unsigned st = kinematics<R>(m, e, tv, src.u, k);
    const R p = k.lam * k.logJ - k.mu;
    R Rq[3][3];
    rq_basis<R>(k.n, Rq);
    R S[3][3], f[3][3];
#pragma unroll
    for (int x = 0; x < 3; ++x)
#pragma unroll
        for (int y = 0; y < 3; ++y) {
            S[x][y] = Rq[x][0] * Rq[y][0] + Rq[x][1] * Rq[y][1] + Rq[x][2] * Rq[y][2];
            f[x][y] = k.FiT[3 * x] * Rq[y][0] + k.FiT[3 * x + 1] * Rq[y][1] + k.FiT[3 * x + 2] * Rq[y][2];
        }
#pragma unroll
    for (int jp = 0; jp < 3; ++jp)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int lp = 0; lp < 3; ++lp)
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    const int r = 3 * jp + i, c = 3 * lp + kk;
                    if (r > c) continue;
                    R v = k.lam * f[i][jp] * f[kk][lp] - p * f[i][lp] * f[kk][jp];
                    if (i == kk) v += k.mu * S[jp][lp];
                    A[sym9(r, c)] = k.vol * v;
                }
    return st;
}

template <typename R>
__device__ __forceinline__ unsigned form_tangent(const MatTangent& src, const DevMesh& m, int e, R* A, R* V) {
    R rec[12];
    load_rec<R>(rec_ptr<R>(m), e, rec);
    R n[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < 3; ++j) n[c + 1][j] = rec[3 * c + j];
#pragma unroll
    for (int j = 0; j < 3; ++j) n[0][j] = -(n[1][j] + n[2][j] + n[3][j]);
    R Rq[3][3];
    rq_basis<R>(n, Rq);
    const R vol = rec[9];
    const double* Ae = src.A + 81 * static_cast<size_t>(e);
    unsigned st = 0;
    // Full M into V (row r = 3 j' + i, column c = 3 l' + k), then the symmetrised upper triangle.
    for (int i = 0; i < 3; ++i)
        for (int kk = 0; kk < 3; ++kk) {
            R T[3][3]; // T[j][l'] = sum_l A[(i,j),(kk,l)] Rq[l'][l]
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                R a3[3];
#pragma unroll
                for (int l = 0; l < 3; ++l) a3[l] = static_cast<R>(__ldg(Ae + (3 * i + j) * 9 + 3 * kk + l));
#pragma unroll
                for (int lp = 0; lp < 3; ++lp) T[j][lp] = a3[0] * Rq[lp][0] + a3[1] * Rq[lp][1] + a3[2] * Rq[lp][2];
            }
#pragma unroll
            for (int jp = 0; jp < 3; ++jp)
#pragma unroll
                for (int lp = 0; lp < 3; ++lp)
                    V[9 * (3 * jp + i) + 3 * lp + kk] =
                        vol * (Rq[jp][0] * T[0][lp] + Rq[jp][1] * T[1][lp] + Rq[jp][2] * T[2][lp]);
        }
    for (int r = 0; r < 9; ++r)
        for (int c = r; c < 9; ++c) {
            const R v = R(0.5) * (V[9 * r + c] + V[9 * c + r]);
            if (!(v == v) || v == R(INFINITY) || v == R(-INFINITY)) st |= ST_NONFINITE_F;
            A[sym9(r, c)] = v;
        }
    return st;
}

template <typename R, class Src>
__global__ void __launch_bounds__(kProjThreads) project_kernel(const DevMesh m, const Src src,
                                                               R* __restrict__ proj, unsigned* status,
                                                               const int* __restrict__ emesh,
                                                               const int* __restrict__ mesh_exact, int* list,
                                                               unsigned* count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* A = reinterpret_cast<R*>(smem_raw) + kProjStride * threadIdx.x;
    R* V = A + 45;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    // Per-mesh state of a batched solve: 0 projected, 1 exact, 2 finished (the element is skipped).
    const int state = (e < m.T && emesh != nullptr) ? mesh_exact[emesh[e]] : 0;
    if (e < m.T && state != 2) {
        st |= form_tangent<R>(src, m, e, A, V);
        // Elements of a mesh marked exact keep their tangent unclamped (the Exact Hessian).
        const bool keep = keeps_exact(src) || state == 1;
        // Positive semi-definiteness test: LDL^T with diagonal pivoting on a copy in the V area
        // (row-major 9x9). Pivots above tol are eliminated; once none is left, M is semi-definite
        // if the remaining Schur complement is below tol everywhere (tol = 64 eps max|diag M|:
        // round-off of a singular semi-definite M, e.g. the rotation modes near rest). Such an M is
        // its own clamp up to that round-off; any other goes to clamp_kernel.
        bool pd = true;
        if (!keep) {
            R scale = 0;
            for (int r = 0; r < 9; ++r) {
                scale = fmax(scale, fabs(A[sym9(r, r)]));
                for (int c = 0; c < 9; ++c) V[9 * r + c] = A[sym9(r, c)];
            }
            pd = semidefinite_ldlt<9>(V, R(64) * Eps<R>::v * scale);
            if (!(scale < R(INFINITY))) pd = false;
        }
        // Semi-definite (or kept exact): final. Otherwise the unclamped tangent is stored and
        // the element is listed for clamp_kernel, which runs the eigenvalue clamp on the listed
        // elements only (a warp of pass 1 then never waits on another lane's Jacobi sweeps).
        R* out = proj + kProjRecord * static_cast<size_t>(e);
        if (pd || keep) {
            blocks_from_q<R>(A, out);
        } else {
            for (int t = 0; t < 45; ++t) out[t] = A[t]; // the clamp reads M here and writes the blocks
            list[atomicAdd(count, 1u)] = e;
        }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Eigenvalue clamp of the listed elements' 9x9 tangents (parallel-ordered cyclic Jacobi):
// M = V max(Lambda, 0) V^T, in place; grid-stride over the list whose length pass 1 counted.
// One thread per element with the packed matrix and the rotations in registers; in FP64 the
// eigenvectors V live in shared memory (81 doubles per thread, an odd stride: conflict-free),
// since A and V together would exceed the register file.
template <typename R, bool VREG, typename VA>
__device__ __forceinline__ void clamp9(R* __restrict__ out, VA& V) {
    R A[45];
#pragma unroll
    for (int t = 0; t < 45; ++t) A[t] = out[t];
    clamp9_packed<R, VREG>(A, V);
    blocks_from_q<R>(A, out); // the clamped M's ten blocks replace M in the element's record
}

constexpr int kClampVStride = 81;
// Resident 64-thread blocks per SM the FP32 clamp's register allocation must allow (6: at most
// 170 registers, a few of them spilled; A, V and the relabelling copy need about 187).
#ifndef LPG_CLAMP_MIN_BLOCKS_F32
#define LPG_CLAMP_MIN_BLOCKS_F32 6
#endif

// Register-budget variants of the clamp (autotuner): FP32 at LPG_CLAMP_MIN_BLOCKS_F32 resident
// blocks or unconstrained (about 187 registers, no spill); FP64 has one.
template <typename R> constexpr int clamp_minb(int v) {
    return sizeof(R) == 8 ? 1 : (v == 0 ? LPG_CLAMP_MIN_BLOCKS_F32 : 1);
}

template <typename R, int MINB>
__global__ void __launch_bounds__(kProjThreads, MINB) clamp_kernel(R* __restrict__ proj, const int* __restrict__ list,
                                                                   const unsigned* __restrict__ count) {
    const unsigned n = *count;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        R* out = proj + kProjRecord * static_cast<size_t>(list[i]);
        if constexpr (sizeof(R) == 8) {
            extern __shared__ __align__(16) unsigned char smem_raw[];
            // volatile: every access goes to shared memory (cached copies would need the
            // registers this layout is there to save).
            volatile R* V = reinterpret_cast<R*>(smem_raw) + kClampVStride * threadIdx.x;
            clamp9<R, false>(out, V);
        } else {
            R V[81];
            clamp9<R, true>(out, V);
        }
    }
}

// Seeded symmetric test matrices for timing the clamp: entry values in [-1, 1) from an integer
// hash (SplitMix64 finaliser) of the element and entry index; list[i] = i.
template <typename R> __global__ void clamp_sample_kernel(R* __restrict__ proj, int* __restrict__ list, int n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    list[e] = e;
    for (int t = 0; t < 45; ++t) {
        unsigned long long z = 45ull * static_cast<unsigned long long>(e) + t + 0x9e3779b97f4a7c15ull;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        proj[kProjRecord * static_cast<size_t>(e) + t] = static_cast<R>(static_cast<double>(z >> 11) * 0x1.0p-52 - 1.0);
    }
}

// Resident-grid facts of one kernel at one dynamic shared-memory size, cached per device: the
// shared-memory opt-in (cudaFuncAttributeMaxDynamicSharedMemorySize) is a per-device attribute
// and the occupancy can differ between devices, so a host thread that drives handles on several
// GPUs sets the attribute and sizes the grid on each of them.
constexpr int kMaxDevices = 64;
struct LaunchCache {
    size_t smem[kMaxDevices];
    int resident[kMaxDevices];
    LaunchCache() {
        for (int d = 0; d < kMaxDevices; ++d) {
            smem[d] = ~size_t(0);
            resident[d] = 0;
        }
    }
};
// Blocks of `kernel` (threads per block, dynamic shared memory smem) that fit on all SMs of the
// current device at once; sets the kernel's shared-memory opt-in there first when smem > 0.
template <typename Kern> int resident_grid(Kern kernel, int threads, size_t smem, LaunchCache& c) {
    int dev = 0;
    LPG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(LPG_EINVAL, "device index out of range");
    if (c.smem[dev] != smem) {
        int sms = 0, per_sm = 0, optin = 0;
        LPG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        if (smem > static_cast<size_t>(optin)) fail(LPG_EINVAL, "mesh cluster needs more shared memory than the GPU has");
        if (smem > 0)
            LPG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        LPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        LPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
        c.resident[dev] = std::max(1, sms * std::max(per_sm, 1));
        c.smem[dev] = smem;
    }
    return c.resident[dev];
}

// ---------------------------------------------------------------------------
// Block slots of the cluster plan (HostPlan::cl_*), used by the block gather below.
// ---------------------------------------------------------------------------
#ifndef LPG_CLUSTER_THREADS
#define LPG_CLUSTER_THREADS 128
#endif
constexpr int kClThreads = LPG_CLUSTER_THREADS;

// Fixed shared memory of the block gather: element ids and a 4-column row table.
constexpr size_t block_gather_fixed() {
    return (static_cast<size_t>(kClusterElems) + 4 * kClusterRows) * sizeof(int);
}

// Position of entry t of block q of a row (first block slot0, nb blocks, solver base sb) in the
// output layout.
__device__ __forceinline__ size_t cl_pos(int layout, int slot0, int nb, int sb, int q, int t) {
    if (layout == LPG_LAYOUT_BSR) return 9 * static_cast<size_t>(slot0 + q) + t;
    if (layout == LPG_LAYOUT_CSC) {
        const int i = t / 3, c = t - 3 * (t / 3);
        return 9 * static_cast<size_t>(slot0) + static_cast<size_t>(i) * 3 * nb + 3 * q + c;
    }
    return static_cast<size_t>(static_cast<int64_t>(sb) + 32 * static_cast<int64_t>(9 * q + t));
}


// ---------------------------------------------------------------------------
// Tet assembly over the tet clusters (E, gradient and Exact Hessian in the BSR, CSC or solver
// layout). One thread block per cluster (persistent over clusters), four passes:
//   stage:   each thread loads one element's record into registers and copies one vertex's
//            displacement into shared memory; the cluster's item table and contributor lists
//            are copied into shared memory with cp.async, and the owned rows' offsets are
//            loaded into registers;
//   element: one thread per element evaluates it once (kinematics as the reference computes
//            it) and keeps h_a = F^-T grad N_a, vol mu grad N_a . grad N_b, vol lambda, vol p
//            and the gradient pieces g_a = vol P grad N_a in shared memory;
//   items:   one thread per diagonal block (with the row's gradient) or edge block sums the
//            block's contributors in ascending element order into registers and writes it into
//            the cluster's output staging (an edge between two owned rows once, at both
//            positions);
//   copy:    one warp per owned row copies the row's staged values to the output: the row's
//            9 nb values are contiguous in the BSR and CSC layouts, so the stores are
//            coalesced.
// The passes are software-pipelined across the block's clusters so that no global read waits
// inside a pass: the next cluster's bounds are read a cluster ahead, its element, vertex and row
// indices during this cluster's item pass, and its stage is issued before this cluster's copy
// pass (whose stores do not wait), so its loads arrive while the copy pass runs.
// ---------------------------------------------------------------------------
constexpr int kTcThreads = 256;
static_assert(kTcThreads >= kTcElems && kTcThreads >= kTcVerts && kTcThreads >= kTcRows,
              "one element, one vertex and one row per thread in the stage");
static_assert(((2 * kTcRows + 31) & ~31) < kTcThreads, "the diagonal lane pairs leave lanes for the edge items");
// Lanes per diagonal item of a cluster with nd owned rows: 4 while they leave at least one warp
// for the edge items, else 2. Part k of the item's S lanes sums contributors
// [ceil(cnt k / S), ceil(cnt (k + 1) / S)); the parts are added as (p0 + p1) + (p2 + p3).
__host__ __device__ constexpr int tc_diag_split(int nd) { return 4 * nd + 32 <= kTcThreads ? 4 : 2; }
// Per-element data in shared memory, one component per kTcElems-long array: h_a (3 a + i),
// vol mu grad N_a . grad N_b (pair order), vol lambda, vol p, g_a (3 a + i).
constexpr int kTcH = 0, kTcCC = 12, kTcL = 22, kTcP = 23, kTcG = 24, kTcComp = 36;
// Owned-row words in shared memory: vertex, staging offset, first block, nb | diagonal block
// index << 8 (solver layout), solver base. A thread holds them one cluster ahead as the words
// loaded (vertex, staging offset, first block, end block, solver base, diagonal slot), so that
// nothing waits on those loads before the next cluster's stage completes.
constexpr int kTcRowInts = 5, kTcRowRaw = 6;
// Launch variants of the Exact-Hessian kernel (autotuner): the resident blocks per SM the
// register allocation must allow, and the unroll depth of the contributor loops. The arithmetic
// and its order are the same, so every variant's results are bitwise identical.
template <typename R> constexpr int tc_minb(int v) { return (sizeof(R) == 8 ? 2 : 3) - (v == 2 ? 1 : 0); }
constexpr int tc_unroll(int v) { return v == 0 ? 1 : 4; }
template <typename R> constexpr size_t tc_ed_bytes() {
    return static_cast<size_t>(kTcComp) * kTcElems * sizeof(R);
}
static_assert(3 * kTcVerts * sizeof(double) <= tc_ed_bytes<float>(), "staged displacements fit the element data");
// Shared memory: reduction scratch (32 doubles), the element data (whose first 3 kTcVerts
// doubles hold the staged displacements until the element pass has read them), the output
// staging, the item table, the contributor lists and two buffers of owned-row words.
template <typename R> constexpr size_t tc_smem_bytes() {
    return 32 * sizeof(double) + tc_ed_bytes<R>() + static_cast<size_t>(kTcVals) * sizeof(R) +
           static_cast<size_t>(kTcItems) * sizeof(uint4) + static_cast<size_t>(kTcEnts) * sizeof(uint16_t) +
           2 * static_cast<size_t>(kTcRows) * kTcRowInts * sizeof(int);
}

// One contributor of an edge block: acc(i, q) = B_q hb_i + (A_i hb_q + acc(i, q)) (A = vol lambda
// h_a, B = -vol p h_a), then + mg on the diagonal entries. In FP32 the nine chains run as packed
// pairs (sm_100 f32x2 FMA); each lane of a pair is rounded as the scalar FMA, so the results are
// bitwise those of the scalar form.
template <typename R>
__device__ __forceinline__ void edge_contrib(R (&acc)[9], const R (&A)[3], const R (&B)[3], const R (&hb)[3], R mg) {
    using X = M<R>;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            acc[3 * i + q] = X::fma(B[q], hb[i], X::fma(A[i], hb[q], acc[3 * i + q]));
            if (i == q) acc[3 * i + q] = X::add(acc[3 * i + q], mg);
        }
}
template <>
__device__ __forceinline__ void edge_contrib<float>(float (&acc)[9], const float (&A)[3], const float (&B)[3],
                                                    const float (&hb)[3], float mg) {
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
        const int i0 = u / 3, q0 = u % 3, i1 = (u + 1) / 3, q1 = (u + 1) % 3;
        float2 t = __ffma2_rn(make_float2(A[i0], A[i1]), make_float2(hb[q0], hb[q1]), make_float2(acc[u], acc[u + 1]));
        t = __ffma2_rn(make_float2(B[q0], B[q1]), make_float2(hb[i0], hb[i1]), t);
        acc[u] = t.x;
        acc[u + 1] = t.y;
    }
    acc[8] = __fmaf_rn(B[2], hb[2], __fmaf_rn(A[2], hb[2], acc[8]));
    acc[0] = __fadd_rn(acc[0], mg);
    acc[4] = __fadd_rn(acc[4], mg);
    acc[8] = __fadd_rn(acc[8], mg);
}

// One contributor of a diagonal block (its upper triangle, 6 sums): acc(i, q) += dv (hh_i hh_q),
// then + mg on the diagonal; FP32 in packed pairs, bitwise as the scalar form.
template <typename R> __device__ __forceinline__ void diag_contrib(R (&acc)[6], const R (&hh)[3], R dv, R mg) {
    using X = M<R>;
    int uix = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int q = i; q < 3; ++q, ++uix) {
            acc[uix] = X::fma(dv, X::mul(hh[i], hh[q]), acc[uix]);
            if (i == q) acc[uix] = X::add(acc[uix], mg);
        }
}
template <>
__device__ __forceinline__ void diag_contrib<float>(float (&acc)[6], const float (&hh)[3], float dv, float mg) {
    // Upper-triangle order: (0,0) (0,1) (0,2) (1,1) (1,2) (2,2).
    const float2 p01 = __fmul2_rn(make_float2(hh[0], hh[0]), make_float2(hh[0], hh[1]));
    const float2 p23 = __fmul2_rn(make_float2(hh[0], hh[1]), make_float2(hh[2], hh[1]));
    const float2 p45 = __fmul2_rn(make_float2(hh[1], hh[2]), make_float2(hh[2], hh[2]));
    const float2 dd = make_float2(dv, dv);
    const float2 a01 = __ffma2_rn(dd, p01, make_float2(acc[0], acc[1]));
    const float2 a23 = __ffma2_rn(dd, p23, make_float2(acc[2], acc[3]));
    const float2 a45 = __ffma2_rn(dd, p45, make_float2(acc[4], acc[5]));
    acc[0] = __fadd_rn(a01.x, mg);
    acc[1] = a01.y;
    acc[2] = a23.x;
    acc[3] = __fadd_rn(a23.y, mg);
    acc[4] = a45.x;
    acc[5] = __fadd_rn(a45.y, mg);
}

// The element pass's outputs for element el: g_a = vol P grad N_a (with the gradient), and
// h_a = F^-T grad N_a, vol lambda, vol p, vol mu grad N_a . grad N_b (with the Hessian), into the
// component-major shared arrays. In FP32 pairs of outputs are formed with packed f32x2 operations,
// each lane rounded as the scalar operation, so the values are bitwise those of the scalar form.
template <typename R, bool WG, bool WH>
__device__ __forceinline__ void tc_element_data(const Kin<R>& k, R p, R* ed, int el) {
    using X = M<R>;
    constexpr int E = kTcElems;
    if constexpr (sizeof(R) == 4) {
        if (WG) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                R P[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) P[j] = X::fma(k.mu, k.F[3 * i + j], X::mul(p, k.FiT[3 * i + j]));
#pragma unroll
                for (int b0 = 0; b0 < 4; b0 += 2) {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        t = __ffma2_rn(make_float2(P[j], P[j]), make_float2(k.n[b0][j], k.n[b0 + 1][j]), t);
                    t = __fmul2_rn(make_float2(k.vol, k.vol), t);
                    ed[(kTcG + 3 * b0 + i) * E + el] = t.x;
                    ed[(kTcG + 3 * (b0 + 1) + i) * E + el] = t.y;
                }
            }
        }
        if (WH) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int b0 = 0; b0 < 4; b0 += 2) {
                    float2 t = __fmul2_rn(make_float2(k.FiT[3 * i], k.FiT[3 * i]), make_float2(k.n[b0][0], k.n[b0 + 1][0]));
                    t = __ffma2_rn(make_float2(k.FiT[3 * i + 1], k.FiT[3 * i + 1]), make_float2(k.n[b0][1], k.n[b0 + 1][1]), t);
                    t = __ffma2_rn(make_float2(k.FiT[3 * i + 2], k.FiT[3 * i + 2]), make_float2(k.n[b0][2], k.n[b0 + 1][2]), t);
                    ed[(kTcH + 3 * b0 + i) * E + el] = t.x;
                    ed[(kTcH + 3 * (b0 + 1) + i) * E + el] = t.y;
                }
            ed[kTcL * E + el] = X::mul(k.vol, k.lam);
            ed[kTcP * E + el] = X::mul(k.vol, p);
            const R mv = X::mul(k.vol, k.mu);
            constexpr int px[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, py[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
#pragma unroll
            for (int c = 0; c < 10; c += 2) {
                const int x1 = px[c], y1 = py[c], x2 = px[c + 1], y2 = py[c + 1];
                float2 t = __fmul2_rn(make_float2(k.n[x1][0], k.n[x2][0]), make_float2(k.n[y1][0], k.n[y2][0]));
                t = __ffma2_rn(make_float2(k.n[x1][1], k.n[x2][1]), make_float2(k.n[y1][1], k.n[y2][1]), t);
                t = __ffma2_rn(make_float2(k.n[x1][2], k.n[x2][2]), make_float2(k.n[y1][2], k.n[y2][2]), t);
                t = __fmul2_rn(make_float2(mv, mv), t);
                ed[(kTcCC + pair10(x1, y1)) * E + el] = t.x;
                ed[(kTcCC + pair10(x2, y2)) * E + el] = t.y;
            }
        }
    } else {
        if (WG) {
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    R sum = 0;
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        sum = X::fma(X::fma(k.mu, k.F[3 * i + j], X::mul(p, k.FiT[3 * i + j])), k.n[bb][j], sum);
                    ed[(kTcG + 3 * bb + i) * E + el] = k.vol * sum;
                }
        }
        if (WH) {
#pragma unroll
            for (int bb = 0; bb < 4; ++bb)
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    ed[(kTcH + 3 * bb + i) * E + el] = X::fma(
                        k.FiT[3 * i + 2], k.n[bb][2], X::fma(k.FiT[3 * i + 1], k.n[bb][1], X::mul(k.FiT[3 * i], k.n[bb][0])));
            ed[kTcL * E + el] = X::mul(k.vol, k.lam);
            ed[kTcP * E + el] = X::mul(k.vol, p);
            const R mv = X::mul(k.vol, k.mu);
#pragma unroll
            for (int xx = 0; xx < 4; ++xx)
#pragma unroll
                for (int y = xx; y < 4; ++y)
                    ed[(kTcCC + pair10(xx, y)) * E + el] = X::mul(
                        mv, X::fma(k.n[xx][2], k.n[y][2], X::fma(k.n[xx][1], k.n[y][1], X::mul(k.n[xx][0], k.n[y][0]))));
        }
    }
}

// Staging index of entry (i, c) of the block at packed position pos (row offset so, block q,
// row length nb): BSR and solver layouts keep blocks row-major one after the other, CSC keeps
// the row's three scalar rows one after the other.
__device__ __forceinline__ int tc_stage(uint32_t pos, bool csc, int i, int c) {
    const int so = static_cast<int>(pos & 0xffffu), q = static_cast<int>((pos >> 16) & 0xffu),
              nb = static_cast<int>(pos >> 24);
    return csc ? so + 3 * nb * i + 3 * q + c : so + 9 * q + 3 * i + c;
}

// Asynchronous global -> shared copies (cp.async; the source is device memory).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Bounds of a tet cluster in the plan's arrays (all zero past the last cluster), field q of
// TcBounds in the order declared.
struct TcBounds {
    int e0 = 0, ne = 0, v0 = 0, nv = 0, i0 = 0, ni = 0, nd = 0, n0 = 0, nn = 0, r0 = 0, nr = 0;
};
constexpr int kTcFields = 12; // the bounds, then the cluster's skip flag (batched solves)
// Field q of cluster cl as the words it is made of: {first, end} of a count field (the count is
// end - first), {value, 0} otherwise. The lanes reading the fields of one cluster take no
// divergent path (the array is selected, the second word's load predicated), and nothing here
// waits on the loads: the count is formed by tc_field_value where the field is used.
__device__ __forceinline__ bool tc_count_field(int q) { return q == 1 || q == 3 || q == 5 || q == 8 || q == 10; }
__device__ __forceinline__ int2 tc_field_words(const DevMesh& m, const unsigned char* skip, int cl, int q) {
    int2 w = make_int2(0, 0);
    if (cl >= m.tc_ncl) return w;
    const int32_t* ptr = q < 2 ? m.tc_el_ptr
                       : q < 4 ? m.tc_vert_ptr
                       : q < 6 ? m.tc_item_ptr
                       : q == 6 ? m.tc_ndiag
                       : q < 9 ? m.tc_ent_ptr
                       : m.tc_row_ptr;
    if (q < 11) w.x = __ldg(ptr + cl);
    if (tc_count_field(q)) w.y = __ldg(ptr + cl + 1);
    if (q == 11 && skip != nullptr) w.x = __ldg(skip + cl) != 0;
    return w;
}
__device__ __forceinline__ int tc_field_value(int2 w, int q) { return tc_count_field(q) ? w.y - w.x : w.x; }
__device__ __forceinline__ int tc_field(const DevMesh& m, const unsigned char* skip, int cl, int q) {
    return tc_field_value(tc_field_words(m, skip, cl, q), q);
}
// A skipped cluster has empty bounds: nothing is staged, evaluated or written.
__device__ __forceinline__ TcBounds tc_bounds(const int* f) {
    TcBounds b;
    if (f[11]) return b;
    b.e0 = f[0], b.ne = f[1], b.v0 = f[2], b.nv = f[3], b.i0 = f[4], b.ni = f[5];
    b.nd = f[6], b.n0 = f[7], b.nn = f[8], b.r0 = f[9], b.nr = f[10];
    return b;
}

// Thread t's indices of a cluster: element t (word and local vertices), vertex t, owned row t.
struct TcIdx {
    uint32_t ew = 0, loc = 0;
    int vert = 0, row = 0, so = 0;
};
__device__ __forceinline__ void tc_load_idx(const DevMesh& m, const TcBounds& b, int t, TcIdx& x) {
    if (t < b.ne) {
        x.ew = __ldg(m.tc_els + b.e0 + t);
        x.loc = __ldg(m.tc_loc + b.e0 + t);
    }
    if (t < b.nv) x.vert = __ldg(m.tc_verts + b.v0 + t);
    if (t < b.nr) {
        x.row = __ldg(m.tc_rows + b.r0 + t);
        x.so = __ldg(m.tc_row_so + b.r0 + t);
    }
}

// Issues thread t's part of a cluster's stage: its element's record into registers, its
// vertex's displacement and its share of the item table and contributor lists into shared memory
// (cp.async, one group), and its owned row's words into registers.
template <typename R, bool ITEMS>
__device__ __forceinline__ void tc_issue(const DevMesh& m, const double* __restrict__ u, const TcBounds& b,
                                         const TcIdx& x, int t, bool sell, double* su, uint4* sitems, uint16_t* sents,
                                         R (&r12)[12], int (&rowv)[kTcRowRaw]) {
    // Without items (energy only) an element the cluster does not own contributes nothing.
    if (t < b.ne && (ITEMS || (x.ew >> 31))) load_rec<R>(rec_ptr<R>(m), static_cast<int>(x.ew & 0x7fffffffu), r12);
    if (t < b.nv) {
#pragma unroll
        for (int i = 0; i < 3; ++i) cp_async8(su + 3 * t + i, u + 3 * static_cast<size_t>(x.vert) + i);
    }
    if (ITEMS) {
        for (int k = t; k < b.ni; k += kTcThreads) cp_async16(sitems + k, m.tc_items + b.i0 + k);
        for (int k = t; k < (b.nn >> 3); k += kTcThreads) cp_async16(sents + 8 * k, m.tc_ents + b.n0 + 8 * k);
    }
    cp_async_commit();
    if (ITEMS && t < b.nr) {
        rowv[0] = x.row;
        rowv[1] = x.so;
        rowv[2] = __ldg(m.row_ptr + x.row);
        rowv[3] = __ldg(m.row_ptr + x.row + 1);
        rowv[4] = 0;
        rowv[5] = 0;
        if (sell) {
            rowv[4] = __ldg(m.sell_base + x.row);
            rowv[5] = __ldg(m.diag_slot + x.row);
        }
    }
}

template <typename R, bool WG, bool WH, int MINB, int UNR>
__global__ void __launch_bounds__(kTcThreads, MINB) tet_cluster_kernel(const DevMesh m, const EvalArgs a) {
    using X = M<R>;
    using HT = typename HOut<R>::T;
    constexpr int E = kTcElems;
    constexpr bool ITEMS = WG || WH;
    constexpr int nw = kTcThreads / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* red = reinterpret_cast<double*>(smem_raw);
    R* ed = reinterpret_cast<R*>(smem_raw + 32 * sizeof(double));
    double* su = reinterpret_cast<double*>(ed); // [nv][3], until the element pass has read it
    R* stage = ed + kTcComp * E;
    uint4* sitems = reinterpret_cast<uint4*>(stage + kTcVals);
    uint16_t* sents = reinterpret_cast<uint16_t*>(sitems + kTcItems);
    int* srow = reinterpret_cast<int*>(sents + kTcEnts);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    HT* hout = reinterpret_cast<HT*>(a.hess);
    const bool csc = a.layout == LPG_LAYOUT_CSC, sell = a.layout == kLayoutSell;
    __shared__ int s_hdr[2][kTcFields]; // bounds of the next cluster, by iteration parity
    unsigned st = 0;
    int cl = blockIdx.x;
    const int grid = static_cast<int>(gridDim.x);
    // Prologue: the first cluster's stage; threads 0 .. kTcFields - 1 hold one field each of the
    // bounds one cluster ahead.
    TcBounds b;
    {
        int f[kTcFields];
#pragma unroll
        for (int q = 0; q < kTcFields; ++q) f[q] = tc_field(m, a.tc_skip, cl, q);
        b = tc_bounds(f);
    }
    TcIdx x;
    tc_load_idx(m, b, tid, x);
    R r12[12];
    int rowv[kTcRowRaw] = {0, 0, 0, 0, 0, 0};
    tc_issue<R, ITEMS>(m, a.u, b, x, tid, sell, su, sitems, sents, r12, rowv);
    int2 ahead = tid < kTcFields ? tc_field_words(m, a.tc_skip, cl + grid, tid) : make_int2(0, 0);
    int ne = b.ne, ni = WH ? b.ni : b.nd, nr = b.nr, ndc = b.nd;
    for (int buf = 0; cl < m.tc_ncl; cl += grid, buf ^= 1) {
        int* rows = srow + buf * kTcRows * kTcRowInts;
        if (ITEMS && tid < nr) {
#pragma unroll
            for (int q = 0; q < 3; ++q) rows[kTcRowInts * tid + q] = rowv[q];
            rows[kTcRowInts * tid + 3] = (rowv[3] - rowv[2]) | (sell ? (rowv[5] - rowv[2]) << 8 : 0);
            rows[kTcRowInts * tid + 4] = rowv[4];
        }
        if (tid < kTcFields) s_hdr[buf][tid] = tc_field_value(ahead, tid);
        cp_async_wait_all();
        __syncthreads(); // the cluster's stage is complete
        // Element pass: every element of the cluster once, one per thread.
        const uint32_t ew = x.ew;
        R Ds[3][3];
        bool in_ok = true;
        if (tid < ne && (ITEMS || (ew >> 31))) {
            double uu[4][3];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int lv = static_cast<int>((x.loc >> (8 * c)) & 0xffu);
#pragma unroll
                for (int i = 0; i < 3; ++i) uu[c][i] = su[3 * lv + i];
            }
            in_ok = edge_differences<R>(uu, Ds);
        }
        __syncthreads(); // the displacements are read; their memory holds element data from here
        double eacc = 0;
        if (tid < ne && (ITEMS || (ew >> 31))) {
            const int el = tid;
            const int e = static_cast<int>(ew & 0x7fffffffu);
            Kin<R> k;
            st |= kinematics_ds<R>(m, e, r12, Ds, in_ok, k);
            if (ew >> 31) {
                const R Ee = k.vol * k.psi;
                eacc += static_cast<double>(Ee);
                if (a.elem_energy) a.elem_energy[e] = static_cast<double>(Ee);
            }
            const R p = X::fma(k.lam, k.logJ, -k.mu);
            tc_element_data<R, WG, WH>(k, p, ed, el);
        }
        // Energy of the cluster's own elements: fixed thread order, fixed tree.
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) eacc += __shfl_xor_sync(0xffffffffu, eacc, off);
        if (lane == 0) red[warp] = eacc;
        __syncthreads(); // element data complete
        if (tid == 0) {
            double t = 0;
            for (int w = 0; w < nw; ++w) t += red[w];
            a.cluster_energy[cl] = t;
            if (!isfinite(t)) st |= ST_NONFINITE_OUT;
        }
        // The next cluster's indices, and the bounds of the one after, arrive while the item pass
        // runs.
        tc_load_idx(m, tc_bounds(s_hdr[buf]), tid, x);
        if (tid < kTcFields) ahead = tc_field_words(m, a.tc_skip, cl + 2 * grid, tid);
        if (ITEMS) {
            // Item pass. The nd diagonal items (the first nd) are summed by groups of S lanes
            // (tc_diag_split), each lane over a contiguous part of the contributor list in
            // ascending order, the parts added by shuffles; they fill whole warps (S nd lanes
            // rounded up to 32), and the edge items follow on the remaining lanes, so no warp runs
            // both kinds and the diagonal sums (the longest lists) take about as long as an edge
            // block.
            const int nd = ndc, sd = tc_diag_split(nd), lsd = sd == 4 ? 2 : 1, dl = sd * nd, dpad = (dl + 31) & ~31;
            if (tid < dpad) {
                // Diagonal block (symmetric: 6 sums, mirrored) and the row's gradient:
                //   H_aa = (vol lambda - vol p) h_a h_a^T + vol mu |grad N_a|^2 I.
                const bool active = tid < dl;
                const int part = tid & (sd - 1);
                uint4 it = make_uint4(0u, 0u, 0u, 0u);
                R acc[6] = {0, 0, 0, 0, 0, 0}, gs[3] = {0, 0, 0};
                if (active) {
                    it = sitems[tid >> lsd];
                    const uint16_t* en = sents + (it.z & 0xfffffu);
                    const int cnt = static_cast<int>(it.z >> 20);
                    const int c0 = (cnt * part + sd - 1) >> lsd, c1 = (cnt * (part + 1) + sd - 1) >> lsd;
#pragma unroll UNR
                    for (int c = c0; c < c1; ++c) {
                        const int w = en[c];
                        const int el = w >> 8, pr = (w >> 4) & 15, la = (w >> 2) & 3;
                        if (WG) {
#pragma unroll
                            for (int i = 0; i < 3; ++i) gs[i] = X::add(gs[i], ed[(kTcG + 3 * la + i) * E + el]);
                        }
                        if (WH) {
                            const R hh[3] = {ed[(kTcH + 3 * la) * E + el], ed[(kTcH + 3 * la + 1) * E + el],
                                             ed[(kTcH + 3 * la + 2) * E + el]};
                            const R dv = X::add(ed[kTcL * E + el], -ed[kTcP * E + el]), mg = ed[(kTcCC + pr) * E + el];
                            diag_contrib<R>(acc, hh, dv, mg);
                        }
                    }
                }
                // The parts added pairwise: (p0 + p1) + (p2 + p3) on the group's first lane.
                for (int off = 1; off < sd; off <<= 1) {
                    if (WG) {
#pragma unroll
                        for (int i = 0; i < 3; ++i) gs[i] = X::add(gs[i], __shfl_xor_sync(0xffffffffu, gs[i], off));
                    }
                    if (WH) {
#pragma unroll
                        for (int u6 = 0; u6 < 6; ++u6)
                            acc[u6] = X::add(acc[u6], __shfl_xor_sync(0xffffffffu, acc[u6], off));
                    }
                }
                if (active && part == 0) {
                    if (WG) {
                        const int v = rows[kTcRowInts * static_cast<int>(it.w & 0xffu)];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            if (!X::finite(gs[i])) st |= ST_NONFINITE_OUT;
                            a.grad[3 * static_cast<size_t>(v) + i] = static_cast<double>(gs[i]);
                        }
                    }
                    if (WH) {
                        constexpr int sym3[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int c = 0; c < 3; ++c) stage[tc_stage(it.x, csc, i, c)] = acc[sym3[3 * i + c]];
                    }
                }
            } else if (WH) {
                for (int kk = nd + tid - dpad; kk < ni; kk += kTcThreads - dpad) {
                    const uint4 it = sitems[kk];
                    // The solver layout keeps only blocks right of the diagonal: an edge to a
                    // lower-numbered row of another cluster is not needed there.
                    if (sell && ((it.w >> 30) & 1u)) continue;
                    const uint16_t* en = sents + (it.z & 0xfffffu);
                    const int cnt = static_cast<int>(it.z >> 20);
                    // Off-diagonal block in the orientation of the lower vertex (a) -> higher (b):
                    //   C += vol lambda h_a h_b^T - vol p h_b h_a^T + vol mu (grad N_a . grad N_b) I.
                    R acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll UNR
                    for (int c = 0; c < cnt; ++c) {
                        const int w = en[c];
                        const int el = w >> 8, pr = (w >> 4) & 15, ra = (w >> 2) & 3, cb = w & 3;
                        R ha[3], hb[3];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            ha[i] = ed[(kTcH + 3 * ra + i) * E + el];
                            hb[i] = ed[(kTcH + 3 * cb + i) * E + el];
                        }
                        const R lv = ed[kTcL * E + el], pv = ed[kTcP * E + el], mg = ed[(kTcCC + pr) * E + el];
                        R A[3], B[3];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            A[i] = X::mul(lv, ha[i]);
                            B[i] = X::mul(-pv, ha[i]);
                        }
                        edge_contrib<R>(acc, A, B, hb, mg);
                    }
                    const bool tr = (it.w >> 30) & 1u;
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int c = 0; c < 3; ++c) stage[tc_stage(it.x, csc, i, c)] = tr ? acc[3 * c + i] : acc[3 * i + c];
                    if (it.y != 0xffffffffu) {
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int c = 0; c < 3; ++c) stage[tc_stage(it.y, csc, i, c)] = acc[3 * c + i];
                    }
                }
            }
        }
        __syncthreads(); // staging complete; items, contributors and element data are dead
        // The next cluster's stage, in flight during the copy pass.
        const int nrc = nr;
        {
            const TcBounds bn = tc_bounds(s_hdr[buf]);
            tc_issue<R, ITEMS>(m, a.u, bn, x, tid, sell, su, sitems, sents, r12, rowv);
            ne = bn.ne;
            ni = WH ? bn.ni : bn.nd;
            nr = bn.nr;
            ndc = bn.nd;
        }
        if (WH) {
            // Copy pass: one warp per owned row.
            for (int j = warp; j < nrc; j += nw) {
                const int* rw = rows + kTcRowInts * j;
                const int so = rw[1], base = rw[2], nb = rw[3] & 0xff;
                bool ok = true;
                if (!sell) {
                    HT* dst = hout + 9 * static_cast<size_t>(base);
                    for (int t = lane; t < 9 * nb; t += 32) {
                        const R val = stage[so + t];
                        ok = ok && X::finite(val);
                        dst[t] = static_cast<HT>(val);
                    }
                } else {
                    const int qd = rw[3] >> 8, sb = rw[4];
                    for (int t = lane; t < 9 * (nb - qd); t += 32) {
                        const int qq = t / 9, tt = t - 9 * qq;
                        const R val = stage[so + 9 * qd + t];
                        ok = ok && X::finite(val);
                        hout[static_cast<int64_t>(sb) + 32 * static_cast<int64_t>(9 * qq + tt)] = static_cast<HT>(val);
                    }
                }
                if (!ok) st |= ST_NONFINITE_OUT;
            }
        }
    }
    cp_async_wait_all();
    st = __reduce_or_sync(0xffffffffu, st);
    if (lane == 0 && st) atomicOr(a.status, st);
}

template <typename R, bool WG, bool WH, int MINB = tc_minb<R>(0), int UNR = tc_unroll(0)>
void launch_tet_cluster(const DevMesh& m, const EvalArgs& a, cudaStream_t s) {
    const size_t sm = tc_smem_bytes<R>();
    thread_local LaunchCache cache;
    const int resident = resident_grid(tet_cluster_kernel<R, WG, WH, MINB, UNR>, kTcThreads, sm, cache);
    const int blocks = std::min(resident, m.tc_ncl);
    if (a.ev_begin) LPG_CUDA(cudaEventRecord(a.ev_begin, s));
    if (blocks > 0) tet_cluster_kernel<R, WG, WH, MINB, UNR><<<blocks, kTcThreads, sm, s>>>(m, a);
    if (a.ev_end) LPG_CUDA(cudaEventRecord(a.ev_end, s));
    LPG_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Hessian assembly from per-element blocks (the projected Hessian: each element's clamped
// tangent as ten 3x3 blocks in a.proj, pair10 order). The cluster plan of the Exact path without
// its element pass: one thread block per cluster stages the cluster's element ids, slot words and
// contributor lists, then each thread sums one block slot's contributors in ascending element
// order and stores the block once, in the lower vertex's orientation (transposed for the other),
// so the result is bitwise symmetric and deterministic. Contributor (a, b) = local indices of the
// lower- and higher-numbered vertex; the stored block is H_{min(a,b) max(a,b)}, read transposed
// when a > b.
// ---------------------------------------------------------------------------
// Cell-size traits of the block gather: K vertices per cell, bits per local index in a
// contributor, values per element in the block scratch, and the pair index of (a, b), a <= b.
template <int K> struct CellBlocks;
template <> struct CellBlocks<4> {
    static constexpr int shift = 2, record = kProjRecord;
    static __device__ __forceinline__ int pair(int a, int b) { return pair10(a, b); }
};
template <> struct CellBlocks<8> {
    static constexpr int shift = 3, record = kHexRecord;
    static __device__ __forceinline__ int pair(int a, int b) {
        const int lo = min(a, b), hi = max(a, b);
        return lo * 8 - (lo * (lo - 1)) / 2 + (hi - lo);
    }
};
template <> struct CellBlocks<64> {
    static constexpr int shift = 6, record = kHermiteRecord;
    static __device__ __forceinline__ int pair(int a, int b) {
        const int lo = min(a, b), hi = max(a, b);
        return lo * 64 - (lo * (lo - 1)) / 2 + (hi - lo);
    }
};

// Contributor word c of a list: one 16-bit word, or two (low half first) for 64-node cells.
template <int K> __device__ __forceinline__ uint32_t contributor(const uint16_t* en, int c) {
    if (K == 64) return static_cast<uint32_t>(en[2 * c]) | (static_cast<uint32_t>(en[2 * c + 1]) << 16);
    return en[c];
}

template <typename R, int K = 4>
__global__ void __launch_bounds__(kClThreads) block_gather_kernel(const DevMesh m, const EvalArgs a) {
    using CB = CellBlocks<K>;
    using HT = typename HOut<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int* sel = reinterpret_cast<int*>(smem_raw); // [kClusterElems] element ids
    int* rt = sel + kClusterElems;               // [4][kClusterRows] row table
    uint32_t* sslot = reinterpret_cast<uint32_t*>(rt + 4 * kClusterRows);
    uint32_t* sslote = sslot + m.cl_max_slots;
    uint16_t* sent = reinterpret_cast<uint16_t*>(smem_raw + block_gather_fixed() +
                                                 (8 * static_cast<size_t>(m.cl_max_slots) + 15) / 16 * 16);
    const R* blocks = reinterpret_cast<const R*>(a.proj);
    HT* hout = reinterpret_cast<HT*>(a.hess);
    const int tid = threadIdx.x, bd = blockDim.x;
    unsigned st = 0;
    for (int cl = blockIdx.x; cl < m.ncl; cl += gridDim.x) {
        if (a.cl_skip != nullptr && __ldg(a.cl_skip + cl) != 0) continue; // its mesh has finished
        const int s0 = __ldg(m.cl_slot_ptr + cl), ns = __ldg(m.cl_slot_ptr + cl + 1) - s0;
        const int eb = __ldg(m.cl_ent_ptr + cl), n16 = (__ldg(m.cl_ent_ptr + cl + 1) - eb) / 8;
        for (int i = tid; i < ns; i += bd) {
            __pipeline_memcpy_async(sslot + i, m.cl_slot + s0 + i, 4);
            __pipeline_memcpy_async(sslote + i, m.cl_slot_ent + s0 + i, 4);
        }
        for (int i = tid; i < n16; i += bd)
            __pipeline_memcpy_async(reinterpret_cast<uint4*>(sent) + i, reinterpret_cast<const uint4*>(m.cl_ents + eb) + i, 16);
        __pipeline_commit();
        const int e0 = __ldg(m.cl_el_ptr + cl), ne = __ldg(m.cl_el_ptr + cl + 1) - e0;
        for (int el = tid; el < ne; el += bd) sel[el] = static_cast<int>(__ldg(m.cl_els + e0 + el) & 0x7fffffffu);
        const int r0 = __ldg(m.cl_row_ptr + cl), nr = __ldg(m.cl_row_ptr + cl + 1) - r0;
        for (int j = tid; j < nr; j += bd) {
            const int v = __ldg(m.cl_rows + r0 + j);
            const int sb = __ldg(m.row_ptr + v);
            rt[j] = sb;
            rt[kClusterRows + j] = __ldg(m.row_ptr + v + 1) - sb;
            if (a.layout == kLayoutSell) rt[2 * kClusterRows + j] = __ldg(m.sell_base + v) - 288 * (__ldg(m.diag_slot + v) - sb);
        }
        __pipeline_wait_prior(0);
        __syncthreads();
        // The solver layout skips the slots left of the diagonal.
        const int first = a.layout == kLayoutSell ? __ldg(m.cl_ntr + cl) : 0;
        for (int s = first + tid; s < ns; s += bd) {
            const uint32_t d = sslot[s], de = sslote[s];
            const int j = d & 0xffu, q = (d >> 8) & 0x3fffffu;
            const uint16_t* en = sent + (de & 0xfffffu);
            const int cnt = static_cast<int>(de >> 20);
            R acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int c = 0; c < cnt; ++c) {
                const uint32_t w = contributor<K>(en, c);
                const int el = static_cast<int>(w >> (2 * CB::shift)), la = (w >> CB::shift) & (K - 1), lb = w & (K - 1);
                const R* blk = blocks + CB::record * static_cast<size_t>(sel[el]) + 9 * CB::pair(la, lb);
                R bv[9];
#pragma unroll
                for (int t = 0; t < 9; ++t) bv[t] = __ldg(blk + t);
                if (la <= lb) {
#pragma unroll
                    for (int t = 0; t < 9; ++t) acc[t] += bv[t];
                } else {
#pragma unroll
                    for (int t = 0; t < 9; ++t) acc[t] += bv[3 * (t % 3) + t / 3];
                }
            }
            const bool tr = (d >> 30) & 1u;
            const int slot0 = rt[j], nb = rt[kClusterRows + j], sb = rt[2 * kClusterRows + j];
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const R val = tr ? acc[3 * (t % 3) + t / 3] : acc[t];
                if (!(val == val) || val == R(INFINITY) || val == R(-INFINITY)) st |= ST_NONFINITE_OUT;
                hout[cl_pos(a.layout, slot0, nb, sb, q, t)] = static_cast<HT>(val);
            }
        }
        __syncthreads(); // the next cluster reuses the shared tables
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((tid & 31) == 0 && st) atomicOr(a.status, st);
}

size_t block_gather_bytes(const DevMesh& m) {
    return block_gather_fixed() + (8 * static_cast<size_t>(m.cl_max_slots) + 15) / 16 * 16 +
           2 * static_cast<size_t>(m.cl_max_ents);
}

template <typename R, int K = 4> void launch_block_gather(const DevMesh& m, const EvalArgs& a, cudaStream_t s) {
    const size_t sm = block_gather_bytes(m);
    thread_local LaunchCache cache;
    const int resident = resident_grid(block_gather_kernel<R, K>, kClThreads, sm, cache);
    const int blocks = std::min(resident, m.ncl);
    if (blocks > 0) block_gather_kernel<R, K><<<blocks, kClThreads, sm, s>>>(m, a);
    LPG_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Rest-position sensitivity of the elastic force. For one element with s = w . g_e =
// vol P : grad w (grad w = sum_a w_a grad N_a^T, H = F - I, Q = dP/dF [grad w] =
// mu grad w + lambda (F^-T : grad w) F^-T - p F^-T grad w^T F^-T):
//   d s / d X_a = vol M grad N_a,   M = (P : grad w) I - H^T Q - grad w^T P,
// from d(Dm^-1) = -Dm^-1 dDm Dm^-1 and d vol = vol tr(Dm^-1 dDm). Per element 12 values;
// a per-vertex pass sums them over the incident elements in element order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) rest_vjp_kernel(const DevMesh m, const double* __restrict__ u,
                                                       const double* __restrict__ w, double* __restrict__ out,
                                                       unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.T) return;
    const int4 tv = __ldg(m.tets + e);
    Kin<double> k;
    unsigned st = kinematics<double>(m, e, tv, u, k);
    const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
    double Wg[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; // row-major grad w
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double wi = __ldg(w + 3 * static_cast<size_t>(vs[a]) + i);
            if (!isfinite(wi)) st |= ST_BAD_INPUT;
#pragma unroll
            for (int j = 0; j < 3; ++j) Wg[3 * i + j] = fma(wi, k.n[a][j], Wg[3 * i + j]);
        }
    const double p = fma(k.lam, k.logJ, -k.mu);
    double P[9], tr = 0, PW = 0;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        P[t] = fma(k.mu, k.F[t], p * k.FiT[t]);
        tr = fma(k.FiT[t], Wg[t], tr);
        PW = fma(P[t], Wg[t], PW);
    }
    double FW[9]; // F^-T grad w^T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int l = 0; l < 3; ++l)
            FW[3 * i + l] = k.FiT[3 * i] * Wg[3 * l] + k.FiT[3 * i + 1] * Wg[3 * l + 1] + k.FiT[3 * i + 2] * Wg[3 * l + 2];
    double Q[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double flip = FW[3 * i] * k.FiT[j] + FW[3 * i + 1] * k.FiT[3 + j] + FW[3 * i + 2] * k.FiT[6 + j];
            Q[3 * i + j] = k.mu * Wg[3 * i + j] + k.lam * tr * k.FiT[3 * i + j] - p * flip;
        }
    double Mx[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double s = r == c ? PW : 0.0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double Hir = k.F[3 * i + r] - (i == r ? 1.0 : 0.0);
                s -= Hir * Q[3 * i + c] + Wg[3 * i + r] * P[3 * i + c];
            }
            Mx[3 * r + c] = s;
        }
    double* o = out + 12 * static_cast<size_t>(e);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double v = k.vol * (Mx[3 * r] * k.n[a][0] + Mx[3 * r + 1] * k.n[a][1] + Mx[3 * r + 2] * k.n[a][2]);
            if (!isfinite(v)) st |= ST_NONFINITE_OUT;
            o[3 * a + r] = v;
        }
    if (st) atomicOr(status, st);
}

// out[v] = sign * sum over the elements of v (ascending) of the per-element vertex values
// (12 per element); vertices of no element are left to zero_rows_kernel.
template <int K = 4>
__global__ void __launch_bounds__(128) vertex_gather_kernel(const DevMesh m, const double* __restrict__ per_elem,
                                                            double sign, double* __restrict__ out) {
    for (int cl = blockIdx.x; cl < m.ncl; cl += gridDim.x) {
        const int s0 = __ldg(m.cl_slot_ptr + cl), ns = __ldg(m.cl_slot_ptr + cl + 1) - s0;
        const int e0 = __ldg(m.cl_el_ptr + cl), r0 = __ldg(m.cl_row_ptr + cl);
        const uint16_t* ents = m.cl_ents + __ldg(m.cl_ent_ptr + cl);
        for (int s = __ldg(m.cl_noff + cl) + threadIdx.x; s < ns; s += blockDim.x) {
            const uint32_t d = __ldg(m.cl_slot + s0 + s), de = __ldg(m.cl_slot_ent + s0 + s);
            const int v = __ldg(m.cl_rows + r0 + (d & 0xffu));
            const uint16_t* en = ents + (de & 0xfffffu);
            double acc[3] = {0, 0, 0};
            for (int c = 0; c < static_cast<int>(de >> 20); ++c) {
                const uint32_t wd = K == 64 ? static_cast<uint32_t>(__ldg(en + 2 * c)) | (static_cast<uint32_t>(__ldg(en + 2 * c + 1)) << 16)
                                            : __ldg(en + c);
                constexpr int sh = cell_bits(K);
                const size_t e = __ldg(m.cl_els + e0 + (wd >> (2 * sh))) & 0x7fffffffu;
                const int a = (wd >> sh) & (K - 1);
#pragma unroll
                for (int i = 0; i < 3; ++i) acc[i] += __ldg(per_elem + 3 * K * e + 3 * a + i);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) out[3 * static_cast<size_t>(v) + i] = sign * acc[i];
        }
    }
}

// ---------------------------------------------------------------------------
// Materials evaluated outside the library (PyVolumetricMaterial, src/python/fem.py:59-109): the
// library exports each element's deformation gradient, the caller evaluates W, dW/dF and
// d2W/dF2 at those points, and the library integrates and assembles them.
// ---------------------------------------------------------------------------
// F = I + grad u per element (row-major, 9 per element), FP64; no plastic field on the handle.
__global__ void __launch_bounds__(256) deformation_gradient_kernel(const DevMesh m, const double* __restrict__ u,
                                                                   double* __restrict__ F, unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const int4 tv = __ldg(m.tets + e);
        const int vs[4] = {tv.x, tv.y, tv.z, tv.w};
        double uu[4][3];
        bool ok = true;
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                uu[c][i] = __ldg(u + 3 * static_cast<size_t>(vs[c]) + i);
                ok = ok && isfinite(uu[c][i]);
            }
        if (!ok) st |= ST_BAD_INPUT;
        const double* rec = m.rec64 + 12 * static_cast<size_t>(e);
        double* o = F + 9 * static_cast<size_t>(e);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double h = (i == j) ? 1.0 : 0.0;
#pragma unroll
                for (int c = 0; c < 3; ++c) h = fma(uu[c + 1][i] - uu[0][i], __ldg(rec + 3 * c + j), h);
                o[3 * i + j] = h;
            }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Per element: vol W and the gradient pieces g_a = vol P grad N_a (12 values, vertex-major),
// from the caller's W (T) and P = dW/dF (9 per element, row-major). Non-finite material outputs
// reject the evaluation.
__global__ void __launch_bounds__(256) material_pieces_kernel(const DevMesh m, const double* __restrict__ W,
                                                              const double* __restrict__ P, double* __restrict__ elemE,
                                                              double* __restrict__ per_elem, unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const double* rec = m.rec64 + 12 * static_cast<size_t>(e);
        const double vol = rec[9];
        double n[4][3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int j = 0; j < 3; ++j) n[c + 1][j] = rec[3 * c + j];
#pragma unroll
        for (int j = 0; j < 3; ++j) n[0][j] = -(n[1][j] + n[2][j] + n[3][j]);
        const double w = __ldg(W + e);
        const double Ee = vol * w;
        if (!isfinite(Ee)) st |= ST_NONFINITE_OUT;
        elemE[e] = Ee;
        if (per_elem) {
            double Pe[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) Pe[t] = __ldg(P + 9 * static_cast<size_t>(e) + t);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double g = vol * (Pe[3 * i] * n[a][0] + Pe[3 * i + 1] * n[a][1] + Pe[3 * i + 2] * n[a][2]);
                    if (!isfinite(g)) st |= ST_NONFINITE_OUT;
                    per_elem[12 * static_cast<size_t>(e) + 3 * a + i] = g;
                }
        }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// ---------------------------------------------------------------------------
// Hex Q1 neo-Hookean element pass (VolumetricFemEnergy<NeoHookean, HexQ1Basis, GaussLegendre3D<n>>,
// volumetric_fem_energy.hpp:78-123 with hex_q1_basis.hpp and gauss_legendre_3d.hpp). One thread
// per (element, vertex pair a <= b): at every quadrature point it forms J = sum_c X_c dN_c^T,
// w = weight det J, grad N = J^-T dN, F = I + (sum_c u_c dN_c^T) J^-1, and accumulates
// H_ab += w [mu (grad N_a . grad N_b) I + lambda h_a h_b^T - p h_b h_a^T], h = F^-T grad N; the
// pair (a, a) threads also accumulate g_a = sum w P grad N_a and the (0, 0) thread the energy.
// FP64 throughout; the blocks are stored in the precision's type. The kinematics are recomputed
// by each of an element's 36 threads (cheap next to reading a per-point cache).
// ---------------------------------------------------------------------------
// The rest geometry at one quadrature point of a hex (dq: the point's table row): J = sum_c X_c
// dN_c^T (corners in order, fma per entry), its determinant and its inverse by cofactors.
__device__ __forceinline__ void hex_point_geometry(const DevMesh& m, const int32_t* cell, const double* dq,
                                                   double (&Ji)[9], double& dJ) {
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
        const int v = __ldg(cell + c);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double X = __ldg(m.hex_X + 3 * static_cast<size_t>(v) + i);
#pragma unroll
            for (int d = 0; d < 3; ++d) J[3 * i + d] = fma(X, __ldg(dq + 3 * c + d), J[3 * i + d]);
        }
    }
    dJ = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
    const double iJ = 1.0 / dJ;
    Ji[0] = (J[4] * J[8] - J[5] * J[7]) * iJ;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) * iJ;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) * iJ;
    Ji[3] = (J[5] * J[6] - J[3] * J[8]) * iJ;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) * iJ;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) * iJ;
    Ji[6] = (J[3] * J[7] - J[4] * J[6]) * iJ;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) * iJ;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) * iJ;
}

__device__ __forceinline__ void hex_pair(int pr, int& a, int& b) {
    a = 0;
    int base = 0;
    while (pr >= base + (8 - a)) {
        base += 8 - a;
        ++a;
    }
    b = a + (pr - base);
}

template <typename R>
__global__ void __launch_bounds__(128) hex_element_kernel(const DevMesh m, const double* __restrict__ u,
                                                          double* __restrict__ elemE, double* __restrict__ per_elem,
                                                          R* __restrict__ blocks, unsigned* status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    const int e = t / 36, pr = t - 36 * (t / 36);
    if (e < m.T) {
        int a, b;
        hex_pair(pr, a, b);
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        const double lam = m.hex_theta[2 * static_cast<size_t>(e)], mu = m.hex_theta[2 * static_cast<size_t>(e) + 1];
        if (!(lam >= 0 && mu > 0 && isfinite(lam) && isfinite(mu))) st |= ST_BAD_THETA;
        double Hb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ga[3] = {0, 0, 0}, E = 0;
        for (int q = 0; q < m.nq; ++q) {
            const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
            // J^-1 (det J > 0 was checked when the mesh was built) and grad u in reference coordinates.
            double Ji[9], dJ;
            hex_point_geometry(m, cell, dq, Ji, dJ);
            double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            bool ok = true;
            for (int c = 0; c < 8; ++c) {
                const int v = __ldg(cell + c);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double uu = __ldg(u + 3 * static_cast<size_t>(v) + i);
                    ok = ok && isfinite(uu);
#pragma unroll
                    for (int d = 0; d < 3; ++d) G[3 * i + d] = fma(uu, __ldg(dq + 3 * c + d), G[3 * i + d]);
                }
            }
            if (!ok) st |= ST_BAD_INPUT;
            const double w = __ldg(dq + 24) * dJ;
            double F[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    F[3 * i + j] = (i == j ? 1.0 : 0.0) + G[3 * i] * Ji[j] + G[3 * i + 1] * Ji[3 + j] + G[3 * i + 2] * Ji[6 + j];
            double C[9]; // cofactors: F^-T = C / det F
            C[0] = F[4] * F[8] - F[5] * F[7];
            C[1] = F[5] * F[6] - F[3] * F[8];
            C[2] = F[3] * F[7] - F[4] * F[6];
            C[3] = F[2] * F[7] - F[1] * F[8];
            C[4] = F[0] * F[8] - F[2] * F[6];
            C[5] = F[1] * F[6] - F[0] * F[7];
            C[6] = F[1] * F[5] - F[2] * F[4];
            C[7] = F[2] * F[3] - F[0] * F[5];
            C[8] = F[0] * F[4] - F[1] * F[3];
            const double detF = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
            if (!(detF > 0) || !isfinite(detF)) {
                st |= isfinite(detF) ? ST_BAD_DET : ST_NONFINITE_F;
                continue;
            }
            const double L = log(detF), p = lam * L - mu;
            double FiT[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) FiT[k] = C[k] / detF;
            // grad N of a and b: rows of dN J^-1.
            double na[3], nb[3];
            const double* dA = dq + 3 * a;
            const double* dB = dq + 3 * b;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                na[j] = __ldg(dA) * Ji[j] + __ldg(dA + 1) * Ji[3 + j] + __ldg(dA + 2) * Ji[6 + j];
                nb[j] = __ldg(dB) * Ji[j] + __ldg(dB + 1) * Ji[3 + j] + __ldg(dB + 2) * Ji[6 + j];
            }
            double ha[3], hb[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                ha[i] = FiT[3 * i] * na[0] + FiT[3 * i + 1] * na[1] + FiT[3 * i + 2] * na[2];
                hb[i] = FiT[3 * i] * nb[0] + FiT[3 * i + 1] * nb[1] + FiT[3 * i + 2] * nb[2];
            }
            const double dn = na[0] * nb[0] + na[1] * nb[1] + na[2] * nb[2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    double v = lam * ha[i] * hb[k] - p * hb[i] * ha[k];
                    if (i == k) v += mu * dn;
                    Hb[3 * i + k] = fma(w, v, Hb[3 * i + k]);
                }
            if (a == b) {
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    double s = 0;
#pragma unroll
                    for (int j = 0; j < 3; ++j) s += (mu * F[3 * i + j] + p * FiT[3 * i + j]) * na[j];
                    ga[i] = fma(w, s, ga[i]);
                }
                if (a == 0) {
                    double ff = 0;
#pragma unroll
                    for (int k = 0; k < 9; ++k) ff += F[k] * F[k];
                    E = fma(w, 0.5 * mu * (ff - 3.0) - mu * L + 0.5 * lam * L * L, E);
                }
            }
        }
        if (a == b) { // a diagonal block: mirror the upper triangle so the matrix is bitwise symmetric
            Hb[3] = Hb[1];
            Hb[6] = Hb[2];
            Hb[7] = Hb[5];
        }
        if (blocks) {
            R* o = blocks + kHexRecord * static_cast<size_t>(e) + 9 * pr;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                if (!isfinite(Hb[k])) st |= ST_NONFINITE_OUT;
                o[k] = static_cast<R>(Hb[k]);
            }
        }
        if (a == b && per_elem) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (!isfinite(ga[i])) st |= ST_NONFINITE_OUT;
                per_elem[24 * static_cast<size_t>(e) + 3 * a + i] = ga[i];
            }
        }
        if (pr == 0) {
            if (!isfinite(E)) st |= ST_NONFINITE_OUT;
            elemE[e] = E;
        }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Force-response parameter VJP of hex meshes (the tet pass's force_vjp_kernel at every
// quadrature point): per element, with grad w = (sum_c w_c dN_c^T) J^-1 at each point,
//   d/dlambda = sum_q w_q log J_q (F_q^-T : grad w_q),   d/dmu = sum_q w_q ((F_q - F_q^-T) : grad w_q),
// w_q = weight det J. One thread per element, points in order; FP64.
__global__ void __launch_bounds__(128) hex_force_vjp_kernel(const DevMesh m, const double* __restrict__ u,
                                                            const double* __restrict__ w, double* out,
                                                            unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        double dl = 0, dm = 0;
        for (int q = 0; q < m.nq; ++q) {
            const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
            double Ji[9], dJ;
            hex_point_geometry(m, cell, dq, Ji, dJ);
            double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Wr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int c = 0; c < 8; ++c) {
                const int v = __ldg(cell + c);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double uu = __ldg(u + 3 * static_cast<size_t>(v) + i);
                    const double ww = __ldg(w + 3 * static_cast<size_t>(v) + i);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double dn = __ldg(dq + 3 * c + d);
                        G[3 * i + d] = fma(uu, dn, G[3 * i + d]);
                        Wr[3 * i + d] = fma(ww, dn, Wr[3 * i + d]);
                    }
                }
            }
            double F[9], Wg[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    F[3 * i + j] = (i == j ? 1.0 : 0.0) + G[3 * i] * Ji[j] + G[3 * i + 1] * Ji[3 + j] +
                                   G[3 * i + 2] * Ji[6 + j];
                    Wg[3 * i + j] = Wr[3 * i] * Ji[j] + Wr[3 * i + 1] * Ji[3 + j] + Wr[3 * i + 2] * Ji[6 + j];
                }
            double C[9];
            C[0] = F[4] * F[8] - F[5] * F[7];
            C[1] = F[5] * F[6] - F[3] * F[8];
            C[2] = F[3] * F[7] - F[4] * F[6];
            C[3] = F[2] * F[7] - F[1] * F[8];
            C[4] = F[0] * F[8] - F[2] * F[6];
            C[5] = F[1] * F[6] - F[0] * F[7];
            C[6] = F[1] * F[5] - F[2] * F[4];
            C[7] = F[2] * F[3] - F[0] * F[5];
            C[8] = F[0] * F[4] - F[1] * F[3];
            const double detF = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
            if (!(detF > 0) || !isfinite(detF)) {
                st |= isfinite(detF) ? ST_BAD_DET : ST_NONFINITE_F;
                continue;
            }
            double hf = 0, ff = 0;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                hf = fma(C[k] / detF, Wg[k], hf);
                ff = fma(F[k], Wg[k], ff);
            }
            const double wq = __ldg(dq + 24) * dJ;
            dl = fma(wq * log(detF), hf, dl);
            dm = fma(wq, ff - hf, dm);
        }
        if (!isfinite(dl) || !isfinite(dm)) st |= ST_NONFINITE_OUT;
        out[2 * static_cast<size_t>(e)] = dl;
        out[2 * static_cast<size_t>(e) + 1] = dm;
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Materials evaluated outside the library on hex meshes (PyVolumetricMaterial over HexQ1Basis):
// F at every quadrature point (row-major, 9 per point, points of an element consecutive), then
// the caller's W, P = dW/dF and A = d2W/dF2 per point integrated and assembled per hex.
__global__ void __launch_bounds__(128) hex_deformation_gradient_kernel(const DevMesh m, const double* __restrict__ u,
                                                                       double* __restrict__ F, unsigned* status) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (t < static_cast<size_t>(m.T) * m.nq) {
        const int e = static_cast<int>(t / m.nq), q = static_cast<int>(t - static_cast<size_t>(m.nq) * e);
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
        double Ji[9], dJ;
        hex_point_geometry(m, cell, dq, Ji, dJ);
        double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        bool ok = true;
        for (int c = 0; c < 8; ++c) {
            const int v = __ldg(cell + c);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double uu = __ldg(u + 3 * static_cast<size_t>(v) + i);
                ok = ok && isfinite(uu);
#pragma unroll
                for (int d = 0; d < 3; ++d) G[3 * i + d] = fma(uu, __ldg(dq + 3 * c + d), G[3 * i + d]);
            }
        }
        if (!ok) st |= ST_BAD_INPUT;
        double* o = F + 9 * t;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                o[3 * i + j] = (i == j ? 1.0 : 0.0) + G[3 * i] * Ji[j] + G[3 * i + 1] * Ji[3 + j] + G[3 * i + 2] * Ji[6 + j];
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// One thread per (element, vertex pair a <= b), 36 per hex, points in order: with grad N = J^-T dN
// and w_q = weight det J,
//   H_ab(i, k) += w_q sum_{j, l} grad N_a[j] As(3 i + j, 3 k + l) grad N_b[l],  As = (A + A^T) / 2,
//   g_a += w_q P grad N_a (pairs (a, a)),  E += w_q W (pair (0, 0)).
// Diagonal blocks are mirrored (bitwise symmetric); A may be null when no Hessian is asked for.
template <typename R>
__global__ void __launch_bounds__(128) hex_material_kernel(const DevMesh m, const double* __restrict__ W,
                                                           const double* __restrict__ P, const double* __restrict__ A,
                                                           double* __restrict__ elemE, double* __restrict__ per_elem,
                                                           R* __restrict__ blocks, unsigned* status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    const int e = t / 36, pr = t - 36 * (t / 36);
    if (e < m.T) {
        int a, b;
        hex_pair(pr, a, b);
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        double Hb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ga[3] = {0, 0, 0}, E = 0;
        for (int q = 0; q < m.nq; ++q) {
            const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
            double Ji[9], dJ;
            hex_point_geometry(m, cell, dq, Ji, dJ);
            const double w = __ldg(dq + 24) * dJ;
            const size_t pt = static_cast<size_t>(e) * m.nq + q;
            double na[3], nb[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                na[j] = __ldg(dq + 3 * a) * Ji[j] + __ldg(dq + 3 * a + 1) * Ji[3 + j] + __ldg(dq + 3 * a + 2) * Ji[6 + j];
                nb[j] = __ldg(dq + 3 * b) * Ji[j] + __ldg(dq + 3 * b + 1) * Ji[3 + j] + __ldg(dq + 3 * b + 2) * Ji[6 + j];
            }
            if (blocks) {
                const double* Aq = A + 81 * pt;
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        double v = 0;
#pragma unroll
                        for (int j = 0; j < 3; ++j)
#pragma unroll
                            for (int l = 0; l < 3; ++l) {
                                const double as = 0.5 * (__ldg(Aq + 9 * (3 * i + j) + 3 * k + l) +
                                                         __ldg(Aq + 9 * (3 * k + l) + 3 * i + j));
                                v = fma(na[j] * as, nb[l], v);
                            }
                        Hb[3 * i + k] = fma(w, v, Hb[3 * i + k]);
                    }
            }
            if (a == b && per_elem) {
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double* Pq = P + 9 * pt + 3 * i;
                    ga[i] = fma(w, __ldg(Pq) * na[0] + __ldg(Pq + 1) * na[1] + __ldg(Pq + 2) * na[2], ga[i]);
                }
            }
            if (pr == 0) E = fma(w, __ldg(W + pt), E);
        }
        if (a == b) {
            Hb[3] = Hb[1];
            Hb[6] = Hb[2];
            Hb[7] = Hb[5];
        }
        if (blocks) {
            R* o = blocks + kHexRecord * static_cast<size_t>(e) + 9 * pr;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                if (!isfinite(Hb[k])) st |= ST_NONFINITE_OUT;
                o[k] = static_cast<R>(Hb[k]);
            }
        }
        if (a == b && per_elem) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (!isfinite(ga[i])) st |= ST_NONFINITE_OUT;
                per_elem[24 * static_cast<size_t>(e) + 3 * a + i] = ga[i];
            }
        }
        if (pr == 0) {
            if (!isfinite(E)) st |= ST_NONFINITE_OUT;
            elemE[e] = E;
        }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// The projection pre-test on a material's own tangents: one thread per (element, point), the
// symmetrised As = (A + A^T) / 2 through the LDL^T test; an element with a point that fails is
// marked in flags (zeroed before).
__global__ void __launch_bounds__(128) hex_material_tangent_test_kernel(const DevMesh m, const double* __restrict__ A,
                                                                        int* __restrict__ flags) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(m.T) * m.nq) return;
    const int e = static_cast<int>(t / m.nq);
    const double* Aq = A + 81 * t;
    double V[81];
    double scale = 0;
    for (int r = 0; r < 9; ++r)
        for (int c = 0; c < 9; ++c) {
            const double v = 0.5 * (__ldg(Aq + 9 * r + c) + __ldg(Aq + 9 * c + r));
            V[9 * r + c] = v;
            if (r == c) scale = fmax(scale, fabs(v));
        }
    if (!(scale < INFINITY) || !semidefinite_ldlt<9>(V, 64 * Eps<double>::v * scale)) flags[e] = 1;
}

// Pre-test of the hex projection: H = sum_q w_q B_q^T A_q B_q (w_q > 0) is semi-definite when
// every quadrature point's tangent A_q = dP/dF is, and then H is its own projection. One thread
// per (element, point) forms
//   A(3 i + j, 3 k + l) = mu d_ik d_jl + lambda G_ij G_kl - p G_il G_kj,  G = F^-T, p = lambda log J - mu
// (bitwise symmetric: each product is formed from the same two factors both ways) and runs the
// LDL^T test with the tet pass's round-off allowance; an element with a point that fails is
// marked in flags (zeroed before) for the eigen-projection. A failed point (det F <= 0 or
// non-finite) marks its element too; the element pass reports it.
__global__ void __launch_bounds__(128) hex_tangent_test_kernel(const DevMesh m, const double* __restrict__ u,
                                                               int* __restrict__ flags) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<size_t>(m.T) * m.nq) return;
    const int e = static_cast<int>(t / m.nq), q = static_cast<int>(t - static_cast<size_t>(m.nq) * e);
    const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
    const double lam = m.hex_theta[2 * static_cast<size_t>(e)], mu = m.hex_theta[2 * static_cast<size_t>(e) + 1];
    const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
    double Ji[9], dJ;
    hex_point_geometry(m, cell, dq, Ji, dJ);
    double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
        const int v = __ldg(cell + c);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double uu = __ldg(u + 3 * static_cast<size_t>(v) + i);
#pragma unroll
            for (int d = 0; d < 3; ++d) G[3 * i + d] = fma(uu, __ldg(dq + 3 * c + d), G[3 * i + d]);
        }
    }
    double F[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            F[3 * i + j] = (i == j ? 1.0 : 0.0) + G[3 * i] * Ji[j] + G[3 * i + 1] * Ji[3 + j] + G[3 * i + 2] * Ji[6 + j];
    double C[9];
    C[0] = F[4] * F[8] - F[5] * F[7];
    C[1] = F[5] * F[6] - F[3] * F[8];
    C[2] = F[3] * F[7] - F[4] * F[6];
    C[3] = F[2] * F[7] - F[1] * F[8];
    C[4] = F[0] * F[8] - F[2] * F[6];
    C[5] = F[1] * F[6] - F[0] * F[7];
    C[6] = F[1] * F[5] - F[2] * F[4];
    C[7] = F[2] * F[3] - F[0] * F[5];
    C[8] = F[0] * F[4] - F[1] * F[3];
    const double detF = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
    if (!(detF > 0) || !isfinite(detF)) {
        flags[e] = 1;
        return;
    }
    double Gt[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Gt[k] = C[k] / detF;
    const double p = lam * log(detF) - mu;
    double A[81];
    double scale = 0;
#pragma unroll
    for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            const int i = r / 3, j = r % 3, k = c / 3, l = c % 3;
            double v = lam * (Gt[r] * Gt[c]) - p * (Gt[3 * i + l] * Gt[3 * k + j]);
            if (r == c) {
                v += mu;
                scale = fmax(scale, fabs(v));
            }
            A[9 * r + c] = v;
        }
    if (!(scale < INFINITY) || !semidefinite_ldlt<9>(A, 64 * Eps<double>::v * scale)) flags[e] = 1;
}

// Projected Hessian of hex meshes (HessianKind::Projected, mesh_energy.cpp:16-27): one warp per
// element loads its record of 36 FP64 blocks (hex_element_kernel) as the 24x24 element Hessian
// into shared memory, runs the parallel-ordered Jacobi iteration (lpg_psd.h) and writes
// V max(L, 0) V^T back as 36 blocks in the precision's type: in place for FP64 (a warp reads its
// whole record before it writes), into a separate FP32 record array for mixed precision. Each
// entry is formed once from the upper triangle, so the diagonal blocks stay bitwise symmetric.
struct WarpTeam {
    int l;
    __device__ int lane() const { return l; }
    __device__ int size() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
    __device__ double sum(double x) const {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        return __shfl_sync(0xffffffffu, x, 0);
    }
};

constexpr int kHexPsdWarps = 4;

template <typename R>
__global__ void __launch_bounds__(32 * kHexPsdWarps) hex_psd_kernel(int T, const double* in, R* out,
                                                                   const int* __restrict__ flags, unsigned* status) {
    using J = PsdJacobi<24>;
    __shared__ double sA[kHexPsdWarps][24 * J::S], sV[kHexPsdWarps][24 * J::S];
    __shared__ double sCS[kHexPsdWarps][J::kCs], sL[kHexPsdWarps][24];
    __shared__ int sPQ[kHexPsdWarps][24];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.x * kHexPsdWarps + w; // uniform over the warp: a warp leaves whole
    if (e >= T) return;
    const double* rec = in + kHexRecord * static_cast<size_t>(e);
    R* o = out + kHexRecord * static_cast<size_t>(e);
    if (flags[e] == 0) { // semi-definite (hex_tangent_test_kernel): the Hessian as it is
        if (static_cast<const void*>(rec) != static_cast<const void*>(o))
            for (int t = lane; t < kHexRecord; t += 32) o[t] = static_cast<R>(rec[t]);
        return;
    }
    double* A = sA[w];
    for (int t = lane; t < kHexRecord; t += 32) {
        int a, b;
        hex_pair(t / 9, a, b);
        const int i = 3 * a + (t % 9) / 3, k = 3 * b + t % 3;
        const double v = rec[t];
        A[i * J::S + k] = v;
        if (a != b) A[k * J::S + i] = v;
    }
    J::eigen(WarpTeam{lane}, A, sV[w], sCS[w], sPQ[w], sL[w]);
    unsigned st = 0;
    for (int t = lane; t < kHexRecord; t += 32) {
        int a, b;
        hex_pair(t / 9, a, b);
        int i = 3 * a + (t % 9) / 3, k = 3 * b + t % 3;
        if (i > k) {
            const int x = i;
            i = k;
            k = x;
        }
        const double v = J::entry(sV[w], sL[w], i, k);
        if (!isfinite(v)) st |= ST_NONFINITE_OUT;
        o[t] = static_cast<R>(v);
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if (lane == 0 && st) atomicOr(status, st);
}

// Feasible step of a hex mesh: at every quadrature point F and dF (the increment's gradient),
// the reference's positive-determinant step, minimum per block.
__global__ void __launch_bounds__(256) hex_feasible_kernel(const DevMesh m, const double* __restrict__ u,
                                                           const double* __restrict__ du, double* block_min,
                                                           unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double alpha = 1.0;
    unsigned st = 0;
    if (e < m.T) {
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        for (int q = 0; q < m.nq && st == 0; ++q) {
            const double* dq = m.hex_q + 25 * static_cast<size_t>(q);
            double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            bool ok = true;
            for (int c = 0; c < 8; ++c) {
                const int v = __ldg(cell + c);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double uu = u[3 * static_cast<size_t>(v) + i], dd = du[3 * static_cast<size_t>(v) + i];
                    ok = ok && isfinite(uu) && isfinite(dd);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double dn = __ldg(dq + 3 * c + d);
                        G[3 * i + d] = fma(uu, dn, G[3 * i + d]);
                        D[3 * i + d] = fma(dd, dn, D[3 * i + d]);
                    }
                }
            }
            if (!ok) {
                st |= ST_BAD_INPUT;
                break;
            }
            double Ji[9], dJ;
            hex_point_geometry(m, cell, dq, Ji, dJ);
            double F[9], dF[9];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    F[3 * i + j] = (i == j ? 1.0 : 0.0) + G[3 * i] * Ji[j] + G[3 * i + 1] * Ji[3 + j] + G[3 * i + 2] * Ji[6 + j];
                    dF[3 * i + j] = D[3 * i] * Ji[j] + D[3 * i + 1] * Ji[3 + j] + D[3 * i + 2] * Ji[6 + j];
                }
            alpha = fmin(alpha, positive_det_step(F, dF, st));
        }
    }
    __shared__ double sm[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) alpha = fmin(alpha, __shfl_xor_sync(0xffffffffu, alpha, off));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = alpha;
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = sm[0];
        for (int w = 1; w < (blockDim.x >> 5); ++w) v = fmin(v, sm[w]);
        block_min[blockIdx.x] = v;
    }
}

// ---------------------------------------------------------------------------
// Tricubic Hermite hexes (VolumetricFemEnergy<NeoHookean, HexHermiteBasis, GaussLegendre3D<n>>,
// hex_hermite_basis.hpp, with the physical DOFs of BasisDofTransform<HexHermiteBasis>,
// basis_dof_transform.hpp:59-148). Elements are axis-aligned boxes of edge lengths h; a vertex
// carries 24 physical DOFs, slots u, u_X, u_Y, u_Z, u_XY, u_XZ, u_YZ, u_XYZ of 3 components, and
// node b = 8 corner + slot of an element is the plan's row 8 v + slot. With the slot scale s_b
// (1, hx, hy, hz, hx hy, hx hz, hy hz, hx hy hz) and G_b = s_b (dN_b / dxi) / h at a point,
// F = I + sum_b d_b G_b^T on the physical DOFs d, so the element's gradient and Hessian come out
// pulled back to physical DOFs (s g, S H S) as in the reference, with w = weight hx hy hz and
//   g_b = sum_q w P G_b,   H_ab = sum_q w [mu (G_a . G_b) I + lambda h_a h_b^T - p h_b h_a^T], h = F^-T G.
// The point table holds, per point, the 64 x 3 reference derivatives and the weight (193 values).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hermite_slot_scale(int slot, double hx, double hy, double hz) {
    switch (slot) {
    case 0: return 1.0;
    case 1: return hx;
    case 2: return hy;
    case 3: return hz;
    case 4: return hx * hy;
    case 5: return hx * hz;
    case 6: return hy * hz;
    default: return hx * hy * hz;
    }
}

// G_b at a point (tq: the point's table row).
__device__ __forceinline__ void hermite_G(const double* tq, int b, const double (&h)[3], double (&G)[3]) {
    const double sb = hermite_slot_scale(b & 7, h[0], h[1], h[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) G[d] = sb * __ldg(tq + 3 * b + d) / h[d];
}

__device__ __forceinline__ void hermite_pair(int pr, int& a, int& b) {
    a = 0;
    int base = 0;
    while (pr >= base + (64 - a)) {
        base += 64 - a;
        ++a;
    }
    b = a + (pr - base);
}

// One CTA per element: the element's 192 DOFs and each point's w, p, F^-T and P in shared
// memory (points by thread), then the energy (thread 0, points in order), the gradient (a thread
// per node) and the 2080 blocks H_ab, a <= b (strided over the CTA; diagonal blocks mirrored so
// the matrix is bitwise symmetric).
constexpr int kHermiteThreads = 128;

// With flags (projected Hessian), flags[e] is set when the tangent d2W/dF2 of some point is not
// positive semi-definite (the element's Hessian then needs the eigenvalue clamp), and cleared
// otherwise: a sum of w B^T A B with semi-definite A is semi-definite.
template <typename R>
__global__ void __launch_bounds__(kHermiteThreads) hermite_element_kernel(const DevMesh m, const double* __restrict__ u,
                                                                          double* __restrict__ elemE,
                                                                          double* __restrict__ per_elem,
                                                                          R* __restrict__ blocks, unsigned* status,
                                                                          int* __restrict__ flags = nullptr) {
    __shared__ int sFlag;
    __shared__ double sD[192];
    __shared__ double sK[64 * 20]; // per point: w, p, F^-T (9), P (9)
    __shared__ double sE[64];
    __shared__ int sOk[64];
    const int e = blockIdx.x, tid = threadIdx.x;
    unsigned st = 0;
    const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
    const double lam = m.hex_theta[2 * static_cast<size_t>(e)], mu = m.hex_theta[2 * static_cast<size_t>(e) + 1];
    if (!(lam >= 0 && mu > 0 && isfinite(lam) && isfinite(mu))) st |= ST_BAD_THETA;
    const double h[3] = {m.herm_h[3 * static_cast<size_t>(e)], m.herm_h[3 * static_cast<size_t>(e) + 1],
                         m.herm_h[3 * static_cast<size_t>(e) + 2]};
    for (int t = tid; t < 192; t += blockDim.x) {
        const double d = __ldg(u + 24 * static_cast<size_t>(__ldg(cell + t / 24)) + t % 24);
        if (!isfinite(d)) st |= ST_BAD_INPUT;
        sD[t] = d;
    }
    if (tid == 0) sFlag = 0;
    __syncthreads();
    for (int q = tid; q < m.nq; q += blockDim.x) {
        const double* tq = m.herm_q + kHermiteTable * static_cast<size_t>(q);
        double Gu[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int b = 0; b < 64; ++b) {
            double G[3];
            hermite_G(tq, b, h, G);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int d = 0; d < 3; ++d) Gu[3 * i + d] = fma(sD[3 * b + i], G[d], Gu[3 * i + d]);
        }
        double F[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = Gu[k] + (k % 4 == 0 ? 1.0 : 0.0);
        double C[9];
        C[0] = F[4] * F[8] - F[5] * F[7];
        C[1] = F[5] * F[6] - F[3] * F[8];
        C[2] = F[3] * F[7] - F[4] * F[6];
        C[3] = F[2] * F[7] - F[1] * F[8];
        C[4] = F[0] * F[8] - F[2] * F[6];
        C[5] = F[1] * F[6] - F[0] * F[7];
        C[6] = F[1] * F[5] - F[2] * F[4];
        C[7] = F[2] * F[3] - F[0] * F[5];
        C[8] = F[0] * F[4] - F[1] * F[3];
        const double detF = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
        double* k = sK + 20 * q;
        if (!(detF > 0) || !isfinite(detF)) {
            st |= isfinite(detF) ? ST_BAD_DET : ST_NONFINITE_F;
            sOk[q] = 0;
            sE[q] = 0;
            continue;
        }
        sOk[q] = 1;
        const double L = log(detF), p = lam * L - mu, w = __ldg(tq + 192) * h[0] * h[1] * h[2];
        k[0] = w;
        k[1] = p;
        if (flags) {
            // The point's tangent A[(3i+j)(3k+l)] = mu d_ik d_jl + lambda H_ij H_kl - p H_il H_kj (H = F^-T).
            double Gt[9], A[81], scale = 0;
#pragma unroll
            for (int t = 0; t < 9; ++t) Gt[t] = C[t] / detF;
            for (int r = 0; r < 9; ++r)
                for (int c = 0; c < 9; ++c) {
                    const int i = r / 3, j = r % 3, kk = c / 3, l = c % 3;
                    double v = lam * (Gt[r] * Gt[c]) - p * (Gt[3 * i + l] * Gt[3 * kk + j]);
                    if (r == c) {
                        v += mu;
                        scale = fmax(scale, fabs(v));
                    }
                    A[9 * r + c] = v;
                }
            if (!(scale < INFINITY) || !semidefinite_ldlt<9>(A, 64 * Eps<double>::v * scale)) sFlag = 1;
        }
        double ff = 0;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const double fit = C[t] / detF;
            k[2 + t] = fit;
            k[11 + t] = mu * F[t] + p * fit;
            ff += F[t] * F[t];
        }
        sE[q] = w * (0.5 * mu * (ff - 3.0) - mu * L + 0.5 * lam * L * L);
    }
    __syncthreads();
    if (tid == 0) {
        double E = 0;
        for (int q = 0; q < m.nq; ++q) E += sE[q];
        if (!isfinite(E)) st |= ST_NONFINITE_OUT;
        elemE[e] = E;
        if (flags) flags[e] = sFlag;
    }
    if (per_elem) {
        for (int b = tid; b < 64; b += blockDim.x) {
            double ga[3] = {0, 0, 0};
            for (int q = 0; q < m.nq; ++q) {
                if (!sOk[q]) continue;
                double G[3];
                hermite_G(m.herm_q + kHermiteTable * static_cast<size_t>(q), b, h, G);
                const double* k = sK + 20 * q;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    ga[i] = fma(k[0], k[11 + 3 * i] * G[0] + k[12 + 3 * i] * G[1] + k[13 + 3 * i] * G[2], ga[i]);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (!isfinite(ga[i])) st |= ST_NONFINITE_OUT;
                per_elem[192 * static_cast<size_t>(e) + 3 * b + i] = ga[i];
            }
        }
    }
    if (blocks) {
        for (int pr = tid; pr < 2080; pr += blockDim.x) {
            int a, b;
            hermite_pair(pr, a, b);
            double Hb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int q = 0; q < m.nq; ++q) {
                if (!sOk[q]) continue;
                const double* tq = m.herm_q + kHermiteTable * static_cast<size_t>(q);
                double Ga[3], Gb[3];
                hermite_G(tq, a, h, Ga);
                hermite_G(tq, b, h, Gb);
                const double* k = sK + 20 * q;
                const double w = k[0], p = k[1];
                double ha[3], hb[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    ha[i] = k[2 + 3 * i] * Ga[0] + k[3 + 3 * i] * Ga[1] + k[4 + 3 * i] * Ga[2];
                    hb[i] = k[2 + 3 * i] * Gb[0] + k[3 + 3 * i] * Gb[1] + k[4 + 3 * i] * Gb[2];
                }
                const double dn = Ga[0] * Gb[0] + Ga[1] * Gb[1] + Ga[2] * Gb[2];
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double v = lam * ha[i] * hb[c] - p * hb[i] * ha[c];
                        if (i == c) v += mu * dn;
                        Hb[3 * i + c] = fma(w, v, Hb[3 * i + c]);
                    }
            }
            if (a == b) {
                Hb[3] = Hb[1];
                Hb[6] = Hb[2];
                Hb[7] = Hb[5];
            }
            R* o = blocks + kHermiteRecord * static_cast<size_t>(e) + 9 * pr;
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                if (!isfinite(Hb[t])) st |= ST_NONFINITE_OUT;
                o[t] = static_cast<R>(Hb[t]);
            }
        }
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((tid & 31) == 0 && st) atomicOr(status, st);
}


// ---------------------------------------------------------------------------
// Projected Hessian of tricubic Hermite hexes: V max(L, 0) V^T of each flagged element's 192 x 192
// Hessian (mesh_energy.cpp:16-27, there Eigen's SelfAdjointEigenSolver). One CTA per element:
// the lower triangle, packed, in shared memory is reduced to tridiagonal form by Householder
// reflections (Golub & Van Loan, Matrix Computations, 8.3.1), the reflections are accumulated
// into Q (column-major, in the CTA's global scratch), and the implicit QL iteration with
// Wilkinson shifts (Golub & Van Loan 8.3.3, in the form of the EISPACK tql2 routine) diagonalises
// the tridiagonal matrix, one thread generating each sweep's plane rotations and every thread
// applying them to its row of Q. The projection is then H - sum_{L_m < 0} L_m v_m v_m^T (or the
// sum over the positive eigenpairs when they are fewer), written back as the element's blocks.
// ---------------------------------------------------------------------------
constexpr int kHermN = 192;
constexpr int kHermPacked = kHermN * (kHermN + 1) / 2;
constexpr int kHermPsdThreads = 256;
constexpr int kHermQlSweeps = 60; // per eigenvalue, far above the few the iteration takes
constexpr size_t kHermPsdSmem = sizeof(double) * (kHermPacked + 6 * kHermN + 32);

__device__ __forceinline__ int hpk(int r, int c) { return r * (r + 1) / 2 + c; } // r >= c
__device__ __forceinline__ double hsym(const double* Ap, int r, int c) { return r >= c ? Ap[hpk(r, c)] : Ap[hpk(c, r)]; }

// Block-wide sum (every thread receives it); red holds 32 doubles.
__device__ __forceinline__ double herm_sum(double v, double* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    return t;
}

template <typename R>
__global__ void __launch_bounds__(kHermPsdThreads) hermite_psd_kernel(int T, double* in, R* out,
                                                                      const int* __restrict__ flags,
                                                                      double* __restrict__ qbuf, unsigned* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* Ap = reinterpret_cast<double*>(smem_raw); // packed lower triangle
    double* d = Ap + kHermPacked;                     // diagonal, then eigenvalues
    double* ev = d + kHermN;                          // off-diagonal
    double* beta = ev + kHermN;                       // reflector coefficients
    double* vp = beta + kHermN;                       // p, then w, of the current reflection
    double* rc = vp + kHermN;                         // a sweep's rotations: c, s (2 per index)
    double* red = rc + 2 * kHermN;
    __shared__ int s_hi, s_count, s_bad;
    const int tid = threadIdx.x, bd = blockDim.x;
    constexpr int n = kHermN;
    double* Q = qbuf + static_cast<size_t>(blockIdx.x) * n * n; // Q(r, c) at c n + r
    unsigned st = 0;
    for (int e = blockIdx.x; e < T; e += gridDim.x) {
        const double* rec = in + kHermiteRecord * static_cast<size_t>(e);
        R* o = out + kHermiteRecord * static_cast<size_t>(e);
        if (!flags[e]) { // semi-definite at every point: its own projection
            if (static_cast<const void*>(o) != static_cast<const void*>(rec))
                for (int t = tid; t < kHermiteRecord; t += bd) o[t] = static_cast<R>(rec[t]);
            continue;
        }
        // The element matrix: block (a, b), a <= b, entry (i, c) is H(3a + i, 3b + c).
        for (int t = tid; t < kHermiteRecord; t += bd) {
            const int pr = t / 9, ic = t - 9 * (t / 9);
            int a, b;
            hermite_pair(pr, a, b);
            const int r = 3 * a + ic / 3, c = 3 * b + ic % 3;
            if (r >= c) Ap[hpk(r, c)] = rec[t];
            else if (a != b) Ap[hpk(c, r)] = rec[t];
        }
        __syncthreads();
        // Householder tridiagonalisation: column k's reflection P = I - beta v v^T maps
        // A[k+1:, k] to (alpha, 0, ...); v is kept in place of the column below the subdiagonal.
        for (int k = 0; k < n - 2; ++k) {
            const int m = n - k - 1;
            double x2 = 0;
            for (int j = tid + 1; j < m; j += bd) {
                const double x = Ap[hpk(k + 1 + j, k)];
                x2 = fma(x, x, x2);
            }
            x2 = herm_sum(x2, red);
            const double x0 = Ap[hpk(k + 1, k)];
            if (x2 == 0.0) { // already tridiagonal in this column
                if (tid == 0) {
                    beta[k] = 0.0;
                    ev[k] = x0;
                }
                __syncthreads();
                continue;
            }
            const double alpha = -copysign(sqrt(fma(x0, x0, x2)), x0);
            const double v0 = x0 - alpha, bk = 1.0 / (alpha * (alpha - x0)); // 2 / v^T v
            __syncthreads();
            if (tid == 0) {
                Ap[hpk(k + 1, k)] = v0;
                beta[k] = bk;
                ev[k] = alpha;
            }
            __syncthreads();
            // p = beta A22 v (row i of the trailing block), then K = beta / 2 p^T v, w = p - K v.
            double pv = 0;
            for (int i = tid; i < m; i += bd) {
                double acc = 0;
                for (int j = 0; j < m; ++j) acc = fma(hsym(Ap, k + 1 + i, k + 1 + j), Ap[hpk(k + 1 + j, k)], acc);
                const double p = bk * acc;
                vp[i] = p;
                pv = fma(p, Ap[hpk(k + 1 + i, k)], pv);
            }
            const double K = 0.5 * bk * herm_sum(pv, red);
            for (int i = tid; i < m; i += bd) vp[i] = fma(-K, Ap[hpk(k + 1 + i, k)], vp[i]);
            __syncthreads();
            // A22 -= v w^T + w v^T on the lower triangle (rows paired for balance).
            for (int t = tid; t < m; t += bd) {
                const int i = t;
                const double vi = Ap[hpk(k + 1 + i, k)], wi = vp[i];
                for (int j = 0; j <= i; ++j) {
                    const double vj = Ap[hpk(k + 1 + j, k)], wj = vp[j];
                    Ap[hpk(k + 1 + i, k + 1 + j)] -= fma(vi, wj, wi * vj);
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < n; i += bd) d[i] = Ap[hpk(i, i)];
        if (tid == 0) {
            ev[n - 2] = Ap[hpk(n - 1, n - 2)];
            beta[n - 2] = 0.0;
            ev[n - 1] = 0.0;
        }
        // Q = P_0 P_1 ... P_{n-3}, accumulated from the last reflection (Q = I to begin with).
        for (int t = tid; t < n * n; t += bd) Q[t] = (t % n == t / n) ? 1.0 : 0.0;
        __syncthreads();
        for (int k = n - 3; k >= 0; --k) {
            const double bk = beta[k];
            if (bk == 0.0) continue;
            const int m = n - k - 1;
            // Columns c of Q with c > k: Q[k+1:, c] -= bk v (v^T Q[k+1:, c]); a warp per column.
            const int warp = tid >> 5, lane = tid & 31;
            for (int c = k + 1 + warp; c < n; c += bd >> 5) {
                double* qc = Q + static_cast<size_t>(c) * n + k + 1;
                double acc = 0;
                for (int j = lane; j < m; j += 32) acc = fma(Ap[hpk(k + 1 + j, k)], qc[j], acc);
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
                const double f = bk * acc;
                for (int j = lane; j < m; j += 32) qc[j] = fma(-f, Ap[hpk(k + 1 + j, k)], qc[j]);
            }
            __syncthreads();
        }
        // Implicit QL with Wilkinson shifts on (d, ev); rotations applied to the rows of Q. An
        // off-diagonal entry is negligible below eps times the tridiagonal matrix's norm bound
        // max |d_i| + |e_i| (as tql2 tests): the element's rigid-body modes are exact zero
        // eigenvalues, next to which a test relative to the neighbouring diagonal entries alone
        // never deflates.
        if (tid == 0) s_bad = 0;
        __syncthreads();
        double tnorm = 0.0;
        if (tid == 0)
            for (int i = 0; i < n; ++i) tnorm = fmax(tnorm, fabs(d[i]) + fabs(ev[i]));
        for (int l = 0; l < n; ++l) {
            for (int iter = 0;; ++iter) {
                if (tid == 0) {
                    int m = l;
                    for (; m < n - 1; ++m)
                        if (fabs(ev[m]) <= 2.220446049250313e-16 * tnorm) break;
                    s_hi = m;
                    s_count = 0;
                    if (m != l) {
                        if (iter >= kHermQlSweeps) {
                            s_bad = 1;
                            s_hi = l;
                        } else {
                            double g = (d[l + 1] - d[l]) / (2.0 * ev[l]);
                            double r = hypot(g, 1.0);
                            g = d[m] - d[l] + ev[l] / (g + copysign(r, g));
                            double sn = 1.0, cs = 1.0, p = 0.0;
                            int i = m - 1;
                            bool split = false;
                            for (; i >= l; --i) {
                                const double f = sn * ev[i], b = cs * ev[i];
                                r = hypot(f, g);
                                ev[i + 1] = r;
                                if (r == 0.0) {
                                    d[i + 1] -= p;
                                    ev[m] = 0.0;
                                    split = true;
                                    break;
                                }
                                sn = f / r;
                                cs = g / r;
                                g = d[i + 1] - p;
                                r = (d[i] - g) * sn + 2.0 * cs * b;
                                p = sn * r;
                                d[i + 1] = g + p;
                                g = cs * r - b;
                                rc[2 * i] = cs;
                                rc[2 * i + 1] = sn;
                                ++s_count;
                            }
                            if (!split) {
                                d[l] -= p;
                                ev[l] = g;
                                ev[m] = 0.0;
                            }
                        }
                    }
                }
                __syncthreads();
                const int m = s_hi, cnt = s_count;
                // Every thread holds the sweep's bounds before thread 0 may write the next ones
                // (after a converged l it goes straight on to l + 1).
                __syncthreads();
                if (m == l) break;
                // Apply rotations i = m-1 .. m-cnt to row r of Q: columns i and i+1.
                for (int r = tid; r < n; r += bd) {
                    double hi = Q[static_cast<size_t>(m) * n + r];
                    for (int i = m - 1; i >= m - cnt; --i) {
                        const double cs = rc[2 * i], sn = rc[2 * i + 1];
                        const double lo = Q[static_cast<size_t>(i) * n + r];
                        Q[static_cast<size_t>(i + 1) * n + r] = fma(sn, lo, cs * hi);
                        hi = fma(cs, lo, -sn * hi);
                    }
                    Q[static_cast<size_t>(m - cnt) * n + r] = hi;
                }
                __syncthreads();
            }
        }
        if (s_bad) st |= ST_NONFINITE_OUT;
        // Reconstruction from the fewer of the negative and positive eigenpairs, staged in the
        // (now free) shared matrix 96 vectors at a time.
        int nneg = 0;
        for (int i = 0; i < n; ++i) nneg += d[i] < 0.0;
        const bool from_neg = nneg <= n / 2;
        constexpr int kStage = 96;
        // Each thread keeps its entries' partial sums in the FP64 record itself (`in` is scratch:
        // it is read and rewritten by the same thread, entry by entry).
        double* acc_rec = in + kHermiteRecord * static_cast<size_t>(e);
        for (int base = 0; base < n; base += kStage) {
            // Stage eigenvectors base .. base + kStage - 1 that take part, scaled by their eigenvalue.
            __syncthreads();
            for (int t = tid; t < kStage * n; t += bd) {
                const int mm = base + t / n, r = t % n;
                double v = 0.0;
                if (mm < n) {
                    const double lm = d[mm];
                    const bool use = from_neg ? lm < 0.0 : lm > 0.0;
                    v = use ? Q[static_cast<size_t>(mm) * n + r] : 0.0;
                }
                Ap[t] = v;
            }
            __syncthreads();
            for (int t = tid; t < kHermiteRecord; t += bd) {
                const int pr = t / 9, ic = t - 9 * (t / 9);
                int a, b;
                hermite_pair(pr, a, b);
                int r = 3 * a + ic / 3, c = 3 * b + ic % 3;
                if (a == b && r > c) { // diagonal blocks: the lower entry mirrors the upper one
                    const int tmp = r;
                    r = c;
                    c = tmp;
                }
                double sum = 0.0;
                for (int k2 = 0; k2 < kStage && base + k2 < n; ++k2)
                    sum = fma(d[base + k2] * Ap[k2 * n + r], Ap[k2 * n + c], sum);
                // The element pass stores diagonal blocks bitwise symmetric, so entry t itself holds
                // the mirrored value.
                const double prev = base == 0 ? (from_neg ? acc_rec[t] : 0.0) : acc_rec[t];
                acc_rec[t] = from_neg ? prev - sum : prev + sum;
            }
        }
        __syncthreads();
        for (int t = tid; t < kHermiteRecord; t += bd) {
            const double v = acc_rec[t];
            if (!isfinite(v)) st |= ST_NONFINITE_OUT;
            o[t] = static_cast<R>(v);
        }
        __syncthreads();
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((tid & 31) == 0 && st) atomicOr(status, st);
}

// Force-response parameter VJP of Hermite hexes (the hex pass's, over the 64 nodes): per element
//   d/dlambda = sum_q w_q log J_q (F_q^-T : grad w_q),   d/dmu = sum_q w_q ((F_q - F_q^-T) : grad w_q),
// grad w = sum_b w_b G_b^T on the weight's physical DOFs. One thread per element; FP64.
__global__ void __launch_bounds__(128) hermite_force_vjp_kernel(const DevMesh m, const double* __restrict__ u,
                                                                const double* __restrict__ w, double* out,
                                                                unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned st = 0;
    if (e < m.T) {
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        const double h[3] = {m.herm_h[3 * static_cast<size_t>(e)], m.herm_h[3 * static_cast<size_t>(e) + 1],
                             m.herm_h[3 * static_cast<size_t>(e) + 2]};
        double dl = 0, dm = 0;
        for (int q = 0; q < m.nq; ++q) {
            const double* tq = m.herm_q + kHermiteTable * static_cast<size_t>(q);
            double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Gw[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int b = 0; b < 64; ++b) {
                double G[3];
                hermite_G(tq, b, h, G);
                const size_t base = 24 * static_cast<size_t>(__ldg(cell + (b >> 3))) + 3 * (b & 7);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double uu = __ldg(u + base + i), ww = __ldg(w + base + i);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        F[3 * i + d] = fma(uu, G[d], F[3 * i + d]);
                        Gw[3 * i + d] = fma(ww, G[d], Gw[3 * i + d]);
                    }
                }
            }
            double C[9];
            C[0] = F[4] * F[8] - F[5] * F[7];
            C[1] = F[5] * F[6] - F[3] * F[8];
            C[2] = F[3] * F[7] - F[4] * F[6];
            C[3] = F[2] * F[7] - F[1] * F[8];
            C[4] = F[0] * F[8] - F[2] * F[6];
            C[5] = F[1] * F[6] - F[0] * F[7];
            C[6] = F[1] * F[5] - F[2] * F[4];
            C[7] = F[2] * F[3] - F[0] * F[5];
            C[8] = F[0] * F[4] - F[1] * F[3];
            const double detF = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
            if (!(detF > 0) || !isfinite(detF)) {
                st |= isfinite(detF) ? ST_BAD_DET : ST_NONFINITE_F;
                continue;
            }
            double hf = 0, ff = 0;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                hf = fma(C[k] / detF, Gw[k], hf);
                ff = fma(F[k], Gw[k], ff);
            }
            const double wq = __ldg(tq + 192) * h[0] * h[1] * h[2];
            dl = fma(wq * log(detF), hf, dl);
            dm = fma(wq, ff - hf, dm);
        }
        if (!isfinite(dl) || !isfinite(dm)) st |= ST_NONFINITE_OUT;
        out[2 * static_cast<size_t>(e)] = dl;
        out[2 * static_cast<size_t>(e) + 1] = dm;
    }
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
}

// Feasible step of a Hermite hex mesh: F and dF at every point, the positive-determinant step,
// minimum per block (as hex_feasible_kernel).
__global__ void __launch_bounds__(256) hermite_feasible_kernel(const DevMesh m, const double* __restrict__ u,
                                                               const double* __restrict__ du, double* block_min,
                                                               unsigned* status) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double alpha = 1.0;
    unsigned st = 0;
    if (e < m.T) {
        const int32_t* cell = m.hex_cells + 8 * static_cast<size_t>(e);
        const double h[3] = {m.herm_h[3 * static_cast<size_t>(e)], m.herm_h[3 * static_cast<size_t>(e) + 1],
                             m.herm_h[3 * static_cast<size_t>(e) + 2]};
        for (int q = 0; q < m.nq && st == 0; ++q) {
            const double* tq = m.herm_q + kHermiteTable * static_cast<size_t>(q);
            double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, dF[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            bool ok = true;
            for (int b = 0; b < 64; ++b) {
                double G[3];
                hermite_G(tq, b, h, G);
                const size_t base = 24 * static_cast<size_t>(__ldg(cell + (b >> 3))) + 3 * (b & 7);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const double uu = u[base + i], dd = du[base + i];
                    ok = ok && isfinite(uu) && isfinite(dd);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        F[3 * i + d] = fma(uu, G[d], F[3 * i + d]);
                        dF[3 * i + d] = fma(dd, G[d], dF[3 * i + d]);
                    }
                }
            }
            if (!ok) {
                st |= ST_BAD_INPUT;
                break;
            }
            alpha = fmin(alpha, positive_det_step(F, dF, st));
        }
    }
    __shared__ double sm[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) alpha = fmin(alpha, __shfl_xor_sync(0xffffffffu, alpha, off));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = alpha;
    st = __reduce_or_sync(0xffffffffu, st);
    if ((threadIdx.x & 31) == 0 && st) atomicOr(status, st);
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = sm[0];
        for (int w = 1; w < (blockDim.x >> 5); ++w) v = fmin(v, sm[w]);
        block_min[blockIdx.x] = v;
    }
}

// Lame parameters of every element record (FP64 and FP32 copies).
__global__ void set_theta_kernel(double* rec64, float* rec32, const double* __restrict__ theta, int per_element, int T) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    const double lam = per_element ? theta[2 * static_cast<size_t>(e)] : theta[0];
    const double mu = per_element ? theta[2 * static_cast<size_t>(e) + 1] : theta[1];
    rec64[12 * static_cast<size_t>(e) + 10] = lam;
    rec64[12 * static_cast<size_t>(e) + 11] = mu;
    rec32[12 * static_cast<size_t>(e) + 10] = static_cast<float>(lam);
    rec32[12 * static_cast<size_t>(e) + 11] = static_cast<float>(mu);
}

// The Hessian-writing tet cluster kernel in the launch variant a.cl_variant.
template <typename R, bool WG> void launch_tet_variant(const DevMesh& m, const EvalArgs& a, cudaStream_t s) {
    switch (a.cl_variant) {
    case 1: launch_tet_cluster<R, WG, true, tc_minb<R>(1), tc_unroll(1)>(m, a, s); break;
    case 2: launch_tet_cluster<R, WG, true, tc_minb<R>(2), tc_unroll(2)>(m, a, s); break;
    default: launch_tet_cluster<R, WG, true>(m, a, s); break;
    }
}

// Launches the element pass; returns the number of per-unit energies it wrote to cluster_energy.
// Energy, gradient and the Exact Hessian come from the tet cluster kernel; the projected Hessian
// is gathered from the per-element clamped blocks by the block gather.
template <typename R> int launch_eval_t(const DevMesh& m, int hessian, const EvalArgs& a, cudaStream_t s) {
    const bool wg = a.grad != nullptr;
    const int wh = a.hess == nullptr ? 0 : (hessian == LPG_HESSIAN_EXACT ? 1 : 2);
    const int units = m.tc_ncl;
    if (wh == 2) {
        // Projected: energy (and gradient) from the element pass, the Hessian gathered from the
        // per-element clamped blocks; the optional events bracket both kernels.
        EvalArgs ea = a;
        ea.ev_end = nullptr;
        ea.hess = nullptr;
        if (wg)
            launch_tet_cluster<R, true, false>(m, ea, s);
        else
            launch_tet_cluster<R, false, false>(m, ea, s);
        launch_block_gather<R>(m, a, s);
        if (a.ev_end) LPG_CUDA(cudaEventRecord(a.ev_end, s));
    } else if (wg && wh == 1) {
        launch_tet_variant<R, true>(m, a, s);
    } else if (!wg && wh == 1) {
        launch_tet_variant<R, false>(m, a, s);
    } else if (wg) {
        launch_tet_cluster<R, true, false>(m, a, s);
    } else {
        launch_tet_cluster<R, false, false>(m, a, s);
    }
    if (wg && m.num_unused > 0)
        zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(a.grad, m.unused_rows, m.num_unused);
    return units;
}

} // namespace

size_t assembly_smem_bytes(const DevMesh& m) {
    const size_t gather = block_gather_bytes(m);
    if (m.K != 4) return gather;
    return std::max(gather, std::max(tc_smem_bytes<double>(), tc_smem_bytes<float>()));
}

void launch_eval(const DevMesh& m, int precision, int hessian, const EvalArgs& a, cudaStream_t s) {
    const int units = precision == LPG_PRECISION_F64 ? launch_eval_t<double>(m, hessian, a, s)
                                                      : launch_eval_t<float>(m, hessian, a, s);
    // Per-unit energies -> partials (stored after the units) -> total.
    sum_partial_kernel<<<kSumBlocks, 256, 0, s>>>(a.cluster_energy, units, a.cluster_energy + units);
    sum_final_kernel<<<1, 256, 0, s>>>(a.cluster_energy + units, kSumBlocks, a.energy);
    LPG_CUDA(cudaGetLastError());
}

void launch_rest_vjp(const DevMesh& m, const double* u, const double* w, double* per_elem, double sign, double* out,
                     unsigned* status, cudaStream_t s) {
    if (m.T > 0) {
        rest_vjp_kernel<<<(m.T + 127) / 128, 128, 0, s>>>(m, u, w, per_elem, status);
        vertex_gather_kernel<4><<<std::min(m.ncl, 148 * 8), 128, 0, s>>>(m, per_elem, sign, out);
    }
    if (m.num_unused > 0) zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(out, m.unused_rows, m.num_unused);
    LPG_CUDA(cudaGetLastError());
}

void launch_set_theta(const DevMesh& m, const double* theta, int per_element, cudaStream_t s) {
    if (m.T > 0) set_theta_kernel<<<(m.T + 255) / 256, 256, 0, s>>>(m.rec64, m.rec32, theta, per_element, m.T);
    LPG_CUDA(cudaGetLastError());
}

size_t project_bytes(const DevMesh& m, int precision) {
    return static_cast<size_t>(m.T) * kProjRecord * (precision == LPG_PRECISION_F64 ? sizeof(double) : sizeof(float));
}

namespace {
template <typename R, int MINB>
void launch_clamp_t(R* proj, const int* list, const unsigned* count, int max_count, cudaStream_t s) {
    const size_t clamp_sm = sizeof(R) == 8 ? sizeof(R) * kClampVStride * kProjThreads : 0;
    thread_local LaunchCache cache; // one wave of this variant
    const int clamp_grid = resident_grid(clamp_kernel<R, MINB>, kProjThreads, clamp_sm, cache);
    const int blocks = (max_count + kProjThreads - 1) / kProjThreads;
    if (blocks > 0) clamp_kernel<R, MINB><<<std::min(clamp_grid, blocks), kProjThreads, clamp_sm, s>>>(proj, list, count);
}
template <typename R>
void launch_clamp_v(R* proj, const int* list, const unsigned* count, int max_count, int variant, cudaStream_t s) {
    if (variant == 1)
        launch_clamp_t<R, clamp_minb<R>(1)>(proj, list, count, max_count, s);
    else
        launch_clamp_t<R, clamp_minb<R>(0)>(proj, list, count, max_count, s);
}

template <typename R, class Src>
void launch_project_t(const DevMesh& m, const Src& src, R* proj, unsigned* status, cudaStream_t s, const int* emesh,
                      const int* mesh_exact, int* list, unsigned* count, int clamp_variant) {
    const size_t sm = sizeof(R) * kProjStride * kProjThreads;
    thread_local LaunchCache cache;
    resident_grid(project_kernel<R, Src>, kProjThreads, sm, cache);
    const int blocks = (m.T + kProjThreads - 1) / kProjThreads;
    LPG_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned), s));
    project_kernel<R, Src><<<blocks, kProjThreads, sm, s>>>(m, src, proj, status, emesh, mesh_exact, list, count);
    launch_clamp_v<R>(proj, list, count, m.T, clamp_variant, s);
}
} // namespace

void launch_project(const DevMesh& m, int precision, int hessian, const double* u, void* proj, unsigned* status,
                    cudaStream_t s, int* list, unsigned* count, const int* emesh, const int* mesh_exact,
                    int clamp_variant) {
    if (hessian != LPG_HESSIAN_PROJECTED) fail(LPG_EINVAL, "projected Hessian kind not available");
    if (m.T == 0) return;
    const NhTangent src{u};
    if (precision == LPG_PRECISION_F64)
        launch_project_t<double>(m, src, static_cast<double*>(proj), status, s, emesh, mesh_exact, list, count,
                                 clamp_variant);
    else
        launch_project_t<float>(m, src, static_cast<float*>(proj), status, s, emesh, mesh_exact, list, count,
                                clamp_variant);
    LPG_CUDA(cudaGetLastError());
}

void launch_clamp(int precision, void* proj, const int* list, const unsigned* count, int max_count, int clamp_variant,
                  cudaStream_t s) {
    if (precision == LPG_PRECISION_F64)
        launch_clamp_v<double>(static_cast<double*>(proj), list, count, max_count, clamp_variant, s);
    else
        launch_clamp_v<float>(static_cast<float*>(proj), list, count, max_count, clamp_variant, s);
    LPG_CUDA(cudaGetLastError());
}

void launch_clamp_sample(int precision, void* proj, int* list, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (precision == LPG_PRECISION_F64)
        clamp_sample_kernel<double><<<(n + 255) / 256, 256, 0, s>>>(static_cast<double*>(proj), list, n);
    else
        clamp_sample_kernel<float><<<(n + 255) / 256, 256, 0, s>>>(static_cast<float*>(proj), list, n);
    LPG_CUDA(cudaGetLastError());
}

int feasible_blocks(const DevMesh& m) { return (m.T + 255) / 256; }

void launch_feasible(const DevMesh& m, const double* u, const double* du, double* block_min, int nblocks,
                     double* alpha, unsigned* status, cudaStream_t s, double* per_elem, const int* emesh,
                     const int* mstate) {
    if (m.K != 4 && per_elem) fail(LPG_EINVAL, "per-element feasible steps are available for tet meshes only");
    if (m.K == 8) {
        launch_hex_feasible(m, u, du, block_min, nblocks, alpha, status, s);
        return;
    }
    if (m.K == 64) {
        if (nblocks > 0) hermite_feasible_kernel<<<nblocks, 256, 0, s>>>(m, u, du, block_min, status);
        min_kernel<<<1, 1024, 0, s>>>(block_min, nblocks, alpha);
        LPG_CUDA(cudaGetLastError());
        return;
    }
    if (nblocks > 0) feasible_kernel<<<nblocks, 256, 0, s>>>(m, u, du, block_min, status, per_elem, emesh, mstate);
    min_kernel<<<1, 1024, 0, s>>>(block_min, nblocks, alpha);
    LPG_CUDA(cudaGetLastError());
}

void launch_force_vjp(const DevMesh& m, const double* u, const double* w, double* out, unsigned* status,
                      cudaStream_t s) {
    if (m.T > 0 && m.K == 8)
        hex_force_vjp_kernel<<<(m.T + 127) / 128, 128, 0, s>>>(m, u, w, out, status);
    else if (m.T > 0 && m.K == 64)
        hermite_force_vjp_kernel<<<(m.T + 127) / 128, 128, 0, s>>>(m, u, w, out, status);
    else if (m.T > 0)
        force_vjp_kernel<<<(m.T + 255) / 256, 256, 0, s>>>(m, u, w, out, status);
    LPG_CUDA(cudaGetLastError());
}

void launch_fp_vjp(const DevMesh& m, const double* u, const double* w, double* out, unsigned* status, cudaStream_t s) {
    if (m.T > 0) fp_vjp_kernel<<<(m.T + 127) / 128, 128, 0, s>>>(m, u, w, out, status);
    LPG_CUDA(cudaGetLastError());
}

void launch_sum_cols9(const double* per_elem, int T, double* partial, int nblocks, double* out9, cudaStream_t s) {
    if (nblocks > 0) sum_cols_partial<9><<<nblocks, 256, 0, s>>>(per_elem, T, partial);
    sum_cols_final<9><<<1, 32, 0, s>>>(partial, nblocks, out9);
    LPG_CUDA(cudaGetLastError());
}

void launch_set_geometry(const DevMesh& m, const double* geo, cudaStream_t s) {
    if (m.T > 0) set_geometry_kernel<<<(m.T + 255) / 256, 256, 0, s>>>(m, geo);
    LPG_CUDA(cudaGetLastError());
}

void launch_sum_pairs(const double* per_elem, int T, double* partial, int nblocks, double* out2, cudaStream_t s) {
    if (nblocks > 0) sum_pairs_partial<<<nblocks, 256, 0, s>>>(per_elem, T, partial);
    sum_pairs_final<<<1, 32, 0, s>>>(partial, nblocks, out2);
    LPG_CUDA(cudaGetLastError());
}

void launch_deformation_gradients(const DevMesh& m, const double* u, double* F, unsigned* status, cudaStream_t s) {
    if (m.T > 0) deformation_gradient_kernel<<<(m.T + 255) / 256, 256, 0, s>>>(m, u, F, status);
    LPG_CUDA(cudaGetLastError());
}

void launch_material_eval(const DevMesh& m, int precision, int hessian, const double* W, const double* P,
                          const double* A, double* elemE, double* per_elem, void* proj, int* list, unsigned* count,
                          int clamp_variant, const EvalArgs& a, cudaStream_t s) {
    if (m.T > 0) {
        material_pieces_kernel<<<(m.T + 255) / 256, 256, 0, s>>>(m, W, P, elemE, a.grad ? per_elem : nullptr, a.status);
        if (a.grad) vertex_gather_kernel<4><<<std::min(m.ncl, 148 * 8), 128, 0, s>>>(m, per_elem, 1.0, a.grad);
    }
    if (a.grad && m.num_unused > 0)
        zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(a.grad, m.unused_rows, m.num_unused);
    // Energy: the per-element energies summed in a fixed order.
    sum_partial_kernel<<<kSumBlocks, 256, 0, s>>>(elemE, m.T, a.cluster_energy);
    sum_final_kernel<<<1, 256, 0, s>>>(a.cluster_energy, kSumBlocks, a.energy);
    if (a.hess && m.T > 0) {
        const MatTangent src{A, hessian == LPG_HESSIAN_EXACT};
        EvalArgs ga = a;
        ga.proj = proj;
        if (precision == LPG_PRECISION_F64) {
            launch_project_t<double>(m, src, static_cast<double*>(proj), a.status, s, nullptr, nullptr, list, count,
                                     clamp_variant);
            launch_block_gather<double>(m, ga, s);
        } else {
            launch_project_t<float>(m, src, static_cast<float*>(proj), a.status, s, nullptr, nullptr, list, count,
                                    clamp_variant);
            launch_block_gather<float>(m, ga, s);
        }
    }
    LPG_CUDA(cudaGetLastError());
}

void launch_hex_deformation_gradients(const DevMesh& m, const double* u, double* F, unsigned* status, cudaStream_t s) {
    const size_t points = static_cast<size_t>(m.T) * m.nq;
    if (points > 0) hex_deformation_gradient_kernel<<<static_cast<int>((points + 127) / 128), 128, 0, s>>>(m, u, F, status);
    LPG_CUDA(cudaGetLastError());
}

void launch_hex_material_eval(const DevMesh& m, int precision, int hessian, const double* W, const double* P,
                              const double* A, double* elemE, double* per_elem, void* blocks, int* flags,
                              const EvalArgs& a, cudaStream_t s) {
    const bool projected = hessian == LPG_HESSIAN_PROJECTED;
    if (m.T > 0) {
        const size_t threads = 36 * static_cast<size_t>(m.T);
        const int grid = static_cast<int>((threads + 127) / 128);
        double* per_grad = a.grad ? per_elem : nullptr;
        if (a.hess && projected) {
            double* records = static_cast<double*>(blocks);
            hex_material_kernel<double><<<grid, 128, 0, s>>>(m, W, P, A, elemE, per_grad, records, a.status);
            LPG_CUDA(cudaMemsetAsync(flags, 0, static_cast<size_t>(m.T) * sizeof(int), s));
            const size_t points = static_cast<size_t>(m.T) * m.nq;
            hex_material_tangent_test_kernel<<<static_cast<int>((points + 127) / 128), 128, 0, s>>>(m, A, flags);
            const int pgrid = (m.T + kHexPsdWarps - 1) / kHexPsdWarps;
            if (precision == LPG_PRECISION_F64) {
                hex_psd_kernel<double><<<pgrid, 32 * kHexPsdWarps, 0, s>>>(m.T, records, records, flags, a.status);
            } else {
                float* out = reinterpret_cast<float*>(records + kHexRecord * static_cast<size_t>(m.T));
                hex_psd_kernel<float><<<pgrid, 32 * kHexPsdWarps, 0, s>>>(m.T, records, out, flags, a.status);
                blocks = out;
            }
        } else if (precision == LPG_PRECISION_F64 || !a.hess) {
            hex_material_kernel<double><<<grid, 128, 0, s>>>(m, W, P, A, elemE, per_grad,
                                                             a.hess ? static_cast<double*>(blocks) : nullptr, a.status);
        } else {
            hex_material_kernel<float><<<grid, 128, 0, s>>>(m, W, P, A, elemE, per_grad, static_cast<float*>(blocks),
                                                            a.status);
        }
        if (a.grad) vertex_gather_kernel<8><<<std::min(m.ncl, 148 * 8), 128, 0, s>>>(m, per_elem, 1.0, a.grad);
        if (a.hess) {
            EvalArgs ga = a;
            ga.proj = blocks;
            if (precision == LPG_PRECISION_F64)
                launch_block_gather<double, 8>(m, ga, s);
            else
                launch_block_gather<float, 8>(m, ga, s);
        }
    }
    if (a.grad && m.num_unused > 0)
        zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(a.grad, m.unused_rows, m.num_unused);
    sum_partial_kernel<<<kSumBlocks, 256, 0, s>>>(elemE, m.T, a.cluster_energy);
    sum_final_kernel<<<1, 256, 0, s>>>(a.cluster_energy, kSumBlocks, a.energy);
    LPG_CUDA(cudaGetLastError());
}

size_t hermite_blocks_bytes(const DevMesh& m, int precision, bool projected) {
    const size_t records = kHermiteRecord * static_cast<size_t>(m.T);
    if (precision == LPG_PRECISION_F64) return records * sizeof(double);
    return records * (projected ? sizeof(double) + sizeof(float) : sizeof(float));
}

int hermite_psd_grid(const DevMesh& m) {
    int dev = 0, sms = 0;
    LPG_CUDA(cudaGetDevice(&dev));
    LPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return std::max(1, std::min(m.T, sms));
}

void launch_hermite_eval(const DevMesh& m, int precision, bool projected, const double* u, double* elemE,
                         double* per_elem, void* blocks, int* flags, double* qbuf, const EvalArgs& a, cudaStream_t s) {
    if (m.T > 0) {
        if (a.ev_begin) LPG_CUDA(cudaEventRecord(a.ev_begin, s));
        double* per_grad = a.grad ? per_elem : nullptr;
        if (a.hess && projected) {
            // FP64 element Hessians with the per-point pre-test, then the clamp of the flagged
            // elements into the precision's records.
            double* records = static_cast<double*>(blocks);
            hermite_element_kernel<double><<<m.T, kHermiteThreads, 0, s>>>(m, u, elemE, per_grad, records, a.status,
                                                                            flags);
            const int grid = hermite_psd_grid(m);
            if (precision == LPG_PRECISION_F64) {
                thread_local LaunchCache cache;
                resident_grid(hermite_psd_kernel<double>, kHermPsdThreads, kHermPsdSmem, cache);
                hermite_psd_kernel<double><<<grid, kHermPsdThreads, kHermPsdSmem, s>>>(m.T, records, records, flags,
                                                                                      qbuf, a.status);
            } else {
                float* out = reinterpret_cast<float*>(records + kHermiteRecord * static_cast<size_t>(m.T));
                thread_local LaunchCache cache;
                resident_grid(hermite_psd_kernel<float>, kHermPsdThreads, kHermPsdSmem, cache);
                hermite_psd_kernel<float><<<grid, kHermPsdThreads, kHermPsdSmem, s>>>(m.T, records, out, flags, qbuf,
                                                                                     a.status);
                blocks = out;
            }
        } else if (precision == LPG_PRECISION_F64 || !a.hess)
            hermite_element_kernel<double><<<m.T, kHermiteThreads, 0, s>>>(
                m, u, elemE, per_grad, a.hess ? static_cast<double*>(blocks) : nullptr, a.status);
        else
            hermite_element_kernel<float><<<m.T, kHermiteThreads, 0, s>>>(m, u, elemE, per_grad,
                                                                          static_cast<float*>(blocks), a.status);
        if (a.grad) vertex_gather_kernel<64><<<std::min(m.ncl, 148 * 8), 128, 0, s>>>(m, per_elem, 1.0, a.grad);
        if (a.hess) {
            EvalArgs ga = a;
            ga.proj = blocks;
            if (precision == LPG_PRECISION_F64)
                launch_block_gather<double, 64>(m, ga, s);
            else
                launch_block_gather<float, 64>(m, ga, s);
        }
        if (a.ev_end) LPG_CUDA(cudaEventRecord(a.ev_end, s));
    }
    if (a.grad && m.num_unused > 0)
        zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(a.grad, m.unused_rows, m.num_unused);
    sum_partial_kernel<<<kSumBlocks, 256, 0, s>>>(elemE, m.T, a.cluster_energy);
    sum_final_kernel<<<1, 256, 0, s>>>(a.cluster_energy, kSumBlocks, a.energy);
    LPG_CUDA(cudaGetLastError());
}

size_t hex_blocks_bytes(const DevMesh& m, int precision, bool projected) {
    const size_t records = kHexRecord * static_cast<size_t>(m.T);
    if (precision == LPG_PRECISION_F64) return records * sizeof(double);
    return records * (projected ? sizeof(double) + sizeof(float) : sizeof(float));
}

void launch_hex_eval(const DevMesh& m, int precision, bool projected, const double* u, double* elemE,
                     double* per_elem, void* blocks, int* flags, const EvalArgs& a, cudaStream_t s) {
    if (m.T > 0) {
        const size_t threads = 36 * static_cast<size_t>(m.T);
        const int grid = static_cast<int>((threads + 127) / 128);
        if (a.ev_begin) LPG_CUDA(cudaEventRecord(a.ev_begin, s));
        double* per_grad = a.grad ? per_elem : nullptr;
        if (a.hess && projected) {
            // FP64 element Hessians, projected into the precision's records.
            double* records = static_cast<double*>(blocks);
            hex_element_kernel<double><<<grid, 128, 0, s>>>(m, u, elemE, per_grad, records, a.status);
            LPG_CUDA(cudaMemsetAsync(flags, 0, static_cast<size_t>(m.T) * sizeof(int), s));
            const size_t points = static_cast<size_t>(m.T) * m.nq;
            hex_tangent_test_kernel<<<static_cast<int>((points + 127) / 128), 128, 0, s>>>(m, u, flags);
            const int pgrid = (m.T + kHexPsdWarps - 1) / kHexPsdWarps;
            if (precision == LPG_PRECISION_F64) {
                hex_psd_kernel<double><<<pgrid, 32 * kHexPsdWarps, 0, s>>>(m.T, records, records, flags, a.status);
            } else {
                float* out = reinterpret_cast<float*>(records + kHexRecord * static_cast<size_t>(m.T));
                hex_psd_kernel<float><<<pgrid, 32 * kHexPsdWarps, 0, s>>>(m.T, records, out, flags, a.status);
                blocks = out;
            }
        } else if (precision == LPG_PRECISION_F64) {
            hex_element_kernel<double><<<grid, 128, 0, s>>>(m, u, elemE, per_grad,
                                                           a.hess ? static_cast<double*>(blocks) : nullptr, a.status);
        } else {
            hex_element_kernel<float><<<grid, 128, 0, s>>>(m, u, elemE, per_grad,
                                                          a.hess ? static_cast<float*>(blocks) : nullptr, a.status);
        }
        if (a.grad) vertex_gather_kernel<8><<<std::min(m.ncl, 148 * 8), 128, 0, s>>>(m, per_elem, 1.0, a.grad);
        if (a.hess) {
            EvalArgs ga = a;
            ga.proj = blocks;
            if (precision == LPG_PRECISION_F64)
                launch_block_gather<double, 8>(m, ga, s);
            else
                launch_block_gather<float, 8>(m, ga, s);
        }
        if (a.ev_end) LPG_CUDA(cudaEventRecord(a.ev_end, s));
    }
    if (a.grad && m.num_unused > 0)
        zero_rows_kernel<<<(m.num_unused + 255) / 256, 256, 0, s>>>(a.grad, m.unused_rows, m.num_unused);
    sum_partial_kernel<<<kSumBlocks, 256, 0, s>>>(elemE, m.T, a.cluster_energy);
    sum_final_kernel<<<1, 256, 0, s>>>(a.cluster_energy, kSumBlocks, a.energy);
    LPG_CUDA(cudaGetLastError());
}

int hex_feasible_blocks(const DevMesh& m) { return (m.T + 255) / 256; }

void launch_hex_feasible(const DevMesh& m, const double* u, const double* du, double* block_min, int nblocks,
                         double* alpha, unsigned* status, cudaStream_t s) {
    if (nblocks > 0) hex_feasible_kernel<<<nblocks, 256, 0, s>>>(m, u, du, block_min, status);
    min_kernel<<<1, 1024, 0, s>>>(block_min, nblocks, alpha);
    LPG_CUDA(cudaGetLastError());
}

} // namespace lpg
