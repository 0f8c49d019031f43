// lpg_solve.cu -- block-CSR SpMV, block-Jacobi PCG, the GPU Newton loop and the adjoint.
//
// Newton follows newton_solve (src/core/solver/newton.cpp:112-183): evaluate E, g and the
// Hessian, stop on the gradient rule, solve the free block for a descent direction
// (shifting the diagonal like LinearSystem::descent_direction, :55-72, when the solve fails
// to give one), then backtrack from the feasible step (:92-108). The reference factors
// the free block directly; here the free block is the 3x3 block-CSR Hessian with fixed DOFs
// masked, solved by block-Jacobi preconditioned CG to a forcing tolerance. All reductions
// are two-stage with a fixed block -> index map, so results do not depend on scheduling.

#include <algorithm>
#include <array>
#include <cmath>
#include <type_traits>
#include <cstring>
#include <string>
#include <vector>

#include "lpg_solver.h"

namespace lpg {
namespace {

constexpr int kThreads = 256;
constexpr int kSpmvGroup = 16;
constexpr double kEps = 2.220446049250313e-16;

int red_blocks(size_t n) { return static_cast<int>(std::max<size_t>(1, std::min<size_t>(512, (n + 4095) / 4096))); }

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (blockDim.x >> 5); ++w) r += sh[w];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double block_max(double v, double* sh) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    __syncthreads();
    return r;
}

// One-block deterministic reduction of k interleaved sums over nb partials: thread t sums
// indices t, t + 1024, ... in order, then a fixed shuffle tree and a fixed warp order.
template <int K>
__device__ __forceinline__ void reduce_partials(const double* __restrict__ part, int nb, double* out) {
    __shared__ double sh[K][32];
    double v[K];
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
#pragma unroll
        for (int c = 0; c < K; ++c) v[c] += part[K * static_cast<size_t>(i) + c];
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], off);
        if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = v[c];
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int c = 0; c < K; ++c) {
            double r = 0;
            for (int w = 0; w < (blockDim.x >> 5); ++w) r += sh[c][w];
            out[c] = r;
        }
}

// Masked statistics of a (and a.b): part[4 * block] = {sum m a b, sum m a^2, max m |a|, sum m b^2}.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kThreads) stats_partial(const TA* __restrict__ a, const TB* __restrict__ b,
                                                          const double* __restrict__ mask, size_t n, double* part) {
    __shared__ double sh[kThreads / 32];
    const size_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const size_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    double s_ab = 0, s_aa = 0, m_a = 0, s_bb = 0;
    for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double m = mask ? mask[i] : 1.0;
        const double ai = m * static_cast<double>(a[i]);
        const double bi = b ? m * static_cast<double>(b[i]) : 0.0;
        s_ab += ai * bi;
        s_aa += ai * ai;
        s_bb += bi * bi;
        m_a = fmax(m_a, fabs(ai));
    }
    s_ab = block_sum(s_ab, sh);
    s_aa = block_sum(s_aa, sh);
    s_bb = block_sum(s_bb, sh);
    m_a = block_max(m_a, sh);
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x] = s_ab;
        part[4 * blockIdx.x + 1] = s_aa;
        part[4 * blockIdx.x + 2] = m_a;
        part[4 * blockIdx.x + 3] = s_bb;
    }
}
__global__ void __launch_bounds__(1024) stats_final(const double* __restrict__ part, int nb, double* out) {
    double s0 = 0, s1 = 0, s3 = 0, m = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        s0 += part[4 * i];
        s1 += part[4 * i + 1];
        m = fmax(m, part[4 * i + 2]);
        s3 += part[4 * i + 3];
    }
    __shared__ double q[4][32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, off);
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        s3 += __shfl_xor_sync(0xffffffffu, s3, off);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    }
    if ((threadIdx.x & 31) == 0) {
        q[0][threadIdx.x >> 5] = s0;
        q[1][threadIdx.x >> 5] = s1;
        q[2][threadIdx.x >> 5] = m;
        q[3][threadIdx.x >> 5] = s3;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0, d = 0;
        for (int w = 0; w < (blockDim.x >> 5); ++w) {
            a += q[0][w];
            b += q[1][w];
            c = fmax(c, q[2][w]);
            d += q[3][w];
        }
        out[0] = a;
        out[1] = b;
        out[2] = c;
        out[3] = d;
    }
}

// y = mask (K x) on the 3x3 block-CSR matrix; a group of 16 lanes walks one block row's
// values contiguously (coalesced), then reduces its three sums with shuffles. With DOT,
// part[block] = sum_i x_i y_i.
template <typename TK, typename TV, typename TO, bool DOT>
__global__ void __launch_bounds__(kThreads) bsr_spmv(const int* __restrict__ row_ptr, const int* __restrict__ col_idx,
                                                     const TK* __restrict__ val, const TV* __restrict__ x,
                                                     const double* __restrict__ mask, TO* __restrict__ y, int V,
                                                     double* part, const int* done) {
    __shared__ double sh[kThreads / 32];
    if (done && *done) return;
    using A = typename std::conditional<(sizeof(TK) == 4 && sizeof(TV) == 4), float, double>::type;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = gid / kSpmvGroup;
    const int lg = threadIdx.x & (kSpmvGroup - 1);
    A a0 = 0, a1 = 0, a2 = 0;
    if (v < V) {
        const int s0 = row_ptr[v], nb = row_ptr[v + 1] - s0;
        const TK* rv = val + 9 * static_cast<size_t>(s0);
        for (int j = lg; j < 9 * nb; j += kSpmvGroup) {
            const int s = j / 9;
            const int r = j - 9 * s;
            const int i = r / 3;
            const int k = r - 3 * i;
            const int c = __ldg(col_idx + s0 + s);
            const A t = static_cast<A>(rv[j]) * static_cast<A>(x[3 * static_cast<size_t>(c) + k]);
            if (i == 0) a0 += t;
            else if (i == 1) a1 += t;
            else a2 += t;
        }
    }
#pragma unroll
    for (int off = kSpmvGroup / 2; off > 0; off >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, off);
        a1 += __shfl_xor_sync(0xffffffffu, a1, off);
        a2 += __shfl_xor_sync(0xffffffffu, a2, off);
    }
    double d = 0;
    if (v < V && lg == 0) {
        const size_t o = 3 * static_cast<size_t>(v);
        const A y0 = mask ? static_cast<A>(mask[o]) * a0 : a0;
        const A y1 = mask ? static_cast<A>(mask[o + 1]) * a1 : a1;
        const A y2 = mask ? static_cast<A>(mask[o + 2]) * a2 : a2;
        y[o] = static_cast<TO>(y0);
        y[o + 1] = static_cast<TO>(y1);
        y[o + 2] = static_cast<TO>(y2);
        if (DOT)
            d = static_cast<double>(x[o]) * static_cast<double>(y0) + static_cast<double>(x[o + 1]) * static_cast<double>(y1) +
                static_cast<double>(x[o + 2]) * static_cast<double>(y2);
    }
    if (DOT) {
        d = block_sum(d, sh);
        if (threadIdx.x == 0) part[blockIdx.x] = d;
    }
}

// Inverse of each masked 3x3 diagonal block (identity on fixed components; identity for a
// vertex without a diagonal block), the block-Jacobi preconditioner.
template <typename TK, typename R>
__global__ void __launch_bounds__(kThreads) block_jacobi(const TK* __restrict__ val, const int* __restrict__ diag_slot,
                                                         const double* __restrict__ mask, R* __restrict__ dinv, int V) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double b[9];
    const int s = diag_slot[v];
    const double m[3] = {mask[3 * static_cast<size_t>(v)], mask[3 * static_cast<size_t>(v) + 1],
                         mask[3 * static_cast<size_t>(v) + 2]};
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            const double kv = s >= 0 ? static_cast<double>(val[9 * static_cast<size_t>(s) + 3 * i + k]) : (i == k ? 1.0 : 0.0);
            b[3 * i + k] = m[i] * m[k] * kv + (i == k ? 1.0 - m[i] : 0.0);
        }
    const double det = b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                       b[2] * (b[3] * b[7] - b[4] * b[6]);
    double r[9];
    if (det != 0 && isfinite(det)) {
        const double id = 1.0 / det;
        r[0] = (b[4] * b[8] - b[5] * b[7]) * id;
        r[1] = (b[2] * b[7] - b[1] * b[8]) * id;
        r[2] = (b[1] * b[5] - b[2] * b[4]) * id;
        r[3] = (b[5] * b[6] - b[3] * b[8]) * id;
        r[4] = (b[0] * b[8] - b[2] * b[6]) * id;
        r[5] = (b[2] * b[3] - b[0] * b[5]) * id;
        r[6] = (b[3] * b[7] - b[4] * b[6]) * id;
        r[7] = (b[1] * b[6] - b[0] * b[7]) * id;
        r[8] = (b[0] * b[4] - b[1] * b[3]) * id;
    } else {
        // Singular block: fall back to the inverse diagonal (scalar Jacobi), 1 where zero.
        for (int t = 0; t < 9; ++t) r[t] = 0;
        for (int i = 0; i < 3; ++i) r[4 * i] = (b[4 * i] != 0 && isfinite(b[4 * i])) ? 1.0 / b[4 * i] : 1.0;
    }
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) dinv[9 * static_cast<size_t>(v) + 3 * i + k] = static_cast<R>(m[i] * m[k] * r[3 * i + k]);
}

struct PcgState {
    double rz, pAp, alpha, beta, rr, bb, tol2;
    int done, breakdown, iters, max_iters;
};

__device__ __forceinline__ void apply_dinv(const float* D, const float* r, float* z) {
    for (int i = 0; i < 3; ++i) z[i] = D[3 * i] * r[0] + D[3 * i + 1] * r[1] + D[3 * i + 2] * r[2];
}
__device__ __forceinline__ void apply_dinv(const double* D, const double* r, double* z) {
    for (int i = 0; i < 3; ++i) z[i] = D[3 * i] * r[0] + D[3 * i + 1] * r[1] + D[3 * i + 2] * r[2];
}

// r = mask b, x = 0, z = M^-1 r, p = z; part = {r.z, r.r} per block.
template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_init(const R* __restrict__ b, const double* __restrict__ mask,
                                                     const R* __restrict__ dinv, R* x, R* r, R* z, R* p, int V,
                                                     double* part) {
    __shared__ double sh[kThreads / 32];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double rz = 0, rr = 0;
    if (v < V) {
        R rv[3], zv[3];
        for (int i = 0; i < 3; ++i) rv[i] = static_cast<R>(mask[3 * static_cast<size_t>(v) + i]) * b[3 * static_cast<size_t>(v) + i];
        apply_dinv(dinv + 9 * static_cast<size_t>(v), rv, zv);
        for (int i = 0; i < 3; ++i) {
            const size_t o = 3 * static_cast<size_t>(v) + i;
            x[o] = 0;
            r[o] = rv[i];
            z[o] = zv[i];
            p[o] = zv[i];
            rz += static_cast<double>(rv[i]) * zv[i];
            rr += static_cast<double>(rv[i]) * rv[i];
        }
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void __launch_bounds__(1024) pcg_start(PcgState* st, const double* part, int nb, double tol, int max_iters) {
    __shared__ double res[2];
    reduce_partials<2>(part, nb, res);
    if (threadIdx.x != 0) return;
    const double rz = res[0], rr = res[1];
    st->rz = rz;
    st->rr = rr;
    st->bb = rr;
    st->tol2 = tol * tol * rr;
    st->iters = 0;
    st->breakdown = 0;
    st->max_iters = max_iters;
    st->done = (rr == 0.0 || max_iters <= 0) ? 1 : 0;
}

__global__ void __launch_bounds__(1024) pcg_alpha(PcgState* st, const double* part, int nb) {
    if (st->done) return;
    __shared__ double res[1];
    reduce_partials<1>(part, nb, res);
    if (threadIdx.x != 0) return;
    const double pap = res[0];
    st->pAp = pap;
    if (!(pap > 0.0) || !isfinite(pap)) {
        st->breakdown = 1;
        st->done = 1;
        return;
    }
    st->alpha = st->rz / pap;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_update(const PcgState* st, const double* __restrict__ mask,
                                                       const R* __restrict__ dinv, R* x, R* r, R* z,
                                                       const R* __restrict__ p, const R* __restrict__ Ap, int V,
                                                       double* part) {
    __shared__ double sh[kThreads / 32];
    if (st->done) return;
    const R alpha = static_cast<R>(st->alpha);
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double rz = 0, rr = 0;
    if (v < V) {
        R rv[3], zv[3];
        for (int i = 0; i < 3; ++i) {
            const size_t o = 3 * static_cast<size_t>(v) + i;
            x[o] += alpha * p[o];
            rv[i] = r[o] - alpha * Ap[o];
            r[o] = rv[i];
        }
        apply_dinv(dinv + 9 * static_cast<size_t>(v), rv, zv);
        for (int i = 0; i < 3; ++i) {
            const size_t o = 3 * static_cast<size_t>(v) + i;
            z[o] = zv[i];
            rz += static_cast<double>(rv[i]) * zv[i];
            rr += static_cast<double>(rv[i]) * rv[i];
        }
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void __launch_bounds__(1024) pcg_beta(PcgState* st, const double* part, int nb) {
    if (st->done) return;
    __shared__ double res[2];
    reduce_partials<2>(part, nb, res);
    if (threadIdx.x != 0) return;
    const double rz = res[0], rr = res[1];
    st->iters += 1;
    st->rr = rr;
    if (rr <= st->tol2 || st->iters >= st->max_iters || !isfinite(rr)) {
        st->done = 1;
        return;
    }
    st->beta = rz / st->rz;
    st->rz = rz;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_pupdate(const PcgState* st, const R* __restrict__ z, R* p, size_t n) {
    if (st->done) return;
    const R beta = static_cast<R>(st->beta);
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
}

template <typename A, typename B> __global__ void convert_kernel(const A* __restrict__ a, B* __restrict__ b, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) b[i] = static_cast<B>(a[i]);
}

// x64 += xR ; optional r64 = b - y (masked) is done by a separate kernel.
template <typename R>
__global__ void add_kernel(double* __restrict__ x64, const R* __restrict__ xr, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) x64[i] += static_cast<double>(xr[i]);
}
__global__ void residual_kernel(const double* __restrict__ b, const double* __restrict__ y,
                                const double* __restrict__ mask, double* __restrict__ r, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) r[i] = mask[i] * (b[i] - y[i]);
}
// g = g_el - f ; out = -g masked (the Newton right-hand side).
__global__ void load_gradient(double* __restrict__ g, const double* __restrict__ f, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n && f) g[i] -= f[i];
}
__global__ void neg_mask(const double* __restrict__ g, const double* __restrict__ mask, double* __restrict__ b, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) b[i] = -mask[i] * g[i];
}
__global__ void axpy_trial(const double* __restrict__ x, double alpha, const double* __restrict__ d,
                           double* __restrict__ t, size_t n, int* moved) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    int mv = 0;
    if (i < n) {
        t[i] = x[i] + alpha * d[i];
        mv = t[i] != x[i];
    }
    mv = __reduce_or_sync(0xffffffffu, mv);
    if ((threadIdx.x & 31) == 0 && mv) atomicOr(moved, 1);
}
__global__ void shift_diag(double* val64, float* val32, const int* __restrict__ diag_slot, int V, double shift) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int s = diag_slot[v];
    if (s < 0) return;
    for (int i = 0; i < 3; ++i) {
        if (val64) val64[9 * static_cast<size_t>(s) + 4 * i] += shift;
        if (val32) val32[9 * static_cast<size_t>(s) + 4 * i] += static_cast<float>(shift);
    }
}
__global__ void diag_absmax_partial(const double* val64, const float* val32, const int* __restrict__ diag_slot,
                                    const double* __restrict__ mask, int V, double* part) {
    __shared__ double sh[kThreads / 32];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0;
    if (v < V && diag_slot[v] >= 0) {
        const size_t s = diag_slot[v];
        for (int i = 0; i < 3; ++i)
            if (mask[3 * static_cast<size_t>(v) + i] != 0)
                m = fmax(m, fabs(val64 ? val64[9 * s + 4 * i] : static_cast<double>(val32[9 * s + 4 * i])));
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = m;
}
__global__ void max_final(const double* part, int nb, double* out) {
    if (threadIdx.x != 0) return;
    double m = 0;
    for (int i = 0; i < nb; ++i) m = fmax(m, part[i]);
    *out = m;
}

inline int grid(size_t n, int threads = kThreads) { return static_cast<int>((n + threads - 1) / threads); }

// ---------------------------------------------------------------------------
// Host-side helpers bound to one handle.
// ---------------------------------------------------------------------------
struct Solver {
    lpg_fem& h;
    cudaStream_t s;
    size_t n;
    int V;
    explicit Solver(lpg_fem& hh) : h(hh), s(hh.stream), n(3 * static_cast<size_t>(hh.dm.V)), V(hh.dm.V) {}

    // {sum m a b, sum m a^2, max m|a|, sum m b^2}
    template <typename TA, typename TB> std::array<double, 4> stats(const TA* a, const TB* b, const double* mask) {
        const int nb = red_blocks(n);
        double* part = h.s_part.as<double>(4 * 1024);
        double* out = h.s_scal.as<double>(64) + 32;
        stats_partial<TA, TB><<<nb, kThreads, 0, s>>>(a, b, mask, n, part);
        stats_final<<<1, 1024, 0, s>>>(part, nb, out);
        LPG_CUDA(cudaGetLastError());
        std::array<double, 4> r{};
        LPG_CUDA(cudaMemcpyAsync(r.data(), out, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
        LPG_CUDA(cudaStreamSynchronize(s));
        return r;
    }

    double energy_dot_f(const double* x, const double* f) {
        if (!f) return 0.0;
        return stats<double, double>(x, f, nullptr)[0];
    }

    // E(x) (FP64) with optional gradient g (FP64, load included); throws on bad status.
    double energy(const double* x, const double* f, double* g) {
        h.eval_async(x, g, LPG_HESSIAN_NONE, LPG_PRECISION_F64, LPG_LAYOUT_BSR, nullptr, nullptr);
        if (g && f) load_gradient<<<grid(n), kThreads, 0, s>>>(g, f, n);
        double e = 0;
        LPG_CUDA(cudaMemcpyAsync(&e, h.d_energy.ptr, sizeof e, cudaMemcpyDeviceToHost, s));
        raise_status(h.take_status());
        return e - energy_dot_f(x, f);
    }

    template <typename R>
    void spmv(const void* K, bool k64, const R* x, const double* mask, R* y, double* part, const int* done, bool dot) {
        const int blocks = grid(static_cast<size_t>(V) * kSpmvGroup);
        if (k64) {
            if (dot) bsr_spmv<double, R, R, true><<<blocks, kThreads, 0, s>>>(h.dm.row_ptr, h.dm.col_idx, static_cast<const double*>(K), x, mask, y, V, part, done);
            else bsr_spmv<double, R, R, false><<<blocks, kThreads, 0, s>>>(h.dm.row_ptr, h.dm.col_idx, static_cast<const double*>(K), x, mask, y, V, part, done);
        } else {
            if (dot) bsr_spmv<float, R, R, true><<<blocks, kThreads, 0, s>>>(h.dm.row_ptr, h.dm.col_idx, static_cast<const float*>(K), x, mask, y, V, part, done);
            else bsr_spmv<float, R, R, false><<<blocks, kThreads, 0, s>>>(h.dm.row_ptr, h.dm.col_idx, static_cast<const float*>(K), x, mask, y, V, part, done);
        }
        LPG_CUDA(cudaGetLastError());
    }

    struct PcgOut {
        int64_t iters = 0;
        bool breakdown = false;
        double rel = 0; // final ||b - K x|| / ||b|| in FP64
    };

    // Solves mask K x = mask b (FP64 b, x): inner PCG in precision R on matrix Kin (typed R),
    // FP64 residual refinement against Kres (FP64 values when res64, else Kin's values).
    template <typename R>
    PcgOut pcg(const void* Kin, const R* dinv, const void* Kres, bool res64, const double* mask, const double* b64,
               double* x64, double tol, int max_iters, int max_refine) {
        PcgOut out;
        R* x = h.s_xcg.as<R>(n);
        R* r = h.s_r.as<R>(n);
        R* z = h.s_z.as<R>(n);
        R* p = h.s_p.as<R>(n);
        R* Ap = h.s_ap.as<R>(n);
        R* bR = reinterpret_cast<R*>(h.s_trial.as<double>(n)); // scratch, reused
        double* r64 = h.s_r64.as<double>(n);
        double* y64 = h.s_b64.as<double>(n);
        const int spmv_blocks = grid(static_cast<size_t>(V) * kSpmvGroup);
        const int vb = grid(static_cast<size_t>(V));
        double* part = h.s_part.as<double>(std::max(4 * 1024, 2 * std::max(spmv_blocks, vb)));
        PcgState* st = reinterpret_cast<PcgState*>(h.s_scal.as<double>(64));
        LPG_CUDA(cudaMemsetAsync(x64, 0, n * sizeof(double), s));
        LPG_CUDA(cudaMemcpyAsync(r64, b64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        const double bnorm = std::sqrt(stats<double, double>(b64, nullptr, mask)[1]);
        if (bnorm == 0) return out;
        double rnorm = bnorm;
        for (int ref = 0; ref <= max_refine; ++ref) {
            const double inner_tol = std::min(0.5, std::max(tol * bnorm / rnorm, sizeof(R) == 4 ? 1e-6 : 1e-14));
            convert_kernel<double, R><<<grid(n), kThreads, 0, s>>>(r64, bR, n);
            pcg_init<R><<<vb, kThreads, 0, s>>>(bR, mask, dinv, x, r, z, p, V, part);
            pcg_start<<<1, 1024, 0, s>>>(st, part, vb, inner_tol, max_iters - static_cast<int>(out.iters));
            LPG_CUDA(cudaGetLastError());
            PcgState hs{};
            for (;;) {
                constexpr int kChunk = 16;
                for (int it = 0; it < kChunk; ++it) {
                    spmv<R>(Kin, sizeof(R) == 8 ? true : false, p, mask, Ap, part, &st->done, true);
                    pcg_alpha<<<1, 1024, 0, s>>>(st, part, spmv_blocks);
                    pcg_update<R><<<vb, kThreads, 0, s>>>(st, mask, dinv, x, r, z, p, Ap, V, part);
                    pcg_beta<<<1, 1024, 0, s>>>(st, part, vb);
                    pcg_pupdate<R><<<grid(n), kThreads, 0, s>>>(st, z, p, n);
                }
                LPG_CUDA(cudaGetLastError());
                LPG_CUDA(cudaMemcpyAsync(&hs, st, sizeof hs, cudaMemcpyDeviceToHost, s));
                LPG_CUDA(cudaStreamSynchronize(s));
                if (hs.done) break;
            }
            out.iters += hs.iters;
            if (hs.breakdown) {
                out.breakdown = true;
                // Negative curvature on the first step: keep the preconditioned residual direction.
                if (hs.iters == 0) LPG_CUDA(cudaMemcpyAsync(x, p, n * sizeof(R), cudaMemcpyDeviceToDevice, s));
            }
            add_kernel<R><<<grid(n), kThreads, 0, s>>>(x64, x, n);
            // FP64 residual r64 = mask (b - Kres x64).
            if (res64)
                bsr_spmv<double, double, double, false><<<spmv_blocks, kThreads, 0, s>>>(
                    h.dm.row_ptr, h.dm.col_idx, static_cast<const double*>(Kres), x64, mask, y64, V, nullptr, nullptr);
            else
                bsr_spmv<float, double, double, false><<<spmv_blocks, kThreads, 0, s>>>(
                    h.dm.row_ptr, h.dm.col_idx, static_cast<const float*>(Kres), x64, mask, y64, V, nullptr, nullptr);
            residual_kernel<<<grid(n), kThreads, 0, s>>>(b64, y64, mask, r64, n);
            LPG_CUDA(cudaGetLastError());
            rnorm = std::sqrt(stats<double, double>(r64, nullptr, mask)[1]);
            out.rel = rnorm / bnorm;
            if (out.breakdown || !(rnorm > tol * bnorm) || out.iters >= max_iters || !std::isfinite(rnorm)) break;
        }
        return out;
    }
};

void make_mask(lpg_fem& h, const int32_t* fixed, int nfixed, double* mask) {
    const int n = 3 * h.dm.V;
    std::vector<int32_t> f(fixed, fixed + std::max(nfixed, 0));
    std::sort(f.begin(), f.end());
    if (std::adjacent_find(f.begin(), f.end()) != f.end()) fail(LPG_EINVAL, "DofReduction fixed DOFs must be unique");
    if (!f.empty() && (f.front() < 0 || f.back() >= n)) fail(LPG_EINVAL, "DofReduction fixed DOFs must lie in [0, num_dofs)");
    std::vector<double> m(static_cast<size_t>(n), 1.0);
    for (int d : f) m[d] = 0.0;
    LPG_CUDA(cudaMemcpyAsync(mask, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    LPG_CUDA(cudaStreamSynchronize(h.stream));
}

const int* diag_slots(lpg_fem& h) { return h.dm.diag_slot; }

} // namespace

void newton_solve(lpg_fem& h, const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                  const lpg_newton_options& o, double* x_out, lpg_newton_result* res) {
    if (!(o.gradient_tolerance >= 0.0) || !std::isfinite(o.gradient_tolerance))
        fail(LPG_EINVAL, "newton_solve: gradient_tolerance must be set to a finite non-negative value");
    if (o.max_iterations < 0 || o.max_line_search_steps < 1)
        fail(LPG_EINVAL, "newton_solve: max_iterations must be >= 0 and max_line_search_steps >= 1");
    if (!(o.line_search_shrink > 0.0 && o.line_search_shrink < 1.0))
        fail(LPG_EINVAL, "newton_solve: line_search_shrink must lie in (0, 1)");
    if (o.hessian != LPG_HESSIAN_EXACT && o.hessian != LPG_HESSIAN_PROJECTED)
        fail(LPG_EINVAL, "newton_solve: invalid Hessian kind");
    if (o.precision != LPG_PRECISION_F64 && o.precision != LPG_PRECISION_MIXED)
        fail(LPG_EINVAL, "newton_solve: invalid precision");
    Solver S(h);
    const size_t n = S.n;
    const int V = S.V;
    cudaStream_t s = h.stream;
    double* mask = h.s_mask.as<double>(std::max<size_t>(n, 1));
    make_mask(h, fixed, nfixed, mask);
    const int* dslot = diag_slots(h);
    cudaEvent_t ev0, ev1;
    LPG_CUDA(cudaEventCreate(&ev0));
    LPG_CUDA(cudaEventCreate(&ev1));
    LPG_CUDA(cudaEventRecord(ev0, s));
    double* x = h.s_x.as<double>(std::max<size_t>(n, 1));
    double* g = h.s_g.as<double>(2 * std::max<size_t>(n, 1));
    double* d = h.s_d.as<double>(std::max<size_t>(n, 1));
    // s_f holds the line-search trial point and, after it, the load vector.
    double* trial = h.s_f.as<double>(2 * std::max<size_t>(n, 1));
    double* f = nullptr;
    const double* fsrc = f_ext ? h.stage_in(f_ext, io_mem, h.d_u2, n) : nullptr;
    if (fsrc) {
        f = trial + n;
        LPG_CUDA(cudaMemcpyAsync(f, fsrc, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    const double* x0d = h.stage_in(x0, io_mem, h.d_u, n);
    LPG_CUDA(cudaMemcpyAsync(x, x0d, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const bool f64 = o.precision == LPG_PRECISION_F64;
    const size_t hbytes = 9 * static_cast<size_t>(h.dm.nnzb) * (f64 ? 8 : 4);
    void* K = h.s_hess.ensure(std::max<size_t>(hbytes, 8));
    void* dinv = h.s_dinv.ensure(9 * static_cast<size_t>(std::max(V, 1)) * (f64 ? 8 : 4));
    double* rhs = h.s_g.as<double>(2 * std::max<size_t>(n, 1)) + std::max<size_t>(n, 1); // second half of s_g
    int* moved = reinterpret_cast<int*>(h.s_flag.as<int>(4));
    lpg_newton_result R{};
    int nfree = 0;
    {
        std::vector<int32_t> ff(fixed, fixed + std::max(nfixed, 0));
        nfree = static_cast<int>(n) - static_cast<int>(ff.size());
    }
    auto finish = [&](int status) {
        R.status = status;
        LPG_CUDA(cudaEventRecord(ev1, s));
        LPG_CUDA(cudaEventSynchronize(ev1));
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0, ev1);
        R.seconds = ms * 1e-3;
        if (io_mem == LPG_MEM_DEVICE)
            LPG_CUDA(cudaMemcpyAsync(x_out, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        else
            LPG_CUDA(cudaMemcpyAsync(x_out, x, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        LPG_CUDA(cudaStreamSynchronize(s));
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        if (res) *res = R;
    };
    if (nfree == 0) {
        R.energy = S.energy(x, f, nullptr);
        finish(0);
        return;
    }
    double gnorm0 = -1;
    for (int it = 0;; ++it) {
        // Energy and FP64 gradient (the Newton residual).
        double E;
        if (f64) {
            h.eval_async(x, g, o.hessian, LPG_PRECISION_F64, LPG_LAYOUT_BSR, K, nullptr);
            if (f) load_gradient<<<grid(n), kThreads, 0, s>>>(g, f, n);
            double e = 0;
            LPG_CUDA(cudaMemcpyAsync(&e, h.d_energy.ptr, sizeof e, cudaMemcpyDeviceToHost, s));
            raise_status(h.take_status());
            E = e - S.energy_dot_f(x, f);
        } else {
            E = S.energy(x, f, g);
        }
        const auto gs = S.stats<double, double>(g, nullptr, mask);
        const double g2 = std::sqrt(gs[1]), gmax = gs[2];
        if (gnorm0 < 0) gnorm0 = g2;
        R.energy = E;
        R.gradient_norm = o.stop_rule == 0 ? gmax : g2;
        R.gradient_norm0 = gnorm0;
        R.iterations = it;
        const bool converged = o.stop_rule == 0 ? gmax <= o.gradient_tolerance : g2 <= o.gradient_tolerance * gnorm0;
        if (converged) return finish(0);
        if (it == o.max_iterations) return finish(1);
        if (!f64) {
            h.eval_async(x, nullptr, o.hessian, LPG_PRECISION_MIXED, LPG_LAYOUT_BSR, K, nullptr);
            raise_status(h.take_status());
        }
        // Descent direction with diagonal shifts (newton.cpp:55-72).
        neg_mask<<<grid(n), kThreads, 0, s>>>(g, mask, rhs, n);
        double dscale = 1.0;
        {
            const int vb = grid(static_cast<size_t>(V));
            double* part = h.s_part.as<double>(std::max(4 * 1024, vb));
            double* outm = h.s_scal.as<double>(64) + 40;
            diag_absmax_partial<<<vb, kThreads, 0, s>>>(f64 ? static_cast<double*>(K) : nullptr,
                                                       f64 ? nullptr : static_cast<float*>(K), dslot, mask, V, part);
            max_final<<<1, 32, 0, s>>>(part, vb, outm);
            double m = 0;
            LPG_CUDA(cudaMemcpyAsync(&m, outm, sizeof m, cudaMemcpyDeviceToHost, s));
            LPG_CUDA(cudaStreamSynchronize(s));
            dscale = std::max(1.0, m);
        }
        double shift = 1e-8 * dscale;
        const double eta = std::min(o.cg_tolerance, std::sqrt(g2 / gnorm0));
        bool found = false;
        double gd = 0;
        for (int shifts = 0;; ++shifts) {
            Solver::PcgOut po;
            if (f64) {
                block_jacobi<double, double><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(
                    static_cast<double*>(K), dslot, mask, static_cast<double*>(dinv), V);
                po = S.pcg<double>(K, static_cast<double*>(dinv), K, true, mask, rhs, d, eta, o.cg_max_iterations, 0);
            } else {
                block_jacobi<float, float><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(
                    static_cast<float*>(K), dslot, mask, static_cast<float*>(dinv), V);
                po = S.pcg<float>(K, static_cast<float*>(dinv), K, false, mask, rhs, d, eta, o.cg_max_iterations, 3);
            }
            R.cg_iterations += po.iters;
            gd = S.stats<double, double>(g, d, mask)[0];
            if (gd < 0.0 && std::isfinite(gd)) {
                found = true;
                break;
            }
            if (shifts == 10) break;
            shift_diag<<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(f64 ? static_cast<double*>(K) : nullptr,
                                                                       f64 ? nullptr : static_cast<float*>(K), dslot, V, shift);
            shift *= 10.0;
        }
        if (!found) return finish(3);
        // Line search (newton.cpp:92-108) from the feasible step.
        const int nb = feasible_blocks(h.dm);
        double* bm = h.d_block.as<double>(std::max(nb, 1));
        double* al = h.d_alpha.as<double>(1);
        launch_feasible(h.dm, x, d, bm, nb, al, h.d_status.as<unsigned>(1), s);
        double alpha = 1;
        LPG_CUDA(cudaMemcpyAsync(&alpha, al, sizeof alpha, cudaMemcpyDeviceToHost, s));
        raise_status(h.take_status());
        bool accepted = false;
        for (int j = 0; j < o.max_line_search_steps; ++j) {
            LPG_CUDA(cudaMemsetAsync(moved, 0, sizeof(int), s));
            axpy_trial<<<grid(n), kThreads, 0, s>>>(x, alpha, d, trial, n, moved);
            int mv = 0;
            LPG_CUDA(cudaMemcpyAsync(&mv, moved, sizeof mv, cudaMemcpyDeviceToHost, s));
            LPG_CUDA(cudaStreamSynchronize(s));
            if (!mv) break;
            ++R.line_search_evaluations;
            const double Et = S.energy(trial, f, nullptr);
            const double noise = 16.0 * kEps * std::max(1.0, std::abs(E));
            const double armijo = o.accept_rule == 1 ? 1e-4 * alpha * gd : 0.0;
            if (Et <= E + armijo + noise) {
                accepted = true;
                break;
            }
            alpha *= o.line_search_shrink;
        }
        if (!accepted) return finish(2);
        LPG_CUDA(cudaMemcpyAsync(x, trial, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
}

void adjoint_theta(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                   int precision, double cg_tolerance, int per_element, double* dtheta, double* lambda_out) {
    if (precision != LPG_PRECISION_F64 && precision != LPG_PRECISION_MIXED) fail(LPG_EINVAL, "invalid precision");
    if (!(cg_tolerance > 0) || !std::isfinite(cg_tolerance)) fail(LPG_EINVAL, "adjoint: cg_tolerance must be positive");
    Solver S(h);
    const size_t n = S.n;
    const int V = S.V;
    const size_t T = static_cast<size_t>(h.dm.T);
    cudaStream_t s = h.stream;
    double* mask = h.s_mask.as<double>(std::max<size_t>(n, 1));
    make_mask(h, fixed, nfixed, mask);
    const int* dslot = diag_slots(h);
    const double* u = h.stage_in(u_star, io_mem, h.d_u, n);
    const double* w = h.stage_in(dLdu, io_mem, h.d_u2, n);
    double* lam = h.s_d.as<double>(std::max<size_t>(n, 1));
    LPG_CUDA(cudaMemsetAsync(lam, 0, n * sizeof(double), s));
    const auto ws = S.stats<double, double>(w, nullptr, mask);
    if (!std::isfinite(ws[1])) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: nonfinite sensitivity right-hand side");
    if (n > 0 && ws[1] > 0) {
        // Exact FP64 Hessian at u*: the residual matrix of the refinement (static_equilibrium_response.cpp:58).
        double* K64 = h.s_hess64.as<double>(std::max<size_t>(9 * static_cast<size_t>(h.dm.nnzb), 1));
        h.eval_async(u, nullptr, LPG_HESSIAN_EXACT, LPG_PRECISION_F64, LPG_LAYOUT_BSR, K64, nullptr);
        raise_status(h.take_status());
        double* rhs = h.s_g.as<double>(std::max<size_t>(n, 1));
        LPG_CUDA(cudaMemcpyAsync(rhs, w, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        Solver::PcgOut po;
        if (precision == LPG_PRECISION_F64) {
            double* dinv = h.s_dinv.as<double>(9 * static_cast<size_t>(std::max(V, 1)));
            block_jacobi<double, double><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(K64, dslot, mask, dinv, V);
            po = S.pcg<double>(K64, dinv, K64, true, mask, rhs, lam, cg_tolerance, 200000, 2);
        } else {
            float* K32 = h.s_hess.as<float>(std::max<size_t>(9 * static_cast<size_t>(h.dm.nnzb), 1));
            const size_t nv = 9 * static_cast<size_t>(h.dm.nnzb);
            if (nv) convert_kernel<double, float><<<grid(nv), kThreads, 0, s>>>(K64, K32, nv);
            float* dinv = h.s_dinv.as<float>(9 * static_cast<size_t>(std::max(V, 1)));
            block_jacobi<float, float><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(K32, dslot, mask, dinv, V);
            po = S.pcg<float>(K32, dinv, K64, true, mask, rhs, lam, cg_tolerance, 200000, 30);
        }
        if (po.breakdown) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: singular or indefinite equilibrium stiffness");
        // Residual check (static_equilibrium_response.cpp:61-68) in FP64 with the exact Hessian.
        const double bn = std::sqrt(ws[1]);
        if (!(po.rel * bn <= 1e-8 * (1.0 + bn))) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: inaccurate sensitivity solve");
    }
    // dtheta = -(dg/dtheta)^T lambda.
    double* pe = h.d_vjp.as<double>(std::max<size_t>(2 * T, 2));
    launch_force_vjp(h.dm, u, lam, pe, h.d_status.as<unsigned>(1), s);
    std::vector<double> host;
    if (per_element) {
        host.resize(2 * T);
        if (T) LPG_CUDA(cudaMemcpyAsync(host.data(), pe, 2 * T * sizeof(double), cudaMemcpyDeviceToHost, s));
    } else {
        const int nb = static_cast<int>(std::min<size_t>(1024, (T + 4095) / 4096));
        double* part = h.d_block.as<double>(std::max(2 * nb, 2));
        double* res = h.d_alpha.as<double>(2);
        launch_sum_pairs(pe, static_cast<int>(T), part, nb, res, s);
        host.resize(2);
        LPG_CUDA(cudaMemcpyAsync(host.data(), res, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    raise_status(h.take_status());
    for (double& v : host) v = -v;
    if (io_mem == LPG_MEM_DEVICE) {
        if (!host.empty()) LPG_CUDA(cudaMemcpyAsync(dtheta, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        if (lambda_out) LPG_CUDA(cudaMemcpyAsync(lambda_out, lam, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
        std::copy(host.begin(), host.end(), dtheta);
        if (lambda_out) LPG_CUDA(cudaMemcpyAsync(lambda_out, lam, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    LPG_CUDA(cudaStreamSynchronize(s));
}

} // namespace lpg
