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

struct PcgState {
    double rz, pAp, alpha, beta, rr, bb, tol2;
    int done, breakdown, iters, max_iters;
    unsigned count_a, count_b; // completion counters of the last-block reductions
};

// 4-wide vector access of padded per-vertex vectors (16-byte float4, two 16-byte double2).
__device__ __forceinline__ void ld4(const float* p, float v[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
// Coherent loads, for vectors the same kernel also writes.
__device__ __forceinline__ void ld4c(const float* p, float v[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
}
__device__ __forceinline__ void ld4c(const double* p, double v[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, float a, float b, float c) {
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, 0.f);
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
    reinterpret_cast<double2*>(p)[1] = make_double2(c, 0.0);
}
// Three components of vertex v of a vector with S (3 or 4) values per vertex.
template <int S, typename T> __device__ __forceinline__ void ld3(const T* p, size_t v, T out[3]) {
    if constexpr (S == 4) {
        T t[4];
        ld4(p + 4 * v, t);
        out[0] = t[0], out[1] = t[1], out[2] = t[2];
    } else {
        out[0] = p[3 * v], out[1] = p[3 * v + 1], out[2] = p[3 * v + 2];
    }
}
template <int S, typename T> __device__ __forceinline__ void st3(T* p, size_t v, T a, T b, T c) {
    if constexpr (S == 4) {
        st4(p + 4 * v, a, b, c);
    } else {
        p[3 * v] = a, p[3 * v + 1] = b, p[3 * v + 2] = c;
    }
}

// Entry t (row-major) of the diagonal block of vertex v in the sliced-ELL layout, or -1.
__device__ __forceinline__ int64_t diag_entry(const DevMesh& m, int v, int t) {
    const int k = m.diag_slot[v];
    if (k < 0) return -1;
    return static_cast<int64_t>(m.sell_base[v]) + 32 * static_cast<int64_t>(9 * (k - m.row_ptr[v]) + t);
}

// y = mask (K x) on the 3x3 block matrix in the sliced-ELL layout (SELL-32): one warp per
// chunk of 32 rows, one lane per row, block slot q of every lane read together, so each of the
// nine value loads and the column load of a slot is one contiguous 128-byte (FP32) run, and a
// lane's slots are independent (no cross-lane reduction). Vectors hold S values per vertex: 4
// for the padded PCG vectors (4th value zero, one 16-byte load per gathered vertex in FP32),
// 3 for plain FP64 vectors. With PCG the vector is z + beta p_old (beta from the state; each
// row writes it to p_new), and the block of the grid that finishes last reduces the partial
// p.Ap sums into alpha; otherwise, with DOT, part[block] = sum x.y. Both reductions use a
// fixed order.
// Resident blocks per SM the register allocation must allow (8 x 256 threads: 32 registers);
// more resident warps hide the gathers' latency better than the registers they cost.
#ifndef LPG_SPMV_MIN_BLOCKS
#define LPG_SPMV_MIN_BLOCKS 8
#endif
template <typename TK, typename TV, typename TO, bool PCG, bool DOT, int S>
__global__ void __launch_bounds__(kThreads, LPG_SPMV_MIN_BLOCKS) spmv_sell(const DevMesh m, const TK* __restrict__ val,
                                                      const TV* __restrict__ x, const TV* __restrict__ p_old,
                                                      const TV* __restrict__ mask, TO* __restrict__ y,
                                                      TV* __restrict__ p_new, PcgState* st, double* part) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    using A = typename std::conditional<(sizeof(TK) == 4 && sizeof(TV) == 4), float, double>::type;
    if (PCG && st->done) return;
    const TV beta = PCG ? static_cast<TV>(st->beta) : TV(0);
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    double dot = 0;
    for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < m.n_sell; c += nwarps) {
        const int row = __ldg(m.sell_row + 32 * static_cast<size_t>(c) + lane);
        const int s0 = __ldg(m.sell_ptr + c);
        const int width = (__ldg(m.sell_ptr + c + 1) - s0) >> 5;
        const int* cp = m.sell_col + s0 + lane;
        const TK* vp = val + 9 * static_cast<size_t>(s0) + lane;
        A a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 4
        for (int q = 0; q < width; ++q) {
            const size_t col = static_cast<size_t>(__ldg(cp + 32 * q));
            TV xz[3];
            ld3<S>(x, col, xz);
            if (PCG) {
                TV xp[3];
                ld3<S>(p_old, col, xp);
#pragma unroll
                for (int i = 0; i < 3; ++i) xz[i] = xz[i] + beta * xp[i];
            }
            const A xv[3] = {static_cast<A>(xz[0]), static_cast<A>(xz[1]), static_cast<A>(xz[2])};
            const TK* vq = vp + 288 * static_cast<size_t>(q);
            A kv[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) kv[e] = static_cast<A>(__ldg(vq + 32 * e));
            a0 += kv[0] * xv[0] + kv[1] * xv[1] + kv[2] * xv[2];
            a1 += kv[3] * xv[0] + kv[4] * xv[1] + kv[5] * xv[2];
            a2 += kv[6] * xv[0] + kv[7] * xv[1] + kv[8] * xv[2];
        }
        if (row >= 0) {
            const size_t o = static_cast<size_t>(row);
            TV mv[3];
            ld3<S>(mask, o, mv);
            const A yv[3] = {static_cast<A>(mv[0]) * a0, static_cast<A>(mv[1]) * a1, static_cast<A>(mv[2]) * a2};
            st3<S, TO>(y, o, static_cast<TO>(yv[0]), static_cast<TO>(yv[1]), static_cast<TO>(yv[2]));
            if (PCG) {
                TV xz[3], xp[3];
                ld3<S>(x, o, xz);
                ld3<S>(p_old, o, xp);
                TV pv[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    pv[i] = xz[i] + beta * xp[i];
                    dot += static_cast<double>(pv[i]) * static_cast<double>(yv[i]);
                }
                st3<S, TV>(p_new, o, pv[0], pv[1], pv[2]);
            } else if (DOT) {
                TV xz[3];
                ld3<S>(x, o, xz);
#pragma unroll
                for (int i = 0; i < 3; ++i) dot += static_cast<double>(xz[i]) * static_cast<double>(yv[i]);
            }
        }
    }
    if (!PCG && !DOT) return;
    dot = block_sum(dot, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = dot;
        // The last block to finish turns the partial sums into alpha (this thread wrote part).
        if (PCG) {
            __threadfence();
            last = atomicAdd(&st->count_a, 1u) == gridDim.x - 1;
        }
    }
    if (!PCG) return;
    __syncthreads();
    if (!last) return;
    double v = 0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) v += __ldcg(part + i);
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        st->count_a = 0;
        st->pAp = v;
        if (!(v > 0.0) || !isfinite(v)) {
            st->breakdown = 1;
            st->done = 1;
        } else {
            st->alpha = st->rz / v;
        }
    }
}

// Inverse of each masked 3x3 diagonal block (identity on fixed components; identity for a
// vertex without a diagonal block), the block-Jacobi preconditioner, stored as 3 padded rows
// of 4 per vertex.
template <typename TK, typename R>
__global__ void __launch_bounds__(kThreads) block_jacobi(const DevMesh m, const TK* __restrict__ val,
                                                         const double* __restrict__ mask, R* __restrict__ dinv, int V) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    double b[9];
    const double mk[3] = {mask[3 * static_cast<size_t>(v)], mask[3 * static_cast<size_t>(v) + 1],
                          mask[3 * static_cast<size_t>(v) + 2]};
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            const int64_t pos = diag_entry(m, v, 3 * i + k);
            const double kv = pos >= 0 ? static_cast<double>(val[pos]) : (i == k ? 1.0 : 0.0);
            b[3 * i + k] = mk[i] * mk[k] * kv + (i == k ? 1.0 - mk[i] : 0.0);
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
        st4(dinv + 12 * static_cast<size_t>(v) + 4 * i, static_cast<R>(mk[i] * mk[0] * r[3 * i]),
            static_cast<R>(mk[i] * mk[1] * r[3 * i + 1]), static_cast<R>(mk[i] * mk[2] * r[3 * i + 2]));
}

// z = D r with D the 3 padded rows of a vertex's preconditioner block.
template <typename R> __device__ __forceinline__ void apply_dinv(const R* D, const R* r, R* z) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R d[4];
        ld4(D + 4 * i, d);
        z[i] = d[0] * r[0] + d[1] * r[1] + d[2] * r[2];
    }
}

// b4 = mask b64 as padded R (4 per vertex, 4th zero).
template <typename R>
__global__ void pad_rhs(const double* __restrict__ b, const double* __restrict__ mask, R* __restrict__ b4, int V) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const size_t o = 3 * static_cast<size_t>(v);
    st4(b4 + 4 * static_cast<size_t>(v), static_cast<R>(mask[o] * b[o]), static_cast<R>(mask[o + 1] * b[o + 1]),
        static_cast<R>(mask[o + 2] * b[o + 2]));
}

// r = b, x = 0, z = M^-1 r, p_old = 0; part = {r.z, r.r} per block (grid-stride, fixed grid).
template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_init(const R* __restrict__ b, const R* __restrict__ dinv, R* x, R* r,
                                                     R* z, R* p_old, int V, double* part) {
    __shared__ double sh[kThreads / 32];
    double rz = 0, rr = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const size_t o = 4 * static_cast<size_t>(v);
        R rv[4], zv[3];
        ld4(b + o, rv);
        apply_dinv(dinv + 12 * static_cast<size_t>(v), rv, zv);
        st4(x + o, R(0), R(0), R(0));
        st4(r + o, rv[0], rv[1], rv[2]);
        st4(z + o, zv[0], zv[1], zv[2]);
        st4(p_old + o, R(0), R(0), R(0));
        for (int i = 0; i < 3; ++i) {
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
    st->beta = 0;
    st->tol2 = tol * tol * rr;
    st->iters = 0;
    st->breakdown = 0;
    st->max_iters = max_iters;
    st->count_a = 0;
    st->count_b = 0;
    st->done = (rr == 0.0 || max_iters <= 0) ? 1 : 0;
}

// x += alpha p, r -= alpha Ap, z = M^-1 r and the partial r.z, r.r; the last block to finish
// computes beta and the stopping test.
template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_update(PcgState* st, const R* __restrict__ dinv, R* x, R* r, R* z,
                                                       const R* __restrict__ p, const R* __restrict__ Ap, int V,
                                                       double* part) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    if (st->done) return;
    const R alpha = static_cast<R>(st->alpha);
    double rz = 0, rr = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const size_t o = 4 * static_cast<size_t>(v);
        R xv[4], pv[4], rv[4], av[4], zv[3];
        ld4c(x + o, xv);
        ld4(p + o, pv);
        ld4c(r + o, rv);
        ld4(Ap + o, av);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            xv[i] += alpha * pv[i];
            rv[i] = rv[i] - alpha * av[i];
        }
        apply_dinv(dinv + 12 * static_cast<size_t>(v), rv, zv);
        st4(x + o, xv[0], xv[1], xv[2]);
        st4(r + o, rv[0], rv[1], rv[2]);
        st4(z + o, zv[0], zv[1], zv[2]);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rz += static_cast<double>(rv[i]) * zv[i];
            rr += static_cast<double>(rv[i]) * rv[i];
        }
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
        __threadfence(); // this thread wrote the partials
        last = atomicAdd(&st->count_b, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        a += __ldcg(part + 2 * i);
        b += __ldcg(part + 2 * i + 1);
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    if (threadIdx.x == 0) {
        st->count_b = 0;
        st->iters += 1;
        st->rr = b;
        if (b <= st->tol2 || st->iters >= st->max_iters || !isfinite(b)) {
            st->done = 1;
        } else {
            st->beta = a / st->rz;
            st->rz = a;
        }
    }
}

template <typename A, typename B> __global__ void convert_kernel(const A* __restrict__ a, B* __restrict__ b, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) b[i] = static_cast<B>(a[i]);
}

// x64 += x (x padded, 4 per vertex).
template <typename R>
__global__ void add_kernel(double* __restrict__ x64, const R* __restrict__ xr, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) x64[i] += static_cast<double>(xr[4 * (i / 3) + i % 3]);
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
__global__ void shift_diag(const DevMesh m, double* val64, float* val32, double shift) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= m.V) return;
    for (int i = 0; i < 3; ++i) {
        const int64_t pos = diag_entry(m, v, 4 * i);
        if (pos < 0) return;
        if (val64) val64[pos] += shift;
        if (val32) val32[pos] += static_cast<float>(shift);
    }
}
__global__ void diag_absmax_partial(const DevMesh m, const double* val64, const float* val32,
                                    const double* __restrict__ mask, double* part) {
    __shared__ double sh[kThreads / 32];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    double mx = 0;
    if (v < m.V)
        for (int i = 0; i < 3; ++i) {
            const int64_t pos = diag_entry(m, v, 4 * i);
            if (pos >= 0 && mask[3 * static_cast<size_t>(v) + i] != 0)
                mx = fmax(mx, fabs(val64 ? val64[pos] : static_cast<double>(val32[pos])));
        }
    mx = block_max(mx, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = mx;
}
__global__ void max_final(const double* part, int nb, double* out) {
    if (threadIdx.x != 0) return;
    double m = 0;
    for (int i = 0; i < nb; ++i) m = fmax(m, part[i]);
    *out = m;
}

inline int grid(size_t n, int threads = kThreads) { return static_cast<int>((n + threads - 1) / threads); }

// Grid of at most `work` blocks that fits in one wave of the device (blocks resident per SM
// for this kernel x SM count), for the grid-stride kernels: a second partial wave would
// double their time.
template <typename Kern> int one_wave(Kern kernel, size_t work) {
    int dev = 0, sms = 0, per = 0;
    LPG_CUDA(cudaGetDevice(&dev));
    LPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    LPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kThreads, 0));
    const size_t wave = static_cast<size_t>(std::max(per, 1)) * static_cast<size_t>(std::max(sms, 1));
    return static_cast<int>(std::max<size_t>(1, std::min(work, wave)));
}

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

    // One warp per sliced-ELL chunk (8 per block). Not persistent: with about one chunk per
    // resident warp, a grid-stride loop would leave a fifth of the warps with two chunks and the
    // rest idle; later blocks instead start as earlier ones finish.
    template <typename Kern> int spmv_grid(Kern) const { return std::max(1, (h.dm.n_sell + 7) / 8); }
    template <typename Kern> int vec_grid(Kern k) const { return one_wave(k, grid(static_cast<size_t>(V))); }

    // y64 = mask (K x64) in FP64 with K stored as TK.
    void residual_spmv(const void* K, bool k64, const double* x64, const double* mask, double* y64) {
        if (k64)
            spmv_sell<double, double, double, false, false, 3>
                <<<spmv_grid(spmv_sell<double, double, double, false, false, 3>), kThreads, 0, s>>>(
                    h.dm, static_cast<const double*>(K), x64, nullptr, mask, y64, nullptr, nullptr, nullptr);
        else
            spmv_sell<float, double, double, false, false, 3>
                <<<spmv_grid(spmv_sell<float, double, double, false, false, 3>), kThreads, 0, s>>>(
                    h.dm, static_cast<const float*>(K), x64, nullptr, mask, y64, nullptr, nullptr, nullptr);
        LPG_CUDA(cudaGetLastError());
    }

    struct PcgOut {
        int64_t iters = 0;
        bool breakdown = false;
        double rel = 0; // final ||b - K x|| / ||b|| in FP64
    };

    // Enqueues `pairs` x 2 PCG iterations on stream gs (two launches per iteration; p_new and
    // p_old swap roles every iteration).
    template <typename R>
    void enqueue_iterations(cudaStream_t gs, const R* K, const R* dinv, const R* mask4, R* x, R* r, R* z, R* pA,
                            R* pB, R* Ap, PcgState* st, double* part, int pairs) {
        const int sg = spmv_grid(spmv_sell<R, R, R, true, false, 4>), ug = vec_grid(pcg_update<R>);
        for (int i = 0; i < pairs; ++i) {
            spmv_sell<R, R, R, true, false, 4><<<sg, kThreads, 0, gs>>>(h.dm, K, z, pA, mask4, Ap, pB, st, part);
            pcg_update<R><<<ug, kThreads, 0, gs>>>(st, dinv, x, r, z, pB, Ap, V, part);
            spmv_sell<R, R, R, true, false, 4><<<sg, kThreads, 0, gs>>>(h.dm, K, z, pB, mask4, Ap, pA, st, part);
            pcg_update<R><<<ug, kThreads, 0, gs>>>(st, dinv, x, r, z, pA, Ap, V, part);
        }
    }

    // Solves mask K x = mask b (FP64 b, x): inner PCG in precision R on Kin (values of type R),
    // FP64 residual refinement against Kres (FP64 values when res64, else Kin's values). The
    // iterations run as a replayed CUDA graph of 32 iterations; the host checks the device
    // state after each replay.
    template <typename R>
    PcgOut pcg(const void* Kin, const R* dinv, const void* Kres, bool res64, const double* mask, const double* b64,
               double* x64, double tol, int max_iters, int max_refine) {
        PcgOut out;
        // The PCG vectors are padded to 4 values per vertex (4th value zero).
        const size_t n4 = 4 * static_cast<size_t>(V);
        R* x = h.s_xcg.as<R>(n4);
        R* r = h.s_r.as<R>(n4);
        R* z = h.s_z.as<R>(n4);
        R* pA = h.s_p.as<R>(n4);
        R* pB = h.s_p2.as<R>(n4);
        R* Ap = h.s_ap.as<R>(n4);
        R* bR = h.s_trial.as<R>(n4);
        R* mask4 = h.s_mask4.as<R>(n4);
        double* r64 = h.s_r64.as<double>(n);
        double* y64 = h.s_b64.as<double>(n);
        const int vg = vec_grid(pcg_init<R>);
        const int pg = std::max(spmv_grid(spmv_sell<R, R, R, true, false, 4>), vec_grid(pcg_update<R>));
        double* part = h.s_part.as<double>(std::max(4 * 1024, 2 * std::max(pg, vg)));
        PcgState* st = reinterpret_cast<PcgState*>(h.s_scal.as<double>(64));
        LPG_CUDA(cudaMemsetAsync(x64, 0, n * sizeof(double), s));
        LPG_CUDA(cudaMemcpyAsync(r64, b64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        const double bnorm = std::sqrt(stats<double, double>(b64, nullptr, mask)[1]);
        if (bnorm == 0) return out;
        pad_rhs<R><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(mask, mask, mask4, V); // 0/1 values: mask^2 = mask
        // The graph of 16 iteration pairs, captured on the handle's own stream and cached.
        constexpr int kPairs = 16;
        constexpr int kKey = 12;
        const void* key[kKey] = {Kin, dinv, mask4, x, r, z, pA, pB, Ap, st, part,
                                 reinterpret_cast<const void*>(sizeof(R) * 1000003u + V)};
        bool same = h.pcg_graph != nullptr;
        for (int i = 0; i < kKey && same; ++i) same = h.pcg_graph_key[i] == key[i];
        cudaStream_t gs = h.own_stream;
        if (!same) {
            if (h.pcg_graph) {
                cudaGraphExecDestroy(h.pcg_graph);
                h.pcg_graph = nullptr;
            }
            cudaGraph_t g = nullptr;
            LPG_CUDA(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
            enqueue_iterations<R>(gs, static_cast<const R*>(Kin), dinv, mask4, x, r, z, pA, pB, Ap, st, part, kPairs);
            LPG_CUDA(cudaStreamEndCapture(gs, &g));
            LPG_CUDA(cudaGraphInstantiate(&h.pcg_graph, g, 0));
            cudaGraphDestroy(g);
            for (int i = 0; i < kKey; ++i) h.pcg_graph_key[i] = key[i];
        }
        cudaEvent_t ev;
        LPG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        double rnorm = bnorm;
        for (int ref = 0; ref <= max_refine; ++ref) {
            const double inner_tol = std::min(0.5, std::max(tol * bnorm / rnorm, sizeof(R) == 4 ? 1e-6 : 1e-14));
            pad_rhs<R><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(r64, mask, bR, V);
            pcg_init<R><<<vg, kThreads, 0, s>>>(bR, dinv, x, r, z, pA, V, part);
            pcg_start<<<1, 1024, 0, s>>>(st, part, vg, inner_tol, max_iters - static_cast<int>(out.iters));
            LPG_CUDA(cudaGetLastError());
            PcgState hs{};
            for (;;) {
                LPG_CUDA(cudaEventRecord(ev, s));
                LPG_CUDA(cudaStreamWaitEvent(gs, ev, 0));
                LPG_CUDA(cudaGraphLaunch(h.pcg_graph, gs));
                LPG_CUDA(cudaEventRecord(ev, gs));
                LPG_CUDA(cudaStreamWaitEvent(s, ev, 0));
                LPG_CUDA(cudaMemcpyAsync(&hs, st, sizeof hs, cudaMemcpyDeviceToHost, s));
                LPG_CUDA(cudaStreamSynchronize(s));
                if (hs.done) break;
            }
            out.iters += hs.iters;
            if (hs.breakdown) {
                out.breakdown = true;
                // Negative curvature on the first step: keep the preconditioned residual direction.
                if (hs.iters == 0) LPG_CUDA(cudaMemcpyAsync(x, pB, n4 * sizeof(R), cudaMemcpyDeviceToDevice, s));
            }
            add_kernel<R><<<grid(n), kThreads, 0, s>>>(x64, x, n);
            residual_spmv(Kres, res64, x64, mask, y64);
            residual_kernel<<<grid(n), kThreads, 0, s>>>(b64, y64, mask, r64, n);
            LPG_CUDA(cudaGetLastError());
            rnorm = std::sqrt(stats<double, double>(r64, nullptr, mask)[1]);
            out.rel = rnorm / bnorm;
            if (out.breakdown || !(rnorm > tol * bnorm) || out.iters >= max_iters || !std::isfinite(rnorm)) break;
        }
        cudaEventDestroy(ev);
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

} // namespace

void newton_solve(lpg_fem& h, const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                  const lpg_newton_options& o, double* x_out, lpg_newton_result* res) {
    if (!(o.gradient_tolerance >= 0.0) || !std::isfinite(o.gradient_tolerance))
        fail(LPG_EINVAL, "newton_solve: gradient_tolerance must be set to a finite non-negative value");
    if (o.max_iterations < 0 || o.max_line_search_steps < 1)
        fail(LPG_EINVAL, "newton_solve: max_iterations must be >= 0 and max_line_search_steps >= 1");
    if (!(o.line_search_shrink > 0.0 && o.line_search_shrink < 1.0))
        fail(LPG_EINVAL, "newton_solve: line_search_shrink must lie in (0, 1)");
    if (!(o.exact_below >= 0.0) || !std::isfinite(o.exact_below))
        fail(LPG_EINVAL, "newton_solve: exact_below must be finite and non-negative");
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
    // Hessian in the sliced-ELL layout; its padding slots are zeroed once and never written.
    const size_t hbytes = 9 * static_cast<size_t>(h.plan.sell_ptr.back()) * (f64 ? 8 : 4);
    void* K = h.s_hess.ensure(std::max<size_t>(hbytes, 8));
    LPG_CUDA(cudaMemsetAsync(K, 0, hbytes, s));
    void* dinv = h.s_dinv.ensure(12 * static_cast<size_t>(std::max(V, 1)) * (f64 ? 8 : 4));
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
    bool exact = false; // the exact_below switch, decided on the previous iteration's gradient
    for (int it = 0;; ++it) {
        const int hk = exact ? LPG_HESSIAN_EXACT : o.hessian;
        // Energy and FP64 gradient (the Newton residual).
        double E;
        if (f64) {
            h.eval_async(x, g, hk, LPG_PRECISION_F64, kLayoutSell, K, nullptr);
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
        if (o.exact_below > 0 && g2 <= o.exact_below * gnorm0) exact = true;
        R.energy = E;
        R.gradient_norm = o.stop_rule == 0 ? gmax : g2;
        R.gradient_norm0 = gnorm0;
        R.iterations = it;
        const bool converged = o.stop_rule == 0 ? gmax <= o.gradient_tolerance : g2 <= o.gradient_tolerance * gnorm0;
        if (converged) return finish(0);
        if (it == o.max_iterations) return finish(1);
        if (!f64) {
            h.eval_async(x, nullptr, hk, LPG_PRECISION_MIXED, kLayoutSell, K, nullptr);
            raise_status(h.take_status());
        }
        // Descent direction with diagonal shifts (newton.cpp:55-72).
        neg_mask<<<grid(n), kThreads, 0, s>>>(g, mask, rhs, n);
        double dscale = 1.0;
        {
            const int vb = grid(static_cast<size_t>(V));
            double* part = h.s_part.as<double>(std::max(4 * 1024, vb));
            double* outm = h.s_scal.as<double>(64) + 40;
            diag_absmax_partial<<<vb, kThreads, 0, s>>>(h.dm, f64 ? static_cast<double*>(K) : nullptr,
                                                       f64 ? nullptr : static_cast<float*>(K), mask, part);
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
                    h.dm, static_cast<double*>(K), mask, static_cast<double*>(dinv), V);
                po = S.pcg<double>(K, static_cast<double*>(dinv), K, true, mask, rhs, d, eta, o.cg_max_iterations, 0);
            } else {
                block_jacobi<float, float><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(
                    h.dm, static_cast<float*>(K), mask, static_cast<float*>(dinv), V);
                po = S.pcg<float>(K, static_cast<float*>(dinv), K, false, mask, rhs, d, eta, o.cg_max_iterations, 3);
            }
            R.cg_iterations += po.iters;
            gd = S.stats<double, double>(g, d, mask)[0];
            if (gd < 0.0 && std::isfinite(gd)) {
                found = true;
                break;
            }
            if (shifts == 10) break;
            shift_diag<<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(h.dm, f64 ? static_cast<double*>(K) : nullptr,
                                                                       f64 ? nullptr : static_cast<float*>(K), shift);
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

namespace {

// The adjoint solve of StaticEquilibriumResponse (static_equilibrium_response.cpp:43-68): the
// Exact FP64 Hessian K at u*, then mask K lambda = mask dL/du by PCG with FP64 refinement and
// the reference's residual check. Returns lambda (device) and u* (device) through out-params.
void adjoint_solve(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                   int precision, double cg_tolerance, const double** u_dev, double** lam_dev) {
    if (precision != LPG_PRECISION_F64 && precision != LPG_PRECISION_MIXED) fail(LPG_EINVAL, "invalid precision");
    if (!(cg_tolerance > 0) || !std::isfinite(cg_tolerance)) fail(LPG_EINVAL, "adjoint: cg_tolerance must be positive");
    Solver S(h);
    const size_t n = S.n;
    const int V = S.V;
    cudaStream_t s = h.stream;
    double* mask = h.s_mask.as<double>(std::max<size_t>(n, 1));
    make_mask(h, fixed, nfixed, mask);
    const double* u = h.stage_in(u_star, io_mem, h.d_u, n);
    const double* w = h.stage_in(dLdu, io_mem, h.d_u2, n);
    double* lam = h.s_d.as<double>(std::max<size_t>(n, 1));
    LPG_CUDA(cudaMemsetAsync(lam, 0, n * sizeof(double), s));
    *u_dev = u;
    *lam_dev = lam;
    const auto ws = S.stats<double, double>(w, nullptr, mask);
    if (!std::isfinite(ws[1])) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: nonfinite sensitivity right-hand side");
    if (n == 0 || !(ws[1] > 0)) return;
    // Exact FP64 Hessian at u*: the residual matrix of the refinement (static_equilibrium_response.cpp:58).
    // Sliced-ELL Hessians; padding slots zeroed (never written by the assembly).
    const size_t nv = 9 * static_cast<size_t>(h.plan.sell_ptr.back());
    double* K64 = h.s_hess64.as<double>(std::max<size_t>(nv, 1));
    LPG_CUDA(cudaMemsetAsync(K64, 0, nv * sizeof(double), s));
    h.eval_async(u, nullptr, LPG_HESSIAN_EXACT, LPG_PRECISION_F64, kLayoutSell, K64, nullptr);
    raise_status(h.take_status());
    double* rhs = h.s_g.as<double>(std::max<size_t>(n, 1));
    LPG_CUDA(cudaMemcpyAsync(rhs, w, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    Solver::PcgOut po;
    if (precision == LPG_PRECISION_F64) {
        double* dinv = h.s_dinv.as<double>(12 * static_cast<size_t>(std::max(V, 1)));
        block_jacobi<double, double><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(h.dm, K64, mask, dinv, V);
        po = S.pcg<double>(K64, dinv, K64, true, mask, rhs, lam, cg_tolerance, 200000, 2);
    } else {
        float* K32 = h.s_hess.as<float>(std::max<size_t>(nv, 1));
        if (nv) convert_kernel<double, float><<<grid(nv), kThreads, 0, s>>>(K64, K32, nv);
        float* dinv = h.s_dinv.as<float>(12 * static_cast<size_t>(std::max(V, 1)));
        block_jacobi<float, float><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(h.dm, K32, mask, dinv, V);
        po = S.pcg<float>(K32, dinv, K64, true, mask, rhs, lam, cg_tolerance, 200000, 30);
    }
    if (po.breakdown) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: singular or indefinite equilibrium stiffness");
    // Residual check (static_equilibrium_response.cpp:61-68) in FP64 with the exact Hessian.
    const double bn = std::sqrt(ws[1]);
    if (!(po.rel * bn <= 1e-8 * (1.0 + bn))) fail(LPG_EDOMAIN, "StaticEquilibriumResponse: inaccurate sensitivity solve");
}

void copy_lambda(lpg_fem& h, const double* lam, int io_mem, double* lambda_out) {
    if (!lambda_out) return;
    const size_t n = 3 * static_cast<size_t>(h.dm.V);
    LPG_CUDA(cudaMemcpyAsync(lambda_out, lam, n * sizeof(double),
                             io_mem == LPG_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h.stream));
}

} // namespace

void adjoint_theta(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                   int precision, double cg_tolerance, int per_element, double* dtheta, double* lambda_out) {
    const double* u = nullptr;
    double* lam = nullptr;
    adjoint_solve(h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, &u, &lam);
    cudaStream_t s = h.stream;
    const size_t T = static_cast<size_t>(h.dm.T);
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
    } else {
        std::copy(host.begin(), host.end(), dtheta);
    }
    copy_lambda(h, lam, io_mem, lambda_out);
    LPG_CUDA(cudaStreamSynchronize(s));
}

void adjoint_rest(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                  int precision, double cg_tolerance, double* dX, double* lambda_out) {
    const double* u = nullptr;
    double* lam = nullptr;
    adjoint_solve(h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, &u, &lam);
    cudaStream_t s = h.stream;
    const size_t n = 3 * static_cast<size_t>(h.dm.V);
    // dX = -(dg/dX)^T lambda.
    double* out = io_mem == LPG_MEM_DEVICE ? dX : h.d_grad.as<double>(std::max<size_t>(n, 1));
    double* pe = h.d_vjp.as<double>(std::max<size_t>(12 * static_cast<size_t>(h.dm.T), 1));
    launch_rest_vjp(h.dm, u, lam, pe, -1.0, out, h.d_status.as<unsigned>(1), s);
    raise_status(h.take_status());
    if (io_mem == LPG_MEM_HOST && n > 0) LPG_CUDA(cudaMemcpyAsync(dX, out, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    copy_lambda(h, lam, io_mem, lambda_out);
    LPG_CUDA(cudaStreamSynchronize(s));
}

} // namespace lpg
