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
#include <chrono>
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
// Two block sums at once (sh holds 2 doubles per warp), each in block_sum's order.
__device__ __forceinline__ double2 block_sum2(double a, double b, double* sh) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[2 * (threadIdx.x >> 5)] = a;
        sh[2 * (threadIdx.x >> 5) + 1] = b;
    }
    __syncthreads();
    double ra = 0, rb = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (blockDim.x >> 5); ++w) {
            ra += sh[2 * w];
            rb += sh[2 * w + 1];
        }
    __syncthreads();
    return make_double2(ra, rb);
}
// Programmatic dependent launch: a kernel launched with programmatic stream serialization may
// start while the kernel before it drains; it waits here until that kernel has completed and
// its memory is visible (a no-op for an ordinary launch), then lets its own dependent launch.
__device__ __forceinline__ void pdl_wait_then_release() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
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

// Entry t (row-major) of the diagonal block of vertex v in the solver layout, or -1.
__device__ __forceinline__ int64_t diag_entry(const DevMesh& m, int v, int t) {
    if (m.diag_slot[v] < 0) return -1;
    return static_cast<int64_t>(m.sell_base[v]) + 32 * t; // own block 0 is the diagonal
}

// y = mask (K x) on the symmetric 3x3 block matrix in the upper-triangle sliced-ELL layout
// (SELL-32): one warp per chunk of 32 rows, one lane per row. Own block slot q of every lane is
// read together, so each of the nine value loads and the column load of a slot is one
// contiguous 128-byte (FP32) run; a borrowed block (left of the diagonal) is the owning row's
// block read transposed, nine 4- or 8-byte loads 32 entries apart (coalesced when the 32 rows'
// owners sit in one chunk, as in a structured ordering). A lane's slots are independent (no
// cross-lane reduction); half the blocks are stored, so the matrix stream is about halved. Vectors hold S values per vertex: 4
// for the padded PCG vectors (4th value zero, one 16-byte load per gathered vertex in FP32),
// 3 for plain FP64 vectors. With PCG the vector is z + beta p_old (beta from the state; each
// row writes it to p_new), and the block of the grid that finishes last reduces the partial
// p.Ap sums into alpha; otherwise, with DOT, part[block] = sum x.y. Both reductions use a
// fixed order.
// Resident blocks per SM the register allocation must allow: 8 x 256 threads (32 registers)
// for FP32 values, where more resident warps hide the gathers' latency better than the
// registers they cost; 4 (64 registers) for FP64, whose nine 8-byte values per block spill at
// 32. Slots unrolled by 2.
#ifndef LPG_SPMV_MIN_BLOCKS_F32
#define LPG_SPMV_MIN_BLOCKS_F32 8
#endif
#ifndef LPG_SPMV_MIN_BLOCKS_F64
#define LPG_SPMV_MIN_BLOCKS_F64 4
#endif
#ifndef LPG_SPMV_UNROLL
#define LPG_SPMV_UNROLL 2
#endif
// Launch variants of the PCG SpMV (autotuner): {resident blocks, slot unroll}. Variant 0 is the
// default; all variants sum each row in the same order, so their results are bitwise identical.
// Variant 2 reads a lane's slots in batches of four: their column indices first,
// then all their vector gathers, then the block values and products, so that a batch of gathers
// per lane is in flight instead of the loop's dependent column -> gather chain of one or two
// slots; the products are summed in the same slot order as the other variants.
template <typename TK, int VAR> struct SpmvCfg {
    static constexpr bool f32 = sizeof(TK) == 4;
    static constexpr int minb = VAR == 0 ? (f32 ? LPG_SPMV_MIN_BLOCKS_F32 : LPG_SPMV_MIN_BLOCKS_F64)
                                         : VAR == 1 ? (f32 ? 8 : 4) : (f32 ? 3 : 2);
    static constexpr int unroll = VAR == 0 ? LPG_SPMV_UNROLL : 4;
    static constexpr bool batched = VAR == 2;
    static constexpr int batch = 4;
};
template <typename TK, typename TV, typename TO, bool PCG, bool DOT, int S, int VAR = 0>
__global__ void __launch_bounds__(kThreads, (SpmvCfg<TK, VAR>::minb)) spmv_sell(const DevMesh m, const TK* __restrict__ val,
                                                      const TV* __restrict__ x, const TV* __restrict__ p_old,
                                                      const TV* __restrict__ mask, TO* __restrict__ y,
                                                      TV* __restrict__ p_new, PcgState* st, double* part) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    using A = typename std::conditional<(sizeof(TK) == 4 && sizeof(TV) == 4), float, double>::type;
    if (PCG) pdl_wait_then_release();
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
        auto gather = [&](size_t col, A xv[3]) {
            TV xz[3];
            ld3<S>(x, col, xz);
            if (PCG) {
                TV xp[3];
                ld3<S>(p_old, col, xp);
#pragma unroll
                for (int i = 0; i < 3; ++i) xz[i] = xz[i] + beta * xp[i];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) xv[i] = static_cast<A>(xz[i]);
        };
        const int b0 = __ldg(m.sell_bptr + c);
        const int bwidth = (__ldg(m.sell_bptr + c + 1) - b0) >> 5;
        const int2* bp = m.sell_bref + b0 + lane;
        if constexpr (SpmvCfg<TK, VAR>::batched) {
            constexpr int kSpmvBatch = SpmvCfg<TK, VAR>::batch;
            // Own blocks (columns >= row), then borrowed blocks, each in batches of kSpmvBatch slots.
            for (int q0 = 0; q0 < width; q0 += kSpmvBatch) {
                int col[kSpmvBatch];
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j) col[j] = q0 + j < width ? __ldg(cp + 32 * (q0 + j)) : 0;
                A xv[kSpmvBatch][3];
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j)
                    if (q0 + j < width) gather(static_cast<size_t>(col[j]), xv[j]);
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j) {
                    if (q0 + j >= width) break;
                    const TK* vq = vp + 288 * static_cast<size_t>(q0 + j);
                    A kv[9];
#pragma unroll
                    for (int e = 0; e < 9; ++e) kv[e] = static_cast<A>(__ldg(vq + 32 * e));
                    a0 += kv[0] * xv[j][0] + kv[1] * xv[j][1] + kv[2] * xv[j][2];
                    a1 += kv[3] * xv[j][0] + kv[4] * xv[j][1] + kv[5] * xv[j][2];
                    a2 += kv[6] * xv[j][0] + kv[7] * xv[j][1] + kv[8] * xv[j][2];
                }
            }
            for (int q0 = 0; q0 < bwidth; q0 += kSpmvBatch) {
                int2 ref[kSpmvBatch];
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j) ref[j] = q0 + j < bwidth ? __ldg(bp + 32 * (q0 + j)) : make_int2(0, 0);
                A xv[kSpmvBatch][3];
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j)
                    if (q0 + j < bwidth) gather(static_cast<size_t>(ref[j].y), xv[j]);
#pragma unroll
                for (int j = 0; j < kSpmvBatch; ++j) {
                    if (q0 + j >= bwidth) break;
                    const TK* vq = val + static_cast<size_t>(ref[j].x);
                    A kv[9];
#pragma unroll
                    for (int e = 0; e < 9; ++e) kv[e] = static_cast<A>(__ldg(vq + 32 * e));
                    a0 += kv[0] * xv[j][0] + kv[3] * xv[j][1] + kv[6] * xv[j][2];
                    a1 += kv[1] * xv[j][0] + kv[4] * xv[j][1] + kv[7] * xv[j][2];
                    a2 += kv[2] * xv[j][0] + kv[5] * xv[j][1] + kv[8] * xv[j][2];
                }
            }
        } else {
            // Own blocks (columns >= row): K_rc x_c.
#pragma unroll (SpmvCfg<TK, VAR>::unroll)
            for (int q = 0; q < width; ++q) {
                A xv[3];
                gather(static_cast<size_t>(__ldg(cp + 32 * q)), xv);
                const TK* vq = vp + 288 * static_cast<size_t>(q);
                A kv[9];
#pragma unroll
                for (int e = 0; e < 9; ++e) kv[e] = static_cast<A>(__ldg(vq + 32 * e));
                a0 += kv[0] * xv[0] + kv[1] * xv[1] + kv[2] * xv[2];
                a1 += kv[3] * xv[0] + kv[4] * xv[1] + kv[5] * xv[2];
                a2 += kv[6] * xv[0] + kv[7] * xv[1] + kv[8] * xv[2];
            }
            // Borrowed blocks (columns < row): K_cr^T x_c from the owning row's block.
#pragma unroll (SpmvCfg<TK, VAR>::unroll)
            for (int q = 0; q < bwidth; ++q) {
                const int2 ref = __ldg(bp + 32 * q);
                A xv[3];
                gather(static_cast<size_t>(ref.y), xv);
                const TK* vq = val + static_cast<size_t>(ref.x);
                A kv[9];
#pragma unroll
                for (int e = 0; e < 9; ++e) kv[e] = static_cast<A>(__ldg(vq + 32 * e));
                a0 += kv[0] * xv[0] + kv[3] * xv[1] + kv[6] * xv[2];
                a1 += kv[1] * xv[0] + kv[4] * xv[1] + kv[7] * xv[2];
                a2 += kv[2] * xv[0] + kv[5] * xv[1] + kv[8] * xv[2];
            }
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
    __shared__ double sh[2 * (kThreads / 32)];
    __shared__ bool last;
    pdl_wait_then_release();
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
    const double2 sums = block_sum2(rz, rr, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sums.x;
        part[2 * blockIdx.x + 1] = sums.y;
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
    {
        const double2 t = block_sum2(a, b, sh);
        a = t.x;
        b = t.y;
    }
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
// y = A x for a scalar CSR matrix (one thread per row, entries in stored order).
__global__ void csr_apply_kernel(const int32_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                 const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                                 int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) acc = fma(val[k], x[col[k]], acc);
    y[i] = acc;
}
// g = w g (+ y when y is given).
__global__ void scale_add_kernel(double* __restrict__ g, double w, const double* __restrict__ y, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    double v = g[i] * w;
    if (y) v += y[i];
    g[i] = v;
}
template <typename R> __global__ void scale_values_kernel(R* __restrict__ v, size_t n, double w) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) v[i] = static_cast<R>(static_cast<double>(v[i]) * w);
}
// Adds the quadratic term's entries at their solver-layout positions (distinct positions).
template <typename R>
__global__ void add_at_kernel(R* __restrict__ K, const int64_t* __restrict__ pos, const double* __restrict__ val, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) K[pos[i]] = static_cast<R>(static_cast<double>(K[pos[i]]) + val[i]);
}

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
// A weighted-sum potential around the elastic energy (lpg_newton_terms) on the device:
//   E = w elastic + 1/2 x^T A x + c (the linear load is handled as f_ext).
struct Potential {
    const lpg_newton_terms* t = nullptr;          // the caller's terms (material and feasible callbacks)
    double w = 1.0, c = 0.0;
    int n = 0;                                    // rows of A (0: no quadratic term)
    int32_t *ptr = nullptr, *col = nullptr;       // A, CSR (duplicates merged)
    double* val = nullptr;
    int nk = 0;                                   // A's entries in the solver layout's upper blocks
    int64_t* kpos = nullptr;
    double* kval = nullptr;
    double* Ax = nullptr;                         // scratch, n values
};

// One evaluation of the elastic term at x (gradient into g if given, Hessian of kind hk into K
// in layout): the handle's own element pass, or with a caller's material the exported F, the
// material's W / P / A and their integration (lpg_fem_eval_material's path). Enqueued on the
// handle's stream; the material callback runs on the host in between.
void eval_elastic_async(lpg_fem& h, const lpg_newton_terms* t, const double* x, double* g, int hk, int prec,
                        int layout, void* K) {
    if (!t || !t->material) {
        h.eval_async(x, g, hk, prec, layout, K, nullptr);
        return;
    }
    const DevMesh& m = h.dm;
    if (m.K == 64) fail(LPG_EINVAL, "newton_solve: materials are not available for Hermite hex meshes");
    if (m.fpinv64) fail(LPG_EINVAL, "newton_solve: a material handle has no plastic field");
    cudaStream_t s = h.stream;
    const bool hex = m.K == 8;
    const size_t rows = static_cast<size_t>(m.T) * (hex ? m.nq : 1), nel = std::max<size_t>(m.T, 1);
    double* F = h.d_mat[4].as<double>(std::max<size_t>(9 * rows, 1));
    double* W = h.d_mat[0].as<double>(std::max<size_t>(rows, 1));
    double* P = h.d_mat[1].as<double>(std::max<size_t>(9 * rows, 1));
    double* A = hk != LPG_HESSIAN_NONE ? h.d_mat[2].as<double>(std::max<size_t>(81 * rows, 1)) : nullptr;
    unsigned* status = h.d_status.as<unsigned>(1);
    if (hex)
        launch_hex_deformation_gradients(m, x, F, status, s);
    else
        launch_deformation_gradients(m, x, F, status, s);
    raise_status(h.take_status());
    const int want = hk != LPG_HESSIAN_NONE ? 2 : g ? 1 : 0;
    if (t->material(F, static_cast<int>(rows), want, W, want >= 1 ? P : nullptr, A, t->material_user) != 0)
        fail(LPG_ESTOPPED, "newton_solve: the material callback stopped the solve");
    EvalArgs a;
    a.grad = g;
    a.hess = hk != LPG_HESSIAN_NONE ? K : nullptr;
    a.layout = layout;
    a.cluster_energy = h.d_cluster_energy.as<double>(static_cast<size_t>(std::max(m.ncl, m.tc_ncl)) + 256);
    a.energy = h.d_energy.as<double>(1);
    a.status = status;
    const int pi = prec == LPG_PRECISION_F64 ? 0 : 1;
    if (hex) {
        const bool projected = hk == LPG_HESSIAN_PROJECTED;
        void* blocks = a.hess ? h.d_proj.ensure(hex_blocks_bytes(m, prec, projected)) : nullptr;
        launch_hex_material_eval(m, prec, hk, W, g ? P : nullptr, A, h.d_mat[3].as<double>(nel), h.d_vjp.as<double>(24 * nel),
                                 blocks, projected && a.hess ? h.d_plist.as<int>(nel) : nullptr, a, s);
    } else {
        void* proj = a.hess ? h.d_proj.ensure(project_bytes(m, prec)) : nullptr;
        launch_material_eval(m, prec, hk, W, g ? P : nullptr, A, h.d_mat[3].as<double>(nel), h.d_vjp.as<double>(12 * nel),
                             proj, h.d_plist.as<int>(nel), h.d_pcount.as<unsigned>(1), h.tune.clamp[pi], a, s);
    }
}

struct Solver {
    lpg_fem& h;
    cudaStream_t s;
    size_t n;
    int V;
    const Potential* P = nullptr;
    explicit Solver(lpg_fem& hh, const Potential* p = nullptr)
        : h(hh), s(hh.stream), n(3 * static_cast<size_t>(hh.dm.V)), V(hh.dm.V), P(p) {}

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
        eval_elastic_async(h, P ? P->t : nullptr, x, g, LPG_HESSIAN_NONE, LPG_PRECISION_F64, LPG_LAYOUT_BSR, nullptr);
        return compose(x, f, g);
    }
    // The potential from the elastic evaluation just enqueued (energy in h.d_energy, gradient
    // in g if given): weight, quadratic term, load and constant.
    double compose(const double* x, const double* f, double* g) {
        double aq = 0;
        if (P && (P->w != 1.0 || P->n > 0)) {
            if (P->n > 0)
                csr_apply_kernel<<<grid(static_cast<size_t>(P->n)), kThreads, 0, s>>>(P->ptr, P->col, P->val, x, P->Ax,
                                                                                    P->n);
            if (g) scale_add_kernel<<<grid(n), kThreads, 0, s>>>(g, P->w, P->n > 0 ? P->Ax : nullptr, n);
            LPG_CUDA(cudaGetLastError());
        }
        if (g && f) load_gradient<<<grid(n), kThreads, 0, s>>>(g, f, n);
        double e = 0;
        LPG_CUDA(cudaMemcpyAsync(&e, h.d_energy.ptr, sizeof e, cudaMemcpyDeviceToHost, s));
        raise_status(h.take_status());
        if (P && P->n > 0) aq = 0.5 * stats<double, double>(x, P->Ax, nullptr)[0];
        if (P) e = P->w * e + aq + P->c;
        return e - energy_dot_f(x, f);
    }
    // The quadratic term and weight applied to a solver-layout Hessian of precision R.
    template <typename R> void compose_hessian(R* K) {
        if (!P) return;
        if (P->w != 1.0) {
            const size_t nv = h.plan.sell_values();
            scale_values_kernel<R><<<grid(nv), kThreads, 0, s>>>(K, nv, P->w);
        }
        if (P->nk > 0) add_at_kernel<R><<<grid(static_cast<size_t>(P->nk)), kThreads, 0, s>>>(K, P->kpos, P->kval, P->nk);
        LPG_CUDA(cudaGetLastError());
    }

    // One warp per sliced-ELL chunk (8 per block). Not persistent: with about one chunk per
    // resident warp, a grid-stride loop would leave a fifth of the warps with two chunks and the
    // rest idle; later blocks instead start as earlier ones finish.
    int spmv_grid(int = 0) const { return std::max(1, (h.dm.n_sell + 7) / 8); }
    template <typename Kern> int vec_grid(Kern k) const { return one_wave(k, grid(static_cast<size_t>(V))); }

    // y64 = mask (K x64) in FP64 with K stored as TK.
    void residual_spmv(const void* K, bool k64, const double* x64, const double* mask, double* y64) {
        if (k64)
            spmv_sell<double, double, double, false, false, 3>
                <<<spmv_grid(), kThreads, 0, s>>>(
                    h.dm, static_cast<const double*>(K), x64, nullptr, mask, y64, nullptr, nullptr, nullptr);
        else
            spmv_sell<float, double, double, false, false, 3>
                <<<spmv_grid(), kThreads, 0, s>>>(
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
    template <typename R, int VAR>
    void enqueue_iterations_v(cudaStream_t gs, const R* K, const R* dinv, const R* mask4, R* x, R* r, R* z, R* pA,
                              R* pB, R* Ap, PcgState* st, double* part, int pairs) {
        const int sg = spmv_grid(0), ug = std::max(1, grid(static_cast<size_t>(V)));
        // Each kernel is launched as a programmatic dependent of the one before it (it waits in
        // griddepcontrol.wait), so its launch overlaps the previous kernel's last blocks.
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cs{}, cu{};
        cs.gridDim = dim3(static_cast<unsigned>(sg));
        cu.gridDim = dim3(static_cast<unsigned>(ug));
        cs.blockDim = cu.blockDim = dim3(kThreads);
        cs.stream = cu.stream = gs;
        cs.attrs = cu.attrs = attr;
        cs.numAttrs = cu.numAttrs = 1;
        const DevMesh& dm = h.dm;
        const R* zc = z;
        for (int i = 0; i < pairs; ++i) {
            LPG_CUDA(cudaLaunchKernelEx(&cs, spmv_sell<R, R, R, true, false, 4, VAR>, dm, K, zc,
                                        static_cast<const R*>(pA), static_cast<const R*>(mask4), Ap, pB, st, part));
            LPG_CUDA(cudaLaunchKernelEx(&cu, pcg_update<R>, st, dinv, x, r, z, static_cast<const R*>(pB),
                                        static_cast<const R*>(Ap), V, part));
            LPG_CUDA(cudaLaunchKernelEx(&cs, spmv_sell<R, R, R, true, false, 4, VAR>, dm, K, zc,
                                        static_cast<const R*>(pB), static_cast<const R*>(mask4), Ap, pA, st, part));
            LPG_CUDA(cudaLaunchKernelEx(&cu, pcg_update<R>, st, dinv, x, r, z, static_cast<const R*>(pA),
                                        static_cast<const R*>(Ap), V, part));
        }
    }
    // The same with the handle's tuned SpMV variant for precision R.
    template <typename R>
    void enqueue_iterations(cudaStream_t gs, const R* K, const R* dinv, const R* mask4, R* x, R* r, R* z, R* pA,
                            R* pB, R* Ap, PcgState* st, double* part, int pairs) {
        switch (h.tune.spmv[sizeof(R) == 8 ? 0 : 1]) {
        case 1: enqueue_iterations_v<R, 1>(gs, K, dinv, mask4, x, r, z, pA, pB, Ap, st, part, pairs); break;
        case 2: enqueue_iterations_v<R, 2>(gs, K, dinv, mask4, x, r, z, pA, pB, Ap, st, part, pairs); break;
        default: enqueue_iterations_v<R, 0>(gs, K, dinv, mask4, x, r, z, pA, pB, Ap, st, part, pairs); break;
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
        const int pg = std::max(spmv_grid(), std::max(1, grid(static_cast<size_t>(V))));
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
                                 reinterpret_cast<const void*>((sizeof(R) * 1000003u + V) * 4u +
                                                               h.tune.spmv[sizeof(R) == 8 ? 0 : 1])};
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

namespace {

// The quadratic term of a weighted-sum potential on the device: A merged and checked on the host
// (symmetric, inside the elastic pattern), its CSR for A x, and its entries of the solver
// layout's upper blocks (row vertex <= column vertex) for the Hessian.
void build_potential(lpg_fem& h, const lpg_newton_terms* t, Potential& P) {
    if (!t) return;
    if (!std::isfinite(t->elastic_weight) || t->elastic_weight == 0.0)
        fail(LPG_EINVAL, "WeightedSumEnergy weights must be finite and nonzero");
    if (!std::isfinite(t->constant)) fail(LPG_EINVAL, "newton_solve: the potential's constant must be finite");
    P.t = t;
    P.w = t->elastic_weight;
    P.c = t->constant;
    if (!t->a_indptr) return;
    const HostPlan& p = h.plan;
    const int n = 3 * p.V;
    if (!t->a_indices || !t->a_values) fail(LPG_EINVAL, "QuadraticEnergy: null CSR arrays");
    if (t->a_indptr[0] != 0) fail(LPG_EINVAL, "QuadraticEnergy: CSR row pointers must start at 0");
    struct Ent {
        int r, c;
        double v;
    };
    std::vector<Ent> ents;
    for (int r = 0; r < n; ++r) {
        if (t->a_indptr[r + 1] < t->a_indptr[r]) fail(LPG_EINVAL, "QuadraticEnergy: CSR row pointers must not decrease");
        for (int k = t->a_indptr[r]; k < t->a_indptr[r + 1]; ++k) {
            const int c = t->a_indices[k];
            const double v = t->a_values[k];
            if (c < 0 || c >= n) fail(LPG_EINVAL, "QuadraticEnergy: column index out of range");
            if (!std::isfinite(v)) fail(LPG_EINVAL, "QuadraticEnergy: A must be finite");
            ents.push_back({r, c, v});
        }
    }
    std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
    std::vector<Ent> m;
    for (const Ent& e : ents) {
        if (!m.empty() && m.back().r == e.r && m.back().c == e.c)
            m.back().v += e.v;
        else
            m.push_back(e);
    }
    // Symmetry: entry (c, r) equals entry (r, c).
    auto find = [&](int r, int c) -> const Ent* {
        auto it = std::lower_bound(m.begin(), m.end(), Ent{r, c, 0},
                                   [](const Ent& a, const Ent& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
        return it != m.end() && it->r == r && it->c == c ? &*it : nullptr;
    };
    std::vector<int32_t> ptr(static_cast<size_t>(n) + 1, 0), col;
    std::vector<double> val;
    std::vector<int64_t> kpos;
    std::vector<double> kval;
    for (const Ent& e : m) {
        const Ent* tr = find(e.c, e.r);
        if (!tr || tr->v != e.v) fail(LPG_EINVAL, "QuadraticEnergy: A must be symmetric on the GPU Newton path");
        ++ptr[e.r + 1];
        col.push_back(e.c);
        val.push_back(e.v);
        const int vr = e.r / 3, vc = e.c / 3;
        const int32_t* beg = p.col_idx.data() + p.row_ptr[vr];
        const int32_t* end = p.col_idx.data() + p.row_ptr[vr + 1];
        const int32_t* at = std::lower_bound(beg, end, vc);
        if (at == end || *at != vc)
            fail(LPG_EINVAL, "QuadraticEnergy: A couples DOFs of vertices that share no element (outside the elastic "
                             "Hessian's pattern), which the GPU Newton path does not support");
        if (vr <= vc && e.v != 0.0) {
            const int k = static_cast<int>(at - p.col_idx.data());
            kpos.push_back(static_cast<int64_t>(p.sell_base[vr]) +
                           32 * static_cast<int64_t>(9 * (k - p.diag_slot[vr]) + 3 * (e.r % 3) + (e.c % 3)));
            kval.push_back(e.v);
        }
    }
    for (int r = 0; r < n; ++r) ptr[r + 1] += ptr[r];
    auto up = [&](lpg::DeviceBuffer& b, const auto& v) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        T* d = b.as<T>(std::max<size_t>(v.size(), 1));
        if (!v.empty()) LPG_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h.stream));
        return d;
    };
    P.n = n;
    P.ptr = up(h.s_q[0], ptr);
    P.col = up(h.s_q[1], col);
    P.val = up(h.s_q[2], val);
    P.nk = static_cast<int>(kpos.size());
    P.kpos = up(h.s_q[3], kpos);
    P.kval = up(h.s_q[4], kval);
    P.Ax = h.s_q[5].as<double>(std::max<size_t>(n, 1));
    LPG_CUDA(cudaStreamSynchronize(h.stream)); // the host vectors go out of scope
}

} // namespace

void newton_solve(lpg_fem& h, const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                  const lpg_newton_options& o, double* x_out, lpg_newton_result* res, const lpg_newton_terms* terms) {
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
    Potential pot;
    build_potential(h, terms, pot);
    Solver S(h, &pot);
    const size_t n = S.n;
    const int V = S.V;
    cudaStream_t s = h.stream;
    double* mask = h.s_mask.as<double>(std::max<size_t>(n, 1));
    make_mask(h, fixed, nfixed, mask);
    // Per-iteration records for the caller's callback (NewtonStep, newton.hpp:34-44).
    lpg_newton_step step{};
    auto report = [&]() {
        if (terms && terms->on_iteration && terms->on_iteration(&step, terms->user) != 0)
            fail(LPG_ESTOPPED, "newton_solve: the on_iteration callback stopped the solve");
    };
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
    const size_t hbytes = h.plan.sell_values() * (f64 ? 8 : 4);
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
        const int64_t cg0 = R.cg_iterations;
        step = lpg_newton_step{};
        step.iteration = it;
        step.pattern_changed = it == 0;
        // Energy and FP64 gradient (the Newton residual).
        double E;
        if (f64) {
            eval_elastic_async(h, terms, x, g, hk, LPG_PRECISION_F64, kLayoutSell, K);
            E = S.compose(x, f, g);
            S.compose_hessian(static_cast<double*>(K));
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
        step.energy = E;
        step.gradient_norm = gmax;
        step.gradient_norm_2 = g2;
        const bool converged = o.stop_rule == 0 ? gmax <= o.gradient_tolerance : g2 <= o.gradient_tolerance * gnorm0;
        if (converged) {
            report();
            return finish(0);
        }
        if (it == o.max_iterations) {
            report();
            return finish(1);
        }
        if (!f64) {
            eval_elastic_async(h, terms, x, nullptr, hk, LPG_PRECISION_MIXED, kLayoutSell, K);
            raise_status(h.take_status());
            S.compose_hessian(static_cast<float*>(K));
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
            step.diagonal_shifts = shifts;
            if (gd < 0.0 && std::isfinite(gd)) {
                found = true;
                break;
            }
            if (shifts == 10) break;
            shift_diag<<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(h.dm, f64 ? static_cast<double*>(K) : nullptr,
                                                                       f64 ? nullptr : static_cast<float*>(K), shift);
            shift *= 10.0;
        }
        step.cg_iterations = R.cg_iterations - cg0;
        if (!found) {
            report();
            return finish(3);
        }
        // Line search (newton.cpp:92-108) from the feasible step.
        const int nb = feasible_blocks(h.dm);
        double* bm = h.d_block.as<double>(std::max(nb, 1));
        double* al = h.d_alpha.as<double>(1);
        double alpha = 1;
        if (terms && terms->feasible) {
            const bool hex = h.dm.K == 8;
            const size_t rows = static_cast<size_t>(h.dm.T) * (hex ? h.dm.nq : 1);
            double* Fx = h.d_mat[4].as<double>(std::max<size_t>(9 * rows, 1));
            double* Gd = h.d_mat[5].as<double>(std::max<size_t>(9 * rows, 1));
            unsigned* stw = h.d_status.as<unsigned>(1);
            if (hex) {
                launch_hex_deformation_gradients(h.dm, x, Fx, stw, s);
                launch_hex_deformation_gradients(h.dm, d, Gd, stw, s);
            } else {
                launch_deformation_gradients(h.dm, x, Fx, stw, s);
                launch_deformation_gradients(h.dm, d, Gd, stw, s);
            }
            raise_status(h.take_status());
            if (terms->feasible(Fx, Gd, static_cast<int>(rows), &alpha, terms->material_user) != 0)
                fail(LPG_ESTOPPED, "newton_solve: the feasible-step callback stopped the solve");
            if (!(alpha >= 0.0 && alpha <= 1.0))
                fail(LPG_ELOGIC, "Energy::max_feasible_step: the energy returned a value outside [0, 1]");
        } else {
            launch_feasible(h.dm, x, d, bm, nb, al, h.d_status.as<unsigned>(1), s);
            LPG_CUDA(cudaMemcpyAsync(&alpha, al, sizeof alpha, cudaMemcpyDeviceToHost, s));
            raise_status(h.take_status());
        }
        step.feasible_step = alpha;
        bool accepted = false;
        for (int j = 0; j < o.max_line_search_steps; ++j) {
            LPG_CUDA(cudaMemsetAsync(moved, 0, sizeof(int), s));
            axpy_trial<<<grid(n), kThreads, 0, s>>>(x, alpha, d, trial, n, moved);
            int mv = 0;
            LPG_CUDA(cudaMemcpyAsync(&mv, moved, sizeof mv, cudaMemcpyDeviceToHost, s));
            LPG_CUDA(cudaStreamSynchronize(s));
            if (!mv) break;
            ++R.line_search_evaluations;
            ++step.line_search_evaluations;
            const double Et = S.energy(trial, f, nullptr);
            const double noise = 16.0 * kEps * std::max(1.0, std::abs(E));
            const double armijo = o.accept_rule == 1 ? 1e-4 * alpha * gd : 0.0;
            if (Et <= E + armijo + noise) {
                accepted = true;
                break;
            }
            alpha *= o.line_search_shrink;
        }
        if (!accepted) {
            report();
            return finish(2);
        }
        step.step = alpha;
        report();
        LPG_CUDA(cudaMemcpyAsync(x, trial, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
}

namespace {

// The adjoint solve of StaticEquilibriumResponse (static_equilibrium_response.cpp:43-68): the
// Exact FP64 Hessian K at u*, then mask K lambda = mask dL/du by PCG with FP64 refinement and
// the reference's residual check. Returns lambda (device) and u* (device) through out-params.
void adjoint_solve(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                   int precision, double cg_tolerance, const double** u_dev, double** lam_dev,
                   const lpg_newton_terms* terms = nullptr) {
    if (precision != LPG_PRECISION_F64 && precision != LPG_PRECISION_MIXED) fail(LPG_EINVAL, "invalid precision");
    if (!(cg_tolerance > 0) || !std::isfinite(cg_tolerance)) fail(LPG_EINVAL, "adjoint: cg_tolerance must be positive");
    Potential pot;
    build_potential(h, terms, pot);
    Solver S(h, &pot);
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
    const size_t nv = h.plan.sell_values();
    double* K64 = h.s_hess64.as<double>(std::max<size_t>(nv, 1));
    LPG_CUDA(cudaMemsetAsync(K64, 0, nv * sizeof(double), s));
    eval_elastic_async(h, terms, u, nullptr, LPG_HESSIAN_EXACT, LPG_PRECISION_F64, kLayoutSell, K64);
    raise_status(h.take_status());
    S.compose_hessian(K64);
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

void adjoint_lambda(lpg_fem& h, const lpg_newton_terms* terms, const double* u_star, const double* dLdu,
                    const int32_t* fixed, int nfixed, int io_mem, int precision, double cg_tolerance, double* lambda_out) {
    const double* u = nullptr;
    double* lam = nullptr;
    adjoint_solve(h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, &u, &lam, terms);
    copy_lambda(h, lam, io_mem, lambda_out);
    LPG_CUDA(cudaStreamSynchronize(h.stream));
}

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

void adjoint_fp(lpg_fem& h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed, int io_mem,
                int precision, double cg_tolerance, int per_element, double* dFp, double* lambda_out) {
    const double* u = nullptr;
    double* lam = nullptr;
    adjoint_solve(h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, &u, &lam);
    cudaStream_t s = h.stream;
    const size_t T = static_cast<size_t>(h.dm.T);
    // dFp = -(dg/dFp)^T lambda.
    double* pe = h.d_vjp.as<double>(std::max<size_t>(9 * T, 9));
    launch_fp_vjp(h.dm, u, lam, pe, h.d_status.as<unsigned>(1), s);
    std::vector<double> host;
    if (per_element) {
        host.resize(9 * T);
        if (T) LPG_CUDA(cudaMemcpyAsync(host.data(), pe, 9 * T * sizeof(double), cudaMemcpyDeviceToHost, s));
    } else {
        const int nb = static_cast<int>(std::min<size_t>(1024, (T + 4095) / 4096));
        double* part = h.d_block.as<double>(std::max(9 * nb, 9));
        double* res = h.d_alpha.as<double>(9);
        launch_sum_cols9(pe, static_cast<int>(T), part, nb, res, s);
        host.resize(9);
        LPG_CUDA(cudaMemcpyAsync(host.data(), res, 9 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    raise_status(h.take_status());
    for (double& v : host) v = -v;
    if (io_mem == LPG_MEM_DEVICE) {
        if (!host.empty()) LPG_CUDA(cudaMemcpyAsync(dFp, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    } else {
        std::copy(host.begin(), host.end(), dFp);
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

// ---------------------------------------------------------------------------
// Batched Newton: many independent meshes as one flat element / vertex stream. The meshes are
// contiguous vertex and element ranges of one handle; assembly, SpMV and the vector kernels run
// once over the union, while every per-mesh quantity (energy, gradient norms, PCG scalars,
// feasible step, line search) is a segmented, fixed-order reduction over its mesh's range.
// ---------------------------------------------------------------------------
namespace {

// One block per mesh over the DOFs [3 voff[m], 3 voff[m+1]): out[4m..] = {sum w a b, sum w a^2,
// max w |a|, sum w b^2} with w = mask (1 where mask is null) and b = 0 where b is null.
__global__ void __launch_bounds__(256) seg_stats(const double* __restrict__ a, const double* __restrict__ b,
                                                 const double* __restrict__ mask, const int* __restrict__ voff,
                                                 double* __restrict__ out) {
    __shared__ double sh[4][8];
    const int m = blockIdx.x;
    const size_t lo = 3 * static_cast<size_t>(voff[m]), hi = 3 * static_cast<size_t>(voff[m + 1]);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double w = mask ? mask[i] : 1.0, av = a[i], bv = b ? b[i] : 0.0;
        s0 += w * av * bv;
        s1 += w * av * av;
        s2 = fmax(s2, w * fabs(av));
        s3 += w * bv * bv;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, off);
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        s2 = fmax(s2, __shfl_xor_sync(0xffffffffu, s2, off));
        s3 += __shfl_xor_sync(0xffffffffu, s3, off);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[0][w] = s0, sh[1][w] = s1, sh[2][w] = s2, sh[3][w] = s3;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[4] = {0, 0, 0, 0};
        for (int k = 0; k < (blockDim.x >> 5); ++k) {
            r[0] += sh[0][k];
            r[1] += sh[1][k];
            r[2] = fmax(r[2], sh[2][k]);
            r[3] += sh[3][k];
        }
        for (int k = 0; k < 4; ++k) out[4 * m + k] = r[k];
    }
}

// One block per mesh over its elements [eoff[m], eoff[m+1]): sum (min_mode 0) or minimum
// starting from 1 (min_mode 1) of a per-element value.
__global__ void __launch_bounds__(256) seg_elem(const double* __restrict__ x, const int* __restrict__ eoff,
                                                int min_mode, double* __restrict__ out) {
    __shared__ double sh[8];
    const int m = blockIdx.x;
    double v = min_mode ? 1.0 : 0.0;
    for (int e = eoff[m] + threadIdx.x; e < eoff[m + 1]; e += blockDim.x) v = min_mode ? fmin(v, x[e]) : v + x[e];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, v, off);
        v = min_mode ? fmin(v, t) : v + t;
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = min_mode ? 1.0 : 0.0;
        for (int k = 0; k < (blockDim.x >> 5); ++k) r = min_mode ? fmin(r, sh[k]) : r + sh[k];
        out[m] = r;
    }
}

// t = x + alpha[mesh] d and diff = t - x (the step actually taken) per DOF.
__global__ void seg_axpy(const double* __restrict__ x, const double* __restrict__ alpha, const int* __restrict__ mov,
                         const double* __restrict__ d, double* __restrict__ t, double* __restrict__ diff, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double v = x[i] + alpha[mov[i / 3]] * d[i];
    t[i] = v;
    diff[i] = v - x[i];
}
// x = src on the DOFs of the meshes with take[mesh] != 0.
__global__ void seg_take(double* __restrict__ x, const double* __restrict__ src, const int* __restrict__ take,
                         const int* __restrict__ mov, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n && take[mov[i / 3]]) x[i] = src[i];
}
// b = -mask g on the active meshes, 0 elsewhere (an inactive mesh gets a zero direction).
__global__ void seg_rhs(const double* __restrict__ g, const double* __restrict__ mask, const int* __restrict__ act,
                        const int* __restrict__ mov, double* __restrict__ b, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n) b[i] = act[mov[i / 3]] ? -mask[i] * g[i] : 0.0;
}

// Per-mesh PCG state (struct of arrays over the meshes).
struct BatchPcg {
    double *rz, *rr, *bb, *tol2, *alpha, *beta;
    int *done, *iters, *brk;
    int max_iters;
};

// r = b, x = 0, z = M^-1 r, p_old = 0 and the per-row r.z, r.r.
template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_b_init(const R* __restrict__ b, const R* __restrict__ dinv, R* x, R* r,
                                                       R* z, R* p_old, int V, double* __restrict__ rowdot2) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const size_t o = 4 * static_cast<size_t>(v);
    R rv[4], zv[3];
    ld4(b + o, rv);
    apply_dinv(dinv + 12 * static_cast<size_t>(v), rv, zv);
    st4(x + o, R(0), R(0), R(0));
    st4(r + o, rv[0], rv[1], rv[2]);
    st4(z + o, zv[0], zv[1], zv[2]);
    st4(p_old + o, R(0), R(0), R(0));
    double rz = 0, rr = 0;
    for (int i = 0; i < 3; ++i) {
        rz += static_cast<double>(rv[i]) * zv[i];
        rr += static_cast<double>(rv[i]) * rv[i];
    }
    rowdot2[2 * static_cast<size_t>(v)] = rz;
    rowdot2[2 * static_cast<size_t>(v) + 1] = rr;
}

// Sums per mesh of n interleaved per-row values (rows [voff[m], voff[m+1])), fixed order.
template <int K>
__device__ __forceinline__ void seg_rows(const double* __restrict__ rd, const int* __restrict__ voff, double* res) {
    __shared__ double sh[K][8];
    const int m = blockIdx.x;
    double v[K];
    for (int k = 0; k < K; ++k) v[k] = 0;
    for (int r = voff[m] + threadIdx.x; r < voff[m + 1]; r += blockDim.x)
        for (int k = 0; k < K; ++k) v[k] += rd[K * static_cast<size_t>(r) + k];
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) {
            double t = 0;
            for (int w = 0; w < (blockDim.x >> 5); ++w) t += sh[k][w];
            res[k] = t;
        }
}

__global__ void __launch_bounds__(256) pcg_b_start(BatchPcg st, const double* __restrict__ rowdot2,
                                                   const int* __restrict__ voff, const double* __restrict__ tol,
                                                   const int* __restrict__ act) {
    double res[2];
    seg_rows<2>(rowdot2, voff, res);
    if (threadIdx.x != 0) return;
    const int m = blockIdx.x;
    st.rz[m] = res[0];
    st.rr[m] = res[1];
    st.bb[m] = res[1];
    st.tol2[m] = tol[m] * tol[m] * res[1];
    st.beta[m] = 0;
    st.alpha[m] = 0;
    st.iters[m] = 0;
    st.brk[m] = 0;
    st.done[m] = (!act[m] || res[1] == 0.0 || st.max_iters <= 0) ? 1 : 0;
}

// Ap = mask (K p) with p = z + beta[mesh] p_old formed on the fly (written to p_new), and the
// per-row p.Ap; the sliced-ELL traversal of spmv_sell, one lane per row.
template <typename R>
__global__ void __launch_bounds__(kThreads, (SpmvCfg<R, 0>::minb))
    spmv_sell_batch(const DevMesh m, const R* __restrict__ val, const R* __restrict__ z, const R* __restrict__ p_old,
                    const R* __restrict__ mask, R* __restrict__ y, R* __restrict__ p_new, BatchPcg st,
                    const int* __restrict__ mov, double* __restrict__ rowdot) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= m.n_sell) return;
    const int row = __ldg(m.sell_row + 32 * static_cast<size_t>(c) + lane);
    const int mesh = row >= 0 ? __ldg(mov + row) : 0;
    const bool live = row >= 0 && !st.done[mesh];
    // A chunk whose rows all belong to finished meshes does nothing: their products, p and
    // row dots are read by no one (the update and the per-mesh reductions skip finished meshes),
    // so the lockstep iterations after most meshes have converged cost only the live chunks.
    if (!__any_sync(0xffffffffu, live)) return;
    const R beta = live ? static_cast<R>(st.beta[mesh]) : R(0);
    const int s0 = __ldg(m.sell_ptr + c);
    const int width = (__ldg(m.sell_ptr + c + 1) - s0) >> 5;
    const int* cp = m.sell_col + s0 + lane;
    const R* vp = val + 9 * static_cast<size_t>(s0) + lane;
    R a0 = 0, a1 = 0, a2 = 0;
    // A block's rows and columns belong to one mesh, so the row's beta applies to its columns.
    auto gather = [&](size_t col, R xv[3]) {
        R xz[3], xp[3];
        ld3<4>(z, col, xz);
        ld3<4>(p_old, col, xp);
#pragma unroll
        for (int i = 0; i < 3; ++i) xv[i] = xz[i] + beta * xp[i];
    };
#pragma unroll (SpmvCfg<R, 0>::unroll)
    for (int q = 0; q < width; ++q) {
        R xv[3];
        gather(static_cast<size_t>(__ldg(cp + 32 * q)), xv);
        const R* vq = vp + 288 * static_cast<size_t>(q);
        R kv[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) kv[e] = __ldg(vq + 32 * e);
        a0 += kv[0] * xv[0] + kv[1] * xv[1] + kv[2] * xv[2];
        a1 += kv[3] * xv[0] + kv[4] * xv[1] + kv[5] * xv[2];
        a2 += kv[6] * xv[0] + kv[7] * xv[1] + kv[8] * xv[2];
    }
    const int b0 = __ldg(m.sell_bptr + c);
    const int bwidth = (__ldg(m.sell_bptr + c + 1) - b0) >> 5;
    const int2* bp = m.sell_bref + b0 + lane;
#pragma unroll (SpmvCfg<R, 0>::unroll)
    for (int q = 0; q < bwidth; ++q) {
        const int2 ref = __ldg(bp + 32 * q);
        R xv[3];
        gather(static_cast<size_t>(ref.y), xv);
        const R* vq = val + static_cast<size_t>(ref.x);
        R kv[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) kv[e] = __ldg(vq + 32 * e);
        a0 += kv[0] * xv[0] + kv[3] * xv[1] + kv[6] * xv[2];
        a1 += kv[1] * xv[0] + kv[4] * xv[1] + kv[7] * xv[2];
        a2 += kv[2] * xv[0] + kv[5] * xv[1] + kv[8] * xv[2];
    }
    if (row < 0) return;
    const size_t o = static_cast<size_t>(row);
    R mv[3], xz[3], xp[3];
    ld3<4>(mask, o, mv);
    ld3<4>(z, o, xz);
    ld3<4>(p_old, o, xp);
    const R yv[3] = {mv[0] * a0, mv[1] * a1, mv[2] * a2};
    st3<4, R>(y, o, yv[0], yv[1], yv[2]);
    R pv[3];
    double dot = 0;
    for (int i = 0; i < 3; ++i) {
        pv[i] = xz[i] + beta * xp[i];
        dot += static_cast<double>(pv[i]) * static_cast<double>(yv[i]);
    }
    st3<4, R>(p_new, o, pv[0], pv[1], pv[2]);
    rowdot[o] = live ? dot : 0.0;
}

__global__ void __launch_bounds__(256) pcg_b_alpha(BatchPcg st, const double* __restrict__ rowdot,
                                                   const int* __restrict__ voff) {
    const int m = blockIdx.x;
    if (st.done[m]) return;
    double res[1];
    seg_rows<1>(rowdot, voff, res);
    if (threadIdx.x != 0) return;
    const double v = res[0];
    if (!(v > 0.0) || !isfinite(v)) {
        st.brk[m] = 1;
        st.done[m] = 1;
        st.alpha[m] = 0;
    } else {
        st.alpha[m] = st.rz[m] / v;
    }
}

template <typename R>
__global__ void __launch_bounds__(kThreads) pcg_b_update(BatchPcg st, const int* __restrict__ mov,
                                                         const R* __restrict__ dinv, R* x, R* r, R* z,
                                                         const R* __restrict__ p, const R* __restrict__ Ap, int V,
                                                         double* __restrict__ rowdot2) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int mesh = __ldg(mov + v);
    if (st.done[mesh]) {
        rowdot2[2 * static_cast<size_t>(v)] = 0;
        rowdot2[2 * static_cast<size_t>(v) + 1] = 0;
        return;
    }
    const R alpha = static_cast<R>(st.alpha[mesh]);
    const size_t o = 4 * static_cast<size_t>(v);
    R xv[4], pv[4], rv[4], av[4], zv[3];
    ld4c(x + o, xv);
    ld4(p + o, pv);
    ld4c(r + o, rv);
    ld4(Ap + o, av);
    for (int i = 0; i < 3; ++i) {
        xv[i] += alpha * pv[i];
        rv[i] = rv[i] - alpha * av[i];
    }
    apply_dinv(dinv + 12 * static_cast<size_t>(v), rv, zv);
    st4(x + o, xv[0], xv[1], xv[2]);
    st4(r + o, rv[0], rv[1], rv[2]);
    st4(z + o, zv[0], zv[1], zv[2]);
    double rz = 0, rr = 0;
    for (int i = 0; i < 3; ++i) {
        rz += static_cast<double>(rv[i]) * zv[i];
        rr += static_cast<double>(rv[i]) * rv[i];
    }
    rowdot2[2 * static_cast<size_t>(v)] = rz;
    rowdot2[2 * static_cast<size_t>(v) + 1] = rr;
}

__global__ void __launch_bounds__(256) pcg_b_beta(BatchPcg st, const double* __restrict__ rowdot2,
                                                  const int* __restrict__ voff) {
    const int m = blockIdx.x;
    if (st.done[m]) return;
    double res[2];
    seg_rows<2>(rowdot2, voff, res);
    if (threadIdx.x != 0) return;
    const double a = res[0], b = res[1];
    st.iters[m] += 1;
    st.rr[m] = b;
    if (b <= st.tol2[m] || st.iters[m] >= st.max_iters || !isfinite(b)) {
        st.done[m] = 1;
    } else {
        st.beta[m] = a / st.rz[m];
        st.rz[m] = a;
    }
}

// Device arrays of one batched solve.
// Skip flags of the two cluster plans from the per-mesh states (2 = finished): a cluster's rows
// all belong to the mesh of its first row (meshes are disconnected, clusters grow through
// vertex adjacency).
__global__ void cluster_skip_kernel(const int* __restrict__ row_ptr, const int* __restrict__ rows, int ncl,
                                    const int* __restrict__ mov, const int* __restrict__ mstate,
                                    unsigned char* __restrict__ skip) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncl) return;
    const int r0 = __ldg(row_ptr + c);
    skip[c] = (__ldg(row_ptr + c + 1) > r0 && mstate[__ldg(mov + __ldg(rows + r0))] == 2) ? 1 : 0;
}

struct BatchDev {
    int M = 0;
    int *voff = nullptr, *eoff = nullptr, *mov = nullptr, *emesh = nullptr;
    int *act = nullptr, *take = nullptr, *exact = nullptr;
    unsigned char *tc_skip = nullptr, *cl_skip = nullptr;
    double *stats = nullptr, *esum = nullptr, *fdot = nullptr, *amin = nullptr, *alpha = nullptr, *tol = nullptr;
    double *rowdot = nullptr, *rowdot2 = nullptr, *elem = nullptr;
    BatchPcg pcg{};
};

struct BatchSolver {
    lpg_fem& h;
    BatchDev& d;
    cudaStream_t s;
    size_t n;
    int V, M;
    BatchSolver(lpg_fem& hh, BatchDev& dd)
        : h(hh), d(dd), s(hh.stream), n(3 * static_cast<size_t>(hh.dm.V)), V(hh.dm.V), M(dd.M) {}

    template <typename T> void down(std::vector<T>& v, const T* p, size_t count) {
        v.resize(count);
        if (count) LPG_CUDA(cudaMemcpyAsync(v.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
        LPG_CUDA(cudaStreamSynchronize(s));
    }
    template <typename T> void up(T* p, const std::vector<T>& v) {
        if (!v.empty()) LPG_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    // Per-mesh {sum w a b, sum w a^2, max w|a|, sum w b^2}.
    std::vector<double> stats(const double* a, const double* b, const double* mask) {
        seg_stats<<<M, 256, 0, s>>>(a, b, mask, d.voff, d.stats);
        LPG_CUDA(cudaGetLastError());
        std::vector<double> r;
        down(r, d.stats, 4 * static_cast<size_t>(M));
        return r;
    }
    // Per-mesh energy at x: element energies summed per mesh, minus f . x.
    std::vector<double> energies(const double* x, const double* f, double* g, int hk, int precision, void* K) {
        h.eval_async(x, g, hk, precision, kLayoutSell, K, d.elem, nullptr, nullptr, d.emesh, d.exact, d.tc_skip,
                     d.cl_skip);
        seg_elem<<<M, 256, 0, s>>>(d.elem, d.eoff, 0, d.esum);
        LPG_CUDA(cudaGetLastError());
        raise_status(h.take_status());
        std::vector<double> e;
        down(e, d.esum, M);
        if (f) {
            const auto fx = stats(x, f, nullptr);
            for (int m = 0; m < M; ++m) e[m] -= fx[4 * m];
        }
        return e;
    }

    struct PcgOut {
        int64_t iters = 0;
        std::vector<int> breakdown;
    };

    template <typename R>
    void enqueue(cudaStream_t gs, const R* K, const R* dinv, const R* mask4, R* x, R* r, R* z, R* pA, R* pB, R* Ap,
                 int pairs) {
        const int sg = std::max(1, (h.dm.n_sell + 7) / 8), vg = grid(static_cast<size_t>(V));
        for (int i = 0; i < pairs; ++i)
            for (int half = 0; half < 2; ++half) {
                R* po = half ? pB : pA;
                R* pn = half ? pA : pB;
                spmv_sell_batch<R><<<sg, kThreads, 0, gs>>>(h.dm, K, z, po, mask4, Ap, pn, d.pcg, d.mov, d.rowdot);
                pcg_b_alpha<<<M, 256, 0, gs>>>(d.pcg, d.rowdot, d.voff);
                pcg_b_update<R><<<vg, kThreads, 0, gs>>>(d.pcg, d.mov, dinv, x, r, z, pn, Ap, V, d.rowdot2);
                pcg_b_beta<<<M, 256, 0, gs>>>(d.pcg, d.rowdot2, d.voff);
            }
    }

    // Solves mask K x = mask b per active mesh (tolerance tol[m] relative to ||b_m||): inner PCG in
    // precision R on Kin, FP64 refinement against Kres; the iterations replay a cached graph.
    template <typename R>
    PcgOut pcg(const void* Kin, const R* dinv, const void* Kres, bool res64, const double* mask, const double* b64,
               double* x64, const std::vector<double>& tol, std::vector<int> act, int max_iters, int max_refine) {
        PcgOut out;
        out.breakdown.assign(M, 0);
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
        LPG_CUDA(cudaMemsetAsync(x64, 0, n * sizeof(double), s));
        LPG_CUDA(cudaMemcpyAsync(r64, b64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        const auto bs = stats(b64, nullptr, mask);
        std::vector<double> bnorm(M), rnorm(M);
        bool any = false;
        for (int m = 0; m < M; ++m) {
            bnorm[m] = rnorm[m] = std::sqrt(bs[4 * m + 1]);
            act[m] = act[m] && bnorm[m] > 0;
            any = any || act[m];
        }
        if (!any) return out;
        pad_rhs<R><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(mask, mask, mask4, V);
        constexpr int kPairs = 16;
        const void* key[12] = {Kin, dinv, mask4, x, r, z, pA, pB, Ap, d.rowdot, d.pcg.rz,
                               reinterpret_cast<const void*>((static_cast<size_t>(d.pcg.max_iters) << 40) ^
                                                             (sizeof(R) * 1000003u + V + 7919u * static_cast<size_t>(M)))};
        bool same = h.batch_graph != nullptr;
        for (int i = 0; i < 12 && same; ++i) same = h.batch_graph_key[i] == key[i];
        cudaStream_t gs = h.own_stream;
        if (!same) {
            if (h.batch_graph) {
                cudaGraphExecDestroy(h.batch_graph);
                h.batch_graph = nullptr;
            }
            cudaGraph_t g = nullptr;
            LPG_CUDA(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
            enqueue<R>(gs, static_cast<const R*>(Kin), dinv, mask4, x, r, z, pA, pB, Ap, kPairs);
            LPG_CUDA(cudaStreamEndCapture(gs, &g));
            LPG_CUDA(cudaGraphInstantiate(&h.batch_graph, g, 0));
            cudaGraphDestroy(g);
            for (int i = 0; i < 12; ++i) h.batch_graph_key[i] = key[i];
        }
        cudaEvent_t ev;
        LPG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        std::vector<double> itol(M);
        std::vector<int> done, iters, brk;
        int used = 0;
        for (int ref = 0; ref <= max_refine; ++ref) {
            for (int m = 0; m < M; ++m)
                itol[m] = act[m] ? std::min(0.5, std::max(tol[m] * bnorm[m] / rnorm[m], sizeof(R) == 4 ? 1e-6 : 1e-14))
                                 : 1.0;
            up(d.tol, itol);
            up(d.act, act);
            pad_rhs<R><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(r64, mask, bR, V);
            pcg_b_init<R><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(bR, dinv, x, r, z, pA, V, d.rowdot2);
            pcg_b_start<<<M, 256, 0, s>>>(d.pcg, d.rowdot2, d.voff, d.tol, d.act);
            LPG_CUDA(cudaGetLastError());
            for (;;) {
                LPG_CUDA(cudaEventRecord(ev, s));
                LPG_CUDA(cudaStreamWaitEvent(gs, ev, 0));
                LPG_CUDA(cudaGraphLaunch(h.batch_graph, gs));
                LPG_CUDA(cudaEventRecord(ev, gs));
                LPG_CUDA(cudaStreamWaitEvent(s, ev, 0));
                down(done, d.pcg.done, M);
                if (std::all_of(done.begin(), done.end(), [](int v) { return v != 0; })) break;
            }
            down(iters, d.pcg.iters, M);
            down(brk, d.pcg.brk, M);
            int mx = 0;
            for (int m = 0; m < M; ++m) {
                if (!act[m]) continue;
                mx = std::max(mx, iters[m]);
                if (brk[m]) out.breakdown[m] = 1;
            }
            used += mx;
            out.iters += mx;
            add_kernel<R><<<grid(n), kThreads, 0, s>>>(x64, x, n);
            if (res64)
                spmv_sell<double, double, double, false, false, 3>
                    <<<std::max(1, (h.dm.n_sell + 7) / 8), kThreads, 0, s>>>(h.dm, static_cast<const double*>(Kres), x64,
                                                                            nullptr, mask, y64, nullptr, nullptr, nullptr);
            else
                spmv_sell<float, double, double, false, false, 3>
                    <<<std::max(1, (h.dm.n_sell + 7) / 8), kThreads, 0, s>>>(h.dm, static_cast<const float*>(Kres), x64,
                                                                            nullptr, mask, y64, nullptr, nullptr, nullptr);
            residual_kernel<<<grid(n), kThreads, 0, s>>>(b64, y64, mask, r64, n);
            LPG_CUDA(cudaGetLastError());
            const auto rs = stats(r64, nullptr, mask);
            any = false;
            for (int m = 0; m < M; ++m) {
                rnorm[m] = std::sqrt(rs[4 * m + 1]);
                act[m] = act[m] && !out.breakdown[m] && rnorm[m] > tol[m] * bnorm[m] && std::isfinite(rnorm[m]);
                any = any || act[m];
            }
            if (!any || used >= max_iters) break;
        }
        cudaEventDestroy(ev);
        return out;
    }
};

} // namespace

void batch_newton_solve(lpg_fem& h, int M, const int32_t* voff_h, const int32_t* eoff_h, const int32_t* fixed,
                        int nfixed, const double* f_ext, const double* x0, int io_mem, const lpg_newton_options& o,
                        double* x_out, lpg_batch_mesh_result* per_mesh, lpg_newton_result* total) {
    const int V = h.dm.V, T = h.dm.T;
    if (M <= 0 || !voff_h || !eoff_h || !per_mesh) fail(LPG_EINVAL, "batch_newton_solve: invalid mesh offsets");
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
    if (!(o.exact_below >= 0.0) || !std::isfinite(o.exact_below))
        fail(LPG_EINVAL, "newton_solve: exact_below must be finite and non-negative");
    if (h.dm.K != 4) fail(LPG_EINVAL, "batch_newton_solve: batched solves are available for tet meshes only");
    // Meshes: contiguous vertex and element ranges; every element inside its mesh's vertices.
    if (voff_h[0] != 0 || voff_h[M] != V || eoff_h[0] != 0 || eoff_h[M] != T)
        fail(LPG_EINVAL, "batch_newton_solve: mesh offsets must start at 0 and end at the vertex / element counts");
    for (int m = 0; m < M; ++m)
        if (voff_h[m + 1] < voff_h[m] || eoff_h[m + 1] < eoff_h[m])
            fail(LPG_EINVAL, "batch_newton_solve: mesh offsets must be non-decreasing");
    cudaStream_t s = h.stream;
    {
        std::vector<int4> tv(static_cast<size_t>(T));
        if (T) LPG_CUDA(cudaMemcpyAsync(tv.data(), h.dm.tets, T * sizeof(int4), cudaMemcpyDeviceToHost, s));
        LPG_CUDA(cudaStreamSynchronize(s));
        for (int m = 0; m < M; ++m)
            for (int e = eoff_h[m]; e < eoff_h[m + 1]; ++e) {
                const int vs[4] = {tv[e].x, tv[e].y, tv[e].z, tv[e].w};
                for (int v : vs)
                    if (v < voff_h[m] || v >= voff_h[m + 1])
                        fail(LPG_EINVAL, "batch_newton_solve: element " + std::to_string(e) +
                                             " references a vertex outside its mesh");
            }
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    const size_t n = 3 * static_cast<size_t>(V);
    BatchDev d;
    d.M = M;
    d.voff = h.bt_int[0].as<int>(M + 1);
    d.eoff = h.bt_int[1].as<int>(M + 1);
    d.mov = h.bt_int[2].as<int>(std::max(V, 1));
    d.act = h.bt_int[3].as<int>(M);
    d.take = h.bt_int[4].as<int>(M);
    d.emesh = h.bt_int[6].as<int>(std::max(T, 1));
    d.exact = h.bt_int[7].as<int>(M);
    d.tc_skip = h.bt_skip[0].as<unsigned char>(static_cast<size_t>(std::max(h.dm.tc_ncl, 1)));
    d.cl_skip = h.bt_skip[1].as<unsigned char>(static_cast<size_t>(std::max(h.dm.ncl, 1)));
    int* pcg_ints = h.bt_int[5].as<int>(3 * static_cast<size_t>(M) + 1);
    d.pcg.done = pcg_ints;
    d.pcg.iters = pcg_ints + M + 1;
    d.pcg.brk = pcg_ints + 2 * M + 1;
    double* dbl = h.bt_dbl[0].as<double>(16 * static_cast<size_t>(M));
    d.stats = dbl;
    d.esum = dbl + 4 * M;
    d.fdot = dbl + 5 * M;
    d.amin = dbl + 6 * M;
    d.alpha = dbl + 7 * M;
    d.tol = dbl + 8 * M;
    d.pcg.rz = dbl + 9 * M;
    d.pcg.rr = dbl + 10 * M;
    d.pcg.bb = dbl + 11 * M;
    d.pcg.tol2 = dbl + 12 * M;
    d.pcg.alpha = dbl + 13 * M;
    d.pcg.beta = dbl + 14 * M;
    d.rowdot = h.bt_dbl[1].as<double>(std::max(V, 1));
    d.rowdot2 = h.bt_dbl[2].as<double>(2 * static_cast<size_t>(std::max(V, 1)));
    d.elem = h.bt_dbl[3].as<double>(std::max(T, 1));
    d.pcg.max_iters = o.cg_max_iterations;
    std::vector<int> mov_h(static_cast<size_t>(V));
    for (int m = 0; m < M; ++m)
        for (int v = voff_h[m]; v < voff_h[m + 1]; ++v) mov_h[v] = m;
    BatchSolver B(h, d);
    B.up(d.voff, std::vector<int>(voff_h, voff_h + M + 1));
    B.up(d.eoff, std::vector<int>(eoff_h, eoff_h + M + 1));
    B.up(d.mov, mov_h);
    {
        std::vector<int> em(static_cast<size_t>(T));
        for (int m = 0; m < M; ++m)
            for (int e = eoff_h[m]; e < eoff_h[m + 1]; ++e) em[e] = m;
        B.up(d.emesh, em);
    }
    double* mask = h.s_mask.as<double>(std::max<size_t>(n, 1));
    make_mask(h, fixed, nfixed, mask);
    double* x = h.s_x.as<double>(std::max<size_t>(n, 1));
    double* g = h.s_g.as<double>(2 * std::max<size_t>(n, 1));
    double* rhs = g + std::max<size_t>(n, 1);
    double* dir = h.s_d.as<double>(std::max<size_t>(n, 1));
    double* trial = h.s_f.as<double>(3 * std::max<size_t>(n, 1));
    double* diff = trial + std::max<size_t>(n, 1);
    double* f = nullptr;
    const double* fsrc = f_ext ? h.stage_in(f_ext, io_mem, h.d_u2, n) : nullptr;
    if (fsrc) {
        f = trial + 2 * std::max<size_t>(n, 1);
        LPG_CUDA(cudaMemcpyAsync(f, fsrc, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    const double* x0d = h.stage_in(x0, io_mem, h.d_u, n);
    LPG_CUDA(cudaMemcpyAsync(x, x0d, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const bool f64 = o.precision == LPG_PRECISION_F64;
    const size_t hbytes = h.plan.sell_values() * (f64 ? 8 : 4);
    void* K = h.s_hess.ensure(std::max<size_t>(hbytes, 8));
    LPG_CUDA(cudaMemsetAsync(K, 0, hbytes, s));
    void* dinv = h.s_dinv.ensure(12 * static_cast<size_t>(std::max(V, 1)) * (f64 ? 8 : 4));
    const int nfeas = feasible_blocks(h.dm);
    double* bm = h.d_block.as<double>(std::max(nfeas, 1));
    double* al = h.d_alpha.as<double>(1);
    // Per-mesh state on the host.
    std::vector<int> status(M, -1), act(M, 1), iters(M, 0), take(M, 0), pending(M, 0);
    std::vector<double> E(M, 0), g2(M, 0), gmax(M, 0), g0(M, -1), secs(M, 0), alpha(M, 0), gd(M, 0);
    {
        std::vector<double> mh;
        B.down(mh, mask, n);
        for (int m = 0; m < M; ++m) {
            bool anyfree = false;
            for (size_t i = 3 * static_cast<size_t>(voff_h[m]); i < 3 * static_cast<size_t>(voff_h[m + 1]); ++i)
                anyfree = anyfree || mh[i] != 0;
            if (!anyfree) act[m] = 0; // nothing to solve: converged at x0
        }
    }
    lpg_newton_result R{};
    // Per-mesh Hessian kind: a mesh whose gradient has fallen to exact_below of its first one
    // switches to the Exact Hessian (its elements skip the projection's clamp).
    std::vector<int> exact(M, o.hessian == LPG_HESSIAN_EXACT ? 1 : 0);
    int it = 0;
    for (;; ++it) {
        // Per-mesh state of this iteration's evaluations: 0 projected, 1 exact, 2 finished (its
        // elements and clusters are skipped; its results were recorded when it finished).
        {
            std::vector<int> state(exact);
            for (int m = 0; m < M; ++m)
                if (status[m] >= 0) state[m] = 2;
            B.up(d.exact, state);
            if (h.dm.tc_ncl > 0)
                cluster_skip_kernel<<<grid(static_cast<size_t>(h.dm.tc_ncl)), kThreads, 0, s>>>(
                    h.dm.tc_row_ptr, h.dm.tc_rows, h.dm.tc_ncl, d.mov, d.exact, d.tc_skip);
            if (h.dm.ncl > 0)
                cluster_skip_kernel<<<grid(static_cast<size_t>(h.dm.ncl)), kThreads, 0, s>>>(
                    h.dm.cl_row_ptr, h.dm.cl_rows, h.dm.ncl, d.mov, d.exact, d.cl_skip);
            LPG_CUDA(cudaGetLastError());
        }
        bool all_exact = true;
        for (int m = 0; m < M; ++m) all_exact = all_exact && (exact[m] || !act[m]);
        const int hk = all_exact ? LPG_HESSIAN_EXACT : LPG_HESSIAN_PROJECTED;
        const std::vector<double> e = f64 ? B.energies(x, f, g, hk, LPG_PRECISION_F64, K)
                                          : B.energies(x, f, g, LPG_HESSIAN_NONE, LPG_PRECISION_F64, nullptr);
        if (f) load_gradient<<<grid(n), kThreads, 0, s>>>(g, f, n);
        const auto gs = B.stats(g, nullptr, mask);
        for (int m = 0; m < M; ++m) {
            if (status[m] >= 0) continue; // finished: skipped by this iteration's evaluation
            E[m] = e[m];
            g2[m] = std::sqrt(gs[4 * m + 1]);
            gmax[m] = gs[4 * m + 2];
            if (g0[m] < 0) g0[m] = g2[m];
            if (!act[m]) {
                status[m] = 0;
                secs[m] = elapsed();
                continue;
            }
            iters[m] = it;
            const bool conv = o.stop_rule == 0 ? gmax[m] <= o.gradient_tolerance : g2[m] <= o.gradient_tolerance * g0[m];
            if (conv || it == o.max_iterations) {
                status[m] = conv ? 0 : 1;
                act[m] = 0;
                secs[m] = elapsed();
            } else if (o.exact_below > 0 && g2[m] <= o.exact_below * g0[m]) {
                exact[m] = 1;
            }
        }
        if (std::none_of(act.begin(), act.end(), [](int v) { return v != 0; })) break;
        if (!f64) {
            // The flags of this iteration's start (d.exact), as the FP64 path uses.
            h.eval_async(x, nullptr, hk, LPG_PRECISION_MIXED, kLayoutSell, K, nullptr, nullptr, nullptr, d.emesh,
                         d.exact, d.tc_skip, d.cl_skip);
            raise_status(h.take_status());
        }
        // Descent directions: per-mesh PCG on the block-diagonal system, forcing term per mesh.
        B.up(d.act, act);
        seg_rhs<<<grid(n), kThreads, 0, s>>>(g, mask, d.act, d.mov, rhs, n);
        std::vector<double> tol(M, 1.0);
        for (int m = 0; m < M; ++m)
            if (act[m]) tol[m] = std::min(o.cg_tolerance, std::sqrt(g2[m] / g0[m]));
        BatchSolver::PcgOut po;
        if (f64) {
            block_jacobi<double, double><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(
                h.dm, static_cast<double*>(K), mask, static_cast<double*>(dinv), V);
            po = B.pcg<double>(K, static_cast<double*>(dinv), K, true, mask, rhs, dir, tol, act, o.cg_max_iterations, 0);
        } else {
            block_jacobi<float, float><<<grid(static_cast<size_t>(V)), kThreads, 0, s>>>(
                h.dm, static_cast<float*>(K), mask, static_cast<float*>(dinv), V);
            po = B.pcg<float>(K, static_cast<float*>(dinv), K, false, mask, rhs, dir, tol, act, o.cg_max_iterations, 3);
        }
        R.cg_iterations += po.iters;
        // A mesh whose direction is not a descent direction (negative curvature at the first PCG
        // step) takes the steepest-descent direction -g for this iteration.
        auto gds = B.stats(g, dir, mask);
        bool fallback = false;
        for (int m = 0; m < M; ++m) {
            take[m] = act[m] && !(gds[4 * m] < 0.0 && std::isfinite(gds[4 * m]));
            fallback = fallback || take[m];
        }
        if (fallback) {
            B.up(d.take, take);
            seg_take<<<grid(n), kThreads, 0, s>>>(dir, rhs, d.take, d.mov, n);
            gds = B.stats(g, dir, mask);
        }
        for (int m = 0; m < M; ++m) gd[m] = gds[4 * m];
        // Line search per mesh from its feasible step.
        launch_feasible(h.dm, x, dir, bm, nfeas, al, h.d_status.as<unsigned>(1), s, d.elem, d.emesh, d.exact);
        seg_elem<<<M, 256, 0, s>>>(d.elem, d.eoff, 1, d.amin);
        raise_status(h.take_status());
        std::vector<double> amin;
        B.down(amin, d.amin, M);
        for (int m = 0; m < M; ++m) {
            pending[m] = act[m];
            alpha[m] = act[m] ? amin[m] : 0.0;
        }
        for (int j = 0; j < o.max_line_search_steps; ++j) {
            if (std::none_of(pending.begin(), pending.end(), [](int v) { return v != 0; })) break;
            std::vector<double> a(M);
            for (int m = 0; m < M; ++m) a[m] = pending[m] ? alpha[m] : 0.0;
            B.up(d.alpha, a);
            seg_axpy<<<grid(n), kThreads, 0, s>>>(x, d.alpha, d.mov, dir, trial, diff, n);
            const auto mv = B.stats(diff, nullptr, nullptr);
            for (int m = 0; m < M; ++m)
                if (pending[m] && !(mv[4 * m + 2] > 0)) {
                    pending[m] = 0;
                    act[m] = 0;
                    status[m] = 2;
                    secs[m] = elapsed();
                }
            ++R.line_search_evaluations;
            std::vector<double> Et = B.energies(trial, f, nullptr, LPG_HESSIAN_NONE, LPG_PRECISION_F64, nullptr);
            for (int m = 0; m < M; ++m) {
                take[m] = 0;
                if (!pending[m]) continue;
                const double noise = 16.0 * kEps * std::max(1.0, std::abs(E[m]));
                const double armijo = o.accept_rule == 1 ? 1e-4 * alpha[m] * gd[m] : 0.0;
                if (Et[m] <= E[m] + armijo + noise) {
                    take[m] = 1;
                    pending[m] = 0;
                } else {
                    alpha[m] *= o.line_search_shrink;
                }
            }
            B.up(d.take, take);
            seg_take<<<grid(n), kThreads, 0, s>>>(x, trial, d.take, d.mov, n);
        }
        for (int m = 0; m < M; ++m)
            if (pending[m]) {
                act[m] = 0;
                status[m] = 2;
                secs[m] = elapsed();
            }
    }
    R.iterations = it;
    R.seconds = elapsed();
    int worst = 0;
    double esum = 0;
    for (int m = 0; m < M; ++m) {
        per_mesh[m].status = status[m] < 0 ? 1 : status[m];
        per_mesh[m].iterations = iters[m];
        per_mesh[m].energy = E[m];
        per_mesh[m].gradient_norm = o.stop_rule == 0 ? gmax[m] : g2[m];
        per_mesh[m].gradient_norm0 = g0[m];
        per_mesh[m].seconds = secs[m];
        worst = std::max(worst, per_mesh[m].status);
        esum += E[m];
    }
    R.status = worst;
    R.energy = esum;
    if (io_mem == LPG_MEM_DEVICE)
        LPG_CUDA(cudaMemcpyAsync(x_out, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        LPG_CUDA(cudaMemcpyAsync(x_out, x, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    LPG_CUDA(cudaStreamSynchronize(s));
    if (total) *total = R;
}

// ---------------------------------------------------------------------------
// Autotuner: times each launch variant of the cluster kernel (Exact Hessian + gradient, BSR),
// the PCG SpMV (the solvers' layout) and the eigenvalue clamp on this handle's mesh and keeps
// the fastest per precision. Inputs: the rest state u = 0 for the first two (their cost does
// not depend on the values), seeded symmetric 9x9 matrices for the clamp. Each timing is the
// mean of 3 launches after one warm-up, CUDA events on the handle's stream. Variants differ in
// register budget and unroll depth only, so the choice never changes a result.
// ---------------------------------------------------------------------------
namespace {
struct TuneTimer {
    cudaStream_t s;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    explicit TuneTimer(cudaStream_t st) : s(st) {
        LPG_CUDA(cudaEventCreate(&e0));
        LPG_CUDA(cudaEventCreate(&e1));
    }
    ~TuneTimer() {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    // Mean ms of `launch` over 3 runs after one warm-up; `prep` runs before each, untimed.
    template <class Prep, class Launch> double time(Prep prep, Launch launch) {
        double total = 0;
        for (int rep = 0; rep < 4; ++rep) {
            prep();
            LPG_CUDA(cudaEventRecord(e0, s));
            launch();
            LPG_CUDA(cudaEventRecord(e1, s));
            LPG_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            LPG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) total += ms;
        }
        return total / 3;
    }
};
int argmin(const double* ms, int n) {
    int best = 0;
    for (int v = 1; v < n; ++v)
        if (ms[v] < ms[best]) best = v;
    return best;
}

template <typename R> void tune_spmv(lpg_fem& h, TuneTimer& tt, const double* u0, double* ms) {
    Solver S(h);
    const int pi = sizeof(R) == 8 ? 0 : 1;
    const int prec = sizeof(R) == 8 ? LPG_PRECISION_F64 : LPG_PRECISION_MIXED;
    DeviceBuffer kb, vb, stb, pb;
    const size_t nv = h.plan.sell_values();
    R* K = kb.as<R>(nv);
    LPG_CUDA(cudaMemsetAsync(K, 0, nv * sizeof(R), h.stream));
    h.eval_async(u0, nullptr, LPG_HESSIAN_EXACT, prec, kLayoutSell, K, nullptr);
    h.take_status(); // timing only: input problems (e.g. bad theta) surface at evaluation
    const size_t n4 = 4 * static_cast<size_t>(std::max(h.dm.V, 1));
    R* vec = vb.as<R>(5 * n4);
    LPG_CUDA(cudaMemsetAsync(vec, 0, 5 * n4 * sizeof(R), h.stream));
    R *z = vec, *pA = vec + n4, *pB = vec + 2 * n4, *mask4 = vec + 3 * n4, *Ap = vec + 4 * n4;
    PcgState* st = stb.as<PcgState>(1);
    const int sg = S.spmv_grid();
    double* part = pb.as<double>(static_cast<size_t>(sg) + 64);
    auto prep = [&] { LPG_CUDA(cudaMemsetAsync(st, 0, sizeof(PcgState), h.stream)); };
    auto run = [&](auto kern) {
        return tt.time(prep, [&] { kern<<<sg, kThreads, 0, h.stream>>>(h.dm, K, z, pA, mask4, Ap, pB, st, part); });
    };
    ms[0] = run(spmv_sell<R, R, R, true, false, 4, 0>);
    ms[1] = run(spmv_sell<R, R, R, true, false, 4, 1>);
    ms[2] = run(spmv_sell<R, R, R, true, false, 4, 2>);
    h.tune.spmv[pi] = argmin(ms, kSpmvVariants);
}
} // namespace

void autotune(lpg_fem& h) {
    Tuning& t = h.tune;
    for (auto& a : t.ms)
        for (auto& b : a)
            for (double& c : b) c = std::nan("");
    t.cl[0] = t.cl[1] = t.spmv[0] = t.spmv[1] = t.clamp[0] = t.clamp[1] = 0;
    const DevMesh& m = h.dm;
    if (m.T == 0) {
        t.tuned = true;
        return;
    }
    cudaStream_t s = h.stream;
    TuneTimer tt(s);
    DeviceBuffer ub, gb;
    const size_t n = 3 * static_cast<size_t>(m.V);
    double* u0 = ub.as<double>(n);
    double* g = gb.as<double>(n);
    LPG_CUDA(cudaMemsetAsync(u0, 0, n * sizeof(double), s));
    const int precs[2] = {LPG_PRECISION_F64, LPG_PRECISION_MIXED};
    for (int pi = 0; pi < 2; ++pi) {
        const int prec = precs[pi];
        // Cluster kernel: E + gradient + Exact Hessian into BSR (the evaluation entry point's work).
        {
            DeviceBuffer hb;
            void* H = hb.ensure(9 * static_cast<size_t>(m.nnzb) * (pi == 0 ? 8 : 4));
            for (int v = 0; v < kClVariants; ++v) {
                t.cl[pi] = v;
                cudaEvent_t b = tt.e0, e = tt.e1;
                double total = 0;
                for (int rep = 0; rep < 4; ++rep) {
                    h.eval_async(u0, g, LPG_HESSIAN_EXACT, prec, LPG_LAYOUT_BSR, H, nullptr, b, e);
                    LPG_CUDA(cudaEventSynchronize(e));
                    float ms = 0;
                    LPG_CUDA(cudaEventElapsedTime(&ms, b, e));
                    if (rep > 0) total += ms;
                }
                t.ms[0][pi][v] = total / 3;
            }
            h.take_status(); // timing only: input problems (e.g. bad theta) surface at evaluation
            t.cl[pi] = argmin(t.ms[0][pi], kClVariants);
        }
        // PCG SpMV.
        if (pi == 0)
            tune_spmv<double>(h, tt, u0, t.ms[1][0]);
        else
            tune_spmv<float>(h, tt, u0, t.ms[1][1]);
        // Eigenvalue clamp (FP32 only has variants) on up to 2^17 seeded matrices.
        if (pi == 1) {
            const int ns = std::min(m.T, 1 << 17);
            DeviceBuffer pb, lb, cb;
            void* proj = pb.ensure(kProjRecord * static_cast<size_t>(ns) * sizeof(float));
            int* list = lb.as<int>(static_cast<size_t>(ns));
            unsigned* count = cb.as<unsigned>(1);
            const unsigned cnt = static_cast<unsigned>(ns);
            LPG_CUDA(cudaMemcpyAsync(count, &cnt, sizeof cnt, cudaMemcpyHostToDevice, s));
            for (int v = 0; v < kClampVariants; ++v)
                t.ms[2][1][v] = tt.time([&] { launch_clamp_sample(prec, proj, list, ns, s); },
                                        [&] { launch_clamp(prec, proj, list, count, ns, v, s); });
            t.clamp[1] = argmin(t.ms[2][1], kClampVariants);
        }
    }
    LPG_CUDA(cudaStreamSynchronize(s));
    t.tuned = true;
}

} // namespace lpg
