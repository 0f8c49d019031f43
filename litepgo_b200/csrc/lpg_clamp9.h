// Eigenvalue clamp of a symmetric 9x9 matrix, M -> V max(Lambda, 0) V^T, by the cyclic Jacobi
// method in a parallel (round-robin) ordering: the projected Hessian's clamp of a tet's tangent in
// the q basis (mesh_energy.cpp:16-27 clamps each element Hessian's eigenvalues at zero). One
// thread per matrix on the GPU (clamp_kernel); compiled for the host as well, where a test checks
// it against an eigensolver.
#pragma once
#ifndef __CUDA_ARCH__
#include <cmath>
#endif
#include <math.h>

#ifdef __CUDACC__
#define LPG_C9 __host__ __device__ __forceinline__
#else
#define LPG_C9 inline
#endif
// The math functions: CUDA's overloads on the device, the standard library's on the host.
#ifdef __CUDA_ARCH__
#define C9F(f) f
#else
#define C9F(f) std::f
#endif

namespace lpg {

// Packed upper-triangle index of a symmetric 9x9 matrix.
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr int sym9(int r, int c) {
    return r <= c ? r * 9 - (r * (r - 1)) / 2 + (c - r) : c * 9 - (c * (c - 1)) / 2 + (r - c);
}

template <typename R> struct Eps;
template <> struct Eps<double> { static constexpr double v = 2.220446049250313e-16; };
template <> struct Eps<float> { static constexpr float v = 1.1920929e-7f; };

template <typename R> LPG_C9 R c9_rsqrt(R x) {
#ifdef __CUDA_ARCH__
    return rsqrt(x);
#else
    return R(1) / std::sqrt(x);
#endif
}

// One round of parallel-ordered Jacobi on a symmetric 9x9 (round-robin ordering: in round r
// index r idles and the pairs (r+i, r-i) mod 9, i = 1..4, are disjoint, so a sweep of 9 rounds
// meets each of the 36 pairs once; Golub & Van Loan 8.5.3 and 8.6 for the ordering). The four
// rotations (Alg. 8.4.1 sym.schur2) are computed from the same A, i.e. four independent
// dependency chains, and applied together as A <- J^T A J with J the block rotation, then
// accumulated into V's columns.
// A is kept relabelled by the round, A_cur(i, j) = A((i + r) mod 9, (j + r) mod 9), so every
// round rotates the fixed pairs (1, 8), (2, 7), (3, 6), (4, 5) of A_cur with literal register
// indices; after the round A_cur is shifted by one label. The loop over rounds therefore stays
// a loop (a fully unrolled sweep of nine rounds overflows the instruction cache). V (register
// array, VREG) is shifted with A; V in shared memory is addressed with the round's offset.
template <typename R, bool VREG, typename VA>
LPG_C9 void jacobi_round(R (&A)[45], VA& V, const int rd) {
    R c[4], sn[4], t[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int P = k + 1, Q = 8 - k;
        // t = sign(tau) / (|tau| + sqrt(1 + tau^2)), tau = d / a2, written with one square
        // root and one division: t = +-|a2| / (|d| + sqrt(d^2 + a2^2)) (A is scaled to
        // max |entry| <= 1, so the squares cannot overflow); c = 1 / sqrt(1 + t^2), s = t c.
        const R apq = A[sym9(P, Q)];
        const R d = A[sym9(Q, Q)] - A[sym9(P, P)], a2 = R(2) * apq;
        const R num = d > R(0) ? a2 : (d < R(0) ? -a2 : C9F(fabs)(a2));
        const R den = C9F(fabs)(d) + C9F(sqrt)(d * d + a2 * a2);
        // den is 0 only when d = 0 and a2^2 underflows (FP32: |apq| below ~1e-23 of the largest
        // entry): the pair is already diagonal to far below the sweep threshold, so no rotation.
        t[k] = (apq == R(0) || !(den > R(0))) ? R(0) : num / den;
        c[k] = c9_rsqrt(R(1) + t[k] * t[k]);
        sn[k] = t[k] * c[k];
    }
    // Off-diagonal 2x2 blocks between pairs k < l: R_k^T A_kl R_l, R = [[c, s], [-s, c]].
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int l = k + 1; l < 4; ++l) {
            const int Pk = k + 1, Qk = 8 - k, Pl = l + 1, Ql = 8 - l;
            const R a = A[sym9(Pk, Pl)], b = A[sym9(Pk, Ql)];
            const R d = A[sym9(Qk, Pl)], e = A[sym9(Qk, Ql)];
            const R a1 = c[l] * a - sn[l] * b, b1 = sn[l] * a + c[l] * b;
            const R d1 = c[l] * d - sn[l] * e, e1 = sn[l] * d + c[l] * e;
            A[sym9(Pk, Pl)] = c[k] * a1 - sn[k] * d1;
            A[sym9(Pk, Ql)] = c[k] * b1 - sn[k] * e1;
            A[sym9(Qk, Pl)] = sn[k] * a1 + c[k] * d1;
            A[sym9(Qk, Ql)] = sn[k] * b1 + c[k] * e1;
        }
    // The idle index 0 against each pair, then each pair's own 2x2 block, then V.
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int P = k + 1, Q = 8 - k;
        const R a = A[sym9(0, P)], b = A[sym9(0, Q)];
        A[sym9(0, P)] = c[k] * a - sn[k] * b;
        A[sym9(0, Q)] = sn[k] * a + c[k] * b;
        const R apq = A[sym9(P, Q)];
        A[sym9(P, P)] -= t[k] * apq;
        A[sym9(Q, Q)] += t[k] * apq;
        A[sym9(P, Q)] = R(0);
        int vp_col = P, vq_col = Q;
        if constexpr (!VREG) {
            vp_col = P + rd >= 9 ? P + rd - 9 : P + rd;
            vq_col = Q + rd >= 9 ? Q + rd - 9 : Q + rd;
        }
#pragma unroll
        for (int x = 0; x < 9; ++x) {
            const R vp = V[9 * x + vp_col], vq = V[9 * x + vq_col];
            V[9 * x + vp_col] = c[k] * vp - sn[k] * vq;
            V[9 * x + vq_col] = sn[k] * vp + c[k] * vq;
        }
    }
    // Relabel for the next round: A_next(i, j) = A_cur(i + 1, j + 1) (indices mod 9).
    R B[45];
#pragma unroll
    for (int u = 0; u < 45; ++u) B[u] = A[u];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = i; j < 9; ++j) A[sym9(i, j)] = B[sym9((i + 1) % 9, (j + 1) % 9)];
    if constexpr (VREG) {
#pragma unroll
        for (int x = 0; x < 9; ++x) {
            const R v0 = V[9 * x];
#pragma unroll
            for (int j = 0; j < 8; ++j) V[9 * x + j] = V[9 * x + j + 1];
            V[9 * x + 8] = v0;
        }
    }
}

// The clamp of the packed upper triangle A (45 values), in place: A <- V max(Lambda, 0) V^T. V
// is 81 values of scratch (a register array when VREG; in FP64 on the GPU, shared memory).
template <typename R, bool VREG, typename VA>
LPG_C9 void clamp9_packed(R (&A)[45], VA& V) {
    R amax = 0;
#pragma unroll
    for (int t = 0; t < 45; ++t) amax = C9F(fmax)(amax, C9F(fabs)(A[t]));
    // Exact power-of-two scaling to max |entry| in [0.5, 1): no overflow in the rotations.
    int ex = 0;
    if (amax > R(0) && amax < R(INFINITY)) C9F(frexp)(amax, &ex);
    const R down = C9F(ldexp)(R(1), -ex), up = C9F(ldexp)(R(1), ex);
    R total = 0;
#pragma unroll
    for (int t = 0; t < 45; ++t) {
        A[t] *= down;
        total += A[t] * A[t];
    }
#pragma unroll
    for (int t = 0; t < 81; ++t) V[t] = (t % 10 == 0) ? R(1) : R(0);
    const R thr = R(16) * Eps<R>::v * Eps<R>::v * total;
#pragma unroll 1
    for (int sweep = 0; sweep < 20; ++sweep) {
        R off = 0;
#pragma unroll
        for (int r = 0; r < 9; ++r)
#pragma unroll
            for (int c = r + 1; c < 9; ++c) off += A[sym9(r, c)] * A[sym9(r, c)];
        if (!(off > thr)) break;
#pragma unroll 1
        for (int rd = 0; rd < 9; ++rd) jacobi_round<R, VREG>(A, V, rd);
    }
    R lam[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) lam[t] = C9F(fmax)(A[sym9(t, t)], R(0)) * up;
#pragma unroll
    for (int k = 0; k < 45; ++k) A[k] = R(0);
    // M+ = sum_t lam_t v_t v_t^T, one eigenvector column at a time (A reused as the sum).
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        R col[9];
#pragma unroll
        for (int r = 0; r < 9; ++r) col[r] = V[9 * r + t];
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const R lr = lam[t] * col[r];
#pragma unroll
            for (int c = r; c < 9; ++c) A[sym9(r, c)] += lr * col[c];
        }
    }
}


} // namespace lpg
