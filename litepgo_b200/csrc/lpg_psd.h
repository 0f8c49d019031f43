// Positive semi-definite projection of a dense symmetric N x N matrix, V max(L, 0) V^T, by the
// cyclic Jacobi eigenvalue method in the round-robin parallel ordering (Brent and Luk, "The
// solution of singular-value and symmetric eigenvalue problems on multiprocessor arrays", 1985):
// a sweep is N - 1 rounds of N / 2 disjoint plane rotations, each round computed from one state
// of the matrix, so a round is three data-parallel phases: the rotations, then every row of
// A J and V J (one row per lane), then every column of J^T (A J) (one column per lane). This is
// the projection HessianKind::Projected applies to every element's local Hessian
// (mesh_energy.cpp:16-27, there by Eigen's SelfAdjointEigenSolver).
//
// The functions are the tasks of one round; eigen() runs them for a team of lanes with a
// barrier after each phase (one warp per matrix on the GPU; plain loops on the host, where a
// test checks this code against an eigensolver).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define LPG_HD __host__ __device__ __forceinline__
#else
#define LPG_HD inline
#endif

namespace lpg {

LPG_HD double inv_sqrt(double x) {
#ifdef __CUDA_ARCH__
    return rsqrt(x);
#else
    return 1.0 / sqrt(x);
#endif
}

template <int N>
struct PsdJacobi {
    static_assert(N % 2 == 0 && N >= 2, "the round-robin ordering pairs an even number of indices");
    static constexpr int S = N + 1;       // row stride (a padded row staggers column reads across banks)
    static constexpr int kPairs = N / 2;  // rotations per round
    static constexpr int kRounds = N - 1; // rounds per sweep: every index pair once
    static constexpr int kCs = 2 * kPairs; // c, s per rotation
    static constexpr int kMaxSweeps = 30;
    // A sweep ends the iteration once the off-diagonal Frobenius norm is below 1e-14 of the
    // matrix's (the projection moves by at most that much: it is non-expansive).
    static constexpr double kOffTol2 = 1e-28;

    // Pair k of round r by the circle method: index N - 1 stays, the others rotate.
    LPG_HD static void pair(int r, int k, int& p, int& q) {
        int x, y;
        if (k == 0) {
            x = N - 1;
            y = r;
        } else {
            x = (r + k) % (N - 1);
            y = (r - k + (N - 1)) % (N - 1);
        }
        p = x < y ? x : y;
        q = x < y ? y : x;
    }

    // The rotation zeroing A(p, q): A' = J^T A J with J_pp = J_qq = c, J_pq = s, J_qp = -s,
    // t = tan phi the smaller root of t^2 + 2 t theta - 1 = 0, theta = (A_qq - A_pp) / (2 A_pq).
    LPG_HD static void rotation(const double* A, int r, int k, double* cs, int* pq) {
        int p, q;
        pair(r, k, p, q);
        const double apq = A[p * S + q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0) {
            const double th = (A[q * S + q] - A[p * S + p]) / (2.0 * apq);
            const double at = fabs(th);
            const double t = at > 1e150 ? 0.5 / th : copysign(1.0, th) / (at + sqrt(th * th + 1.0));
            c = inv_sqrt(t * t + 1.0);
            s = t * c;
        }
        cs[2 * k] = c;
        cs[2 * k + 1] = s;
        pq[2 * k] = p;
        pq[2 * k + 1] = q;
    }

    // One row (or column) of the round's rotations applied from the right (or left): the round's
    // pairs partition the indices, so the row's 2 kPairs entries are distinct and all of them are
    // loaded before any is stored (one load latency per row instead of one per pair).
    // x(m) addresses entry m of the row; zero_p / zero_q: set entries (row, q_k) / (row, p_k) of
    // the pair whose p_k / q_k is the row itself to zero (the entries the rotations annihilate).
    template <class Addr>
    LPG_HD static void rotate_line(const double* cs, const int* pq, Addr x, int row, bool zero) {
        double a[kPairs], b[kPairs], c[kPairs], s[kPairs];
        int p[kPairs], q[kPairs];
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
        for (int k = 0; k < kPairs; ++k) {
            p[k] = pq[2 * k];
            q[k] = pq[2 * k + 1];
            c[k] = cs[2 * k];
            s[k] = cs[2 * k + 1];
        }
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
        for (int k = 0; k < kPairs; ++k) {
            a[k] = *x(p[k]);
            b[k] = *x(q[k]);
        }
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
        for (int k = 0; k < kPairs; ++k) {
            *x(p[k]) = zero && row == q[k] ? 0.0 : c[k] * a[k] - s[k] * b[k];
            *x(q[k]) = zero && row == p[k] ? 0.0 : s[k] * a[k] + c[k] * b[k];
        }
    }

    // Row i of A J and of V J: columns p_k and q_k of every pair k.
    LPG_HD static void right(double* A, double* V, const double* cs, const int* pq, int i) {
        double* a = A + i * S;
        double* v = V + i * S;
        rotate_line(cs, pq, [a](int m) { return a + m; }, i, false);
        rotate_line(cs, pq, [v](int m) { return v + m; }, i, false);
    }

    // Column j of J^T (A J): rows p_k and q_k of every pair k; the entries the rotations
    // annihilate, (p_k, q_k) and (q_k, p_k), are set to zero.
    LPG_HD static void left(double* A, const double* cs, const int* pq, int j) {
        rotate_line(cs, pq, [A, j](int m) { return A + m * S + j; }, j, true);
    }

    // Entry (i, j), i <= j, of V diag(L) V^T for the clamped eigenvalues L (summed in index order).
    LPG_HD static double entry(const double* V, const double* L, int i, int j) {
        double sum = 0.0;
        for (int m = 0; m < N; ++m) sum = fma(V[i * S + m] * L[m], V[j * S + m], sum);
        return sum;
    }

    // The eigen-iteration by a team of lanes (lane(), size(), sync(), and sum(), which returns
    // the same total to every lane). A holds the symmetric matrix (row stride S) on entry and its
    // rotated diagonal form on exit; V (N S), cs (kCs), pq (N) and L (N) are scratch shared by the
    // team, and on exit V holds the eigenvectors (columns) and L the eigenvalues clamped at zero.
    // Returns the sweeps run; a non-finite A stops at once (its output is non-finite or zero,
    // and the caller flags it).
#ifdef __CUDACC__
#pragma nv_exec_check_disable
#endif
    template <class Team>
    LPG_HD static int eigen(const Team& team, double* A, double* V, double* cs, int* pq, double* L) {
        const int lane = team.lane(), nl = team.size();
        team.sync();
        double tot = 0.0;
        for (int t = lane; t < N * N; t += nl) {
            const int i = t / N, j = t - N * i;
            V[i * S + j] = i == j ? 1.0 : 0.0;
            const double a = A[i * S + j];
            tot = fma(a, a, tot);
        }
        tot = team.sum(tot);
        team.sync();
        int sweep = 0;
        for (; sweep < kMaxSweeps; ++sweep) {
            double off = 0.0;
            for (int t = lane; t < N * N; t += nl) {
                const int i = t / N, j = t - N * i;
                const double a = A[i * S + j];
                if (i != j) off = fma(a, a, off);
            }
            off = team.sum(off);
            if (!(off > kOffTol2 * tot)) break;
            for (int r = 0; r < kRounds; ++r) {
                for (int k = lane; k < kPairs; k += nl) rotation(A, r, k, cs, pq);
                team.sync();
                for (int i = lane; i < N; i += nl) right(A, V, cs, pq, i);
                team.sync();
                for (int j = lane; j < N; j += nl) left(A, cs, pq, j);
                team.sync();
            }
        }
        for (int m = lane; m < N; m += nl) {
            const double d = A[m * S + m];
            L[m] = d > 0.0 ? d : 0.0;
        }
        team.sync();
        return sweep;
    }
};

// Semi-definiteness test by LDL^T with diagonal pivoting on V (row-major N x N, overwritten):
// pivots above tol are eliminated; once none is left, V is semi-definite if the remaining Schur
// complement is below tol everywhere. tol is the round-off allowance of a singular semi-definite
// matrix (e.g. 64 eps max|diag V|): such a matrix is its own projection up to that round-off.
template <int N, typename R>
LPG_HD bool semidefinite_ldlt(R* V, R tol) {
    static_assert(N <= 32, "the remaining pivots are a 32-bit mask");
    bool pd = true;
    unsigned left = N == 32 ? 0xffffffffu : (1u << N) - 1u;
    for (int k = 0; k < N && pd; ++k) {
        int piv = -1;
        R best = tol;
        for (int i = 0; i < N; ++i)
            if (((left >> i) & 1u) && V[N * i + i] > best) best = V[N * i + i], piv = i;
        if (piv < 0) {
            for (int i = 0; i < N && pd; ++i)
                for (int j = 0; j < N; ++j)
                    if (((left >> i) & (left >> j) & 1u) && !(fabs(V[N * i + j]) <= tol)) {
                        pd = false;
                        break;
                    }
            break;
        }
        left &= ~(1u << piv);
        const R inv = R(1) / best;
        for (int i = 0; i < N; ++i) {
            if (!((left >> i) & 1u)) continue;
            const R li = V[N * i + piv] * inv;
            for (int j = 0; j < N; ++j)
                if ((left >> j) & 1u) V[N * i + j] -= li * V[N * piv + j];
        }
    }
    return pd;
}

// A team of one: the host form of the loops above.
struct SerialTeam {
    LPG_HD int lane() const { return 0; }
    LPG_HD int size() const { return 1; }
    LPG_HD void sync() const {}
    LPG_HD double sum(double x) const { return x; }
};

} // namespace lpg
