// Positive semi-definite projection of a dense symmetric N x N matrix, V max(L, 0) V^T, by the
// cyclic Jacobi eigenvalue method in the round-robin parallel ordering (Brent and Luk, "The
// solution of singular-value and symmetric eigenvalue problems on multiprocessor arrays", 1985):
// a sweep is N - 1 rounds of N / 2 disjoint plane rotations, each round computed from one state
// of the matrix, so the rotations of a round, their row updates and their column updates are
// independent tasks. This is the projection HessianKind::Projected applies to every element's
// local Hessian (mesh_energy.cpp:16-27, there by Eigen's SelfAdjointEigenSolver).
//
// The functions are the tasks of one round; a caller runs rotation() for k < N/2, then
// update() for t < kUpdateTasks, with a barrier after each phase (one warp per matrix on the
// GPU; plain loops on the host, where a test checks this code against an eigensolver).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define LPG_HD __host__ __device__ __forceinline__
#else
#define LPG_HD inline
#endif

namespace lpg {

template <int N>
struct PsdJacobi {
    static_assert(N % 2 == 0 && N >= 2, "the round-robin ordering pairs an even number of indices");
    static constexpr int S = N + 1;       // row stride (a padded row staggers column reads across banks)
    static constexpr int kPairs = N / 2;  // rotations per round
    static constexpr int kRounds = N - 1; // rounds per sweep: every index pair once
    static constexpr int kCs = 3 * kPairs; // c, s, t per rotation
    static constexpr int kBlockTasks = kPairs * (kPairs + 1) / 2; // 2x2 blocks (k, l), k <= l
    static constexpr int kUpdateTasks = kBlockTasks + kPairs * N;  // ... then V's rows
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
        double c = 1.0, s = 0.0, t = 0.0;
        if (apq != 0.0) {
            const double th = (A[q * S + q] - A[p * S + p]) / (2.0 * apq);
            const double at = fabs(th);
            t = at > 1e150 ? 0.5 / th : copysign(1.0, th) / (at + sqrt(th * th + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
        }
        cs[3 * k] = c;
        cs[3 * k + 1] = s;
        cs[3 * k + 2] = t;
        pq[2 * k] = p;
        pq[2 * k + 1] = q;
    }

    // Task t of a round's update. t < kBlockTasks: the 2x2 block of A at rows (p_k, q_k) and
    // columns (p_l, q_l), k <= l, becomes J_k^T X J_l and is mirrored to (l, k); on a diagonal
    // block (k = l) the rotation's own entry is annihilated exactly, a'_pp = a_pp - t a_pq,
    // a'_qq = a_qq + t a_pq, a'_pq = 0, so A stays bitwise symmetric. Otherwise: columns p_k
    // and q_k of V J at row i (t - kBlockTasks = k N + i).
    LPG_HD static void update(double* A, double* V, const double* cs, const int* pq, int t) {
        if (t >= kBlockTasks) {
            const int u = t - kBlockTasks, k = u / N, i = u - N * k;
            const double c = cs[3 * k], s = cs[3 * k + 1];
            double* v = V + i * S;
            const int p = pq[2 * k], q = pq[2 * k + 1];
            const double x = v[p], y = v[q];
            v[p] = c * x - s * y;
            v[q] = s * x + c * y;
            return;
        }
        int k = 0, l = t;
        while (l >= kPairs - k) {
            l -= kPairs - k;
            ++k;
        }
        l += k;
        const int p = pq[2 * k], q = pq[2 * k + 1];
        if (l == k) {
            const double apq = A[p * S + q], tk = cs[3 * k + 2];
            A[p * S + p] -= tk * apq;
            A[q * S + q] += tk * apq;
            A[p * S + q] = 0.0;
            A[q * S + p] = 0.0;
            return;
        }
        const int pl = pq[2 * l], ql = pq[2 * l + 1];
        const double ck = cs[3 * k], sk = cs[3 * k + 1], cl = cs[3 * l], sl = cs[3 * l + 1];
        const double x00 = A[p * S + pl], x01 = A[p * S + ql], x10 = A[q * S + pl], x11 = A[q * S + ql];
        const double y00 = ck * x00 - sk * x10, y01 = ck * x01 - sk * x11; // rows: J_k^T X
        const double y10 = sk * x00 + ck * x10, y11 = sk * x01 + ck * x11;
        const double z00 = cl * y00 - sl * y01, z01 = sl * y00 + cl * y01; // columns: (J_k^T X) J_l
        const double z10 = cl * y10 - sl * y11, z11 = sl * y10 + cl * y11;
        A[p * S + pl] = z00;
        A[p * S + ql] = z01;
        A[q * S + pl] = z10;
        A[q * S + ql] = z11;
        A[pl * S + p] = z00;
        A[ql * S + p] = z01;
        A[pl * S + q] = z10;
        A[ql * S + q] = z11;
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
                for (int t = lane; t < kUpdateTasks; t += nl) update(A, V, cs, pq, t);
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
