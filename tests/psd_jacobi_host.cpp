// Test harness: the GPU's element projections run on the host, for tests/test_psd_jacobi.py (built
// there with g++ into a temporary folder): the hex projection (litepgo_b200/csrc/lpg_psd.h) by a
// team of one lane, and the tet tangent's 9x9 clamp (litepgo_b200/csrc/lpg_clamp9.h).
#include <vector>

#include "lpg_clamp9.h"
#include "lpg_psd.h"

namespace {

template <int N>
int project(const double* in, double* out, double* eig) {
    using J = lpg::PsdJacobi<N>;
    std::vector<double> A(N * J::S), V(N * J::S), cs(J::kCs), L(N);
    std::vector<int> pq(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[i * J::S + j] = in[i * N + j];
    const int sweeps = J::eigen(lpg::SerialTeam{}, A.data(), V.data(), cs.data(), pq.data(), L.data());
    for (int i = 0; i < N; ++i) {
        eig[i] = A[i * J::S + i];
        for (int j = i; j < N; ++j) out[i * N + j] = out[j * N + i] = J::entry(V.data(), L.data(), i, j);
    }
    return sweeps;
}

} // namespace

// Projects the row-major n x n matrix in (n = 2, 8 or 24) into out and writes the unclamped
// eigenvalues (unsorted) to eig; returns the sweeps taken, or -1 for an unsupported n.
extern "C" int psd_project(int n, const double* in, double* out, double* eig) {
    switch (n) {
    case 2: return project<2>(in, out, eig);
    case 8: return project<8>(in, out, eig);
    case 24: return project<24>(in, out, eig);
    default: return -1;
    }
}

// Pairs of round r of the n-index round-robin ordering (n = 24), 2 * n / 2 ints.
extern "C" void psd_round_pairs(int r, int* out) {
    for (int k = 0; k < 12; ++k) lpg::PsdJacobi<24>::pair(r, k, out[2 * k], out[2 * k + 1]);
}

// The semi-definiteness test of the projection passes on a row-major 9 x 9 copy of V.
extern "C" int psd_semidefinite9(const double* V, double tol) {
    double W[81];
    for (int i = 0; i < 81; ++i) W[i] = V[i];
    return lpg::semidefinite_ldlt<9>(W, tol) ? 1 : 0;
}

// The same test in FP32 (the mixed-precision tet projection's instantiation).
extern "C" int psd_semidefinite9f(const float* V, float tol) {
    float W[81];
    for (int i = 0; i < 81; ++i) W[i] = V[i];
    return lpg::semidefinite_ldlt<9>(W, tol) ? 1 : 0;
}

// The 9x9 clamp of the row-major symmetric matrix in (upper triangle used) into out, in FP32
// (fp32 != 0) or FP64, as clamp_kernel runs it.
template <typename R> void clamp9_run(const double* in, double* out) {
    R A[45];
    R V[81];
    for (int r = 0; r < 9; ++r)
        for (int c = r; c < 9; ++c) A[lpg::sym9(r, c)] = static_cast<R>(in[9 * r + c]);
    lpg::clamp9_packed<R, true>(A, V);
    for (int r = 0; r < 9; ++r)
        for (int c = 0; c < 9; ++c) out[9 * r + c] = static_cast<double>(A[lpg::sym9(r, c)]);
}
extern "C" void clamp9_host(int fp32, const double* in, double* out) {
    if (fp32)
        clamp9_run<float>(in, out);
    else
        clamp9_run<double>(in, out);
}
