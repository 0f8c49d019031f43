// lpg_oracle.cpp -- CPU restatement of the litepgo volumetric neo-Hookean hot path.
//
// TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline); see lpg_oracle.h.
// Every function cites the reference file:line it restates. The code is written
// from the reference's behaviour with plain arrays in place of Eigen; the dense
// products, the 12x12 eigen-projection (cyclic Jacobi, Golub & Van Loan,
// "Matrix Computations", Alg. 8.5.2/8.5.3) and the direct solver (envelope
// LDL^T) are this project's own stand-ins for Eigen's routines.

#include "lpg_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_error;
int g_threads = 0;

struct Error {
    int code;
    std::string what;
};
[[noreturn]] void fail(int code, const std::string& what) { throw Error{code, what}; }

template <class F> int guarded(F&& f) {
    try {
        f();
        return ORC_OK;
    } catch (const Error& e) {
        g_error = e.what;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "out of memory";
        return ORC_ELOGIC;
    } catch (const std::exception& e) {
        g_error = e.what();
        return ORC_ELOGIC;
    }
}

constexpr double kEps = std::numeric_limits<double>::epsilon();

// ---------------------------------------------------------------------------
// 3x3 helpers, column-major: m[i + 3 j].
// ---------------------------------------------------------------------------
using M3 = std::array<double, 9>;

inline double at(const M3& m, int i, int j) { return m[i + 3 * j]; }
inline bool finite9(const double* m) {
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(m[k])) return false;
    return true;
}
inline double det3(const M3& m) {
    return at(m, 0, 0) * (at(m, 1, 1) * at(m, 2, 2) - at(m, 2, 1) * at(m, 1, 2)) -
           at(m, 1, 0) * (at(m, 0, 1) * at(m, 2, 2) - at(m, 2, 1) * at(m, 0, 2)) +
           at(m, 2, 0) * (at(m, 0, 1) * at(m, 1, 2) - at(m, 1, 1) * at(m, 0, 2));
}
// Inverse through the adjugate; the caller checks finiteness.
inline M3 inv3(const M3& m) {
    const double d = det3(m);
    M3 r;
    r[0 + 3 * 0] = (at(m, 1, 1) * at(m, 2, 2) - at(m, 1, 2) * at(m, 2, 1)) / d;
    r[0 + 3 * 1] = (at(m, 0, 2) * at(m, 2, 1) - at(m, 0, 1) * at(m, 2, 2)) / d;
    r[0 + 3 * 2] = (at(m, 0, 1) * at(m, 1, 2) - at(m, 0, 2) * at(m, 1, 1)) / d;
    r[1 + 3 * 0] = (at(m, 1, 2) * at(m, 2, 0) - at(m, 1, 0) * at(m, 2, 2)) / d;
    r[1 + 3 * 1] = (at(m, 0, 0) * at(m, 2, 2) - at(m, 0, 2) * at(m, 2, 0)) / d;
    r[1 + 3 * 2] = (at(m, 0, 2) * at(m, 1, 0) - at(m, 0, 0) * at(m, 1, 2)) / d;
    r[2 + 3 * 0] = (at(m, 1, 0) * at(m, 2, 1) - at(m, 1, 1) * at(m, 2, 0)) / d;
    r[2 + 3 * 1] = (at(m, 0, 1) * at(m, 2, 0) - at(m, 0, 0) * at(m, 2, 1)) / d;
    r[2 + 3 * 2] = (at(m, 0, 0) * at(m, 1, 1) - at(m, 0, 1) * at(m, 1, 0)) / d;
    return r;
}
inline M3 mul3(const M3& a, const M3& b) {
    M3 r{};
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += at(a, i, k) * at(b, k, j);
            r[i + 3 * j] = s;
        }
    return r;
}
inline M3 transpose3(const M3& a) {
    M3 r;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) r[i + 3 * j] = a[j + 3 * i];
    return r;
}
inline M3 load3(const double* p) {
    M3 r;
    std::memcpy(r.data(), p, sizeof(double) * 9);
    return r;
}
inline M3 eye3() { return M3{1, 0, 0, 0, 1, 0, 0, 0, 1}; }

// ---------------------------------------------------------------------------
// MultiplicativeKinematics (multiplicative_kinematics.cpp:9-51) and NeoHookean
// (neo_hookean.cpp:14-146).
// ---------------------------------------------------------------------------
struct Kinematics {
    M3 inv_Fp, Fe;
    double det_Fp;
};

// multiplicative_kinematics.cpp:9-22
Kinematics make_kinematics(const M3& F, const M3& Fp) {
    if (!finite9(F.data()) || !finite9(Fp.data()))
        fail(ORC_EINVAL, "MultiplicativeKinematics requires finite F and Fp");
    Kinematics k;
    k.det_Fp = det3(Fp);
    if (!std::isfinite(k.det_Fp) || k.det_Fp <= 0.0)
        fail(ORC_EDOMAIN, "MultiplicativeKinematics requires finite det(Fp) > 0");
    k.inv_Fp = inv3(Fp);
    k.Fe = mul3(F, k.inv_Fp);
    if (!finite9(k.inv_Fp.data()) || !finite9(k.Fe.data()))
        fail(ORC_EDOMAIN, "MultiplicativeKinematics: non-finite inverse or elastic gradient");
    return k;
}

// neo_hookean.cpp:14-23
double log_det_Fe(const M3& Fe, const double* theta) {
    if (!std::isfinite(theta[0]) || !std::isfinite(theta[1]) || theta[0] < 0.0 || theta[1] <= 0.0)
        fail(ORC_EINVAL, "NeoHookean requires finite lambda >= 0 and mu > 0");
    const double d = det3(Fe);
    if (!std::isfinite(d) || d <= 0.0) fail(ORC_EDOMAIN, "NeoHookean requires finite det(Fe) > 0");
    return std::log(d);
}

// neo_hookean.cpp:25-31
M3 inv_Fe_T(const M3& Fe) {
    const M3 r = transpose3(inv3(Fe));
    if (!finite9(r.data())) fail(ORC_EDOMAIN, "NeoHookean: non-finite elastic inverse");
    return r;
}

// neo_hookean.cpp:33-36
double psi(const M3& Fe, const double* theta, double L) {
    double sq = 0;
    for (double v : Fe) sq += v * v;
    return 0.5 * theta[1] * (sq - 3.0) - theta[1] * L + 0.5 * theta[0] * L * L;
}

// neo_hookean.cpp:38-41
M3 dpsi_dFe(const M3& Fe, const double* theta, double L, const M3& iFT) {
    M3 r;
    for (int k = 0; k < 9; ++k) r[k] = theta[1] * Fe[k] + (theta[0] * L - theta[1]) * iFT[k];
    return r;
}

// neo_hookean.cpp:43-60 ; 9x9 column-major: A[r + 9 c] with r = i + 3j, c = m + 3l.
void d2psi_dFe2(const double* theta, double L, const M3& iFT, double* A) {
    const double lambda = theta[0], mu = theta[1];
    const double pressure = lambda * L - mu;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m)
                    A[(i + 3 * j) + 9 * (m + 3 * l)] = mu * ((i == m && j == l) ? 1.0 : 0.0) +
                                                       lambda * at(iFT, i, j) * at(iFT, m, l) -
                                                       pressure * at(iFT, i, l) * at(iFT, m, j);
}

// multiplicative_kinematics.cpp:24-29
double kin_W(const Kinematics& k, double ps) {
    const double W = k.det_Fp * ps;
    if (!std::isfinite(W)) fail(ORC_EDOMAIN, "MultiplicativeKinematics: non-finite density");
    return W;
}
// multiplicative_kinematics.cpp:31-36
M3 kin_dW_dF(const Kinematics& k, const M3& dpsi) {
    M3 g = mul3(dpsi, transpose3(k.inv_Fp));
    for (double& v : g) v *= k.det_Fp;
    if (!finite9(g.data())) fail(ORC_EDOMAIN, "MultiplicativeKinematics: non-finite F gradient");
    return g;
}
// multiplicative_kinematics.cpp:38-51: det_Fp * D^T A D with D = dFe/dF,
// D block (3i, 3j) = inv_Fp(j, i) * I3.
void kin_d2W_dF2(const Kinematics& k, const double* A, double* out) {
    double D[81] = {0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int d = 0; d < 3; ++d) D[(3 * i + d) + 9 * (3 * j + d)] = at(k.inv_Fp, j, i);
    double AD[81];
    for (int c = 0; c < 9; ++c)
        for (int r = 0; r < 9; ++r) {
            double s = 0;
            for (int t = 0; t < 9; ++t) s += A[r + 9 * t] * D[t + 9 * c];
            AD[r + 9 * c] = s;
        }
    for (int c = 0; c < 9; ++c)
        for (int r = 0; r < 9; ++r) {
            double s = 0;
            for (int t = 0; t < 9; ++t) s += D[t + 9 * r] * AD[t + 9 * c];
            out[r + 9 * c] = k.det_Fp * s;
        }
    for (int t = 0; t < 81; ++t)
        if (!std::isfinite(out[t])) fail(ORC_EDOMAIN, "MultiplicativeKinematics: non-finite F Hessian");
}

// neo_hookean.cpp:64-70
double nh_W(const M3& F, const M3& Fp, const double* theta) {
    const Kinematics k = make_kinematics(F, Fp);
    const double L = log_det_Fe(k.Fe, theta);
    return kin_W(k, psi(k.Fe, theta, L));
}
// neo_hookean.cpp:72-78
M3 nh_P(const M3& F, const M3& Fp, const double* theta) {
    const Kinematics k = make_kinematics(F, Fp);
    const double L = log_det_Fe(k.Fe, theta);
    return kin_dW_dF(k, dpsi_dFe(k.Fe, theta, L, inv_Fe_T(k.Fe)));
}
// neo_hookean.cpp:80-86
void nh_A(const M3& F, const M3& Fp, const double* theta, double* out) {
    const Kinematics k = make_kinematics(F, Fp);
    const double L = log_det_Fe(k.Fe, theta);
    double A[81];
    d2psi_dFe2(theta, L, inv_Fe_T(k.Fe), A);
    kin_d2W_dF2(k, A, out);
}
// neo_hookean.cpp:88-101
void nh_dP_dtheta(const M3& F, const M3& Fp, const double* theta, double* out) {
    const Kinematics k = make_kinematics(F, Fp);
    const double L = log_det_Fe(k.Fe, theta);
    const M3 iFT = inv_Fe_T(k.Fe);
    M3 a, b;
    for (int t = 0; t < 9; ++t) {
        a[t] = L * iFT[t];
        b[t] = k.Fe[t] - iFT[t];
    }
    const M3 dl = kin_dW_dF(k, a), dm = kin_dW_dF(k, b);
    for (int t = 0; t < 9; ++t) {
        out[t] = dl[t];
        out[9 + t] = dm[t];
    }
}
// neo_hookean.cpp:103-128
void nh_dP_dFp(const M3& F, const M3& Fp, const double* theta, double* out) {
    const Kinematics k = make_kinematics(F, Fp);
    const double L = log_det_Fe(k.Fe, theta);
    const M3 iFT = inv_Fe_T(k.Fe);
    const M3 inv_Fp = inv3(Fp);
    double tangent[81];
    d2psi_dFe2(theta, L, iFT, tangent);
    const M3 P = kin_dW_dF(k, dpsi_dFe(k.Fe, theta, L, iFT));
    const M3 iFpT = transpose3(inv_Fp);
    for (int column = 0; column < 9; ++column) {
        M3 dFp{};
        dFp[column] = 1;
        M3 dFe = mul3(mul3(k.Fe, dFp), inv_Fp);
        for (double& v : dFe) v = -v;
        M3 dstress;
        for (int r = 0; r < 9; ++r) {
            double s = 0;
            for (int t = 0; t < 9; ++t) s += tangent[r + 9 * t] * dFe[t];
            dstress[r] = s;
        }
        const M3 tr_m = mul3(inv_Fp, dFp);
        const double tr = tr_m[0] + tr_m[4] + tr_m[8];
        const M3 second = mul3(dstress, iFpT);
        const M3 third = mul3(mul3(P, transpose3(dFp)), iFpT);
        for (int t = 0; t < 9; ++t) out[t + 9 * column] = tr * P[t] + k.det_Fp * second[t] - third[t];
    }
    for (int t = 0; t < 81; ++t)
        if (!std::isfinite(out[t])) fail(ORC_EDOMAIN, "NeoHookean: non-finite plastic mixed derivative");
}

// positive_det_feasible_step.cpp:13-84
double positive_det_step(const M3& A, const M3& dA) {
    if (!finite9(A.data()) || !finite9(dA.data()))
        fail(ORC_EINVAL, "Positive determinant step requires finite matrices");
    const double det_A = det3(A);
    if (!std::isfinite(det_A) || det_A <= 0) fail(ORC_EDOMAIN, "Positive determinant step requires finite det(A)>0");
    // Column scaling by the larger max-abs entry of A and dA in that column.
    M3 a, d;
    for (int j = 0; j < 3; ++j) {
        double s = 0;
        for (int i = 0; i < 3; ++i) s = std::max(s, std::abs(at(A, i, j)));
        double t = 0;
        for (int i = 0; i < 3; ++i) t = std::max(t, std::abs(at(dA, i, j)));
        const double scale = std::max(s, t);
        for (int i = 0; i < 3; ++i) {
            a[i + 3 * j] = at(A, i, j) / scale;
            d[i + 3 * j] = at(dA, i, j) / scale;
        }
    }
    auto col = [](const M3& m, int j) { return std::array<double, 3>{m[3 * j], m[3 * j + 1], m[3 * j + 2]}; };
    auto cross = [](const std::array<double, 3>& x, const std::array<double, 3>& y) {
        return std::array<double, 3>{x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
    };
    auto dot = [](const std::array<double, 3>& x, const std::array<double, 3>& y) {
        return x[0] * y[0] + x[1] * y[1] + x[2] * y[2];
    };
    const auto a0 = col(a, 0), a1 = col(a, 1), a2 = col(a, 2);
    const auto d0 = col(d, 0), d1 = col(d, 1), d2 = col(d, 2);
    const double c0 = det3(a);
    const double c1 = dot(d0, cross(a1, a2)) + dot(a0, cross(d1, a2)) + dot(a0, cross(a1, d2));
    const double c2 = dot(d0, cross(d1, a2)) + dot(d0, cross(a1, d2)) + dot(a0, cross(d1, d2));
    const double c3 = det3(d);
    if (!(c0 > 0)) return 0;
    auto value = [&](double t) { return std::fma(std::fma(std::fma(c3, t, c2), t, c1), t, c0); };
    auto tolerance = [&](double t) {
        return 64 * kEps * (((std::abs(c3) * t + std::abs(c2)) * t + std::abs(c1)) * t + c0);
    };
    std::array<double, 4> knots{0, 1, 0, 0};
    int count = 2;
    auto add_knot = [&](double t) {
        if (t > 0 && t < 1) knots[count++] = t;
    };
    const double qa = 3 * c3, qb = 2 * c2, qc = c1;
    if (qa == 0) {
        if (qb != 0) add_knot(-qc / qb);
    } else {
        double disc = std::fma(qb, qb, -4 * qa * qc);
        const double err = 8 * kEps * (qb * qb + std::abs(4 * qa * qc));
        if (disc >= -err) {
            disc = std::max(0.0, disc);
            const double q = -0.5 * (qb + std::copysign(std::sqrt(disc), qb));
            if (q == 0)
                add_knot(-qb / (2 * qa));
            else {
                add_knot(q / qa);
                add_knot(qc / q);
            }
        }
    }
    for (int i = 1; i < count; ++i) // insertion sort of at most four knots
        for (int j = i; j > 0 && knots[j - 1] > knots[j]; --j) std::swap(knots[j - 1], knots[j]);
    for (int i = 1; i < count; ++i) {
        double lo = knots[i - 1], hi = knots[i];
        if (value(hi) > tolerance(hi)) continue;
        for (;;) {
            const double mid = lo + (hi - lo) / 2;
            if (mid == lo || mid == hi) break;
            if (value(mid) > tolerance(mid))
                lo = mid;
            else
                hi = mid;
        }
        return 0.9 * lo;
    }
    return 1;
}

// neo_hookean.cpp:130-146
double nh_feasible_step(const M3& F, const M3& Fp, const double* theta, const M3& dF, const M3& dFp,
                        const double* dtheta) {
    if (!finite9(dF.data()) || !finite9(dFp.data()) || !std::isfinite(dtheta[0]) || !std::isfinite(dtheta[1]))
        fail(ORC_EINVAL, "NeoHookean step requires finite, compatible input increments");
    nh_W(F, Fp, theta);
    double alpha = std::min(positive_det_step(F, dF), positive_det_step(Fp, dFp));
    for (int j = 0; j < 2; ++j) {
        if (dtheta[j] < 0)
            alpha = std::min(alpha, 0.9 * (theta[j] / -dtheta[j]));
        else if (dtheta[j] > 0)
            alpha = std::min(alpha, 0.9 * ((std::numeric_limits<double>::max() - theta[j]) / dtheta[j]));
    }
    return alpha;
}

// ---------------------------------------------------------------------------
// Cyclic Jacobi eigen-decomposition of a symmetric matrix (Golub & Van Loan,
// Alg. 8.5.2 sym.schur2 + 8.5.3 cyclic sweeps). Stand-in for Eigen's
// SelfAdjointEigenSolver in project_hessian (mesh_energy.cpp:16-27).
// ---------------------------------------------------------------------------
void jacobi_eigen(int n, std::vector<double>& A, std::vector<double>& V) {
    V.assign(static_cast<size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
    auto a = [&](int i, int j) -> double& { return A[i + static_cast<size_t>(n) * j]; };
    double total = 0;
    for (double v : A) total += v * v;
    if (total == 0) return;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                if (i != j) off += a(i, j) * a(i, j);
        if (off <= 1e-32 * total) break;
        bool rotated = false;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a(p, q);
                if (apq == 0) continue;
                const double tau = (a(q, q) - a(p, p)) / (2 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (std::abs(tau) + std::sqrt(1 + tau * tau));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                if (s == 0) continue;
                rotated = true;
                // A <- J^T A J with J the Givens rotation in the (p, q) plane.
                for (int k = 0; k < n; ++k) {
                    const double akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * akq;
                    a(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * aqk;
                    a(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[k + n * p], vkq = V[k + n * q];
                    V[k + n * p] = c * vkp - s * vkq;
                    V[k + n * q] = s * vkp + c * vkq;
                }
            }
        if (!rotated) break;
    }
}

// mesh_energy.cpp:16-27: symmetrise, eigen-decompose, clamp eigenvalues at 0.
void project_psd(int n, const double* H, double* out) {
    std::vector<double> S(static_cast<size_t>(n) * n), V;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) S[i + n * j] = 0.5 * H[i + n * j] + 0.5 * H[j + n * i];
    jacobi_eigen(n, S, V);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int k = 0; k < n; ++k) s += V[i + n * k] * std::max(S[k + n * k], 0.0) * V[j + n * k];
            out[i + n * j] = s;
        }
    for (int t = 0; t < n * n; ++t)
        if (!std::isfinite(out[t])) fail(ORC_EDOMAIN, "MeshEnergy: non-finite projected Hessian");
}

} // namespace

// ---------------------------------------------------------------------------
// Mesh energy: VolumetricFemEnergy<NeoHookean, TetP1Basis, TetCentroidQuadrature>
// (volumetric_fem_energy.hpp:29-210) + MeshEnergy (mesh_energy.cpp:29-107) +
// EnergyAssembler (energy_assembler.cpp:22-170).
// ---------------------------------------------------------------------------
struct orc_mesh {
    int V = 0, T = 0, n = 0; // n = number of DOFs
    std::vector<int> tets;   // T*4
    // Per element: B (9x12, column-major), w = (1/6) det J, Fp, theta.
    std::vector<double> B, w, Fp, theta;
    bool has_Fp = false;
    // Assembler.
    std::vector<int> outer, inner;                    // CSC pattern
    std::vector<int> offsets;                         // T * 144, (i + 12 j) -> value position
    std::vector<int> contrib_ptr, contrib_elem, contrib_local; // per column, element order
};

namespace {

// TetP1Basis::eval_dN_dxi (tet_p1_basis.cpp:11-15).
const double kdN[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

// VolumetricElement3D ctor (volumetric_element.hpp:23-39) + deformation_gradient_sampling_response
// (deformation_gradient_sampling_response.hpp:15-45) for one tet with rest corners Xc[4][3].
void build_element(const double* Xc, double* Bout, double* wout) {
    for (int k = 0; k < 12; ++k)
        if (!std::isfinite(Xc[k])) fail(ORC_EINVAL, "VolumetricElement3D: invalid reference Jacobian");
    // J_X(:, j) = d X / d xi_j = sum_a X_a dN_a/dxi_j  (InterpolatedResponse<TetP1Basis>).
    M3 J{};
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = 0;
            for (int a = 0; a < 4; ++a) s += Xc[3 * a + i] * kdN[a][j];
            J[i + 3 * j] = s;
        }
    const double det = det3(J);
    const double w = det / 6.0; // TetCentroidQuadrature weight 1/6
    if (!std::isfinite(det) || det <= 0 || !std::isfinite(w))
        fail(ORC_EINVAL, "VolumetricElement3D: invalid reference determinant or volume weight");
    const M3 Ji = inv3(J);
    // gradient (4x3) = dN_dxi * J^{-1}; B = kron(gradient^T, I3): B(3j+i, 3a+k) = grad(a, j) delta_ik.
    double grad[4][3];
    for (int a = 0; a < 4; ++a)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int t = 0; t < 3; ++t) s += kdN[a][t] * at(Ji, t, j);
            grad[a][j] = s;
        }
    for (int k = 0; k < 108; ++k) Bout[k] = 0;
    for (int a = 0; a < 4; ++a)
        for (int j = 0; j < 3; ++j) {
            if (!std::isfinite(grad[a][j]))
                fail(ORC_EINVAL, "Deformation gradient sampling: non-finite physical gradient");
            for (int i = 0; i < 3; ++i) Bout[(3 * j + i) + 9 * (3 * a + i)] = grad[a][j];
        }
    *wout = w;
}

// EnergyAssembler ctor (energy_assembler.cpp:22-68) for vertex-major 3-DOF tets.
void build_assembler(orc_mesh& m) {
    const int n = m.n;
    std::vector<std::vector<int>> rows(static_cast<size_t>(n));
    for (int e = 0; e < m.T; ++e) {
        int idx[12];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) idx[3 * a + c] = 3 * m.tets[4 * e + a] + c;
        for (int column : idx)
            for (int row : idx) rows[column].push_back(row);
    }
    m.outer.assign(n + 1, 0);
    for (int c = 0; c < n; ++c) {
        auto& r = rows[c];
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        m.outer[c + 1] = m.outer[c] + static_cast<int>(r.size());
    }
    m.inner.resize(static_cast<size_t>(m.outer[n]));
    for (int c = 0; c < n; ++c) std::copy(rows[c].begin(), rows[c].end(), m.inner.begin() + m.outer[c]);
    // Contributions per DOF column in element / local-DOF order (energy_assembler.cpp:49-54).
    std::vector<int> count(n + 1, 0);
    for (int e = 0; e < m.T; ++e)
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) ++count[3 * m.tets[4 * e + a] + c + 1];
    m.contrib_ptr.assign(n + 1, 0);
    for (int c = 0; c < n; ++c) m.contrib_ptr[c + 1] = m.contrib_ptr[c] + count[c + 1];
    m.contrib_elem.resize(static_cast<size_t>(m.contrib_ptr[n]));
    m.contrib_local.resize(static_cast<size_t>(m.contrib_ptr[n]));
    std::vector<int> fill(m.contrib_ptr.begin(), m.contrib_ptr.end() - 1);
    for (int e = 0; e < m.T; ++e)
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) {
                const int d = 3 * m.tets[4 * e + a] + c;
                m.contrib_elem[fill[d]] = e;
                m.contrib_local[fill[d]] = 3 * a + c;
                ++fill[d];
            }
    // Per-element value offsets by lower_bound (energy_assembler.cpp:56-67), index i + 12 j.
    m.offsets.resize(static_cast<size_t>(m.T) * 144);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < m.T; ++e) {
        int idx[12];
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) idx[3 * a + c] = 3 * m.tets[4 * e + a] + c;
        for (int j = 0; j < 12; ++j) {
            const int column = idx[j];
            const int* b = m.inner.data() + m.outer[column];
            const int* en = m.inner.data() + m.outer[column + 1];
            for (int i = 0; i < 12; ++i)
                m.offsets[static_cast<size_t>(e) * 144 + i + 12 * j] =
                    static_cast<int>(std::lower_bound(b, en, idx[i]) - m.inner.data());
        }
    }
}

// Local coefficients c (12, row-major u_a,k) -> F = I + reshape(B c) (volumetric_fem_energy.hpp:186-192).
M3 element_F(const orc_mesh& m, int e, const double* c) {
    const double* B = m.B.data() + static_cast<size_t>(e) * 108;
    M3 F;
    for (int r = 0; r < 9; ++r) {
        double s = 0;
        for (int k = 0; k < 12; ++k) s += B[r + 9 * k] * c[k];
        F[r] = s;
    }
    F[0] += 1;
    F[4] += 1;
    F[8] += 1;
    if (!finite9(F.data())) fail(ORC_EDOMAIN, "VolumetricFemEnergy: non-finite deformation gradient");
    return F;
}

void gather_local(const orc_mesh& m, int e, const double* x, double* c) {
    for (int a = 0; a < 4; ++a)
        for (int k = 0; k < 3; ++k) c[3 * a + k] = x[3 * m.tets[4 * e + a] + k];
}

const double* elem_theta(const orc_mesh& m, int e) { return m.theta.data() + 2 * static_cast<size_t>(e); }
M3 elem_Fp(const orc_mesh& m, int e) {
    return m.has_Fp ? load3(m.Fp.data() + 9 * static_cast<size_t>(e)) : eye3();
}

// One element's E, g (12) and H (144, column-major) through the dense B products
// (volumetric_fem_energy.hpp:195-210; dof_derivatives.cpp:22-51).
double eval_element(const orc_mesh& m, int e, const double* x, double* g, double* H) {
    double c[12];
    gather_local(m, e, x, c);
    const M3 F = element_F(m, e, c);
    const M3 Fp = elem_Fp(m, e);
    const double* th = elem_theta(m, e);
    const double W = nh_W(F, Fp, th);
    const double w = m.w[e];
    const double* B = m.B.data() + static_cast<size_t>(e) * 108;
    if (g) {
        const M3 P = nh_P(F, Fp, th);
        for (int k = 0; k < 12; ++k) {
            double s = 0;
            for (int r = 0; r < 9; ++r) s += B[r + 9 * k] * P[r];
            g[k] = w * s;
        }
    }
    if (H) {
        double A[81];
        nh_A(F, Fp, th, A);
        double BtA[12 * 9];
        for (int r = 0; r < 9; ++r)
            for (int k = 0; k < 12; ++k) {
                double s = 0;
                for (int t = 0; t < 9; ++t) s += B[t + 9 * k] * A[t + 9 * r];
                BtA[k + 12 * r] = s;
            }
        for (int j = 0; j < 12; ++j)
            for (int i = 0; i < 12; ++i) {
                double s = 0;
                for (int t = 0; t < 9; ++t) s += BtA[i + 12 * t] * B[t + 9 * j];
                H[i + 12 * j] = w * s;
            }
    }
    const double E = w * W;
    // VolumetricElement3D::eval_into finite checks (volumetric_element.hpp:59-60).
    bool ok = std::isfinite(E);
    if (g)
        for (int k = 0; k < 12; ++k) ok = ok && std::isfinite(g[k]);
    if (H)
        for (int k = 0; k < 144; ++k) ok = ok && std::isfinite(H[k]);
    if (!ok) fail(ORC_EDOMAIN, "VolumetricElement3D: non-finite integrated outputs");
    return E;
}

// Runs body(e) over all elements in parallel; the first error (lowest element) wins.
template <class Body> void for_elements(int T, Body&& body) {
    int err_elem = T;
    Error first{ORC_OK, ""};
#pragma omp parallel for schedule(static)
    for (int e = 0; e < T; ++e) {
        try {
            body(e);
        } catch (const Error& x) {
#pragma omp critical
            {
                if (e < err_elem) {
                    err_elem = e;
                    first = x;
                }
            }
        }
    }
    if (err_elem < T) throw first;
}

// MeshEnergy::eval_values (mesh_energy.cpp:48-87) + EnergyAssembler::assemble (energy_assembler.cpp:123-170).
double mesh_eval(orc_mesh& m, const double* u, double* grad, int hessian, double* values, double* elem_E_out,
                 double* elem_g_out, double* elem_H_out) {
    for (int k = 0; k < m.n; ++k)
        if (!std::isfinite(u[k])) fail(ORC_EINVAL, "Energy::eval: x must have num_dofs finite entries");
    const bool want_g = grad || elem_g_out;
    const bool want_H = hessian != 0;
    std::vector<double> Ee(static_cast<size_t>(m.T));
    std::vector<double> ge(want_g ? static_cast<size_t>(m.T) * 12 : 0);
    std::vector<double> He(want_H ? static_cast<size_t>(m.T) * 144 : 0);
    for_elements(m.T, [&](int e) {
        double* g = want_g ? ge.data() + 12 * static_cast<size_t>(e) : nullptr;
        double* H = want_H ? He.data() + 144 * static_cast<size_t>(e) : nullptr;
        Ee[e] = eval_element(m, e, u, g, H);
        if (H && hessian == 2) {
            double P[144];
            project_psd(12, H, P);
            std::memcpy(H, P, sizeof P);
        }
    });
    if (grad || values) {
        const int n = m.n;
        // A task owns whole CSC columns (grain 64 in the reference); order within a column is fixed.
#pragma omp parallel for schedule(static, 64)
        for (int column = 0; column < n; ++column) {
            if (values)
                for (int k = m.outer[column]; k < m.outer[column + 1]; ++k) values[k] = 0.0;
            double g = 0;
            for (int t = m.contrib_ptr[column]; t < m.contrib_ptr[column + 1]; ++t) {
                const int e = m.contrib_elem[t], j = m.contrib_local[t];
                if (grad) g += ge[12 * static_cast<size_t>(e) + j];
                if (values) {
                    const double* H = He.data() + 144 * static_cast<size_t>(e);
                    const int* off = m.offsets.data() + 144 * static_cast<size_t>(e);
                    for (int i = 0; i < 12; ++i) values[off[i + 12 * j]] += H[i + 12 * j];
                }
            }
            if (grad) grad[column] = g;
        }
    }
    double E = 0;
    for (double v : Ee) E += v; // std::accumulate in element order (mesh_energy.cpp:83)
    if (!std::isfinite(E)) fail(ORC_EDOMAIN, "MeshEnergy: non-finite energy sum");
    if (elem_E_out) std::copy(Ee.begin(), Ee.end(), elem_E_out);
    if (elem_g_out) std::copy(ge.begin(), ge.end(), elem_g_out);
    if (elem_H_out) std::copy(He.begin(), He.end(), elem_H_out);
    return E;
}

// VolumetricFemEnergy::eval_feasible_step_batch (volumetric_fem_energy.hpp:156-185) +
// MeshEnergy::feasible_step (mesh_energy.cpp:88-107).
double mesh_feasible_step(orc_mesh& m, const double* u, const double* du) {
    for (int k = 0; k < m.n; ++k)
        if (!std::isfinite(u[k])) fail(ORC_EINVAL, "Energy::max_feasible_step: x must have num_dofs finite entries");
    for (int k = 0; k < m.n; ++k)
        if (!std::isfinite(du[k])) fail(ORC_EINVAL, "Energy::max_feasible_step: dx must have num_dofs finite entries");
    std::vector<double> steps(static_cast<size_t>(m.T));
    for_elements(m.T, [&](int e) {
        double c[12], dc[12];
        gather_local(m, e, u, c);
        gather_local(m, e, du, dc);
        const M3 F = element_F(m, e, c);
        const double* B = m.B.data() + static_cast<size_t>(e) * 108;
        M3 dF;
        for (int r = 0; r < 9; ++r) {
            double s = 0;
            for (int k = 0; k < 12; ++k) s += B[r + 9 * k] * dc[k];
            dF[r] = s;
        }
        if (!finite9(dF.data())) fail(ORC_EDOMAIN, "VolumetricFemEnergy: non-finite input increment");
        const double zero2[2] = {0, 0};
        const M3 Z{};
        const double b = nh_feasible_step(F, elem_Fp(m, e), elem_theta(m, e), dF, Z, zero2);
        if (!(b >= 0 && b <= 1)) fail(ORC_ELOGIC, "VolumetricElement3D: local feasible step outside [0,1]");
        steps[e] = b;
    });
    double alpha = 1;
    for (double s : steps) alpha = std::min(alpha, s);
    return alpha;
}

// VolumetricFemForceResponse::eval_row (detail/volumetric_fem_force_response.hpp:155-179) with
// MeshResponse::product transpose (mesh_response.cpp:70-98): per element (B^T dP/dtheta w_dV)^T w_e.
void force_vjp_theta(orc_mesh& m, const double* u, const double* wvec, double* out) {
    for_elements(m.T, [&](int e) {
        double c[12], we[12];
        gather_local(m, e, u, c);
        gather_local(m, e, wvec, we);
        const M3 F = element_F(m, e, c);
        double mixed[18];
        nh_P(F, elem_Fp(m, e), elem_theta(m, e)); // stress finite check as in eval_row
        nh_dP_dtheta(F, elem_Fp(m, e), elem_theta(m, e), mixed);
        const double* B = m.B.data() + static_cast<size_t>(e) * 108;
        const double w = m.w[e];
        for (int p = 0; p < 2; ++p) {
            // J(:, p) = w * B^T mixed(:, p); out_p = sum_k J(k, p) we[k].
            double s = 0;
            for (int k = 0; k < 12; ++k) {
                double jk = 0;
                for (int r = 0; r < 9; ++r) jk += B[r + 9 * k] * mixed[r + 9 * p];
                s += (w * jk) * we[k];
            }
            out[2 * static_cast<size_t>(e) + p] = s;
        }
    });
}

// VolumetricFemForceFpResponse::eval_vjp (volumetric_fem_force_fp_response.hpp:8-10 through
// detail/volumetric_fem_force_response.hpp:155-179 and MeshResponse::product,
// mesh_response.cpp:70-98): per element J = w B^T dP/dFp (12 x 9, dP/dFp from
// NeoHookean::eval_d2W_dF_dFp, neo_hookean.cpp:103-128) and out_c = sum_k J(k, c) w_e[k].
void force_vjp_fp(orc_mesh& m, const double* u, const double* wvec, double* out) {
    for_elements(m.T, [&](int e) {
        double c[12], we[12];
        gather_local(m, e, u, c);
        gather_local(m, e, wvec, we);
        const M3 F = element_F(m, e, c);
        double mixed[81];
        nh_P(F, elem_Fp(m, e), elem_theta(m, e)); // stress finite check as in eval_row
        nh_dP_dFp(F, elem_Fp(m, e), elem_theta(m, e), mixed);
        const double* B = m.B.data() + static_cast<size_t>(e) * 108;
        const double w = m.w[e];
        for (int p = 0; p < 9; ++p) {
            double s = 0;
            for (int k = 0; k < 12; ++k) {
                double jk = 0;
                for (int r = 0; r < 9; ++r) jk += B[r + 9 * k] * mixed[r + 9 * p];
                s += (w * jk) * we[k];
            }
            out[9 * static_cast<size_t>(e) + p] = s;
        }
    });
}

// Rest-position sensitivity of the force (no reference counterpart; pinned by central finite
// differences of the force in the rest positions). Per element s = w_e . g_e = vol P : grad w;
// with H = F - I and Q = A : grad w (A the material tangent of nh_A),
//   d s / d X_a = vol M grad N_a,  M = (P : grad w) I - H^T Q - grad w^T P.
// Per-vertex sums run over the elements in ascending order.
void force_vjp_rest(orc_mesh& m, const double* u, const double* wvec, double* out) {
    if (m.has_Fp) fail(ORC_EINVAL, "rest-position sensitivity needs vertex rest positions and no plastic field");
    std::vector<double> pe(12 * static_cast<size_t>(m.T));
    for_elements(m.T, [&](int e) {
        double c[12], we[12];
        gather_local(m, e, u, c);
        gather_local(m, e, wvec, we);
        const M3 F = element_F(m, e, c);
        const M3 I = eye3();
        const M3 P = nh_P(F, I, elem_theta(m, e));
        double A[81];
        nh_A(F, I, elem_theta(m, e), A);
        const double* B = m.B.data() + static_cast<size_t>(e) * 108;
        double gN[4][3];
        for (int a = 0; a < 4; ++a)
            for (int j = 0; j < 3; ++j) gN[a][j] = B[(3 * j) + 9 * (3 * a)];
        M3 Wg{};
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                double t = 0;
                for (int a = 0; a < 4; ++a) t += we[3 * a + i] * gN[a][j];
                Wg[i + 3 * j] = t;
            }
        M3 Q{};
        double PW = 0;
        for (int r = 0; r < 9; ++r) {
            double t = 0;
            for (int col = 0; col < 9; ++col) t += A[r + 9 * col] * Wg[col];
            Q[r] = t;
            PW += P[r] * Wg[r];
        }
        M3 Mx{};
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) {
                double t = k == l ? PW : 0.0;
                for (int i = 0; i < 3; ++i) t -= (at(F, i, k) - I[i + 3 * k]) * at(Q, i, l) + at(Wg, i, k) * at(P, i, l);
                Mx[k + 3 * l] = t;
            }
        for (int a = 0; a < 4; ++a)
            for (int k = 0; k < 3; ++k) {
                double t = 0;
                for (int l = 0; l < 3; ++l) t += at(Mx, k, l) * gN[a][l];
                pe[12 * static_cast<size_t>(e) + 3 * a + k] = m.w[e] * t;
            }
    });
    std::fill(out, out + m.n, 0.0);
    for (int e = 0; e < m.T; ++e)
        for (int a = 0; a < 4; ++a)
            for (int k = 0; k < 3; ++k) out[3 * m.tets[4 * e + a] + k] += pe[12 * static_cast<size_t>(e) + 3 * a + k];
}

// ---------------------------------------------------------------------------
// Free-DOF reduction (dof_reduction.cpp, reduced_matrix.cpp) and linear solvers.
// ---------------------------------------------------------------------------
struct Reduction {
    int n = 0;
    std::vector<int> free_dofs, free_index;
};

Reduction make_reduction(int n, const int* fixed, int nf) {
    Reduction r;
    r.n = n;
    std::vector<int> f(fixed, fixed + nf);
    std::sort(f.begin(), f.end());
    if (std::adjacent_find(f.begin(), f.end()) != f.end()) fail(ORC_EINVAL, "DofReduction fixed DOFs must be unique");
    if (!f.empty() && (f.front() < 0 || f.back() >= n)) fail(ORC_EINVAL, "DofReduction fixed DOFs must lie in [0, num_dofs)");
    r.free_index.assign(n, -1);
    size_t next = 0;
    for (int d = 0; d < n; ++d) {
        if (next < f.size() && f[next] == d) {
            ++next;
            continue;
        }
        r.free_index[d] = static_cast<int>(r.free_dofs.size());
        r.free_dofs.push_back(d);
    }
    return r;
}

// Free block of a CSC matrix with its whole diagonal (reduced_matrix.cpp:21-66), as CSC.
struct Csc {
    int n = 0;
    std::vector<int> outer, inner;
    std::vector<double> val;
};
Csc reduce_matrix(const Reduction& r, const std::vector<int>& outer, const std::vector<int>& inner,
                  const std::vector<double>& values) {
    Csc out;
    const int nf = static_cast<int>(r.free_dofs.size());
    out.n = nf;
    out.outer.assign(nf + 1, 0);
    for (int column = 0; column < nf; ++column) {
        const int full = r.free_dofs[column];
        bool has_diag = false;
        auto add = [&](int row, double v) {
            if (row == column) has_diag = true;
            out.inner.push_back(row);
            out.val.push_back(v);
        };
        for (int k = outer[full]; k < outer[full + 1]; ++k) {
            const int row = r.free_index[inner[k]];
            if (row < 0) continue;
            if (!has_diag && row > column) add(column, 0.0);
            add(row, values[k]);
        }
        if (!has_diag) add(column, 0.0);
        out.outer[column + 1] = static_cast<int>(out.inner.size());
    }
    return out;
}

// Envelope (skyline) LDL^T without pivoting; stand-in for the reference's direct solvers.
struct Ldlt {
    int n = 0;
    std::vector<long long> start; // row i stores columns [first[i], i]
    std::vector<int> first;
    std::vector<double> L, D;
    std::vector<double> solve(const std::vector<double>& b) const {
        std::vector<double> y = b;
        for (int i = 0; i < n; ++i) {
            const double* ri = L.data() + start[i];
            double s = y[i];
            for (int k = first[i]; k < i; ++k) s -= ri[k - first[i]] * y[k];
            y[i] = s;
        }
        for (int i = 0; i < n; ++i) y[i] /= D[i];
        for (int i = n - 1; i >= 0; --i) {
            const double* ri = L.data() + start[i];
            const double yi = y[i];
            for (int k = first[i]; k < i; ++k) y[k] -= ri[k - first[i]] * yi;
        }
        return y;
    }
};

// Row-oriented LDL^T with the correct ordering of partial sums: within row i, g_ij = K_ij -
// sum_{k<j} g_ik L_jk, where g_ik (k<j) is kept in a scratch row and L_jk is final.
bool ldlt_factor(Ldlt& f, const Csc& K) {
    const int n = K.n;
    f.n = n;
    f.first.assign(n, 0);
    for (int i = 0; i < n; ++i) f.first[i] = i;
    for (int c = 0; c < n; ++c)
        for (int k = K.outer[c]; k < K.outer[c + 1]; ++k) {
            const int row = K.inner[k];
            if (row > c) f.first[row] = std::min(f.first[row], c);
        }
    f.start.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) f.start[i + 1] = f.start[i] + (i - f.first[i] + 1);
    f.L.assign(static_cast<size_t>(f.start[n]), 0.0);
    f.D.assign(n, 0.0);
    for (int c = 0; c < n; ++c)
        for (int k = K.outer[c]; k < K.outer[c + 1]; ++k) {
            const int row = K.inner[k];
            if (row >= c) f.L[f.start[row] + (c - f.first[row])] = K.val[k];
        }
    std::vector<double> g;
    for (int i = 0; i < n; ++i) {
        double* ri = f.L.data() + f.start[i];
        const int fi = f.first[i];
        g.assign(ri, ri + (i - fi + 1));
        for (int j = fi; j < i; ++j) {
            const double* rj = f.L.data() + f.start[j];
            const int fj = f.first[j];
            double s = g[j - fi];
            for (int k = std::max(fi, fj); k < j; ++k) s -= g[k - fi] * rj[k - fj];
            g[j - fi] = s;
        }
        double d = g[i - fi];
        for (int j = fi; j < i; ++j) {
            const double lij = g[j - fi] / f.D[j];
            d -= g[j - fi] * lij;
            ri[j - fi] = lij;
        }
        if (!std::isfinite(d) || d == 0.0) return false;
        f.D[i] = d;
        ri[i - fi] = 1.0;
    }
    return true;
}

double dotv(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

void csc_matvec(const Csc& K, const std::vector<double>& x, std::vector<double>& y) {
    // K is symmetric: y_i = sum_j K(i, j) x_j = column-wise accumulation.
    y.assign(K.n, 0.0);
    for (int c = 0; c < K.n; ++c) {
        const double xc = x[c];
        for (int k = K.outer[c]; k < K.outer[c + 1]; ++k) y[K.inner[k]] += K.val[k] * xc;
    }
}

// Block-Jacobi (3x3 per vertex on the free DOFs) preconditioned CG on K d = b, relative tolerance
// tol; stops on negative curvature. Returns iterations; d holds the iterate.
int block_jacobi_pcg(const Csc& K, const Reduction& r, const std::vector<double>& b, double tol, int max_it,
                     std::vector<double>& d, bool* breakdown) {
    const int nf = K.n;
    // Diagonal 3x3 blocks over free DOFs of the same vertex.
    std::vector<int> vert(nf);
    for (int i = 0; i < nf; ++i) vert[i] = r.free_dofs[i] / 3;
    std::vector<double> Minv(static_cast<size_t>(nf) * 3, 0.0); // row i: coefficients for its vertex-mates
    std::vector<int> mate(static_cast<size_t>(nf) * 3, -1);
    for (int i = 0; i < nf; ++i) {
        int cnt = 0;
        for (int j = std::max(0, i - 2); j < std::min(nf, i + 3); ++j)
            if (vert[j] == vert[i]) mate[3 * i + cnt++] = j;
    }
    // Invert each vertex block (size 1..3).
    std::vector<char> done(nf, 0);
    for (int i = 0; i < nf; ++i) {
        if (done[i]) continue;
        int ids[3], m = 0;
        for (int t = 0; t < 3; ++t)
            if (mate[3 * i + t] >= 0) ids[m++] = mate[3 * i + t];
        double blk[9] = {0};
        for (int a = 0; a < m; ++a)
            for (int k = K.outer[ids[a]]; k < K.outer[ids[a] + 1]; ++k)
                for (int bb = 0; bb < m; ++bb)
                    if (K.inner[k] == ids[bb]) blk[bb + 3 * a] = K.val[k];
        double inv[9] = {0};
        if (m == 1) {
            inv[0] = 1.0 / blk[0];
        } else if (m == 2) {
            const double det = blk[0] * blk[4] - blk[3] * blk[1];
            inv[0] = blk[4] / det;
            inv[4] = blk[0] / det;
            inv[3] = -blk[3] / det;
            inv[1] = -blk[1] / det;
        } else {
            M3 b3;
            for (int t = 0; t < 9; ++t) b3[t] = blk[t];
            const M3 i3 = inv3(b3);
            for (int t = 0; t < 9; ++t) inv[t] = i3[t];
        }
        for (int a = 0; a < m; ++a) {
            done[ids[a]] = 1;
            for (int bb = 0; bb < m; ++bb) Minv[3 * static_cast<size_t>(ids[a]) + bb] = inv[a + 3 * bb];
        }
    }
    auto apply_M = [&](const std::vector<double>& x, std::vector<double>& z) {
        z.assign(nf, 0.0);
        for (int i = 0; i < nf; ++i) {
            double s = 0;
            for (int t = 0; t < 3; ++t)
                if (mate[3 * i + t] >= 0) s += Minv[3 * static_cast<size_t>(i) + t] * x[mate[3 * i + t]];
            z[i] = s;
        }
    };
    d.assign(nf, 0.0);
    std::vector<double> res = b, z, p, Ap;
    apply_M(res, z);
    p = z;
    double rz = dotv(res, z);
    const double bnorm = std::sqrt(dotv(b, b));
    *breakdown = false;
    if (bnorm == 0) return 0;
    int it = 0;
    for (; it < max_it; ++it) {
        csc_matvec(K, p, Ap);
        const double pAp = dotv(p, Ap);
        if (!(pAp > 0)) {
            *breakdown = true;
            if (it == 0) d = p; // first direction is still a preconditioned descent direction
            break;
        }
        const double alpha = rz / pAp;
        for (int i = 0; i < nf; ++i) {
            d[i] += alpha * p[i];
            res[i] -= alpha * Ap[i];
        }
        if (std::sqrt(dotv(res, res)) <= tol * bnorm) {
            ++it;
            break;
        }
        apply_M(res, z);
        const double rz_new = dotv(res, z);
        const double beta = rz_new / rz;
        rz = rz_new;
        for (int i = 0; i < nf; ++i) p[i] = z[i] + beta * p[i];
    }
    return it;
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* orc_last_error(void) { return g_error.c_str(); }

void orc_set_threads(int threads) {
    g_threads = threads;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_nh_W(const double F[9], const double Fp[9], const double theta[2], double* W) {
    return guarded([&] { *W = nh_W(load3(F), load3(Fp), theta); });
}
int orc_nh_dW_dF(const double F[9], const double Fp[9], const double theta[2], double P[9]) {
    return guarded([&] {
        const M3 r = nh_P(load3(F), load3(Fp), theta);
        std::memcpy(P, r.data(), sizeof(double) * 9);
    });
}
int orc_nh_d2W_dF2(const double F[9], const double Fp[9], const double theta[2], double A[81]) {
    return guarded([&] { nh_A(load3(F), load3(Fp), theta, A); });
}
int orc_nh_d2W_dF_dtheta(const double F[9], const double Fp[9], const double theta[2], double out[18]) {
    return guarded([&] { nh_dP_dtheta(load3(F), load3(Fp), theta, out); });
}
int orc_nh_d2W_dF_dFp(const double F[9], const double Fp[9], const double theta[2], double out[81]) {
    return guarded([&] { nh_dP_dFp(load3(F), load3(Fp), theta, out); });
}
int orc_nh_feasible_step(const double F[9], const double Fp[9], const double theta[2], const double dF[9],
                         const double dFp[9], const double dtheta[2], double* alpha) {
    return guarded([&] { *alpha = nh_feasible_step(load3(F), load3(Fp), theta, load3(dF), load3(dFp), dtheta); });
}
int orc_positive_det_step(const double A[9], const double dA[9], double* alpha) {
    return guarded([&] { *alpha = positive_det_step(load3(A), load3(dA)); });
}
int orc_project_psd(int n, const double* H, double* out) {
    return guarded([&] {
        if (n <= 0) fail(ORC_EINVAL, "project_psd: n must be positive");
        project_psd(n, H, out);
    });
}

int orc_mesh_create(int V, const double* X, int T, const int* tets, const double* Xe, const double* theta,
                    int theta_per_element, const double* Fp, orc_mesh** out) {
    *out = nullptr;
    return guarded([&] {
        if (V < 0 || T < 0 || V > std::numeric_limits<int>::max() / 3) fail(ORC_EINVAL, "invalid mesh sizes");
        auto m = std::make_unique<orc_mesh>();
        m->V = V;
        m->T = T;
        m->n = 3 * V;
        m->tets.assign(tets, tets + 4 * static_cast<size_t>(T));
        // MeshTopology ctor (mesh_topology.hpp:25-44): indices in range and distinct per cell.
        for (int e = 0; e < T; ++e) {
            int s[4];
            std::copy(tets + 4 * e, tets + 4 * e + 4, s);
            std::sort(s, s + 4);
            if (s[0] < 0 || s[3] >= V) fail(ORC_EINVAL, "MeshTopology cell has vertex indices outside [0, num_vertices)");
            if (s[0] == s[1] || s[1] == s[2] || s[2] == s[3]) fail(ORC_EINVAL, "MeshTopology cell must contain distinct vertices");
        }
        m->B.resize(static_cast<size_t>(T) * 108);
        m->w.resize(T);
        m->theta.resize(2 * static_cast<size_t>(T));
        for (int e = 0; e < T; ++e) {
            m->theta[2 * e] = theta_per_element ? theta[2 * e] : theta[0];
            m->theta[2 * e + 1] = theta_per_element ? theta[2 * e + 1] : theta[1];
        }
        if (Fp) {
            m->has_Fp = true;
            m->Fp.assign(Fp, Fp + 9 * static_cast<size_t>(T));
        }
        for_elements(T, [&](int e) {
            double Xc[12];
            for (int a = 0; a < 4; ++a)
                for (int k = 0; k < 3; ++k)
                    Xc[3 * a + k] = Xe ? Xe[12 * static_cast<size_t>(e) + 3 * a + k] : X[3 * tets[4 * e + a] + k];
            build_element(Xc, m->B.data() + 108 * static_cast<size_t>(e), &m->w[e]);
        });
        build_assembler(*m);
        *out = m.release();
    });
}

void orc_mesh_destroy(orc_mesh* m) { delete m; }
int orc_mesh_num_dofs(const orc_mesh* m) { return m->n; }
long long orc_mesh_nnz(const orc_mesh* m) { return m->outer.back(); }

int orc_mesh_pattern(const orc_mesh* m, int* outer, int* inner) {
    std::copy(m->outer.begin(), m->outer.end(), outer);
    std::copy(m->inner.begin(), m->inner.end(), inner);
    return ORC_OK;
}

int orc_mesh_eval(orc_mesh* m, const double* u, double* E, double* grad, int hessian, double* values,
                  double* elem_E, double* elem_g, double* elem_H) {
    return guarded([&] {
        if (hessian < 0 || hessian > 2) fail(ORC_EINVAL, "Energy: invalid Hessian kind");
        const double v = mesh_eval(*m, u, grad, hessian, values, elem_E, elem_g, elem_H);
        if (E) *E = v;
    });
}

int orc_mesh_feasible_step(orc_mesh* m, const double* u, const double* du, double* alpha) {
    return guarded([&] { *alpha = mesh_feasible_step(*m, u, du); });
}

int orc_mesh_force_vjp_theta(orc_mesh* m, const double* u, const double* w, double* out) {
    return guarded([&] { force_vjp_theta(*m, u, w, out); });
}

int orc_mesh_force_vjp_fp(orc_mesh* m, const double* u, const double* w, double* out) {
    return guarded([&] { force_vjp_fp(*m, u, w, out); });
}

int orc_mesh_force_vjp_rest(orc_mesh* m, const double* u, const double* w, double* out) {
    return guarded([&] { force_vjp_rest(*m, u, w, out); });
}

// newton_solve (newton.cpp:112-183) with the load term E = elastic - f . u, plus the
// relative-2-norm / Armijo variant and a PCG linear solver option.
int orc_newton_solve(orc_mesh* m, const int* fixed, int nfixed, const double* f_ext, const double* x0,
                     const orc_newton_options* o, double* x_out, orc_newton_result* res) {
    return orc_newton_solve_ex(m, nullptr, fixed, nfixed, f_ext, x0, o, x_out, res, nullptr, 0, nullptr);
}

// The same over a weighted-sum potential (WeightedSumEnergy of the elastic energy and
// QuadraticEnergy terms) with the NewtonStep trace.
int orc_newton_solve_ex(orc_mesh* m, const orc_terms* terms, const int* fixed, int nfixed, const double* f_ext,
                        const double* x0, const orc_newton_options* o, double* x_out, orc_newton_result* res,
                        double* trace, int trace_cap, int* trace_len) {
    return guarded([&] {
        const int n = m->n;
        const double w = terms ? terms->elastic_weight : 1.0, cst = terms ? terms->constant : 0.0;
        const bool has_a = terms && terms->a_indptr;
        // A's entries at their positions in the elastic CSC values (A symmetric: CSR row r is column r).
        std::vector<std::pair<int, double>> apos;
        if (has_a) {
            for (int r = 0; r < n; ++r)
                for (int k = terms->a_indptr[r]; k < terms->a_indptr[r + 1]; ++k) {
                    const int c = terms->a_indices[k];
                    const int* beg = m->inner.data() + m->outer[r];
                    const int* end = m->inner.data() + m->outer[r + 1];
                    const int* at = std::lower_bound(beg, end, c);
                    if (at == end || *at != c) fail(ORC_EINVAL, "QuadraticEnergy: A outside the elastic pattern");
                    apos.emplace_back(static_cast<int>(at - m->inner.data()), terms->a_values[k]);
                }
        }
        int nsteps = 0;
        if (trace_len) *trace_len = 0;
        auto report = [&](int it, double E, double gmax, int shifts, double feas, double step, int lse) {
            if (trace && nsteps < trace_cap) {
                double* t = trace + 7 * static_cast<size_t>(nsteps);
                t[0] = it;
                t[1] = E;
                t[2] = gmax;
                t[3] = shifts;
                t[4] = feas;
                t[5] = step;
                t[6] = lse;
            }
            ++nsteps;
            if (trace_len) *trace_len = std::min(nsteps, trace_cap);
        };
        if (!(o->gradient_tolerance >= 0) || !std::isfinite(o->gradient_tolerance))
            fail(ORC_EINVAL, "newton_solve: gradient_tolerance must be set to a finite non-negative value");
        if (o->max_iterations < 0 || o->max_line_search_steps < 1)
            fail(ORC_EINVAL, "newton_solve: max_iterations must be >= 0 and max_line_search_steps >= 1");
        if (!(o->line_search_shrink > 0.0 && o->line_search_shrink < 1.0))
            fail(ORC_EINVAL, "newton_solve: line_search_shrink must lie in (0, 1)");
        const Reduction red = make_reduction(n, fixed, nfixed);
        std::vector<double> x(x0, x0 + n), f(n, 0.0);
        if (f_ext) f.assign(f_ext, f_ext + n);
        auto energy = [&](const std::vector<double>& y, std::vector<double>* g, std::vector<double>* vals) {
            double E = mesh_eval(*m, y.data(), g ? g->data() : nullptr, vals ? o->hessian : 0,
                                 vals ? vals->data() : nullptr, nullptr, nullptr, nullptr);
            if (terms) {
                E *= w;
                if (g)
                    for (double& v : *g) v *= w;
                if (vals)
                    for (double& v : *vals) v *= w;
                if (has_a) {
                    double q = 0;
                    for (int r = 0; r < n; ++r) {
                        double ax = 0;
                        for (int k = terms->a_indptr[r]; k < terms->a_indptr[r + 1]; ++k)
                            ax += terms->a_values[k] * y[terms->a_indices[k]];
                        q += y[r] * ax;
                        if (g) (*g)[r] += ax;
                    }
                    E += 0.5 * q;
                    if (vals)
                        for (const auto& pa : apos) (*vals)[pa.first] += pa.second;
                }
                E += cst;
            }
            for (int k = 0; k < n; ++k) E -= f[k] * y[k];
            if (g)
                for (int k = 0; k < n; ++k) (*g)[k] -= f[k];
            return E;
        };
        *res = orc_newton_result{};
        const int nf = static_cast<int>(red.free_dofs.size());
        if (nf == 0) {
            res->status = 0;
            res->energy = energy(x, nullptr, nullptr);
            std::copy(x.begin(), x.end(), x_out);
            return;
        }
        std::vector<double> g(n), vals(m->outer.back()), gf(nf), df, dir(n, 0.0), trial(n);
        double gnorm0 = -1;
        for (int it = 0;; ++it) {
            const double E = energy(x, &g, &vals);
            for (int i = 0; i < nf; ++i) gf[i] = g[red.free_dofs[i]];
            double gmax = 0, g2 = 0;
            for (double v : gf) {
                gmax = std::max(gmax, std::abs(v));
                g2 += v * v;
            }
            g2 = std::sqrt(g2);
            if (gnorm0 < 0) gnorm0 = g2;
            const double gn = o->stop_rule == 0 ? gmax : g2;
            res->energy = E;
            res->gradient_norm = gn;
            res->gradient_norm0 = gnorm0;
            res->iterations = it;
            const bool converged = o->stop_rule == 0 ? gn <= o->gradient_tolerance : g2 <= o->gradient_tolerance * gnorm0;
            if (converged) {
                res->status = 0;
                report(it, E, gmax, 0, 0.0, 0.0, 0);
                break;
            }
            if (it == o->max_iterations) {
                res->status = 1;
                report(it, E, gmax, 0, 0.0, 0.0, 0);
                break;
            }
            Csc K = reduce_matrix(red, m->outer, m->inner, vals);
            std::vector<double> rhs(nf);
            for (int i = 0; i < nf; ++i) rhs[i] = -gf[i];
            // descent_direction (newton.cpp:55-72): diagonal shifts until a descent direction.
            double dscale = 1.0;
            std::vector<int> diag_pos(nf);
            for (int c = 0; c < nf; ++c)
                for (int k = K.outer[c]; k < K.outer[c + 1]; ++k)
                    if (K.inner[k] == c) {
                        diag_pos[c] = k;
                        dscale = std::max(dscale, std::abs(K.val[k]));
                    }
            double shift = 1e-8 * dscale;
            bool found = false;
            int nshift = 0;
            for (int shifts = 0;; ++shifts) {
                nshift = shifts;
                bool ok = false;
                if (o->linear_solver == 0) {
                    Ldlt fct;
                    if (ldlt_factor(fct, K)) {
                        df = fct.solve(rhs);
                        ok = true;
                    }
                } else {
                    bool brk = false;
                    const double eta = std::min(o->cg_tolerance, std::sqrt(g2 / gnorm0));
                    res->cg_iterations += block_jacobi_pcg(K, red, rhs, eta, o->cg_max_iterations, df, &brk);
                    ok = true;
                }
                if (ok) {
                    double gd = 0;
                    for (int i = 0; i < nf; ++i) gd += gf[i] * df[i];
                    if (gd < 0.0) {
                        found = true;
                        break;
                    }
                }
                if (shifts == 10) break;
                for (int c = 0; c < nf; ++c) K.val[diag_pos[c]] += shift;
                shift *= 10.0;
            }
            if (!found) {
                res->status = 3;
                report(it, E, gmax, 10, 0.0, 0.0, 0);
                break;
            }
            std::fill(dir.begin(), dir.end(), 0.0);
            for (int i = 0; i < nf; ++i) dir[red.free_dofs[i]] = df[i];
            double gd = 0;
            for (int i = 0; i < nf; ++i) gd += gf[i] * df[i];
            // line_search (newton.cpp:92-108)
            double alpha = mesh_feasible_step(*m, x.data(), dir.data());
            const double feas = alpha;
            int lse = 0;
            bool accepted = false;
            for (int j = 0; j < o->max_line_search_steps; ++j) {
                bool moved = false;
                for (int k = 0; k < n; ++k) {
                    trial[k] = x[k] + alpha * dir[k];
                    moved = moved || trial[k] != x[k];
                }
                if (!moved) break;
                ++res->line_search_evaluations;
                ++lse;
                const double Et = energy(trial, nullptr, nullptr);
                const double noise = 16.0 * kEps * std::max(1.0, std::abs(E));
                const double armijo = o->accept_rule == 1 ? 1e-4 * alpha * gd : 0.0;
                if (Et <= E + armijo + noise) {
                    accepted = true;
                    break;
                }
                alpha *= o->line_search_shrink;
            }
            if (!accepted) {
                res->status = 2;
                report(it, E, gmax, nshift, feas, 0.0, lse);
                break;
            }
            report(it, E, gmax, nshift, feas, alpha, lse);
            x = trial;
        }
        std::copy(x.begin(), x.end(), x_out);
    });
}

int orc_adjoint_theta(orc_mesh* m, const double* u_star, const double* dLdu, const int* fixed, int nfixed,
                      int linear_solver, double cg_tolerance, double* dtheta, double* lambda_out) {
    return guarded([&] {
        const int n = m->n;
        const Reduction red = make_reduction(n, fixed, nfixed);
        const int nf = static_cast<int>(red.free_dofs.size());
        std::vector<double> lam(n, 0.0);
        if (nf > 0) {
            std::vector<double> vals(m->outer.back());
            mesh_eval(*m, u_star, nullptr, 1, vals.data(), nullptr, nullptr, nullptr);
            const Csc K = reduce_matrix(red, m->outer, m->inner, vals);
            std::vector<double> rhs(nf), sol;
            for (int i = 0; i < nf; ++i) rhs[i] = dLdu[red.free_dofs[i]];
            for (double v : rhs)
                if (!std::isfinite(v)) fail(ORC_EDOMAIN, "StaticEquilibriumResponse: nonfinite sensitivity right-hand side");
            if (linear_solver == 0) {
                Ldlt fct;
                if (!ldlt_factor(fct, K)) fail(ORC_EDOMAIN, "StaticEquilibriumResponse: singular equilibrium stiffness");
                sol = fct.solve(rhs);
            } else {
                bool brk = false;
                block_jacobi_pcg(K, red, rhs, cg_tolerance, 100000, sol, &brk);
                if (brk) fail(ORC_EDOMAIN, "StaticEquilibriumResponse: indefinite equilibrium stiffness");
            }
            // Residual check (static_equilibrium_response.cpp:61-68).
            std::vector<double> Ks;
            csc_matvec(K, sol, Ks);
            double rn = 0, bn = 0;
            for (int i = 0; i < nf; ++i) {
                rn += (Ks[i] - rhs[i]) * (Ks[i] - rhs[i]);
                bn += rhs[i] * rhs[i];
            }
            const double tol = linear_solver == 0 ? 1e-8 : std::max(1e-8, cg_tolerance * 10);
            if (!(std::sqrt(rn) <= tol * (1 + std::sqrt(bn))))
                fail(ORC_EDOMAIN, "StaticEquilibriumResponse: inaccurate sensitivity solve");
            for (int i = 0; i < nf; ++i) lam[red.free_dofs[i]] = sol[i];
        }
        force_vjp_theta(*m, u_star, lam.data(), dtheta);
        for (size_t k = 0; k < 2 * static_cast<size_t>(m->T); ++k) dtheta[k] = -dtheta[k];
        if (lambda_out) std::copy(lam.begin(), lam.end(), lambda_out);
    });
}

} // extern "C"
