// Test harness: the tet assembly kernel's plan-driven work (tet_cluster_kernel in
// litepgo_b200/csrc/lpg_assemble.cu) replayed on the host in FP64, for tests/test_tet_plan_host.py
// (built there with g++ together with litepgo_b200/csrc/lpg_plan.cpp). It builds the library's own
// assembly plan, then for every cluster: the element pass (h_a, vol mu grad N_a . grad N_b, vol
// lambda, vol p, g_a per element), the item pass into the cluster's output staging (positions,
// transposes and contributor lists exactly as the plan gives them), and the row copy-out into the
// BSR or CSC values. The test compares the result with the oracle's assembly, so the plan's
// item positions, orientations and contributor lists are checked without a GPU.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "lpg_internal.h"

namespace lpg {
[[noreturn]] void fail(int code, const std::string& what) { throw Error{code, what}; }
void check_cuda(cudaError_t, const char*) {}
} // namespace lpg

namespace {

constexpr int pair10h(int a, int b) {
    const int x = a < b ? a : b, y = a < b ? b : a;
    return x * 4 - (x * (x - 1)) / 2 + (y - x);
}

int stage_index(uint32_t pos, bool csc, int i, int c) {
    const int so = static_cast<int>(pos & 0xffffu), q = static_cast<int>((pos >> 16) & 0xffu),
              nb = static_cast<int>(pos >> 24);
    return csc ? so + 3 * nb * i + 3 * q + c : so + 9 * q + 3 * i + c;
}

} // namespace

// theta: T x 2 (lambda, mu). layout 0: BSR values (9 nnzb), 1: CSC values. Returns 0, or -1 with
// the message in err on a plan failure.
extern "C" int tet_assemble(int V, const double* X, int T, const int32_t* tets, const double* theta, const double* u,
                            int layout, double* energy, double* grad, double* vals, char* err, int errlen) {
    using namespace lpg;
    try {
        HostPlan p;
        build_plan(V, T, tets, p, 4);
        const bool csc = layout == 1;
        const int ncl = static_cast<int>(p.tc_row_ptr.size()) - 1;
        double Etot = 0;
        std::vector<double> ed, stage;
        for (int cl = 0; cl < ncl; ++cl) {
            const int e0 = p.tc_el_ptr[cl], ne = p.tc_el_ptr[cl + 1] - e0;
            const int v0 = p.tc_vert_ptr[cl];
            const int E = ne;
            ed.assign(36 * static_cast<size_t>(E), 0.0);
            for (int el = 0; el < ne; ++el) {
                const uint32_t ew = p.tc_els[e0 + el];
                const int e = static_cast<int>(ew & 0x7fffffffu);
                const uint32_t loc = p.tc_loc[e0 + el];
                int vs[4];
                for (int c = 0; c < 4; ++c) vs[c] = p.tc_verts[v0 + ((loc >> (8 * c)) & 0xffu)];
                for (int c = 0; c < 4; ++c)
                    if (vs[c] != tets[4 * e + c]) throw Error{LPG_ELOGIC, "local vertex index"};
                // Rest geometry: G = Dm^-1 (rows grad N_1..3), vol = det Dm / 6.
                double Dm[9];
                for (int i = 0; i < 3; ++i)
                    for (int c = 0; c < 3; ++c) Dm[3 * i + c] = X[3 * vs[c + 1] + i] - X[3 * vs[0] + i];
                const double dD = Dm[0] * (Dm[4] * Dm[8] - Dm[5] * Dm[7]) - Dm[1] * (Dm[3] * Dm[8] - Dm[5] * Dm[6]) +
                                  Dm[2] * (Dm[3] * Dm[7] - Dm[4] * Dm[6]);
                double G[9];
                G[0] = (Dm[4] * Dm[8] - Dm[5] * Dm[7]) / dD;
                G[1] = (Dm[2] * Dm[7] - Dm[1] * Dm[8]) / dD;
                G[2] = (Dm[1] * Dm[5] - Dm[2] * Dm[4]) / dD;
                G[3] = (Dm[5] * Dm[6] - Dm[3] * Dm[8]) / dD;
                G[4] = (Dm[0] * Dm[8] - Dm[2] * Dm[6]) / dD;
                G[5] = (Dm[2] * Dm[3] - Dm[0] * Dm[5]) / dD;
                G[6] = (Dm[3] * Dm[7] - Dm[4] * Dm[6]) / dD;
                G[7] = (Dm[1] * Dm[6] - Dm[0] * Dm[7]) / dD;
                G[8] = (Dm[0] * Dm[4] - Dm[1] * Dm[3]) / dD;
                const double vol = dD / 6.0, lam = theta[2 * e], mu = theta[2 * e + 1];
                double n[4][3];
                for (int c = 0; c < 3; ++c)
                    for (int j = 0; j < 3; ++j) n[c + 1][j] = G[3 * c + j];
                for (int j = 0; j < 3; ++j) n[0][j] = -(n[1][j] + n[2][j] + n[3][j]);
                double F[9];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double s = i == j ? 1.0 : 0.0;
                        for (int c = 0; c < 3; ++c) s += (u[3 * vs[c + 1] + i] - u[3 * vs[0] + i]) * G[3 * c + j];
                        F[3 * i + j] = s;
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
                const double J = F[0] * C[0] + F[1] * C[1] + F[2] * C[2];
                if (!(J > 0)) throw Error{LPG_EDOMAIN, "det F <= 0"};
                const double L = std::log(J), p_ = lam * L - mu;
                double ff = 0, FiT[9];
                for (int t = 0; t < 9; ++t) {
                    ff += F[t] * F[t];
                    FiT[t] = C[t] / J;
                }
                if (ew >> 31) Etot += vol * (0.5 * mu * (ff - 3.0) - mu * L + 0.5 * lam * L * L);
                for (int b = 0; b < 4; ++b)
                    for (int i = 0; i < 3; ++i) {
                        double h = 0, g = 0;
                        for (int j = 0; j < 3; ++j) {
                            h += FiT[3 * i + j] * n[b][j];
                            g += (mu * F[3 * i + j] + p_ * FiT[3 * i + j]) * n[b][j];
                        }
                        ed[(0 + 3 * b + i) * E + el] = h;
                        ed[(24 + 3 * b + i) * E + el] = vol * g;
                    }
                ed[22 * E + el] = vol * lam;
                ed[23 * E + el] = vol * p_;
                for (int x = 0; x < 4; ++x)
                    for (int y = x; y < 4; ++y)
                        ed[(12 + pair10h(x, y)) * E + el] =
                            vol * mu * (n[x][0] * n[y][0] + n[x][1] * n[y][1] + n[x][2] * n[y][2]);
            }
            const int i0 = p.tc_item_ptr[cl], ni = p.tc_item_ptr[cl + 1] - i0;
            const int r0 = p.tc_row_ptr[cl], nr = p.tc_row_ptr[cl + 1] - r0;
            const int last_v = p.tc_rows[r0 + nr - 1];
            stage.assign(static_cast<size_t>(p.tc_row_so[r0 + nr - 1] + 9 * (p.row_ptr[last_v + 1] - p.row_ptr[last_v])),
                         std::nan(""));
            const uint16_t* ents = p.tc_ents.data() + p.tc_ent_ptr[cl];
            for (int k = 0; k < ni; ++k) {
                const uint32_t* it = p.tc_items.data() + 4 * static_cast<size_t>(i0 + k);
                const uint16_t* en = ents + (it[2] & 0xfffffu);
                const int cnt = static_cast<int>(it[2] >> 20);
                if (it[3] >> 31) {
                    // The list in S contiguous parts summed apart (the kernel's lane group: S = 4
                    // while 4 nd + 32 <= 256, else 2), then added as (p0 + p1) + (p2 + p3).
                    const int nd = p.tc_ndiag[cl], S = 4 * nd + 32 <= 256 ? 4 : 2;
                    double pa[4][9] = {}, pg[4][3] = {};
                    for (int part = 0; part < S; ++part) {
                        double* ap = pa[part];
                        double* gp = pg[part];
                        const int c0 = (cnt * part + S - 1) / S, c1 = (cnt * (part + 1) + S - 1) / S;
                        for (int c = c0; c < c1; ++c) {
                            const int w = en[c], el = w >> 8, pr = (w >> 4) & 15, la = (w >> 2) & 3;
                            for (int i = 0; i < 3; ++i) gp[i] += ed[(24 + 3 * la + i) * E + el];
                            const double dv = ed[22 * E + el] - ed[23 * E + el], mg = ed[(12 + pr) * E + el];
                            for (int i = 0; i < 3; ++i)
                                for (int cc = 0; cc < 3; ++cc)
                                    ap[3 * i + cc] += dv * (ed[(3 * la + i) * E + el] * ed[(3 * la + cc) * E + el]) +
                                                      (i == cc ? mg : 0.0);
                        }
                    }
                    for (int off = 1; off < S; off <<= 1)
                        for (int part = 0; part < S; part += 2 * off) {
                            for (int t = 0; t < 9; ++t) pa[part][t] += pa[part + off][t];
                            for (int i = 0; i < 3; ++i) pg[part][i] += pg[part + off][i];
                        }
                    const double* acc = pa[0];
                    const double* gs = pg[0];
                    const int v = p.tc_rows[r0 + static_cast<int>(it[3] & 0xffu)];
                    for (int i = 0; i < 3; ++i) grad[3 * v + i] = gs[i];
                    for (int i = 0; i < 3; ++i)
                        for (int c = 0; c < 3; ++c) stage[stage_index(it[0], csc, i, c)] = acc[3 * i + c];
                } else {
                    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    for (int c = 0; c < cnt; ++c) {
                        const int w = en[c], el = w >> 8, pr = (w >> 4) & 15, ra = (w >> 2) & 3, cb = w & 3;
                        const double lv = ed[22 * E + el], pv = ed[23 * E + el], mg = ed[(12 + pr) * E + el];
                        for (int i = 0; i < 3; ++i)
                            for (int kk = 0; kk < 3; ++kk) {
                                const double ha_i = ed[(3 * ra + i) * E + el], hb_k = ed[(3 * cb + kk) * E + el];
                                const double hb_i = ed[(3 * cb + i) * E + el], ha_k = ed[(3 * ra + kk) * E + el];
                                acc[3 * i + kk] += lv * ha_i * hb_k - pv * hb_i * ha_k + (i == kk ? mg : 0.0);
                            }
                    }
                    const bool tr = (it[3] >> 30) & 1u;
                    for (int i = 0; i < 3; ++i)
                        for (int c = 0; c < 3; ++c)
                            stage[stage_index(it[0], csc, i, c)] = tr ? acc[3 * c + i] : acc[3 * i + c];
                    if (it[1] != 0xffffffffu)
                        for (int i = 0; i < 3; ++i)
                            for (int c = 0; c < 3; ++c) stage[stage_index(it[1], csc, i, c)] = acc[3 * c + i];
                }
            }
            for (int j = 0; j < nr; ++j) {
                const int v = p.tc_rows[r0 + j], so = p.tc_row_so[r0 + j];
                const int base = p.row_ptr[v], nb = p.row_ptr[v + 1] - base;
                for (int t = 0; t < 9 * nb; ++t) {
                    if (std::isnan(stage[so + t])) throw Error{LPG_ELOGIC, "staging value not written"};
                    vals[9 * static_cast<size_t>(base) + t] = stage[so + t];
                }
            }
        }
        *energy = Etot;
        return 0;
    } catch (const Error& e) {
        std::snprintf(err, errlen, "%s", e.what.c_str());
        return -1;
    }
}
