// lpg_plan.cpp -- host-side assembly plan: block-CSR pattern, vertex incidence, the
// solvers' upper-triangle sliced ELL, and the vertex clusters with per-slot contributor lists.
//
// The scalar pattern of the reference is the union over elements of local x local DOF
// pairs, both triangles (src/core/dof/energy_assembler.cpp:38-47). For 3 DOFs per vertex
// in vertex-major order it is exactly the 3x3 expansion of the vertex adjacency, so the
// block-CSR rows below expand to the reference's CSC columns bit for bit. Contributions to
// one block are kept in ascending element order, the order of the reference's per-column
// contribution lists (energy_assembler.cpp:49-54).

#include <algorithm>
#include <cstring>
#include <exception>
#include <limits>
#include <string>
#include <thread>
#include <utility>

#include "lpg_internal.h"

namespace lpg {

namespace {

// Vertex clusters for the element-once assembly. A cluster grows breadth-first over the vertex
// adjacency from the lowest unassigned vertex until it owns kClusterRows rows or one more row
// would bring its distinct incident elements above kClusterElems (such a row is left for a
// later cluster). Each block slot of an owned row lists its contributing elements in ascending
// element order (the reference's summation order per block); an off-diagonal slot is
// evaluated in the orientation of its lower-numbered vertex, so slot (v, w) and slot (w, v)
// are computed by the same operations and are exact transposes.
void build_clusters(HostPlan& p, const int32_t* tets, const std::vector<int32_t>& inc) {
    const int V = p.V, T = p.T;
    const int ishift = inc_shift(p.K), kMaskE = (1 << ishift) - 1;
    const int K = p.K, sh = cell_bits(K); // vertices per cell, bits per local index in a contributor
    const bool wide = K == 64;             // 32-bit contributors, stored as two 16-bit halves (low first)
    const int max_rows = wide ? kClusterRowsWide : kClusterRows;
    std::vector<int32_t> cl_of(static_cast<size_t>(V), -1), qstamp(static_cast<size_t>(V), -1);
    std::vector<int32_t> estamp(static_cast<size_t>(T), -1);
    std::vector<int32_t> queue;
    int ncl = 0;
    for (int seed = 0; seed < V; ++seed) {
        if (cl_of[seed] >= 0 || p.inc_ptr[seed + 1] == p.inc_ptr[seed]) continue;
        const int c = ncl++;
        queue.assign(1, seed);
        qstamp[seed] = c;
        int nr = 0, ne = 0;
        for (size_t qi = 0; qi < queue.size() && nr < max_rows; ++qi) {
            const int v = queue[qi];
            if (cl_of[v] >= 0) continue;
            int add = 0;
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) add += estamp[inc[k] & kMaskE] != c;
            if (ne + add > kClusterElems) continue;
            cl_of[v] = c;
            ++nr;
            ne += add;
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) estamp[inc[k] & kMaskE] = c;
            for (int k = p.row_ptr[v]; k < p.row_ptr[v + 1]; ++k) {
                const int w = p.col_idx[k];
                if (cl_of[w] < 0 && qstamp[w] != c && p.inc_ptr[w + 1] > p.inc_ptr[w]) {
                    qstamp[w] = c;
                    queue.push_back(w);
                }
            }
        }
    }
    // Rows of each cluster, ascending.
    p.cl_row_ptr.assign(static_cast<size_t>(ncl) + 1, 0);
    for (int v = 0; v < V; ++v)
        if (cl_of[v] >= 0) ++p.cl_row_ptr[cl_of[v] + 1];
    for (int c = 0; c < ncl; ++c) p.cl_row_ptr[c + 1] += p.cl_row_ptr[c];
    p.cl_rows.assign(static_cast<size_t>(p.cl_row_ptr[ncl]), 0);
    {
        std::vector<int32_t> fill(p.cl_row_ptr.begin(), p.cl_row_ptr.end() - 1);
        for (int v = 0; v < V; ++v)
            if (cl_of[v] >= 0) p.cl_rows[fill[cl_of[v]]++] = v;
    }
    p.cl_el_ptr.assign(1, 0);
    p.cl_slot_ptr.assign(1, 0);
    p.cl_ent_ptr.assign(1, 0);
    p.cl_els.clear();
    p.cl_noff.clear();
    p.cl_ntr.clear();
    p.cl_slot.clear();
    p.cl_slot_ent.clear();
    p.cl_ents.clear();
    std::vector<int32_t> eloc(static_cast<size_t>(T), -1), els, colq(static_cast<size_t>(V), -1);
    // A row's off-diagonal contributor words grouped by block (counting sort, each block's words
    // in iteration order), and the cluster's diagonal words row after row.
    std::vector<uint32_t> roww, rowpool, dpool;
    std::vector<int32_t> rowq, qstart, qfill, dstart;
    // Appends a contributor list to cl_ents: one 16-bit word each, or two for wide cells.
    auto append = [&](const uint32_t* first, const uint32_t* last) {
        for (; first != last; ++first) {
            p.cl_ents.push_back(static_cast<uint16_t>(*first & 0xffffu));
            if (wide) p.cl_ents.push_back(static_cast<uint16_t>(*first >> 16));
        }
    };
    std::vector<std::pair<uint32_t, uint32_t>> left, right; // (slot word, entry word)
    for (int c = 0; c < ncl; ++c) {
        const int r0 = p.cl_row_ptr[c], nr = p.cl_row_ptr[c + 1] - r0;
        els.clear();
        for (int j = 0; j < nr; ++j) {
            const int v = p.cl_rows[r0 + j];
            // Each distinct element once (eloc -2 marks one already listed), then ascending.
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE;
                if (eloc[e] == -1) {
                    eloc[e] = -2;
                    els.push_back(e);
                }
            }
        }
        std::sort(els.begin(), els.end());
        for (size_t i = 0; i < els.size(); ++i) {
            const int e = els[i];
            eloc[e] = static_cast<int32_t>(i);
            const bool owner = cl_of[tets[K * static_cast<size_t>(e)]] == c;
            p.cl_els.push_back(static_cast<uint32_t>(e) | (owner ? 0x80000000u : 0u));
        }
        p.cl_el_ptr.push_back(static_cast<int32_t>(p.cl_els.size()));
        const size_t ent0 = p.cl_ents.size();
        dpool.clear();
        dstart.assign(static_cast<size_t>(nr) + 1, 0);
        left.clear();
        right.clear();
        int noff = 0;
        for (int j = 0; j < nr; ++j) {
            const int v = p.cl_rows[r0 + j];
            const int rb = p.row_ptr[v], nb = p.row_ptr[v + 1] - rb;
            // Block index within the row of each column: every vertex of an element incident to v
            // is in v's pattern, so the entries looked up below are always this row's.
            for (int q = 0; q < nb; ++q) colq[p.col_idx[rb + q]] = q;
            rowq.clear();
            roww.clear();
            qstart.assign(static_cast<size_t>(nb) + 1, 0);
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE, a = static_cast<int>(static_cast<uint32_t>(inc[k]) >> ishift);
                const uint32_t el = static_cast<uint32_t>(eloc[e]) << (2 * sh);
                for (int b = 0; b < K; ++b) {
                    const int w = tets[K * static_cast<size_t>(e) + b];
                    if (w == v) {
                        dpool.push_back(el | static_cast<uint32_t>((a << sh) | a));
                        continue;
                    }
                    const int q = colq[w];
                    rowq.push_back(q);
                    roww.push_back(el | static_cast<uint32_t>(v < w ? ((a << sh) | b) : ((b << sh) | a)));
                    ++qstart[static_cast<size_t>(q) + 1];
                }
            }
            dstart[j + 1] = static_cast<int32_t>(dpool.size());
            for (int q = 0; q < nb; ++q) qstart[q + 1] += qstart[q];
            rowpool.resize(roww.size());
            qfill.assign(qstart.begin(), qstart.end() - 1);
            for (size_t i = 0; i < roww.size(); ++i) rowpool[qfill[rowq[i]]++] = roww[i];
            for (int q = 0; q < nb; ++q) {
                const int w = p.col_idx[rb + q];
                if (w == v) continue;
                const uint32_t word = static_cast<uint32_t>(j) | (static_cast<uint32_t>(q) << 8) | (v > w ? 1u << 30 : 0u);
                const uint32_t ent = static_cast<uint32_t>(p.cl_ents.size() - ent0) |
                                     (static_cast<uint32_t>(qstart[q + 1] - qstart[q]) << 20);
                (v > w ? left : right).emplace_back(word, ent);
                append(rowpool.data() + qstart[q], rowpool.data() + qstart[q + 1]);
                ++noff;
            }
        }
        // Slots left of the diagonal first: the solver layout stores only the others.
        for (const auto* side : {&left, &right})
            for (const auto& we : *side) {
                p.cl_slot.push_back(we.first);
                p.cl_slot_ent.push_back(we.second);
            }
        p.cl_ntr.push_back(static_cast<int32_t>(left.size()));
        for (int j = 0; j < nr; ++j) {
            const int v = p.cl_rows[r0 + j];
            const int q = p.diag_slot[v] - p.row_ptr[v];
            p.cl_slot.push_back(static_cast<uint32_t>(j) | (static_cast<uint32_t>(q) << 8) | (1u << 31));
            p.cl_slot_ent.push_back(static_cast<uint32_t>(p.cl_ents.size() - ent0) |
                                    (static_cast<uint32_t>(dstart[j + 1] - dstart[j]) << 20));
            append(dpool.data() + dstart[j], dpool.data() + dstart[j + 1]);
        }
        if (p.cl_ents.size() - ent0 >= (1u << 20) ||
            p.cl_ents.size() >= static_cast<size_t>(std::numeric_limits<int32_t>::max()))
            fail(LPG_EINVAL, "mesh too large for the assembly plan's index ranges");
        while (p.cl_ents.size() % 8 != 0) p.cl_ents.push_back(0); // 16-byte aligned per cluster
        p.cl_noff.push_back(noff);
        p.cl_slot_ptr.push_back(static_cast<int32_t>(p.cl_slot.size()));
        p.cl_ent_ptr.push_back(static_cast<int32_t>(p.cl_ents.size()));
        for (int e : els) eloc[e] = -1;
    }
}

// Tet assembly clusters (HostPlan::tc_*). Growth as build_clusters (breadth-first from the lowest
// unassigned vertex), under the tet limits: a row joins while the cluster's distinct elements
// stay within kTcElems and their distinct vertices within kTcVerts.
void build_tet_clusters(HostPlan& p, const int32_t* tets, const std::vector<int32_t>& inc) {
    const int V = p.V, T = p.T;
    const int kMaskE = (1 << inc_shift(4)) - 1;
    auto vert = [&](int e, int a) { return tets[4 * static_cast<size_t>(e) + a]; };
    std::vector<int32_t> cl_of(static_cast<size_t>(V), -1), qstamp(static_cast<size_t>(V), -1);
    std::vector<int32_t> estamp(static_cast<size_t>(T), -1), vstamp(static_cast<size_t>(V), -1);
    std::vector<int32_t> queue;
    int ncl = 0;
    for (int seed = 0; seed < V; ++seed) {
        if (cl_of[seed] >= 0 || p.inc_ptr[seed + 1] == p.inc_ptr[seed]) continue;
        const int c = ncl++;
        queue.assign(1, seed);
        qstamp[seed] = c;
        int nr = 0, ne = 0, nv = 0, nvals = 0, nents = 0;
        for (size_t qi = 0; qi < queue.size() && nr < kTcRows; ++qi) {
            const int v = queue[qi];
            if (cl_of[v] >= 0) continue;
            int add_e = 0, add_v = 0;
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE;
                if (estamp[e] == c) continue;
                ++add_e;
                for (int a = 0; a < 4; ++a) {
                    const int w = vert(e, a);
                    if (vstamp[w] != c && vstamp[w] != -2 - c) {
                        vstamp[w] = -2 - c; // counted once while sizing this row
                        ++add_v;
                    }
                }
            }
            // Undo the provisional vertex marks.
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k)
                for (int a = 0; a < 4; ++a)
                    if (vstamp[vert(inc[k] & kMaskE, a)] == -2 - c) vstamp[vert(inc[k] & kMaskE, a)] = -1;
            const int add_vals = 9 * (p.row_ptr[v + 1] - p.row_ptr[v]);
            // Contributor words of the row's blocks: at most four per incident element.
            const int add_ents = 4 * (p.inc_ptr[v + 1] - p.inc_ptr[v]);
            if (ne + add_e > kTcElems || nv + add_v > kTcVerts || nvals + add_vals > kTcVals ||
                nents + add_ents > kTcEnts - 7) {
                if (nr == 0) fail(LPG_EINVAL, "vertex neighbourhood exceeds the assembly cluster limits");
                continue;
            }
            cl_of[v] = c;
            ++nr;
            ne += add_e;
            nv += add_v;
            nvals += add_vals;
            nents += add_ents;
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE;
                estamp[e] = c;
                for (int a = 0; a < 4; ++a) vstamp[vert(e, a)] = c;
            }
            for (int k = p.row_ptr[v]; k < p.row_ptr[v + 1]; ++k) {
                const int w = p.col_idx[k];
                if (cl_of[w] < 0 && qstamp[w] != c && p.inc_ptr[w + 1] > p.inc_ptr[w]) {
                    qstamp[w] = c;
                    queue.push_back(w);
                }
            }
        }
    }
    p.tc_row_ptr.assign(static_cast<size_t>(ncl) + 1, 0);
    for (int v = 0; v < V; ++v)
        if (cl_of[v] >= 0) ++p.tc_row_ptr[cl_of[v] + 1];
    for (int c = 0; c < ncl; ++c) p.tc_row_ptr[c + 1] += p.tc_row_ptr[c];
    p.tc_rows.assign(static_cast<size_t>(p.tc_row_ptr[ncl]), 0);
    {
        std::vector<int32_t> fill(p.tc_row_ptr.begin(), p.tc_row_ptr.end() - 1);
        for (int v = 0; v < V; ++v)
            if (cl_of[v] >= 0) p.tc_rows[fill[cl_of[v]]++] = v;
    }
    p.tc_row_so.assign(p.tc_rows.size(), 0);
    p.tc_el_ptr.assign(1, 0);
    p.tc_vert_ptr.assign(1, 0);
    p.tc_item_ptr.assign(1, 0);
    p.tc_ent_ptr.assign(1, 0);
    p.tc_els.clear();
    p.tc_loc.clear();
    p.tc_verts.clear();
    p.tc_items.clear();
    p.tc_ndiag.clear();
    p.tc_ents.clear();
    std::vector<int32_t> eloc(static_cast<size_t>(T), -1), vloc(static_cast<size_t>(V), -1), rloc(static_cast<size_t>(V), -1);
    std::vector<int32_t> colq(static_cast<size_t>(V), -1);
    std::vector<int32_t> els, verts;
    // An item's contributor words are pool[start, start + cnt): the cluster's words, block by block.
    struct Item {
        uint32_t w0, w1, w3;
        int start, cnt;
    };
    std::vector<Item> diag, edge;
    std::vector<uint16_t> pool, roww;
    std::vector<int32_t> rowq, qstart, qfill;
    auto pack = [](int so, int q, int nb) {
        return static_cast<uint32_t>(so) | (static_cast<uint32_t>(q) << 16) | (static_cast<uint32_t>(nb) << 24);
    };
    for (int c = 0; c < ncl; ++c) {
        const int r0 = p.tc_row_ptr[c], nr = p.tc_row_ptr[c + 1] - r0;
        els.clear();
        verts.clear();
        int so = 0;
        for (int j = 0; j < nr; ++j) {
            const int v = p.tc_rows[r0 + j];
            rloc[v] = j;
            p.tc_row_so[r0 + j] = so;
            const int nb = p.row_ptr[v + 1] - p.row_ptr[v];
            if (nb > 255) fail(LPG_EINVAL, "vertex has more than 254 neighbours (assembly plan limit)");
            so += 9 * nb;
            // Each distinct element once (eloc -2 marks one already listed), then ascending.
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE;
                if (eloc[e] == -1) {
                    eloc[e] = -2;
                    els.push_back(e);
                }
            }
        }
        if (so > 65535) fail(LPG_EINVAL, "assembly cluster output exceeds its staging index range");
        std::sort(els.begin(), els.end());
        for (int e : els)
            for (int a = 0; a < 4; ++a)
                if (vloc[vert(e, a)] == -1) {
                    vloc[vert(e, a)] = -2;
                    verts.push_back(vert(e, a));
                }
        std::sort(verts.begin(), verts.end());
        for (size_t i = 0; i < verts.size(); ++i) {
            vloc[verts[i]] = static_cast<int32_t>(i);
            p.tc_verts.push_back(verts[i]);
        }
        for (size_t i = 0; i < els.size(); ++i) {
            const int e = els[i];
            eloc[e] = static_cast<int32_t>(i);
            const bool owner = cl_of[vert(e, 0)] == c;
            p.tc_els.push_back(static_cast<uint32_t>(e) | (owner ? 0x80000000u : 0u));
            uint32_t loc = 0;
            for (int a = 0; a < 4; ++a) loc |= static_cast<uint32_t>(vloc[vert(e, a)]) << (8 * a);
            p.tc_loc.push_back(loc);
        }
        diag.clear();
        edge.clear();
        pool.clear();
        for (int j = 0; j < nr; ++j) {
            const int v = p.tc_rows[r0 + j];
            const int rb = p.row_ptr[v], nb = p.row_ptr[v + 1] - rb;
            // Block index within the row of each column: every vertex of an element incident to v
            // is in v's pattern, so the entries looked up below are always this row's.
            for (int q = 0; q < nb; ++q) colq[p.col_idx[rb + q]] = q;
            // Contributors of every block of row v, in element order (the incidence is ascending):
            // each incident element gives one word to each of four blocks; the words are counted
            // per block and then placed block after block, each block's in that order.
            rowq.clear();
            roww.clear();
            qstart.assign(static_cast<size_t>(nb) + 1, 0);
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & kMaskE;
                const int a = static_cast<int>(static_cast<uint32_t>(inc[k]) >> inc_shift(4));
                const uint32_t el = static_cast<uint32_t>(eloc[e]) << 8;
                for (int b = 0; b < 4; ++b) {
                    const int w = vert(e, b);
                    const int q = colq[w];
                    const int lo = v <= w ? a : b, hi = v <= w ? b : a;
                    const int x = std::min(a, b), y = std::max(a, b);
                    const int pr = x * 4 - (x * (x - 1)) / 2 + (y - x); // element block pair index (a <= b order)
                    rowq.push_back(q);
                    roww.push_back(static_cast<uint16_t>(el | static_cast<uint32_t>((pr << 4) | (lo << 2) | hi)));
                    ++qstart[static_cast<size_t>(q) + 1];
                }
            }
            for (int q = 0; q < nb; ++q) qstart[q + 1] += qstart[q];
            const int base = static_cast<int>(pool.size());
            pool.resize(pool.size() + roww.size());
            qfill.assign(qstart.begin(), qstart.end() - 1);
            for (size_t i = 0; i < roww.size(); ++i) pool[base + qfill[rowq[i]]++] = roww[i];
            for (int q = 0; q < nb; ++q) {
                const int w = p.col_idx[rb + q];
                const int start = base + qstart[q], cnt = qstart[q + 1] - qstart[q];
                if (w == v) {
                    diag.push_back({pack(p.tc_row_so[r0 + j], q, nb), 0xffffffffu, 0x80000000u | static_cast<uint32_t>(j),
                                    start, cnt});
                } else if (cl_of[w] == c) {
                    if (v > w) continue; // summed with the lower row's item
                    const int k = rloc[w];
                    const int wb = p.row_ptr[w], wn = p.row_ptr[w + 1] - wb;
                    const int qw = static_cast<int>(std::lower_bound(p.col_idx.data() + wb, p.col_idx.data() + wb + wn, v) -
                                                    (p.col_idx.data() + wb));
                    edge.push_back({pack(p.tc_row_so[r0 + j], q, nb), pack(p.tc_row_so[r0 + k], qw, wn), 0u, start, cnt});
                } else {
                    edge.push_back({pack(p.tc_row_so[r0 + j], q, nb), 0xffffffffu, v > w ? 0x40000000u : 0u, start, cnt});
                }
            }
        }
        auto by_count = [](const Item& x, const Item& y) { return x.cnt > y.cnt; };
        std::stable_sort(diag.begin(), diag.end(), by_count);
        std::stable_sort(edge.begin(), edge.end(), by_count);
        const size_t ent0 = p.tc_ents.size();
        for (const auto* group : {&diag, &edge})
            for (const Item& it : *group) {
                const size_t first = p.tc_ents.size() - ent0;
                if (first >= (1u << 20) || it.cnt >= (1 << 12))
                    fail(LPG_EINVAL, "mesh too large for the assembly plan's index ranges");
                p.tc_items.insert(p.tc_items.end(),
                                  {it.w0, it.w1, static_cast<uint32_t>(first) | (static_cast<uint32_t>(it.cnt) << 20), it.w3});
                p.tc_ents.insert(p.tc_ents.end(), pool.begin() + it.start, pool.begin() + it.start + it.cnt);
            }
        while (p.tc_ents.size() % 8 != 0) p.tc_ents.push_back(0); // 16-byte aligned per cluster
        p.tc_ndiag.push_back(static_cast<int32_t>(diag.size()));
        p.tc_el_ptr.push_back(static_cast<int32_t>(p.tc_els.size()));
        p.tc_vert_ptr.push_back(static_cast<int32_t>(p.tc_verts.size()));
        p.tc_item_ptr.push_back(static_cast<int32_t>(p.tc_items.size() / 4));
        p.tc_ent_ptr.push_back(static_cast<int32_t>(p.tc_ents.size()));
        if (p.tc_ents.size() >= static_cast<size_t>(std::numeric_limits<int32_t>::max()))
            fail(LPG_EINVAL, "mesh too large for the assembly plan's index ranges");
        for (int e : els) eloc[e] = -1;
        for (int w : verts) vloc[w] = -1;
        for (int j = 0; j < nr; ++j) rloc[p.tc_rows[r0 + j]] = -1;
    }
}

} // namespace

void build_plan(int V, int T, const int32_t* tets, HostPlan& p, int K) {
    p.K = K;
    if (V < 0 || T < 0) fail(LPG_EINVAL, "MeshTopology requires a non-negative vertex count");
    if (V > std::numeric_limits<int>::max() / 3) fail(LPG_EINVAL, "VertexDofMap requires total DOFs fitting in int");
    if (K != 4 && K != 8 && K != 64) fail(LPG_EINVAL, "cells must have 4 (tet), 8 (hex) or 64 (Hermite hex) nodes");
    const int ishift = inc_shift(K);
    if (T >= (1 << ishift))
        fail(LPG_EINVAL, "mesh has too many elements for the assembly plan (limit 2^" + std::to_string(ishift) + ")");
    for (int e = 0; e < T; ++e) {
        int s[64];
        std::memcpy(s, tets + K * static_cast<size_t>(e), K * sizeof(int));
        std::sort(s, s + K);
        if (s[0] < 0 || s[K - 1] >= V)
            fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " has vertex indices outside [0, num_vertices)");
        for (int a = 1; a < K; ++a)
            if (s[a] == s[a - 1])
                fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " must contain distinct vertices");
    }
    p.V = V;
    p.T = T;
    // Incidence (row -> pairs in element order), by counting sort.
    p.inc_ptr.assign(static_cast<size_t>(V) + 1, 0);
    for (int64_t k = 0; k < K * static_cast<int64_t>(T); ++k) ++p.inc_ptr[tets[k] + 1];
    for (int v = 0; v < V; ++v) p.inc_ptr[v + 1] += p.inc_ptr[v];
    const int64_t npairs = p.inc_ptr[V];
    std::vector<int32_t> inc(static_cast<size_t>(npairs));
    {
        std::vector<int32_t> fill(p.inc_ptr.begin(), p.inc_ptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int a = 0; a < K; ++a) {
                const int v = tets[K * static_cast<size_t>(e) + a];
                inc[fill[v]++] = e | (a << ishift);
            }
    }
    int maxdeg = 0;
    for (int v = 0; v < V; ++v) maxdeg = std::max(maxdeg, p.inc_ptr[v + 1] - p.inc_ptr[v]);
    // A vertex's elements must fit in one assembly cluster.
    if (maxdeg > kClusterElems)
        fail(LPG_EINVAL, "vertex valence " + std::to_string(maxdeg) + " exceeds the supported maximum of " +
                             std::to_string(kClusterElems));
    // Block-CSR pattern: sorted unique neighbours (including the vertex itself).
    p.row_ptr.assign(static_cast<size_t>(V) + 1, 0);
    {
        std::vector<int32_t> cols;
        cols.reserve(static_cast<size_t>(npairs) * 2);
        std::vector<int32_t> buf;
        for (int v = 0; v < V; ++v) {
            buf.clear();
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & ((1 << ishift) - 1);
                for (int b = 0; b < K; ++b) buf.push_back(tets[K * static_cast<size_t>(e) + b]);
            }
            std::sort(buf.begin(), buf.end());
            buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
            cols.insert(cols.end(), buf.begin(), buf.end());
            p.row_ptr[v + 1] = static_cast<int32_t>(cols.size());
            if (cols.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max() / 9))
                fail(LPG_EINVAL, "Hessian has too many entries for int32 CSC indices");
        }
        p.col_idx.swap(cols);
    }
    p.diag_slot.assign(static_cast<size_t>(V), -1);
    for (int v = 0; v < V; ++v)
        for (int k = p.row_ptr[v]; k < p.row_ptr[v + 1]; ++k)
            if (p.col_idx[k] == v) p.diag_slot[v] = k;
    // Upper-triangle sliced ELL (SELL-32): rows sorted by block count (descending, then by
    // index) within windows of kSellWindow rows, cut into chunks of 32. Own slots (columns >=
    // row, diagonal first) are as wide as the chunk's longest own list, padding pointing at the
    // row itself (values stay zero); borrowed slots (columns < row) reference the owning row's
    // block, padding the zero block after the own slots.
    {
        const int nch = (V + 31) / 32;
        std::vector<int32_t> order(static_cast<size_t>(V));
        for (int v = 0; v < V; ++v) order[v] = v;
        for (int w0 = 0; w0 < V; w0 += kSellWindow) {
            const int w1 = std::min(V, w0 + kSellWindow);
            std::stable_sort(order.begin() + w0, order.begin() + w1, [&](int a, int b) {
                return p.row_ptr[a + 1] - p.row_ptr[a] > p.row_ptr[b + 1] - p.row_ptr[b];
            });
        }
        // Own list of v: [diag, row end); borrowed: [row start, diag). A vertex in no element
        // has neither.
        auto own0 = [&](int v) { return p.diag_slot[v] >= 0 ? p.diag_slot[v] : p.row_ptr[v + 1]; };
        p.sell_ptr.assign(static_cast<size_t>(nch) + 1, 0);
        p.sell_bptr.assign(static_cast<size_t>(nch) + 1, 0);
        p.sell_row.assign(32 * static_cast<size_t>(nch), -1);
        p.sell_base.assign(static_cast<size_t>(V), 0);
        int64_t slots = 0, bslots = 0;
        for (int c = 0; c < nch; ++c) {
            int width = 0, bwidth = 0;
            for (int l = 0; l < 32 && 32 * c + l < V; ++l) {
                const int r = order[32 * c + l];
                p.sell_row[32 * static_cast<size_t>(c) + l] = r;
                width = std::max(width, p.row_ptr[r + 1] - own0(r));
                bwidth = std::max(bwidth, own0(r) - p.row_ptr[r]);
                p.sell_base[r] = static_cast<int32_t>(std::min<int64_t>(9 * slots + l, std::numeric_limits<int32_t>::max()));
            }
            slots += 32 * static_cast<int64_t>(width);
            bslots += 32 * static_cast<int64_t>(bwidth);
            if (9 * slots + 9 * 32 >= std::numeric_limits<int32_t>::max() ||
                bslots >= std::numeric_limits<int32_t>::max() / 2)
                fail(LPG_EINVAL, "mesh too large for the solver's int32 Hessian offsets");
            p.sell_ptr[c + 1] = static_cast<int32_t>(slots);
            p.sell_bptr[c + 1] = static_cast<int32_t>(bslots);
        }
        const int32_t zero = static_cast<int32_t>(9 * slots);
        p.sell_col.assign(static_cast<size_t>(slots), 0);
        p.sell_bref.assign(2 * static_cast<size_t>(bslots), 0);
        for (int c = 0; c < nch; ++c) {
            const int width = (p.sell_ptr[c + 1] - p.sell_ptr[c]) / 32;
            const int bwidth = (p.sell_bptr[c + 1] - p.sell_bptr[c]) / 32;
            for (int l = 0; l < 32; ++l) {
                const int r = p.sell_row[32 * static_cast<size_t>(c) + l];
                const int o0 = r < 0 ? 0 : own0(r);
                const int no = r < 0 ? 0 : p.row_ptr[r + 1] - o0;
                const int nbr = r < 0 ? 0 : o0 - p.row_ptr[r];
                for (int q = 0; q < width; ++q)
                    p.sell_col[p.sell_ptr[c] + 32 * static_cast<size_t>(q) + l] = q < no ? p.col_idx[o0 + q] : std::max(r, 0);
                for (int q = 0; q < bwidth; ++q) {
                    int32_t idx = zero, col = std::max(r, 0);
                    if (q < nbr) {
                        col = p.col_idx[p.row_ptr[r] + q];
                        // Block (col, r) is own block k - own0(col) of row col.
                        const int32_t* beg = p.col_idx.data() + own0(col);
                        const int32_t* end = p.col_idx.data() + p.row_ptr[col + 1];
                        const int k = static_cast<int>(std::lower_bound(beg, end, r) - p.col_idx.data());
                        if (k >= p.row_ptr[col + 1] || p.col_idx[k] != r) fail(LPG_ELOGIC, "Hessian pattern is not symmetric");
                        idx = p.sell_base[col] + 32 * 9 * (k - own0(col));
                    }
                    const size_t at = 2 * (p.sell_bptr[c] + 32 * static_cast<size_t>(q) + l);
                    p.sell_bref[at] = idx;
                    p.sell_bref[at + 1] = col;
                }
            }
        }
    }
    p.unused_rows.clear();
    for (int v = 0; v < V; ++v)
        if (p.inc_ptr[v + 1] == p.inc_ptr[v]) p.unused_rows.push_back(v); // no element: zero gradient, no blocks
    if (K != 4) {
        build_clusters(p, tets, inc);
        return;
    }
    // The two cluster plans read the pattern and incidence only and write disjoint fields (cl_*
    // and tc_*): they are built side by side. An error of the first is reported before one of
    // the second, as when they ran in turn.
    std::exception_ptr tet_error;
    std::thread tet([&] {
        try {
            build_tet_clusters(p, tets, inc);
        } catch (...) {
            tet_error = std::current_exception();
        }
    });
    try {
        build_clusters(p, tets, inc);
    } catch (...) {
        tet.join();
        throw;
    }
    tet.join();
    if (tet_error) std::rethrow_exception(tet_error);
}

void check_clusters(const HostPlan& p, const int32_t* tets) {
    const int V = p.V, T = p.T;
    const int ncl = static_cast<int>(p.cl_row_ptr.size()) - 1;
    auto bad = [](const char* what) { fail(LPG_ELOGIC, std::string("assembly cluster plan: ") + what); };
    const int K = p.K, sh = cell_bits(K);
    const bool wide = K == 64;
    auto vert = [&](int e, int a) { return tets[K * static_cast<size_t>(e) + a]; };
    // Incidence (vertex -> elements, ascending), independent of the plan's own.
    std::vector<int32_t> ptr(static_cast<size_t>(V) + 1, 0), inc(K * static_cast<size_t>(T));
    for (size_t k = 0; k < K * static_cast<size_t>(T); ++k) ++ptr[tets[k] + 1];
    for (int v = 0; v < V; ++v) ptr[v + 1] += ptr[v];
    {
        std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int a = 0; a < K; ++a) inc[fill[vert(e, a)]++] = e;
    }
    std::vector<int> owner(static_cast<size_t>(V), -1), energy_count(static_cast<size_t>(T), 0);
    for (int c = 0; c < ncl; ++c)
        for (int k = p.cl_row_ptr[c]; k < p.cl_row_ptr[c + 1]; ++k) {
            if (owner[p.cl_rows[k]] >= 0) bad("vertex owned twice");
            owner[p.cl_rows[k]] = c;
        }
    for (int v = 0; v < V; ++v)
        if ((owner[v] >= 0) != (ptr[v + 1] > ptr[v])) bad("referenced vertex without a cluster");
    for (int c = 0; c < ncl; ++c) {
        const int e0 = p.cl_el_ptr[c], ne = p.cl_el_ptr[c + 1] - e0;
        if (p.cl_row_ptr[c + 1] - p.cl_row_ptr[c] > (wide ? kClusterRowsWide : kClusterRows) || ne > kClusterElems)
            bad("cluster over its limits");
        for (int i = 0; i < ne; ++i) {
            const int e = static_cast<int>(p.cl_els[e0 + i] & 0x7fffffffu);
            if (i > 0 && e <= static_cast<int>(p.cl_els[e0 + i - 1] & 0x7fffffffu)) bad("elements not ascending");
            bool touches = false;
            for (int a = 0; a < K; ++a) touches = touches || owner[vert(e, a)] == c;
            if (!touches) bad("element not incident to the cluster");
            if (p.cl_els[e0 + i] >> 31) {
                if (owner[vert(e, 0)] != c) bad("energy counted by a non-owner");
                ++energy_count[e];
            }
        }
        const int s0 = p.cl_slot_ptr[c], ns = p.cl_slot_ptr[c + 1] - s0;
        int rows_slots = 0;
        for (int k = p.cl_row_ptr[c]; k < p.cl_row_ptr[c + 1]; ++k)
            rows_slots += p.row_ptr[p.cl_rows[k] + 1] - p.row_ptr[p.cl_rows[k]];
        if (ns != rows_slots) bad("slot count differs from the rows' blocks");
        std::vector<char> seen(static_cast<size_t>(rows_slots), 0);
        std::vector<int> first(static_cast<size_t>(p.cl_row_ptr[c + 1] - p.cl_row_ptr[c]) + 1, 0);
        for (int j = 0; j + 1 < static_cast<int>(first.size()); ++j) {
            const int v = p.cl_rows[p.cl_row_ptr[c] + j];
            first[j + 1] = first[j] + p.row_ptr[v + 1] - p.row_ptr[v];
        }
        for (int s = 0; s < ns; ++s) {
            const uint32_t d = p.cl_slot[s0 + s], de = p.cl_slot_ent[s0 + s];
            const int j = d & 0xffu, q = (d >> 8) & 0x3fffffu;
            const bool diag = d >> 31, tr = (d >> 30) & 1u;
            if ((s >= p.cl_noff[c]) != diag) bad("slot order");
            if (!diag && (s < p.cl_ntr[c]) != tr) bad("slot order (left of the diagonal first)");
            if (j >= static_cast<int>(first.size()) - 1) bad("slot row outside the cluster");
            const int v = p.cl_rows[p.cl_row_ptr[c] + j];
            if (q >= p.row_ptr[v + 1] - p.row_ptr[v]) bad("slot position outside its row");
            if (seen[first[j] + q]++) bad("slot listed twice");
            const int w = p.col_idx[p.row_ptr[v] + q];
            if (diag != (v == w) || tr != (v > w)) bad("slot flags");
            const int lo = std::min(v, w), hi = std::max(v, w);
            // Expected contributors: the elements holding both vertices, ascending.
            std::vector<int> expect;
            for (int k = ptr[v]; k < ptr[v + 1]; ++k) {
                const int e = inc[k];
                bool has = false;
                for (int a = 0; a < K; ++a) has = has || vert(e, a) == w;
                if (has) expect.push_back(e);
            }
            if ((de >> 20) != expect.size()) bad("slot contributor count");
            const size_t off = p.cl_ent_ptr[c] + (de & 0xfffffu);
            for (size_t t = 0; t < expect.size(); ++t) {
                const uint32_t en = wide ? p.cl_ents[off + 2 * t] | (static_cast<uint32_t>(p.cl_ents[off + 2 * t + 1]) << 16)
                                         : p.cl_ents[off + t];
                const int el = en >> (2 * sh), a = (en >> sh) & (K - 1), b = en & (K - 1);
                if (el >= ne) bad("contributor outside the cluster");
                const int e = static_cast<int>(p.cl_els[e0 + el] & 0x7fffffffu);
                if (e != expect[t]) bad("contributor list differs from the elements sharing the block");
                if (vert(e, a) != lo || vert(e, b) != hi) bad("contributor local indices");
            }
        }
    }
    for (int e = 0; e < T; ++e)
        if (energy_count[e] != 1) bad("element energy not counted exactly once");
    size_t contributors = 0;
    for (uint32_t de : p.cl_slot_ent) contributors += de >> 20;
    if (contributors != static_cast<size_t>(K) * K * T) bad("contributor total differs from K^2 per element");
    for (int c = 0; c < ncl; ++c)
        if (p.cl_ent_ptr[c] % 8 != 0) bad("contributor lists not 16-byte aligned");
}

void check_tet_clusters(const HostPlan& p, const int32_t* tets) {
    auto bad = [](const char* what) { fail(LPG_ELOGIC, std::string("tet assembly plan: ") + what); };
    if (p.K != 4) {
        if (!p.tc_items.empty()) bad("tet clusters on a non-tet mesh");
        return;
    }
    const int V = p.V, T = p.T;
    auto vert = [&](int e, int a) { return tets[4 * static_cast<size_t>(e) + a]; };
    const int ncl = static_cast<int>(p.tc_row_ptr.size()) - 1;
    std::vector<int> owner(static_cast<size_t>(V), -1), energy_count(static_cast<size_t>(T), 0);
    for (int c = 0; c < ncl; ++c)
        for (int k = p.tc_row_ptr[c]; k < p.tc_row_ptr[c + 1]; ++k) {
            if (owner[p.tc_rows[k]] >= 0) bad("vertex owned twice");
            owner[p.tc_rows[k]] = c;
        }
    for (int v = 0; v < V; ++v)
        if ((owner[v] >= 0) != (p.inc_ptr[v + 1] > p.inc_ptr[v])) bad("referenced vertex without a cluster");
    // Every block of every row must be written exactly once, with the right contributors.
    std::vector<char> written(static_cast<size_t>(p.nnzb()), 0);
    std::vector<int> incident;
    for (int c = 0; c < ncl; ++c) {
        const int r0 = p.tc_row_ptr[c], nr = p.tc_row_ptr[c + 1] - r0;
        const int e0 = p.tc_el_ptr[c], ne = p.tc_el_ptr[c + 1] - e0;
        const int v0 = p.tc_vert_ptr[c], nv = p.tc_vert_ptr[c + 1] - v0;
        if (nr > kTcRows || ne > kTcElems || nv > kTcVerts) bad("cluster over its limits");
        if (p.tc_item_ptr[c + 1] - p.tc_item_ptr[c] > kTcItems) bad("cluster items over their limit");
        {
            const int nn = p.tc_ent_ptr[c + 1] - p.tc_ent_ptr[c];
            if (nn > kTcEnts || nn % 8 != 0 || p.tc_ent_ptr[c] % 8 != 0) bad("cluster contributor lists over their limit");
        }
        if (nr == 0) bad("cluster without rows");
        {
            const int vl = p.tc_rows[r0 + nr - 1];
            if (p.tc_row_so[r0 + nr - 1] + 9 * (p.row_ptr[vl + 1] - p.row_ptr[vl]) > kTcVals)
                bad("cluster staging over its limit");
        }
        for (int i = 0; i < nv; ++i)
            if (i > 0 && p.tc_verts[v0 + i] <= p.tc_verts[v0 + i - 1]) bad("vertices not ascending");
        for (int i = 0; i < ne; ++i) {
            const int e = static_cast<int>(p.tc_els[e0 + i] & 0x7fffffffu);
            if (e >= T || (i > 0 && e <= static_cast<int>(p.tc_els[e0 + i - 1] & 0x7fffffffu))) bad("elements not ascending");
            bool touches = false;
            for (int a = 0; a < 4; ++a) {
                const int lv = static_cast<int>((p.tc_loc[e0 + i] >> (8 * a)) & 0xffu);
                if (lv >= nv || p.tc_verts[v0 + lv] != vert(e, a)) bad("local vertex index");
                touches = touches || owner[vert(e, a)] == c;
            }
            if (!touches) bad("element not incident to the cluster");
            if (p.tc_els[e0 + i] >> 31) {
                if (owner[vert(e, 0)] != c) bad("energy counted by a non-owner");
                ++energy_count[e];
            }
        }
        // Staging offsets: rows back to back.
        int so = 0;
        for (int j = 0; j < nr; ++j) {
            const int v = p.tc_rows[r0 + j];
            if (j > 0 && v <= p.tc_rows[r0 + j - 1]) bad("rows not ascending");
            if (p.tc_row_so[r0 + j] != so) bad("row staging offset");
            so += 9 * (p.row_ptr[v + 1] - p.row_ptr[v]);
        }
        const int i0 = p.tc_item_ptr[c], ni = p.tc_item_ptr[c + 1] - i0;
        const int nd = p.tc_ndiag[c];
        if (nd != nr) bad("one diagonal item per row");
        size_t prev = ~size_t(0);
        for (int it = 0; it < ni; ++it) {
            const uint32_t* w = p.tc_items.data() + 4 * static_cast<size_t>(i0 + it);
            const bool dg = w[3] >> 31, tr = (w[3] >> 30) & 1u;
            if ((it < nd) != dg) bad("diagonal items first");
            const size_t cnt = w[2] >> 20;
            if (it == nd) prev = ~size_t(0);
            if (cnt > prev) bad("items not sorted by contributor count");
            prev = cnt;
            // Decode a staging position into (row j, block q) and check its packing.
            auto locate = [&](uint32_t pos, int& j, int& q) {
                const int s0 = static_cast<int>(pos & 0xffffu), qq = static_cast<int>((pos >> 16) & 0xffu),
                          nb = static_cast<int>(pos >> 24);
                j = -1;
                for (int r = 0; r < nr; ++r)
                    if (p.tc_row_so[r0 + r] == s0) j = r;
                if (j < 0) bad("staging position is not a row start");
                const int v = p.tc_rows[r0 + j];
                if (nb != p.row_ptr[v + 1] - p.row_ptr[v] || qq >= nb) bad("staging position row length");
                q = qq;
            };
            int j1, q1;
            locate(w[0], j1, q1);
            const int v = p.tc_rows[r0 + j1];
            const int x = p.col_idx[p.row_ptr[v] + q1];
            if (dg != (x == v)) bad("diagonal flag");
            if (dg && static_cast<int>(w[3] & 0xffu) != j1) bad("diagonal row index");
            if (written[p.row_ptr[v] + q1]++) bad("block written twice");
            if (w[1] != 0xffffffffu) {
                int j2, q2;
                locate(w[1], j2, q2);
                const int xv = p.tc_rows[r0 + j2];
                if (dg || owner[x] != c || xv != x || p.col_idx[p.row_ptr[x] + q2] != v || v > x || tr)
                    bad("second position of an owned edge");
                if (written[p.row_ptr[x] + q2]++) bad("block written twice");
            } else if (!dg) {
                if (owner[x] == c) bad("owned edge without its transpose");
                if (tr != (v > x)) bad("transpose flag");
            }
            const int lo = std::min(v, x), hi = std::max(v, x);
            // Expected contributors: the elements holding both vertices, ascending.
            incident.clear();
            for (int e = 0; e < ne; ++e) {
                const int ge = static_cast<int>(p.tc_els[e0 + e] & 0x7fffffffu);
                bool hv = false, hx = false;
                for (int a = 0; a < 4; ++a) {
                    hv = hv || vert(ge, a) == v;
                    hx = hx || vert(ge, a) == x;
                }
                if (hv && hx) incident.push_back(e);
            }
            if (cnt != incident.size()) bad("item contributor count");
            const size_t off = static_cast<size_t>(p.tc_ent_ptr[c]) + (w[2] & 0xfffffu);
            for (size_t t = 0; t < cnt; ++t) {
                const uint16_t en = p.tc_ents[off + t];
                const int el = en >> 8, pr = (en >> 4) & 15, a = (en >> 2) & 3, b = en & 3;
                if (el != incident[t]) bad("contributor list differs from the elements sharing the block");
                const int ge = static_cast<int>(p.tc_els[e0 + el] & 0x7fffffffu);
                if (vert(ge, a) != lo || vert(ge, b) != hi) bad("contributor local indices");
                const int x = std::min(a, b), y = std::max(a, b);
                if (pr != x * 4 - (x * (x - 1)) / 2 + (y - x)) bad("contributor pair index");
            }
        }
        if (p.tc_ent_ptr[c] % 8 != 0) bad("contributor lists not 16-byte aligned");
    }
    for (int64_t k = 0; k < p.nnzb(); ++k)
        if (!written[k]) bad("block not written");
    for (int e = 0; e < T; ++e)
        if (energy_count[e] != 1) bad("element energy not counted exactly once");
}

void check_solver_layout(const HostPlan& p) {
    auto bad = [](const char* what) { fail(LPG_ELOGIC, std::string("solver layout: ") + what); };
    const int V = p.V;
    const int nch = static_cast<int>(p.sell_ptr.size()) - 1;
    if (nch != (V + 31) / 32 || p.sell_bptr.size() != p.sell_ptr.size()) bad("chunk count");
    // (row, column) -> value index of entry 0, from the own slots as stored.
    std::vector<std::vector<std::pair<int, int64_t>>> own(static_cast<size_t>(V));
    std::vector<char> seen(static_cast<size_t>(V), 0);
    for (int c = 0; c < nch; ++c) {
        const int width = (p.sell_ptr[c + 1] - p.sell_ptr[c]) / 32;
        if (p.sell_ptr[c + 1] - p.sell_ptr[c] != 32 * width || width < 0) bad("own slots not a multiple of 32");
        for (int l = 0; l < 32; ++l) {
            const int r = p.sell_row[32 * static_cast<size_t>(c) + l];
            if (r < 0) continue;
            if (r >= V || seen[r]++) bad("row listed twice or out of range");
            if (p.sell_base[r] != 9 * p.sell_ptr[c] + l) bad("row base");
            std::vector<int> upper;
            for (int k = p.row_ptr[r]; k < p.row_ptr[r + 1]; ++k)
                if (p.col_idx[k] >= r) upper.push_back(p.col_idx[k]);
            if (static_cast<int>(upper.size()) > width) bad("chunk narrower than a row");
            if (!upper.empty() && upper[0] != r) bad("diagonal is not the first own block");
            for (int q = 0; q < width; ++q) {
                const int col = p.sell_col[p.sell_ptr[c] + 32 * static_cast<size_t>(q) + l];
                if (q < static_cast<int>(upper.size())) {
                    if (col != upper[q]) bad("own column");
                    own[r].emplace_back(col, static_cast<int64_t>(9) * p.sell_ptr[c] + 32 * 9 * static_cast<int64_t>(q) + l);
                } else if (col != r) {
                    bad("own padding column");
                }
            }
        }
    }
    for (int v = 0; v < V; ++v)
        if (!seen[v]) bad("row missing");
    const int64_t zero = p.sell_zero();
    for (int c = 0; c < nch; ++c) {
        const int bwidth = (p.sell_bptr[c + 1] - p.sell_bptr[c]) / 32;
        if (p.sell_bptr[c + 1] - p.sell_bptr[c] != 32 * bwidth || bwidth < 0) bad("borrowed slots not a multiple of 32");
        for (int l = 0; l < 32; ++l) {
            const int r = p.sell_row[32 * static_cast<size_t>(c) + l];
            std::vector<int> lower;
            if (r >= 0)
                for (int k = p.row_ptr[r]; k < p.row_ptr[r + 1]; ++k)
                    if (p.col_idx[k] < r) lower.push_back(p.col_idx[k]);
            if (static_cast<int>(lower.size()) > bwidth) bad("chunk narrower than a borrowed list");
            for (int q = 0; q < bwidth; ++q) {
                const size_t at = 2 * (p.sell_bptr[c] + 32 * static_cast<size_t>(q) + l);
                const int64_t idx = p.sell_bref[at];
                const int col = p.sell_bref[at + 1];
                if (q < static_cast<int>(lower.size())) {
                    if (col != lower[q]) bad("borrowed column");
                    int64_t want = -1;
                    for (const auto& ce : own[col])
                        if (ce.first == r) want = ce.second;
                    if (want < 0 || idx != want) bad("borrowed block does not reference the owning row's block");
                } else if (idx != zero || col < 0 || col >= std::max(V, 1)) {
                    bad("borrowed padding");
                }
            }
        }
    }
}

} // namespace lpg
