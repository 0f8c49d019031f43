// lpg_plan.cpp -- host-side assembly plan: block-CSR pattern, vertex incidence,
// warp tiles and per-slot contributor lists.
//
// The scalar pattern of the reference is the union over elements of local x local DOF
// pairs, both triangles (src/core/dof/energy_assembler.cpp:38-47). For 3 DOFs per vertex
// in vertex-major order it is exactly the 3x3 expansion of the vertex adjacency, so the
// block-CSR rows below expand to the reference's CSC columns bit for bit. Contributions to
// one block are kept in ascending element order, the order of the reference's per-column
// contribution lists (energy_assembler.cpp:49-54).

#include <algorithm>
#include <cstring>
#include <limits>
#include <string>

#include "lpg_internal.h"

namespace lpg {

void build_plan(int V, int T, const int32_t* tets, HostPlan& p) {
    if (V < 0 || T < 0) fail(LPG_EINVAL, "MeshTopology requires a non-negative vertex count");
    if (V > std::numeric_limits<int>::max() / 3) fail(LPG_EINVAL, "VertexDofMap requires total DOFs fitting in int");
    if (T >= (1 << 30)) fail(LPG_EINVAL, "mesh has too many elements for the assembly plan (limit 2^30)");
    for (int e = 0; e < T; ++e) {
        int s[4];
        std::memcpy(s, tets + 4 * static_cast<size_t>(e), sizeof s);
        std::sort(s, s + 4);
        if (s[0] < 0 || s[3] >= V)
            fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " has vertex indices outside [0, num_vertices)");
        if (s[0] == s[1] || s[1] == s[2] || s[2] == s[3])
            fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(e) + " must contain distinct vertices");
    }
    p.V = V;
    p.T = T;
    // Incidence (row -> pairs in element order), by counting sort.
    p.inc_ptr.assign(static_cast<size_t>(V) + 1, 0);
    for (int64_t k = 0; k < 4 * static_cast<int64_t>(T); ++k) ++p.inc_ptr[tets[k] + 1];
    for (int v = 0; v < V; ++v) p.inc_ptr[v + 1] += p.inc_ptr[v];
    const int64_t npairs = p.inc_ptr[V];
    std::vector<int32_t> inc(static_cast<size_t>(npairs));
    {
        std::vector<int32_t> fill(p.inc_ptr.begin(), p.inc_ptr.end() - 1);
        for (int e = 0; e < T; ++e)
            for (int a = 0; a < 4; ++a) {
                const int v = tets[4 * static_cast<size_t>(e) + a];
                inc[fill[v]++] = e | (a << 30);
            }
    }
    int maxdeg = 0;
    for (int v = 0; v < V; ++v) maxdeg = std::max(maxdeg, p.inc_ptr[v + 1] - p.inc_ptr[v]);
    if (maxdeg > 64)
        fail(LPG_EINVAL, "vertex valence " + std::to_string(maxdeg) + " exceeds the supported maximum of 64");
    p.cap = maxdeg > 32 ? 64 : 32;
    // Block-CSR pattern: sorted unique neighbours (including the vertex itself).
    p.row_ptr.assign(static_cast<size_t>(V) + 1, 0);
    {
        std::vector<int32_t> cols;
        cols.reserve(static_cast<size_t>(npairs) * 2);
        std::vector<int32_t> buf;
        for (int v = 0; v < V; ++v) {
            buf.clear();
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int e = inc[k] & ((1 << 30) - 1);
                for (int b = 0; b < 4; ++b) buf.push_back(tets[4 * static_cast<size_t>(e) + b]);
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
    // SpMV tiles: runs of consecutive rows holding at most 32 blocks (a row without blocks counts
    // as one), one warp lane per block; a row with more than 32 blocks is a tile of its own.
    p.spmv_tile_row.assign(1, 0);
    {
        int lanes = 0, rows = 0;
        for (int v = 0; v < V; ++v) {
            const int need = std::max(1, p.row_ptr[v + 1] - p.row_ptr[v]);
            if (rows > 0 && (lanes + need > 32 || rows == 32)) {
                p.spmv_tile_row.push_back(v);
                lanes = rows = 0;
            }
            lanes += need;
            ++rows;
            if (need > 32) {
                p.spmv_tile_row.push_back(v + 1);
                lanes = rows = 0;
            }
        }
        if (rows > 0) p.spmv_tile_row.push_back(V);
        p.spmv_row_tile.assign(static_cast<size_t>(V), 0);
        for (size_t t = 0; t + 1 < p.spmv_tile_row.size(); ++t)
            for (int v = p.spmv_tile_row[t]; v < p.spmv_tile_row[t + 1]; ++v) p.spmv_row_tile[v] = static_cast<int32_t>(t);
    }
    // Warp tiles: whole rows, at most `cap` pairs and 32 rows per tile. First fit over a
    // short window of open tiles keeps rows of one tile close in memory.
    struct Open {
        int tile, pairs, rows;
    };
    std::vector<std::vector<int32_t>> tiles;
    std::vector<int> tile_pairs;
    std::vector<Open> open;
    constexpr int kWindow = 8;
    p.unused_rows.clear();
    for (int v = 0; v < V; ++v) {
        const int deg = p.inc_ptr[v + 1] - p.inc_ptr[v];
        if (deg == 0) {
            p.unused_rows.push_back(v); // no element references v: zero gradient, no Hessian slots
            continue;
        }
        int chosen = -1;
        for (size_t k = 0; k < open.size(); ++k)
            if (open[k].pairs + deg <= p.cap && open[k].rows < 32) {
                chosen = static_cast<int>(k);
                break;
            }
        if (chosen < 0) {
            tiles.emplace_back();
            tile_pairs.push_back(0);
            open.push_back({static_cast<int>(tiles.size()) - 1, 0, 0});
            if (open.size() > kWindow) open.erase(open.begin());
            chosen = static_cast<int>(open.size()) - 1;
        }
        Open& o = open[chosen];
        tiles[o.tile].push_back(v);
        o.pairs += deg;
        o.rows += 1;
        tile_pairs[o.tile] = o.pairs;
        if (o.pairs == p.cap || o.rows == 32) open.erase(open.begin() + chosen);
    }
    const int ntiles = static_cast<int>(tiles.size());
    p.tile_pair_ptr.assign(static_cast<size_t>(ntiles) + 1, 0);
    p.tile_row_ptr.assign(static_cast<size_t>(ntiles) + 1, 0);
    p.tile_slot_ptr.assign(static_cast<size_t>(ntiles) + 1, 0);
    p.tile_rows.clear();
    p.tile_rows.reserve(V);
    p.pair_elem.resize(static_cast<size_t>(npairs));
    p.contrib.assign(static_cast<size_t>(npairs) * 4, 0xff);
    p.slot_desc.clear();
    p.slot_desc.reserve(static_cast<size_t>(p.nnzb()));
    p.diag_slot.assign(static_cast<size_t>(V), -1);
    for (int v = 0; v < V; ++v)
        for (int k = p.row_ptr[v]; k < p.row_ptr[v + 1]; ++k)
            if (p.col_idx[k] == v) p.diag_slot[v] = k;
    std::vector<std::vector<int>> bucket;
    int64_t pair_cursor = 0;
    for (int t = 0; t < ntiles; ++t) {
        const int64_t pair_base = pair_cursor;
        int64_t slots = 0;
        int count = 0; // off-diagonal blocks of the tile placed so far
        for (int j = 0; j < static_cast<int>(tiles[t].size()); ++j) {
            const int v = tiles[t][j];
            p.tile_rows.push_back(v);
            const int r0 = p.row_ptr[v], nb_v = p.row_ptr[v + 1] - p.row_ptr[v];
            bucket.assign(static_cast<size_t>(nb_v), {});
            for (int k = p.inc_ptr[v]; k < p.inc_ptr[v + 1]; ++k) {
                const int local = static_cast<int>(pair_cursor - pair_base);
                p.pair_elem[pair_cursor++] = inc[k];
                const int e = inc[k] & ((1 << 30) - 1);
                for (int b = 0; b < 4; ++b) {
                    const int w = tets[4 * static_cast<size_t>(e) + b];
                    if (w == v) continue; // the diagonal block is reduced in registers
                    const int32_t* beg = p.col_idx.data() + r0;
                    const int q = static_cast<int>(std::lower_bound(beg, beg + nb_v, w) - beg);
                    bucket[q].push_back(4 * local + b);
                }
            }
            // Off-diagonal slots in column order; each slot's blocks contiguous, in element order.
            for (int q = 0; q < nb_v; ++q) {
                if (p.col_idx[r0 + q] == v) continue;
                p.slot_desc.push_back(static_cast<uint32_t>(count) | (static_cast<uint32_t>(j) << 8) |
                                      (static_cast<uint32_t>(q) << 13));
                for (int c : bucket[q]) p.contrib[4 * pair_base + c] = static_cast<uint8_t>(count++);
                ++slots;
            }
        }
        p.tile_pair_ptr[t + 1] = static_cast<int32_t>(pair_cursor);
        p.tile_row_ptr[t + 1] = static_cast<int32_t>(p.tile_rows.size());
        p.tile_slot_ptr[t + 1] = static_cast<int32_t>(p.tile_slot_ptr[t] + slots);
    }
}

} // namespace lpg
