// lpg_internal.h -- shared host-side definitions of the litepgo_b200 CUDA library.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/litepgo_b200.h"

namespace lpg {

// Device status word bits, OR-ed by kernels that find a bad element or input.
enum : unsigned {
    ST_BAD_INPUT = 1u << 0,    // non-finite u / du           -> LPG_EINVAL
    ST_BAD_THETA = 1u << 1,    // lambda < 0, mu <= 0, NaN     -> LPG_EINVAL
    ST_NONFINITE_F = 1u << 2,  // non-finite F or increment    -> LPG_EDOMAIN
    ST_BAD_DET = 1u << 3,      // det F <= 0                   -> LPG_EDOMAIN
    ST_NONFINITE_OUT = 1u << 4  // non-finite E, g or H         -> LPG_EDOMAIN
};

struct Error {
    int code;
    std::string what;
};
[[noreturn]] void fail(int code, const std::string& what);
void check_cuda(cudaError_t e, const char* what);
#define LPG_CUDA(call) ::lpg::check_cuda((call), #call)

// Host-side assembly plan (built once per mesh, lpg_plan.cpp). Rows of the 3x3 block-CSR
// Hessian are vertices; a "pair" is (row vertex v, element e incident to v, local index a of v
// in e).
struct HostPlan {
    int V = 0, T = 0;
    int K = 4; // vertices per cell: 4 (tet) or 8 (hex)
    std::vector<int32_t> row_ptr, col_idx;   // BSR pattern (V+1, nnzb)
    std::vector<int32_t> inc_ptr;            // V+1: pairs per row, natural order
    std::vector<int32_t> diag_slot;          // V: block index of (v, v), -1 for an unused vertex
    std::vector<int32_t> unused_rows;        // vertices referenced by no element
    // Upper-triangle sliced ELL of the solvers (SELL-32 with rows sorted by block count within
    // windows of kSellWindow rows). The matrix is symmetric, so each row stores only its blocks
    // with column >= row ("own" blocks, the diagonal first) and reads its blocks left of the
    // diagonal as the transposes of the owning rows' blocks ("borrowed" blocks).
    //   Own: chunk c holds 32 rows (sell_row, -1 past the end) and sell_ptr[c + 1] - sell_ptr[c]
    //   = 32 x (its most own blocks) slots; own block q of the row in lane l is slot
    //   sell_ptr[c] + 32 q + l, its column sell_col (the row itself for padding), and entry t of
    //   the 3x3 block is value 9 sell_ptr[c] + (9 q + t) 32 + l = sell_base[row] + 32 (9 q + t).
    //   Borrowed: slots [sell_bptr[c], sell_bptr[c + 1]), 32 per borrowed block of the chunk's
    //   longest such list; slot sell_bptr[c] + 32 q + l holds {value index of entry 0 of the
    //   owning row's block, its column}; entry t is at that index + 32 t. Padding points at a
    //   zero block stored after the own slots (sell_zero()).
    std::vector<int32_t> sell_ptr, sell_row, sell_col, sell_base;
    std::vector<int32_t> sell_bptr, sell_bref;
    // Vertex clusters of the element-once assembly (one thread block per cluster): the rows a
    // cluster owns, the elements incident to them (ascending; bit 31 set on the elements whose
    // energy the cluster counts, those whose first vertex it owns), and its block slots:
    // off-diagonal slots left of the diagonal (cl_ntr of them), off-diagonal slots right of
    // it, then the diagonal slots (cl_noff off-diagonal in all). Slot word: bits 0-7 the row within the cluster, bits
    // 8-29 the slot's position within its row, bit 30 "store the transpose", bit 31 diagonal.
    // Entry word of a slot: bits 0-19 first contributor (within the cluster), 20-31 count.
    // Contributors (uint16): element within the cluster << 2s | a << s | b (s = 2 bits for tets,
    // 3 for hexes), where (a, b) are the local indices of the lower- and higher-numbered vertex
    // of the slot (a = b diagonal).
    std::vector<int32_t> cl_row_ptr, cl_rows;
    std::vector<int32_t> cl_el_ptr;
    std::vector<uint32_t> cl_els;
    std::vector<int32_t> cl_slot_ptr, cl_noff, cl_ntr;
    std::vector<uint32_t> cl_slot, cl_slot_ent;
    std::vector<int32_t> cl_ent_ptr;
    std::vector<uint16_t> cl_ents;
    // Tet assembly clusters (tet_cluster_kernel; empty for other cells). A cluster owns
    // up to kTcRows rows; its elements (those incident to the rows, ascending, at most kTcElems;
    // bit 31 on the ones whose energy it counts: those whose first vertex it owns) touch at most
    // kTcVerts vertices (tc_verts, ascending); tc_loc packs each element's four local vertex
    // indices (one byte each, vertex order). Output staging: row j of the cluster (tc_rows) keeps
    // its 9 nb_j values at offset tc_row_so[j] (values), so_j = 9 sum_{i<j} nb_i.
    // Items (4 words each): the cluster's diagonal blocks first (tc_ndiag of them), then its
    // edge blocks, each group sorted by contributor count (descending):
    //   w0: primary staging position (so 16 bits | block position q in the row << 16 | nb << 24)
    //   w1: second position (same packing; the transposed block of an edge between two owned
    //       rows) or 0xffffffff
    //   w2: first contributor (within the cluster's list, 20 bits) | count << 20
    //   w3: bit 31 diagonal, bit 30 the primary position stores the transpose; bits 0-7 the row
    //       j of a diagonal block (its gradient row)
    // An edge between two owned rows is summed once and stored at both positions; an edge to a
    // row of another cluster is summed by each of the two clusters for its own row, in the same
    // orientation (lower-numbered vertex first) and order, so both blocks are exact transposes.
    // Contributors (uint16): element within the cluster << 8 | its block pair index (pair10 of
    // the two local indices) << 4 | a << 2 | b, (a, b) the local indices of the lower- and
    // higher-numbered vertex (a = b for a diagonal block), ascending by element (the
    // reference's per-column order).
    std::vector<int32_t> tc_row_ptr, tc_rows, tc_row_so;
    std::vector<int32_t> tc_el_ptr, tc_vert_ptr, tc_verts, tc_item_ptr, tc_ndiag, tc_ent_ptr;
    std::vector<uint32_t> tc_els, tc_loc, tc_items;
    std::vector<uint16_t> tc_ents;
    // Value count of the solver layout: 9 per own slot, then the 9 x 32 zero block.
    int64_t sell_zero() const { return 9 * static_cast<int64_t>(sell_ptr.back()); }
    size_t sell_values() const { return static_cast<size_t>(sell_zero()) + 9 * 32; }
    int64_t nnzb() const { return static_cast<int64_t>(col_idx.size()); }
};

// Size limits of an assembly cluster: owned rows, and distinct incident elements (the
// element data of a cluster is held in shared memory).
constexpr int kSellWindow = 128;

#ifndef LPG_CLUSTER_ROWS
#define LPG_CLUSTER_ROWS 24
#endif
#ifndef LPG_CLUSTER_ELEMS
#define LPG_CLUSTER_ELEMS 224
#endif
constexpr int kClusterRows = LPG_CLUSTER_ROWS;
constexpr int kClusterElems = LPG_CLUSTER_ELEMS;
// Limits of a tet assembly cluster (HostPlan::tc_*): owned rows, distinct incident elements
// (their data is held in shared memory) and distinct vertices of those elements.
#ifndef LPG_TC_ROWS
#define LPG_TC_ROWS 64
#endif
#ifndef LPG_TC_ELEMS
#define LPG_TC_ELEMS 256
#endif
#ifndef LPG_TC_VALS
#define LPG_TC_VALS 3072
#endif
#ifndef LPG_TC_ENTS
#define LPG_TC_ENTS 2048
#endif
constexpr int kTcRows = LPG_TC_ROWS;
constexpr int kTcElems = LPG_TC_ELEMS;
constexpr int kTcVerts = 256;
constexpr int kTcVals = LPG_TC_VALS; // output staging values of a cluster (its rows' 9 nb)
// Items of a cluster (at most one per block of its rows) and contributor words (padded to a
// multiple of 8); both are staged in shared memory.
constexpr int kTcItems = kTcVals / 9;
constexpr int kTcEnts = LPG_TC_ENTS;
static_assert(kTcEnts % 8 == 0, "contributor lists are staged in 16-byte chunks");
static_assert(kTcElems <= 256 && kTcRows <= 256, "tet cluster indices are 8-bit");
// Clusters of 64-node cells (Hermite hexes: 8 slot rows per vertex, ~216 blocks per row) hold at
// most one vertex's rows, so a cluster's slot and contributor tables fit in shared memory.
constexpr int kClusterRowsWide = 8;
// Bits of a node index inside a contributor word (2, 3 or 6), and the bit where the plan's
// incidence words keep a node's local index above its element id.
constexpr int cell_bits(int K) { return K == 4 ? 2 : K == 8 ? 3 : 6; }
constexpr int inc_shift(int K) { return K == 64 ? 26 : 29; }

// VEG volume-mesh files (lpg_veg.cpp; src/core/mesh/io/veg.cpp).
struct VegMesh {
    int num_vertices = 0;
    int width = 0;                 // 4 (TET) or 8 (CUBIC)
    std::vector<double> positions; // 3 per vertex
    std::vector<int32_t> cells;    // width per cell, 0-based
};
void read_veg(const std::string& path, VegMesh& mesh);
void write_veg(const std::string& path, int V, const double* positions, int T, int width, const int32_t* cells);
// MeshData::validate + MeshTopology checks (LPG_EINVAL).
void validate_volume_mesh(int V, const std::vector<double>& positions, int width, const std::vector<int32_t>& cells);

// Validates connectivity (mesh_topology.hpp:25-44) and builds the plan.
void build_plan(int V, int T, const int32_t* cells, HostPlan& plan, int K = 4);
// Checks the cluster plan's invariants (throws LPG_ELOGIC on a violation).
void check_clusters(const HostPlan& plan, const int32_t* tets);
// Checks the tet assembly clusters (HostPlan::tc_*) against the mesh (throws LPG_ELOGIC).
void check_tet_clusters(const HostPlan& plan, const int32_t* tets);
// Checks the solvers' upper-triangle sliced-ELL layout against the BSR pattern (LPG_ELOGIC).
void check_solver_layout(const HostPlan& plan);

// Device mirror of the plan and of the per-element records.
struct DevMesh {
    int V = 0, T = 0;
    int64_t nnzb = 0;
    int32_t *row_ptr = nullptr, *col_idx = nullptr, *inc_ptr = nullptr;
    int32_t* diag_slot = nullptr;
    int32_t* unused_rows = nullptr;
    int num_unused = 0;
    int32_t *sell_ptr = nullptr, *sell_row = nullptr, *sell_col = nullptr, *sell_base = nullptr;
    int32_t* sell_bptr = nullptr;
    int2* sell_bref = nullptr; // {value index, column} per borrowed slot
    int n_sell = 0; // SELL chunks
    int ncl = 0, cl_max_slots = 0, cl_max_ents = 0;
    int32_t *cl_row_ptr = nullptr, *cl_rows = nullptr, *cl_el_ptr = nullptr, *cl_slot_ptr = nullptr, *cl_noff = nullptr,
            *cl_ntr = nullptr, *cl_ent_ptr = nullptr;
    uint32_t *cl_els = nullptr, *cl_slot = nullptr, *cl_slot_ent = nullptr;
    uint16_t* cl_ents = nullptr;
    // Tet assembly clusters (HostPlan::tc_*), and their largest element, vertex, row and staging
    // counts.
    int tc_ncl = 0, tc_max_els = 0, tc_max_verts = 0, tc_max_vals = 0;
    int32_t *tc_row_ptr = nullptr, *tc_rows = nullptr, *tc_row_so = nullptr, *tc_el_ptr = nullptr,
            *tc_vert_ptr = nullptr, *tc_verts = nullptr, *tc_item_ptr = nullptr, *tc_ndiag = nullptr,
            *tc_ent_ptr = nullptr;
    uint32_t *tc_els = nullptr, *tc_loc = nullptr;
    uint4* tc_items = nullptr;
    uint16_t* tc_ents = nullptr;
    int4* tets = nullptr;
    // Per-element record: G (3x3 row-major, rows = grad N_1..3 in rest coordinates, times Fp^-1),
    // vol (= det(Dm)/6 * det Fp), lambda, mu. 12 values, 16-byte aligned.
    double* rec64 = nullptr;
    float* rec32 = nullptr;
    // Fp^-1 row-major (9 per element) when the mesh has a plastic field, else null.
    double* fpinv64 = nullptr;
    float* fpinv32 = nullptr;
    // Hex Q1 meshes (K = 8): rest positions (3 per vertex), cells (8 per element), [lambda, mu]
    // per element, and per quadrature point the 8 x 3 reference derivatives dN/dxi and the
    // weight (25 values per point, nq points).
    int K = 4, nq = 0;
    double* hex_X = nullptr;
    int32_t* hex_cells = nullptr;
    double* hex_theta = nullptr;
    double* hex_q = nullptr;
    // Tricubic Hermite hexes (K = 64 plan nodes, 8 per vertex; hex_cells and hex_theta as
    // above): per point the 64 x 3 reference derivatives and the weight (193 values), and each
    // element's box edge lengths (3 per element).
    double* herm_q = nullptr;
    double* herm_h = nullptr;
};

// Internal Hessian layout of the solvers: the upper-triangle sliced ELL of HostPlan::sell_*
// (blocks left of the diagonal are not stored).
constexpr int kLayoutSell = 2;

// ---- kernel launchers (lpg_assemble.cu) ----
struct EvalArgs {
    const double* u = nullptr;  // device, 3V
    double* grad = nullptr;     // device, 3V or null
    void* hess = nullptr;       // device values or null
    int layout = LPG_LAYOUT_BSR;
    double* cluster_energy = nullptr; // device, one per cluster (always written)
    double* energy = nullptr;      // device scalar (always written)
    double* elem_energy = nullptr; // device, T, or null
    const void* proj = nullptr;    // projected per-element 9x9 tangents (hessian PROJECTED*), or null
    unsigned* status = nullptr;    // device status word
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr; // optional: bracket the assembly kernel
    int cl_variant = 0; // register-budget variant of the Exact-Hessian cluster kernel (autotuner)
    // Batched solves: per-cluster flags (tet clusters, block-gather clusters) of clusters whose
    // mesh has finished; such a cluster writes nothing. Null: every cluster runs.
    const unsigned char* tc_skip = nullptr;
    const unsigned char* cl_skip = nullptr;
};

// Autotuned launch variants (register budgets and unroll depths; every variant of a kernel
// computes bitwise the same results). Index [0] FP64, [1] FP32 / mixed.
constexpr int kClVariants = 3;    // cluster kernel, Exact Hessian
constexpr int kSpmvVariants = 3;  // PCG sliced-ELL SpMV
constexpr int kClampVariants = 2; // eigenvalue clamp (FP32 only; FP64 has one)
struct Tuning {
    int cl[2] = {0, 0};
    int spmv[2] = {0, 0};
    int clamp[2] = {0, 0};
    // Mean ms per launch of each variant as measured ([family][precision][variant]); NaN if not run.
    double ms[3][2][3];
    bool tuned = false;
};
void launch_eval(const DevMesh& m, int precision, int hessian, const EvalArgs& a, cudaStream_t s);
// Largest dynamic shared memory any assembly kernel of this mesh's cell type needs for its
// largest cluster (the same formulas the launches use).
size_t assembly_smem_bytes(const DevMesh& m);
// Per-element clamped tangents for the projected Hessians (45 values / element, upper triangle).
// list (T ints) and count (1) are scratch: the elements whose tangent needs the eigenvalue
// clamp. With emesh (element -> mesh) and mesh_exact (per mesh), the elements of the meshes
// marked exact keep their tangent unclamped.
void launch_project(const DevMesh& m, int precision, int hessian, const double* u, void* proj, unsigned* status,
                    cudaStream_t s, int* list, unsigned* count, const int* emesh = nullptr,
                    const int* mesh_exact = nullptr, int clamp_variant = 0);
// The eigenvalue clamp alone on `count` listed elements of proj (autotuner timing).
void launch_clamp(int precision, void* proj, const int* list, const unsigned* count, int max_count, int clamp_variant,
                  cudaStream_t s);
// Fills n packed symmetric 9x9 matrices (45 values each) with seeded values in [-1, 1] and
// list[i] = i (autotuner timing input for the clamp).
void launch_clamp_sample(int precision, void* proj, int* list, int n, cudaStream_t s);
size_t project_bytes(const DevMesh& m, int precision);
// Values per element of the projected-Hessian scratch: the element's ten 3x3 blocks (pair10
// order), or, for an element listed for the clamp until it is clamped, its 9x9 tangent (45).
constexpr int kProjRecord = 90;
// Values per element of the hex block scratch: 36 blocks (a <= b of 8 vertices) of 3x3.
constexpr int kHexRecord = 324;
constexpr int kHermiteRecord = 2080 * 9; // tricubic Hermite hex: 64 nodes, 2080 blocks (a <= b)
constexpr int kHermiteTable = 193;       // per quadrature point: 64 x 3 reference derivatives, weight
// per_elem (T doubles, optional) receives each element's step.
// With emesh / mstate (batched solves: element -> mesh, per-mesh state), the elements of a mesh in
// state 2 (finished) are skipped.
void launch_feasible(const DevMesh& m, const double* u, const double* du, double* block_min, int nblocks,
                     double* alpha, unsigned* status, cudaStream_t s, double* per_elem = nullptr,
                     const int* emesh = nullptr, const int* mstate = nullptr);
int feasible_blocks(const DevMesh& m);
void launch_force_vjp(const DevMesh& m, const double* u, const double* w, double* out_per_elem, unsigned* status,
                      cudaStream_t s);
// Rest-position force VJP: out (3V) = sign * (d g / d X)^T w; per_elem: 12 T doubles of scratch.
void launch_rest_vjp(const DevMesh& m, const double* u, const double* w, double* per_elem, double sign, double* out,
                     unsigned* status, cudaStream_t s);
void launch_set_theta(const DevMesh& m, const double* theta, int per_element, cudaStream_t s);
void launch_sum_pairs(const double* per_elem, int T, double* partial, int nblocks, double* out2, cudaStream_t s);
// Hex Q1 element pass (K = 8): energy per element into elemE (T), gradient pieces (24 per element)
// into per_elem when a.grad is set, the 36 blocks per element (precision's type) into blocks when
// a.hess is set, then the gradient gather, the energy sum and the block gather. With projected,
// every element's 24x24 Hessian is first projected to PSD (flags: T ints of scratch marking the
// elements that need the eigen-projection); blocks then holds hex_blocks_bytes().
void launch_hex_eval(const DevMesh& m, int precision, bool projected, const double* u, double* elemE,
                     double* per_elem, void* blocks, int* flags, const EvalArgs& a, cudaStream_t s);
// Python/Torch materials on hex meshes: F at every quadrature point (9 per point, T * nq rows,
// element-major), and the caller's W (T nq), P (9 T nq) and A (81 T nq, or null without a
// Hessian) integrated per hex and assembled (blocks and flags as for launch_hex_eval).
void launch_hex_deformation_gradients(const DevMesh& m, const double* u, double* F, unsigned* status, cudaStream_t s);
void launch_hex_material_eval(const DevMesh& m, int precision, int hessian, const double* W, const double* P,
                              const double* A, double* elemE, double* per_elem, void* blocks, int* flags,
                              const EvalArgs& a, cudaStream_t s);
// Tricubic Hermite hex element pass (Exact Hessian): energy per element into elemE, gradient
// pieces (192 per element) into per_elem when a.grad is set, the 2080 blocks per element
// (precision's type, kHermiteRecord values) into blocks when a.hess is set, then the gathers.
// With projected, each element's 192 x 192 Hessian is first projected to PSD where its per-point
// pre-test fails (flags: T ints of scratch; qbuf: hermite_psd_grid() x 192^2 doubles of scratch);
// blocks then holds hermite_blocks_bytes().
void launch_hermite_eval(const DevMesh& m, int precision, bool projected, const double* u, double* elemE,
                         double* per_elem, void* blocks, int* flags, double* qbuf, const EvalArgs& a, cudaStream_t s);
size_t hermite_blocks_bytes(const DevMesh& m, int precision, bool projected);
int hermite_psd_grid(const DevMesh& m);
// Bytes of the block records launch_hex_eval needs: FP64 records, plus FP32 ones for a
// projected mixed-precision Hessian (the projection runs in FP64).
size_t hex_blocks_bytes(const DevMesh& m, int precision, bool projected);
// Largest step along du keeping det F > 0 at every quadrature point of every hex (x 0.9 as the
// reference), minimum over the mesh into *alpha (device).
void launch_hex_feasible(const DevMesh& m, const double* u, const double* du, double* block_min, int nblocks,
                         double* alpha, unsigned* status, cudaStream_t s);
int hex_feasible_blocks(const DevMesh& m);
// Materials evaluated by the caller: F (9 T, row-major) at u, then integration and assembly of
// the caller's W (T), P = dW/dF (9 T) and, for a Hessian, A = d2W/dF2 (81 T) — energy into
// a.energy (a.cluster_energy is scratch of >= 256 values), gradient into a.grad if set, Hessian
// (Exact, or projected: clamped) into a.hess in a.layout. elemE (T), per_elem (12 T), proj
// (project_bytes), list (T) and count (1) are scratch.
void launch_deformation_gradients(const DevMesh& m, const double* u, double* F, unsigned* status, cudaStream_t s);
void launch_material_eval(const DevMesh& m, int precision, int hessian, const double* W, const double* P,
                          const double* A, double* elemE, double* per_elem, void* proj, int* list, unsigned* count,
                          int clamp_variant, const EvalArgs& a, cudaStream_t s);
// Plastic force VJP: out (9 T, column-major per element) = (d g_e / d vec Fp_e)^T w_e.
void launch_fp_vjp(const DevMesh& m, const double* u, const double* w, double* out, unsigned* status, cudaStream_t s);
void launch_sum_cols9(const double* per_elem, int T, double* partial, int nblocks, double* out9, cudaStream_t s);
// geo: 10 doubles per element (G row-major, vol) written into rec64 / rec32 (theta kept).
void launch_set_geometry(const DevMesh& m, const double* geo, cudaStream_t s);

} // namespace lpg
