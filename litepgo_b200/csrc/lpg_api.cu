// lpg_api.cu -- the C ABI (include/litepgo_b200.h): handle, element records, I/O.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "lpg_internal.h"
#include "lpg_solver.h"

namespace lpg {

thread_local std::string g_last_error;

void fail(int code, const std::string& what) { throw Error{code, what}; }

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(LPG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return LPG_OK;
    } catch (const Error& e) {
        g_last_error = e.what;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return LPG_ELOGIC;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return LPG_ELOGIC;
    }
}

// Device allocations made by the library since the process started (reported by lpg_build_info).
std::atomic<long long> g_device_allocations{0};

DeviceBuffer::~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
}
void* DeviceBuffer::ensure(size_t n) {
    if (n <= bytes) return ptr;
    if (ptr) LPG_CUDA(cudaFree(ptr));
    ptr = nullptr;
    bytes = 0;
    LPG_CUDA(cudaMalloc(&ptr, n > 0 ? n : 1));
    g_device_allocations.fetch_add(1);
    bytes = n;
    return ptr;
}

namespace {

template <class T> T* upload(DeviceBuffer& b, const std::vector<T>& v) {
    T* p = b.as<T>(v.size());
    if (!v.empty()) LPG_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

// Copies the host plan's arrays to the device mirror (every mesh kind).
void upload_plan(lpg_fem& hh, int V, int T) {
    lpg_fem* h = &hh;
    const HostPlan& p = h->plan;
    DevMesh& m = h->dm;
    m.V = V;
    m.T = T;
    m.nnzb = p.nnzb();
    m.row_ptr = upload(h->b_row_ptr, p.row_ptr);
    m.col_idx = upload(h->b_col_idx, p.col_idx);
    m.inc_ptr = upload(h->b_inc_ptr, p.inc_ptr);
    m.diag_slot = upload(h->b_diag_slot, p.diag_slot);
    m.unused_rows = upload(h->b_unused, p.unused_rows);
    m.num_unused = static_cast<int>(p.unused_rows.size());
    m.sell_ptr = upload(h->b_sell[0], p.sell_ptr);
    m.sell_row = upload(h->b_sell[1], p.sell_row);
    m.sell_col = upload(h->b_sell[2], p.sell_col);
    m.sell_base = upload(h->b_sell[3], p.sell_base);
    m.sell_bptr = upload(h->b_sell[4], p.sell_bptr);
    m.sell_bref = reinterpret_cast<int2*>(upload(h->b_sell[5], p.sell_bref));
    m.n_sell = static_cast<int>(p.sell_ptr.size()) - 1;
    m.ncl = static_cast<int>(p.cl_row_ptr.size()) - 1;
    m.cl_row_ptr = upload(h->b_cl[0], p.cl_row_ptr);
    m.cl_rows = upload(h->b_cl[1], p.cl_rows);
    m.cl_el_ptr = upload(h->b_cl[2], p.cl_el_ptr);
    m.cl_els = upload(h->b_cl[3], p.cl_els);
    m.cl_slot_ptr = upload(h->b_cl[4], p.cl_slot_ptr);
    m.cl_noff = upload(h->b_cl[5], p.cl_noff);
    m.cl_slot = upload(h->b_cl[6], p.cl_slot);
    m.cl_slot_ent = upload(h->b_cl[7], p.cl_slot_ent);
    m.cl_ent_ptr = upload(h->b_cl[8], p.cl_ent_ptr);
    m.cl_ents = upload(h->b_cl[9], p.cl_ents);
    m.cl_ntr = upload(h->b_cl[10], p.cl_ntr);
    m.tc_ncl = p.tc_row_ptr.empty() ? 0 : static_cast<int>(p.tc_row_ptr.size()) - 1;
    if (m.tc_ncl > 0) {
        m.tc_row_ptr = upload(h->b_tc[0], p.tc_row_ptr);
        m.tc_rows = upload(h->b_tc[1], p.tc_rows);
        m.tc_row_so = upload(h->b_tc[2], p.tc_row_so);
        m.tc_el_ptr = upload(h->b_tc[3], p.tc_el_ptr);
        m.tc_vert_ptr = upload(h->b_tc[4], p.tc_vert_ptr);
        m.tc_verts = upload(h->b_tc[5], p.tc_verts);
        m.tc_item_ptr = upload(h->b_tc[6], p.tc_item_ptr);
        m.tc_ndiag = upload(h->b_tc[7], p.tc_ndiag);
        m.tc_ent_ptr = upload(h->b_tc[8], p.tc_ent_ptr);
        m.tc_els = upload(h->b_tc[9], p.tc_els);
        m.tc_loc = upload(h->b_tc[10], p.tc_loc);
        m.tc_items = reinterpret_cast<uint4*>(upload(h->b_tc[11], p.tc_items));
        m.tc_ents = upload(h->b_tc[12], p.tc_ents);
        m.tc_max_els = m.tc_max_verts = m.tc_max_vals = 0;
        for (int c = 0; c < m.tc_ncl; ++c) {
            m.tc_max_els = std::max(m.tc_max_els, p.tc_el_ptr[c + 1] - p.tc_el_ptr[c]);
            m.tc_max_verts = std::max(m.tc_max_verts, p.tc_vert_ptr[c + 1] - p.tc_vert_ptr[c]);
        }
    }
    m.cl_max_slots = m.cl_max_ents = 0;
    for (int c = 0; c < m.ncl; ++c) {
        m.cl_max_slots = std::max(m.cl_max_slots, p.cl_slot_ptr[c + 1] - p.cl_slot_ptr[c]);
        m.cl_max_ents = std::max(m.cl_max_ents, p.cl_ent_ptr[c + 1] - p.cl_ent_ptr[c]);
    }
    // The assembly kernels stage a cluster's element data, row table, slot words and contributor
    // lists in shared memory: a mesh whose largest cluster would not fit is rejected here rather
    // than at its first evaluation.
    const size_t need = assembly_smem_bytes(m);
    int optin = 0;
    LPG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    if (need > static_cast<size_t>(optin))
        fail(LPG_EINVAL, "mesh valence too high for the assembly plan: a cluster needs " +
                             std::to_string(need / 1024) + " KB of shared memory (device limit " +
                             std::to_string(optin / 1024) + " KB)");
}

// Entry points whose kernels exist for tet meshes only.
// Gauss-Legendre points and weights on [0, 1] for 2 or 4 points (gauss_legendre_3d.hpp).
void gauss_legendre_01(int n, double* t1, double* w1) {
    if (n == 2) {
        t1[0] = 0.5 - 0.5 / std::sqrt(3.0);
        t1[1] = 0.5 + 0.5 / std::sqrt(3.0);
        w1[0] = w1[1] = 0.5;
    } else {
        const double outer = std::sqrt((3 + 2 * std::sqrt(6.0 / 5)) / 7), inner = std::sqrt((3 - 2 * std::sqrt(6.0 / 5)) / 7);
        t1[0] = 0.5 * (1 - outer);
        t1[1] = 0.5 * (1 - inner);
        t1[2] = 0.5 * (1 + inner);
        t1[3] = 0.5 * (1 + outer);
        w1[0] = w1[3] = (18 - std::sqrt(30.0)) / 72;
        w1[1] = w1[2] = (18 + std::sqrt(30.0)) / 72;
    }
}

// HexQ1Basis / HexHermiteBasis corner order on [0,1]^3.
constexpr int kHexCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

// Entry points whose kernels do not exist for tricubic Hermite hexes.
void not_hermite(const lpg_fem& h, const char* what) {
    if (h.dm.K == 64) fail(LPG_EINVAL, std::string(what) + " is not available for Hermite hex meshes");
}

void tet_only(const lpg_fem& h, const char* what) {
    if (h.dm.K != 4) fail(LPG_EINVAL, std::string(what) + " is available for tet meshes only");
}

// 3x3 row-major helpers for the element records.
double det3(const double* a) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
void inv3(const double* a, double* r) {
    const double d = det3(a);
    r[0] = (a[4] * a[8] - a[5] * a[7]) / d;
    r[1] = (a[2] * a[7] - a[1] * a[8]) / d;
    r[2] = (a[1] * a[5] - a[2] * a[4]) / d;
    r[3] = (a[5] * a[6] - a[3] * a[8]) / d;
    r[4] = (a[0] * a[8] - a[2] * a[6]) / d;
    r[5] = (a[2] * a[3] - a[0] * a[5]) / d;
    r[6] = (a[3] * a[7] - a[4] * a[6]) / d;
    r[7] = (a[1] * a[6] - a[0] * a[7]) / d;
    r[8] = (a[0] * a[4] - a[1] * a[3]) / d;
}

} // namespace

// Maps status bits to the reference's exception classes and messages.
void raise_status(unsigned st) {
    if (st & ST_BAD_INPUT) fail(LPG_EINVAL, "Energy: x must have num_dofs finite entries");
    if (st & ST_BAD_THETA) fail(LPG_EINVAL, "NeoHookean requires finite lambda >= 0 and mu > 0");
    if (st & ST_NONFINITE_F) fail(LPG_EDOMAIN, "VolumetricFemEnergy: non-finite deformation gradient");
    if (st & ST_BAD_DET) fail(LPG_EDOMAIN, "NeoHookean requires finite det(Fe) > 0");
    if (st & ST_NONFINITE_OUT) fail(LPG_EDOMAIN, "VolumetricElement3D: non-finite integrated outputs");
}

} // namespace lpg

using namespace lpg;

struct BusyGuard {
    std::atomic<bool>& b;
    explicit BusyGuard(std::atomic<bool>& f) : b(f) {
        if (b.exchange(true)) fail(LPG_EBUSY, "MeshEnergy is already in use by another call");
    }
    ~BusyGuard() { b.store(false); }
};

lpg_fem::~lpg_fem() {
    if (pcg_graph) cudaGraphExecDestroy(pcg_graph);
    if (batch_graph) cudaGraphExecDestroy(batch_graph);
    if (own_stream) cudaStreamDestroy(own_stream);
}

void lpg_fem::sync() { LPG_CUDA(cudaStreamSynchronize(stream)); }

unsigned lpg_fem::take_status() {
    unsigned st = 0;
    LPG_CUDA(cudaMemcpyAsync(&st, d_status.ptr, sizeof st, cudaMemcpyDeviceToHost, stream));
    LPG_CUDA(cudaMemsetAsync(d_status.ptr, 0, sizeof(unsigned), stream));
    sync();
    return st;
}

// Device pointer of an input array: the caller's when device memory, else staged.
const double* lpg_fem::stage_in(const double* p, int mem, DeviceBuffer& buf, size_t n) {
    if (!p) return nullptr;
    if (mem == LPG_MEM_DEVICE) return p;
    if (mem != LPG_MEM_HOST) fail(LPG_EINVAL, "invalid memory flag");
    double* d = buf.as<double>(n);
    LPG_CUDA(cudaMemcpyAsync(d, p, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    return d;
}

void lpg_fem::eval_async(const double* du, double* dgrad, int hessian, int precision, int layout, void* dhess,
                         double* delem, cudaEvent_t ev_begin, cudaEvent_t ev_end, const int* emesh,
                         const int* mesh_exact, const unsigned char* tc_skip, const unsigned char* cl_skip) {
    if (hessian != LPG_HESSIAN_NONE && hessian != LPG_HESSIAN_EXACT && hessian != LPG_HESSIAN_PROJECTED)
        fail(LPG_EINVAL, "Energy: invalid Hessian kind");
    if (precision != LPG_PRECISION_F64 && precision != LPG_PRECISION_MIXED) fail(LPG_EINVAL, "invalid precision");
    if (layout != LPG_LAYOUT_BSR && layout != LPG_LAYOUT_CSC && layout != kLayoutSell)
        fail(LPG_EINVAL, "invalid Hessian layout");
    EvalArgs a;
    a.u = du;
    a.grad = dgrad;
    a.hess = hessian != LPG_HESSIAN_NONE ? dhess : nullptr;
    a.layout = layout;
    // Per-cluster energies, then partial sums.
    a.cluster_energy = d_cluster_energy.as<double>(static_cast<size_t>(std::max(dm.ncl, dm.tc_ncl)) + 256);
    a.energy = d_energy.as<double>(1);
    a.elem_energy = delem;
    a.status = d_status.as<unsigned>(1);
    a.ev_begin = ev_begin;
    a.ev_end = ev_end;
    const int pi = precision == LPG_PRECISION_F64 ? 0 : 1;
    a.cl_variant = tune.cl[pi];
    a.tc_skip = tc_skip;
    a.cl_skip = cl_skip;
    if (dm.K == 64) {
        const bool projected = hessian == LPG_HESSIAN_PROJECTED;
        const size_t T = static_cast<size_t>(dm.T);
        double* elemE = delem ? delem : d_mat[3].as<double>(std::max<size_t>(T, 1));
        void* blocks = a.hess ? d_proj.ensure(hermite_blocks_bytes(dm, precision, projected)) : nullptr;
        int* flags = projected && a.hess ? d_plist.as<int>(std::max<size_t>(T, 1)) : nullptr;
        double* qbuf = projected && a.hess && T > 0
                           ? d_herm_q.as<double>(static_cast<size_t>(hermite_psd_grid(dm)) * 192 * 192)
                           : nullptr;
        launch_hermite_eval(dm, precision, projected, du, elemE, d_vjp.as<double>(std::max<size_t>(192 * T, 1)), blocks,
                            flags, qbuf, a, stream);
        return;
    }
    if (dm.K == 8) {
        const bool projected = hessian == LPG_HESSIAN_PROJECTED;
        const size_t T = static_cast<size_t>(dm.T);
        double* elemE = delem ? delem : d_mat[3].as<double>(std::max<size_t>(T, 1));
        void* blocks = a.hess ? d_proj.ensure(hex_blocks_bytes(dm, precision, projected)) : nullptr;
        a.cluster_energy = d_cluster_energy.as<double>(static_cast<size_t>(std::max(dm.ncl, dm.tc_ncl)) + 256);
        int* flags = projected && a.hess ? d_plist.as<int>(std::max<size_t>(T, 1)) : nullptr;
        launch_hex_eval(dm, precision, projected, du, elemE, d_vjp.as<double>(std::max<size_t>(24 * T, 1)), blocks,
                        flags, a, stream);
        return;
    }
    if (a.hess && hessian == LPG_HESSIAN_PROJECTED) {
        void* proj = d_proj.ensure(project_bytes(dm, precision));
        launch_project(dm, precision, hessian, du, proj, a.status, stream,
                       d_plist.as<int>(std::max<size_t>(static_cast<size_t>(dm.T), 1)), d_pcount.as<unsigned>(1), emesh,
                       mesh_exact, tune.clamp[pi]);
        a.proj = proj;
    }
    launch_eval(dm, precision, hessian, a, stream);
}

extern "C" {

const char* lpg_last_error(void) { return g_last_error.c_str(); }
int lpg_abi_version(void) { return LPG_ABI_VERSION; }

int lpg_build_info(char* buf, size_t size) {
    return guarded([&] {
        int rt = 0, drv = 0;
        cudaRuntimeGetVersion(&rt);
        cudaDriverGetVersion(&drv);
        std::snprintf(buf, size, "litepgo_b200 abi %d; CUDA runtime %d, driver %d; built for sm_100a; device allocations %lld",
                      LPG_ABI_VERSION, rt, drv, g_device_allocations.load());
    });
}

int lpg_mesh_pattern_bsr(int V, int T, const int32_t* tets, int64_t* nnzb, int32_t* row_ptr, int32_t* col_idx) {
    return guarded([&] {
        if (T > 0 && !tets) fail(LPG_EINVAL, "lpg_mesh_pattern_bsr: null tets");
        HostPlan p;
        build_plan(V, T, tets, p);
        if (nnzb) *nnzb = p.nnzb();
        if (row_ptr) std::copy(p.row_ptr.begin(), p.row_ptr.end(), row_ptr);
        if (col_idx) std::copy(p.col_idx.begin(), p.col_idx.end(), col_idx);
    });
}

int lpg_mesh_cluster_summary(int V, int T, const int32_t* tets, int64_t out[5]) {
    return lpg_mesh_cluster_summary_cells(V, T, tets, 4, out);
}

int lpg_mesh_cluster_summary_cells(int V, int T, const int32_t* tets, int cell_width, int64_t out[5]) {
    return guarded([&] {
        if (T > 0 && !tets) fail(LPG_EINVAL, "lpg_mesh_cluster_summary: null cells");
        HostPlan p;
        build_plan(V, T, tets, p, cell_width);
        check_clusters(p, tets);
        check_tet_clusters(p, tets);
        check_solver_layout(p);
        const int ncl = static_cast<int>(p.cl_row_ptr.size()) - 1;
        int64_t max_rows = 0, max_els = 0;
        for (int c = 0; c < ncl; ++c) {
            max_rows = std::max<int64_t>(max_rows, p.cl_row_ptr[c + 1] - p.cl_row_ptr[c]);
            max_els = std::max<int64_t>(max_els, p.cl_el_ptr[c + 1] - p.cl_el_ptr[c]);
        }
        out[0] = ncl;
        out[1] = max_rows;
        out[2] = max_els;
        out[3] = static_cast<int64_t>(p.cl_els.size());
        int64_t contributors = 0;
        for (uint32_t de : p.cl_slot_ent) contributors += de >> 20;
        out[4] = contributors;
    });
}

int lpg_fem_create(int V, const double* X, int T, const int32_t* tets, const double* Xe, const double* theta,
                   int theta_per_element, const double* Fp, int device, lpg_fem_t* out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out) fail(LPG_EINVAL, "lpg_fem_create: null output handle");
        if (T > 0 && (!tets || !theta || (!X && !Xe))) fail(LPG_EINVAL, "lpg_fem_create: null input array");
        auto h = std::make_unique<lpg_fem>();
        h->device = device;
        LPG_CUDA(cudaSetDevice(device));
        LPG_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
        h->stream = h->own_stream;
        build_plan(V, T, tets, h->plan);
        h->from_vertices = Xe == nullptr;
        // Element records (VolumetricElement3D ctor, volumetric_element.hpp:23-39, and the
        // sampled B of deformation_gradient_sampling_response.hpp:24-41).
        std::vector<double> rec(12 * static_cast<size_t>(T));
        std::vector<double> fpinv(Fp ? 9 * static_cast<size_t>(T) : 0);
        h->geo_base.assign(10 * static_cast<size_t>(T), 0.0);
        for (int e = 0; e < T; ++e) {
            double Xc[4][3];
            for (int a = 0; a < 4; ++a)
                for (int k = 0; k < 3; ++k)
                    Xc[a][k] = Xe ? Xe[12 * static_cast<size_t>(e) + 3 * a + k] : X[3 * static_cast<size_t>(tets[4 * e + a]) + k];
            bool finite = true;
            for (int a = 0; a < 4; ++a)
                for (int k = 0; k < 3; ++k) finite = finite && std::isfinite(Xc[a][k]);
            if (!finite) fail(LPG_EINVAL, "VolumetricElement3D: invalid reference Jacobian");
            double J[9]; // row-major, column j = X_{j+1} - X_0
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) J[3 * i + j] = Xc[j + 1][i] - Xc[0][i];
            const double det = det3(J);
            const double w = det / 6.0;
            if (!std::isfinite(det) || det <= 0 || !std::isfinite(w))
                fail(LPG_EINVAL, "VolumetricElement3D: invalid reference determinant or volume weight");
            double G[9];
            inv3(J, G); // rows of J^-1 = grad N_1..3
            for (double g : G)
                if (!std::isfinite(g)) fail(LPG_EINVAL, "Deformation gradient sampling: non-finite physical gradient");
            double vol = w;
            std::copy(G, G + 9, &h->geo_base[10 * static_cast<size_t>(e)]);
            h->geo_base[10 * static_cast<size_t>(e) + 9] = w;
            if (Fp) {
                double P[9]; // row-major from column-major input
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) P[3 * i + j] = Fp[9 * static_cast<size_t>(e) + i + 3 * j];
                bool pf = true;
                for (double v : P) pf = pf && std::isfinite(v);
                if (!pf) fail(LPG_EINVAL, "MultiplicativeKinematics requires finite F and Fp");
                const double dp = det3(P);
                if (!std::isfinite(dp) || dp <= 0) fail(LPG_EDOMAIN, "MultiplicativeKinematics requires finite det(Fp) > 0");
                double Pi[9];
                inv3(P, Pi);
                double G2[9];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        G2[3 * i + j] = G[3 * i] * Pi[j] + G[3 * i + 1] * Pi[3 + j] + G[3 * i + 2] * Pi[6 + j];
                std::memcpy(G, G2, sizeof G);
                std::memcpy(&fpinv[9 * static_cast<size_t>(e)], Pi, sizeof Pi);
                vol = w * dp;
            }
            double* r = &rec[12 * static_cast<size_t>(e)];
            std::memcpy(r, G, sizeof G);
            r[9] = vol;
            r[10] = theta_per_element ? theta[2 * static_cast<size_t>(e)] : theta[0];
            r[11] = theta_per_element ? theta[2 * static_cast<size_t>(e) + 1] : theta[1];
        }
        std::vector<float> rec32(rec.begin(), rec.end());
        upload_plan(*h, V, T);
        DevMesh& m = h->dm;
        std::vector<int32_t> tv(tets, tets + 4 * static_cast<size_t>(T));
        m.tets = reinterpret_cast<int4*>(upload(h->b_tets, tv));
        m.rec64 = upload(h->b_rec64, rec);
        m.rec32 = upload(h->b_rec32, rec32);
        if (Fp) {
            std::vector<float> f32(fpinv.begin(), fpinv.end());
            m.fpinv64 = upload(h->b_fpinv64, fpinv);
            m.fpinv32 = upload(h->b_fpinv32, f32);
        }
        LPG_CUDA(cudaMemset(h->d_status.as<unsigned>(1), 0, sizeof(unsigned)));
        LPG_CUDA(cudaDeviceSynchronize());
        // Launch variants tuned on this mesh unless LPG_AUTOTUNE=0 (then the defaults stay).
        const char* at = std::getenv("LPG_AUTOTUNE");
        if (!(at && std::strcmp(at, "0") == 0)) autotune(*h);
        *out = h.release();
    });
}

int lpg_fem_create_hex_hermite(int V, const double* X, int T, const int32_t* cells, const double* theta,
                               int theta_per_element, int points_per_axis, int device, lpg_fem_t* out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out) fail(LPG_EINVAL, "lpg_fem_create_hex_hermite: null output handle");
        if (T > 0 && (!cells || !theta || !X)) fail(LPG_EINVAL, "lpg_fem_create_hex_hermite: null input array");
        if (points_per_axis != 2 && points_per_axis != 4)
            fail(LPG_EINVAL, "GaussLegendre3D is instantiated for 2 or 4 points per axis");
        if (V < 0 || T < 0 || V > std::numeric_limits<int>::max() / 24)
            fail(LPG_EINVAL, "VertexDofMap requires total DOFs fitting in int");
        for (size_t k = 0; k < 8 * static_cast<size_t>(T); ++k)
            if (cells[k] < 0 || cells[k] >= V)
                fail(LPG_EINVAL, "MeshTopology cell " + std::to_string(k / 8) + " has vertex indices outside [0, num_vertices)");
        auto h = std::make_unique<lpg_fem>();
        h->device = device;
        LPG_CUDA(cudaSetDevice(device));
        LPG_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
        h->stream = h->own_stream;
        // Plan rows: node 8 v + slot (3 DOFs each, so DOF 24 v + 3 slot + c); cell nodes in basis
        // order 8 corner + slot.
        std::vector<int32_t> nodes(64 * static_cast<size_t>(T));
        for (size_t e = 0; e < static_cast<size_t>(T); ++e)
            for (int b = 0; b < 64; ++b) nodes[64 * e + b] = 8 * cells[8 * e + b / 8] + b % 8;
        build_plan(8 * V, T, nodes.data(), h->plan, 64);
        // BasisDofTransform<HexHermiteBasis> (basis_dof_transform.hpp:59-92): every element a
        // positive axis-aligned box in corner order; its edge lengths scale the DOF slots.
        std::vector<double> hb(3 * static_cast<size_t>(T));
        for (size_t e = 0; e < static_cast<size_t>(T); ++e) {
            const double* o = X + 3 * static_cast<size_t>(cells[8 * e]);
            const double len[3] = {X[3 * static_cast<size_t>(cells[8 * e + 1])] - o[0],
                                   X[3 * static_cast<size_t>(cells[8 * e + 3]) + 1] - o[1],
                                   X[3 * static_cast<size_t>(cells[8 * e + 4]) + 2] - o[2]};
            for (int d = 0; d < 3; ++d)
                if (!std::isfinite(len[d]) || !(len[d] > 0))
                    fail(LPG_EINVAL, "Hermite DOF transform requires positive axis-aligned box dimensions");
            for (int c = 0; c < 8; ++c)
                for (int d = 0; d < 3; ++d) {
                    const double r = (X[3 * static_cast<size_t>(cells[8 * e + c]) + d] - o[d]) / len[d];
                    if (!std::isfinite(r) || std::fabs(r - kHexCorner[c][d]) > 1e-12)
                        fail(LPG_EINVAL, "Hermite DOF transform requires axis-aligned boxes in Hex corner order");
                }
            for (int d = 0; d < 3; ++d) hb[3 * e + d] = len[d];
        }
        // Per point the tricubic Hermite reference derivatives (hex_hermite_basis.hpp: function
        // 8 corner + slot is the product of 1D cubic Hermite factors 2 corner_d + order_d, ordered
        // u(0), u'(0), u(1), u'(1), cubic_hermite_basis.hpp) and the weight.
        static const int order[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                        {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
        const int n = points_per_axis, nq = n * n * n;
        double t1[4], w1[4];
        gauss_legendre_01(n, t1, w1);
        std::vector<double> qt(kHermiteTable * static_cast<size_t>(nq));
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    const int q = (i * n + j) * n + k;
                    const double xi[3] = {t1[i], t1[j], t1[k]};
                    double f[3][4], df[3][4];
                    for (int d = 0; d < 3; ++d) {
                        const double t = xi[d], t2 = t * t, t3 = t2 * t;
                        const double fv[4] = {2 * t3 - 3 * t2 + 1, t3 - 2 * t2 + t, -2 * t3 + 3 * t2, t3 - t2};
                        const double dv[4] = {6 * t2 - 6 * t, 3 * t2 - 4 * t + 1, -6 * t2 + 6 * t, 3 * t2 - 2 * t};
                        for (int r = 0; r < 4; ++r) {
                            f[d][r] = fv[r];
                            df[d][r] = dv[r];
                        }
                    }
                    for (int b = 0; b < 64; ++b) {
                        int ix[3];
                        for (int d = 0; d < 3; ++d) ix[d] = 2 * kHexCorner[b / 8][d] + order[b % 8][d];
                        qt[kHermiteTable * q + 3 * b] = df[0][ix[0]] * f[1][ix[1]] * f[2][ix[2]];
                        qt[kHermiteTable * q + 3 * b + 1] = f[0][ix[0]] * df[1][ix[1]] * f[2][ix[2]];
                        qt[kHermiteTable * q + 3 * b + 2] = f[0][ix[0]] * f[1][ix[1]] * df[2][ix[2]];
                    }
                    qt[kHermiteTable * q + 192] = w1[i] * w1[j] * w1[k];
                }
        std::vector<double> th(2 * static_cast<size_t>(T));
        for (int e = 0; e < T; ++e)
            for (int c = 0; c < 2; ++c) th[2 * static_cast<size_t>(e) + c] = theta_per_element ? theta[2 * static_cast<size_t>(e) + c] : theta[c];
        upload_plan(*h, 8 * V, T);
        DevMesh& m = h->dm;
        m.K = 64;
        m.nq = nq;
        m.hex_X = upload(h->b_hex[0], std::vector<double>(X, X + 3 * static_cast<size_t>(V)));
        m.hex_cells = upload(h->b_hex[1], std::vector<int32_t>(cells, cells + 8 * static_cast<size_t>(T)));
        m.hex_theta = upload(h->b_hex[2], th);
        m.herm_q = upload(h->b_hex[3], qt);
        m.herm_h = upload(h->b_herm, hb);
        LPG_CUDA(cudaMemset(h->d_status.as<unsigned>(1), 0, sizeof(unsigned)));
        LPG_CUDA(cudaDeviceSynchronize());
        *out = h.release();
    });
}

int lpg_fem_create_hex(int V, const double* X, int T, const int32_t* cells, const double* theta,
                       int theta_per_element, int points_per_axis, int device, lpg_fem_t* out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out) fail(LPG_EINVAL, "lpg_fem_create_hex: null output handle");
        if (T > 0 && (!cells || !theta || !X)) fail(LPG_EINVAL, "lpg_fem_create_hex: null input array");
        if (points_per_axis != 2 && points_per_axis != 4)
            fail(LPG_EINVAL, "GaussLegendre3D is instantiated for 2 or 4 points per axis");
        auto h = std::make_unique<lpg_fem>();
        h->device = device;
        LPG_CUDA(cudaSetDevice(device));
        LPG_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
        h->stream = h->own_stream;
        build_plan(V, T, cells, h->plan, 8);
        // Gauss-Legendre points on [0,1]^3, last axis fastest (gauss_legendre_3d.hpp), and the
        // trilinear basis derivatives at each (hex_q1_basis.hpp corner order).
        const int n = points_per_axis, nq = n * n * n;
        double t1[4], w1[4];
        gauss_legendre_01(n, t1, w1);
        std::vector<double> qt(25 * static_cast<size_t>(nq));
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    const int q = (i * n + j) * n + k;
                    const double xi[3] = {t1[i], t1[j], t1[k]};
                    for (int a = 0; a < 8; ++a) {
                        double f[3], df[3];
                        for (int d = 0; d < 3; ++d) {
                            f[d] = kHexCorner[a][d] ? xi[d] : 1 - xi[d];
                            df[d] = kHexCorner[a][d] ? 1.0 : -1.0;
                        }
                        qt[25 * q + 3 * a] = df[0] * f[1] * f[2];
                        qt[25 * q + 3 * a + 1] = f[0] * df[1] * f[2];
                        qt[25 * q + 3 * a + 2] = f[0] * f[1] * df[2];
                    }
                    qt[25 * q + 24] = w1[i] * w1[j] * w1[k];
                }
        // Construction checks of VolumetricElement3D (volumetric_element.hpp:23-39) at every point.
        for (size_t v = 0; v < 3 * static_cast<size_t>(V); ++v)
            if (!std::isfinite(X[v])) fail(LPG_EINVAL, "VolumetricElement3D: invalid reference Jacobian");
        for (int e = 0; e < T; ++e)
            for (int q = 0; q < nq; ++q) {
                double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int a = 0; a < 8; ++a) {
                    const double* Xa = X + 3 * static_cast<size_t>(cells[8 * static_cast<size_t>(e) + a]);
                    for (int i = 0; i < 3; ++i)
                        for (int d = 0; d < 3; ++d) J[3 * i + d] += Xa[i] * qt[25 * q + 3 * a + d];
                }
                const double det = det3(J), w = qt[25 * q + 24] * det;
                if (!std::isfinite(det) || det <= 0 || !std::isfinite(w))
                    fail(LPG_EINVAL, "VolumetricElement3D: invalid reference determinant or volume weight");
            }
        std::vector<double> th(2 * static_cast<size_t>(T));
        for (int e = 0; e < T; ++e)
            for (int c = 0; c < 2; ++c) th[2 * static_cast<size_t>(e) + c] = theta_per_element ? theta[2 * static_cast<size_t>(e) + c] : theta[c];
        upload_plan(*h, V, T);
        DevMesh& m = h->dm;
        m.K = 8;
        m.nq = nq;
        m.hex_X = upload(h->b_hex[0], std::vector<double>(X, X + 3 * static_cast<size_t>(V)));
        m.hex_cells = upload(h->b_hex[1], std::vector<int32_t>(cells, cells + 8 * static_cast<size_t>(T)));
        m.hex_theta = upload(h->b_hex[2], th);
        m.hex_q = upload(h->b_hex[3], qt);
        LPG_CUDA(cudaMemset(h->d_status.as<unsigned>(1), 0, sizeof(unsigned)));
        LPG_CUDA(cudaDeviceSynchronize());
        *out = h.release();
    });
}

int lpg_fem_destroy(lpg_fem_t h) {
    return guarded([&] {
        if (!h) return;
        cudaSetDevice(h->device);
        if (h->own_stream) cudaStreamSynchronize(h->own_stream);
        if (h->stream && h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
        delete h;
    });
}

int lpg_fem_set_stream(lpg_fem_t h, void* stream) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    });
}

int lpg_fem_sizes(lpg_fem_t h, int* V, int* T, int* n, int64_t* nnzb, int64_t* nnz) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        if (V) *V = h->dm.V;
        if (T) *T = h->dm.T;
        if (n) *n = 3 * h->dm.V;
        if (nnzb) *nnzb = h->dm.nnzb;
        if (nnz) *nnz = 9 * h->dm.nnzb;
    });
}

int lpg_fem_pattern_bsr(lpg_fem_t h, int32_t* row_ptr, int32_t* col_idx) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        if (row_ptr) std::copy(h->plan.row_ptr.begin(), h->plan.row_ptr.end(), row_ptr);
        if (col_idx) std::copy(h->plan.col_idx.begin(), h->plan.col_idx.end(), col_idx);
    });
}

int lpg_fem_solver_layout(lpg_fem_t h, int64_t* num_slots, int* num_chunks, int32_t* sell_ptr, int32_t* sell_row) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        const HostPlan& p = h->plan;
        if (num_slots) *num_slots = p.sell_ptr.back();
        if (num_chunks) *num_chunks = static_cast<int>(p.sell_ptr.size()) - 1;
        if (sell_ptr) std::copy(p.sell_ptr.begin(), p.sell_ptr.end(), sell_ptr);
        if (sell_row) std::copy(p.sell_row.begin(), p.sell_row.end(), sell_row);
    });
}

int lpg_fem_pattern_csc(lpg_fem_t h, int32_t* outer, int32_t* inner) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        const HostPlan& p = h->plan;
        // Column 3v + k holds rows 3w + i for the sorted block columns w of row v.
        for (int v = 0; v < p.V; ++v) {
            const int s0 = p.row_ptr[v], nb = p.row_ptr[v + 1] - s0;
            for (int k = 0; k < 3; ++k) {
                const int64_t start = 9 * static_cast<int64_t>(s0) + 3 * static_cast<int64_t>(nb) * k;
                if (outer) outer[3 * v + k] = static_cast<int32_t>(start);
                if (inner)
                    for (int q = 0; q < nb; ++q)
                        for (int i = 0; i < 3; ++i) inner[start + 3 * q + i] = 3 * p.col_idx[s0 + q] + i;
            }
        }
        if (outer) outer[3 * p.V] = static_cast<int32_t>(9 * p.nnzb());
    });
}

int lpg_fem_eval(lpg_fem_t h, const double* u, int io_mem, double* energy, double* grad, int hessian, int precision,
                 int layout, void* hess, int hess_mem) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        if (!u && n > 0) fail(LPG_EINVAL, "lpg_fem_eval: null u");
        if (hessian != LPG_HESSIAN_NONE && !hess) fail(LPG_EINVAL, "lpg_fem_eval: null Hessian output");
        if (layout != LPG_LAYOUT_BSR && layout != LPG_LAYOUT_CSC) fail(LPG_EINVAL, "invalid Hessian layout");
        const double* du = h->stage_in(u, io_mem, h->d_u, n);
        double* dgrad = nullptr;
        if (grad) dgrad = io_mem == LPG_MEM_DEVICE ? grad : h->d_grad.as<double>(n);
        const size_t hbytes = 9 * static_cast<size_t>(h->dm.nnzb) * (precision == LPG_PRECISION_F64 ? 8 : 4);
        void* dhess = nullptr;
        if (hessian != LPG_HESSIAN_NONE) {
            if (hess_mem != LPG_MEM_HOST && hess_mem != LPG_MEM_DEVICE) fail(LPG_EINVAL, "invalid memory flag");
            dhess = hess_mem == LPG_MEM_DEVICE ? hess : h->d_hess.ensure(hbytes);
        }
        h->eval_async(du, dgrad, hessian, precision, layout, dhess, nullptr);
        double e = 0;
        LPG_CUDA(cudaMemcpyAsync(&e, h->d_energy.ptr, sizeof e, cudaMemcpyDeviceToHost, h->stream));
        if (grad && io_mem == LPG_MEM_HOST)
            LPG_CUDA(cudaMemcpyAsync(grad, dgrad, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        if (dhess && hess_mem == LPG_MEM_HOST)
            LPG_CUDA(cudaMemcpyAsync(hess, dhess, hbytes, cudaMemcpyDeviceToHost, h->stream));
        raise_status(h->take_status());
        if (!std::isfinite(e)) fail(LPG_EDOMAIN, "MeshEnergy: non-finite energy sum");
        if (energy) *energy = e;
    });
}

int lpg_fem_deformation_gradients(lpg_fem_t h, const double* u, int io_mem, double* F) {
    return guarded([&] {
        if (!h || !F) fail(LPG_EINVAL, "lpg_fem_deformation_gradients: null argument");
        not_hermite(*h, "lpg_fem_deformation_gradients");
        if (h->dm.fpinv64) fail(LPG_EINVAL, "lpg_fem_deformation_gradients: the handle has a plastic field");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const bool hex = h->dm.K == 8;
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const size_t rows = static_cast<size_t>(h->dm.T) * (hex ? h->dm.nq : 1); // one F per quadrature point
        const double* du = h->stage_in(u, io_mem, h->d_u, n);
        double* dF = io_mem == LPG_MEM_DEVICE ? F : h->d_vjp.as<double>(std::max<size_t>(9 * rows, 1));
        if (hex)
            launch_hex_deformation_gradients(h->dm, du, dF, h->d_status.as<unsigned>(1), h->stream);
        else
            launch_deformation_gradients(h->dm, du, dF, h->d_status.as<unsigned>(1), h->stream);
        if (io_mem == LPG_MEM_HOST && rows > 0)
            LPG_CUDA(cudaMemcpyAsync(F, dF, 9 * rows * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        raise_status(h->take_status());
    });
}

int lpg_fem_eval_material(lpg_fem_t h, const double* W, const double* P, const double* A, int in_mem, double* energy,
                          double* grad, int hessian, int precision, int layout, void* hess, int out_mem) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        not_hermite(*h, "lpg_fem_eval_material");
        if (h->dm.fpinv64) fail(LPG_EINVAL, "lpg_fem_eval_material: the handle has a plastic field");
        const bool hex = h->dm.K == 8;
        // Material rows: one per element (tets) or per quadrature point (hexes).
        const size_t T = static_cast<size_t>(h->dm.T) * (hex ? h->dm.nq : 1), n = 3 * static_cast<size_t>(h->dm.V);
        if (T > 0 && (!W || (grad && !P))) fail(LPG_EINVAL, "lpg_fem_eval_material: null material output");
        if (hessian != LPG_HESSIAN_NONE && hessian != LPG_HESSIAN_EXACT && hessian != LPG_HESSIAN_PROJECTED)
            fail(LPG_EINVAL, "Energy: invalid Hessian kind");
        if (hessian != LPG_HESSIAN_NONE && (!hess || (T > 0 && !A)))
            fail(LPG_EINVAL, "lpg_fem_eval_material: a Hessian needs d2W/dF2 and an output");
        if (precision != LPG_PRECISION_F64 && precision != LPG_PRECISION_MIXED) fail(LPG_EINVAL, "invalid precision");
        if (layout != LPG_LAYOUT_BSR && layout != LPG_LAYOUT_CSC) fail(LPG_EINVAL, "invalid Hessian layout");
        if (out_mem != LPG_MEM_HOST && out_mem != LPG_MEM_DEVICE) fail(LPG_EINVAL, "invalid memory flag");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        // Inputs on the device (staged through the handle's scratch when on the host).
        auto stage = [&](const double* p, size_t count, DeviceBuffer& buf) -> const double* {
            if (!p || count == 0 || in_mem == LPG_MEM_DEVICE) return p;
            if (in_mem != LPG_MEM_HOST) fail(LPG_EINVAL, "invalid memory flag");
            double* d = buf.as<double>(count);
            LPG_CUDA(cudaMemcpyAsync(d, p, count * sizeof(double), cudaMemcpyHostToDevice, s));
            return d;
        };
        const double* dW = stage(W, T, h->d_mat[0]);
        const double* dP = grad ? stage(P, 9 * T, h->d_mat[1]) : nullptr;
        const double* dA = hessian != LPG_HESSIAN_NONE ? stage(A, 81 * T, h->d_mat[2]) : nullptr;
        EvalArgs a;
        a.grad = grad ? (out_mem == LPG_MEM_DEVICE ? grad : h->d_grad.as<double>(std::max<size_t>(n, 1))) : nullptr;
        const size_t hbytes = 9 * static_cast<size_t>(h->dm.nnzb) * (precision == LPG_PRECISION_F64 ? 8 : 4);
        a.hess = hessian != LPG_HESSIAN_NONE ? (out_mem == LPG_MEM_DEVICE ? hess : h->d_hess.ensure(hbytes)) : nullptr;
        a.layout = layout;
        a.cluster_energy = h->d_cluster_energy.as<double>(static_cast<size_t>(std::max(h->dm.ncl, h->dm.tc_ncl)) + 256);
        a.energy = h->d_energy.as<double>(1);
        a.status = h->d_status.as<unsigned>(1);
        const int pi = precision == LPG_PRECISION_F64 ? 0 : 1;
        const size_t nel = std::max<size_t>(static_cast<size_t>(h->dm.T), 1);
        if (hex) {
            const bool projected = hessian == LPG_HESSIAN_PROJECTED;
            void* blocks = a.hess ? h->d_proj.ensure(hex_blocks_bytes(h->dm, precision, projected)) : nullptr;
            launch_hex_material_eval(h->dm, precision, hessian, dW, dP, dA, h->d_mat[3].as<double>(nel),
                                     h->d_vjp.as<double>(24 * nel), blocks,
                                     projected && a.hess ? h->d_plist.as<int>(nel) : nullptr, a, s);
        } else {
            void* proj = a.hess ? h->d_proj.ensure(project_bytes(h->dm, precision)) : nullptr;
            launch_material_eval(h->dm, precision, hessian, dW, dP, dA, h->d_mat[3].as<double>(nel),
                                 h->d_vjp.as<double>(12 * nel), proj, h->d_plist.as<int>(nel),
                                 h->d_pcount.as<unsigned>(1), h->tune.clamp[pi], a, s);
        }
        double e = 0;
        LPG_CUDA(cudaMemcpyAsync(&e, a.energy, sizeof e, cudaMemcpyDeviceToHost, s));
        if (grad && out_mem == LPG_MEM_HOST && n > 0)
            LPG_CUDA(cudaMemcpyAsync(grad, a.grad, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (a.hess && out_mem == LPG_MEM_HOST) LPG_CUDA(cudaMemcpyAsync(hess, a.hess, hbytes, cudaMemcpyDeviceToHost, s));
        raise_status(h->take_status());
        if (!std::isfinite(e)) fail(LPG_EDOMAIN, "MeshEnergy: non-finite energy sum");
        if (energy) *energy = e;
    });
}

int lpg_fem_time_eval(lpg_fem_t h, const double* u, double* grad, int hessian, int precision, int layout, void* hess,
                      int launches, int flush_l2, double* ms_assemble, double* ms_eval) {
    return guarded([&] {
        if (!h || !u || launches <= 0) fail(LPG_EINVAL, "lpg_fem_time_eval: invalid arguments");
        if (hessian != LPG_HESSIAN_NONE && !hess) fail(LPG_EINVAL, "lpg_fem_time_eval: null Hessian output");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t flush_bytes = size_t(512) << 20; // four times the 126 MB L2
        void* fl = flush_l2 ? h->d_flush.ensure(flush_bytes) : nullptr;
        std::vector<cudaEvent_t> ev(4 * static_cast<size_t>(launches));
        for (auto& e : ev) LPG_CUDA(cudaEventCreate(&e));
        for (int i = 0; i < launches; ++i) {
            if (fl) LPG_CUDA(cudaMemsetAsync(fl, i & 0xff, flush_bytes, h->stream));
            LPG_CUDA(cudaEventRecord(ev[4 * i], h->stream));
            h->eval_async(u, grad, hessian, precision, layout, hess, nullptr, ev[4 * i + 1], ev[4 * i + 2]);
            LPG_CUDA(cudaEventRecord(ev[4 * i + 3], h->stream));
        }
        const unsigned st = h->take_status();
        double ta = 0, te = 0;
        for (int i = 0; i < launches; ++i) {
            float a = 0, b = 0;
            LPG_CUDA(cudaEventElapsedTime(&a, ev[4 * i + 1], ev[4 * i + 2]));
            LPG_CUDA(cudaEventElapsedTime(&b, ev[4 * i], ev[4 * i + 3]));
            ta += a;
            te += b;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        raise_status(st);
        if (ms_assemble) *ms_assemble = ta / launches;
        if (ms_eval) *ms_eval = te / launches;
    });
}

int lpg_fem_element_energies(lpg_fem_t h, const double* u, int io_mem, double* elem_energy) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const double* du = h->stage_in(u, io_mem, h->d_u, n);
        double* de = io_mem == LPG_MEM_DEVICE ? elem_energy : h->d_vjp.as<double>(std::max(h->dm.T, 1));
        h->eval_async(du, nullptr, LPG_HESSIAN_NONE, LPG_PRECISION_F64, LPG_LAYOUT_BSR, nullptr, de);
        if (io_mem == LPG_MEM_HOST && h->dm.T > 0)
            LPG_CUDA(cudaMemcpyAsync(elem_energy, de, h->dm.T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        raise_status(h->take_status());
    });
}

int lpg_fem_feasible_step(lpg_fem_t h, const double* u, const double* du, int io_mem, double* alpha) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const double* d_u = h->stage_in(u, io_mem, h->d_u, n);
        const double* d_du = h->stage_in(du, io_mem, h->d_u2, n);
        const int nb = feasible_blocks(h->dm);
        double* bm = h->d_block.as<double>(std::max(nb, 1));
        double* al = h->d_alpha.as<double>(1);
        launch_feasible(h->dm, d_u, d_du, bm, nb, al, h->d_status.as<unsigned>(1), h->stream);
        double v = 1;
        LPG_CUDA(cudaMemcpyAsync(&v, al, sizeof v, cudaMemcpyDeviceToHost, h->stream));
        const unsigned st = h->take_status();
        // Energy::max_feasible_step validates x and dx first (energy.cpp:35-41).
        if (st & ST_BAD_INPUT) fail(LPG_EINVAL, "Energy::max_feasible_step: x and dx must have num_dofs finite entries");
        raise_status(st);
        if (!(v >= 0.0 && v <= 1.0)) fail(LPG_ELOGIC, "Energy::max_feasible_step: the energy returned a value outside [0, 1]");
        if (alpha) *alpha = v;
    });
}

int lpg_fem_force_vjp_theta(lpg_fem_t h, const double* u, const double* w, int io_mem, int per_element, double* out) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const double* d_u = h->stage_in(u, io_mem, h->d_u, n);
        const double* d_w = h->stage_in(w, io_mem, h->d_u2, n);
        const size_t T = static_cast<size_t>(h->dm.T);
        double* pe = (per_element && io_mem == LPG_MEM_DEVICE) ? out : h->d_vjp.as<double>(std::max<size_t>(2 * T, 2));
        launch_force_vjp(h->dm, d_u, d_w, pe, h->d_status.as<unsigned>(1), h->stream);
        if (per_element) {
            if (io_mem == LPG_MEM_HOST && T > 0)
                LPG_CUDA(cudaMemcpyAsync(out, pe, 2 * T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        } else {
            const int nb = static_cast<int>(std::min<size_t>(1024, (T + 4095) / 4096));
            double* part = h->d_block.as<double>(std::max(2 * nb, 2));
            double* res = io_mem == LPG_MEM_DEVICE ? out : h->d_alpha.as<double>(2);
            launch_sum_pairs(pe, static_cast<int>(T), part, nb, res, h->stream);
            if (io_mem == LPG_MEM_HOST)
                LPG_CUDA(cudaMemcpyAsync(out, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        }
        raise_status(h->take_status());
    });
}

void lpg_newton_default_options(lpg_newton_options* o) {
    if (!o) return;
    o->gradient_tolerance = std::nan("");
    o->max_iterations = 50;
    o->hessian = LPG_HESSIAN_PROJECTED;
    o->max_line_search_steps = 30;
    o->line_search_shrink = 0.5;
    o->stop_rule = 0;
    o->accept_rule = 0;
    o->precision = LPG_PRECISION_F64;
    o->cg_tolerance = 1e-2;
    o->cg_max_iterations = 20000;
    o->exact_below = 0.0;
}

int lpg_newton_solve(lpg_fem_t h, const int32_t* fixed, int nfixed, const double* f_ext, const double* x0,
                     int io_mem, const lpg_newton_options* o, double* x_out, lpg_newton_result* res) {
    return guarded([&] {
        if (!h || !o || !x0 || !x_out) fail(LPG_EINVAL, "lpg_newton_solve: null argument");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        newton_solve(*h, fixed, nfixed, f_ext, x0, io_mem, *o, x_out, res);
    });
}

int lpg_newton_solve_terms(lpg_fem_t h, const lpg_newton_terms* terms, const int32_t* fixed, int nfixed,
                           const double* f_ext, const double* x0, int io_mem, const lpg_newton_options* o,
                           double* x_out, lpg_newton_result* res) {
    return guarded([&] {
        if (!h || !o || !x0 || !x_out) fail(LPG_EINVAL, "lpg_newton_solve_terms: null argument");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        newton_solve(*h, fixed, nfixed, f_ext, x0, io_mem, *o, x_out, res, terms);
    });
}

int lpg_adjoint_solve_terms(lpg_fem_t h, const lpg_newton_terms* terms, const double* u_star, const double* dLdu,
                            const int32_t* fixed, int nfixed, int io_mem, int precision, double cg_tolerance,
                            double* lambda_out) {
    return guarded([&] {
        if (!h || !u_star || !dLdu || !lambda_out) fail(LPG_EINVAL, "lpg_adjoint_solve_terms: null argument");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        adjoint_lambda(*h, terms, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, lambda_out);
    });
}

int lpg_fem_set_fp(lpg_fem_t h, const double* Fp, int fp_per_element) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        tet_only(*h, "lpg_fem_set_fp");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        DevMesh& m = h->dm;
        const size_t T = static_cast<size_t>(m.T);
        std::vector<double> geo(h->geo_base);
        std::vector<double> fpinv(Fp ? 9 * T : 0);
        for (size_t e = 0; e < T && Fp; ++e) {
            const double* src = Fp + (fp_per_element ? 9 * e : 0);
            double P[9]; // row-major from column-major input
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) P[3 * i + j] = src[i + 3 * j];
            for (double v : P)
                if (!std::isfinite(v)) fail(LPG_EINVAL, "MultiplicativeKinematics requires finite F and Fp");
            const double dp = det3(P);
            if (!std::isfinite(dp) || dp <= 0) fail(LPG_EDOMAIN, "MultiplicativeKinematics requires finite det(Fp) > 0");
            double Pi[9];
            inv3(P, Pi);
            double* g = &geo[10 * e];
            double G2[9];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) G2[3 * i + j] = g[3 * i] * Pi[j] + g[3 * i + 1] * Pi[3 + j] + g[3 * i + 2] * Pi[6 + j];
            std::copy(G2, G2 + 9, g);
            g[9] *= dp;
            std::copy(Pi, Pi + 9, &fpinv[9 * e]);
        }
        if (T > 0) {
            double* d = h->d_vjp.as<double>(10 * T);
            LPG_CUDA(cudaMemcpyAsync(d, geo.data(), 10 * T * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            launch_set_geometry(m, d, h->stream);
        }
        if (Fp) {
            std::vector<float> f32(fpinv.begin(), fpinv.end());
            LPG_CUDA(cudaStreamSynchronize(h->stream));
            m.fpinv64 = upload(h->b_fpinv64, fpinv);
            m.fpinv32 = upload(h->b_fpinv32, f32);
        } else {
            m.fpinv64 = nullptr;
            m.fpinv32 = nullptr;
        }
        LPG_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int lpg_fem_force_vjp_fp(lpg_fem_t h, const double* u, const double* w, int io_mem, int per_element, double* out) {
    return guarded([&] {
        if (!h || !out) fail(LPG_EINVAL, "lpg_fem_force_vjp_fp: null argument");
        tet_only(*h, "lpg_fem_force_vjp_fp");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const double* d_u = h->stage_in(u, io_mem, h->d_u, n);
        const double* d_w = h->stage_in(w, io_mem, h->d_u2, n);
        const size_t T = static_cast<size_t>(h->dm.T);
        double* pe = (per_element && io_mem == LPG_MEM_DEVICE) ? out : h->d_vjp.as<double>(std::max<size_t>(9 * T, 9));
        launch_fp_vjp(h->dm, d_u, d_w, pe, h->d_status.as<unsigned>(1), h->stream);
        if (per_element) {
            if (io_mem == LPG_MEM_HOST && T > 0)
                LPG_CUDA(cudaMemcpyAsync(out, pe, 9 * T * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        } else {
            const int nb = static_cast<int>(std::min<size_t>(1024, (T + 4095) / 4096));
            double* part = h->d_block.as<double>(std::max(9 * nb, 9));
            double* res = io_mem == LPG_MEM_DEVICE ? out : h->d_alpha.as<double>(9);
            launch_sum_cols9(pe, static_cast<int>(T), part, nb, res, h->stream);
            if (io_mem == LPG_MEM_HOST)
                LPG_CUDA(cudaMemcpyAsync(out, res, 9 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        }
        raise_status(h->take_status());
    });
}

int lpg_adjoint_fp(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed_dofs, int num_fixed,
                   int io_mem, int precision, double cg_tolerance, int per_element, double* dFp, double* lambda_out) {
    return guarded([&] {
        if (!h || !u_star || !dLdu || !dFp) fail(LPG_EINVAL, "lpg_adjoint_fp: null argument");
        tet_only(*h, "lpg_adjoint_fp");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        adjoint_fp(*h, u_star, dLdu, fixed_dofs, num_fixed, io_mem, precision, cg_tolerance, per_element, dFp,
                   lambda_out);
    });
}

int lpg_read_veg(const char* path, int* num_vertices, int* num_cells, int* cell_width, double* positions,
                 int32_t* cells) {
    return guarded([&] {
        if (!path) fail(LPG_EINVAL, "lpg_read_veg: null path");
        // A sizes-only call keeps the parsed mesh for the next call on this thread with the same
        // path (and unchanged file), so the usual two calls parse the file once.
        thread_local std::string cached_key;
        thread_local VegMesh cached;
        std::error_code ec;
        const auto stamp = std::filesystem::last_write_time(path, ec);
        const auto bytes = std::filesystem::file_size(path, ec);
        const std::string key = std::string(path) + '\n' + std::to_string(stamp.time_since_epoch().count()) + '\n' +
                                std::to_string(ec ? 0 : bytes);
        VegMesh m;
        if (!ec && key == cached_key) {
            m = std::move(cached);
            cached_key.clear();
        } else {
            read_veg(path, m);
        }
        if (!positions && !cells && !ec) {
            cached = m;
            cached_key = key;
        }
        if (num_vertices) *num_vertices = m.num_vertices;
        if (num_cells) *num_cells = m.width ? static_cast<int>(m.cells.size() / m.width) : 0;
        if (cell_width) *cell_width = m.width;
        if (positions) std::copy(m.positions.begin(), m.positions.end(), positions);
        if (cells) std::copy(m.cells.begin(), m.cells.end(), cells);
    });
}

int lpg_write_veg(const char* path, int num_vertices, const double* positions, int num_cells, int cell_width,
                  const int32_t* cells) {
    return guarded([&] {
        if (!path || (num_vertices > 0 && !positions) || (num_cells > 0 && !cells))
            fail(LPG_EINVAL, "lpg_write_veg: null argument");
        write_veg(path, num_vertices, positions, num_cells, cell_width, cells);
    });
}

int lpg_fem_autotune(lpg_fem_t h) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        autotune(*h);
    });
}

int lpg_fem_get_tuning(lpg_fem_t h, int32_t choice[6], double ms[18]) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        const Tuning& t = h->tune;
        if (choice) {
            const int32_t c[6] = {t.cl[0], t.cl[1], t.spmv[0], t.spmv[1], t.clamp[0], t.clamp[1]};
            std::copy(c, c + 6, choice);
        }
        if (ms)
            for (int f = 0; f < 3; ++f)
                for (int p = 0; p < 2; ++p)
                    for (int v = 0; v < 3; ++v) ms[6 * f + 3 * p + v] = t.tuned ? t.ms[f][p][v] : std::nan("");
    });
}

int lpg_fem_set_tuning(lpg_fem_t h, const int32_t choice[6]) {
    return guarded([&] {
        if (!h || !choice) fail(LPG_EINVAL, "lpg_fem_set_tuning: null argument");
        const int lim[6] = {kClVariants, kClVariants, kSpmvVariants, kSpmvVariants, 1, kClampVariants};
        for (int i = 0; i < 6; ++i)
            if (choice[i] < -1 || choice[i] >= lim[i]) fail(LPG_EINVAL, "lpg_fem_set_tuning: variant out of range");
        BusyGuard busy(h->busy);
        Tuning& t = h->tune;
        int* dst[6] = {&t.cl[0], &t.cl[1], &t.spmv[0], &t.spmv[1], &t.clamp[0], &t.clamp[1]};
        for (int i = 0; i < 6; ++i)
            if (choice[i] >= 0) *dst[i] = choice[i];
    });
}

int lpg_fem_set_theta(lpg_fem_t h, const double* theta, int theta_per_element) {
    return guarded([&] {
        if (!h) fail(LPG_EINVAL, "null handle");
        if (!theta && h->dm.T > 0) fail(LPG_EINVAL, "lpg_fem_set_theta: null theta");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = theta_per_element ? 2 * static_cast<size_t>(h->dm.T) : 2;
        for (size_t k = 0; k < n && h->dm.T > 0; ++k)
            if (!std::isfinite(theta[k])) fail(LPG_EINVAL, "VolumetricFemEnergy: theta must be finite");
        if (h->dm.T == 0) return;
        if (h->dm.K != 4) { // hexes keep theta per element, read at every evaluation
            const size_t T = static_cast<size_t>(h->dm.T);
            std::vector<double> th(2 * T);
            for (size_t e = 0; e < T; ++e)
                for (int c = 0; c < 2; ++c) th[2 * e + c] = theta_per_element ? theta[2 * e + c] : theta[c];
            LPG_CUDA(cudaMemcpyAsync(h->dm.hex_theta, th.data(), 2 * T * sizeof(double),
                                     cudaMemcpyHostToDevice, h->stream));
            LPG_CUDA(cudaStreamSynchronize(h->stream));
            return;
        }
        double* d = h->d_u2.as<double>(n);
        LPG_CUDA(cudaMemcpyAsync(d, theta, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        launch_set_theta(h->dm, d, theta_per_element, h->stream);
        LPG_CUDA(cudaStreamSynchronize(h->stream));
    });
}

int lpg_fem_force_vjp_rest(lpg_fem_t h, const double* u, const double* w, int io_mem, double* out) {
    return guarded([&] {
        if (!h || !out) fail(LPG_EINVAL, "lpg_fem_force_vjp_rest: null argument");
        tet_only(*h, "lpg_fem_force_vjp_rest");
        if (!h->from_vertices || h->dm.fpinv64)
            fail(LPG_EINVAL, "rest-position sensitivity needs vertex rest positions and no plastic field");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        const size_t n = 3 * static_cast<size_t>(h->dm.V);
        const double* d_u = h->stage_in(u, io_mem, h->d_u, n);
        const double* d_w = h->stage_in(w, io_mem, h->d_u2, n);
        double* d_out = io_mem == LPG_MEM_DEVICE ? out : h->d_grad.as<double>(std::max<size_t>(n, 1));
        double* pe = h->d_vjp.as<double>(std::max<size_t>(12 * static_cast<size_t>(h->dm.T), 1));
        launch_rest_vjp(h->dm, d_u, d_w, pe, 1.0, d_out, h->d_status.as<unsigned>(1), h->stream);
        if (io_mem == LPG_MEM_HOST && n > 0)
            LPG_CUDA(cudaMemcpyAsync(out, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        raise_status(h->take_status());
    });
}

int lpg_adjoint_rest(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed,
                     int io_mem, int precision, double cg_tolerance, double* dX, double* lambda_out) {
    return guarded([&] {
        if (!h || !u_star || !dLdu || !dX) fail(LPG_EINVAL, "lpg_adjoint_rest: null argument");
        tet_only(*h, "lpg_adjoint_rest");
        if (!h->from_vertices || h->dm.fpinv64)
            fail(LPG_EINVAL, "rest-position sensitivity needs vertex rest positions and no plastic field");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        adjoint_rest(*h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, dX, lambda_out);
    });
}

int lpg_batch_newton_solve(lpg_fem_t h, int num_meshes, const int32_t* vertex_offsets, const int32_t* element_offsets,
                           const int32_t* fixed, int nfixed, const double* f_ext, const double* x0, int io_mem,
                           const lpg_newton_options* o, double* x_out, lpg_batch_mesh_result* per_mesh,
                           lpg_newton_result* result) {
    return guarded([&] {
        if (!h || !o || !x_out || (!x0 && h->dm.V > 0)) fail(LPG_EINVAL, "lpg_batch_newton_solve: null argument");
        tet_only(*h, "lpg_batch_newton_solve");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        batch_newton_solve(*h, num_meshes, vertex_offsets, element_offsets, fixed, nfixed, f_ext, x0, io_mem, *o, x_out,
                           per_mesh, result);
    });
}

int lpg_adjoint_theta(lpg_fem_t h, const double* u_star, const double* dLdu, const int32_t* fixed, int nfixed,
                      int io_mem, int precision, double cg_tolerance, int per_element, double* dtheta,
                      double* lambda_out) {
    return guarded([&] {
        if (!h || !u_star || !dLdu || !dtheta) fail(LPG_EINVAL, "lpg_adjoint_theta: null argument");
        BusyGuard busy(h->busy);
        LPG_CUDA(cudaSetDevice(h->device));
        adjoint_theta(*h, u_star, dLdu, fixed, nfixed, io_mem, precision, cg_tolerance, per_element, dtheta,
                      lambda_out);
    });
}

} // extern "C"
