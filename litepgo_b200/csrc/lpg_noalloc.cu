// lpg_noalloc.cu -- the feasible step without any device allocation.
//
// Some callers must not call cudaMalloc at the moment they need a feasible step: solvers
// embedded in a framework whose device memory is owned by its own pool (a training loop on
// PyTorch's caching allocator, an application with a fixed memory budget), where a library
// allocation mid-step fragments or exceeds that budget. lpg_fem_feasible_step may allocate
// its per-block scratch on first use; this variant takes that scratch from a fixed array in
// the library image instead. It serves tet, hex and Hermite handles (one thread per element
// in every case) and returns synchronously.
//
// The scratch is one file-scope __device__ array of kMaxBlocks + 4 doubles (about 512 KB):
// the per-block minima of the feasible-step reduction, the result and the status word. Every
// GPU that loads the library holds it until the process exits. All calls on a device share
// it, so two calls that overlap on the GPU (on different streams, or through different
// handles) race on it; callers must order them. The status word is cleared by each call; the
// block minima are overwritten before they are read.

#include <cmath>
#include <mutex>
#include <string>

#include "lpg_solver.h"

namespace lpg {

extern thread_local std::string g_last_error;

namespace {

// 65,536 blocks of 256 elements: meshes of up to 16,777,216 elements.
constexpr int kMaxBlocks = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_feasible_scratch[kMaxBlocks + 4];

std::mutex g_scratch_mutex;
double* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on `device`, looked up once per device with that device
// current. In host code the array's name is only a host-side stand-in, so kernels must be given
// this address, never the symbol itself.
double* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) fail(LPG_EINVAL, "lpg_fem_feasible_step_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[device]) {
        void* p = nullptr;
        LPG_CUDA(cudaGetSymbolAddress(&p, g_feasible_scratch));
        g_scratch_address[device] = static_cast<double*>(p);
    }
    return g_scratch_address[device];
}

// u and du must be device (or managed) memory on the handle's GPU: a host pointer given to the
// kernel would fault, so it is rejected here.
void check_device_array(const void* p, int device, const char* name) {
    cudaPointerAttributes at{};
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(LPG_EINVAL, std::string("lpg_fem_feasible_step_noalloc: ") + name + " is not a device pointer");
    }
    const bool ok = at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == device);
    if (!ok)
        fail(LPG_EINVAL, std::string("lpg_fem_feasible_step_noalloc: ") + name +
                             " must be device memory on the handle's GPU");
}

} // namespace
} // namespace lpg

extern "C" int lpg_fem_feasible_step_noalloc(lpg_fem_t h, const double* u, const double* du, double* alpha) {
    using namespace lpg;
    try {
        if (!h || !u || !du || !alpha) fail(LPG_EINVAL, "lpg_fem_feasible_step_noalloc: null argument");
        if (h->busy.exchange(true)) fail(LPG_EBUSY, "MeshEnergy is already in use by another call");
        struct Release {
            std::atomic<bool>& b;
            ~Release() { b.store(false); }
        } release{h->busy};
        LPG_CUDA(cudaSetDevice(h->device));
        check_device_array(u, h->device, "u");
        check_device_array(du, h->device, "du");
        const int nb = feasible_blocks(h->dm);
        if (nb > kMaxBlocks)
            fail(LPG_EINVAL, "lpg_fem_feasible_step_noalloc: at most 16,777,216 elements (" +
                                 std::to_string(h->dm.T) + " given); use lpg_fem_feasible_step");
        double* scratch = scratch_address(h->device);
        double* block_min = scratch;
        double* result = scratch + kMaxBlocks;
        unsigned* status = reinterpret_cast<unsigned*>(scratch + kMaxBlocks + 2);
        LPG_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned), h->stream));
        launch_feasible(h->dm, u, du, block_min, nb, result, status, h->stream);
        double a = 1;
        unsigned st = 0;
        LPG_CUDA(cudaMemcpyAsync(&a, result, sizeof a, cudaMemcpyDeviceToHost, h->stream));
        LPG_CUDA(cudaMemcpyAsync(&st, status, sizeof st, cudaMemcpyDeviceToHost, h->stream));
        LPG_CUDA(cudaStreamSynchronize(h->stream));
        if (st & ST_BAD_INPUT) fail(LPG_EINVAL, "Energy::max_feasible_step: x and dx must have num_dofs finite entries");
        raise_status(st);
        if (!(a >= 0.0 && a <= 1.0)) fail(LPG_ELOGIC, "Energy::max_feasible_step: the energy returned a value outside [0, 1]");
        *alpha = a;
        return LPG_OK;
    } catch (const Error& e) {
        g_last_error = e.what;
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return LPG_ELOGIC;
    }
}
