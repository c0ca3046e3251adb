// dA/dt at mesh nodes without any device allocation by the library.
//
// Some callers cannot let a library allocate GPU memory: a process whose device memory is already
// reserved in full by another framework's caching allocator (a cudaMalloc from here would fail, or
// would fragment the caller's budget), or code that has to stay on a fixed, audited memory budget
// set up front. This entry point serves them: the caller passes every input and output in device
// memory, and the only scratch the computation needs -- the coil's dipoles rotated into each
// placement's frame -- lives in a fixed-size array compiled into the library.
//
// When that array takes device memory: the array belongs to this library's CUDA module. With the
// CUDA runtime's default lazy module loading (CUDA_MODULE_LOADING=LAZY), a device gets the module
// -- the array and the kernel code -- at the first call on that device, not when the library is
// loaded; under CUDA_MODULE_LOADING=EAGER it gets it when the context is created. Either way the
// device holds it until the process exits.
#include <cuda.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/cunibs_b200.h"
#include "internal.hpp"

namespace cunibs {
namespace {

// Room for k * n_dip rotated dipole records; at 48 bytes each this is 768 KiB per GPU.
constexpr std::size_t kNoAllocRecords = CUNIBS_DADT_NOALLOC_MAX_RECORDS;
constexpr std::size_t kNoAllocBytes = kNoAllocRecords * 48;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_dipoles[kNoAllocBytes];

// The array's device address per device, with the id of the context it was looked up in. A context
// id is unique for the life of the process (cuCtxGetId), so a context torn down and made again
// (cudaDeviceReset, or another driver-API context made current) is seen as new and the address is
// looked up again instead of being reused.
struct ScratchSlot {
    unsigned long long ctx_id = 0;
    bool valid = false;
    void* ptr = nullptr;
};

std::mutex g_mu;
ScratchSlot g_slots[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// The current context's id, through the driver entry points the runtime hands out (no link to the
// driver library). Returns false when no context is current on this thread yet.
bool current_context_id(unsigned long long* id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
    });
    if (!get_current || !get_id) fail(kECuda, "cunibs_dadt_noalloc: the driver lacks cuCtxGetCurrent/cuCtxGetId");
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    if (get_id(ctx, id) != CUDA_SUCCESS) fail(kECuda, "cunibs_dadt_noalloc: cuCtxGetId failed");
    return true;
}

// The device address of the scratch array on the current device. In host code the symbol itself is
// only a host-side stand-in, so kernels are handed this address. The lookup (cudaGetSymbolAddress,
// with the device current) is made once per device, and again if that device's context changed.
void* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) fail(kEInval, "device ordinal out of range");
    unsigned long long id = 0;
    const bool bound = current_context_id(&id);
    std::lock_guard<std::mutex> lock(g_mu);
    ScratchSlot& slot = g_slots[device];
    if (bound && slot.valid && slot.ctx_id == id) return slot.ptr;
    void* p = nullptr;
    // With no context current yet, this call is also what makes the runtime bind the device's
    // primary context (and, under lazy loading, load the module holding the array).
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_dipoles);
    if (rc != cudaSuccess) fail(kECuda, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
    if (!bound && !current_context_id(&id)) fail(kECuda, "cunibs_dadt_noalloc: no current CUDA context");
    slot.ptr = p;
    slot.ctx_id = id;
    slot.valid = true;
    return slot.ptr;
}

}  // namespace
}  // namespace cunibs

using namespace cunibs;

extern "C" int cunibs_dadt_noalloc(const double* nodes_mm, int n_nodes, const double* dip_pos_m,
                                   const double* dip_moment, int n_dip, const double* transforms, int k, double didt,
                                   float* out, void* stream) {
    try {
        if (!nodes_mm || !dip_pos_m || !dip_moment || !transforms || !out) fail(kEInval, "NULL argument");
        if (n_nodes < 1 || n_dip < 1 || k < 1) fail(kEInval, "n_nodes, n_dip and k must be positive");
        if (static_cast<std::size_t>(n_dip) * static_cast<std::size_t>(k) > kNoAllocRecords) {
            fail(kEInval, "cunibs_dadt_noalloc: k * n_dip = " + std::to_string(static_cast<long long>(n_dip) * k) +
                              " exceeds the fixed scratch of " + std::to_string(kNoAllocRecords) +
                              " dipole records (CUNIBS_DADT_NOALLOC_MAX_RECORDS); split the placements into "
                              "smaller batches");
        }
        if (packed_dipole_bytes() != 48) fail(kEInternal, "dipole record size changed");
        // An error left by the caller's own earlier work would otherwise be read back below as this
        // call's launch error (and cleared). Report it as what it is and leave it pending.
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess)
            fail(kECuda, std::string("cunibs_dadt_noalloc: a CUDA error from earlier work is pending: ") +
                             cudaGetErrorString(pending));
        int device = 0;
        check(cudaGetDevice(&device), "cudaGetDevice");
        void* scratch = scratch_address(device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // Every record the kernel reads is written first, so nothing needs clearing.
        prep_dipoles(dip_pos_m, dip_moment, n_dip, transforms, k, scratch, s);
        dadt_nodes_raw(nodes_mm, n_nodes, static_cast<const float*>(scratch), n_dip, transforms, k, didt, out, s);
        check(cudaGetLastError(), "dadt launch");
        return CUNIBS_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return CUNIBS_EINTERNAL;
    }
}
