// dA/dt at mesh nodes without any device allocation by the library.
//
// Some callers cannot let a library allocate GPU memory: a process whose device memory is already
// reserved in full by another framework's caching allocator (a cudaMalloc from here would fail, or
// would fragment the caller's budget), or code that has to stay on a fixed, audited memory budget
// set up front. This entry point serves them: the caller passes every input and output in device
// memory, and the only scratch the computation needs -- the coil's dipoles rotated into each
// placement's frame -- lives in a fixed-size array compiled into the library, which every GPU that
// loads the library holds from load to process exit.
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

std::mutex g_mu;
void* g_scratch[kMaxDevices] = {};

// The device address of the scratch array on the current device, looked up once per device. In
// host code the symbol itself is only a host-side stand-in, so kernels are handed this address.
void* scratch_address(int device) {
    if (device < 0 || device >= kMaxDevices) fail(kEInval, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_scratch[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_dipoles);
        if (rc != cudaSuccess) fail(kECuda, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
        g_scratch[device] = p;
    }
    return g_scratch[device];
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
