// Device memory behind DevArray: blocks the library frees are kept per device and size and handed
// out again, instead of going back to the driver.
//
// Measured on this build's B200 boxes: cudaMalloc and cudaFree usually take well under a millisecond,
// but now and then one takes 100-400 ms (a 88 MB cudaMalloc 420 ms, a cudaFree 96 ms, in 60 pairs of
// each). The calls that build their workspace anew every time (an adjoint solve of the auxiliary
// dipole method: 7.5-238 ms over ten identical calls; a conductivity study's begin; a reciprocity
// field sampling) inherited those stalls. With freed blocks reused, a repeated call allocates from
// the cache.
//
// A freed block is reused only once the work queued on its device has finished: dev_free
// synchronises the device first, which is what cudaFree's own implicit synchronisation guaranteed.
// Sizes are rounded up (512 bytes below 1 MiB, 2 MiB above) so that nearly equal requests share a
// bucket. At most kCacheCap bytes are kept idle; past that, and whenever a cudaMalloc runs out of
// memory (the cache is emptied and the allocation retried), blocks go back to the driver.
#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.cuh"

namespace cunibs {
namespace {

constexpr std::size_t kSmallQuantum = 512;
constexpr std::size_t kLargeQuantum = std::size_t{2} << 20;
constexpr std::size_t kLargeFrom = std::size_t{1} << 20;
constexpr std::size_t kCacheCap = std::size_t{8} << 30;

struct Pool {
    std::mutex mu;
    std::unordered_map<void*, std::pair<int, std::size_t>> live;           // block -> (device, bytes)
    std::map<std::pair<int, std::size_t>, std::vector<void*>> idle;        // (device, bytes) -> blocks
    std::size_t idle_bytes = 0;
};

// Never destroyed: blocks still cached at exit go back with the process.
Pool& pool() {
    static Pool* p = new Pool();
    return *p;
}

std::size_t rounded(std::size_t bytes) {
    const std::size_t q = bytes >= kLargeFrom ? kLargeQuantum : kSmallQuantum;
    return (bytes + q - 1) / q * q;
}

// Returns every idle block of `device` to the driver (the pool's lock held).
void drop_idle(Pool& P, int device) {
    for (auto it = P.idle.begin(); it != P.idle.end();) {
        if (it->first.first == device) {
            for (void* b : it->second) {
                cudaFree(b);
                P.idle_bytes -= it->first.second;
            }
            it = P.idle.erase(it);
        } else {
            ++it;
        }
    }
}

}  // namespace

void* dev_alloc(std::size_t bytes) {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    const std::size_t rb = rounded(bytes ? bytes : 1);
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> lock(P.mu);
        auto it = P.idle.find({device, rb});
        if (it != P.idle.end() && !it->second.empty()) {
            void* b = it->second.back();
            it->second.pop_back();
            P.idle_bytes -= rb;
            P.live[b] = {device, rb};
            return b;
        }
    }
    void* b = nullptr;
    cudaError_t rc = cudaMalloc(&b, rb);
    if (rc == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        std::lock_guard<std::mutex> lock(P.mu);
        drop_idle(P, device);
        rc = cudaMalloc(&b, rb);
    }
    check(rc, "cudaMalloc");
    std::lock_guard<std::mutex> lock(P.mu);
    P.live[b] = {device, rb};
    return b;
}

void dev_free(void* b) noexcept {
    if (b == nullptr) return;
    Pool& P = pool();
    std::pair<int, std::size_t> info;
    {
        std::lock_guard<std::mutex> lock(P.mu);
        auto it = P.live.find(b);
        if (it == P.live.end()) {
            cudaFree(b);
            return;
        }
        info = it->second;
        P.live.erase(it);
    }
    int current = 0;
    const bool other = cudaGetDevice(&current) == cudaSuccess && current != info.first;
    if (other) cudaSetDevice(info.first);
    const cudaError_t sync = cudaDeviceSynchronize();
    std::lock_guard<std::mutex> lock(P.mu);
    if (sync != cudaSuccess || P.idle_bytes + info.second > kCacheCap) {
        cudaFree(b);
    } else {
        P.idle[{info.first, info.second}].push_back(b);
        P.idle_bytes += info.second;
    }
    if (other) cudaSetDevice(current);
}

}  // namespace cunibs
