// Shared device/host helpers for the cunibs_b200 CUDA library (sm_100a only).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace cunibs {

// Status codes of the C-ABI (mirrored in include/cunibs_b200.h).
enum Status : int {
    kOk = 0,
    kEInval = 1,
    kENoMem = 2,
    kECuda = 3,
    kENoConv = 4,
    kETimeout = 5,
    kEInternal = 6,
};

// An error that carries its C-ABI status. Every entry point catches these and returns the code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void check(cudaError_t rc, const char* what) {
    if (rc != cudaSuccess) {
        const int code = (rc == cudaErrorMemoryAllocation) ? kENoMem : kECuda;
        fail(code, std::string(what) + ": " + cudaGetErrorString(rc));
    }
}

#define CUNIBS_CHECK(expr) ::cunibs::check((expr), #expr)
#define CUNIBS_LAUNCH_CHECK(what) ::cunibs::check(cudaGetLastError(), what)

// Kernels this process has enqueued through the library (graph replays count their kernel nodes).
inline std::atomic<long long>& launch_counter() {
    static std::atomic<long long> c{0};
    return c;
}
inline void count_launch(long long n = 1) { launch_counter().fetch_add(n, std::memory_order_relaxed); }

constexpr int kWarp = 32;
constexpr int kBlock = 256;

inline unsigned grid_for(std::int64_t n, int per_block = kBlock) {
    if (n <= 0) return 0;
    return static_cast<unsigned>((n + per_block - 1) / per_block);
}

// Device memory for DevArray (devmem.cu): freed blocks are cached per device and size and reused.
// dev_alloc throws Error on failure; dev_free synchronises the block's device before the block can
// be handed out again.
void* dev_alloc(std::size_t bytes);
void dev_free(void* p) noexcept;

// Owning device allocation. Move-only; frees on destruction.
template <typename T>
class DevArray {
  public:
    DevArray() = default;
    explicit DevArray(std::size_t n) { resize(n); }
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevArray& operator=(DevArray&& o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    ~DevArray() { release(); }

    void resize(std::size_t n) {
        if (n == n_ && p_ != nullptr) return;
        release();
        if (n == 0) return;
        p_ = static_cast<T*>(dev_alloc(n * sizeof(T)));
        n_ = n;
    }
    // Grow-only resize: keeps the allocation when it is already large enough.
    void reserve(std::size_t n) {
        if (n > n_) resize(n);
    }
    void release() noexcept {
        if (p_) dev_free(p_);
        p_ = nullptr;
        n_ = 0;
    }
    void upload(const T* host, std::size_t n, cudaStream_t s) {
        resize(n);
        if (n) check(cudaMemcpyAsync(p_, host, n * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    }
    void download(T* host, std::size_t n, cudaStream_t s) const {
        if (n) check(cudaMemcpyAsync(host, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
    }
    std::vector<T> to_host(cudaStream_t s) const {
        std::vector<T> h(n_);
        download(h.data(), n_, s);
        check(cudaStreamSynchronize(s), "to_host sync");
        return h;
    }
    void zero(cudaStream_t s) {
        if (n_) check(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s), "memset");
    }

    T* get() const { return p_; }
    std::size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }

  private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

// Device CSR with int32 indices.
template <typename T>
struct DevCsr {
    int n = 0;
    int ncol = 0;
    long nnz = 0;
    DevArray<int> ptr;
    DevArray<int> col;
    DevArray<T> val;
};

// Fixed-order shuffle reduction into lane 0 of each WIDTH-wide lane group.
template <int WIDTH, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int off = WIDTH / 2; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off, WIDTH);
    return v;
}

}  // namespace cunibs
