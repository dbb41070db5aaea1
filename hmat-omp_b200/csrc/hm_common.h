// Shared definitions for the B200 hierarchical-matrix library (host + device).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hmat_b200.h"

namespace hm {

// An error with an ABI status code; thrown by host code, converted at the C boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HM_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            (void)cudaGetLastError();                                                      \
            throw ::hm::Error(HM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + \
                                               " at " __FILE__ ":" + std::to_string(__LINE__)); \
        }                                                                                  \
    } while (0)

#define HM_CHECK(cond, code, msg)                                     \
    do {                                                              \
        if (!(cond)) throw ::hm::Error((code), std::string(msg));     \
    } while (0)

// max that propagates NaN (std::max(a, NaN) returns a): a residual norm that is NaN in
// one column must make the whole check fail, not vanish from it.
inline double max_nan(double a, double b) { return (a != a || b != b) ? (a != a ? a : b) : (a < b ? b : a); }

// Device-side status word bits (written by kernels, read by the host after a phase).
enum : int {
    ST_SINGULAR = 1,        // zero / non-finite pivot in an inversion
    ST_NO_CONVERGE = 2,     // Jacobi sweeps hit their limit
    ST_NONFINITE = 4,       // non-finite value met where a finite one is required
    ST_TIMEOUT = 8,         // a kernel's bounded wait on its own pipeline gave up
};

// A typed device allocation with RAII.
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) HM_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void zero(cudaStream_t s) {
        if (n) HM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
};

// Raise a kernel's dynamic shared-memory limit to `bytes` (once per larger request).
template <typename K>
inline void ensure_dyn_smem(K kernel, size_t bytes, size_t& current) {
    if (bytes <= current || bytes <= 48 * 1024) return;
    HM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    current = bytes;
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace hm
