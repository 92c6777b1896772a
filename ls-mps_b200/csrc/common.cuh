// Shared device/host definitions of the LS-MPS sm_100a library: the context, grow-only
// device buffers, error plumbing and small device helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <utility>

#include "lsmps_gpu.h"

namespace lsmps_gpu {

constexpr int K = 9;  // second-order WLS basis size in 3-D

// ---- status plumbing -----------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define LSMPS_CUDA(call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::lsmps_gpu::Error{LSMPS_ERR_CUDA, std::string(#call) + ": " +              \
                                                         cudaGetErrorString(e_)};             \
    } while (0)

// Kernel launches issued by this library (graph replays add their kernel nodes).
void note_launches(uint64_t n);

#define LSMPS_CHECK_LAUNCH()                   \
    do {                                       \
        LSMPS_CUDA(cudaGetLastError());        \
        ::lsmps_gpu::note_launches(1);         \
    } while (0)

#define LSMPS_REQUIRE(cond, code, text)                         \
    do {                                                        \
        if (!(cond)) throw ::lsmps_gpu::Error{(code), (text)};  \
    } while (0)

// ---- grow-only device buffer --------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T>
    T* get() const { return static_cast<T*>(p); }
    template <class T>
    T* ensure(size_t count) {
        size_t need = count * sizeof(T);
        if (need == 0) need = sizeof(T);
        if (need > bytes) {
            if (p) cudaFree(p);
            p = nullptr;
            bytes = 0;
            size_t cap = need + need / 8;  // headroom so a growing step series re-allocates rarely
            cudaError_t e = cudaMalloc(&p, cap);
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Error{LSMPS_ERR_ALLOC, "cudaMalloc of " + std::to_string(cap) + " bytes: " +
                                                 cudaGetErrorString(e)};
            }
            bytes = cap;
        }
        return static_cast<T*>(p);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// ---- device error flags (bounded waits and device-side checks set these) ------------
enum DeviceFlag : int {
    DFLAG_NONFINITE = 1,
    DFLAG_TIMEOUT = 2,
    DFLAG_CELL_OVERFLOW = 4,
    DFLAG_INDEX = 8,
    DFLAG_STENCIL = 16,  // a PPE coupling spans more than one neighbor-grid cell (multigrid setup)
};

// ---- small device helpers ------------------------------------------------------------
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Exactly rounded FP64 operations that the compiler may not contract into FMAs; used
// wherever results must equal the reference's x86-64 (non-FMA) arithmetic bit for bit.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// |d|^2 as the reference's n2 (src/lsmps.cpp:21): (x*x + y*y) + z*z, no contraction.
__device__ __forceinline__ double xnorm2(double dx, double dy, double dz) {
    return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// weight (src/lsmps.cpp:22): (re/r - 1)^2 for 1e-12 < r < re, else 0; exact ops.
__device__ __forceinline__ double xweight(double r, double re) {
    if (r <= 1e-12 || r >= re) return 0.0;
    double q = xsub(xdiv(re, r), 1.0);
    return xmul(q, q);
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Programmatic dependent launch (sm_90+): a kernel launched with launch_pdl may start while
// the kernel before it in the stream drains. It calls pdl_begin() first: that waits until the
// previous kernel has completed and its writes are visible, then lets the next PDL kernel
// launch once every block of this one has passed the wait. So at most one grid waits ahead of
// the running one. Triggering before the wait let a whole chain of dependent grids launch
// ahead and hold SM slots while the running kernel still worked, and the grids that then found
// their slots late ran unevenly spread over the SMs (measured on the multigrid BiCGStab at 1M:
// 12.8 ms per solve against 10.1 ms with the wait first, 10.8 ms without PDL). Launched
// without the attribute, both instructions return at once.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LSMPS_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

inline unsigned blocks_for(size_t n, unsigned threads) {
    return (unsigned)((n + threads - 1) / threads);
}

}  // namespace lsmps_gpu
