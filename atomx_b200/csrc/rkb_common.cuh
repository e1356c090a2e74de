// Shared device helpers and host-side status plumbing for the rkb200 library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../include/rkb200.h"

namespace rkb {

// ------------------------------------------------------------------ host side
void set_error(const char *fmt, ...);
int cuda_status(cudaError_t err, const char *what);

#define RKB_CHECK_ARG(cond, ...)                      \
    do {                                              \
        if (!(cond)) {                                \
            ::rkb::set_error(__VA_ARGS__);            \
            return RKB_EINVAL;                        \
        }                                             \
    } while (0)

#define RKB_CUDA(call)                                                     \
    do {                                                                   \
        cudaError_t e__ = (call);                                          \
        if (e__ != cudaSuccess) return ::rkb::cuda_status(e__, #call);     \
    } while (0)

#define RKB_LAUNCHED(what)                                                 \
    do {                                                                   \
        cudaError_t e__ = cudaGetLastError();                              \
        if (e__ != cudaSuccess) return ::rkb::cuda_status(e__, what);      \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline long ceil_div(long a, long b) { return (a + b - 1) / b; }

// Number of SMs on the current device (cached per device).
int sm_count();

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device,
// size): later launches (e.g. while a stream is being captured into a CUDA
// graph) make no attribute call.
cudaError_t set_smem_once(const void *func, int bytes);
template <class F>
inline cudaError_t set_smem(F *func, int bytes) { return set_smem_once(reinterpret_cast<const void *>(func), bytes); }

// ---------------------------------------------------------------- device side
// x^n for integer n by square-and-multiply, negative n as 1/x^|n|: the same
// operation sequence Numba emits for float**int, so powers agree bit for bit
// with the reference's r**k and r**(-(k+1)).
__device__ __forceinline__ double int_pow(double x, int n) {
    bool inv = n < 0;
    unsigned e = inv ? (unsigned)(-n) : (unsigned)n;
    double r = 1.0, a = x;
    while (e != 0u) {
        if (e & 1u) r = __dmul_rn(r, a);
        e >>= 1;
        a = __dmul_rn(a, a);
    }
    return inv ? __ddiv_rn(1.0, r) : r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Inclusive prefix sum over the 32 lanes.
__device__ __forceinline__ double warp_inclusive_scan(double v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = __dadd_rn(v, t);
    }
    return v;
}

}  // namespace rkb
