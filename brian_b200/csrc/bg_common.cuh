// bg_common.cuh -- shared device/host helpers for the brian_b200 engine.
#pragma once
#ifdef __CUDACC_RTC__
// compiled at run time by NVRTC (generated network models): no host headers
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
typedef unsigned long long uintptr_t;
#else
#include <cstdint>
#include <cuda_runtime.h>
#endif

#define BG_OK 0
#define BG_EINVAL (-1)
#define BG_ENOMEM (-2)
#define BG_ECUDA (-3)
#define BG_ETIMEOUT (-4)
#define BG_ENUMERIC (-5)
#define BG_ESTATE (-6)
#define BG_ENOSYS (-7)
#define BG_ECOMPILE (-8)

#ifndef __CUDACC_RTC__
// Records the calling thread's error message for bg_last_error (library
// internal; defined in bg_net.cu).
int bg_internal_fail(int code, const char *msg);
#endif

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).  One 4x32 block per
// (seed, clock step, neuron index): the Poisson source of PoissonGroup
// (threshold.py:461-471) becomes a pure function of its coordinates, so the
// CPU restatement and the device draw the same numbers.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void bg_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// Uniform double in [0,1) built from 53 random bits (27 from word 0, 26 from
// word 1): exact in binary64.
__host__ __device__ __forceinline__ double bg_philox_uniform(uint64_t seed, int64_t step, int64_t i) {
    uint32_t c[4] = {(uint32_t)step, (uint32_t)((uint64_t)step >> 32), (uint32_t)i,
                     (uint32_t)((uint64_t)i >> 32)};
    bg_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = c[0] >> 5, b = c[1] >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
}

// Two uniform floats in [0,1) with 24 random bits each (PSO draws).
__host__ __device__ __forceinline__ void bg_philox_uniform2f(uint64_t seed, uint64_t ctr_hi, uint64_t ctr_lo,
                                                            float *u0, float *u1) {
    uint32_t c[4] = {(uint32_t)ctr_lo, (uint32_t)(ctr_lo >> 32), (uint32_t)ctr_hi, (uint32_t)(ctr_hi >> 32)};
    bg_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    *u0 = (float)(c[0] >> 8) * (1.0f / 16777216.0f);
    *u1 = (float)(c[1] >> 8) * (1.0f / 16777216.0f);
}

// Exactly-rounded arithmetic without contraction, spelled out so that no
// compiler flag can fuse a multiply into an add on the bit-exact path.
template <typename T> struct rn;
template <> struct rn<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
};
template <> struct rn<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
};

// Per-network control block in device memory.  Kernels of one step all read
// `nstep`; the last kernel of the step advances it (last-arriving block), so
// a captured CUDA graph of many steps needs no host-side parameter update.
struct DevCtl {
    long long nstep;       // steps executed since the network was prepared
    long long clock_off;   // clock step = nstep + clock_off
    unsigned int done;     // arrival counter of the step's last kernel
    int err;               // first error code raised on the device (0 = none)
    long long err_info;    // detail for err
};

#define BG_DERR_MONITOR_OVERFLOW 1
#define BG_DERR_RANGE 2
#define BG_DERR_TIMEOUT 3      // a bounded inter-block wait gave up
#define BG_DERR_NONFINITE 4    // a state variable is NaN or infinite (finite-state check)

// Spin limit of inter-block waits: about a second of polling.
#define BG_SPIN_LIMIT (1u << 22)

__device__ __forceinline__ void bg_finish_step(DevCtl *ctl, int last) {
    if (!last) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
        const unsigned int prev = atomicAdd(&ctl->done, 1u);
        if (prev == nb - 1) {
            ctl->done = 0;
            __threadfence();
            ctl->nstep = ctl->nstep + 1;
        }
    }
}

__device__ __forceinline__ void bg_raise(DevCtl *ctl, int code, long long info) {
    if (atomicCAS(&ctl->err, 0, code) == 0) ctl->err_info = info;
}
