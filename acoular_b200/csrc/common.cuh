// Shared helpers for the acoular_b200 CUDA kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/acoular_b200.h"

namespace acb {

// Record the last CUDA error text for acb_last_cuda_error().
void set_cuda_error(cudaError_t e);

// Limit of one bounded device-side wait of the tensor-core kernels (acb_tc_set_wait_limit_ns).
uint64_t tc_wait_limit_ns();

inline int check_launch()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_cuda_error(e);
        return ACB_ERR_CUDA;
    }
    return ACB_OK;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kNumSMs = 148;

// Distance |g - m| with the contraction order the reference's fastmath dist_mat compiles to:
// sqrt(fma(d2, d2, fma(d1, d1, d0 * d0))) (acoular/environments.py:65-103).
__device__ __forceinline__ double dist3(double g0, double g1, double g2, double m0, double m1, double m2)
{
    const double d0 = __dsub_rn(g0, m0);
    const double d1 = __dsub_rn(g1, m1);
    const double d2 = __dsub_rn(g2, m2);
    return __dsqrt_rn(__fma_rn(d2, d2, __fma_rn(d1, d1, __dmul_rn(d0, d0))));
}

// Look up float32 argument `x` in the sincos exception table (open addressing, linear probing).
// Entry layout: bits 63..32 = float bits of x, bits 15..8 = int8 ulp delta of cos, bits 7..0 =
// int8 ulp delta of sin; an all-ones word marks an empty slot.
__device__ __forceinline__ void sincos_exception(const uint64_t *__restrict__ table, uint64_t mask, float x,
                                                 int &dcos, int &dsin)
{
    const uint32_t key = __float_as_uint(x);
    uint64_t slot = (static_cast<uint64_t>(key) * 0x9E3779B97F4A7C15ull) >> 20;
    dcos = 0;
    dsin = 0;
    for (int probe = 0; probe < 64; ++probe) {  // bounded: the table is built at < 50 % load
        const uint64_t e = __ldg(table + (slot & mask));
        if (e == ~0ull) return;
        if (static_cast<uint32_t>(e >> 32) == key) {
            dcos = static_cast<int8_t>((e >> 8) & 0xff);
            dsin = static_cast<int8_t>(e & 0xff);
            return;
        }
        ++slot;
    }
}

// Float32 cos/sin of a float32 argument: correctly rounded value through FP64 evaluation,
// optionally corrected to the host C library's cosf/sinf by the exception table.  The table holds
// non-negative arguments; a negative one is looked up by its magnitude (the C library's cosf is even
// and its sinf odd, bit for bit, and a delta on the bits of a float changes its magnitude).
__device__ __forceinline__ void sincos_f32_arg(float x, const uint64_t *table, uint64_t mask, bool faithful,
                                               float &c, float &s)
{
    double sd, cd;
    sincos(static_cast<double>(x), &sd, &cd);
    c = __double2float_rn(cd);
    s = __double2float_rn(sd);
    if (faithful) {
        int dc, ds;
        sincos_exception(table, mask, fabsf(x), dc, ds);
        if (dc) c = __int_as_float(__float_as_int(c) + dc);
        if (ds) s = __int_as_float(__float_as_int(s) + ds);
    }
}

}  // namespace acb
