// Device self-checks exported through the C ABI.
//   lgcr_selftest_reciprocal: rcpAtLeastOne (the guided taps' reciprocal of
//   1 + non-negative terms) against the IEEE quotient 1.0f / x for every
//   float x in [1, +inf] (2^30 + 1 arguments: the fast range [1, 2^64) and
//   the IEEE-division range above it), bit for bit.
#include "impl.h"
#include "recon.cuh"

using namespace lgcr_b200;

namespace {

__global__ void k_check_reciprocal(uint32_t lo, uint32_t hi, unsigned long long *bad) {
    unsigned long long local = 0;
    for (uint64_t b = lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b <= hi;
         b += (uint64_t)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((uint32_t)b);
        if (__float_as_uint(rcpAtLeastOne(x)) != __float_as_uint(1.0f / x))
            ++local;
    }
    if (local)
        atomicAdd(bad, local);
}

} // namespace

extern "C" int lgcr_selftest_reciprocal(uint64_t *mismatches) {
    if (!mismatches)
        return LGCR_E_ARGUMENT;
    unsigned long long *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_selftest_reciprocal");
    unsigned long long h = 0;
    e = cudaMemset(d, 0, sizeof(h));
    if (e == cudaSuccess) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_check_reciprocal<<<sms * 8, 256>>>(0x3f800000u, 0x7f800000u, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_selftest_reciprocal");
    *mismatches = h;
    return LGCR_OK;
}
