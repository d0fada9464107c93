// Self-check of the two-cell pass's division (mpdata_check_division): the
// round-to-nearest division without a slow-path call (div_nearest,
// common.cuh) against IEEE division (__fdiv_rn) on seeded random operands of
// the ranges the pass divides: divisors in [FLT_MIN, 2^100), numerators of
// either sign from 0 and subnormals up to 2^100.
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "mpdata_b200.h"
#include "solver.h"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

__global__ void k_check_division(long long n, unsigned long long seed, unsigned long long* bad)
{
    unsigned long long local = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const uint64_t h1 = mix64(seed ^ (uint64_t)t * 0x9e3779b97f4a7c15ULL);
        const uint64_t h2 = mix64(h1 + 0x632be59bd9b4e019ULL);
        // divisor: exponent field 1 .. 226 (FLT_MIN .. 2^100), any mantissa
        const uint32_t eb = 1 + (uint32_t)(h1 % 226);
        const float b = __uint_as_float((eb << 23) | (uint32_t)(h1 >> 40 & 0x7fffff));
        // numerator: exponent field 0 .. 226 (zero and subnormals included), any sign
        const uint32_t ea = (uint32_t)(h2 % 227);
        uint32_t abits = (ea << 23) | (uint32_t)(h2 >> 40 & 0x7fffff);
        if ((h2 >> 20 & 0xff) == 0) abits = 0;  // exact zeros, 1 in 256
        const float a = __uint_as_float(abits | (uint32_t)(h2 >> 63) << 31);
        const float q = mpd::div_nearest(a, b), ref = __fdiv_rn(a, b);
        const float qc = mpd::div_nearest<true>(fabsf(a), b), refc = fminf(__fdiv_rn(fabsf(a), b), 1.0f);
        if (__float_as_uint(q) != __float_as_uint(ref)) local++;
        if (__float_as_uint(qc) != __float_as_uint(refc)) local++;
    }
    if (local) atomicAdd(bad, local);
}

}  // namespace

extern "C" int mpdata_check_division(long long n, unsigned long long seed, long long* mismatches)
{
    if (n < 0 || !mismatches) return mpd::fail(MPDATA_ERR_ARG, "bad arguments");
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess)
        return mpd::fail(MPDATA_ERR_NOMEM, "check_division: device allocation failed");
    unsigned long long h = 0;
    cudaError_t e = cudaMemset(d, 0, sizeof(*d));
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        k_check_division<<<sms * 8, 256>>>(n, seed, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess)
        return mpd::fail(MPDATA_ERR_CUDA, "check_division: %s", cudaGetErrorString(e));
    *mismatches = (long long)h;
    return 0;
}
