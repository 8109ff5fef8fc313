// microbench.cuh -- measured integer peaks of this GPU for the roofline.
//
// The driver's measured-peak file holds HBM and bf16 tensor peaks only; this
// path is integer-ALU bound, so its denominators are measured here:
//  kind 0: "plane-word tests" per second -- the filter's elemental operation,
//          one funnel shift plus one three-input logic op (xor-and-not) on
//          32-bit words, 8 independent chains per thread, all SMs;
//  kind 1: 32-bit Montgomery products per second (4 integer multiplies each),
//          8 independent chains per thread.
#pragma once
#include "common.cuh"

namespace cz {

__global__ void mb_alu_kernel(u32 iters, u32 seed, u32 *sink) {
    u32 x[8], acc[8];
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; ++i) { x[i] = seed * (t + 7u * i) + i; acc[i] = ~0u; }
    const u32 y = seed ^ t;
    for (u32 it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const u32 w = __funnelshift_r(x[i], y, it + i);
            acc[i] &= ~(w ^ x[(i + 1) & 7]);
            x[i] = w;
        }
    }
    u32 r = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r ^= acc[i] ^ x[i];
    if (r == 0x12345678u) sink[0] = r;
}

__global__ void mb_mont_kernel(u32 iters, u32 p, u32 ninv, u32 *sink) {
    u32 v[8];
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (t * 2654435761u + 97u * i) % p;
    for (u32 it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = mmul(v[i], v[i], p, ninv);
    }
    u32 r = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) r ^= v[i];
    if (r == 0x12345678u) sink[0] = r;
}

}  // namespace cz
