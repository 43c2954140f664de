// Device helpers shared by the count pass (sj_join.cu) and the emission pass
// (sj_emit.cu): the warp bit-matrix transpose and the candidate-validity masks
// of a block of 32 stream positions.  Both passes must agree bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sjdev {

__device__ __forceinline__ uint32_t transpose32(uint32_t x, uint32_t lane)
{
    // Lane i holds row i of a 32x32 bit matrix; afterwards lane j holds column j.
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t lo = (s == 16) ? 0x0000ffffu
                          : (s == 8)  ? 0x00ff00ffu
                          : (s == 4)  ? 0x0f0f0f0fu
                          : (s == 2)  ? 0x33333333u
                                      : 0x55555555u;
        uint32_t y = __shfl_xor_sync(0xffffffffu, x, s);
        if (lane & s) x = (x & ~lo) | ((y & ~lo) >> s);
        else x = (x & lo) | ((y & lo) << s);
    }
    return x;
}

// Candidate-validity masks of a block of 32 stream positions starting at blk.
// Inside a symmetric home segment (stream positions < homeEnd are the home
// cell's points from the query tile's first point on) a query keeps candidates
// at or after itself; the mirrored direction drops the query itself.
__device__ __forceinline__ uint32_t home_bits(uint32_t blk, uint32_t homeEnd, bool sym)
{
    if (!sym || blk >= homeEnd) return 0u;
    const uint32_t hn = homeEnd - blk;
    return hn >= 32 ? 0xffffffffu : ((1u << hn) - 1u);
}

__device__ __forceinline__ uint32_t row_keep(uint32_t qi, uint32_t blk, uint32_t hb)
{
    const int lo = (int)qi - (int)blk;   // home candidate index >= query index
    const uint32_t ge = lo <= 0 ? 0xffffffffu : (lo >= 32 ? 0u : (0xffffffffu << lo));
    return ~hb | (hb & ge);
}

__device__ __forceinline__ uint32_t mir_keep(uint32_t qi, uint32_t blk, uint32_t hb)
{
    const int lo = (int)qi - (int)blk;
    return (lo >= 0 && lo < 32) ? ~(hb & (1u << lo)) : 0xffffffffu;
}

}  // namespace sjdev
