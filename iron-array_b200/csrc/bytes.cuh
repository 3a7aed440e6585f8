// Byte-plane helpers shared by the codec and the split product's reconstruction (which can
// write its output straight into the encoder's shuffled block image).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace iab {

// 4x4 byte transpose: o_i holds byte i of a, b, c, d (in that order).
__device__ __forceinline__ void transpose4x4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t &o0, uint32_t &o1,
                                             uint32_t &o2, uint32_t &o3)
{
    const uint32_t ab_lo = __byte_perm(a, b, 0x5140), ab_hi = __byte_perm(a, b, 0x7362);
    const uint32_t cd_lo = __byte_perm(c, d, 0x5140), cd_hi = __byte_perm(c, d, 0x7362);
    o0 = __byte_perm(ab_lo, cd_lo, 0x5410);
    o1 = __byte_perm(ab_lo, cd_lo, 0x7632);
    o2 = __byte_perm(ab_hi, cd_hi, 0x5410);
    o3 = __byte_perm(ab_hi, cd_hi, 0x7632);
}

}  // namespace iab
