// Zero-block skipping of the block-pair products (iarray_opt_gemm and its variants,
// iarray_opt_gemv): the reference skips the product of a K-block pair when either block
// is a zero block (src/linalg/iarray_gemm.c:17-77, used at :146-168 and :206-211;
// iarray_gemm_a.c:127-146, iarray_gemm_b.c:127-146, iarray_gemv.c:131-164).  The GPU
// product multiplies the decoded operands densely, which gives the same sums except where
// a skipped pair's other block holds a NaN or an infinity (0 x NaN).  So:
//   - the tensor-core kernels leave out every k-tile of an output tile for which all the
//     A blocks under the tile's rows, or all the B blocks under its columns, are zero
//     blocks (an exact saving: those pairs are skipped by the reference too);
//   - afterwards every output block whose row or column meets a skipped pair with a
//     non-finite partner is recomputed with the reference's rule (k_zero_fix).
// Flags are kept on the logical block grid of each operand: block row ib covers rows
// [ic * chunk + bi * block, min(+block, (ic + 1) * chunk)) with ic = ib / bg, bi = ib % bg
// (bg = blocks per chunk along that dimension); blocks past a chunk's edge are empty.
#pragma once
#include <stdint.h>

namespace iab {

struct ZeroSkip {
    const uint8_t *za;     // [RB][KB]: 1 = the pair's A block is skipped
    const uint8_t *zb;     // [KB][JB]: 1 = the pair's B block is skipped
    int64_t r_chunk, r_block, r_bg;   // rows of A (and of C)
    int64_t k_chunk, k_block, k_bg;   // K: columns of A, rows of B
    int64_t c_chunk, c_block, c_bg;   // columns of B (and of C)
    int64_t RB, KB, JB;               // logical block counts
};

// First index past the block that holds coordinate x, and that block's grid index.
__host__ __device__ __forceinline__ int64_t zs_block_of(int64_t x, int64_t chunk, int64_t block, int64_t bg,
                                                        int64_t *next)
{
    const int64_t ic = x / chunk, off = x - ic * chunk, bi = off / block;
    const int64_t end = ic * chunk + ((bi + 1) * block < chunk ? (bi + 1) * block : chunk);
    *next = end;
    return ic * bg + bi;
}

// Start and end of block index ib along one dimension (empty when past the chunk's edge).
__host__ __device__ __forceinline__ void zs_block_range(int64_t ib, int64_t chunk, int64_t block, int64_t bg,
                                                        int64_t *lo, int64_t *hi)
{
    const int64_t ic = ib / bg, bi = ib - ic * bg;
    const int64_t s = bi * block;
    *lo = ic * chunk + (s < chunk ? s : chunk);
    *hi = ic * chunk + (s + block < chunk ? s + block : chunk);
}

// All A blocks under rows [r0, r1) at K block kb are skipped.
__device__ __forceinline__ bool zs_rows_zero(const ZeroSkip &z, int64_t r0, int64_t r1, int64_t kb)
{
    for (int64_t r = r0; r < r1;) {
        int64_t nx;
        const int64_t ib = zs_block_of(r, z.r_chunk, z.r_block, z.r_bg, &nx);
        if (!z.za[ib * z.KB + kb]) return false;
        r = nx;
    }
    return true;
}

__device__ __forceinline__ bool zs_cols_zero(const ZeroSkip &z, int64_t c0, int64_t c1, int64_t kb)
{
    for (int64_t c = c0; c < c1;) {
        int64_t nx;
        const int64_t jb = zs_block_of(c, z.c_chunk, z.c_block, z.c_bg, &nx);
        if (!z.zb[kb * z.JB + jb]) return false;
        c = nx;
    }
    return true;
}

// Whether the output tile rows [r0, r1) x columns [c0, c1) needs K range [k0, k1): some
// K block of the range has a non-skipped A block under the rows and a non-skipped B
// block under the columns.  (Ranges are clipped to the matrices by the caller.)
__device__ __forceinline__ bool zs_tile_active(const ZeroSkip &z, int64_t r0, int64_t r1, int64_t c0, int64_t c1,
                                               int64_t k0, int64_t k1)
{
    if (r0 >= r1 || c0 >= c1 || k0 >= k1) return false;
    for (int64_t k = k0; k < k1;) {
        int64_t nx;
        const int64_t kb = zs_block_of(k, z.k_chunk, z.k_block, z.k_bg, &nx);
        if (!zs_rows_zero(z, r0, r1, kb) && !zs_cols_zero(z, c0, c1, kb)) return true;
        k = nx;
    }
    return false;
}

}  // namespace iab
