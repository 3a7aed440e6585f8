// Zero-block rule of the block-pair products on the GPU (see zskip.cuh): the flag grids
// built from the decoders' per-block flags, the non-finite scan of the decoded operands,
// and the recomputation of the output blocks where the dense product and the reference's
// skipping differ (src/linalg/iarray_gemm.c:146-211: a skipped pair contributes nothing,
// so a NaN or an infinity facing a zero block does not reach C).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "zskip.cuh"

namespace iab {

// Logical block grid [RB][CB] of a container from the decoder's per (chunk, block) flags:
// 1 where the block is skipped (block_is_zeros, or chunk_is_zeros when `use_chunk`).
__global__ void k_zero_grid(Geom g, const uint8_t *__restrict__ zf, int use_chunk, uint8_t *__restrict__ grid)
{
    const int64_t RB = g.cgrid[0] * g.bgrid[0], CB = g.cgrid[1] * g.bgrid[1];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < RB * CB; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ib = t / CB, jb = t - ib * CB;
        const int64_t ic = ib / g.bgrid[0], bi = ib - ic * g.bgrid[0];
        const int64_t jc = jb / g.bgrid[1], bj = jb - jc * g.bgrid[1];
        const uint8_t f = zf[(ic * g.cgrid[1] + jc) * g.nblocks + bi * g.bgrid[1] + bj];
        grid[t] = (f & 1) || (use_chunk && (f & 2)) ? 1 : 0;
    }
}

// flags[rb * CB + cb] = 1 when the block holds a NaN or an infinity (rows x cols dense,
// leading dimension ld; blocks as in zskip.cuh).  `flags` starts zeroed.
template <typename T>
__global__ void k_block_nonfinite(int64_t rows, int64_t cols, const T *__restrict__ x, int64_t ld, int64_t r_chunk,
                                  int64_t r_block, int64_t r_bg, int64_t c_chunk, int64_t c_block, int64_t c_bg,
                                  int64_t CB, uint8_t *__restrict__ flags)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < rows * cols; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / cols, j = t - i * cols;
        if (!isfinite(x[i * ld + j])) {
            int64_t nx;
            const int64_t rb = zs_block_of(i, r_chunk, r_block, r_bg, &nx);
            const int64_t cb = zs_block_of(j, c_chunk, c_block, c_bg, &nx);
            flags[rb * CB + cb] = 1;
        }
    }
}

// One CTA per output block (jb, ib): when some skipped pair of the block faces a
// non-finite partner, the block is recomputed as the sum over its non-skipped pairs
// (in T, as the reference's cblas_dgemm / cblas_sgemm accumulate); other blocks return.
template <typename T>
__global__ void __launch_bounds__(256) k_zero_fix(int64_t M, int64_t N, int64_t K, const T *__restrict__ A, int64_t lda,
                                                  const T *__restrict__ B, int64_t ldb, T *__restrict__ C, int64_t ldc,
                                                  ZeroSkip z, const uint8_t *__restrict__ nfa,
                                                  const uint8_t *__restrict__ nfb)
{
    for (int64_t t = blockIdx.x; t < z.RB * z.JB; t += gridDim.x) {     // block-uniform loop
        const int64_t ib = t / z.JB, jb = t - ib * z.JB;
        int hit = 0;
        for (int64_t kb = threadIdx.x; kb < z.KB; kb += blockDim.x) {
            const bool skip = z.za[ib * z.KB + kb] || z.zb[kb * z.JB + jb];
            const bool nf = nfa[ib * z.KB + kb] || nfb[kb * z.JB + jb];
            hit |= skip && nf;
        }
        if (!__syncthreads_or(hit)) continue;
        int64_t r0, r1, c0, c1;
        zs_block_range(ib, z.r_chunk, z.r_block, z.r_bg, &r0, &r1);
        zs_block_range(jb, z.c_chunk, z.c_block, z.c_bg, &c0, &c1);
        r1 = r1 < M ? r1 : M;
        c1 = c1 < N ? c1 : N;
        if (r0 >= r1 || c0 >= c1) continue;
        const int64_t nc = c1 - c0, cnt = (r1 - r0) * nc;
        for (int64_t e = threadIdx.x; e < cnt; e += blockDim.x) {
            const int64_t i = r0 + e / nc, j = c0 + e % nc;
            T acc = 0;
            for (int64_t kb = 0; kb < z.KB; kb++) {
                if (z.za[ib * z.KB + kb] || z.zb[kb * z.JB + jb]) continue;
                int64_t k0, k1;
                zs_block_range(kb, z.k_chunk, z.k_block, z.k_bg, &k0, &k1);
                k1 = k1 < K ? k1 : K;
                for (int64_t k = k0; k < k1; k++) acc = fma(A[i * lda + k], B[k * ldb + j], acc);
            }
            C[i * ldc + j] = acc;
        }
    }
}

static int grid_of(int64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
}

void zero_grid(const Geom &g, const uint8_t *zf, bool use_chunk, uint8_t *grid, cudaStream_t st)
{
    const int64_t n = g.cgrid[0] * g.bgrid[0] * g.cgrid[1] * g.bgrid[1];
    if (n == 0) return;
    IAB_TIMED("k_zero_grid", st, k_zero_grid<<<grid_of(n), 256, 0, st>>>(g, zf, use_chunk ? 1 : 0, grid));
}

void block_nonfinite(int itemsize, int64_t rows, int64_t cols, const void *x, int64_t ld, int64_t r_chunk,
                     int64_t r_block, int64_t r_bg, int64_t c_chunk, int64_t c_block, int64_t c_bg, int64_t CB,
                     uint8_t *flags, cudaStream_t st)
{
    if (rows * cols == 0) return;
    if (itemsize == 8)
        IAB_TIMED("k_block_nonfinite", st, k_block_nonfinite<double><<<grid_of(rows * cols), 256, 0, st>>>(
            rows, cols, (const double *)x, ld, r_chunk, r_block, r_bg, c_chunk, c_block, c_bg, CB, flags));
    else
        IAB_TIMED("k_block_nonfinite", st, k_block_nonfinite<float><<<grid_of(rows * cols), 256, 0, st>>>(
            rows, cols, (const float *)x, ld, r_chunk, r_block, r_bg, c_chunk, c_block, c_bg, CB, flags));
}

void zero_fix(int itemsize, int64_t M, int64_t N, int64_t K, const void *A, int64_t lda, const void *B, int64_t ldb,
              void *C, int64_t ldc, const ZeroSkip &z, const uint8_t *nfa, const uint8_t *nfb, cudaStream_t st)
{
    if (z.RB == 0 || z.JB == 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::min<int64_t>(z.RB * z.JB, (int64_t)sms * 16);
    if (itemsize == 8)
        IAB_TIMED("k_zero_fix", st, k_zero_fix<double><<<grid, 256, 0, st>>>(M, N, K, (const double *)A, lda,
                                                                            (const double *)B, ldb, (double *)C, ldc,
                                                                            z, nfa, nfb));
    else
        IAB_TIMED("k_zero_fix", st, k_zero_fix<float><<<grid, 256, 0, st>>>(M, N, K, (const float *)A, lda,
                                                                          (const float *)B, ldb, (float *)C, ldc,
                                                                          z, nfa, nfb));
}

}  // namespace iab
