// Native products on decoded operands.
//
// Replaces the MKL calls of ironArray's matmul path: cblas_dgemm / cblas_sgemm of the
// block-pair path (src/linalg/iarray_gemm.c:276-290, iarray_gemm_a.c:160-176) and the
// panel path (src/linalg/matmul/gemm.c:97-101), cblas_dgemv / cblas_sgemv
// (src/linalg/iarray_gemv.c:211-228, src/linalg/matmul/gemv.c:93-97).  Operands were
// decoded once into dense row-major arrays, so one launch covers every block pair
// (sum over K blocks of A_blk * B_blk == the dense product over the padded extents,
// because Caterva's padding is zero).
//
// FP64: DMMA tensor-core tiles (mma.sync m16n8k16 .f64), 128x128x32 CTA tile,
//       8 warps (64x32 each), 3-stage cp.async pipeline with zero-filled edges.
// FP32: FFMA SIMT tiles, 128x128x8, 8x8 outer product per thread, double buffer.
// GEMV: one warp per row, 16-byte loads.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "zskip.cuh"

namespace iab {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Copies `bytes` (0, 8 or 16) from global memory into a 16-byte shared slot; the rest of the
// slot is zero-filled, so nothing past a matrix edge is read.
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(sdst)), "l"(gsrc), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ============================================================================ FP64 DMMA
namespace f64k {
constexpr int STAGES = 3;
// BK: k-depth of a pipeline stage (16 or 32; the single product uses 32, the grouped
// autotuner tries both).  Row strides are 4 mod 16 doubles: conflict-free fragments.
template <int BM, int BN, int BK> struct Cfg {
    static constexpr int SA = BK + 4, SB = BN + 4;
    static constexpr int A_STAGE = BM * SA, B_STAGE = BK * SB;
    static constexpr int SMEM = STAGES * (A_STAGE + B_STAGE) * 8;
    static constexpr int MI = BM / 32, NJ = BN / 32;     // 2 x 4 warps, warp tile (BM/2) x (BN/4)
};
constexpr int BK_SINGLE = 32;
}

// D += A B for one 16x8 tile over k = 16 (a: rows g, g + 8 at columns q + 4u; b: rows q + 4u
// at column g).  The products are summed in k order, as sixteen m16n8k1 steps would.
__device__ __forceinline__ void dmma_16x8x16(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
          "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// One BM x BN tile of C = A B at (m0, n0), 256 threads.  Requires lda, ldb even and
// 16-byte aligned bases (true for the library's dense buffers).  With `klist`, only the
// nk k-tiles it lists (ascending) are multiplied: the others are pairs of zero blocks the
// block-pair product skips; without it, all k-tiles.
template <int BM, int BN, int BK>
__device__ __forceinline__ void f64_tile(int M, int N, int K, const double *__restrict__ A, int64_t lda,
                                         const double *__restrict__ B, int64_t ldb, double *__restrict__ C,
                                         int64_t ldc, int m0, int n0, double *smf64, const uint16_t *klist = nullptr,
                                         int nk = -1)
{
    using namespace f64k;
    using G = Cfg<BM, BN, BK>;
    constexpr int SA = G::SA;
    double *sA = smf64, *sB = smf64 + STAGES * G::A_STAGE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int ktiles = klist ? nk : (K + BK - 1) / BK;
    auto kt_of = [&](int li) { return klist ? (int)klist[li] : li; };

    auto load_tile = [&](int kt, int s) {
        const int k0 = kt * BK;
        double *a = sA + s * G::A_STAGE, *b = sB + s * G::B_STAGE;
#pragma unroll
        for (int i = 0; i < BM * BK / 512; i++) {      // A: BM rows x BK/2 16-byte pieces
            const int idx = tid + i * 256, r = idx / (BK / 2), cpc = (idx % (BK / 2)) * 2;
            const int gr = m0 + r, gk = k0 + cpc;
            // the two doubles at gk, gk + 1 that lie inside the row (K may be odd: the padding
            // column after it is never read, it may hold anything)
            const int nb = gr < M ? 8 * max(0, min(2, K - gk)) : 0;
            cp_async16(a + r * SA + cpc, nb ? (const void *)(A + (int64_t)gr * lda + gk) : (const void *)A, nb);
        }
#pragma unroll
        for (int i = 0; i < BN * BK / 512; i++) {      // B: BK rows x BN/2 pieces
            const int idx = tid + i * 256, r = idx / (BN / 2), cpc = (idx % (BN / 2)) * 2;
            const int gk = k0 + r, gn = n0 + cpc;
            const int nb = gk < K ? 8 * max(0, min(2, N - gn)) : 0;
            cp_async16(b + r * G::SB + cpc, nb ? (const void *)(B + (int64_t)gk * ldb + gn) : (const void *)B, nb);
        }
    };

    double acc[G::MI][G::NJ][4];
#pragma unroll
    for (int i = 0; i < G::MI; i++)
#pragma unroll
        for (int j = 0; j < G::NJ; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < ktiles) load_tile(kt_of(s), s);
        cp_async_commit();
    }
    const int g = lane >> 2, q = lane & 3;
    for (int kt = 0; kt < ktiles; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nxt = kt + STAGES - 1;
        if (nxt < ktiles) load_tile(kt_of(nxt), nxt % STAGES);
        cp_async_commit();
        const double *a = sA + (kt % STAGES) * G::A_STAGE + (wm * (BM / 2)) * SA;
        const double *b = sB + (kt % STAGES) * G::B_STAGE + wn * (BN / 4);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            double bf[G::NJ][4];
#pragma unroll
            for (int j = 0; j < G::NJ; j++)
#pragma unroll
                for (int u = 0; u < 4; u++) bf[j][u] = b[(kk + q + 4 * u) * G::SB + j * 8 + g];
#pragma unroll
            for (int i = 0; i < G::MI; i++) {
                double af[8];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    af[2 * u] = a[(i * 16 + g) * SA + kk + q + 4 * u];
                    af[2 * u + 1] = a[(i * 16 + g + 8) * SA + kk + q + 4 * u];
                }
#pragma unroll
                for (int j = 0; j < G::NJ; j++) dmma_16x8x16(acc[i][j], af, bf[j]);
            }
        }
    }
    cp_async_wait<0>();
    // epilogue: fragment rows g, g+8; cols 2q, 2q+1
#pragma unroll
    for (int i = 0; i < G::MI; i++)
#pragma unroll
        for (int j = 0; j < G::NJ; j++) {
            const int r0 = m0 + wm * (BM / 2) + i * 16 + g, c0 = n0 + wn * (BN / 4) + j * 8 + 2 * q;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = r0 + h * 8;
                if (r >= M) continue;
                double *cp = C + (int64_t)r * ldc + c0;
                if (c0 + 1 < N) {
                    *reinterpret_cast<double2 *>(cp) = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
                } else if (c0 < N) {
                    cp[0] = acc[i][j][2 * h];
                }
            }
        }
}

__global__ void __launch_bounds__(256) k_gemm_f64(int M, int N, int K, const double *__restrict__ A, int64_t lda,
                                                  const double *__restrict__ B, int64_t ldb, double *__restrict__ C,
                                                  int64_t ldc)
{
    extern __shared__ __align__(16) double smf64[];
    f64_tile<128, 128, f64k::BK_SINGLE>(M, N, K, A, lda, B, ldb, C, ldc, blockIdx.y * 128, blockIdx.x * 128, smf64);
}

// The same product where the K ranges of zero-block pairs are left out: each CTA lists the
// k-tiles its tile needs (zs_tile_active) in shared memory, compacted by warp ballots, and
// multiplies only those.  K <= ZS_MAX_K.
constexpr int ZS_MAX_K = 65536;
constexpr int ZS_LIST_BYTES = (ZS_MAX_K / f64k::BK_SINGLE) * 3 + 64;    // flags + uint16 list + count
__global__ void __launch_bounds__(256) k_gemm_f64_skip(int M, int N, int K, const double *__restrict__ A, int64_t lda,
                                                       const double *__restrict__ B, int64_t ldb, double *__restrict__ C,
                                                       int64_t ldc, ZeroSkip z)
{
    constexpr int BK = f64k::BK_SINGLE;
    using G = f64k::Cfg<128, 128, BK>;
    extern __shared__ __align__(16) double smf64[];
    uint8_t *extra = reinterpret_cast<uint8_t *>(smf64 + f64k::STAGES * (G::A_STAGE + G::B_STAGE));
    const int ktiles = (K + BK - 1) / BK;
    int *count = reinterpret_cast<int *>(extra);
    uint16_t *list = reinterpret_cast<uint16_t *>(extra + 16);
    uint8_t *flag = extra + 16 + 2 * ktiles;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * 128;
    const int64_t r1 = min(m0 + 128, M), c1 = min(n0 + 128, N);
    for (int kt = threadIdx.x; kt < ktiles; kt += blockDim.x)
        flag[kt] = zs_tile_active(z, m0, r1, n0, c1, (int64_t)kt * BK, min((kt + 1) * BK, K)) ? 1 : 0;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int c = 0;
        for (int base = 0; base < ktiles; base += 32) {
            const bool f = base + lane < ktiles && flag[base + lane];
            const unsigned m = __ballot_sync(0xffffffffu, f);
            if (f) list[c + __popc(m & ((1u << lane) - 1))] = (uint16_t)(base + lane);
            c += __popc(m);
        }
        if (lane == 0) *count = c;
    }
    __syncthreads();
    f64_tile<128, 128, BK>(M, N, K, A, lda, B, ldb, C, ldc, m0, n0, smf64, list, *count);
}

void gemm_f64_native(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
                     double *C, int64_t ldc, cudaStream_t st, const ZeroSkip *zs)
{
    using G = f64k::Cfg<128, 128, f64k::BK_SINGLE>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        cudaFuncSetAttribute(k_gemm_f64_skip, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM + ZS_LIST_BYTES);
        attr = true;
    }
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)((M + 127) / 128));
    if (zs && K <= ZS_MAX_K) {
        const int ktiles = (int)((K + f64k::BK_SINGLE - 1) / f64k::BK_SINGLE);
        const int smem = G::SMEM + 3 * ktiles + 64;
        IAB_TIMED("k_gemm_f64", st, k_gemm_f64_skip<<<grid, 256, smem, st>>>((int)M, (int)N, (int)K, A, lda, B, ldb, C,
                                                                           ldc, *zs));
        return;
    }
    IAB_TIMED("k_gemm_f64", st, k_gemm_f64<<<grid, 256, G::SMEM, st>>>((int)M, (int)N, (int)K, A, lda, B, ldb, C, ldc));
}

// Grouped form: one persistent launch over the tiles of many independent products.
// Problem p owns global tiles [tile_start, tile_start + tiles_m * tiles_n); CTAs take
// tiles round-robin and find their problem by binary search.
template <int BM, int BN, int BK>
__global__ void __launch_bounds__(256) k_gemm_f64_grouped(const GemmProblem *__restrict__ probs, int nprob,
                                                          int total_tiles)
{
    extern __shared__ __align__(16) double smf64[];
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (probs[mid].tile_start <= t) lo = mid; else hi = mid - 1;
        }
        const GemmProblem &p = probs[lo];
        const int local = t - p.tile_start, tn_count = (p.N + BN - 1) / BN;
        const int tm = local / tn_count, tn = local - tm * tn_count;
        f64_tile<BM, BN, BK>(p.M, p.N, p.K, p.A, p.lda, p.B, p.ldb, p.C, p.ldc, tm * BM, tn * BN, smf64);
        __syncthreads();
    }
}

// Tile configuration cfg: shape (cfg & 3: 128x128, 64x128, 128x64, 64x64), stage depth
// (cfg < 4: 16, else 32 k per stage).
int gemm_f64_grouped_tiles(int cfg, int M, int N)
{
    const int s = cfg & 3;
    const int bm = (s == 0 || s == 2) ? 128 : 64, bn = (s == 0 || s == 1) ? 128 : 64;
    return ((M + bm - 1) / bm) * ((N + bn - 1) / bn);
}

template <int BM, int BN, int BK>
static void launch_grouped(const GemmProblem *d_probs, int nprob, int total, int ctas, cudaStream_t st)
{
    using G = f64k::Cfg<BM, BN, BK>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_f64_grouped<BM, BN, BK>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
        attr = true;
    }
    IAB_TIMED("k_gemm_f64_grouped", st, k_gemm_f64_grouped<BM, BN, BK><<<(unsigned)std::max(1, std::min(ctas, total)), 256, G::SMEM, st>>>(
        d_probs, nprob, total));
}

template <int BM, int BN, int BK>
static int grouped_ctas()
{
    using G = f64k::Cfg<BM, BN, BK>;
    cudaFuncSetAttribute(k_gemm_f64_grouped<BM, BN, BK>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gemm_f64_grouped<BM, BN, BK>, 256, G::SMEM) != cudaSuccess)
        per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, per_sm) * std::max(1, sms);
}

int gemm_f64_grouped_ctas(int cfg)
{
    switch (cfg) {
    case 0: return grouped_ctas<128, 128, 16>();
    case 1: return grouped_ctas<64, 128, 16>();
    case 2: return grouped_ctas<128, 64, 16>();
    case 3: return grouped_ctas<64, 64, 16>();
    case 4: return grouped_ctas<128, 128, 32>();
    case 5: return grouped_ctas<64, 128, 32>();
    case 6: return grouped_ctas<128, 64, 32>();
    default: return grouped_ctas<64, 64, 32>();
    }
}

void gemm_f64_grouped(int cfg, const GemmProblem *d_probs, int nprob, int total_tiles, int ctas, cudaStream_t st)
{
    switch (cfg) {
    case 0: launch_grouped<128, 128, 16>(d_probs, nprob, total_tiles, ctas, st); break;
    case 1: launch_grouped<64, 128, 16>(d_probs, nprob, total_tiles, ctas, st); break;
    case 2: launch_grouped<128, 64, 16>(d_probs, nprob, total_tiles, ctas, st); break;
    case 3: launch_grouped<64, 64, 16>(d_probs, nprob, total_tiles, ctas, st); break;
    case 4: launch_grouped<128, 128, 32>(d_probs, nprob, total_tiles, ctas, st); break;
    case 5: launch_grouped<64, 128, 32>(d_probs, nprob, total_tiles, ctas, st); break;
    case 6: launch_grouped<128, 64, 32>(d_probs, nprob, total_tiles, ctas, st); break;
    default: launch_grouped<64, 64, 32>(d_probs, nprob, total_tiles, ctas, st); break;
    }
}

// ============================================================================ FP32 FFMA
namespace f32k {
constexpr int BM = 128, BN = 128, BK = 8;
}

// Requires lda, ldb multiples of 4 and 16-byte aligned bases.
__global__ void __launch_bounds__(256) k_gemm_f32(int M, int N, int K, const float *__restrict__ A, int64_t lda,
                                                  const float *__restrict__ B, int64_t ldb, float *__restrict__ C,
                                                  int64_t ldc)
{
    using namespace f32k;
    __shared__ __align__(16) float sA[2][BK][BM + 4];
    __shared__ __align__(16) float sB[2][BK][BN];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;   // 16 x 16 threads, 8x8 each
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
    // A loads: 128 rows x 8 k = 256 float4 (row r, k-quad); stored transposed
    const int ar = tid >> 1, ak = (tid & 1) * 4;
    // B loads: 8 rows x 128 = 256 float4
    const int br = tid >> 5, bc = (tid & 31) * 4;
    const int ktiles = (K + BK - 1) / BK;
    float4 ra, rb;
    auto gload = [&](int kt) {
        const int k0 = kt * BK;
        const int gr = m0 + ar, gk = k0 + ak;
        ra = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gr < M) {
            const float *p = A + (int64_t)gr * lda + gk;
            if (gk + 3 < K) ra = *reinterpret_cast<const float4 *>(p);
            else {
                if (gk < K) ra.x = p[0];
                if (gk + 1 < K) ra.y = p[1];
                if (gk + 2 < K) ra.z = p[2];
            }
        }
        const int gk2 = k0 + br, gn = n0 + bc;
        rb = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gk2 < K) {
            const float *p = B + (int64_t)gk2 * ldb + gn;
            if (gn + 3 < N) rb = *reinterpret_cast<const float4 *>(p);
            else {
                if (gn < N) rb.x = p[0];
                if (gn + 1 < N) rb.y = p[1];
                if (gn + 2 < N) rb.z = p[2];
            }
        }
    };
    auto sstore = [&](int s) {
        sA[s][ak + 0][ar] = ra.x; sA[s][ak + 1][ar] = ra.y; sA[s][ak + 2][ar] = ra.z; sA[s][ak + 3][ar] = ra.w;
        *reinterpret_cast<float4 *>(&sB[s][br][bc]) = rb;
    };
    gload(0);
    sstore(0);
    __syncthreads();
    for (int kt = 0; kt < ktiles; kt++) {
        const int s = kt & 1;
        if (kt + 1 < ktiles) gload(kt + 1);
#pragma unroll
        for (int k = 0; k < BK; k++) {
            float a[8], b[8];
            const float4 a0 = *reinterpret_cast<const float4 *>(&sA[s][k][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&sA[s][k][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4 *>(&sB[s][k][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4 *>(&sB[s][k][64 + tx * 4]);
            a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w; a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
            b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w; b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < ktiles) {
            sstore(s ^ 1);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
        if (r >= M) continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int c = n0 + h * 64 + tx * 4;
            float *cp = C + (int64_t)r * ldc + c;
            const float v0 = acc[i][h * 4 + 0], v1 = acc[i][h * 4 + 1], v2 = acc[i][h * 4 + 2], v3 = acc[i][h * 4 + 3];
            if (c + 3 < N) *reinterpret_cast<float4 *>(cp) = make_float4(v0, v1, v2, v3);
            else {
                if (c < N) cp[0] = v0;
                if (c + 1 < N) cp[1] = v1;
                if (c + 2 < N) cp[2] = v2;
            }
        }
    }
}

void gemm_f32_native(int64_t M, int64_t N, int64_t K, const float *A, int64_t lda, const float *B, int64_t ldb,
                     float *C, int64_t ldc, cudaStream_t st)
{
    using namespace f32k;
    dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)((M + BM - 1) / BM));
    IAB_TIMED("k_gemm_f32", st, k_gemm_f32<<<grid, 256, 0, st>>>((int)M, (int)N, (int)K, A, lda, B, ldb, C, ldc));
}

// ============================================================================ GEMV
template <typename T>
__global__ void __launch_bounds__(256) k_gemv(int M, int K, const T *__restrict__ A, int64_t lda,
                                              const T *__restrict__ x, T *__restrict__ y)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= M) return;
    const T *row = A + (int64_t)warp * lda;
    T acc = 0;
    constexpr int V = 16 / sizeof(T);
    const int kv = K / V;
    for (int i = lane; i < kv; i += 32) {
        if constexpr (sizeof(T) == 8) {
            const double2 a = __ldcs(reinterpret_cast<const double2 *>(row) + i);
            const double2 b = __ldg(reinterpret_cast<const double2 *>(x) + i);
            acc = fma(a.x, b.x, acc);
            acc = fma(a.y, b.y, acc);
        } else {
            const float4 a = __ldcs(reinterpret_cast<const float4 *>(row) + i);
            const float4 b = __ldg(reinterpret_cast<const float4 *>(x) + i);
            acc = fmaf(a.x, b.x, acc);
            acc = fmaf(a.y, b.y, acc);
            acc = fmaf(a.z, b.z, acc);
            acc = fmaf(a.w, b.w, acc);
        }
    }
    for (int i = kv * V + lane; i < K; i += 32) acc += row[i] * x[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) y[warp] = acc;
}

void gemv_native(int dtype, int64_t M, int64_t K, const void *A, int64_t lda, const void *x, void *y, cudaStream_t st)
{
    const int blocks = (int)((M * 32 + 255) / 256);
    if (dtype == 0) { IAB_TIMED("k_gemv", st, k_gemv<double><<<blocks, 256, 0, st>>>((int)M, (int)K, (const double *)A, lda, (const double *)x, (double *)y)); }
    else { IAB_TIMED("k_gemv", st, k_gemv<float><<<blocks, 256, 0, st>>>((int)M, (int)K, (const float *)A, lda, (const float *)x, (float *)y)); }
}

// ============================================================================ helpers
template <typename T>
__global__ void k_arange(int64_t M, int64_t N, int64_t ld, double start, double step, T *out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M * N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / N, c = i - r * N;
        out[r * ld + c] = (T)(start + (double)i * step);
    }
}

void fill_arange(int dtype, int64_t M, int64_t N, int64_t ld, double start, double step, void *out, cudaStream_t st)
{
    const int64_t n = M * N;
    const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32);
    if (n == 0) return;
    if (dtype == 0) { IAB_TIMED("k_arange", st, k_arange<double><<<blocks, 256, 0, st>>>(M, N, ld, start, step, (double *)out)); }
    else { IAB_TIMED("k_arange", st, k_arange<float><<<blocks, 256, 0, st>>>(M, N, ld, start, step, (float *)out)); }
}

template <typename T>
__global__ void k_transpose(int64_t rows, int64_t cols, const T *__restrict__ in, int64_t ldin, T *__restrict__ out,
                            int64_t ldout)
{
    __shared__ T tile[32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = in[r * ldin + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t r = c0 + k, c = r0 + threadIdx.x;   // out is cols x rows
        if (r < cols && c < rows) out[r * ldout + c] = tile[threadIdx.x][k];
    }
}

void transpose_dense(int itemsize, int64_t rows, int64_t cols, const void *in, int64_t ldin, void *out, int64_t ldout,
                     cudaStream_t st)
{
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32)), block(32, 8);
    if (itemsize == 8) { IAB_TIMED("k_transpose", st, k_transpose<double><<<grid, block, 0, st>>>(rows, cols, (const double *)in, ldin, (double *)out, ldout)); }
    else { IAB_TIMED("k_transpose", st, k_transpose<float><<<grid, block, 0, st>>>(rows, cols, (const float *)in, ldin, (float *)out, ldout)); }
}

}  // namespace iab
