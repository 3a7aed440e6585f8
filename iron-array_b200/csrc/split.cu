// Split-precision float64 product on the INT8 tensor cores (Ozaki scheme II, the
// Chinese-remainder form), for the block-pair GEMM of ironArray's matmul path
// (src/linalg/iarray_gemm.c:276-290 computes the same product with cblas_dgemm).
//
//   1. Scaling.  Row i of A is scaled by 2^sA_i and rounded to an integer matrix A'
//      (|A'_ik| < 2^52), column j of B by 2^sB_j -> B'.  The shifts are chosen from the
//      row / column 2-norms so that ||A'_i||_2 * ||B'_j||_2 < P / 8, where P is the
//      product of the moduli; by Cauchy-Schwarz every entry of C' = A' B' then lies in
//      (-P/8, P/8) and is recovered exactly from its residues.
//   2. Residues.  For each modulus m_l (pairwise coprime, <= 256) the symmetric residues
//      A'_l = A' mod m_l and B'_l = B' mod m_l fit in int8 (B'_l is stored transposed,
//      K-major, for the tensor-core operand layout).
//   3. INT8 GEMM per modulus on tcgen05 (kind::i8, INT32 accumulate in TMEM, exact since
//      K * 128 * 128 < 2^31), fused epilogue reducing every entry modulo m_l to a byte.
//   4. Reconstruction.  C'_ij = sum_l r_l w_l mod P (w_l the CRT basis, held in 40-bit
//      chunks so that the sums are exact in FP64), centred, rounded to float64 and scaled
//      back by 2^-(sA_i + sB_j).
// FP64 (non-tensor) arithmetic is used for the scaling, the residues and the
// reconstruction; every step before the final rounding is exact.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "bytes.cuh"
#include "common.cuh"
#include "tc_common.cuh"
#include "zskip.cuh"

namespace iab {

// ============================================================================ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

bool make_tmap_3d(CUtensorMap *map, CUtensorMapDataType dt, const void *base, uint64_t d0, uint64_t d1, uint64_t d2,
                  uint64_t stride1, uint64_t stride2, uint32_t box0, uint32_t box1, CUtensorMapSwizzle sw)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {stride1, stride2};
    const cuuint32_t box[3] = {box0, box1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ============================================================================ moduli + CRT basis
constexpr int MAX_MODULI = 20;
static const int kModuli[MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                        223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

constexpr int CRT_BITS = 34;                       // chunk width of the reconstruction
struct CrtConst {
    int L;
    int np;                                        // residue pairs (m_2p, m_2p+1); the last is single when L is odd
    int nc;                                        // CRT_BITS-bit chunks needed for P (1..4)
    int mod[MAX_MODULI];
    double inv_mod[MAX_MODULI];
    float inv_modf[MAX_MODULI];
    uint32_t pm0[8], pm1[8];                       // pair moduli (pm1 = 1: single)
    uint32_t pinv[8], pmagic[8];                   // pm0^-1 mod pm1, ceil(2^32 / pm1)
    double pw[8][4];                               // CRT basis of the pair moduli M_p = pm0 pm1:
                                                   // (P/M_p) ((P/M_p)^-1 mod M_p) mod P, in chunks
    double pp[4];                                  // P in chunks (least significant first)
    double inv_p;                                  // 1/P (rounded)
    double log2p;
};

__constant__ CrtConst c_crt;

static bool build_crt(int L, CrtConst *c)
{
    if (L < 2 || L > 16) return false;   // P < 2^126: at most four chunks
    typedef unsigned __int128 u128;
    const u128 mask = ((u128)1 << CRT_BITS) - 1;
    u128 P = 1;
    for (int l = 0; l < L; l++) P *= (u128)kModuli[l];
    memset(c, 0, sizeof(*c));
    c->L = L;
    int bits = 0;
    for (u128 t = P; t; t >>= 1) bits++;
    c->nc = (bits + CRT_BITS - 1) / CRT_BITS;
    double lp = 0;
    for (int l = 0; l < L; l++) {
        const int m = kModuli[l];
        c->mod[l] = m;
        c->inv_mod[l] = 1.0 / m;
        c->inv_modf[l] = 1.0f / (float)m;
        lp += log2((double)m);
    }
    auto inverse = [](uint64_t a, uint64_t m) -> uint64_t {   // a^-1 mod m (m > 1, gcd 1)
        for (uint64_t x = 1; x < m; x++)
            if ((a * x) % m == 1) return x;
        return 0;
    };
    c->np = (L + 1) / 2;
    for (int p = 0; p < c->np; p++) {
        const uint64_t m0 = (uint64_t)kModuli[2 * p], m1 = 2 * p + 1 < L ? (uint64_t)kModuli[2 * p + 1] : 1;
        c->pm0[p] = (uint32_t)m0;
        c->pm1[p] = (uint32_t)m1;
        if (m1 > 1) {
            c->pinv[p] = (uint32_t)inverse(m0 % m1, m1);
            c->pmagic[p] = (uint32_t)(((uint64_t)1 << 32) / m1 + 1);   // ceil(2^32 / m1): m1 is odd
            if (!c->pinv[p]) return false;
        }
        const u128 Mp = (u128)(m0 * m1), Q = P / Mp;
        const uint64_t inv = inverse((uint64_t)(Q % Mp), (uint64_t)Mp);
        if (!inv) return false;
        const u128 w = (Q * (u128)inv) % P;
        for (int k = 0; k < 4; k++) c->pw[p][k] = (double)(uint64_t)((w >> (CRT_BITS * k)) & mask);
    }
    for (int k = 0; k < 4; k++) c->pp[k] = (double)(uint64_t)((P >> (CRT_BITS * k)) & mask);
    c->inv_p = 1.0 / ((double)(uint64_t)(P >> 64) * 18446744073709551616.0 + (double)(uint64_t)P);
    c->log2p = lp;
    return true;
}

// ============================================================================ scaling
// Shift value of a row / column that holds a NaN or an infinity: its residues are zero and
// its outputs are recomputed by k_nonfinite_fix.
constexpr int kNonFinite = -0x7fffffff - 1;

// Shift for one row / column: the largest s with max|x| * 2^s < 2^52 and
// ||x||_2 * 2^s <= 2^(gamma - 1); lg2nrm = log2 ||x||_2.
__device__ __forceinline__ int pick_shift(double amax, double lg2nrm, double gamma)
{
    if (!(amax > 0.0)) return 0;
    int e;
    frexp(amax, &e);                      // amax < 2^e
    const int s1 = 52 - e;
    const int s2 = (int)floor(gamma - lg2nrm) - 1;
    return min(s1, s2);
}

// Largest magnitude for which the plain sum of squares of up to 65536 entries neither
// overflows nor loses the largest square to underflow (2^-480 .. 2^480); outside it the
// norm is taken again from the entries scaled by 2^-e.
__device__ __forceinline__ bool norm_needs_rescale(double amax) { return amax > 0x1p480 || amax < 0x1p-480; }

__global__ void __launch_bounds__(256) k_row_shift(int M, int K, const double *__restrict__ A, int64_t lda, double gamma,
                                                   int *__restrict__ shift)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= M) return;
    const double *row = A + (int64_t)warp * lda;
    double mx = 0.0, ss = 0.0;
    for (int k = lane; k < K; k += 32) {
        const double v = fabs(row[k]);
        mx = fmax(mx, v);
        ss = fma(v, v, ss);
    }
    for (int o = 16; o; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    // a NaN reaches ss (fmax drops it), an infinity reaches mx
    if (isnan(ss) || isinf(mx)) {
        if (lane == 0) shift[warp] = kNonFinite;
        return;
    }
    double lg = 0.5 * log2(ss);
    if (mx > 0.0 && norm_needs_rescale(mx)) {
        int e;
        frexp(mx, &e);
        double s2 = 0.0;
        for (int k = lane; k < K; k += 32) {
            const double v = ldexp(fabs(row[k]), -e);
            s2 = fma(v, v, s2);
        }
        for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        lg = 0.5 * log2(s2) + e;
    }
    if (lane == 0) shift[warp] = pick_shift(mx, lg, gamma);
}

constexpr int COL_SEGS = 64;

__global__ void __launch_bounds__(256) k_col_partial(int K, int N, const double *__restrict__ B, int64_t ldb,
                                                     double *__restrict__ pmax, double *__restrict__ pss)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, seg = blockIdx.y;
    if (j >= N) return;
    const int per = (K + COL_SEGS - 1) / COL_SEGS, k0 = seg * per, k1 = min(K, k0 + per);
    double mx = 0.0, ss = 0.0;
    for (int k = k0; k < k1; k++) {
        const double v = fabs(B[(int64_t)k * ldb + j]);
        mx = fmax(mx, v);
        ss = fma(v, v, ss);
    }
    pmax[(int64_t)seg * N + j] = mx;
    pss[(int64_t)seg * N + j] = ss;
}

__global__ void k_col_shift(int K, int N, const double *__restrict__ B, int64_t ldb, const double *__restrict__ pmax,
                            const double *__restrict__ pss, double gamma, int *__restrict__ shift)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    double mx = 0.0, ss = 0.0;
    for (int s = 0; s < COL_SEGS; s++) {
        mx = fmax(mx, pmax[(int64_t)s * N + j]);
        ss += pss[(int64_t)s * N + j];
    }
    if (isnan(ss) || isinf(mx)) {
        shift[j] = kNonFinite;
        return;
    }
    double lg = 0.5 * log2(ss);
    if (mx > 0.0 && norm_needs_rescale(mx)) {
        int e;
        frexp(mx, &e);
        double s2 = 0.0;
        for (int k = 0; k < K; k++) {
            const double v = ldexp(fabs(B[(int64_t)k * ldb + j]), -e);
            s2 = fma(v, v, s2);
        }
        lg = 0.5 * log2(s2) + e;
    }
    shift[j] = pick_shift(mx, lg, gamma);
}

// Outputs whose row of A or column of B holds a NaN or an infinity are recomputed as plain
// dot products (one FMA per k, in order), so they carry the native product's IEEE
// propagation.  One warp per row (warp index < M, flag rflag[i] == flagval) or column
// (warp index - M); warps of rows and columns without such values return at once.
// Offset of item (i, j) of a container in its encoder's shuffled block image (plane 0; plane
// p is p * blockn further).
__device__ __forceinline__ int64_t img_item_offset(const Geom &g, int64_t i, int64_t j)
{
    const int64_t ci = i / g.chunk[0], ii = i - ci * g.chunk[0], bi = ii / g.block[0];
    const int64_t cj = j / g.chunk[1], jj = j - cj * g.chunk[1], bj = jj / g.block[1];
    const int64_t t = (ci * g.cgrid[1] + cj) * g.nblocks + bi * g.bgrid[1] + bj;
    return t * g.blocksize + (ii - bi * g.block[0]) * g.block[1] + (jj - bj * g.block[1]);
}

// Store of one output of the non-finite fix: dense C, or (IMG, float64 only) the eight bytes of
// the item in the output container's shuffled block image.
template <typename T, bool IMG>
__device__ __forceinline__ void fix_store(T *C, int64_t ldc, const Geom &g, uint8_t *img, int64_t i, int64_t j, T v)
{
    if constexpr (IMG) {
        const uint64_t x = (uint64_t)__double_as_longlong((double)v);
        uint8_t *o = img + img_item_offset(g, i, j);
#pragma unroll
        for (int p = 0; p < 8; p++) o[(int64_t)p * g.blockn] = (uint8_t)(x >> (8 * p));
    } else {
        C[i * ldc + j] = v;
    }
}

template <typename T, bool IMG>
__global__ void __launch_bounds__(256) k_nonfinite_fix(int M, int N, int K, const T *__restrict__ A, int64_t lda,
                                                      const T *__restrict__ B, int64_t ldb, T *__restrict__ C,
                                                      int64_t ldc, const int *__restrict__ rflag,
                                                      const int *__restrict__ cflag, int flagval, Geom g, uint8_t *img)
{
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w < M) {
        const int i = (int)w;
        if (rflag[i] != flagval) return;
        for (int j = lane; j < N; j += 32) {
            T acc = 0;
            for (int k = 0; k < K; k++) acc = fma(A[(int64_t)i * lda + k], B[(int64_t)k * ldb + j], acc);
            fix_store<T, IMG>(C, ldc, g, img, i, j, acc);
        }
    } else if (w < (int64_t)M + N) {
        const int j = (int)(w - M);
        if (cflag[j] != flagval) return;
        for (int i = lane; i < M; i += 32) {
            T acc = 0;
            for (int k = 0; k < K; k++) acc = fma(A[(int64_t)i * lda + k], B[(int64_t)k * ldb + j], acc);
            fix_store<T, IMG>(C, ldc, g, img, i, j, acc);
        }
    }
}

template <typename T>
static void launch_nonfinite_fix(int64_t M, int64_t N, int64_t K, const T *A, int64_t lda, const T *B, int64_t ldb,
                                 T *C, int64_t ldc, const int *rflag, const int *cflag, int flagval, cudaStream_t st,
                                 const CImage *cimg = nullptr)
{
    const int64_t threads = (M + N) * 32;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    if (cimg) {
        IAB_TIMED("k_nonfinite_fix", st, k_nonfinite_fix<T, true><<<grid, 256, 0, st>>>(
            (int)M, (int)N, (int)K, A, lda, B, ldb, C, ldc, rflag, cflag, flagval, cimg->g, cimg->img));
    } else {
        Geom g0;
        memset(&g0, 0, sizeof(g0));
        IAB_TIMED("k_nonfinite_fix", st, k_nonfinite_fix<T, false><<<grid, 256, 0, st>>>(
            (int)M, (int)N, (int)K, A, lda, B, ldb, C, ldc, rflag, cflag, flagval, g0, nullptr));
    }
}

// ============================================================================ residues
// Rounding by the 1.5 * 2^52 constant: for |y| < 2^51, (y + kRound) is the double of ulp 1
// nearest to y + kRound, so (y + kRound) - kRound = rint(y), and the low 32 bits of
// y + kRound hold rint(y) in two's complement.  This keeps the per-modulus work on the
// FP64 pipe (no float/int conversions).
constexpr double kRound = 6755399441055744.0;
constexpr double kTwo52 = 4503599627370496.0;

// 2^s for -1022 <= s <= 1023.
__device__ __forceinline__ double pow2i(int s) { return __hiloint2double((1023 + s) << 20, 0); }

// x = rint(a * 2^s), the scaled entry of an operand row or column (|x| < 2^52), and the low
// 32 bits of x as an integer: y + copysign(2^52, y) holds |x| in its mantissa field.
__device__ __forceinline__ double scaled_int(double a, int s, bool pow2_ok, double f, uint32_t &xlo)
{
    const double y = pow2_ok ? a * f : ldexp(a, s);
    if (!pow2_ok) {
        const double x = rint(y);
        xlo = (uint32_t)__double2ll_rn(x);
        return x;
    }
    const double c = copysign(kTwo52, y);
    const double t = y + c;
    const uint32_t mag = (uint32_t)__double2loint(t);
    xlo = y < 0.0 ? 0u - mag : mag;
    return t - c;
}

// Residue of the integer x (|x| < 2^52, low 32 bits xlo) modulo m_l, as the byte of an int8
// in [-128, 127].  The INT8 products need only some representative of the class, not the
// centred one.  l = 0 is m = 256: the low byte.  Otherwise q = rint(x / m) comes from one
// FMA (its low 32 bits sit in the low word of x / m + 1.5 * 2^52); q may be one off near a
// half-integer, so x - q m lies in [-m/2 - 1, m/2 + 1] and one correction brings it below 128.
__device__ __forceinline__ uint32_t residue_byte(double x, uint32_t xlo, int l)
{
    if (l == 0) return xlo & 0xffu;
    const uint32_t m = (uint32_t)c_crt.mod[l];
    const uint32_t q = (uint32_t)__double2loint(fma(x, c_crt.inv_mod[l], kRound));
    int r = (int)(xlo - q * m);
    if (r > 127) r -= (int)m;
    return (uint32_t)r & 0xffu;
}

// A (M x K, row-major) -> res[l][i][k] (int8, row pitch Kp), 8 consecutive k per thread.
__global__ void __launch_bounds__(256) k_residues_rows(int M, int K, int Kp, const double *__restrict__ A, int64_t lda,
                                                       const int *__restrict__ shift, int8_t *__restrict__ res)
{
    const int groups = Kp / 8;
    const int64_t total = (int64_t)M * groups;
    const int L = c_crt.L;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / groups), k0 = (int)(t - (int64_t)i * groups) * 8;
        const int s = shift[i];
        const bool p2 = s >= -1022 && s <= 1023, fin = s != kNonFinite;
        const double f = p2 ? pow2i(s) : 0.0;
        double x[8];
        uint32_t xl[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int k = k0 + u;
            xl[u] = 0u;
            x[u] = k < K && fin ? scaled_int(A[(int64_t)i * lda + k], s, p2, f, xl[u]) : 0.0;
        }
#pragma unroll
        for (int l = 0; l < 16; l++) {
            if (l < L) {
                uint32_t w0 = 0, w1 = 0;
#pragma unroll
                for (int u = 0; u < 4; u++) w0 |= residue_byte(x[u], xl[u], l) << (8 * u);
#pragma unroll
                for (int u = 0; u < 4; u++) w1 |= residue_byte(x[4 + u], xl[4 + u], l) << (8 * u);
                *reinterpret_cast<uint2 *>(res + ((int64_t)l * M + i) * Kp + k0) = make_uint2(w0, w1);
            }
        }
    }
}

// B (K x N, row-major) -> res[l][j][k] (int8, transposed, row pitch Kp), via 64x64 tiles.
__global__ void __launch_bounds__(256) k_residues_cols(int K, int N, int Kp, const double *__restrict__ B, int64_t ldb,
                                                       const int *__restrict__ shift, int8_t *__restrict__ res)
{
    __shared__ double tile[64][65];
    const int k0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int r = e >> 6, c = e & 63;
        const int k = k0 + r, j = j0 + c;
        tile[r][c] = (k < K && j < N) ? B[(int64_t)k * ldb + j] : 0.0;
    }
    __syncthreads();
    const int L = c_crt.L;
    for (int e = threadIdx.x; e < 64 * 8; e += blockDim.x) {
        const int c = e >> 3, kg = (e & 7) * 8;
        const int j = j0 + c;
        if (j >= N || k0 + kg >= Kp) continue;
        const int s = shift[j];
        const bool p2 = s >= -1022 && s <= 1023, fin = s != kNonFinite;
        const double f = p2 ? pow2i(s) : 0.0;
        double x[8];
        uint32_t xl[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            xl[u] = 0u;
            x[u] = fin ? scaled_int(tile[kg + u][c], s, p2, f, xl[u]) : 0.0;
        }
#pragma unroll
        for (int l = 0; l < 16; l++) {
            if (l < L) {
                uint32_t w0 = 0, w1 = 0;
#pragma unroll
                for (int u = 0; u < 4; u++) w0 |= residue_byte(x[u], xl[u], l) << (8 * u);
#pragma unroll
                for (int u = 0; u < 4; u++) w1 |= residue_byte(x[4 + u], xl[4 + u], l) << (8 * u);
                *reinterpret_cast<uint2 *>(res + ((int64_t)l * N + j) * Kp + k0 + kg) = make_uint2(w0, w1);
            }
        }
    }
}

// ============================================================================ INT8 tcgen05 GEMM
namespace oz {
constexpr int BM = 128, BN = 256, BK = 128, STAGES = 4;
constexpr int A_BYTES = BM * BK, B_BYTES = BN * BK, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int THREADS = 192;
// The grouped form's many small-K tiles leave the epilogue little MMA time to hide behind:
// it drains each accumulator with eight warps (two per TMEM lane quarter, one column half
// each) instead of four.
template <bool GROUPED> constexpr int threads_of() { return GROUPED ? 320 : THREADS; }
template <bool GROUPED> constexpr int epi_warps() { return GROUPED ? 8 : 4; }
constexpr int SMEM = 1024 + STAGES * STAGE_BYTES + 256;
constexpr uint32_t IDESC = tc::make_idesc(2 /*S32*/, 1 /*s8*/, 1 /*s8*/, BM, BN);
}

// Tile order of the persistent tensor-core kernels: tile rows are taken in groups of
// TILE_GROUP; inside a group the walk is column by column, so the CTAs of one wave share a
// few B column panels and the group's A row panels stay in L2 across the whole group.
constexpr int TILE_GROUP = 32;
__device__ __forceinline__ void tile_of(int local, int tiles_m, int tiles_n, int &tm, int &tn)
{
    const int per_group = TILE_GROUP * tiles_n;
    const int g = local / per_group, rem = local - g * per_group;
    const int rows = min(TILE_GROUP, tiles_m - g * TILE_GROUP);
    tn = rem / rows;
    tm = g * TILE_GROUP + (rem - tn * rows);
}

// One product of a grouped split-precision launch (device table, one entry per product).
struct OzGProb {
    int M, N, K, Kp;
    int tiles_m, tiles_n;
    int64_t row0, col0;          // first row / column of this product in the concatenated row / column index
    int64_t task_r0;             // first task of the grouped row-residue kernel (8 k per task)
    int64_t tile_c0;             // first 64 x 64 tile of the grouped column-residue kernel
    int64_t item0;               // first item (modulus, tile) of the grouped INT8 GEMM
    int64_t crt0;                // first task (row, 4 columns) of the grouped reconstruction
    const double *A, *B;
    double *C;
    int64_t lda, ldb, ldc;
    int8_t *ra, *rb;             // residues [L][M][Kp], [L][N][Kp]
    uint8_t *R;                  // residues of the product [L][M][ldr]
    int64_t ldr;
    Geom gc;                     // image output (OzGroupWork::img): C's geometry, its encoder image,
    uint8_t *cimg;               // and the first work unit of the grouped image reconstruction
    int64_t unit0;
};

// Index of the product whose range [key(q), key(q + 1)) holds v: the last q with key(q) <= v
// (products with empty ranges share their start with the next one).
template <typename F>
__device__ __forceinline__ int oz_find(const OzGProb *__restrict__ pr, int np, int64_t v, F key)
{
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (key(pr[mid]) <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// oz_find for a loop whose values only increase: from the previous product qh (-1: none yet)
// a few steps forward, a binary search when the value has moved further.
template <typename F>
__device__ __forceinline__ int oz_walk(const OzGProb *__restrict__ pr, int np, int64_t v, F key, int &qh)
{
    int q = qh;
    if (q >= 0)
        for (int k = 0; k < 8 && q + 1 < np && key(pr[q + 1]) <= v; k++) q++;
    if (q < 0 || (q + 1 < np && key(pr[q + 1]) <= v)) q = oz_find(pr, np, v, key);
    qh = q;
    return q;
}

struct I8Params {
    int M, N, K, Kp, L, tiles_m, tiles_n;
    uint8_t *R;        // [L][M][ldr] residues of the products
    int64_t ldr;
    int *err;
    int use_skip;      // leave out the k-tiles of zero-block pairs (zskip.cuh)
    ZeroSkip zs;
    // grouped launch: items of every product of the table, tensor maps 2q (A) and 2q + 1 (B)
    const OzGProb *probs;
    int nprob;
    int64_t total;
    const CUtensorMap *maps;
};

// The work of item t: product tile (tm, tn) for modulus l.
struct I8Tile {
    const CUtensorMap *ma, *mb;
    int l, tm, tn, M, N, ktiles;
    uint8_t *R;
    int64_t ldr;
};

// The product of grouped item t, walking forward from the product *qh of the caller's previous
// item (a CTA's items only increase, by the grid size, so the walk is usually one compare).
__device__ __forceinline__ int oz_item_prob(const I8Params &p, int64_t t, int &qh)
{
    int q = qh;
    if (q < 0) q = oz_find(p.probs, p.nprob, t, [](const OzGProb &x) { return x.item0; });
    while (q + 1 < p.nprob && p.probs[q + 1].item0 <= t) q++;
    qh = q;
    return q;
}

template <bool GROUPED>
__device__ __forceinline__ I8Tile i8_tile(const I8Params &p, const CUtensorMap *tmA, const CUtensorMap *tmB, int64_t t,
                                          int &qh)
{
    I8Tile r;
    if constexpr (!GROUPED) {
        r.l = (int)(t / (p.tiles_m * p.tiles_n));
        const int rem = (int)(t - (int64_t)r.l * p.tiles_m * p.tiles_n);
        tile_of(rem, p.tiles_m, p.tiles_n, r.tm, r.tn);
        r.ma = tmA; r.mb = tmB;
        r.M = p.M; r.N = p.N; r.ktiles = p.Kp / oz::BK;
        r.R = p.R; r.ldr = p.ldr;
    } else {
        const int q = oz_item_prob(p, t, qh);
        const OzGProb &pr = p.probs[q];
        const int per = pr.tiles_m * pr.tiles_n;
        const int64_t local = t - pr.item0;
        r.l = (int)(local / per);
        tile_of((int)(local - (int64_t)r.l * per), pr.tiles_m, pr.tiles_n, r.tm, r.tn);
        r.ma = p.maps + 2 * q; r.mb = p.maps + 2 * q + 1;
        r.M = pr.M; r.N = pr.N; r.ktiles = pr.Kp / oz::BK;
        r.R = pr.R; r.ldr = pr.ldr;
    }
    return r;
}

// Bit kt of mask[kt / 32] = k-tile kt of output tile (tm, tn) is needed (some K block in it
// pairs a non-zero A block under the tile's rows with a non-zero B block under its
// columns).  Called by a whole warp; K <= 65536 keeps the mask within 16 words.
__device__ __forceinline__ void i8_kmask(const I8Params &p, int tm, int tn, int ktiles, uint32_t *mask)
{
    const int lane = threadIdx.x & 31;
    const int64_t r0 = (int64_t)tm * oz::BM, r1 = min(r0 + oz::BM, (int64_t)p.M);
    const int64_t c0 = (int64_t)tn * oz::BN, c1 = min(c0 + oz::BN, (int64_t)p.N);
    for (int w = 0; w < (ktiles + 31) / 32; w++) {
        const int kt = w * 32 + lane;
        const bool f = kt < ktiles && zs_tile_active(p.zs, r0, r1, c0, c1, (int64_t)kt * oz::BK,
                                                      min((int64_t)(kt + 1) * oz::BK, (int64_t)p.K));
        const uint32_t b = __ballot_sync(0xffffffffu, f);
        if (lane == 0) mask[w] = b;
    }
    __syncwarp();
}

// Whether output tile (tm, tn) needs any k-tile (whole warp).
__device__ __forceinline__ bool i8_tile_any(const I8Params &p, int tm, int tn, int ktiles)
{
    const int lane = threadIdx.x & 31;
    const int64_t r0 = (int64_t)tm * oz::BM, r1 = min(r0 + oz::BM, (int64_t)p.M);
    const int64_t c0 = (int64_t)tn * oz::BN, c1 = min(c0 + oz::BN, (int64_t)p.N);
    for (int w = 0; w < (ktiles + 31) / 32; w++) {
        const int kt = w * 32 + lane;
        const bool f = kt < ktiles && zs_tile_active(p.zs, r0, r1, c0, c1, (int64_t)kt * oz::BK,
                                                      min((int64_t)(kt + 1) * oz::BK, (int64_t)p.K));
        if (__ballot_sync(0xffffffffu, f)) return true;
    }
    return false;
}

// Persistent, warp-specialised: warp 0 issues TMA loads, warp 1 issues tcgen05.mma into
// one of two TMEM accumulators (128 x 256 int32 each), warps 2-5 drain the other
// accumulator: r = C mod m_l in [0, m_l), stored as one byte per entry.  With use_skip,
// the k-tiles of zero-block pairs are neither loaded nor multiplied (every role derives the
// same mask); a tile that needs none is written as zero residues.
template <bool SKIP, bool GROUPED>
__global__ void __launch_bounds__(oz::threads_of<GROUPED>(), 1) k_i8gemm_mod(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB, I8Params p)
{
    static_assert(!(SKIP && GROUPED), "the grouped form does not skip zero blocks");
    using namespace oz;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA = smem, *sB = smem + STAGES * A_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    uint32_t *pmask = reinterpret_cast<uint32_t *>(smem + STAGES * STAGE_BYTES + 112);   // producer's k-tile mask
    uint32_t *mmask = pmask + 16;                                                        // MMA issuer's
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { tc::mbar_init(&full[s], 1); tc::mbar_init(&empty[s], 1); }
        for (int b = 0; b < 2; b++) { tc::mbar_init(&tfull[b], 1); tc::mbar_init(&tempty[b], epi_warps<GROUPED>()); }
        tc::mbar_init(drain, 1);
        tc::fence_barrier_init();
        if constexpr (!GROUPED) {
            tc::tma_prefetch_desc(&tmA);
            tc::tma_prefetch_desc(&tmB);
        }
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int64_t total = GROUPED ? p.total : (int64_t)p.L * p.tiles_m * p.tiles_n;
    const int ktiles = p.Kp / BK;            // (SKIP only: the single product's k-tiles)
    auto needed = [&](const uint32_t *mask, int kt) {
        if constexpr (SKIP) return ((mask[kt >> 5] >> (kt & 31)) & 1u) != 0;
        else return true;
    };

    int qh = -1;                             // grouped form: product of this warp's previous item
    if (warp == 0) {
        int stage = 0;
        uint32_t phase = 0;
        int64_t issued = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {  // the whole warp walks the tiles
            const I8Tile tl = i8_tile<GROUPED>(p, &tmA, &tmB, t, qh);
            const int l = tl.l, tm = tl.tm, tn = tl.tn;
            if constexpr (GROUPED) {
                // the tensor maps of this CTA's next item (often another product's) are fetched
                // while this item's loads run
                const int64_t tn2 = t + gridDim.x;
                if (lane == 0 && tn2 < total) {
                    int q2 = qh;
                    while (q2 + 1 < p.nprob && p.probs[q2 + 1].item0 <= tn2) q2++;
                    tc::tma_prefetch_desc(p.maps + 2 * q2);
                    tc::tma_prefetch_desc(p.maps + 2 * q2 + 1);
                }
            }
            if constexpr (SKIP) i8_kmask(p, tm, tn, ktiles, pmask);
            if (lane == 0) {
                for (int kt = 0; kt < tl.ktiles; kt++) {
                    if (!needed(pmask, kt)) continue;
                    if (!tc::mbar_wait(&empty[stage], phase ^ 1, p.err)) { ok = false; break; }
                    tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                    tc::tma_load_3d(sA + stage * A_BYTES, tl.ma, kt * BK, tm * BM, l, &full[stage]);
                    tc::tma_load_3d(sB + stage * B_BYTES, tl.mb, kt * BK, tn * BN, l, &full[stage]);
                    issued++;
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            }
            if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) break;
        }
        // every load issued has landed before the CTA may exit (bounded waits on the
        // full barriers of the last STAGES loads)
        if (lane == 0)
            for (int64_t it = issued > STAGES ? issued - STAGES : 0; it < issued; it++)
                tc::mbar_wait(&full[it % STAGES], (uint32_t)((it / STAGES) & 1), p.err, 1u << 20);
    } else if (warp == 1) {
        int stage = 0, acc = 0;
        uint32_t phase = 0, acc_phase = 0;
        bool ok = true;
        for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
            const I8Tile tl = i8_tile<GROUPED>(p, &tmA, &tmB, t, qh);
            if constexpr (SKIP) i8_kmask(p, tl.tm, tl.tn, ktiles, mmask);
            if (lane == 0) {
                if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, p.err)) {
                    ok = false;
                } else {
                    tc::tc_fence_after();
                    const uint32_t dt = tmem_base + (uint32_t)(acc * BN);
                    bool any = false;
                    for (int kt = 0; kt < tl.ktiles; kt++) {
                        if (!needed(mmask, kt)) continue;
                        if (!tc::mbar_wait(&full[stage], phase, p.err)) { ok = false; break; }
                        tc::tc_fence_after();
                        const uint32_t a0 = tc::smem_addr(sA + stage * A_BYTES), b0 = tc::smem_addr(sB + stage * B_BYTES);
#pragma unroll
                        for (int kk = 0; kk < BK / 32; kk++) {
                            tc::mma_i8(dt, tc::sw128_kmajor_desc(a0 + kk * 32), tc::sw128_kmajor_desc(b0 + kk * 32),
                                       IDESC, (any || kk != 0) ? 1u : 0u);
                        }
                        any = true;
                        tc::tc_commit(&empty[stage]);
                        if (++stage == STAGES) { stage = 0; phase ^= 1; }
                    }
                    if (ok) {
                        // an empty tile touches no TMEM: the epilogue writes zeros for it
                        if (any) tc::tc_commit(&tfull[acc]);
                        else tc::mbar_arrive(&tfull[acc]);
                        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
                    }
                }
            }
            if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) break;
        }
        // all issued MMAs complete before TMEM is released
        if (lane == 0) {
            tc::tc_commit(drain);
            tc::mbar_wait(drain, 0, p.err, 1u << 20);
        }
    } else {
        const int q = warp & 3;   // TMEM lane quarter this warp may access
        int c_lo = 0, c_hi = BN;                                  // this warp's columns
        if constexpr (GROUPED) {
            c_lo = ((warp - 2) / 4) * (BN / 2);
            c_hi = c_lo + BN / 2;
        }
        int acc = 0;
        uint32_t acc_phase = 0;
        for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
            const I8Tile tl = i8_tile<GROUPED>(p, &tmA, &tmB, t, qh);
            const int l = tl.l, tm = tl.tm, tn = tl.tn;
            bool active = true;
            if constexpr (SKIP) active = i8_tile_any(p, tm, tn, ktiles);
            if (!tc::mbar_wait(&tfull[acc], acc_phase, p.err)) break;
            tc::tc_fence_after();
            const int m = c_crt.mod[l];
            const float invm = c_crt.inv_modf[l];
            const int row = tm * BM + q * 32 + lane;
            uint8_t *out = tl.R + ((int64_t)l * tl.M + row) * tl.ldr + (int64_t)tn * BN;
            for (int c = c_lo; c < c_hi; c += 32) {
                uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                if (active) {
                    uint32_t v[32];
                    tc::tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + c), v);
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        uint32_t packed = 0;
#pragma unroll
                        for (int b = 0; b < 4; b++) {
                            const int x = (int)v[u * 4 + b];
                            const int qq = __float2int_rn((float)x * invm);
                            int r = x - qq * m;
                            r += (r < 0) ? m : 0;
                            r -= (r >= m) ? m : 0;
                            packed |= (uint32_t)r << (8 * b);
                        }
                        w[u] = packed;
                    }
                }
                const int col = tn * BN + c;
                if (row < tl.M) {
                    if (col + 32 <= tl.N) {
                        uint4 *o4 = reinterpret_cast<uint4 *>(out + c);
                        o4[0] = make_uint4(w[0], w[1], w[2], w[3]);
                        o4[1] = make_uint4(w[4], w[5], w[6], w[7]);
                    } else {
#pragma unroll
                        for (int b = 0; b < 32; b++)
                            if (col + b < tl.N) out[c + b] = (uint8_t)(w[b >> 2] >> (8 * (b & 3)));
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&tempty[acc]);
            if (++acc == 2) { acc = 0; acc_phase ^= 1; }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 1) tc::tmem_dealloc(tmem_base, 512);
}

// ============================================================================ reconstruction
// X = sum_l r_l w_l mod P, centred into (-P/2, P/2), in exact arithmetic.  The residues of
// each pair of moduli (m0, m1) are first combined in integers (Garner: y = r0 + m0 t with
// t = (r1 - r0) m0^-1 mod m1, so y = X mod m0 m1 < 2^16), then X = sum_p y_p W_p mod P over
// the pair moduli.  Each W_p is held as NC chunks of CRT_BITS = 34 bits, so with at most 8
// pairs every partial sum S_k = sum_p y_p W_pk stays below 2^53 and is exact in FP64.  The
// quotient q = rint(S / P) < 2^19 comes from a rounded estimate of S: the scaling keeps |X|
// below P / 8 (both norms are held to 2^(gamma - 1)), so S / P stays far from a half-integer
// compared with the estimate's error (about 2^-34 of one unit), and q is exact.  Then every
// D_k = S_k - q P_k is exact (q P_k < 2^53); with the low chunks carried into [0, 2^34),
// X = sum_k D_k 2^(34 k) is formed by Horner steps that are exact whenever X is
// representable (every partial floor(X / 2^(34 j)) then is too) and otherwise stay within
// about one ulp.
constexpr double kTwoCB = 17179869184.0;           // 2^CRT_BITS
constexpr double kInvTwoCB = 0x1p-34;

template <int NC>
__device__ __forceinline__ double crt_value(const double (&S)[NC])
{
    double s = S[NC - 1];
#pragma unroll
    for (int k = NC - 2; k >= 0; k--) s = fma(s, kTwoCB, S[k]);
    const double q = fma(s, c_crt.inv_p, kRound) - kRound;
    double D[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) D[k] = fma(-q, c_crt.pp[k], S[k]);
    // carry the low chunks into [0, 2^34) (every step exact: integers below 2^53)
#pragma unroll
    for (int k = 0; k < NC - 1; k++) {
        const double c = floor(D[k] * kInvTwoCB);
        D[k] = fma(-c, kTwoCB, D[k]);
        D[k + 1] += c;
    }
    double x = D[NC - 1];
#pragma unroll
    for (int k = NC - 2; k >= 0; k--) x = fma(x, kTwoCB, D[k]);
    return x;
}

// x * 2^-e, exact scaling (one rounding when the result is subnormal).
__device__ __forceinline__ double unscale(double x, int e)
{
    return (e >= -1023 && e <= 1022) ? x * pow2i(-e) : ldexp(x, -e);
}

// C_ij = 2^-(sA_i + sB_j) * centred( sum_l r_l w_l mod P ); four entries per thread.
// Outputs j0 .. j0 + 3 of row i of one product: reconstruction from the L residue planes
// R[l][i][j] (plane = M ldr bytes), unscaled by the row and column shifts (j0 % 4 == 0; the
// four residue bytes are read as one word, inside the row's ldr bytes).
template <int NC>
__device__ __forceinline__ void crt_quad_values(int N, const uint8_t *__restrict__ R, int64_t ldr, int64_t plane, int si,
                                                const int *__restrict__ sB, int i, int j0, double (&v)[4])
{
    const int L = c_crt.L;
    const uint8_t *rp = R + (int64_t)i * ldr + j0;
    uint32_t w[16];
#pragma unroll
    for (int l = 0; l < 16; l++) w[l] = l < L ? *reinterpret_cast<const uint32_t *>(rp + l * plane) : 0u;  // ldr % 16 == 0
    double S[4][NC];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int k = 0; k < NC; k++) S[u][k] = 0.0;
    const int np = c_crt.np;
#pragma unroll
    for (int p = 0; p < 8; p++) {
        if (p < np) {
            const uint32_t m0 = c_crt.pm0[p], m1 = c_crt.pm1[p], inv = c_crt.pinv[p], mg = c_crt.pmagic[p];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t r0 = (w[2 * p] >> (8 * u)) & 0xffu;
                uint32_t y = r0;
                if (m1 > 1) {
                    const uint32_t r1 = (w[2 * p + 1] >> (8 * u)) & 0xffu;
                    const uint32_t prod = (r1 + 2 * m1 - r0) * inv;           // < 2^18
                    const uint32_t t = prod - __umulhi(prod, mg) * m1;         // prod mod m1, exact
                    y = r0 + m0 * t;
                }
                // y as a double: 2^52 + y, less 2^52
                const double yd = __hiloint2double(0x43300000, (int)y) - kTwo52;
#pragma unroll
                for (int k = 0; k < NC; k++) S[u][k] = fma(yd, c_crt.pw[p][k], S[u][k]);
            }
        }
    }
    bool ok[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int sj = j0 + u < N ? sB[j0 + u] : kNonFinite;
        // rows / columns with NaN or infinity are recomputed by k_nonfinite_fix
        ok[u] = si != kNonFinite && sj != kNonFinite;
        v[u] = crt_value<NC>(S[u]);
        v[u] = unscale(v[u], ok[u] ? si + sj : 0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = ok[u] ? v[u] : 0.0;
}

template <int NC>
__device__ __forceinline__ void crt_quad(int N, const uint8_t *__restrict__ R, int64_t ldr, int64_t plane, int si,
                                         const int *__restrict__ sB, double *__restrict__ C, int64_t ldc, int i, int j0)
{
    double v[4];
    crt_quad_values<NC>(N, R, ldr, plane, si, sB, i, j0, v);
    double *cp = C + (int64_t)i * ldc + j0;
    if (j0 + 3 < N && (reinterpret_cast<uintptr_t>(cp) & 15) == 0) {
        reinterpret_cast<double2 *>(cp)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(cp)[1] = make_double2(v[2], v[3]);
    } else {
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (j0 + u < N) cp[u] = v[u];
    }
}

// Rows of a block per work unit of the image reconstruction: up to 128, fewer when the images
// hold fewer than 128 x 8 x SMs block rows, so that small products still spread over the SMs.
constexpr int CRT_SLICE_MAX = 128;
static int crt_slice_rows(int64_t block_rows_total, int nsm)
{
    const int64_t s = block_rows_total / ((int64_t)nsm * 8);
    return (int)std::max<int64_t>(1, std::min<int64_t>(CRT_SLICE_MAX, s));
}

// The reconstruction written into the output container's shuffled block image (CImage): work
// units are slices of `slice` rows of one block; each thread takes 4 consecutive items of a
// block row (one 4-byte word per byte plane), the logical ones reconstructed, chunk and array
// padding zero, exactly the image the encoder's gather would write from the dense product.
// Needs block[1] % 4 == 0 and chunk[1] % 4 == 0 (every quad starts at a column j0 % 4 == 0).
//
// One work unit of it: rows [slice sl, slice (sl + 1)) of block t of the output's image
// (unit un = t x slices-per-block + sl); sA / sB are the product's row and column shifts.
template <int NC>
__device__ __forceinline__ void crt_img_unit(const Geom &g, const uint8_t *__restrict__ R, int64_t ldr,
                                             const int *__restrict__ sA, const int *__restrict__ sB,
                                             uint8_t *__restrict__ img, int64_t un, int slice)
{
    const int M = (int)g.shape[0], N = (int)g.shape[1];
    const int64_t plane = (int64_t)M * ldr;
    const int qpr = (int)(g.block[1] / 4);
    const int step_r = (int)blockDim.x / qpr, step_q = (int)blockDim.x - step_r * qpr;
    const int spb = (int)((g.block[0] + slice - 1) / slice);
    const int64_t units = g.nchunks * g.nblocks * spb;
    const bool small = units < (int64_t(1) << 31) && g.cgrid[1] < (int64_t(1) << 31);
    int64_t t, c, b, ci0, ci1, bi0, bi1;
    int sl;
    if (small) {                         // 32-bit divisions (the usual case)
        const uint32_t t32 = (uint32_t)un / (uint32_t)spb, c32 = t32 / (uint32_t)g.nblocks;
        const uint32_t b32 = t32 - c32 * (uint32_t)g.nblocks;
        sl = (int)((uint32_t)un - t32 * (uint32_t)spb);
        t = t32; c = c32; b = b32;
        ci0 = c32 / (uint32_t)g.cgrid[1]; ci1 = c32 - (uint32_t)ci0 * (uint32_t)g.cgrid[1];
        bi0 = b32 / (uint32_t)g.bgrid[1]; bi1 = b32 - (uint32_t)bi0 * (uint32_t)g.bgrid[1];
    } else {
        t = un / spb;
        sl = (int)(un - t * spb);
        c = t / g.nblocks; b = t - c * g.nblocks;
        ci0 = c / g.cgrid[1]; ci1 = c - ci0 * g.cgrid[1];
        bi0 = b / g.bgrid[1]; bi1 = b - bi0 * g.bgrid[1];
    }
    const int64_t row0 = ci0 * g.chunk[0] + bi0 * g.block[0], col0 = ci1 * g.chunk[1] + bi1 * g.block[1];
    const int nr = (int)max((int64_t)0, min(min(g.block[0], g.chunk[0] - bi0 * g.block[0]), g.shape[0] - row0));
    const int nc = (int)max((int64_t)0, min(min(g.block[1], g.chunk[1] - bi1 * g.block[1]), g.shape[1] - col0));
    uint8_t *blk = img + t * g.blocksize;
    const int r_lo = sl * slice, r_hi = (int)min((int64_t)r_lo + slice, g.block[0]);
    const int nq = (r_hi - r_lo) * qpr;
    // (row, quad column) of each thread's quad, advanced by a fixed step per iteration
    int r = r_lo + (int)threadIdx.x / qpr, q = (int)threadIdx.x % qpr;
    for (int k = threadIdx.x; k < nq; k += blockDim.x, r += step_r, q += step_q) {
        if (q >= qpr) { q -= qpr; r++; }
        const int cc = q * 4;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        if (r < nr && cc < nc) {
            const int i = (int)row0 + r;
            crt_quad_values<NC>(N, R, ldr, plane, sA[i], sB, i, (int)col0 + cc, v);
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (cc + u >= nc) v[u] = 0.0;                  // chunk or array padding
        }
        uint64_t x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) x[u] = (uint64_t)__double_as_longlong(v[u]);
        uint32_t o[8];
        transpose4x4((uint32_t)x[0], (uint32_t)x[1], (uint32_t)x[2], (uint32_t)x[3], o[0], o[1], o[2], o[3]);
        transpose4x4((uint32_t)(x[0] >> 32), (uint32_t)(x[1] >> 32), (uint32_t)(x[2] >> 32), (uint32_t)(x[3] >> 32),
                     o[4], o[5], o[6], o[7]);
        const int64_t i0 = (int64_t)r * g.block[1] + cc;
#pragma unroll
        for (int p = 0; p < 8; p++) *reinterpret_cast<uint32_t *>(blk + (int64_t)p * g.blockn + i0) = o[p];
    }
}

// Work units: slices of `slice` rows of one block of the image.  Held to 80 registers (three
// CTAs per SM): 0.70 ms instead of 0.79 ms at 8192^2 with 102.
template <int NC>
__global__ void __launch_bounds__(256, 3) k_crt_img(Geom g, const uint8_t *__restrict__ R, int64_t ldr,
                                                    const int *__restrict__ sA, const int *__restrict__ sB,
                                                    uint8_t *__restrict__ img, int slice)
{
    const int64_t units = g.nchunks * g.nblocks * ((g.block[0] + slice - 1) / slice);
    for (int64_t un = blockIdx.x; un < units; un += gridDim.x) crt_img_unit<NC>(g, R, ldr, sA, sB, img, un, slice);
}

template <int NC>
__global__ void __launch_bounds__(256) k_crt(int M, int N, const uint8_t *__restrict__ R, int64_t ldr,
                                             const int *__restrict__ sA, const int *__restrict__ sB,
                                             double *__restrict__ C, int64_t ldc)
{
    const int64_t plane = (int64_t)M * ldr;
    const int nq = (N + 3) / 4;
    const int64_t total = (int64_t)M * nq;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nq), j0 = (int)(e - (int64_t)i * nq) * 4;
        crt_quad<NC>(N, R, ldr, plane, sA[i], sB, C, ldc, i, j0);
    }
}

static void launch_crt(int nc, unsigned grid, int M, int N, const uint8_t *R, int64_t ldr, const int *sA,
                       const int *sB, double *C, int64_t ldc, cudaStream_t st)
{
    switch (nc) {
    case 1: IAB_TIMED("k_crt", st, k_crt<1><<<grid, 256, 0, st>>>(M, N, R, ldr, sA, sB, C, ldc)); break;
    case 2: IAB_TIMED("k_crt", st, k_crt<2><<<grid, 256, 0, st>>>(M, N, R, ldr, sA, sB, C, ldc)); break;
    case 3: IAB_TIMED("k_crt", st, k_crt<3><<<grid, 256, 0, st>>>(M, N, R, ldr, sA, sB, C, ldc)); break;
    default: IAB_TIMED("k_crt", st, k_crt<4><<<grid, 256, 0, st>>>(M, N, R, ldr, sA, sB, C, ldc)); break;
    }
}

static void launch_crt_img(int nc, int nsm, const Geom &g, const uint8_t *R, int64_t ldr, const int *sA,
                           const int *sB, uint8_t *img, cudaStream_t st)
{
    const int slice = crt_slice_rows(g.nchunks * g.nblocks * g.block[0], nsm);
    const int64_t units = g.nchunks * g.nblocks * ceil_div(g.block[0], (int64_t)slice);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)nsm * 8));
    switch (nc) {
    case 1: IAB_TIMED("k_crt_img", st, k_crt_img<1><<<grid, 256, 0, st>>>(g, R, ldr, sA, sB, img, slice)); break;
    case 2: IAB_TIMED("k_crt_img", st, k_crt_img<2><<<grid, 256, 0, st>>>(g, R, ldr, sA, sB, img, slice)); break;
    case 3: IAB_TIMED("k_crt_img", st, k_crt_img<3><<<grid, 256, 0, st>>>(g, R, ldr, sA, sB, img, slice)); break;
    default: IAB_TIMED("k_crt_img", st, k_crt_img<4><<<grid, 256, 0, st>>>(g, R, ldr, sA, sB, img, slice)); break;
    }
}

// ============================================================================ host driver
static int sms()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

static bool device_is_sm100()
{
    int dev = 0, major = 0, minor = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return major == 10 && minor == 0;
}

int gemm_f64_ozaki(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
                   double *C, int64_t ldc, int nterms, cudaStream_t st, const ZeroSkip *zs, const CImage *cimg)
{
    if (cimg && (cimg->g.shape[0] != M || cimg->g.shape[1] != N || cimg->g.itemsize != 8 || (cimg->g.block[1] & 3) ||
                 (cimg->g.chunk[1] & 3) || M > (1 << 30) || N > (1 << 30)))
        return -1;
    OzakiWork w;
    w.zs = zs;
    w.cimg = cimg;
    const int r = gemm_f64_ozaki_launch(M, N, K, A, lda, B, ldb, C, ldc, nterms, &w, st);
    if (r) return r;
    return gemm_f64_ozaki_finish(&w, st);
}

int gemm_f64_ozaki_finish(OzakiWork *w, cudaStream_t st)
{
    if (!w->err.p) return 0;
    int h_err = 0;
    cudaMemcpyAsync(&h_err, w->err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    return h_err ? -3 : 0;
}

// CRT constants for L moduli, copied to the device constant bank on `st`.
static bool set_crt(int L, CrtConst *out, cudaStream_t st)
{
    static std::mutex mu;
    static CrtConst cached;
    static int cached_L = -1;
    std::lock_guard<std::mutex> lk(mu);
    if (cached_L != L) {
        if (!build_crt(L, &cached)) return false;
        cached_L = L;
    }
    *out = cached;
    return cudaMemcpyToSymbolAsync(c_crt, &cached, sizeof(CrtConst), 0, cudaMemcpyHostToDevice, st) == cudaSuccess;
}

int gemm_f64_ozaki_setup(int64_t K, int64_t N, int nterms, OzakiB *ob, cudaStream_t st)
{
    if (!device_is_sm100()) return -1;
    // |sum_k a*b| <= K * 2^14 must keep the epilogue's float quotient within one of the
    // true quotient (K * 2^14 * 2^-24 / 173 < 0.5) and the int32 accumulator exact
    if (K <= 0 || N <= 0 || K > 65536 || N > (1 << 30)) return -1;
    const int L = nterms > 0 ? nterms : 14;
    CrtConst cc;
    if (!set_crt(L, &cc, st)) return -1;
    ob->L = L;
    ob->nc = cc.nc;
    ob->K = K;
    ob->N = N;
    ob->Kp = round_up(K, oz::BK);
    ob->gamma = (cc.log2p - 1.0) / 2.0 - 0.01;
    return 0;
}

int gemm_f64_ozaki_b_kernels(const double *B, int64_t ldb, OzakiB *ob, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int L = ob->L;
    const int64_t K = ob->K, N = ob->N, Kp = ob->Kp;
    ob->B = B;
    ob->ldb = ldb;
    if (!ob->rb.allocate((size_t)(L * N * Kp), dev) || !ob->sb.allocate((size_t)N * 4, dev) ||
        !ob->pm.allocate((size_t)COL_SEGS * N * 8, dev) || !ob->ps.allocate((size_t)COL_SEGS * N * 8, dev))
        return -100;
    IAB_TIMED("k_col_partial", st, k_col_partial<<<dim3((unsigned)((N + 255) / 256), COL_SEGS), 256, 0, st>>>(
        (int)K, (int)N, B, ldb, ob->pm.as<double>(), ob->ps.as<double>()));
    IAB_TIMED("k_col_shift", st, k_col_shift<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
        (int)K, (int)N, B, ldb, ob->pm.as<double>(), ob->ps.as<double>(), ob->gamma, ob->sb.as<int>()));
    IAB_TIMED("k_residues_cols", st, k_residues_cols<<<dim3((unsigned)((N + 63) / 64), (unsigned)((Kp + 63) / 64)), 256, 0, st>>>(
        (int)K, (int)N, (int)Kp, B, ldb, ob->sb.as<int>(), ob->rb.as<int8_t>()));
    static_assert(sizeof(CUtensorMap) <= sizeof(ob->tmB), "tensor map storage");
    if (!make_tmap_3d(reinterpret_cast<CUtensorMap *>(ob->tmB), CU_TENSOR_MAP_DATA_TYPE_UINT8, ob->rb.p, (uint64_t)Kp,
                      (uint64_t)N, (uint64_t)L, (uint64_t)Kp, (uint64_t)(Kp * N), oz::BK, oz::BN,
                      CU_TENSOR_MAP_SWIZZLE_128B))
        return -1;
    return 0;
}

int gemm_f64_ozaki_prepare_b(int64_t K, int64_t N, const double *B, int64_t ldb, int nterms, OzakiB *ob, cudaStream_t st)
{
    const int r = gemm_f64_ozaki_setup(K, N, nterms, ob, st);
    return r ? r : gemm_f64_ozaki_b_kernels(B, ldb, ob, st);
}

int gemm_f64_ozaki_rows_prep(int64_t M, const double *A, int64_t lda, const OzakiB &ob, OzakiWork *w, cudaStream_t st)
{
    if (M <= 0) return 0;
    if (M > (1 << 30)) return -1;
    const int L = ob.L;
    const int64_t N = ob.N, K = ob.K, Kp = ob.Kp;
    const int64_t ldr = round_up(N, 16);
    int dev = 0;
    cudaGetDevice(&dev);
    DevBuf &ra = w->ra, &rr = w->rr, &sa = w->sa, &err = w->err;
    if (!ra.allocate((size_t)(L * M * Kp), dev) || !rr.allocate((size_t)(L * M * ldr), dev) ||
        !sa.allocate((size_t)M * 4, dev) || !err.allocate(16, dev))
        return -100;
    cudaMemsetAsync(err.p, 0, 16, st);
    const int nsm = sms();
    IAB_TIMED("k_row_shift", st, k_row_shift<<<(unsigned)((M * 32 + 255) / 256), 256, 0, st>>>((int)M, (int)K, A, lda, ob.gamma, sa.as<int>()));
    IAB_TIMED("k_residues_rows", st, k_residues_rows<<<(unsigned)(nsm * 16), 256, 0, st>>>((int)M, (int)K, (int)Kp, A, lda, sa.as<int>(), ra.as<int8_t>()));
    static_assert(sizeof(CUtensorMap) <= sizeof(w->tmA), "tensor map storage");
    if (!make_tmap_3d(reinterpret_cast<CUtensorMap *>(w->tmA), CU_TENSOR_MAP_DATA_TYPE_UINT8, ra.p, (uint64_t)Kp,
                      (uint64_t)M, (uint64_t)L, (uint64_t)Kp, (uint64_t)(Kp * M), oz::BK, oz::BM,
                      CU_TENSOR_MAP_SWIZZLE_128B))
        return -1;
    return 0;
}

int gemm_f64_ozaki_rows_product(int64_t M, const double *A, int64_t lda, const OzakiB &ob, double *C, int64_t ldc,
                                OzakiWork *w, cudaStream_t st)
{
    if (M <= 0) return 0;
    const int L = ob.L;
    const int64_t N = ob.N, K = ob.K, Kp = ob.Kp;
    const int64_t ldr = round_up(N, 16);
    const int nsm = sms();
    I8Params prm;
    memset(&prm, 0, sizeof(prm));
    prm.M = (int)M; prm.N = (int)N; prm.K = (int)K; prm.Kp = (int)Kp; prm.L = L;
    if (w->zs) {
        prm.use_skip = 1;
        prm.zs = *w->zs;
    }
    prm.tiles_m = (int)ceil_div(M, oz::BM); prm.tiles_n = (int)ceil_div(N, oz::BN);
    prm.R = w->rr.as<uint8_t>(); prm.ldr = ldr; prm.err = w->err.as<int>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_i8gemm_mod<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz::SMEM);
        cudaFuncSetAttribute(k_i8gemm_mod<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz::SMEM);
        attr = true;
    }
    const int tiles = L * prm.tiles_m * prm.tiles_n;
    const CUtensorMap &tmA = *reinterpret_cast<const CUtensorMap *>(w->tmA);
    const CUtensorMap &tmB = *reinterpret_cast<const CUtensorMap *>(ob.tmB);
    if (prm.use_skip)
        IAB_TIMED("k_i8gemm_mod", st, k_i8gemm_mod<true, false><<<(unsigned)std::min(tiles, nsm), oz::THREADS, oz::SMEM, st>>>(tmA, tmB, prm));
    else
        IAB_TIMED("k_i8gemm_mod", st, k_i8gemm_mod<false, false><<<(unsigned)std::min(tiles, nsm), oz::THREADS, oz::SMEM, st>>>(tmA, tmB, prm));
    if (w->cimg) {
        launch_crt_img(ob.nc, nsm, w->cimg->g, w->rr.as<uint8_t>(), ldr, w->sa.as<int>(), ob.sb.as<int>(), w->cimg->img,
                       st);
    } else {
        launch_crt(ob.nc, (unsigned)(nsm * 8), (int)M, (int)N, w->rr.as<uint8_t>(), ldr, w->sa.as<int>(), ob.sb.as<int>(), C,
                   ldc, st);
    }
    launch_nonfinite_fix<double>(M, N, K, A, lda, ob.B, ob.ldb, C, ldc, w->sa.as<int>(), ob.sb.as<int>(), kNonFinite, st,
                                 w->cimg);
    return 0;
}

int gemm_f64_ozaki_rows(int64_t M, const double *A, int64_t lda, const OzakiB &ob, double *C, int64_t ldc,
                        OzakiWork *w, cudaStream_t st)
{
    const int r = gemm_f64_ozaki_rows_prep(M, A, lda, ob, w, st);
    return r ? r : gemm_f64_ozaki_rows_product(M, A, lda, ob, C, ldc, w, st);
}

int gemm_f64_ozaki_launch(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
                          double *C, int64_t ldc, int nterms, OzakiWork *w, cudaStream_t st)
{
    if (!device_is_sm100()) return -1;
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (K > 65536 || M > (1 << 30) || N > (1 << 30)) return -1;
    const int r = gemm_f64_ozaki_prepare_b(K, N, B, ldb, nterms, &w->b, st);
    if (r) return r;
    return gemm_f64_ozaki_rows(M, A, lda, w->b, C, ldc, w, st);
}

// ============================================================================ grouped form
// Many independent products C_q = A_q B_q in one pipeline: every kernel of the split
// product runs once over a table of products (OzGProb), with the products' rows, columns,
// residue tasks and GEMM items numbered consecutively, so a batch costs seven launches
// however many products it holds.  The INT8 GEMM reads each product's residues through
// that product's tensor maps, kept in a device array.
__global__ void __launch_bounds__(256) k_row_shift_g(const OzGProb *__restrict__ pr, int np, int64_t rows,
                                                     double gamma, int *__restrict__ shift)
{
    const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= rows) return;
    const OzGProb &q = pr[oz_find(pr, np, g, [](const OzGProb &x) { return x.row0; })];
    const double *row = q.A + (g - q.row0) * q.lda;
    const int K = q.K;
    double mx = 0.0, ss = 0.0;
    for (int k = lane; k < K; k += 32) {
        const double v = fabs(row[k]);
        mx = fmax(mx, v);
        ss = fma(v, v, ss);
    }
    for (int o = 16; o; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if (isnan(ss) || isinf(mx)) {
        if (lane == 0) shift[g] = kNonFinite;
        return;
    }
    double lg = 0.5 * log2(ss);
    if (mx > 0.0 && norm_needs_rescale(mx)) {
        int e;
        frexp(mx, &e);
        double s2 = 0.0;
        for (int k = lane; k < K; k += 32) {
            const double v = ldexp(fabs(row[k]), -e);
            s2 = fma(v, v, s2);
        }
        for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        lg = 0.5 * log2(s2) + e;
    }
    if (lane == 0) shift[g] = pick_shift(mx, lg, gamma);
}

__global__ void __launch_bounds__(256) k_residues_rows_g(const OzGProb *__restrict__ pr, int np, int64_t tasks,
                                                         const int *__restrict__ shift)
{
    const int L = c_crt.L;
    int qh = -1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tasks; t += (int64_t)gridDim.x * blockDim.x) {
        const OzGProb &q = pr[oz_walk(pr, np, t, [](const OzGProb &x) { return x.task_r0; }, qh)];
        const int groups = q.Kp / 8;
        const int64_t lt = t - q.task_r0;
        const int i = (int)(lt / groups), k0 = (int)(lt - (int64_t)i * groups) * 8;
        const int s = shift[q.row0 + i];
        const bool p2 = s >= -1022 && s <= 1023, fin = s != kNonFinite;
        const double f = p2 ? pow2i(s) : 0.0;
        double x[8];
        uint32_t xl[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int k = k0 + u;
            xl[u] = 0u;
            x[u] = k < q.K && fin ? scaled_int(q.A[(int64_t)i * q.lda + k], s, p2, f, xl[u]) : 0.0;
        }
#pragma unroll
        for (int l = 0; l < 16; l++) {
            if (l < L) {
                uint32_t w0 = 0, w1 = 0;
#pragma unroll
                for (int u = 0; u < 4; u++) w0 |= residue_byte(x[u], xl[u], l) << (8 * u);
#pragma unroll
                for (int u = 0; u < 4; u++) w1 |= residue_byte(x[4 + u], xl[4 + u], l) << (8 * u);
                *reinterpret_cast<uint2 *>(q.ra + ((int64_t)l * q.M + i) * q.Kp + k0) = make_uint2(w0, w1);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_col_partial_g(const OzGProb *__restrict__ pr, int np, int64_t cols,
                                                       double *__restrict__ pmax, double *__restrict__ pss)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int seg = blockIdx.y;
    if (g >= cols) return;
    const OzGProb &q = pr[oz_find(pr, np, g, [](const OzGProb &x) { return x.col0; })];
    const int64_t j = g - q.col0;
    const int K = q.K, per = (K + COL_SEGS - 1) / COL_SEGS, k0 = seg * per, k1 = min(K, k0 + per);
    double mx = 0.0, ss = 0.0;
    for (int k = k0; k < k1; k++) {
        const double v = fabs(q.B[(int64_t)k * q.ldb + j]);
        mx = fmax(mx, v);
        ss = fma(v, v, ss);
    }
    pmax[(int64_t)seg * cols + g] = mx;
    pss[(int64_t)seg * cols + g] = ss;
}

__global__ void k_col_shift_g(const OzGProb *__restrict__ pr, int np, int64_t cols, const double *__restrict__ pmax,
                              const double *__restrict__ pss, double gamma, int *__restrict__ shift)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= cols) return;
    const OzGProb &q = pr[oz_find(pr, np, g, [](const OzGProb &x) { return x.col0; })];
    const int64_t j = g - q.col0;
    double mx = 0.0, ss = 0.0;
    for (int sg = 0; sg < COL_SEGS; sg++) {
        mx = fmax(mx, pmax[(int64_t)sg * cols + g]);
        ss += pss[(int64_t)sg * cols + g];
    }
    if (isnan(ss) || isinf(mx)) {
        shift[g] = kNonFinite;
        return;
    }
    double lg = 0.5 * log2(ss);
    if (mx > 0.0 && norm_needs_rescale(mx)) {
        int e;
        frexp(mx, &e);
        double s2 = 0.0;
        for (int k = 0; k < q.K; k++) {
            const double v = ldexp(fabs(q.B[(int64_t)k * q.ldb + j]), -e);
            s2 = fma(v, v, s2);
        }
        lg = 0.5 * log2(s2) + e;
    }
    shift[g] = pick_shift(mx, lg, gamma);
}

// One 64 x 64 tile of one product's B per CTA step (as k_residues_cols).
__global__ void __launch_bounds__(256) k_residues_cols_g(const OzGProb *__restrict__ pr, int np, int64_t tiles,
                                                         const int *__restrict__ shift)
{
    __shared__ double tile[64][65];
    const int L = c_crt.L;
    int qh = -1;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {                 // block-uniform loop
        const OzGProb &q = pr[oz_walk(pr, np, t, [](const OzGProb &x) { return x.tile_c0; }, qh)];
        const int tx_n = (q.N + 63) / 64;
        const int64_t lt = t - q.tile_c0;
        const int ty = (int)(lt / tx_n), tx = (int)(lt - (int64_t)ty * tx_n);
        const int k0 = ty * 64, j0 = tx * 64;
        __syncthreads();                                                       // the previous tile is read
        for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
            const int r = e >> 6, c = e & 63;
            const int k = k0 + r, j = j0 + c;
            tile[r][c] = (k < q.K && j < q.N) ? q.B[(int64_t)k * q.ldb + j] : 0.0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < 64 * 8; e += blockDim.x) {
            const int c = e >> 3, kg = (e & 7) * 8;
            const int j = j0 + c;
            if (j >= q.N || k0 + kg >= q.Kp) continue;
            const int s = shift[q.col0 + j];
            const bool p2 = s >= -1022 && s <= 1023, fin = s != kNonFinite;
            const double f = p2 ? pow2i(s) : 0.0;
            double x[8];
            uint32_t xl[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                xl[u] = 0u;
                x[u] = fin ? scaled_int(tile[kg + u][c], s, p2, f, xl[u]) : 0.0;
            }
#pragma unroll
            for (int l = 0; l < 16; l++) {
                if (l < L) {
                    uint32_t w0 = 0, w1 = 0;
#pragma unroll
                    for (int u = 0; u < 4; u++) w0 |= residue_byte(x[u], xl[u], l) << (8 * u);
#pragma unroll
                    for (int u = 0; u < 4; u++) w1 |= residue_byte(x[4 + u], xl[4 + u], l) << (8 * u);
                    *reinterpret_cast<uint2 *>(q.rb + ((int64_t)l * q.N + j) * q.Kp + k0 + kg) = make_uint2(w0, w1);
                }
            }
        }
    }
}

template <int NC>
__global__ void __launch_bounds__(256) k_crt_g(const OzGProb *__restrict__ pr, int np, int64_t tasks,
                                               const int *__restrict__ sA, const int *__restrict__ sB)
{
    int qh = -1;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tasks; e += (int64_t)gridDim.x * blockDim.x) {
        const OzGProb &q = pr[oz_walk(pr, np, e, [](const OzGProb &x) { return x.crt0; }, qh)];
        const int nq = (q.N + 3) / 4;
        const int64_t lt = e - q.crt0;
        const int i = (int)(lt / nq), j0 = (int)(lt - (int64_t)i * nq) * 4;
        crt_quad<NC>(q.N, q.R, q.ldr, (int64_t)q.M * q.ldr, sA[q.row0 + i], sB + q.col0, q.C, q.ldc, i, j0);
    }
}

// The grouped reconstruction into the products' encoder images: the work units of every image
// numbered consecutively (unit0), each unit as in k_crt_img.
template <int NC>
__global__ void __launch_bounds__(256, 3) k_crt_img_g(const OzGProb *__restrict__ pr, int np, int64_t units,
                                                      const int *__restrict__ sA, const int *__restrict__ sB, int slice)
{
    int qh = -1;
    for (int64_t un = blockIdx.x; un < units; un += gridDim.x) {
        const OzGProb &q = pr[oz_walk(pr, np, un, [](const OzGProb &x) { return x.unit0; }, qh)];
        // the product's fields read once (the image stores could alias the table as far as the
        // compiler can tell, which would reload every field after each store)
        const Geom g = q.gc;
        const uint8_t *R = q.R;
        uint8_t *img = q.cimg;
        const int64_t ldr = q.ldr, row0 = q.row0, col0 = q.col0, unit0 = q.unit0;
        crt_img_unit<NC>(g, R, ldr, sA + row0, sB + col0, img, un - unit0, slice);
    }
}

// Output (i, j) of product q: its dense C, or its encoder image's eight bytes.
__device__ __forceinline__ void oz_store(const OzGProb &q, int64_t i, int64_t j, double v)
{
    if (q.cimg) {
        const uint64_t x = (uint64_t)__double_as_longlong(v);
        uint8_t *o = q.cimg + img_item_offset(q.gc, i, j);
#pragma unroll
        for (int p = 0; p < 8; p++) o[(int64_t)p * q.gc.blockn] = (uint8_t)(x >> (8 * p));
    } else {
        q.C[i * q.ldc + j] = v;
    }
}

// Rows and columns holding NaN or infinity, of every product: one warp per row (global row
// index < rows) or column (the rest), recomputing its outputs as plain dot products.
__global__ void __launch_bounds__(256) k_nonfinite_fix_g(const OzGProb *__restrict__ pr, int np, int64_t rows,
                                                         int64_t cols, const int *__restrict__ sA,
                                                         const int *__restrict__ sB)
{
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w < rows) {
        if (sA[w] != kNonFinite) return;
        const OzGProb &q = pr[oz_find(pr, np, w, [](const OzGProb &x) { return x.row0; })];
        const int64_t i = w - q.row0;
        for (int j = lane; j < q.N; j += 32) {
            double acc = 0;
            for (int k = 0; k < q.K; k++) acc = fma(q.A[i * q.lda + k], q.B[(int64_t)k * q.ldb + j], acc);
            oz_store(q, i, j, acc);
        }
    } else if (w < rows + cols) {
        const int64_t g = w - rows;
        if (sB[g] != kNonFinite) return;
        const OzGProb &q = pr[oz_find(pr, np, g, [](const OzGProb &x) { return x.col0; })];
        const int64_t j = g - q.col0;
        for (int i = lane; i < q.M; i += 32) {
            double acc = 0;
            for (int k = 0; k < q.K; k++) acc = fma(q.A[(int64_t)i * q.lda + k], q.B[(int64_t)k * q.ldb + j], acc);
            oz_store(q, i, j, acc);
        }
    }
}

int gemm_f64_ozaki_grouped_setup(const std::vector<OzGroupItem> &items, int nterms, OzGroupWork *w, cudaStream_t st)
{
    if (!device_is_sm100()) return -1;
    int dev = 0;
    cudaGetDevice(&dev);
    const int L = nterms > 0 ? nterms : 14;
    CrtConst cc;
    if (!set_crt(L, &cc, st)) return -1;
    w->L = L;
    w->nc = cc.nc;
    w->gamma = (cc.log2p - 1.0) / 2.0 - 0.01;
    std::vector<OzGProb> hp;
    int64_t rows = 0, cols = 0, tr = 0, tc = 0, items_total = 0, crt = 0, units = 0;
    size_t ra_bytes = 0, rb_bytes = 0, r_bytes = 0;
    // image output: every item has one (then no item may be skipped: its image must be written)
    const bool img = !items.empty() && items[0].cimg;
    int slice = CRT_SLICE_MAX;
    if (img) {
        int64_t brows = 0;
        for (const OzGroupItem &it : items) brows += it.gc.nchunks * it.gc.nblocks * it.gc.block[0];
        slice = crt_slice_rows(brows, sms());
    }
    for (const OzGroupItem &it : items) {
        if ((it.cimg != nullptr) != img) return -1;
        if (img && (it.M <= 0 || it.N <= 0 || it.K <= 0 || it.gc.shape[0] != it.M || it.gc.shape[1] != it.N ||
                    it.gc.itemsize != 8 || (it.gc.block[1] & 3) || (it.gc.chunk[1] & 3)))
            return -1;
        if (it.M <= 0 || it.N <= 0 || it.K <= 0) continue;
        if (it.K > 65536 || it.M > (1 << 30) || it.N > (1 << 30)) return -1;
        OzGProb q;
        memset(&q, 0, sizeof(q));
        q.M = (int)it.M; q.N = (int)it.N; q.K = (int)it.K; q.Kp = (int)round_up(it.K, oz::BK);
        q.tiles_m = (int)ceil_div(it.M, oz::BM); q.tiles_n = (int)ceil_div(it.N, oz::BN);
        q.row0 = rows; q.col0 = cols; q.task_r0 = tr; q.tile_c0 = tc; q.item0 = items_total; q.crt0 = crt;
        q.A = it.A; q.B = it.B; q.C = it.C; q.lda = it.lda; q.ldb = it.ldb; q.ldc = it.ldc;
        q.ldr = round_up(it.N, 16);
        if (img) {
            q.gc = it.gc;
            q.cimg = it.cimg;
            q.unit0 = units;
            units += it.gc.nchunks * it.gc.nblocks * ceil_div(it.gc.block[0], (int64_t)slice);
        }
        rows += it.M; cols += it.N;
        tr += it.M * (q.Kp / 8);
        tc += ceil_div(it.N, 64) * ceil_div(q.Kp, 64);
        items_total += (int64_t)L * q.tiles_m * q.tiles_n;
        crt += it.M * ceil_div(it.N, 4);
        ra_bytes += round_up((int64_t)L * it.M * q.Kp, 256);
        rb_bytes += round_up((int64_t)L * it.N * q.Kp, 256);
        r_bytes += round_up((int64_t)L * it.M * q.ldr, 256);
        hp.push_back(q);
    }
    w->np = (int)hp.size();
    w->rows = rows; w->cols = cols; w->tasks_r = tr; w->tiles_c = tc; w->items = items_total; w->crt = crt;
    w->img = img;
    w->units = units;
    w->slice = slice;
    if (hp.empty()) return 0;
    if (!w->ra.allocate(ra_bytes, dev) || !w->rb.allocate(rb_bytes, dev) || !w->rr.allocate(r_bytes, dev) ||
        !w->sa.allocate((size_t)rows * 4, dev) || !w->sb.allocate((size_t)cols * 4, dev) ||
        !w->pm.allocate((size_t)COL_SEGS * cols * 8, dev) || !w->ps.allocate((size_t)COL_SEGS * cols * 8, dev) ||
        !w->probs.allocate(sizeof(OzGProb) * hp.size(), dev) ||
        !w->maps.allocate(sizeof(CUtensorMap) * 2 * hp.size(), dev) || !w->err.allocate(16, dev))
        return -100;
    std::vector<CUtensorMap> hm(2 * hp.size());
    size_t oa = 0, ob = 0, orr = 0;
    for (size_t k = 0; k < hp.size(); k++) {
        OzGProb &q = hp[k];
        q.ra = w->ra.as<int8_t>() + oa;
        q.rb = w->rb.as<int8_t>() + ob;
        q.R = w->rr.as<uint8_t>() + orr;
        oa += round_up((int64_t)L * q.M * q.Kp, 256);
        ob += round_up((int64_t)L * q.N * q.Kp, 256);
        orr += round_up((int64_t)L * q.M * q.ldr, 256);
        if (!make_tmap_3d(&hm[2 * k], CU_TENSOR_MAP_DATA_TYPE_UINT8, q.ra, (uint64_t)q.Kp, (uint64_t)q.M, (uint64_t)L,
                          (uint64_t)q.Kp, (uint64_t)q.Kp * q.M, oz::BK, oz::BM, CU_TENSOR_MAP_SWIZZLE_128B) ||
            !make_tmap_3d(&hm[2 * k + 1], CU_TENSOR_MAP_DATA_TYPE_UINT8, q.rb, (uint64_t)q.Kp, (uint64_t)q.N,
                          (uint64_t)L, (uint64_t)q.Kp, (uint64_t)q.Kp * q.N, oz::BK, oz::BN, CU_TENSOR_MAP_SWIZZLE_128B))
            return -1;
    }
    // the tables are written once here, outside any captured work, and only read after
    if (cudaMemcpy(w->probs.p, hp.data(), sizeof(OzGProb) * hp.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(w->maps.p, hm.data(), sizeof(CUtensorMap) * hm.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return -2;
    return 0;
}

int gemm_f64_ozaki_grouped_launch(OzGroupWork *w, cudaStream_t st)
{
    if (w->np == 0) return 0;
    const int nsm = sms();
    const OzGProb *pr = w->probs.as<OzGProb>();
    cudaMemsetAsync(w->err.p, 0, 16, st);
    IAB_TIMED("k_row_shift", st, k_row_shift_g<<<(unsigned)((w->rows * 32 + 255) / 256), 256, 0, st>>>(
        pr, w->np, w->rows, w->gamma, w->sa.as<int>()));
    IAB_TIMED("k_residues_rows", st, k_residues_rows_g<<<(unsigned)(nsm * 16), 256, 0, st>>>(pr, w->np, w->tasks_r,
                                                                                       w->sa.as<int>()));
    IAB_TIMED("k_col_partial", st, k_col_partial_g<<<dim3((unsigned)((w->cols + 255) / 256), COL_SEGS), 256, 0, st>>>(
        pr, w->np, w->cols, w->pm.as<double>(), w->ps.as<double>()));
    IAB_TIMED("k_col_shift", st, k_col_shift_g<<<(unsigned)((w->cols + 255) / 256), 256, 0, st>>>(
        pr, w->np, w->cols, w->pm.as<double>(), w->ps.as<double>(), w->gamma, w->sb.as<int>()));
    IAB_TIMED("k_residues_cols", st, k_residues_cols_g<<<(unsigned)std::min<int64_t>(w->tiles_c, (int64_t)nsm * 8), 256, 0, st>>>(
        pr, w->np, w->tiles_c, w->sb.as<int>()));
    I8Params prm;
    memset(&prm, 0, sizeof(prm));
    prm.L = w->L;
    prm.err = w->err.as<int>();
    prm.probs = pr;
    prm.nprob = w->np;
    prm.total = w->items;
    prm.maps = w->maps.as<CUtensorMap>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_i8gemm_mod<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz::SMEM);
        attr = true;
    }
    // the tensor maps of the kernel parameters are unused in the grouped form
    CUtensorMap unused;
    memset(&unused, 0, sizeof(unused));
    IAB_TIMED("k_i8gemm_mod", st, k_i8gemm_mod<false, true><<<(unsigned)std::min<int64_t>(w->items, nsm), oz::threads_of<true>(),
                                                               oz::SMEM, st>>>(unused, unused, prm));
    const unsigned cg = (unsigned)std::min<int64_t>((w->crt + 255) / 256, (int64_t)nsm * 8);
    if (w->img) {
        const unsigned ig = (unsigned)std::max<int64_t>(1, std::min<int64_t>(w->units, (int64_t)nsm * 8));
        switch (w->nc) {
        case 1: IAB_TIMED("k_crt_img", st, k_crt_img_g<1><<<ig, 256, 0, st>>>(pr, w->np, w->units, w->sa.as<int>(), w->sb.as<int>(), w->slice)); break;
        case 2: IAB_TIMED("k_crt_img", st, k_crt_img_g<2><<<ig, 256, 0, st>>>(pr, w->np, w->units, w->sa.as<int>(), w->sb.as<int>(), w->slice)); break;
        case 3: IAB_TIMED("k_crt_img", st, k_crt_img_g<3><<<ig, 256, 0, st>>>(pr, w->np, w->units, w->sa.as<int>(), w->sb.as<int>(), w->slice)); break;
        default: IAB_TIMED("k_crt_img", st, k_crt_img_g<4><<<ig, 256, 0, st>>>(pr, w->np, w->units, w->sa.as<int>(), w->sb.as<int>(), w->slice)); break;
        }
    } else {
        switch (w->nc) {
        case 1: IAB_TIMED("k_crt", st, k_crt_g<1><<<cg, 256, 0, st>>>(pr, w->np, w->crt, w->sa.as<int>(), w->sb.as<int>())); break;
        case 2: IAB_TIMED("k_crt", st, k_crt_g<2><<<cg, 256, 0, st>>>(pr, w->np, w->crt, w->sa.as<int>(), w->sb.as<int>())); break;
        case 3: IAB_TIMED("k_crt", st, k_crt_g<3><<<cg, 256, 0, st>>>(pr, w->np, w->crt, w->sa.as<int>(), w->sb.as<int>())); break;
        default: IAB_TIMED("k_crt", st, k_crt_g<4><<<cg, 256, 0, st>>>(pr, w->np, w->crt, w->sa.as<int>(), w->sb.as<int>())); break;
        }
    }
    IAB_TIMED("k_nonfinite_fix", st, k_nonfinite_fix_g<<<(unsigned)(((w->rows + w->cols) * 32 + 255) / 256), 256, 0, st>>>(
        pr, w->np, w->rows, w->cols, w->sa.as<int>(), w->sb.as<int>()));
    return 0;
}

int gemm_f64_ozaki_grouped_finish(OzGroupWork *w, cudaStream_t st)
{
    if (!w->err.p) return 0;
    int h_err = 0;
    cudaMemcpyAsync(&h_err, w->err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    return h_err ? -3 : 0;
}

// Normwise difference over many products (the split form's autotuner): per product, one CTA
// sums (x - y)^2 and y^2 over its M x N outputs.
__global__ void __launch_bounds__(256) k_normdiff(const DiffItem *__restrict__ it, double *__restrict__ out)
{
    __shared__ double s1[256], s2[256];
    const DiffItem d = it[blockIdx.x];
    double a = 0.0, b = 0.0;
    for (int64_t e = threadIdx.x; e < d.M * d.N; e += blockDim.x) {
        const int64_t i = e / d.N, j = e - i * d.N;
        const double x = d.X[i * d.ld + j], y = d.Y[i * d.ld + j];
        a = fma(x - y, x - y, a);
        b = fma(y, y, b);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) { s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[2 * blockIdx.x] = s1[0]; out[2 * blockIdx.x + 1] = s2[0]; }
}

double normwise_diff_grouped(const std::vector<DiffItem> &items, cudaStream_t st)
{
    if (items.empty()) return 0.0;
    int dev = 0;
    cudaGetDevice(&dev);
    DevBuf di, dout;
    if (!di.allocate(sizeof(DiffItem) * items.size(), dev) || !dout.allocate(16 * items.size(), dev)) return -1.0;
    cudaMemcpyAsync(di.p, items.data(), sizeof(DiffItem) * items.size(), cudaMemcpyHostToDevice, st);
    IAB_TIMED("k_normdiff", st, k_normdiff<<<(unsigned)items.size(), 256, 0, st>>>(di.as<DiffItem>(), dout.as<double>()));
    std::vector<double> h(2 * items.size());
    cudaMemcpyAsync(h.data(), dout.p, 16 * items.size(), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1.0;
    double a = 0.0, b = 0.0;
    for (size_t i = 0; i < items.size(); i++) { a += h[2 * i]; b += h[2 * i + 1]; }
    return b > 0.0 ? sqrt(a / b) : sqrt(a);
}

// ============================================================================ float32: BF16 splits
// A float32 x is split into bfloat16 words.  Two words: hi = bf16(x), lo = bf16(x - hi)
// hold x to about 2^-17 relative, and C = A_lo B_hi + A_hi B_lo + A_hi B_hi (three
// products; lo x lo is below that precision).  Three words: x1 = bf16(x),
// x2 = bf16(x - x1), x3 = bf16(x - x1 - x2) hold x to about 2^-25 (every difference is
// exact in float32), and C = A3 B1 + A1 B3 + A2 B2 + A2 B1 + A1 B2 + A1 B1 (six products,
// the dropped ones below float32 resolution).  Each product is a tcgen05.mma kind::f16
// pass over K (bf16 x bf16 -> fp32 in TMEM).
//
// Accuracy of the sums.  The tensor core adds each K = 16 slice into its FP32 accumulator
// with a truncating alignment, so one long accumulation loses precision in proportion to
// its length (measured on a B200: normwise 4.4e-6 at K = 4096 with exact bf16 operands,
// against 1.1e-6 for FFMA).  Two changes keep the error at float32 level:
//   - passes run smallest first, so the small cross products are never added to an
//     accumulator that already holds the large A1 B1 sums;
//   - the pass sequence is cut into segments of SEG_KT k-tiles (512 K).  Each segment
//     starts a fresh TMEM accumulator (two alternate, so the tensor core never waits for
//     the drain), and the epilogue warps add every segment into FP32 registers with
//     round-to-nearest.  The truncation error is then bounded by one segment's length
//     instead of the whole K.
namespace bfs {
constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;        // BK bf16 = 128 bytes per row
constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int EPI_WARPS = 8;                                  // two per TMEM lane quarter, 128 columns each
constexpr int THREADS = 64 + 32 * EPI_WARPS;
constexpr int SMEM = 1024 + STAGES * STAGE_BYTES + 256;
constexpr int SEG_KT = 8;                                     // k-tiles per accumulation segment (512 K)
constexpr int MAX_PASS = 6;
constexpr uint32_t IDESC = tc::make_idesc(1 /*F32*/, 1 /*BF16*/, 1 /*BF16*/, BM, BN);
}

struct BfsParams {
    int M, N, Kp, tiles_m, tiles_n;
    int npass;                         // 3 or 6 products
    int pa[bfs::MAX_PASS], pb[bfs::MAX_PASS];   // word plane of A and of B in each pass
    float *C;
    int64_t ldc;
    int *err;
};

__device__ __forceinline__ void split_words(float x, int words, __nv_bfloat16 (&w)[3])
{
    w[0] = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(w[0]);                  // exact
    w[1] = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(w[1]);                 // exact
    w[2] = words == 3 ? __float2bfloat16_rn(r2) : __float2bfloat16_rn(0.f);
}

// Row-major A (M x K) -> `words` planes [words][M][Kp] of bf16, K padded with zeros.
// A row (column) holding a value whose leading bf16 word is not finite (NaN, infinity, or
// a float beyond bf16's range) sets its flag; its outputs are recomputed by
// k_nonfinite_fix.
__global__ void __launch_bounds__(256) k_split_rows(int M, int K, int Kp, int words, const float *__restrict__ A,
                                                    int64_t lda, __nv_bfloat16 *__restrict__ P, int *__restrict__ rflag)
{
    const int groups = Kp / 4;
    const int64_t total = (int64_t)M * groups, plane = (int64_t)M * Kp;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / groups), k0 = (int)(t - (int64_t)i * groups) * 4;
        __nv_bfloat16 h[3][4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const float x = k0 + u < K ? A[(int64_t)i * lda + k0 + u] : 0.f;
            __nv_bfloat16 w[3];
            split_words(x, words, w);
            h[0][u] = w[0]; h[1][u] = w[1]; h[2][u] = w[2];
            if (!isfinite(__bfloat162float(w[0]))) rflag[i] = 1;
        }
        __nv_bfloat16 *ph = P + (int64_t)i * Kp + k0;
        for (int wd = 0; wd < words; wd++)
            *reinterpret_cast<uint2 *>(ph + wd * plane) = *reinterpret_cast<const uint2 *>(h[wd]);
    }
}

// Row-major B (K x N) -> `words` planes [words][N][Kp] of bf16 (transposed, K-major).
__global__ void __launch_bounds__(256) k_split_cols(int K, int N, int Kp, int words, const float *__restrict__ B,
                                                    int64_t ldb, __nv_bfloat16 *__restrict__ P, int *__restrict__ cflag)
{
    __shared__ float tile[64][65];
    const int k0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
        const int r = e >> 6, c = e & 63;
        const int k = k0 + r, j = j0 + c;
        tile[r][c] = (k < K && j < N) ? B[(int64_t)k * ldb + j] : 0.f;
    }
    __syncthreads();
    const int64_t plane = (int64_t)N * Kp;
    for (int e = threadIdx.x; e < 64 * 16; e += blockDim.x) {
        const int c = e >> 4, kg = (e & 15) * 4;
        const int j = j0 + c;
        if (j >= N || k0 + kg >= Kp) continue;
        __nv_bfloat16 h[3][4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            __nv_bfloat16 w[3];
            split_words(tile[kg + u][c], words, w);
            h[0][u] = w[0]; h[1][u] = w[1]; h[2][u] = w[2];
            if (!isfinite(__bfloat162float(w[0]))) cflag[j] = 1;
        }
        __nv_bfloat16 *ph = P + (int64_t)j * Kp + k0 + kg;
        for (int wd = 0; wd < words; wd++)
            *reinterpret_cast<uint2 *>(ph + wd * plane) = *reinterpret_cast<const uint2 *>(h[wd]);
    }
}

// Persistent, warp-specialised: warp 0 loads (TMA), warp 1 issues the MMAs, warps 2-9
// drain.  Per output tile the k-tile sequence of all passes (pass-major) is cut into
// segments of SEG_KT k-tiles; each segment accumulates into one of two 128 x 256 FP32
// TMEM accumulators from zero, and the epilogue adds it into FP32 registers (warp w reads
// TMEM lane quarter w % 4, columns 128 (w - 2) / 4 .. + 127), storing the tile as float32
// rows of C after its last segment.
__global__ void __launch_bounds__(bfs::THREADS, 1) k_bf16s_gemm(const __grid_constant__ CUtensorMap tmA,
                                                                 const __grid_constant__ CUtensorMap tmB, BfsParams p)
{
    using namespace bfs;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA = smem, *sB = smem + STAGES * A_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { tc::mbar_init(&full[s], 1); tc::mbar_init(&empty[s], 1); }
        for (int b = 0; b < 2; b++) { tc::mbar_init(&tfull[b], 1); tc::mbar_init(&tempty[b], EPI_WARPS); }
        tc::mbar_init(drain, 1);
        tc::fence_barrier_init();
        tc::tma_prefetch_desc(&tmA);
        tc::tma_prefetch_desc(&tmB);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int total = p.tiles_m * p.tiles_n;
    const int ktiles = p.Kp / BK;
    const int steps = p.npass * ktiles;                  // k-tiles per output tile
    const int nseg = (steps + SEG_KT - 1) / SEG_KT;

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
                int tm, tn;
                tile_of(t, p.tiles_m, p.tiles_n, tm, tn);
                for (int st = 0; st < steps; st++) {
                    const int pass = st / ktiles, kt = st - pass * ktiles;
                    if (!tc::mbar_wait(&empty[stage], phase ^ 1, p.err)) { ok = false; break; }
                    tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                    tc::tma_load_3d(sA + stage * A_BYTES, &tmA, kt * BK, tm * BM, p.pa[pass], &full[stage]);
                    tc::tma_load_3d(sB + stage * B_BYTES, &tmB, kt * BK, tn * BN, p.pb[pass], &full[stage]);
                    issued++;
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            }
            for (int64_t it = issued > STAGES ? issued - STAGES : 0; it < issued; it++)
                tc::mbar_wait(&full[it % STAGES], (uint32_t)((it / STAGES) & 1), p.err, 1u << 20);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0, acc = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
                for (int sg = 0; sg < nseg && ok; sg++) {
                    if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, p.err)) { ok = false; break; }
                    tc::tc_fence_after();
                    const uint32_t dt = tmem_base + (uint32_t)(acc * BN);
                    const int s0 = sg * SEG_KT, s1 = min(steps, s0 + SEG_KT);
                    for (int st = s0; st < s1; st++) {
                        if (!tc::mbar_wait(&full[stage], phase, p.err)) { ok = false; break; }
                        tc::tc_fence_after();
                        const uint32_t a0 = tc::smem_addr(sA + stage * A_BYTES), b0 = tc::smem_addr(sB + stage * B_BYTES);
#pragma unroll
                        for (int kk = 0; kk < BK / 16; kk++) {
                            tc::mma_f16(dt, tc::sw128_kmajor_desc(a0 + kk * 32), tc::sw128_kmajor_desc(b0 + kk * 32),
                                        IDESC, (st != s0 || kk != 0) ? 1u : 0u);
                        }
                        tc::tc_commit(&empty[stage]);
                        if (++stage == STAGES) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    tc::tc_commit(&tfull[acc]);
                    if (++acc == 2) { acc = 0; acc_phase ^= 1; }
                }
            }
            tc::tc_commit(drain);
            tc::mbar_wait(drain, 0, p.err, 1u << 20);
        }
    } else {
        const int q = warp & 3;                          // TMEM lane quarter this warp may access
        const int half = (warp - 2) >> 2;                // columns 128 * half .. + 127
        int acc = 0;
        uint32_t acc_phase = 0;
        bool ok = true;
        float sum[128];
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int tm, tn;
            tile_of(t, p.tiles_m, p.tiles_n, tm, tn);
#pragma unroll
            for (int u = 0; u < 128; u++) sum[u] = 0.f;
            for (int sg = 0; sg < nseg; sg++) {
                if (!tc::mbar_wait(&tfull[acc], acc_phase, p.err)) { ok = false; break; }
                tc::tc_fence_after();
                const uint32_t ta = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN + half * 128);
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    uint32_t v[32];
                    tc::tmem_ld32(ta + (uint32_t)(c * 32), v);
#pragma unroll
                    for (int u = 0; u < 32; u++) sum[c * 32 + u] = __fadd_rn(sum[c * 32 + u], __uint_as_float(v[u]));
                }
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&tempty[acc]);
                if (++acc == 2) { acc = 0; acc_phase ^= 1; }
            }
            if (!ok) break;
            const int row = tm * BM + q * 32 + lane;
            const int col0 = tn * BN + half * 128;
            if (row < p.M) {
                float *out = p.C + (int64_t)row * p.ldc + col0;
                if (col0 + 128 <= p.N && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
                    float4 *o4 = reinterpret_cast<float4 *>(out);
#pragma unroll
                    for (int u = 0; u < 32; u++)
                        o4[u] = make_float4(sum[4 * u], sum[4 * u + 1], sum[4 * u + 2], sum[4 * u + 3]);
                } else {
#pragma unroll
                    for (int b = 0; b < 128; b++)
                        if (col0 + b < p.N) out[b] = sum[b];
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 1) tc::tmem_dealloc(tmem_base, 512);
}

int gemm_f32_bf16_split(int64_t M, int64_t N, int64_t K, const float *A, int64_t lda, const float *B, int64_t ldb,
                        float *C, int64_t ldc, int products, cudaStream_t st)
{
    if (!device_is_sm100()) return -1;
    if (products == 0) products = 6;
    if (products != 3 && products != 6) return -4;
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (M > (1 << 30) || N > (1 << 30) || K > (1 << 30)) return -1;
    int dev = 0;
    cudaGetDevice(&dev);
    const int words = products == 6 ? 3 : 2;
    const int64_t Kp = round_up(K, bfs::BK);
    DevBuf pa, pb, err, flg;
    if (!pa.allocate((size_t)(words * M * Kp * 2), dev) || !pb.allocate((size_t)(words * N * Kp * 2), dev) ||
        !err.allocate(16, dev) || !flg.allocate((size_t)(M + N) * 4, dev))
        return -100;
    cudaMemsetAsync(err.p, 0, 16, st);
    cudaMemsetAsync(flg.p, 0, (size_t)(M + N) * 4, st);
    int *rflag = flg.as<int>(), *cflag = rflag + M;
    const int nsm = sms();
    IAB_TIMED("k_split_rows", st, k_split_rows<<<(unsigned)(nsm * 16), 256, 0, st>>>(
        (int)M, (int)K, (int)Kp, words, A, lda, pa.as<__nv_bfloat16>(), rflag));
    IAB_TIMED("k_split_cols", st, k_split_cols<<<dim3((unsigned)((N + 63) / 64), (unsigned)((Kp + 63) / 64)), 256, 0, st>>>(
        (int)K, (int)N, (int)Kp, words, B, ldb, pb.as<__nv_bfloat16>(), cflag));
    CUtensorMap tmA, tmB;
    if (!make_tmap_3d(&tmA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, pa.p, (uint64_t)Kp, (uint64_t)M, (uint64_t)words,
                      (uint64_t)Kp * 2, (uint64_t)(Kp * M * 2), bfs::BK, bfs::BM, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !make_tmap_3d(&tmB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, pb.p, (uint64_t)Kp, (uint64_t)N, (uint64_t)words,
                      (uint64_t)Kp * 2, (uint64_t)(Kp * N * 2), bfs::BK, bfs::BN, CU_TENSOR_MAP_SWIZZLE_128B))
        return -1;
    BfsParams prm;
    memset(&prm, 0, sizeof(prm));
    prm.M = (int)M; prm.N = (int)N; prm.Kp = (int)Kp;
    prm.tiles_m = (int)ceil_div(M, bfs::BM); prm.tiles_n = (int)ceil_div(N, bfs::BN);
    // word planes of each pass, smallest products first (A word, B word; 0 = leading)
    static const int kPa3[3] = {1, 0, 0}, kPb3[3] = {0, 1, 0};
    static const int kPa6[6] = {2, 0, 1, 1, 0, 0}, kPb6[6] = {0, 2, 1, 0, 1, 0};
    prm.npass = products;
    for (int i = 0; i < products; i++) {
        prm.pa[i] = products == 6 ? kPa6[i] : kPa3[i];
        prm.pb[i] = products == 6 ? kPb6[i] : kPb3[i];
    }
    prm.C = C; prm.ldc = ldc; prm.err = err.as<int>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_bf16s_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, bfs::SMEM);
        attr = true;
    }
    const int tiles = prm.tiles_m * prm.tiles_n;
    IAB_TIMED("k_bf16s_gemm", st, k_bf16s_gemm<<<(unsigned)std::min(tiles, nsm), bfs::THREADS, bfs::SMEM, st>>>(tmA, tmB, prm));
    launch_nonfinite_fix<float>(M, N, K, A, lda, B, ldb, C, ldc, rflag, cflag, 1, st);
    int h_err = 0;
    cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -2;
    return h_err ? -3 : 0;
}

}  // namespace iab
