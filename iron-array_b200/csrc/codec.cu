// Blosc2 LZ4+SHUFFLE chunk decoder and encoder on the GPU.
//
// Replaces, for ironArray's matmul path, the Blosc2 block decode done by
// blosc2_getitem_ctx / blosc2_decompress_ctx (src/linalg/iarray_gemm.c:259-274,
// src/linalg/iarray_gemm_a.c:316, src/linalg/iarray_gemv.c:194-209, and the panel
// slices of src/iarray_container.c:628-737) and the output encode done by
// blosc2_compress_ctx (src/linalg/iarray_gemm.c:405-422, src/linalg/matmul/gemm.c:216-233),
// plus Caterva's padded blocked layout (iarray_from_buffer / iarray_to_buffer,
// src/iarray_constructor.c:218-305).
//
// Decode = parse (one thread per block walks its stream headers and queues its LZ4 streams)
// -> LZ4 (one CTA per LZ4 stream from a job queue that may span several containers; each
// window of the stream decoded in parallel: token chain by pointer doubling, output resolved
// in shared memory by pointer jumping) -> unshuffle/scatter (slices of interior blocks staged
// in shared memory by bulk asynchronous copies, items written to the dense row-major array;
// a general path for the other blocks).  Raw and run streams are never copied before the
// scatter.
//
// Encode = gather/shuffle (dense -> byte-plane image) -> LZ4 -> layout (per chunk: stream
// kinds, offsets, memcpy fallback; exclusive scan of chunk sizes) -> emit (copy payloads
// into the final contiguous chunk buffer).  Two LZ4 encoders: one warp per stream
// reproducing liblz4 1.9.4 LZ4_compress_fast(acceleration 1) output byte for byte (the codec
// c-blosc2 calls for BLOSC_LZ4: 16 KiB hash table in shared memory, 32 match probes
// evaluated per step), and a parallel-parse encoder (one CTA per stream, valid LZ4 with
// different bytes).  Stream-kind selection (zero/run, raw when LZ4 does not fit, memcpyed
// chunk when the output would exceed nbytes + 32) follows c-blosc2's blosc_c rules.
#include <cuda_runtime.h>
#include <stdint.h>

#include "bytes.cuh"
#include "common.cuh"
#include "tc_common.cuh"

namespace iab {

#define FULLMASK 0xffffffffu

__device__ __forceinline__ int32_t ld_s32(const uint8_t *p)
{
    return (int32_t)((uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24));
}

__device__ __forceinline__ void dev_fail(int *err, int code) { atomicCAS(err, 0, code); }

// ============================================================================ decode
// D0: parse one (chunk, block) per thread.
// zf (optional): per (chunk, block) zero flags of the reference's block-pair products:
// bit 0 = block_is_zeros (src/linalg/iarray_gemm.c:28-77: no memcpyed or special chunk, and
// the first typesize csize words from the block's bstart are all 0: Blosc2 v5 chunks always
// carry the flag bit the reference reads as "split"), bit 1 = chunk_is_zeros (:17-26:
// special value ZERO); nzero counts the flagged blocks.
__device__ __forceinline__ void parse_block(const Geom &g, const uint8_t *__restrict__ ch, const int64_t *__restrict__ off,
                                            const int32_t *__restrict__ len, BlockDesc *bd, StreamDesc *sd,
                                            Lz4Job *jobs, int *njobs, int64_t jcap, int *err, uint8_t *scratch,
                                            uint8_t *zf, int *nzero, int64_t t)
{
    do {
        const int64_t c = t / g.nblocks, b = t % g.nblocks;
        const uint8_t *p = ch + off[c];
        const int32_t clen = len[c];
        BlockDesc d;
        d.mode = BM_PLAIN; d.nstreams = 1; d.neblock = (int32_t)g.blocksize; d.pad = 0; d.value_src = 0;
        StreamDesc *s = sd + t * 8;
        for (int j = 0; j < 8; j++) { s[j].kind = SK_RUN; s[j].len = 0; s[j].src = 0; }
        bool ok = clen >= 32;
        int32_t nbytes = 0, bsz = 0, cbytes = 0;
        uint8_t flags = 0, ts = 0, bflags = 0;
        if (ok) {
            flags = p[2]; ts = p[3]; bflags = p[31];
            nbytes = ld_s32(p + 4); bsz = ld_s32(p + 8); cbytes = ld_s32(p + 12);
            ok = (flags & 0x05) == 0x05 && nbytes == g.chunk_nbytes && cbytes >= 32 && cbytes <= clen;
        }
        if (!ok) { dev_fail(err, DE_HEADER); bd[t] = d; if (zf) zf[t] = 0; continue; }
        const int special = (bflags >> 4) & 7;
        if (zf) {
            uint8_t zflag = special == 1 ? 2 : 0;
            if (!special && !(flags & 0x02) && 32 + 4 * (b + 1) <= cbytes) {
                const int64_t q0 = ld_s32(p + 32 + 4 * b);
                bool z = q0 >= 32 && q0 + 4 * (int64_t)ts <= cbytes;
                for (int j = 0; z && j < ts; j++) z = ld_s32(p + q0 + 4 * j) == 0;
                if (z) zflag |= 1;
            }
            zf[t] = zflag;
            if (zflag && nzero) atomicAdd(nzero, 1);
        }
        if (special) {
            if (special == 2) d.mode = BM_NAN;
            else if (special == 3) {
                if (cbytes < 32 + (int32_t)g.itemsize) dev_fail(err, DE_HEADER);
                d.mode = BM_VALUE; d.value_src = off[c] + 32;
            } else if (special != 1 && special != 4) dev_fail(err, DE_HEADER);
            bd[t] = d;
            continue;
        }
        if (flags & 0x02) {                      // memcpyed: raw blocked items
            if (cbytes < 32 + nbytes) { dev_fail(err, DE_BOUNDS); bd[t] = d; continue; }
            s[0].kind = SK_RAW; s[0].len = (int32_t)g.blocksize; s[0].src = off[c] + 32 + b * g.blocksize;
            bd[t] = d;
            continue;
        }
        // filters: only SHUFFLE (slot 5 == 1) or none are produced on this path
        bool filt_ok = p[16] == 0 && p[17] == 0 && p[18] == 0 && p[19] == 0 && p[20] == 0 && p[21] <= 1;
        if (bsz != g.blocksize || ts != g.itemsize || !filt_ok) { dev_fail(err, DE_HEADER); bd[t] = d; continue; }
        const bool split = !(flags & 0x10);
        const bool shuffle = p[21] == 1 && ts > 1;
        const int nstreams = split ? ts : 1;
        const int neblock = (int)(g.blocksize / nstreams);
        d.mode = shuffle ? BM_SHUFFLED : BM_PLAIN;
        d.nstreams = nstreams; d.neblock = neblock;
        const int64_t bs_end = 32 + 4 * g.nblocks;
        if (bs_end > cbytes) { d.mode = BM_PLAIN; dev_fail(err, DE_BOUNDS); bd[t] = d; continue; }
        int64_t q = ld_s32(p + 32 + 4 * b);
        if (q < bs_end || q >= cbytes) { d.mode = BM_PLAIN; dev_fail(err, DE_BOUNDS); bd[t] = d; continue; }
        for (int j = 0; j < nstreams; j++) {
            if (q + 4 > cbytes) { dev_fail(err, DE_BOUNDS); ok = false; break; }
            const int32_t cs = ld_s32(p + q);
            q += 4;
            if (cs == 0) { s[j].kind = SK_RUN; s[j].len = 0; s[j].src = 0; continue; }
            if (cs < 0) {
                if (q + 1 > cbytes || !(p[q] & 1) || cs < -255) { dev_fail(err, DE_RUN_TOKEN); ok = false; break; }
                q += 1;
                s[j].kind = SK_RUN; s[j].len = -cs; s[j].src = 0;
                continue;
            }
            if (q + cs > cbytes || cs > neblock) { dev_fail(err, DE_BOUNDS); ok = false; break; }
            s[j].src = off[c] + q;
            s[j].len = cs;
            if (cs == neblock) {
                s[j].kind = SK_RAW;
            } else {
                s[j].kind = SK_LZ4;
                const int k = atomicAdd(njobs, 1);
                if (k < jcap) {
                    Lz4Job jb;
                    jb.src = ch + off[c] + q; jb.dst = scratch + t * g.blocksize + (int64_t)j * neblock; jb.err = err;
                    jb.csize = cs; jb.dlen = neblock;
                    jobs[k] = jb;
                } else {
                    dev_fail(err, DE_BOUNDS);                            // queue full: left undecoded
                }
            }
            q += cs;
        }
        if (!ok) { for (int j = 0; j < nstreams; j++) { s[j].kind = SK_RUN; s[j].len = 0; } }
        bd[t] = d;
    } while (false);
}

__global__ void k_parse(Geom g, const uint8_t *__restrict__ ch, const int64_t *__restrict__ off,
                        const int32_t *__restrict__ len, BlockDesc *bd, StreamDesc *sd, Lz4Job *jobs,
                        int *njobs, int64_t jcap, int *err, uint8_t *scratch, uint8_t *zf, int *nzero)
{
    const int64_t total = g.nchunks * g.nblocks;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x)
        parse_block(g, ch, off, len, bd, sd, jobs, njobs, jcap, err, scratch, zf, nzero, t);
}

// D1: LZ4 stream decode, one CTA (256 threads) per stream, streams handed out
// dynamically from a job queue (which may hold the streams of several containers: each job
// carries its source, destination and status word).  The stream is consumed in windows of up to DW compressed bytes staged in
// shared memory, and each window is decoded without any serial walk:
//  1. for every byte q of the window, next[q] = where the following token would start if
//     a sequence began at q (STOP when that sequence does not end inside the window,
//     ENDS when it is the stream's last, literal-only sequence);
//  2. the chain of token positions from the window start is built by pointer doubling
//     (next, next^2, next^4, ... composed in two ping-pong tables, the chain doubled
//     alongside), so the window's sequences are all located in O(log) parallel steps;
//  3. their literal and match lengths are read in parallel and an exclusive scan gives
//     each sequence's output offset;
//  4. the output is resolved in groups of at most DCAP bytes in shared memory: a literal
//     byte takes its value from the window, a match byte points at its source (a source
//     inside the same match is folded back below the match start modulo the offset), and
//     pointer jumping settles every byte in O(log depth) rounds; sources before the group
//     are read from the already written output;
//  5. a sequence with more than DCAP output bytes is copied straight in global memory
//     (all its sources lie before its own match start), and a sequence too long for a
//     window is decoded alone with its header read from global memory.
namespace dcta {
constexpr int THREADS = 256;
constexpr int DW = 2048;                   // compressed bytes per window
constexpr int MAXS = DW / 3 + 2;           // sequences per window (a non-final one takes >= 3 bytes)
constexpr int PATH = 1024;                 // >= 2 * the largest power of two below MAXS + 1
constexpr int HB = 4096;                   // output history kept in shared memory for match sources
constexpr int LONGSEQ = 64;                // longer sequences are filled by the whole CTA
constexpr int DCAP = 4096;                 // output bytes resolved in shared memory at once
constexpr int WALK_MAX = 24;               // chains of at most this many sequences are walked
constexpr uint16_t STOP = 0xFFFF, ENDS = 0xFFFE;
constexpr uint32_t RES = 0x80000000u;      // resolved output byte (value in the low 8 bits)
struct Smem {
    union {
        uint32_t st[DCAP];                 // per output byte: RES | value, or the source's index
        uint16_t J[2][DW];                 // next-token tables (dead once the window's chain is known)
    };
    int32_t ostart[MAXS + 1];              // output offset of each sequence in the window
    int32_t llen[MAXS];
    int32_t mlen[MAXS];
    uint16_t lpos[MAXS];
    uint16_t off[MAXS];
    uint16_t path[PATH];
    uint8_t win[DW + 16];
    uint8_t hist[HB];                      // the last HB output bytes (ring, by absolute position)
    int32_t longs[DCAP / (LONGSEQ + 1) + 1];  // sequences of a group longer than LONGSEQ bytes
    int32_t nlong;
    int32_t wsum[THREADS / 32];
    int32_t scal[9];
};
}  // namespace dcta

// next[q] for a sequence starting at window offset q (n valid bytes, rem bytes left in
// the stream from the window start).
__device__ __forceinline__ uint16_t dcta_next(const uint8_t *win, int q, int n, int rem)
{
    int r = q + 1;
    const int tok = win[q];
    int lit = tok >> 4;
    if (lit == 15) {
        int b = 255;
        while (b == 255) {
            if (r >= n) return dcta::STOP;
            b = win[r++];
            lit += b;
        }
    }
    r += lit;
    if (r > n) return dcta::STOP;
    if (r == rem) return dcta::ENDS;      // literals reach the stream end: the last sequence
    if (r + 2 > n) return dcta::STOP;
    r += 2;
    if ((tok & 15) == 15) {
        int b = 255;
        while (b == 255) {
            if (r >= n) return dcta::STOP;
            b = win[r++];
        }
    }
    return (uint16_t)r;                   // r <= n; r == n: the next token starts the next window
}

__global__ void __launch_bounds__(dcta::THREADS, 6) k_lz4_decode_cta(const Lz4Job *__restrict__ jobs,
                                                                  const int *__restrict__ njobs_p, int64_t jcap,
                                                                  unsigned *next_job)
{
    using namespace dcta;
    extern __shared__ __align__(16) uint8_t sm_dcta[];
    Smem &S = *reinterpret_cast<Smem *>(sm_dcta);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int njobs = (int)min((int64_t)*njobs_p, jcap);
    if (tid == 0) S.nlong = 0;                     // first use follows the barriers below
    for (;;) {
        __syncthreads();
        if (tid == 0) S.scal[0] = (int)atomicAdd(next_job, 1u);
        __syncthreads();
        const int jid = S.scal[0];
        if (jid >= njobs) break;
        const Lz4Job jb = jobs[jid];
        const uint8_t *__restrict__ in = jb.src;
        const int isz = jb.csize;
        uint8_t *out = jb.dst;
        const int osz = jb.dlen;
        int p = 0, op = 0;                 // window start in the input, output written so far
        int hist_from = 0;                 // S.hist holds output bytes [hist_from, written)
        bool bad = false, done = false;    // block-uniform
        bool walk = true;                  // block-uniform: walk this window's chain (sparse windows)
        while (!done && !bad) {
            const int rem = isz - p, n = min(DW, rem);
            __syncthreads();
            {                                          // every load issued before any store
                uint8_t v[DW / THREADS];
#pragma unroll
                for (int k = 0; k < DW / THREADS; k++) {
                    const int x = tid + k * THREADS;
                    v[k] = x < n ? __ldg(in + p + x) : (uint8_t)0;
                }
#pragma unroll
                for (int k = 0; k < DW / THREADS; k++) S.win[tid + k * THREADS] = v[k];
            }
            __syncthreads();
            // Windows of few sequences (long literal runs, long matches): one thread walks the
            // chain of token positions, at most WALK_MAX steps; when the chain does not leave the
            // window by then, and for the windows that follow a dense one, the chain is built by
            // doubling.  Both leave path[0 .. cnt) = token positions, path[cnt] >= n.
            int cnt = -1;
            if (walk) {
                if (tid == 0) {
                    int q = 0, k = 0, res = -1;
                    S.path[0] = 0;
                    for (;;) {
                        const uint16_t v = dcta_next(S.win, q, n, rem);
                        S.path[++k] = v;
                        if (v >= n) { res = k; break; }
                        if (k >= WALK_MAX) break;
                        q = v;
                    }
                    S.scal[8] = res;
                }
                __syncthreads();
                cnt = S.scal[8];
            }
            if (cnt < 0) {
#pragma unroll
            for (int k = 0; k < DW / THREADS; k++) {      // eight independent table entries per thread
                const int q = tid + k * THREADS;
                if (q < n) S.J[0][q] = dcta_next(S.win, q, n, rem);
            }
            if (tid == 0) { S.path[0] = 0; S.scal[1] = PATH; }
            __syncthreads();
            // chain of token positions by doubling: after level k, path[0 .. 2^(k+1)) known
            int len = 1, cur = 0;
            for (;;) {
                for (int j = tid; j < len; j += THREADS) {
                    const uint16_t pj = S.path[j];
                    const uint16_t v = pj < n ? S.J[cur][pj] : pj;
                    S.path[len + j] = v;
                    if (v >= n) atomicMin(&S.scal[1], len + j);
                }
                __syncthreads();
                const int t = S.scal[1];
                if (t < 2 * len) { cnt = t; break; }
                // J_{k+1} = J_k o J_k (a thread's loads issued together, then its stores)
                {
                    uint16_t v[DW / THREADS], w[DW / THREADS];
#pragma unroll
                    for (int k = 0; k < DW / THREADS; k++) {
                        const int q = tid + k * THREADS;
                        v[k] = q < n ? S.J[cur][q] : (uint16_t)0xFFFF;
                    }
#pragma unroll
                    for (int k = 0; k < DW / THREADS; k++) w[k] = v[k] < n ? S.J[cur][v[k]] : v[k];
#pragma unroll
                    for (int k = 0; k < DW / THREADS; k++) {
                        const int q = tid + k * THREADS;
                        if (q < n) S.J[cur ^ 1][q] = w[k];
                    }
                }
                cur ^= 1;
                len *= 2;
                __syncthreads();
            }
            }
            walk = cnt <= WALK_MAX;
            const uint16_t term = S.path[cnt];          // n, ENDS or STOP
            const int nseq = term == STOP ? cnt - 1 : cnt;
            if (nseq > 0) {
                // sequence fields and validity
                if (tid == 0) S.scal[2] = 0;
                int part = 0;
                constexpr int PER = (MAXS + THREADS - 1) / THREADS;
                const int i0 = tid * PER;
                for (int i = i0; i < min(i0 + PER, nseq); i++) {
                    const int q = S.path[i];
                    const int tok = S.win[q];
                    int r = q + 1, lit = tok >> 4;
                    if (lit == 15) {
                        int b = 255;
                        while (b == 255) { b = S.win[r++]; lit += b; }
                    }
                    S.lpos[i] = (uint16_t)r;
                    S.llen[i] = lit;
                    r += lit;
                    int ml = 0, mo = 0;
                    if (!(i == nseq - 1 && term == ENDS)) {
                        mo = S.win[r] | (S.win[r + 1] << 8);
                        r += 2;
                        ml = tok & 15;
                        if (ml == 15) {
                            int b = 255;
                            while (b == 255) { b = S.win[r++]; ml += b; }
                        }
                        ml += 4;
                    }
                    S.off[i] = (uint16_t)mo;
                    S.mlen[i] = ml;
                    part += lit + ml;
                }
                // exclusive scan of the output lengths
                int incl = part;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULLMASK, incl, o);
                    if (lane >= o) incl += v;
                }
                if (lane == 31) S.wsum[warp] = incl;
                __syncthreads();
                int wbase = 0;
                for (int w = 0; w < warp; w++) wbase += S.wsum[w];
                int acc = wbase + incl - part;
                for (int i = i0; i < min(i0 + PER, nseq); i++) {
                    S.ostart[i] = acc;
                    const int ms = op + acc + S.llen[i];             // absolute match start
                    if (S.mlen[i] > 0 && (S.off[i] == 0 || S.off[i] > ms)) S.scal[2] = 1;
                    acc += S.llen[i] + S.mlen[i];
                }
                if (tid == THREADS - 1) S.ostart[nseq] = acc;      // nseq <= MAXS: the last thread holds the total
                __syncthreads();
                const int total = S.ostart[nseq];
                if (S.scal[2] || total > osz - op) { bad = true; break; }
                // output in groups of at most DCAP bytes
                int a = 0;
                while (a < nseq) {
                    const int base = S.ostart[a];
                    int lo = a + 1, hi = nseq;                      // largest b with ostart[b] - base <= DCAP
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (S.ostart[mid] - base <= DCAP) lo = mid; else hi = mid - 1;
                    }
                    const int b = lo;
                    if (S.ostart[b] - base <= DCAP) {
                        const int span = S.ostart[b] - base;
                        // a match byte's source, relative to the group (>= 0: a pointer into st),
                        // or its value when it precedes the group (the ring, else global memory)
                        auto src_entry = [&](int src) -> uint32_t {
                            if (src >= 0) return (uint32_t)src;
                            const int abs = op + base + src;
                            return RES | (abs >= hist_from ? (uint32_t)S.hist[abs & (HB - 1)] : (uint32_t)__ldcg(out + abs));
                        };
                        // Sequence-parallel fill: a thread writes whole sequences (match byte k at
                        // m0 + k takes its source at m0 - d + (k mod d): below the match start even
                        // when the match overlaps itself); sequences longer than LONGSEQ bytes are
                        // listed and filled by the whole CTA after.
                        for (int i = a + tid; i < b; i += THREADS) {
                            const int s0 = S.ostart[i] - base, lit = S.llen[i], ml = S.mlen[i];
                            if (lit + ml > LONGSEQ) {
                                S.longs[atomicAdd(&S.nlong, 1)] = i;
                                continue;
                            }
                            const int lp = S.lpos[i], d = S.off[i], m0 = s0 + lit;
                            for (int r = 0; r < lit; r++) S.st[s0 + r] = RES | S.win[lp + r];
                            int km = 0;                                  // k mod d
                            for (int k = 0; k < ml; k++) {
                                S.st[m0 + k] = src_entry(m0 - d + km);
                                if (++km == d) km = 0;
                            }
                        }
                        __syncthreads();
                        const int nlong = S.nlong;
                        for (int j = 0; j < nlong; j++) {
                            const int i = S.longs[j];
                            const int s0 = S.ostart[i] - base, lit = S.llen[i], ml = S.mlen[i];
                            const int lp = S.lpos[i], d = S.off[i], m0 = s0 + lit;
                            for (int x = tid; x < lit + ml; x += THREADS)
                                S.st[s0 + x] = x < lit ? RES | S.win[lp + x] : src_entry(m0 - d + (x - lit) % d);
                        }
                        __syncthreads();
                        if (tid == 0) S.nlong = 0;                     // read above, before the barrier
                        for (;;) {                                 // pointer jumping
                            int open = 0;
                            for (int x = tid; x < span; x += THREADS) {
                                const uint32_t v = S.st[x];
                                if (!(v & RES)) {
                                    const uint32_t t = S.st[v];
                                    S.st[x] = t;
                                    open |= !(t & RES);
                                }
                            }
                            if (!__syncthreads_or(open)) break;
                        }
                        uint8_t *o = out + op + base;
                        for (int x = tid; x < span; x += THREADS) {
                            const uint8_t byte = (uint8_t)S.st[x];
                            o[x] = byte;
                            S.hist[(op + base + x) & (HB - 1)] = byte;
                        }
                        hist_from = max(hist_from, op + base + span - HB);
                        a = b;
                    } else {
                        // one sequence larger than DCAP: literals, then the match from global memory
                        const int abs0 = op + base, lit = S.llen[a], ml = S.mlen[a], d = S.off[a];
                        for (int x = tid; x < lit; x += THREADS) out[abs0 + x] = S.win[S.lpos[a] + x];
                        __syncthreads();
                        const int m0 = abs0 + lit;
                        for (int x = tid; x < ml; x += THREADS) out[m0 + x] = __ldcg(out + m0 - d + (d > x ? x : x % d));
                        hist_from = m0 + ml;                        // the ring missed this sequence
                        a = a + 1;
                    }
                    __syncthreads();
                }
                op += total;
                if (term == ENDS) { done = true; break; }
                p += term == STOP ? S.path[cnt - 1] : n;
                continue;
            }
            // the sequence at p does not fit in a window: decode it alone, header from global
            if (tid == 0) {
                int r = p, f = 0, lit = 0, mo = 0, ml = 0, fin = 0;
                const int tok = __ldg(in + r++);
                lit = tok >> 4;
                if (lit == 15) {
                    int bb = 255;
                    while (bb == 255) {
                        if (r >= isz) { f = 1; break; }
                        bb = __ldg(in + r++);
                        lit += bb;
                    }
                }
                const int lp = r;
                if (!f && (lit > isz - r || lit > osz - op)) f = 1;
                if (!f) {
                    r += lit;
                    if (r == isz) {
                        fin = 1;
                    } else if (isz - r < 2) {
                        f = 1;
                    } else {
                        mo = __ldg(in + r) | (__ldg(in + r + 1) << 8);
                        r += 2;
                        ml = tok & 15;
                        if (ml == 15) {
                            int bb = 255;
                            while (bb == 255) {
                                if (r >= isz) { f = 1; break; }
                                bb = __ldg(in + r++);
                                ml += bb;
                            }
                        }
                        ml += 4;
                        if (!f && (mo == 0 || mo > op + lit || ml > osz - op - lit)) f = 1;
                    }
                }
                S.scal[2] = f; S.scal[3] = lit; S.scal[4] = lp; S.scal[5] = mo; S.scal[6] = ml; S.scal[7] = fin ? -1 : r;
            }
            __syncthreads();
            if (S.scal[2]) { bad = true; break; }
            {
                const int lit = S.scal[3], lp = S.scal[4], mo = S.scal[5], ml = S.scal[6], nr = S.scal[7];
                for (int x = tid; x < lit; x += THREADS) out[op + x] = __ldg(in + lp + x);
                __syncthreads();
                const int m0 = op + lit;
                for (int x = tid; x < ml; x += THREADS) out[m0 + x] = __ldcg(out + m0 - mo + (mo > x ? x : x % mo));
                __syncthreads();
                op += lit + ml;
                hist_from = op;                            // the ring missed this sequence
                if (nr < 0) done = true; else p = nr;
            }
        }
        if (!bad && op != osz) bad = true;
        if (bad && tid == 0) dev_fail(jb.err, DE_LZ4);
    }
}

constexpr int TILE = 1024;

__device__ __forceinline__ void store_item(uint8_t *o, int ts, uint64_t v)
{
    switch (ts) {
    case 8: *reinterpret_cast<uint64_t *>(o) = v; break;
    case 4: *reinterpret_cast<uint32_t *>(o) = (uint32_t)v; break;
    case 2: *reinterpret_cast<uint16_t *>(o) = (uint16_t)v; break;
    default: for (int j = 0; j < ts; j++) o[j] = (uint8_t)(v >> (8 * j)); break;
    }
}

__device__ __forceinline__ uint64_t load_item(const uint8_t *o, int ts)
{
    switch (ts) {
    case 8: return *reinterpret_cast<const uint64_t *>(o);
    case 4: return *reinterpret_cast<const uint32_t *>(o);
    case 2: return *reinterpret_cast<const uint16_t *>(o);
    default: { uint64_t v = 0; for (int j = 0; j < ts; j++) v |= (uint64_t)o[j] << (8 * j); return v; }
    }
}

// An item at any byte offset (a special-value chunk's value sits right after the chunk's
// 32-byte header, and chunks lie back to back at arbitrary offsets).
__device__ __forceinline__ uint64_t load_item_bytes(const uint8_t *o, int ts)
{
    uint64_t v = 0;
    for (int j = 0; j < ts; j++) v |= (uint64_t)__ldg(o + j) << (8 * j);
    return v;
}

// Map item i of block b of chunk c to its logical (row, col); false if it is padding.
__device__ __forceinline__ bool item_pos(const Geom &g, int64_t c, int64_t b, int64_t i, int64_t &row, int64_t &col)
{
    const int64_t ci0 = c / g.cgrid[1], ci1 = c - ci0 * g.cgrid[1];
    const int64_t bi0 = b / g.bgrid[1], bi1 = b - bi0 * g.bgrid[1];
    const int64_t r = i / g.block[1], cc = i - r * g.block[1];
    const int64_t rin = bi0 * g.block[0] + r, cin = bi1 * g.block[1] + cc;
    if (rin >= g.chunk[0] || cin >= g.chunk[1]) return false;
    row = ci0 * g.chunk[0] + rin;
    col = ci1 * g.chunk[1] + cin;
    return row < g.shape[0] && col < g.shape[1];
}

// Partitions whose block rows hold whole groups of 4 items of 4 or 8 bytes take the
// word-level fast paths below, edge blocks included.
__device__ __forceinline__ bool geom_fast(const Geom &g)
{
    return !(g.block[1] & 3) && (g.itemsize == 4 || g.itemsize == 8);
}

// Block b of chunk c: its first logical row and column, and how many of its rows (nr) and
// columns (nc) hold logical items (the rest is chunk or array padding; 0 when none do).
// q = a / b, r = a - q b for a >= 0, b > 0: 32-bit division when both fit (the usual case),
// 64-bit otherwise.
__device__ __forceinline__ void divmod(int64_t a, int64_t b, int64_t &q, int64_t &r)
{
    if (((a | b) >> 31) == 0) {
        const uint32_t q32 = (uint32_t)a / (uint32_t)b;
        q = q32;
        r = a - (int64_t)q32 * b;
    } else {
        q = a / b;
        r = a - q * b;
    }
}

struct BlockSpan {
    int64_t row0, col0;
    int nr, nc;
};
__device__ __forceinline__ BlockSpan block_span(const Geom &g, int64_t c, int64_t b)
{
    BlockSpan s;
    int64_t ci0, ci1, bi0, bi1;
    divmod(c, g.cgrid[1], ci0, ci1);
    divmod(b, g.bgrid[1], bi0, bi1);
    s.row0 = ci0 * g.chunk[0] + bi0 * g.block[0];
    s.col0 = ci1 * g.chunk[1] + bi1 * g.block[1];
    s.nr = (int)max((int64_t)0, min(min(g.block[0], g.chunk[0] - bi0 * g.block[0]), g.shape[0] - s.row0));
    s.nc = (int)max((int64_t)0, min(min(g.block[1], g.chunk[1] - bi1 * g.block[1]), g.shape[1] - s.col0));
    return s;
}

// D2 fast path: shuffled, split blocks of partitions whose block rows hold whole groups of 4
// items, in slices of SC_ITEMS items (one CTA per slice at a time).  One thread stages the
// slice's bytes of every byte plane (read in place from raw streams or the LZ4 scratch) into
// shared memory with bulk asynchronous copies completing on an mbarrier; then each thread
// rebuilds 4 consecutive items from one 4-byte word per plane and writes the logical ones to
// the dense row (edge blocks: the items in chunk or array padding are not written; slices of
// padding only are skipped).  Every other block is appended to the list `rest` for the
// general path.
constexpr int SC_ITEMS = 4096;
constexpr int SC_PLANE = SC_ITEMS + 32;            // a slice of a plane from its 16-byte boundary
constexpr uint32_t SC_WAIT_POLLS = 1u << 22;

__device__ __forceinline__ void bulk_g2s(void *sdst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(tc::smem_addr(sdst)), "l"(gsrc), "r"(bytes), "r"(tc::smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool sc_wait(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < SC_WAIT_POLLS; i++)
        if (tc::mbar_try_wait(bar, parity)) return true;
    return false;
}

// One slice (t, sl) of the fast scatter; false when a bounded wait gave up (the CTA must
// leave).  rest_id: the block's entry for the general path's list.
template <int TS>
__device__ __forceinline__ bool scatter_fast_unit(const Geom &g, const uint8_t *__restrict__ ch, const uint8_t *ch_end,
                                                  const BlockDesc *__restrict__ bd, const StreamDesc *__restrict__ sd,
                                                  const uint8_t *__restrict__ scratch, const uint8_t *scratch_end,
                                                  uint8_t *__restrict__ out, int64_t ld, int *rest, int *nrest,
                                                  int rest_id, int *err, int64_t t, int sl, uint8_t (*stage)[SC_PLANE],
                                                  uint64_t *bar, uint32_t &parity, int *abort_all)
{
    const int tid = threadIdx.x;
    const int qpr = (int)(g.block[1] / 4);
    int64_t c, b;
    divmod(t, g.nblocks, c, b);
    const BlockDesc d = bd[t];
    if (d.mode != BM_SHUFFLED || d.nstreams != TS || !geom_fast(g)) {
        if (tid == 0 && sl == 0) rest[atomicAdd(nrest, 1)] = rest_id;   // left to k_scatter
        return true;
    }
    const BlockSpan sp = block_span(g, c, b);
    const int i0s = sl * SC_ITEMS, cnt = (int)min((int64_t)SC_ITEMS, g.blockn - i0s);
    if (sp.nc == 0 || i0s / (qpr * 4) >= sp.nr) return true;          // the slice holds only padding
    // per plane: its slice starts at src, 16-byte word a16 = src - shift; the bulk copy
    // takes the whole words of [a16, a16 + want) before the buffer end lim, threads copy
    // the bytes that the buffer end cuts off (zeros past it)
    auto plane = [&](int j, const uint8_t *&src, const uint8_t *&lim, int &want, int &bulk) {
        const StreamDesc q = sd[t * 8 + j];
        src = nullptr; lim = nullptr;
        if (q.kind == SK_RAW) { src = ch + q.src + i0s; lim = ch_end; }
        else if (q.kind == SK_LZ4) { src = scratch + t * g.blocksize + (int64_t)j * d.neblock + i0s; lim = scratch_end; }
        want = bulk = 0;
        if (src) {
            const uint8_t *a16 = src - (reinterpret_cast<uintptr_t>(src) & 15);
            want = ((int)(src - a16) + cnt + 15) & ~15;
            bulk = (int)min((int64_t)want, (lim - a16) & ~int64_t(15));
        }
        return q;
    };
    if (tid == 0) {
        uint32_t tx = 0;
#pragma unroll
        for (int j = 0; j < TS; j++) {
            const uint8_t *src, *lim;
            int want, bulk;
            plane(j, src, lim, want, bulk);
            tx += (uint32_t)bulk;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of stage precede the copies
        tc::mbar_arrive_expect_tx(bar, tx);
#pragma unroll
        for (int j = 0; j < TS; j++) {
            const uint8_t *src, *lim;
            int want, bulk;
            plane(j, src, lim, want, bulk);
            if (bulk > 0) bulk_g2s(stage[j], src - (reinterpret_cast<uintptr_t>(src) & 15), (uint32_t)bulk, bar);
        }
    }
    int code[TS];                                  // 0..15: the plane's shift in stage; 256 + v: a run of byte v
#pragma unroll
    for (int j = 0; j < TS; j++) {
        const uint8_t *src, *lim;
        int want, bulk;
        const StreamDesc q = plane(j, src, lim, want, bulk);
        code[j] = src ? (int)(reinterpret_cast<uintptr_t>(src) & 15) : 256 + (q.kind == SK_RUN ? (q.len & 255) : 0);
        if (bulk < want) {
            const uint8_t *a16 = src - code[j];
            for (int x = bulk + tid; x < want; x += blockDim.x) stage[j][x] = a16 + x < lim ? __ldg(a16 + x) : (uint8_t)0;
        }
    }
    const bool ok = sc_wait(bar, parity);
    parity ^= 1;
    if (!ok) *abort_all = 1;
    __syncthreads();
    if (*abort_all) {                              // the copies did not complete: report, wait once more, leave
        if (tid == 0) {
            dev_fail(err, DE_WAIT);
            sc_wait(bar, parity ^ 1);
        }
        return false;
    }
    uint8_t *const obase = out + (sp.row0 * ld + sp.col0) * TS;
    const int nr = sp.nr, nc = sp.nc;
    // (row, column) of each thread's quad, advanced by a fixed step per iteration (one
    // division per slice instead of one per quad)
    const int rowlen = qpr * 4, step = (int)blockDim.x * 4;
    const int step_r = step / rowlen, step_c = step - step_r * rowlen;
    int r = (i0s + tid * 4) / rowlen, cc = i0s + tid * 4 - r * rowlen;
    for (int qd = tid; qd < cnt / 4; qd += blockDim.x, r += step_r, cc += step_c) {
        if (cc >= rowlen) { cc -= rowlen; r++; }
        if (r >= nr || cc >= nc) continue;                                // padding items
        uint32_t w[TS];
#pragma unroll
        for (int j = 0; j < TS; j++) {
            if (code[j] >= 256) { w[j] = (uint32_t)(code[j] - 256) * 0x01010101u; continue; }
            const uint32_t *pw = reinterpret_cast<const uint32_t *>(stage[j]);
            const int byte = code[j] + qd * 4, wi = byte >> 2, sh = (byte & 3) * 8;
            w[j] = sh ? __funnelshift_r(pw[wi], pw[wi + 1], sh) : pw[wi];
        }
        uint8_t *o = obase + ((int64_t)r * ld + cc) * TS;
        uint32_t v[4];
        transpose4x4(w[0], w[1], w[2], w[3], v[0], v[1], v[2], v[3]);
        const bool whole = cc + 4 <= nc;
        const bool o16a = (reinterpret_cast<uintptr_t>(o) & 15) == 0;
        if constexpr (TS == 8) {
            uint32_t h[4];
            transpose4x4(w[4], w[5], w[6], w[7], h[0], h[1], h[2], h[3]);
            if (whole && o16a) {
                uint4 *o16 = reinterpret_cast<uint4 *>(o);
                o16[0] = make_uint4(v[0], h[0], v[1], h[1]);
                o16[1] = make_uint4(v[2], h[2], v[3], h[3]);
            } else {
                uint64_t *o8 = reinterpret_cast<uint64_t *>(o);
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (cc + u < nc) o8[u] = ((uint64_t)h[u] << 32) | v[u];
            }
        } else {
            if (whole && o16a) {
                *reinterpret_cast<uint4 *>(o) = make_uint4(v[0], v[1], v[2], v[3]);
            } else {
                uint32_t *o4 = reinterpret_cast<uint32_t *>(o);
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (cc + u < nc) o4[u] = v[u];
            }
        }
    }
    __syncthreads();                               // stage is read before the next slice's copies
    return true;
}

template <int TS>
__global__ void __launch_bounds__(256, 6) k_scatter_fast(Geom g, const uint8_t *__restrict__ ch, const uint8_t *ch_end,
                                                      const BlockDesc *__restrict__ bd,
                                                      const StreamDesc *__restrict__ sd,
                                                      const uint8_t *__restrict__ scratch, const uint8_t *scratch_end,
                                                      uint8_t *__restrict__ out, int64_t ld, int *rest, int *nrest,
                                                      int *err)
{
    __shared__ __align__(128) uint8_t stage[TS][SC_PLANE];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_all;
    const int tid = threadIdx.x;
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_barrier_init();
        abort_all = 0;
    }
    __syncthreads();
    const int64_t nbl = g.nchunks * g.nblocks;
    const int64_t nsl = (g.blockn + SC_ITEMS - 1) / SC_ITEMS;
    uint32_t parity = 0;
    for (int64_t u = blockIdx.x; u < nbl * nsl; u += gridDim.x) {
        int64_t t, s64;
        divmod(u, nsl, t, s64);
        const int sl = (int)s64;
        if (!scatter_fast_unit<TS>(g, ch, ch_end, bd, sd, scratch, scratch_end, out, ld, rest, nrest, (int)t, err, t, sl,
                                   stage, &bar, parity, &abort_all))
            return;
    }
}

// D2 general path: unshuffle one tile of TILE items of one block through shared memory
// and scatter it to the dense array (padded edge blocks, other item sizes, plain and
// special chunks).  With a `rest` list, only the blocks listed there; else every block.
__device__ __forceinline__ void scatter_tile(const Geom &g, const uint8_t *__restrict__ ch,
                                             const BlockDesc *__restrict__ bd, const StreamDesc *__restrict__ sd,
                                             const uint8_t *__restrict__ scratch, uint8_t *__restrict__ out, int64_t ld,
                                             int64_t t, int64_t i0, uint8_t *planes)
{
    const int ts = g.itemsize;
    const int cnt = (int)min((int64_t)TILE, g.blockn - i0);
    const int64_t c = t / g.nblocks, b = t - c * g.nblocks;
    const BlockDesc d = bd[t];
    const StreamDesc *s = sd + t * 8;
    const uint8_t *blk_scratch = scratch + t * g.blocksize;
    if (d.mode == BM_SHUFFLED) {
        for (int j = 0; j < ts; j++) {
            const int64_t pos = (int64_t)j * g.blockn + i0;
            const int sidx = (int)(pos / d.neblock);
            const int64_t so = pos - (int64_t)sidx * d.neblock;
            const StreamDesc q = s[sidx];
            uint8_t *pl = planes + j * TILE;
            if (q.kind == SK_RUN) {
                for (int x = threadIdx.x; x < cnt; x += blockDim.x) pl[x] = (uint8_t)q.len;
            } else if (q.kind == SK_RAW) {
                const uint8_t *src = ch + q.src + so;
                for (int x = threadIdx.x; x < cnt; x += blockDim.x) pl[x] = __ldg(src + x);
            } else {
                const uint8_t *src = blk_scratch + (int64_t)sidx * d.neblock + so;
                for (int x = threadIdx.x; x < cnt; x += blockDim.x) pl[x] = __ldcg(src + x);
            }
        }
    } else if (d.mode == BM_PLAIN) {
        for (int x = threadIdx.x; x < cnt * ts; x += blockDim.x) {
            const int64_t pos = i0 * ts + x;
            const int sidx = (int)(pos / d.neblock);
            const int64_t so = pos - (int64_t)sidx * d.neblock;
            const StreamDesc q = s[sidx];
            uint8_t v;
            if (q.kind == SK_RUN) v = (uint8_t)q.len;
            else if (q.kind == SK_RAW) v = __ldg(ch + q.src + so);
            else v = __ldcg(blk_scratch + (int64_t)sidx * d.neblock + so);
            planes[x] = v;
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < cnt; x += blockDim.x) {
        int64_t row, col;
        if (!item_pos(g, c, b, i0 + x, row, col)) continue;
        uint8_t *o = out + (row * ld + col) * ts;
        uint64_t v = 0;
        if (d.mode == BM_SHUFFLED) {
            for (int j = 0; j < ts; j++) v |= (uint64_t)planes[j * TILE + x] << (8 * j);
        } else if (d.mode == BM_PLAIN) {
            for (int j = 0; j < ts; j++) v |= (uint64_t)planes[x * ts + j] << (8 * j);
        } else if (d.mode == BM_NAN) {
            v = ts == 8 ? 0x7FF8000000000000ull : 0x7FC00000ull;
        } else {
            v = load_item_bytes(ch + d.value_src, ts);
        }
        store_item(o, ts, v);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_scatter(Geom g, const int *__restrict__ rest, const int *__restrict__ nrest,
                                                 const uint8_t *__restrict__ ch,
                                                 const BlockDesc *__restrict__ bd, const StreamDesc *__restrict__ sd,
                                                 const uint8_t *__restrict__ scratch, uint8_t *__restrict__ out, int64_t ld)
{
    __shared__ __align__(16) uint8_t planes[8 * TILE];
    const int64_t tpb = (g.blockn + TILE - 1) / TILE;
    const int64_t nwork = (rest ? (int64_t)*nrest : g.nchunks * g.nblocks) * tpb;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t k = w / tpb, t = rest ? rest[k] : k, i0 = (w - k * tpb) * TILE;
        scatter_tile(g, ch, bd, sd, scratch, out, ld, t, i0, planes);
    }
}

// ============================================================================ encode
// E1 fast path: shuffle on, block rows of whole groups of 4 items; each thread reads 4
// consecutive items of a block row (zero for the items in chunk or array padding) and
// writes one 4-byte word into each byte plane of the image.
template <int TS>
__device__ __forceinline__ void gather_fast_block(const Geom &g, const uint8_t *__restrict__ in, int64_t ld,
                                                  uint8_t *__restrict__ img, int64_t t)
{
    if (!geom_fast(g)) return;
    const int qpr = (int)(g.block[1] / 4), nq = (int)(g.blockn / 4);
    int64_t c, b;
    divmod(t, g.nblocks, c, b);
    const BlockSpan sp = block_span(g, c, b);
    uint8_t *blk = img + t * g.blocksize;
    // (row, quad column) of each thread's quad, advanced by a fixed step per iteration
    const int step_r = (int)blockDim.x / qpr, step_q = (int)blockDim.x - step_r * qpr;
    int r = (int)threadIdx.x / qpr, q = (int)threadIdx.x - r * qpr;
    for (int qd = threadIdx.x; qd < nq; qd += blockDim.x, r += step_r, q += step_q) {
        if (q >= qpr) { q -= qpr; r++; }
        const int i0 = qd * 4, cc = q * 4;
        const uint8_t *src = in + ((sp.row0 + r) * ld + sp.col0 + cc) * TS;
        uint64_t x[4] = {0, 0, 0, 0};                 // padding items are zero, as in Caterva
        if (r < sp.nr && cc + 4 <= sp.nc) {
            if constexpr (TS == 8) {
                const uint64_t *s8 = reinterpret_cast<const uint64_t *>(src);
#pragma unroll
                for (int u = 0; u < 4; u++) x[u] = __ldg(s8 + u);
            } else {
                const uint32_t *s4 = reinterpret_cast<const uint32_t *>(src);
#pragma unroll
                for (int u = 0; u < 4; u++) x[u] = __ldg(s4 + u);
            }
        } else if (r < sp.nr) {
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (cc + u < sp.nc) x[u] = TS == 8 ? __ldg(reinterpret_cast<const uint64_t *>(src) + u)
                                                   : __ldg(reinterpret_cast<const uint32_t *>(src) + u);
        }
        uint32_t o[TS];
        transpose4x4((uint32_t)x[0], (uint32_t)x[1], (uint32_t)x[2], (uint32_t)x[3], o[0], o[1], o[2], o[3]);
        if constexpr (TS == 8)
            transpose4x4((uint32_t)(x[0] >> 32), (uint32_t)(x[1] >> 32), (uint32_t)(x[2] >> 32), (uint32_t)(x[3] >> 32),
                         o[4], o[5], o[6], o[7]);
#pragma unroll
        for (int j = 0; j < TS; j++) *reinterpret_cast<uint32_t *>(blk + (int64_t)j * g.blockn + i0) = o[j];
    }
}

template <int TS>
__global__ void __launch_bounds__(256) k_gather_fast(Geom g, const uint8_t *__restrict__ in, int64_t ld,
                                                     uint8_t *__restrict__ img)
{
    const int64_t nbl = g.nchunks * g.nblocks;
    for (int64_t t = blockIdx.x; t < nbl; t += gridDim.x) gather_fast_block<TS>(g, in, ld, img, t);
}

// E1 general path: dense -> byte-plane image (shuffled: plane j holds byte j of every
// item; plain: items back to back).  Padding items are zero, as in Caterva.  With
// skip_fast, nothing is done for partitions the fast path handles.
__device__ __forceinline__ void gather_tile(const Geom &g, const uint8_t *__restrict__ in, int64_t ld, bool shuffle,
                                            uint8_t *__restrict__ img, int64_t t, int64_t i0, uint8_t *planes)
{
    const int ts = g.itemsize;
    const int cnt = (int)min((int64_t)TILE, g.blockn - i0);
    const int64_t c = t / g.nblocks, b = t - c * g.nblocks;
    for (int x = threadIdx.x; x < cnt; x += blockDim.x) {
        int64_t row, col;
        uint64_t v = 0;
        if (item_pos(g, c, b, i0 + x, row, col)) v = load_item(in + (row * ld + col) * ts, ts);
        if (shuffle) {
            for (int j = 0; j < ts; j++) planes[j * TILE + x] = (uint8_t)(v >> (8 * j));
        } else {
            for (int j = 0; j < ts; j++) planes[x * ts + j] = (uint8_t)(v >> (8 * j));
        }
    }
    __syncthreads();
    uint8_t *blk = img + t * g.blocksize;
    if (shuffle) {
        for (int j = 0; j < ts; j++) {
            uint8_t *dst = blk + (int64_t)j * g.blockn + i0;
            for (int x = threadIdx.x; x < cnt; x += blockDim.x) dst[x] = planes[j * TILE + x];
        }
    } else {
        uint8_t *dst = blk + i0 * ts;
        for (int x = threadIdx.x; x < cnt * ts; x += blockDim.x) dst[x] = planes[x];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_gather(Geom g, bool skip_fast, const uint8_t *__restrict__ in, int64_t ld,
                                                bool shuffle, uint8_t *__restrict__ img)
{
    __shared__ __align__(16) uint8_t planes[8 * TILE];
    const int64_t tpb = (g.blockn + TILE - 1) / TILE;
    const int64_t nwork = g.nchunks * g.nblocks * tpb;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t t = w / tpb, i0 = (w - t * tpb) * TILE;
        if (skip_fast && geom_fast(g)) continue;
        gather_tile(g, in, ld, shuffle, img, t, i0, planes);
    }
}

// ---------------------------------------------------------------- LZ4 encoder (warp)
// Unaligned little-endian reads from a source whose stream base is 4-byte aligned: two
// aligned word loads and a funnel shift.  Callers only read where p + 7 stays inside the
// stream (hash positions are at most n - 12; match candidates lie before them).
__device__ __forceinline__ uint32_t ld4u(const uint8_t *p)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
    return __funnelshift_r(__ldg(w), __ldg(w + 1), (uint32_t)(a & 3) * 8);
}

// Position offset of the t-th probe of a search, relative to its start: the step is
// 1 for probes 0..64 and grows by one every 64 probes after that.
__device__ __forceinline__ int64_t probe_offset(int64_t t)
{
    if (t <= 0) return 0;
    const int64_t m = 62 + t, q = m >> 6, r = m - (q << 6);
    return 1 + 64 * (q * (q - 1) / 2) + q * (r + 1);
}

// Shared-memory window over one stream for the encoder: positions [lo, hi) sit at
// r[x & (ERING - 1)], the first 16 ring bytes mirrored past its end so that 4-byte reads
// never wrap.  The window follows the parse position; reads outside it (far search
// probes, old match candidates) go to global memory.  Without it the candidate reads of
// low-entropy streams, spread over the last few KiB, mostly miss L1.
constexpr int ERING = 4096, ESEG = 1024, ELOOK = 512;

struct EncSrc {
    const uint8_t *g;   // the stream in global memory
    uint8_t *r;         // ERING + 16 bytes, 16-byte aligned
    int lo, hi, n;
};

__device__ __forceinline__ uint32_t es_byte(const EncSrc &s, int x)
{
    return (x >= s.lo && x < s.hi) ? (uint32_t)s.r[x & (ERING - 1)] : (uint32_t)__ldg(s.g + x);
}

__device__ __forceinline__ uint32_t es_rd32(const EncSrc &s, int x)
{
    if (x >= s.lo && x + 4 <= s.hi) {
        const int o = x & (ERING - 1);
        const uint32_t *w = reinterpret_cast<const uint32_t *>(s.r) + (o >> 2);
        return __funnelshift_r(w[0], w[1], (uint32_t)(o & 3) * 8);
    }
    return ld4u(s.g + x);
}

// liblz4's hash of the 4 (byU16 tables) or 5 (byU32 tables) bytes at p.
__device__ __forceinline__ uint32_t es_hash(const EncSrc &s, int p, bool small)
{
    if (small) return (es_rd32(s, p) * 2654435761u) >> (32 - 13);
    const uint64_t v = (uint64_t)es_rd32(s, p) | ((uint64_t)es_byte(s, p + 4) << 32);
    return (uint32_t)(((v << 24) * 889523592379ull) >> (64 - 12));
}

// Extends the window up to position `want` (warp-uniform) in ESEG pieces.
__device__ __forceinline__ void es_fill(EncSrc &s, int want)
{
    const int lane = threadIdx.x & 31;
    while (s.hi < s.n && s.hi < want) {
        const int base = s.hi, cnt = min(ESEG, s.n - base);
        __syncwarp();                                    // reads of the slots being replaced are done
        for (int x = lane * 4; x < cnt; x += 128) {
            uint32_t v = 0;
            if (base + x + 8 <= s.n) {
                v = ld4u(s.g + base + x);
            } else {
                for (int k = 0; k < 4; k++)
                    if (base + x + k < s.n) v |= (uint32_t)__ldg(s.g + base + x + k) << (8 * k);
            }
            const int o = (base + x) & (ERING - 1);
            *reinterpret_cast<uint32_t *>(s.r + o) = v;
            if (o < 16) *reinterpret_cast<uint32_t *>(s.r + ERING + o) = v;
        }
        s.hi = base + cnt;
        s.lo = max(s.lo, base + ESEG - ERING);
        __syncwarp();
    }
}

// Shared-memory accesses through 32-bit shared-window addresses (volatile: they keep
// their order relative to each other, which the table updates rely on).
__device__ __forceinline__ uint32_t lds32(uint32_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t lds_tab(uint32_t a, bool small)
{
    uint32_t v;
    if (small) {
        uint16_t h;
        asm volatile("ld.shared.u16 %0, [%1];" : "=h"(h) : "r"(a) : "memory");
        v = h;
    } else {
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    }
    return v;
}
__device__ __forceinline__ void sts_tab(uint32_t a, uint32_t v, bool small)
{
    if (small) asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"((uint16_t)v) : "memory");
    else asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

// liblz4's hash of the 4 bytes v4 at a position (byU16 tables) or of those and the fifth
// byte b4 (byU32 tables).
template <bool SMALL>
__device__ __forceinline__ uint32_t lz_hash_v(uint32_t v4, uint32_t b4)
{
    if (SMALL) return (v4 * 2654435761u) >> (32 - 13);
    const uint64_t v = (uint64_t)v4 | ((uint64_t)b4 << 32);
    return (uint32_t)(((v << 24) * 889523592379ull) >> (64 - 12));
}

// Warp-cooperative LZ4 block compressor in limited-output mode with capacity `cap`.
// Returns the compressed size, or 0 when it does not fit; *need_out receives the
// smallest capacity for which it would have fit.  All lanes must call it; every
// position, candidate and output offset below is warp-uniform.  SMALL selects liblz4's
// byU16 table (inputs below 64 KiB + 11 bytes: 13-bit hash of 4 bytes) over its byU32
// table (12-bit hash of 5 bytes, 65535-byte distance limit).
//
// Two regimes.  Searching (no match at the parse position): one step evaluates 32
// consecutive probes of liblz4's search (its step schedule), resolving probes that share
// a hash bucket in probe order with __match_any_sync.  Right after a match liblz4
// inserts ip - 2 and tests ip itself; on low-entropy data that test nearly always
// succeeds, so it runs as a short scalar path that every lane executes identically (the
// window bytes around ip and around the candidate come from a few aligned shared-memory
// words, the match length from one 64-bit compare, table updates written by all lanes
// with the same value), leaving the warp-wide machinery for long matches and searches.
template <bool SMALL>
__device__ __forceinline__ int warp_lz4_compress(const uint8_t *__restrict__ src, int n, uint8_t *__restrict__ dst,
                                                 int cap, uint32_t *tab, uint8_t *ring, int *need_out)
{
    const int lane = threadIdx.x & 31;
    uint16_t *tab16 = reinterpret_cast<uint16_t *>(tab);
    for (int i = lane; i < 4096; i += 32) tab[i] = 0u;
    EncSrc s;
    s.g = src; s.r = ring; s.lo = 0; s.hi = 0; s.n = n;
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring), tab_s = (uint32_t)__cvta_generic_to_shared(tab);
    constexpr uint32_t TSH = SMALL ? 1 : 2;             // table entry size: 2 or 4 bytes
    __syncwarp();
    int need = 0, op = 0, anchor = 0, ip = 1, mt = 0;
    int token_pos = 0, token_val = 0;
    const int mfl1 = n - 12 + 1, mlimit = n - 5;
#define TGET(h) (SMALL ? (uint32_t)tab16[h] : tab[h])
#define TPUT(h, v) do { if (SMALL) tab16[h] = (uint16_t)(v); else tab[h] = (uint32_t)(v); } while (0)
#define NEED(x) do { const int nx_ = (x); need = max(need, nx_); if (nx_ > cap) { *need_out = need; return 0; } } while (0)
    if (n < 13) goto last_literals;
    es_fill(s, ELOOK);
    if (lane == 0) TPUT(es_hash(s, 0, SMALL), 0);
    __syncwarp();
    for (;;) {
        // ---- search from ip: probes p0 + probe_offset(t), t = 0, 1, ...
        {
            const int p0 = ip;
            int64_t t0 = 0;
            for (;;) {
                es_fill(s, p0 + (int)(probe_offset(t0) < n ? probe_offset(t0) : (int64_t)n) + ELOOK);
                const int64_t t = t0 + lane;
                // the step is 1 for the first 66 probes: positions are p0 + t there
                const bool dense = t0 + 32 <= 65;
                const int64_t p = dense ? p0 + t : p0 + probe_offset(t);
                const int64_t pn = dense ? p + 1 : p0 + probe_offset(t + 1);
                const bool valid = pn <= mfl1;
                const uint32_t h = valid ? es_hash(s, (int)p, SMALL) : (0x80000000u | (uint32_t)lane);
                const uint32_t ctab = valid ? TGET(h) : 0u;
                const unsigned peers = __match_any_sync(FULLMASK, h);
                const unsigned lower = peers & ((1u << lane) - 1u);
                const int srcl = lower ? 31 - __clz(lower) : lane;
                const int pl = __shfl_sync(FULLMASK, (int)p, srcl);
                const uint32_t cand = lower ? (uint32_t)pl : ctab;
                const bool m = valid && (SMALL || cand + 65535u >= (uint32_t)p) &&
                               es_rd32(s, (int)cand) == es_rd32(s, (int)p);
                const unsigned mm = __ballot_sync(FULLMASK, m), em = __ballot_sync(FULLMASK, !valid);
                const int W = mm ? __ffs(mm) - 1 : 32, E = em ? __ffs(em) - 1 : 32;
                const int lastw = min(W, E - 1);
                __syncwarp();
                if (lane <= lastw) {
                    const unsigned upto = (lastw >= 31) ? FULLMASK : ((2u << lastw) - 1u);
                    const unsigned higher = peers & ~((2u << lane) - 1u) & upto;
                    if (!higher) TPUT(h, (uint32_t)p);
                }
                __syncwarp();
                if (W < E) {
                    ip = __shfl_sync(FULLMASK, (int)p, W);
                    mt = (int)__shfl_sync(FULLMASK, cand, W);
                    break;
                }
                if (E < 32) goto last_literals;
                t0 += 32;
            }
        }
        for (;;) {   // extend the match backwards
            const int k = lane + 1;
            const bool ok = (ip - k >= anchor) && (mt - k >= 0) && es_byte(s, ip - k) == es_byte(s, mt - k);
            const unsigned badm = __ballot_sync(FULLMASK, !ok);
            const int ext = badm ? __ffs(badm) - 1 : 32;
            ip -= ext;
            mt -= ext;
            if (ext < 32) break;
        }
        {   // literals
            const int lit = ip - anchor;
            token_pos = op;
            op += 1;
            NEED(op + lit + 8 + lit / 255);
            if (lit >= 15) {
                token_val = 15 << 4;
                const int rem = lit - 15, nff = rem / 255;
                for (int x = lane; x < nff; x += 32) dst[op + x] = 255;
                if (lane == 0) dst[op + nff] = (uint8_t)(rem % 255);
                op += nff + 1;
            } else {
                token_val = lit << 4;
            }
            for (int x = lane; x < lit; x += 32) dst[op + x] = (uint8_t)es_byte(s, anchor + x);
            op += lit;
        }
        {   // the match found by the search: offset, length (warp-wide compare), token
            const int mo = ip - mt;
            if (lane == 0) { dst[op] = (uint8_t)mo; dst[op + 1] = (uint8_t)(mo >> 8); }
            op += 2;
            int mc = 0;
            for (int a = ip + 4, bpos = mt + 4;; a += 32, bpos += 32) {
                es_fill(s, a + 32 + ELOOK);
                const int pa = a + lane;
                const bool eq = pa < mlimit && es_byte(s, pa) == es_byte(s, bpos + lane);
                const unsigned ne = __ballot_sync(FULLMASK, !eq);
                const int cnum = ne ? __ffs(ne) - 1 : 32;
                mc += cnum;
                if (cnum < 32) break;
            }
            ip += mc + 4;
            NEED(op + 6 + (mc + 240) / 255);
            if (mc >= 15) {
                token_val += 15;
                const int rem = mc - 15, nff = rem / 255;
                for (int x = lane; x < nff; x += 32) dst[op + x] = 255;
                if (lane == 0) dst[op + nff] = (uint8_t)(rem % 255);
                op += nff + 1;
            } else {
                token_val += mc;
            }
            if (lane == 0) dst[token_pos] = (uint8_t)token_val;
        }
        // ---- after each match: insert ip - 2, look ip up, insert it; a hit is a match with
        // no literals (scalar path, identical on every lane)
        for (;;) {
            anchor = ip;
            if (ip >= mfl1) goto last_literals;
            if (ip + 64 > s.hi) es_fill(s, ip + ELOOK);
            uint32_t a0, a1, a2, a3;                         // bytes ip-2 .. ip+13
            {
                const uint32_t o = (uint32_t)(ip - 2) & (ERING - 1);
                const uint32_t wa = ring_s + (o & ~3u);
                const uint32_t sh = (o & 3) * 8;
                const uint32_t w0 = lds32(wa), w1 = lds32(wa + 4), w2 = lds32(wa + 8), w3 = lds32(wa + 12),
                               w4 = lds32(wa + 16);
                a0 = __funnelshift_r(w0, w1, sh);
                a1 = __funnelshift_r(w1, w2, sh);
                a2 = __funnelshift_r(w2, w3, sh);
                a3 = __funnelshift_r(w3, w4, sh);
            }
            const uint32_t v0 = __funnelshift_r(a0, a1, 16);   // bytes ip .. ip+3
            const uint32_t h2 = lz_hash_v<SMALL>(a0, a1 & 0xffu), h0 = lz_hash_v<SMALL>(v0, (a1 >> 16) & 0xffu);
            const uint32_t c = (h0 == h2) ? (uint32_t)(ip - 2) : lds_tab(tab_s + (h0 << TSH), SMALL);
            sts_tab(tab_s + (h2 << TSH), (uint32_t)(ip - 2), SMALL);
            sts_tab(tab_s + (h0 << TSH), (uint32_t)ip, SMALL);
            uint32_t cv, cn0, cn1;                            // bytes c .. c+11
            if ((int)c >= s.lo) {
                const uint32_t o = c & (ERING - 1);
                const uint32_t wa = ring_s + (o & ~3u);
                const uint32_t sh = (o & 3) * 8;
                const uint32_t w0 = lds32(wa), w1 = lds32(wa + 4), w2 = lds32(wa + 8), w3 = lds32(wa + 12);
                cv = __funnelshift_r(w0, w1, sh);
                cn0 = __funnelshift_r(w1, w2, sh);
                cn1 = __funnelshift_r(w2, w3, sh);
            } else {
                cv = ld4u(src + c);
                cn0 = ld4u(src + c + 4);
                cn1 = ld4u(src + c + 8);
            }
            if (!((SMALL || c + 65535u >= (uint32_t)ip) && cv == v0)) {
                ip += 1;
                __syncwarp();
                break;                                        // back to searching from ip + 1
            }
            const uint64_t nx = ((uint64_t)__funnelshift_r(a2, a3, 16) << 32) | __funnelshift_r(a1, a2, 16);
            const uint64_t x = nx ^ (((uint64_t)cn1 << 32) | cn0);
            const int lim = mlimit - (ip + 4);
            int mc = x ? (__ffsll((long long)x) - 1) >> 3 : 8;
            if (mc >= lim) {
                mc = lim;
            } else if (mc == 8) {                            // long match: warp-wide compare from ip + 12
                for (int a = ip + 12, bpos = (int)c + 12;; a += 32, bpos += 32) {
                    es_fill(s, a + 32 + ELOOK);
                    const int pa = a + lane;
                    const bool eq = pa < mlimit && es_byte(s, pa) == es_byte(s, bpos + lane);
                    const unsigned ne = __ballot_sync(FULLMASK, !eq);
                    const int cnum = ne ? __ffs(ne) - 1 : 32;
                    mc += cnum;
                    if (cnum < 32) break;
                }
            }
            const int mo = ip - (int)c;
            NEED(op + 9 + (mc >= 15 ? (mc + 240) / 255 : 0));
            if (lane == 0) {
                uint8_t *dp = dst + op;
                dp[0] = (uint8_t)(mc >= 15 ? 15 : mc);
                dp[1] = (uint8_t)mo;
                dp[2] = (uint8_t)(mo >> 8);
            }
            op += 3;
            if (mc >= 15) {
                const int rem = mc - 15, nff = rem / 255;
                for (int xx = lane; xx < nff; xx += 32) dst[op + xx] = 255;
                if (lane == 0) dst[op + nff] = (uint8_t)(rem % 255);
                op += nff + 1;
            }
            ip += mc + 4;
        }
    }
last_literals:
    {
        const int last = n - anchor;
        NEED(op + last + 1 + (last + 255 - 15) / 255);
        if (last >= 15) {
            const int rem = last - 15, nff = rem / 255;
            if (lane == 0) dst[op] = 15 << 4;
            for (int x = lane; x < nff; x += 32) dst[op + 1 + x] = 255;
            if (lane == 0) dst[op + 1 + nff] = (uint8_t)(rem % 255);
            op += nff + 2;
        } else {
            if (lane == 0) dst[op] = (uint8_t)(last << 4);
            op += 1;
        }
        for (int x = lane; x < last; x += 32) dst[op + x] = (uint8_t)es_byte(s, anchor + x);
        op += last;
    }
#undef TGET
#undef TPUT
#undef NEED
    __syncwarp();
    *need_out = need;
    return op;
}

// E2: one warp per stream: run check, then LZ4 into the stream's slot (capacity =
// stream length; a stream that does not shrink is stored raw).
// Streams are handed out dynamically (one atomic per stream): compressible streams cost
// far more than incompressible ones, and in shuffled float data they recur at a fixed
// stride, which a static round-robin assignment would pile onto the same warps.
__global__ void __launch_bounds__(32, 10) k_lz4_encode(const uint8_t *__restrict__ img, int64_t nstreams_total,
                                                    int neblock, uint8_t *slots, EncStream *es,
                                                    unsigned long long *next)
{
    extern __shared__ __align__(16) uint32_t sm_tab[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *tab = sm_tab + warp * (4096 + (ERING + 16) / 4);
    uint8_t *ring = reinterpret_cast<uint8_t *>(tab + 4096);
    for (;;) {
        unsigned long long got = 0;
        if (lane == 0) got = atomicAdd(next, 1ull);
        const int64_t sid = (int64_t)__shfl_sync(FULLMASK, got, 0);
        if (sid >= nstreams_total) break;
        const uint8_t *src = img + sid * neblock;
        const uint8_t first = __ldg(src);
        bool run = true;
        for (int base = 0; base < neblock && run; base += 32 * 16) {
            bool mine = true;
            for (int k = 0; k < 16; k++) {
                const int x = base + k * 32 + lane;
                if (x < neblock && __ldg(src + x) != first) mine = false;
            }
            run = __all_sync(FULLMASK, mine);
        }
        EncStream e;
        e.out = -1;
        if (run) {
            e.kind = SK_RUN; e.csize = first; e.need = 0;
        } else {
            int need = 0;
            const int cs = neblock < 65536 + 12 - 1
                               ? warp_lz4_compress<true>(src, neblock, slots + sid * neblock, neblock, tab, ring, &need)
                               : warp_lz4_compress<false>(src, neblock, slots + sid * neblock, neblock, tab, ring, &need);
            if (cs > 0 && cs < neblock) { e.kind = SK_LZ4; e.csize = cs; e.need = need; }
            else { e.kind = SK_RAW; e.csize = neblock; e.need = need; }
        }
        if (lane == 0) es[sid] = e;
        __syncwarp();
    }
}

// ---------------------------------------------------------------- LZ4 encoder, parallel parse
// The second encoder mode.  It writes standard LZ4 blocks (any LZ4 decoder, liblz4 and the
// reference's Blosc2 included, reads them back bit-exactly) but does not retrace liblz4's
// serial search, so its bytes differ from liblz4's.  One CTA of PT threads encodes one
// stream; per window of PW positions:
//  A. every position is hashed (4 bytes, 12 bits); its candidate is the latest position of
//     its bucket among the previous rounds of PT positions (the table keeps the largest
//     position written, so it is the same whatever the order of the writes), and the
//     previous position is a second candidate (runs); the longer match is kept, measured
//     up to PCAP bytes.  Every position enters the table.
//  B. the greedy parse (from the parse position, take the first position with a match of
//     at least 4 bytes, continue after it) is a chain over match positions: J[q] = the first
//     match position at or after q + L(q).  The chain is located by pointer doubling (J,
//     J^2, J^4, ... in two ping-pong tables, the chain doubled alongside), the sequences'
//     output sizes are prefix-summed across the CTA, and every thread writes its own
//     sequences.  A chain ends at the window end, after the window's last match, or at a
//     match of PCAP bytes or more, which is extended exactly before it is written.
// Format rules kept: offsets 1..65535, matches start at least 12 bytes before the end and
// end at least 5 bytes before it, so the block ends with >= 5 literals.
constexpr int PW = 1024;
constexpr int PT = 128;                   // threads per stream
constexpr int PCAP = 128;                 // match lengths measured in phase A (PCAP: at least PCAP)
constexpr uint16_t PJ_NONE = 0xFFFF, PJ_OUT = 0xFFFE, PJ_LONG = 0xFFFD;
constexpr int PSTAGE = 1024 + 16;         // staged bytes per probe window (from 4 before it)

struct ParSmem {              // per CTA
    union {
        uint16_t tab16[8192]; // liblz4 search (byU16); probe: four tables of 2048
        uint32_t tab32[4096]; // parallel parse: position + 1 of each bucket (0: empty); liblz4 byU32
    };
    uint8_t ring[ERING + 16];
    union {
        struct {
            uint16_t cw[PW];  // match distance of each window position
            uint8_t lw[PW];   // match length (0: none, 4..PCAP; PCAP: at least PCAP)
            uint16_t J[PW];   // the match after the one at each position, or why the chain stops
            uint16_t path[PW / 4 + 2];
        } w;
        uint8_t stage[4][PSTAGE];
    };
    uint32_t bits[32];        // match flags, one word per 32 positions
    int32_t nchain;           // matches on the window's chain
    int32_t red[8];           // block reductions
    long long sid;
};

// First match position at or after window offset rel (PJ_NONE: none left in the window).
__device__ __forceinline__ uint32_t par_next_match(const uint32_t *bits, int rel)
{
    if (rel >= PW) return PJ_OUT;
    int wi = rel >> 5;
    uint32_t m = bits[wi] & (0xFFFFFFFFu << (rel & 31));
    while (!m && ++wi < 32) m = bits[wi];
    return m ? (uint32_t)(wi * 32 + __ffs((int)m) - 1) : PJ_NONE;
}

__device__ __forceinline__ int lz4_seq_bytes(int lit, int ml)
{
    return 1 + (lit >= 15 ? 1 + (lit - 15) / 255 : 0) + lit + 2 + (ml >= 15 ? 1 + (ml - 15) / 255 : 0);
}

// One sequence (literals src[anchor, q), match at q, distance d, length L) at dst + o.
__device__ __forceinline__ void lz4_put_seq(const EncSrc &s, uint8_t *o, int anchor, int q, int d, int L)
{
    const int lit = q - anchor, ml = L - 4;
    int k = 1;
    if (lit >= 15) {
        int rem = lit - 15;
        for (; rem >= 255; rem -= 255) o[k++] = 255;
        o[k++] = (uint8_t)rem;
    }
    for (int x = 0; x < lit; x++) o[k + x] = (uint8_t)es_byte(s, anchor + x);
    k += lit;
    o[0] = (uint8_t)(((lit >= 15 ? 15 : lit) << 4) | (ml >= 15 ? 15 : ml));
    o[k] = (uint8_t)d;
    o[k + 1] = (uint8_t)(d >> 8);
    k += 2;
    if (ml >= 15) {
        int rem = ml - 15;
        for (; rem >= 255; rem -= 255) o[k++] = 255;
        o[k] = (uint8_t)rem;
    }
}

// 4 bytes at stream position x from the window (x must be inside it).
__device__ __forceinline__ uint32_t par_rd32(uint32_t ring_s, int x)
{
    const uint32_t o = (uint32_t)x & (ERING - 1);
    const uint32_t wa = ring_s + (o & ~3u);
    return __funnelshift_r(lds32(wa), lds32(wa + 4), (o & 3) * 8);
}

// es_fill for a whole CTA (every thread calls it with the same `want`).
__device__ __forceinline__ void cta_fill(EncSrc &s, int want)
{
    while (s.hi < s.n && s.hi < want) {
        const int base = s.hi, cnt = min(ESEG, s.n - base);
        __syncthreads();                                 // reads of the slots being replaced are done
        for (int x = threadIdx.x * 4; x < cnt; x += PT * 4) {
            uint32_t v = 0;
            if (base + x + 8 <= s.n) {
                v = ld4u(s.g + base + x);
            } else {
                for (int k = 0; k < 4; k++)
                    if (base + x + k < s.n) v |= (uint32_t)__ldg(s.g + base + x + k) << (8 * k);
            }
            const int o = (base + x) & (ERING - 1);
            *reinterpret_cast<uint32_t *>(s.r + o) = v;
            if (o < 16) *reinterpret_cast<uint32_t *>(s.r + ERING + o) = v;
        }
        s.hi = base + cnt;
        s.lo = max(s.lo, base + ESEG - ERING);
        __syncthreads();
    }
}

// Block-wide sum / min of one int per thread (uses red[]; ends with every thread holding
// the result and red[] free again).
__device__ __forceinline__ int cta_sum(int v, int32_t *red)
{
    v = (int)__reduce_add_sync(FULLMASK, (unsigned)v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int t = red[0] + red[1] + red[2] + red[3];
    __syncthreads();
    return t;
}

__device__ __forceinline__ int cta_min(int v, int32_t *red)
{
    v = (int)__reduce_min_sync(FULLMASK, (unsigned)v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int t = min(min(red[0], red[1]), min(red[2], red[3]));
    __syncthreads();
    return t;
}

__device__ __forceinline__ int cta_lz4_compress_par(const uint8_t *__restrict__ src, int n,
                                                    uint8_t *__restrict__ dst, int cap, ParSmem &S)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(S.ring);
    for (int i = tid; i < 4096 / 4; i += PT) reinterpret_cast<uint4 *>(S.tab32)[i] = make_uint4(0u, 0u, 0u, 0u);
    EncSrc s;
    s.g = src; s.r = S.ring; s.lo = 0; s.hi = 0; s.n = n;
    __syncthreads();
    int op = 0, anchor = 0, pos = 0;
    const int mfl1 = n - 11, mlimit = n - 5;
    for (int w0 = 0; n >= 13 && w0 < mfl1; w0 += PW) {
        const int wend = min(w0 + PW, mfl1), wn = wend - w0;
        cta_fill(s, wend + PCAP + 32);
        // ---- A: candidates and lengths.  Positions p .. p + PCAP + 4 lie in the window;
        // a candidate is read from the window when it is still there, else from global memory.
        // Rounds of 2 PT positions (two per thread; a round's positions see the table as it was
        // before the round).  The stream's first PT positions go in rounds of 32 and the next PT
        // in one round of PT, so that short streams keep table candidates for most positions.
        for (int q0 = 0, rsz; q0 < PW; q0 += rsz) {
            rsz = w0 + q0 < PT ? 32 : w0 + q0 < 2 * PT ? PT : 2 * PT;
            int p2[2];
            bool valid[2];
            uint32_t v2[2], h2[2], tv2[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int q = q0 + tid + k * PT;
                p2[k] = w0 + q;
                valid[k] = tid + k * PT < rsz && p2[k] < wend;
                v2[k] = valid[k] ? par_rd32(ring_s, p2[k]) : 0u;
                h2[k] = (v2[k] * 2654435761u) >> (32 - 12);
                tv2[k] = valid[k] ? S.tab32[h2[k]] : 0u;
            }
            __syncthreads();                             // every read of this round precedes its writes
#pragma unroll
            for (int k = 0; k < 2; k++)
                if (valid[k]) atomicMax(&S.tab32[h2[k]], (uint32_t)p2[k] + 1u);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int p = p2[k];
                const uint32_t v = v2[k];
                const int cand = (int)tv2[k] - 1;
                int L = 0, best = cand;
                const int lim = min(mlimit - p, PCAP);
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const int c = t ? p - 1 : cand;
                    if (!valid[k] || c >= p || c < 0 || p - c > 65535 || (t && c == cand)) continue;
                    // the previous position matches only inside a run: the 4 bytes at p are equal
                    if (t && v != (v & 0xFFu) * 0x01010101u) continue;
                    const bool inring = c >= s.lo;
                    if ((inring ? par_rd32(ring_s, c) : ld4u(src + c)) != v) continue;
                    int l = 4;
                    while (l < lim) {
                        const uint32_t x = par_rd32(ring_s, p + l) ^ (inring ? par_rd32(ring_s, c + l) : ld4u(src + c + l));
                        if (x) { l += (__ffs((int)x) - 1) >> 3; break; }
                        l += 4;
                    }
                    l = min(l, lim);
                    if (l > L) { L = l; best = c; }
                }
                const int q = q0 + tid + k * PT;
                if (tid + k * PT < rsz) {
                    S.w.cw[q] = (uint16_t)(p - best);
                    S.w.lw[q] = (uint8_t)L;
                }
                const unsigned bb = __ballot_sync(FULLMASK, L >= 4);
                if (lane == 0 && k * PT + warp * 32 < rsz) S.bits[((q0 + k * PT) >> 5) + warp] = bb;
            }
            __syncthreads();                             // this round's writes precede the next reads
        }
        // ---- B: chains of matches from the parse position
        while (pos < wend) {
            const uint32_t s0 = par_next_match(S.bits, pos - w0);
            if (s0 >= (uint32_t)wn) { pos = wend; break; }   // no match left: literals run on
            // J[q]: the match after the one at q, or why the chain stops there
            for (int q = tid; q < wn; q += PT) {
                const int L = S.w.lw[q];
                uint16_t j = PJ_NONE;
                if (L >= PCAP) j = PJ_LONG;
                else if (L >= 4) {
                    const uint32_t nx = par_next_match(S.bits, q + L);
                    j = nx >= (uint32_t)wn ? (q + L >= wn ? PJ_OUT : PJ_NONE) : (uint16_t)nx;
                }
                S.w.J[q] = j;
            }
            __syncthreads();
            // The chain from s0 by segment walks (warp 0): lane t walks J from the first match
            // at or after 32 t, recording the matches it visits; then, in rounds, lane t takes
            // the exit of lane t - 1 as its entry (lane 0: s0), follows its own walk once the
            // chain meets it and publishes its exit, until no exit changes.
            if (warp == 0) {
                const int lo = lane * 32, hi = lo + 32;
                const int nl = (wn + 31) / 32;              // lanes whose segment holds window positions
                const bool act = lane < nl;
                uint32_t mask = 0;
                int ex = PJ_NONE;
                if (act) {
                    int q = (int)par_next_match(S.bits, lo);
                    ex = q;
                    if (q < hi && q < wn) {
                        for (;;) {                          // positions grow: at most 32 steps
                            mask |= 1u << (q - lo);
                            const int v = S.w.J[q];
                            if (v >= hi || v >= wn) { ex = v; break; }
                            q = v;
                        }
                    }
                }
                uint32_t fm = 0;
                int cur = ex;
                for (int round = 0; round < 32; round++) {  // one round settles at least one more lane
                    int entry = __shfl_up_sync(FULLMASK, cur, 1);
                    if (lane == 0) entry = (int)s0;
                    uint32_t m = 0;
                    int e2 = entry;
                    if (act && entry < hi && entry < wn) {
                        int q = entry;
                        for (;;) {
                            const int b = q - lo;
                            if ((mask >> b) & 1u) { m |= mask & (~0u << b); e2 = ex; break; }
                            m |= 1u << b;
                            const int v = S.w.J[q];
                            if (v >= hi || v >= wn) { e2 = v; break; }
                            q = v;
                        }
                    }
                    const bool changed = act && e2 != cur;
                    fm = m;
                    cur = e2;
                    if (!__any_sync(FULLMASK, changed)) break;
                }
                const int chain_end = __shfl_sync(FULLMASK, cur, max(nl, 1) - 1);
                const int c = __popc(fm);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULLMASK, incl, o);
                    if (lane >= o) incl += v;
                }
                int o = incl - c;
                for (uint32_t x = fm; x; x &= x - 1) S.w.path[o++] = (uint16_t)(lo + __ffs((int)x) - 1);
                if (lane == 31) {
                    S.w.path[incl] = (uint16_t)chain_end;   // PJ_NONE, PJ_OUT or PJ_LONG
                    S.nchain = incl;
                }
            }
            __syncthreads();
            const int cnt = S.nchain;
            const uint16_t term = S.w.path[cnt];                // why the chain stopped
            // a capped last match: extend it exactly (CTA-wide) before writing it
            int lastL = S.w.lw[S.w.path[cnt - 1]];
            const int lastq = w0 + S.w.path[cnt - 1], lastd = S.w.cw[S.w.path[cnt - 1]];
            if (term == PJ_LONG) {
                for (;;) {
                    const int a = lastq + lastL;
                    cta_fill(s, a + PT + ELOOK);
                    const bool eq = a + tid < mlimit && es_byte(s, a + tid) == es_byte(s, a - lastd + tid);
                    const unsigned ne = __ballot_sync(FULLMASK, !eq);
                    const int cnum = cta_min(ne ? warp * 32 + __ffs((int)ne) - 1 : PT, S.red);
                    lastL += cnum;
                    if (cnum < PT) break;
                }
            }
            // output sizes
            int mine = 0;
            for (int i = tid; i < cnt; i += PT) {
                const int q = w0 + S.w.path[i];
                const int prev_end = i ? w0 + S.w.path[i - 1] + S.w.lw[S.w.path[i - 1]] : anchor;
                const int L = (i == cnt - 1) ? lastL : S.w.lw[S.w.path[i]];
                mine += lz4_seq_bytes(q - prev_end, L - 4);
            }
            const int total = cta_sum(mine, S.red);
            if (op + total + 1 + 6 > cap) return 0;
            // write: exclusive scan per round of PT sequences
            int base = op;
            for (int i0 = 0; i0 < cnt; i0 += PT) {
                const int i = i0 + tid;
                int sz = 0, q = 0, prev_end = 0, L = 0, d = 0;
                if (i < cnt) {
                    q = w0 + S.w.path[i];
                    prev_end = i ? w0 + S.w.path[i - 1] + S.w.lw[S.w.path[i - 1]] : anchor;
                    L = (i == cnt - 1) ? lastL : S.w.lw[S.w.path[i]];
                    d = S.w.cw[S.w.path[i]];
                    sz = lz4_seq_bytes(q - prev_end, L - 4);
                }
                int incl = sz;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(FULLMASK, incl, o);
                    if (lane >= o) incl += t;
                }
                if (lane == 31) S.red[warp] = incl;
                __syncthreads();
                int before = 0, all = 0;
#pragma unroll
                for (int k = 0; k < PT / 32; k++) {
                    const int t = S.red[k];
                    before += k < warp ? t : 0;
                    all += t;
                }
                if (i < cnt) lz4_put_seq(s, dst + base + before + incl - sz, prev_end, q, d, L);
                base += all;
                __syncthreads();
            }
            op = base;
            anchor = lastq + lastL;
            pos = anchor;
            if (term == PJ_NONE) { pos = max(pos, wend); }
        }
    }
    {
        const int last = n - anchor;
        if (op + 1 + last + (last + 240) / 255 > cap) return 0;
        uint8_t *o = dst + op;
        int k = 1;
        if (last >= 15) {
            const int rem = last - 15, nff = rem / 255;
            for (int x = tid; x < nff; x += PT) o[1 + x] = 255;
            if (tid == 0) o[1 + nff] = (uint8_t)(rem % 255);
            k += nff + 1;
        }
        if (tid == 0) o[0] = (uint8_t)((last >= 15 ? 15 : last) << 4);
        for (int x = tid; x < last; x += PT) o[k + x] = (uint8_t)es_byte(s, anchor + x);
        op += k + last;
    }
    __syncthreads();
    return op;
}

// Matches found in four sampled windows of 1024 positions (at 0, 1/4, 1/2 and 3/4 of the
// stream), one window per warp: positions with a 4-byte match against the warp's table of
// recent positions of the window (11-bit hash) or against the previous position.  Each
// window is staged in shared memory first by one round of coalesced word loads.  Returns
// the CTA's total.
__device__ __forceinline__ uint32_t stage_rd32(const uint8_t *stage, int o)
{
    const uint32_t *w = reinterpret_cast<const uint32_t *>(stage) + (o >> 2);
    return __funnelshift_r(w[0], w[1], (uint32_t)(o & 3) * 8);
}

__device__ __forceinline__ int cta_probe(const uint8_t *__restrict__ src, int n, ParSmem &S)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint16_t *tab = S.tab16 + w * 2048;
    uint8_t *stage = S.stage[w];
    for (int i = lane; i < 2048 / 8; i += 32) reinterpret_cast<uint4 *>(tab)[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
    const int base = (int)(((int64_t)(n - 11) * w / 4) & ~31);
    const int lim = min(n - 11, base + 1024);
    const int b0 = base >= 4 ? base - 4 : 0;                 // word aligned: base is a multiple of 32
    const int cnt = min(PSTAGE, n - b0);
    for (int x = lane * 4; x < cnt; x += 128) {
        uint32_t v = 0;
        if (b0 + x + 8 <= n) {                               // ld4u reads 8 bytes
            v = ld4u(src + b0 + x);
        } else {
            for (int k = 0; k < 4; k++)
                if (b0 + x + k < n) v |= (uint32_t)__ldg(src + b0 + x + k) << (8 * k);
        }
        *reinterpret_cast<uint32_t *>(stage + x) = v;
    }
    __syncwarp();
    int hits = 0;
    for (int r = 0; r < 32; r++) {
        const int p = base + r * 32 + lane;
        const bool valid = p < lim;
        const uint32_t v = valid ? stage_rd32(stage, p - b0) : 0u;
        const uint32_t h = (v * 2654435761u) >> (32 - 11);
        const uint32_t c = valid ? tab[h] : 0xFFFFu;
        __syncwarp();
        if (valid) tab[h] = (uint16_t)p;
        const bool m = valid && ((c < (uint32_t)p && c >= (uint32_t)b0 && stage_rd32(stage, (int)c - b0) == v) ||
                                 (p > b0 && stage_rd32(stage, p - 1 - b0) == v));
        hits += __popc(__ballot_sync(FULLMASK, m));
    }
    return cta_sum(lane == 0 ? hits : 0, S.red);
}

// E2 (parallel mode): one CTA of PT threads per stream, streams handed out dynamically.  A
// probe of four sampled windows routes each stream: almost no matches (incompressible
// byte planes): stored raw; few matches: the liblz4 search (one warp), whose accelerating
// skip makes them cheap; the rest: the parallel parse.
__global__ void __launch_bounds__(PT, 8) k_lz4_encode_par(const uint8_t *__restrict__ img, int64_t nstreams_total,
                                                       int neblock, uint8_t *slots, EncStream *es,
                                                       unsigned long long *next)
{
    extern __shared__ __align__(16) uint8_t sm_par[];
    ParSmem &S = *reinterpret_cast<ParSmem *>(sm_par);
    const int tid = threadIdx.x, warp = tid >> 5;
    for (;;) {
        if (tid == 0) S.sid = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const int64_t sid = S.sid;
        __syncthreads();
        if (sid >= nstreams_total) break;
        const uint8_t *src = img + sid * neblock;
        const uint8_t first = __ldg(src);
        bool run = true;
        for (int b = 0; b < neblock && run; b += PT * 16) {
            bool mine = true;
            for (int k = 0; k < 16; k++) {
                const int x = b + k * PT + tid;
                if (x < neblock && __ldg(src + x) != first) mine = false;
            }
            run = __syncthreads_and(mine);
        }
        EncStream e;
        e.out = -1;
        if (run) {
            e.kind = SK_RUN; e.csize = first; e.need = 0;
        } else {
            const int hits = cta_probe(src, neblock, S);
            if (hits < 16) {                     // no matches to speak of: store the stream raw
                e.kind = SK_RAW; e.csize = neblock; e.need = neblock + 1;
            } else if (hits < 256) {
                if (warp == 0) {
                    int need = 0;
                    const int cs = neblock < 65536 + 12 - 1
                                       ? warp_lz4_compress<true>(src, neblock, slots + sid * neblock, neblock, S.tab32, S.ring, &need)
                                       : warp_lz4_compress<false>(src, neblock, slots + sid * neblock, neblock, S.tab32, S.ring, &need);
                    if (cs > 0 && cs < neblock) { e.kind = SK_LZ4; e.csize = cs; e.need = need; }
                    else { e.kind = SK_RAW; e.csize = neblock; e.need = need; }
                }
            } else {
                const int cs = cta_lz4_compress_par(src, neblock, slots + sid * neblock, neblock, S);
                if (cs > 0 && cs < neblock) { e.kind = SK_LZ4; e.csize = cs; e.need = cs; }
                else { e.kind = SK_RAW; e.csize = neblock; e.need = neblock + 1; }
            }
        }
        if (tid == 0) es[sid] = e;
        __syncthreads();
    }
}

// E3: per chunk (one CTA each), the stream layout blosc_c produces: streams in order, each a
// 4-byte csize word and its payload (a run: one byte or none), an LZ4 stream only where its
// output fits the space left (else raw); a chunk that does not fit nbytes + 32 is stored
// memcpyed.  The space left only binds near the end of a chunk, so sizes are prefix-summed
// as if it never binds, and thread 0 replays the stream-by-stream walk from the first stream
// where it could.
constexpr int LAYOUT_T = 256;

// The blosc_c walk for one stream from running size ntb; false: the chunk does not fit.
__device__ __forceinline__ bool layout_step(EncStream &e, int64_t &ntb, int64_t destsize, int neblock)
{
    ntb += 4;
    if (e.kind == SK_RUN) {
        if (ntb > destsize) return false;
        e.out = (int32_t)(ntb - 4);
        if (e.csize != 0) {
            if (ntb + 1 > destsize) return false;
            ntb += 1;
        }
        return true;
    }
    int64_t maxout = neblock;
    if (ntb + maxout > destsize) {
        maxout = destsize - ntb;
        if (maxout <= 0) return false;
    }
    int64_t sz;
    if (e.kind == SK_LZ4 && e.need <= maxout) {
        sz = e.csize;
    } else {
        if (ntb + neblock > destsize) return false;
        e.kind = SK_RAW;
        sz = neblock;
    }
    e.out = (int32_t)(ntb - 4);
    ntb += sz;
    return true;
}

// memcpy_only (compression level 0): c-blosc2 stores every chunk memcpyed.
__device__ __forceinline__ void layout_chunk(const Geom &g, int nstreams, int neblock, EncStream *es, EncChunk *ec,
                                             int memcpy_only, int64_t c, int64_t *wsum, int64_t &s_before, int &s_first)
{
    const int64_t destsize = g.chunk_nbytes + 32, ns = g.nblocks * nstreams;
    if (memcpy_only) {
        if (threadIdx.x == 0) { ec[c].memcpyed = 1; ec[c].cbytes = (int32_t)destsize; }
        return;
    }
    const int64_t ntb0 = 32 + 4 * g.nblocks;
    EncStream *e0 = es + c * ns;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_first = 0x7FFFFFFF;
    __syncthreads();
    int64_t base = ntb0;
    for (int64_t r0 = 0; ntb0 <= destsize && r0 < ns; r0 += LAYOUT_T) {
        const int64_t i = r0 + threadIdx.x;
        EncStream e;
        e.kind = SK_RAW; e.csize = 0; e.need = 0; e.out = -1;
        int64_t sz = 0;
        if (i < ns) {
            e = e0[i];
            sz = e.kind == SK_RUN ? 4 + (e.csize != 0) : e.kind == SK_LZ4 ? 4 + (int64_t)e.csize : 4 + (int64_t)neblock;
        }
        int64_t incl = sz;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(FULLMASK, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        int64_t before = base + incl - sz, all = 0;
#pragma unroll
        for (int w = 0; w < LAYOUT_T / 32; w++) {
            before += w < warp ? wsum[w] : 0;
            all += wsum[w];
        }
        // the unconstrained choice holds while the stream (raw, at worst) still fits
        const bool safe = e.kind == SK_RUN ? before + sz <= destsize
                                           : before + 4 + neblock <= destsize && (e.kind != SK_LZ4 || e.need <= neblock);
        if (i < ns && !safe) atomicMin(&s_first, (int)i);
        __syncthreads();
        const int first = s_first;
        if (i < ns && i < first) e0[i].out = (int32_t)before;
        if (i == first) s_before = before;
        base += all;
        __syncthreads();
        if (first != 0x7FFFFFFF) break;
    }
    if (threadIdx.x == 0) {
        bool ok = ntb0 <= destsize;
        int64_t ntb = base;
        if (ok && s_first != 0x7FFFFFFF) {
            ntb = s_before;
            for (int64_t i = s_first; ok && i < ns; i++) ok = layout_step(e0[i], ntb, destsize, neblock);
        }
        ec[c].memcpyed = ok ? 0 : 1;
        ec[c].cbytes = (int32_t)(ok ? ntb : destsize);
    }
}

__global__ void __launch_bounds__(LAYOUT_T) k_layout(Geom g, int nstreams, int neblock, EncStream *es, EncChunk *ec,
                                                    int memcpy_only)
{
    __shared__ int64_t wsum[LAYOUT_T / 32];
    __shared__ int64_t s_before;
    __shared__ int s_first;
    layout_chunk(g, nstreams, neblock, es, ec, memcpy_only, blockIdx.x, wsum, s_before, s_first);
}

// Chunk offsets: exclusive scan of the chunk sizes (one CTA).
__device__ __forceinline__ void chunk_offsets(int64_t nchunks, EncChunk *ec, int64_t *total, int64_t *wsum)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t base = 0;
    for (int64_t r0 = 0; r0 < nchunks; r0 += 1024) {
        const int64_t i = r0 + threadIdx.x;
        const int64_t v = i < nchunks ? ec[i].cbytes : 0;
        int64_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(FULLMASK, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        int64_t before = base + incl - v, all = 0;
        for (int w = 0; w < 32; w++) {
            before += w < warp ? wsum[w] : 0;
            all += wsum[w];
        }
        if (i < nchunks) ec[i].offset = before;
        base += all;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = base;
}

__global__ void __launch_bounds__(1024) k_chunk_offsets(int64_t nchunks, EncChunk *ec, int64_t *total)
{
    __shared__ int64_t wsum[32];
    chunk_offsets(nchunks, ec, total, wsum);
}

// Copies len bytes with the whole CTA: 16-byte aligned stores to dst, each fed by five
// aligned 32-bit loads of src funnel-shifted into place.  Source words are only read
// inside [lo, hi); pieces whose words would leave it are copied bytewise.
__device__ __forceinline__ void cta_copy(uint8_t *__restrict__ dst, const uint8_t *__restrict__ src, int len,
                                         const uint8_t *lo, const uint8_t *hi)
{
    int head = (int)((16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15);
    if (head > len) head = len;
    for (int x = threadIdx.x; x < head; x += blockDim.x) dst[x] = __ldg(src + x);
    const int nvec = (len - head) >> 4;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const int s = head + (v << 4);
        const uint8_t *sp = src + s;
        const uint8_t *sa = reinterpret_cast<const uint8_t *>(reinterpret_cast<uintptr_t>(sp) & ~uintptr_t(3));
        uint4 o;
        if (sa >= lo && sa + 20 <= hi) {
            const uint32_t *w = reinterpret_cast<const uint32_t *>(sa);
            const uint32_t sh = (uint32_t)(reinterpret_cast<uintptr_t>(sp) & 3) * 8;
            const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2), w3 = __ldg(w + 3), w4 = __ldg(w + 4);
            o.x = __funnelshift_r(w0, w1, sh);
            o.y = __funnelshift_r(w1, w2, sh);
            o.z = __funnelshift_r(w2, w3, sh);
            o.w = __funnelshift_r(w3, w4, sh);
        } else {
            uint32_t b[4];
            for (int k = 0; k < 4; k++)
                b[k] = (uint32_t)__ldg(sp + 4 * k) | ((uint32_t)__ldg(sp + 4 * k + 1) << 8) |
                       ((uint32_t)__ldg(sp + 4 * k + 2) << 16) | ((uint32_t)__ldg(sp + 4 * k + 3) << 24);
            o = make_uint4(b[0], b[1], b[2], b[3]);
        }
        *reinterpret_cast<uint4 *>(dst + s) = o;
    }
    for (int x = head + (nvec << 4) + threadIdx.x; x < len; x += blockDim.x) dst[x] = __ldg(src + x);
}

// E5: write headers, bstarts, csize words and payloads.  One CTA per (chunk, block).
__device__ __forceinline__ void emit_block(const Geom &g, int nstreams, int neblock, bool shuffle, int splitflag,
                                           const uint8_t *__restrict__ img, const uint8_t *__restrict__ slots,
                                           int64_t img_bytes, const EncStream *__restrict__ es,
                                           const EncChunk *__restrict__ ec, uint8_t *__restrict__ outbuf, int64_t t)
{
    const int ts = g.itemsize;
    do {
        const int64_t c = t / g.nblocks, b = t - c * g.nblocks;
        const EncChunk cc = ec[c];
        uint8_t *chunk = outbuf + cc.offset;
        if (b == 0 && threadIdx.x < 32) {
            const int flags = 0x05 | (1 << 5) | (splitflag ? 0 : 0x10) | (cc.memcpyed ? 0x02 : 0);
            uint8_t hb = 0;
            const int x = threadIdx.x;
            if (x == 0) hb = 5;
            else if (x == 1) hb = 1;
            else if (x == 2) hb = (uint8_t)flags;
            else if (x == 3) hb = (uint8_t)ts;
            else if (x >= 4 && x < 8) hb = (uint8_t)(g.chunk_nbytes >> (8 * (x - 4)));
            else if (x >= 8 && x < 12) hb = (uint8_t)(g.blocksize >> (8 * (x - 8)));
            else if (x >= 12 && x < 16) hb = (uint8_t)((uint32_t)cc.cbytes >> (8 * (x - 12)));
            else if (x == 21) hb = shuffle ? 1 : 0;
            else if (x == 22) hb = 1;   // compcode LZ4
            chunk[x] = hb;
        }
        const uint8_t *blk_img = img + t * g.blocksize;
        if (cc.memcpyed) {
            uint8_t *dst = chunk + 32 + b * g.blocksize;
            for (int64_t x = threadIdx.x; x < g.blocksize; x += blockDim.x) {
                uint8_t v;
                if (shuffle) { const int64_t i = x / ts, j = x - i * ts; v = blk_img[j * g.blockn + i]; }
                else v = blk_img[x];
                dst[x] = v;
            }
            continue;
        }
        const EncStream *bs = es + t * nstreams;
        if (threadIdx.x == 0) {
            const int32_t bstart = bs[0].out;
            uint8_t *p = chunk + 32 + 4 * b;
            p[0] = (uint8_t)bstart; p[1] = (uint8_t)(bstart >> 8); p[2] = (uint8_t)(bstart >> 16); p[3] = (uint8_t)(bstart >> 24);
        }
        for (int j = 0; j < nstreams; j++) {
            const EncStream e = bs[j];
            uint8_t *w = chunk + e.out;
            int32_t word;
            const uint8_t *payload = nullptr;
            int plen = 0;
            if (e.kind == SK_RUN) { word = -e.csize; }
            else if (e.kind == SK_LZ4) { word = e.csize; payload = slots + (t * nstreams + j) * (int64_t)neblock; plen = e.csize; }
            else { word = neblock; payload = blk_img + (int64_t)j * neblock; plen = neblock; }
            if (threadIdx.x < 4) w[threadIdx.x] = (uint8_t)((uint32_t)word >> (8 * threadIdx.x));
            if (e.kind == SK_RUN && e.csize != 0 && threadIdx.x == 4) w[4] = 1;
            if (plen > 0) {
                const uint8_t *base = e.kind == SK_LZ4 ? slots : img;
                cta_copy(w + 4, payload, plen, base, base + img_bytes);
            }
        }
    } while (false);
}

__global__ void __launch_bounds__(256) k_emit(Geom g, int nstreams, int neblock, bool shuffle, int splitflag,
                                              const uint8_t *__restrict__ img, const uint8_t *__restrict__ slots,
                                              int64_t img_bytes,
                                              const EncStream *__restrict__ es, const EncChunk *__restrict__ ec,
                                              uint8_t *__restrict__ outbuf)
{
    for (int64_t t = blockIdx.x; t < g.nchunks * g.nblocks; t += gridDim.x)
        emit_block(g, nstreams, neblock, shuffle, splitflag, img, slots, img_bytes, es, ec, outbuf, t);
}

// ============================================================================ host launchers
static int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int decode_container(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, const int64_t *d_off, const int32_t *d_len,
                     void *out, int64_t ld, cudaStream_t st)
{
    DecodeWork w;
    int r = decode_launch(g, d_chunks, chunks_bytes, d_off, d_len, out, ld, st, &w);
    if (r) return r;
    return decode_finish(&w, st);
}

int decode_finish(DecodeWork *w, cudaStream_t st)
{
    int h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int *cnt = w->ext_counters ? w->ext_counters : w->counters.as<int>();
    cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -101;
    w->nzero = h[4];
    return h[1];
}

// Grid of the fast scatter: the CTAs resident at once (one wave), at most one per slice.
template <int TS>
static int64_t scatter_fast_grid(const Geom &g, int64_t nbl)
{
    static int per_sm = 0;
    if (!per_sm) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_scatter_fast<TS>, 256, 0) != cudaSuccess || n < 1) {
            cudaGetLastError();
            n = 4;
        }
        per_sm = n;
    }
    const int64_t units = nbl * ((g.blockn + SC_ITEMS - 1) / SC_ITEMS);
    return std::max<int64_t>(std::min<int64_t>(units, (int64_t)sm_count() * per_sm), 1);
}

int64_t decode_max_jobs(const Geom &g) { return g.nchunks * g.nblocks * 8; }

int decode_queue_init(DecodeQueue *q, int64_t max_jobs, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (!q->jobs.allocate(sizeof(Lz4Job) * (size_t)std::max<int64_t>(max_jobs, 1), dev) || !q->counters.allocate(64, dev))
        return -100;
    q->cap = max_jobs;
    cudaMemsetAsync(q->counters.p, 0, 64, st);
    return 0;
}

int decode_parse(const DecodeArgs &a, DecodeQueue *q, DecodeWork *w, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const Geom &g = a.g;
    const int64_t nbl = g.nchunks * g.nblocks;
    if (!w->bd.allocate(sizeof(BlockDesc) * nbl, dev) || !w->sd.allocate(sizeof(StreamDesc) * nbl * 8, dev) ||
        !w->scratch.allocate((size_t)(nbl * g.blocksize), dev) || (!w->ext_counters && !w->counters.allocate(64, dev)))
        return -100;
    int *cnt = w->ext_counters ? w->ext_counters : w->counters.as<int>();
    cudaMemsetAsync(cnt, 0, 64, st);
    const int threads = 128;
    const int64_t blocks = std::min<int64_t>((nbl + threads - 1) / threads, (int64_t)sm_count() * 16);
    if (!w->zf.allocate((size_t)std::max<int64_t>(nbl, 1), dev)) return -100;
    IAB_TIMED("k_parse", st, k_parse<<<(unsigned)std::max<int64_t>(blocks, 1), threads, 0, st>>>(
        g, a.chunks, a.off, a.len, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), q->jobs.as<Lz4Job>(),
        q->counters.as<int>(), q->cap, cnt + 1, w->scratch.as<uint8_t>(), w->zf.as<uint8_t>(), cnt + 4));
    return 0;
}

int decode_lz4(DecodeQueue *q, cudaStream_t st)
{
    static bool attr = false;
    const int smem = (int)sizeof(dcta::Smem);
    if (!attr) {
        cudaFuncSetAttribute(k_lz4_decode_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    int *qc = q->counters.as<int>();
    IAB_TIMED("k_lz4_decode_cta", st, k_lz4_decode_cta<<<sm_count() * 6, dcta::THREADS, smem, st>>>(
        q->jobs.as<Lz4Job>(), qc, q->cap, reinterpret_cast<unsigned *>(qc + 1)));
    return 0;
}

int decode_scatter(const DecodeArgs &a, DecodeWork *w, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const Geom &g = a.g;
    const int64_t nbl = g.nchunks * g.nblocks;
    int *cnt = w->ext_counters ? w->ext_counters : w->counters.as<int>();
    const int sms = sm_count();
    const uint8_t *scratch = w->scratch.as<uint8_t>();
    const int64_t tpb = (g.blockn + TILE - 1) / TILE;
    const int64_t blocks = std::min<int64_t>(nbl * tpb, (int64_t)sms * 8);
    const bool fast = g.itemsize == 4 || g.itemsize == 8;
    int *rest = nullptr, *nrest = cnt + 3;
    if (fast) {
        if (!w->rest.allocate(sizeof(int) * (size_t)nbl, dev)) return -100;
        rest = w->rest.as<int>();
        const uint8_t *cend = a.chunks + a.chunks_bytes, *send = scratch + nbl * g.blocksize;
        if (g.itemsize == 8)
            IAB_TIMED("k_scatter_fast", st, k_scatter_fast<8><<<(unsigned)scatter_fast_grid<8>(g, nbl), 256, 0, st>>>(
                g, a.chunks, cend, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), scratch, send, (uint8_t *)a.out, a.ld,
                rest, nrest, cnt + 1));
        else
            IAB_TIMED("k_scatter_fast", st, k_scatter_fast<4><<<(unsigned)scatter_fast_grid<4>(g, nbl), 256, 0, st>>>(
                g, a.chunks, cend, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), scratch, send, (uint8_t *)a.out, a.ld,
                rest, nrest, cnt + 1));
    }
    IAB_TIMED("k_scatter", st, k_scatter<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(
        g, rest, nrest, a.chunks, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), scratch, (uint8_t *)a.out, a.ld));
    return 0;
}

int decode_launch(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, const int64_t *d_off, const int32_t *d_len, void *out,
                  int64_t ld, cudaStream_t st, DecodeWork *w)
{
    const DecodeArgs a{g, d_chunks, chunks_bytes, d_off, d_len, out, ld};
    int r = decode_queue_init(&w->queue, decode_max_jobs(g), st);
    if (!r) r = decode_parse(a, &w->queue, w, st);
    if (!r) r = decode_lz4(&w->queue, st);
    if (!r) r = decode_scatter(a, w, st);
    return r;
}

// c-blosc2's split rule for LZ4 (always / never / automatic: LZ4 + shuffle, typesize <= 16
// and at least 32 items per block); a split block has one stream per item byte.
static bool encode_split(const Geom &g, bool shuffle, int splitmode)
{
    if (splitmode == 1) return true;
    if (splitmode == 2) return false;
    return shuffle && g.itemsize <= 16 && (g.blocksize / g.itemsize) >= 32;
}

int encode_nstreams(const Geom &g, bool shuffle, int splitmode)
{
    return encode_split(g, shuffle, splitmode) ? g.itemsize : 1;
}

int encode_gather(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode, EncodeWork *w, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int ts = g.itemsize;
    const int64_t nbl = g.nchunks * g.nblocks;
    const int64_t img_bytes = nbl * g.blocksize;
    const int nstreams = encode_nstreams(g, shuffle, splitmode);
    const bool ext = w->ext_img != nullptr;
    const bool ready = w->img_ready && !ext && w->img.n >= (size_t)img_bytes;
    if ((!ext && ((!ready && !w->img.allocate(img_bytes, dev)) || !w->slots.allocate(img_bytes, dev) ||
                  !w->es.allocate(sizeof(EncStream) * nbl * nstreams, dev))) ||
        (!w->ext_chunks && !w->ec.allocate(sizeof(EncChunk) * g.nchunks, dev)) || !w->tot.allocate(64, dev))
        return -100;
    w->nchunks = g.nchunks;
    uint8_t *img = ext ? w->ext_img : w->img.as<uint8_t>();
    cudaMemsetAsync(w->tot.p, 0, 64, st);
    if (ready) return 0;                   // the product wrote the image
    const int sms = sm_count();
    const int64_t tpb = (g.blockn + TILE - 1) / TILE;
    const int64_t blocks = std::min<int64_t>(nbl * tpb, (int64_t)sms * 8);
    const bool fast = shuffle && (ts == 4 || ts == 8);
    if (fast) {
        const int64_t fb = std::min<int64_t>(nbl, (int64_t)sms * 8);
        if (ts == 8)
            IAB_TIMED("k_gather_fast", st, k_gather_fast<8><<<(unsigned)std::max<int64_t>(fb, 1), 256, 0, st>>>(
                g, (const uint8_t *)in, ld, img));
        else
            IAB_TIMED("k_gather_fast", st, k_gather_fast<4><<<(unsigned)std::max<int64_t>(fb, 1), 256, 0, st>>>(
                g, (const uint8_t *)in, ld, img));
    }
    // the general gather covers the partitions the fast one does not take
    const bool all_fast = fast && !(g.block[1] & 3);
    if (!all_fast)
        IAB_TIMED("k_gather", st, k_gather<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(
            g, fast, (const uint8_t *)in, ld, shuffle, img));
    return 0;
}

void encode_streams(const uint8_t *img, int64_t ns, int neblock, uint8_t *slots, EncStream *es,
                    unsigned long long *cursor, bool exact_lz4, cudaStream_t st)
{
    const int sms = sm_count();
    if (exact_lz4) {
        static bool attr = false;
        // per warp: 16 KiB hash table + the source window; 1 warp per CTA, 10 CTAs per SM
        const int wpb = 1, smem = wpb * (4096 * 4 + ERING + 16);
        if (!attr) {
            cudaFuncSetAttribute(k_lz4_encode, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            attr = true;
        }
        const int64_t blocks = std::min<int64_t>((ns + wpb - 1) / wpb, (int64_t)sms * 10);
        IAB_TIMED("k_lz4_encode", st, k_lz4_encode<<<(unsigned)std::max<int64_t>(blocks, 1), wpb * 32, smem, st>>>(
            img, ns, neblock, slots, es, cursor));
    } else {
        static bool attr = false;
        const int smem = (int)sizeof(ParSmem);                 // one stream per CTA of PT threads, 8 CTAs per SM
        if (!attr) {
            cudaFuncSetAttribute(k_lz4_encode_par, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            attr = true;
        }
        const int64_t blocks = std::min<int64_t>(ns, (int64_t)sms * 8);
        IAB_TIMED("k_lz4_encode_par", st, k_lz4_encode_par<<<(unsigned)std::max<int64_t>(blocks, 1), PT, smem, st>>>(
            img, ns, neblock, slots, es, cursor));
    }
}

int encode_emit(const Geom &g, bool shuffle, int splitmode, DevBuf *d_out, EncodeWork *w, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int64_t nbl = g.nchunks * g.nblocks;
    const int64_t img_bytes = nbl * g.blocksize;
    const int nstreams = encode_nstreams(g, shuffle, splitmode);
    const int neblock = (int)(g.blocksize / nstreams);
    if (!d_out->allocate((size_t)(g.nchunks * (g.chunk_nbytes + 32)), dev)) return -100;
    const bool ext = w->ext_img != nullptr;
    const uint8_t *img = ext ? w->ext_img : w->img.as<uint8_t>();
    const uint8_t *slots = ext ? w->ext_slots : w->slots.as<uint8_t>();
    EncStream *es = ext ? w->ext_es : w->es.as<EncStream>();
    EncChunk *ec = w->ext_chunks ? w->ext_chunks : w->ec.as<EncChunk>();
    IAB_TIMED("k_layout", st, k_layout<<<(unsigned)std::max<int64_t>(g.nchunks, 1), LAYOUT_T, 0, st>>>(
        g, nstreams, neblock, es, ec, w->memcpy_only ? 1 : 0));
    IAB_TIMED("k_chunk_offsets", st, k_chunk_offsets<<<1, 1024, 0, st>>>(g.nchunks, ec, w->tot.as<int64_t>()));
    const int64_t blocks = std::min<int64_t>(nbl, (int64_t)sm_count() * 8);
    IAB_TIMED("k_emit", st, k_emit<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(
        g, nstreams, neblock, shuffle, encode_split(g, shuffle, splitmode) ? 1 : 0, img, slots, img_bytes, es, ec,
        d_out->as<uint8_t>()));
    return 0;
}

int encode_launch(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode, DevBuf *d_out, EncodeWork *w,
                  cudaStream_t st)
{
    w->ext_img = nullptr;
    w->ext_slots = nullptr;
    w->ext_es = nullptr;
    const int r = encode_gather(g, in, ld, shuffle, splitmode, w, st);
    if (r) return r;
    const int nstreams = encode_nstreams(g, shuffle, splitmode);
    if (!w->memcpy_only)
        encode_streams(w->img.as<uint8_t>(), g.nchunks * g.nblocks * nstreams, (int)(g.blocksize / nstreams),
                       w->slots.as<uint8_t>(), w->es.as<EncStream>(),
                       reinterpret_cast<unsigned long long *>(w->tot.as<int64_t>() + 1), w->exact_lz4, st);
    return encode_emit(g, shuffle, splitmode, d_out, w, st);
}

int encode_finish(EncodeWork *w, std::vector<int64_t> *h_off, std::vector<int32_t> *h_len, cudaStream_t st)
{
    const int64_t n = w->nchunks;
    std::vector<EncChunk> hc((size_t)n);
    const EncChunk *ec = w->ext_chunks ? w->ext_chunks : w->ec.as<EncChunk>();
    cudaMemcpyAsync(hc.data(), ec, sizeof(EncChunk) * n, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -101;
    h_off->resize((size_t)n);
    h_len->resize((size_t)n);
    for (int64_t c = 0; c < n; c++) { (*h_off)[c] = hc[c].offset; (*h_len)[c] = hc[c].cbytes; }
    return 0;
}

bool encode_image_ok(const Geom &g, bool shuffle, bool memcpy_only)
{
    return g.ndim == 2 && g.itemsize == 8 && shuffle && !memcpy_only && g.nchunks > 0 && !(g.block[1] & 3) &&
           !(g.chunk[1] & 3) && g.blocksize > 0;
}

int encode_image_prepare(const Geom &g, EncodeWork *w)
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (!w->img.allocate((size_t)(g.nchunks * g.nblocks * g.blocksize), dev)) return -100;
    w->img_ready = true;
    return 0;
}

int encode_image_finish(const Geom &g, bool shuffle, int splitmode, DevBuf *d_out, std::vector<int64_t> *h_off,
                        std::vector<int32_t> *h_len, cudaStream_t st, bool exact_lz4, EncodeWork *w)
{
    if (!w->img_ready) return -1;
    w->exact_lz4 = exact_lz4;
    w->memcpy_only = false;
    const int r = encode_launch(g, nullptr, 0, shuffle, splitmode, d_out, w, st);
    if (r) return r;
    return encode_finish(w, h_off, h_len, st);
}

int encode_container(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode, DevBuf *d_out,
                     std::vector<int64_t> *h_off, std::vector<int32_t> *h_len, cudaStream_t st, bool exact_lz4,
                     bool memcpy_only)
{
    EncodeWork w;
    w.exact_lz4 = exact_lz4;
    w.memcpy_only = memcpy_only;
    const int r = encode_launch(g, in, ld, shuffle, splitmode, d_out, &w, st);
    if (r) return r;
    return encode_finish(&w, h_off, h_len, st);
}

// ============================================================================ decode-fused GEMV
// y = A x straight from A's chunks, after the parse and the LZ4 launch: the dense A is never
// written.  A unit is one slice of whole rows of one block (SC_ITEMS / block[1] rows): its items
// are rebuilt as the scatter rebuilds them (word-level from the staged byte planes for shuffled
// split blocks, item by item from the stream descriptors otherwise), multiplied by x over the
// block's columns, and each row's sum is stored in part[jb * M + row] (jb: the block's column in
// the global block grid); k_gemv_rows then sums part over jb in order.  Every sum runs in a fixed
// order, so the result does not vary from run to run.

// Item i of a block from its stream descriptors (any block mode).
__device__ __forceinline__ uint64_t item_bits(const Geom &g, const uint8_t *__restrict__ ch, const BlockDesc &d,
                                              const StreamDesc *__restrict__ s, const uint8_t *__restrict__ blk_scratch,
                                              int64_t i)
{
    const int ts = g.itemsize;
    if (d.mode == BM_NAN) return ts == 8 ? 0x7FF8000000000000ull : 0x7FC00000ull;
    if (d.mode == BM_VALUE) return load_item_bytes(ch + d.value_src, ts);
    uint64_t v = 0;
    for (int j = 0; j < ts; j++) {
        const int64_t pos = d.mode == BM_SHUFFLED ? (int64_t)j * g.blockn + i : i * ts + j;
        const int sidx = (int)(pos / d.neblock);
        const int64_t so = pos - (int64_t)sidx * d.neblock;
        const StreamDesc q = s[sidx];
        uint8_t b;
        if (q.kind == SK_RUN) b = (uint8_t)q.len;
        else if (q.kind == SK_RAW) b = __ldg(ch + q.src + so);
        else b = __ldcg(blk_scratch + (int64_t)sidx * d.neblock + so);
        v |= (uint64_t)b << (8 * j);
    }
    return v;
}

template <typename T> __device__ __forceinline__ T bits_as(uint64_t v);
template <> __device__ __forceinline__ float bits_as<float>(uint64_t v) { return __uint_as_float((uint32_t)v); }
template <> __device__ __forceinline__ double bits_as<double>(uint64_t v) { return __longlong_as_double((long long)v); }

// One unit of the fused GEMV: one slice of whole rows of one block (block-uniform values).
struct GvUnit {
    int64_t t, jb;
    BlockSpan sp;
    BlockDesc d;
    int r0, nrow, i0s, cnt;
    bool active, fast;         // active: the slice holds logical items; fast: word-level path
};

__device__ __forceinline__ GvUnit gv_unit(const Geom &g, const BlockDesc *__restrict__ bd, int64_t u, int64_t nsl,
                                          int rps, int ts)
{
    GvUnit w;
    int64_t s64, c, b, cq, cr, bq, br;
    divmod(u, nsl, w.t, s64);
    divmod(w.t, g.nblocks, c, b);
    w.sp = block_span(g, c, b);
    w.r0 = (int)s64 * rps;
    w.active = w.sp.nc > 0 && w.r0 < w.sp.nr;
    w.nrow = w.active ? min(rps, w.sp.nr - w.r0) : 0;
    w.i0s = w.r0 * (int)g.block[1];
    w.cnt = w.nrow * (int)g.block[1];
    w.d = bd[w.t];
    w.fast = w.d.mode == BM_SHUFFLED && w.d.nstreams == ts;
    divmod(c, g.cgrid[1], cq, cr);
    divmod(b, g.bgrid[1], bq, br);
    w.jb = cr * g.bgrid[1] + br;
    return w;
}

// Plane j of a fast unit: its slice starts at src (nullptr for a run), 16-byte word a16 =
// src - shift; the bulk copy takes the whole words of [a16, a16 + want) before the buffer end
// lim, threads copy the bytes that the buffer end cuts off (zeros past it).
__device__ __forceinline__ StreamDesc gv_plane(const Geom &g, const uint8_t *ch, const uint8_t *ch_end,
                                               const StreamDesc *__restrict__ sd, const uint8_t *scratch,
                                               const uint8_t *scratch_end, const GvUnit &w, int j,
                                               const uint8_t *&src, const uint8_t *&lim, int &want, int &bulk)
{
    const StreamDesc q = sd[w.t * 8 + j];
    src = nullptr; lim = nullptr;
    if (q.kind == SK_RAW) { src = ch + q.src + w.i0s; lim = ch_end; }
    else if (q.kind == SK_LZ4) { src = scratch + w.t * g.blocksize + (int64_t)j * w.d.neblock + w.i0s; lim = scratch_end; }
    want = bulk = 0;
    if (src) {
        const uint8_t *a16 = src - (reinterpret_cast<uintptr_t>(src) & 15);
        want = ((int)(src - a16) + w.cnt + 15) & ~15;
        bulk = (int)min((int64_t)want, (lim - a16) & ~int64_t(15));
    }
    return q;
}

template <int TS, typename T>
__global__ void __launch_bounds__(256, 4) k_scatter_gemv(Geom g, const uint8_t *__restrict__ ch, const uint8_t *ch_end,
                                                      const BlockDesc *__restrict__ bd,
                                                      const StreamDesc *__restrict__ sd,
                                                      const uint8_t *__restrict__ scratch, const uint8_t *scratch_end,
                                                      const T *__restrict__ x, T *__restrict__ part, int64_t M,
                                                      int *err)
{
    __shared__ __align__(128) uint8_t stage[TS][SC_PLANE];
    __shared__ T qsum[SC_ITEMS / 4];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_all;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_barrier_init();
        abort_all = 0;
    }
    __syncthreads();
    const int qpr = (int)(g.block[1] / 4);
    const int rps = (int)(SC_ITEMS / g.block[1]);            // whole rows per slice (>= 1: checked by the host)
    const int64_t nsl = (g.block[0] + rps - 1) / rps;
    const int64_t total = g.nchunks * g.nblocks * nsl;
    uint32_t parity = 0;
    for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {          // block-uniform loop
        const GvUnit w = gv_unit(g, bd, u, nsl, rps, TS);
        if (!w.active) continue;                              // padding only
        const T *__restrict__ xb = x + w.sp.col0;
        if (w.fast) {
            if (tid == 0) {
                uint32_t tx = 0;
#pragma unroll
                for (int j = 0; j < TS; j++) {
                    const uint8_t *src, *lim;
                    int want, bulk;
                    gv_plane(g, ch, ch_end, sd, scratch, scratch_end, w, j, src, lim, want, bulk);
                    tx += (uint32_t)bulk;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of stage precede the copies
                tc::mbar_arrive_expect_tx(&bar, tx);
#pragma unroll
                for (int j = 0; j < TS; j++) {
                    const uint8_t *src, *lim;
                    int want, bulk;
                    gv_plane(g, ch, ch_end, sd, scratch, scratch_end, w, j, src, lim, want, bulk);
                    if (bulk > 0) bulk_g2s(stage[j], src - (reinterpret_cast<uintptr_t>(src) & 15), (uint32_t)bulk, &bar);
                }
            }
            int code[TS];
#pragma unroll
            for (int j = 0; j < TS; j++) {
                const uint8_t *src, *lim;
                int want, bulk;
                const StreamDesc q = gv_plane(g, ch, ch_end, sd, scratch, scratch_end, w, j, src, lim, want, bulk);
                code[j] = src ? (int)(reinterpret_cast<uintptr_t>(src) & 15) : 256 + (q.kind == SK_RUN ? (q.len & 255) : 0);
                if (bulk < want) {
                    const uint8_t *a16 = src - code[j];
                    for (int xx = bulk + tid; xx < want; xx += blockDim.x)
                        stage[j][xx] = a16 + xx < lim ? __ldg(a16 + xx) : (uint8_t)0;
                }
            }
            const bool ok = sc_wait(&bar, parity);
            parity ^= 1;
            if (!ok) abort_all = 1;
            __syncthreads();
            if (abort_all) {                                  // the copies did not complete: report, wait once more, leave
                if (tid == 0) {
                    dev_fail(err, DE_WAIT);
                    sc_wait(&bar, parity ^ 1);
                }
                return;
            }
            const int step_r = (int)blockDim.x / qpr, step_q = (int)blockDim.x - step_r * qpr;
            int q = tid - (tid / qpr) * qpr;
            for (int qd = tid; qd < w.cnt / 4; qd += blockDim.x, q += step_q) {
                if (q >= qpr) q -= qpr;
                const int cc = q * 4;
                T sum = 0;
                if (cc < w.sp.nc) {
                    uint32_t wd[TS];
#pragma unroll
                    for (int j = 0; j < TS; j++) {
                        if (code[j] >= 256) { wd[j] = (uint32_t)(code[j] - 256) * 0x01010101u; continue; }
                        const uint32_t *pw = reinterpret_cast<const uint32_t *>(stage[j]);
                        const int byte = code[j] + qd * 4, wi = byte >> 2, sh = (byte & 3) * 8;
                        wd[j] = sh ? __funnelshift_r(pw[wi], pw[wi + 1], sh) : pw[wi];
                    }
                    uint32_t v[4];
                    transpose4x4(wd[0], wd[1], wd[2], wd[3], v[0], v[1], v[2], v[3]);
                    uint64_t item[4];
                    if constexpr (TS == 8) {
                        uint32_t h[4];
                        transpose4x4(wd[4], wd[5], wd[6], wd[7], h[0], h[1], h[2], h[3]);
#pragma unroll
                        for (int k = 0; k < 4; k++) item[k] = ((uint64_t)h[k] << 32) | v[k];
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++) item[k] = v[k];
                    }
                    const T *xq = xb + cc;
                    if (cc + 4 <= w.sp.nc && (reinterpret_cast<uintptr_t>(xq) & 15) == 0) {
                        T xv[4];
                        if constexpr (TS == 8) {
                            const double2 x0 = __ldg(reinterpret_cast<const double2 *>(xq));
                            const double2 x1 = __ldg(reinterpret_cast<const double2 *>(xq) + 1);
                            xv[0] = x0.x; xv[1] = x0.y; xv[2] = x1.x; xv[3] = x1.y;
                        } else {
                            const float4 x0 = __ldg(reinterpret_cast<const float4 *>(xq));
                            xv[0] = x0.x; xv[1] = x0.y; xv[2] = x0.z; xv[3] = x0.w;
                        }
#pragma unroll
                        for (int k = 0; k < 4; k++) sum = fma(bits_as<T>(item[k]), xv[k], sum);
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            if (cc + k < w.sp.nc) sum = fma(bits_as<T>(item[k]), xq[k], sum);
                    }
                }
                qsum[qd] = sum;
            }
        } else {
            const StreamDesc *s = sd + w.t * 8;
            const uint8_t *bs = scratch + w.t * g.blocksize;
            for (int qd = tid; qd < w.cnt / 4; qd += blockDim.x) {
                const int cc = (qd % qpr) * 4;
                T sum = 0;
                for (int k = 0; k < 4; k++)
                    if (cc + k < w.sp.nc)
                        sum = fma(bits_as<T>(item_bits(g, ch, w.d, s, bs, w.i0s + qd * 4 + k)), xb[cc + k], sum);
                qsum[qd] = sum;
            }
        }
        __syncthreads();
        // row sums: warp w takes rows w, w + 8, ...; lanes stride the row's quads, then a shuffle tree
        for (int rr = warp; rr < w.nrow; rr += blockDim.x / 32) {
            T acc = 0;
            for (int q = lane; q < qpr; q += 32) acc += qsum[rr * qpr + q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULLMASK, acc, o);
            if (lane == 0) part[w.jb * M + w.sp.row0 + w.r0 + rr] = acc;
        }
        __syncthreads();                                  // stage and qsum are read before the next slice
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_gemv_rows(const T *__restrict__ part, int64_t JB, int64_t M, T *__restrict__ y)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
        T acc = 0;
        for (int64_t jb = 0; jb < JB; jb++) acc += part[jb * M + i];
        y[i] = acc;
    }
}

bool decode_gemv_fits(const Geom &g)
{
    return g.ndim == 2 && (g.itemsize == 4 || g.itemsize == 8) && !(g.block[1] & 3) && g.block[1] <= SC_ITEMS &&
           g.block[1] > 0;
}

int64_t decode_gemv_part_items(const Geom &g) { return g.cgrid[1] * g.bgrid[1] * g.shape[0]; }

int decode_gemv(const DecodeArgs &a, DecodeWork *w, const void *x, void *part, void *y, cudaStream_t st)
{
    const Geom &g = a.g;
    if (!decode_gemv_fits(g)) return -102;
    const int64_t M = g.shape[0], JB = g.cgrid[1] * g.bgrid[1], nbl = g.nchunks * g.nblocks;
    cudaMemsetAsync(part, 0, (size_t)(JB * M * g.itemsize), st);
    int *cnt = w->ext_counters ? w->ext_counters : w->counters.as<int>();
    const uint8_t *scratch = w->scratch.as<uint8_t>();
    const uint8_t *cend = a.chunks + a.chunks_bytes, *send = scratch + nbl * g.blocksize;
    const int rps = (int)(SC_ITEMS / g.block[1]);
    const int64_t units = nbl * ((g.block[0] + rps - 1) / rps);
    static int per_sm[2] = {0, 0};
    const int slot = g.itemsize == 8;
    if (!per_sm[slot]) {
        int m = 0;
        const cudaError_t e = slot ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_scatter_gemv<8, double>, 256, 0)
                                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_scatter_gemv<4, float>, 256, 0);
        if (e != cudaSuccess || m < 1) { cudaGetLastError(); m = 4; }
        per_sm[slot] = m;
    }
    const int64_t grid = std::max<int64_t>(std::min<int64_t>(units, (int64_t)sm_count() * per_sm[slot]), 1);
    const unsigned rb = (unsigned)std::max<int64_t>(std::min<int64_t>((M + 255) / 256, (int64_t)sm_count() * 8), 1);
    if (slot) {
        IAB_TIMED("k_scatter_gemv", st, k_scatter_gemv<8, double><<<(unsigned)grid, 256, 0, st>>>(
            g, a.chunks, cend, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), scratch, send, (const double *)x,
            (double *)part, M, cnt + 1));
        IAB_TIMED("k_gemv_rows", st, k_gemv_rows<double><<<rb, 256, 0, st>>>((const double *)part, JB, M, (double *)y));
    } else {
        IAB_TIMED("k_scatter_gemv", st, k_scatter_gemv<4, float><<<(unsigned)grid, 256, 0, st>>>(
            g, a.chunks, cend, w->bd.as<BlockDesc>(), w->sd.as<StreamDesc>(), scratch, send, (const float *)x,
            (float *)part, M, cnt + 1));
        IAB_TIMED("k_gemv_rows", st, k_gemv_rows<float><<<rb, 256, 0, st>>>((const float *)part, JB, M, (float *)y));
    }
    return 0;
}

// ============================================================================ grouped codec
// Largest k with start[k] <= u (containers with no units share their start with the next).
__device__ __forceinline__ int group_find(const int64_t *__restrict__ start, int n, int64_t u)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_group_reset(const CodecItem *__restrict__ items, int n)
{
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < (int64_t)n * 16) items[x >> 4].cnt[x & 15] = 0;
}

__global__ void k_parse_g(const CodecItem *__restrict__ items, const int64_t *__restrict__ bstart, int n, int64_t nbl,
                          Lz4Job *jobs, int *njobs, int64_t jcap)
{
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nbl; u += (int64_t)gridDim.x * blockDim.x) {
        const int k = group_find(bstart, n, u);
        const CodecItem &it = items[k];
        parse_block(it.g, it.ch, it.off, it.len, it.bd, it.sd, jobs, njobs, jcap, it.cnt + 1, it.scratch, nullptr,
                    nullptr, u - bstart[k]);
    }
}

template <int TS>
__global__ void __launch_bounds__(256, 4) k_scatter_fast_g(const CodecItem *__restrict__ items,
                                                        const int64_t *__restrict__ bstart,
                                                        const int64_t *__restrict__ sstart, int n, int64_t nsf,
                                                        int *rest, int *nrest)
{
    __shared__ __align__(128) uint8_t stage[TS][SC_PLANE];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_all;
    const int tid = threadIdx.x;
    if (tid == 0) {
        tc::mbar_init(&bar, 1);
        tc::fence_barrier_init();
        abort_all = 0;
    }
    __syncthreads();
    uint32_t parity = 0;
    for (int64_t u = blockIdx.x; u < nsf; u += gridDim.x) {
        const int k = group_find(sstart, n, u);
        const CodecItem &it = items[k];
        const int64_t nsl = (it.g.blockn + SC_ITEMS - 1) / SC_ITEMS;
        const int64_t lu = u - sstart[k], t = lu / nsl;
        const int sl = (int)(lu - t * nsl);
        const int64_t nbk = it.g.nchunks * it.g.nblocks;
        if (!scatter_fast_unit<TS>(it.g, it.ch, it.ch + it.ch_bytes, it.bd, it.sd, it.scratch,
                                   it.scratch + nbk * it.g.blocksize, it.dense, it.ld, rest, nrest,
                                   (int)(bstart[k] + t), it.cnt + 1, t, sl, stage, &bar, parity, &abort_all))
            return;
    }
}

// General scatter over the listed blocks (global block numbers), or every block without a list.
__global__ void __launch_bounds__(256) k_scatter_g(const CodecItem *__restrict__ items, const int64_t *__restrict__ bstart,
                                                   int n, const int *__restrict__ rest, const int *__restrict__ nrest,
                                                   int64_t nbl, int64_t tpb)
{
    __shared__ __align__(16) uint8_t planes[8 * TILE];
    const int64_t nwork = (rest ? (int64_t)*nrest : nbl) * tpb;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t kk = w / tpb, gb = rest ? rest[kk] : kk, i0 = (w - kk * tpb) * TILE;
        const int k = group_find(bstart, n, gb);
        const CodecItem &it = items[k];
        if (i0 >= it.g.blockn) continue;
        scatter_tile(it.g, it.ch, it.bd, it.sd, it.scratch, it.dense, it.ld, gb - bstart[k], i0, planes);
    }
}

template <int TS>
__global__ void __launch_bounds__(256) k_gather_fast_g(const CodecItem *__restrict__ items,
                                                       const int64_t *__restrict__ bstart, int n, int64_t nbl)
{
    for (int64_t u = blockIdx.x; u < nbl; u += gridDim.x) {
        const int k = group_find(bstart, n, u);
        const CodecItem &it = items[k];
        gather_fast_block<TS>(it.g, it.dense, it.ld, it.img, u - bstart[k]);
    }
}

__global__ void __launch_bounds__(256) k_gather_g(const CodecItem *__restrict__ items, const int64_t *__restrict__ bstart,
                                                  int n, int64_t nbl, int64_t tpb, bool skip_fast, bool shuffle)
{
    __shared__ __align__(16) uint8_t planes[8 * TILE];
    for (int64_t w = blockIdx.x; w < nbl * tpb; w += gridDim.x) {
        const int64_t gb = w / tpb, i0 = (w - gb * tpb) * TILE;
        const int k = group_find(bstart, n, gb);
        const CodecItem &it = items[k];
        if (i0 >= it.g.blockn) continue;
        if (skip_fast && geom_fast(it.g)) continue;
        gather_tile(it.g, it.dense, it.ld, shuffle, it.img, gb - bstart[k], i0, planes);
    }
}

__global__ void __launch_bounds__(LAYOUT_T) k_layout_g(const CodecItem *__restrict__ items,
                                                      const int64_t *__restrict__ cstart, int n, int nstreams,
                                                      int neblock, int memcpy_only)
{
    __shared__ int64_t wsum[LAYOUT_T / 32];
    __shared__ int64_t s_before;
    __shared__ int s_first;
    const int64_t u = blockIdx.x;
    const int k = group_find(cstart, n, u);
    const CodecItem &it = items[k];
    layout_chunk(it.g, nstreams, neblock, it.es, it.ec, memcpy_only, u - cstart[k], wsum, s_before, s_first);
}

__global__ void __launch_bounds__(1024) k_chunk_offsets_g(CodecItem *items)
{
    __shared__ int64_t wsum[32];
    CodecItem &it = items[blockIdx.x];
    chunk_offsets(it.g.nchunks, it.ec, &it.out_bytes, wsum);
}

__global__ void __launch_bounds__(256) k_emit_g(const CodecItem *__restrict__ items, const int64_t *__restrict__ bstart,
                                                int n, int64_t nbl, int nstreams, int neblock, bool shuffle, int splitflag)
{
    for (int64_t u = blockIdx.x; u < nbl; u += gridDim.x) {
        const int k = group_find(bstart, n, u);
        const CodecItem &it = items[k];
        const int64_t img_bytes = it.g.nchunks * it.g.nblocks * it.g.blocksize;
        emit_block(it.g, nstreams, neblock, shuffle, splitflag, it.img, it.slots, img_bytes, it.es, it.ec, it.outbuf,
                   u - bstart[k]);
    }
}

// Start tables (blocks, fast-scatter slices, chunks; n + 1 entries each) and the item table
// on the device.  Synchronises `st` (setup only, before any capture).
static int group_upload(CodecGroup *grp, cudaStream_t st)
{
    const int n = grp->n;
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<int64_t> s(3 * (size_t)(n + 1), 0);
    for (int k = 0; k < n; k++) {
        const Geom &g = grp->h[(size_t)k].g;
        const int64_t nbl = g.nchunks * g.nblocks;
        s[(size_t)k + 1] = s[(size_t)k] + nbl;
        s[(size_t)(n + 1) + k + 1] = s[(size_t)(n + 1) + k] + nbl * ((g.blockn + SC_ITEMS - 1) / SC_ITEMS);
        s[(size_t)(2 * (n + 1)) + k + 1] = s[(size_t)(2 * (n + 1)) + k] + g.nchunks;
    }
    grp->nbl = s[(size_t)n];
    grp->nsf = s[(size_t)(2 * n + 1)];
    grp->nch = s[(size_t)(3 * n + 2)];
    if (grp->nbl > INT32_MAX) return -102;
    if (!grp->items.allocate(sizeof(CodecItem) * (size_t)n, dev) || !grp->starts.allocate(sizeof(int64_t) * s.size(), dev))
        return -100;
    cudaMemcpyAsync(grp->items.p, grp->h.data(), sizeof(CodecItem) * (size_t)n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(grp->starts.p, s.data(), sizeof(int64_t) * s.size(), cudaMemcpyHostToDevice, st);
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : -101;
}

int decode_group_setup(const std::vector<DecodeArgs> &a, const std::vector<int *> &cnt, CodecGroup *grp, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int n = (int)a.size();
    if (n <= 0 || cnt.size() != a.size()) return -102;
    grp->n = n;
    grp->ts = a[0].g.itemsize;
    int64_t nbl = 0, img = 0, jobs = 0;
    grp->max_tpb = 1;
    for (const DecodeArgs &x : a) {
        if (x.g.itemsize != grp->ts) return 1;
        nbl += x.g.nchunks * x.g.nblocks;
        img += x.g.nchunks * x.g.nblocks * x.g.blocksize;
        jobs += decode_max_jobs(x.g);
        grp->max_tpb = std::max<int64_t>(grp->max_tpb, (x.g.blockn + TILE - 1) / TILE);
    }
    if (!grp->bd.allocate(sizeof(BlockDesc) * (size_t)std::max<int64_t>(nbl, 1), dev) ||
        !grp->sd.allocate(sizeof(StreamDesc) * 8 * (size_t)std::max<int64_t>(nbl, 1), dev) ||
        !grp->scratch.allocate((size_t)std::max<int64_t>(img, 16), dev) ||
        !grp->rest.allocate(sizeof(int) * (size_t)std::max<int64_t>(nbl, 1), dev) || !grp->counters.allocate(128, dev))
        return -100;
    int r = decode_queue_init(&grp->q, jobs, st);
    if (r) return r;
    grp->h.assign((size_t)n, CodecItem{});
    int64_t bo = 0, io = 0;
    for (int k = 0; k < n; k++) {
        const DecodeArgs &x = a[(size_t)k];
        CodecItem &it = grp->h[(size_t)k];
        it.g = x.g;
        it.ch = x.chunks; it.ch_bytes = x.chunks_bytes; it.off = x.off; it.len = x.len;
        it.bd = grp->bd.as<BlockDesc>() + bo;
        it.sd = grp->sd.as<StreamDesc>() + bo * 8;
        it.scratch = grp->scratch.as<uint8_t>() + io;
        it.dense = static_cast<uint8_t *>(x.out);
        it.ld = x.ld;
        it.cnt = cnt[(size_t)k];
        bo += x.g.nchunks * x.g.nblocks;
        io += x.g.nchunks * x.g.nblocks * x.g.blocksize;
    }
    return group_upload(grp, st);
}

int decode_group_launch(CodecGroup *grp, cudaStream_t st)
{
    const int n = grp->n, sms = sm_count();
    const CodecItem *items = grp->items.as<CodecItem>();
    const int64_t *bstart = grp->starts.as<int64_t>(), *sstart = bstart + (n + 1);
    int *gc = grp->counters.as<int>();
    cudaMemsetAsync(grp->q.counters.p, 0, 64, st);
    cudaMemsetAsync(gc, 0, 128, st);
    IAB_TIMED("k_group_reset", st, k_group_reset<<<(unsigned)((n * 16 + 255) / 256), 256, 0, st>>>(items, n));
    if (grp->nbl == 0) return 0;
    const int64_t pb = std::min<int64_t>((grp->nbl + 127) / 128, (int64_t)sms * 16);
    IAB_TIMED("k_parse", st, k_parse_g<<<(unsigned)pb, 128, 0, st>>>(items, bstart, n, grp->nbl, grp->q.jobs.as<Lz4Job>(),
                                                                     grp->q.counters.as<int>(), grp->q.cap));
    int r = decode_lz4(&grp->q, st);
    if (r) return r;
    const bool fast = grp->ts == 4 || grp->ts == 8;
    if (fast) {
        static int per_sm[2] = {0, 0};
        const int slot = grp->ts == 8;
        if (!per_sm[slot]) {
            int m = 0;
            const cudaError_t e = slot ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_scatter_fast_g<8>, 256, 0)
                                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_scatter_fast_g<4>, 256, 0);
            if (e != cudaSuccess || m < 1) { cudaGetLastError(); m = 4; }
            per_sm[slot] = m;
        }
        const int64_t grid = std::max<int64_t>(std::min<int64_t>(grp->nsf, (int64_t)sms * per_sm[slot]), 1);
        if (slot)
            IAB_TIMED("k_scatter_fast", st, k_scatter_fast_g<8><<<(unsigned)grid, 256, 0, st>>>(
                items, bstart, sstart, n, grp->nsf, grp->rest.as<int>(), gc));
        else
            IAB_TIMED("k_scatter_fast", st, k_scatter_fast_g<4><<<(unsigned)grid, 256, 0, st>>>(
                items, bstart, sstart, n, grp->nsf, grp->rest.as<int>(), gc));
    }
    const int64_t sb = std::min<int64_t>(grp->nbl * grp->max_tpb, (int64_t)sms * 8);
    IAB_TIMED("k_scatter", st, k_scatter_g<<<(unsigned)std::max<int64_t>(sb, 1), 256, 0, st>>>(
        items, bstart, n, fast ? grp->rest.as<int>() : nullptr, fast ? gc : nullptr, grp->nbl, grp->max_tpb));
    return 0;
}

int encode_group_setup(const std::vector<Geom> &g, const std::vector<const void *> &dense, const std::vector<int64_t> &ld,
                       const std::vector<EncChunk *> &ec, std::vector<DevBuf> *out, CodecGroup *grp, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int n = (int)g.size();
    if (n <= 0 || dense.size() != g.size() || ld.size() != g.size() || ec.size() != g.size() || out->size() != g.size())
        return -102;
    grp->n = n;
    grp->ts = g[0].itemsize;
    grp->shuffle = true;
    grp->nstreams = encode_nstreams(g[0], true, 3 /* automatic split */);
    grp->split = encode_split(g[0], true, 3);
    grp->neblock = (int)(g[0].blocksize / grp->nstreams);
    grp->max_tpb = 1;
    int64_t img = 0, ns = 0;
    for (const Geom &x : g) {
        const int nsx = encode_nstreams(x, true, 3);
        if (x.itemsize != grp->ts || nsx != grp->nstreams || x.blocksize / nsx != grp->neblock ||
            encode_split(x, true, 3) != grp->split)
            return 1;
        img += x.nchunks * x.nblocks * x.blocksize;
        ns += x.nchunks * x.nblocks * nsx;
        grp->max_tpb = std::max<int64_t>(grp->max_tpb, (x.blockn + TILE - 1) / TILE);
    }
    if (!grp->img.allocate((size_t)std::max<int64_t>(img, 16), dev) || !grp->slots.allocate((size_t)std::max<int64_t>(img, 16), dev) ||
        !grp->es.allocate(sizeof(EncStream) * (size_t)std::max<int64_t>(ns, 1), dev) || !grp->counters.allocate(128, dev))
        return -100;
    grp->h.assign((size_t)n, CodecItem{});
    int64_t io = 0, so = 0;
    for (int k = 0; k < n; k++) {
        const Geom &x = g[(size_t)k];
        if (!(*out)[(size_t)k].allocate((size_t)std::max<int64_t>(x.nchunks * (x.chunk_nbytes + 32), 16), dev)) return -100;
        CodecItem &it = grp->h[(size_t)k];
        it.g = x;
        it.dense = const_cast<uint8_t *>(static_cast<const uint8_t *>(dense[(size_t)k]));
        it.ld = ld[(size_t)k];
        it.img = grp->img.as<uint8_t>() + io;
        it.slots = grp->slots.as<uint8_t>() + io;
        it.es = grp->es.as<EncStream>() + so;
        it.ec = ec[(size_t)k];
        it.outbuf = (*out)[(size_t)k].as<uint8_t>();
        io += x.nchunks * x.nblocks * x.blocksize;
        so += x.nchunks * x.nblocks * grp->nstreams;
    }
    return group_upload(grp, st);
}

int encode_group_launch(CodecGroup *grp, bool exact_lz4, bool memcpy_only, cudaStream_t st)
{
    const int n = grp->n, sms = sm_count(), ts = grp->ts;
    CodecItem *items = grp->items.as<CodecItem>();
    const int64_t *bstart = grp->starts.as<int64_t>(), *cstart = bstart + 2 * (n + 1);
    if (grp->nbl == 0) return 0;
    cudaMemsetAsync(grp->counters.p, 0, 128, st);
    const bool fast = grp->shuffle && (ts == 4 || ts == 8);
    bool all_fast = fast;
    for (const CodecItem &it : grp->h) {
        const Geom &g = it.g;
        all_fast = all_fast && !(g.block[1] & 3);
    }
    const int64_t gb = std::max<int64_t>(std::min<int64_t>(grp->nbl, (int64_t)sms * 8), 1);
    if (fast && !grp->img_ready) {
        if (ts == 8)
            IAB_TIMED("k_gather_fast", st, k_gather_fast_g<8><<<(unsigned)gb, 256, 0, st>>>(items, bstart, n, grp->nbl));
        else
            IAB_TIMED("k_gather_fast", st, k_gather_fast_g<4><<<(unsigned)gb, 256, 0, st>>>(items, bstart, n, grp->nbl));
    }
    if (!all_fast && !grp->img_ready) {
        const int64_t tb = std::max<int64_t>(std::min<int64_t>(grp->nbl * grp->max_tpb, (int64_t)sms * 8), 1);
        IAB_TIMED("k_gather", st, k_gather_g<<<(unsigned)tb, 256, 0, st>>>(items, bstart, n, grp->nbl, grp->max_tpb, fast,
                                                                           grp->shuffle));
    }
    if (!memcpy_only)
        encode_streams(grp->img.as<uint8_t>(), grp->nbl * grp->nstreams, grp->neblock, grp->slots.as<uint8_t>(),
                       grp->es.as<EncStream>(), reinterpret_cast<unsigned long long *>(grp->counters.as<uint8_t>() + 64),
                       exact_lz4, st);
    IAB_TIMED("k_layout", st, k_layout_g<<<(unsigned)std::max<int64_t>(grp->nch, 1), LAYOUT_T, 0, st>>>(
        items, cstart, n, grp->nstreams, grp->neblock, memcpy_only ? 1 : 0));
    IAB_TIMED("k_chunk_offsets", st, k_chunk_offsets_g<<<(unsigned)n, 1024, 0, st>>>(items));
    IAB_TIMED("k_emit", st, k_emit_g<<<(unsigned)gb, 256, 0, st>>>(items, bstart, n, grp->nbl, grp->nstreams, grp->neblock,
                                                                   grp->shuffle, grp->split ? 1 : 0));
    return 0;
}

// ============================================================================ decode without allocation
// For callers that cannot call cudaMalloc: engines whose device memory belongs to their own
// arena or memory-budget manager and that hand the library only buffers they already hold,
// and latency-bound loops that must not pay the device synchronisation of cudaMalloc and
// cudaFree.  decode_noalloc runs the same kernels as decode_launch, but its work buffers (chunk
// index, block and stream descriptors, LZ4 jobs, the decoded-stream image and the
// status counters) live in one file-scope device array instead of pool allocations.
// The array is part of the library's device image: every GPU on which the library's
// kernels are loaded holds it until the process exits, and every call shares it, so
// calls whose kernels overlap on the GPU (two streams, two host threads) race on it.
constexpr int64_t NA_MAX_BLOCKS = NOALLOC_MAX_BLOCKS;
constexpr size_t na_align(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t NA_COUNTERS = 0;
constexpr size_t NA_OFF = 256;
constexpr size_t NA_LEN = na_align(NA_OFF + sizeof(int64_t) * NA_MAX_BLOCKS);
constexpr size_t NA_BD = na_align(NA_LEN + sizeof(int32_t) * NA_MAX_BLOCKS);
constexpr size_t NA_SD = na_align(NA_BD + sizeof(BlockDesc) * NA_MAX_BLOCKS);
constexpr size_t NA_JOBS = na_align(NA_SD + sizeof(StreamDesc) * 8 * NA_MAX_BLOCKS);
constexpr size_t NA_REST = na_align(NA_JOBS + sizeof(Lz4Job) * 8 * NA_MAX_BLOCKS);
constexpr size_t NA_IMG = na_align(NA_REST + sizeof(int) * NA_MAX_BLOCKS);
constexpr size_t NA_TOTAL = NA_IMG + (size_t)NOALLOC_MAX_BYTES;

static __device__ __align__(256) uint8_t g_noalloc_scratch[NA_TOTAL];

// Chunk index of back-to-back chunks: one thread walks the headers (cbytes at byte 12).
// A header that does not fit the buffer yields length 0, which the parse kernel reports
// as a header error.
__global__ void k_chunk_walk(const uint8_t *__restrict__ ch, int64_t bytes, int64_t n, int64_t *off, int32_t *len)
{
    if (blockIdx.x || threadIdx.x) return;
    int64_t pos = 0;
    for (int64_t c = 0; c < n; c++) {
        int32_t cb = 0;
        if (pos + 32 <= bytes) {
            cb = ld_s32(ch + pos + 12);
            if (cb < 32 || (int64_t)cb > bytes - pos) cb = 0;
        }
        off[c] = pos;
        len[c] = cb;
        pos = cb ? pos + cb : bytes;
    }
}

// Device address of g_noalloc_scratch on the current device.  The first call on a device
// looks the address up (the symbol's host name is only a stand-in, not a device address)
// and sets the decoder's shared-memory attribute; later calls reuse the cached address.
static uint8_t *noalloc_scratch()
{
    constexpr int MAXDEV = 64;
    static std::mutex mu;
    static uint8_t *ptr[MAXDEV] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAXDEV) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) { cudaGetLastError(); return nullptr; }
        if (cudaFuncSetAttribute(k_lz4_decode_cta, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(dcta::Smem)) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        ptr[dev] = static_cast<uint8_t *>(p);
    }
    return ptr[dev];
}

int decode_noalloc(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, void *out, int64_t ld, cudaStream_t st)
{
    if (!noalloc_fits(g)) return -102;
    const int64_t nbl = g.nchunks * g.nblocks;
    if (nbl == 0) return 0;
    uint8_t *base = noalloc_scratch();
    if (!base) return -101;
    int *counters = reinterpret_cast<int *>(base + NA_COUNTERS);
    int64_t *off = reinterpret_cast<int64_t *>(base + NA_OFF);
    int32_t *len = reinterpret_cast<int32_t *>(base + NA_LEN);
    BlockDesc *bd = reinterpret_cast<BlockDesc *>(base + NA_BD);
    StreamDesc *sd = reinterpret_cast<StreamDesc *>(base + NA_SD);
    Lz4Job *jobs = reinterpret_cast<Lz4Job *>(base + NA_JOBS);
    uint8_t *img = base + NA_IMG;
    int *njobs = counters, *err = counters + 1;
    // the job count, the status word and the job cursor must start at zero; descriptors,
    // the chunk index and the image are fully rewritten before they are read
    if (cudaMemsetAsync(counters, 0, 64, st) != cudaSuccess) return -101;
    const int sms = sm_count();
    IAB_TIMED("k_chunk_walk", st, k_chunk_walk<<<1, 32, 0, st>>>(d_chunks, chunks_bytes, g.nchunks, off, len));
    {
        const int threads = 128;
        const int64_t blocks = std::min<int64_t>((nbl + threads - 1) / threads, (int64_t)sms * 16);
        IAB_TIMED("k_parse", st, k_parse<<<(unsigned)std::max<int64_t>(blocks, 1), threads, 0, st>>>(g, d_chunks, off, len, bd, sd, jobs, njobs,
                                                                                      8 * NA_MAX_BLOCKS, err, img,
                                                                                      nullptr, nullptr));
    }
    {
        IAB_TIMED("k_lz4_decode_cta", st, k_lz4_decode_cta<<<sms * 6, dcta::THREADS, (int)sizeof(dcta::Smem), st>>>(
            jobs, njobs, 8 * NA_MAX_BLOCKS, reinterpret_cast<unsigned *>(counters + 2)));
    }
    {
        const int64_t tpb = (g.blockn + TILE - 1) / TILE;
        const int64_t blocks = std::min<int64_t>(nbl * tpb, (int64_t)sms * 8);
        const bool fast = g.itemsize == 4 || g.itemsize == 8;
        int *rest = fast ? reinterpret_cast<int *>(base + NA_REST) : nullptr, *nrest = counters + 3;
        if (fast) {
            const uint8_t *cend = d_chunks + chunks_bytes, *send = img + nbl * g.blocksize;
            if (g.itemsize == 8)
                IAB_TIMED("k_scatter_fast", st, k_scatter_fast<8><<<(unsigned)scatter_fast_grid<8>(g, nbl), 256, 0, st>>>(
                    g, d_chunks, cend, bd, sd, img, send, (uint8_t *)out, ld, rest, nrest, err));
            else
                IAB_TIMED("k_scatter_fast", st, k_scatter_fast<4><<<(unsigned)scatter_fast_grid<4>(g, nbl), 256, 0, st>>>(
                    g, d_chunks, cend, bd, sd, img, send, (uint8_t *)out, ld, rest, nrest, err));
        }
        IAB_TIMED("k_scatter", st, k_scatter<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, st>>>(
            g, rest, nrest, d_chunks, bd, sd, img, (uint8_t *)out, ld));
    }
    // a launch that failed (a bad configuration, or an error left by earlier work) never
    // wrote the status word: report it instead of the zero it still holds
    if (cudaPeekAtLastError() != cudaSuccess) return -101;
    int h_err = 0;
    if (cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -101;
    if (cudaStreamSynchronize(st) != cudaSuccess) return -101;
    return h_err;
}

}  // namespace iab
