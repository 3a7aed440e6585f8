/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C CPU restatement of the pieces of ironArray's blocked matmul path that
 * the GPU library replaces, used by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg as the checker.  The product (libiarray_b200.so) never links,
 * loads or calls this file.
 *
 * What it restates:
 *   - LZ4 block format decoder and the liblz4 1.9.4 LZ4_compress_fast(acceleration=1)
 *     greedy encoder in "limited output" mode.  c-blosc2 (the reference's codec,
 *     an un-vendored submodule `contribs/caterva/contribs/c-blosc2`, version not
 *     pinned in the checkout) bundles liblz4 and always calls it with acceleration 1.
 *     Parity pin: the reference's golden frames (tests/data/*.iarray: every LZ4 stream
 *     re-encodes byte-identically) and liblz4.so.1 itself (random + structured inputs).
 *   - Blosc2 chunk format v5 with the 32-byte extended header, SHUFFLE filter,
 *     split streams, zero / run / raw / LZ4 stream kinds, memcpyed chunks and the
 *     special-value chunks (zeros, NaN, uninit).  Layout pinned on the golden frames.
 *   - Caterva's blocked, zero-padded chunk layout (chunk = extchunkshape, blocks
 *     row-major inside the chunk, items row-major inside a block).
 *   - ironArray's zero-skip predicates chunk_is_zeros / block_is_zeros
 *     (src/linalg/iarray_gemm.c:17-77).
 *   - The loop orders of iarray_opt_gemm (src/linalg/iarray_gemm.c:91-312),
 *     iarray_opt_gemm_a/_b (src/linalg/iarray_gemm_a.c:87-188, iarray_gemm_b.c),
 *     iarray_opt_gemv (src/linalg/iarray_gemv.c:88-246), the panel GEMM
 *     (src/linalg/matmul/gemm.c:71-249) and panel GEMV (src/linalg/matmul/gemv.c:71-190),
 *     with the block products done as plain k-ascending loops (the reference calls MKL
 *     there; MKL's internal order is not observable).
 *   - A double-double (TwoProd via fma + TwoSum) reference for sampled rows of A*B,
 *     used to measure normwise error.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* little-endian helpers                                                      */
/* ------------------------------------------------------------------------- */
static inline uint32_t rd32(const uint8_t *p) { uint32_t v; memcpy(&v, p, 4); return v; }
static inline uint64_t rd64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
static inline int32_t rds32(const uint8_t *p) { int32_t v; memcpy(&v, p, 4); return v; }
static inline void wr32(uint8_t *p, int32_t v) { memcpy(p, &v, 4); }

/* ------------------------------------------------------------------------- */
/* LZ4 block format                                                          */
/* ------------------------------------------------------------------------- */
/* Sequence = token (hi nibble literal length, lo nibble match length - 4),
 * optional length extension bytes (255 = continue), literals, 2-byte LE offset,
 * optional match length extension bytes.  The last sequence has literals only. */

/* Returns the number of decoded bytes (== dst_len on success) or a negative error.
 * Every read and write is bounds-checked; a malformed stream never overruns. */
EXPORT int ora_lz4_decompress(const uint8_t *src, int src_len, uint8_t *dst, int dst_len)
{
    const uint8_t *ip = src, *iend = src + src_len;
    uint8_t *op = dst, *oend = dst + dst_len;
    if (src_len <= 0) return -1;
    for (;;) {
        if (ip >= iend) return -2;
        unsigned token = *ip++;
        size_t lit = token >> 4;
        if (lit == 15) {
            unsigned s;
            do { if (ip >= iend) return -3; s = *ip++; lit += s; } while (s == 255);
        }
        if ((size_t)(iend - ip) < lit || (size_t)(oend - op) < lit) return -4;
        memcpy(op, ip, lit); ip += lit; op += lit;
        if (ip == iend) break;                     /* last sequence: literals only */
        if (iend - ip < 2) return -5;
        size_t off = (size_t)ip[0] | ((size_t)ip[1] << 8); ip += 2;
        if (off == 0 || off > (size_t)(op - dst)) return -6;
        size_t ml = token & 15;
        if (ml == 15) {
            unsigned s;
            do { if (ip >= iend) return -7; s = *ip++; ml += s; } while (s == 255);
        }
        ml += 4;
        if ((size_t)(oend - op) < ml) return -8;
        const uint8_t *m = op - off;
        for (size_t i = 0; i < ml; i++) op[i] = m[i];   /* byte-wise: overlap allowed */
        op += ml;
    }
    return (int)(op - dst);
}

/* Encoder restating liblz4 1.9.4's single-segment greedy compressor as called by
 * LZ4_compress_fast(src, dst, n, cap, 1) when cap < LZ4_compressBound(n):
 * "limited output" mode, which gives up (returns 0) as soon as a conservative
 * size check says the output may not fit in `cap` bytes.
 *   table: 2^13 16-bit positions hashed from 4 bytes when n < 65547,
 *          else 2^12 32-bit positions hashed from 5 bytes (64-bit build);
 *   search: step starts at 1 and grows by one every 64 failed probes;
 *   a match needs 4 equal bytes, distance <= 65535, and is extended backwards;
 *   the last 5 bytes are always literals and no match starts in the last 12. */
#define LZ4_MINMATCH 4
#define LZ4_MFLIMIT 12
#define LZ4_LASTLITERALS 5
#define LZ4_MIN_LENGTH (LZ4_MFLIMIT + 1)
#define LZ4_SMALL_LIMIT (65536 + LZ4_MFLIMIT - 1)
#define LZ4_MAX_DISTANCE 65535

static inline uint32_t lz4_hash(const uint8_t *p, int small)
{
    if (small) return (rd32(p) * 2654435761u) >> (32 - 13);
    return (uint32_t)(((rd64(p) << 24) * 889523592379ull) >> (64 - 12));
}

static inline unsigned lz4_count(const uint8_t *a, const uint8_t *b, const uint8_t *alimit)
{
    const uint8_t *s = a;
    while (a < alimit && *a == *b) { a++; b++; }
    return (unsigned)(a - s);
}

EXPORT int ora_lz4_compress_limited(const uint8_t *src, int n, uint8_t *dst, int cap)
{
    if (n < 0 || n > 0x7E000000) return 0;
    if (n == 0) { if (cap <= 0) return 0; dst[0] = 0; return 1; }
    const int small = n < LZ4_SMALL_LIMIT;
    uint32_t table[8192];
    memset(table, 0, sizeof(table));
    const uint8_t *ip = src, *anchor = src, *iend = src + n;
    const uint8_t *mflimit_plus1 = iend - LZ4_MFLIMIT + 1;
    const uint8_t *matchlimit = iend - LZ4_LASTLITERALS;
    uint8_t *op = dst, *olimit = dst + cap;
    uint32_t fwd_h;
    const uint8_t *match;
    uint8_t *token;

    if (n < LZ4_MIN_LENGTH) goto last_literals;
    table[lz4_hash(ip, small)] = 0;
    ip++;
    fwd_h = lz4_hash(ip, small);

    for (;;) {
        {   /* find a match */
            const uint8_t *fwd_ip = ip;
            int step = 1, probes = 1 << 6;
            for (;;) {
                uint32_t h = fwd_h;
                uint32_t cur = (uint32_t)(fwd_ip - src);
                uint32_t midx = table[h];
                ip = fwd_ip;
                fwd_ip += step;
                step = probes++ >> 6;
                if (fwd_ip > mflimit_plus1) goto last_literals;
                match = src + midx;
                fwd_h = lz4_hash(fwd_ip, small);
                table[h] = small ? (cur & 0xFFFFu) : cur;
                if (!small && midx + LZ4_MAX_DISTANCE < cur) continue;
                if (rd32(match) == rd32(ip)) break;
            }
        }
        /* extend backwards */
        while (ip > anchor && match > src && ip[-1] == match[-1]) { ip--; match--; }
        {   /* literals */
            unsigned lit = (unsigned)(ip - anchor);
            token = op++;
            if (op + lit + (2 + 1 + LZ4_LASTLITERALS) + (lit / 255) > olimit) return 0;
            if (lit >= 15) {
                unsigned len = lit - 15;
                *token = 15 << 4;
                for (; len >= 255; len -= 255) *op++ = 255;
                *op++ = (uint8_t)len;
            } else {
                *token = (uint8_t)(lit << 4);
            }
            memcpy(op, anchor, lit);
            op += lit;
        }
next_match:
        {   /* offset + match length */
            uint16_t off = (uint16_t)(ip - match);
            op[0] = (uint8_t)off; op[1] = (uint8_t)(off >> 8); op += 2;
            unsigned mc = lz4_count(ip + LZ4_MINMATCH, match + LZ4_MINMATCH, matchlimit);
            ip += mc + LZ4_MINMATCH;
            if (op + (1 + LZ4_LASTLITERALS) + (mc + 240) / 255 > olimit) return 0;
            if (mc >= 15) {
                *token += 15;
                mc -= 15;
                for (; mc >= 255; mc -= 255) *op++ = 255;
                *op++ = (uint8_t)mc;
            } else {
                *token += (uint8_t)mc;
            }
        }
        anchor = ip;
        if (ip >= mflimit_plus1) break;
        table[lz4_hash(ip - 2, small)] = (uint32_t)(ip - 2 - src);
        {   /* immediate re-match at ip */
            uint32_t h = lz4_hash(ip, small);
            uint32_t cur = (uint32_t)(ip - src);
            uint32_t midx = table[h];
            match = src + midx;
            table[h] = cur;
            if ((small || midx + LZ4_MAX_DISTANCE >= cur) && rd32(match) == rd32(ip)) {
                token = op++;
                *token = 0;
                goto next_match;
            }
        }
        fwd_h = lz4_hash(++ip, small);
    }

last_literals:
    {
        size_t last = (size_t)(iend - anchor);
        if (op + last + 1 + ((last + 255 - 15) / 255) > olimit) return 0;
        if (last >= 15) {
            size_t acc = last - 15;
            *op++ = 15 << 4;
            for (; acc >= 255; acc -= 255) *op++ = 255;
            *op++ = (uint8_t)acc;
        } else {
            *op++ = (uint8_t)(last << 4);
        }
        memcpy(op, anchor, last);
        op += last;
    }
    return (int)(op - dst);
}

/* ------------------------------------------------------------------------- */
/* Byte shuffle                                                               */
/* ------------------------------------------------------------------------- */
/* shuffled[j*nitems + i] = src[i*ts + j]; bytes past nitems*ts are copied as-is. */
EXPORT void ora_shuffle(int ts, int nbytes, const uint8_t *src, uint8_t *dst)
{
    int nitems = nbytes / ts;
    for (int j = 0; j < ts; j++)
        for (int i = 0; i < nitems; i++) dst[j * nitems + i] = src[i * ts + j];
    memcpy(dst + nitems * ts, src + nitems * ts, nbytes - nitems * ts);
}

EXPORT void ora_unshuffle(int ts, int nbytes, const uint8_t *src, uint8_t *dst)
{
    int nitems = nbytes / ts;
    for (int j = 0; j < ts; j++)
        for (int i = 0; i < nitems; i++) dst[i * ts + j] = src[j * nitems + i];
    memcpy(dst + nitems * ts, src + nitems * ts, nbytes - nitems * ts);
}

/* ------------------------------------------------------------------------- */
/* Blosc2 chunk (format version 5, 32-byte extended header)                  */
/* ------------------------------------------------------------------------- */
/* header:  [0] version=5  [1] codec format version=1  [2] flags  [3] typesize
 *          [4..7] nbytes  [8..11] blocksize  [12..15] cbytes
 *          [16..21] filters[6] (SHUFFLE=1 in slot 5)  [22] compcode  [23] compcode meta
 *          [24..29] filters meta  [30] reserved  [31] blosc2 flags
 * flags:   bit0|bit2 = extended header, bit1 = memcpyed, bit4 = streams not split,
 *          bits5-7 = codec (1 = LZ4).
 * blosc2 flags: bits4-6 special value (1 zeros, 2 NaN, 3 value, 4 uninit), bit3 lazy.
 * body:    int32 bstarts[nblocks] (any order), then per block `nstreams` x
 *          (int32 csize, payload): csize 0 = run of 0x00, csize < 0 = run of byte
 *          (-csize) followed by a 1-byte token (bit0 set), csize == stream length = raw,
 *          otherwise an LZ4 block. */
#define HDR 32
enum { SPLIT_ALWAYS = 1, SPLIT_NEVER = 2, SPLIT_AUTO = 3, SPLIT_FORWARD_COMPAT = 4 };
enum { CODEC_BLOSCLZ = 0, CODEC_LZ4 = 1 };

EXPORT int ora_split_decision(int splitmode, int compcode, int shuffle, int typesize, int blocksize)
{
    if (splitmode == SPLIT_ALWAYS) return 1;
    if (splitmode == SPLIT_NEVER) return 0;
    return (compcode == CODEC_BLOSCLZ || compcode == CODEC_LZ4) && shuffle &&
           typesize <= 16 && (blocksize / typesize) >= 32;
}

static int all_same(const uint8_t *p, int n)
{
    for (int i = 1; i < n; i++) if (p[i] != p[0]) return 0;
    return 1;
}

static void write_header(uint8_t *d, int flags, int typesize, int nbytes, int blocksize, int cbytes,
                         int shuffle, int compcode)
{
    memset(d, 0, HDR);
    d[0] = 5; d[1] = 1; d[2] = (uint8_t)flags; d[3] = (uint8_t)typesize;
    wr32(d + 4, nbytes); wr32(d + 8, blocksize); wr32(d + 12, cbytes);
    d[16 + 5] = shuffle ? 1 : 0;
    d[22] = (uint8_t)compcode;
}

/* Compress one chunk of `nbytes` (typesize, blocksize as stored in the header) with
 * LZ4 + optional SHUFFLE.  `dst` must hold nbytes + 32 bytes; `destsize` is the
 * caller's capacity (Blosc2's callers pass nbytes + BLOSC2_MAX_OVERHEAD = nbytes + 32).
 * Blocks are written in order 0..nblocks-1.  Returns cbytes or < 0 on error. */
EXPORT int ora_chunk_compress(const uint8_t *src, int nbytes, int typesize, int blocksize,
                              int shuffle, int splitmode, uint8_t *dst, int destsize)
{
    if (typesize < 1 || typesize > 255 || blocksize <= 0 || nbytes < 0) return -1;
    if (blocksize > nbytes) blocksize = nbytes;
    const int compcode = CODEC_LZ4;
    int nblocks = nbytes == 0 ? 0 : (nbytes + blocksize - 1) / blocksize;
    int leftover = nbytes % (blocksize ? blocksize : 1);
    int split = ora_split_decision(splitmode, compcode, shuffle, typesize, blocksize);
    int flags = 0x05 | (compcode << 5) | (split ? 0 : 0x10);
    uint8_t *tmp = (uint8_t *)malloc(blocksize ? blocksize : 1);
    int32_t ntbytes = HDR + 4 * nblocks;
    int ok = ntbytes <= destsize;
    for (int b = 0; ok && b < nblocks; b++) {
        int bsize = (b == nblocks - 1 && leftover) ? leftover : blocksize;
        const uint8_t *blk = src + (size_t)b * blocksize;
        const uint8_t *s = blk;
        if (shuffle && typesize > 1) { ora_shuffle(typesize, bsize, blk, tmp); s = tmp; }
        wr32(dst + HDR + 4 * b, ntbytes);
        int nstreams = (split && !(b == nblocks - 1 && leftover)) ? typesize : 1;
        int neblock = bsize / nstreams;
        for (int j = 0; j < nstreams; j++) {
            const uint8_t *ip = s + j * neblock;
            uint8_t *csz = dst + ntbytes;
            ntbytes += 4;
            if (ntbytes > destsize) { ok = 0; break; }
            if (all_same(ip, neblock)) {
                int v = ip[0];
                wr32(csz, -v);
                if (v != 0) {                       /* non-zero runs carry a token byte */
                    if (ntbytes + 1 > destsize) { ok = 0; break; }
                    dst[ntbytes++] = 0x01;
                }
                continue;
            }
            int maxout = neblock;
            if (ntbytes + maxout > destsize) {
                maxout = destsize - ntbytes;
                if (maxout <= 0) { ok = 0; break; }
            }
            int cb = ora_lz4_compress_limited(ip, neblock, dst + ntbytes, maxout);
            if (cb == 0 || cb >= neblock) {
                if (ntbytes + neblock > destsize) { ok = 0; break; }
                memcpy(dst + ntbytes, ip, neblock);
                cb = neblock;
            }
            wr32(csz, cb);
            ntbytes += cb;
        }
    }
    free(tmp);
    if (!ok) {                                     /* fall back to a memcpyed chunk */
        if (nbytes + HDR > destsize) return -2;
        write_header(dst, flags | 0x02, typesize, nbytes, blocksize, nbytes + HDR, shuffle, compcode);
        memcpy(dst + HDR, src, nbytes);
        return nbytes + HDR;
    }
    write_header(dst, flags, typesize, nbytes, blocksize, ntbytes, shuffle, compcode);
    return ntbytes;
}

/* Decode a whole chunk into dst (dst_len >= nbytes).  Returns nbytes or < 0. */
EXPORT int ora_chunk_decompress(const uint8_t *chunk, int chunk_len, uint8_t *dst, int dst_len)
{
    if (chunk_len < HDR) return -1;
    int flags = chunk[2], typesize = chunk[3];
    int nbytes = rds32(chunk + 4), blocksize = rds32(chunk + 8), cbytes = rds32(chunk + 12);
    int bflags = chunk[31];
    if (chunk[0] < 2 || (flags & 0x05) != 0x05) return -2;      /* extended header only */
    if (nbytes < 0 || cbytes > chunk_len || cbytes < HDR || dst_len < nbytes) return -3;
    int special = (bflags >> 4) & 7;
    if (special) {
        if (special == 1 || special == 4) { memset(dst, 0, nbytes); return nbytes; }
        if (special == 2) {
            if (typesize == 8) { double v = NAN; for (int i = 0; i < nbytes / 8; i++) memcpy(dst + 8 * i, &v, 8); }
            else if (typesize == 4) { float v = NAN; for (int i = 0; i < nbytes / 4; i++) memcpy(dst + 4 * i, &v, 4); }
            else return -4;
            return nbytes;
        }
        if (special == 3) {                               /* value repeated, stored after header */
            if (cbytes < HDR + typesize) return -4;
            for (int i = 0; i < nbytes / typesize; i++) memcpy(dst + (size_t)i * typesize, chunk + HDR, typesize);
            return nbytes;
        }
        return -4;
    }
    if (flags & 0x02) {                                           /* memcpyed */
        if (cbytes < HDR + nbytes) return -5;
        memcpy(dst, chunk + HDR, nbytes);
        return nbytes;
    }
    if (blocksize <= 0) return -6;
    int nblocks = (nbytes + blocksize - 1) / blocksize;
    int leftover = nbytes % blocksize;
    int split = !(flags & 0x10);
    int shuffle = chunk[16 + 5] == 1;
    if (HDR + 4 * nblocks > cbytes) return -7;
    uint8_t *tmp = (uint8_t *)malloc(blocksize);
    for (int b = 0; b < nblocks; b++) {
        int bsize = (b == nblocks - 1 && leftover) ? leftover : blocksize;
        int32_t bstart = rds32(chunk + HDR + 4 * b);
        if (bstart < HDR + 4 * nblocks || bstart > cbytes) { free(tmp); return -8; }
        int nstreams = (split && !(b == nblocks - 1 && leftover)) ? typesize : 1;
        int neblock = bsize / nstreams;
        uint8_t *out = (shuffle && typesize > 1) ? tmp : dst + (size_t)b * blocksize;
        const uint8_t *p = chunk + bstart, *pend = chunk + cbytes;
        for (int j = 0; j < nstreams; j++) {
            if (pend - p < 4) { free(tmp); return -9; }
            int32_t cs = rds32(p); p += 4;
            uint8_t *o = out + j * neblock;
            if (cs == 0) { memset(o, 0, neblock); continue; }
            if (cs < 0) {
                if (pend - p < 1 || !(p[0] & 1) || cs < -255) { free(tmp); return -10; }
                p += 1;
                memset(o, -cs, neblock);
                continue;
            }
            if (cs > pend - p) { free(tmp); return -11; }
            if (cs == neblock) memcpy(o, p, neblock);
            else if (ora_lz4_decompress(p, cs, o, neblock) != neblock) { free(tmp); return -12; }
            p += cs;
        }
        if (shuffle && typesize > 1) ora_unshuffle(typesize, bsize, tmp, dst + (size_t)b * blocksize);
    }
    free(tmp);
    return nbytes;
}

/* ironArray's chunk_is_zeros (src/linalg/iarray_gemm.c:17-26). */
EXPORT int ora_chunk_is_zeros(const uint8_t *chunk)
{
    return ((chunk[31] >> 4) & 7) == 1;
}

/* ironArray's block_is_zeros (src/linalg/iarray_gemm.c:29-77), non-lazy chunks:
 * true when every stream of the block has csize 0.  Memcpyed and special chunks
 * are never "zero blocks". */
EXPORT int ora_block_is_zeros(const uint8_t *chunk, int nblock)
{
    int flags = chunk[2];
    int memcpyed = flags & 0x02, split = flags & 0x04;   /* bit2 is set for every v5 chunk */
    int special = (chunk[31] >> 4) & 7;
    if (memcpyed || special) return 0;
    int32_t bstart = rds32(chunk + HDR + 4 * nblock);
    const uint8_t *p = chunk + bstart, *pend = chunk + rds32(chunk + 12);
    int n = split ? chunk[3] : 1;
    for (int i = 0; i < n; i++) {
        if (pend - p < 4) return 0;            /* guard: never read past cbytes */
        int32_t cs = rds32(p);
        if (cs != 0) return 0;
        p += 4 + cs;
    }
    return 1;
}

/* ------------------------------------------------------------------------- */
/* Caterva layout: logical row-major buffer <-> padded blocked chunk          */
/* ------------------------------------------------------------------------- */
typedef struct {
    int ndim, itemsize;
    int64_t shape[8], chunk[8], block[8];
} ora_geom_t;

static int64_t ceil_to(int64_t a, int64_t b) { return ((a + b - 1) / b) * b; }

/* Gather chunk `nchunk` (row-major chunk index) from the logical buffer into its
 * padded blocked byte layout (extchunk items; padding = 0). */
EXPORT void ora_chunk_from_buffer(const ora_geom_t *g, const uint8_t *buf, int64_t nchunk, uint8_t *out)
{
    int nd = g->ndim, is = g->itemsize;
    int64_t ext[8], cgrid[8], bgrid[8], cidx[8];
    int64_t rem = nchunk;
    for (int d = nd - 1; d >= 0; d--) {
        ext[d] = ceil_to(g->chunk[d], g->block[d]);
        cgrid[d] = ceil_to(g->shape[d], g->chunk[d]) / g->chunk[d];
        bgrid[d] = ext[d] / g->block[d];
        cidx[d] = rem % cgrid[d]; rem /= cgrid[d];
    }
    int64_t blockn = 1, nblocks = 1;
    for (int d = 0; d < nd; d++) { blockn *= g->block[d]; nblocks *= bgrid[d]; }
    for (int64_t b = 0; b < nblocks; b++) {
        int64_t bi[8], r = b;
        for (int d = nd - 1; d >= 0; d--) { bi[d] = r % bgrid[d]; r /= bgrid[d]; }
        for (int64_t e = 0; e < blockn; e++) {
            int64_t ei[8], q = e, flat = 0, inside = 1;
            for (int d = nd - 1; d >= 0; d--) { ei[d] = q % g->block[d]; q /= g->block[d]; }
            for (int d = 0; d < nd; d++) {
                int64_t within = bi[d] * g->block[d] + ei[d];      /* coordinate inside chunk */
                int64_t gl = cidx[d] * g->chunk[d] + within;
                if (within >= g->chunk[d] || gl >= g->shape[d]) inside = 0;
                flat = flat * g->shape[d] + gl;
            }
            uint8_t *o = out + (b * blockn + e) * is;
            if (inside) memcpy(o, buf + flat * is, is); else memset(o, 0, is);
        }
    }
}

EXPORT void ora_chunk_to_buffer(const ora_geom_t *g, const uint8_t *chunkdata, int64_t nchunk, uint8_t *buf)
{
    int nd = g->ndim, is = g->itemsize;
    int64_t ext[8], cgrid[8], bgrid[8], cidx[8];
    int64_t rem = nchunk;
    for (int d = nd - 1; d >= 0; d--) {
        ext[d] = ceil_to(g->chunk[d], g->block[d]);
        cgrid[d] = ceil_to(g->shape[d], g->chunk[d]) / g->chunk[d];
        bgrid[d] = ext[d] / g->block[d];
        cidx[d] = rem % cgrid[d]; rem /= cgrid[d];
    }
    int64_t blockn = 1, nblocks = 1;
    for (int d = 0; d < nd; d++) { blockn *= g->block[d]; nblocks *= bgrid[d]; }
    for (int64_t b = 0; b < nblocks; b++) {
        int64_t bi[8], r = b;
        for (int d = nd - 1; d >= 0; d--) { bi[d] = r % bgrid[d]; r /= bgrid[d]; }
        for (int64_t e = 0; e < blockn; e++) {
            int64_t ei[8], q = e, flat = 0, inside = 1;
            for (int d = nd - 1; d >= 0; d--) { ei[d] = q % g->block[d]; q /= g->block[d]; }
            for (int d = 0; d < nd; d++) {
                int64_t within = bi[d] * g->block[d] + ei[d];
                int64_t gl = cidx[d] * g->chunk[d] + within;
                if (within >= g->chunk[d] || gl >= g->shape[d]) inside = 0;
                flat = flat * g->shape[d] + gl;
            }
            if (inside) memcpy(buf + flat * is, chunkdata + (b * blockn + e) * is, is);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Blocked GEMM / GEMV restated on decoded chunks                            */
/* ------------------------------------------------------------------------- */
/* A "super-chunk" here is an array of chunk pointers + lengths in row-major chunk
 * order.  Every product below accumulates block products in the reference's order;
 * the block product itself is C[i][j] += sum_k A[i][k]*B[k][j] with k ascending. */
typedef struct {
    ora_geom_t g;
    const uint8_t *const *chunks;
    const int32_t *chunk_len;
} ora_schunk_t;

static int64_t ext_of(const ora_geom_t *g, int d) { return ceil_to(g->shape[d], g->chunk[d]); }
static int64_t extc_of(const ora_geom_t *g, int d) { return ceil_to(g->chunk[d], g->block[d]); }

/* Decode block `nblock` of chunk `ch` into out (blockn items). */
static int decode_block(const ora_schunk_t *s, int64_t ch, int64_t nblock, uint8_t *scratch_chunk, uint8_t *out)
{
    int64_t blockn = 1;
    for (int d = 0; d < s->g.ndim; d++) blockn *= s->g.block[d];
    int64_t extcn = 1;
    for (int d = 0; d < s->g.ndim; d++) extcn *= extc_of(&s->g, d);
    int nb = (int)(extcn * s->g.itemsize);
    if (ora_chunk_decompress(s->chunks[ch], s->chunk_len[ch], scratch_chunk, nb) != nb) return -1;
    memcpy(out, scratch_chunk + nblock * blockn * s->g.itemsize, blockn * s->g.itemsize);
    return 0;
}

#define DEF_BLOCK_GEMM(T, NAME)                                                       \
static void NAME(int64_t M, int64_t N, int64_t K, const T *a, int64_t lda,           \
                 const T *b, int64_t ldb, T *c, int64_t ldc)                          \
{                                                                                    \
    for (int64_t i = 0; i < M; i++)                                                  \
        for (int64_t j = 0; j < N; j++) {                                            \
            T acc = c[i * ldc + j];                                                  \
            for (int64_t k = 0; k < K; k++) acc += a[i * lda + k] * b[k * ldb + j];  \
            c[i * ldc + j] = acc;                                                    \
        }                                                                            \
}
DEF_BLOCK_GEMM(double, bgemm_d)
DEF_BLOCK_GEMM(float, bgemm_f)

/* iarray_opt_gemm (src/linalg/iarray_gemm.c:91-312, :392-425): for every output
 * chunk, every output block: zero it, then for each K chunk (skipping special-zero
 * chunks of B then A) and each K block (skipping all-zero blocks of A then B),
 * trim M/K/N at the container edge and accumulate A_blk * B_blk with the full
 * block leading dimensions.  Writes C's padded chunk data (c_chunks[n] holds
 * extchunk items of chunk n).  dtype 0 = double, 1 = float. */
EXPORT int ora_opt_gemm_rule(const ora_schunk_t *A, const ora_schunk_t *B, const ora_geom_t *Cg,
                             int dtype, uint8_t *const *c_chunks, int chunk_rule);

EXPORT int ora_opt_gemm(const ora_schunk_t *A, const ora_schunk_t *B, const ora_geom_t *Cg,
                        int dtype, uint8_t *const *c_chunks)
{
    return ora_opt_gemm_rule(A, B, Cg, dtype, c_chunks, 3);
}

/* The same loop with the chunk-level skip of each operand switchable: chunk_rule bit 0 =
 * skip A's special-zero chunks, bit 1 = B's.  iarray_opt_gemm uses both (3);
 * iarray_opt_gemm_a only B's (2: src/linalg/iarray_gemm_a.c:127-146, where A's blocks are
 * judged by block_is_zeros alone, :313); iarray_opt_gemm_b only A's (1: iarray_gemm_b.c). */
EXPORT int ora_opt_gemm_rule(const ora_schunk_t *A, const ora_schunk_t *B, const ora_geom_t *Cg,
                             int dtype, uint8_t *const *c_chunks, int chunk_rule)
{
    const ora_geom_t *ag = &A->g, *bg = &B->g;
    int is = ag->itemsize;
    int64_t Mch = ext_of(ag, 0) / ag->chunk[0], Kch = ext_of(ag, 1) / ag->chunk[1];
    int64_t Nch = ext_of(bg, 1) / bg->chunk[1];
    int64_t Kbl = extc_of(ag, 1) / ag->block[1], Nbl = extc_of(bg, 1) / bg->block[1];
    int64_t Mbl = extc_of(ag, 0) / ag->block[0];
    int64_t a_extcn = extc_of(ag, 0) * extc_of(ag, 1), b_extcn = extc_of(bg, 0) * extc_of(bg, 1);
    uint8_t *adec = malloc(a_extcn * is), *bdec = malloc(b_extcn * is);
    int64_t cbn = Cg->block[0] * Cg->block[1];
    for (int64_t cn = 0; cn < Mch * Nch; cn++) {
        int64_t ci0 = cn / Nch, ci1 = cn % Nch;
        uint8_t *cchunk = c_chunks[cn];
        memset(cchunk, 0, extc_of(Cg, 0) * extc_of(Cg, 1) * is);
        for (int64_t cb = 0; cb < Mbl * Nbl; cb++) {
            int64_t cb0 = cb / Nbl, cb1 = cb % Nbl;
            uint8_t *out = cchunk + cb * cbn * is;
            for (int64_t kc = 0; kc < Kch; kc++) {
                int64_t an = ci0 * Kch + kc, bn = kc * Nch + ci1;
                if ((chunk_rule & 2) && ora_chunk_is_zeros(B->chunks[bn])) continue;
                if ((chunk_rule & 1) && ora_chunk_is_zeros(A->chunks[an])) continue;
                if (ora_chunk_decompress(A->chunks[an], A->chunk_len[an], adec, (int)(a_extcn * is)) < 0) goto fail;
                if (ora_chunk_decompress(B->chunks[bn], B->chunk_len[bn], bdec, (int)(b_extcn * is)) < 0) goto fail;
                int pad_m = ag->shape[0] != ext_of(ag, 0) && ci0 == Mch - 1;
                int pad_k = ag->shape[1] != ext_of(ag, 1) && kc == Kch - 1;
                int pad_n = bg->shape[1] != ext_of(bg, 1) && ci1 == Nch - 1;
                for (int64_t kb = 0; kb < Kbl; kb++) {
                    int64_t anb = cb0 * Kbl + kb, bnb = kb * Nbl + cb1;
                    if (ora_block_is_zeros(A->chunks[an], (int)anb)) continue;
                    if (ora_block_is_zeros(B->chunks[bn], (int)bnb)) continue;
                    int64_t M = ag->block[0], K = ag->block[1], N = bg->block[1];
                    int64_t lda = K, ldb = N, ldc = N;
                    if (pad_m) {
                        int64_t s = ci0 * ag->chunk[0] + cb0 * ag->block[0], e = s + ag->block[0];
                        if (ag->shape[0] <= s) continue;
                        M = ag->shape[0] < e ? ag->shape[0] - s : e - s;
                    }
                    if (pad_k) {
                        int64_t s = kc * ag->chunk[1] + kb * ag->block[1], e = s + ag->block[1];
                        if (ag->shape[1] <= s) continue;
                        K = ag->shape[1] < e ? ag->shape[1] - s : e - s;
                    }
                    if (pad_n) {
                        int64_t s = ci1 * bg->chunk[1] + cb1 * bg->block[1], e = s + bg->block[1];
                        if (bg->shape[1] <= s) continue;
                        N = bg->shape[1] < e ? bg->shape[1] - s : e - s;
                    }
                    const uint8_t *ab = adec + anb * ag->block[0] * ag->block[1] * is;
                    const uint8_t *bb = bdec + bnb * bg->block[0] * bg->block[1] * is;
                    if (dtype == 0) bgemm_d(M, N, K, (const double *)ab, lda, (const double *)bb, ldb, (double *)out, ldc);
                    else bgemm_f(M, N, K, (const float *)ab, lda, (const float *)bb, ldb, (float *)out, ldc);
                }
            }
        }
    }
    free(adec); free(bdec);
    return 0;
fail:
    free(adec); free(bdec);
    return -1;
}

/* iarray_opt_gemv (src/linalg/iarray_gemv.c:88-246, :320-344): per output chunk and
 * output block, for each K chunk (B chunk checked first for special zeros) and K block
 * (zero blocks skipped), trim rows/cols at the edge and accumulate A_blk * x_blk. */
EXPORT int ora_opt_gemv(const ora_schunk_t *A, const ora_schunk_t *X, const ora_geom_t *Cg,
                        int dtype, uint8_t *const *c_chunks)
{
    const ora_geom_t *ag = &A->g, *xg = &X->g;
    int is = ag->itemsize;
    int64_t Mch = ext_of(ag, 0) / ag->chunk[0], Kch = ext_of(ag, 1) / ag->chunk[1];
    int64_t Mbl = extc_of(ag, 0) / ag->block[0], Kbl = extc_of(ag, 1) / ag->block[1];
    int64_t a_extcn = extc_of(ag, 0) * extc_of(ag, 1), x_extcn = extc_of(xg, 0);
    uint8_t *adec = malloc(a_extcn * is), *xdec = malloc(x_extcn * is);
    for (int64_t cn = 0; cn < Mch; cn++) {
        uint8_t *cchunk = c_chunks[cn];
        memset(cchunk, 0, extc_of(Cg, 0) * is);
        for (int64_t cb = 0; cb < Mbl; cb++) {
            uint8_t *out = cchunk + cb * Cg->block[0] * is;
            for (int64_t kc = 0; kc < Kch; kc++) {
                int64_t an = cn * Kch + kc;
                if (ora_chunk_is_zeros(X->chunks[kc])) continue;
                if (ora_chunk_is_zeros(A->chunks[an])) continue;
                if (ora_chunk_decompress(A->chunks[an], A->chunk_len[an], adec, (int)(a_extcn * is)) < 0) goto fail;
                if (ora_chunk_decompress(X->chunks[kc], X->chunk_len[kc], xdec, (int)(x_extcn * is)) < 0) goto fail;
                for (int64_t kb = 0; kb < Kbl; kb++) {
                    int64_t anb = cb * Kbl + kb;
                    if (ora_block_is_zeros(A->chunks[an], (int)anb)) continue;
                    if (ora_block_is_zeros(X->chunks[kc], (int)kb)) continue;
                    int64_t r0 = ag->chunk[0] * cn + ag->block[0] * cb, rows, cols;
                    if (r0 > ag->shape[0]) continue;
                    rows = (r0 + ag->block[0] > ag->shape[0]) ? ag->shape[0] - r0 : ag->block[0];
                    int64_t c0 = ag->chunk[1] * kc + ag->block[1] * kb;
                    if (c0 > ag->shape[1]) continue;
                    cols = (c0 + ag->block[1] > ag->shape[1]) ? ag->shape[1] - c0 : ag->block[1];
                    const uint8_t *ab = adec + anb * ag->block[0] * ag->block[1] * is;
                    const uint8_t *xb = xdec + kb * xg->block[0] * is;
                    if (dtype == 0) bgemm_d(rows, 1, cols, (const double *)ab, ag->block[1], (const double *)xb, 1, (double *)out, 1);
                    else bgemm_f(rows, 1, cols, (const float *)ab, ag->block[1], (const float *)xb, 1, (float *)out, 1);
                }
            }
        }
    }
    free(adec); free(xdec);
    return 0;
fail:
    free(adec); free(xdec);
    return -1;
}

/* Dense products on logical row-major buffers, k ascending (the panel path's block
 * product with k = the full K, src/linalg/matmul/gemm.c:97, gemv.c:93). */
EXPORT void ora_dense_gemm(int dtype, int64_t M, int64_t N, int64_t K, const void *a, const void *b, void *c)
{
    if (dtype == 0) { memset(c, 0, M * N * 8); bgemm_d(M, N, K, a, K, b, N, c, N); }
    else { memset(c, 0, M * N * 4); bgemm_f(M, N, K, a, K, b, N, c, N); }
}

/* ------------------------------------------------------------------------- */
/* Double-double reference rows: C[r,:] = sum_k A[r,k] * B[k,:]               */
/* ------------------------------------------------------------------------- */
/* Error-free TwoProd (via fma) and TwoSum; accumulates hi+lo per output element.
 * The relative error of hi+lo is ~K * 2^-104, far below every form measured here.
 * Work is split over `nthreads` POSIX threads by (row, 256-column strip). */
typedef struct {
    const double *A, *B; int64_t N, K; const int64_t *rows; int64_t nrows;
    double *hi, *lo; int64_t ntasks; int64_t next; pthread_mutex_t mu;
} dd_job_t;

static void dd_task(dd_job_t *jb, int64_t t)
{
    int64_t strips = (jb->N + 255) / 256;
    int64_t ri = t / strips, j0 = (t % strips) * 256;
    int64_t j1 = j0 + 256 < jb->N ? j0 + 256 : jb->N, w = j1 - j0;
    int64_t r = jb->rows[ri], N = jb->N, K = jb->K;
    double hi[256], lo[256];
    for (int64_t j = 0; j < w; j++) { hi[j] = 0; lo[j] = 0; }
    for (int64_t k = 0; k < K; k++) {
        double a = jb->A[r * K + k];
        const double *brow = jb->B + k * N + j0;
        for (int64_t j = 0; j < w; j++) {
            double p = a * brow[j];
            double pe = fma(a, brow[j], -p);
            double s = hi[j] + p;
            double bb = s - hi[j];
            double se = (hi[j] - (s - bb)) + (p - bb);
            hi[j] = s;
            lo[j] += se + pe;
        }
    }
    for (int64_t j = 0; j < w; j++) {
        double s = hi[j] + lo[j];
        jb->lo[ri * N + j0 + j] = lo[j] - (s - hi[j]);
        jb->hi[ri * N + j0 + j] = s;
    }
}

static void *dd_worker(void *arg)
{
    dd_job_t *jb = (dd_job_t *)arg;
    for (;;) {
        pthread_mutex_lock(&jb->mu);
        int64_t t = jb->next++;
        pthread_mutex_unlock(&jb->mu);
        if (t >= jb->ntasks) break;
        dd_task(jb, t);
    }
    return NULL;
}

EXPORT void ora_dd_rows(const double *A, const double *B, int64_t M, int64_t N, int64_t K,
                        const int64_t *rows, int64_t nrows, double *out_hi, double *out_lo, int nthreads)
{
    (void)M;
    dd_job_t jb = { A, B, N, K, rows, nrows, out_hi, out_lo, nrows * ((N + 255) / 256), 0 };
    pthread_mutex_init(&jb.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, dd_worker, &jb);
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&jb.mu);
}

/* ------------------------------------------------------------------------- */
/* CPU baseline: the reference's block-pair loop, timed (bench only)          */
/* ------------------------------------------------------------------------- */
/* Computes output chunk `cn` of iarray_opt_gemm exactly as the reference's prefilter
 * does (src/linalg/iarray_gemm.c:91-312): one worker per output block (Blosc2's
 * thread pool with MKL pinned to one thread, src/linalg/matmul/gemm.c:261-264), each
 * worker decoding the A and B block of every K block pair again and accumulating with a
 * single-threaded BLAS dgemm (beta = 1), then Blosc2-compressing the finished chunk.
 * `dgemm` is a cblas_dgemm-compatible function pointer (row-major); `lz4_dec` /
 * `lz4_enc` optionally point at liblz4's LZ4_decompress_safe / LZ4_compress_fast (the
 * codec the reference's Blosc2 bundles); NULL selects this file's restatement. */
typedef void (*cblas_dgemm_fn)(int, int, int, int, int, int, double, const double *, int, const double *, int,
                               double, double *, int);
typedef int (*lz4_dec_fn)(const char *, char *, int, int);

typedef struct {
    const ora_schunk_t *A, *B;
    const ora_geom_t *Cg;
    int64_t cn;
    cblas_dgemm_fn dgemm;
    lz4_dec_fn dec;
    uint8_t *cchunk;
    /* per-block compression (whole-product form): block b's Blosc2 payload (its streams,
     * csize words included) goes to bout + b * bcap, its length to blen[b]; -1 when the
     * block does not compress into its own size (the chunk is then compressed whole) */
    uint8_t *bout;
    int64_t bcap;
    int32_t *blen;
    int64_t next;
    pthread_mutex_t mu;
    int err;
} bl_job_t;

/* Decode one block of a chunk with the block's own streams (blosc2_getitem_ctx). */
static int bl_decode_block(const uint8_t *chunk, int nblock, uint8_t *out, uint8_t *tmp, lz4_dec_fn dec)
{
    int flags = chunk[2], ts = chunk[3];
    int blocksize = rds32(chunk + 8);
    if (((chunk[31] >> 4) & 7) == 1) { memset(out, 0, blocksize); return 0; }
    if (flags & 0x02) { memcpy(out, chunk + HDR + (size_t)nblock * blocksize, blocksize); return 0; }
    int split = !(flags & 0x10), shuffle = chunk[21] == 1;
    int nstreams = split ? ts : 1, neblock = blocksize / nstreams;
    const uint8_t *p = chunk + rds32(chunk + HDR + 4 * nblock);
    uint8_t *o = (shuffle && ts > 1) ? tmp : out;
    for (int j = 0; j < nstreams; j++) {
        int32_t cs = rds32(p); p += 4;
        if (cs == 0) memset(o + j * neblock, 0, neblock);
        else if (cs < 0) { memset(o + j * neblock, -cs, neblock); p += 1; cs = 0; }
        else if (cs == neblock) memcpy(o + j * neblock, p, neblock);
        else {
            int r = dec ? dec((const char *)p, (char *)(o + j * neblock), cs, neblock)
                        : ora_lz4_decompress(p, cs, o + j * neblock, neblock);
            if (r != neblock) return -1;
        }
        if (cs > 0) p += cs;
    }
    if (shuffle && ts > 1) ora_unshuffle(ts, blocksize, tmp, out);
    return 0;
}

static void *bl_worker(void *arg)
{
    bl_job_t *jb = (bl_job_t *)arg;
    const ora_geom_t *ag = &jb->A->g, *bg = &jb->B->g;
    int64_t Kch = ext_of(ag, 1) / ag->chunk[1], Nch = ext_of(bg, 1) / bg->chunk[1];
    int64_t Kbl = extc_of(ag, 1) / ag->block[1], Nbl = extc_of(bg, 1) / bg->block[1];
    int64_t Mbl = extc_of(ag, 0) / ag->block[0];
    int64_t ci0 = jb->cn / Nch, ci1 = jb->cn % Nch;
    int64_t bm = ag->block[0], bk = ag->block[1], bn = bg->block[1];
    uint8_t *ablk = malloc(bm * bk * 8), *bblk = malloc(bk * bn * 8);
    uint8_t *tmp = malloc((bm * bk > bk * bn ? bm * bk : bk * bn) * 8);
    for (;;) {
        pthread_mutex_lock(&jb->mu);
        int64_t cb = jb->next++;
        pthread_mutex_unlock(&jb->mu);
        if (cb >= Mbl * Nbl) break;
        int64_t cb0 = cb / Nbl, cb1 = cb % Nbl;
        double *out = (double *)(jb->cchunk + cb * jb->Cg->block[0] * jb->Cg->block[1] * 8);
        memset(out, 0, bm * bn * 8);
        for (int64_t kc = 0; kc < Kch; kc++) {
            const uint8_t *ach = jb->A->chunks[ci0 * Kch + kc], *bch = jb->B->chunks[kc * Nch + ci1];
            if (ora_chunk_is_zeros(ach) || ora_chunk_is_zeros(bch)) continue;
            for (int64_t kb = 0; kb < Kbl; kb++) {
                int anb = (int)(cb0 * Kbl + kb), bnb = (int)(kb * Nbl + cb1);
                if (ora_block_is_zeros(ach, anb) || ora_block_is_zeros(bch, bnb)) continue;
                if (bl_decode_block(ach, anb, ablk, tmp, jb->dec) || bl_decode_block(bch, bnb, bblk, tmp, jb->dec)) {
                    jb->err = 1;
                    continue;
                }
                jb->dgemm(101, 111, 111, (int)bm, (int)bn, (int)bk, 1.0, (const double *)ablk, (int)bk,
                          (const double *)bblk, (int)bn, 1.0, out, (int)bn);
            }
        }
        if (jb->bout) {
            /* Blosc2 compresses each block in the thread that filled it: shuffle + split
             * streams of this block alone (a one-block chunk holds exactly those bytes
             * after its header and its single bstart) */
            const int bsz = (int)(bm * bn * 8);
            uint8_t *cb1 = malloc((size_t)bsz + HDR + 64);
            int r = ora_chunk_compress((const uint8_t *)out, bsz, 8, bsz, 1, SPLIT_AUTO, cb1, bsz + HDR);
            int32_t plen = -1;
            if (r > 0 && !(cb1[2] & 0x02) && r - HDR - 4 <= jb->bcap) {
                plen = r - HDR - 4;
                memcpy(jb->bout + cb * jb->bcap, cb1 + HDR + 4, (size_t)plen);
            }
            jb->blen[cb] = plen;
            free(cb1);
        }
    }
    free(ablk); free(bblk); free(tmp);
    return NULL;
}




/* The whole product: every output chunk of iarray_opt_gemm in the reference's order
 * (src/linalg/iarray_gemm.c:399-425: one blosc2_compress_ctx per output chunk, its
 * prefilter run by `nthreads` workers over the chunk's blocks).  Each worker computes
 * an output block and compresses it at once, as Blosc2's workers do; the chunk is then
 * assembled from the block payloads (header, bstarts, payloads in block order).  Output
 * chunk c goes to outs[c] (capacity chunk_nbytes + 32), its size to out_len[c].
 * Returns 0, or < 0 on error. */
EXPORT int ora_cpu_opt_gemm(const ora_schunk_t *A, const ora_schunk_t *B, const ora_geom_t *Cg, int nthreads,
                            void *dgemm, void *lz4_dec, uint8_t **outs, int32_t *out_len)
{
    const int64_t ext0 = extc_of(Cg, 0), ext1 = extc_of(Cg, 1);
    const int64_t cnb = ext0 * ext1 * 8;
    const int64_t nch = (ext_of(Cg, 0) / Cg->chunk[0]) * (ext_of(Cg, 1) / Cg->chunk[1]);
    const int64_t nbl = (ext0 / Cg->block[0]) * (ext1 / Cg->block[1]);
    const int64_t bsz = Cg->block[0] * Cg->block[1] * 8;
    const int64_t bcap = bsz + 8 * 4 + 8;          /* streams no larger than the block, csize words */
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    uint8_t *cchunk = malloc((size_t)cnb), *bout = malloc((size_t)(nbl * bcap));
    int32_t *blen = malloc((size_t)nbl * 4);
    int rc = 0;
    for (int64_t cn = 0; cn < nch && rc == 0; cn++) {
        bl_job_t jb;
        memset(&jb, 0, sizeof(jb));
        jb.A = A; jb.B = B; jb.Cg = Cg; jb.cn = cn;
        jb.dgemm = (cblas_dgemm_fn)dgemm; jb.dec = (lz4_dec_fn)lz4_dec;
        jb.cchunk = cchunk; jb.bout = bout; jb.bcap = bcap; jb.blen = blen;
        pthread_mutex_init(&jb.mu, NULL);
        pthread_t th[256];
        for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, bl_worker, &jb);
        for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
        pthread_mutex_destroy(&jb.mu);
        if (jb.err) { rc = -1; break; }
        int64_t pos = HDR + 4 * nbl;
        int whole = 0;
        for (int64_t b = 0; b < nbl; b++) {
            if (blen[b] < 0 || pos + blen[b] > cnb) { whole = 1; break; }
            wr32(outs[cn] + HDR + 4 * b, (int32_t)pos);
            memcpy(outs[cn] + pos, bout + b * bcap, (size_t)blen[b]);
            pos += blen[b];
        }
        if (whole) {
            int r = ora_chunk_compress(cchunk, (int)cnb, 8, (int)bsz, 1, SPLIT_AUTO, outs[cn], (int)cnb + 32);
            if (r < 0) { rc = -2; break; }
            out_len[cn] = r;
        } else {
            const int split = ora_split_decision(SPLIT_AUTO, CODEC_LZ4, 1, 8, (int)bsz);
            write_header(outs[cn], 0x05 | (CODEC_LZ4 << 5) | (split ? 0 : 0x10), 8, (int)cnb, (int)bsz, (int)pos, 1,
                         CODEC_LZ4);
            out_len[cn] = (int32_t)pos;
        }
    }
    free(cchunk); free(bout); free(blen);
    return rc;
}

/* Returns the compressed size of the output chunk written to `out` (capacity
 * chunk_nbytes + 32), or < 0 on error. */
EXPORT int ora_cpu_opt_gemm_chunk(const ora_schunk_t *A, const ora_schunk_t *B, const ora_geom_t *Cg, int64_t cn,
                                  int nthreads, void *dgemm, void *lz4_dec, uint8_t *out)
{
    int64_t cnb = extc_of(Cg, 0) * extc_of(Cg, 1) * 8;
    bl_job_t jb;
    memset(&jb, 0, sizeof(jb));
    jb.A = A; jb.B = B; jb.Cg = Cg; jb.cn = cn;
    jb.dgemm = (cblas_dgemm_fn)dgemm; jb.dec = (lz4_dec_fn)lz4_dec;
    jb.cchunk = malloc(cnb);
    pthread_mutex_init(&jb.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, bl_worker, &jb);
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&jb.mu);
    int r = jb.err ? -1 : ora_chunk_compress(jb.cchunk, (int)cnb, 8, (int)(Cg->block[0] * Cg->block[1] * 8), 1,
                                             SPLIT_AUTO, out, (int)cnb + 32);
    free(jb.cchunk);
    return r;
}
