// Shared definitions for the B200 kernels and the host runtime.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <mutex>
#include <map>
#include <vector>

namespace iab {

// ------------------------------------------------------------------ geometry
// A container's partition, viewed as 2-D: 1-D arrays of n items are 1 x n with
// chunk 1 x c and block 1 x b (Caterva's 1-D layout is the same byte sequence).
struct Geom {
    int itemsize;
    int ndim;
    int64_t shape[2], chunk[2], block[2];
    int64_t extc[2];       // extchunkshape = chunk rounded up to block
    int64_t cgrid[2];      // chunks per dimension (extshape / chunkshape)
    int64_t bgrid[2];      // blocks per dimension inside a chunk
    int64_t nchunks;       // cgrid[0] * cgrid[1]
    int64_t nblocks;       // blocks per chunk
    int64_t blockn;        // items per block
    int64_t blocksize;     // bytes per block
    int64_t chunk_nbytes;  // bytes per (padded) chunk
};

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
static inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

struct ZeroSkip;   // zskip.cuh

// Builds the geometry; returns false when the partition is invalid.
bool make_geom(int ndim, const int64_t *shape, const int64_t *chunk, const int64_t *block,
               int itemsize, Geom *g);

// ------------------------------------------------------------------ codec descriptors
enum StreamKind : int32_t { SK_RUN = 0, SK_RAW = 1, SK_LZ4 = 2 };
enum BlockMode : int32_t { BM_SHUFFLED = 0, BM_PLAIN = 1, BM_NAN = 2, BM_VALUE = 3 };

struct StreamDesc {   // one compressed stream of one block, found by the parse kernel
    int32_t kind;     // StreamKind
    int32_t len;      // csize for LZ4 / raw, byte value for runs
    int64_t src;      // byte offset of the payload in the container's chunk buffer
};

struct BlockDesc {
    int32_t mode;      // BlockMode
    int32_t nstreams;  // typesize when split, else 1
    int32_t neblock;   // bytes per stream
    int32_t pad;
    int64_t value_src; // BM_VALUE: offset of the repeated item
};

struct Lz4Job {       // decode job: one LZ4 stream
    const uint8_t *src;  // payload in the container's chunk buffer
    uint8_t *dst;        // its place in the container's decoded-stream image
    int *err;            // the container's status word
    int32_t csize;
    int32_t dlen;
};

struct EncStream {    // per-stream result of the LZ4 encoder
    int32_t kind;     // SK_RUN / SK_RAW / SK_LZ4
    int32_t csize;    // LZ4: compressed size; RUN: byte value
    int32_t need;     // LZ4: the smallest output capacity for which limited mode succeeds
    int32_t out;      // final offset of the stream's csize word inside its chunk (-1: none)
};

struct EncChunk {
    int32_t cbytes;
    int32_t memcpyed;
    int64_t offset;   // byte offset of the chunk in the container buffer
};

// Error codes reported by kernels through a device status word (first error wins).
enum DevErr : int32_t {
    DE_OK = 0,
    DE_HEADER = 1,      // chunk header does not match the container geometry
    DE_BOUNDS = 2,      // a bstart / csize points outside the chunk
    DE_LZ4 = 3,         // malformed LZ4 stream
    DE_RUN_TOKEN = 4,   // negative csize without a valid run token
    DE_WAIT = 5,        // a bounded wait for an asynchronous copy gave up
};

// ------------------------------------------------------------------ device memory pool
// Caching allocator: freed blocks are kept per size class and reused, so steady-state
// calls do no cudaMalloc.  One pool per device, shared by all contexts.
class DevicePool {
public:
    static DevicePool &get(int device);
    void *alloc(size_t bytes);
    void release(void *p);
    void trim();
private:
    std::mutex mu_;
    std::multimap<size_t, void *> free_;
    std::map<void *, size_t> used_;
};

struct DevBuf {   // RAII handle over a pool allocation
    void *p = nullptr;
    size_t n = 0;
    int dev = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept { p = o.p; n = o.n; dev = o.dev; o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept { reset(); p = o.p; n = o.n; dev = o.dev; o.p = nullptr; o.n = 0; return *this; }
    ~DevBuf() { reset(); }
    bool allocate(size_t bytes, int device);
    void reset();
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// ------------------------------------------------------------------ kernel entry points
// Every kernel launch of the library adds to this counter (read through the C ABI).
extern std::atomic<uint64_t> g_launches;
#define IAB_LAUNCHED(n) (::iab::g_launches.fetch_add((n), std::memory_order_relaxed))
// Counts and (while kernel profiling is on) times one launch statement on stream `st`.
#define IAB_TIMED(name, st, ...)                   \
    do {                                           \
        ::iab::KernelTimer iab_kt_((name), (st));  \
        IAB_LAUNCHED(1);                           \
        __VA_ARGS__;                               \
    } while (0)

// Brackets one kernel launch with CUDA events on its stream while kernel profiling is on
// (iarray_b200_profile_kernels); does nothing otherwise.  Construct it right before the
// launch, in the launch's scope.
class KernelTimer {
public:
    KernelTimer(const char *name, cudaStream_t st);
    ~KernelTimer();
    KernelTimer(const KernelTimer &) = delete;
    KernelTimer &operator=(const KernelTimer &) = delete;
private:
    const char *name_;
    cudaStream_t st_;
    cudaEvent_t e0_ = nullptr;
};

// Switches kernel profiling on or off without clearing it; returns the previous state.
bool kprof_enable(bool on);

struct CodecStats { int32_t err; };

// Decode `g.nchunks` chunks (buffer d_chunks, offsets d_off) into a dense row-major
// array `out` with leading dimension `ld` items.  Returns a DevErr (synchronises).
int decode_container(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, const int64_t *d_off,
                     const int32_t *d_len, void *out, int64_t ld, cudaStream_t st);

struct DecodeArgs {
    Geom g;
    const uint8_t *chunks;  // the container's chunks, back to back
    int64_t chunks_bytes;
    const int64_t *off;     // chunk offsets and lengths (device)
    const int32_t *len;
    void *out;              // dense row-major destination
    int64_t ld;             // its leading dimension in items
};
struct DecodeQueue {
    DevBuf jobs, counters;  // counters: [0] jobs queued, [1] the next job to hand out
    int64_t cap = 0;
};
// Asynchronous form: decode_launch enqueues the kernels on `st` (work buffers held in
// *w until decode_finish, which synchronises `st` and returns the DevErr).
struct DecodeWork {
    DevBuf bd, sd, scratch, counters, rest;
    DevBuf zf;                     // per (chunk, block) zero flags of the block-pair products (k_parse)
    DecodeQueue queue;             // the job queue of decode_launch (unused by decode_parse / _scatter)
    int *ext_counters = nullptr;   // optional caller-owned 16-int status slot (device) instead of `counters`
    int nzero = 0;                 // flagged blocks, read back by decode_finish
};
int decode_launch(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, const int64_t *d_off, const int32_t *d_len,
                  void *out, int64_t ld, cudaStream_t st, DecodeWork *w);
int decode_finish(DecodeWork *w, cudaStream_t st);

// Several containers decoded with one LZ4 launch: decode_queue_init (on the stream that
// will run the LZ4 launch), then decode_parse of each container (any streams ordered after
// the init), decode_lz4 once (ordered after every parse), then decode_scatter of each
// container (after the LZ4 launch); decode_finish(w) per container as above.  The LZ4
// streams of all containers are handed out from one queue, so the LZ4 kernel's CTAs stay
// busy across container boundaries.
int decode_queue_init(DecodeQueue *q, int64_t max_jobs, cudaStream_t st);
int64_t decode_max_jobs(const Geom &g);
int decode_parse(const DecodeArgs &a, DecodeQueue *q, DecodeWork *w, cudaStream_t st);
int decode_lz4(DecodeQueue *q, cudaStream_t st);
int decode_scatter(const DecodeArgs &a, DecodeWork *w, cudaStream_t st);
// Decode-fused GEMV y = A x in place of decode_scatter(A) (after decode_parse and decode_lz4
// of A; x dense on the device): part holds decode_gemv_part_items(g) items of A's type (row
// sums per block column), y gets the M sums.  The dense A is never written.  Partitions of
// 2-D float32 / float64 containers whose block rows hold whole groups of 4 items and at most
// 4096 items (decode_gemv_fits).
bool decode_gemv_fits(const Geom &g);
int64_t decode_gemv_part_items(const Geom &g);
int decode_gemv(const DecodeArgs &a, DecodeWork *w, const void *x, void *part, void *y, cudaStream_t st);

// Decode without allocating: the work buffers live in a fixed device array of the library
// (at most NOALLOC_MAX_BYTES decoded bytes and NOALLOC_MAX_BLOCKS blocks per call; larger
// geometries return -102).  d_chunks holds g.nchunks chunks back to back.  Returns a
// DevErr (synchronises `st`), -101 on a CUDA error.
constexpr int64_t NOALLOC_MAX_BYTES = int64_t(8) << 20;
constexpr int64_t NOALLOC_MAX_BLOCKS = 4096;
// Whether g fits those limits; the products are checked by division, so a huge geometry
// cannot wrap around and pass.
inline bool noalloc_fits(const Geom &g)
{
    if (g.nchunks == 0) return true;
    return g.chunk_nbytes <= NOALLOC_MAX_BYTES / g.nchunks && g.nblocks <= NOALLOC_MAX_BLOCKS / g.nchunks;
}
int decode_noalloc(const Geom &g, const uint8_t *d_chunks, int64_t chunks_bytes, void *out, int64_t ld, cudaStream_t st);

// Encode a dense row-major array into Blosc2 chunks.  On return *d_out holds the
// chunks back-to-back, h_off / h_len (host) their offsets and lengths.
// exact_lz4: streams byte-identical to liblz4 1.9.4 LZ4_compress_fast(acceleration 1); else
// the parallel-parse encoder (valid LZ4, different bytes).
// memcpy_only: compression level 0, every chunk stored memcpyed.
int encode_container(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode,
                     DevBuf *d_out, std::vector<int64_t> *h_off, std::vector<int32_t> *h_len,
                     cudaStream_t st, bool exact_lz4, bool memcpy_only = false);
// Asynchronous form: encode_launch enqueues the kernels (no host synchronisation; work
// buffers held in *w), encode_finish synchronises and reads the chunk table.
struct EncodeWork {
    DevBuf img, slots, es, ec, tot;
    bool exact_lz4 = true;            // liblz4-identical streams (see encode_container)
    bool memcpy_only = false;         // compression level 0: every chunk stored memcpyed (c-blosc2's clevel 0)
    bool img_ready = false;           // img already holds the byte-plane image (written by the product)
    EncChunk *ext_chunks = nullptr;   // optional caller-owned chunk table (device) instead of `ec`
    // optional caller-owned byte-plane image, LZ4 output slots and stream results (device)
    // instead of img / slots / es: slices of buffers shared by several containers
    uint8_t *ext_img = nullptr, *ext_slots = nullptr;
    EncStream *ext_es = nullptr;
    int64_t nchunks = 0;
};
int encode_launch(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode, DevBuf *d_out,
                  EncodeWork *w, cudaStream_t st);
// Encoding from an image the caller writes: encode_image_ok says whether a container of
// geometry g can take it (float64, shuffled, LZ4, block[1] and chunk[1] multiples of 4);
// encode_image_prepare allocates w->img for the caller to fill; encode_image_finish encodes it
// (no gather) and returns the chunk table as encode_container does.
bool encode_image_ok(const Geom &g, bool shuffle, bool memcpy_only);
int encode_image_prepare(const Geom &g, EncodeWork *w);
int encode_image_finish(const Geom &g, bool shuffle, int splitmode, DevBuf *d_out, std::vector<int64_t> *h_off,
                        std::vector<int32_t> *h_len, cudaStream_t st, bool exact_lz4, EncodeWork *w);

// encode_launch in stages, so that several containers can share one LZ4 launch:
// encode_gather (dense -> byte-plane image), encode_streams (LZ4 over ns streams of neblock
// bytes each; the streams of several containers when their images, slots and results lie
// back to back), encode_emit (chunk layout, offsets, payloads into *d_out).  The stream
// cursor `cursor` must be zero before encode_streams.
int encode_nstreams(const Geom &g, bool shuffle, int splitmode);
int encode_gather(const Geom &g, const void *in, int64_t ld, bool shuffle, int splitmode, EncodeWork *w, cudaStream_t st);
void encode_streams(const uint8_t *img, int64_t ns, int neblock, uint8_t *slots, EncStream *es,
                    unsigned long long *cursor, bool exact_lz4, cudaStream_t st);
int encode_emit(const Geom &g, bool shuffle, int splitmode, DevBuf *d_out, EncodeWork *w, cudaStream_t st);
int encode_finish(EncodeWork *w, std::vector<int64_t> *h_off, std::vector<int32_t> *h_len, cudaStream_t st);

// Grouped codec (batches): every stage of the decode (parse, LZ4, scatter) or of the encode
// (gather, LZ4, layout, chunk offsets, emit) is one launch over the blocks or chunks of all
// containers of the group; a unit finds its container by binary search of the group's start
// tables.  The containers share one item size (and, for the encode, one stream size).
struct CodecItem {                // one container of a group (device table entry)
    Geom g;
    const uint8_t *ch;            // decode: the container's chunks back to back
    int64_t ch_bytes;
    const int64_t *off;           // decode: chunk offsets and lengths
    const int32_t *len;
    BlockDesc *bd;                // decode work: descriptors, decoded-stream image
    StreamDesc *sd;
    uint8_t *scratch;
    uint8_t *dense;               // decode destination / encode source (row-major)
    int64_t ld;                   // its leading dimension in items
    int *cnt;                     // the container's status words ([1] decode error)
    uint8_t *img, *slots;         // encode: byte-plane image, LZ4 slots, stream results,
    EncStream *es;                // chunk table and output chunks (slices of shared buffers)
    EncChunk *ec;
    uint8_t *outbuf;
    int64_t out_bytes;            // total size of the output chunks (written by the encode)
};
struct CodecGroup {
    int n = 0, ts = 0;
    int nstreams = 0, neblock = 0;         // encode: the shared stream shape
    int64_t nbl = 0, nch = 0, nsf = 0;     // blocks, chunks, fast-scatter slices of all containers
    int64_t max_tpb = 0;                   // general-path tiles per block (largest over containers)
    bool shuffle = true, split = true;     // encode: byte shuffle, one stream per item byte
    std::vector<CodecItem> h;              // host copy of the table
    DevBuf items, starts;                  // device table; starts: blocks, slices, chunks ([n + 1] each)
    DevBuf bd, sd, scratch, rest, counters;   // decode work shared by the group; counters: [0] rest length, [2..] LZ4 cursor
    DevBuf img, slots, es, outsz;          // encode work shared by the group
    bool img_ready = false;                // encode: the producer writes img itself (no gather)
    DecodeQueue q;
};
// Decode group: a[i] is container i (all of item size ts), cnt[i] its 16-int status slot.
int decode_group_setup(const std::vector<DecodeArgs> &a, const std::vector<int *> &cnt, CodecGroup *grp, cudaStream_t st);
// Enqueues the decode of every container of the group (three kernel launches and the resets).
int decode_group_launch(CodecGroup *grp, cudaStream_t st);
// Encode group: container i from dense[i] (leading dimension ld[i]) into out[i] (allocated
// here), chunk table ec[i] (device, g[i].nchunks entries).  Returns 1 when the containers do
// not share one item size and one stream shape (the caller encodes them one by one).
int encode_group_setup(const std::vector<Geom> &g, const std::vector<const void *> &dense, const std::vector<int64_t> &ld,
                       const std::vector<EncChunk *> &ec, std::vector<DevBuf> *out, CodecGroup *grp, cudaStream_t st);
int encode_group_launch(CodecGroup *grp, bool exact_lz4, bool memcpy_only, cudaStream_t st);

// Dense products (row-major, leading dimensions in items).
// zs (optional): leave out the K ranges of zero-block pairs (zskip.cuh)
void gemm_f64_native(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda,
                     const double *B, int64_t ldb, double *C, int64_t ldc, cudaStream_t st,
                     const ZeroSkip *zs = nullptr);
void gemm_f32_native(int64_t M, int64_t N, int64_t K, const float *A, int64_t lda,
                     const float *B, int64_t ldb, float *C, int64_t ldc, cudaStream_t st);
void gemv_native(int dtype, int64_t M, int64_t K, const void *A, int64_t lda, const void *x,
                 void *y, cudaStream_t st);
// Grouped FP64 product: many independent C_p = A_p B_p in one persistent launch.
// tile_start is the first global tile of problem p for the chosen tile configuration
// (cfg & 3 the tile shape, 0: 128x128, 1: 64x128, 2: 128x64, 3: 64x64; cfg < 4: 16 k per
// pipeline stage, else 32); problems are listed in tile order.
constexpr int GEMM_F64_GROUPED_CONFIGS = 8;
struct GemmProblem {
    int M, N, K, tile_start;
    const double *A;
    const double *B;
    double *C;
    int64_t lda, ldb, ldc;
};
int gemm_f64_grouped_tiles(int cfg, int M, int N);
int gemm_f64_grouped_ctas(int cfg);          // resident CTAs of the persistent launch (SMs x occupancy)
void gemm_f64_grouped(int cfg, const GemmProblem *d_probs, int nprob, int total_tiles, int ctas, cudaStream_t st);

// The output of a float64 split product written straight into the byte-plane image of the
// output container's encoder (shuffled blocks, the layout the encoder's gather would write:
// block t = chunk * nblocks + block at t * blocksize, byte j of every item in plane j, padding
// items zero) instead of a dense matrix.  Needs itemsize 8, block[1] and chunk[1] multiples of 4.
struct CImage {
    Geom g;          // the output container's geometry (shape M x N)
    uint8_t *img;    // nchunks x nblocks x blocksize bytes
};

// Split-precision forms; return 0 on success, < 0 when unsupported on this device.
// With cimg, C and ldc are not used: the product goes into cimg->img.
int gemm_f64_ozaki(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda,
                   const double *B, int64_t ldb, double *C, int64_t ldc, int nterms, cudaStream_t st,
                   const ZeroSkip *zs = nullptr, const CImage *cimg = nullptr);
// Asynchronous form with caller-owned work buffers (no host synchronisation until finish).
// The B side (column scaling, residues, tensor map) is prepared once and can serve several
// row bands of A (gemm_f64_ozaki_rows), each with its own OzakiWork.
struct OzakiB {
    DevBuf rb, sb, pm, ps;
    int L = 0, nc = 0;
    int64_t K = 0, N = 0, Kp = 0;
    double gamma = 0;
    const double *B = nullptr;
    int64_t ldb = 0;
    alignas(64) unsigned char tmB[128];   // CUtensorMap of the residues of B
};
struct OzakiWork {
    DevBuf ra, rr, sa, err;
    const ZeroSkip *zs = nullptr;          // optional: leave out zero-block pairs (zskip.cuh)
    const CImage *cimg = nullptr;          // optional: write the product into an encoder image, not C
    alignas(64) unsigned char tmA[128];   // CUtensorMap of the residues of A (rows_prep -> rows_product)
    OzakiB b;                              // used by gemm_f64_ozaki_launch
};
int gemm_f64_ozaki_launch(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B,
                          int64_t ldb, double *C, int64_t ldc, int nterms, OzakiWork *w, cudaStream_t st);
int gemm_f64_ozaki_prepare_b(int64_t K, int64_t N, const double *B, int64_t ldb, int nterms, OzakiB *ob, cudaStream_t st);
// The same in two parts: setup (CRT constants on `st`, the B side's sizes) and the B kernels;
// and rows = rows_prep (scaling and residues of the A rows) + rows_product (INT8 GEMM, CRT).
// The CRT constants are read by every kernel after setup: other streams must wait for `st`.
int gemm_f64_ozaki_setup(int64_t K, int64_t N, int nterms, OzakiB *ob, cudaStream_t st);
int gemm_f64_ozaki_b_kernels(const double *B, int64_t ldb, OzakiB *ob, cudaStream_t st);
int gemm_f64_ozaki_rows_prep(int64_t M, const double *A, int64_t lda, const OzakiB &ob, OzakiWork *w, cudaStream_t st);
int gemm_f64_ozaki_rows_product(int64_t M, const double *A, int64_t lda, const OzakiB &ob, double *C, int64_t ldc,
                                OzakiWork *w, cudaStream_t st);
int gemm_f64_ozaki_rows(int64_t M, const double *A, int64_t lda, const OzakiB &ob, double *C, int64_t ldc,
                        OzakiWork *w, cudaStream_t st);
int gemm_f64_ozaki_finish(OzakiWork *w, cudaStream_t st);
// Grouped split-precision form: many independent products in one pipeline of seven kernel
// launches over a table of products (split.cu).  setup allocates every buffer and writes the
// tables (synchronously; call it outside stream capture); launch enqueues the kernels on `st`
// (capturable); finish reads the status word.
struct OzGroupItem {
    int64_t M, N, K;
    const double *A;
    const double *B;
    double *C;
    int64_t lda, ldb, ldc;
    // optional (every item or none): C's encoder image and geometry, written instead of C
    // (the CImage layout)
    uint8_t *cimg = nullptr;
    Geom gc = {};
};
struct OzGroupWork {
    DevBuf ra, rb, rr, sa, sb, pm, ps, probs, maps, err;
    int L = 0, nc = 0, np = 0;
    double gamma = 0;
    int64_t rows = 0, cols = 0, tasks_r = 0, tiles_c = 0, items = 0, crt = 0;
    bool img = false;                // the reconstruction writes the items' encoder images
    int64_t units = 0;               // its work units (block slices of every image)
    int slice = 0;                   // rows per work unit
};
int gemm_f64_ozaki_grouped_setup(const std::vector<OzGroupItem> &items, int nterms, OzGroupWork *w, cudaStream_t st);
int gemm_f64_ozaki_grouped_launch(OzGroupWork *w, cudaStream_t st);
int gemm_f64_ozaki_grouped_finish(OzGroupWork *w, cudaStream_t st);
// sqrt(sum_i ||X_i - Y_i||_F^2 / sum_i ||Y_i||_F^2) over M_i x N_i float64 matrices (row pitch
// ld_i); synchronises st; < 0 on a CUDA error.
struct DiffItem {
    const double *X;
    const double *Y;
    int64_t M, N, ld;
};
double normwise_diff_grouped(const std::vector<DiffItem> &items, cudaStream_t st);

// float32 split form: each operand split into bf16 words, `products` BF16 tensor-core
// products (3: two words; 6: three words; 0: 6) summed in FP32 segments.
int gemm_f32_bf16_split(int64_t M, int64_t N, int64_t K, const float *A, int64_t lda,
                        const float *B, int64_t ldb, float *C, int64_t ldc, int products, cudaStream_t st);

// Zero-block rule of the block-pair products (zero.cu, zskip.cuh).
void zero_grid(const Geom &g, const uint8_t *zf, bool use_chunk, uint8_t *grid, cudaStream_t st);
void block_nonfinite(int itemsize, int64_t rows, int64_t cols, const void *x, int64_t ld, int64_t r_chunk,
                     int64_t r_block, int64_t r_bg, int64_t c_chunk, int64_t c_block, int64_t c_bg, int64_t CB,
                     uint8_t *flags, cudaStream_t st);
void zero_fix(int itemsize, int64_t M, int64_t N, int64_t K, const void *A, int64_t lda, const void *B, int64_t ldb,
              void *C, int64_t ldc, const ZeroSkip &z, const uint8_t *nfa, const uint8_t *nfb, cudaStream_t st);

void fill_arange(int dtype, int64_t M, int64_t N, int64_t ld, double start, double step, void *out,
                 cudaStream_t st);
void transpose_dense(int itemsize, int64_t rows, int64_t cols, const void *in, int64_t ldin, void *out,
                     int64_t ldout, cudaStream_t st);

}  // namespace iab
