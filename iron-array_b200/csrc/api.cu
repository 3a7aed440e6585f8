// Host runtime behind include/iarray_b200.h: contexts, GPU-resident containers,
// persistence, and the matmul entry points of ironArray (src/linalg/matmul.c,
// src/linalg/matmul/gemm.c, gemv.c, src/linalg/iarray_gemm.c, iarray_gemm_a.c,
// iarray_gemm_b.c, iarray_gemv.c).
//
// A container keeps its Blosc2 chunks in device memory, back to back, with host-side
// offsets.  A product decodes each operand once into a dense row-major device array
// (the reference decodes every A block N_blocks x N_chunks times), runs one product
// kernel over the whole matrices, and re-encodes the result into `storage`'s
// partition.  Calls are synchronous on one internal CUDA stream per context.
#include <cuda_runtime.h>
#include <dirent.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/iarray_b200.h"
#include "common.cuh"
#include "expr.h"
#include "frame.h"
#include "zskip.cuh"

using iab::DevBuf;
using iab::Geom;

// ============================================================================ pool + geometry
namespace iab {

std::atomic<uint64_t> g_launches{0};

DevicePool &DevicePool::get(int device)
{
    static std::mutex mu;
    static std::map<int, DevicePool *> pools;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return *it->second;
    DevicePool *p = new DevicePool();
    pools[device] = p;
    return *p;
}

static size_t size_class(size_t n)
{
    if (n <= (1u << 20)) {
        size_t s = 256;
        while (s < n) s <<= 1;
        return s;
    }
    return round_up((int64_t)n, (int64_t)2 << 20);
}

void *DevicePool::alloc(size_t bytes)
{
    const size_t sc = size_class(std::max<size_t>(bytes, 1));
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.lower_bound(sc);
        if (it != free_.end() && it->first <= sc + sc / 4) {
            void *p = it->second;
            used_[p] = it->first;
            free_.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaMalloc(&p, sc) != cudaSuccess) {
        cudaGetLastError();
        trim();
        if (cudaMalloc(&p, sc) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    }
    std::lock_guard<std::mutex> lk(mu_);
    used_[p] = sc;
    return p;
}

void DevicePool::release(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = used_.find(p);
    if (it == used_.end()) return;
    free_.emplace(it->second, p);
    used_.erase(it);
}

void DevicePool::trim()
{
    std::lock_guard<std::mutex> lk(mu_);
    cudaDeviceSynchronize();
    for (auto &kv : free_) cudaFree(kv.second);
    free_.clear();
}

bool DevBuf::allocate(size_t bytes, int device)
{
    reset();
    dev = device;
    p = DevicePool::get(device).alloc(bytes);
    n = p ? bytes : 0;
    return p != nullptr;
}

void DevBuf::reset()
{
    if (p) DevicePool::get(dev).release(p);
    p = nullptr;
    n = 0;
}

bool make_geom(int ndim, const int64_t *shape, const int64_t *chunk, const int64_t *block, int itemsize, Geom *g)
{
    if (ndim < 1 || ndim > 2) return false;
    memset(g, 0, sizeof(*g));
    g->itemsize = itemsize;
    g->ndim = ndim;
    // every extent is held below 2^48 and every product below is checked by division
    // first, so no size computed here can wrap around
    constexpr int64_t kMaxExtent = int64_t(1) << 48;
    for (int d = 0; d < 2; d++) {
        const int s = d - (2 - ndim);   // 1-D arrays are 1 x n
        g->shape[d] = s < 0 ? 1 : shape[s];
        g->chunk[d] = s < 0 ? 1 : chunk[s];
        g->block[d] = s < 0 ? 1 : block[s];
        if (g->shape[d] < 0 || g->chunk[d] <= 0 || g->block[d] <= 0) return false;
        if (g->shape[d] > kMaxExtent || g->chunk[d] > kMaxExtent) return false;
        if (g->block[d] > g->chunk[d]) return false;
        g->extc[d] = round_up(g->chunk[d], g->block[d]);
        g->cgrid[d] = g->shape[d] == 0 ? 0 : ceil_div(g->shape[d], g->chunk[d]);
        g->bgrid[d] = g->extc[d] / g->block[d];
    }
    // Blosc2 chunks are below 2 GiB: extc0 * extc1 * itemsize < 2^31 - 64
    const int64_t kChunkMax = (int64_t)INT32_MAX - 64;
    if (g->extc[0] > kChunkMax / g->extc[1] / itemsize) return false;
    if (g->cgrid[1] && g->cgrid[0] > INT64_MAX / 2 / g->cgrid[1]) return false;
    g->nchunks = g->cgrid[0] * g->cgrid[1];
    g->nblocks = g->bgrid[0] * g->bgrid[1];
    g->blockn = g->block[0] * g->block[1];
    g->blocksize = g->blockn * itemsize;
    g->chunk_nbytes = g->extc[0] * g->extc[1] * itemsize;
    if (g->chunk_nbytes > kChunkMax) return false;
    return true;
}

}  // namespace iab

// ============================================================================ objects
struct ChunkStore {
    int device = 0;
    DevBuf buf;                    // chunk bytes, back to back
    DevBuf d_off, d_len;           // device copies of off / len
    std::vector<int64_t> off;      // byte offset of each chunk in buf
    std::vector<int32_t> len;      // cbytes of each chunk
    int64_t cbytes = 0;
    bool upload_index()
    {
        const size_t n = off.size();
        if (!d_off.allocate(std::max<size_t>(n, 1) * 8, device) || !d_len.allocate(std::max<size_t>(n, 1) * 4, device))
            return false;
        if (n) {
            cudaMemcpy(d_off.p, off.data(), n * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(d_len.p, len.data(), n * 4, cudaMemcpyHostToDevice);
        }
        cbytes = 0;
        for (int32_t l : len) cbytes += l;
        return true;
    }
};

struct iarray_context_s {
    iarray_config_t cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    int form = IARRAY_B200_FORM_NATIVE;
    int split_terms = 0;
    int split_products_f32 = 0;              // float32 split form: 3 or 6 BF16 products (0: 6)
    int encoder = IARRAY_B200_ENCODER_LIBLZ4;
    double timings[5] = {0, 0, 0, 0, 0};
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaStream_t stream2 = nullptr;          // second stream (operand decode of the pipelined call)
    cudaEvent_t fork = nullptr, join = nullptr;
    // iarray_b200_opt_gemm_cframes: copy streams, the encode stream, the chunk-table copy
    // stream and pinned staging for chunk tables
    cudaStream_t up = nullptr, down = nullptr, enc = nullptr, tabs = nullptr;
    void *pin = nullptr;
    size_t pin_n = 0;
};

struct iarray_container_s {
    iarray_dtshape_t dtshape;      // logical shape (a transposed view has it reversed)
    iarray_storage_t storage;      // partition of the stored chunks
    std::string urlpath;
    Geom geom;                     // geometry of the stored chunks
    std::shared_ptr<ChunkStore> store;
    bool transposed = false;
    bool view = false;
    bool shuffle = true;
    int splitmode = IARRAY_AUTO_SPLIT;
    int clevel = 5;
};

// ============================================================================ errors
static ina_rc_t rc_err(uint32_t msg) { return INA_RC_ERROR_BIT | (ina_rc_t)msg; }

static bool g_initialized = false;
static int g_device = -1;

INA_API(const char *) iarray_err_strerror(ina_rc_t error)
{
    if (!INA_FAILED(error)) return "Success";
    switch (INA_RC_MSG(error)) {
    case IARRAY_ERR_INVALID_DTYPE: return "Invalid dtype";
    case IARRAY_ERR_INVALID_SHAPE: return "Invalid shape";
    case IARRAY_ERR_INVALID_CHUNKSHAPE: return "Invalid chunkshape";
    case IARRAY_ERR_INVALID_BLOCKSHAPE: return "Invalid blockshape";
    case IARRAY_ERR_INVALID_NDIM: return "Invalid ndim";
    case IARRAY_ERR_INVALID_STORAGE: return "Invalid storage";
    case IARRAY_ERR_TOO_SMALL_BUFFER: return "Buffer too small";
    case IARRAY_ERR_BLOSC_FAILED: return "Blosc chunk failed to encode or decode";
    case IARRAY_ERR_ASSERTION_FAILED: return "Assertion failed";
    case IARRAY_ERR_PERSISTENCY_FAILED: return "Persistence failed";
    case IARRAY_ERR_GPU_FAILED: return "GPU failed or unavailable";
    case IARRAY_ERR_GPU_OUT_OF_MEMORY: return "GPU out of memory";
    case IARRAY_ERR_NOT_SUPPORTED: return "Not supported";
    case INA_ERR_INVALID_ARGUMENT: return "Invalid argument";
    case INA_ERR_NOT_INITIALIZED: return "Library not initialized";
    case IARRAY_ERR_NOALLOC_TOO_LARGE: return "Geometry exceeds the fixed scratch of iarray_b200_decode_noalloc";
    default: return "Error";
    }
}

#define CHECK_ARG(x) do { if (!(x)) return rc_err(INA_ERR_INVALID_ARGUMENT); } while (0)

static ina_rc_t cuda_rc(cudaError_t e)
{
    if (e == cudaSuccess) return INA_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return rc_err(IARRAY_ERR_GPU_FAILED);
}

// ============================================================================ runtime
INA_API(ina_rc_t) iarray_init(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    int dev = 0;
    cudaGetDevice(&dev);
    g_device = dev;
    g_initialized = true;
    return INA_SUCCESS;
}

INA_API(void) iarray_destroy(void)
{
    if (g_initialized && g_device >= 0) iab::DevicePool::get(g_device).trim();
    g_initialized = false;
}

INA_API(ina_rc_t) iarray_context_new(iarray_config_t *cfg, iarray_context_t **ctx)
{
    CHECK_ARG(cfg && ctx);
    if (!g_initialized) return rc_err(INA_ERR_NOT_INITIALIZED);
    if (cfg->compression_codec != IARRAY_COMPRESSION_LZ4) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    if (cfg->filter_flags & ~IARRAY_COMP_SHUFFLE) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    // level 0 stores chunks memcpyed, as c-blosc2 does (src/iarray.c:391-439 passes it on)
    if (cfg->compression_level < 0 || cfg->compression_level > 9) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    iarray_context_t *c = new iarray_context_t();
    c->cfg = *cfg;
    c->device = g_device;
    cudaSetDevice(c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    for (auto &e : c->ev) cudaEventCreate(&e);
    cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming);
    *ctx = c;
    return INA_SUCCESS;
}

INA_API(void) iarray_context_free(iarray_context_t **ctx)
{
    if (!ctx || !*ctx) return;
    iarray_context_t *c = *ctx;
    if (c->stream) { cudaStreamSynchronize(c->stream); cudaStreamDestroy(c->stream); }
    if (c->stream2) { cudaStreamSynchronize(c->stream2); cudaStreamDestroy(c->stream2); }
    if (c->up) { cudaStreamSynchronize(c->up); cudaStreamDestroy(c->up); }
    if (c->down) { cudaStreamSynchronize(c->down); cudaStreamDestroy(c->down); }
    if (c->enc) { cudaStreamSynchronize(c->enc); cudaStreamDestroy(c->enc); }
    if (c->tabs) { cudaStreamSynchronize(c->tabs); cudaStreamDestroy(c->tabs); }
    if (c->pin) cudaFreeHost(c->pin);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    for (auto &e : c->ev) if (e) cudaEventDestroy(e);
    delete c;
    *ctx = nullptr;
}

INA_API(ina_rc_t) iarray_b200_set_encoder(iarray_context_t *ctx, iarray_b200_encoder_t encoder)
{
    CHECK_ARG(ctx && (encoder == IARRAY_B200_ENCODER_PARALLEL || encoder == IARRAY_B200_ENCODER_LIBLZ4));
    ctx->encoder = encoder;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_set_form(iarray_context_t *ctx, iarray_b200_form_t form)
{
    CHECK_ARG(ctx && (form == IARRAY_B200_FORM_NATIVE || form == IARRAY_B200_FORM_SPLIT));
    ctx->form = form;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_set_split_terms(iarray_context_t *ctx, int nterms)
{
    CHECK_ARG(ctx && nterms >= 0 && nterms <= 32);
    ctx->split_terms = nterms;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_set_split_products_f32(iarray_context_t *ctx, int nproducts)
{
    CHECK_ARG(ctx && (nproducts == 0 || nproducts == 3 || nproducts == 6));
    ctx->split_products_f32 = nproducts;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_last_timings(iarray_context_t *ctx, double *ms5)
{
    CHECK_ARG(ctx && ms5);
    for (int i = 0; i < 5; i++) ms5[i] = ctx->timings[i];
    return INA_SUCCESS;
}

INA_API(uint64_t) iarray_b200_kernel_launches(void) { return iab::g_launches.load(); }

INA_API(ina_rc_t) iarray_b200_get_stream(iarray_context_t *ctx, void **stream)
{
    CHECK_ARG(ctx && stream);
    *stream = (void *)ctx->stream;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_synchronize(iarray_context_t *ctx)
{
    CHECK_ARG(ctx);
    return cuda_rc(cudaStreamSynchronize(ctx->stream));
}

// ============================================================================ containers
static int dtype_size(int dtype)
{
    switch (dtype) {
    case IARRAY_DATA_TYPE_DOUBLE: case IARRAY_DATA_TYPE_INT64: case IARRAY_DATA_TYPE_UINT64: return 8;
    case IARRAY_DATA_TYPE_FLOAT: case IARRAY_DATA_TYPE_INT32: case IARRAY_DATA_TYPE_UINT32: return 4;
    case IARRAY_DATA_TYPE_INT16: case IARRAY_DATA_TYPE_UINT16: return 2;
    case IARRAY_DATA_TYPE_INT8: case IARRAY_DATA_TYPE_UINT8: case IARRAY_DATA_TYPE_BOOL: return 1;
    default: return 0;
    }
}

static ina_rc_t new_container(iarray_context_t *ctx, iarray_dtshape_t *dtshape, iarray_storage_t *storage,
                              iarray_container_t **out)
{
    CHECK_ARG(ctx && dtshape && storage && out);
    const int isz = dtype_size(dtshape->dtype);
    if (!isz) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (dtshape->ndim < 1 || dtshape->ndim > 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    for (int i = 0; i < dtshape->ndim; i++) {
        if (dtshape->shape[i] < 0) return rc_err(IARRAY_ERR_INVALID_SHAPE);
        if (storage->chunkshape[i] <= 0) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
        if (storage->blockshape[i] <= 0 || storage->blockshape[i] > storage->chunkshape[i])
            return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    }
    Geom g;
    if (!iab::make_geom(dtshape->ndim, dtshape->shape, storage->chunkshape, storage->blockshape, isz, &g))
        return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    iarray_container_t *c = new iarray_container_t();
    c->dtshape = *dtshape;
    c->dtshape.dtype_size = isz;
    c->storage = *storage;
    c->storage.urlpath = nullptr;
    if (storage->urlpath) c->urlpath = storage->urlpath;
    c->geom = g;
    c->store = std::make_shared<ChunkStore>();
    c->store->device = ctx->device;
    c->shuffle = (ctx->cfg.filter_flags & IARRAY_COMP_SHUFFLE) != 0;
    c->splitmode = ctx->cfg.splitmode;
    c->clevel = ctx->cfg.compression_level;
    *out = c;
    return INA_SUCCESS;
}

static ina_rc_t save_if_urlpath(iarray_context_t *ctx, iarray_container_t *c);

// Fill a container with Blosc2 special-zero chunks (header only).
static ina_rc_t fill_zero_chunks(iarray_container_t *c)
{
    const Geom &g = c->geom;
    std::vector<uint8_t> h((size_t)g.nchunks * 32, 0);
    for (int64_t k = 0; k < g.nchunks; k++) {
        uint8_t *p = &h[k * 32];
        p[0] = 5; p[1] = 1; p[2] = 0x05 | (1 << 5); p[3] = (uint8_t)g.itemsize;
        const int32_t nb = (int32_t)g.chunk_nbytes, bs = (int32_t)g.blocksize, cb = 32;
        memcpy(p + 4, &nb, 4); memcpy(p + 8, &bs, 4); memcpy(p + 12, &cb, 4);
        p[21] = c->shuffle ? 1 : 0;
        p[22] = 1;
        p[31] = 1 << 4;   // special value: zeros
    }
    ChunkStore &s = *c->store;
    if (!s.buf.allocate(std::max<size_t>(h.size(), 1), s.device)) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (!h.empty() && cudaMemcpy(s.buf.p, h.data(), h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return rc_err(IARRAY_ERR_GPU_FAILED);
    s.off.resize((size_t)g.nchunks);
    s.len.assign((size_t)g.nchunks, 32);
    for (int64_t k = 0; k < g.nchunks; k++) s.off[k] = k * 32;
    if (!s.upload_index()) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_empty(iarray_context_t *ctx, iarray_dtshape_t *dtshape, iarray_storage_t *storage,
                               iarray_container_t **container)
{
    ina_rc_t rc = new_container(ctx, dtshape, storage, container);
    if (INA_FAILED(rc)) return rc;
    rc = fill_zero_chunks(*container);
    if (INA_FAILED(rc)) { iarray_container_free(ctx, container); return rc; }
    return save_if_urlpath(ctx, *container);
}

INA_API(ina_rc_t) iarray_zeros(iarray_context_t *ctx, iarray_dtshape_t *dtshape, iarray_storage_t *storage,
                               iarray_container_t **container)
{
    return iarray_empty(ctx, dtshape, storage, container);
}

INA_API(void) iarray_container_free(iarray_context_t *ctx, iarray_container_t **container)
{
    (void)ctx;
    if (!container || !*container) return;
    delete *container;
    *container = nullptr;
}

// Encode a dense device array (row-major, leading dimension ld) into c's store.
static ina_rc_t encode_into(iarray_context_t *ctx, iarray_container_t *c, const void *dense, int64_t ld)
{
    ChunkStore &s = *c->store;
    DevBuf out;
    std::vector<int64_t> off;
    std::vector<int32_t> len;
    int r = iab::encode_container(c->geom, dense, ld, c->shuffle, c->splitmode, &out, &off, &len, ctx->stream,
                                  ctx->encoder == IARRAY_B200_ENCODER_LIBLZ4, c->clevel == 0);
    if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (r != 0) return rc_err(IARRAY_ERR_GPU_FAILED);
    s.buf = std::move(out);
    s.off = std::move(off);
    s.len = std::move(len);
    if (!s.upload_index()) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return INA_SUCCESS;
}

// encode_into for an image the product wrote (iab::encode_image_prepare).
static ina_rc_t encode_into_image(iarray_context_t *ctx, iarray_container_t *c, iab::EncodeWork *w)
{
    ChunkStore &s = *c->store;
    DevBuf out;
    std::vector<int64_t> off;
    std::vector<int32_t> len;
    int r = iab::encode_image_finish(c->geom, c->shuffle, c->splitmode, &out, &off, &len, ctx->stream,
                                     ctx->encoder == IARRAY_B200_ENCODER_LIBLZ4, w);
    if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (r != 0) return rc_err(IARRAY_ERR_GPU_FAILED);
    s.buf = std::move(out);
    s.off = std::move(off);
    s.len = std::move(len);
    if (!s.upload_index()) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return INA_SUCCESS;
}

// A decoder's status word: malformed chunk data is a codec failure; a bounded wait on an
// asynchronous copy that gave up (DE_WAIT) is a GPU failure, not bad data.
static ina_rc_t status_rc(int status)
{
    if (status == 0) return INA_SUCCESS;
    return rc_err(status == iab::DE_WAIT ? IARRAY_ERR_GPU_FAILED : IARRAY_ERR_BLOSC_FAILED);
}

static ina_rc_t decode_rc(int r)
{
    if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (r < 0) return rc_err(IARRAY_ERR_GPU_FAILED);
    return status_rc(r);
}

// Decode the stored chunks of c (its base geometry, not the view) into dense memory.
static ina_rc_t decode_store(iarray_context_t *ctx, const iarray_container_t *c, void *dense, int64_t ld)
{
    const Geom &g = c->geom;
    if (g.nchunks == 0) return INA_SUCCESS;
    if (ld != g.shape[1] || g.nchunks * g.nblocks == 0) {
        // callers of iarray_b200_decode_to_device get defined padding columns
        cudaMemsetAsync(dense, 0, (size_t)(g.shape[0] * ld * g.itemsize), ctx->stream);
    }
    const ChunkStore &s = *c->store;
    const int r = iab::decode_container(g, s.buf.as<uint8_t>(), (int64_t)s.buf.n, s.d_off.as<int64_t>(), s.d_len.as<int32_t>(), dense, ld,
                                        ctx->stream);
    return decode_rc(r);
}

// Decode two stored (non-view) containers on the context's stream with one LZ4 launch for
// the streams of both (one job queue), then each container's scatter; returns after both
// finished.
// zf / nzero (optional): each container's per (chunk, block) zero flags and their count.
static ina_rc_t decode_pair(iarray_context_t *ctx, const iarray_container_t *a, void *da, int64_t lda,
                            const iarray_container_t *b, void *db, int64_t ldb, DevBuf *zf = nullptr,
                            int *nzero = nullptr)
{
    // the padding columns past each row are left as they are: no product reads them
    const iarray_container_t *x[2] = {a, b};
    const iab::DecodeArgs args[2] = {
        {a->geom, a->store->buf.as<uint8_t>(), (int64_t)a->store->buf.n, a->store->d_off.as<int64_t>(),
         a->store->d_len.as<int32_t>(), da, lda},
        {b->geom, b->store->buf.as<uint8_t>(), (int64_t)b->store->buf.n, b->store->d_off.as<int64_t>(),
         b->store->d_len.as<int32_t>(), db, ldb}};
    iab::DecodeQueue q;
    iab::DecodeWork w[2];
    int r = iab::decode_queue_init(&q, iab::decode_max_jobs(a->geom) + iab::decode_max_jobs(b->geom), ctx->stream);
    for (int k = 0; k < 2 && !r; k++)
        if (x[k]->geom.nchunks) r = iab::decode_parse(args[k], &q, &w[k], ctx->stream);
    if (!r) r = iab::decode_lz4(&q, ctx->stream);
    for (int k = 0; k < 2 && !r; k++)
        if (x[k]->geom.nchunks) r = iab::decode_scatter(args[k], &w[k], ctx->stream);
    for (int k = 0; k < 2 && !r; k++)
        if (x[k]->geom.nchunks) r = iab::decode_finish(&w[k], ctx->stream);
    if (r) cudaStreamSynchronize(ctx->stream);     // the work buffers go back to the pool idle
    for (int k = 0; k < 2 && !r; k++) {
        if (zf) zf[k] = std::move(w[k].zf);
        if (nzero) nzero[k] = x[k]->geom.nchunks ? w[k].nzero : 0;
    }
    return decode_rc(r);
}

static int64_t rows_of(const iarray_dtshape_t &d) { return d.ndim == 2 ? d.shape[0] : 1; }
static int64_t cols_of(const iarray_dtshape_t &d) { return d.ndim == 2 ? d.shape[1] : d.shape[0]; }
static int64_t pad_ld(int64_t cols) { return std::max<int64_t>(iab::round_up(cols, 32), 32); }

// Decode a container (honouring a transposed view) into dense memory, logical
// rows x cols with leading dimension ld.
static ina_rc_t decode_logical(iarray_context_t *ctx, const iarray_container_t *c, void *dense, int64_t ld)
{
    if (!c->transposed) return decode_store(ctx, c, dense, ld);
    const Geom &g = c->geom;
    DevBuf tmp;
    const int64_t bld = pad_ld(g.shape[1]);
    if (!tmp.allocate((size_t)(std::max<int64_t>(g.shape[0], 1) * bld * g.itemsize), ctx->device))
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    ina_rc_t rc = decode_store(ctx, c, tmp.p, bld);
    if (INA_FAILED(rc)) return rc;
    if (ld != g.shape[0]) cudaMemsetAsync(dense, 0, (size_t)(g.shape[1] * ld * g.itemsize), ctx->stream);
    iab::transpose_dense(g.itemsize, g.shape[0], g.shape[1], tmp.p, bld, dense, ld, ctx->stream);
    return cuda_rc(cudaStreamSynchronize(ctx->stream));
}

INA_API(ina_rc_t) iarray_from_buffer(iarray_context_t *ctx, iarray_dtshape_t *dtshape, void *buffer, int64_t buflen,
                                     iarray_storage_t *storage, iarray_container_t **container)
{
    CHECK_ARG(buffer);
    ina_rc_t rc = new_container(ctx, dtshape, storage, container);
    if (INA_FAILED(rc)) return rc;
    iarray_container_t *c = *container;
    const int64_t n = rows_of(c->dtshape) * cols_of(c->dtshape);
    if (buflen < n * c->geom.itemsize) { iarray_container_free(ctx, container); return rc_err(IARRAY_ERR_TOO_SMALL_BUFFER); }
    DevBuf dense;
    if (!dense.allocate((size_t)std::max<int64_t>(n * c->geom.itemsize, 1), ctx->device)) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    }
    cudaMemcpyAsync(dense.p, buffer, (size_t)(n * c->geom.itemsize), cudaMemcpyHostToDevice, ctx->stream);
    if (c->geom.nchunks == 0) rc = fill_zero_chunks(c);
    else rc = encode_into(ctx, c, dense.p, cols_of(c->dtshape));
    if (INA_FAILED(rc)) { iarray_container_free(ctx, container); return rc; }
    return save_if_urlpath(ctx, c);
}

INA_API(ina_rc_t) iarray_to_buffer(iarray_context_t *ctx, iarray_container_t *container, void *buffer, int64_t buflen)
{
    CHECK_ARG(ctx && container && buffer);
    const iarray_container_t *c = container;
    const int64_t rows = rows_of(c->dtshape), cols = cols_of(c->dtshape);
    const int64_t nb = rows * cols * c->geom.itemsize;
    if (buflen < nb) return rc_err(IARRAY_ERR_TOO_SMALL_BUFFER);
    if (nb == 0) return INA_SUCCESS;
    DevBuf dense;
    if (!dense.allocate((size_t)nb, ctx->device)) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    ina_rc_t rc = decode_logical(ctx, c, dense.p, cols);
    if (INA_FAILED(rc)) return rc;
    cudaMemcpyAsync(buffer, dense.p, (size_t)nb, cudaMemcpyDeviceToHost, ctx->stream);
    return cuda_rc(cudaStreamSynchronize(ctx->stream));
}

INA_API(ina_rc_t) iarray_arange(iarray_context_t *ctx, iarray_dtshape_t *dtshape, double start, double step,
                                iarray_storage_t *storage, iarray_container_t **container)
{
    ina_rc_t rc = new_container(ctx, dtshape, storage, container);
    if (INA_FAILED(rc)) return rc;
    iarray_container_t *c = *container;
    if (c->dtshape.dtype != IARRAY_DATA_TYPE_DOUBLE && c->dtshape.dtype != IARRAY_DATA_TYPE_FLOAT) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_INVALID_DTYPE);
    }
    const int64_t rows = rows_of(c->dtshape), cols = cols_of(c->dtshape);
    DevBuf dense;
    if (!dense.allocate((size_t)std::max<int64_t>(rows * cols * c->geom.itemsize, 1), ctx->device)) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    }
    iab::fill_arange(c->dtshape.dtype == IARRAY_DATA_TYPE_DOUBLE ? 0 : 1, rows, cols, cols, start, step, dense.p,
                     ctx->stream);
    rc = c->geom.nchunks ? encode_into(ctx, c, dense.p, cols) : fill_zero_chunks(c);
    if (INA_FAILED(rc)) { iarray_container_free(ctx, container); return rc; }
    return save_if_urlpath(ctx, c);
}

INA_API(ina_rc_t) iarray_linspace(iarray_context_t *ctx, iarray_dtshape_t *dtshape, double start, double stop,
                                  iarray_storage_t *storage, iarray_container_t **container)
{
    CHECK_ARG(dtshape);
    int64_t n = 1;
    for (int i = 0; i < dtshape->ndim; i++) n *= dtshape->shape[i];
    const double step = n > 1 ? (stop - start) / (double)(n - 1) : 0.0;
    return iarray_arange(ctx, dtshape, start, step, storage, container);
}

INA_API(ina_rc_t) iarray_container_info(iarray_container_t *container, int64_t *nbytes, int64_t *cbytes)
{
    CHECK_ARG(container && nbytes && cbytes);
    *nbytes = container->geom.nchunks * container->geom.chunk_nbytes;
    *cbytes = container->store->cbytes;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_get_dtshape(iarray_context_t *ctx, iarray_container_t *c, iarray_dtshape_t *dtshape)
{
    (void)ctx;
    CHECK_ARG(c && dtshape);
    *dtshape = c->dtshape;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_get_storage(iarray_context_t *ctx, iarray_container_t *c, iarray_storage_t *storage)
{
    (void)ctx;
    CHECK_ARG(c && storage);
    *storage = c->storage;
    storage->urlpath = c->urlpath.empty() ? nullptr : (char *)c->urlpath.c_str();
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_is_view(iarray_context_t *ctx, iarray_container_t *c, bool *view)
{
    (void)ctx;
    CHECK_ARG(c && view);
    *view = c->view;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_nchunks(iarray_container_t *c, int64_t *nchunks)
{
    CHECK_ARG(c && nchunks);
    *nchunks = c->geom.nchunks;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_get_chunk(iarray_context_t *ctx, iarray_container_t *c, int64_t nchunk, uint8_t *buf,
                                        int64_t *len)
{
    CHECK_ARG(ctx && c && len && nchunk >= 0 && nchunk < c->geom.nchunks);
    const ChunkStore &s = *c->store;
    const int32_t l = s.len[nchunk];
    if (!buf) { *len = l; return INA_SUCCESS; }
    if (*len < l) return rc_err(IARRAY_ERR_TOO_SMALL_BUFFER);
    *len = l;
    cudaMemcpyAsync(buf, s.buf.as<uint8_t>() + s.off[nchunk], (size_t)l, cudaMemcpyDeviceToHost, ctx->stream);
    return cuda_rc(cudaStreamSynchronize(ctx->stream));
}

static ina_rc_t upload_chunks(iarray_context_t *ctx, iarray_container_t *c, const uint8_t *const *chunks,
                              const int64_t *lens)
{
    const Geom &g = c->geom;
    ChunkStore &s = *c->store;
    int64_t total = 0;
    for (int64_t k = 0; k < g.nchunks; k++) {
        if (lens[k] < 32 || lens[k] > g.chunk_nbytes + 64) return rc_err(IARRAY_ERR_BLOSC_FAILED);
        total += lens[k];
    }
    if (!s.buf.allocate((size_t)std::max<int64_t>(total, 1), s.device)) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    // one staging copy keeps the H2D transfer to a single large cudaMemcpyAsync
    std::vector<uint8_t> stage((size_t)total);
    s.off.resize((size_t)g.nchunks);
    s.len.resize((size_t)g.nchunks);
    int64_t acc = 0;
    for (int64_t k = 0; k < g.nchunks; k++) {
        memcpy(stage.data() + acc, chunks[k], (size_t)lens[k]);
        s.off[k] = acc;
        s.len[k] = (int32_t)lens[k];
        acc += lens[k];
    }
    if (total) cudaMemcpyAsync(s.buf.p, stage.data(), (size_t)total, cudaMemcpyHostToDevice, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    if (!s.upload_index()) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_from_chunks(iarray_context_t *ctx, iarray_dtshape_t *dtshape, iarray_storage_t *storage,
                                          int64_t nchunks, const uint8_t *const *chunks, const int64_t *chunk_lens,
                                          iarray_container_t **container)
{
    CHECK_ARG(chunks && chunk_lens);
    ina_rc_t rc = new_container(ctx, dtshape, storage, container);
    if (INA_FAILED(rc)) return rc;
    if (nchunks != (*container)->geom.nchunks) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_INVALID_STORAGE);
    }
    rc = upload_chunks(ctx, *container, chunks, chunk_lens);
    if (INA_FAILED(rc)) iarray_container_free(ctx, container);
    return rc;
}

INA_API(ina_rc_t) iarray_b200_decode_to_device(iarray_context_t *ctx, iarray_container_t *c, void *dptr, int64_t ld)
{
    CHECK_ARG(ctx && c && dptr && ld >= cols_of(c->dtshape));
    return decode_logical(ctx, c, dptr, ld);
}

INA_API(ina_rc_t) iarray_b200_decode_noalloc(int8_t ndim, const int64_t *shape, const int64_t *chunkshape,
                                             const int64_t *blockshape, int32_t itemsize, const void *chunks,
                                             int64_t chunks_len, void *dptr, int64_t ld, void *stream)
{
    CHECK_ARG(shape && chunkshape && blockshape && chunks && dptr && chunks_len >= 0);
    CHECK_ARG(itemsize == 1 || itemsize == 2 || itemsize == 4 || itemsize == 8);
    Geom g;
    if (!iab::make_geom(ndim, shape, chunkshape, blockshape, itemsize, &g)) return rc_err(INA_ERR_INVALID_ARGUMENT);
    CHECK_ARG(ld >= g.shape[1]);
    static_assert(IARRAY_B200_NOALLOC_MAX_BYTES == iab::NOALLOC_MAX_BYTES &&
                  IARRAY_B200_NOALLOC_MAX_BLOCKS == iab::NOALLOC_MAX_BLOCKS, "no-allocation limits");
    if (!iab::noalloc_fits(g)) return rc_err(IARRAY_ERR_NOALLOC_TOO_LARGE);
    const int r = iab::decode_noalloc(g, static_cast<const uint8_t *>(chunks), chunks_len, dptr, ld,
                                      static_cast<cudaStream_t>(stream));
    if (r == -102) return rc_err(IARRAY_ERR_NOALLOC_TOO_LARGE);
    if (r < 0) return rc_err(IARRAY_ERR_GPU_FAILED);
    return status_rc(r);
}

INA_API(ina_rc_t) iarray_b200_encode_from_device(iarray_context_t *ctx, iarray_dtshape_t *dtshape, const void *dptr,
                                                 int64_t ld, iarray_storage_t *storage, iarray_container_t **container)
{
    CHECK_ARG(dptr);
    ina_rc_t rc = new_container(ctx, dtshape, storage, container);
    if (INA_FAILED(rc)) return rc;
    if (ld < cols_of((*container)->dtshape)) { iarray_container_free(ctx, container); return rc_err(INA_ERR_INVALID_ARGUMENT); }
    rc = (*container)->geom.nchunks ? encode_into(ctx, *container, dptr, ld) : fill_zero_chunks(*container);
    if (INA_FAILED(rc)) iarray_container_free(ctx, container);
    return rc;
}

INA_API(ina_rc_t) iarray_container_almost_equal(iarray_container_t *a, iarray_container_t *b, double tol)
{
    CHECK_ARG(a && b);
    if (a->dtshape.dtype != b->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (a->dtshape.ndim != b->dtshape.ndim) return rc_err(IARRAY_ERR_INVALID_NDIM);
    for (int i = 0; i < a->dtshape.ndim; i++)
        if (a->dtshape.shape[i] != b->dtshape.shape[i]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    iarray_config_t cfg = IARRAY_CONFIG_DEFAULTS;
    iarray_context_t *ctx = nullptr;
    ina_rc_t rc = iarray_context_new(&cfg, &ctx);
    if (INA_FAILED(rc)) return rc;
    const int64_t n = rows_of(a->dtshape) * cols_of(a->dtshape);
    const int isz = a->geom.itemsize;
    std::vector<uint8_t> ha((size_t)(n * isz)), hb((size_t)(n * isz));
    rc = iarray_to_buffer(ctx, a, ha.data(), n * isz);
    if (INA_SUCCEED(rc)) rc = iarray_to_buffer(ctx, b, hb.data(), n * isz);
    iarray_context_free(&ctx);
    if (INA_FAILED(rc)) return rc;
    // relative difference |a - b| / a, as src/iarray_container.c:1252-1279 computes it
    for (int64_t i = 0; i < n; i++) {
        double va, vb;
        if (isz == 8) { va = ((double *)ha.data())[i]; vb = ((double *)hb.data())[i]; }
        else { va = ((float *)ha.data())[i]; vb = ((float *)hb.data())[i]; }
        const double r = fabs(va - vb) / va;
        if (r > tol) return rc_err(IARRAY_ERR_ASSERTION_FAILED);
    }
    return INA_SUCCESS;
}

// ============================================================================ persistence
static iab::FrameInfo frame_info(iarray_context_t *ctx, const iarray_container_t *c)
{
    const Geom &g = c->geom;
    iab::FrameInfo fi;
    fi.ndim = c->dtshape.ndim;
    const iarray_dtshape_t &d = c->dtshape;
    for (int i = 0; i < fi.ndim; i++) {
        fi.shape[i] = d.shape[i];
        fi.chunk[i] = c->storage.chunkshape[i];
        fi.block[i] = c->storage.blockshape[i];
    }
    fi.dtype = d.dtype;
    fi.typesize = g.itemsize;
    fi.nbytes = g.nchunks * g.chunk_nbytes;
    fi.blocksize = (int32_t)g.blocksize;
    fi.chunksize = (int32_t)g.chunk_nbytes;
    fi.codec = 1;
    fi.clevel = c->clevel;
    fi.nthreads = std::max(1, ctx->cfg.max_num_threads);
    fi.shuffle = c->shuffle;
    return fi;
}

// Serialise c as a contiguous frame into buf (capacity cap bytes); *len receives the
// frame size (buf == NULL only queries it).  Chunk bytes go device -> buf directly.
static ina_rc_t frame_into(iarray_context_t *ctx, iarray_container_t *c, uint8_t *buf, int64_t cap, int64_t *len)
{
    const Geom &g = c->geom;
    const ChunkStore &s = *c->store;
    const iab::FrameInfo fi = frame_info(ctx, c);
    const std::vector<uint8_t> head = iab::frame_header(fi, s.cbytes, g.nchunks);
    const std::vector<uint8_t> tail = iab::frame_tail(s.len);
    const int64_t total = (int64_t)head.size() + s.cbytes + (int64_t)tail.size();
    *len = total;
    if (!buf) return INA_SUCCESS;
    if (cap < total) return rc_err(IARRAY_ERR_TOO_SMALL_BUFFER);
    memcpy(buf, head.data(), head.size());
    uint8_t *data = buf + head.size();
    bool in_order = true;
    int64_t acc = 0;
    for (int64_t k = 0; k < g.nchunks; k++) {
        if (s.off[k] != acc) in_order = false;
        acc += s.len[k];
    }
    if (in_order) {
        if (s.cbytes) cudaMemcpyAsync(data, s.buf.p, (size_t)s.cbytes, cudaMemcpyDeviceToHost, ctx->stream);
    } else {
        acc = 0;
        for (int64_t k = 0; k < g.nchunks; k++) {
            cudaMemcpyAsync(data + acc, s.buf.as<uint8_t>() + s.off[k], (size_t)s.len[k], cudaMemcpyDeviceToHost,
                            ctx->stream);
            acc += s.len[k];
        }
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
    memcpy(data + s.cbytes, tail.data(), tail.size());
    return INA_SUCCESS;
}

static ina_rc_t to_frame(iarray_context_t *ctx, iarray_container_t *c, std::vector<uint8_t> *out)
{
    int64_t n = 0;
    ina_rc_t rc = frame_into(ctx, c, nullptr, 0, &n);
    if (INA_FAILED(rc)) return rc;
    out->resize((size_t)n);
    return frame_into(ctx, c, out->data(), n, &n);
}

INA_API(ina_rc_t) iarray_b200_to_cframe_into(iarray_context_t *ctx, iarray_container_t *c, uint8_t *buf, int64_t cap,
                                             int64_t *len)
{
    CHECK_ARG(ctx && c && len);
    if (c->view) return rc_err(IARRAY_ERR_INVALID_STORAGE);
    return frame_into(ctx, c, buf, cap, len);
}

INA_API(ina_rc_t) iarray_to_cframe(iarray_context_t *ctx, iarray_container_t *src, uint8_t **frame, int64_t *frame_len,
                                   bool *needs_free)
{
    CHECK_ARG(ctx && src && frame && frame_len && needs_free);
    if (src->view) return rc_err(IARRAY_ERR_INVALID_STORAGE);
    int64_t n = 0;
    ina_rc_t rc = frame_into(ctx, src, nullptr, 0, &n);
    if (INA_FAILED(rc)) return rc;
    uint8_t *p = (uint8_t *)malloc((size_t)n);
    if (!p) return rc_err(INA_ERR_OUT_OF_MEMORY);
    rc = frame_into(ctx, src, p, n, &n);
    if (INA_FAILED(rc)) { free(p); return rc; }
    *frame = p;
    *frame_len = n;
    *needs_free = true;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_from_cframe(iarray_context_t *ctx, uint8_t *frame, int64_t frame_len, bool copy,
                                     iarray_container_t **container)
{
    (void)copy;   // chunks are always copied to the GPU
    CHECK_ARG(ctx && frame && container && frame_len > 0);
    iab::FrameInfo fi;
    std::vector<std::pair<int64_t, int32_t>> chunks;
    std::string why;
    if (!iab::read_frame(frame, (size_t)frame_len, &fi, &chunks, &why)) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    iarray_dtshape_t d;
    memset(&d, 0, sizeof(d));
    d.dtype = (iarray_data_type_t)fi.dtype;
    d.ndim = (int8_t)fi.ndim;
    iarray_storage_t st;
    memset(&st, 0, sizeof(st));
    for (int i = 0; i < fi.ndim; i++) { d.shape[i] = fi.shape[i]; st.chunkshape[i] = fi.chunk[i]; st.blockshape[i] = fi.block[i]; }
    ina_rc_t rc = new_container(ctx, &d, &st, container);
    if (INA_FAILED(rc)) return rc;
    iarray_container_t *c = *container;
    if (fi.typesize != c->geom.itemsize || fi.chunksize != c->geom.chunk_nbytes ||
        (int64_t)chunks.size() != c->geom.nchunks) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    }
    c->shuffle = fi.shuffle;
    c->clevel = fi.clevel;
    // the chunks occupy one region of the frame: copy it once, keep the frame's offsets
    int64_t lo = INT64_MAX, hi = 0;
    for (auto &pr : chunks) {
        if (pr.second > c->geom.chunk_nbytes + 64) { iarray_container_free(ctx, container); return rc_err(IARRAY_ERR_BLOSC_FAILED); }
        lo = std::min(lo, pr.first);
        hi = std::max(hi, pr.first + (int64_t)pr.second);
    }
    ChunkStore &s = *c->store;
    if (chunks.empty()) lo = hi = 0;
    if (!s.buf.allocate((size_t)std::max<int64_t>(hi - lo, 1), s.device)) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    }
    if (hi > lo) cudaMemcpyAsync(s.buf.p, frame + lo, (size_t)(hi - lo), cudaMemcpyHostToDevice, ctx->stream);
    s.off.clear();
    s.len.clear();
    for (auto &pr : chunks) { s.off.push_back(pr.first - lo); s.len.push_back(pr.second); }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || !s.upload_index()) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    return INA_SUCCESS;
}

static ina_rc_t write_file(const char *path, const std::vector<uint8_t> &f)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    const size_t w = fwrite(f.data(), 1, f.size(), fp);
    fclose(fp);
    return w == f.size() ? INA_SUCCESS : rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
}

// Sparse (directory) frame, c-blosc2's layout for storage.contiguous == false: the
// directory `dir` holds the index frame chunks.b2frame (header and metalayers, no chunk
// bytes, offsets holding chunk file numbers) and chunk n in the file %08X.chunk (n in
// upper-case hexadecimal, eight digits).
static std::string chunk_file(const std::string &dir, int64_t n)
{
    char name[32];
    snprintf(name, sizeof(name), "/%08X.chunk", (unsigned)n);
    return dir + name;
}

static ina_rc_t write_sparse(iarray_context_t *ctx, iarray_container_t *c, const std::string &dir)
{
    struct stat sb;
    if (stat(dir.c_str(), &sb) == 0) {
        if (!S_ISDIR(sb.st_mode)) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    } else if (mkdir(dir.c_str(), 0755) != 0) {
        return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    }
    const ChunkStore &s = *c->store;
    iab::FrameInfo fi = frame_info(ctx, c);
    fi.sparse = true;
    std::vector<uint8_t> f = iab::frame_header(fi, s.cbytes, c->geom.nchunks);
    const std::vector<uint8_t> tail = iab::frame_tail(s.len, true);
    f.insert(f.end(), tail.begin(), tail.end());
    ina_rc_t rc = write_file((dir + "/chunks.b2frame").c_str(), f);
    std::vector<uint8_t> chunk;
    for (int64_t k = 0; k < c->geom.nchunks && INA_SUCCEED(rc); k++) {
        chunk.resize((size_t)s.len[k]);
        if (cudaMemcpy(chunk.data(), s.buf.as<uint8_t>() + s.off[k], chunk.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
            return rc_err(IARRAY_ERR_GPU_FAILED);
        rc = write_file(chunk_file(dir, k).c_str(), chunk);
    }
    return rc;
}

static ina_rc_t save_if_urlpath(iarray_context_t *ctx, iarray_container_t *c)
{
    if (c->urlpath.empty()) return INA_SUCCESS;
    if (!c->storage.contiguous) return write_sparse(ctx, c, c->urlpath);
    std::vector<uint8_t> f;
    ina_rc_t rc = to_frame(ctx, c, &f);
    if (INA_FAILED(rc)) return rc;
    return write_file(c->urlpath.c_str(), f);
}

INA_API(ina_rc_t) iarray_container_save(iarray_context_t *ctx, iarray_container_t *container, char *urlpath)
{
    CHECK_ARG(ctx && container && urlpath);
    if (container->view) return rc_err(IARRAY_ERR_INVALID_STORAGE);   // src/iarray_container.c:57-61
    if (!container->urlpath.empty()) return rc_err(IARRAY_ERR_INVALID_STORAGE);
    std::vector<uint8_t> f;
    ina_rc_t rc = to_frame(ctx, container, &f);
    if (INA_FAILED(rc)) return rc;
    return write_file(urlpath, f);
}

static bool read_file(const std::string &path, std::vector<uint8_t> *f)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) return false;
    fseek(fp, 0, SEEK_END);
    const long n = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    f->resize((size_t)std::max(n, 0L));
    const size_t r = n > 0 ? fread(f->data(), 1, (size_t)n, fp) : 0;
    fclose(fp);
    return n > 0 && r == (size_t)n;
}

// Open a sparse (directory) frame: its index frame, then every chunk file it names.
static ina_rc_t load_sparse(iarray_context_t *ctx, const std::string &dir, iarray_container_t **container)
{
    std::vector<uint8_t> f;
    if (!read_file(dir + "/chunks.b2frame", &f)) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    iab::FrameInfo fi;
    std::vector<std::pair<int64_t, int32_t>> index;
    std::string why;
    if (!iab::read_frame(f.data(), f.size(), &fi, &index, &why) || !fi.sparse)
        return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    std::vector<std::vector<uint8_t>> chunks(index.size());
    std::vector<const uint8_t *> ptrs;
    std::vector<int64_t> lens;
    for (size_t k = 0; k < index.size(); k++) {
        if (!read_file(chunk_file(dir, index[k].first), &chunks[k]) || chunks[k].size() < 32)
            return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
        ptrs.push_back(chunks[k].data());
        lens.push_back((int64_t)chunks[k].size());
    }
    iarray_dtshape_t d;
    memset(&d, 0, sizeof(d));
    d.dtype = (iarray_data_type_t)fi.dtype;
    d.ndim = (int8_t)fi.ndim;
    iarray_storage_t st;
    memset(&st, 0, sizeof(st));
    st.contiguous = false;
    for (int i = 0; i < fi.ndim; i++) { d.shape[i] = fi.shape[i]; st.chunkshape[i] = fi.chunk[i]; st.blockshape[i] = fi.block[i]; }
    ina_rc_t rc = new_container(ctx, &d, &st, container);
    if (INA_FAILED(rc)) return rc;
    iarray_container_t *c = *container;
    if (fi.typesize != c->geom.itemsize || fi.chunksize != c->geom.chunk_nbytes ||
        (int64_t)index.size() != c->geom.nchunks) {
        iarray_container_free(ctx, container);
        return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    }
    c->shuffle = fi.shuffle;
    c->clevel = fi.clevel;
    rc = upload_chunks(ctx, c, ptrs.data(), lens.data());
    if (INA_FAILED(rc)) iarray_container_free(ctx, container);
    return rc;
}

static ina_rc_t load_file(iarray_context_t *ctx, char *urlpath, iarray_container_t **container, bool keep_path)
{
    CHECK_ARG(ctx && urlpath && container);
    struct stat sb;
    if (stat(urlpath, &sb) != 0) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    ina_rc_t rc;
    if (S_ISDIR(sb.st_mode)) {
        rc = load_sparse(ctx, urlpath, container);
    } else {
        std::vector<uint8_t> f;
        if (!read_file(urlpath, &f)) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
        rc = iarray_from_cframe(ctx, f.data(), (int64_t)f.size(), true, container);
        if (INA_SUCCEED(rc)) (*container)->storage.contiguous = true;
    }
    if (INA_SUCCEED(rc) && keep_path) (*container)->urlpath = urlpath;
    return rc;
}

// iarray.h:617 (src/iarray_container.c:219-225, blosc2_remove_urlpath): removes a
// contiguous frame file, or a sparse frame's directory with its index and chunk files.
INA_API(ina_rc_t) iarray_container_remove(char *urlpath)
{
    CHECK_ARG(urlpath);
    struct stat sb;
    if (stat(urlpath, &sb) != 0) return rc_err(IARRAY_ERR_BLOSC_FAILED);
    if (!S_ISDIR(sb.st_mode)) return unlink(urlpath) == 0 ? INA_SUCCESS : rc_err(IARRAY_ERR_BLOSC_FAILED);
    DIR *dp = opendir(urlpath);
    if (!dp) return rc_err(IARRAY_ERR_BLOSC_FAILED);
    bool ok = true;
    for (struct dirent *e = readdir(dp); e; e = readdir(dp)) {
        const std::string n = e->d_name;
        const bool chunk = n.size() == 14 && n.compare(8, 6, ".chunk") == 0;
        if (chunk || n == "chunks.b2frame") ok &= unlink((std::string(urlpath) + "/" + n).c_str()) == 0;
    }
    closedir(dp);
    ok &= rmdir(urlpath) == 0;
    return ok ? INA_SUCCESS : rc_err(IARRAY_ERR_BLOSC_FAILED);
}

INA_API(ina_rc_t) iarray_container_open(iarray_context_t *ctx, char *urlpath, iarray_container_t **container)
{
    return load_file(ctx, urlpath, container, true);
}

INA_API(ina_rc_t) iarray_container_load(iarray_context_t *ctx, char *urlpath, iarray_container_t **container)
{
    return load_file(ctx, urlpath, container, false);
}

// ============================================================================ linear algebra
INA_API(ina_rc_t) iarray_linalg_transpose(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t **b)
{
    (void)ctx;
    CHECK_ARG(a && b);
    if (a->view) return rc_err(IARRAY_ERR_NOT_SUPPORTED);          // src/linalg/transpose.c:23-26
    if (a->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    iarray_container_t *v = new iarray_container_t(*a);
    v->dtshape.shape[0] = a->dtshape.shape[1];
    v->dtshape.shape[1] = a->dtshape.shape[0];
    v->transposed = true;
    v->view = true;
    v->urlpath.clear();
    *b = v;
    return INA_SUCCESS;
}

struct Timer {
    iarray_context_t *ctx;
    explicit Timer(iarray_context_t *c) : ctx(c) { cudaEventRecord(ctx->ev[0], ctx->stream); }
    void mark(int i) { cudaEventRecord(ctx->ev[i], ctx->stream); }
    void finish()
    {
        cudaEventSynchronize(ctx->ev[4]);
        float t;
        for (int i = 0; i < 4; i++) {
            cudaEventElapsedTime(&t, ctx->ev[i], ctx->ev[i + 1]);
            ctx->timings[i] = t;
        }
        cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[4]);
        ctx->timings[4] = t;
    }
};

// Run the product on dense device operands with the context's form.
// zs (optional): leave out the K ranges of zero-block pairs in the float64 products.
// cimg (optional, split form, float64): the product goes into the output container's encoder
// image instead of C.
static ina_rc_t dense_product(iarray_context_t *ctx, int dtype, int64_t M, int64_t N, int64_t K, const void *A,
                              int64_t lda, const void *B, int64_t ldb, void *C, int64_t ldc,
                              const iab::ZeroSkip *zs = nullptr, const iab::CImage *cimg = nullptr)
{
    if (ctx->form == IARRAY_B200_FORM_SPLIT) {
        int r;
        if (dtype == IARRAY_DATA_TYPE_DOUBLE)
            r = iab::gemm_f64_ozaki(M, N, K, (const double *)A, lda, (const double *)B, ldb, (double *)C, ldc,
                                    ctx->split_terms, ctx->stream, zs, cimg);
        else
            r = iab::gemm_f32_bf16_split(M, N, K, (const float *)A, lda, (const float *)B, ldb, (float *)C, ldc,
                                         ctx->split_products_f32, ctx->stream);
        if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        if (r != 0) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    } else if (dtype == IARRAY_DATA_TYPE_DOUBLE) {
        iab::gemm_f64_native(M, N, K, (const double *)A, lda, (const double *)B, ldb, (double *)C, ldc, ctx->stream, zs);
    } else {
        iab::gemm_f32_native(M, N, K, (const float *)A, lda, (const float *)B, ldb, (float *)C, ldc, ctx->stream);
    }
    return cuda_rc(cudaGetLastError());
}

INA_API(ina_rc_t) iarray_b200_dense_gemm(iarray_context_t *ctx, int dtype, int64_t M, int64_t N, int64_t K,
                                         const void *A, int64_t lda, const void *B, int64_t ldb, void *C, int64_t ldc)
{
    CHECK_ARG(ctx && A && B && C && M >= 0 && N >= 0 && K >= 0);
    CHECK_ARG(dtype == IARRAY_DATA_TYPE_DOUBLE || dtype == IARRAY_DATA_TYPE_FLOAT);
    const int64_t align = dtype == IARRAY_DATA_TYPE_DOUBLE ? 2 : 4;
    CHECK_ARG(lda % align == 0 && ldb % align == 0 && ldc % align == 0);
    CHECK_ARG(lda >= K && ldb >= N && ldc >= N);
    if (M == 0 || N == 0) return INA_SUCCESS;
    return dense_product(ctx, dtype, M, N, K, A, lda, B, ldb, C, ldc);
}

// Decode -> product -> encode into the already-created container c.
// Zero-block rule of the entry point (which operands' special-zero chunks are skipped
// besides zero blocks): none for the panel products (src/linalg/matmul/gemm.c, gemv.c
// multiply whole panels), both for iarray_opt_gemm and iarray_opt_gemv
// (src/linalg/iarray_gemm.c:146-168, iarray_gemv.c:131-150), B's only for
// iarray_opt_gemm_a (iarray_gemm_a.c:127-146: A's blocks come from block_is_zeros alone),
// A's only for iarray_opt_gemm_b (iarray_gemm_b.c:127-146).
enum SkipRule { SKIP_NONE = 0, SKIP_BOTH, SKIP_B_CHUNKS, SKIP_A_CHUNKS };

// The zero-block rule around a product of decoded operands: flag grids from the decoders'
// per-block flags, and (after the product) the recomputation of output blocks whose
// skipped pairs face a NaN or an infinity.
struct ZeroRule {
    DevBuf za, zb, nfa, nfb;
    iab::ZeroSkip zs;
    bool on = false;
    bool build(iarray_context_t *ctx, const Geom &ga, const Geom &gb, bool vec, const DevBuf *zf, int rule)
    {
        const int64_t RB = ga.cgrid[0] * ga.bgrid[0], KB = ga.cgrid[1] * ga.bgrid[1];
        const int64_t JB = vec ? 1 : gb.cgrid[1] * gb.bgrid[1];
        if (RB * KB == 0 || KB * JB == 0) return true;
        if (!za.allocate((size_t)(RB * KB), ctx->device) || !zb.allocate((size_t)(KB * JB), ctx->device) ||
            !nfa.allocate((size_t)(RB * KB), ctx->device) || !nfb.allocate((size_t)(KB * JB), ctx->device))
            return false;
        iab::zero_grid(ga, zf[0].as<uint8_t>(), rule == SKIP_BOTH || rule == SKIP_A_CHUNKS, za.as<uint8_t>(), ctx->stream);
        iab::zero_grid(gb, zf[1].as<uint8_t>(), rule == SKIP_BOTH || rule == SKIP_B_CHUNKS, zb.as<uint8_t>(), ctx->stream);
        zs = iab::ZeroSkip{za.as<uint8_t>(), zb.as<uint8_t>(),
                           ga.chunk[0], ga.block[0], ga.bgrid[0],
                           ga.chunk[1], ga.block[1], ga.bgrid[1],
                           vec ? 1 : gb.chunk[1], vec ? 1 : gb.block[1], vec ? 1 : gb.bgrid[1],
                           RB, KB, JB};
        on = true;
        return true;
    }
    void fix(iarray_context_t *ctx, int isz, int64_t M, int64_t N, int64_t K, const void *A, int64_t lda, const void *B,
             int64_t ldb, void *C, int64_t ldc)
    {
        if (!on) return;
        cudaMemsetAsync(nfa.p, 0, nfa.n, ctx->stream);
        cudaMemsetAsync(nfb.p, 0, nfb.n, ctx->stream);
        iab::block_nonfinite(isz, M, K, A, lda, zs.r_chunk, zs.r_block, zs.r_bg, zs.k_chunk, zs.k_block, zs.k_bg, zs.KB,
                             nfa.as<uint8_t>(), ctx->stream);
        iab::block_nonfinite(isz, K, N, B, ldb, zs.k_chunk, zs.k_block, zs.k_bg, zs.c_chunk, zs.c_block, zs.c_bg, zs.JB,
                             nfb.as<uint8_t>(), ctx->stream);
        iab::zero_fix(isz, M, N, K, A, lda, B, ldb, C, ldc, zs, nfa.as<uint8_t>(), nfb.as<uint8_t>(), ctx->stream);
    }
};

// y = A x with the GEMV fused into A's decode (iab::decode_gemv): x is decoded into dx, A's
// streams through the parse and the LZ4 launch, then its items straight into the row sums.  When
// the entry point's zero-block rule applies and the parse found zero blocks, A is also scattered
// densely into *dA (leading dimension lda) from the same decoded streams and *zr is built, for
// the caller's recomputation of the outputs the rule changes.
static ina_rc_t gemv_fused(iarray_context_t *ctx, const iarray_container_t *a, const iarray_container_t *b, void *dx,
                           void *dy, int skip, DevBuf *dA, int64_t lda, ZeroRule *zr)
{
    const Geom &g = a->geom;
    DevBuf part;
    if (!part.allocate((size_t)std::max<int64_t>(iab::decode_gemv_part_items(g) * g.itemsize, 16), ctx->device))
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    const iab::DecodeArgs args[2] = {
        {g, a->store->buf.as<uint8_t>(), (int64_t)a->store->buf.n, a->store->d_off.as<int64_t>(),
         a->store->d_len.as<int32_t>(), nullptr, lda},
        {b->geom, b->store->buf.as<uint8_t>(), (int64_t)b->store->buf.n, b->store->d_off.as<int64_t>(),
         b->store->d_len.as<int32_t>(), dx, b->geom.shape[1]}};
    iab::DecodeQueue q;
    iab::DecodeWork w[2];
    const bool xc = b->geom.nchunks > 0;
    int r = iab::decode_queue_init(&q, iab::decode_max_jobs(g) + iab::decode_max_jobs(b->geom), ctx->stream);
    if (!r) r = iab::decode_parse(args[0], &q, &w[0], ctx->stream);
    if (!r && xc) r = iab::decode_parse(args[1], &q, &w[1], ctx->stream);
    if (!r) r = iab::decode_lz4(&q, ctx->stream);
    if (!r && xc) r = iab::decode_scatter(args[1], &w[1], ctx->stream);
    if (!r) r = iab::decode_gemv(args[0], &w[0], dx, part.p, dy, ctx->stream);
    if (!r) r = iab::decode_finish(&w[0], ctx->stream);
    if (!r && xc) r = iab::decode_finish(&w[1], ctx->stream);
    if (!r && skip != SKIP_NONE && w[0].nzero + (xc ? w[1].nzero : 0) > 0) {
        if (!dA->allocate((size_t)std::max<int64_t>(g.shape[0] * lda * g.itemsize, 16), ctx->device)) {
            cudaStreamSynchronize(ctx->stream);
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        }
        iab::DecodeArgs da = args[0];
        da.out = dA->p;
        r = iab::decode_scatter(da, &w[0], ctx->stream);
        if (!r) r = iab::decode_finish(&w[0], ctx->stream);
        DevBuf zf[2];
        zf[0] = std::move(w[0].zf);
        if (xc) zf[1] = std::move(w[1].zf);
        if (!r && !zr->build(ctx, g, b->geom, true, zf, skip)) {
            cudaStreamSynchronize(ctx->stream);
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        }
    }
    if (r) cudaStreamSynchronize(ctx->stream);     // the work buffers go back to the pool idle
    return decode_rc(r);
}

static ina_rc_t run_matmul(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b, iarray_container_t *c,
                           int skip = SKIP_NONE)
{
    const int dtype = a->dtshape.dtype;
    const int isz = a->geom.itemsize;
    const int64_t M = a->dtshape.shape[0], K = a->dtshape.shape[1];
    const bool vec = b->dtshape.ndim == 1;
    const int64_t N = vec ? 1 : b->dtshape.shape[1];
    const int64_t lda = pad_ld(K), ldb = vec ? 1 : pad_ld(N), ldc = vec ? 1 : pad_ld(N);
    Timer tm(ctx);
    DevBuf dA, dB, dC;
    // decode-fused GEMV: A's items go from its chunks straight into the row sums
    const bool fused = vec && !a->transposed && !b->transposed && K > 0 && M > 0 && a->geom.nchunks &&
                       b->geom.nchunks && iab::decode_gemv_fits(a->geom);
    // split float64 product straight into C's encoder image (no dense C, no gather)
    bool direct = !vec && K > 0 && ctx->form == IARRAY_B200_FORM_SPLIT && dtype == IARRAY_DATA_TYPE_DOUBLE &&
                  iab::encode_image_ok(c->geom, c->shuffle, c->clevel == 0);
    if ((!fused && !dA.allocate((size_t)std::max<int64_t>(M * lda * isz, 16), ctx->device)) ||
        !dB.allocate((size_t)std::max<int64_t>((vec ? pad_ld(K) : K * ldb) * isz, 16), ctx->device) ||
        (!direct && !dC.allocate((size_t)std::max<int64_t>((vec ? pad_ld(M) : M * ldc) * isz, 16), ctx->device)))
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (vec) cudaMemsetAsync(dB.p, 0, (size_t)(pad_ld(K) * isz), ctx->stream);
    ina_rc_t rc;
    ZeroRule zr;
    if (fused) {
        rc = gemv_fused(ctx, a, b, dB.p, dC.p, skip, &dA, lda, &zr);
        if (INA_FAILED(rc)) return rc;
        tm.mark(1);
        tm.mark(2);
        if (zr.on) {
            zr.fix(ctx, isz, M, N, K, dA.p, lda, dB.p, 1, dC.p, 1);
            rc = cuda_rc(cudaGetLastError());
            if (INA_FAILED(rc)) return rc;
        }
    } else if (!a->transposed && !b->transposed) {
        // both operands at once: one LZ4 launch over the streams of A and B
        DevBuf zf[2];
        int nz[2] = {0, 0};
        rc = decode_pair(ctx, a, dA.p, lda, b, dB.p, vec ? K : ldb, zf, nz);
        if (INA_FAILED(rc)) return rc;
        if (skip != SKIP_NONE && nz[0] + nz[1] > 0 && K > 0 &&
            !zr.build(ctx, a->geom, b->geom, vec, zf, skip))
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        tm.mark(1);
        tm.mark(2);
    } else {
        rc = decode_logical(ctx, a, dA.p, lda);
        if (INA_FAILED(rc)) return rc;
        tm.mark(1);
        rc = decode_logical(ctx, b, dB.p, vec ? K : ldb);
        if (INA_FAILED(rc)) return rc;
        tm.mark(2);
    }
    // the zero-block rule's fix works on a dense C
    if (direct && zr.on) {
        direct = false;
        if (!dC.allocate((size_t)std::max<int64_t>(M * ldc * isz, 16), ctx->device)) {
            cudaStreamSynchronize(ctx->stream);
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        }
    }
    iab::EncodeWork ew;
    iab::CImage cimg;
    if (direct) {
        if (iab::encode_image_prepare(c->geom, &ew) != 0) {
            cudaStreamSynchronize(ctx->stream);
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        }
        cimg.g = c->geom;
        cimg.img = ew.img.as<uint8_t>();
    }
    if (fused) {
    } else if (K == 0) {
        cudaMemsetAsync(dC.p, 0, (size_t)((vec ? M : M * ldc) * isz), ctx->stream);
    } else if (vec) {
        iab::gemv_native(dtype == IARRAY_DATA_TYPE_DOUBLE ? 0 : 1, M, K, dA.p, lda, dB.p, dC.p, ctx->stream);
        rc = cuda_rc(cudaGetLastError());
    } else {
        rc = dense_product(ctx, dtype, M, N, K, dA.p, lda, dB.p, ldb, dC.p, ldc, zr.on ? &zr.zs : nullptr,
                           direct ? &cimg : nullptr);
    }
    if (INA_FAILED(rc)) return rc;
    if (zr.on && !fused) {
        zr.fix(ctx, isz, M, N, K, dA.p, lda, dB.p, vec ? 1 : ldb, dC.p, vec ? 1 : ldc);
        rc = cuda_rc(cudaGetLastError());
        if (INA_FAILED(rc)) return rc;
    }
    tm.mark(3);
    // dA and dB stay allocated until the encode below has synchronised the stream: the pool is
    // shared by every context, so memory released while the product may still read it could be
    // handed to another stream
    if (direct) rc = encode_into_image(ctx, c, &ew);
    else rc = c->geom.nchunks ? encode_into(ctx, c, dC.p, vec ? M : ldc) : fill_zero_chunks(c);
    if (INA_FAILED(rc)) return rc;
    tm.mark(4);
    tm.finish();
    return save_if_urlpath(ctx, c);
}

static ina_rc_t output_container(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                 iarray_storage_t *storage, iarray_container_t **c)
{
    iarray_dtshape_t d;
    memset(&d, 0, sizeof(d));
    d.dtype = a->dtshape.dtype;
    d.ndim = b->dtshape.ndim;
    d.shape[0] = a->dtshape.shape[0];
    if (d.ndim > 1) d.shape[1] = b->dtshape.shape[1];
    ina_rc_t rc = new_container(ctx, &d, storage, c);
    if (INA_FAILED(rc)) return rc;
    (*c)->shuffle = true;   // blosc2 cparams defaults keep SHUFFLE in the last filter slot
    return INA_SUCCESS;
}

static ina_rc_t check_operands(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b, iarray_storage_t *storage,
                               iarray_container_t **c)
{
    CHECK_ARG(ctx && a && b && storage && c);
    if (a->dtshape.dtype != IARRAY_DATA_TYPE_DOUBLE && a->dtshape.dtype != IARRAY_DATA_TYPE_FLOAT)
        return rc_err(IARRAY_ERR_INVALID_DTYPE);
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_linalg_matmul(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                       iarray_storage_t *storage, iarray_container_t **c)
{
    CHECK_ARG(ctx && a && b && storage && c);
    // src/linalg/matmul.c:31-55
    if (a->dtshape.ndim != 2 || (b->dtshape.ndim != 1 && b->dtshape.ndim != 2)) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    ina_rc_t rc = check_operands(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    const int64_t oshape[2] = {a->dtshape.shape[0], b->dtshape.ndim > 1 ? b->dtshape.shape[1] : 0};
    for (int i = 0; i < b->dtshape.ndim; i++)
        if (oshape[i] < storage->chunkshape[i]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    rc = output_container(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    rc = run_matmul(ctx, a, b, *c);
    if (INA_FAILED(rc)) iarray_container_free(ctx, c);
    return rc;
}

INA_API(ina_rc_t) iarray_gemm(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b, iarray_container_t *c)
{
    CHECK_ARG(ctx && a && b && c);
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 2 || c->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0] || c->dtshape.shape[0] != a->dtshape.shape[0] ||
        c->dtshape.shape[1] != b->dtshape.shape[1])
        return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype || c->dtshape.dtype != a->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    c->shuffle = true;
    return run_matmul(ctx, a, b, c);
}

INA_API(ina_rc_t) iarray_gemv(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b, iarray_container_t *c)
{
    CHECK_ARG(ctx && a && b && c);
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 1 || c->dtshape.ndim != 1) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0] || c->dtshape.shape[0] != a->dtshape.shape[0])
        return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype || c->dtshape.dtype != a->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    c->shuffle = true;
    return run_matmul(ctx, a, b, c);
}

// Partition checks of iarray_opt_gemm (src/linalg/iarray_gemm.c:327-364).
INA_API(ina_rc_t) iarray_opt_gemm(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                  iarray_storage_t *storage, iarray_container_t **c)
{
    ina_rc_t rc = check_operands(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    const int64_t *ac = a->storage.chunkshape, *bc = b->storage.chunkshape, *ab = a->storage.blockshape,
                  *bb = b->storage.blockshape;
    if (a->transposed || b->transposed) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    if (ac[0] != storage->chunkshape[0] || ac[1] != bc[0] || bc[1] != storage->chunkshape[1])
        return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    if (ab[0] != storage->blockshape[0] || ab[1] != bb[0] || bb[1] != storage->blockshape[1])
        return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    rc = output_container(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    rc = run_matmul(ctx, a, b, *c, SKIP_BOTH);
    if (INA_FAILED(rc)) iarray_container_free(ctx, c);
    return rc;
}

// Partition checks of iarray_opt_gemm_a (src/linalg/iarray_gemm_a.c:212-263); with
// `swap`, the mirrored checks of iarray_opt_gemm_b (src/linalg/iarray_gemm_b.c).
static ina_rc_t opt_gemm_ab(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                            iarray_storage_t *storage, iarray_container_t **c, bool swap)
{
    ina_rc_t rc = check_operands(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (a->transposed || b->transposed) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    const int64_t *ac = a->storage.chunkshape, *bc = b->storage.chunkshape, *ab = a->storage.blockshape,
                  *bb = b->storage.blockshape, *as = a->dtshape.shape, *bs = b->dtshape.shape;
    const int64_t *cc = storage->chunkshape, *cb = storage->blockshape;
    if (!swap) {
        if (ac[1] < as[1] || bc[0] < bs[0] || ac[1] != bc[0]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
        if (ac[0] != cc[0] || bs[1] > cc[1]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
        if (ac[0] != cb[0] || bc[1] != cb[1] || ac[0] != ab[0] || bc[1] != bb[1] || ab[1] != bb[0])
            return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    } else {
        if (ac[1] < as[1] || bc[0] < bs[0] || ac[1] != bc[0]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
        if (bc[1] != cc[1] || as[0] > cc[0]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
        if (ac[0] != cb[0] || bc[1] != cb[1] || ac[0] != ab[0] || bc[1] != bb[1] || ab[1] != bb[0])
            return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    }
    rc = output_container(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    rc = run_matmul(ctx, a, b, *c, swap ? SKIP_A_CHUNKS : SKIP_B_CHUNKS);
    if (INA_FAILED(rc)) iarray_container_free(ctx, c);
    return rc;
}

INA_API(ina_rc_t) iarray_opt_gemm_a(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                    iarray_storage_t *storage, iarray_container_t **c)
{
    return opt_gemm_ab(ctx, a, b, storage, c, false);
}

INA_API(ina_rc_t) iarray_opt_gemm_b(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                    iarray_storage_t *storage, iarray_container_t **c)
{
    return opt_gemm_ab(ctx, a, b, storage, c, true);
}

// Partition checks of iarray_opt_gemv (src/linalg/iarray_gemv.c:261-286).
INA_API(ina_rc_t) iarray_opt_gemv(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                  iarray_storage_t *storage, iarray_container_t **c)
{
    ina_rc_t rc = check_operands(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 1) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    if (a->dtshape.dtype != b->dtshape.dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (a->transposed) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    const int64_t *ac = a->storage.chunkshape, *bc = b->storage.chunkshape, *ab = a->storage.blockshape,
                  *bb = b->storage.blockshape;
    if (ac[0] != storage->chunkshape[0] || ac[1] != bc[0]) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    if (ab[0] != storage->blockshape[0] || ab[1] != bb[0]) return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    rc = output_container(ctx, a, b, storage, c);
    if (INA_FAILED(rc)) return rc;
    rc = run_matmul(ctx, a, b, *c, SKIP_BOTH);
    if (INA_FAILED(rc)) iarray_container_free(ctx, c);
    return rc;
}

// ============================================================================ product of host frames, pipelined
// iarray_b200_opt_gemm_cframes: iarray_opt_gemm for operands held as contiguous frames in
// host memory, with the result written as a contiguous frame into host memory.  The work is
// cut into row bands of C, one chunk row each.  All uploads are queued at once on the upload
// stream (B's chunk rows, then A's); the context stream decodes each chunk row as soon as its
// bytes are on the device, multiplies each band of A with the whole of B and encodes the
// band; the download stream copies a band's chunks to their final place in the output frame
// as soon as their sizes are known.  Uploads, kernels and downloads of different bands
// overlap; with pinned host buffers the step approaches the time of the uploads.
namespace {
struct FrameView {
    iab::FrameInfo fi;
    std::vector<std::pair<int64_t, int32_t>> chunks;   // (offset in the frame, cbytes)
    Geom g;
};

ina_rc_t view_frame(const uint8_t *f, int64_t n, FrameView *v)
{
    std::string why;
    if (!iab::read_frame(f, (size_t)n, &v->fi, &v->chunks, &why)) return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    const int isz = dtype_size(v->fi.dtype);
    if (!isz) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (v->fi.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (!iab::make_geom(2, v->fi.shape, v->fi.chunk, v->fi.block, isz, &v->g)) return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    if (v->fi.typesize != isz || v->fi.chunksize != v->g.chunk_nbytes || (int64_t)v->chunks.size() != v->g.nchunks)
        return rc_err(IARRAY_ERR_PERSISTENCY_FAILED);
    for (auto &pr : v->chunks)
        if (pr.first < 0 || pr.second <= 0 || pr.second > v->g.chunk_nbytes + 64 || pr.first + pr.second > n)
            return rc_err(IARRAY_ERR_BLOSC_FAILED);
    return INA_SUCCESS;
}

// One matrix's chunks on the device: the frame region [lo, hi) and the chunk index.
struct DevChunks {
    DevBuf buf, d_off, d_len;
    int64_t lo = 0, hi = 0;
};

bool upload_index(const FrameView &v, DevChunks *d, int device)
{
    d->lo = INT64_MAX;
    d->hi = 0;
    for (auto &pr : v.chunks) {
        d->lo = std::min(d->lo, pr.first);
        d->hi = std::max(d->hi, pr.first + (int64_t)pr.second);
    }
    const size_t n = v.chunks.size();
    std::vector<int64_t> off(n);
    std::vector<int32_t> len(n);
    for (size_t k = 0; k < n; k++) { off[k] = v.chunks[k].first - d->lo; len[k] = v.chunks[k].second; }
    if (!d->buf.allocate((size_t)(d->hi - d->lo), device) || !d->d_off.allocate(n * 8, device) ||
        !d->d_len.allocate(n * 4, device))
        return false;
    return cudaMemcpy(d->d_off.p, off.data(), n * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(d->d_len.p, len.data(), n * 4, cudaMemcpyHostToDevice) == cudaSuccess;
}

// Queues the upload of chunk row r of v (its byte range in the frame) and records ev.
void upload_row(const FrameView &v, const uint8_t *frame, DevChunks &d, int64_t r, cudaStream_t up, cudaEvent_t ev)
{
    const int64_t per = v.g.cgrid[1];
    int64_t lo = INT64_MAX, hi = 0;
    for (int64_t k = r * per; k < (r + 1) * per; k++) {
        lo = std::min(lo, v.chunks[(size_t)k].first);
        hi = std::max(hi, v.chunks[(size_t)k].first + (int64_t)v.chunks[(size_t)k].second);
    }
    cudaMemcpyAsync(d.buf.as<uint8_t>() + (lo - d.lo), frame + lo, (size_t)(hi - lo), cudaMemcpyHostToDevice, up);
    cudaEventRecord(ev, up);
}

// Geometry of rows [r * chunk0, ...) of g: one chunk row.
Geom row_geom(const Geom &g, int64_t r)
{
    Geom b;
    const int64_t rows = std::min(g.chunk[0], g.shape[0] - r * g.chunk[0]);
    const int64_t shape[2] = {rows, g.shape[1]};
    iab::make_geom(2, shape, g.chunk, g.block, g.itemsize, &b);
    return b;
}

struct EventSet {
    std::vector<cudaEvent_t> ev;
    explicit EventSet(size_t n) : ev(n, nullptr)
    {
        for (auto &e : ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    ~EventSet()
    {
        for (auto &e : ev) if (e) cudaEventDestroy(e);
    }
};
}  // namespace

// The same product without the pipeline (degenerate sizes).
static ina_rc_t opt_gemm_cframes_plain(iarray_context_t *ctx, const uint8_t *a_frame, int64_t a_len,
                                       const uint8_t *b_frame, int64_t b_len, iarray_storage_t *storage, uint8_t *out,
                                       int64_t out_cap, int64_t *out_len)
{
    iarray_container_t *a = nullptr, *b = nullptr, *c = nullptr;
    ina_rc_t rc = iarray_from_cframe(ctx, const_cast<uint8_t *>(a_frame), a_len, true, &a);
    if (INA_SUCCEED(rc)) rc = iarray_from_cframe(ctx, const_cast<uint8_t *>(b_frame), b_len, true, &b);
    if (INA_SUCCEED(rc)) rc = iarray_opt_gemm(ctx, a, b, storage, &c);
    if (INA_SUCCEED(rc)) rc = frame_into(ctx, c, out, out_cap, out_len);
    iarray_container_free(ctx, &a);
    iarray_container_free(ctx, &b);
    iarray_container_free(ctx, &c);
    return rc;
}

INA_API(ina_rc_t) iarray_b200_opt_gemm_cframes(iarray_context_t *ctx, const uint8_t *a_frame, int64_t a_len,
                                               const uint8_t *b_frame, int64_t b_len, iarray_storage_t *storage,
                                               uint8_t *out, int64_t out_cap, int64_t *out_len)
{
    CHECK_ARG(ctx && a_frame && b_frame && storage && out_len && a_len > 0 && b_len > 0 && out_cap >= 0);
    CHECK_ARG(!storage->urlpath);
    FrameView fa, fb;
    ina_rc_t rc = view_frame(a_frame, a_len, &fa);
    if (INA_FAILED(rc)) return rc;
    rc = view_frame(b_frame, b_len, &fb);
    if (INA_FAILED(rc)) return rc;
    // iarray_opt_gemm's checks (src/linalg/iarray_gemm.c:327-364)
    const int dtype = fa.fi.dtype;
    if (dtype != fb.fi.dtype || (dtype != IARRAY_DATA_TYPE_DOUBLE && dtype != IARRAY_DATA_TYPE_FLOAT))
        return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (fa.fi.shape[1] != fb.fi.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    const int64_t *ac = fa.fi.chunk, *bc = fb.fi.chunk, *ab = fa.fi.block, *bb = fb.fi.block;
    if (ac[0] != storage->chunkshape[0] || ac[1] != bc[0] || bc[1] != storage->chunkshape[1])
        return rc_err(IARRAY_ERR_INVALID_CHUNKSHAPE);
    if (ab[0] != storage->blockshape[0] || ab[1] != bb[0] || bb[1] != storage->blockshape[1])
        return rc_err(IARRAY_ERR_INVALID_BLOCKSHAPE);
    const int64_t M = fa.fi.shape[0], K = fa.fi.shape[1], N = fb.fi.shape[1];
    const bool split = ctx->form == IARRAY_B200_FORM_SPLIT;
    if (M == 0 || N == 0 || K == 0 || (split && dtype == IARRAY_DATA_TYPE_FLOAT))
        return opt_gemm_cframes_plain(ctx, a_frame, a_len, b_frame, b_len, storage, out, out_cap, out_len);

    // output container (host object only: its geometry and frame fields)
    iarray_dtshape_t d;
    memset(&d, 0, sizeof(d));
    d.dtype = (iarray_data_type_t)dtype;
    d.ndim = 2;
    d.shape[0] = M;
    d.shape[1] = N;
    iarray_container_t *cc = nullptr;
    rc = new_container(ctx, &d, storage, &cc);
    if (INA_FAILED(rc)) return rc;
    std::unique_ptr<iarray_container_t, void (*)(iarray_container_t *)> cguard(cc, [](iarray_container_t *p) { delete p; });
    cc->shuffle = true;
    const Geom gc = cc->geom;
    const iab::FrameInfo fic = frame_info(ctx, cc);
    const int64_t hsize = (int64_t)iab::frame_header(fic, 0, gc.nchunks).size();
    const int64_t tsize = (int64_t)iab::frame_tail(std::vector<int32_t>((size_t)gc.nchunks, 0)).size();

    if (!ctx->up) cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking);
    if (!ctx->down) cudaStreamCreateWithFlags(&ctx->down, cudaStreamNonBlocking);
    if (!ctx->enc) cudaStreamCreateWithFlags(&ctx->enc, cudaStreamNonBlocking);
    if (!ctx->tabs) cudaStreamCreateWithFlags(&ctx->tabs, cudaStreamNonBlocking);
    if (!ctx->up || !ctx->down || !ctx->enc || !ctx->tabs || !ctx->stream2) return rc_err(IARRAY_ERR_GPU_FAILED);
    cudaStream_t st = ctx->stream;
    const int isz = fa.g.itemsize;
    const int64_t lda = pad_ld(K), ldb = pad_ld(N), ldc = pad_ld(N);
    const int64_t rowsA = fa.g.cgrid[0], rowsB = fb.g.cgrid[0], bands = gc.cgrid[0];
    DevChunks da, db;
    DevBuf dA, dB, dC, status;
    if (!upload_index(fa, &da, ctx->device) || !upload_index(fb, &db, ctx->device) ||
        !dA.allocate((size_t)(M * lda * isz), ctx->device) || !dB.allocate((size_t)(K * ldb * isz), ctx->device) ||
        !dC.allocate((size_t)(M * ldc * isz), ctx->device) ||
        !status.allocate((size_t)(rowsA + rowsB) * 16 * 4, ctx->device))
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    const size_t tab_bytes = (size_t)gc.nchunks * sizeof(iab::EncChunk);
    if (ctx->pin_n < tab_bytes) {
        if (ctx->pin) cudaFreeHost(ctx->pin);
        ctx->pin = nullptr;
        ctx->pin_n = 0;
        if (cudaHostAlloc(&ctx->pin, tab_bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        }
        ctx->pin_n = tab_bytes;
    }
    iab::EncChunk *htab = static_cast<iab::EncChunk *>(ctx->pin);
    cudaMemsetAsync(status.p, 0, status.n, st);
    // everything above is ordered before the uploads
    cudaEventRecord(ctx->fork, st);
    cudaStreamWaitEvent(ctx->up, ctx->fork, 0);
    EventSet evB((size_t)rowsB), evA((size_t)rowsA), evE((size_t)bands);
    for (int64_t r = 0; r < rowsB; r++) upload_row(fb, b_frame, db, r, ctx->up, evB.ev[(size_t)r]);
    for (int64_t r = 0; r < rowsA; r++) upload_row(fa, a_frame, da, r, ctx->up, evA.ev[(size_t)r]);

    // Three compute streams: the second stream decodes (B's chunk rows, then A's, each as
    // soon as it is uploaded), the context stream prepares B and multiplies each band, the
    // encode stream encodes each finished band.  A band's decode and the previous band's
    // encode are both latency-bound and run side by side.
    cudaStream_t sd = ctx->stream2, se = ctx->enc;
    cudaStreamWaitEvent(sd, ctx->fork, 0);
    cudaStreamWaitEvent(se, ctx->fork, 0);
    Timer tm(ctx);                 // timings: [0] B decoded and prepared, [3] the bands, [4] total
    tm.mark(1);
    int err = 0;
    EventSet evD((size_t)rowsA + 1), evP((size_t)bands), evK((size_t)bands);
    std::vector<iab::DecodeWork> decB((size_t)rowsB), decA((size_t)rowsA);
    for (int64_t r = 0; r < rowsB && !err; r++) {
        cudaStreamWaitEvent(sd, evB.ev[(size_t)r], 0);
        const Geom g = row_geom(fb.g, r);
        decB[(size_t)r].ext_counters = status.as<int>() + r * 16;
        err = iab::decode_launch(g, db.buf.as<uint8_t>(), (int64_t)db.buf.n, db.d_off.as<int64_t>() + r * fb.g.cgrid[1],
                                 db.d_len.as<int32_t>() + r * fb.g.cgrid[1],
                                 dB.as<uint8_t>() + r * fb.g.chunk[0] * ldb * isz, ldb, sd, &decB[(size_t)r]);
    }
    cudaEventRecord(evD.ev[(size_t)rowsA], sd);                 // all of B decoded
    for (int64_t k = 0; k < rowsA && !err; k++) {
        cudaStreamWaitEvent(sd, evA.ev[(size_t)k], 0);
        const Geom ga = row_geom(fa.g, k);
        decA[(size_t)k].ext_counters = status.as<int>() + (rowsB + k) * 16;
        err = iab::decode_launch(ga, da.buf.as<uint8_t>(), (int64_t)da.buf.n, da.d_off.as<int64_t>() + k * fa.g.cgrid[1],
                                 da.d_len.as<int32_t>() + k * fa.g.cgrid[1],
                                 dA.as<uint8_t>() + k * fa.g.chunk[0] * lda * isz, lda, sd, &decA[(size_t)k]);
        cudaEventRecord(evD.ev[(size_t)k], sd);
    }
    cudaStreamWaitEvent(st, evD.ev[(size_t)rowsA], 0);
    iab::OzakiB ob;
    if (!err && split) err = iab::gemm_f64_ozaki_prepare_b(K, N, dB.as<double>(), ldb, ctx->split_terms, &ob, st);
    tm.mark(2);
    tm.mark(3);
    std::vector<iab::OzakiWork> oz((size_t)bands);
    std::vector<iab::EncodeWork> enc((size_t)bands);
    std::vector<DevBuf> cbuf((size_t)bands);
    std::vector<int32_t> lens((size_t)gc.nchunks, 0);
    int64_t acc = 0;
    bool small = false;
    // band k's chunks to the output frame (after its encode and chunk table are done)
    auto drain = [&](int64_t k) {
        cudaEventSynchronize(evE.ev[(size_t)k]);
        const int64_t per = gc.cgrid[1], c0 = k * per;
        int64_t bytes = 0, first = htab[c0].offset;
        for (int64_t c = c0; c < c0 + per; c++) {
            lens[(size_t)c] = htab[c].cbytes;
            bytes += htab[c].cbytes;
        }
        if (hsize + acc + bytes + tsize > out_cap || !out) small = true;
        if (!small) {
            cudaStreamWaitEvent(ctx->down, evE.ev[(size_t)k], 0);
            cudaMemcpyAsync(out + hsize + acc, cbuf[(size_t)k].as<uint8_t>() + first, (size_t)bytes,
                            cudaMemcpyDeviceToHost, ctx->down);
        }
        acc += bytes;
    };
    int64_t queued = 0;            // bands whose encode is queued
    for (int64_t k = 0; k < bands && !err; k++) {
        cudaStreamWaitEvent(st, evD.ev[(size_t)k], 0);
        // split form: a band's product (about 1.6 ms for 2048 x 8192 x 8192) is shorter than
        // the download of an encoded band, so the downloads bound the call once the first
        // band is out; each product waits for the previous band's encode kernels, which then
        // run alone instead of sharing the SMs with the product (the native form's products
        // are the longer part and keep overlapping the encodes)
        if (split && k > 0) cudaStreamWaitEvent(st, evK.ev[(size_t)k - 1], 0);
        const int64_t r0 = k * gc.chunk[0], mk = row_geom(fa.g, k).shape[0];
        uint8_t *a_k = dA.as<uint8_t>() + r0 * lda * isz, *c_k = dC.as<uint8_t>() + r0 * ldc * isz;
        const Geom gk = row_geom(gc, k);
        iab::EncodeWork &w = enc[(size_t)k];
        // split float64: the band's reconstruction goes straight into its encoder image
        iab::CImage cimg;
        if (split && dtype == IARRAY_DATA_TYPE_DOUBLE && iab::encode_image_ok(gk, cc->shuffle, cc->clevel == 0)) {
            err = iab::encode_image_prepare(gk, &w);
            if (err) break;
            cimg.g = gk;
            cimg.img = w.img.as<uint8_t>();
            oz[(size_t)k].cimg = &cimg;
        }
        if (split) {
            err = iab::gemm_f64_ozaki_rows(mk, (const double *)a_k, lda, ob, (double *)c_k, ldc, &oz[(size_t)k], st);
            oz[(size_t)k].cimg = nullptr;                 // read at launch only
        } else if (dtype == IARRAY_DATA_TYPE_DOUBLE) {
            iab::gemm_f64_native(mk, N, K, (const double *)a_k, lda, dB.as<double>(), ldb, (double *)c_k, ldc, st);
        } else {
            iab::gemm_f32_native(mk, N, K, (const float *)a_k, lda, dB.as<float>(), ldb, (float *)c_k, ldc, st);
        }
        if (err) break;
        cudaEventRecord(evP.ev[(size_t)k], st);
        cudaStreamWaitEvent(se, evP.ev[(size_t)k], 0);
        w.exact_lz4 = ctx->encoder == IARRAY_B200_ENCODER_LIBLZ4;
        w.memcpy_only = cc->clevel == 0;
        err = iab::encode_launch(gk, c_k, ldc, cc->shuffle, cc->splitmode, &cbuf[(size_t)k], &w, se);
        if (err) break;
        // the chunk table goes to the host on its own stream: a device-to-host copy queued on
        // the encode stream would wait behind the previous band's download and hold up the
        // next band's encode
        cudaEventRecord(evK.ev[(size_t)k], se);
        cudaStreamWaitEvent(ctx->tabs, evK.ev[(size_t)k], 0);
        cudaMemcpyAsync(htab + k * gc.cgrid[1], w.ec.p, (size_t)gk.nchunks * sizeof(iab::EncChunk),
                        cudaMemcpyDeviceToHost, ctx->tabs);
        cudaEventRecord(evE.ev[(size_t)k], ctx->tabs);
        queued = k + 1;
        if (k > 0) drain(k - 1);
    }
    if (!err) drain(bands - 1);
    // the context stream waits for the other compute streams before the final timestamp
    cudaEventRecord(ctx->join, sd);
    cudaStreamWaitEvent(st, ctx->join, 0);
    if (queued) cudaStreamWaitEvent(st, evE.ev[(size_t)queued - 1], 0);
    tm.mark(4);
    const cudaError_t ce1 = cudaStreamSynchronize(st), ce2 = cudaStreamSynchronize(ctx->down),
                      ce3 = cudaStreamSynchronize(ctx->up), ce4 = cudaStreamSynchronize(sd),
                      ce5 = cudaStreamSynchronize(se), ce6 = cudaStreamSynchronize(ctx->tabs);
    tm.finish();
    if (err == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (err || ce1 != cudaSuccess || ce2 != cudaSuccess || ce3 != cudaSuccess || ce4 != cudaSuccess ||
        ce5 != cudaSuccess || ce6 != cudaSuccess)
        return rc_err(IARRAY_ERR_GPU_FAILED);
    // decode status words, then the split product's error flags
    std::vector<int> hs((size_t)(rowsA + rowsB) * 16);
    if (cudaMemcpy(hs.data(), status.p, hs.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return rc_err(IARRAY_ERR_GPU_FAILED);
    for (int64_t r = 0; r < rowsA + rowsB; r++)
        if (hs[(size_t)(r * 16 + 1)]) return status_rc(hs[(size_t)(r * 16 + 1)]);
    for (auto &w : oz)
        if (w.err.p && iab::gemm_f64_ozaki_finish(&w, st)) return rc_err(IARRAY_ERR_GPU_FAILED);
    *out_len = hsize + acc + tsize;
    if (small) return rc_err(IARRAY_ERR_TOO_SMALL_BUFFER);
    const std::vector<uint8_t> head = iab::frame_header(fic, acc, gc.nchunks);
    const std::vector<uint8_t> tail = iab::frame_tail(lens);
    memcpy(out, head.data(), head.size());
    memcpy(out + hsize + acc, tail.data(), tail.size());
    return INA_SUCCESS;
}

// ============================================================================ batched products
// A batch of independent float64 products C_i = A_i * B_i with their own shapes and
// partitions.  iarray_b200_batch_new allocates every buffer the batch needs, decodes the
// operands once, runs the autotuner (native form: the grouped product's tile and stage
// configurations; split form: the moduli count), runs the whole batch once eagerly, and
// captures decode -> product -> encode of all problems in one CUDA graph.
// iarray_b200_batch_run replays the graph and turns the encoded outputs into containers.
// Every stage is one launch over all problems: the grouped codec (decode of every operand,
// encode of every output when they share a stream shape), and the product: native form, one
// persistent grouped DMMA launch over the tiles of all problems (tiles ordered by descending
// K); split form, one grouped Ozaki pipeline over all problems.
struct iarray_b200_batch_s {
    iarray_context_t *ctx = nullptr;
    int form = IARRAY_B200_FORM_NATIVE;
    int64_t n = 0;
    std::vector<iarray_container_t *> a, b;
    std::vector<iarray_storage_t> storage;
    std::vector<Geom> cgeom;
    std::vector<int64_t> M, N, K, lda, ldb, ldc;
    std::vector<DevBuf> dA, dB, dC, cbuf;
    iab::CodecGroup dgrp;             // every operand's decode: one launch per stage
    iab::CodecGroup egrp;             // every output's encode, when they share one stream shape
    bool egroup = false;
    std::vector<iab::EncodeWork> enc; // else each output's encode on the branches
    iab::OzGroupWork ozg;             // split form: every product in one grouped pipeline
    int split_terms = 0;              // split form: moduli in use (context's choice or the autotuner's)
    double split_err_native = -1;     // autotuner: normwise error of the native product vs 16 moduli
    double split_tune_ms[5] = {-1, -1, -1, -1, -1};    // autotuner: 16, 15, 14, 13, 12 moduli
    double split_tune_err[5] = {-1, -1, -1, -1, -1};
    DevBuf status;                    // 16 ints per decode: [2i] operand A, [2i + 1] operand B
    DevBuf chunks;                    // chunk tables of all outputs
    std::vector<int64_t> chunk_base;  // first entry of output i in `chunks`
    DevBuf probs;
    std::vector<iab::GemmProblem> hprobs;
    int cfg = 0, ctas = 0, total_tiles = 0;
    double tune_ms[iab::GEMM_F64_GROUPED_CONFIGS] = {-1, -1, -1, -1, -1, -1, -1, -1};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t nodes = 0;
    // independent containers are decoded / encoded on parallel branches
    std::vector<cudaStream_t> br;
    std::vector<cudaEvent_t> brev;
    cudaEvent_t fork = nullptr;
    ~iarray_b200_batch_s()
    {
        for (cudaStream_t x : br)
            if (x) cudaStreamDestroy(x);
        for (cudaEvent_t e : brev)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
    }
};

namespace {
std::mutex g_tune_mu;
std::map<std::string, int> g_tune_cache;   // problem-set signature -> tile configuration

void batch_problems(iarray_b200_batch_t *bt, int cfg, std::vector<iab::GemmProblem> *out, int *total)
{
    std::vector<int64_t> order((size_t)bt->n);
    for (int64_t i = 0; i < bt->n; i++) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return bt->K[(size_t)x] > bt->K[(size_t)y]; });
    out->clear();
    int t = 0;
    for (int64_t i : order) {
        iab::GemmProblem p;
        p.M = (int)bt->M[(size_t)i]; p.N = (int)bt->N[(size_t)i]; p.K = (int)bt->K[(size_t)i];
        p.tile_start = t;
        p.A = bt->dA[(size_t)i].as<double>(); p.B = bt->dB[(size_t)i].as<double>(); p.C = bt->dC[(size_t)i].as<double>();
        p.lda = bt->lda[(size_t)i]; p.ldb = bt->ldb[(size_t)i]; p.ldc = bt->ldc[(size_t)i];
        if (p.M > 0 && p.N > 0) {
            out->push_back(p);
            t += iab::gemm_f64_grouped_tiles(cfg, p.M, p.N);
        }
    }
    *total = t;
}

// Enqueues decode (parts & 1), product (parts & 2) and encode (parts & 4) of the whole
// batch on the context stream.
// Branch streams: fork from the context stream, join back into it.
void batch_fork(iarray_b200_batch_t *bt)
{
    cudaEventRecord(bt->fork, bt->ctx->stream);
    for (cudaStream_t x : bt->br) cudaStreamWaitEvent(x, bt->fork, 0);
}
void batch_join(iarray_b200_batch_t *bt)
{
    for (size_t k = 0; k < bt->br.size(); k++) {
        cudaEventRecord(bt->brev[k], bt->br[k]);
        cudaStreamWaitEvent(bt->ctx->stream, bt->brev[k], 0);
    }
}

int batch_enqueue(iarray_b200_batch_t *bt, int parts)
{
    cudaStream_t st = bt->ctx->stream;
    const size_t nbr = bt->br.size();
    if (parts & 1) {
        const int r = iab::decode_group_launch(&bt->dgrp, st);
        if (r) return r;
    }
    if (!(parts & 2)) {
    } else if (bt->form == IARRAY_B200_FORM_SPLIT) {
        const int r = iab::gemm_f64_ozaki_grouped_launch(&bt->ozg, st);
        if (r) return r;
    } else if (bt->total_tiles > 0) {
        iab::gemm_f64_grouped(bt->cfg, bt->probs.as<iab::GemmProblem>(), (int)bt->hprobs.size(), bt->total_tiles,
                              bt->ctas, st);
    }
    if (!(parts & 4)) return 0;
    const bool exact = bt->ctx->encoder == IARRAY_B200_ENCODER_LIBLZ4;
    if (bt->egroup) return iab::encode_group_launch(&bt->egrp, exact, bt->ctx->cfg.compression_level == 0, st);
    batch_fork(bt);
    for (int64_t i = 0; i < bt->n; i++) {
        const Geom &g = bt->cgeom[(size_t)i];
        if (!g.nchunks) continue;
        bt->enc[(size_t)i].ext_chunks = bt->chunks.as<iab::EncChunk>() + bt->chunk_base[(size_t)i];
        bt->enc[(size_t)i].exact_lz4 = exact;
        bt->enc[(size_t)i].memcpy_only = bt->ctx->cfg.compression_level == 0;
        const int r = iab::encode_launch(g, bt->dC[(size_t)i].p, bt->ldc[(size_t)i], true, IARRAY_AUTO_SPLIT,
                                         &bt->cbuf[(size_t)i], &bt->enc[(size_t)i], bt->br[(size_t)i % nbr]);
        if (r) { batch_join(bt); return r; }
    }
    batch_join(bt);
    return 0;
}

ina_rc_t batch_rc(int r)
{
    if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    return rc_err(IARRAY_ERR_GPU_FAILED);
}

// Reads the decode status words: a failed decode is a codec failure.
ina_rc_t batch_status(iarray_b200_batch_t *bt)
{
    std::vector<int> h((size_t)(bt->n * 32));
    if (cudaMemcpy(h.data(), bt->status.p, h.size() * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return rc_err(IARRAY_ERR_GPU_FAILED);
    for (int64_t i = 0; i < 2 * bt->n; i++)
        if (h[(size_t)(i * 16 + 1)]) return status_rc(h[(size_t)(i * 16 + 1)]);
    if (bt->form == IARRAY_B200_FORM_SPLIT && iab::gemm_f64_ozaki_grouped_finish(&bt->ozg, bt->ctx->stream))
        return rc_err(IARRAY_ERR_GPU_FAILED);
    return INA_SUCCESS;
}
}  // namespace

// Split form: the number of moduli.  With the context's count fixed
// (iarray_b200_set_split_terms), that count; else an error-checked autotuner on the batch's
// own decoded operands: the products with 16 moduli (about 2^-59 relative per scaled operand:
// exact against float64 rounding) serve as the reference, the native grouped FP64 product's
// normwise error against it sets the bar, and of 15, 14, 13 and 12 moduli the fastest whose
// error stays within 4x the native error is kept (16 when none is).  The choice is cached per
// set of shapes.  The grouped pipeline's buffers and tables are then written for the chosen
// count, before any capture.
static ina_rc_t batch_tune_split(iarray_b200_batch_t *bt)
{
    iarray_context_t *ctx = bt->ctx;
    const size_t un = (size_t)bt->n;
    auto items_into = [&](std::vector<DevBuf> *out) {
        std::vector<iab::OzGroupItem> items(un);
        for (size_t i = 0; i < un; i++)
            items[i] = iab::OzGroupItem{bt->M[i], bt->N[i], bt->K[i], bt->dA[i].as<double>(), bt->dB[i].as<double>(),
                                        out ? (*out)[i].as<double>() : bt->dC[i].as<double>(), bt->lda[i], bt->ldb[i],
                                        bt->ldc[i]};
        return items;
    };
    int L = ctx->split_terms;
    std::string sig = "split";
    for (size_t i = 0; i < un; i++)
        sig += ";" + std::to_string(bt->M[i]) + "x" + std::to_string(bt->N[i]) + "x" + std::to_string(bt->K[i]);
    if (L <= 0) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(sig);
        if (it != g_tune_cache.end()) L = it->second;
    }
    if (L <= 0) {
        // decode every operand once (also sets up the codec kernels)
        int r = batch_enqueue(bt, 1);
        if (r) return batch_rc(r);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
        ina_rc_t rc = batch_status(bt);
        if (INA_FAILED(rc)) return rc;
        std::vector<DevBuf> cref(un), cnat(un);
        for (size_t i = 0; i < un; i++)
            if (!cref[i].allocate(bt->dC[i].n, ctx->device) || !cnat[i].allocate(bt->dC[i].n, ctx->device))
                return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        auto diff_vs_ref = [&](const std::vector<DevBuf> &x) {
            std::vector<iab::DiffItem> d(un);
            for (size_t i = 0; i < un; i++)
                d[i] = iab::DiffItem{x[i].as<double>(), cref[i].as<double>(), bt->M[i], bt->N[i], bt->ldc[i]};
            return iab::normwise_diff_grouped(d, ctx->stream);
        };
        {   // reference: 16 moduli
            iab::OzGroupWork w;
            r = iab::gemm_f64_ozaki_grouped_setup(items_into(&cref), 16, &w, ctx->stream);
            if (!r) r = iab::gemm_f64_ozaki_grouped_launch(&w, ctx->stream);
            if (!r) r = iab::gemm_f64_ozaki_grouped_finish(&w, ctx->stream);
            if (r) return rc_err(r == -100 ? IARRAY_ERR_GPU_OUT_OF_MEMORY : IARRAY_ERR_GPU_FAILED);
        }
        {   // the native grouped FP64 product sets the bar
            std::vector<iab::GemmProblem> hp;
            int total = 0;
            batch_problems(bt, 0, &hp, &total);
            std::vector<iab::GemmProblem> hn = hp;
            for (auto &q : hn)
                for (size_t i = 0; i < un; i++)
                    if (q.C == bt->dC[i].as<double>()) q.C = cnat[i].as<double>();
            DevBuf dp;
            if (!dp.allocate(std::max<size_t>(hn.size(), 1) * sizeof(iab::GemmProblem), ctx->device))
                return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
            cudaMemcpyAsync(dp.p, hn.data(), hn.size() * sizeof(iab::GemmProblem), cudaMemcpyHostToDevice, ctx->stream);
            if (total > 0)
                iab::gemm_f64_grouped(0, dp.as<iab::GemmProblem>(), (int)hn.size(), total, iab::gemm_f64_grouped_ctas(0),
                                      ctx->stream);
            bt->split_err_native = diff_vs_ref(cnat);
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        double best = -1.0;
        L = 16;
        for (int cand = 16; cand >= 12; cand--) {
            iab::OzGroupWork w;
            r = iab::gemm_f64_ozaki_grouped_setup(items_into(nullptr), cand, &w, ctx->stream);
            if (r) break;
            iab::gemm_f64_ozaki_grouped_launch(&w, ctx->stream);               // warm-up
            cudaEventRecord(e0, ctx->stream);
            for (int rep = 0; rep < 2; rep++) iab::gemm_f64_ozaki_grouped_launch(&w, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            if (iab::gemm_f64_ozaki_grouped_finish(&w, ctx->stream)) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double err = diff_vs_ref(bt->dC);
            bt->split_tune_ms[16 - cand] = ms / 2;
            bt->split_tune_err[16 - cand] = err;
            const bool within = err >= 0.0 && err <= 4.0 * bt->split_err_native;
            if (within && (best < 0.0 || ms / 2 < best)) { best = ms / 2; L = cand; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (cudaGetLastError() != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[sig] = L;
    }
    bt->split_terms = L;
    // the graph's reconstruction writes the outputs' encoder images straight away (no dense C,
    // no gather) when the outputs are encoded as one group and every one can take it
    std::vector<iab::OzGroupItem> items = items_into(nullptr);
    bool img = bt->egroup && ctx->cfg.compression_level != 0;
    for (size_t i = 0; i < un && img; i++)
        img = bt->M[i] > 0 && bt->N[i] > 0 && bt->K[i] > 0 && iab::encode_image_ok(bt->cgeom[i], true, false);
    if (img)
        for (size_t i = 0; i < un; i++) {
            items[i].cimg = bt->egrp.h[i].img;
            items[i].gc = bt->cgeom[i];
        }
    const int r = iab::gemm_f64_ozaki_grouped_setup(items, L, &bt->ozg, ctx->stream);
    if (r == -100) return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    if (r) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    bt->egrp.img_ready = img;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_batch_new(iarray_context_t *ctx, int64_t n, iarray_container_t *const *a,
                                        iarray_container_t *const *b, const iarray_storage_t *storage,
                                        iarray_b200_batch_t **batch)
{
    CHECK_ARG(ctx && a && b && storage && batch && n > 0);
    for (int64_t i = 0; i < n; i++) {
        CHECK_ARG(a[i] && b[i]);
        if (a[i]->dtshape.dtype != IARRAY_DATA_TYPE_DOUBLE || b[i]->dtshape.dtype != IARRAY_DATA_TYPE_DOUBLE)
            return rc_err(IARRAY_ERR_INVALID_DTYPE);
        if (a[i]->dtshape.ndim != 2 || b[i]->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
        if (a[i]->dtshape.shape[1] != b[i]->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
        if (a[i]->transposed || b[i]->transposed) return rc_err(IARRAY_ERR_NOT_SUPPORTED);
    }
    std::unique_ptr<iarray_b200_batch_s> bt(new iarray_b200_batch_s());
    bt->ctx = ctx;
    {
        const int nbr = (int)std::min<int64_t>(n, 16);
        bt->br.resize((size_t)nbr);
        bt->brev.resize((size_t)nbr);
        for (int k = 0; k < nbr; k++) {
            if (cudaStreamCreateWithFlags(&bt->br[(size_t)k], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&bt->brev[(size_t)k], cudaEventDisableTiming) != cudaSuccess)
                return rc_err(IARRAY_ERR_GPU_FAILED);
        }
        if (cudaEventCreateWithFlags(&bt->fork, cudaEventDisableTiming) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    bt->form = ctx->form;
    bt->n = n;
    const size_t un = (size_t)n;
    bt->a.assign(a, a + n);
    bt->b.assign(b, b + n);
    bt->storage.assign(storage, storage + n);
    bt->cgeom.resize(un);
    bt->M.resize(un); bt->N.resize(un); bt->K.resize(un); bt->lda.resize(un); bt->ldb.resize(un); bt->ldc.resize(un);
    bt->dA.resize(un); bt->dB.resize(un); bt->dC.resize(un); bt->cbuf.resize(un);
    bt->enc.resize(un);
    bt->chunk_base.resize(un);
    int64_t nch = 0;
    for (size_t i = 0; i < un; i++) {
        const int64_t M = a[i]->dtshape.shape[0], K = a[i]->dtshape.shape[1], N = b[i]->dtshape.shape[1];
        bt->M[i] = M; bt->N[i] = N; bt->K[i] = K;
        bt->lda[i] = pad_ld(K); bt->ldb[i] = pad_ld(N); bt->ldc[i] = pad_ld(N);
        const int64_t shape[2] = {M, N};
        if (!iab::make_geom(2, shape, storage[i].chunkshape, storage[i].blockshape, 8, &bt->cgeom[i]))
            return rc_err(IARRAY_ERR_INVALID_STORAGE);
        if (!bt->dA[i].allocate((size_t)std::max<int64_t>(M * bt->lda[i] * 8, 16), ctx->device) ||
            !bt->dB[i].allocate((size_t)std::max<int64_t>(K * bt->ldb[i] * 8, 16), ctx->device) ||
            !bt->dC[i].allocate((size_t)std::max<int64_t>(M * bt->ldc[i] * 8, 16), ctx->device))
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        bt->chunk_base[i] = nch;
        nch += bt->cgeom[i].nchunks;
    }
    if (!bt->status.allocate((size_t)(n * 32 * sizeof(int)), ctx->device) ||
        !bt->chunks.allocate((size_t)std::max<int64_t>(nch, 1) * sizeof(iab::EncChunk), ctx->device))
        return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
    {   // the grouped decode of every operand and, when the outputs share a stream shape, encode
        std::vector<iab::DecodeArgs> da;
        std::vector<int *> dc;
        for (size_t i = 0; i < un; i++)
            for (int k = 0; k < 2; k++) {
                const iarray_container_t *x = k ? b[i] : a[i];
                da.push_back(iab::DecodeArgs{x->geom, x->store->buf.as<uint8_t>(), (int64_t)x->store->buf.n,
                                             x->store->d_off.as<int64_t>(), x->store->d_len.as<int32_t>(),
                                             (k ? bt->dB : bt->dA)[i].p, k ? bt->ldb[i] : bt->lda[i]});
                dc.push_back(bt->status.as<int>() + (2 * i + k) * 16);
            }
        int r = iab::decode_group_setup(da, dc, &bt->dgrp, ctx->stream);
        if (r) return r == -100 ? rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY) : rc_err(IARRAY_ERR_GPU_FAILED);
        std::vector<const void *> dense(un);
        std::vector<iab::EncChunk *> ec(un);
        for (size_t i = 0; i < un; i++) {
            dense[i] = bt->dC[i].p;
            ec[i] = bt->chunks.as<iab::EncChunk>() + bt->chunk_base[i];
        }
        r = iab::encode_group_setup(bt->cgeom, dense, bt->ldc, ec, &bt->cbuf, &bt->egrp, ctx->stream);
        if (r < 0) return r == -100 ? rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY) : rc_err(IARRAY_ERR_GPU_FAILED);
        bt->egroup = r == 0;
    }
    if (bt->form == IARRAY_B200_FORM_SPLIT) {
        ina_rc_t rc = batch_tune_split(bt.get());
        if (INA_FAILED(rc)) return rc;
    }
    cudaMemsetAsync(bt->status.p, 0, bt->status.n, ctx->stream);
    // autotuner (native form): time every tile configuration of the grouped kernel on the
    // decoded operands of this batch; the choice is cached per problem-set signature
    std::string sig;
    for (size_t i = 0; i < un; i++)
        sig += std::to_string(bt->M[i]) + "x" + std::to_string(bt->N[i]) + "x" + std::to_string(bt->K[i]) + ";";
    bt->cfg = 0;
    if (bt->form != IARRAY_B200_FORM_SPLIT) {
        bool cached = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune_cache.find(sig);
            if (it != g_tune_cache.end()) { bt->cfg = it->second; cached = true; }
        }
        // first eager pass: decode every operand (also sets up the codec kernels)
        {
            const int r = batch_enqueue(bt.get(), 1);
            if (r) return batch_rc(r);
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
            ina_rc_t rc = batch_status(bt.get());
            if (INA_FAILED(rc)) return rc;
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int cfg = 0; cfg < iab::GEMM_F64_GROUPED_CONFIGS && !cached; cfg++) {
            std::vector<iab::GemmProblem> hp;
            int total = 0;
            batch_problems(bt.get(), cfg, &hp, &total);
            DevBuf dp;
            if (!dp.allocate(std::max<size_t>(hp.size(), 1) * sizeof(iab::GemmProblem), ctx->device)) break;
            cudaMemcpyAsync(dp.p, hp.data(), hp.size() * sizeof(iab::GemmProblem), cudaMemcpyHostToDevice, ctx->stream);
            const int ctas = iab::gemm_f64_grouped_ctas(cfg);
            iab::gemm_f64_grouped(cfg, dp.as<iab::GemmProblem>(), (int)hp.size(), total, ctas, ctx->stream);
            cudaEventRecord(e0, ctx->stream);
            for (int rep = 0; rep < 2; rep++)
                iab::gemm_f64_grouped(cfg, dp.as<iab::GemmProblem>(), (int)hp.size(), total, ctas, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            bt->tune_ms[cfg] = ms / 2;
            if (bt->tune_ms[bt->cfg] < 0 || bt->tune_ms[cfg] < bt->tune_ms[bt->cfg]) bt->cfg = cfg;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (cudaGetLastError() != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
        if (!cached) {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune_cache[sig] = bt->cfg;
        }
        batch_problems(bt.get(), bt->cfg, &bt->hprobs, &bt->total_tiles);
        bt->ctas = iab::gemm_f64_grouped_ctas(bt->cfg);
        if (!bt->probs.allocate(std::max<size_t>(bt->hprobs.size(), 1) * sizeof(iab::GemmProblem), ctx->device))
            return rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
        cudaMemcpyAsync(bt->probs.p, bt->hprobs.data(), bt->hprobs.size() * sizeof(iab::GemmProblem),
                        cudaMemcpyHostToDevice, ctx->stream);
    }
    // one complete eager pass, then the capture (every buffer above is owned by the batch,
    // so the graph's pointers stay valid until iarray_b200_batch_free)
    {
        const int r = batch_enqueue(bt.get(), 7);
        if (r) return batch_rc(r);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
        ina_rc_t rc = batch_status(bt.get());
        if (INA_FAILED(rc)) return rc;
    }
    // kernel profiling records events around launches: keep it out of the capture
    const bool prof = iab::kprof_enable(false);
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        iab::kprof_enable(prof);
        return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    const int r = batch_enqueue(bt.get(), 7);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    iab::kprof_enable(prof);
    if (r || ce != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return r ? batch_rc(r) : rc_err(IARRAY_ERR_GPU_FAILED);
    }
    bt->graph = graph;
    if (cudaGraphInstantiate(&bt->exec, graph, 0) != cudaSuccess) {
        cudaGetLastError();
        return rc_err(IARRAY_ERR_GPU_FAILED);
    }
    size_t nodes = 0;
    cudaGraphGetNodes(graph, nullptr, &nodes);
    bt->nodes = (int64_t)nodes;
    *batch = bt.release();
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_batch_run(iarray_b200_batch_t *bt, iarray_container_t **c)
{
    CHECK_ARG(bt && c);
    iarray_context_t *ctx = bt->ctx;
    const size_t un = (size_t)bt->n;
    for (size_t i = 0; i < un; i++) c[i] = nullptr;
    cudaEventRecord(ctx->ev[0], ctx->stream);
    if (cudaGraphLaunch(bt->exec, ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
    cudaEventRecord(ctx->ev[4], ctx->stream);
    int64_t nch = bt->chunk_base.empty() ? 0 : bt->chunk_base.back() + bt->cgeom.back().nchunks;
    std::vector<iab::EncChunk> hc((size_t)std::max<int64_t>(nch, 1));
    cudaMemcpyAsync(hc.data(), bt->chunks.p, (size_t)nch * sizeof(iab::EncChunk), cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return rc_err(IARRAY_ERR_GPU_FAILED);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[4]);
    for (int k = 0; k < 4; k++) ctx->timings[k] = 0;
    ctx->timings[2] = ms;
    ctx->timings[4] = ms;
    ina_rc_t rc = batch_status(bt);
    if (INA_FAILED(rc)) return rc;
    for (size_t i = 0; i < un && INA_SUCCEED(rc); i++) {
        iarray_dtshape_t d;
        memset(&d, 0, sizeof(d));
        d.dtype = IARRAY_DATA_TYPE_DOUBLE;
        d.ndim = 2;
        d.shape[0] = bt->M[i];
        d.shape[1] = bt->N[i];
        iarray_storage_t st = bt->storage[i];
        rc = new_container(ctx, &d, &st, &c[i]);
        if (INA_FAILED(rc)) break;
        iarray_container_t *ci = c[i];
        if (!ci->geom.nchunks) { rc = fill_zero_chunks(ci); continue; }
        ChunkStore &s = *ci->store;
        const int64_t n = ci->geom.nchunks, base = bt->chunk_base[i];
        s.off.resize((size_t)n);
        s.len.resize((size_t)n);
        int64_t total = 0;
        for (int64_t k = 0; k < n; k++) {
            s.off[(size_t)k] = hc[(size_t)(base + k)].offset;
            s.len[(size_t)k] = hc[(size_t)(base + k)].cbytes;
            total = std::max<int64_t>(total, s.off[(size_t)k] + s.len[(size_t)k]);
        }
        if (!s.buf.allocate((size_t)std::max<int64_t>(total, 1), ctx->device) ||
            !s.d_off.allocate((size_t)n * 8, ctx->device) || !s.d_len.allocate((size_t)n * 4, ctx->device)) {
            rc = rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY);
            break;
        }
        cudaMemcpyAsync(s.buf.p, bt->cbuf[i].p, (size_t)total, cudaMemcpyDeviceToDevice, ctx->stream);
        cudaMemcpyAsync(s.d_off.p, s.off.data(), (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(s.d_len.p, s.len.data(), (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream);
        s.cbytes = 0;
        for (int32_t l : s.len) s.cbytes += l;
    }
    if (INA_SUCCEED(rc) && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = rc_err(IARRAY_ERR_GPU_FAILED);
    if (INA_FAILED(rc))
        for (size_t i = 0; i < un; i++)
            if (c[i]) iarray_container_free(ctx, &c[i]);
    return rc;
}

INA_API(ina_rc_t) iarray_b200_batch_info(iarray_b200_batch_t *bt, int *tile_config, double *tune_ms,
                                         int64_t *graph_nodes)
{
    CHECK_ARG(bt);
    if (tile_config) *tile_config = bt->form == IARRAY_B200_FORM_SPLIT ? -1 : bt->cfg;
    if (tune_ms)
        for (int k = 0; k < iab::GEMM_F64_GROUPED_CONFIGS; k++) tune_ms[k] = bt->tune_ms[k];
    if (graph_nodes) *graph_nodes = bt->nodes;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_b200_batch_split_tuning(iarray_b200_batch_t *bt, int *nterms, double *err_native,
                                                 double *tune_ms, double *tune_err)
{
    CHECK_ARG(bt);
    if (bt->form != IARRAY_B200_FORM_SPLIT) return rc_err(INA_ERR_INVALID_ARGUMENT);
    if (nterms) *nterms = bt->split_terms;
    if (err_native) *err_native = bt->split_err_native;
    for (int i = 0; i < 5; i++) {
        if (tune_ms) tune_ms[i] = bt->split_tune_ms[i];
        if (tune_err) tune_err[i] = bt->split_tune_err[i];
    }
    return INA_SUCCESS;
}

INA_API(void) iarray_b200_batch_free(iarray_b200_batch_t **batch)
{
    if (!batch || !*batch) return;
    iarray_b200_batch_t *bt = *batch;
    // the context may already be gone: wait on the device, not on the context's stream
    cudaDeviceSynchronize();
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    delete bt;
    *batch = nullptr;
}

// ============================================================================ expressions
// iarray_expr_* / iarray_eval (include/libiarray/iarray.h:830-846, src/iarray_expression.c):
// element-wise expressions over containers of one shape, evaluated on the GPU (expr.cu).  The
// operands are decoded into dense device arrays, one kernel runs the compiled program for
// every element, and the result is encoded into the output partition.  B200 addition:
// iarray_b200_expr_bind_matmul binds a variable to the product A * B, computed on the GPU in
// the context's form and consumed by the expression in device memory (the product is never
// encoded): the expression acts as the product's epilogue.
struct iarray_expression_s {
    iarray_context_t *ctx = nullptr;
    int dtype = IARRAY_DATA_TYPE_DOUBLE;
    std::vector<std::string> names;
    std::vector<iarray_container_t *> conts;                                  // nullptr for a product
    std::vector<std::pair<iarray_container_t *, iarray_container_t *>> prods;  // {a, b} of a product operand
    std::vector<std::pair<std::string, double>> scalars;
    bool out_set = false, compiled = false;
    iarray_dtshape_t out_dtshape;
    iarray_storage_t out_storage;
    std::string out_urlpath;
    std::vector<iab::ExprOp> prog;
};

INA_API(ina_rc_t) iarray_expr_new(iarray_context_t *ctx, iarray_data_type_t dtype, iarray_expression_t **e)
{
    CHECK_ARG(ctx && e);
    if (dtype != IARRAY_DATA_TYPE_DOUBLE && dtype != IARRAY_DATA_TYPE_FLOAT) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    *e = new iarray_expression_t();
    (*e)->ctx = ctx;
    (*e)->dtype = dtype;
    return INA_SUCCESS;
}

INA_API(void) iarray_expr_free(iarray_context_t *ctx, iarray_expression_t **e)
{
    (void)ctx;
    if (!e || !*e) return;
    delete *e;
    *e = nullptr;
}

static ina_rc_t expr_add_operand(iarray_expression_t *e, const char *var, iarray_container_t *c, iarray_container_t *a,
                                 iarray_container_t *b)
{
    CHECK_ARG(e && var && var[0]);
    if ((int)e->names.size() >= iab::EXPR_MAX_OPERANDS) return rc_err(INA_ERR_FULL);
    for (const std::string &n : e->names)
        if (n == var) return rc_err(INA_ERR_INVALID_ARGUMENT);
    e->names.push_back(var);
    e->conts.push_back(c);
    e->prods.emplace_back(a, b);
    e->compiled = false;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_expr_bind(iarray_expression_t *e, const char *var, iarray_container_t *val)
{
    CHECK_ARG(e && val);
    if (val->dtshape.dtype != e->dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    return expr_add_operand(e, var, val, nullptr, nullptr);
}

INA_API(ina_rc_t) iarray_b200_expr_bind_matmul(iarray_expression_t *e, const char *var, iarray_container_t *a,
                                               iarray_container_t *b)
{
    CHECK_ARG(e && a && b);
    if (a->dtshape.dtype != e->dtype || b->dtshape.dtype != e->dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    if (a->dtshape.ndim != 2 || b->dtshape.ndim != 2) return rc_err(IARRAY_ERR_INVALID_NDIM);
    if (a->dtshape.shape[1] != b->dtshape.shape[0]) return rc_err(IARRAY_ERR_INVALID_SHAPE);
    return expr_add_operand(e, var, nullptr, a, b);
}

INA_API(ina_rc_t) iarray_expr_bind_out_properties(iarray_expression_t *e, iarray_dtshape_t *dtshape,
                                                  iarray_storage_t *store)
{
    CHECK_ARG(e && dtshape && store);
    e->out_dtshape = *dtshape;
    e->out_storage = *store;
    e->out_urlpath = store->urlpath ? store->urlpath : "";
    e->out_storage.urlpath = nullptr;
    e->out_set = true;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_expr_bind_param(iarray_expression_t *e, iarray_user_param_t val)
{
    (void)e;
    (void)val;
    return rc_err(IARRAY_ERR_NOT_SUPPORTED);        // parameters of user-defined functions (LLVM bitcode)
}

static ina_rc_t expr_add_scalar(iarray_expression_t *e, const char *var, double val)
{
    CHECK_ARG(e && var && var[0]);
    for (auto &sc : e->scalars)
        if (sc.first == var) { sc.second = val; e->compiled = false; return INA_SUCCESS; }
    e->scalars.emplace_back(var, val);
    e->compiled = false;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_expr_bind_scalar_float(iarray_expression_t *e, const char *var, float val)
{
    return expr_add_scalar(e, var, (double)val);
}

INA_API(ina_rc_t) iarray_expr_bind_scalar_double(iarray_expression_t *e, const char *var, double val)
{
    return expr_add_scalar(e, var, val);
}

INA_API(ina_rc_t) iarray_expr_compile(iarray_expression_t *e, const char *expr)
{
    CHECK_ARG(e && expr);
    std::string why;
    if (!iab::expr_compile(expr, e->names, e->scalars, &e->prog, &why)) {
        e->compiled = false;
        return rc_err(INA_ERR_INVALID_ARGUMENT);
    }
    e->compiled = true;
    return INA_SUCCESS;
}

INA_API(ina_rc_t) iarray_expr_compile_udf(iarray_expression_t *e, int llvm_bc_len, const char *llvm_bc,
                                          const char *name)
{
    (void)e; (void)llvm_bc_len; (void)llvm_bc; (void)name;
    return rc_err(IARRAY_ERR_NOT_SUPPORTED);        // user-defined functions come as LLVM bitcode
}

INA_API(ina_rc_t) iarray_eval(iarray_expression_t *e, iarray_container_t **container)
{
    CHECK_ARG(e && container);
    if (!e->compiled || !e->out_set) return rc_err(INA_ERR_NOT_COMPLETE);
    iarray_context_t *ctx = e->ctx;
    iarray_dtshape_t od = e->out_dtshape;
    if (od.dtype != e->dtype) return rc_err(IARRAY_ERR_INVALID_DTYPE);
    iarray_storage_t os = e->out_storage;
    os.urlpath = e->out_urlpath.empty() ? nullptr : (char *)e->out_urlpath.c_str();
    iarray_container_t *out = nullptr;
    ina_rc_t rc = new_container(ctx, &od, &os, &out);
    if (INA_FAILED(rc)) return rc;
    const int64_t rows = rows_of(out->dtshape), cols = cols_of(out->dtshape), ld = pad_ld(cols);
    const int isz = out->geom.itemsize;
    auto fail = [&](ina_rc_t r) { iarray_container_free(ctx, &out); return r; };
    // operands: shapes, then dense device copies
    for (size_t k = 0; k < e->names.size(); k++) {
        if (e->conts[k]) {
            const iarray_dtshape_t &d = e->conts[k]->dtshape;
            if (d.ndim != od.ndim) return fail(rc_err(IARRAY_ERR_INVALID_NDIM));
            for (int i = 0; i < od.ndim; i++)
                if (d.shape[i] != od.shape[i]) return fail(rc_err(IARRAY_ERR_INVALID_SHAPE));
        } else if (od.ndim != 2 || e->prods[k].first->dtshape.shape[0] != od.shape[0] ||
                   e->prods[k].second->dtshape.shape[1] != od.shape[1]) {
            return fail(rc_err(IARRAY_ERR_INVALID_SHAPE));
        }
    }
    std::vector<DevBuf> dense(e->names.size());
    iab::ExprArgs args;
    memset(&args, 0, sizeof(args));
    for (size_t k = 0; k < e->names.size(); k++) {
        if (!dense[k].allocate((size_t)std::max<int64_t>(rows * ld * isz, 16), ctx->device))
            return fail(rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY));
        if (e->conts[k]) {
            rc = decode_logical(ctx, e->conts[k], dense[k].p, ld);
        } else {
            iarray_container_t *a = e->prods[k].first, *b = e->prods[k].second;
            const int64_t K = a->dtshape.shape[1], lda = pad_ld(K);
            DevBuf dA, dB;
            if (!dA.allocate((size_t)std::max<int64_t>(rows * lda * isz, 16), ctx->device) ||
                !dB.allocate((size_t)std::max<int64_t>(K * ld * isz, 16), ctx->device))
                return fail(rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY));
            rc = decode_logical(ctx, a, dA.p, lda);
            if (INA_SUCCEED(rc)) rc = decode_logical(ctx, b, dB.p, ld);
            if (INA_SUCCEED(rc)) {
                if (K == 0) cudaMemsetAsync(dense[k].p, 0, (size_t)(rows * ld * isz), ctx->stream);
                else rc = dense_product(ctx, e->dtype, rows, cols, K, dA.p, lda, dB.p, ld, dense[k].p, ld);
            }
            if (INA_SUCCEED(rc)) rc = cuda_rc(cudaStreamSynchronize(ctx->stream));   // dA, dB go back to the pool idle
        }
        if (INA_FAILED(rc)) return fail(rc);
        args.in[k] = dense[k].p;
        args.ld[k] = ld;
    }
    args.nops = (int)e->prog.size();
    for (int i = 0; i < args.nops; i++) args.ops[i] = e->prog[(size_t)i];
    DevBuf res;
    if (!res.allocate((size_t)std::max<int64_t>(rows * ld * isz, 16), ctx->device))
        return fail(rc_err(IARRAY_ERR_GPU_OUT_OF_MEMORY));
    iab::expr_eval(isz, rows, cols, args, res.p, ld, ctx->stream);
    rc = cuda_rc(cudaGetLastError());
    if (INA_FAILED(rc)) return fail(rc);
    rc = out->geom.nchunks ? encode_into(ctx, out, res.p, ld) : fill_zero_chunks(out);
    if (INA_SUCCEED(rc)) rc = save_if_urlpath(ctx, out);
    if (INA_FAILED(rc)) return fail(rc);
    *container = out;
    return INA_SUCCESS;
}
