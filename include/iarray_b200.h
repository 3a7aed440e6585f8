/*
 * iarray_b200.h — C ABI of the B200-native blocked matrix product over
 * Blosc2-compressed chunked containers.
 *
 * The entry points, types and argument meanings follow ironArray's public header
 * include/libiarray/iarray.h so that C code written against the reference for the
 * matmul path compiles and links unchanged against libiarray_b200.so.  Every
 * declaration names the reference interface it replaces (file:line in the
 * reference project).  Containers live in GPU memory as Blosc2 LZ4+SHUFFLE chunks
 * laid out exactly like Caterva's (chunkshape / blockshape, zero padding, blocks
 * row-major inside a chunk); decode, products and re-encode run as CUDA kernels
 * on one B200.  There is no CPU fallback: on a machine without a usable GPU every
 * compute entry point returns IARRAY_ERR_GPU_FAILED.
 *
 * Return codes follow libinac's 64-bit RC layout (doc/inac/error.md in the
 * reference): bit 63 = error flag, bits 16..23 = adjective/verb code, bit 15 =
 * negate flag, bits 0..14 = subject.  The subject numbers (IARRAY_ES_*) are the
 * reference's; the adjective/verb numbers behind INA_ERR_* are this library's own,
 * because libinac, which defines them, is not part of the reference's sources.
 * Compare return codes with the IARRAY_ERR_* / INA_ERR_* macros of this header, not
 * with raw numbers taken from a libinac build.
 */
#ifndef IARRAY_B200_H
#define IARRAY_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define INA_API(x) __attribute__((visibility("default"))) x
#else
#define INA_API(x) x
#endif

/* ---------------------------------------------------------------- return codes */
typedef uint64_t ina_rc_t;

#define INA_SUCCESS ((ina_rc_t)0)
#define INA_RC_ERROR_BIT (1ULL << 63)
#define INA_FAILED(rc) ((((ina_rc_t)(rc)) & INA_RC_ERROR_BIT) != 0)
#define INA_SUCCEED(rc) (!INA_FAILED(rc))
/* error message (code | negate | subject) of an RC, comparable with IARRAY_ERR_* */
#define INA_RC_MSG(rc) ((uint32_t)((rc) & 0xFFFFFFu))

#define INA_ERR_CODE(c) ((uint32_t)(c) << 16)
#define INA_ERR_NEGATE (1u << 15)
#define INA_ERR_INVALID INA_ERR_CODE(1)
#define INA_ERR_FAILED INA_ERR_CODE(2)
#define INA_ERR_EMPTY INA_ERR_CODE(3)
#define INA_ERR_FULL INA_ERR_CODE(4)
#define INA_ERR_TOO_SMALL INA_ERR_CODE(5)
#define INA_ERR_OUT_OF_RANGE INA_ERR_CODE(6)
#define INA_ERR_COMPILED INA_ERR_CODE(7)
#define INA_ERR_COMPLETE INA_ERR_CODE(8)
#define INA_ERR_NOT_COMPLETE (INA_ERR_CODE(8) | INA_ERR_NEGATE)
#define INA_ERR_OUT_OF_MEMORY INA_ERR_CODE(9)
#define INA_ERR_NOT_SUPPORTED (INA_ERR_CODE(10) | INA_ERR_NEGATE)
#define INA_ERR_INVALID_ARGUMENT (INA_ERR_INVALID | 1u)
#define INA_ERR_NOT_INITIALIZED (INA_ERR_CODE(11) | INA_ERR_NEGATE)
#define INA_ERR_NOT_FOUND (INA_ERR_CODE(12) | INA_ERR_NEGATE)

#define INA_ES_USER_DEFINED 1024u
/* subjects: include/libiarray/iarray.h:28-50 */
#define IARRAY_ES_CONTAINER (INA_ES_USER_DEFINED + 1)
#define IARRAY_ES_DTSHAPE (INA_ES_USER_DEFINED + 2)
#define IARRAY_ES_SHAPE (INA_ES_USER_DEFINED + 3)
#define IARRAY_ES_CHUNKSHAPE (INA_ES_USER_DEFINED + 4)
#define IARRAY_ES_NDIM (INA_ES_USER_DEFINED + 5)
#define IARRAY_ES_DTYPE (INA_ES_USER_DEFINED + 6)
#define IARRAY_ES_STORAGE (INA_ES_USER_DEFINED + 7)
#define IARRAY_ES_PERSISTENCY (INA_ES_USER_DEFINED + 8)
#define IARRAY_ES_BUFFER (INA_ES_USER_DEFINED + 9)
#define IARRAY_ES_CATERVA (INA_ES_USER_DEFINED + 10)
#define IARRAY_ES_BLOSC (INA_ES_USER_DEFINED + 11)
#define IARRAY_ES_ASSERTION (INA_ES_USER_DEFINED + 12)
#define IARRAY_ES_BLOCKSHAPE (INA_ES_USER_DEFINED + 13)
#define IARRAY_ES_GPU (INA_ES_USER_DEFINED + 100) /* B200 build: CUDA runtime failures */

/* messages: include/libiarray/iarray.h:53-90 */
#define IARRAY_ERR_EMPTY_CONTAINER (INA_ERR_EMPTY | IARRAY_ES_CONTAINER)
#define IARRAY_ERR_INVALID_DTSHAPE (INA_ERR_INVALID | IARRAY_ES_DTSHAPE)
#define IARRAY_ERR_INVALID_DTYPE (INA_ERR_INVALID | IARRAY_ES_DTYPE)
#define IARRAY_ERR_INVALID_SHAPE (INA_ERR_INVALID | IARRAY_ES_SHAPE)
#define IARRAY_ERR_INVALID_CHUNKSHAPE (INA_ERR_INVALID | IARRAY_ES_CHUNKSHAPE)
#define IARRAY_ERR_INVALID_BLOCKSHAPE (INA_ERR_INVALID | IARRAY_ES_BLOCKSHAPE)
#define IARRAY_ERR_INVALID_NDIM (INA_ERR_INVALID | IARRAY_ES_NDIM)
#define IARRAY_ERR_INVALID_STORAGE (INA_ERR_INVALID | IARRAY_ES_STORAGE)
#define IARRAY_ERR_TOO_SMALL_BUFFER (INA_ERR_TOO_SMALL | IARRAY_ES_BUFFER)
#define IARRAY_ERR_CATERVA_FAILED (INA_ERR_FAILED | IARRAY_ES_CATERVA)
#define IARRAY_ERR_BLOSC_FAILED (INA_ERR_FAILED | IARRAY_ES_BLOSC)
#define IARRAY_ERR_ASSERTION_FAILED (INA_ERR_FAILED | IARRAY_ES_ASSERTION)
#define IARRAY_ERR_PERSISTENCY_FAILED (INA_ERR_FAILED | IARRAY_ES_PERSISTENCY)
#define IARRAY_ERR_GPU_FAILED (INA_ERR_FAILED | IARRAY_ES_GPU)
#define IARRAY_ERR_GPU_OUT_OF_MEMORY (INA_ERR_OUT_OF_MEMORY | IARRAY_ES_GPU)
#define IARRAY_ERR_NOT_SUPPORTED (INA_ERR_NOT_SUPPORTED | IARRAY_ES_CONTAINER)

/* ---------------------------------------------------------------- types */
#define IARRAY_DIMENSION_MAX 8 /* include/libiarray/iarray.h:20 */

typedef struct iarray_context_s iarray_context_t;     /* iarray.h:134 */
typedef struct iarray_container_s iarray_container_t; /* iarray.h:135 */

/* include/libiarray/iarray.h:152-168 */
typedef enum iarray_data_type_e {
    IARRAY_DATA_TYPE_DOUBLE = 0,
    IARRAY_DATA_TYPE_FLOAT = 1,
    IARRAY_DATA_TYPE_INT64 = 10,
    IARRAY_DATA_TYPE_INT32 = 11,
    IARRAY_DATA_TYPE_INT16 = 12,
    IARRAY_DATA_TYPE_INT8 = 13,
    IARRAY_DATA_TYPE_UINT64 = 16,
    IARRAY_DATA_TYPE_UINT32 = 17,
    IARRAY_DATA_TYPE_UINT16 = 18,
    IARRAY_DATA_TYPE_UINT8 = 19,
    IARRAY_DATA_TYPE_BOOL = 24,
    IARRAY_DATA_TYPE_MAX
} iarray_data_type_t;

/* include/libiarray/iarray.h:182-187 */
typedef enum iarray_filter_flags_e {
    IARRAY_COMP_SHUFFLE = 0x1,
    IARRAY_COMP_BITSHUFFLE = 0x2,
    IARRAY_COMP_DELTA = 0x4,
    IARRAY_COMP_TRUNC_PREC = 0x8,
} iarray_filter_flags_t;

/* include/libiarray/iarray.h:195-205 */
typedef enum iarray_compression_codec_e {
    IARRAY_COMPRESSION_BLOSCLZ = 0,
    IARRAY_COMPRESSION_LZ4,
    IARRAY_COMPRESSION_LZ4HC,
    IARRAY_COMPRESSION_SNAPPY,
    IARRAY_COMPRESSION_ZLIB,
    IARRAY_COMPRESSION_ZSTD,
    IARRAY_COMPRESSION_ZFP_FIXED_ACCURACY,
    IARRAY_COMPRESSION_ZFP_FIXED_PRECISION,
    IARRAY_COMPRESSION_ZFP_FIXED_RATE
} iarray_compression_codec_t;

typedef enum iarray_compression_favor_e {
    IARRAY_COMPRESSION_FAVOR_BALANCE = 0,
    IARRAY_COMPRESSION_FAVOR_SPEED,
    IARRAY_COMPRESSION_FAVOR_CRATIO,
} iarray_compression_favor_t;

/* include/libiarray/iarray.h:213-218 */
typedef enum iarray_split_mode_e {
    IARRAY_ALWAYS_SPLIT = 1,
    IARRAY_NEVER_SPLIT = 2,
    IARRAY_AUTO_SPLIT = 3,
    IARRAY_FORWARD_COMPAT_SPLIT = 4,
} iarray_split_mode_t;

typedef enum iarray_eval_method_e {
    IARRAY_EVAL_METHOD_AUTO = 0u,
    IARRAY_EVAL_METHOD_ITERCHUNK = 1u,
    IARRAY_EVAL_METHOD_ITERBLOSC = 2u,
} iarray_eval_method_t;

/* include/libiarray/iarray.h:214-226: same member order and types */
typedef struct iarray_config_s {
    iarray_compression_codec_t compression_codec;
    int compression_level;
    iarray_compression_favor_t compression_favor;
    int use_dict;
    int splitmode;
    int filter_flags;
    unsigned int eval_method;
    int max_num_threads;
    uint8_t fp_mantissa_bits;
    bool btune;
    uint8_t compression_meta;
} iarray_config_t;

/* include/libiarray/iarray.h:228-233 */
typedef struct iarray_dtshape_s {
    iarray_data_type_t dtype;
    int32_t dtype_size;
    int8_t ndim;
    int64_t shape[IARRAY_DIMENSION_MAX];
} iarray_dtshape_t;

/* include/libiarray/iarray.h:235-240 */
typedef struct iarray_storage_s {
    char *urlpath;
    bool contiguous;
    int64_t chunkshape[IARRAY_DIMENSION_MAX];
    int64_t blockshape[IARRAY_DIMENSION_MAX];
} iarray_storage_t;

/* include/libiarray/iarray.h:275-287.  btune is accepted and ignored: the GPU
 * encoder always writes the configured codec (the reference's parity runs disable
 * btune, examples/example_gemm.c:48). */
static const iarray_config_t IARRAY_CONFIG_DEFAULTS = {
    IARRAY_COMPRESSION_LZ4, 5, IARRAY_COMPRESSION_FAVOR_BALANCE, 0, IARRAY_AUTO_SPLIT,
    IARRAY_COMP_SHUFFLE, IARRAY_EVAL_METHOD_ITERBLOSC, 1, 0, true, 0};

/* ---------------------------------------------------------------- runtime */
/* iarray.h:337 (src/iarray.c:77-105).  Picks the current CUDA device. */
INA_API(ina_rc_t) iarray_init(void);
/* iarray.h:338 (src/iarray.c:108-120). */
INA_API(void) iarray_destroy(void);
/* iarray.h:340. */
INA_API(const char *) iarray_err_strerror(ina_rc_t error);
/* iarray.h:342 (src/iarray.c:361-380).  Unlike the reference, calling this before
 * iarray_init returns an error instead of exit(1). */
INA_API(ina_rc_t) iarray_context_new(iarray_config_t *cfg, iarray_context_t **ctx);
/* iarray.h:343. */
INA_API(void) iarray_context_free(iarray_context_t **ctx);

/* ---------------------------------------------------------------- containers */
/* iarray.h:451 (src/iarray_constructor.c:16-45): an all-zero container. */
INA_API(ina_rc_t) iarray_empty(iarray_context_t *ctx, iarray_dtshape_t *dtshape,
                               iarray_storage_t *storage, iarray_container_t **container);
/* iarray.h:456. */
INA_API(ina_rc_t) iarray_zeros(iarray_context_t *ctx, iarray_dtshape_t *dtshape,
                               iarray_storage_t *storage, iarray_container_t **container);
/* iarray.h:403-409 (src/constructors/iarray_constructor_arange.c:40): val = start + i*step. */
INA_API(ina_rc_t) iarray_arange(iarray_context_t *ctx, iarray_dtshape_t *dtshape, double start,
                                double step, iarray_storage_t *storage, iarray_container_t **container);
/* iarray.h:411-416 (src/constructors/iarray_constructor_linspace.c:42,117). */
INA_API(ina_rc_t) iarray_linspace(iarray_context_t *ctx, iarray_dtshape_t *dtshape, double start,
                                  double stop, iarray_storage_t *storage, iarray_container_t **container);
/* iarray.h:664-669 (src/iarray_constructor.c:218-262): host buffer (row-major) ->
 * container; the buffer is copied to the GPU and encoded there. */
INA_API(ina_rc_t) iarray_from_buffer(iarray_context_t *ctx, iarray_dtshape_t *dtshape, void *buffer,
                                     int64_t buflen, iarray_storage_t *storage,
                                     iarray_container_t **container);
/* iarray.h:671-674 (src/iarray_constructor.c:265-305): decoded on the GPU, copied out. */
INA_API(ina_rc_t) iarray_to_buffer(iarray_context_t *ctx, iarray_container_t *container, void *buffer,
                                   int64_t buflen);
/* iarray.h:679 (src/iarray_container.c:1200-1210). */
INA_API(ina_rc_t) iarray_container_info(iarray_container_t *container, int64_t *nbytes, int64_t *cbytes);
/* iarray.h:681 (src/iarray_container.c:1438-1461). */
INA_API(void) iarray_container_free(iarray_context_t *ctx, iarray_container_t **container);
/* iarray.h:645-651. */
INA_API(ina_rc_t) iarray_get_dtshape(iarray_context_t *ctx, iarray_container_t *c, iarray_dtshape_t *dtshape);
INA_API(ina_rc_t) iarray_get_storage(iarray_context_t *ctx, iarray_container_t *c, iarray_storage_t *storage);
/* iarray.h:661. */
INA_API(ina_rc_t) iarray_is_view(iarray_context_t *ctx, iarray_container_t *c, bool *view);
/* iarray.h:690 (src/iarray_container.c:1212-1288): max relative difference |a-b|/|a| <= tol. */
INA_API(ina_rc_t) iarray_container_almost_equal(iarray_container_t *a, iarray_container_t *b, double tol);

/* ---------------------------------------------------------------- persistence */
/* iarray.h:601-603 (src/iarray_container.c:50-76): contiguous Blosc2 frame on disk. */
INA_API(ina_rc_t) iarray_container_save(iarray_context_t *ctx, iarray_container_t *container, char *urlpath);
/* iarray.h:597-599 (src/iarray_container.c:79-217). */
INA_API(ina_rc_t) iarray_container_open(iarray_context_t *ctx, char *urlpath, iarray_container_t **container);
/* iarray.h:593-595. */
INA_API(ina_rc_t) iarray_container_load(iarray_context_t *ctx, char *urlpath, iarray_container_t **container);
/* iarray.h:617 (src/iarray_container.c:219-225): removes a frame file, or a sparse frame's
 * directory.  A container created with storage->urlpath set and storage->contiguous false
 * is written as a sparse (directory) frame, c-blosc2's layout: <urlpath>/chunks.b2frame
 * (header, metalayers and the offsets index, whose entries are chunk file numbers) and one
 * file <urlpath>/%08X.chunk per chunk; iarray_container_open / _load read either kind. */
INA_API(ina_rc_t) iarray_container_remove(char *urlpath);
/* iarray.h:605-609 (src/iarray_container.c:228-260): serialise to a contiguous frame in
 * host memory; *needs_free tells the caller to free(*frame). */
INA_API(ina_rc_t) iarray_to_cframe(iarray_context_t *ctx, iarray_container_t *src, uint8_t **frame,
                                   int64_t *frame_len, bool *needs_free);
/* iarray.h:611-615 (src/iarray_container.c:262-300). */
INA_API(ina_rc_t) iarray_from_cframe(iarray_context_t *ctx, uint8_t *frame, int64_t frame_len, bool copy,
                                     iarray_container_t **container);

/* ---------------------------------------------------------------- linear algebra */
/* iarray.h:760-764 (src/linalg/matmul.c:19-67): C = A*B (2-D B) or y = A*x (1-D B);
 * C is created with `storage`'s partition and returned through *c. */
INA_API(ina_rc_t) iarray_linalg_matmul(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                       iarray_storage_t *storage, iarray_container_t **c);
/* iarray.h:766-768 (src/linalg/transpose.c:18-45): a transposed view sharing a's chunks. */
INA_API(ina_rc_t) iarray_linalg_transpose(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t **b);
/* src/linalg/matmul/gemm.h:15-18 (src/linalg/matmul/gemm.c:252-267): C preallocated. */
INA_API(ina_rc_t) iarray_gemm(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                              iarray_container_t *c);
/* src/linalg/matmul/gemv.h:15-18 (src/linalg/matmul/gemv.c:193-208). */
INA_API(ina_rc_t) iarray_gemv(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                              iarray_container_t *c);
/* iarray.h:866-870 (src/linalg/iarray_gemm.c:315-432): matched partitions required. */
INA_API(ina_rc_t) iarray_opt_gemm(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                  iarray_storage_t *storage, iarray_container_t **c);
/* iarray.h:878-882 (src/linalg/iarray_gemm_a.c:191-358). */
INA_API(ina_rc_t) iarray_opt_gemm_a(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                    iarray_storage_t *storage, iarray_container_t **c);
/* iarray.h:872-876 (src/linalg/iarray_gemm_b.c:191-358). */
INA_API(ina_rc_t) iarray_opt_gemm_b(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                    iarray_storage_t *storage, iarray_container_t **c);
/* iarray.h:860-864 (src/linalg/iarray_gemv.c:249-351). */
INA_API(ina_rc_t) iarray_opt_gemv(iarray_context_t *ctx, iarray_container_t *a, iarray_container_t *b,
                                  iarray_storage_t *storage, iarray_container_t **c);

/* ---------------------------------------------------------------- expressions */
/* include/libiarray/iarray.h:317-332 (opaque here) and :308-314. */
typedef struct iarray_expression_s iarray_expression_t;
typedef union {
    float f32;
    double f64;
    int32_t i32;
    int64_t i64;
    bool b;
} iarray_user_param_t;

/* iarray.h:830-846 (src/iarray_expression.c:59-120, :780).  Element-wise expressions over
 * containers of the output's shape, float64 or float32, evaluated on the GPU: operands are
 * decoded in device memory and one kernel runs the compiled program for every element.
 * Grammar: numbers, bound variables and scalars, pi, e, + - * / ** (right-associative),
 * unary minus, parentheses, and the functions abs, sqrt, exp, expm1, log, log10, log1p, sin,
 * cos, tan, asin, acos, atan, sinh, cosh, tanh, ceil, floor, negative (one argument), atan2,
 * pow, min, max, fmod (two), with numpy's aliases absolute, arcsin, arccos, arctan, arctan2,
 * power, minimum, maximum.  At most 16 operands.  iarray_expr_compile returns
 * INA_ERR_INVALID_ARGUMENT for a malformed expression or an unbound name; iarray_eval returns
 * INA_ERR_NOT_COMPLETE before compile / bind_out_properties and IARRAY_ERR_INVALID_SHAPE when
 * an operand's shape differs from the output's.  User-defined functions (LLVM bitcode:
 * iarray_expr_compile_udf, iarray_expr_bind_param) return IARRAY_ERR_NOT_SUPPORTED. */
INA_API(ina_rc_t) iarray_expr_new(iarray_context_t *ctx, iarray_data_type_t dtype, iarray_expression_t **e);
INA_API(void) iarray_expr_free(iarray_context_t *ctx, iarray_expression_t **e);
INA_API(ina_rc_t) iarray_expr_bind(iarray_expression_t *e, const char *var, iarray_container_t *val);
INA_API(ina_rc_t) iarray_expr_bind_out_properties(iarray_expression_t *e, iarray_dtshape_t *dtshape,
                                                  iarray_storage_t *store);
INA_API(ina_rc_t) iarray_expr_bind_param(iarray_expression_t *e, iarray_user_param_t val);
INA_API(ina_rc_t) iarray_expr_bind_scalar_float(iarray_expression_t *e, const char *var, float val);
INA_API(ina_rc_t) iarray_expr_bind_scalar_double(iarray_expression_t *e, const char *var, double val);
INA_API(ina_rc_t) iarray_expr_compile(iarray_expression_t *e, const char *expr);
INA_API(ina_rc_t) iarray_expr_compile_udf(iarray_expression_t *e, int llvm_bc_len, const char *llvm_bc,
                                          const char *name);
INA_API(ina_rc_t) iarray_eval(iarray_expression_t *e, iarray_container_t **container);

/* ================================================================ B200 additions
 * No counterpart in the reference: the split-precision and batching forms named in
 * the project goal, plus chunk-level access used by the parity tests. */

/* Arithmetic form used by the float64 / float32 products of this context. */
typedef enum iarray_b200_form_e {
    IARRAY_B200_FORM_NATIVE = 0,   /* FP64 DMMA / FP32 FFMA, the plain drop-in */
    IARRAY_B200_FORM_SPLIT = 1,    /* float64: Ozaki INT8 slices on tcgen05;
                                      float32: BF16 word splits on tcgen05 (6 or 3
                                      products) with FP32 accumulation */
} iarray_b200_form_t;

INA_API(ina_rc_t) iarray_b200_set_form(iarray_context_t *ctx, iarray_b200_form_t form);
/* LZ4 encoder used when this context writes chunks.  Both write standard LZ4 blocks that
 * the reference's Blosc2 decodes bit-exactly.  LIBLZ4 (default) reproduces liblz4 1.9.4
 * LZ4_compress_fast(acceleration 1), c-blosc2's codec, byte for byte, so chunks equal the
 * reference's own; PARALLEL parses each window of every stream in parallel (different
 * bytes, compression ratio within a few percent on typical data). */
typedef enum iarray_b200_encoder_e {
    IARRAY_B200_ENCODER_PARALLEL = 0,
    IARRAY_B200_ENCODER_LIBLZ4 = 1,
} iarray_b200_encoder_t;
INA_API(ina_rc_t) iarray_b200_set_encoder(iarray_context_t *ctx, iarray_b200_encoder_t encoder);
/* Binds expression variable `var` to the matrix product a * b (B200 addition; the
 * reference's expressions take containers only, so a product is first written to a
 * container by iarray_linalg_matmul).  The product is computed on the GPU in the context's
 * form when iarray_eval runs and is consumed by the expression in device memory without
 * being encoded: the expression is the product's epilogue, e.g. "max(ab, 0) + bias". */
INA_API(ina_rc_t) iarray_b200_expr_bind_matmul(iarray_expression_t *e, const char *var, iarray_container_t *a,
                                               iarray_container_t *b);
/* Number of INT8 moduli/slices the float64 split form uses (0 = automatic). */
INA_API(ina_rc_t) iarray_b200_set_split_terms(iarray_context_t *ctx, int nterms);
/* Number of BF16 tensor-core products of the float32 split form: 6 (each operand split
 * into three bf16 words; float32 accuracy) or 3 (two words, "3xBF16": each operand held
 * to about 2^-17 relative, so the result carries about 4e-6 normwise error on random data
 * whatever the accumulation); 0 = automatic (6).  Both sum their products in FP32. */
INA_API(ina_rc_t) iarray_b200_set_split_products_f32(iarray_context_t *ctx, int nproducts);

/* Per-call timing of the last product on this context, in milliseconds (CUDA events):
 * [0] decode A, [1] decode B, [2] product, [3] encode C, [4] total device time. */
INA_API(ina_rc_t) iarray_b200_last_timings(iarray_context_t *ctx, double *ms5);

/* Container built from raw Blosc2 chunks (host memory, row-major chunk order);
 * chunk bytes are copied to the GPU as-is. */
INA_API(ina_rc_t) iarray_b200_from_chunks(iarray_context_t *ctx, iarray_dtshape_t *dtshape,
                                          iarray_storage_t *storage, int64_t nchunks,
                                          const uint8_t *const *chunks, const int64_t *chunk_lens,
                                          iarray_container_t **container);
/* Copy chunk `nchunk`'s compressed bytes to host `buf`; *len gets its cbytes
 * (pass buf = NULL to query the size). */
INA_API(ina_rc_t) iarray_b200_get_chunk(iarray_context_t *ctx, iarray_container_t *c, int64_t nchunk,
                                        uint8_t *buf, int64_t *len);
INA_API(ina_rc_t) iarray_b200_nchunks(iarray_container_t *c, int64_t *nchunks);

/* Decode a container into caller-provided device memory (row-major, leading dimension
 * `ld` items, ld >= last dimension) on the context's stream, without host copies. */
INA_API(ina_rc_t) iarray_b200_decode_to_device(iarray_context_t *ctx, iarray_container_t *c, void *dptr,
                                               int64_t ld);
/* Encode caller-provided device memory (row-major, leading dimension `ld`) into a new
 * container with the given partition. */
INA_API(ina_rc_t) iarray_b200_encode_from_device(iarray_context_t *ctx, iarray_dtshape_t *dtshape,
                                                 const void *dptr, int64_t ld, iarray_storage_t *storage,
                                                 iarray_container_t **container);
/* Dense product of device matrices C = A*B (row-major, leading dimensions lda/ldb/ldc),
 * float64 (dtype 0) or float32 (dtype 1), using the context's form. */
INA_API(ina_rc_t) iarray_b200_dense_gemm(iarray_context_t *ctx, int dtype, int64_t M, int64_t N,
                                         int64_t K, const void *A, int64_t lda, const void *B,
                                         int64_t ldb, void *C, int64_t ldc);
/* Synchronise the context's stream. */
INA_API(ina_rc_t) iarray_b200_synchronize(iarray_context_t *ctx);
/* Number of CUDA kernels this library has launched in this process. */
INA_API(uint64_t) iarray_b200_kernel_launches(void);
/* The context's CUDA stream (a cudaStream_t), for callers that record their own
 * events around library calls. */
INA_API(ina_rc_t) iarray_b200_get_stream(iarray_context_t *ctx, void **stream);
/* Serialise a container as a contiguous frame (the layout of iarray_to_cframe) into a
 * caller buffer of `cap` bytes, e.g. pinned host memory; *len receives the frame size.
 * buf = NULL only queries the size. */
INA_API(ina_rc_t) iarray_b200_to_cframe_into(iarray_context_t *ctx, iarray_container_t *c, uint8_t *buf,
                                             int64_t cap, int64_t *len);

/* B200 addition (no reference counterpart; it fuses the reference sequence
 * iarray_from_cframe (iarray.h:611-615) for a and b + iarray_opt_gemm (iarray.h:866-870) +
 * iarray_to_cframe (iarray.h:605-609) into one call).  C = A * B with A and B given as
 * contiguous frames in host memory and C written as a contiguous frame into host memory
 * `out` (capacity out_cap bytes; *out_len receives the frame's length, also when it does
 * not fit, in which case IARRAY_ERR_TOO_SMALL_BUFFER is returned).  Partition rules,
 * context form and encoder are those of iarray_opt_gemm; storage->urlpath must be NULL.
 * The work runs in row bands of C (one chunk row each) so that the uploads of later bands,
 * the kernels of the current one and the download of earlier ones overlap; with pinned
 * host memory (cudaHostAlloc) the call approaches the time of the uploads.  A capacity of
 * M * N * itemsize rounded up to whole chunks, plus 64 bytes per chunk, plus 4 KiB always
 * suffices.  Implemented by iarray_b200_opt_gemm_cframes in api.cu. */
INA_API(ina_rc_t) iarray_b200_opt_gemm_cframes(iarray_context_t *ctx, const uint8_t *a_frame, int64_t a_len,
                                               const uint8_t *b_frame, int64_t b_len, iarray_storage_t *storage,
                                               uint8_t *out, int64_t out_cap, int64_t *out_len);

/* Batched products (B200 addition; the reference has no counterpart: its callers loop over
 * iarray_opt_gemm).  C_i = A_i * B_i for i < n, float64, each pair with its own shapes
 * (A_i: M_i x K_i, B_i: K_i x N_i) and partitions, output i partitioned by storage[i].
 * iarray_b200_batch_new decodes the operands, times the grouped product's tile
 * configurations on them (autotuner; choice cached per set of shapes), runs the batch once
 * and captures decode -> product -> encode of every problem in one CUDA graph: in the
 * native form the products of all problems are one persistent grouped kernel launch, in
 * the split form (context form IARRAY_B200_FORM_SPLIT) one grouped split-precision
 * pipeline (seven launches over all problems: scaling, residues, one persistent INT8
 * tensor-core launch over every problem's tiles and moduli, reconstruction).  iarray_b200_batch_run replays the graph and returns n new containers in c
 * (free each with iarray_container_free).  The operand containers are borrowed: they must
 * stay alive and unchanged until iarray_b200_batch_free.  Operands must not be transposed
 * views. */
typedef struct iarray_b200_batch_s iarray_b200_batch_t;
INA_API(ina_rc_t) iarray_b200_batch_new(iarray_context_t *ctx, int64_t n, iarray_container_t *const *a,
                                        iarray_container_t *const *b, const iarray_storage_t *storage,
                                        iarray_b200_batch_t **batch);
INA_API(ina_rc_t) iarray_b200_batch_run(iarray_b200_batch_t *batch, iarray_container_t **c);
/* Tile configuration chosen by the autotuner (-1 in the split form): cfg & 3 is the tile
 * shape (0: 128x128, 1: 64x128, 2: 128x64, 3: 64x64), cfg < 4 pipeline stages 16 deep in
 * k, cfg >= 4 32 deep; the tuning times of the IARRAY_B200_BATCH_TILE_CONFIGS
 * configurations in ms (-1: not measured, e.g. a cached choice); and the number of nodes
 * of the captured graph. */
#define IARRAY_B200_BATCH_TILE_CONFIGS 8
INA_API(ina_rc_t) iarray_b200_batch_info(iarray_b200_batch_t *batch, int *tile_config, double *tune_ms,
                                         int64_t *graph_nodes);
/* Split form: the number of moduli the batch uses.  When the context's count is automatic
 * (iarray_b200_set_split_terms(ctx, 0)), iarray_b200_batch_new tunes it on the batch's own
 * operands: 16 moduli serve as the reference, the native FP64 product's normwise error
 * against it sets the bar, and of 16..12 moduli the fastest whose error stays within 4x that
 * bar is kept (cached per set of shapes).  *err_native receives the bar's base error,
 * tune_ms[5] / tune_err[5] the time and error of 16, 15, 14, 13, 12 moduli (-1: not measured,
 * e.g. a cached choice or a count fixed by the context).  IARRAY_ERR invalid argument for a
 * batch in the native form. */
INA_API(ina_rc_t) iarray_b200_batch_split_tuning(iarray_b200_batch_t *batch, int *nterms, double *err_native,
                                                 double *tune_ms, double *tune_err);
INA_API(void) iarray_b200_batch_free(iarray_b200_batch_t **batch);

/* Per-kernel device time (B200 addition; the reference has no counterpart).  While
 * enabled, every kernel launch of the library is bracketed by CUDA events on its stream;
 * iarray_b200_profile_kernels(1) clears the totals and starts, (0) stops.
 * iarray_b200_kernel_profile writes one line per kernel, "name launches total_ms\n",
 * NUL-terminated, into `buf` (cap bytes; buf = NULL only queries *len). */
INA_API(ina_rc_t) iarray_b200_profile_kernels(int on);
INA_API(ina_rc_t) iarray_b200_kernel_profile(char *buf, int64_t cap, int64_t *len);

/* Decode without allocating.  No counterpart in the reference (whose decoders allocate
 * through Blosc2 contexts): this entry point is for callers that cannot call cudaMalloc,
 * such as engines whose device memory is owned by their own arena or memory-budget
 * manager and that hand the library only buffers they already hold, or latency-bound
 * loops that must not pay the device synchronisation cudaMalloc / cudaFree bring.
 *
 * Decodes `nchunks = prod(ceil(shape / chunkshape))` Blosc2 chunks stored back to back
 * in device memory (`chunks`, `chunks_len` bytes, row-major chunk order, the layout of a
 * frame's chunk region) into the device array `dptr` (row-major, leading dimension `ld`
 * items, ld >= last dimension; columns past the last dimension are left untouched), on
 * the CUDA stream `stream` (a cudaStream_t; NULL = the legacy default stream), and
 * waits for it.  The kernels are the ones iarray_b200_decode_to_device runs; their work
 * buffers live in one fixed device array of the library instead of allocations, so the
 * call allocates nothing.  Limits per call: nchunks x padded chunk bytes <=
 * IARRAY_B200_NOALLOC_MAX_BYTES and nchunks x blocks per chunk <=
 * IARRAY_B200_NOALLOC_MAX_BLOCKS; larger geometries return IARRAY_ERR_NOALLOC_TOO_LARGE
 * (decode a large container chunk by chunk, passing chunkshape as the shape).
 * The fixed array (about 9.7 MiB) is held by every GPU that loads the library's kernels
 * until the process exits.  The first call on each device looks up the array's device
 * address and sets a kernel attribute; make that first call before any stream capture.
 * Every call waits for `stream` before it returns (it reads the decoders' status word
 * back to the host).  All calls share the array and it keeps the last call's contents:
 * calls whose work overlaps on the GPU (other streams, other host threads) race on it
 * and must be serialised by the caller. */
#define IARRAY_B200_NOALLOC_MAX_BYTES (8LL << 20)
#define IARRAY_B200_NOALLOC_MAX_BLOCKS 4096LL
#define IARRAY_ERR_NOALLOC_TOO_LARGE (INA_ERR_OUT_OF_RANGE | IARRAY_ES_BUFFER)
INA_API(ina_rc_t) iarray_b200_decode_noalloc(int8_t ndim, const int64_t *shape, const int64_t *chunkshape,
                                             const int64_t *blockshape, int32_t itemsize, const void *chunks,
                                             int64_t chunks_len, void *dptr, int64_t ld, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IARRAY_B200_H */
