/*
 * gpuspmv_b200.h -- C ABI of the B200 SpMV engine.
 *
 * Two layers, both plain C (no CUDA or torch types in any signature; streams are passed
 * as an opaque pointer that holds a cudaStream_t):
 *
 *  1. Drop-in layer.  The format structs, converters and per-format SpMV entry points of
 *     the reference program (edoardoCB/gpu_spmv, canonical source cudaSpmv.cu, built with
 *     FP_TYPE=FP_DOUBLE as its gc.sh does), with the same names, argument meaning and
 *     struct layouts, so that a driver written against cudaSpmv.cu links against this
 *     library unchanged.  The converters run on the GPU and return bit-identical host
 *     arrays; the entry points run sm_100a kernels.  Differences in error behaviour: the
 *     reference prints and exit()s; this library never exits -- it prints the same kind of
 *     message, marks the result (name "error", times 0) and records the reason for
 *     gs_last_error().
 *
 *  2. Native layer (gs_*).  Device-resident matrices built on the GPU from a device CSR,
 *     status-returning, stream-ordered SpMV / SpMM / adjoint calls on device pointers.
 *
 * Index type is the reference's UIN (32-bit unsigned) throughout, so every length is
 * below 2^32.
 */
#ifndef GPUSPMV_B200_H
#define GPUSPMV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================================
 * 1. Drop-in layer (reference: cudaSpmv.cu)
 * ==================================================================================== */

#ifndef GS_UIN_DEFINED
#define GS_UIN_DEFINED
typedef unsigned int UIN; /* cudaSpmv.cu:78-80 */
typedef double FPT;       /* cudaSpmv.cu:64-74 with FP_TYPE == FP_DOUBLE */
#endif

/* GS_API_GEN2 selects the reference's second API generation (gpuSpmv_header.h) for the
 * drop-in names instead of the first (cudaSpmv.cu); see gpuspmv_b200_gen2.h. */
#ifdef GS_API_GEN2
#ifdef __cplusplus
}
#endif
#include "gpuspmv_b200_gen2.h"
#ifdef __cplusplus
extern "C" {
#endif
#else

/* cudaSpmv.cu:261 */
typedef struct {
    char name[48];
    UIN nrows;
    UIN nnz;
    UIN rmin;
    FPT rave;
    UIN rmax;
    FPT rsd;
    UIN bw;
    FPT *val;
    UIN *row;
    UIN *rowStart;
    UIN *rowEnd;
    UIN *col;
    UIN *rl;
} str_matCSR;

/* cudaSpmv.cu:385 */
typedef struct {
    char name[48];
    double mfp;
    double beta;
    double ct;
} str_formatData;

/* cudaSpmv.cu:470 */
typedef struct {
    double aErr;
    double rErr;
    UIN pos;
} str_err;

/* cudaSpmv.cu:499 */
typedef struct {
    char name[48];
    double et;
    double ot;
    double flops;
    str_err sErr;
} str_res;

/* cudaSpmv.cu:712 */
typedef struct {
    UIN nrows;
    UIN nnz;
    UIN chunkNum;
    UIN lenVC;
    UIN *permi;
    UIN *nmc;
    UIN *chp;
    FPT *val;
    UIN *col;
} str_matK1;

/* cudaSpmv.cu:933 */
typedef struct {
    UIN nrows;
    UIN nnz;
    UIN hbs;
    UIN lenAX;
    UIN lenBRP;
    UIN lenMAPX;
    FPT *ax;
    UIN *brp;
    UIN *mapx;
} str_matAXC;

/* cudaSpmv.cu:1154 */
typedef struct {
    char name[48];
    UIN nrows;
    UIN nnz;
    char mode[8];
    UIN tileHW;
    UIN tileH;
    UIN logTH;
    UIN tileN;
    UIN lenAX;
    UIN lenSEC;
    UIN lenCON;
    UIN log;
    UIN bs;
    FPT *ax;
    UIN *sec;
    UIN *con;
} str_matAXT;

/* Matrix I/O and statistics.
 * matrixReading replaces cudaSpmv.cu:265-328 (.csr text / .bin raw reader).  On failure
 * the returned struct has nrows = nnz = 0 and NULL arrays (the reference exits).
 * printMatrixStats replaces cudaSpmv.cu:332-381: fills rl[] and the statistics and writes
 * "<name up to the first '.'>.sta". */
str_matCSR matrixReading(const char *matFileName);
void printMatrixStats(const char *matFileName, str_matCSR *matCSR);
/* Writes the reference's raw .bin layout (u32 nrows, u32 nnz, FPT val[nnz], u32 col[nnz],
 * u32 row[nrows+1]); returns 0 on success.  No counterpart in the reference (which only
 * reads .bin files); provided so generated matrices can be fed to either program. */
int matrixWritingBin(const char *matFileName, const str_matCSR *matCSR);

/* cudaSpmv.cu:403-436: rowStart/rowEnd copies of row[] (calloc'd), footprint, beta = 1. */
str_formatData getFormatDataCSR(str_matCSR *matCSR);

/* cudaSpmv.cu:440-447: vec[i] = i. */
void init_vec(const UIN ompNT, const UIN len, FPT *vec);

/* cudaSpmv.cu:451-466: res = A vec.  Runs on the GPU (sequential per-row order for short
 * rows, so results match the reference's CPU loop to the last bit for rows that fit one
 * lane's share; ompNT is accepted and ignored). */
void ncsr(const UIN ompNT, const str_matCSR matCSR, const FPT *vec, FPT *res);

/* cudaSpmv.cu:474-495. */
void get_errors(const UIN len, const FPT *ar, const FPT *ac, str_err *sErr);

/* Converters (cudaSpmv.cu:782, 1004, 1391).  They run on the GPU and fill the struct with
 * calloc'd host arrays that are bit-identical to the reference's CPU converters (x baked
 * into ax exactly as the reference does).  matCSR.rl must be filled (printMatrixStats).
 * fd.ct is the device conversion time in seconds.  The caller frees the arrays with
 * free(), as with the reference. */
str_formatData getFormatDataK1(const UIN blockSize, const str_matCSR matCSR, const FPT *vec,
                               str_matK1 *matK1);
str_formatData getFormatDataAXC(const UIN ompNT, const UIN hbs, const str_matCSR matCSR,
                                const FPT *vec, str_matAXC *matAXC);
str_formatData getFormatDataAXT(const UIN ompNT, const UIN bs, const UIN thw, const UIN th,
                                const char *mode, const str_matCSR matCSR, const FPT *vec,
                                str_matAXT *matAXT);

/* Per-format SpMV entry points (cudaSpmv.cu:547, 629, 871, 1100, 1603, 1714, 1854, 1963,
 * 2101, 2213).  Each copies the host struct to the device, times NUM_ITE launches of the
 * engine's kernel for that format with CUDA events, copies y back and scores it against
 * ref with get_errors.  NUM_ITE defaults to 250 (cudaSpmv.cu:96-98) and is set with
 * gs_set_num_ite().  The launch-shape arguments (cudaBlockSize, wpw, tpw) name the result
 * as in the reference; the engine picks its own B200 launch shape. */
str_res test_gcsr(const UIN cudaBlockSize, const str_matCSR matCSR, const FPT *vec,
                  const FPT *ref);
str_res test_gcucsr(const str_matCSR matCSR, const FPT *vec, const FPT *ref);
str_res test_gk1(const UIN cudaBlockSize, const str_matK1 matK1, const FPT *vec,
                 const FPT *ref);
str_res test_gaxc(const UIN cudaBlockSize, const str_matAXC matAXC, const FPT *ref);
str_res test_gaxtuh1hw16w(const UIN wpw, const UIN cbs, const str_matAXT matAXT,
                          const FPT *ref);
str_res test_gaxtuh1hw08w(const UIN wpw, const UIN cbs, const str_matAXT matAXT,
                          const FPT *ref);
str_res test_gaxtuh1hw04w(const UIN wpw, const UIN cbs, const str_matAXT matAXT,
                          const FPT *ref);
str_res test_gaxtuh(const UIN tpw, const UIN cbs, const str_matAXT matAXT, const FPT *ref);
str_res test_gaxtch1(const UIN cudaBlockSize, const str_matAXT matAXT, const FPT *ref);
str_res test_gaxtch(const UIN cudaBlockSize, const str_matAXT matAXT, const FPT *ref);
#endif /* GS_API_GEN2 */

/* ======================================================================================
 * 2. Native layer
 * ==================================================================================== */

typedef int gs_status;
#define GS_OK 0
#define GS_ERR_INVALID 1     /* bad argument / malformed input */
#define GS_ERR_CUDA 2        /* a CUDA runtime call failed */
#define GS_ERR_ALLOC 3       /* device or host allocation failed */
#define GS_ERR_OVERFLOW 4    /* a 32-bit length or packed header would overflow */
#define GS_ERR_UNSUPPORTED 5 /* parameter combination not supported */
#define GS_ERR_DEVICE 6      /* a kernel reported an error through its status word */

typedef enum { GS_F64 = 0, GS_F32 = 1, GS_BF16 = 2 } gs_dtype;
typedef enum { GS_IDX_U32 = 0, GS_IDX_U16 = 1 } gs_itype;
typedef enum { GS_FMT_CSR = 0, GS_FMT_K1 = 1, GS_FMT_AXC = 2, GS_FMT_AXT = 3 } gs_format;
typedef enum { GS_AXT_UNC = 0, GS_AXT_COM = 1 } gs_axt_mode;

/* Opaque handle for a cudaStream_t (NULL = the legacy default stream). */
typedef void *gs_stream;

const char *gs_status_string(gs_status s);
/* Text of the most recent error raised on the calling thread ("" if none). */
const char *gs_last_error(void);
/* Library version string. */
const char *gs_version(void);
/* Number of timed launches used by the drop-in test_* entry points (default 250). */
void gs_set_num_ite(UIN num_ite);
UIN gs_get_num_ite(void);
/* The y of the calling thread's most recent drop-in test_* product (test_gcsr, test_gk1,
 * test_gaxc, test_gaxt*, and their second-generation names), in row order, copied into
 * out[0..n) when cap >= n; returns n (0 before any product).  No counterpart in the
 * reference, whose test_* entry points only report get_errors' sign-blind summary: this
 * lets a caller check every row of the product it timed. */
UIN gs_dropin_last_y(FPT *out, UIN cap);

/* Conversion parameters for gs_matrix_create.
 *  format  : GS_FMT_CSR / K1 / AXC / AXT
 *  tileHW, tileH, bs, mode : AXT tile half-width, tile height, COM header block size and
 *            mode -- the arguments of getFormatDataAXT (cudaSpmv.cu:1391)
 *  hbs     : AXC brick half-size (getFormatDataAXC, cudaSpmv.cu:1004)
 *  vtype   : stored value type (GS_F64 / GS_F32 / GS_BF16)
 *  itype   : stored column type (GS_IDX_U32, or GS_IDX_U16 = 16-bit offsets from a 32-bit
 *            base per 32-row block; conversion fails with GS_ERR_UNSUPPORTED if a block's
 *            column spread exceeds 65535)
 *  keep_layout : keep the reference layout's metadata (sec, con, mapx) on the device so
 *            it can be read back and compared with the reference converters. */
typedef struct {
    gs_format format;
    UIN tileHW;
    UIN tileH;
    UIN bs;
    gs_axt_mode mode;
    UIN hbs;
    gs_dtype vtype;
    gs_itype itype;
    UIN keep_layout;
} gs_convert_params;

typedef struct gs_matrix gs_matrix;

/* Build a device-resident matrix from a device CSR (row[nrows+1], col[nnz], val[nnz] of
 * type val_type).  Runs on `stream`; returns after the conversion has completed. */
gs_status gs_matrix_create(gs_matrix **out, const gs_convert_params *params, UIN nrows,
                           UIN ncols, UIN nnz, const UIN *d_row, const UIN *d_col,
                           const void *d_val, gs_dtype val_type, gs_stream stream);
/* The same from host CSR arrays (copied to the device on `stream`, then converted), for
 * callers without a CUDA runtime of their own. */
gs_status gs_matrix_create_host(gs_matrix **out, const gs_convert_params *params, UIN nrows,
                                UIN ncols, UIN nnz, const UIN *h_row, const UIN *h_col,
                                const void *h_val, gs_dtype val_type, gs_stream stream);
gs_status gs_matrix_destroy(gs_matrix *A);

/* Sizes and device arrays of a converted matrix (pointers stay owned by the matrix). */
typedef struct {
    gs_format format;
    UIN nrows, ncols, nnz;
    /* AXT (str_matAXT fields) */
    UIN tileHW, tileH, logTH, tileN, lenAX, lenSEC, lenCON, log, bs;
    gs_axt_mode mode;
    /* AXC (str_matAXC fields) */
    UIN hbs, lenBRP, lenMAPX;
    /* K1 (str_matK1 fields) */
    UIN chunkNum, lenVC;
    /* native streams: nslots value/column slots in the format's slot order; slot s of an
     * AXT/AXC layout is the value half of ax[(s/w)*2w + s%w], w = tileHW or hbs */
    UIN nslots;
    gs_dtype vtype;
    gs_itype itype;
    const void *d_val;
    const void *d_col;
    const UIN *d_colbase; /* per 32-row block column base (GS_IDX_U16 only) */
    const UIN *d_sec, *d_con, *d_brp, *d_mapx, *d_permi, *d_nmc, *d_chp;
    /* row table used by the kernels: first position of each row (nrows+1) and real
     * lengths (NULL when rows are unpadded) */
    const UIN *d_rpos;
    const UIN *d_rlen;
    double conv_ms; /* device time of the conversion */
    double mfp;     /* memory footprint as the reference counts it (bytes) */
    double beta;    /* occupancy nnz / stored slots */
    UIN lane_positions; /* consecutive positions per lane of the row-stream kernel (0: the
                         * matrix runs on the K1 or the tile kernel) */
    UIN tiles_per_step; /* UNC layouts of 32-wide tiles, tileH 2 or 4: tiles a warp takes
                         * per step (2 when the x gathers are close to random, else 1);
                         * 0 for every other layout */
} gs_matrix_info;
gs_status gs_matrix_get_info(const gs_matrix *A, gs_matrix_info *info);

/* Algorithmic (format-independent) bytes of one SpMV with k right-hand sides:
 * nnz*(s_v+s_i) + 4*(nrows+1) + s_x*ncols*k + s_y*nrows*k. */
double gs_algorithmic_bytes(UIN nrows, UIN ncols, UIN nnz, UIN k, UIN s_v, UIN s_i, UIN s_x,
                            UIN s_y);

/* SpMV flags */
#define GS_FLAG_NONE 0u
#define GS_FLAG_ACC_F64 1u /* FP32-stored values: FP32 products, FP64 row reduction */
#define GS_FLAG_TMA 2u        /* tileH > 1 layouts with tileHW = 32: stage the value/column
                                 tiles in shared memory with TMA bulk copies instead of
                                 plain loads (kernel variant, for tuning / comparison) */
#define GS_FLAG_STRIPED 4u    /* CSR / COM tileH = 1 layouts: one position per lane per
                                 32-position chunk instead of 8 consecutive positions per
                                 lane (kernel variant) */

/* Device status word of a matrix's kernels: bit 0 = a bounded wait on a TMA stage timed
 * out (the kernel gave up and its y is incomplete).  Synchronises the device; `reset`
 * clears the word. */
gs_status gs_matrix_device_status(const gs_matrix *A, UIN *word, int reset);

/* y = A x on the device.  x has ncols entries of xtype, y nrows entries of ytype.
 * F64 matrices take F64 x/y; F32/BF16 matrices take F32 x and F32 or F64 y.
 * Deterministic: every y entry is written once, with a fixed summation order.
 * Products on one matrix (gs_spmv, gs_spmm, gs_spmm_adjoint, batches holding it) share its
 * K1 split-chunk counters and status word: calls that could overlap in time (other
 * streams, other threads) must be ordered by the caller. */
gs_status gs_spmv(const gs_matrix *A, const void *d_x, gs_dtype xtype, void *d_y,
                  gs_dtype ytype, UIN flags, gs_stream stream);

/* Same product through host buffers: copies x to the device, runs gs_spmv, copies y
 * back, all on `stream`, and returns when y is on the host.  d_xbuf/d_ybuf are
 * caller-provided device staging buffers (ncols / nrows elements). */
gs_status gs_spmv_host(const gs_matrix *A, const void *h_x, void *d_xbuf, gs_dtype xtype,
                       void *h_y, void *d_ybuf, gs_dtype ytype, UIN flags, gs_stream stream);

/* `count` products y_k = A x_k streamed from host memory: x_k at h_x + k x_stride
 * elements, y_k to h_y + k y_stride (strides may be 0: the same host vector every time).
 * Each x_k is copied in and each y_k copied out; uploads, products and downloads of
 * consecutive vectors overlap on three streams with two device buffers each (made on the
 * first call and kept with the matrix).  Host buffers should be pinned for the copies to
 * overlap.  Returns when every y_k is on the host. */
gs_status gs_spmv_host_stream(const gs_matrix *A, const void *h_x, size_t x_stride,
                              gs_dtype xtype, void *h_y, size_t y_stride, gs_dtype ytype,
                              UIN count, UIN flags, gs_stream stream);

/* Synchronous device -> host copy of `bytes` bytes (for bindings that read a matrix's
 * device arrays back without a CUDA runtime of their own). */
gs_status gs_copy_to_host(void *h_dst, const void *d_src, size_t bytes);

/* CSR SpMV straight from device CSR arrays: y = A x, FP64.  Builds the kernel's row-start
 * plan on every call and returns when y is complete; for repeated products convert once
 * with gs_matrix_create(GS_FMT_CSR) and call gs_spmv.  val and col must be 16-byte
 * aligned. */
gs_status gs_csr_spmv_f64(UIN nrows, UIN ncols, UIN nnz, const UIN *d_row, const UIN *d_col,
                          const double *d_val, const double *d_x, double *d_y,
                          gs_stream stream);

/* ---- multi-RHS products and the adjoint of y = A(v) x (K1 matrices, FP64 or FP32 values,
 * 32-bit columns).  No counterpart in the reference, which has one right-hand side and no
 * derivative.  X is row-major [ncols][k], Y row-major [nrows][k], k in {1,2,4,8,16,32},
 * operands of the matrix's value type and 32-byte aligned. */
typedef enum {
    GS_ADJ_DETERMINISTIC = 0, /* transposed K1 layout: fixed summation order, no atomics */
    GS_ADJ_ATOMIC = 1         /* forward layout with atomic adds into Xbar */
} gs_adjoint_mode;

/* Order of a value (or value-gradient) array: the CSR order of creation (nnz entries), or
 * the slot order of the adjoint layout (gs_matrix_value_slots entries, padding slots 0),
 * in which the deterministic adjoint writes vbar without scattering. */
typedef enum { GS_VALUES_CSR = 0, GS_VALUES_SLOTS = 1 } gs_value_order;

/* Y = A X.  The first call sizes the matrix's multi-RHS scratch (allocates, synchronises). */
gs_status gs_spmm(gs_matrix *A, const void *d_X, void *d_Y, gs_dtype dtype, UIN k,
                  gs_stream stream);
/* Builds what the adjoint needs from the CSR structure the matrix was created from (the
 * same d_row / d_col): the map from K1 slots to CSR indices and the K1 layout of A^T with
 * its values.  Once per matrix; allocates and synchronises. */
gs_status gs_matrix_prepare_adjoint(gs_matrix *A, const UIN *d_row, const UIN *d_col,
                                    gs_stream stream);
/* Replaces the stored values (forward and transposed layouts) by d_val, of the matrix's
 * value type, in the given order.  Needs the adjoint prepared. */
gs_status gs_matrix_set_values(gs_matrix *A, const void *d_val, gs_dtype dtype,
                               gs_value_order order, gs_stream stream);
/* Number of slots of the adjoint layout (length of a GS_VALUES_SLOTS array). */
gs_status gs_matrix_value_slots(const gs_matrix *A, UIN *nslots);
/* Converts a value array between the two orders (CSR -> slots fills padding with 0). */
gs_status gs_matrix_convert_values(const gs_matrix *A, const void *d_in,
                                   gs_value_order in_order, void *d_out, gs_dtype dtype,
                                   gs_stream stream);
/* Xbar = A^T Ybar (Xbar [ncols][k], overwritten) and, when d_vbar is given,
 * vbar[e] = sum_r Ybar[row_e][r] * X[col_e][r] for every stored element e, in vbar_order
 * (the gradient with respect to the values; d_X is then required).  X, Ybar and Xbar are
 * 32-byte aligned.  A CSR-order vbar is formed in slot order in a buffer of the matrix and
 * gathered into CSR order (coalesced writes), so calls on one matrix must not overlap.
 * The atomic mode without d_vbar reads neither X nor a second copy of the values. */
gs_status gs_spmm_adjoint(gs_matrix *A, const void *d_Ybar, const void *d_X, void *d_Xbar,
                          void *d_vbar, gs_dtype dtype, UIN k, gs_adjoint_mode mode,
                          gs_value_order vbar_order, gs_stream stream);

/* ---- batched uneven multi-RHS products: Y_i = A_i X_i for many K1 matrices in one
 * persistent launch (no counterpart in the reference).  All matrices share one value type
 * (FP64 or FP32, 32-bit columns); matrix i has k_i right-hand sides (1..32), stored padded
 * to kpad_i = the next power of two: X_i row-major [ncols_i][kpad_i], Y_i [nrows_i][kpad_i],
 * 32-byte aligned (the padding columns of Y_i receive A_i times the padding of X_i). */
typedef struct gs_batch gs_batch;
/* Builds the work list (K1 units or row blocks of each matrix, per right-hand-side block),
 * longest first; allocates and synchronises.  Each matrix starts with one block of kpad_i
 * columns and the path GS_BATCH_AUTO. */
gs_status gs_batch_create(gs_batch **out, UIN count, gs_matrix *const *mats, const UIN *k,
                          gs_stream stream);
gs_status gs_batch_destroy(gs_batch *B);
/* Number of work items, each matrix's kpad (array of count, optional) and the batch's
 * FLOPs per run (2 sum nnz_i k_i). */
gs_status gs_batch_info(const gs_batch *B, UIN *nitems, UIN *kpad, double *flops);
/* Device pointers of every X_i and Y_i (host arrays of count pointers); synchronises.
 * Replaces the operands without invalidating a captured graph. */
gs_status gs_batch_set_operands(gs_batch *B, void *const *d_X, void *const *d_Y,
                                gs_stream stream);
/* Right-hand-side block width of each matrix (a power of two dividing kpad_i): kpad_i/kb_i
 * passes over A_i, each gathering kb_i values per stored element.  Rebuilds the work list
 * (and drops a captured graph). */
gs_status gs_batch_set_blocking(gs_batch *B, const UIN *kb, gs_stream stream);
/* How each matrix of a batch runs.  GS_BATCH_K1: warps over its K1 units, gathering X rows
 * through L1 / L2.  GS_BATCH_BAND: thread blocks over blocks of consecutive rows, each
 * staging its value and column segments and the rows of X its columns reach into shared
 * memory (for banded matrices); the matrix's CSR arrays are rebuilt once from its K1
 * layout (nnz (4 + value size) bytes more device memory).  GS_BATCH_AUTO (the default):
 * row blocks when every row with its X band fits a block's shared memory at the current
 * block width, else K1 units.  Both give the same bits. */
#define GS_BATCH_AUTO 0u
#define GS_BATCH_K1 1u
#define GS_BATCH_BAND 2u
/* Sets the requested path of every matrix and rebuilds the work list (drops a captured
 * graph); GS_ERR_UNSUPPORTED (nothing changed) if a matrix held to GS_BATCH_BAND does not
 * fit at its block width (gs_batch_set_blocking refuses such a width the same way). */
gs_status gs_batch_set_paths(gs_batch *B, const UIN *path, gs_stream stream);
/* The path each matrix runs on (GS_BATCH_K1 or GS_BATCH_BAND; array of count). */
gs_status gs_batch_paths(const gs_batch *B, UIN *path);
/* Height of each matrix's row blocks: at most rows_max[i] consecutive rows per block
 * (32..4096, default 4096; a block also ends where its rows and X band would overflow the
 * shared-memory stage).  The analogue of the reference's tileHeight for the row-block path:
 * lower heights give more, smaller work items.  Re-plans the changed matrices' blocks and
 * rebuilds the work list (drops a captured graph); the sums and their order do not depend
 * on it. */
gs_status gs_batch_set_row_blocks(gs_batch *B, const UIN *rows_max, gs_stream stream);
/* Each matrix's row-block height and its number of row blocks (0 when it runs as K1
 * units); either array may be NULL. */
gs_status gs_batch_row_blocks(const gs_batch *B, UIN *rows_max, UIN *blocks);
/* Reads and clears the batch's device status word (synchronises): bit 0 set when a row
 * block's shared-memory copies did not arrive within the bounded wait (its products were
 * not written). */
gs_status gs_batch_status(gs_batch *B, UIN *flags, gs_stream stream);
/* One run: a counter reset and one persistent kernel launch on `stream`. */
gs_status gs_batch_run(gs_batch *B, gs_stream stream);
/* The same run replayed from a CUDA graph captured on the first call. */
gs_status gs_batch_run_graph(gs_batch *B, gs_stream stream);

/* K1 SpMV that allocates nothing: y[permi[r]] = row r of the K1 layout times x, FP64, from
 * the arrays the reference's gk1 kernel takes (cudaSpmv.cu:851), all on the device, in the
 * str_matK1 layout (chunkNum = ceil(nrows / 32), permi of chunkNum * 32 entries, lenVC
 * slots of val / col).  No counterpart in the reference: gk1 runs each chunk in one warp
 * with no scratch; this runs the engine's split-chunk K1 kernel, whose piece partial sums
 * and arrival counters live in a static device array of 8.25 MiB per device instead of
 * memory allocated per matrix or per call.  For callers that cannot allocate: ones whose
 * device memory belongs to another allocator (a framework's caching pool that has
 * reserved the device), and loops that must not synchronise (cudaFree synchronises the
 * device).  Layouts above GS_K1_STATIC_MAX_SLOTS slots are refused with
 * GS_ERR_UNSUPPORTED.  The first call on each device looks the scratch up and zeroes its
 * counters, synchronising the device: make it before any stream capture or timed loop.
 * Calls on one device share the scratch, so calls that could overlap (other streams, other
 * threads) must be serialised by the caller.  Asynchronous on `stream`. */
#define GS_K1_STATIC_MAX_SLOTS 134217728ull
gs_status gs_k1_spmv_f64_static(UIN nrows, UIN chunkNum, UIN lenVC, const double *d_val,
                                const UIN *d_col, const UIN *d_nmc, const UIN *d_chp,
                                const UIN *d_permi, const double *d_x, double *d_y,
                                gs_stream stream);

/* Synthetic matrices (host, deterministic for a given seed, any thread count).  Each
 * returns a CSR in malloc'd host arrays the caller frees with gs_free_host. */
gs_status gs_gen_laplacian2d(UIN grid, UIN **row, UIN **col, double **val, UIN *nrows,
                             UIN *nnz);
gs_status gs_gen_powerlaw(UIN nrows, uint64_t target_nnz, double mu, double sigma,
                          UIN max_len, uint64_t seed, UIN **row, UIN **col, double **val,
                          UIN *nnz);
gs_status gs_gen_stencil27(UIN grid, uint64_t seed, UIN **row, UIN **col, double **val,
                           UIN *nrows, UIN *nnz);
gs_status gs_gen_banded(UIN nrows, UIN half_bw, UIN min_len, UIN max_len, uint64_t seed,
                        UIN **row, UIN **col, double **val, UIN *nnz);
/* Fill v[0..n) with uniform [lo, hi) (dist 0) or N(0,1) (dist 1). */
gs_status gs_gen_vector(uint64_t n, int dist, double lo, double hi, uint64_t seed,
                        double *v);
void gs_free_host(void *p);

#ifdef __cplusplus
}
#endif
#endif /* GPUSPMV_B200_H */
