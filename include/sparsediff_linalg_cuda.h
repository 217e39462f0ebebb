/* sparsediff_linalg B200 extension API.
 *
 * The drop-in headers under sparsediff_linalg/ keep the upstream host-pointer API.
 * This header adds what a GPU-resident caller needs and upstream has no
 * counterpart for:
 *   - status codes and error text instead of exit(1);
 *   - device-resident products, transposes and duplicate coalescing whose
 *     operands and results stay in HBM (all pointers below are DEVICE pointers
 *     unless a comment says otherwise);
 *   - the batched refill engine and the learned row scheduler.
 * Every function is extern "C" with plain pointers and sizes. Streams are passed
 * as void* (a cudaStream_t); NULL means the library's own stream. The library
 * works on one device per process: the device current when it is first used
 * (one process per GPU, as torch.distributed and torchrun arrange it). */
#ifndef SPARSEDIFF_LINALG_CUDA_H
#define SPARSEDIFF_LINALG_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "sparsediff_linalg/COO_matrix.h"
#include "sparsediff_linalg/CSC_matrix.h"
#include "sparsediff_linalg/CSR_matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sdl_status
{
    SDL_OK = 0,
    SDL_ERR_NO_DEVICE = 1,   /* no usable CUDA device */
    SDL_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    SDL_ERR_INVALID = 3,     /* malformed input (bad pointers, sizes, indices) */
    SDL_ERR_OVERFLOW = 4,    /* a result does not fit int32 indexing */
    SDL_ERR_OOM = 5,         /* device allocation failed */
    SDL_ERR_UNSUPPORTED = 6, /* operand combination not provided by this build */
    SDL_ERR_TIMEOUT = 7,     /* a bounded device wait gave up */
    SDL_ERR_INTERNAL = 8     /* a device-side consistency check failed */
} sdl_status;

/* Status and message of the last failing call on this thread (SDL_OK / "" when
   none). */
sdl_status sdl_last_status(void);
const char *sdl_last_error(void);
void sdl_clear_error(void);

/* The upstream API has no error returns: by default a device failure inside one
   of its entry points prints the message to stderr and exits(1), as upstream does
   on its own fatal conditions. With fatal = 0 those entry points instead record
   the status (sdl_last_status) and return NULL / leave outputs unchanged. */
void sdl_set_fatal_errors(int fatal);

/* 1 if a CUDA device is usable (initialises the library runtime on it). */
int sdl_device_available(void);
/* Number of device allocations / kernel launches the library has made so far. */
unsigned long long sdl_device_alloc_count(void);
unsigned long long sdl_kernel_launch_count(void);
/* The library keeps device memory it has freed (plans' scratch, destroyed
   products) in a cache for its next allocations, up to a quarter of the device's
   memory; this returns the current device's cached blocks to the driver (after a
   device synchronisation), e.g. before a large allocation of the application's own. */
void sdl_release_cached_memory(void);
/* The library's stream (a cudaStream_t) and a full synchronisation of it. */
void *sdl_stream(void);
sdl_status sdl_synchronize(void);
/* Frees a buffer the library allocated and handed out (device pointer). */
void sdl_free(void *device_ptr);

/* ------------------------------------------------------------------------
   Device-resident sparse product  C = kron(I_blocks, L) diag(d) A.
   L is given by rows (Lp, Li): for B^T D A, L is the CSC of B (its columns);
   for C = B A, L is B's CSR. A is CSR with A_m = blocks * (rows of A per block).
   L_map (optional) makes the value of L entry ii equal Lx[L_map[ii]], which lets
   the fill read B's values straight from its CSR (L_map = the CSR position of
   each CSC entry) with no separate CSC refresh.
   ------------------------------------------------------------------------ */
typedef struct sdl_product sdl_product;

typedef struct sdl_product_desc
{
    const int *Lp;
    const int *Li;
    const int *L_map; /* may be NULL */
    int L_m, L_nnz;
    int blocks; /* >= 1 */
    const int *Ap;
    const int *Ai;
    int A_m, A_n, A_nnz;
} sdl_product_desc;

/* Symbolic phase (exact structure, rows sorted ascending, unique) and the
   numeric schedule. The operand structure arrays must stay alive and unchanged
   while the product is used. Synchronises the stream. */
sdl_status sdl_product_create(const sdl_product_desc *desc, void *stream,
                              sdl_product **out);
/* Shape, nnz and device pointers to C's row offsets / column indices (owned by
   the product). */
sdl_status sdl_product_info(const sdl_product *P, int *m, int *n, int *nnz,
                            long long *terms, const int **Cp, const int **Ci);
/* Numeric phase: Cx[0 .. nnz) = values of C. Lx (NULL = every L value is 1.0),
   d (A_m values, NULL = identity), Ax. Asynchronous on the stream; never
   allocates; each entry is summed in the upstream order with the upstream
   roundings (no FMA). */
sdl_status sdl_product_fill(const sdl_product *P, const double *Lx, const double *d,
                            const double *Ax, double *Cx, void *stream);
void sdl_product_destroy(sdl_product *P);

/* No upstream counterpart: autotuner. Re-plans P for its own pattern (structure
   and values are unchanged; only the schedule moves). Candidate symbolic bin
   thresholds (warp-kernel row limit 128 / 512 terms, 4 / 8 / 16 warps per CTA)
   are timed on the pattern; then candidate tile budgets (TILE_T, 3/4, 1/2 of it)
   and resident refill CTAs per SM (all that fit, 4, 3), and the small-tile
   refill (128-thread CTAs over tiles and tile rows of at most TILE_T / 2 terms),
   by `reps` refills each with placeholder values, L2 flushed before each; P keeps
   the fastest plan
   (the as-given plan unless a candidate beats it). The row offsets / column
   indices sdl_product_info returned before are released: ask again. Allocates;
   synchronises the stream. */
sdl_status sdl_product_autotune(sdl_product *P, int reps, void *stream);
/* The configuration P runs with and, after sdl_product_autotune, what the tuner
   measured (microseconds of the chosen and of the as-given refill; candidates
   timed; milliseconds the tuning took). Any pointer may be NULL. */
sdl_status sdl_product_tuning(const sdl_product *P, int *warp_max_terms, int *rows_per_cta_warp,
                              int *tile_budget, int *refill_ctas_per_sm, double *refill_us,
                              double *default_refill_us, int *candidates, double *tune_ms);
/* Re-plans P with a given refill configuration (structure unchanged): tile budget
   and largest tile row in terms (0: TILE_T = 1024), refill CTA threads (256, or 128:
   used when every tile window fits the small-tile refill, i.e. budget and largest
   row at most 512), resident refill CTAs per SM (0: all that fit). The row offsets
   / column indices sdl_product_info returned before are released. Allocates;
   synchronises the stream. */
sdl_status sdl_product_replan(sdl_product *P, int tile_budget, int tile_max_terms, int refill_threads,
                              int refill_ctas_per_sm, void *stream);
/* Threads of P's refill CTAs (256, or 128 for the small-tile refill) and the largest
   row (terms) its tiles take. Any pointer may be NULL. */
sdl_status sdl_product_refill_shape(const sdl_product *P, int *refill_threads, int *tile_max_terms);
/* No upstream counterpart. Chooses between the two refills of P's tiles: the
   pipelined one (on = 1, the default: each tile's term words and entry records are
   copied into shared memory two tiles ahead and its A.x / V values one tile ahead,
   so computing a tile reads shared memory only), used when every tile of the plan
   holds at most 1024 terms, 512 entries and 1024 outputs (plans of at most 512-term
   tiles, which sdl_product_replan and the autotuner make), or the direct one
   (on = 0, the default; the autotuner times both). Both give the same bits. *used
   (may be NULL) reports whether the pipelined refill will run. */
sdl_status sdl_product_set_refill_pipe(sdl_product *P, int on, int *used);
/* Whether P's tiles are refilled by the pipelined refill (1) or the direct one (0). */
sdl_status sdl_product_refill_pipe_used(const sdl_product *P, int *used);
/* The staged direct refill (on = 1: each tile's term words and entry records are
   bulk-copied into shared memory by one thread while the tile before it runs, so a
   term step issues only the V and A.x gathers to global memory), used when two
   slots for the plan's largest tile fit a 64 KB CTA; on = 0 the plain direct
   refill. Turning it on turns the pipelined refill off. Same bits either way.
   *used (may be NULL) reports whether it will run. */
sdl_status sdl_product_set_refill_staged(sdl_product *P, int on, int *used);
sdl_status sdl_product_refill_staged_used(const sdl_product *P, int *used);

/* No upstream counterpart (it generalises upstream's fixed plan-vs-accumulator
   threshold GUSTAVSON_PLAN_MAX_RATIO, src/internal/gustavson.h:52, used at
   src/sparse/sparse_matrix.c:270-277): the tuning table. sdl_product_autotune
   records its choice under P's pattern key -- rows of C, columns of A, terms per
   row, terms per output and the histogram of C's row lengths over power-of-two
   classes -- in a table of the process; sdl_product_apply_tuned re-plans a product
   with the configuration recorded for its key (structure unchanged; *found = 0 and
   nothing changes when the key is absent). The table is saved to and loaded from a
   text file (one entry per line), so a later process takes tuned plans without
   timing candidates; loading adds to the table (an entry replaces one of the same
   key) and rejects a malformed file as a whole. The pattern key is written into
   buf (NUL-terminated; len bytes available). apply_tuned and pattern_key
   synchronise the stream; apply_tuned allocates. */
sdl_status sdl_product_apply_tuned(sdl_product *P, int *found, void *stream);
sdl_status sdl_product_pattern_key(const sdl_product *P, char *buf, int len, void *stream);
sdl_status sdl_tune_table_save(const char *path);
sdl_status sdl_tune_table_load(const char *path, int *entries);
sdl_status sdl_tune_table_clear(void);
sdl_status sdl_tune_table_size(int *entries);

/* No upstream counterpart. Same result as sdl_product_fill, bit for bit, for
   callers that cannot call cudaMalloc while they refill: device memory wholly
   owned by another allocator, a fixed device-memory budget that may not grow, or
   a latency-critical loop that must not pay cudaMalloc's implicit
   synchronisation. It allocates nothing: the scratch of the rows with more than
   8192 outputs is a 16 MiB array inside the library (held by every GPU that
   loads the library until the process exits), so A may have at most 4194304
   (4 Mi) columns; larger products are rejected with SDL_ERR_INVALID. The first
   call on a device looks the array's address up once (with that device
   current); make that first call before any stream capture. Every call shares
   the array, so calls that overlap on the GPU race; it needs no clearing between
   calls. */
sdl_status sdl_product_fill_noalloc(const sdl_product *P, const double *Lx, const double *d,
                                    const double *Ax, double *Cx, void *stream);

/* ------------------------------------------------------------------------
   Batched refill: many products (uneven sizes, fixed patterns) refilled by a few
   persistent launches over the union of their compiled tile schedules, captured
   into a CUDA graph on the first refill and replayed afterwards. The products are
   cut, in order, into groups whose entry values and entry records (16 bytes per
   entry) reach a size (64 MiB by default); each group's entry values are computed
   on a side stream while the previous group is refilled. Rows with more than the
   tile budget of terms are refilled by per-product launches inside the same graph.
   ------------------------------------------------------------------------ */
typedef struct sdl_batch sdl_batch;
/* The products must outlive the batch. Synchronises the stream. */
sdl_status sdl_batch_create(sdl_product *const *products, int count, void *stream,
                            sdl_batch **out);
/* Device value arrays of product i used by the following refills (as in
   sdl_product_fill). Rebinding after the first refill is allowed: the graph reads
   the pointers from a device table. The table is written synchronously, so rebind
   only while no refill of the batch is in flight. */
sdl_status sdl_batch_bind(sdl_batch *B, int i, const double *Lx, const double *d,
                          const double *Ax, double *Cx);
/* Bytes of entry values and records per group (0: one group for the whole batch).
   Only before the first sdl_batch_refill. */
sdl_status sdl_batch_set_group_bytes(sdl_batch *B, long long bytes);
/* Number of product groups of the batch. */
sdl_status sdl_batch_groups(const sdl_batch *B, int *groups);
/* No upstream counterpart: the batch's autotuner. Before the batch's first refill
   (its graph does not exist yet) and with every product bound, times `reps`
   refills (eagerly, on `stream`, which must not be the legacy default stream) at
   each candidate group size -- 16, 32, 64, 128, 256 MiB of entry values and
   records per group, and one group -- and keeps the fastest. Reports the chosen
   size (0: one group) and its milliseconds per refill (either pointer may be
   NULL). The refills it runs write the bound outputs. */
sdl_status sdl_batch_autotune(sdl_batch *B, int reps, void *stream, long long *group_bytes, double *ms);
/* One refill of every product of the batch, asynchronous on the stream. */
sdl_status sdl_batch_refill(sdl_batch *B, void *stream);
/* The same refill as sdl_batch_refill done the plain way: one sdl_product_fill
   per product (separate launches, no graph). For comparisons. */
sdl_status sdl_batch_refill_unbatched(sdl_batch *B, void *stream);
/* Tiles / larger rows of the batch (for reporting). */
sdl_status sdl_batch_info(const sdl_batch *B, int *tiles, int *big_rows, long long *terms);
void sdl_batch_destroy(sdl_batch *B);

/* ------------------------------------------------------------------------
   Learned row scheduler. An 8 -> 32 -> 32 -> 4 FP32 MLP over per-row statistics
   (L-row length, term count, longest referenced A row, A's width, and ratios of
   them) predicts each output row's nnz (log1p, regression) and its accumulator
   class (<= 512, <= 8192, > 8192 outputs). It is trained on the labels the exact
   symbolic pass produces, by the library's own CUDA forward / backward / Adam
   kernels. It only changes the schedule: sdl_product_create_learned sizes each
   row's column scratch from the prediction and redoes the rows that do not fit
   with the exact pass, so the product is exactly the one sdl_product_create
   builds.
   ------------------------------------------------------------------------ */
#define SDL_MLP_INPUTS 8
#define SDL_MLP_OUTPUTS 4
#define SDL_MLP_NPARAMS 1476
typedef struct sdl_mlp sdl_mlp;
sdl_status sdl_mlp_create(unsigned long long seed, sdl_mlp **out);
void sdl_mlp_destroy(sdl_mlp *net);
/* Parameters as SDL_MLP_NPARAMS host floats: W1[32][8], b1[32], W2[32][32], b2[32],
   W3[4][32], b3[4]. */
sdl_status sdl_mlp_get_params(const sdl_mlp *net, float *host_params);
sdl_status sdl_mlp_set_params(sdl_mlp *net, const float *host_params);
/* Row statistics of a product: features (device, rows x 8) and, from its exact
   structure, labels (device, rows x 2: log1p(nnz), class). */
sdl_status sdl_product_row_stats(const sdl_product *P, float *feat, float *label, void *stream);
/* Mean loss and its gradient (host, SDL_MLP_NPARAMS floats) over n samples. */
sdl_status sdl_mlp_gradient(const sdl_mlp *net, const float *feat, const float *label, int n,
                            float *host_grad, float *loss);
/* Adam over shuffled mini-batches; *final_loss = mean loss of the last epoch. */
sdl_status sdl_mlp_train(sdl_mlp *net, const float *feat, const float *label, long long n,
                         int epochs, int batch, float lr, unsigned long long seed,
                         float *final_loss);
/* out (device, n x 4): log1p(nnz) prediction and the three class logits. */
sdl_status sdl_mlp_predict(const sdl_mlp *net, const float *feat, long long n, float *out,
                           void *stream);
typedef struct sdl_learned_stats
{
    long long rows;           /* output rows */
    long long term_bound;     /* sum of the rows' term counts (the plain scratch size) */
    long long capacity;       /* sum of the learned capacities (the learned scratch size) */
    long long fallback_rows;  /* rows redone by the exact pass */
    long long fallback_terms; /* their term counts */
    long long class_hits;     /* rows whose predicted class was right */
    long long scratch_bytes;  /* column scratch used, fallback included */
} sdl_learned_stats;
sdl_status sdl_product_create_learned(const sdl_product_desc *desc, const sdl_mlp *net,
                                      float margin, void *stream, sdl_product **out,
                                      sdl_learned_stats *stats);
/* No upstream counterpart: the learned one-shot product, for a pattern met for the
   first time (it replaces upstream's gustavson_alloc passes 1 and 2 and the first
   gustavson_fill_values, src/sparse/gustavson.c:26-143). Structure and values of
   C = kron(I, L) diag(d) A come out of one pass over the terms: every row of up to
   8192 terms is sorted together with its term values into the slots the network
   predicts for it (capacity = predicted nnz x (1 + margin) + 8, at most its term
   count), its columns and its sums -- each in upstream's visiting order, from
   +0.0 -- written at once; a row whose outputs do not fit is flagged and redone
   exactly; larger rows take the exact bitmap pass for their columns and an
   accumulating kernel for their values. No refill plan is built: the product's
   values are at sdl_product_values (device memory owned by P, nnz doubles), and
   sdl_product_fill refuses P until sdl_product_complete_plan has built the plan (a
   pattern that recurs). The result is bit-identical to sdl_product_create followed
   by sdl_product_fill. Lx, d as for sdl_product_fill; Ax is required. Allocates;
   synchronises the stream. sdl_product_plan_ready reports whether P can be refilled. */
sdl_status sdl_product_create_learned_filled(const sdl_product_desc *desc, const sdl_mlp *net, float margin,
                                             const double *Lx, const double *d, const double *Ax, void *stream,
                                             sdl_product **out, sdl_learned_stats *stats);
sdl_status sdl_product_values(const sdl_product *P, const double **Cx);
sdl_status sdl_product_complete_plan(sdl_product *P, void *stream);
sdl_status sdl_product_plan_ready(const sdl_product *P, int *ready);
/* Column scratch bytes the symbolic pass of a product used. */
sdl_status sdl_product_scratch_bytes(const sdl_product *P, long long *bytes);

/* ------------------------------------------------------------------------
   Device-resident stable transpose of a compressed structure (CSR -> CSC,
   CSC -> CSR, A -> A^T). The source is rows x cols with nnz entries; the result
   has cols + 1 offsets, the source row of each entry (ascending within each
   output row) and the source position of each entry (src).
   ------------------------------------------------------------------------ */
typedef struct sdl_transpose sdl_transpose;
sdl_status sdl_transpose_create(const int *p, const int *idx, int rows, int cols,
                                int nnz, void *stream, sdl_transpose **out);
sdl_status sdl_transpose_info(const sdl_transpose *T, const int **Tp,
                              const int **Ti, const int **src);
/* Tx[q] = x[src[q]]. */
sdl_status sdl_transpose_fill(const sdl_transpose *T, const double *x, double *Tx,
                              void *stream);
void sdl_transpose_destroy(sdl_transpose *T);

/* ------------------------------------------------------------------------
   Duplicate coalescing: COO triplets -> CSR with sorted unique columns per row,
   duplicates summed in ascending triplet order (the order upstream's row_reduce
   sums sources in). Two phases: the plan (structure) and the fill (values).
   ------------------------------------------------------------------------ */
typedef struct sdl_coalesce sdl_coalesce;
sdl_status sdl_coalesce_create(const int *rows, const int *cols, int nnz_in, int m,
                               int n, void *stream, sdl_coalesce **out);
sdl_status sdl_coalesce_info(const sdl_coalesce *C, int *nnz_out, const int **Cp,
                             const int **Ci);
sdl_status sdl_coalesce_fill(const sdl_coalesce *C, const double *x, double *Cx,
                             void *stream);
void sdl_coalesce_destroy(sdl_coalesce *C);

/* ------------------------------------------------------------------------
   Dense blocks times a sparse CSR, device-resident: C_k = B_k S[col_perm_k, :]
   for source blocks B_k of shape m0[k] x n0[k] whose columns are the rows
   col_perm[k] (strictly increasing) of S (S_m x S_n). Replaces upstream's
   BA_spd_csr_alloc / BA_spd_csr_fill_values (src/stacked_pd/stacked_pd_linalg.c:
   657-671) and, with one block, BA_pd_csr_alloc / BA_pd_csr_fill_values
   (src/permuted_dense/permuted_dense_linalg.c:313-430). Output block k has
   upstream's shape: B's rows times the columns of S that its rows reach
   (ascending); with keep_empty = 0, blocks without such columns are dropped, as
   upstream's stacked_pd product does. The structure (Sp, Si, col_perm) is read
   from host memory at create; the fill reads device values: B_vals holds the
   source blocks in order, each m0 x n0 row-major (a stacked_pd's value buffer),
   C_vals receives the output blocks in order, each m0 x n0_C row-major. Every
   output is summed in upstream's order, bit for bit.
   ------------------------------------------------------------------------ */
typedef struct sdl_blocks_csr sdl_blocks_csr;
sdl_status sdl_blocks_csr_create(int n_blocks, const int *m0, const int *n0,
                                 const int *const *col_perm, const int *Sp, const int *Si,
                                 int S_m, int S_n, int keep_empty, void *stream,
                                 sdl_blocks_csr **out);
/* Number of output blocks, and the lengths of the C and B value arrays. */
sdl_status sdl_blocks_csr_info(const sdl_blocks_csr *P, int *out_blocks, long long *c_values,
                               long long *b_values);
/* Output block k: its source block, rows, columns and (host) column indices. */
sdl_status sdl_blocks_csr_block(const sdl_blocks_csr *P, int k, int *src_block, int *m0,
                                int *n0_C, const int **col_perm);
sdl_status sdl_blocks_csr_fill(const sdl_blocks_csr *P, const double *B_vals,
                               const double *S_x, double *C_vals, void *stream);
void sdl_blocks_csr_destroy(sdl_blocks_csr *P);

/* ------------------------------------------------------------------------
   A^T diag(d) A of dense blocks, device-resident (upstream ATA_spd_alloc /
   ATDA_spd_fill_values, src/stacked_pd/stacked_pd_linalg.c:197-237; with one
   block ATA_pd_alloc / ATDA_pd_fill_values, src/permuted_dense/
   permuted_dense_linalg.c:87-112). Block k is m0[k] x n0[k] at rows row_perm[k]
   of m and columns col_perm[k] (strictly increasing) of n. Each block's
   X^T diag(d) X runs on the FP64 tensor cores; the partials are coalesced as
   upstream does (output blocks grouped by the set of blocks that hold a row;
   each cell summed from +0.0 in block order). The dgemm inside upstream has no
   specified summation order, so results agree within rounding (about 1e-15 of
   the sum of |terms|), not bit for bit. X_vals: the blocks' values in order,
   row-major; d: m values or NULL (identity); C_vals: the output blocks in order,
   row-major.
   ------------------------------------------------------------------------ */
typedef struct sdl_blocks_ata sdl_blocks_ata;
sdl_status sdl_blocks_ata_create(int n_blocks, const int *m0, const int *n0,
                                 const int *const *row_perm, const int *const *col_perm, int m,
                                 int n, void *stream, sdl_blocks_ata **out);
sdl_status sdl_blocks_ata_info(const sdl_blocks_ata *P, int *out_blocks, long long *c_values,
                               long long *x_values);
sdl_status sdl_blocks_ata_block(const sdl_blocks_ata *P, int k, int *m0, int *n0,
                                const int **rows, const int **cols);
sdl_status sdl_blocks_ata_fill(const sdl_blocks_ata *P, const double *X_vals, const double *d,
                               double *C_vals, void *stream);
void sdl_blocks_ata_destroy(sdl_blocks_ata *P);

/* Host-pointer form for COO_matrix users (no upstream counterpart): the
   coalesced CSR of A (m x n), and a refill of its values from A->x. */
CSR_matrix *COO_coalesce_alloc(const COO_matrix *A);
void COO_coalesce_fill_values(const COO_matrix *A, CSR_matrix *C);

#ifdef __cplusplus
}
#endif

#endif /* SPARSEDIFF_LINALG_CUDA_H */
