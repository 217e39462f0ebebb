// Internal C++ interface of the B200 sparse-product library.
//
// Everything here is device-resident: pointers named d_* or held in DevBuf are
// device memory on the library's device, and every launch goes to the stream the
// caller passes (the library stream by default). The C ABI layers (capi_*.cpp,
// ext_api.cpp) translate host structs and status codes onto these types.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "sparsediff_linalg_cuda.h"

namespace sdl {

// Named span of a host-side phase (symbolic pass, refill plan, refill, host
// transfers) on an Nsight Systems timeline; free when no profiler is attached.
struct NvtxRange
{
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------------- errors
struct Error : std::runtime_error
{
    sdl_status code;
    Error(sdl_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(sdl_status code, const std::string &msg);
[[noreturn]] void cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define SDL_CUDA(call)                                                                 \
    do                                                                                 \
    {                                                                                  \
        cudaError_t sdl_e_ = (call);                                                   \
        if (sdl_e_ != cudaSuccess) ::sdl::cuda_fail(sdl_e_, #call, __FILE__, __LINE__); \
    } while (0)

// Every kernel launch of the library goes through this so launches are counted
// and launch errors surface at the call site.
extern std::atomic<unsigned long long> g_launches;
#define SDL_LAUNCH(kernel, grid, block, smem, stream, ...)                         \
    do                                                                             \
    {                                                                              \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                \
        ::sdl::g_launches.fetch_add(1, std::memory_order_relaxed);                 \
        SDL_CUDA(cudaGetLastError());                                              \
    } while (0)

// ---------------------------------------------------------------- runtime
struct Runtime
{
    int device = -1;
    cudaStream_t stream = nullptr; // library default stream (non-blocking)
    int num_sms = 0;
    int smem_optin = 0; // max dynamic shared memory per block (opt-in)
    int l2_bytes = 0;
    int *d_error = nullptr; // device error word (kernel-side checks), 0 = ok
};

// Initialises on first use (device = current device at that moment). Throws
// Error(SDL_ERR_NO_DEVICE) when no CUDA device is usable.
Runtime &runtime();
inline cudaStream_t pick_stream(void *s)
{
    return s ? static_cast<cudaStream_t>(s) : runtime().stream;
}

// Reads and clears the device error word (synchronises the stream).
int take_device_error(cudaStream_t s);

// ---------------------------------------------------------------- memory
void *dev_alloc(size_t bytes); // from the block cache or cudaMalloc, counted; throws on failure
void dev_free(void *p);         // into the block cache (after a device synchronisation) or cudaFree
void release_cached_device_memory(); // frees the current device's cached blocks
extern std::atomic<unsigned long long> g_dev_allocs;

template <class T>
struct DevBuf
{
    T *ptr = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { reset(count); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), n(o.n)
    {
        o.ptr = nullptr;
        o.n = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o)
        {
            release();
            ptr = o.ptr;
            n = o.n;
            o.ptr = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void reset(size_t count)
    {
        release();
        n = count;
        if (count) ptr = static_cast<T *>(dev_alloc(count * sizeof(T)));
    }
    void release()
    {
        if (ptr) dev_free(ptr);
        ptr = nullptr;
        n = 0;
    }
    T *get() const { return ptr; }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------- primitives
// out[0] = 0, out[k + 1] = in[0] + ... + in[k]; out has n + 1 entries. Returns the
// total (synchronises). For the int variant the caller checks the total fits.
long long exclusive_scan_i64(const long long *d_in, long long *d_out, long long n,
                             cudaStream_t s);
// Exclusive scan of int counts into int offsets; fails with SDL_ERR_OVERFLOW if
// the total exceeds INT_MAX. Returns the total.
int exclusive_scan_i32_checked(const int *d_in, int *d_out, int n, cudaStream_t s);
void fill_iota(int *d, int n, cudaStream_t s);

// Validates a compressed structure (p has rows + 1 entries, indices in [0, cols)):
// p[0] == 0, p non-decreasing, p[rows] == nnz, 0 <= idx < cols. Throws
// SDL_ERR_INVALID otherwise.
void validate_compressed(const int *d_p, const int *d_idx, int rows, int cols, int nnz,
                         const char *what, cudaStream_t s);

// ---------------------------------------------------------------- transpose
// Stable transpose of a compressed structure (rows x cols, nnz entries): Tp has
// cols + 1 offsets, Ti the source row of each transposed entry (ascending inside
// every output row), src the source position of each transposed entry. With
// d_p == nullptr the source is the "one entry per row" structure p = 0..rows.
struct TransposePlan
{
    int rows = 0, cols = 0, nnz = 0;
    DevBuf<int> Tp, Ti, src;
};
void transpose_build(const int *d_p, const int *d_idx, int rows, int cols, int nnz,
                     TransposePlan &out, cudaStream_t s);
// Tx[q] = x[src[q]].
void gather_values(const int *d_src, const double *d_x, double *d_out, int n,
                   cudaStream_t s);

// ---------------------------------------------------------------- coalescing
// Bucketed refill plan of a coalescing (coalesce.cu): for inputs of at least
// COALESCE_BUCKET_MIN triplets the refill first writes the values, chunk by chunk,
// into output-range buckets (lperm: each chunk's triplets in bucket order; cbound:
// each bucket's first position in a chunk's order, nb + 1 per chunk; dst: start of
// every (chunk, bucket) run in buf, chunk-major), then sums every output from its
// bucket (perm2: the buf position of every output-order slot). buf is the plan's
// refill scratch.
constexpr int COALESCE_BUCKET_MIN = 1 << 22;
struct CoalesceBuckets
{
    int n = 0, nb = 0, nchunks = 0;
    DevBuf<unsigned short> lperm;
    DevBuf<int> cbound, perm2;
    DevBuf<long long> dst;
    DevBuf<double> buf;
    bool active() const { return nb > 0; }
};
void coalesce_bucket_build(const int *ostart, const int *perm, int n, int nout, CoalesceBuckets &B, cudaStream_t s);
void coalesce_bucket_fill(const CoalesceBuckets &B, const int *ostart, const double *x, const double *f, int nout,
                          double *C, cudaStream_t s);
// dst[k] = src[k] (int -> long long), k < n.
void widen_i32(const int *d_src, long long *d_dst, long long n, cudaStream_t s);

// ---------------------------------------------------------------- Gustavson
// Row classes of the row-wise product. Thresholds are tunable (autotuner).
enum
{
    SYM_W32 = 0,
    SYM_W128,
    SYM_W512,
    SYM_C2K,
    SYM_C8K,
    SYM_BITMAP,
    SYM_NBINS
};
enum
{
    NUM_TILE = 0, // rows with at most TILE_T terms: row-tile kernel
    NUM_C2K,      // larger rows with <= 2048 / 8192 entries: CTA per row
    NUM_C8K,
    NUM_GMEM, // larger rows: CTA per row, accumulator in C.x itself
    NUM_NBINS
};
// Term budget of a row tile. A tile row costs TILE_T / 256 extra units and a larger
// row TILE_T, so a tile holds at most 256 rows, at most 2 * TILE_T terms and
// outputs, and a larger row is always the last row of its tile (the outputs of a
// tile's rows are one contiguous range of C).
#ifndef SDL_TILE_T
#define SDL_TILE_T 1024
#endif
constexpr int TILE_T = SDL_TILE_T;
constexpr int TILE_THREADS = 256;

// Compiled refill schedule of the tile rows (built once per pattern), entry-major:
// the terms of a tile in upstream's visiting order (the tile's L entries in order,
// each entry's A row in order), one 32-bit word per term:
//   bits 0..11   p, the term's output inside the tile window;
//   bits 12..13  kind: TERM_ONE (the output's only term), TERM_PAIR (one of exactly
//                two), TERM_LIST (one of three or more: summed by the list pass);
//   bits 14..31  e, the term's entry among the tile's L entries.
// With ES[vbase + e] = {bq, slot}, term u of a tile is V[slot] * A.x[bq + u]: V holds
// the entry values L.x * d[k] of one refill (entry-value kernel), bq = A.p[k] minus
// the offset of the entry's first term in its tile. A tile's entries are the
// consecutive entries vbase, vbase + 1, ... (b * L_nnz + ii) of its rows.
constexpr unsigned TERM_ONE = 0u, TERM_PAIR = 1u, TERM_LIST = 2u;
struct TileDesc
{
    int vbase;       // ES index of the tile's first entry
    int word_begin;  // first term word of the tile
    int nterms;      // terms of the tile
    int out_begin;   // first output of the tile in C.x
    int nout;        // outputs of the tile (the window)
    int x_begin;     // list section: nlist + 1 headers (p | start << 12), then term indices
    int nlist;       // outputs with three or more terms
    int prod;        // product index (batched refills), 0 for a single product
};
// Value arrays of one refill of one product.
struct ProdPtrs
{
    const double *Lx, *d, *Ax;
    double *Cx;
};
// Refill schedule of one product as the kernels read it.
struct ProdSched
{
    const unsigned *W; // term words of the tile rows
    const unsigned *X; // list sections
    double *V;         // entry values (refill scratch, nV)
    const int2 *ES;    // per entry: {A.p[k] - tile term offset, slot of its value in V}
    const int *Li, *L_map;
    const int *kv;     // V in L's value order: row of A of each value (else null)
    long long nV, nA; // entries of kron(I_blocks, L), entries of A
    int L_nnz, n_L, blocks, pad;
};
// A run of one product's entries (batched entry values).
struct EntChunk
{
    long long begin;
    int count;
    int prod;
};

// Run-time parameters of a product's plan (the autotuner picks them per pattern).
struct TuneConfig
{
    // symbolic pass: rows with at most 32 / 128 / 512 terms go to the warp kernel of
    // that capacity, rows above warp_max_terms (128 or 512) to the CTA kernels
    int warp_max_terms = 512;
    int rows_per_cta_warp = 8;  // warps per CTA of the warp kernels
    int cta_threads_2k = 256;   // threads of the CTA kernel for rows up to 2048 terms
    int cta_threads_8k = 512;
    int gmem_threads = 512;
    // refill: weight (terms plus per-row costs) of a row tile, at most TILE_T, and
    // resident refill CTAs per SM (0: as many as fit)
    int tile_budget = 0; // 0: TILE_T
    int refill_ctas_per_sm = 0;
    // rows with more terms leave the tiles for the larger-row kernels (0: TILE_T);
    // refill CTA threads: 256, or 128 for plans whose tiles have at most TILE_T
    // outputs (tile budget and tile_max_terms at most TILE_T / 2)
    int tile_max_terms = 0;
    int refill_threads = 256;
    // the pipelined refill (tile data staged ahead by asynchronous copies) for plans
    // whose tiles all fit its stages (1), or the direct one (0, the default: on the
    // patterns measured so far the direct refill is faster; the autotuner tries both)
    int refill_pipe = 0;
    // the staged direct refill (1: tile words and entry records bulk-copied into
    // shared memory a tile ahead) where its slots fit, or the plain direct one (0);
    // the autotuner tries both
    int refill_es = 0;
};
// Autotuner results: the chosen configuration and what it measured.
struct TuneResult
{
    TuneConfig best;
    double sym_ms = 0, refill_us = 0, default_refill_us = 0, tune_ms = 0;
    int candidates = 0;
};

// Operand description of C = kron(I_blocks, L) diag(d) A.
struct ProductDesc
{
    const int *Lp = nullptr; // L_m + 1
    const int *Li = nullptr; // column index of each L entry (row of A within a block)
    const int *L_map = nullptr; // optional: value of L entry ii is Lx[L_map[ii]]
    int L_m = 0, L_nnz = 0;
    int blocks = 1;
    const int *Ap = nullptr, *Ai = nullptr;
    int A_m = 0, A_n = 0, A_nnz = 0;
};

struct Product
{
    ProductDesc desc;
    int m_out = 0, n = 0, nnz = 0, n_L = 0;
    long long terms = 0;
    long long scratch_bytes = 0; // column scratch the symbolic pass used
    DevBuf<int> Cp, Ci;
    DevBuf<int> num_rows; // row ids grouped by numeric class
    int num_count[NUM_NBINS] = {0};
    int num_offset[NUM_NBINS + 1] = {0};
    // Compiled refill schedule of the tile rows.
    int ntiles = 0;
    int max_tile_out = 0; // largest tile window of the plan
    int max_tile_terms = 0, max_tile_ent = 0; // largest term / entry count of a tile
    DevBuf<int> tile_nent; // entries of every tile
    DevBuf<TileDesc> tiles;
    DevBuf<unsigned> W, X; // term words, list sections
    DevBuf<int2> ES;       // per entry: {A.p[k] - tile term offset, V slot} (L_nnz * blocks)
    DevBuf<int> kv;        // V in L's value order (L_map a permutation): row of A per value
    DevBuf<double> V;      // entry values of the current refill (L_nnz * blocks)
    DevBuf<int> gmem_scratch; // posmap scratch for NUM_GMEM rows (slots x n ints)
    int gmem_slots = 0;
    // Rows beyond the tile budget, output-major: every output's terms as {A
    // position, entry-value slot} pairs in upstream's visiting order (big_lists).
    bool big_lists = false;
    int nbig = 0, big_outputs = 0;
    DevBuf<int> brows;          // the rows (big row i = brows[i])
    DevBuf<int> bout_off;       // outputs of big rows before big row i (nbig + 1)
    DevBuf<int> bostart;        // first pair of every big-row output (big_outputs + 1)
    DevBuf<uint2> bpairs;       // the pairs
    TuneConfig cfg;
    // per-row statistics kept for the learned scheduler (optional)
    DevBuf<long long> row_terms; // ub per row
    // false for a product made by the learned one-shot pass until its refill plan is
    // built (product_complete_plan); its fills are refused until then
    bool plan_ready = true;
};

// Re-plans P with configuration c (same structure; the schedule follows c).
void product_replan(Product &P, const TuneConfig &c, cudaStream_t s);

// Autotuner: re-plans P (built by product_symbolic) for its own pattern. Candidate
// symbolic configurations are timed on the pattern, then candidate tile budgets and
// refill CTAs per SM by refills with placeholder values (L2 flushed before each);
// P ends up planned with the fastest, which is returned with its timings.
TuneResult product_autotune(Product &P, int reps, cudaStream_t s);
// Key of P's pattern for the tuning table: rows of C, columns of A, terms per row,
// terms per output and the histogram of C's row lengths over power-of-two classes
// (each class's share of the rows in eighths). Synchronises the stream.
std::string product_pattern_key(const Product &P, cudaStream_t s);
// The process's tuning table (tune_table.cpp): the configuration recorded for a
// pattern key (record replaces an earlier one), and its lookup.
void tune_table_record(const std::string &key, const TuneConfig &c, double refill_us);
bool tune_table_lookup(const std::string &key, TuneConfig &c);
// Symbolic phase: fills P.Cp, P.Ci, P.nnz and the numeric schedule.
void product_symbolic(const ProductDesc &d, const TuneConfig &cfg, Product &P,
                      cudaStream_t s, bool keep_row_terms = false);
// Learned one-shot pass of a pattern met for the first time: C's structure and
// values (Cx, allocated here) in one pass over the terms -- rows of up to 8192 terms
// sorted with their values into the network's predicted capacity (rows that do not
// fit are redone exactly), larger rows by the exact bitmap pass and an accumulating
// kernel -- without building the refill plan. P then holds C's structure with
// plan_ready = false; product_complete_plan builds the plan for later refills.
struct LearnedStats;
struct Mlp;
void product_oneshot_learned(const ProductDesc &d, const TuneConfig &cfg, const Mlp &net, float margin,
                             const double *Lx, const double *dvec, const double *Ax, Product &P,
                             DevBuf<double> &Cx, LearnedStats &st, cudaStream_t s);
void product_complete_plan(Product &P, cudaStream_t s);
// Statistics of a learned symbolic pass.
struct LearnedStats
{
    long long rows = 0, ub_total = 0, cap_total = 0, fallback_terms = 0, fallback_rows = 0,
              class_hits = 0;
};
struct Mlp;
// Symbolic phase with the learned row scheduler: each row's column scratch is
// sized from the network's predicted nnz (times 1 + margin) instead of its term
// count; rows that do not fit are redone by the exact pass. The structure is the
// exact one in every case.
void product_symbolic_learned(const ProductDesc &d, const TuneConfig &cfg, const Mlp &net, float margin,
                              Product &P, LearnedStats &st, cudaStream_t s);

// Numeric phase. Lx: values of L (indexed through L_map when set), or nullptr for
// a unit L (every L value 1.0). d: A_m values or nullptr. Never allocates.
void product_numeric(const Product &P, const double *Lx, const double *d,
                     const double *Ax, double *Cx, cudaStream_t s);
// The schedule of a product as the refill kernels read it.
ProdSched sched_of(const Product &P);
// Entry values V of one product for the given values (first kernel of a refill).
void entry_values(const ProdSched &S, const ProdPtrs &vals, cudaStream_t s);
// Entry values of many products: chunks of their entries, pointers from the tables.
void entry_values_batched(const EntChunk *chunks, int nchunks, const ProdPtrs *ptrs,
                          const ProdSched *scheds, cudaStream_t s);
// Chunks of at most `chunk` entries covering nV entries of product `prod`.
void append_entry_chunks(long long nV, int prod, int chunk, std::vector<EntChunk> &out);
// The tile refill over a descriptor list that may mix products (batched refills):
// tile t reads its pointers from ptrs[tiles[t].prod] / scheds[tiles[t].prod], or,
// with null tables, from `vals` / `sched`.
void tile_refill(const TileDesc *tiles, int ntiles, const ProdPtrs *ptrs, const ProdSched *scheds,
                 cudaStream_t s, ProdPtrs vals = ProdPtrs{}, ProdSched sched = ProdSched{},
                 int ctas_per_sm = 0, bool small = false, const int *tile_nent = nullptr, int wcap = 0,
                 int ecap = 0);
// Whether a single product's refill runs the staged direct kernel (each tile's term
// words and entry records bulk-copied into shared memory while the tile before it
// runs), and that kernel's slot capacities (words, records) for P's tiles.
bool es_refill(const Product &P);
void staged_caps(const Product &P, int &wcap, int &ecap);
// Whether a single product's refill runs the 128-thread small-tile kernel.
bool small_tile_refill(const Product &P);
// Whether P's tiles are refilled by the pipelined kernel (its configuration asks for
// it and every tile fits the kernel's stages).
bool pipe_refill(const Product &P);
// Whether a product's entry values are L.x itself (no d, one block, values in L's
// value order or no L_map): the refill then reads L.x and skips the entry values.
bool entry_values_are_lx(const Product &P, const double *Lx, const double *dvec);
// Copies `n` descriptors, setting `prod`.
void rebase_tiles(const TileDesc *src, int n, int prod, TileDesc *dst, cudaStream_t s);
// The larger rows of one product from their output-major term lists (needs
// P.big_lists), values as in tile_refill.
// V: the entry values to read (null: the product's own scratch).
void big_lists_refill(const Product &P, const ProdPtrs *ptrs, cudaStream_t s, ProdPtrs vals = ProdPtrs{},
                      const double *V = nullptr);
// The larger rows of one product (CTA kernels), for the given values; with `vals`
// (a device ProdPtrs) the kernels read the value pointers from there instead.
void big_rows_refill(const Product &P, const double *Lx, const double *d, const double *Ax,
                     double *Cx, cudaStream_t s, const ProdPtrs *vals = nullptr);

} // namespace sdl
