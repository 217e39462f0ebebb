#include <cstring>
// Device-resident extension API (sparsediff_linalg_cuda.h): products, transposes
// and duplicate coalescing whose operands and results stay in HBM.
#include <memory>

#include "capi_common.h"

using namespace sdl;

struct sdl_product
{
    Product P;
    TuneResult tuned;
    DevBuf<double> values; // C's values from the learned one-shot pass
};

struct sdl_transpose
{
    TransposePlan T;
};

// Coalescing = group triplets by row (stable transpose of the one-entry-per-row
// structure rows[]), then a unit-valued row-wise product with the triplet matrix
// (row t = {(cols[t], x[t])}): each output entry sums its duplicates in ascending
// triplet order, starting from +0.0, as upstream's row_reduce does. The product's
// symbolic pass gives the output structure; value refills gather in output order
// (coalesce.cu), which sums in the same order.
struct sdl_coalesce
{
    int m = 0, n = 0, nnz_in = 0, nout = 0;
    DevBuf<int> Cp, Ci;       // the coalesced CSR structure
    DevBuf<int> perm, ostart; // triplets in output order; first slot of every output
    CoalesceBuckets buckets;  // bucketed refill plan (large inputs)
};

namespace sdl {
void coalesce_fill_scaled(const sdl_coalesce *C, const double *x, const double *d, double *Cx, cudaStream_t s);
int coalesce_sorted_build(const int *rows, const int *cols, int n, int m, int ncols, DevBuf<int> &Cp, DevBuf<int> &Ci,
                          DevBuf<int> &perm, DevBuf<int> &ostart, cudaStream_t s);
void coalesce_order_fill(const int *ostart, const int *perm, const double *x, const double *f, int nout, double *C,
                         cudaStream_t s);
} // namespace sdl

extern "C" int sdl_device_available(void)
{
    try
    {
        runtime();
        return 1;
    }
    catch (...)
    {
        return 0;
    }
}

extern "C" unsigned long long sdl_device_alloc_count(void) { return g_dev_allocs.load(); }

extern "C" void sdl_release_cached_memory(void) { release_cached_device_memory(); }
extern "C" unsigned long long sdl_kernel_launch_count(void) { return g_launches.load(); }

extern "C" void *sdl_stream(void)
{
    try
    {
        return runtime().stream;
    }
    catch (...)
    {
        return nullptr;
    }
}

extern "C" sdl_status sdl_synchronize(void)
{
    return guard_status("sdl_synchronize", [&]() { SDL_CUDA(cudaStreamSynchronize(runtime().stream)); });
}

extern "C" void sdl_free(void *device_ptr) { dev_free(device_ptr); }

// ------------------------------------------------------------------ product
extern "C" sdl_status sdl_product_create(const sdl_product_desc *desc, void *stream,
                                         sdl_product **out)
{
    return guard_status("sdl_product_create", [&]() {
        if (!desc || !out) fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        ProductDesc d;
        d.Lp = desc->Lp;
        d.Li = desc->Li;
        d.L_map = desc->L_map;
        d.L_m = desc->L_m;
        d.L_nnz = desc->L_nnz;
        d.blocks = desc->blocks;
        d.Ap = desc->Ap;
        d.Ai = desc->Ai;
        d.A_m = desc->A_m;
        d.A_n = desc->A_n;
        d.A_nnz = desc->A_nnz;
        if (!d.Lp || !d.Ap) fail(SDL_ERR_INVALID, "NULL structure pointer");
        auto p = std::make_unique<sdl_product>();
        product_symbolic(d, TuneConfig{}, p->P, pick_stream(stream));
        *out = p.release();
    });
}

extern "C" sdl_status sdl_product_autotune(sdl_product *P, int reps, void *stream)
{
    return guard_status("sdl_product_autotune", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        cudaStream_t s = pick_stream(stream);
        P->tuned = product_autotune(P->P, reps, s);
        tune_table_record(product_pattern_key(P->P, s), P->P.cfg, P->tuned.refill_us);
    });
}

extern "C" sdl_status sdl_product_apply_tuned(sdl_product *P, int *found, void *stream)
{
    return guard_status("sdl_product_apply_tuned", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        if (found) *found = 0;
        cudaStream_t s = pick_stream(stream);
        TuneConfig c;
        if (!tune_table_lookup(product_pattern_key(P->P, s), c)) return;
        product_replan(P->P, c, s);
        P->tuned = TuneResult{};
        P->tuned.best = c;
        if (found) *found = 1;
    });
}

extern "C" sdl_status sdl_product_pattern_key(const sdl_product *P, char *buf, int len, void *stream)
{
    return guard_status("sdl_product_pattern_key", [&]() {
        if (!P || !buf || len <= 0) fail(SDL_ERR_INVALID, "NULL argument");
        const std::string k = product_pattern_key(P->P, pick_stream(stream));
        if ((int)k.size() >= len) fail(SDL_ERR_INVALID, "key buffer too short");
        std::memcpy(buf, k.c_str(), k.size() + 1);
    });
}

extern "C" sdl_status sdl_product_tuning(const sdl_product *P, int *warp_max_terms, int *rows_per_cta_warp,
                                         int *tile_budget, int *refill_ctas_per_sm, double *refill_us,
                                         double *default_refill_us, int *candidates, double *tune_ms)
{
    return guard_status("sdl_product_tuning", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        const TuneConfig &c = P->P.cfg;
        if (warp_max_terms) *warp_max_terms = c.warp_max_terms;
        if (rows_per_cta_warp) *rows_per_cta_warp = c.rows_per_cta_warp;
        if (tile_budget) *tile_budget = c.tile_budget > 0 ? c.tile_budget : TILE_T;
        if (refill_ctas_per_sm) *refill_ctas_per_sm = c.refill_ctas_per_sm;
        if (refill_us) *refill_us = P->tuned.refill_us;
        if (default_refill_us) *default_refill_us = P->tuned.default_refill_us;
        if (candidates) *candidates = P->tuned.candidates;
        if (tune_ms) *tune_ms = P->tuned.tune_ms;
    });
}

extern "C" sdl_status sdl_product_replan(sdl_product *P, int tile_budget, int tile_max_terms,
                                         int refill_threads, int refill_ctas_per_sm, void *stream)
{
    return guard_status("sdl_product_replan", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        TuneConfig c = P->P.cfg;
        c.tile_budget = tile_budget;
        c.tile_max_terms = tile_max_terms;
        c.refill_threads = refill_threads;
        c.refill_ctas_per_sm = refill_ctas_per_sm;
        product_replan(P->P, c, pick_stream(stream));
    });
}

extern "C" sdl_status sdl_product_set_refill_pipe(sdl_product *P, int on, int *used)
{
    return guard_status("sdl_product_set_refill_pipe", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        P->P.cfg.refill_pipe = on ? 1 : 0;
        if (on) P->P.cfg.refill_es = 0;
        if (used) *used = pipe_refill(P->P) ? 1 : 0;
    });
}

extern "C" sdl_status sdl_product_set_refill_staged(sdl_product *P, int on, int *used)
{
    return guard_status("sdl_product_set_refill_staged", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        P->P.cfg.refill_es = on ? 1 : 0;
        if (on) P->P.cfg.refill_pipe = 0;
        if (used) *used = es_refill(P->P) ? 1 : 0;
    });
}

extern "C" sdl_status sdl_product_refill_staged_used(const sdl_product *P, int *used)
{
    return guard_status("sdl_product_refill_staged_used", [&]() {
        if (!P || !used) fail(SDL_ERR_INVALID, "NULL argument");
        *used = es_refill(P->P) ? 1 : 0;
    });
}

extern "C" sdl_status sdl_product_refill_pipe_used(const sdl_product *P, int *used)
{
    return guard_status("sdl_product_refill_pipe_used", [&]() {
        if (!P || !used) fail(SDL_ERR_INVALID, "NULL argument");
        *used = pipe_refill(P->P) ? 1 : 0;
    });
}

extern "C" sdl_status sdl_product_refill_shape(const sdl_product *P, int *refill_threads, int *tile_max_terms)
{
    return guard_status("sdl_product_refill_shape", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        const TuneConfig &c = P->P.cfg;
        if (refill_threads) *refill_threads = small_tile_refill(P->P) ? c.refill_threads : 256;
        if (tile_max_terms) *tile_max_terms = c.tile_max_terms > 0 ? c.tile_max_terms : TILE_T;
    });
}

extern "C" sdl_status sdl_product_info(const sdl_product *P, int *m, int *n, int *nnz,
                                       long long *terms, const int **Cp, const int **Ci)
{
    return guard_status("sdl_product_info", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        if (m) *m = P->P.m_out;
        if (n) *n = P->P.n;
        if (nnz) *nnz = P->P.nnz;
        if (terms) *terms = P->P.terms;
        if (Cp) *Cp = P->P.Cp.get();
        if (Ci) *Ci = P->P.Ci.get();
    });
}

extern "C" sdl_status sdl_product_fill(const sdl_product *P, const double *Lx, const double *d,
                                       const double *Ax, double *Cx, void *stream)
{
    return guard_status("sdl_product_fill", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        if (P->P.nnz > 0 && (!Ax || !Cx)) fail(SDL_ERR_INVALID, "NULL value pointer");
        product_numeric(P->P, Lx, d, Ax, Cx, pick_stream(stream));
    });
}

extern "C" void sdl_product_destroy(sdl_product *P) { delete P; }

namespace sdl {
const Product *product_of(const sdl_product *P) { return P ? &P->P : nullptr; }

sdl_product *product_new_learned(const ProductDesc &d, const Mlp &net, float margin, LearnedStats &st,
                                 cudaStream_t s)
{
    auto p = std::make_unique<sdl_product>();
    product_symbolic_learned(d, TuneConfig{}, net, margin, p->P, st, s);
    return p.release();
}

sdl_product *product_new_learned_oneshot(const ProductDesc &d, const Mlp &net, float margin, const double *Lx,
                                         const double *dvec, const double *Ax, LearnedStats &st, cudaStream_t s)
{
    auto p = std::make_unique<sdl_product>();
    product_oneshot_learned(d, TuneConfig{}, net, margin, Lx, dvec, Ax, p->P, p->values, st, s);
    return p.release();
}
} // namespace sdl

extern "C" sdl_status sdl_product_values(const sdl_product *P, const double **Cx)
{
    return guard_status("sdl_product_values", [&]() {
        if (!P || !Cx) fail(SDL_ERR_INVALID, "NULL argument");
        *Cx = P->values.get();
    });
}

extern "C" sdl_status sdl_product_complete_plan(sdl_product *P, void *stream)
{
    return guard_status("sdl_product_complete_plan", [&]() {
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        product_complete_plan(P->P, pick_stream(stream));
    });
}

extern "C" sdl_status sdl_product_plan_ready(const sdl_product *P, int *ready)
{
    return guard_status("sdl_product_plan_ready", [&]() {
        if (!P || !ready) fail(SDL_ERR_INVALID, "NULL argument");
        *ready = P->P.plan_ready ? 1 : 0;
    });
}

namespace sdl {
} // namespace sdl

// ------------------------------------------------------------------ transpose
extern "C" sdl_status sdl_transpose_create(const int *p, const int *idx, int rows, int cols, int nnz,
                                           void *stream, sdl_transpose **out)
{
    return guard_status("sdl_transpose_create", [&]() {
        if (!out) fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        cudaStream_t s = pick_stream(stream);
        validate_compressed(p, idx, rows, cols, nnz, "transpose operand", s);
        auto t = std::make_unique<sdl_transpose>();
        transpose_build(p, idx, rows, cols, nnz, t->T, s);
        *out = t.release();
    });
}

extern "C" sdl_status sdl_transpose_info(const sdl_transpose *T, const int **Tp, const int **Ti,
                                         const int **src)
{
    return guard_status("sdl_transpose_info", [&]() {
        if (!T) fail(SDL_ERR_INVALID, "NULL transpose");
        if (Tp) *Tp = T->T.Tp.get();
        if (Ti) *Ti = T->T.Ti.get();
        if (src) *src = T->T.src.get();
    });
}

extern "C" sdl_status sdl_transpose_fill(const sdl_transpose *T, const double *x, double *Tx,
                                         void *stream)
{
    return guard_status("sdl_transpose_fill", [&]() {
        if (!T) fail(SDL_ERR_INVALID, "NULL transpose");
        gather_values(T->T.src.get(), x, Tx, T->T.nnz, pick_stream(stream));
    });
}

extern "C" void sdl_transpose_destroy(sdl_transpose *T) { delete T; }

// ------------------------------------------------------------------ coalesce
extern "C" sdl_status sdl_coalesce_create(const int *rows, const int *cols, int nnz_in, int m, int n,
                                          void *stream, sdl_coalesce **out)
{
    return guard_status("sdl_coalesce_create", [&]() {
        if (!out) fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        if (nnz_in < 0 || m < 0 || n < 0) fail(SDL_ERR_INVALID, "negative size");
        cudaStream_t s = pick_stream(stream);
        validate_compressed(nullptr, rows, 0, m, nnz_in, "coalesce rows", s);
        validate_compressed(nullptr, cols, 0, n, nnz_in, "coalesce cols", s);
        auto c = std::make_unique<sdl_coalesce>();
        c->m = m;
        c->n = n;
        c->nnz_in = nnz_in;
        c->nout = coalesce_sorted_build(rows, cols, nnz_in, m, n, c->Cp, c->Ci, c->perm, c->ostart, s);
        coalesce_bucket_build(c->ostart.get(), c->perm.get(), nnz_in, c->nout, c->buckets, s);
        *out = c.release();
    });
}

extern "C" sdl_status sdl_coalesce_info(const sdl_coalesce *C, int *nnz_out, const int **Cp,
                                        const int **Ci)
{
    return guard_status("sdl_coalesce_info", [&]() {
        if (!C) fail(SDL_ERR_INVALID, "NULL plan");
        if (nnz_out) *nnz_out = C->nout;
        if (Cp) *Cp = C->Cp.get();
        if (Ci) *Ci = C->Ci.get();
    });
}

extern "C" sdl_status sdl_coalesce_fill(const sdl_coalesce *C, const double *x, double *Cx,
                                        void *stream)
{
    return guard_status("sdl_coalesce_fill", [&]() {
        if (!C) fail(SDL_ERR_INVALID, "NULL plan");
        coalesce_fill_scaled(C, x, nullptr, Cx, pick_stream(stream));
    });
}

extern "C" void sdl_coalesce_destroy(sdl_coalesce *C) { delete C; }

namespace sdl {
// Coalesce with a factor per input triplet: each output sums (1 * d[t]) * x[t]
// over its duplicates in ascending t, from +0.0 (d null: x[t]).
void coalesce_fill_scaled(const sdl_coalesce *C, const double *x, const double *d, double *Cx, cudaStream_t s)
{
    if (C->buckets.active())
        coalesce_bucket_fill(C->buckets, C->ostart.get(), x, d, C->nout, Cx, s);
    else
        coalesce_order_fill(C->ostart.get(), C->perm.get(), x, d, C->nout, Cx, s);
}
} // namespace sdl
