// Batched refill engine (sdl_batch_*): many products refilled by a few launches
// over the union of their compiled schedules, replayed from a CUDA graph. The
// products are cut into consecutive groups whose entry values and entry records
// fit in L2 next to the next group's; per group, one launch computes the entry
// values of every product of the group (on a side stream) and one persistent
// launch refills every tile of the group (on the caller's stream, after it), so
// the refill reads the entry values from L2 instead of HBM, and the entry values
// of group g + 1 are computed while group g is refilled (they wait for the refill
// of group g - 1 only, so they do not run further ahead). The plain alternative --
// one sdl_product_fill per product -- pays two launches (and their ramp-up and
// tail) per product. Each product's schedule and entry-value scratch stay where the
// product keeps them; the kernels find them through per-product pointer tables.
#include <memory>
#include <vector>

#include "capi_common.h"

// default bytes of entry values and entry records (16 per entry) of a group
constexpr long long kGroupBytes = 64LL << 20;

namespace sdl {
const Product *product_of(const sdl_product *P);
} // namespace sdl

using namespace sdl;

struct sdl_batch
{
    std::vector<const Product *> prods;
    int ntiles = 0;
    long long terms = 0;
    int big_rows = 0;
    DevBuf<TileDesc> tiles;
    DevBuf<ProdSched> scheds;
    DevBuf<EntChunk> chunks;
    int nchunks = 0;
    unsigned long long launches_per_refill = 0; // kernels one refill launches (graph replays)
    DevBuf<ProdPtrs> ptrs;
    std::vector<ProdPtrs> host_ptrs;
    std::vector<int> with_big; // products that have rows beyond the tile budget
    // per product: end of its tiles / entry chunks, bytes of its entry values and records
    std::vector<int> prod_tile_end, prod_chunk_end;
    std::vector<long long> prod_bytes;
    // group g: tiles [group_tiles[g], group_tiles[g + 1]) and entry chunks
    // [group_chunks[g], group_chunks[g + 1])
    long long group_bytes = kGroupBytes;
    std::vector<int> group_tiles, group_chunks;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // side stream of the entry-value launches and the events that order them
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    std::vector<cudaEvent_t> entry_done, refill_done; // per group
    void drop_group_events()
    {
        for (cudaEvent_t e : entry_done) cudaEventDestroy(e);
        for (cudaEvent_t e : refill_done) cudaEventDestroy(e);
        entry_done.clear();
        refill_done.clear();
    }
    ~sdl_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        drop_group_events();
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
    }
};

namespace {
// Cuts the products, in order, into groups: a group closes once its products'
// entry values and records reach B.group_bytes (0: one group).
void make_groups(sdl_batch &B)
{
    B.group_tiles.assign(1, 0);
    B.group_chunks.assign(1, 0);
    long long in_group = 0;
    const size_t n = B.prods.size();
    for (size_t i = 0; i < n; ++i)
    {
        in_group += B.prod_bytes[i];
        if (B.group_bytes > 0 && in_group >= B.group_bytes)
        {
            B.group_tiles.push_back(B.prod_tile_end[i]);
            B.group_chunks.push_back(B.prod_chunk_end[i]);
            in_group = 0;
        }
    }
    if (B.ntiles > B.group_tiles.back() || B.nchunks > B.group_chunks.back())
    {
        B.group_tiles.push_back(B.ntiles);
        B.group_chunks.push_back(B.nchunks);
    }
    B.drop_group_events();
    const size_t ngroups = B.group_tiles.size() - 1;
    B.entry_done.assign(ngroups, nullptr);
    B.refill_done.assign(ngroups, nullptr);
    for (size_t g = 0; g < ngroups; ++g)
    {
        SDL_CUDA(cudaEventCreateWithFlags(&B.entry_done[g], cudaEventDisableTiming));
        SDL_CUDA(cudaEventCreateWithFlags(&B.refill_done[g], cudaEventDisableTiming));
    }
}
} // namespace

extern "C" sdl_status sdl_batch_create(sdl_product *const *products, int count, void *stream,
                                       sdl_batch **out)
{
    return guard_status("sdl_batch_create", [&]() {
        if (!out || (count > 0 && !products)) fail(SDL_ERR_INVALID, "NULL argument");
        *out = nullptr;
        cudaStream_t s = pick_stream(stream);
        auto B = std::make_unique<sdl_batch>();
        for (int i = 0; i < count; ++i)
        {
            const Product *P = product_of(products[i]);
            if (!P) fail(SDL_ERR_INVALID, "NULL product in batch");
            for (const Product *Q : B->prods)
                if (Q == P) fail(SDL_ERR_INVALID, "a product appears twice in the batch");
            B->prods.push_back(P);
            B->ntiles += P->num_count[NUM_TILE] ? P->ntiles : 0;
            B->terms += P->terms;
            int big = P->num_count[NUM_C2K] + P->num_count[NUM_C8K] + P->num_count[NUM_GMEM];
            B->big_rows += big;
            if (big) B->with_big.push_back(i);
        }
        B->tiles.reset(std::max(1, B->ntiles));
        B->ptrs.reset(std::max(1, count));
        B->scheds.reset(std::max(1, count));
        B->host_ptrs.assign(count, ProdPtrs{nullptr, nullptr, nullptr, nullptr});
        std::vector<ProdSched> hs(count);
        std::vector<EntChunk> chunks;
        int t_off = 0;
        B->prod_tile_end.assign(count, 0);
        B->prod_chunk_end.assign(count, 0);
        B->prod_bytes.assign(count, 0);
        for (int i = 0; i < count; ++i)
        {
            const Product *P = B->prods[i];
            hs[i] = sched_of(*P);
            if (P->num_count[NUM_TILE] && P->ntiles)
            {
                rebase_tiles(P->tiles.get(), P->ntiles, i, B->tiles.get() + t_off, s);
                t_off += P->ntiles;
            }
            if ((P->num_count[NUM_TILE] && P->ntiles) || P->big_lists)
            {
                append_entry_chunks(hs[i].nV, i, 2048, chunks);
                B->prod_bytes[i] = 16 * hs[i].nV;
            }
            B->prod_tile_end[i] = t_off;
            B->prod_chunk_end[i] = (int)chunks.size();
        }
        SDL_CUDA(cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking));
        SDL_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
        SDL_CUDA(cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming));
        if (count)
            SDL_CUDA(cudaMemcpyAsync(B->scheds.get(), hs.data(), count * sizeof(ProdSched),
                                     cudaMemcpyHostToDevice, s));
        B->nchunks = (int)chunks.size();
        make_groups(*B);
        B->chunks.reset(std::max<size_t>(1, chunks.size()));
        if (!chunks.empty())
            SDL_CUDA(cudaMemcpyAsync(B->chunks.get(), chunks.data(), chunks.size() * sizeof(EntChunk),
                                     cudaMemcpyHostToDevice, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        *out = B.release();
    });
}

extern "C" sdl_status sdl_batch_set_group_bytes(sdl_batch *B, long long bytes)
{
    return guard_status("sdl_batch_set_group_bytes", [&]() {
        if (!B || bytes < 0) fail(SDL_ERR_INVALID, "bad batch or group size");
        if (B->exec) fail(SDL_ERR_INVALID, "the batch has been refilled: its groups are fixed");
        B->group_bytes = bytes;
        make_groups(*B);
    });
}

extern "C" sdl_status sdl_batch_groups(const sdl_batch *B, int *groups)
{
    return guard_status("sdl_batch_groups", [&]() {
        if (!B || !groups) fail(SDL_ERR_INVALID, "NULL argument");
        *groups = (int)B->entry_done.size();
    });
}

extern "C" sdl_status sdl_batch_bind(sdl_batch *B, int i, const double *Lx, const double *d,
                                     const double *Ax, double *Cx)
{
    return guard_status("sdl_batch_bind", [&]() {
        if (!B || i < 0 || i >= (int)B->prods.size()) fail(SDL_ERR_INVALID, "bad batch index");
        const Product *P = B->prods[i];
        if (P->nnz > 0 && (!Ax || !Cx)) fail(SDL_ERR_INVALID, "NULL value pointer");
        B->host_ptrs[i] = ProdPtrs{Lx, d, Ax, Cx};
        SDL_CUDA(cudaMemcpy(B->ptrs.get() + i, &B->host_ptrs[i], sizeof(ProdPtrs), cudaMemcpyHostToDevice));
    });
}

namespace {
// One refill of the batch, enqueued on s: per group, the entry values of its products
// on the side stream (after the refill of group g - 2, so they run at most one group
// ahead), then the group's tiles on s; then the rows beyond the tile budget.
void batch_enqueue(sdl_batch &Bq, cudaStream_t s)
{
    sdl_batch *B = &Bq;
    SDL_CUDA(cudaEventRecord(B->fork, s));
    SDL_CUDA(cudaStreamWaitEvent(B->side, B->fork, 0));
    for (size_t g = 0; g < B->entry_done.size(); ++g)
    {
        const int c0 = B->group_chunks[g], t0 = B->group_tiles[g];
        if (g >= 2) SDL_CUDA(cudaStreamWaitEvent(B->side, B->refill_done[g - 2], 0));
        entry_values_batched(B->chunks.get() + c0, B->group_chunks[g + 1] - c0, B->ptrs.get(), B->scheds.get(),
                             B->side);
        SDL_CUDA(cudaEventRecord(B->entry_done[g], B->side));
        SDL_CUDA(cudaStreamWaitEvent(s, B->entry_done[g], 0));
        tile_refill(B->tiles.get() + t0, B->group_tiles[g + 1] - t0, B->ptrs.get(), B->scheds.get(), s);
        SDL_CUDA(cudaEventRecord(B->refill_done[g], s));
    }
    SDL_CUDA(cudaEventRecord(B->join, B->side));
    SDL_CUDA(cudaStreamWaitEvent(s, B->join, 0));
    for (int i : B->with_big)
    {
        const ProdPtrs &pp = B->host_ptrs[i];
        if (B->prods[i]->big_lists)
            big_lists_refill(*B->prods[i], B->ptrs.get() + i, s);
        else
            big_rows_refill(*B->prods[i], pp.Lx, pp.d, pp.Ax, pp.Cx, s, B->ptrs.get() + i);
    }
}

void check_bound(const sdl_batch &B)
{
    for (size_t i = 0; i < B.prods.size(); ++i)
        if (B.prods[i]->nnz > 0 && !B.host_ptrs[i].Cx)
            fail(SDL_ERR_INVALID, "product " + std::to_string(i) + " has no bound values");
}
} // namespace

extern "C" sdl_status sdl_batch_autotune(sdl_batch *B, int reps, void *stream, long long *group_bytes, double *ms)
{
    return guard_status("sdl_batch_autotune", [&]() {
        if (!B) fail(SDL_ERR_INVALID, "NULL batch");
        if (B->exec) fail(SDL_ERR_INVALID, "the batch has been refilled: its groups are fixed");
        check_bound(*B);
        cudaStream_t s = pick_stream(stream);
        if (s == cudaStreamLegacy) fail(SDL_ERR_INVALID, "batched refills need a non-default stream");
        reps = std::max(1, std::min(reps, 20));
        cudaEvent_t e0, e1;
        SDL_CUDA(cudaEventCreate(&e0));
        SDL_CUDA(cudaEventCreate(&e1));
        const long long cands[] = {16LL << 20, 32LL << 20, 64LL << 20, 128LL << 20, 256LL << 20, 0};
        long long best_bytes = B->group_bytes;
        double best = 1e30;
        for (long long c : cands)
        {
            B->group_bytes = c;
            make_groups(*B);
            batch_enqueue(*B, s); // warm
            SDL_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r) batch_enqueue(*B, s);
            SDL_CUDA(cudaEventRecord(e1, s));
            SDL_CUDA(cudaEventSynchronize(e1));
            float t = 0;
            SDL_CUDA(cudaEventElapsedTime(&t, e0, e1));
            if (t / reps < best)
            {
                best = t / reps;
                best_bytes = c;
            }
        }
        SDL_CUDA(cudaEventDestroy(e0));
        SDL_CUDA(cudaEventDestroy(e1));
        B->group_bytes = best_bytes;
        make_groups(*B);
        if (group_bytes) *group_bytes = best_bytes;
        if (ms) *ms = best;
    });
}

extern "C" sdl_status sdl_batch_refill(sdl_batch *B, void *stream)
{
    return guard_status("sdl_batch_refill", [&]() {
        if (!B) fail(SDL_ERR_INVALID, "NULL batch");
        check_bound(*B);
        cudaStream_t s = pick_stream(stream);
        if (s == cudaStreamLegacy)
            fail(SDL_ERR_INVALID, "batched refills need a non-default stream (graph capture)");
        auto enqueue = [&]() { batch_enqueue(*B, s); };
        if (!B->exec)
        {
            // first refill runs eagerly (every lazily set kernel attribute is set
            // outside any capture), then the same launches are captured once
            const unsigned long long l0 = g_launches.load();
            enqueue();
            B->launches_per_refill = g_launches.load() - l0;
            SDL_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try
            {
                enqueue();
            }
            catch (...)
            {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            SDL_CUDA(cudaStreamEndCapture(s, &B->graph));
            // captured launches are not executions: only replays count
            g_launches.fetch_sub(B->launches_per_refill, std::memory_order_relaxed);
            SDL_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
            return;
        }
        SDL_CUDA(cudaGraphLaunch(B->exec, s));
        g_launches.fetch_add(B->launches_per_refill, std::memory_order_relaxed);
    });
}

extern "C" sdl_status sdl_batch_refill_unbatched(sdl_batch *B, void *stream)
{
    return guard_status("sdl_batch_refill_unbatched", [&]() {
        if (!B) fail(SDL_ERR_INVALID, "NULL batch");
        cudaStream_t s = pick_stream(stream);
        for (size_t i = 0; i < B->prods.size(); ++i)
        {
            const ProdPtrs &pp = B->host_ptrs[i];
            if (B->prods[i]->nnz > 0 && !pp.Cx)
                fail(SDL_ERR_INVALID, "product " + std::to_string(i) + " has no bound values");
            product_numeric(*B->prods[i], pp.Lx, pp.d, pp.Ax, pp.Cx, s);
        }
    });
}

extern "C" sdl_status sdl_batch_info(const sdl_batch *B, int *tiles, int *big_rows, long long *terms)
{
    return guard_status("sdl_batch_info", [&]() {
        if (!B) fail(SDL_ERR_INVALID, "NULL batch");
        if (tiles) *tiles = B->ntiles;
        if (big_rows) *big_rows = B->big_rows;
        if (terms) *terms = B->terms;
    });
}

extern "C" void sdl_batch_destroy(sdl_batch *B) { delete B; }
