// Batched refill engine (sdl_batch_*): many products refilled by two launches over
// the union of their compiled schedules (the entry values of every product, then
// every product's tiles), replayed from a CUDA graph. The plain alternative -- one
// sdl_product_fill per product -- pays two launches (and their ramp-up and tail)
// per product; here all products share one grid and one graph launch. Each
// product's schedule and entry-value scratch stay where the product keeps them;
// the kernels find them through per-product pointer tables.
#include <memory>
#include <vector>

#include "capi_common.h"

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
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    ~sdl_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

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
        for (int i = 0; i < count; ++i)
        {
            const Product *P = B->prods[i];
            hs[i] = sched_of(*P);
            if (P->num_count[NUM_TILE] && P->ntiles)
            {
                rebase_tiles(P->tiles.get(), P->ntiles, i, B->tiles.get() + t_off, s);
                t_off += P->ntiles;
            }
            if ((P->num_count[NUM_TILE] && P->ntiles) || P->big_lists) append_entry_chunks(hs[i].nV, i, 2048, chunks);
        }
        if (count)
            SDL_CUDA(cudaMemcpyAsync(B->scheds.get(), hs.data(), count * sizeof(ProdSched),
                                     cudaMemcpyHostToDevice, s));
        B->nchunks = (int)chunks.size();
        B->chunks.reset(std::max<size_t>(1, chunks.size()));
        if (!chunks.empty())
            SDL_CUDA(cudaMemcpyAsync(B->chunks.get(), chunks.data(), chunks.size() * sizeof(EntChunk),
                                     cudaMemcpyHostToDevice, s));
        SDL_CUDA(cudaStreamSynchronize(s));
        *out = B.release();
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

extern "C" sdl_status sdl_batch_refill(sdl_batch *B, void *stream)
{
    return guard_status("sdl_batch_refill", [&]() {
        if (!B) fail(SDL_ERR_INVALID, "NULL batch");
        for (size_t i = 0; i < B->prods.size(); ++i)
            if (B->prods[i]->nnz > 0 && !B->host_ptrs[i].Cx)
                fail(SDL_ERR_INVALID, "product " + std::to_string(i) + " has no bound values");
        cudaStream_t s = pick_stream(stream);
        if (s == cudaStreamLegacy)
            fail(SDL_ERR_INVALID, "batched refills need a non-default stream (graph capture)");
        auto enqueue = [&]() {
            entry_values_batched(B->chunks.get(), B->nchunks, B->ptrs.get(), B->scheds.get(), s);
            tile_refill(B->tiles.get(), B->ntiles, B->ptrs.get(), B->scheds.get(), s);
            for (int i : B->with_big)
            {
                const ProdPtrs &pp = B->host_ptrs[i];
                if (B->prods[i]->big_lists)
                    big_lists_refill(*B->prods[i], B->ptrs.get() + i, s);
                else
                    big_rows_refill(*B->prods[i], pp.Lx, pp.d, pp.Ax, pp.Cx, s, B->ptrs.get() + i);
            }
        };
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
