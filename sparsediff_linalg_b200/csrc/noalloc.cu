// Refill of a product that makes no device allocation, for callers that cannot
// call cudaMalloc while their refill loop runs: a caller whose device memory is
// wholly owned by another allocator (a framework pool that has reserved the free
// memory), a caller held to a fixed device-memory budget that may not grow during
// the loop, or a latency-critical loop that must not pay cudaMalloc's implicit
// device-wide synchronisation.
//
// sdl_product_fill already allocates nothing, but its rows with more than 8192
// outputs use a column -> position map that sdl_product_create allocates for the
// product. This variant gives those rows a file-scope __device__ array instead:
// STATIC_POSMAP_INTS ints (16 MiB), which every GPU that loads the library holds
// until the process exits. Each CTA of the large-row kernel owns one slice of A_n
// ints, so the array serves products whose A has at most STATIC_POSMAP_INTS
// columns; larger ones are rejected with SDL_ERR_INVALID.
#include <mutex>
#include <unordered_map>

#include "capi_common.h"

namespace sdl {
const Product *product_of(const sdl_product *P);
void big_rows_refill_scratch(const Product &P, const double *Lx, const double *dvec, const double *Ax,
                             double *Cx, int *posmap, int slots, cudaStream_t s);
} // namespace sdl

using namespace sdl;

namespace {

constexpr long long STATIC_POSMAP_INTS = 4LL * 1024 * 1024;

// Only rows of the product being refilled are ever looked up in the map, and each
// call writes those rows' entries before reading them, so the array needs no
// clearing between calls. Calls that overlap on the GPU share it and race.
__device__ __align__(256) int g_static_posmap[STATIC_POSMAP_INTS];

std::mutex g_addr_mu;
std::unordered_map<int, int *> g_addr; // device -> device address of g_static_posmap

// The host-side name g_static_posmap is only a stand-in for the array, not a
// device address: the address is looked up once per device, with that device
// current, and handed to the kernel.
int *static_posmap_address()
{
    int dev = 0;
    SDL_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_addr_mu);
    auto it = g_addr.find(dev);
    if (it != g_addr.end()) return it->second;
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_posmap);
    if (e != cudaSuccess || !ptr)
    {
        cudaGetLastError();
        fail(SDL_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                               cudaGetErrorString(e));
    }
    g_addr[dev] = static_cast<int *>(ptr);
    return static_cast<int *>(ptr);
}

} // namespace

extern "C" sdl_status sdl_product_fill_noalloc(const sdl_product *Ph, const double *Lx,
                                               const double *d, const double *Ax, double *Cx,
                                               void *stream)
{
    return guard_status("sdl_product_fill_noalloc", [&]() {
        const Product *P = product_of(Ph);
        if (!P) fail(SDL_ERR_INVALID, "NULL product");
        if (P->nnz > 0 && (!Ax || !Cx)) fail(SDL_ERR_INVALID, "NULL value pointer");
        if ((long long)P->n > STATIC_POSMAP_INTS)
            fail(SDL_ERR_INVALID, "A has " + std::to_string(P->n) +
                                      " columns; the static scratch serves at most " +
                                      std::to_string(STATIC_POSMAP_INTS) + " columns");
        if (P->nnz == 0) return;
        cudaStream_t s = pick_stream(stream);
        int *posmap = static_posmap_address();
        const int slots = (int)std::max<long long>(
            1, std::min<long long>(runtime().num_sms, STATIC_POSMAP_INTS / std::max(1, P->n)));
        if (P->num_count[NUM_TILE])
        {
            ProdSched S = sched_of(*P);
            const ProdPtrs vals{Lx, d, Ax, Cx};
            if (entry_values_are_lx(*P, Lx, d))
                S.V = const_cast<double *>(Lx); // read only
            else
                entry_values(S, vals, s);
            tile_refill(P->tiles.get(), P->ntiles, nullptr, nullptr, s, vals, S, P->cfg.refill_ctas_per_sm,
                        small_tile_refill(*P));
        }
        big_rows_refill_scratch(*P, Lx, d, Ax, Cx, posmap, slots, s);
    });
}
