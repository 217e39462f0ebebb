// Library runtime: device selection, the library stream, error words, counted
// device allocations, and the scan / iota / validation primitives every phase
// uses.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <unordered_map>
#include <mutex>
#include <string>

#include "sdl_internal.h"
#include "sdl_device.cuh"

namespace sdl {

std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned long long> g_dev_allocs{0};

void fail(sdl_status code, const std::string &msg) { throw Error(code, msg); }

void cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    std::string m = std::string("CUDA error '") + cudaGetErrorString(e) + "' in " + what +
                    " (" + file + ":" + std::to_string(line) + ")";
    sdl_status code = (e == cudaErrorMemoryAllocation) ? SDL_ERR_OOM : SDL_ERR_CUDA;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = SDL_ERR_NO_DEVICE;
    throw Error(code, m);
}

static std::mutex g_rt_mu;
static Runtime g_rt;
static bool g_rt_ready = false;

Runtime &runtime()
{
    std::lock_guard<std::mutex> lk(g_rt_mu);
    if (g_rt_ready) return g_rt;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        throw Error(SDL_ERR_NO_DEVICE, "no CUDA device available to the sparsediff_linalg "
                                       "B200 library");
    }
    SDL_CUDA(cudaGetDevice(&g_rt.device));
    cudaDeviceProp prop{};
    SDL_CUDA(cudaGetDeviceProperties(&prop, g_rt.device));
    g_rt.num_sms = prop.multiProcessorCount;
    g_rt.smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
    g_rt.l2_bytes = prop.l2CacheSize;
    SDL_CUDA(cudaStreamCreateWithFlags(&g_rt.stream, cudaStreamNonBlocking));
    SDL_CUDA(cudaMalloc(&g_rt.d_error, sizeof(int)));
    SDL_CUDA(cudaMemset(g_rt.d_error, 0, sizeof(int)));
    g_rt_ready = true;
    return g_rt;
}

int take_device_error(cudaStream_t s)
{
    Runtime &rt = runtime();
    int h = 0;
    SDL_CUDA(cudaMemcpyAsync(&h, rt.d_error, sizeof(int), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    if (h) SDL_CUDA(cudaMemsetAsync(rt.d_error, 0, sizeof(int), s));
    return h;
}

// Device memory: a cache of freed blocks per device in front of cudaMalloc, so that
// plans built again and again (new patterns, re-plans) reuse their scratch instead of
// paying cudaMalloc / cudaFree for several GB each time. A block is cached only after
// a device synchronisation -- what cudaFree implies -- so no kernel still in flight
// uses it when it is handed out again. Sizes above 1 MiB are rounded up to 2 MiB; a
// request takes the smallest cached block of its device between its size and twice
// it. The cache holds at most a quarter of the device's memory; an allocation that
// fails empties it and tries once more; sdl_release_cached_memory empties it.
namespace {
struct DevCache
{
    std::mutex mu;
    std::unordered_map<void *, std::pair<size_t, int>> live; // block -> (bytes, device)
    std::multimap<std::pair<int, size_t>, void *> idle;        // (device, bytes) -> block
    std::unordered_map<int, size_t> idle_bytes, cap;           // per device
};
DevCache &dev_cache()
{
    static DevCache c;
    return c;
}

size_t round_block(size_t bytes)
{
    const size_t q = bytes > (1u << 20) ? (2u << 20) : 512u;
    return (bytes + q - 1) / q * q;
}

// Frees every idle block of `dev` (the caller holds the lock).
void release_idle(DevCache &c, int dev)
{
    for (auto it = c.idle.lower_bound({dev, 0}); it != c.idle.end() && it->first.first == dev;)
    {
        cudaFree(it->second);
        it = c.idle.erase(it);
    }
    c.idle_bytes[dev] = 0;
}
} // namespace

void *dev_alloc(size_t bytes)
{
    runtime();
    const size_t want = round_block(bytes);
    int dev = 0;
    SDL_CUDA(cudaGetDevice(&dev));
    DevCache &c = dev_cache();
    std::lock_guard<std::mutex> g(c.mu);
    g_dev_allocs.fetch_add(1, std::memory_order_relaxed);
    auto it = c.idle.lower_bound({dev, want});
    if (it != c.idle.end() && it->first.first == dev && it->first.second <= 2 * want)
    {
        void *p = it->second;
        const size_t have = it->first.second;
        c.idle.erase(it);
        c.idle_bytes[dev] -= have;
        c.live[p] = {have, dev};
        return p;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        release_idle(c, dev);
        e = cudaMalloc(&p, want);
    }
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        throw Error(SDL_ERR_OOM, "device allocation of " + std::to_string(bytes) +
                                     " bytes failed: " + cudaGetErrorString(e));
    }
    c.live[p] = {want, dev};
    if (!c.cap.count(dev))
    {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        c.cap[dev] = tot / 4;
    }
    return p;
}

void dev_free(void *p)
{
    if (!p) return;
    DevCache &c = dev_cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end())
    {
        cudaFree(p);
        return;
    }
    const size_t bytes = it->second.first;
    const int dev = it->second.second;
    c.live.erase(it);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev || c.idle_bytes[dev] + bytes > c.cap[dev] || cudaDeviceSynchronize() != cudaSuccess)
    {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    c.idle.insert({{dev, bytes}, p});
    c.idle_bytes[dev] += bytes;
}

void release_cached_device_memory()
{
    DevCache &c = dev_cache();
    std::lock_guard<std::mutex> g(c.mu);
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
    {
        cudaDeviceSynchronize();
        release_idle(c, dev);
    }
}

// ------------------------------------------------------------------ scan
// Three-phase scan: per-tile sums, a single-CTA scan of the tile sums, then
// per-tile scans seeded with the tile prefix. Sums are carried in 64 bits.
namespace {
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class Tin>
__global__ void k_scan_tile_sums(const Tin *in, long long n, long long *tile_sums)
{
    long long base = (long long)blockIdx.x * SCAN_TILE;
    long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k)
    {
        long long idx = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += (long long)in[idx];
    }
    s = block_reduce_sum_ll<SCAN_THREADS>(s);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = s;
}

__global__ void k_scan_tile_prefix(long long *tile_sums, long long ntiles, long long *total)
{
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < ntiles; base += SCAN_THREADS)
    {
        long long idx = base + threadIdx.x;
        long long v = idx < ntiles ? tile_sums[idx] : 0;
        long long incl = block_incl_scan_ll<SCAN_THREADS>(v);
        long long c = carry;
        if (idx < ntiles) tile_sums[idx] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == SCAN_THREADS - 1) carry = c + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

template <class Tin, class Tout>
__global__ void k_scan_tiles(const Tin *in, long long n, const long long *tile_prefix,
                             Tout *out)
{
    // each thread owns SCAN_ITEMS consecutive items of the tile
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    long long v[SCAN_ITEMS];
    long long local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
    {
        long long idx = base + k;
        v[k] = idx < n ? (long long)in[idx] : 0;
        local += v[k];
    }
    long long incl = block_incl_scan_ll<SCAN_THREADS>(local);
    long long run = tile_prefix[blockIdx.x] + incl - local;
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
    {
        long long idx = base + k;
        run += v[k];
        if (idx < n) out[idx + 1] = (Tout)run;
    }
}

template <class Tin, class Tout>
long long scan_impl(const Tin *in, Tout *out, long long n, cudaStream_t s)
{
    if (n <= 0)
    {
        SDL_CUDA(cudaMemsetAsync(out, 0, sizeof(Tout), s));
        return 0;
    }
    long long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DevBuf<long long> tiles(ntiles + 1);
    SDL_LAUNCH(k_scan_tile_sums<Tin>, (unsigned)ntiles, SCAN_THREADS, 0, s, in, n, tiles.get());
    SDL_LAUNCH(k_scan_tile_prefix, 1, SCAN_THREADS, 0, s, tiles.get(), ntiles,
               tiles.get() + ntiles);
    SDL_LAUNCH((k_scan_tiles<Tin, Tout>), (unsigned)ntiles, SCAN_THREADS, 0, s, in, n,
               tiles.get(), out);
    long long total = 0;
    SDL_CUDA(cudaMemcpyAsync(&total, tiles.get() + ntiles, sizeof(long long),
                             cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    return total;
}
} // namespace

long long exclusive_scan_i64(const long long *d_in, long long *d_out, long long n,
                             cudaStream_t s)
{
    return scan_impl<long long, long long>(d_in, d_out, n, s);
}

int exclusive_scan_i32_checked(const int *d_in, int *d_out, int n, cudaStream_t s)
{
    long long total = scan_impl<int, int>(d_in, d_out, n, s);
    if (total > 2147483647LL)
        fail(SDL_ERR_OVERFLOW, "result has more than INT_MAX entries (" +
                                   std::to_string(total) + ")");
    return static_cast<int>(total);
}

// ------------------------------------------------------------------ iota
namespace {
__global__ void k_iota(int *d, int n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        d[k] = (int)k;
}
} // namespace

void fill_iota(int *d, int n, cudaStream_t s)
{
    if (n <= 0) return;
    int grid = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    SDL_LAUNCH(k_iota, grid, 256, 0, s, d, n);
}

// ------------------------------------------------------------------ validation
namespace {
// bit 1: p[0] != 0 or p[rows] != nnz; bit 2: p decreasing; bit 4: index out of range
__global__ void k_validate(const int *p, const int *idx, int rows, int cols, int nnz,
                           int *flags)
{
    long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    int f = 0;
    if (tid == 0 && p)
    {
        if (p[0] != 0 || p[rows] != nnz) f |= 1;
    }
    if (p)
        for (long long r = tid; r < rows; r += stride)
            if (p[r + 1] < p[r]) f |= 2;
    for (long long k = tid; k < nnz; k += stride)
    {
        int c = idx[k];
        if (c < 0 || c >= cols) f |= 4;
    }
    if (f) atomicOr(flags, f);
}
} // namespace

void validate_compressed(const int *d_p, const int *d_idx, int rows, int cols, int nnz,
                         const char *what, cudaStream_t s)
{
    if (rows < 0 || cols < 0 || nnz < 0) fail(SDL_ERR_INVALID, std::string(what) + ": negative size");
    if (nnz > 0 && !d_idx) fail(SDL_ERR_INVALID, std::string(what) + ": null index array");
    Runtime &rt = runtime();
    long long work = std::max<long long>(rows, nnz);
    int grid = (int)std::max<long long>(1, std::min<long long>((work + 255) / 256, 148LL * 8));
    DevBuf<int> flags(1);
    SDL_CUDA(cudaMemsetAsync(flags.get(), 0, sizeof(int), s));
    SDL_LAUNCH(k_validate, grid, 256, 0, s, d_p, d_idx, rows, cols, nnz, flags.get());
    int h = 0;
    SDL_CUDA(cudaMemcpyAsync(&h, flags.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SDL_CUDA(cudaStreamSynchronize(s));
    (void)rt;
    if (h & 1) fail(SDL_ERR_INVALID, std::string(what) + ": offsets must start at 0 and end at nnz");
    if (h & 2) fail(SDL_ERR_INVALID, std::string(what) + ": offsets must be non-decreasing");
    if (h & 4) fail(SDL_ERR_INVALID, std::string(what) + ": index out of range");
}

// ------------------------------------------------------------------ widen
namespace {
__global__ void k_widen(const int *__restrict__ src, long long *__restrict__ dst, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        dst[k] = src[k];
}
} // namespace

void widen_i32(const int *d_src, long long *d_dst, long long n, cudaStream_t s)
{
    if (n <= 0) return;
    const int grid = (int)std::min<long long>((n + 255) / 256, (long long)runtime().num_sms * 8);
    SDL_LAUNCH(k_widen, grid, 256, 0, s, d_src, d_dst, n);
}

// ------------------------------------------------------------------ gather
namespace {
// out[k] = x[src[k]], four consecutive positions per thread: one 16-byte load of
// their sources, four independent gathers, two 16-byte stores. The positions and
// the output are streamed (evict-first), so the gathered array keeps its place in
// L2 while the permutation revisits it. The last n % 4 positions go to the first
// threads of the grid.
__global__ void k_gather(const int4 *__restrict__ src4, const double *__restrict__ x, double2 *__restrict__ out2,
                         long long n4, const int *__restrict__ src_tail, double *__restrict__ out_tail, int ntail)
{
    const long long first = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long k = first; k < n4; k += step)
    {
        const int4 q = __ldcs(src4 + k);
        const double a = x[q.x], b = x[q.y], c = x[q.z], d = x[q.w];
        __stcs(out2 + 2 * k, make_double2(a, b));
        __stcs(out2 + 2 * k + 1, make_double2(c, d));
    }
    if (first < ntail) out_tail[first] = x[src_tail[first]];
}

// The same for buffers that are not 16-byte aligned.
__global__ void k_gather_unaligned(const int *__restrict__ src, const double *__restrict__ x,
                                   double *__restrict__ out, int n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        out[k] = x[src[k]];
}
} // namespace

void gather_values(const int *d_src, const double *d_x, double *d_out, int n, cudaStream_t s)
{
    if (n <= 0) return;
    Runtime &rt = runtime();
    if (((uintptr_t)d_src | (uintptr_t)d_out) & 15)
    {
        int grid = (int)std::min<long long>((n + 255) / 256, (long long)rt.num_sms * 8);
        SDL_LAUNCH(k_gather_unaligned, grid, 256, 0, s, d_src, d_x, d_out, n);
        return;
    }
    const long long n4 = n / 4;
    const int ntail = n - (int)(4 * n4);
    int grid = (int)std::max<long long>(1, std::min<long long>((n4 + 255) / 256, (long long)rt.num_sms * 8));
    SDL_LAUNCH(k_gather, grid, 256, 0, s, reinterpret_cast<const int4 *>(d_src), d_x,
               reinterpret_cast<double2 *>(d_out), n4, d_src + 4 * n4, d_out + 4 * n4, ntail);
}

} // namespace sdl
