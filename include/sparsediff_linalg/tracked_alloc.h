/* sparsediff_linalg drop-in (B200/CUDA build): host allocation wrappers.
 *
 * Same inline API as upstream include/sparsediff_linalg/tracked_alloc.h:24-136:
 * with SP_TRACK_MEMORY defined the sp_* wrappers count live and peak host bytes
 * (the basis of the "fills never allocate" checks), otherwise they are plain
 * malloc/calloc/realloc/free. Device memory is counted separately
 * (sdl_device_alloc_count in sparsediff_linalg_cuda.h). */
#ifndef SDL_TRACKED_ALLOC_H
#define SDL_TRACKED_ALLOC_H

#include <stddef.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifdef SP_TRACK_MEMORY
#include <malloc.h>
extern size_t g_allocated_bytes;
extern size_t g_peak_bytes;
void sp_memory_stats(size_t *live_bytes, size_t *peak_bytes);
void sp_memory_reset_peak(void);

static inline void sp_track_add_(void *p)
{
    if (p)
    {
        g_allocated_bytes += malloc_usable_size(p);
        if (g_allocated_bytes > g_peak_bytes) g_peak_bytes = g_allocated_bytes;
    }
}
static inline void *sp_malloc(size_t size)
{
    void *p = malloc(size);
    sp_track_add_(p);
    return p;
}
static inline void *sp_calloc(size_t count, size_t size)
{
    void *p = calloc(count, size);
    sp_track_add_(p);
    return p;
}
static inline void sp_free(void *ptr)
{
    if (ptr)
    {
        g_allocated_bytes -= malloc_usable_size(ptr);
        free(ptr);
    }
}
static inline void *sp_realloc(void *ptr, size_t size)
{
    size_t old = ptr ? malloc_usable_size(ptr) : 0;
    void *p = realloc(ptr, size);
    if (p)
    {
        g_allocated_bytes -= old;
        sp_track_add_(p);
    }
    return p;
}
#else
static inline void *sp_malloc(size_t size) { return malloc(size); }
static inline void *sp_calloc(size_t count, size_t size) { return calloc(count, size); }
static inline void sp_free(void *ptr) { free(ptr); }
static inline void *sp_realloc(void *ptr, size_t size) { return realloc(ptr, size); }
#endif

#ifdef __cplusplus
}
#endif

#endif /* SDL_TRACKED_ALLOC_H */
