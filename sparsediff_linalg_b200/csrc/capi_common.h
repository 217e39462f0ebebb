// Shared plumbing of the C ABI: status bookkeeping, the fatal-error policy of the
// upstream-compatible entry points, and host <-> device copy helpers.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "sdl_internal.h"

namespace sdl {

void set_status(sdl_status code, const std::string &msg);
bool fatal_errors();

// Runs f(); on failure records the status and either exits (upstream entry points
// with fatal errors on) or returns `on_error`.
template <class R, class F>
R guard_upstream(const char *fn, R on_error, F &&f)
{
    try
    {
        return f();
    }
    catch (const Error &e)
    {
        set_status(e.code, std::string(fn) + ": " + e.what());
        if (fatal_errors())
        {
            std::fprintf(stderr, "Error in %s: %s\n", fn, e.what());
            std::exit(1);
        }
    }
    catch (const std::bad_alloc &)
    {
        set_status(SDL_ERR_OOM, std::string(fn) + ": host allocation failed");
        if (fatal_errors())
        {
            std::fprintf(stderr, "Error in %s: host allocation failed\n", fn);
            std::exit(1);
        }
    }
    catch (const std::exception &e)
    {
        set_status(SDL_ERR_INTERNAL, std::string(fn) + ": " + e.what());
        if (fatal_errors())
        {
            std::fprintf(stderr, "Error in %s: %s\n", fn, e.what());
            std::exit(1);
        }
    }
    return on_error;
}

template <class F>
void guard_upstream_void(const char *fn, F &&f)
{
    guard_upstream<int>(fn, 0, [&]() {
        f();
        return 0;
    });
}

// Status-returning form for the extension API.
template <class F>
sdl_status guard_status(const char *fn, F &&f)
{
    try
    {
        f();
        return SDL_OK;
    }
    catch (const Error &e)
    {
        set_status(e.code, std::string(fn) + ": " + e.what());
        return e.code;
    }
    catch (const std::bad_alloc &)
    {
        set_status(SDL_ERR_OOM, std::string(fn) + ": host allocation failed");
        return SDL_ERR_OOM;
    }
    catch (const std::exception &e)
    {
        set_status(SDL_ERR_INTERNAL, std::string(fn) + ": " + e.what());
        return SDL_ERR_INTERNAL;
    }
}

// Host arrays allocated by this library's constructors (new_CSR_matrix, ...) are
// page-locked in place (cudaHostRegister) the first time a large transfer touches
// them, so copies run at full link speed; they are unregistered before the library
// frees or reallocates them. Arrays the caller allocated are never registered.
void host_track(void *p, size_t bytes);
void host_untrack(void *p);
void host_pin_if_owned(const void *p, size_t bytes);

template <class T>
void h2d(T *dst, const T *src, size_t count, cudaStream_t s)
{
    if (!count) return;
    host_pin_if_owned(src, count * sizeof(T));
    SDL_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
}
template <class T>
void d2h(T *dst, const T *src, size_t count, cudaStream_t s)
{
    if (!count) return;
    host_pin_if_owned(dst, count * sizeof(T));
    SDL_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s));
}
template <class T>
DevBuf<T> upload(const T *src, size_t count, cudaStream_t s)
{
    DevBuf<T> b(count ? count : 1);
    h2d(b.get(), src, count, s);
    return b;
}

// Throws if a device-side consistency check fired since the last call.
void check_device_errors(cudaStream_t s, const char *what);

} // namespace sdl
