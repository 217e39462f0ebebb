// Persisted tuning table (sdl_tune_table_*): the autotuner's choices keyed by
// pattern statistics, so that a later process -- or another product of a similar
// pattern in this one -- takes a tuned plan without timing candidates again. It
// generalises upstream's one fixed plan-vs-accumulator threshold
// (GUSTAVSON_PLAN_MAX_RATIO, src/internal/gustavson.h:52, applied at
// src/sparse/sparse_matrix.c:270-277) into per-pattern measured choices.
//
// File format (text, one entry per line, '#' starts a comment line):
//   <key> <warp_max_terms> <rows_per_cta_warp> <cta_threads_2k> <cta_threads_8k>
//         <gmem_threads> <tile_budget> <refill_ctas_per_sm> <tile_max_terms>
//         <refill_threads> <refill_kind> <refill_us>
// refill_kind: 0 direct, 1 pipelined, 2 staged direct. Lines without it (the
// first version of the format) load as direct.
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "capi_common.h"

namespace sdl {
namespace {
struct TuneEntry
{
    TuneConfig cfg;
    double refill_us = 0;
};
std::mutex g_mu;
std::map<std::string, TuneEntry> g_table;

bool valid(const TuneConfig &c)
{
    auto pos = [](int v) { return v > 0 && v <= 4096; };
    return (c.warp_max_terms == 128 || c.warp_max_terms == 512) && pos(c.rows_per_cta_warp) &&
           pos(c.cta_threads_2k) && pos(c.cta_threads_8k) && pos(c.gmem_threads) && c.tile_budget >= 0 &&
           c.tile_budget <= TILE_T && c.tile_max_terms >= 0 && c.tile_max_terms <= TILE_T &&
           c.refill_ctas_per_sm >= 0 && c.refill_ctas_per_sm <= 64 &&
           (c.refill_threads == 256 || c.refill_threads == 128) && (c.refill_pipe == 0 || c.refill_es == 0);
}

int refill_kind(const TuneConfig &c) { return c.refill_pipe ? 1 : c.refill_es ? 2 : 0; }
} // namespace

void tune_table_record(const std::string &key, const TuneConfig &c, double refill_us)
{
    std::lock_guard<std::mutex> g(g_mu);
    g_table[key] = TuneEntry{c, refill_us};
}

bool tune_table_lookup(const std::string &key, TuneConfig &c)
{
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_table.find(key);
    if (it == g_table.end()) return false;
    c = it->second.cfg;
    return true;
}
} // namespace sdl

using namespace sdl;

extern "C" sdl_status sdl_tune_table_save(const char *path)
{
    return guard_status("sdl_tune_table_save", [&]() {
        if (!path) fail(SDL_ERR_INVALID, "NULL path");
        std::lock_guard<std::mutex> g(g_mu);
        std::ofstream f(path, std::ios::trunc);
        if (!f) fail(SDL_ERR_INVALID, std::string("cannot write ") + path);
        f << "# sparsediff_linalg_b200 tuning table v2: key warp_max_terms rows_per_cta_warp cta_threads_2k "
             "cta_threads_8k gmem_threads tile_budget refill_ctas_per_sm tile_max_terms refill_threads "
             "refill_kind refill_us\n";
        char num[32];
        for (const auto &kv : g_table)
        {
            const TuneConfig &c = kv.second.cfg;
            std::snprintf(num, sizeof num, "%.3f", kv.second.refill_us);
            f << kv.first << ' ' << c.warp_max_terms << ' ' << c.rows_per_cta_warp << ' ' << c.cta_threads_2k << ' '
              << c.cta_threads_8k << ' ' << c.gmem_threads << ' ' << c.tile_budget << ' ' << c.refill_ctas_per_sm
              << ' ' << c.tile_max_terms << ' ' << c.refill_threads << ' ' << refill_kind(c) << ' ' << num << '\n';
        }
        if (!f) fail(SDL_ERR_INVALID, std::string("write failed: ") + path);
    });
}

extern "C" sdl_status sdl_tune_table_load(const char *path, int *entries)
{
    return guard_status("sdl_tune_table_load", [&]() {
        if (!path) fail(SDL_ERR_INVALID, "NULL path");
        std::ifstream f(path);
        if (!f) fail(SDL_ERR_INVALID, std::string("cannot read ") + path);
        std::map<std::string, TuneEntry> loaded;
        std::string line;
        int lineno = 0;
        while (std::getline(f, line))
        {
            ++lineno;
            if (line.empty() || line[0] == '#') continue;
            std::istringstream in(line);
            std::vector<std::string> tok;
            for (std::string t; in >> t;) tok.push_back(t);
            TuneEntry e;
            TuneConfig &c = e.cfg;
            bool ok = tok.size() == 11 || tok.size() == 12;
            if (ok)
            {
                int *fields[] = {&c.warp_max_terms, &c.rows_per_cta_warp, &c.cta_threads_2k, &c.cta_threads_8k,
                                 &c.gmem_threads, &c.tile_budget, &c.refill_ctas_per_sm, &c.tile_max_terms,
                                 &c.refill_threads};
                int kind = 0;
                size_t used = 0;
                try
                {
                    for (int q = 0; q < 9 && ok; ++q)
                    {
                        *fields[q] = std::stoi(tok[1 + q], &used);
                        ok = used == tok[1 + q].size();
                    }
                    if (ok && tok.size() == 12)
                    {
                        kind = std::stoi(tok[10], &used);
                        ok = used == tok[10].size() && kind >= 0 && kind <= 2;
                    }
                    if (ok)
                    {
                        const std::string &u = tok.back();
                        e.refill_us = std::stod(u, &used);
                        ok = used == u.size();
                    }
                }
                catch (const std::exception &)
                {
                    ok = false;
                }
                c.refill_pipe = kind == 1;
                c.refill_es = kind == 2;
            }
            if (!ok || !valid(c))
                fail(SDL_ERR_INVALID, std::string(path) + ": malformed tuning entry on line " + std::to_string(lineno));
            loaded[tok[0]] = e;
        }
        std::lock_guard<std::mutex> g(g_mu);
        for (auto &kv : loaded) g_table[kv.first] = kv.second;
        if (entries) *entries = (int)loaded.size();
    });
}

extern "C" sdl_status sdl_tune_table_clear(void)
{
    return guard_status("sdl_tune_table_clear", [&]() {
        std::lock_guard<std::mutex> g(g_mu);
        g_table.clear();
    });
}

extern "C" sdl_status sdl_tune_table_size(int *entries)
{
    return guard_status("sdl_tune_table_size", [&]() {
        if (!entries) fail(SDL_ERR_INVALID, "NULL argument");
        std::lock_guard<std::mutex> g(g_mu);
        *entries = (int)g_table.size();
    });
}
