// The autotuners' cache file, free of CUDA so that it can be tested on its
// own.  Text, one line per tuned batch (cola_batch_autotune_cached):
//     <key> <unroll> <grid_pct> <blocks_per_sm> <best_ms>
// The first line whose key matches and whose values are valid wins; lines that
// do not parse or hold invalid values are skipped.
#pragma once
#include <cstdio>
#include <string>

namespace cola {

struct TuneEntry {
    int unroll = 4, grid_pct = 100, blocks_per_sm = 3;
    float ms = 0.f;
};

// The values the batched launch accepts (the autotuner's search space).
inline bool tune_entry_valid(const TuneEntry &e)
{
    return (e.unroll == 2 || e.unroll == 4) && e.grid_pct >= 10 && e.grid_pct <= 100 &&
           (e.blocks_per_sm == 3 || e.blocks_per_sm == 4);
}

// Looks `key` up in the cache file; false when the file is missing or holds no
// valid line for the key.  Keys are at most 599 characters.
inline bool tune_cache_find(const char *path, const std::string &key, TuneEntry &out)
{
    FILE *f = std::fopen(path, "r");
    if (!f)
        return false;
    char line[1024];
    bool found = false;
    while (!found && std::fgets(line, sizeof line, f)) {
        char k[600];
        TuneEntry e;
        if (std::sscanf(line, "%599s %d %d %d %f", k, &e.unroll, &e.grid_pct, &e.blocks_per_sm, &e.ms) == 5 &&
            key == k && tune_entry_valid(e)) {
            out = e;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

// Appends one line for `key`; false when the file cannot be written.
inline bool tune_cache_append(const char *path, const std::string &key, const TuneEntry &e)
{
    FILE *f = std::fopen(path, "a");
    if (!f)
        return false;
    std::fprintf(f, "%s %d %d %d %.6f\n", key.c_str(), e.unroll, e.grid_pct, e.blocks_per_sm, e.ms);
    const bool err = std::ferror(f) != 0;
    return std::fclose(f) == 0 && !err;
}

// The single-graph tuner's lines (cola_spmm_autotune):
//     <key> <k_tile> <unroll> <min_blocks> <gather_batch_rows> <best_ms>
// with keys that start with "spmm|", so they never match a batch's key.
struct SpmmTuneEntry {
    int k_tile = 0, unroll = 0, min_blocks = 0, gather_batch_rows = 0;
    float ms = 0.f;
};

// The values cola_spmm accepts for these options (0 = the library's choice).
inline bool spmm_tune_entry_valid(const SpmmTuneEntry &e)
{
    const int kt = e.k_tile;
    const bool kt_ok = kt == 0 || kt == 64 || kt == 128 || kt == 256 || kt == 512 || kt == 1024;
    const bool u_ok = e.unroll == 0 || e.unroll == 2 || e.unroll == 4 || e.unroll == 6 || e.unroll == 8;
    const bool mb_ok = e.min_blocks == 0 || (e.min_blocks >= 3 && e.min_blocks <= 8);
    const bool gb_ok = e.gather_batch_rows >= 0 && e.gather_batch_rows <= (1 << 24);
    return kt_ok && u_ok && mb_ok && gb_ok;
}

inline bool spmm_tune_cache_find(const char *path, const std::string &key, SpmmTuneEntry &out)
{
    FILE *f = std::fopen(path, "r");
    if (!f)
        return false;
    char line[1024];
    bool found = false;
    while (!found && std::fgets(line, sizeof line, f)) {
        char k[600];
        SpmmTuneEntry e;
        if (std::sscanf(line, "%599s %d %d %d %d %f", k, &e.k_tile, &e.unroll, &e.min_blocks, &e.gather_batch_rows,
                        &e.ms) == 6 &&
            key == k && spmm_tune_entry_valid(e)) {
            out = e;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

inline bool spmm_tune_cache_append(const char *path, const std::string &key, const SpmmTuneEntry &e)
{
    FILE *f = std::fopen(path, "a");
    if (!f)
        return false;
    std::fprintf(f, "%s %d %d %d %d %.6f\n", key.c_str(), e.k_tile, e.unroll, e.min_blocks, e.gather_batch_rows,
                 e.ms);
    const bool err = std::ferror(f) != 0;
    return std::fclose(f) == 0 && !err;
}

}  // namespace cola
