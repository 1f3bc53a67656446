// The batched autotuner's cache file, free of CUDA so that it can be tested on
// its own.  Text, one line per tuned batch:
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

}  // namespace cola
