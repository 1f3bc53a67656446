// Exercises the batched autotuner's cache file (cola_b200/csrc/tune_cache.h,
// the functions cola_batch_autotune_cached calls) on the CPU, for
// tests/test_tune_cache.py.
//
//   tune_cache_main find <path> <key>      prints "hit u gp bps ms" or "miss"
//   tune_cache_main append <path> <key> <u> <gp> <bps> <ms>   exit 0 on success
//   tune_cache_main sfind <path> <key>     single-graph lines: "hit kt u mb gb ms" or "miss"
//   tune_cache_main sappend <path> <key> <kt> <u> <mb> <gb> <ms>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "tune_cache.h"

int main(int argc, char **argv)
{
    if (argc >= 4 && !std::strcmp(argv[1], "find")) {
        cola::TuneEntry e;
        if (cola::tune_cache_find(argv[2], argv[3], e))
            std::printf("hit %d %d %d %.6f\n", e.unroll, e.grid_pct, e.blocks_per_sm, e.ms);
        else
            std::printf("miss\n");
        return 0;
    }
    if (argc >= 8 && !std::strcmp(argv[1], "append")) {
        cola::TuneEntry e;
        e.unroll = std::atoi(argv[4]);
        e.grid_pct = std::atoi(argv[5]);
        e.blocks_per_sm = std::atoi(argv[6]);
        e.ms = (float)std::atof(argv[7]);
        return cola::tune_cache_append(argv[2], argv[3], e) ? 0 : 1;
    }
    if (argc >= 4 && !std::strcmp(argv[1], "sfind")) {
        cola::SpmmTuneEntry e;
        if (cola::spmm_tune_cache_find(argv[2], argv[3], e))
            std::printf("hit %d %d %d %d %.6f\n", e.k_tile, e.unroll, e.min_blocks, e.gather_batch_rows, e.ms);
        else
            std::printf("miss\n");
        return 0;
    }
    if (argc >= 9 && !std::strcmp(argv[1], "sappend")) {
        cola::SpmmTuneEntry e;
        e.k_tile = std::atoi(argv[4]);
        e.unroll = std::atoi(argv[5]);
        e.min_blocks = std::atoi(argv[6]);
        e.gather_batch_rows = std::atoi(argv[7]);
        e.ms = (float)std::atof(argv[8]);
        return cola::spmm_tune_cache_append(argv[2], argv[3], e) ? 0 : 1;
    }
    return 2;
}
