// A reference-style host program built against include/cola/compat.h: it reads
// one partition's .bin files with bin2vec and splits them with nnz_split, as
// src/distSpMM_ppl_batch.cu:79-99 does, and prints the chunk arrays.  No GPU
// call is made, so it runs on a machine without a GPU.
#include <cstdio>
#include <string>
#include <vector>

#include "cola/compat.h"

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    const std::string dir = argv[1];
    const std::string pos = std::string(argv[2]) + "_" + argv[3];
    auto rowPtr = bin2vec<int>(dir + "csr_rowPtr_l_" + pos + ".bin");
    auto colIdx = bin2vec<int>(dir + "csr_colIdx_l_" + pos + ".bin");
    auto rowIdx = bin2vec<int>(dir + "csr_rowIdx_l_" + pos + ".bin");
    std::vector<int> target, ptr;
    nnz_split(rowIdx, rowPtr, colIdx, target, ptr, 0, true);
    printf("T");
    for (int t : target)
        printf(" %d", t);
    printf("\nP");
    for (int p : ptr)
        printf(" %d", p);
    printf("\n");
    try {
        bin2vec<int>(dir + "missing.bin");
    } catch (const cola_compat::error &e) {
        printf("E %d\n", (int)e.status);
    }
    return 0;
}
