// A host program written the way the reference's src/distSpMM_ppl_batch.cu
// main is (read the partition .bin files, nnz_split both blocks, upload the
// zip holders, run_distSpMM_ppl_batch with validation and profiling), built
// against include/cola/compat.h for one GPU with P virtual PEs.
//   usage: compat_gpu_main <graph dir> <N> <P> <dim>
// Prints "PE <p> ms <t>" per PE, or "E <status>" when the library throws.
#include <algorithm>
#include <cmath>
#include <memory>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "cola/compat.h"

int main(int argc, char **argv)
{
    if (argc != 5)
        return 2;
    const std::string dir = argv[1];
    const int N = std::atoi(argv[2]), P = std::atoi(argv[3]), dim = std::atoi(argv[4]);
    const int npp = (N + P - 1) / P;
    try {
        std::vector<int> g_rowPtr = bin2vec<int>(dir + "/global_rowPtr.bin");
        std::vector<int> g_colIdx = bin2vec<int>(dir + "/global_colIdx.bin");
        std::vector<float> h_in((size_t)P * npp * dim, 0.f);
        for (size_t i = 0; i < (size_t)N * dim; i++)
            h_in[i] = (float)((i * 7919u) % 23u) * 0.125f - 1.0f;
        float *d_in = nullptr, *d_out = nullptr;
        cola_compat::check_cuda(cudaMalloc((void **)&d_in, h_in.size() * sizeof(float)), "main");
        cola_compat::check_cuda(cudaMalloc((void **)&d_out, h_in.size() * sizeof(float)), "main");
        cola_compat::check_cuda(cudaMemcpy(d_in, h_in.data(), h_in.size() * sizeof(float), cudaMemcpyHostToDevice),
                                "main");
        cola_compat::check_cuda(cudaMemset(d_out, 0, h_in.size() * sizeof(float)), "main");
        cudaStream_t stream;
        cola_compat::check_cuda(cudaStreamCreate(&stream), "main");
        const std::string gdir = dir + "/GPU" + std::to_string(P) + "/";
        std::vector<std::unique_ptr<d_csr_zip>> csrs;
        std::vector<std::unique_ptr<d_csc_zip>> cscs;
        std::vector<std::vector<int>> offs;  // per PE: local offsets (2), remote offsets (2)
        for (int p = 0; p < P; p++) {
            const std::string pos = "_" + std::to_string(P) + "_" + std::to_string(p) + ".bin";
            std::vector<int> rowPtr_l = bin2vec<int>(gdir + "csr_rowPtr_l" + pos);
            std::vector<int> colIdx_l = bin2vec<int>(gdir + "csr_colIdx_l" + pos);
            std::vector<int> rowIdx_l = bin2vec<int>(gdir + "csr_rowIdx_l" + pos);
            std::vector<int> colPtr_r = bin2vec<int>(gdir + "csc_colPtr_r" + pos);
            std::vector<int> rowIdx_r = bin2vec<int>(gdir + "csc_rowIdx_r" + pos);
            std::vector<int> colIdx_r = bin2vec<int>(gdir + "csc_colIdx_r" + pos);
            std::vector<int> zrow, zptr, zcol, zcptr;
            nnz_split(rowIdx_l, rowPtr_l, colIdx_l, zrow, zptr, p, true);
            nnz_split(colIdx_r, colPtr_r, rowIdx_r, zcol, zcptr, p, false);
            csrs.emplace_back(new d_csr_zip(zptr, colIdx_l, zrow, std::vector<float>(colIdx_l.size(), 1.0f)));
            cscs.emplace_back(new d_csc_zip(zcptr, rowIdx_r, zcol, std::vector<float>(rowIdx_r.size(), 1.0f)));
            offs.push_back({0, (int)zrow.size(), 0, (int)zcol.size()});
            const int lb = p * npp, ub = std::min(N, (p + 1) * npp);
            const double ms = run_distSpMM_ppl_batch<true, true>(
                P, d_out + (size_t)p * npp * dim, d_in + (size_t)p * npp * dim, nullptr, nullptr, nullptr,
                offs.back().data(), offs.back().data() + 2, nullptr, nullptr, nullptr, csrs.back().get(),
                cscs.back().get(), lb, ub, dim, npp, P, p, g_rowPtr.data(), g_colIdx.data(), h_in.data(), stream);
            printf("PE %d ms %.4f\n", p, ms);
        }
        // every PE in one call (single stage: one row view of all PEs' chunks), against
        // the per-PE results above (those accumulated 1 + 50 + 200 SpMMs: compare per SpMM)
        {
            float *d_all = nullptr;
            cola_compat::check_cuda(cudaMalloc((void **)&d_all, h_in.size() * sizeof(float)), "main");
            cola_compat::check_cuda(cudaMemset(d_all, 0, h_in.size() * sizeof(float)), "main");
            std::vector<int *> lo, ro;
            std::vector<d_csr_zip *> cl;
            std::vector<d_csc_zip *> cr;
            for (int p = 0; p < P; p++) {
                lo.push_back(offs[(size_t)p].data());
                ro.push_back(offs[(size_t)p].data() + 2);
                cl.push_back(csrs[(size_t)p].get());
                cr.push_back(cscs[(size_t)p].get());
            }
            for (int rep = 0; rep < 2; rep++)  // the first call builds the view, the second reuses it
                distSpMM_ppl_batch_all(P, d_all, d_in, nullptr, lo.data(), ro.data(), nullptr, nullptr, nullptr,
                                       cl.data(), cr.data(), dim, npp, P, stream);
            cola_compat::check_cuda(cudaStreamSynchronize(stream), "main");
            std::vector<float> a(h_in.size()), b(h_in.size());
            cudaMemcpy(a.data(), d_all, a.size() * sizeof(float), cudaMemcpyDeviceToHost);
            cudaMemcpy(b.data(), d_out, b.size() * sizeof(float), cudaMemcpyDeviceToHost);
            double num = 0, den = 0;
            for (size_t i = 0; i < a.size(); i++) {
                const double want = (double)b[i] / 251.0 * 2.0;  // 251 SpMMs there, 2 here
                num += (a[i] - want) * (a[i] - want);
                den += want * want;
            }
            printf("ALL rel %.3e\n", den > 0 ? std::sqrt(num / den) : 0.0);
            cudaFree(d_all);
        }
        cudaStreamDestroy(stream);
        cudaFree(d_in);
        cudaFree(d_out);
    } catch (const cola_compat::error &e) {
        printf("E %d %s\n", (int)e.status, e.what());
        return 1;
    }
    return 0;
}
