/* Declarations the reference's run_distSpMM_ppl_batch template names
 * (include/dist_spmm_ppl_batch.cuh:972-981); one process, no MPI.
 * TEST INFRASTRUCTURE (oracle/ only). */
#pragma once
#include <chrono>
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline double MPI_Wtime()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
