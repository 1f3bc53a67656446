/*
 * Single-GPU stand-in for the NVSHMEM calls the reference's kernel header
 * (include/dist_spmm_ppl_batch.cuh) makes, so that header compiles unmodified
 * for sm_100a as a GPU checker.  TEST INFRASTRUCTURE (oracle/ only).
 *
 * Emulation: the P virtual PEs' symmetric buffers of one kind are laid out back
 * to back in one device allocation, `cola_shim_pe_stride` elements apart, so the
 * copy of PE `pe` of a symmetric address `a` held by PE `me` is
 * a + (pe - me) * stride.  `cola_shim_me` (device) / `cola_shim_host_me` (host)
 * name the PE whose launch is being issued; the launcher sets both before every
 * launch on the launch stream.
 */
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

/* Defined here: exactly one translation unit (ref_kernels.cu) includes this. */
__device__ int cola_shim_me = 0;
__device__ long long cola_shim_pe_stride = 0;
inline int cola_shim_host_me = 0;
inline long long cola_shim_host_pe_stride = 0;

/* nvshmemx_float_get_warp: one warp copies n floats of PE pe's copy of src. */
__device__ __forceinline__ void cola_shim_float_get_warp(float *dest, const float *src, size_t n, int pe)
{
    const float *s = src + (long long)(pe - cola_shim_me) * cola_shim_pe_stride;
    for (size_t i = threadIdx.x % 32; i < n; i += 32)
        dest[i] = s[i];
    __syncwarp();
}
#define nvshmemx_float_get_warp(d, s, n, pe) cola_shim_float_get_warp((d), (s), (n), (pe))

/* nvshmemx_float_put_nbi_on_stream: ordered on `stream` (one GPU, one stream). */
inline void nvshmemx_float_put_nbi_on_stream(float *dest, const float *src, size_t n, int pe, cudaStream_t stream)
{
    if (n == 0)
        return;
    float *d = dest + (long long)(pe - cola_shim_host_me) * cola_shim_host_pe_stride;
    cudaMemcpyAsync(d, src, n * sizeof(float), cudaMemcpyDeviceToDevice, stream);
}

/* Stream order already serialises the emulated PEs. */
inline void nvshmemx_barrier_all_on_stream(cudaStream_t) {}
