// Stand-ins for the legacy texture-reference API that CUDA 12 removed
// (texture<T, dim>, tex2D/tex3D on references, cudaBindTexture*), so that the
// reference's .cu files compile here for their HOST code (the path-table
// builders).  Nothing in the oracle launches the reference's kernels: these
// device functions return 0 and the bind calls do nothing.
#pragma once
#include <cuda_runtime.h>

template <typename T, int Dim = 1, int Mode = 0>
struct texture {
    int normalized = 0;
    cudaTextureFilterMode filterMode = cudaFilterModePoint;
    cudaTextureAddressMode addressMode[3] = {cudaAddressModeClamp, cudaAddressModeClamp, cudaAddressModeClamp};
};
template <typename T, int D, int M>
__device__ inline T tex1Dfetch(const texture<T, D, M>&, int) { return T(); }
template <typename T, int D, int M>
__device__ inline T tex2D(const texture<T, D, M>&, float, float) { return T(); }
template <typename T, int D, int M>
__device__ inline T tex3D(const texture<T, D, M>&, float, float, float) { return T(); }
template <typename T, int D, int M>
inline cudaError_t cudaBindTexture(size_t*, const texture<T, D, M>&, const void*, const cudaChannelFormatDesc&,
                                   size_t = ~(size_t)0) {
    return cudaSuccess;
}
template <typename T, int D, int M>
inline cudaError_t cudaBindTexture2D(size_t*, const texture<T, D, M>&, const void*, const cudaChannelFormatDesc&,
                                     size_t, size_t, size_t) {
    return cudaSuccess;
}
template <typename T, int D, int M>
inline cudaError_t cudaUnbindTexture(const texture<T, D, M>&) { return cudaSuccess; }
