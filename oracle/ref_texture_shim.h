// ref_texture_shim.h — force-included when compiling the reference's CUDA
// translation unit (src/gsop.cu) for sm_100a.  CUDA 12 removed texture
// references; the reference's TEA integrator still declares three of them
// (src/Integrators/bdhitea.cu:17-19, bound at :80-82).  This header gives
// those declarations a device-global pointer and makes tex1Dfetch a plain
// global load of the bound array, which is what a 1-D element fetch returns.
// TEST INFRASTRUCTURE ONLY (the reference GPU golden harness).
#pragma once
#include <cuda_runtime.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct sopref_texref {
    const T* ptr;
};

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ __forceinline__ T tex1Dfetch(const sopref_texref<T, Dim, Mode>& t, int i) {
    return t.ptr[i];
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaBindTexture(size_t* offset, const sopref_texref<T, Dim, Mode>& t, const void* p, size_t) {
    const T* q = static_cast<const T*>(p);
    if (offset) *offset = 0;
    return cudaMemcpyToSymbol(t, &q, sizeof(q));
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaUnbindTexture(const sopref_texref<T, Dim, Mode>&) {
    return cudaSuccess;
}

#define texture __device__ sopref_texref
