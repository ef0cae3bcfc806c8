// ref_compat.h -- forced include (nvcc -include) for the comparator build of
// the reference's GPU step (iwf_mfree_gpu_3d, CUDA 8 era) on CUDA 12 / sm_100a.
//
// CUDA 12 removed texture references (texture<T, 1, mode>, tex1Dfetch on a
// reference, cudaBindTexture, cudaUnbindTexture), which the reference's pair
// kernels read through (src/interactions_gpu.cu:41-57,482-513).  The build
// recipe (build_ref_gpu.sh) turns each texture declaration into a __device__
// ref_texture<T, 1, mode> holding a device pointer; the functions below give
// the same calls their old meaning: binding stores the pointer in the device
// variable, a fetch is a read-only-cache load of element i (what a linear
// texture fetch returned), unbinding does nothing.  Element values are the same
// as the texture path's, so the reference's arithmetic is unchanged.
#pragma once
#include "ref_prelude.h"

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct ref_texture {
    const T *ptr;
};

template <class T, int dim, enum cudaTextureReadMode mode>
__device__ __forceinline__ T tex1Dfetch(const ref_texture<T, dim, mode> &t, int i) {
    return __ldg(t.ptr + i);
}

template <class T, int dim, enum cudaTextureReadMode mode>
inline cudaError_t cudaBindTexture(size_t *, const ref_texture<T, dim, mode> &tex, const void *p, size_t) {
    const T *q = static_cast<const T *>(p);
    return cudaMemcpyToSymbol(tex, &q, sizeof(q));
}

template <class T, int dim, enum cudaTextureReadMode mode>
inline cudaError_t cudaUnbindTexture(const ref_texture<T, dim, mode> &) {
    return cudaSuccess;
}
