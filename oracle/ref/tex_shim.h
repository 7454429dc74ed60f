/*
 * tex_shim.h -- lets the reference's test/bfs/test_bfs.cu compile with CUDA 12.
 *
 * TEST INFRASTRUCTURE ONLY (force-included by oracle/Makefile when building
 * oracle/_ref).  CUDA 12 removed texture references and pre-Volta __any; the
 * reference's GPU enactors name both.  These stand-ins only make the
 * translation unit compile: the shimmed GPU enactors are never called, and the
 * oracle uses the reference's host code alone (SimpleReferenceBfs, builders,
 * CsrGraph::FromCoo).
 */
#pragma once
#include <cuda_runtime.h>

template <class T, int Dim = 1, int Mode = 0>
struct texture {
    typedef T value_type;
    cudaChannelFormatDesc channelDesc;
};
#ifndef cudaTextureType1D
#define cudaTextureType1D 1
#endif
/* Never evaluates the reference: yields a zero of the texel type. */
#define tex1Dfetch(ref, idx) ((typename std::remove_reference<decltype(ref)>::type::value_type)(0))
template <class T, int D, int M>
static inline cudaError_t cudaBindTexture(size_t *, texture<T, D, M> &, const void *,
                                          const cudaChannelFormatDesc &, size_t) {
    return cudaSuccess;
}
#define __any(p) __any_sync(0xffffffffu, (p))
#include <type_traits>
