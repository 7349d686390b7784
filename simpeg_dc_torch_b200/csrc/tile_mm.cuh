// Register-tiled shared-memory products used by the factor and solve kernels
// (256 threads per CTA).
#pragma once
#include <cuda_runtime.h>

namespace dct {

// acc[p][q] += sum_{k<K} S1[k*LD1 + a] * S2[k*LD2 + j], a = ag + 16p,
// j = jg + 16q, jg = tid%16, ag = tid/16, for the first NP of the four
// a-groups (NP = ceil(valid a / 16)).  A 64 x 64 output tile, 4 x 4 per thread.
template <typename T, int NP, int LD1, int LD2>
__device__ __forceinline__ void mm64_np(const T* __restrict__ S1,
                                        const T* __restrict__ S2, int K,
                                        T (&acc)[4][4]) {
  const int jg = threadIdx.x & 15, ag = threadIdx.x >> 4;
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    T a[NP], b[4];
#pragma unroll
    for (int p = 0; p < NP; ++p) a[p] = S1[k * LD1 + ag + 16 * p];
#pragma unroll
    for (int q = 0; q < 4; ++q) b[q] = S2[k * LD2 + jg + 16 * q];
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * b[q];
  }
}

template <typename T, int LD1, int LD2>
__device__ __forceinline__ void mm64(const T* __restrict__ S1,
                                     const T* __restrict__ S2, int K, int arows,
                                     T (&acc)[4][4]) {
  switch ((arows + 15) >> 4) {
    case 1: mm64_np<T, 1, LD1, LD2>(S1, S2, K, acc); break;
    case 2: mm64_np<T, 2, LD1, LD2>(S1, S2, K, acc); break;
    case 3: mm64_np<T, 3, LD1, LD2>(S1, S2, K, acc); break;
    default: mm64_np<T, 4, LD1, LD2>(S1, S2, K, acc); break;
  }
}

template <typename T>
__device__ __forceinline__ void zero_acc(T (&acc)[4][4]) {
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = T(0);
}

}  // namespace dct
