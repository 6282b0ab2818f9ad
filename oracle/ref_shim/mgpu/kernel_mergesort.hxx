// Compile-only stand-in for ModernGPU's kernel_mergesort.hxx, a third-party library the
// reference's PageRank includes (src/static_page_rank/pr.cu:15) and that is absent here: the
// three names it uses (standard_context_t, greater_t, mergesort of keys with values), with the
// sort done by CUB's radix sort of pairs (descending for greater_t). Build support for running the
// reference's own algorithm sources; nothing in the library uses it.
#pragma once

#include <cub/cub.cuh>

namespace mgpu {

struct standard_context_t {
  explicit standard_context_t(bool print_prop = true) { (void)print_prop; }
};

template <class T>
struct greater_t {};

template <class K, class V, class C>
void mergesort(K* keys, V* vals, int count, C comp, standard_context_t& context) {
  (void)comp;
  (void)context;
  K* k2 = nullptr;
  V* v2 = nullptr;
  void* tmp = nullptr;
  size_t bytes = 0;
  cudaMalloc(&k2, sizeof(K) * count);
  cudaMalloc(&v2, sizeof(V) * count);
  cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, keys, k2, vals, v2, count);
  cudaMalloc(&tmp, bytes);
  cub::DeviceRadixSort::SortPairsDescending(tmp, bytes, keys, k2, vals, v2, count);
  cudaMemcpy(keys, k2, sizeof(K) * count, cudaMemcpyDeviceToDevice);
  cudaMemcpy(vals, v2, sizeof(V) * count, cudaMemcpyDeviceToDevice);
  cudaFree(tmp);
  cudaFree(k2);
  cudaFree(v2);
}

}  // namespace mgpu
