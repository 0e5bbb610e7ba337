// TanasicSort (P2P sort, src/tanasic_sort.cuh:176-299 of the reference) with its
// g per-GPU partitions mapped onto g chunks of one GPU's HBM.
//
// The control flow is the reference's: pad n to a multiple of g with the type's
// maximum (:231-238, :255-259), sort every chunk, then MergePartitions (:176-204):
// recurse on both halves, find the pivot between the halves (FindPivot, :45-87),
// exchange the pivot ranges between mirrored chunks (SwapPartitions, :89-146),
// merge the two boundary chunks (MergeLocalPartitions, :148-174), recurse again.
//
// What changes on one GPU: a chunk's data is a pointer into a pool of 2g
// chunk-sized HBM blocks. A fully exchanged mirrored pair swaps its block
// pointers (no copy); the boundary pair's "copy then merge" becomes two merges
// that read the tail of one chunk and the head of the other in place and write
// into free blocks. Per merge step only 2 chunks' worth of keys are read and
// written, instead of the reference's peer copies of every exchanged chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <limits>
#include <vector>

#include "../kernels/engine_types.h"
#include "../kernels/merge.cuh"
#include "../kernels/radix_sort.cuh"
#include "chunk_sort.h"
#include "context.h"

namespace mgs {

namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// numeric_limits<T>::max() of the dtype, as raw bits (the reference's filler).
uint64_t type_max_bits(int dtype) {
  switch (dtype) {
    case 0: return 0xFFFFFFFFull;
    case 1: return 0x7FFFFFFFull;
    case 2: {
      float f = std::numeric_limits<float>::max();
      uint32_t b;
      std::memcpy(&b, &f, 4);
      return b;
    }
    case 3: return 0xFFFFFFFFFFFFFFFFull;
    case 4: return 0x7FFFFFFFFFFFFFFFull;
    default: {
      double d = std::numeric_limits<double>::max();
      uint64_t b;
      std::memcpy(&b, &d, 8);
      return b;
    }
  }
}

cudaError_t fill_pattern(void* dst, size_t count, size_t w, uint64_t bits, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  // Fillers are fewer than g keys: stage them in a small host pattern.
  std::vector<unsigned char> host(count * w);
  for (size_t i = 0; i < count; ++i) std::memcpy(host.data() + i * w, &bits, w);
  return cudaMemcpyAsync(dst, host.data(), count * w, cudaMemcpyHostToDevice, s);
}

struct ChunkTree {
  Context* c;
  int dtype;
  size_t w, ps;
  cudaStream_t s;
  std::vector<char*> data;  // logical chunk -> block holding its keys
  std::vector<char*> free_blocks;
  void* merge_temp;
  size_t merge_temp_bytes;
  uint64_t* d_pivot;
  uint64_t* h_pivot;

  cudaError_t find_pivot(const std::vector<int>& devs, size_t* pivot) {
    const int half = int(devs.size() / 2);
    std::vector<const void*> left(half), right(half);
    for (int i = 0; i < half; ++i) {
      left[i] = data[devs[i]];
      right[i] = data[devs[half + i]];
    }
    cudaError_t e = pivot_search(dtype, left.data(), right.data(), half, ps, d_pivot, s, &c->recorder);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_pivot, d_pivot, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    *pivot = size_t(*h_pivot);
    return e;
  }

  cudaError_t merge_into(const char* a, size_t na, const char* b, size_t nb, char* out) {
    const void* runs[2] = {a, b};
    const size_t lens[2] = {na, nb};
    if (na == 0 || nb == 0) {
      const void* src = na ? a : b;
      return cudaMemcpyAsync(out, src, (na + nb) * w, cudaMemcpyDeviceToDevice, s);
    }
    return kway_merge(dtype, runs, lens, 2, out, merge_temp, merge_temp_bytes, s, &c->recorder);
  }

  // SwapPartitions + MergeLocalPartitions for one step (pivot > 0).
  cudaError_t exchange(size_t pivot, const std::vector<int>& devs) {
    const size_t half = devs.size() / 2;
    size_t full = pivot / ps;
    size_t part = pivot % ps;
    if (pivot == ps * half) {  // every mirrored pair is exchanged completely
      full = half;
      part = 0;
    }
    for (size_t i = 0; i < full; ++i) std::swap(data[devs[half - i - 1]], data[devs[half + i]]);
    if (part == 0) return cudaSuccess;
    const int left = devs[half - full - 1];
    const int right = devs[half + full];
    char* L = data[left];
    char* R = data[right];
    char* nl = free_blocks.back();
    free_blocks.pop_back();
    char* nr = free_blocks.back();
    free_blocks.pop_back();
    // left keeps its head and receives right's head; right receives left's tail
    // and keeps its own tail; each is merged (first range first on ties).
    cudaError_t e = merge_into(L, ps - part, R, part, nl);
    if (e == cudaSuccess) e = merge_into(L + (ps - part) * w, part, R + part * w, ps - part, nr);
    data[left] = nl;
    data[right] = nr;
    free_blocks.push_back(L);
    free_blocks.push_back(R);
    return e;
  }

  cudaError_t merge_partitions(const std::vector<int>& devs) {
    const size_t h = devs.size() / 2;
    cudaError_t e = cudaSuccess;
    if (devs.size() > 2) {
      e = merge_partitions(std::vector<int>(devs.begin(), devs.begin() + h));
      if (e == cudaSuccess) e = merge_partitions(std::vector<int>(devs.begin() + h, devs.end()));
      if (e != cudaSuccess) return e;
    }
    size_t pivot = 0;
    e = find_pivot(devs, &pivot);
    if (e != cudaSuccess) return e;
    if (pivot > 0) {
      e = exchange(pivot, devs);
      if (e != cudaSuccess) return e;
    }
    if (devs.size() > 2) {
      e = merge_partitions(std::vector<int>(devs.begin(), devs.begin() + h));
      if (e == cudaSuccess) e = merge_partitions(std::vector<int>(devs.begin() + h, devs.end()));
    }
    return e;
  }
};

}  // namespace

ChunkPlan plan_chunks(size_t n, int g) {
  // src/tanasic_sort.cuh:231-238: pad to a multiple of g; halve g while a
  // chunk would be shorter than the padding.
  ChunkPlan p;
  size_t gg = size_t(g);
  size_t fillers = (n % gg != 0) ? (gg - n % gg) : 0;
  size_t bs = (n + fillers) / gg;
  while (bs < fillers) {
    gg /= 2;
    fillers = (n % gg != 0) ? (gg - n % gg) : 0;
    bs = (n + fillers) / gg;
  }
  p.g = int(gg);
  p.fillers = fillers;
  p.chunk = bs;
  return p;
}

size_t chunk_sort_temp_bytes(int dtype, size_t n, int g) {
  const ChunkPlan p = plan_chunks(n, g);
  const size_t w = dtype_bytes(dtype);
  const size_t blk = align256(p.chunk * w);
  return 2 * size_t(p.g) * blk + align256(radix_sort_temp_bytes(dtype, p.chunk)) +
         align256(kway_merge_temp_bytes(dtype, 2, 2 * p.chunk)) + 256;
}

cudaError_t chunk_sort(Context& c, int dtype, const void* h_in, void* h_out, void* d_io, size_t n, int g,
                       void* temp, size_t temp_bytes, cudaStream_t s) {
  const size_t w = dtype_bytes(dtype);
  const ChunkPlan p = plan_chunks(n, g);
  const size_t ps = p.chunk;
  const size_t blk = align256(ps * w);
  if (temp_bytes < chunk_sort_temp_bytes(dtype, n, g)) return cudaErrorInvalidValue;
  char* base = static_cast<char*>(temp);
  std::vector<char*> blocks(2 * p.g);
  for (int i = 0; i < 2 * p.g; ++i) blocks[i] = base + size_t(i) * blk;
  char* radix_temp = base + 2 * size_t(p.g) * blk;
  const size_t radix_bytes = align256(radix_sort_temp_bytes(dtype, ps));
  char* merge_temp = radix_temp + radix_bytes;
  const size_t merge_bytes = align256(kway_merge_temp_bytes(dtype, 2, 2 * ps));
  uint64_t* d_pivot = reinterpret_cast<uint64_t*>(merge_temp + merge_bytes);

  // Load: chunk i holds keys [i*ps, (i+1)*ps), the last one padded with fillers.
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < p.g && e == cudaSuccess; ++i) {
    const size_t cnt = ps - (i == p.g - 1 ? p.fillers : 0);
    if (h_in) {
      e = cudaMemcpyAsync(blocks[i], static_cast<const char*>(h_in) + i * ps * w, cnt * w, cudaMemcpyHostToDevice, s);
    } else {
      e = cudaMemcpyAsync(blocks[i], static_cast<const char*>(d_io) + i * ps * w, cnt * w, cudaMemcpyDeviceToDevice,
                          s);
    }
  }
  if (e == cudaSuccess && p.fillers)
    e = fill_pattern(blocks[p.g - 1] + (ps - p.fillers) * w, p.fillers, w, type_max_bits(dtype), s);
  for (int i = 0; i < p.g && e == cudaSuccess; ++i)
    e = radix_sort(dtype, blocks[i], ps, radix_temp, radix_bytes, s, c.d_status, &c.recorder);
  if (e != cudaSuccess) return e;

  ChunkTree tree{&c, dtype, w, ps, s, {}, {}, merge_temp, merge_bytes, d_pivot, c.h_status64};
  tree.data.assign(blocks.begin(), blocks.begin() + p.g);
  tree.free_blocks.assign(blocks.begin() + p.g, blocks.end());
  if (p.g > 1) {
    std::vector<int> devs(p.g);
    for (int i = 0; i < p.g; ++i) devs[i] = i;
    e = tree.merge_partitions(devs);
    if (e != cudaSuccess) return e;
  }
  // Store without the fillers (src/tanasic_sort.cuh:282-292).
  for (int i = 0; i < p.g && e == cudaSuccess; ++i) {
    const size_t cnt = ps - (i == p.g - 1 ? p.fillers : 0);
    if (h_out) {
      e = cudaMemcpyAsync(static_cast<char*>(h_out) + i * ps * w, tree.data[i], cnt * w, cudaMemcpyDeviceToHost, s);
    } else {
      e = cudaMemcpyAsync(static_cast<char*>(d_io) + i * ps * w, tree.data[i], cnt * w, cudaMemcpyDeviceToDevice, s);
    }
  }
  return e;
}

}  // namespace mgs
