// TanasicSort over g chunks of one GPU (see chunk_sort.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace mgs {

struct Context;

struct ChunkPlan {
  int g;           // chunks actually used (halved while chunks would be shorter than the padding)
  size_t fillers;  // padding keys at the end of the last chunk
  size_t chunk;    // keys per chunk
};

ChunkPlan plan_chunks(size_t n, int g);
size_t chunk_sort_temp_bytes(int dtype, size_t n, int g);

// Sorts n keys with the P2P merge tree over g chunks. Input from h_in (host)
// or d_io (device); output to h_out (host) or d_io (device). temp must hold
// chunk_sort_temp_bytes(). Stream-ordered on s; the pivot readbacks synchronize s.
cudaError_t chunk_sort(Context& c, int dtype, const void* h_in, void* h_out, void* d_io, size_t n, int g, void* temp,
                       size_t temp_bytes, cudaStream_t s);

}  // namespace mgs
