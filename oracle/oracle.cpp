// ORACLE — test infrastructure only. Not part of the product.
//
// A plain-C++ CPU restatement of the reference's sort path
// (hpides/multi-gpu-sorting), used as the checker by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline leg. Nothing in the
// engine (multi-gpu-sorting_b200/) links or calls it.
//
// Order of keys: the order thrust::sort gives for arithmetic keys
// (src/tanasic_sort.cuh:264), i.e. CUB DeviceRadixSort 2.8.2 (the thrust/CUB
// bundled with CUDA 12.9; the reference's own thrust submodule commit is not
// recoverable): unsigned by value; signed by value; IEEE-754 by value with -0.0
// equal to +0.0 (stable, so they keep input order) and NaNs placed by their bit
// pattern after the sign transform. The same order is used for the merge
// steps; for NaN-free keys it coincides with the operator< / operator<= the
// reference's merges use (src/tanasic_sort.cuh:35,163).
//
// Pinned against: the reference's own DataGenerator, gnu-parallel sort,
// multiway merge and TanasicSort compiled from its sources into oracle/_ref
// (oracle/Makefile). tests/golden holds hashes of the reference
// DataGenerator's output (tests/golden/make_golden.py); the sort results are
// compared with the reference's TanasicSort / CUB at test time, on the GPU.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <queue>
#include <vector>

namespace {

template <typename U, int KIND>
struct Order {
  static constexpr int kBits = int(sizeof(U) * 8);
  static constexpr U kSign = U(1) << (kBits - 1);
  static U key(U b) {
    if (KIND == 0) return b;
    if (KIND == 1) return b ^ kSign;
    if (b == kSign) b = 0;  // -0.0 ranks as +0.0
    return (b & kSign) ? U(~b) : U(b ^ kSign);
  }
  static bool less(U a, U b) { return key(a) < key(b); }
};

// Largest key value of the reference's element type T, as bits
// (std::numeric_limits<T>::max(), the filler of src/tanasic_sort.cuh:256-259).
template <typename U, int KIND>
U type_max_bits() {
  if (KIND == 0) return std::numeric_limits<U>::max();
  if (KIND == 1) return std::numeric_limits<U>::max() >> 1;
  if (sizeof(U) == 4) {
    float f = std::numeric_limits<float>::max();
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return U(b);
  }
  double d = std::numeric_limits<double>::max();
  uint64_t b;
  std::memcpy(&b, &d, 8);
  return U(b);
}

template <typename U, int KIND>
void stable_sort_keys(U* p, size_t n) {
  // LSD counting sort by the radix order, 8-bit digits: stable and O(n).
  if (n < 2) return;
  std::vector<U> tmp(n);
  U* src = p;
  U* dst = tmp.data();
  for (int pass = 0; pass < int(sizeof(U)); ++pass) {
    size_t count[257] = {0};
    for (size_t i = 0; i < n; ++i) ++count[((Order<U, KIND>::key(src[i]) >> (8 * pass)) & 0xFF) + 1];
    bool trivial = false;
    for (int d = 1; d <= 256; ++d) trivial |= (count[d] == n);
    if (trivial) continue;
    for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
    for (size_t i = 0; i < n; ++i) dst[count[(Order<U, KIND>::key(src[i]) >> (8 * pass)) & 0xFF]++] = src[i];
    std::swap(src, dst);
  }
  if (src != p) std::memcpy(p, src, n * sizeof(U));
}

// thrust::merge semantics (src/tanasic_sort.cuh:163-167): stable; on ties the
// element of the first range comes first.
template <typename U, int KIND>
void merge_two(const U* a, size_t na, const U* b, size_t nb, U* out) {
  size_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) out[k++] = Order<U, KIND>::less(b[j], a[i]) ? b[j++] : a[i++];
  while (i < na) out[k++] = a[i++];
  while (j < nb) out[k++] = b[j++];
}

// ---- TanasicSort restated over g partitions of host memory ----------------
template <typename U, int KIND>
struct Partitions {
  size_t psize;
  std::vector<std::vector<U>> primary, secondary;  // flipped together per partition like DeviceBuffers::Flip
  void flip(int p) { std::swap(primary[p], secondary[p]); }
};

// SelectPivot/FindPivot (src/tanasic_sort.cuh:15-87): binary search for the
// largest p such that local[N - p] > remote[p - 1] over the virtual
// concatenations of the left and right halves.
template <typename U, int KIND>
size_t find_pivot(Partitions<U, KIND>& P, const std::vector<int>& devs) {
  const size_t half = devs.size() / 2;
  auto local = [&](size_t idx) { return P.primary[devs[idx / P.psize]][idx % P.psize]; };
  auto remote = [&](size_t idx) { return P.primary[devs[half + idx / P.psize]][idx % P.psize]; };
  size_t low = 0, high = P.psize * half;
  while (low < high) {
    const size_t mid = high - (high - low) / 2;
    const U a = local(P.psize * half - mid);
    const U b = remote(mid - 1);
    if (!Order<U, KIND>::less(b, a)) {  // a <= b
      high = mid - 1;
    } else {
      low = mid;
    }
  }
  return low;
}

// SwapPartitions (src/tanasic_sort.cuh:89-146).
template <typename U, int KIND>
std::pair<int, int> swap_partitions(Partitions<U, KIND>& P, size_t pivot, const std::vector<int>& devs) {
  const size_t ps = P.psize;
  const size_t half = devs.size() / 2;
  size_t to_swap = pivot / ps;
  if (pivot == ps * half) {
    --to_swap;
    pivot = ps;
  } else {
    pivot %= ps;
  }
  std::pair<int, int> merge_pair{-1, -1};
  for (size_t i = 0; i <= to_swap; ++i) {
    const int left = devs[half - i - 1];
    const int right = devs[half + i];
    const size_t num = (i == to_swap) ? pivot : ps;
    std::copy(P.primary[right].begin(), P.primary[right].begin() + num, P.secondary[left].begin() + (ps - num));
    std::copy(P.primary[left].begin() + (ps - num), P.primary[left].end(), P.secondary[right].begin());
    if (i == to_swap) {
      merge_pair = {left, right};
      const int pair[2] = {left, right};
      for (int j = 0; j < 2; ++j) {
        const size_t off = size_t(j) * pivot;
        std::copy(P.primary[pair[j]].begin() + off, P.primary[pair[j]].begin() + off + (ps - pivot),
                  P.secondary[pair[j]].begin() + off);
      }
    }
    P.flip(left);
    P.flip(right);
  }
  return merge_pair;
}

// MergeLocalPartitions (src/tanasic_sort.cuh:148-174).
template <typename U, int KIND>
void merge_local(Partitions<U, KIND>& P, size_t pivot, std::pair<int, int> mp, const std::vector<int>& devs) {
  const size_t ps = P.psize;
  pivot %= ps;
  for (size_t i = 0; i < devs.size(); ++i) {
    const int d = devs[i];
    if (d != mp.first && d != mp.second) continue;
    const size_t off = i >= devs.size() / 2 ? pivot : ps - pivot;
    merge_two<U, KIND>(P.primary[d].data(), off, P.primary[d].data() + off, ps - off, P.secondary[d].data());
    P.flip(d);
  }
}

// MergePartitions (src/tanasic_sort.cuh:176-204).
template <typename U, int KIND>
void merge_partitions(Partitions<U, KIND>& P, const std::vector<int>& devs) {
  const size_t h = devs.size() / 2;
  if (devs.size() > 2) {
    merge_partitions(P, std::vector<int>(devs.begin(), devs.begin() + h));
    merge_partitions(P, std::vector<int>(devs.begin() + h, devs.end()));
  }
  const size_t pivot = find_pivot(P, devs);
  if (pivot > 0) {
    auto mp = swap_partitions(P, pivot, devs);
    merge_local(P, pivot, mp, devs);
  }
  if (devs.size() > 2) {
    merge_partitions(P, std::vector<int>(devs.begin(), devs.begin() + h));
    merge_partitions(P, std::vector<int>(devs.begin() + h, devs.end()));
  }
}

// TanasicSort (src/tanasic_sort.cuh:223-299) with g partitions, in place.
template <typename U, int KIND>
void tanasic_sort(U* keys, size_t n, size_t g) {
  if (n == 0 || g == 0) return;
  size_t fillers = (n % g != 0) ? (g - n % g) : 0;
  size_t bs = (n + fillers) / g;
  while (bs < fillers) {
    g /= 2;
    fillers = (n % g != 0) ? (g - n % g) : 0;
    bs = (n + fillers) / g;
  }
  Partitions<U, KIND> P;
  P.psize = bs;
  P.primary.assign(g, std::vector<U>(bs));
  P.secondary.assign(g, std::vector<U>(bs));
  const U filler = type_max_bits<U, KIND>();
  for (size_t i = 0; i < g; ++i) {
    const size_t cnt = bs - (i == g - 1 ? fillers : 0);
    std::copy(keys + i * bs, keys + i * bs + cnt, P.primary[i].begin());
    if (i == g - 1) std::fill(P.primary[i].end() - fillers, P.primary[i].end(), filler);
    stable_sort_keys<U, KIND>(P.primary[i].data(), bs);
  }
  if (g > 1) {
    std::vector<int> devs(g);
    std::iota(devs.begin(), devs.end(), 0);
    merge_partitions(P, devs);
  }
  for (size_t i = 0; i < g; ++i) {
    const size_t cnt = bs - (i == g - 1 ? fillers : 0);
    std::copy(P.primary[i].begin(), P.primary[i].begin() + cnt, keys + i * bs);
  }
}

// Stable k-way merge (ties: the lower run index first). The reference merges
// with __gnu_parallel::multiway_merge (src/gowanlock_sort.cuh:73-74,91-92),
// which is not stable; for keys without equal-comparing distinct bit patterns
// (all integer keys, floats without -0.0/+0.0 pairs or NaN) the outputs agree.
template <typename U, int KIND>
void kway_merge(const U* const* runs, const size_t* lens, int k, U* out) {
  using Item = std::pair<U, int>;
  auto cmp = [](const Item& x, const Item& y) {
    if (Order<U, KIND>::less(x.first, y.first)) return false;
    if (Order<U, KIND>::less(y.first, x.first)) return true;
    return x.second > y.second;
  };
  std::priority_queue<Item, std::vector<Item>, decltype(cmp)> pq(cmp);
  std::vector<size_t> pos(k, 0);
  for (int r = 0; r < k; ++r)
    if (lens[r] > 0) pq.push({runs[r][0], r});
  size_t o = 0;
  while (!pq.empty()) {
    Item it = pq.top();
    pq.pop();
    out[o++] = it.first;
    const int r = it.second;
    if (++pos[r] < lens[r]) pq.push({runs[r][pos[r]], r});
  }
}

template <typename Fn>
int dispatch(int dtype, Fn&& fn) {
  switch (dtype) {
    case 0: fn(Order<uint32_t, 0>{}); return 0;
    case 1: fn(Order<uint32_t, 1>{}); return 0;
    case 2: fn(Order<uint32_t, 2>{}); return 0;
    case 3: fn(Order<uint64_t, 0>{}); return 0;
    case 4: fn(Order<uint64_t, 1>{}); return 0;
    case 5: fn(Order<uint64_t, 2>{}); return 0;
    default: return 1;
  }
}

template <typename O>
struct Parts;
template <typename U, int KIND>
struct Parts<Order<U, KIND>> {
  using Bits = U;
  static constexpr int kKind = KIND;
};

}  // namespace

extern "C" {

// Stable ascending sort in the thrust::sort order (src/tanasic_sort.cuh:264).
int oracle_sort(int dtype, void* keys, size_t n) {
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    stable_sort_keys<typename P::Bits, P::kKind>(static_cast<typename P::Bits*>(keys), n);
  });
}

// Key-value sort in the thrust::sort_by_key order (the reference's sort order,
// stable: values of equal keys keep their input order). value_bytes is 4 or 8;
// values are opaque payloads that follow their keys.
int oracle_sort_pairs(int dtype, void* keys, void* values, size_t value_bytes, size_t n) {
  if (value_bytes != 4 && value_bytes != 8) return 1;
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    U* k = static_cast<U*>(keys);
    std::vector<size_t> perm(n);
    std::iota(perm.begin(), perm.end(), size_t(0));
    std::stable_sort(perm.begin(), perm.end(),
                     [&](size_t a, size_t b) { return Order<U, P::kKind>::less(k[a], k[b]); });
    std::vector<U> kk(n);
    std::vector<unsigned char> vv(n * value_bytes);
    const unsigned char* v = static_cast<const unsigned char*>(values);
    for (size_t i = 0; i < n; ++i) {
      kk[i] = k[perm[i]];
      std::memcpy(&vv[i * value_bytes], v + perm[i] * value_bytes, value_bytes);
    }
    if (n) {
      std::memcpy(keys, kk.data(), n * sizeof(U));
      std::memcpy(values, vv.data(), n * value_bytes);
    }
  });
}

// CUB's begin_bit / end_bit and descending forms (the library behind the
// reference's thrust::sort): stable sort by bits [begin, end) of the ordered
// key, reversed when descending; values (value_bytes 4 or 8, 0 = none) follow.
int oracle_sort_range(int dtype, void* keys, void* values, size_t value_bytes, size_t n, int begin, int end,
                      int descending) {
  if (value_bytes != 0 && value_bytes != 4 && value_bytes != 8) return 1;
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    U* k = static_cast<U*>(keys);
    const int width = end - begin;
    auto bits = [&](U x) -> U {
      if (width <= 0) return U(0);
      U full = Order<U, P::kKind>::key(x);
      // CUB's onesweep maps both zeros of IEEE keys to the ordered pattern of -0.0 when descending
      // (cub/block/radix_rank_sort_operations.cuh, BaseDigitExtractor), of +0.0 when ascending.
      if (P::kKind == 2 && descending && full == Order<U, P::kKind>::kSign) full = Order<U, P::kKind>::kSign - 1;
      const U ord = full >> begin;
      return width >= int(sizeof(U) * 8) ? ord : U(ord & ((U(1) << width) - 1));
    };
    std::vector<size_t> perm(n);
    std::iota(perm.begin(), perm.end(), size_t(0));
    std::stable_sort(perm.begin(), perm.end(), [&](size_t a, size_t b) {
      return descending ? bits(k[b]) < bits(k[a]) : bits(k[a]) < bits(k[b]);
    });
    std::vector<U> kk(n);
    for (size_t i = 0; i < n; ++i) kk[i] = k[perm[i]];
    if (n) std::memcpy(keys, kk.data(), n * sizeof(U));
    if (value_bytes) {
      std::vector<unsigned char> vv(n * value_bytes);
      const unsigned char* v = static_cast<const unsigned char*>(values);
      for (size_t i = 0; i < n; ++i) std::memcpy(&vv[i * value_bytes], v + perm[i] * value_bytes, value_bytes);
      if (n) std::memcpy(values, vv.data(), n * value_bytes);
    }
  });
}

// thrust::merge of two sorted ranges (src/tanasic_sort.cuh:163-167).
int oracle_merge(int dtype, const void* a, size_t na, const void* b, size_t nb, void* out) {
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    merge_two<U, P::kKind>(static_cast<const U*>(a), na, static_cast<const U*>(b), nb, static_cast<U*>(out));
  });
}

// FindPivot over g sorted partitions given back to back in `keys` (partition
// size psize); returns the pivot of the top-level merge step.
int oracle_find_pivot(int dtype, const void* keys, size_t psize, int g, size_t* pivot) {
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    Partitions<U, P::kKind> parts;
    parts.psize = psize;
    for (int i = 0; i < g; ++i) {
      const U* p = static_cast<const U*>(keys) + size_t(i) * psize;
      parts.primary.emplace_back(p, p + psize);
    }
    std::vector<int> devs(g);
    std::iota(devs.begin(), devs.end(), 0);
    *pivot = find_pivot(parts, devs);
  });
}

// TanasicSort with g partitions (src/tanasic_sort.cuh:223-299), in place.
int oracle_tanasic_sort(int dtype, void* keys, size_t n, int g) {
  if (g <= 0 || (g & (g - 1)) != 0) return 1;
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    tanasic_sort<typename P::Bits, P::kKind>(static_cast<typename P::Bits*>(keys), n, size_t(g));
  });
}

// Stable k-way merge of sorted runs (HET sort's merge, src/gowanlock_sort.cuh:29-95).
int oracle_kway_merge(int dtype, const void* const* runs, const size_t* lens, int k, void* out) {
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    kway_merge<U, P::kKind>(reinterpret_cast<const U* const*>(runs), lens, k, static_cast<U*>(out));
  });
}

// Each segment [offsets[i], offsets[i+1]) sorted stably on its own.
int oracle_segmented_sort(int dtype, void* keys, const uint64_t* offsets, size_t num_segments) {
  return dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    for (size_t s = 0; s < num_segments; ++s) {
      U* p = static_cast<U*>(keys) + offsets[s];
      stable_sort_keys<U, P::kKind>(p, size_t(offsets[s + 1] - offsets[s]));
    }
  });
}

// Radix-order key of one value (for tests that check order properties).
uint64_t oracle_order_key(int dtype, uint64_t bits) {
  uint64_t r = 0;
  dispatch(dtype, [&](auto o) {
    using P = Parts<decltype(o)>;
    using U = typename P::Bits;
    r = uint64_t(Order<U, P::kKind>::key(U(bits)));
  });
  return r;
}

}  // extern "C"
