// Merge kernels for one B200 (sm_100a).
//
//   K3 pivot_search    : SelectPivot/FindPivot of P2P sort (src/tanasic_sort.cuh:
//                        15-87) as one warp doing a 32-ary search over the
//                        virtual concatenations of the left and right chunks
//                        (about log32(N) dependent rounds instead of log2(N)).
//   K4 merge_partition : merge-path diagonal search for a two-way merge, one
//                        thread per output tile boundary.
//   K7a kway_partition : exact multi-sequence selection for a k-way merge, one
//                        warp per output tile boundary: bisection over the radix
//                        order key space, every lane narrowing the index window of
//                        its runs, then ties split by run index (stable).
//                        Hierarchical: coarser levels (every 256, then every
//                        16 tiles) bound the finer searches.
//   K5/K7b tile_merge  : per output tile, the k input ranges are staged in shared
//                        memory in run order and merged by ceil(log2 k) rounds of
//                        pairwise merge-path merges in shared memory, then stored
//                        coalesced. k = 2 is thrust::merge (src/tanasic_sort.cuh:
//                        163-167); k > 2 replaces __gnu_parallel::multiway_merge
//                        (src/gowanlock_sort.cuh:73-74,91-92).
// Order: radix order of the keys (KeyTraits::Ordered); on ties the lower run
// (the first range) comes first.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "device_common.cuh"
#include "dispatch.cuh"
#include "merge.cuh"
#include "radix_sort.cuh"

namespace mgs {
namespace {

using u64 = unsigned long long;

template <typename Bits>
struct ChunkTable {
  const Bits* left[kMaxPivotHalf];
  const Bits* right[kMaxPivotHalf];
};

// ---------------------------------------------------------------- K3 --------
template <class Tr>
__global__ __launch_bounds__(32) void pivot_search_kernel(ChunkTable<typename Tr::Bits> tab, int half, u64 psize,
                                                          u64* __restrict__ out) {
  const int lane = threadIdx.x;
  const u64 N = psize * u64(half);
  auto L = [&](u64 i) { return tab.left[i / psize][i % psize]; };
  auto R = [&](u64 i) { return tab.right[i / psize][i % psize]; };
  // f(p) = left[N - p] > right[p - 1] is true exactly for p <= pivot.
  u64 lo = 0, hi = N;
  while (lo < hi) {
    const u64 step = (hi - lo + 31) / 32;
    const u64 p = min(lo + u64(lane + 1) * step, hi);
    const bool t = Tr::Less(R(p - 1), L(N - p));
    const uint32_t bal = __ballot_sync(0xffffffffu, t);
    const int c = __popc(bal);
    if (c == 0) {
      hi = lo + step - 1;
    } else {
      const u64 nlo = min(lo + u64(c) * step, hi);
      const u64 nhi = (c < 32) ? min(lo + u64(c + 1) * step, hi) - 1 : hi;
      lo = nlo;
      hi = nhi;
    }
  }
  if (lane == 0) *out = lo;
}

// ---------------------------------------------------------------- K4 --------
template <class Tr>
__global__ __launch_bounds__(256) void merge_partition_kernel(const typename Tr::Bits* __restrict__ a, u64 na,
                                                              const typename Tr::Bits* __restrict__ b, u64 nb,
                                                              u64 spacing, u64 num_diag, u64* __restrict__ splits) {
  const u64 j = u64(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= num_diag) return;
  const u64 d = min(j * spacing, na + nb);
  u64 lo = d > nb ? d - nb : 0, hi = min(d, na);
  while (lo < hi) {
    const u64 mid = (lo + hi) / 2;
    if (!Tr::Less(b[d - 1 - mid], a[mid])) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  splits[2 * j] = lo;
  splits[2 * j + 1] = d - lo;
}

// ---------------------------------------------------------------- K7a -------
template <typename Bits>
__device__ __forceinline__ u64 warp_sum_u64(u64 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// First index in [lo, hi) whose radix-order key is > v (upper) or >= v (lower).
template <class Tr, bool UPPER>
__device__ __forceinline__ u64 bound_search(const typename Tr::Bits* run, u64 lo, u64 hi, typename Tr::Bits v) {
  while (lo < hi) {
    const u64 mid = (lo + hi) / 2;
    const typename Tr::Bits o = Tr::Ordered(run[mid]);
    if (UPPER ? (o <= v) : (o < v)) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo;
}

constexpr int kMaxRunsPerLane = kMaxKwayRuns / 32;
static_assert(kMaxKwayTileRuns >= kMaxKwayRuns, "the radix tiles take every k-way merge");

// One warp per diagonal d: splits[r] = number of elements of run r among the
// first d outputs of the stable k-way merge. Optional coarse level: the
// splits / ub / lt / v* of the enclosing coarse diagonals bound the search.
// Lane l handles runs l, l + 32, ... (PER_LANE of them, PER_LANE >= k / 32),
// with its per-run search windows in registers.
template <class Tr, int PER_LANE>
__global__ __launch_bounds__(128) void kway_partition_kernel(
    const typename Tr::Bits* const* __restrict__ runs, const u64* __restrict__ lens, int k, u64 total, u64 spacing,
    u64 num_diag, const u64* __restrict__ c_splits, const u64* __restrict__ c_ub, const u64* __restrict__ c_lt,
    const typename Tr::Bits* __restrict__ c_vstar, u64 c_spacing, u64* __restrict__ splits, u64* __restrict__ ub_out,
    u64* __restrict__ lt_out, typename Tr::Bits* __restrict__ vstar_out) {
  using Bits = typename Tr::Bits;
  const u64 w = (u64(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= num_diag) return;
  const u64 d = min(w * spacing, total);
  if (d >= total) {
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
      const int r = lane + 32 * i;
      if (r < k) {
        splits[w * k + r] = lens[r];
        if (ub_out) ub_out[w * k + r] = lens[r];
        if (lt_out) lt_out[w * k + r] = lens[r];
      }
    }
    if (vstar_out && lane == 0) vstar_out[w] = ~Bits(0);
    return;
  }
  u64 a[PER_LANE], b[PER_LANE], base[PER_LANE];
  Bits vlo = 0, vhi = ~Bits(0);
  u64 c0 = 0, c1 = 0;
  if (c_splits) {
    c0 = d / c_spacing;
    c1 = c0 + 1;
    vlo = c_vstar[c0];
    vhi = c_vstar[c1];
  }
#pragma unroll
  for (int i = 0; i < PER_LANE; ++i) {
    const int r = lane + 32 * i;
    if (r < k) {
      a[i] = c_splits ? c_splits[c0 * k + r] : 0;
      base[i] = c_splits ? c_lt[c0 * k + r] : 0;
      b[i] = c_splits ? c_ub[c1 * k + r] : lens[r];
    } else {
      a[i] = b[i] = base[i] = 0;
    }
  }
  // Bisection for v* = the smallest v with (number of keys <= v) > d.
  while (vlo < vhi) {
    u64 width = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) width += b[i] - a[i];
    if (warp_sum_u64<Bits>(width) == 0) break;  // no key strictly inside: v* = vlo
    const Bits vmid = vlo + (vhi - vlo) / 2;
    u64 u[PER_LANE];
    u64 cnt = 0;
#pragma unroll
    for (int i = 0; i < PER_LANE; ++i) {
      const int r = lane + 32 * i;
      u[i] = (r < k) ? bound_search<Tr, true>(runs[r], a[i], b[i], vmid) : 0;
      cnt += u[i];
    }
    const u64 le = warp_sum_u64<Bits>(cnt);
    if (le > d) {
      vhi = vmid;
#pragma unroll
      for (int i = 0; i < PER_LANE; ++i) b[i] = u[i];
    } else {
      vlo = vmid + 1;
#pragma unroll
      for (int i = 0; i < PER_LANE; ++i) a[i] = base[i] = u[i];
    }
  }
  const Bits vs = vlo;
  // Keys equal to v* are split across runs in run order (stability).
  u64 lt[PER_LANE], eq[PER_LANE];
  u64 lt_sum = 0;
#pragma unroll
  for (int i = 0; i < PER_LANE; ++i) {
    const int r = lane + 32 * i;
    if (r < k) {
      lt[i] = bound_search<Tr, false>(runs[r], base[i], b[i], vs);
      const u64 ubr = bound_search<Tr, true>(runs[r], max(a[i], lt[i]), b[i], vs);
      eq[i] = ubr - lt[i];
      if (ub_out) ub_out[w * k + r] = ubr;
      if (lt_out) lt_out[w * k + r] = lt[i];
    } else {
      lt[i] = eq[i] = 0;
    }
    lt_sum += lt[i];
  }
  const u64 rem = d - warp_sum_u64<Bits>(lt_sum);
  u64 before = 0;  // equal keys in all runs with a lower index
#pragma unroll
  for (int i = 0; i < PER_LANE; ++i) {
    u64 incl = eq[i];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const u64 excl = before + incl - eq[i];
    const int r = lane + 32 * i;
    if (r < k) {
      const u64 take = rem > excl ? min(rem - excl, eq[i]) : 0;
      splits[w * k + r] = lt[i] + take;
    }
    before += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (vstar_out && lane == 0) vstar_out[w] = vs;
}

// ---------------------------------------------------------------- K5/K7b ----
// One output tile (BLOCK * ITEMS keys) of a stable k-way merge. The tile's
// slice of every run (from the split matrix) is staged back to back in run
// order in shared memory; then ceil(log2 k) rounds merge neighbouring slices
// pairwise. In a round every thread finds where its ITEMS consecutive outputs
// start in their pair (merge-path search) and merges them serially into
// registers, with one comparison, one select and one shared-memory load per
// key; the last round stores its registers straight to global memory.
// The shared buffers carry one pad element per 128 bytes (a thread's outputs
// sit ITEMS positions from its neighbour's, which without the pad fall into a
// few banks) and spare elements at the end (the serial merge may load one key
// past its slice; that key is never used).
template <typename Bits>
__device__ __forceinline__ uint32_t tile_pad(uint32_t i) {
  return i + i / uint32_t(128 / sizeof(Bits));
}
template <typename Bits>
constexpr size_t tile_buffer_elems(size_t tile) {
  return (tile + tile / (128 / sizeof(Bits)) + 1 + 3) / 4 * 4;
}

template <class Tr, int BLOCK, int ITEMS>
__global__ __launch_bounds__(BLOCK, BLOCK == 256 ? 5 : BLOCK == 512 ? 3 : 1) void tile_merge_kernel(const typename Tr::Bits* const* __restrict__ runs, int k,
                                                           const u64* __restrict__ splits,
                                                           typename Tr::Bits* __restrict__ out, u64 total, u64 tile0) {
  using Bits = typename Tr::Bits;
  constexpr int kTile = BLOCK * ITEMS;
  constexpr uint32_t kBuf = uint32_t(tile_buffer_elems<Bits>(kTile));
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Bits* buf0 = reinterpret_cast<Bits*>(smem_raw);
  Bits* buf1 = buf0 + kBuf;
  const Bits** sptr = reinterpret_cast<const Bits**>(buf1 + kBuf);  // this tile's first key of every run
  uint32_t* seg0 = reinterpret_cast<uint32_t*>(sptr + k);
  uint32_t* seg1 = seg0 + (k + 1);
  __shared__ uint32_t scan_tmp[BLOCK / 32 + 1];

  const int tid = threadIdx.x;
  const u64 j = tile0 + blockIdx.x;
  const u64 d0 = j * u64(kTile);
  const uint32_t cnt = uint32_t(min(u64(kTile), total - d0));

  // Segment offsets of the k input slices (exclusive scan of their lengths).
  const int per_thread = (k + BLOCK - 1) / BLOCK;
  uint32_t local = 0;
  for (int i = 0; i < per_thread; ++i) {
    const int r = tid * per_thread + i;
    if (r < k) {
      const u64 s = splits[j * k + r];
      sptr[r] = runs[r] + s;
      local += uint32_t(splits[(j + 1) * k + r] - s);
    }
  }
  uint32_t tot;
  uint32_t run_off = block_exclusive_scan<BLOCK>(local, scan_tmp, &tot);
  for (int i = 0; i < per_thread; ++i) {
    const int r = tid * per_thread + i;
    if (r < k) {
      seg0[r] = run_off;
      run_off += uint32_t(splits[(j + 1) * k + r] - splits[j * k + r]);
    }
  }
  if (tid == 0) seg0[k] = cnt;
  __syncthreads();

  // Stage the slices back to back: consecutive threads read consecutive keys;
  // every thread issues its ITEMS loads before storing any. A thread's
  // elements are BLOCK apart, so its slice index only moves forward.
  {
    Bits v[ITEMS];
    int r = 0;
    {
      int lo = 0, hi = k;  // largest r with seg0[r] <= tid
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (seg0[mid] <= uint32_t(tid)) {
          lo = mid;
        } else {
          hi = mid;
        }
      }
      r = lo;
    }
    // The current slice in registers: its end and the address of tile
    // position 0 in its run (slice start minus the slice's tile offset).
    uint32_t r_end = seg0[r + 1];
    const Bits* r_base = sptr[r] - seg0[r];
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
      const uint32_t i = uint32_t(t) * BLOCK + tid;
      if (i < cnt) {
        if (i >= r_end) {
          do {
            ++r;
          } while (seg0[r + 1] <= i);  // seg0[k] = cnt > i ends the walk
          r_end = seg0[r + 1];
          r_base = sptr[r] - seg0[r];
        }
        v[t] = __ldg(r_base + i);
      }
    }
#pragma unroll
    for (int t = 0; t < ITEMS; ++t) {
      const uint32_t i = uint32_t(t) * BLOCK + tid;
      if (i < cnt) buf0[tile_pad<Bits>(i)] = v[t];
    }
  }
  __syncthreads();

  // Pairwise merge rounds.
  Bits* src = buf0;
  Bits* dst = buf1;
  uint32_t* so = seg0;
  uint32_t* no = seg1;
  int m = k;
  const uint32_t p0 = uint32_t(tid) * ITEMS;
  const uint32_t nv = p0 < cnt ? min(uint32_t(ITEMS), cnt - p0) : 0u;  // outputs of this thread
  for (;;) {
    const int m2 = (m + 1) / 2;
    for (int i = tid; i <= m2; i += BLOCK) no[i] = (i < m2) ? so[2 * i] : cnt;
    __syncthreads();
    Bits v[ITEMS];
    if (nv > 0) {
      int q = 0, hi = m2;  // pair holding p0: largest q with no[q] <= p0
      while (hi - q > 1) {
        const int mid = (q + hi) >> 1;
        if (no[mid] <= p0) {
          q = mid;
        } else {
          hi = mid;
        }
      }
      // Pair q: A = [a0, a1), B = [a1, b1) (B empty for the odd slice out).
      uint32_t a0 = so[2 * q], a1 = so[min(2 * q + 1, m)], b1 = so[min(2 * q + 2, m)];
      const uint32_t la = a1 - a0, lb = b1 - a1;
      const uint32_t diag = p0 - a0;
      uint32_t s_lo = diag > lb ? diag - lb : 0, s_hi = min(diag, la);
      while (s_lo < s_hi) {
        const uint32_t mid = (s_lo + s_hi) >> 1;
        if (!Tr::Less(src[tile_pad<Bits>(a1 + diag - 1 - mid)], src[tile_pad<Bits>(a0 + mid)])) {
          s_lo = mid + 1;
        } else {
          s_hi = mid;
        }
      }
      uint32_t ia = a0 + s_lo, ib = a1 + (diag - s_lo), a_end = a1, b_end = b1;
      Bits ka = src[tile_pad<Bits>(ia)];
      Bits kb = src[tile_pad<Bits>(ib)];
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        if (uint32_t(i) < nv) {
          while (p0 + i == b_end) {  // this thread's outputs continue in the next non-empty pair
            ++q;
            ia = b_end;
            a_end = so[min(2 * q + 1, m)];
            ib = a_end;
            b_end = so[min(2 * q + 2, m)];
            ka = src[tile_pad<Bits>(ia)];
            kb = src[tile_pad<Bits>(ib)];
          }
          const bool take_a = ia < a_end && (ib >= b_end || !Tr::Less(kb, ka));
          v[i] = take_a ? ka : kb;
          ia += take_a ? 1u : 0u;
          ib += take_a ? 0u : 1u;
          const Bits kn = src[tile_pad<Bits>(take_a ? ia : ib)];
          ka = take_a ? kn : ka;
          kb = take_a ? kb : kn;
        }
      }
    }
    if (m2 == 1) {
      Bits* o = out + d0 + p0;
      if (nv == uint32_t(ITEMS) && (reinterpret_cast<uintptr_t>(o) & 15u) == 0) {
        constexpr int kPerVec = 16 / int(sizeof(Bits));
#pragma unroll
        for (int i = 0; i < ITEMS; i += kPerVec) {
          uint4 q4;
          if constexpr (sizeof(Bits) == 4) {
            q4 = make_uint4(uint32_t(v[i]), uint32_t(v[i + 1]), uint32_t(v[i + 2]), uint32_t(v[i + 3]));
          } else {
            q4 = make_uint4(uint32_t(v[i]), uint32_t(uint64_t(v[i]) >> 32), uint32_t(v[i + 1]),
                            uint32_t(uint64_t(v[i + 1]) >> 32));
          }
          *reinterpret_cast<uint4*>(o + i) = q4;
        }
      } else {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
          if (uint32_t(i) < nv) o[i] = v[i];
      }
      return;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (uint32_t(i) < nv) dst[tile_pad<Bits>(p0 + i)] = v[i];
    __syncthreads();
    Bits* t = src;
    src = dst;
    dst = t;
    uint32_t* ts = so;
    so = no;
    no = ts;
    m = m2;
  }
}

// ---------------------------------------------------------------- host ------
size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Merge tile shapes: 256, 512 or 1024 threads, each merging 16 (4-byte keys)
// or 8 (8-byte keys) outputs; a larger tile means fewer tile boundaries to
// partition and fewer slices per run to stage.
constexpr int kMergeShapes = 3;
template <int KEY_BYTES, int SHAPE>
struct MergeShape {
  static constexpr int kBlock = 256 << SHAPE;
  static constexpr int kItems = KEY_BYTES == 4 ? 16 : 8;
};
constexpr u64 merge_tile_keys(size_t key_bytes, int shape) { return u64(256 << shape) * (key_bytes == 4 ? 16 : 8); }

// The shape a merge of k runs uses: 256 threads for two runs, 512 for more
// (measured on a B200, 2^31 u32 keys: k = 2 6.96 ms against 7.53 with 512
// threads; k = 8 / 32 / 64: 16.27 / 27.50 / 37.48 ms with 256 threads, 16.06 /
// 26.51 / 34.89 with 512, 17.61 / 27.84 / 35.49 with 1024). MGS_MERGE_SHAPE
// (0-2) overrides it for experiments.
int merge_shape(int k) {
  static const int env = [] {
    const char* e = getenv("MGS_MERGE_SHAPE");
    return (e && e[0] >= '0' && e[0] < '0' + kMergeShapes && e[1] == 0) ? e[0] - '0' : -1;
  }();
  if (env >= 0) return env;
  return k <= 2 ? 0 : 1;
}

// The C ABI dtype of a key traits type.
template <class Tr>
constexpr int dtype_of() {
  return (sizeof(typename Tr::Bits) == 4 ? 0 : 3) + Tr::kKind;
}

// Merges of at least this many runs of 4-byte keys sort their output tiles in
// shared memory (kway_radix_tiles: 16384-key tiles, range-limited LSD passes,
// two for uniform keys) instead of ceil(log2 k) pairwise merge rounds over
// 8192-key tiles. Measured on a B200, 2^31 u32 keys in Dirichlet(1) runs,
// sorted tiles against merged tiles (partition included): k = 8: 18.2 / 14.8
// ms, 16: 18.9 / 18.3, 32: 21.4 / 24.6, 64: 25.2 / 32.8. MGS_KWAY_RADIX_MIN_RUNS
// overrides it for experiments (0: never).
int kway_radix_min_runs() {
  static const int env = [] {
    const char* e = getenv("MGS_KWAY_RADIX_MIN_RUNS");
    return e ? atoi(e) : -1;
  }();
  return env >= 0 ? (env == 0 ? kMaxKwayRuns + 1 : env) : 24;
}

// Output tile of a k-way merge: a radix tile or a merge tile.
template <class Tr>
u64 kway_tile_keys(int k, bool* radix) {
  const size_t rt = kway_radix_tile_keys(dtype_of<Tr>());
  *radix = k > 2 && rt != 0 && k >= kway_radix_min_runs();
  return *radix ? u64(rt) : merge_tile_keys(sizeof(typename Tr::Bits), merge_shape(k));
}

// The exact splits of a k-way merge (k > 2) are found level by level: every
// 256 output tiles, then every 16 tiles within those bounds, then at every
// tile boundary within those. A level bounds the next one's value bisection
// and per-run index windows, so the fine searches start from windows of about
// 16 tiles / k keys per run. A level exists only when the merge spans more
// than two of its spacings. Measured on a B200, 2^31 u32 keys, k = 64: the
// partition took 6.3 ms with the 256-tile level alone.
constexpr int kBoundLevels = 2;
constexpr u64 kBoundTiles[kBoundLevels] = {256, 16};  // tiles per diagonal of each bounding level

struct KwayLayout {
  size_t ptrs_off, lens_off, splits_off, total;
  size_t b_splits_off[kBoundLevels], b_ub_off[kBoundLevels], b_lt_off[kBoundLevels], b_vstar_off[kBoundLevels];
  u64 tile, num_tiles;
  u64 b_diag[kBoundLevels];  // diagonals of each bounding level (0: level absent)
  bool radix;
};

template <class Tr>
KwayLayout kway_layout(int k, size_t total) {
  KwayLayout L;
  const u64 kTile = kway_tile_keys<Tr>(k, &L.radix);
  L.tile = kTile;
  L.num_tiles = (total + kTile - 1) / kTile;
  size_t off = 0;
  L.ptrs_off = off;
  off += align_up(size_t(k) * 8, 256);
  L.lens_off = off;
  off += align_up(size_t(k) * 8, 256);
  L.splits_off = off;
  off += align_up(size_t(L.num_tiles + 1) * k * 8, 256);
  for (int l = 0; l < kBoundLevels; ++l) {
    const u64 spacing = kTile * kBoundTiles[l];
    const bool on = (k > 2) && (L.num_tiles > 2 * kBoundTiles[l]);
    L.b_diag[l] = on ? (total + spacing - 1) / spacing + 1 : 0;
    const size_t cn = size_t(L.b_diag[l]);
    L.b_splits_off[l] = off;
    off += align_up(cn * k * 8, 256);
    L.b_ub_off[l] = off;
    off += align_up(cn * k * 8, 256);
    L.b_lt_off[l] = off;
    off += align_up(cn * k * 8, 256);
    L.b_vstar_off[l] = off;
    off += align_up(cn * sizeof(typename Tr::Bits), 256);
  }
  L.total = off;
  return L;
}

// kway_partition_kernel with the smallest runs-per-lane count that covers k.
template <class Tr, typename... Args>
cudaError_t launch_partition(LaunchRecorder* rec, int k, dim3 grid, cudaStream_t stream, Args... args) {
  const int per_lane = (k + 31) / 32;
#define MGS_PARTITION(L) \
  launch_kernel(rec, "kway_partition", kway_partition_kernel<Tr, L>, grid, dim3(128), 0, stream, args...)
  if (per_lane <= 1) return MGS_PARTITION(1);
  if (per_lane <= 2) return MGS_PARTITION(2);
  if (per_lane <= 4) return MGS_PARTITION(4);
  if (per_lane <= 8) return MGS_PARTITION(8);
  return MGS_PARTITION(kMaxRunsPerLane);
#undef MGS_PARTITION
}

// The tile-merge launches of one merge, window by window.
template <class Tr, class Shape>
cudaError_t launch_tile_merges(const typename Tr::Bits* const* d_runs, int k, const u64* d_splits,
                               typename Tr::Bits* out, u64 total, u64 num_tiles, size_t window_keys,
                               const MergeWindowFn& on_window, cudaStream_t stream, LaunchRecorder* rec) {
  using Bits = typename Tr::Bits;
  constexpr u64 kTile = u64(Shape::kBlock) * Shape::kItems;
  auto kernel = tile_merge_kernel<Tr, Shape::kBlock, Shape::kItems>;
  const size_t bufs = 2 * tile_buffer_elems<Bits>(kTile) * sizeof(Bits);
  const size_t smem = bufs + size_t(k) * 8 + size_t(2 * (k + 1)) * 4;
  static SmemLimitOnce attr;
  cudaError_t e = attr.ensure(kernel, bufs + size_t(kMaxKwayRuns) * 8 + size_t(2 * (kMaxKwayRuns + 1)) * 4);
  if (e != cudaSuccess) return e;
  // Output tiles in windows of about window_keys keys (one window when 0).
  const u64 per_window = window_keys == 0 ? num_tiles : std::max<u64>(1, (u64(window_keys) + kTile - 1) / kTile);
  for (u64 t0 = 0; t0 < num_tiles; t0 += per_window) {
    const u64 t1 = std::min<u64>(num_tiles, t0 + per_window);
    e = launch_kernel(rec, k == 2 ? "merge_tiles" : "kway_merge_tiles", kernel, dim3(unsigned(t1 - t0)),
                      dim3(Shape::kBlock), smem, stream, d_runs, k, d_splits, out, total, t0);
    if (e != cudaSuccess) return e;
    if (on_window) {
      const u64 first = t0 * kTile, last = std::min<u64>(total, t1 * kTile);
      e = on_window(size_t(first), size_t(last - first));
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

template <class Tr>
cudaError_t kway_merge_typed(const void* const* runs_v, const size_t* lens, int k, void* out_v, void* temp,
                             size_t temp_bytes, size_t window_keys, const MergeWindowFn& on_window,
                             cudaStream_t stream, LaunchRecorder* rec) {
  using Bits = typename Tr::Bits;
  if (k <= 0 || k > kMaxKwayRuns) return cudaErrorInvalidValue;
  const int shape = merge_shape(k);
  size_t total = 0;
  for (int r = 0; r < k; ++r) total += lens[r];
  if (total == 0) return cudaSuccess;
  Bits* out = static_cast<Bits*>(out_v);
  if (k == 1) {
    cudaError_t e = cudaMemcpyAsync(out, runs_v[0], lens[0] * sizeof(Bits), cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess && on_window) e = on_window(0, total);
    return e;
  }
  const KwayLayout L = kway_layout<Tr>(k, total);
  const u64 kTile = L.tile;
  if (temp == nullptr || temp_bytes < L.total) return cudaErrorInvalidValue;
  char* tb = static_cast<char*>(temp);
  const Bits** d_runs = reinterpret_cast<const Bits**>(tb + L.ptrs_off);
  u64* d_lens = reinterpret_cast<u64*>(tb + L.lens_off);
  u64* d_splits = reinterpret_cast<u64*>(tb + L.splits_off);
  {
    // Pageable-source copies are staged by the runtime before the call returns.
    std::vector<u64> hp(k), hl(k);
    for (int r = 0; r < k; ++r) {
      hp[r] = reinterpret_cast<u64>(runs_v[r]);
      hl[r] = lens[r];
    }
    cudaError_t e = cudaMemcpyAsync(d_runs, hp.data(), size_t(k) * 8, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_lens, hl.data(), size_t(k) * 8, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return e;
  }
  const u64 num_diag = L.num_tiles + 1;
  cudaError_t e;
  if (k == 2) {
    e = launch_kernel(rec, "merge_partition", merge_partition_kernel<Tr>, dim3(unsigned((num_diag + 255) / 256)),
                      dim3(256), 0, stream, static_cast<const Bits*>(runs_v[0]), u64(lens[0]),
                      static_cast<const Bits*>(runs_v[1]), u64(lens[1]), kTile, num_diag, d_splits);
  } else {
    // Bounding levels, coarsest first, each bounded by the one before; then every tile boundary.
    const u64* c_splits = nullptr;
    const u64* c_ub = nullptr;
    const u64* c_lt = nullptr;
    const Bits* c_vstar = nullptr;
    u64 c_spacing = 1;
    for (int l = 0; l < kBoundLevels; ++l) {
      if (L.b_diag[l] == 0) continue;
      u64* cs = reinterpret_cast<u64*>(tb + L.b_splits_off[l]);
      u64* cu = reinterpret_cast<u64*>(tb + L.b_ub_off[l]);
      u64* cl = reinterpret_cast<u64*>(tb + L.b_lt_off[l]);
      Bits* cv = reinterpret_cast<Bits*>(tb + L.b_vstar_off[l]);
      const u64 spacing = kTile * kBoundTiles[l];
      const u64 cdiag = L.b_diag[l];
      e = launch_partition<Tr>(rec, k, dim3(unsigned((cdiag * 32 + 127) / 128)), stream, d_runs, d_lens, k,
                               u64(total), spacing, cdiag, c_splits, c_ub, c_lt, c_vstar, c_spacing, cs, cu, cl,
                               cv);
      if (e != cudaSuccess) return e;
      c_splits = cs;
      c_ub = cu;
      c_lt = cl;
      c_vstar = cv;
      c_spacing = spacing;
    }
    e = launch_partition<Tr>(rec, k, dim3(unsigned((num_diag * 32 + 127) / 128)), stream, d_runs, d_lens, k,
                             u64(total), kTile, num_diag, c_splits, c_ub, c_lt, c_vstar, c_spacing, d_splits,
                             static_cast<u64*>(nullptr), static_cast<u64*>(nullptr), static_cast<Bits*>(nullptr));
  }
  if (e != cudaSuccess) return e;
  const Bits* const* cruns = d_runs;
  const u64* csplits = d_splits;
  if (L.radix) {
    // Output tiles in windows of about window_keys keys (one window when 0), as launch_tile_merges.
    const u64 per_window =
        window_keys == 0 ? L.num_tiles : std::max<u64>(1, (u64(window_keys) + kTile - 1) / kTile);
    for (u64 t0 = 0; t0 < L.num_tiles; t0 += per_window) {
      const u64 t1 = std::min<u64>(L.num_tiles, t0 + per_window);
      e = kway_radix_tiles(dtype_of<Tr>(), cruns, k, reinterpret_cast<const uint64_t*>(d_splits), out, u64(total), t0,
                           t1 - t0, stream, rec);
      if (e != cudaSuccess) return e;
      if (on_window) {
        const u64 first = t0 * kTile, last = std::min<u64>(total, t1 * kTile);
        e = on_window(size_t(first), size_t(last - first));
        if (e != cudaSuccess) return e;
      }
    }
    return cudaSuccess;
  }
  switch (shape) {
    case 0:
      return launch_tile_merges<Tr, MergeShape<sizeof(Bits), 0>>(cruns, k, csplits, out, u64(total), L.num_tiles,
                                                                 window_keys, on_window, stream, rec);
    case 1:
      return launch_tile_merges<Tr, MergeShape<sizeof(Bits), 1>>(cruns, k, csplits, out, u64(total), L.num_tiles,
                                                                 window_keys, on_window, stream, rec);
    default:
      return launch_tile_merges<Tr, MergeShape<sizeof(Bits), 2>>(cruns, k, csplits, out, u64(total), L.num_tiles,
                                                                 window_keys, on_window, stream, rec);
  }
}

template <class Tr>
cudaError_t pivot_search_typed(const void* const* left, const void* const* right, int half, size_t psize,
                               uint64_t* d_pivot, cudaStream_t stream, LaunchRecorder* rec) {
  using Bits = typename Tr::Bits;
  if (half <= 0 || half > kMaxPivotHalf || psize == 0) return cudaErrorInvalidValue;
  ChunkTable<Bits> tab{};
  for (int i = 0; i < half; ++i) {
    tab.left[i] = static_cast<const Bits*>(left[i]);
    tab.right[i] = static_cast<const Bits*>(right[i]);
  }
  return launch_kernel(rec, "pivot_search", pivot_search_kernel<Tr>, dim3(1), dim3(32), 0, stream, tab, half,
                       u64(psize), reinterpret_cast<u64*>(d_pivot));
}

}  // namespace

size_t kway_merge_temp_bytes(int dtype, int k, size_t total) {
  size_t bytes = 0;
  if (k < 1) k = 1;
  dispatch_dtype(dtype, [&](auto tr) { bytes = kway_layout<decltype(tr)>(k, total).total; });
  return bytes;
}

cudaError_t kway_merge(int dtype, const void* const* runs, const size_t* lens, int k, void* out, void* d_temp,
                       size_t temp_bytes, cudaStream_t stream, LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    result = kway_merge_typed<decltype(tr)>(runs, lens, k, out, d_temp, temp_bytes, 0, MergeWindowFn(), stream, rec);
  });
  return result;
}

cudaError_t kway_merge_windowed(int dtype, const void* const* runs, const size_t* lens, int k, void* out,
                                void* d_temp, size_t temp_bytes, size_t window_keys, const MergeWindowFn& on_window,
                                cudaStream_t stream, LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    result = kway_merge_typed<decltype(tr)>(runs, lens, k, out, d_temp, temp_bytes, window_keys, on_window, stream,
                                            rec);
  });
  return result;
}

cudaError_t pivot_search(int dtype, const void* const* left, const void* const* right, int half, size_t psize,
                         uint64_t* d_pivot, cudaStream_t stream, LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    result = pivot_search_typed<decltype(tr)>(left, right, half, psize, d_pivot, stream, rec);
  });
  return result;
}

}  // namespace mgs
