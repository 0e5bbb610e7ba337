// Onesweep LSD radix sort for one B200 (sm_100a): the engine's replacement of
// thrust::sort -> CUB DeviceRadixSort, which the reference calls for every
// partition / chunk sort (src/tanasic_sort.cuh:264-266,
// src/gowanlock_sort.cuh:188-190,337-339, src/sort_benchmark.cu:89).
//
// Per sort of n keys of w bytes (P = w 8-bit digit passes):
//   K1 radix_histogram : one streaming read of the keys builds all P digit
//                        histograms at once (16-byte loads; one shared-memory
//                        copy of the histograms per lane, so that the atomics of
//                        a warp never share a bank) and clears the first
//                        look-back array.
//   K1b radix_scan     : exclusive scan per pass -> global bucket starts; marks
//                        passes whose digit is the same for every key (the
//                        stable counting pass is then the identity and is skipped).
//   K2 radix_onesweep  : one launch per pass. Each CTA takes the next tile in
//                        launch order from an atomic counter, stages it in shared
//                        memory with a TMA bulk copy, ranks the keys by digit
//                        (peer groups from ballots for half of the items and
//                        from shared-memory masks for the other half; per-warp
//                        shared-memory counters),
//                        publishes its digit counts, resolves its global offsets
//                        by decoupled look-back over earlier tiles, and scatters
//                        the tile from shared memory in digit order.
//   K3 radix_finalize  : when an odd number of passes ran, copies the result back
//                        into the caller's buffer; reports device status words.
// Algorithmic HBM traffic: n*w*(2P+1) bytes (+ n*w*2 for an odd pass count).
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "device_common.cuh"
#include "dispatch.cuh"
#include "radix_sort.cuh"

namespace mgs {
namespace {

constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;

struct RadixState {
  uint32_t counts[kMaxPasses][kRadix];        // global digit counts (atomically accumulated)
  uint32_t bucket_start[kMaxPasses][kRadix];  // exclusive scan of counts
  uint32_t tile_counter[kMaxPasses];          // launch-order tile ids per pass
  uint32_t skip[kMaxPasses];                  // 1 = every key has the same digit in this pass
  uint32_t error;                             // DeviceStatus bits
  uint32_t pad[7];
};

// Tile shapes per key width: threads x keys per thread, CTAs per SM, ranking
// chains per warp. The default (shape 5: 512 threads x 32 keys, 16384-key
// tiles) is the fastest measured on B200 without register spills.
template <int KEY_BYTES, int SHAPE>
struct OnesweepShape;
#define MGS_SHAPE(W, S, B, I, M, C)                                                 \
  template <>                                                                      \
  struct OnesweepShape<W, S> {                                                     \
    static constexpr int kBlock = B, kItems = I, kMinBlocks = M, kChains = C;      \
  };
MGS_SHAPE(4, 0, 512, 16, 1, 1)
MGS_SHAPE(4, 1, 256, 16, 2, 1)
MGS_SHAPE(4, 2, 512, 24, 1, 1)
MGS_SHAPE(4, 3, 512, 24, 1, 2)
MGS_SHAPE(4, 4, 512, 32, 1, 2)
MGS_SHAPE(4, 5, 512, 32, 1, 1)
MGS_SHAPE(4, 6, 512, 40, 1, 1)
MGS_SHAPE(8, 0, 512, 8, 1, 1)
MGS_SHAPE(8, 1, 256, 8, 2, 1)
MGS_SHAPE(8, 2, 512, 12, 1, 1)
MGS_SHAPE(8, 3, 512, 12, 1, 2)
MGS_SHAPE(8, 4, 512, 16, 1, 2)
MGS_SHAPE(8, 5, 512, 16, 1, 1)
MGS_SHAPE(8, 6, 512, 20, 1, 1)
#undef MGS_SHAPE
constexpr int kNumShapes = 7;
constexpr int kDefaultShape = 5;
constexpr int kSegShape = kDefaultShape;  // tile shape of the segmented sort's kernels

constexpr int kHistBlock = 1024;
constexpr int kHistUnroll = 4;
// Histogram copies per CTA: counter (pass, digit, copy) lives at word
// (pass * 256 + digit) * copies + copy, and lane l updates copy l % copies.
// With 32 copies every atomic of a warp hits its own bank whatever the digits
// are (random digits into one shared histogram cost about 3.5 bank wavefronts
// per warp atomic, equal digits up to 32). 8-byte keys keep 16 copies so that
// both widths use 128 KB.
template <class Tr>
struct HistCopies {
  static constexpr int kCopies = Tr::kPasses <= 4 ? 32 : 16;
  static constexpr size_t kSmemBytes = size_t(Tr::kPasses) * kRadix * kCopies * sizeof(uint32_t);
};
constexpr uint32_t kLookbackSpinLimit = 1u << 25;  // default bound of one look-back wait (polls)
constexpr uint32_t kTmaWaitLimit = 1u << 24;       // default bound of one tile-copy wait (polls)
constexpr uint32_t kNoHeldTile = 0xFFFFFFFFu;
constexpr int kLookahead = 8;  // predecessor statuses fetched per look-back round

// Bounds of the device-side waits and a failure-injection hook, kept in this
// module's device memory so that a test can change them between sorts
// (set_wait_control). hold_tile: the plain sort's tile of that id never
// publishes its look-back status, so the look-back of the tiles after it waits
// on a word that nothing sets until its bound runs out; the sort then reports
// a look-back timeout instead of hanging. The output of such a sort is
// unspecified (every scatter stays inside the array); the next sort is exact
// again. Default: the bounds above, no tile held.
struct WaitControl {
  uint32_t lookback_spins;
  uint32_t tma_polls;
  uint32_t hold_tile;
  uint32_t pad;
};
__device__ WaitControl g_wait_control = {kLookbackSpinLimit, kTmaWaitLimit, kNoHeldTile, 0u};

// Look-back status word: 0 = not published yet; (count + 1) with the top bit
// clear = this tile's own digit count (aggregate); top bit set = inclusive
// prefix over this tile and all earlier ones.
template <typename StatusT>
struct LookbackWord;
template <>
struct LookbackWord<uint32_t> {
  static constexpr uint32_t kPrefix = 0x80000000u;
  __device__ __forceinline__ static uint32_t load(const uint32_t* p) { return ld_volatile_u32(p); }
  __device__ __forceinline__ static void store(uint32_t* p, uint32_t v) { st_volatile_u32(p, v); }
};
template <>
struct LookbackWord<unsigned long long> {
  static constexpr unsigned long long kPrefix = 0x8000000000000000ull;
  __device__ __forceinline__ static unsigned long long load(const unsigned long long* p) {
    return ld_volatile_u64(p);
  }
  __device__ __forceinline__ static void store(unsigned long long* p, unsigned long long v) {
    st_volatile_u64(p, v);
  }
};

template <typename Bits>
__device__ __forceinline__ void unpack_v4(const uint4& q, Bits (&k)[16 / sizeof(Bits)]);
template <>
__device__ __forceinline__ void unpack_v4<uint32_t>(const uint4& q, uint32_t (&k)[4]) {
  k[0] = q.x;
  k[1] = q.y;
  k[2] = q.z;
  k[3] = q.w;
}
template <>
__device__ __forceinline__ void unpack_v4<unsigned long long>(const uint4& q, unsigned long long (&k)[2]) {
  k[0] = (static_cast<unsigned long long>(q.y) << 32) | q.x;
  k[1] = (static_cast<unsigned long long>(q.w) << 32) | q.z;
}

// ---------------------------------------------------------------- K1 --------
template <class Tr, class Dg = PlainDigits>
__global__ __launch_bounds__(kHistBlock, 1) void radix_histogram_kernel(const typename Tr::Bits* __restrict__ keys,
                                                                     uint32_t n, RadixState* __restrict__ st,
                                                                     uint4* __restrict__ lb0, size_t lb0_vecs, Dg dg) {
  using Bits = typename Tr::Bits;
  constexpr int P = Tr::kPasses;
  constexpr int C = HistCopies<Tr>::kCopies;
  constexpr int kWords = P * kRadix * C;
  constexpr int kPerVec = 16 / int(sizeof(Bits));
  extern __shared__ __align__(16) uint32_t hist_smem[];
  for (int i = threadIdx.x; i < kWords / 4; i += kHistBlock)
    reinterpret_cast<uint4*>(hist_smem)[i] = make_uint4(0u, 0u, 0u, 0u);

  const size_t gtid = size_t(blockIdx.x) * kHistBlock + threadIdx.x;
  const size_t gstride = size_t(gridDim.x) * kHistBlock;
  for (size_t i = gtid; i < lb0_vecs; i += gstride) lb0[i] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();

  uint32_t* const copy = hist_smem + (threadIdx.x & (C - 1));
  auto count_key = [&](Bits k) {
#pragma unroll
    for (int p = 0; p < P; ++p) atomicAdd(copy + (p * kRadix + dg.template digit<Tr>(k, p)) * C, 1u);
  };

  const uintptr_t addr = reinterpret_cast<uintptr_t>(keys);
  size_t head = ((16u - (addr & 15u)) & 15u) / sizeof(Bits);
  if (head > n) head = n;
  const size_t nvec = (n - head) / kPerVec;
  const uint4* kv = reinterpret_cast<const uint4*>(keys + head);
  if (blockIdx.x == 0) {
    for (size_t i = threadIdx.x; i < head; i += kHistBlock) count_key(keys[i]);
    for (size_t i = head + nvec * kPerVec + threadIdx.x; i < n; i += kHistBlock) count_key(keys[i]);
  }
  size_t v = gtid;
  for (; v + (kHistUnroll - 1) * gstride < nvec; v += kHistUnroll * gstride) {
    uint4 q[kHistUnroll];
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) q[u] = ld_stream_v4(kv + v + u * gstride);
#pragma unroll
    for (int u = 0; u < kHistUnroll; ++u) {
      Bits k[kPerVec];
      unpack_v4<Bits>(q[u], k);
#pragma unroll
      for (int j = 0; j < kPerVec; ++j) count_key(k[j]);
    }
  }
  for (; v < nvec; v += gstride) {
    Bits k[kPerVec];
    unpack_v4<Bits>(ld_stream_v4(kv + v), k);
#pragma unroll
    for (int j = 0; j < kPerVec; ++j) count_key(k[j]);
  }
  __syncthreads();
  // Fold the copies: a warp reads 32 consecutive words (32 / C counters) and
  // sums each counter's C copies with shuffles.
  const int lane = threadIdx.x & 31;
  for (int w0 = (threadIdx.x >> 5) * 32; w0 < kWords; w0 += kHistBlock) {
    uint32_t c = hist_smem[w0 + lane];
#pragma unroll
    for (int off = C / 2; off >= 1; off >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, off);
    const int row = (w0 + lane) / C;
    if ((lane & (C - 1)) == 0 && c != 0u) atomicAdd(&st->counts[row / kRadix][row % kRadix], c);
  }
}

// ---------------------------------------------------------------- K1b -------
__global__ __launch_bounds__(kRadix) void radix_scan_kernel(RadixState* __restrict__ st, uint32_t n) {
  __shared__ uint32_t tmp[kRadix / 32 + 1];
  const int p = blockIdx.x, d = threadIdx.x;
  const uint32_t c = st->counts[p][d];
  if (c == n) st->skip[p] = 1u;
  uint32_t total;
  const uint32_t ex = block_exclusive_scan<kRadix>(c, tmp, &total);
  st->bucket_start[p][d] = ex;
}

// ---------------------------------------------------------------- K2 --------
// Value payload of a key-value sort (uint32_t or unsigned long long, opaque
// to the sort); NoValue for a keys-only sort, for which every value step below
// compiles to nothing.
struct NoValue {};
template <typename V>
constexpr bool kHasValues = !std::is_same<V, NoValue>::value;
template <typename V, int N>
struct ValueTiles {
  alignas(16) V v[2][N + 16 / sizeof(V)];  // the values of the two key buffers (+ 16 bytes: aligned window)
};
template <int N>
struct ValueTiles<NoValue, N> {};

template <class Tr, int BLOCK, int ITEMS, int CHAINS, typename V = NoValue>
struct OnesweepSmem {
  static constexpr int kTile = BLOCK * ITEMS;
  static constexpr int kWarps = BLOCK / 32;
  static constexpr int kChains = kWarps * CHAINS;  // ranking chains (CHAINS per warp)
  // Double buffer: tile being sorted / next tile in flight. A tile arrives as
  // the 16-byte-aligned window that covers it, so a row holds 16 bytes more.
  alignas(16) typename Tr::Bits keys[2][kTile + 16 / sizeof(typename Tr::Bits)];
  ValueTiles<V, kTile> vals;
  uint32_t ccount[kChains * kRadix];     // per-chain digit counters -> tile positions
  uint32_t masks[kChains * 2 * kRadix];  // per-chain peer masks (shared-memory multisplit)
  uint32_t tile_start[kRadix];           // exclusive scan of the tile's digit counts
  uint32_t gbase[kRadix];                // global scatter base per digit
  uint32_t scan_tmp[kWarps + 1];
  uint32_t tile_id[2];
  alignas(8) uint64_t bar[2];
  alignas(16) unsigned char span[2][48];  // TileSpan of the current / prefetched tile
};

// Peer mask of lanes holding the same digit (the warp multisplit step), two
// measured ways:
//   MATCH 2: per-chain shared-memory masks: every lane ORs its bit into the
//            mask of its digit, reads the mask back, and the last lane of each
//            group clears it (masks alternate between two arrays per item).
//   MATCH 3: ballots (8, one per digit bit) for half of the items (alternate
//            items, or chain 0 of two), shared-memory masks for the rest, so
//            that the integer-ALU work of one item overlaps the shared-memory
//            latency of the next.
// `ok` separates padding lanes of a partial tile (their digit is 256 + lane).
template <int MATCH, int CHAINS>
__device__ __forceinline__ constexpr bool rank_by_ballot(int h, int j) {
  return MATCH == 3 && (CHAINS == 1 ? (j & 1) == 0 : h == 0);
}

// The peer mask from 8 ballots, one per digit bit: lane k (and k + 16) forms
// the masks of the lanes whose low / high nibble equals k & 15 (four ballots
// each, with k's bits as lane constants), and every lane fetches the two masks
// of its own nibbles with two shuffles: fewer integer operations per item than
// combining all eight ballots in every lane.
template <bool FULL>
__device__ __forceinline__ uint32_t ballot_peers(uint32_t d, bool ok) {
  const uint32_t k = threadIdx.x & 15u;
  uint32_t mlo = 0xffffffffu, mhi = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const uint32_t kb = ((k >> b) & 1u) - 1u;  // 0 where k has bit b, all ones where it has not
    mlo &= __ballot_sync(0xffffffffu, (d >> b) & 1u) ^ kb;
    mhi &= __ballot_sync(0xffffffffu, (d >> (b + 4)) & 1u) ^ kb;
  }
  uint32_t peers =
      __shfl_sync(0xffffffffu, mlo, int(d & 15u)) & __shfl_sync(0xffffffffu, mhi, int((d >> 4) & 15u));
  if (!FULL) {
    const uint32_t bal = __ballot_sync(0xffffffffu, ok);
    peers &= ok ? bal : ~bal;
  }
  return peers;
}

// Phases 1-2 of ranking a tile held in shared memory: stable rank of `valid`
// keys of `src` by the digit of `pass`, written in digit order into `dst`
// (dst may be src). Warp w owns tile positions [w*32*ITEMS, (w+1)*32*ITEMS);
// item i of lane l is position w*32*ITEMS + i*32 + l, so (warp, item, lane) is
// input order. With CHAINS = 2 the warp's items split into two halves ranked as
// independent chains (own counters and masks), interleaved so that their
// shared-memory latencies overlap; the second half's counters start after the
// first half's keys of the same digit. on_counts(count) runs on threads
// d < 256 with the tile's count of digit d before the ranks are formed (the
// onesweep publishes its look-back aggregate there). With ALLOW_SKIP, a digit
// shared by every key makes the pass the identity: nothing is written and the
// function returns true (block-uniform). sm.tile_start receives the exclusive
// scan of the digit counts. between(count) runs on every thread once the
// counts and tile starts are final and before the thread's warp ranks its keys
// (count = the tile's count of digit tid for tid < 256): warps that do extra
// work there rank later, while the other warps rank at once. The caller
// synchronizes before reading dst.
// With values, src_val/dst_val are the value buffers of src/dst: every value
// goes to the slot its key goes to.
// With SPREAD (partial tiles, one chain per warp) the keys may be spread
// thinner: warp w owns positions [w*32*warp_items, (w+1)*32*warp_items), so
// that a short tile keeps every warp busy, and a warp stops at its first item
// that lies wholly past `valid`. Without it the code is the fixed-span form
// the onesweep kernel is tuned on.
//
// LEAN (the onesweep kernel's form) keeps the block barriers per tile at
// three: the per-chain counters of a warp are zero on entry (each warp clears
// its own rows after the tile's scatter), the first barrier also reduces
// `arrived` (false on any thread: the tile's copy never completed; returns
// kRankAborted before anything is written) and is followed by after_a() (the
// next tile's copy may be issued into the other buffer from then on), and the
// tile scan is a warp scan over the first eight warps plus one barrier.
struct NoOp {
  __device__ __forceinline__ void operator()() const {}
};
constexpr int kRankDone = 0, kRankSkipped = 1, kRankAborted = 2;

template <class Tr, int BLOCK, int ITEMS, int CHAINS, int MATCH, bool FULL, bool ALLOW_SKIP, bool SPREAD = false,
          bool LEAN = false, typename V = NoValue, class OnCounts = void, class Between = void,
          class Dg = PlainDigits, class AfterA = NoOp>
__device__ __forceinline__ int rank_tile(OnesweepSmem<Tr, BLOCK, ITEMS, CHAINS, V>& sm, const typename Tr::Bits* src,
                                         typename Tr::Bits* dst, uint32_t valid, int pass, uint32_t* tile_count_out,
                                         OnCounts on_counts, Between between, const V* src_val = nullptr,
                                         V* dst_val = nullptr, Dg dg = Dg{}, uint32_t warp_items = ITEMS,
                                         bool arrived = true, AfterA after_a = AfterA{}) {
  using Bits = typename Tr::Bits;
  constexpr int kTile = BLOCK * ITEMS;
  constexpr int kChains = (BLOCK / 32) * CHAINS;
  constexpr int kPerChain = ITEMS / CHAINS;
  static_assert(ITEMS % CHAINS == 0, "items split evenly into chains");
  static_assert(MATCH == 2 || MATCH == 3, "ranking modes: shared-memory masks, or half ballots");
  static_assert(!(LEAN && ALLOW_SKIP), "the lean form has no identity-pass exit");
  static_assert(BLOCK >= kRadix, "one thread per digit");
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  constexpr bool kSpread = SPREAD && !FULL && CHAINS == 1;
  const int witems = kSpread ? int(warp_items) : ITEMS;
  const int wbase = warp * 32 * witems;
  // Warp-uniform: item i of this warp holds no key of the tile.
  auto item_done = [&](int i) { return kSpread && (i >= witems || uint32_t(wbase + i * 32) >= valid); };

  if constexpr (!LEAN) {
    for (int i = tid; i < kChains * kRadix; i += BLOCK) sm.ccount[i] = 0u;
    __syncthreads();
  }
  // Phase 1: per-chain digit counts.
  Bits key[ITEMS];
  V val[kHasValues<V> ? ITEMS : 1];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (item_done(i)) break;  // positions grow with i: the rest lie past `valid` too
    const uint32_t idx = wbase + i * 32 + lane;
    key[i] = src[idx];
    if constexpr (kHasValues<V>) val[i] = src_val[idx];
    uint32_t* cc = sm.ccount + (warp * CHAINS + i / kPerChain) * kRadix;
    if (FULL || idx < valid) atomicAdd(&cc[dg.template digit<Tr>(key[i], pass)], 1u);
  }
  if constexpr (LEAN) {
    if (__syncthreads_or(!arrived)) return kRankAborted;
  } else {
    __syncthreads();
  }
  after_a();

  uint32_t tile_count = 0;
  if (tid < kRadix) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) tile_count += sm.ccount[c * kRadix + tid];
    on_counts(tile_count);
  }
  *tile_count_out = tile_count;
  if (ALLOW_SKIP) {
    if (__syncthreads_or(tid < kRadix && tile_count == valid)) return kRankSkipped;
  }
  uint32_t tstart = 0;
  if constexpr (LEAN) {
    // exclusive scan of the 256 digit counts: a shuffle scan within each of the
    // first eight warps, then the totals of the warps before.
    uint32_t incl = tile_count;
    if (tid < kRadix) {
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane == 31) sm.scan_tmp[warp] = incl;
    }
    __syncthreads();
    if (tid < kRadix) {
      uint32_t before = 0;
#pragma unroll
      for (int w = 0; w < kRadix / 32; ++w) before += (w < warp) ? sm.scan_tmp[w] : 0u;
      tstart = before + incl - tile_count;
    }
  } else {
    uint32_t total;
    tstart = block_exclusive_scan<BLOCK>(tid < kRadix ? tile_count : 0u, sm.scan_tmp, &total);
  }
  if (tid < kRadix) {
    sm.tile_start[tid] = tstart;
    uint32_t run = tstart;
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      const uint32_t v = sm.ccount[c * kRadix + tid];
      sm.ccount[c * kRadix + tid] = run;
      run += v;
    }
  }
  __syncthreads();
  between(tile_count);

  // Phase 2: stable rank within each chain (peer groups of equal digit, in lane
  // order); each key goes straight to its slot of the tile in digit order.
  const uint32_t lmask = lanemask_lt();
  const uint32_t lmask_gt = lanemask_gt();
#pragma unroll
  for (int j = 0; j < kPerChain; ++j) {
    if (item_done(j)) break;  // chain 0's item j comes first: every chain's item j lies past `valid`
    uint32_t d[CHAINS], peers[CHAINS], pos[CHAINS];
    bool ok[CHAINS];
    uint32_t* cc[CHAINS];
    uint32_t* mm[CHAINS];
#pragma unroll
    for (int h = 0; h < CHAINS; ++h) {
      const int i = h * kPerChain + j;
      const uint32_t idx = wbase + i * 32 + lane;
      ok[h] = FULL || idx < valid;
      d[h] = ok[h] ? dg.template digit<Tr>(key[i], pass) : (256u + lane);
      cc[h] = sm.ccount + (warp * CHAINS + h) * kRadix;
      mm[h] = sm.masks + (warp * CHAINS + h) * 2 * kRadix + (j & 1) * kRadix;
    }
#pragma unroll
    for (int h = 0; h < CHAINS; ++h)
      if (!rank_by_ballot<MATCH, CHAINS>(h, j) && ok[h]) atomicOr(&mm[h][d[h]], 1u << lane);
    __syncwarp();
#pragma unroll
    for (int h = 0; h < CHAINS; ++h)
      peers[h] = rank_by_ballot<MATCH, CHAINS>(h, j) ? ballot_peers<FULL>(d[h], ok[h])
                                                       : (ok[h] ? mm[h][d[h]] : (1u << lane));
#pragma unroll
    for (int h = 0; h < CHAINS; ++h) pos[h] = ok[h] ? cc[h][d[h]] + __popc(peers[h] & lmask) : 0u;
    __syncwarp();
#pragma unroll
    for (int h = 0; h < CHAINS; ++h) {
      if (ok[h] && (peers[h] & lmask_gt) == 0) {
        cc[h][d[h]] = pos[h] + 1u;  // the last lane of each peer group advances the counter
        if (!rank_by_ballot<MATCH, CHAINS>(h, j)) mm[h][d[h]] = 0u;
      }
    }
    // The next item's first __syncwarp orders these counter updates (and mask
    // clears) before its counter reads.
#pragma unroll
    for (int h = 0; h < CHAINS; ++h) {
      if (ok[h] && pos[h] < uint32_t(kTile)) {
        dst[pos[h]] = key[h * kPerChain + j];
        if constexpr (kHasValues<V>) dst_val[pos[h]] = val[h * kPerChain + j];
      }
    }
  }
  return kRankDone;
}

// Where one onesweep tile's keys come from and go to. For the plain sort the
// whole array is one segment; for the segmented sort every large segment is
// its own run of tiles (a tile never spans two segments).
template <class Tr>
struct alignas(16) TileSpan {
  const typename Tr::Bits* src;  // the segment's first key in the source buffer
  typename Tr::Bits* dst;        // the segment's first key in the destination buffer
  uint32_t first_tile;           // global id of the segment's first tile (look-back stops there)
  uint32_t seg_len;              // keys in the segment
  const uint32_t* bucket;        // 256 bucket starts of this pass within the segment
};

// Where a key-value sort's values come from and go to (the whole array).
template <typename V>
struct ValueSpan {
  const V* src;
  V* dst;
};

// One tile: count digits in shared memory (publishing the tile's counts for
// the look-back as soon as they are known), look back over the segment's
// earlier tiles while the other warps rank, scatter the digit runs (with their
// values, svals being the tile's value buffer, when V is a value type).
// SPREAD: a partial tile is ranked over all warps (ceil(valid / BLOCK) keys per
// lane), as the segmented sort's many short last tiles want.
// Returns true (block-uniform) when the tile's copy never completed; nothing
// was written then. Otherwise the calling warp's counter rows are zero again on
// return, and the tile's shared-memory buffer is no longer read.
template <class Tr, int BLOCK, int ITEMS, int CHAINS, typename StatusT, int MATCH, bool FULL, bool SPREAD, typename V,
          class Dg, class AfterA>
__device__ __forceinline__ bool onesweep_tile(OnesweepSmem<Tr, BLOCK, ITEMS, CHAINS, V>& sm, typename Tr::Bits* skeys,
                                              RadixState* __restrict__ st, StatusT* __restrict__ lb_cur,
                                              const TileSpan<Tr>& span, uint32_t tile, uint32_t valid, int pass,
                                              V* svals, const ValueSpan<V>& vspan, Dg dg, uint32_t spin_limit,
                                              bool publish, bool arrived, AfterA after_a) {
  using Bits = typename Tr::Bits;
  using LW = LookbackWord<StatusT>;
  const int tid = threadIdx.x;
  // Decoupled look-back (one thread per digit: the first 256 threads) runs
  // between the counting and the ranking of the tile: it walks back over
  // earlier tiles of the segment, summing their aggregates until it meets an
  // inclusive prefix, with the statuses of kLookahead predecessors fetched per
  // round. With 512 threads the other eight warps rank their keys meanwhile, so
  // the waits on other tiles overlap ranking. A segment's first tile has no
  // predecessor and its last tile places its keys from the bucket ends, so
  // neither waits (in the segmented sort a short last tile would otherwise
  // wait on its predecessor for most of a full tile's time).
  uint32_t tile_count = 0;
  const uint32_t warp_items = (SPREAD && !FULL) ? (valid + BLOCK - 1) / BLOCK : uint32_t(ITEMS);
  const int ranked = rank_tile<Tr, BLOCK, ITEMS, CHAINS, MATCH, FULL, false, SPREAD, true>(
      sm, skeys, skeys, valid, pass, &tile_count,
      [&](uint32_t count) {
        StatusT* slot = lb_cur + size_t(tile) * kRadix + tid;
        if (publish) LW::store(slot, tile == span.first_tile ? (LW::kPrefix | StatusT(count)) : StatusT(count + 1u));
      },
      [&](uint32_t count) {
        if (tid >= kRadix) return;
        StatusT excl = 0;
        if (tile > span.first_tile &&
            (uint64_t(tile - span.first_tile) + 1u) * uint64_t(BLOCK * ITEMS) >= uint64_t(span.seg_len)) {
          // The last tile of a segment (or of the array) needs no look-back: the digit totals of its span are
          // known (the bucket starts), so its keys of digit d end the digit's bucket. No tile looks back at it.
          const uint32_t end = tid + 1 < kRadix ? span.bucket[tid + 1] : span.seg_len;
          excl = StatusT(end - span.bucket[tid] - count);
        } else if (tile > span.first_tile) {
          const long long first = span.first_tile;
          long long jt = static_cast<long long>(tile) - 1;
          uint32_t spins = 0;
          bool done = false;
          while (!done && jt >= first) {
            StatusT sv[kLookahead];
#pragma unroll
            for (int q = 0; q < kLookahead; ++q)
              sv[q] = (jt - q >= first) ? LW::load(lb_cur + size_t(jt - q) * kRadix + tid) : (LW::kPrefix | StatusT(0));
            int used = 0;
#pragma unroll
            for (int q = 0; q < kLookahead; ++q) {
              if (done || used != q) continue;
              const StatusT v = sv[q];
              if (v == 0) continue;  // not published yet: poll it again
              if (v & LW::kPrefix) {
                excl += v & ~LW::kPrefix;
                done = true;
              } else {
                excl += v - 1;
                ++used;
              }
            }
            jt -= used;
            if (!done && used == 0) {
              if (++spins >= spin_limit) {
                atomicOr(&st->error, kStatusLookbackTimeout);
                break;
              }
              if (spins > 8) __nanosleep(32);
            }
          }
          if (publish) LW::store(lb_cur + size_t(tile) * kRadix + tid, LW::kPrefix | (excl + count));
        }
        sm.gbase[tid] = span.bucket[tid] + uint32_t(excl) - sm.tile_start[tid];
      },
      svals, svals, dg, warp_items, arrived, after_a);
  if (ranked == kRankAborted) return true;
  __syncthreads();

  // Phase 3: consecutive threads write consecutive positions of one digit run.
  // The bound check only fails after a look-back timeout (status already set).
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const uint32_t idx = i * BLOCK + tid;
    if (FULL || idx < valid) {
      const Bits k = skeys[idx];
      const uint32_t gpos = sm.gbase[dg.template digit<Tr>(k, pass)] + idx;
      if (gpos < span.seg_len) {
        span.dst[gpos] = k;
        if constexpr (kHasValues<V>) vspan.dst[gpos] = svals[idx];
      }
    }
  }
  // This warp's counter rows back to zero for the next tile: no other warp
  // touches them before the next tile's first barrier.
  uint32_t* own = sm.ccount + (tid >> 5) * CHAINS * kRadix;
  for (int j = tid & 31; j < CHAINS * kRadix; j += 32) own[j] = 0u;
  __syncwarp();
  return false;
}

// Large segments of a segmented sort, as seen by the onesweep kernels.
struct SegLarge {
  const unsigned long long* offsets;  // segment offsets (nseg + 1)
  const uint32_t* ids;                // large segment ids, in segment order
  const uint32_t* tile_prefix;        // first global tile of each large segment (n_large + 1)
  const uint32_t* counts;             // [n_small, n_medium, n_large, large_tiles]
  const uint32_t* bucket;             // [n_large][P][256] bucket starts
  // Per large tile, its segment's {first key, keys, first tile, index into ids}, written by seg_histogram: a
  // tile's span is one 16-byte load (first keys fit 32 bits: segmented sorts take n < 2^32).
  const uint4* tile_info;
};

// The 16-byte-aligned window that covers [p, p + count): it starts at p
// rounded down to 16 bytes and ends at p + count rounded up (the bulk copy's
// alignment rule), and the tile starts `shift` elements into it. ok only when
// the window lies inside the array [lo, hi).
template <typename T>
struct AlignedWindow {
  const T* start;
  uint32_t bytes;
  uint32_t shift;
  bool ok;
};
template <typename T>
__device__ __forceinline__ AlignedWindow<T> aligned_window(const T* p, uint32_t count, const T* lo, const T* hi) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uintptr_t a0 = a & ~uintptr_t(15);
  const uintptr_t e1 = (a + uintptr_t(count) * sizeof(T) + 15) & ~uintptr_t(15);
  AlignedWindow<T> w;
  w.start = reinterpret_cast<const T*>(a0);
  w.bytes = uint32_t(e1 - a0);
  w.shift = uint32_t((a - a0) / sizeof(T));
  w.ok = a0 >= reinterpret_cast<uintptr_t>(lo) && e1 <= reinterpret_cast<uintptr_t>(hi);
  return w;
}

// vbuf0/vbuf1: the value buffers of buf0/buf1 (key-value sort), else null.
template <class Tr, int BLOCK, int ITEMS, int MINB, int CHAINS, typename StatusT, int MATCH, bool SEG,
          typename V = NoValue, class Dg = PlainDigits>
__global__ __launch_bounds__(BLOCK, MINB) void radix_onesweep_kernel(typename Tr::Bits* buf0, typename Tr::Bits* buf1,
                                                                     RadixState* __restrict__ st,
                                                                     StatusT* __restrict__ lb_cur,
                                                                     StatusT* __restrict__ lb_next, uint32_t n,
                                                                     uint32_t num_tiles_arg, int pass, int use_tma,
                                                                     SegLarge sg, V* vbuf0, V* vbuf1, Dg dg) {
  using Bits = typename Tr::Bits;
  using Smem = OnesweepSmem<Tr, BLOCK, ITEMS, CHAINS, V>;
  static_assert(!(SEG && kHasValues<V>), "the segmented sort carries no values");
  constexpr int kTile = Smem::kTile;
  constexpr int kChains = Smem::kChains;
  static_assert(BLOCK >= kRadix, "one thread per digit");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x;
  const uint32_t num_tiles = SEG ? sg.counts[3] : num_tiles_arg;

  // The next pass uses the other look-back array; clear it (grid-stride).
  if (lb_next != nullptr) {
    const size_t words = size_t(num_tiles) * kRadix;
    for (size_t i = size_t(blockIdx.x) * BLOCK + tid; i < words; i += size_t(gridDim.x) * BLOCK) lb_next[i] = 0;
  }
  if (st->skip[pass]) return;  // one digit for every key: identity permutation
  const WaitControl wc = g_wait_control;
  const uint32_t held = SEG ? kNoHeldTile : wc.hold_tile;
  int sel = 0;
  for (int q = 0; q < pass; ++q) sel ^= (st->skip[q] == 0u) ? 1 : 0;
  const Bits* src = sel ? buf1 : buf0;
  Bits* dst = sel ? buf0 : buf1;
  const ValueSpan<V> vspan{sel ? vbuf1 : vbuf0, sel ? vbuf0 : vbuf1};

  // A segmented tile's span comes from its 16-byte record (loaded by the leader when it claims the tile); a
  // plain tile's span is the whole array.
  auto span_of = [&](const uint4& rec) {
    if (SEG) {
      TileSpan<Tr> sp{src + rec.x, dst + rec.x, rec.z, rec.y,
                      sg.bucket + (size_t(rec.w) * Tr::kPasses + pass) * kRadix};
      return sp;
    }
    TileSpan<Tr> sp{src, dst, 0u, n, st->bucket_start[pass]};
    return sp;
  };
  auto record_of = [&](uint32_t t) { return SEG ? sg.tile_info[t] : make_uint4(0u, 0u, 0u, 0u); };
  // Tile t's keys (and values) as aligned windows of the source arrays. The
  // keys of a segment or of an unaligned buffer start anywhere; the window
  // copy still goes through the TMA, and the tile is read `shift` keys into
  // the buffer. Only a window that would leave the array (the first or last
  // tile of an unaligned array) takes plain loads.
  struct Windows {
    AlignedWindow<Bits> k;
    AlignedWindow<V> v;
    bool tma;
  };
  auto windows_of = [&](const TileSpan<Tr>& sp, uint32_t t) {
    const size_t off = size_t(t - sp.first_tile) * kTile;
    const uint32_t count = uint32_t(min(size_t(kTile), size_t(sp.seg_len) - off));
    Windows w;
    w.k = aligned_window<Bits>(sp.src + off, count, src, src + n);
    w.tma = use_tma && w.k.ok;
    if constexpr (kHasValues<V>) {
      const size_t voff = size_t(sp.src - src) + off;
      w.v = aligned_window<V>(vspan.src + voff, count, vspan.src, vspan.src + n);
      w.tma = w.tma && w.v.ok;
    } else {
      w.v = AlignedWindow<V>{nullptr, 0u, 0u, true};
    }
    return w;
  };
  // One tile's windows into buffer b with the TMA, completing on bar[b].
  auto issue_copy = [&](int b, const Windows& w) {
    mbar_arrive_expect_tx(&sm.bar[b], w.k.bytes + (kHasValues<V> ? w.v.bytes : 0u));
    bulk_copy_g2s(sm.keys[b], w.k.start, w.k.bytes, &sm.bar[b]);
    if constexpr (kHasValues<V>) bulk_copy_g2s(sm.vals.v[b], w.v.start, w.v.bytes, &sm.bar[b]);
  };

  // Persistent CTA: tiles come in launch order from an atomic counter. The
  // leader claims the next tile at the top of each iteration and loads its
  // span record (segmented sort); after the first barrier (every warp is past
  // it, so the other buffer's previous tile is fully scattered) it works out
  // the next tile's span and issues its TMA bulk copy into the other buffer,
  // so loads overlap ranking. A CTA's current tile is always older than its
  // prefetched one, so the oldest unfinished tile is always being processed
  // and the look-back makes progress. (Claiming one tile further ahead made a
  // lone 2^30-key sort 0.6 % faster but slowed sorts that share the GPU with
  // others: in the serving loop it cut the full mix's peak from 28.2 to 24.4
  // Gkeys/s and raised its p99 at 0.9 load from about 4 to 17-24 ms.)
  static_assert(sizeof(TileSpan<Tr>) <= sizeof(sm.span[0]), "span slot");
  TileSpan<Tr>* spans = reinterpret_cast<TileSpan<Tr>*>(sm.span);
  for (int i = tid; i < kChains * 2 * kRadix; i += BLOCK) sm.masks[i] = 0u;
  for (int i = tid; i < kChains * kRadix; i += BLOCK) sm.ccount[i] = 0u;  // then kept zero by each warp
  // The thread that claims tiles and issues their copies: a thread of the last
  // warp (the first eight warps run the tile scan and the look-back; a
  // segmented tile's claim is followed by the load of its span record).
  constexpr int kLeader = BLOCK - 32;
  if (tid == kLeader) {
    mbar_init(&sm.bar[0], 1);
    mbar_init(&sm.bar[1], 1);
    fence_mbar_init();
    const uint32_t t = atomicAdd(&st->tile_counter[pass], 1u);
    sm.tile_id[0] = t;
    if (t < num_tiles) {
      const TileSpan<Tr> sp = span_of(record_of(t));
      spans[0] = sp;
      const Windows w = windows_of(sp, t);
      if (w.tma) issue_copy(0, w);
    }
  }
  __syncthreads();
  uint32_t parity = 0;  // bit b = phase parity of bar[b]
  int cur = 0;
  for (;;) {
    const uint32_t tile = sm.tile_id[cur];
    if (tile >= num_tiles) break;
    // Every thread read tile_id / spans of the other slot one iteration ago.
    uint32_t next_tile = num_tiles;
    uint4 next_rec = make_uint4(0u, 0u, 0u, 0u);
    if (tid == kLeader) {
      next_tile = atomicAdd(&st->tile_counter[pass], 1u);
      sm.tile_id[cur ^ 1] = next_tile;
      if (next_tile < num_tiles) next_rec = record_of(next_tile);
    }
    auto issue_next = [&] {
      if (tid == kLeader && next_tile < num_tiles) {
        const TileSpan<Tr> sp = span_of(next_rec);
        spans[cur ^ 1] = sp;
        const Windows w = windows_of(sp, next_tile);
        if (w.tma) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue_copy(cur ^ 1, w);
        }
      }
    };
    const TileSpan<Tr> span = spans[cur];
    const size_t base = size_t(tile - span.first_tile) * kTile;
    const uint32_t valid = uint32_t(min(size_t(kTile), size_t(span.seg_len) - base));
    const Windows win = windows_of(span, tile);
    Bits* skeys = sm.keys[cur];
    V* svals = nullptr;
    if constexpr (kHasValues<V>) svals = sm.vals.v[cur];
    bool arrived = true;
    if (win.tma) {
      // (the first barrier of the tile reduces `arrived`: a block-uniform exit when the copy never completed)
      arrived = mbar_wait_bounded(&sm.bar[cur], (parity >> cur) & 1u, wc.tma_polls);
      parity ^= 1u << cur;
      skeys += win.k.shift;
      if constexpr (kHasValues<V>) svals += win.v.shift;
    } else {
      for (uint32_t i = tid; i < valid; i += BLOCK) skeys[i] = span.src[base + i];
      if constexpr (kHasValues<V>)
        for (uint32_t i = tid; i < valid; i += BLOCK) svals[i] = vspan.src[size_t(span.src - src) + base + i];
      __syncthreads();
    }
    bool aborted;
    if (valid == uint32_t(kTile)) {
      aborted = onesweep_tile<Tr, BLOCK, ITEMS, CHAINS, StatusT, MATCH, true, false>(
          sm, skeys, st, lb_cur, span, tile, valid, pass, svals, vspan, dg, wc.lookback_spins, tile != held, arrived,
          issue_next);
    } else {
      // Partial tiles are spread over all warps in the segmented sort only: the
      // plain sort has one partial tile per pass, and its kernel keeps the
      // fixed-span code it is tuned on.
      aborted = onesweep_tile<Tr, BLOCK, ITEMS, CHAINS, StatusT, MATCH, false, SEG>(
          sm, skeys, st, lb_cur, span, tile, valid, pass, svals, vspan, dg, wc.lookback_spins, tile != held, arrived,
          issue_next);
    }
    if (aborted) {
      if (tid == 0) atomicOr(&st->error, kStatusTmaTimeout);
      return;
    }
    cur ^= 1;
  }
}

// ---------------------------------------------------------------- segmented -
// Batched segmented sort: every segment [offsets[s], offsets[s+1]) of one key
// array is sorted on its own (stably), all segments in a fixed number of
// launches. Segments fall into size classes:
//   small  (2..one warp's share of a tile buffer: 1024 4-byte or 512 8-byte
//          keys)                one warp each, LSD passes in warp-private
//                               shared memory;
//   medium (..one tile of keys) one CTA each, LSD passes entirely in shared
//                               memory (load once, store once);
//   large  (more than a tile)   the onesweep pipeline over all large segments
//                               at once: per-segment histograms and bucket
//                               starts, tiles that never span segments, and a
//                               look-back that stops at the segment's first tile.
// Small and medium segments share one persistent launch.

struct SegPlanHeader {
  uint32_t counts[4];     // n_small, n_medium, n_large, large tiles
  uint32_t work_counter;  // next medium segment (one CTA each)
  uint32_t small_counter; // next small segment (one warp each)
  uint32_t pad[2];
};

// Classifies the segments (ids in segment order per class) and lays out the
// large segments' tiles. One CTA; thread t of a round classifies ITEMS
// consecutive segments, and one block scan per round (of the three class
// counts packed into one 64-bit word, 21 bits each, and the tile count) places
// them, so a round covers BLOCK x ITEMS segments.
template <int BLOCK, int ITEMS>
__global__ __launch_bounds__(BLOCK) void seg_classify_kernel(const unsigned long long* __restrict__ offsets,
                                                             uint32_t nseg, unsigned long long n, uint32_t tile,
                                                             uint32_t small_cap, uint32_t medium_cap,
                                                             SegPlanHeader* __restrict__ hdr,
                                                             uint32_t* __restrict__ small_ids,
                                                             uint32_t* __restrict__ medium_ids,
                                                             uint32_t* __restrict__ large_ids,
                                                             uint32_t* __restrict__ tile_prefix,
                                                             uint32_t* __restrict__ d_status) {
  constexpr int kWarps = BLOCK / 32;
  constexpr int kField = 21;
  static_assert(BLOCK * ITEMS < (1 << kField), "a round's class counts must fit their fields");
  constexpr unsigned long long kFieldMask = (1ull << kField) - 1;
  __shared__ unsigned long long s_cls[kWarps];
  __shared__ uint32_t s_tiles[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t cnt_small = 0, cnt_medium = 0, cnt_large = 0, tiles = 0;
  for (uint64_t base = 0; base < nseg; base += uint64_t(BLOCK) * ITEMS) {
    const uint64_t s0 = base + uint64_t(threadIdx.x) * ITEMS;
    int cls[ITEMS];
    uint32_t seg_tiles[ITEMS];
    unsigned long long packed = 0;
    uint32_t my_tiles = 0;
    unsigned long long b = s0 < nseg ? offsets[s0] : 0ull;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      unsigned long long len = 0;
      if (s0 + j < nseg) {
        const unsigned long long e = offsets[s0 + j + 1];
        if (e < b || e > n) {
          if (d_status) atomicOr(d_status, kStatusBadInput);
        } else {
          len = e - b;
        }
        b = e;
      }
      cls[j] = len <= 1 ? 0 : len <= small_cap ? 1 : len <= medium_cap ? 2 : 3;
      seg_tiles[j] = cls[j] == 3 ? uint32_t((len + tile - 1) / tile) : 0u;
      packed += cls[j] == 0 ? 0ull : 1ull << (kField * (cls[j] - 1));
      my_tiles += seg_tiles[j];
    }
    unsigned long long pin = packed;
    uint32_t tin = my_tiles;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned long long pu = __shfl_up_sync(0xFFFFFFFFu, pin, off);
      const uint32_t tu = __shfl_up_sync(0xFFFFFFFFu, tin, off);
      if (lane >= off) {
        pin += pu;
        tin += tu;
      }
    }
    if (lane == 31) {
      s_cls[warp] = pin;
      s_tiles[warp] = tin;
    }
    __syncthreads();
    if (warp == 0) {
      unsigned long long wp = lane < kWarps ? s_cls[lane] : 0ull;
      uint32_t wt = lane < kWarps ? s_tiles[lane] : 0u;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long pu = __shfl_up_sync(0xFFFFFFFFu, wp, off);
        const uint32_t tu = __shfl_up_sync(0xFFFFFFFFu, wt, off);
        if (lane >= off) {
          wp += pu;
          wt += tu;
        }
      }
      if (lane < kWarps) {
        s_cls[lane] = wp;
        s_tiles[lane] = wt;
      }
    }
    __syncthreads();
    const unsigned long long pex = (warp ? s_cls[warp - 1] : 0ull) + pin - packed;
    uint32_t xt = tiles + (warp ? s_tiles[warp - 1] : 0u) + tin - my_tiles;
    const unsigned long long ptot = s_cls[kWarps - 1];
    const uint32_t ttot = s_tiles[kWarps - 1];
    uint32_t xs = cnt_small + uint32_t(pex & kFieldMask);
    uint32_t xm = cnt_medium + uint32_t((pex >> kField) & kFieldMask);
    uint32_t xl = cnt_large + uint32_t(pex >> (2 * kField));
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t s = uint32_t(s0 + j);
      if (cls[j] == 1) small_ids[xs++] = s;
      if (cls[j] == 2) medium_ids[xm++] = s;
      if (cls[j] == 3) {
        large_ids[xl] = s;
        tile_prefix[xl] = xt;
        ++xl;
        xt += seg_tiles[j];
      }
    }
    cnt_small += uint32_t(ptot & kFieldMask);
    cnt_medium += uint32_t((ptot >> kField) & kFieldMask);
    cnt_large += uint32_t(ptot >> (2 * kField));
    tiles += ttot;
    __syncthreads();  // s_cls / s_tiles are rewritten by the next round
  }
  if (threadIdx.x == 0) {
    tile_prefix[cnt_large] = tiles;
    hdr->counts[0] = cnt_small;
    hdr->counts[1] = cnt_medium;
    hdr->counts[2] = cnt_large;
    hdr->counts[3] = tiles;
    hdr->work_counter = 0;
    hdr->small_counter = 0;
  }
}

// Sorts one small segment (len <= CAP) with one warp: LSD passes of 8-bit
// digits between two warp-private shared buffers of CAP keys; passes whose
// digit is the same for every key are skipped. Each pass counts the digits
// (shared atomics), scans the 256 counters across the lanes, then places the
// keys 32 at a time in index order: the lanes holding one digit find each
// other through a shared bit mask, take consecutive slots in lane order, and
// the highest of them advances the digit's counter (stable).
template <class Tr, uint32_t CAP>
__device__ __forceinline__ void warp_sort_small(typename Tr::Bits* __restrict__ keys, uint32_t len,
                                                typename Tr::Bits* A, typename Tr::Bits* B, uint32_t* cnt,
                                                uint32_t* mm) {
  using Bits = typename Tr::Bits;
  const int lane = threadIdx.x & 31;
  const uint32_t lmask = lanemask_lt(), lmask_gt = lanemask_gt();
  const uint32_t steps = (len + 31) / 32;
  for (uint32_t i = lane; i < len; i += 32) A[i] = keys[i];
  __syncwarp();
  for (int pass = 0; pass < Tr::kPasses; ++pass) {
#pragma unroll
    for (int q = 0; q < 8; ++q) cnt[lane * 8 + q] = 0u;
    __syncwarp();
    for (uint32_t i = lane; i < len; i += 32) atomicAdd(&cnt[Tr::Digit(A[i], pass)], 1u);
    __syncwarp();
    uint32_t c[8], local = 0;
    bool uniform = false;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      c[q] = cnt[lane * 8 + q];
      uniform |= (c[q] == len);
      local += c[q];
    }
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t run = incl - local;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      cnt[lane * 8 + q] = run;
      run += c[q];
    }
    if (__any_sync(0xffffffffu, uniform)) {
      __syncwarp();
      continue;  // identity permutation
    }
    __syncwarp();
    for (uint32_t j = 0; j < steps; ++j) {
      const uint32_t idx = j * 32 + lane;
      const bool ok = idx < len;
      const Bits k = ok ? A[idx] : Bits(0);
      const uint32_t d = ok ? Tr::Digit(k, pass) : 0u;
      uint32_t* m = mm + (j & 1) * kRadix;
      if (ok) atomicOr(&m[d], 1u << lane);
      __syncwarp();
      const uint32_t peers = ok ? m[d] : 0u;
      const uint32_t pos = ok ? cnt[d] + __popc(peers & lmask) : 0u;
      __syncwarp();
      if (ok && (peers & lmask_gt) == 0) {
        cnt[d] = pos + 1u;
        m[d] = 0u;
      }
      __syncwarp();
      if (ok && pos < CAP) B[pos] = k;
    }
    __syncwarp();
    Bits* t = A;
    A = B;
    B = t;
  }
  for (uint32_t i = lane; i < len; i += 32) keys[i] = A[i];
  __syncwarp();
}

// Keys a warp sorts alone in the segmented sort: one warp's share of a tile
// buffer (1024 4-byte or 512 8-byte keys with the default 512 x 32 / 512 x 16
// tiles).
template <class Tr>
constexpr uint32_t seg_small_cap() {
  using Shape = OnesweepShape<sizeof(typename Tr::Bits), kSegShape>;
  return uint32_t(Shape::kItems) * 32u;
}

// Medium segments first, one CTA each (grabbed through work_counter), then
// small segments, one warp each (grabbed per warp through small_counter, so a
// warp never waits for the others of its CTA).
template <class Tr, int BLOCK, int ITEMS, int MINB, int CHAINS, int MATCH>
__global__ __launch_bounds__(BLOCK, MINB) void seg_small_medium_kernel(typename Tr::Bits* __restrict__ keys,
                                                                       const unsigned long long* __restrict__ offsets,
                                                                       SegPlanHeader* __restrict__ hdr,
                                                                       const uint32_t* __restrict__ small_ids,
                                                                       const uint32_t* __restrict__ medium_ids) {
  using Bits = typename Tr::Bits;
  using Smem = OnesweepSmem<Tr, BLOCK, ITEMS, CHAINS>;
  constexpr int kWarps = BLOCK / 32;
  constexpr int kChains = Smem::kChains;
  constexpr uint32_t kCap = uint32_t(ITEMS) * 32u;
  static_assert(kWarps * kCap <= Smem::kTile, "warp buffers fit in one tile buffer");
  static_assert(CHAINS == 1, "one mask/counter region per warp");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  __shared__ uint32_t s_work;
  __shared__ Bits s_min[kWarps], s_max[kWarps];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kChains * 2 * kRadix; i += BLOCK) sm.masks[i] = 0u;
  for (int i = tid; i < kChains * kRadix; i += BLOCK) sm.ccount[i] = 0u;  // lean passes: zero on entry
  const uint32_t n_small = hdr->counts[0], n_medium = hdr->counts[1];
  for (;;) {
    __syncthreads();
    if (tid == 0) s_work = atomicAdd(&hdr->work_counter, 1u);
    __syncthreads();
    const uint32_t work = s_work;
    if (work >= n_medium) break;
    const uint32_t seg = medium_ids[work];
    const unsigned long long b = offsets[seg];
    const uint32_t len = uint32_t(offsets[seg + 1] - b);
    Bits* g = keys + b;
    // Load, with the range of the ordered keys: LSD passes over (ordered key - minimum), as many as the range's
    // bits need, with the onesweep kernel's lean ranking (each warp clears its counter rows after its scatter).
    Bits lo = ~Bits(0), hi = Bits(0);
    for (uint32_t i = tid; i < len; i += BLOCK) {
      const Bits k = g[i];
      sm.keys[0][i] = k;
      const Bits o = Tr::Ordered(k);
      lo = o < lo ? o : lo;
      hi = o > hi ? o : hi;
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      const Bits ol = __shfl_xor_sync(0xFFFFFFFFu, lo, off), oh = __shfl_xor_sync(0xFFFFFFFFu, hi, off);
      lo = ol < lo ? ol : lo;
      hi = oh > hi ? oh : hi;
    }
    if (lane == 0) {
      s_min[warp] = lo;
      s_max[warp] = hi;
    }
    __syncthreads();
    lo = s_min[0];
    hi = s_max[0];
#pragma unroll
    for (int w = 1; w < kWarps; ++w) {
      lo = s_min[w] < lo ? s_min[w] : lo;
      hi = s_max[w] > hi ? s_max[w] : hi;
    }
    const Bits range = hi - lo;  // len >= 2: lo <= hi
    int bits = 0;
    if constexpr (sizeof(Bits) == 4) {
      bits = range ? 32 - __clz(int(range)) : 0;
    } else {
      bits = range ? 64 - __clzll((long long)range) : 0;
    }
    const int passes = (bits + 7) / 8;
    const OffsetDigits<Bits> dg{lo};
    const uint32_t span = (len + BLOCK - 1) / BLOCK;  // keys per lane: every warp takes a share
    int cur = 0;
    for (int pass = 0; pass < passes; ++pass) {
      uint32_t tc;
      rank_tile<Tr, BLOCK, ITEMS, CHAINS, MATCH, false, false, true, true>(
          sm, sm.keys[cur], sm.keys[cur ^ 1], len, pass, &tc, [](uint32_t) {}, [](uint32_t) {},
          static_cast<const NoValue*>(nullptr), static_cast<NoValue*>(nullptr), dg, span);
      for (int i = lane; i < kRadix; i += 32) sm.ccount[warp * kRadix + i] = 0u;
      __syncthreads();
      cur ^= 1;
    }
    for (uint32_t i = tid; i < len; i += BLOCK) g[i] = sm.keys[cur][i];
  }
  for (;;) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(&hdr->small_counter, 1u);
    idx = __shfl_sync(0xFFFFFFFFu, idx, 0);
    if (idx >= n_small) break;
    const uint32_t seg = small_ids[idx];
    const unsigned long long b = offsets[seg];
    warp_sort_small<Tr, kCap>(keys + b, uint32_t(offsets[seg + 1] - b), sm.keys[0] + warp * kCap,
                              sm.keys[1] + warp * kCap, sm.ccount + warp * kRadix, sm.masks + warp * 2 * kRadix);
  }
}

// Per large segment and pass: digit counts (one read of the large segments),
// the span of every large tile (tile_info, for the onesweep kernels), and the
// first look-back array cleared. One CTA per SM; CTA b of G takes the
// contiguous large tiles [b T / G, (b + 1) T / G) (T large tiles in all), so
// its range crosses only a few segment boundaries. Keys are counted into
// per-lane histogram copies (the layout of radix_histogram: no bank conflicts
// whatever the digits) with 16-byte streaming loads, and the copies are folded
// into the segment's global histogram, and cleared, each time the range
// leaves a segment. The next segment's bounds are fetched while the current
// one is counted.
template <class Tr, class Dg>
__global__ __launch_bounds__(kHistBlock, 1) void seg_histogram_kernel(const typename Tr::Bits* __restrict__ keys,
                                                                   SegLarge sg, uint32_t tile,
                                                                   uint32_t* __restrict__ seg_hist,
                                                                   uint32_t* __restrict__ lb0,
                                                                   uint4* __restrict__ tile_info, Dg dg) {
  using Bits = typename Tr::Bits;
  constexpr int P = Tr::kPasses;
  constexpr int C = HistCopies<Tr>::kCopies;
  constexpr int kCounters = P * kRadix;
  constexpr int kVecsPerCounter = C / 4;  // 16-byte words holding one counter's copies
  constexpr int kRotDiv = 32 / C;         // see the fold below
  constexpr int kPerVec = 16 / int(sizeof(Bits));
  extern __shared__ __align__(16) uint32_t hist_smem[];
  uint4* const rows = reinterpret_cast<uint4*>(hist_smem);

  const uint32_t num_tiles = sg.counts[3];
  const uint32_t n_large = sg.counts[2];
  for (size_t i = size_t(blockIdx.x) * kHistBlock + threadIdx.x; i < size_t(num_tiles) * kRadix;
       i += size_t(gridDim.x) * kHistBlock)
    lb0[i] = 0u;
  const uint32_t t0 = uint32_t(uint64_t(num_tiles) * blockIdx.x / gridDim.x);
  const uint32_t t1 = uint32_t(uint64_t(num_tiles) * (blockIdx.x + 1) / gridDim.x);
  if (t0 >= t1) return;  // the whole CTA
  for (int i = threadIdx.x; i < kCounters * kVecsPerCounter; i += kHistBlock) rows[i] = make_uint4(0u, 0u, 0u, 0u);

  // The large segment holding tile t0: the largest s with tile_prefix[s] <= t0
  // (tile_prefix is strictly increasing, every large segment has two tiles or
  // more). Each round probes kHistBlock evenly spaced entries at once.
  uint32_t lo = 0, hi = n_large;
  while (hi - lo > 1) {
    const uint32_t step = (hi - lo + kHistBlock - 1) / kHistBlock;
    const uint32_t j = lo + (threadIdx.x + 1) * step;
    const uint32_t c = uint32_t(__syncthreads_count(j < hi && sg.tile_prefix[j] <= t0));
    lo += c * step;
    hi = min(hi, lo + step);
  }

  struct Seg {
    uint32_t begin, len, first, end;  // first key; keys; first tile; one past the last tile
  };
  auto seg_at = [&](uint32_t s) {
    const uint32_t id = sg.ids[s];
    const unsigned long long b = sg.offsets[id];
    return Seg{uint32_t(b), uint32_t(sg.offsets[id + 1] - b), sg.tile_prefix[s], sg.tile_prefix[s + 1]};
  };
  uint32_t* const copy = hist_smem + (threadIdx.x & (C - 1));
  auto count_key = [&](Bits k) {
#pragma unroll
    for (int p = 0; p < P; ++p) atomicAdd(copy + (p * kRadix + dg.template digit<Tr>(k, p)) * C, 1u);
  };

  uint32_t si = lo;
  Seg cur = seg_at(si);
  __syncthreads();  // copies cleared
  for (uint32_t t = t0; t < t1;) {
    const uint32_t ct1 = min(t1, cur.end);
    const Seg nxt = ct1 < t1 ? seg_at(si + 1) : cur;
    for (uint32_t x = t + threadIdx.x; x < ct1; x += kHistBlock)
      tile_info[x] = make_uint4(cur.begin, cur.len, cur.first, si);
    const uint32_t k0 = (t - cur.first) * tile;
    const uint32_t cnt = min(cur.len, (ct1 - cur.first) * tile) - k0;
    const Bits* const src = keys + cur.begin + k0;
    const uint32_t head =
        min(cnt, uint32_t(((16u - (reinterpret_cast<uintptr_t>(src) & 15u)) & 15u) / sizeof(Bits)));
    const uint32_t nvec = (cnt - head) / kPerVec;
    const uint32_t tail = head + nvec * kPerVec;
    if (threadIdx.x < head) count_key(src[threadIdx.x]);
    if (threadIdx.x < cnt - tail) count_key(src[tail + threadIdx.x]);
    const uint4* kv = reinterpret_cast<const uint4*>(src + head);
    uint32_t v = threadIdx.x;
    for (; v + (kHistUnroll - 1) * kHistBlock < nvec; v += kHistUnroll * kHistBlock) {
      uint4 q[kHistUnroll];
#pragma unroll
      for (int u = 0; u < kHistUnroll; ++u) q[u] = ld_stream_v4(kv + v + u * kHistBlock);
#pragma unroll
      for (int u = 0; u < kHistUnroll; ++u) {
        Bits k[kPerVec];
        unpack_v4<Bits>(q[u], k);
#pragma unroll
        for (int j = 0; j < kPerVec; ++j) count_key(k[j]);
      }
    }
    for (; v < nvec; v += kHistBlock) {
      Bits k[kPerVec];
      unpack_v4<Bits>(ld_stream_v4(kv + v), k);
#pragma unroll
      for (int j = 0; j < kPerVec; ++j) count_key(k[j]);
    }
    __syncthreads();
    // Fold: thread r sums counter r's C copies (kVecsPerCounter 16-byte words)
    // and clears them. The words are visited in a rotated order so that the 8
    // threads of each quarter-warp touch 8 different 16-byte bank groups.
    for (int r = threadIdx.x; r < kCounters; r += kHistBlock) {
      uint4* const row = rows + r * kVecsPerCounter;
      uint32_t sum = 0u;
#pragma unroll
      for (int q = 0; q < kVecsPerCounter; ++q) {
        const int w = (q + r / kRotDiv) & (kVecsPerCounter - 1);
        const uint4 c4 = row[w];
        row[w] = make_uint4(0u, 0u, 0u, 0u);
        sum += c4.x + c4.y + c4.z + c4.w;
      }
      if (sum) atomicAdd(&seg_hist[size_t(si) * kCounters + r], sum);
    }
    __syncthreads();
    t = ct1;
    ++si;
    cur = nxt;
  }
}

// ---------------------------------------------------------------- K7c -------
// One output tile of a stable k-way merge of 4-byte keys, sorted instead of
// merged: the tile's slice of every run (from the split matrix) is staged back
// to back in run order in shared memory, exactly as the pairwise-merge tiles
// stage it, and then sorted by LSD passes over the ordered keys minus the
// tile's smallest one. All of the tile's keys lie between the smallest slice
// head and the largest slice tail, so ceil(bits(max - min) / 8) passes order
// it (two for 16384 uniform keys out of 2^31). The passes are stable and the
// staging order is run order, so equal keys keep the merge's order (lower run
// first). Replaces the ceil(log2 k) pairwise rounds when k is large.
template <class Tr, int BLOCK, int ITEMS, int MATCH>
__global__ __launch_bounds__(BLOCK, 1) void kway_radix_tile_kernel(const typename Tr::Bits* const* __restrict__ runs,
                                                                   int k, const unsigned long long* __restrict__ splits,
                                                                   typename Tr::Bits* __restrict__ out,
                                                                   unsigned long long total, unsigned long long tile0) {
  using Bits = typename Tr::Bits;
  using u64 = unsigned long long;
  using Smem = OnesweepSmem<Tr, BLOCK, ITEMS, 1>;
  static_assert(sizeof(Bits) == 4, "4-byte keys");
  static_assert(sizeof(Smem) % 16 == 0, "run table after the sort buffers");
  constexpr uint32_t kTile = uint32_t(BLOCK) * ITEMS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const Bits** sptr = reinterpret_cast<const Bits**>(smem_raw + sizeof(Smem));  // this tile's first key of every run
  uint32_t* seg0 = reinterpret_cast<uint32_t*>(sptr + k);                        // slice offsets in the tile (k + 1)
  __shared__ uint32_t scan_tmp[BLOCK / 32 + 1];
  __shared__ uint32_t s_min, s_max;
  const int tid = threadIdx.x;
  const u64 j = tile0 + blockIdx.x;
  const u64 d0 = j * u64(kTile);
  const uint32_t cnt = uint32_t(min(u64(kTile), total - d0));
  if (tid == 0) {
    s_min = 0xFFFFFFFFu;
    s_max = 0u;
  }
  for (int i = tid; i < Smem::kChains * 2 * kRadix; i += BLOCK) sm.masks[i] = 0u;

  // Slice offsets (exclusive scan of the slice lengths) and the key range.
  const int per_thread = (k + BLOCK - 1) / BLOCK;
  uint32_t local = 0, lmin = 0xFFFFFFFFu, lmax = 0u;
  for (int i = 0; i < per_thread; ++i) {
    const int r = tid * per_thread + i;
    if (r < k) {
      const u64 s = splits[j * k + r], e = splits[(j + 1) * k + r];
      sptr[r] = runs[r] + s;
      local += uint32_t(e - s);
      if (e > s) {
        lmin = min(lmin, uint32_t(Tr::Ordered(runs[r][s])));
        lmax = max(lmax, uint32_t(Tr::Ordered(runs[r][e - 1])));
      }
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
  if (local) {
    atomicMin(&s_min, lmin);
    atomicMax(&s_max, lmax);
  }
  __syncthreads();

  // Stage the slices back to back: consecutive threads read consecutive keys;
  // every thread issues its loads before storing any, and its slice index
  // only moves forward (its keys are BLOCK apart).
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
      if (i < cnt) sm.keys[0][i] = v[t];
    }
  }
  __syncthreads();

  // Lean passes (the onesweep kernel's ranking: counters zero on entry, each
  // warp clearing its own rows after its scatter); a full tile takes the
  // fixed-span form, the last, shorter one spreads its keys over every warp.
  const uint32_t range = cnt ? s_max - s_min : 0u;
  const int passes = range == 0u ? 0 : (32 - __clz(int(range)) + 7) / 8;
  const OffsetDigits<uint32_t> dg{s_min};
  const int warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < Smem::kChains * kRadix; i += BLOCK) sm.ccount[i] = 0u;
  __syncthreads();
  int cur = 0;
  for (int pass = 0; pass < passes; ++pass) {
    uint32_t tc;
    if (cnt == kTile) {
      rank_tile<Tr, BLOCK, ITEMS, 1, MATCH, true, false, false, true>(
          sm, sm.keys[cur], sm.keys[cur ^ 1], cnt, pass, &tc, [](uint32_t) {}, [](uint32_t) {},
          static_cast<const NoValue*>(nullptr), static_cast<NoValue*>(nullptr), dg);
    } else {
      rank_tile<Tr, BLOCK, ITEMS, 1, MATCH, false, false, true, true>(
          sm, sm.keys[cur], sm.keys[cur ^ 1], cnt, pass, &tc, [](uint32_t) {}, [](uint32_t) {},
          static_cast<const NoValue*>(nullptr), static_cast<NoValue*>(nullptr), dg, (cnt + BLOCK - 1) / BLOCK);
    }
    for (int i = lane; i < kRadix; i += 32) sm.ccount[warp * kRadix + i] = 0u;
    __syncthreads();
    cur ^= 1;
  }
  Bits* o = out + d0;
  for (uint32_t i = tid; i < cnt; i += BLOCK) o[i] = sm.keys[cur][i];
}

template <int P>
__global__ __launch_bounds__(kRadix) void seg_scan_kernel(const uint32_t* __restrict__ counts,
                                                          const uint32_t* __restrict__ seg_hist,
                                                          uint32_t* __restrict__ seg_bucket) {
  __shared__ uint32_t tmp[kRadix / 32 + 1];
  const uint32_t units = counts[2] * P;
  for (uint32_t u = blockIdx.x; u < units; u += gridDim.x) {
    uint32_t total;
    const uint32_t c = seg_hist[size_t(u) * kRadix + threadIdx.x];
    seg_bucket[size_t(u) * kRadix + threadIdx.x] = block_exclusive_scan<kRadix>(c, tmp, &total);
  }
}

// ---------------------------------------------------------------- K3 --------
// Copies buf1 back into buf0 when an odd number of passes ran (the sorted data
// then sits in the ping-pong buffer); reports the sort's status word.
template <int P, typename T>
__device__ __forceinline__ void copy_back_if_odd(T* __restrict__ buf0, const T* __restrict__ buf1,
                                                 const RadixState* __restrict__ st, uint32_t n,
                                                 uint32_t* __restrict__ d_status) {
  int live = 0;
#pragma unroll
  for (int p = 0; p < P; ++p) live += (st->skip[p] == 0u) ? 1 : 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && d_status != nullptr && st->error != 0u) atomicOr(d_status, st->error);
  if ((live & 1) == 0) return;
  const size_t gtid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t gstride = size_t(gridDim.x) * blockDim.x;
  const bool aligned = ((reinterpret_cast<uintptr_t>(buf0) | reinterpret_cast<uintptr_t>(buf1)) & 15u) == 0;
  if (aligned) {
    constexpr int kPerVec = 16 / int(sizeof(T));
    const size_t nvec = n / kPerVec;
    const uint4* s = reinterpret_cast<const uint4*>(buf1);
    uint4* d = reinterpret_cast<uint4*>(buf0);
    for (size_t i = gtid; i < nvec; i += gstride) d[i] = ld_stream_v4(s + i);
    for (size_t i = nvec * kPerVec + gtid; i < n; i += gstride) buf0[i] = buf1[i];
  } else {
    for (size_t i = gtid; i < n; i += gstride) buf0[i] = buf1[i];
  }
}

template <class Tr>
__global__ __launch_bounds__(256) void radix_finalize_kernel(typename Tr::Bits* __restrict__ buf0,
                                                             const typename Tr::Bits* __restrict__ buf1,
                                                             const RadixState* __restrict__ st, uint32_t n,
                                                             uint32_t* __restrict__ d_status) {
  copy_back_if_odd<Tr::kPasses>(buf0, buf1, st, n, d_status);
}

// Key-value sort: the keys and the values go back when an odd number of passes ran.
template <class Tr, typename V>
__global__ __launch_bounds__(256) void radix_finalize_pairs_kernel(typename Tr::Bits* __restrict__ buf0,
                                                                   const typename Tr::Bits* __restrict__ buf1,
                                                                   V* __restrict__ vbuf0, const V* __restrict__ vbuf1,
                                                                   const RadixState* __restrict__ st, uint32_t n,
                                                                   uint32_t* __restrict__ d_status) {
  copy_back_if_odd<Tr::kPasses>(buf0, buf1, st, n, d_status);
  copy_back_if_odd<Tr::kPasses>(vbuf0, vbuf1, st, n, nullptr);
}

// ---------------------------------------------------------------- host ------
size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct RadixLayout {
  size_t state_off, lb0_off, lb1_off, keys_off, vals_off, total;
  size_t num_tiles, status_bytes;
};

// ---------------------------------------------------------------- variants --
// Onesweep variant (tile shape x ranking mode) per key width and size class.
// The table starts at shape 5 with ranking mode 3 everywhere, is replaced by a
// tuning file when one is found (load_default_tuning, on first use), and can be
// set or measured at run time (set_sort_variant, autotune). The
// MGS_ONESWEEP_SHAPE / MGS_RANK_MODE environment variables override the table
// for experiments.
constexpr int kDefaultRankMode = 3;
std::atomic<int> g_variant[2][kSizeClasses];  // shape * 10 + mode; 0 = not set

int env_override(const char* name, int lo, int hi) {
  const char* e = getenv(name);
  return (e && e[0] >= '0' + lo && e[0] <= '0' + hi && e[1] == 0) ? e[0] - '0' : -1;
}

}  // namespace

int size_class(size_t n) {
  if (n < (size_t(1) << 16)) return 0;
  if (n < (size_t(1) << 18)) return 1;
  if (n < (size_t(1) << 20)) return 2;
  if (n < (size_t(1) << 22)) return 3;
  if (n < (size_t(1) << 26)) return 4;
  return 5;
}

size_t size_class_sample(int c) {
  static const size_t sample[kSizeClasses] = {3u << 14, 3u << 16, 3u << 18, 3u << 20, size_t(1) << 24,
                                              size_t(1) << 28};
  return sample[c < 0 ? 0 : (c >= kSizeClasses ? kSizeClasses - 1 : c)];
}

bool valid_variant(SortVariant v) {
  return v.shape >= 0 && v.shape < kNumShapes && (v.mode == 2 || v.mode == 3);
}

void ensure_default_tuning() {
  static std::once_flag once;
  std::call_once(once, [] { load_default_tuning(); });
}

bool store_sort_variant(int key_bytes, int size_class_index, SortVariant v) {
  if ((key_bytes != 4 && key_bytes != 8) || size_class_index < 0 || size_class_index >= kSizeClasses ||
      !valid_variant(v))
    return false;
  g_variant[key_bytes == 8][size_class_index].store(v.shape * 10 + v.mode, std::memory_order_relaxed);
  return true;
}

bool set_sort_variant(int key_bytes, int size_class_index, SortVariant v) {
  ensure_default_tuning();  // the default file must not overwrite this entry later
  return store_sort_variant(key_bytes, size_class_index, v);
}

SortVariant table_variant(int key_bytes, int size_class_index) {
  ensure_default_tuning();
  const int c = size_class_index < 0 ? 0 : (size_class_index >= kSizeClasses ? kSizeClasses - 1 : size_class_index);
  const int code = g_variant[key_bytes == 8][c].load(std::memory_order_relaxed);
  return code ? SortVariant{code / 10, code % 10} : SortVariant{kDefaultShape, kDefaultRankMode};
}

SortVariant sort_variant(int key_bytes, size_t n) {
  static const int env_shape = env_override("MGS_ONESWEEP_SHAPE", 0, kNumShapes - 1);
  static const int env_mode = env_override("MGS_RANK_MODE", 2, 3);
  SortVariant v = table_variant(key_bytes, size_class(n));
  if (env_shape >= 0) v.shape = env_shape;
  if (env_mode >= 0) v.mode = env_mode;
  return v;
}

namespace {

template <int KEY_BYTES, int SHAPE>
constexpr size_t shape_tile() {
  return size_t(OnesweepShape<KEY_BYTES, SHAPE>::kBlock) * OnesweepShape<KEY_BYTES, SHAPE>::kItems;
}

// Key-value tiles: 512 threads x kItems keys, sized so that two tiles of keys
// and values fit in shared memory beside the per-warp counters and masks
// (8-byte pairs: 16 keys per thread, 12-byte pairs: 12, 16-byte pairs: 8).
template <int KEY_BYTES, int VALUE_BYTES>
struct PairShape {
  static constexpr int kBlock = 512;
  static constexpr int kItems = (KEY_BYTES + VALUE_BYTES == 8) ? 16 : ((KEY_BYTES + VALUE_BYTES == 12) ? 12 : 8);
  static constexpr int kMinBlocks = 1, kChains = 1;
};

template <class Tr, typename V = NoValue, class Dg = PlainDigits>
RadixLayout radix_layout(size_t n) {
  constexpr int w = int(sizeof(typename Tr::Bits));
  size_t tile;
  if constexpr (kHasValues<V>) {
    tile = size_t(PairShape<w, int(sizeof(V))>::kBlock) * PairShape<w, int(sizeof(V))>::kItems;
  } else if constexpr (!std::is_same<Dg, PlainDigits>::value) {
    tile = shape_tile<w, kDefaultShape>();  // range sorts run the default shape
  } else {
    constexpr size_t tiles[kNumShapes] = {shape_tile<w, 0>(), shape_tile<w, 1>(), shape_tile<w, 2>(),
                                           shape_tile<w, 3>(), shape_tile<w, 4>(), shape_tile<w, 5>(),
                                           shape_tile<w, 6>()};
    tile = tiles[sort_variant(w, n).shape];
  }
  // The look-back arrays are sized for the smallest tile, so every shape (and the key-value tiles) fits.
  constexpr size_t min_tile = shape_tile<w, 1>();
  RadixLayout L;
  L.num_tiles = (n + tile - 1) / tile;
  L.status_bytes = (n < (size_t(1) << 31)) ? 4 : 8;
  const size_t lb_bytes = ((n + min_tile - 1) / min_tile) * kRadix * L.status_bytes;
  L.state_off = 0;
  L.lb0_off = align_up(sizeof(RadixState), 256);
  L.lb1_off = L.lb0_off + align_up(lb_bytes, 256);
  L.keys_off = L.lb1_off + align_up(lb_bytes, 256);
  L.total = L.keys_off + align_up(n * sizeof(typename Tr::Bits), 256);
  L.vals_off = 0;
  if constexpr (kHasValues<V>) {
    L.vals_off = L.total;
    L.total += align_up(n * sizeof(V), 256);
  }
  return L;
}

int device_sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

template <class Tr, int SHAPE, typename StatusT, int MATCH, class Dg = PlainDigits>
cudaError_t launch_onesweep_passes(typename Tr::Bits* keys, typename Tr::Bits* tmp, RadixState* st, char* tbase,
                                   const RadixLayout& L, uint32_t n, bool use_tma, cudaStream_t stream,
                                   LaunchRecorder* rec, Dg dg = Dg{}) {
  using Shape = OnesweepShape<sizeof(typename Tr::Bits), SHAPE>;
  using Smem = OnesweepSmem<Tr, Shape::kBlock, Shape::kItems, Shape::kChains>;
  auto kernel = radix_onesweep_kernel<Tr, Shape::kBlock, Shape::kItems, Shape::kMinBlocks, Shape::kChains, StatusT,
                                      MATCH, false, NoValue, Dg>;
  static SmemLimitOnce attr;
  cudaError_t e = attr.ensure(kernel, sizeof(Smem));
  if (e != cudaSuccess) return e;
  static std::once_flag once;
  static int ctas_per_sm = 1;
  std::call_once(once, [&] {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, Shape::kBlock, sizeof(Smem)) == cudaSuccess &&
        occ > 0)
      ctas_per_sm = occ;
  });
  const size_t grid = std::min<size_t>(L.num_tiles, size_t(device_sm_count()) * ctas_per_sm);
  StatusT* lb[2] = {reinterpret_cast<StatusT*>(tbase + L.lb0_off), reinterpret_cast<StatusT*>(tbase + L.lb1_off)};
  for (int p = 0; p < Tr::kPasses; ++p) {
    StatusT* cur = lb[p & 1];
    StatusT* next = (p + 1 < Tr::kPasses) ? lb[(p + 1) & 1] : nullptr;
    e = launch_kernel(rec, "radix_onesweep", kernel, dim3(unsigned(grid)), dim3(Shape::kBlock), sizeof(Smem), stream,
                      keys, tmp, st, cur, next, n, uint32_t(L.num_tiles), p, use_tma ? 1 : 0, SegLarge{},
                      static_cast<NoValue*>(nullptr), static_cast<NoValue*>(nullptr), dg);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <class Tr, typename StatusT>
cudaError_t launch_onesweep_variant(typename Tr::Bits* keys, typename Tr::Bits* tmp, RadixState* st, char* tbase,
                                    const RadixLayout& L, uint32_t n, bool use_tma, cudaStream_t stream,
                                    LaunchRecorder* rec) {
#define MGS_LAUNCH(S, M) launch_onesweep_passes<Tr, S, StatusT, M>(keys, tmp, st, tbase, L, n, use_tma, stream, rec)
#define MGS_SHAPES(M)                \
  switch (v.shape) {                 \
    case 0: return MGS_LAUNCH(0, M); \
    case 1: return MGS_LAUNCH(1, M); \
    case 2: return MGS_LAUNCH(2, M); \
    case 3: return MGS_LAUNCH(3, M); \
    case 4: return MGS_LAUNCH(4, M); \
    case 6: return MGS_LAUNCH(6, M); \
    default: return MGS_LAUNCH(5, M); \
  }
  // The same choice as radix_layout made for this n (the table is read once per sort there and here;
  // set_sort_variant must not run while sorts are being issued).
  const SortVariant v = sort_variant(int(sizeof(typename Tr::Bits)), n);
  if (v.mode == 2) MGS_SHAPES(2)
  MGS_SHAPES(3)
#undef MGS_SHAPES
#undef MGS_LAUNCH
}

// Key-value passes: one fixed tile shape per (key, value) width and ranking mode 3.
template <class Tr, typename V, typename StatusT, class Dg>
cudaError_t launch_onesweep_pairs(typename Tr::Bits* keys, typename Tr::Bits* tmp, V* vals, V* vtmp, RadixState* st,
                                  char* tbase, const RadixLayout& L, uint32_t n, bool use_tma, cudaStream_t stream,
                                  LaunchRecorder* rec, Dg dg) {
  using Shape = PairShape<int(sizeof(typename Tr::Bits)), int(sizeof(V))>;
  using Smem = OnesweepSmem<Tr, Shape::kBlock, Shape::kItems, Shape::kChains, V>;
  auto kernel = radix_onesweep_kernel<Tr, Shape::kBlock, Shape::kItems, Shape::kMinBlocks, Shape::kChains, StatusT,
                                      3, false, V, Dg>;
  static SmemLimitOnce attr;
  cudaError_t e = attr.ensure(kernel, sizeof(Smem));
  if (e != cudaSuccess) return e;
  const size_t grid = std::min<size_t>(L.num_tiles, size_t(device_sm_count()));
  StatusT* lb[2] = {reinterpret_cast<StatusT*>(tbase + L.lb0_off), reinterpret_cast<StatusT*>(tbase + L.lb1_off)};
  for (int p = 0; p < Tr::kPasses; ++p) {
    StatusT* cur = lb[p & 1];
    StatusT* next = (p + 1 < Tr::kPasses) ? lb[(p + 1) & 1] : nullptr;
    e = launch_kernel(rec, "radix_onesweep_pairs", kernel, dim3(unsigned(grid)), dim3(Shape::kBlock), sizeof(Smem),
                      stream, keys, tmp, st, cur, next, n, uint32_t(L.num_tiles), p, use_tma ? 1 : 0, SegLarge{}, vals,
                      vtmp, dg);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Sorts keys (and, with a value type V, the values beside them) in place.
template <class Tr, typename V = NoValue, class Dg = PlainDigits>
cudaError_t radix_sort_impl(typename Tr::Bits* keys, V* vals, size_t n, void* temp, size_t temp_bytes,
                            cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec, Dg dg = Dg{}) {
  using Bits = typename Tr::Bits;
  if (n == 0) return cudaSuccess;
  if (n >= (size_t(1) << 32)) return cudaErrorInvalidValue;
  const RadixLayout L = radix_layout<Tr, V, Dg>(n);
  if (temp == nullptr || temp_bytes < L.total) return cudaErrorInvalidValue;
  char* tb = static_cast<char*>(temp);
  RadixState* st = reinterpret_cast<RadixState*>(tb + L.state_off);
  Bits* tmp = reinterpret_cast<Bits*>(tb + L.keys_off);
  const uint32_t n32 = uint32_t(n);
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(RadixState), stream);
  if (e != cudaSuccess) return e;

  const int sms = device_sm_count();
  const size_t vecs = n * sizeof(Bits) / 16 + 1;
  const size_t want = (vecs + size_t(kHistBlock) * kHistUnroll - 1) / (size_t(kHistBlock) * kHistUnroll);
  const unsigned hist_grid = unsigned(std::max<size_t>(1, std::min<size_t>(size_t(sms), want)));
  const size_t lb0_vecs = L.num_tiles * kRadix * L.status_bytes / 16;
  static SmemLimitOnce hist_attr;
  e = hist_attr.ensure(radix_histogram_kernel<Tr, Dg>, HistCopies<Tr>::kSmemBytes);
  if (e != cudaSuccess) return e;
  e = launch_kernel(rec, "radix_histogram", radix_histogram_kernel<Tr, Dg>, dim3(hist_grid), dim3(kHistBlock),
                    HistCopies<Tr>::kSmemBytes, stream, keys, n32, st, reinterpret_cast<uint4*>(tb + L.lb0_off),
                    lb0_vecs, dg);
  if (e != cudaSuccess) return e;
  e = launch_kernel(rec, "radix_scan", radix_scan_kernel, dim3(Tr::kPasses), dim3(kRadix), 0, stream, st, n32);
  if (e != cudaSuccess) return e;

  const unsigned fin_grid = unsigned(std::max<size_t>(1, std::min<size_t>(size_t(sms) * 8, (n + 1023) / 1024)));
  if constexpr (kHasValues<V>) {
    V* vtmp = reinterpret_cast<V*>(tb + L.vals_off);
    const bool use_tma = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals)) & 15u) == 0;
    if (L.status_bytes == 4) {
      e = launch_onesweep_pairs<Tr, V, uint32_t>(keys, tmp, vals, vtmp, st, tb, L, n32, use_tma, stream, rec, dg);
    } else {
      e = launch_onesweep_pairs<Tr, V, unsigned long long>(keys, tmp, vals, vtmp, st, tb, L, n32, use_tma, stream,
                                                           rec, dg);
    }
    if (e != cudaSuccess) return e;
    return launch_kernel(rec, "radix_finalize", radix_finalize_pairs_kernel<Tr, V>, dim3(fin_grid), dim3(256), 0,
                         stream, keys, static_cast<const typename Tr::Bits*>(tmp), vals, static_cast<const V*>(vtmp),
                         static_cast<const RadixState*>(st), n32, d_status);
  } else {
    (void)vals;
    const bool use_tma = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
    if constexpr (!std::is_same<Dg, PlainDigits>::value) {
      if (L.status_bytes == 4) {
        e = launch_onesweep_passes<Tr, kDefaultShape, uint32_t, 3, Dg>(keys, tmp, st, tb, L, n32, use_tma, stream,
                                                                       rec, dg);
      } else {
        e = launch_onesweep_passes<Tr, kDefaultShape, unsigned long long, 3, Dg>(keys, tmp, st, tb, L, n32, use_tma,
                                                                                 stream, rec, dg);
      }
    } else if (L.status_bytes == 4) {
      e = launch_onesweep_variant<Tr, uint32_t>(keys, tmp, st, tb, L, n32, use_tma, stream, rec);
    } else {
      e = launch_onesweep_variant<Tr, unsigned long long>(keys, tmp, st, tb, L, n32, use_tma, stream, rec);
    }
    if (e != cudaSuccess) return e;
    return launch_kernel(rec, "radix_finalize", radix_finalize_kernel<Tr>, dim3(fin_grid), dim3(256), 0, stream, keys,
                         tmp, st, n32, d_status);
  }
}

template <class Tr>
cudaError_t radix_sort_typed(typename Tr::Bits* keys, size_t n, void* temp, size_t temp_bytes, cudaStream_t stream,
                             uint32_t* d_status, LaunchRecorder* rec) {
  return radix_sort_impl<Tr, NoValue>(keys, static_cast<NoValue*>(nullptr), n, temp, temp_bytes, stream, d_status,
                                      rec);
}

// ---------------------------------------------------------------- segmented host
struct SegLayout {
  size_t state_off, hdr_off, small_off, medium_off, large_off, prefix_off, hist_off, bucket_off, lb0_off, lb1_off,
      tile_info_off, keys_off, total;
  size_t max_large, max_tiles, hist_bytes;
};

template <class Tr>
SegLayout seg_layout(size_t n, size_t nseg) {
  constexpr int w = int(sizeof(typename Tr::Bits));
  constexpr size_t tile = shape_tile<w, kSegShape>();
  SegLayout L;
  L.max_large = std::min(nseg, n / (tile + 1) + 1);
  L.max_tiles = n / tile + L.max_large + 1;
  L.hist_bytes = L.max_large * Tr::kPasses * kRadix * 4;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align_up(bytes, 256);
    return at;
  };
  L.state_off = take(sizeof(RadixState));
  L.hdr_off = take(sizeof(SegPlanHeader));
  L.small_off = take(nseg * 4);
  L.medium_off = take(nseg * 4);
  L.large_off = take(nseg * 4);
  L.prefix_off = take((nseg + 1) * 4);
  L.hist_off = take(L.hist_bytes);
  L.bucket_off = take(L.hist_bytes);
  L.lb0_off = take(L.max_tiles * kRadix * 4);
  L.lb1_off = take(L.max_tiles * kRadix * 4);
  L.tile_info_off = take(L.max_tiles * 16);
  L.keys_off = take(n * sizeof(typename Tr::Bits));
  L.total = off;
  return L;
}

template <class Tr>
cudaError_t segmented_sort_typed(typename Tr::Bits* keys, size_t n, const uint64_t* d_offsets, size_t nseg,
                                 void* temp, size_t temp_bytes, cudaStream_t stream, uint32_t* d_status,
                                 LaunchRecorder* rec) {
  using Bits = typename Tr::Bits;
  using Shape = OnesweepShape<sizeof(Bits), kSegShape>;
  using Smem = OnesweepSmem<Tr, Shape::kBlock, Shape::kItems, Shape::kChains>;
  constexpr uint32_t kTile = uint32_t(shape_tile<int(sizeof(Bits)), kSegShape>());
  if (n == 0 || nseg == 0) return cudaSuccess;
  if (n >= (size_t(1) << 32) || nseg >= (size_t(1) << 32) - 1) return cudaErrorInvalidValue;
  const SegLayout L = seg_layout<Tr>(n, nseg);
  if (temp == nullptr || temp_bytes < L.total) return cudaErrorInvalidValue;
  char* tb = static_cast<char*>(temp);
  RadixState* st = reinterpret_cast<RadixState*>(tb + L.state_off);
  SegPlanHeader* hdr = reinterpret_cast<SegPlanHeader*>(tb + L.hdr_off);
  uint32_t* small_ids = reinterpret_cast<uint32_t*>(tb + L.small_off);
  uint32_t* medium_ids = reinterpret_cast<uint32_t*>(tb + L.medium_off);
  uint32_t* large_ids = reinterpret_cast<uint32_t*>(tb + L.large_off);
  uint32_t* prefix = reinterpret_cast<uint32_t*>(tb + L.prefix_off);
  uint32_t* hist = reinterpret_cast<uint32_t*>(tb + L.hist_off);
  uint32_t* bucket = reinterpret_cast<uint32_t*>(tb + L.bucket_off);
  uint32_t* lb[2] = {reinterpret_cast<uint32_t*>(tb + L.lb0_off), reinterpret_cast<uint32_t*>(tb + L.lb1_off)};
  uint4* tile_info = reinterpret_cast<uint4*>(tb + L.tile_info_off);
  Bits* tmp = reinterpret_cast<Bits*>(tb + L.keys_off);
  const unsigned long long* offs = reinterpret_cast<const unsigned long long*>(d_offsets);

  cudaError_t e = cudaMemsetAsync(tb, 0, L.small_off, stream);  // RadixState + plan header
  if (e == cudaSuccess && L.hist_bytes) e = cudaMemsetAsync(hist, 0, L.hist_bytes, stream);
  if (e != cudaSuccess) return e;
  e = launch_kernel(rec, "seg_classify", seg_classify_kernel<1024, 8>, dim3(1), dim3(1024), 0, stream, offs,
                    uint32_t(nseg), (unsigned long long)n, kTile, seg_small_cap<Tr>(), kTile, hdr, small_ids,
                    medium_ids, large_ids, prefix, d_status);
  if (e != cudaSuccess) return e;

  const int sms = device_sm_count();
  {
    auto kernel = seg_small_medium_kernel<Tr, Shape::kBlock, Shape::kItems, Shape::kMinBlocks, Shape::kChains, 3>;
    static SmemLimitOnce attr;
    e = attr.ensure(kernel, sizeof(Smem));
    if (e != cudaSuccess) return e;
    e = launch_kernel(rec, "seg_small_medium", kernel, dim3(unsigned(sms)), dim3(Shape::kBlock), sizeof(Smem),
                      stream, keys, offs, hdr, static_cast<const uint32_t*>(small_ids),
                      static_cast<const uint32_t*>(medium_ids));
    if (e != cudaSuccess) return e;
  }
  SegLarge sg{offs, large_ids, prefix, hdr->counts, bucket, tile_info};
  {
    auto kernel = seg_histogram_kernel<Tr, PlainDigits>;
    static SmemLimitOnce attr;
    e = attr.ensure(kernel, HistCopies<Tr>::kSmemBytes);
    if (e != cudaSuccess) return e;
    e = launch_kernel(rec, "seg_histogram", kernel, dim3(unsigned(sms)), dim3(kHistBlock), HistCopies<Tr>::kSmemBytes,
                      stream, static_cast<const Bits*>(keys), sg, kTile, hist, lb[0], tile_info, PlainDigits{});
    if (e != cudaSuccess) return e;
  }
  e = launch_kernel(rec, "seg_scan", seg_scan_kernel<Tr::kPasses>, dim3(unsigned(sms * 4)), dim3(kRadix), 0, stream,
                    static_cast<const uint32_t*>(hdr->counts), static_cast<const uint32_t*>(hist), bucket);
  if (e != cudaSuccess) return e;
  {
    auto kernel = radix_onesweep_kernel<Tr, Shape::kBlock, Shape::kItems, Shape::kMinBlocks, Shape::kChains,
                                        uint32_t, 3, true>;
    static SmemLimitOnce attr;
    e = attr.ensure(kernel, sizeof(Smem));
    if (e != cudaSuccess) return e;
    for (int p = 0; p < Tr::kPasses; ++p) {
      uint32_t* next = (p + 1 < Tr::kPasses) ? lb[(p + 1) & 1] : nullptr;
      e = launch_kernel(rec, "seg_onesweep", kernel, dim3(unsigned(sms)), dim3(Shape::kBlock), sizeof(Smem), stream,
                        keys, tmp, st, lb[p & 1], next, uint32_t(n), 0u, p, 1, sg, static_cast<NoValue*>(nullptr),
                        static_cast<NoValue*>(nullptr), PlainDigits{});
      if (e != cudaSuccess) return e;
    }
  }
  // Passes are never skipped here (an even number ran): only the status report.
  return launch_kernel(rec, "radix_finalize", radix_finalize_kernel<Tr>, dim3(1), dim3(256), 0, stream, keys,
                       static_cast<const Bits*>(tmp), static_cast<const RadixState*>(st), 0u, d_status);
}

}  // namespace

size_t kway_radix_tile_keys(int dtype) {
  size_t keys = 0;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    if constexpr (sizeof(typename Tr::Bits) == 4) keys = shape_tile<4, kDefaultShape>();
  });
  return keys;
}

cudaError_t kway_radix_tiles(int dtype, const void* d_runs, int k, const uint64_t* d_splits, void* out,
                             uint64_t total, uint64_t tile0, uint64_t tiles, cudaStream_t stream,
                             LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  if (k < 1 || k > kMaxKwayTileRuns || tiles == 0 || tiles > 0x7FFFFFFFull) return result;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    using Bits = typename Tr::Bits;
    if constexpr (sizeof(Bits) == 4) {
      using Shape = OnesweepShape<4, kDefaultShape>;
      using Smem = OnesweepSmem<Tr, Shape::kBlock, Shape::kItems, 1>;
      auto kernel = kway_radix_tile_kernel<Tr, Shape::kBlock, Shape::kItems, 3>;
      static SmemLimitOnce attr;
      result = attr.ensure(kernel, sizeof(Smem) + size_t(kMaxKwayTileRuns) * 12 + 4);
      if (result != cudaSuccess) return;
      result = launch_kernel(rec, "kway_radix_tiles", kernel, dim3(unsigned(tiles)), dim3(Shape::kBlock),
                             sizeof(Smem) + size_t(k) * 12 + 4, stream, static_cast<const Bits* const*>(d_runs), k,
                             reinterpret_cast<const unsigned long long*>(d_splits), static_cast<Bits*>(out),
                             (unsigned long long)total, (unsigned long long)tile0);
    }
  });
  return result;
}

cudaError_t set_wait_control(uint32_t lookback_spins, uint32_t tma_polls, uint32_t hold_tile) {
  const WaitControl wc{lookback_spins ? lookback_spins : kLookbackSpinLimit, tma_polls ? tma_polls : kTmaWaitLimit,
                       hold_tile, 0u};
  return cudaMemcpyToSymbol(g_wait_control, &wc, sizeof(wc));
}

size_t radix_sort_temp_bytes(int dtype, size_t n) {
  size_t bytes = 0;
  dispatch_dtype(dtype, [&](auto tr) { bytes = radix_layout<decltype(tr)>(n).total; });
  return bytes;
}

size_t radix_sort_pairs_temp_bytes(int dtype, size_t value_bytes, size_t n) {
  size_t bytes = 0;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    if (value_bytes == 4) bytes = radix_layout<Tr, uint32_t>(n).total;
    if (value_bytes == 8) bytes = radix_layout<Tr, unsigned long long>(n).total;
  });
  return bytes;
}

cudaError_t radix_sort_pairs(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n, void* d_temp,
                             size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec) {
  if (value_bytes != 4 && value_bytes != 8) return cudaErrorInvalidValue;
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    using Bits = typename Tr::Bits;
    if (value_bytes == 4) {
      result = radix_sort_impl<Tr, uint32_t>(static_cast<Bits*>(d_keys), static_cast<uint32_t*>(d_values), n, d_temp,
                                             temp_bytes, stream, d_status, rec);
    } else {
      result = radix_sort_impl<Tr, unsigned long long>(static_cast<Bits*>(d_keys),
                                                       static_cast<unsigned long long*>(d_values), n, d_temp,
                                                       temp_bytes, stream, d_status, rec);
    }
  });
  return result;
}

namespace {
template <typename V>
__global__ void iota_kernel(V* __restrict__ out, size_t n) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = V(i);
}
}  // namespace

cudaError_t radix_sort_range(int dtype, void* d_keys, void* d_values, size_t value_bytes, size_t n, int begin_bit,
                             int end_bit, int descending, void* d_temp, size_t temp_bytes, cudaStream_t stream,
                             uint32_t* d_status, LaunchRecorder* rec) {
  if (value_bytes != 0 && value_bytes != 4 && value_bytes != 8) return cudaErrorInvalidValue;
  const RangeDigits dg{begin_bit, end_bit, descending ? 1 : 0};
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    using Bits = typename Tr::Bits;
    if (begin_bit < 0 || end_bit > Tr::kBits || begin_bit > end_bit) return;
    Bits* k = static_cast<Bits*>(d_keys);
    if (value_bytes == 0) {
      result = radix_sort_impl<Tr, NoValue, RangeDigits>(k, static_cast<NoValue*>(nullptr), n, d_temp, temp_bytes,
                                                         stream, d_status, rec, dg);
    } else if (value_bytes == 4) {
      result = radix_sort_impl<Tr, uint32_t, RangeDigits>(k, static_cast<uint32_t*>(d_values), n, d_temp,
                                                          temp_bytes, stream, d_status, rec, dg);
    } else {
      result = radix_sort_impl<Tr, unsigned long long, RangeDigits>(
          k, static_cast<unsigned long long*>(d_values), n, d_temp, temp_bytes, stream, d_status, rec, dg);
    }
  });
  return result;
}

cudaError_t radix_argsort(int dtype, void* d_keys, void* d_indices, size_t index_bytes, size_t n, void* d_temp,
                          size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec) {
  if (index_bytes != 4 && index_bytes != 8) return cudaErrorInvalidValue;
  if (n == 0) return cudaSuccess;
  const unsigned grid = unsigned(std::max<size_t>(1, std::min<size_t>(size_t(device_sm_count()) * 8, (n + 255) / 256)));
  cudaError_t e = index_bytes == 4
                      ? launch_kernel(rec, "iota", iota_kernel<uint32_t>, dim3(grid), dim3(256), 0, stream,
                                      static_cast<uint32_t*>(d_indices), n)
                      : launch_kernel(rec, "iota", iota_kernel<unsigned long long>, dim3(grid), dim3(256), 0, stream,
                                      static_cast<unsigned long long*>(d_indices), n);
  if (e != cudaSuccess) return e;
  return radix_sort_pairs(dtype, d_keys, d_indices, index_bytes, n, d_temp, temp_bytes, stream, d_status, rec);
}

int radix_sort_launches(int dtype, size_t n) {
  if (n == 0) return 0;
  const size_t w = dtype_bytes(dtype);
  return int(3 + w);  // histogram + scan + one onesweep per 8-bit digit + finalize
}

size_t segmented_sort_temp_bytes(int dtype, size_t n, size_t num_segments) {
  size_t bytes = 0;
  dispatch_dtype(dtype, [&](auto tr) { bytes = seg_layout<decltype(tr)>(n, num_segments).total; });
  return bytes;
}

cudaError_t segmented_sort(int dtype, void* d_keys, size_t n, const uint64_t* d_offsets, size_t num_segments,
                           void* d_temp, size_t temp_bytes, cudaStream_t stream, uint32_t* d_status,
                           LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    result = segmented_sort_typed<Tr>(static_cast<typename Tr::Bits*>(d_keys), n, d_offsets, num_segments, d_temp,
                                      temp_bytes, stream, d_status, rec);
  });
  return result;
}

cudaError_t radix_sort(int dtype, void* d_keys, size_t n, void* d_temp, size_t temp_bytes, cudaStream_t stream,
                       uint32_t* d_status, LaunchRecorder* rec) {
  cudaError_t result = cudaErrorInvalidValue;
  dispatch_dtype(dtype, [&](auto tr) {
    using Tr = decltype(tr);
    result = radix_sort_typed<Tr>(static_cast<typename Tr::Bits*>(d_keys), n, d_temp, temp_bytes, stream, d_status,
                                  rec);
  });
  return result;
}

}  // namespace mgs
