// Device input generator (see generate.cuh). Each distribution is the host
// generator's own arithmetic, restated so that every rounding step is the same:
//
// * mt19937 streams (reference "uniform", "sorted", "reverse-sorted",
//   "staggered", "bucket-sorted"; src/data_generator.cuh:40-191): the host runs
//   128 logical threads, each with its own std::mt19937 over a contiguous index
//   block. Here every logical thread is one warp holding the engine state in
//   shared memory. A twist regenerates the 624 words in chunks of 32 (the
//   recurrence of word k reads words k, k+1 and k+397 mod 624; a chunk reads
//   before it writes, so each read sees the value the sequential order sees);
//   then each lane tempers two words into one double exactly as
//   std::generate_canonical<double, 53> does (low word + high word * 2^32,
//   rounded once, scaled by 2^-64, clamped below 1) and applies
//   uniform_real_distribution's (u * (b - a)) + a with separately rounded
//   operations (no fused multiply-add). The initial states come from the host
//   engine itself (mt19937_seed_state).
// * counter-based distributions ("full-uniform", "zipf", "-specials", "all-equal"):
//   SplitMix64 of (seed, stream, index), the same integer arithmetic; the Zipf
//   CDF and rank keys are the host's tables, searched with a guide table that
//   only narrows the same lower_bound.
// * sorted forms: the engine's own radix sort (ascending, or descending by the
//   bit-range sort) and, for "bucket-sorted", its segmented sort. The keys of
//   these distributions hold no -0.0 and no NaN, so any correct sort gives the
//   host's bytes.
// * "nearly-sorted-swaps": the host applies n/100 random transpositions one
//   after another. Here every transposition j adds the events (a_j, j -> b_j)
//   and (b_j, j -> a_j); sorting the events by (position, j) lets each touched
//   position walk back through the swaps that moved its final key (latest
//   earlier swap of the current position, then its partner, ...) to the
//   position the key started from; a gather then a scatter apply the result.
#include <algorithm>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#include "../host/data_generator.h"
#include "engine_types.h"
#include "generate.cuh"
#include "radix_sort.cuh"

namespace mgs {
namespace {

// ------------------------------------------------------------- mt19937 ------
constexpr int kMtN = 624;
constexpr int kMtM = 397;
constexpr uint32_t kMtMatrixA = 0x9908B0DFu;
constexpr uint32_t kMtUpper = 0x80000000u;
constexpr uint32_t kMtLower = 0x7FFFFFFFu;
constexpr int kStreamWarpThreads = 32;

// One logical generator thread: its engine state and where its values go. A
// stream's values fill seg 0 then seg 1; with range_draw the first value sets
// the bounds of the rest (one staggered bucket).
struct MtStream {
  unsigned long long dst[2];
  unsigned long long len[2];
  uint32_t state;       // index of the stream's 624-word initial state
  uint32_t range_draw;  // 0 or 1
};

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9D2C5680u;
  y ^= (y << 15) & 0xEFC60000u;
  y ^= y >> 18;
  return y;
}

// std::generate_canonical<double, 53> over a 32-bit engine: two draws.
__device__ __forceinline__ double mt_canonical(uint32_t lo, uint32_t hi) {
  const double sum = __dadd_rn(static_cast<double>(lo), __dmul_rn(static_cast<double>(hi), 4294967296.0));
  double r = __dmul_rn(sum, 0x1p-64);  // / 2^64, exact
  if (r >= 1.0) r = 0x1.fffffffffffffp-1;  // nextafter(1, 0)
  return r;
}

// uniform_real_distribution<double>(a, b): (u * (b - a)) + a.
__device__ __forceinline__ double uniform_ab(double u, double a, double b) {
  return __dadd_rn(__dmul_rn(u, __dsub_rn(b, a)), a);
}

// Bounds of one staggered bucket from its first draw, with the host's
// expressions and types (src/data_generator.cuh:95-101).
template <typename T>
__device__ __forceinline__ void staggered_bounds(double draw, double* a, double* b) {
  const size_t num_buckets = 10;
  T upper = static_cast<T>(draw);
  T lower = num_buckets > upper ? 0 : upper - num_buckets;
  *a = static_cast<double>(lower);
  *b = static_cast<double>(upper);
}

template <typename T>
__global__ __launch_bounds__(kStreamWarpThreads) void mt_streams_kernel(T* __restrict__ out,
                                                                         const MtStream* __restrict__ streams,
                                                                         const uint32_t* __restrict__ states,
                                                                         double a0, double b0) {
  __shared__ uint32_t x[kMtN];
  const int lane = threadIdx.x;
  const MtStream st = streams[blockIdx.x];
  for (int i = lane; i < kMtN; i += 32) x[i] = states[size_t(st.state) * kMtN + i];
  __syncwarp();
  double a = a0, b = b0;
  const unsigned long long total = st.range_draw + st.len[0] + st.len[1];
  for (unsigned long long base = 0; base < total; base += kMtN / 2) {
    for (int c = 0; c < kMtN; c += 32) {
      const int k = c + lane;
      uint32_t next = 0;
      if (k < kMtN) {
        const uint32_t y = (x[k] & kMtUpper) | (x[k + 1 < kMtN ? k + 1 : 0] & kMtLower);
        next = x[k + kMtM < kMtN ? k + kMtM : k + kMtM - kMtN] ^ (y >> 1) ^ ((y & 1u) ? kMtMatrixA : 0u);
      }
      __syncwarp();
      if (k < kMtN) x[k] = next;
      __syncwarp();
    }
    for (int v0 = 0; v0 < kMtN / 2; v0 += 32) {
      const int v = v0 + lane;
      double u = 0.0;
      if (v < kMtN / 2) u = mt_canonical(mt_temper(x[2 * v]), mt_temper(x[2 * v + 1]));
      if (st.range_draw && base == 0 && v0 == 0) {
        const double first = __shfl_sync(0xFFFFFFFFu, u, 0);
        staggered_bounds<T>(uniform_ab(first, a0, b0), &a, &b);
      }
      const unsigned long long k = base + v;
      if (v < kMtN / 2 && k >= st.range_draw && k < total) {
        const unsigned long long j = k - st.range_draw;
        const unsigned long long pos = j < st.len[0] ? st.dst[0] + j : st.dst[1] + (j - st.len[0]);
        out[pos] = static_cast<T>(uniform_ab(u, a, b));
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------- counter-based ------
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ unsigned long long draw(uint32_t seed, unsigned long long s, unsigned long long k) {
  return splitmix64(splitmix64((static_cast<unsigned long long>(seed) << 8) ^ s) ^
                    splitmix64(k * 0xD1B54A32D192ED03ull + s));
}
__device__ __forceinline__ double unit(unsigned long long r) {
  return __dmul_rn(static_cast<double>(r >> 11), 1.0 / 9007199254740992.0);
}

template <typename T>
__device__ __forceinline__ T from_bits(unsigned long long r) {
  T v;
  if constexpr (sizeof(T) == 4) {
    const uint32_t b = static_cast<uint32_t>(r);
    memcpy(&v, &b, 4);
  } else {
    memcpy(&v, &r, 8);
  }
  return v;
}

template <typename T>
__global__ __launch_bounds__(256) void full_uniform_kernel(T* __restrict__ out, size_t n, uint32_t seed, double maxv) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long r = draw(seed, 1, i);
    if constexpr (std::numeric_limits<T>::is_integer) {
      out[i] = from_bits<T>(r);
    } else {
      out[i] = static_cast<T>(__dmul_rn(__dadd_rn(__dmul_rn(2.0, unit(r)), -1.0), maxv));
    }
  }
}

template <typename T>
__global__ __launch_bounds__(256) void fill_value_kernel(T* __restrict__ out, size_t n, T v) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = v;
}

constexpr int kZipfGuideBits = 16;
constexpr uint32_t kZipfGuide = 1u << kZipfGuideBits;

template <typename T>
__global__ __launch_bounds__(256) void zipf_kernel(T* __restrict__ out, size_t n, uint32_t seed,
                                                   const double* __restrict__ cdf, const T* __restrict__ value,
                                                   const uint32_t* __restrict__ guide, uint32_t distinct) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double u = unit(draw(seed, 3, i));
    const uint32_t g = static_cast<uint32_t>(__dmul_rn(u, double(kZipfGuide)));  // u < 1: g < kZipfGuide
    uint32_t lo = guide[g], hi = guide[g + 1];  // the first cdf >= u lies in [lo, hi]
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo) >> 1);
      if (cdf[mid] < u) {
        lo = mid + 1;
      } else {
        hi = mid;
      }
    }
    out[i] = value[lo < distinct ? lo : distinct - 1];
  }
}

template <typename T>
__global__ __launch_bounds__(256) void specials_kernel(T* __restrict__ out, size_t n, uint32_t seed) {
  using U = typename std::conditional<sizeof(T) == 4, uint32_t, unsigned long long>::type;
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long r = draw(seed, 5, i) % 1000;
    if (r > 1) continue;
    U b;
    if (r == 0) {
      b = U(1) << (sizeof(U) * 8 - 1);
    } else {
      const unsigned long long pick = draw(seed, 6, i) % 6;
      if constexpr (sizeof(U) == 4) {
        const uint32_t p4[6] = {0x7FC00000u, 0xFFC00000u, 0x7FC00001u, 0xFFC12345u, 0x7F800001u, 0xFF800002u};
        b = U(p4[pick]);
      } else {
        const unsigned long long p8[6] = {0x7FF8000000000000ull, 0xFFF8000000000000ull, 0x7FF8000000000001ull,
                                          0xFFF8000000012345ull, 0x7FF0000000000001ull, 0xFFF0000000000002ull};
        b = U(p8[pick]);
      }
    }
    memcpy(&out[i], &b, sizeof(U));
  }
}

// --------------------------------------------------------------- swaps ------
__global__ __launch_bounds__(256) void swap_events_kernel(unsigned long long* __restrict__ ev_key,
                                                          uint32_t* __restrict__ ev_other, size_t m, size_t n,
                                                          uint32_t seed) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < m; j += stride) {
    const unsigned long long a = draw(seed, 4, 2 * j) % n;
    const unsigned long long b = draw(seed, 4, 2 * j + 1) % n;
    ev_key[2 * j] = (a << 32) | j;
    ev_other[2 * j] = uint32_t(b);
    ev_key[2 * j + 1] = (b << 32) | j;
    ev_other[2 * j + 1] = uint32_t(a);
  }
}

__device__ __forceinline__ bool last_event_of_position(const unsigned long long* ev_key, size_t e, size_t ne) {
  return e + 1 == ne || (ev_key[e + 1] >> 32) != (ev_key[e] >> 32);
}

// For the last event of every touched position: the position its final key
// started at, found by walking back through the swaps; the key is gathered.
template <typename T>
__global__ __launch_bounds__(256) void swap_trace_kernel(const unsigned long long* __restrict__ ev_key,
                                                         const uint32_t* __restrict__ ev_other, size_t ne, uint32_t m,
                                                         const T* __restrict__ data, T* __restrict__ moved) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < ne; e += stride) {
    if (!last_event_of_position(ev_key, e, ne)) continue;
    unsigned long long cur = ev_key[e] >> 32;
    unsigned long long limit = m;  // swaps before this one may have moved the key
    for (;;) {                     // `limit` falls at every step: at most m steps
      const unsigned long long probe = (cur << 32) | limit;
      size_t lo = 0, hi = ne;
      while (lo < hi) {
        const size_t mid = lo + ((hi - lo) >> 1);
        if (ev_key[mid] < probe) {
          lo = mid + 1;
        } else {
          hi = mid;
        }
      }
      if (lo == 0 || (ev_key[lo - 1] >> 32) != cur) break;
      limit = ev_key[lo - 1] & 0xFFFFFFFFull;
      cur = ev_other[lo - 1];
    }
    moved[e] = data[cur];
  }
}

template <typename T>
__global__ __launch_bounds__(256) void swap_scatter_kernel(const unsigned long long* __restrict__ ev_key, size_t ne,
                                                           const T* __restrict__ moved, T* __restrict__ data) {
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < ne; e += stride)
    if (last_event_of_position(ev_key, e, ne)) data[ev_key[e] >> 32] = moved[e];
}

// ---------------------------------------------------------------- host ------
enum class Dist {
  kZero,
  kUniform,
  kSorted,
  kReverseSorted,
  kStaggered,
  kBucketSorted,
  kFullUniform,
  kZipf,
  kSortedFull,
  kReverseSortedFull,
  kNearlySortedSwaps,
  kAllEqual,
};

bool parse(int dtype, const char* distribution, Dist* d, bool* specials, std::string* why) {
  std::string s(distribution ? distribution : "");
  const std::string suffix = "-specials";
  *specials = false;
  if (s.size() > suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0) {
    if (dtype != 2 && dtype != 5) {
      *why = "the -specials suffix applies to f32 and f64 keys only";
      return false;
    }
    *specials = true;
    s.resize(s.size() - suffix.size());
  }
  static const struct {
    const char* name;
    Dist d;
  } kNames[] = {{"zero", Dist::kZero},
                {"uniform", Dist::kUniform},
                {"sorted", Dist::kSorted},
                {"reverse-sorted", Dist::kReverseSorted},
                {"staggered", Dist::kStaggered},
                {"bucket-sorted", Dist::kBucketSorted},
                {"full-uniform", Dist::kFullUniform},
                {"zipf", Dist::kZipf},
                {"sorted-full", Dist::kSortedFull},
                {"reverse-sorted-full", Dist::kReverseSortedFull},
                {"nearly-sorted-swaps", Dist::kNearlySortedSwaps},
                {"all-equal", Dist::kAllEqual}};
  for (const auto& e : kNames) {
    if (s == e.name) {
      *d = e.d;
      return true;
    }
  }
  if (s == "normal" || s == "nearly-sorted" || s == "normal0") {
    *why = "'" + s + "' draws through the host C library's log/cos, which the device does not reproduce bit for bit; "
           "use mgs_generate";
  } else {
    *why = "unknown distribution '" + s + "'";
  }
  return false;
}

constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

size_t streams_bytes() {
  return align_up(sizeof(uint32_t) * kMtN * (kGeneratorThreads + 1)) +
         align_up(sizeof(MtStream) * (kGeneratorThreads + 1));
}

size_t swaps_bytes(size_t w, size_t n) {
  const size_t ne = 2 * (n / 100);
  if (ne == 0) return 0;
  return align_up(ne * 8) + align_up(ne * 4) + align_up(ne * w) + radix_sort_pairs_temp_bytes(3, 4, ne);
}

size_t temp_bytes_for(Dist d, int dtype, size_t n) {
  const size_t w = dtype_bytes(dtype);
  switch (d) {
    case Dist::kZero:
    case Dist::kFullUniform:
    case Dist::kAllEqual:
      return 0;
    case Dist::kUniform:
    case Dist::kStaggered:
      return streams_bytes();
    case Dist::kSorted:
    case Dist::kReverseSorted:
      return std::max(streams_bytes(), radix_sort_temp_bytes(dtype, n));
    case Dist::kBucketSorted:
      return std::max(streams_bytes(), align_up(12 * sizeof(uint64_t)) + segmented_sort_temp_bytes(dtype, n, 11));
    case Dist::kZipf:
      return align_up(kZipfDistinct * 8) + align_up(kZipfDistinct * w) + align_up((kZipfGuide + 1) * 4);
    case Dist::kSortedFull:
    case Dist::kReverseSortedFull:
      return radix_sort_temp_bytes(dtype, n);
    case Dist::kNearlySortedSwaps:
      return std::max(radix_sort_temp_bytes(dtype, n), swaps_bytes(w, n));
  }
  return 0;
}

unsigned grid_for(size_t n) {
  const size_t blocks = (n + 255) / 256;
  return unsigned(std::min<size_t>(blocks, 148 * 16));
}

template <typename T>
struct Generator {
  T* out;
  size_t n;
  uint32_t seed;
  char* temp;
  size_t temp_bytes;
  cudaStream_t s;
  uint32_t* d_status;
  LaunchRecorder* rec;
  int dtype;

  static double maxv() { return static_cast<double>(std::numeric_limits<T>::max()); }

  // Streams of the mt19937 distributions: states seeded with seed + logical
  // thread (or seed + 128 for the staggered tail), values placed as the host
  // loops place them.
  cudaError_t run_streams(const std::vector<MtStream>& streams) {
    if (streams.empty()) return cudaSuccess;
    std::vector<uint32_t> states(streams.size() * kMtN);
    std::vector<MtStream> table(streams);
    for (size_t i = 0; i < streams.size(); ++i) {
      if (!mt19937_seed_state(seed + streams[i].state, states.data() + i * kMtN)) return cudaErrorUnknown;
      table[i].state = uint32_t(i);
    }
    uint32_t* d_states = reinterpret_cast<uint32_t*>(temp);
    MtStream* d_table = reinterpret_cast<MtStream*>(temp + align_up(sizeof(uint32_t) * kMtN * (kGeneratorThreads + 1)));
    cudaError_t e = cudaMemcpyAsync(d_states, states.data(), states.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_table, table.data(), table.size() * sizeof(MtStream), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = launch_kernel(rec, "generate_mt_streams", mt_streams_kernel<T>, dim3(unsigned(table.size())),
                        dim3(kStreamWarpThreads), 0, s, out, d_table, d_states, 0.0, maxv());
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host vectors go out of scope
    return e;
  }

  cudaError_t uniform() {  // src/data_generator.cuh:40-52
    std::vector<MtStream> streams;
    for (int t = 0; t < kGeneratorThreads; ++t) {
      size_t b, e;
      generator_static_block(n, t, &b, &e);
      if (e > b) streams.push_back(MtStream{{b, 0}, {e - b, 0}, uint32_t(t), 0});
    }
    return run_streams(streams);
  }

  cudaError_t staggered() {  // src/data_generator.cuh:81-115
    const size_t num_buckets = 10, bucket_size = n / num_buckets;
    if (bucket_size == 0) return cudaSuccess;
    const size_t loop_n = n / bucket_size;  // at most 19
    std::vector<MtStream> streams;
    for (int t = 0; t < kGeneratorThreads; ++t) {
      size_t b, e;
      generator_static_block(loop_n, t, &b, &e);
      if (e == b) continue;
      if (e - b != 1) return cudaErrorInvalidValue;  // one bucket per logical thread
      streams.push_back(MtStream{{b * bucket_size, 0}, {bucket_size, 0}, uint32_t(t), 1});
    }
    const size_t tail = n % bucket_size;
    if (tail) streams.push_back(MtStream{{n - tail, 0}, {tail, 0}, uint32_t(kGeneratorThreads), 1});
    return run_streams(streams);
  }

  cudaError_t bucket_sorted() {  // src/data_generator.cuh:164-191
    const size_t num_buckets = 10, bucket_size = n / num_buckets;
    if (bucket_size == 0) return cudaSuccess;
    const size_t tail_begin = n - n % bucket_size;
    std::vector<MtStream> streams;
    for (int t = 0; t < kGeneratorThreads; ++t) {
      size_t b, e, tb, te;
      generator_static_block(num_buckets, t, &b, &e);
      generator_static_block(n - tail_begin, t, &tb, &te);
      if (e > b || te > tb)
        streams.push_back(MtStream{{b * bucket_size, tail_begin + tb}, {(e - b) * bucket_size, te - tb}, uint32_t(t), 0});
    }
    cudaError_t err = run_streams(streams);
    if (err != cudaSuccess) return err;
    // Buckets 0..10 (the eleventh is the remainder) sorted on their own.
    std::vector<uint64_t> offs(12);
    for (size_t i = 0; i <= num_buckets + 1; ++i) offs[i] = std::min(i * bucket_size, n);
    uint64_t* d_offs = reinterpret_cast<uint64_t*>(temp);
    err = cudaMemcpyAsync(d_offs, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) return err;
    const size_t off = align_up(12 * sizeof(uint64_t));
    return segmented_sort(dtype, out, n, d_offs, num_buckets + 1, temp + off, temp_bytes - off, s, d_status, rec);
  }

  cudaError_t full_uniform() {
    return launch_kernel(rec, "generate_full_uniform", full_uniform_kernel<T>, dim3(grid_for(n)), dim3(256), 0, s, out,
                         n, seed, maxv());
  }

  cudaError_t fill(T v) {
    return launch_kernel(rec, "generate_fill", fill_value_kernel<T>, dim3(grid_for(n)), dim3(256), 0, s, out, n, v);
  }

  cudaError_t zipf() {
    std::vector<double> cdf;
    std::vector<unsigned char> values;
    if (!zipf_tables(dtype, seed, &cdf, &values)) return cudaErrorInvalidValue;
    std::vector<uint32_t> guide(kZipfGuide + 1);
    for (uint32_t g = 0; g <= kZipfGuide; ++g)
      guide[g] = uint32_t(std::lower_bound(cdf.begin(), cdf.end(), double(g) / double(kZipfGuide)) - cdf.begin());
    double* d_cdf = reinterpret_cast<double*>(temp);
    T* d_val = reinterpret_cast<T*>(temp + align_up(kZipfDistinct * 8));
    uint32_t* d_guide = reinterpret_cast<uint32_t*>(temp + align_up(kZipfDistinct * 8) + align_up(kZipfDistinct * sizeof(T)));
    cudaError_t e = cudaMemcpyAsync(d_cdf, cdf.data(), cdf.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_val, values.data(), values.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_guide, guide.data(), guide.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = launch_kernel(rec, "generate_zipf", zipf_kernel<T>, dim3(grid_for(n)), dim3(256), 0, s, out, n, seed, d_cdf,
                        d_val, d_guide, uint32_t(kZipfDistinct));
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  }

  cudaError_t sort(bool descending) {
    if (!descending) return radix_sort(dtype, out, n, temp, temp_bytes, s, d_status, rec);
    return radix_sort_range(dtype, out, nullptr, 0, n, 0, int(8 * sizeof(T)), 1, temp, temp_bytes, s, d_status, rec);
  }

  cudaError_t swaps() {  // the host's swap_one_percent
    const size_t m = n / 100, ne = 2 * m;
    if (n < 2 || m == 0) return cudaSuccess;
    unsigned long long* ev_key = reinterpret_cast<unsigned long long*>(temp);
    uint32_t* ev_other = reinterpret_cast<uint32_t*>(temp + align_up(ne * 8));
    T* moved = reinterpret_cast<T*>(temp + align_up(ne * 8) + align_up(ne * 4));
    char* sort_temp = temp + align_up(ne * 8) + align_up(ne * 4) + align_up(ne * sizeof(T));
    const size_t sort_bytes = temp_bytes - size_t(sort_temp - temp);
    cudaError_t e = launch_kernel(rec, "generate_swap_events", swap_events_kernel, dim3(grid_for(m)), dim3(256), 0, s,
                                  ev_key, ev_other, m, n, seed);
    if (e == cudaSuccess) e = radix_sort_pairs(3, ev_key, ev_other, 4, ne, sort_temp, sort_bytes, s, d_status, rec);
    if (e == cudaSuccess)
      e = launch_kernel(rec, "generate_swap_trace", swap_trace_kernel<T>, dim3(grid_for(ne)), dim3(256), 0, s, ev_key,
                        ev_other, ne, uint32_t(m), static_cast<const T*>(out), moved);
    if (e == cudaSuccess)
      e = launch_kernel(rec, "generate_swap_scatter", swap_scatter_kernel<T>, dim3(grid_for(ne)), dim3(256), 0, s,
                        ev_key, ne, static_cast<const T*>(moved), out);
    return e;
  }

  cudaError_t specials() {
    return launch_kernel(rec, "generate_specials", specials_kernel<T>, dim3(grid_for(n)), dim3(256), 0, s, out, n, seed);
  }

  cudaError_t run(Dist d, bool with_specials) {
    cudaError_t e = cudaSuccess;
    switch (d) {
      case Dist::kZero: e = fill(T(0)); break;
      case Dist::kUniform: e = uniform(); break;
      case Dist::kSorted:
      case Dist::kReverseSorted:
        e = uniform();
        if (e == cudaSuccess) e = sort(d == Dist::kReverseSorted);
        break;
      case Dist::kStaggered: e = staggered(); break;
      case Dist::kBucketSorted: e = bucket_sorted(); break;
      case Dist::kFullUniform: e = full_uniform(); break;
      case Dist::kZipf: e = zipf(); break;
      case Dist::kSortedFull:
      case Dist::kReverseSortedFull:
      case Dist::kNearlySortedSwaps:
        e = full_uniform();
        if (e == cudaSuccess) e = sort(d == Dist::kReverseSortedFull);
        if (e == cudaSuccess && d == Dist::kNearlySortedSwaps) e = swaps();
        break;
      case Dist::kAllEqual:
        e = fill(std::numeric_limits<T>::is_integer ? static_cast<T>(0x5A) : static_cast<T>(1.5));
        break;
    }
    if (e == cudaSuccess && with_specials) e = specials();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
  }
};

template <typename T>
cudaError_t run_typed(Dist d, bool with_specials, int dtype, uint32_t seed, void* d_out, size_t n, void* d_temp,
                      size_t temp_bytes, cudaStream_t s, uint32_t* d_status, LaunchRecorder* rec) {
  Generator<T> g{static_cast<T*>(d_out), n, seed, static_cast<char*>(d_temp), temp_bytes, s, d_status, rec, dtype};
  return g.run(d, with_specials);
}

}  // namespace

bool generate_device_temp_bytes(int dtype, const char* distribution, size_t n, size_t* bytes, std::string* why) {
  Dist d;
  bool specials;
  if (dtype_bytes(dtype) == 0) {
    *why = "unknown dtype";
    return false;
  }
  if (!parse(dtype, distribution, &d, &specials, why)) return false;
  *bytes = n ? temp_bytes_for(d, dtype, n) : 0;
  return true;
}

cudaError_t generate_device(int dtype, const char* distribution, uint32_t seed, void* d_out, size_t n, void* d_temp,
                            size_t temp_bytes, cudaStream_t stream, uint32_t* d_status, LaunchRecorder* rec) {
  Dist d;
  bool specials;
  std::string why;
  if (!parse(dtype, distribution, &d, &specials, &why)) return cudaErrorInvalidValue;
  if (n == 0) return cudaSuccess;
  if (temp_bytes < temp_bytes_for(d, dtype, n)) return cudaErrorInvalidValue;
  switch (dtype) {
    case 0: return run_typed<uint32_t>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    case 1: return run_typed<int32_t>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    case 2: return run_typed<float>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    case 3: return run_typed<uint64_t>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    case 4: return run_typed<int64_t>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    case 5: return run_typed<double>(d, specials, dtype, seed, d_out, n, d_temp, temp_bytes, stream, d_status, rec);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mgs
