// Seeded input generation for the sort engine.
//
// Part 1 reproduces DataGenerator::ComputeDistribution<T> of the reference
// (src/data_generator.cuh:18-211) value for value: 128 logical generator
// threads (kNumThreads, :210), each with its own std::mt19937 seeded through
// std::seed_seq from the bit-rotated seed + thread index (:193-205), iterating
// the contiguous block of indices that OpenMP's schedule(static) gives that
// thread. The logical threads are mapped onto however many OS threads exist,
// so the output does not depend on the machine's core count.
//
// Part 2 adds the seeded distributions of the sort engine's workload sweep
// (full-range uniform, normal(0, 2^20), Zipf(1.1), 1% random swaps, all-equal,
// and -0.0 / NaN specials for floating-point keys). These use a counter-based
// generator (SplitMix64 of seed and index), so any index range can be produced
// independently and in parallel.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <parallel/algorithm>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "data_generator.h"

namespace mgs {
namespace {

// Same seeding procedure as src/data_generator.cuh:193-205: fill a seed
// sequence as long as the generator state with successive left-rotations of
// the 32-bit seed.
std::mt19937 seeded_generator(uint32_t seed) {
  const size_t seeds_bytes = sizeof(std::mt19937::result_type) * std::mt19937::state_size;
  const size_t seeds_length = seeds_bytes / sizeof(std::seed_seq::result_type);
  std::vector<std::seed_seq::result_type> seeds(seeds_length);
  for (auto& s : seeds) {
    seed = (seed << 1) | (seed >> 31);
    s = seed;
  }
  std::seed_seq sequence(seeds.begin(), seeds.end());
  return std::mt19937{sequence};
}

// Iteration block of logical thread t under OpenMP schedule(static) without a
// chunk size (libgomp: the first n % T threads get one extra iteration).
inline void static_block(size_t n, int t, size_t* begin, size_t* end) {
  const size_t q = n / kGeneratorThreads, r = n % kGeneratorThreads;
  const size_t ut = static_cast<size_t>(t);
  if (ut < r) {
    *begin = ut * (q + 1);
    *end = *begin + q + 1;
  } else {
    *begin = ut * q + r;
    *end = *begin + q;
  }
}

// Runs body(t) for each of the 128 logical generator threads.
template <typename Fn>
void for_each_logical_thread(Fn&& body) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int t = 0; t < kGeneratorThreads; ++t) body(t);
}

template <typename T>
void ref_uniform(T* out, size_t n, uint32_t seed) {
  for_each_logical_thread([&](int t) {
    std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(t));
    std::uniform_real_distribution<double> dist(0, std::numeric_limits<T>::max());
    size_t b, e;
    static_block(n, t, &b, &e);
    for (size_t i = b; i < e; ++i) out[i] = static_cast<T>(dist(rng));
  });
}

template <typename T>
void ref_normal(T* out, size_t n, uint32_t seed) {
  const double mean = std::numeric_limits<T>::max() / 2.0;
  const double stddev = mean / 3.0;
  for_each_logical_thread([&](int t) {
    std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(t));
    std::normal_distribution<double> dist(mean, stddev);
    size_t b, e;
    static_block(n, t, &b, &e);
    for (size_t i = b; i < e; ++i) out[i] = static_cast<T>(std::fabs(dist(rng)));
  });
}

template <typename T>
void ref_zero(T* out, size_t n) {
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) out[i] = 0;
}

// The bucket bounds below keep the reference's expression `num_buckets > upper`
// (size_t against T) and its implicit conversions, on purpose.
#pragma GCC diagnostic ignored "-Wsign-compare"
// src/data_generator.cuh:81-115. Ten buckets; each bucket is uniform over a
// window of width 10 below a random upper bound; the tail that does not fill a
// bucket uses a separate generator seeded with seed + 128.
template <typename T>
void ref_staggered(T* out, size_t n, uint32_t seed) {
  const size_t num_buckets = 10;
  const size_t bucket_size = n / num_buckets;
  if (bucket_size == 0) return;  // the reference divides by zero here (n < 10)
  const size_t loop_n = n / bucket_size;
  for_each_logical_thread([&](int t) {
    std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(t));
    std::uniform_real_distribution<double> range_dist(0, std::numeric_limits<T>::max());
    size_t b, e;
    static_block(loop_n, t, &b, &e);
    for (size_t i = b; i < e; ++i) {
      T upper = range_dist(rng);
      T lower = num_buckets > upper ? 0 : upper - num_buckets;
      std::uniform_real_distribution<double> dist(lower, upper);
      for (size_t j = i * bucket_size; j < (i + 1) * bucket_size; ++j) out[j] = static_cast<T>(dist(rng));
    }
  });
  std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(kGeneratorThreads));
  std::uniform_real_distribution<double> range_dist(0, std::numeric_limits<T>::max());
  T upper = range_dist(rng);
  T lower = num_buckets > upper ? 0 : upper - num_buckets;
  std::uniform_real_distribution<double> dist(lower, upper);
  for (size_t i = n - (n % bucket_size); i < n; ++i) out[i] = static_cast<T>(dist(rng));
}

template <typename T>
void ref_sorted(T* out, size_t n, uint32_t seed, bool reverse) {
  ref_uniform<T>(out, n, seed);
  if (reverse) {
    __gnu_parallel::sort(out, out + n, std::greater<T>());
  } else {
    __gnu_parallel::sort(out, out + n);
  }
}

// src/data_generator.cuh:132-161: sorted input, then each element but the last
// is raised by |N(0, 2*gap)| (gap = distance to its successor), saturating at
// the type maximum. The reference reads the successor while another thread may
// already have raised it (a data race at the 127 block boundaries); this
// version always reads the successor's sorted value.
template <typename T>
void ref_nearly_sorted(T* out, size_t n, uint32_t seed) {
  ref_sorted<T>(out, n, seed, false);
  if (n < 2) return;
  std::vector<T> boundary(kGeneratorThreads + 1);
  for (int t = 0; t < kGeneratorThreads; ++t) {
    size_t b, e;
    static_block(n - 1, t, &b, &e);
    boundary[t] = e < n ? out[e] : T(0);
  }
  for_each_logical_thread([&](int t) {
    std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(t));
    size_t b, e;
    static_block(n - 1, t, &b, &e);
    for (size_t i = b; i < e; ++i) {
      const double mean = 0.0;
      const T next = (i + 1 == e) ? boundary[t] : out[i + 1];
      double stddev = next - out[i];
      if (stddev < std::numeric_limits<double>::max() / 2.0) stddev *= 2.0;
      std::normal_distribution<double> dist(mean, stddev);
      T diff = static_cast<T>(std::fabs(dist(rng)));
      if (out[i] > std::numeric_limits<T>::max() - diff) {
        out[i] = std::numeric_limits<T>::max();
      } else {
        out[i] += diff;
      }
    }
  });
}

// src/data_generator.cuh:164-191: ten uniform buckets (plus the remainder),
// each bucket then sorted on its own.
template <typename T>
void ref_bucket_sorted(T* out, size_t n, uint32_t seed) {
  const size_t num_buckets = 10;
  const size_t bucket_size = n / num_buckets;
  if (bucket_size == 0) return;  // the reference divides by zero here (n < 10)
  const size_t tail_begin = n - n % bucket_size;
  for_each_logical_thread([&](int t) {
    std::mt19937 rng = seeded_generator(seed + static_cast<uint32_t>(t));
    std::uniform_real_distribution<double> dist(0, std::numeric_limits<T>::max());
    size_t b, e;
    static_block(num_buckets, t, &b, &e);
    for (size_t i = b; i < e; ++i)
      for (size_t j = i * bucket_size; j < (i + 1) * bucket_size; ++j) out[j] = static_cast<T>(dist(rng));
    static_block(n - tail_begin, t, &b, &e);
    for (size_t i = tail_begin + b; i < tail_begin + e; ++i) out[i] = static_cast<T>(dist(rng));
  });
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i <= num_buckets; ++i) {
    T* lo = out + i * bucket_size;
    T* hi = std::min(out + (i + 1) * bucket_size, out + n);
    if (lo < hi) std::sort(lo, hi);
  }
}

// ---------------------------------------------------------------- part 2 ----
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Counter-based stream: value `k` of stream `s` for seed `seed`.
inline uint64_t draw(uint32_t seed, uint64_t s, uint64_t k) {
  return splitmix64(splitmix64((uint64_t(seed) << 8) ^ s) ^ splitmix64(k * 0xD1B54A32D192ED03ull + s));
}
inline double unit(uint64_t r) { return double(r >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)

template <typename T>
T from_bits(uint64_t r) {
  T v;
  if (sizeof(T) == 4) {
    uint32_t b = uint32_t(r);
    std::memcpy(&v, &b, 4);
  } else {
    std::memcpy(&v, &r, 8);
  }
  return v;
}

template <typename T>
void full_uniform(T* out, size_t n, uint32_t seed) {
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    const uint64_t r = draw(seed, 1, i);
    if (std::is_floating_point<T>::value) {
      // uniform real over [-max, max]
      const double u = unit(r);
      out[i] = static_cast<T>((2.0 * u - 1.0) * double(std::numeric_limits<T>::max()));
    } else {
      out[i] = from_bits<T>(r);  // uniform over every bit pattern = the full range
    }
  }
}

template <typename T>
void normal0(T* out, size_t n, uint32_t seed) {
  const double sd = 1048576.0;  // 2^20
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    // Box-Muller on two counter draws
    const double u1 = 1.0 - unit(draw(seed, 2, 2 * i));
    const double u2 = unit(draw(seed, 2, 2 * i + 1));
    const double x = sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    if (std::is_floating_point<T>::value) {
      out[i] = static_cast<T>(x);
    } else {
      // rounded; negative values of unsigned types wrap modulo 2^w
      out[i] = static_cast<T>(static_cast<long long>(std::llround(x)));
    }
  }
}

// Zipf(s) over `distinct` ranks by inverse CDF; rank k maps to a fixed scattered
// key value so that every digit position varies.
template <typename T>
void zipf_tables_typed(uint32_t seed, double s, size_t distinct, std::vector<double>* cdf_out,
                       std::vector<T>* value_out) {
  std::vector<double>& cdf = *cdf_out;
  cdf.assign(distinct, 0.0);
  double acc = 0.0;
  for (size_t k = 0; k < distinct; ++k) {
    acc += std::pow(double(k + 1), -s);
    cdf[k] = acc;
  }
  for (auto& c : cdf) c /= acc;
  std::vector<T>& value = *value_out;
  value.assign(distinct, T(0));
  for (size_t k = 0; k < distinct; ++k) {
    const uint64_t r = splitmix64(uint64_t(seed) * 0x100000001B3ull + k);
    if (std::is_floating_point<T>::value) {
      value[k] = static_cast<T>((unit(r) * 2.0 - 1.0) * 1.0e6);
    } else {
      value[k] = from_bits<T>(r);
    }
  }
}

template <typename T>
void zipf(T* out, size_t n, uint32_t seed, double s, size_t distinct) {
  std::vector<double> cdf;
  std::vector<T> value;
  zipf_tables_typed<T>(seed, s, distinct, &cdf, &value);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    const double u = unit(draw(seed, 3, i));
    size_t k = size_t(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
    if (k >= distinct) k = distinct - 1;
    out[i] = value[k];
  }
}

template <typename T>
void all_equal(T* out, size_t n) {
  const T v = std::is_floating_point<T>::value ? static_cast<T>(1.5) : static_cast<T>(0x5A);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) out[i] = v;
}

template <typename T>
void swap_one_percent(T* out, size_t n, uint32_t seed) {
  if (n < 2) return;
  const size_t swaps = n / 100;
  for (size_t j = 0; j < swaps; ++j) {
    const size_t a = size_t(draw(seed, 4, 2 * j) % n);
    const size_t b = size_t(draw(seed, 4, 2 * j + 1) % n);
    std::swap(out[a], out[b]);
  }
}

// Replace 0.1% of the keys with -0.0 and 0.1% with NaNs (quiet and signalling
// patterns with both sign bits and several payloads).
template <typename T>
void add_specials(T* out, size_t n, uint32_t seed) {
  using U = typename std::conditional<sizeof(T) == 4, uint32_t, uint64_t>::type;
  const U sign = U(1) << (sizeof(U) * 8 - 1);
  const U nan_patterns4[] = {0x7FC00000u, 0xFFC00000u, 0x7FC00001u, 0xFFC12345u, 0x7F800001u, 0xFF800002u};
  const uint64_t nan_patterns8[] = {0x7FF8000000000000ull, 0xFFF8000000000000ull, 0x7FF8000000000001ull,
                                    0xFFF8000000012345ull, 0x7FF0000000000001ull, 0xFFF0000000000002ull};
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; ++i) {
    const uint64_t r = draw(seed, 5, i) % 1000;
    if (r == 0) {
      U b = sign;
      std::memcpy(&out[i], &b, sizeof(U));
    } else if (r == 1) {
      const uint64_t pick = draw(seed, 6, i) % 6;
      U b = sizeof(U) == 4 ? U(nan_patterns4[pick]) : U(nan_patterns8[pick]);
      std::memcpy(&out[i], &b, sizeof(U));
    }
  }
}

template <typename T>
bool generate_typed(const std::string& dist_in, uint32_t seed, T* out, size_t n) {
  std::string dist = dist_in;
  bool specials = false;
  const std::string suffix = "-specials";
  if (dist.size() > suffix.size() && dist.compare(dist.size() - suffix.size(), suffix.size(), suffix) == 0) {
    if (!std::is_floating_point<T>::value) return false;
    specials = true;
    dist.resize(dist.size() - suffix.size());
  }
  if (dist == "uniform") {
    ref_uniform<T>(out, n, seed);
  } else if (dist == "normal") {
    ref_normal<T>(out, n, seed);
  } else if (dist == "zero") {
    ref_zero<T>(out, n);
  } else if (dist == "staggered") {
    ref_staggered<T>(out, n, seed);
  } else if (dist == "sorted") {
    ref_sorted<T>(out, n, seed, false);
  } else if (dist == "reverse-sorted") {
    ref_sorted<T>(out, n, seed, true);
  } else if (dist == "nearly-sorted") {
    ref_nearly_sorted<T>(out, n, seed);
  } else if (dist == "bucket-sorted") {
    ref_bucket_sorted<T>(out, n, seed);
  } else if (dist == "full-uniform") {
    full_uniform<T>(out, n, seed);
  } else if (dist == "normal0") {
    normal0<T>(out, n, seed);
  } else if (dist == "zipf") {
    zipf<T>(out, n, seed, kZipfExponent, kZipfDistinct);
  } else if (dist == "sorted-full" || dist == "reverse-sorted-full" || dist == "nearly-sorted-swaps") {
    full_uniform<T>(out, n, seed);
    if (dist == "reverse-sorted-full") {
      __gnu_parallel::sort(out, out + n, std::greater<T>());
    } else {
      __gnu_parallel::sort(out, out + n);
    }
    if (dist == "nearly-sorted-swaps") swap_one_percent<T>(out, n, seed);
  } else if (dist == "all-equal") {
    all_equal<T>(out, n);
  } else {
    return false;
  }
  if (specials) add_specials<T>(out, n, seed);
  return true;
}

template <typename T>
void zipf_tables_bytes(uint32_t seed, std::vector<double>* cdf, std::vector<unsigned char>* bytes) {
  std::vector<T> value;
  zipf_tables_typed<T>(seed, kZipfExponent, kZipfDistinct, cdf, &value);
  bytes->resize(value.size() * sizeof(T));
  std::memcpy(bytes->data(), value.data(), bytes->size());
}

}  // namespace

void generator_static_block(size_t n, int t, size_t* begin, size_t* end) { static_block(n, t, begin, end); }

bool mt19937_seed_state(uint32_t seed, uint32_t* state624) {
  // The engine's textual form is its state: the 624 words, then (libstdc++)
  // the position of the next output, which is 624 for a freshly seeded engine.
  std::ostringstream os;
  os << seeded_generator(seed);
  std::istringstream is(os.str());
  for (size_t i = 0; i < std::mt19937::state_size; ++i) {
    unsigned long long v;
    if (!(is >> v) || v > 0xFFFFFFFFull) return false;
    state624[i] = static_cast<uint32_t>(v);
  }
  unsigned long long p;
  return bool(is >> p) && p == std::mt19937::state_size;
}

bool zipf_tables(int dtype, uint32_t seed, std::vector<double>* cdf, std::vector<unsigned char>* values) {
  switch (dtype) {
    case 0: zipf_tables_bytes<uint32_t>(seed, cdf, values); return true;
    case 1: zipf_tables_bytes<int32_t>(seed, cdf, values); return true;
    case 2: zipf_tables_bytes<float>(seed, cdf, values); return true;
    case 3: zipf_tables_bytes<uint64_t>(seed, cdf, values); return true;
    case 4: zipf_tables_bytes<int64_t>(seed, cdf, values); return true;
    case 5: zipf_tables_bytes<double>(seed, cdf, values); return true;
    default: return false;
  }
}

// dtype codes follow mgs_dtype (u32, i32, f32, u64, i64, f64).
bool generate_keys(int dtype, const char* distribution, uint32_t seed, void* out, size_t n) {
  const std::string d(distribution);
  switch (dtype) {
    case 0: return generate_typed<uint32_t>(d, seed, static_cast<uint32_t*>(out), n);
    case 1: return generate_typed<int32_t>(d, seed, static_cast<int32_t*>(out), n);
    case 2: return generate_typed<float>(d, seed, static_cast<float*>(out), n);
    case 3: return generate_typed<uint64_t>(d, seed, static_cast<uint64_t*>(out), n);
    case 4: return generate_typed<int64_t>(d, seed, static_cast<int64_t*>(out), n);
    case 5: return generate_typed<double>(d, seed, static_cast<double*>(out), n);
    default: return false;
  }
}

}  // namespace mgs
