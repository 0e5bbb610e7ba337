// sort_benchmark: the reference's benchmark CLI (src/sort_benchmark.cu) on the
// engine. Same options, defaults and CSV line:
//   num_elements,"algorithm","gpus","data_type","distribution",seed,threads,
//   chunk_size,merge_group_size,num_buffers,memory_allocation,sort_phase,
//   memory_deallocation,total
// followed by "Error: Invalid sort order." when the output is not sorted
// (exit code 0, as in the reference). Added option: --chunks <g> sorts with
// TanasicSort over g chunks of the first GPU (the reference's g partitions).
// "boost" and "paradis" are CPU baselines whose sources are not available
// (empty submodules); "std" runs std::sort.
#include <omp.h>

#include <algorithm>
#include <iomanip>
#include <iostream>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "argument_limits.h"
#include "data_generator.h"
#include "gowanlock_sort.h"
#include "host_vector.h"
#include "tanasic_sort.h"
#include "time_durations.h"

namespace {

void Usage() {
  std::cout << "Usage: ./sort_benchmark <num_elements> [options]\n\n"
            << "--algorithm\t\t<algorithm>\t\t" << ArgumentLimits::Join(ArgumentLimits::Algorithms()) << " (= tanasic)\n"
            << "--gpus\t\t\t<gpus>\t\t\tThe visible GPUs, e.g. 0 or {0,1} (= 0)\n"
            << "--chunks\t\t<g>\t\t\tTanasicSort over g chunks of the first GPU (= number of gpus)\n"
            << "--num_threads\t\t<num_threads>\t\t[1, " << omp_get_num_procs() << "] (= " << omp_get_num_procs()
            << ")\n"
            << "--data_type\t\t<data_type>\t\t" << ArgumentLimits::Join(ArgumentLimits::DataTypes()) << " (= int)\n"
            << "--distribution_type\t<distribution_type>\t" << ArgumentLimits::Join(ArgumentLimits::Distributions())
            << " (= uniform)\n"
            << "--distribution_seed\t<distribution_seed>\t[0, 4294967295] (= 2147483647)\n\n"
            << "[--algorithm gowanlock]\n"
            << "--chunk_size\t\t<chunk_size>\t\t(= auto)\n"
            << "--merge_group_size\t<merge_group_size>\t(= auto)\n"
            << "--num_buffers\t\t<num_buffers>\t\t{2, 3} (= 2)\n";
  std::exit(1);
}

void Fail(const std::string& what) {
  std::cout << "Error: " << what << "\n\n";
  Usage();
}

bool Option(const std::vector<std::string>& args, const std::string& name, std::string* value) {
  auto it = std::find(args.begin(), args.end(), name);
  if (it == args.end() || it + 1 == args.end()) return false;
  *value = *(it + 1);
  return true;
}

template <typename T>
bool Run(size_t n, const std::string& algorithm, const std::vector<int>& gpus, int chunks, const std::string& data_type,
         const std::string& dist, uint32_t seed, int threads, size_t chunk_size, size_t merge_group_size,
         size_t num_buffers) {
  DataGenerator generator(seed);
  HostVector<T> elements(n);
  if (n > 0) generator.ComputeDistribution<T>(elements.data(), n, dist);

  if (algorithm == "tanasic") {
    SetupTanasicSort(gpus);
    std::vector<int> parts(chunks, gpus.front());
    TanasicSort<T>(&elements, parts);
  } else if (algorithm == "gowanlock") {
    SetupGowanlockSort(gpus, threads);
    GowanlockSort<T>(&elements, chunk_size, merge_group_size, num_buffers, gpus);
  } else if (algorithm == "thrust") {
    mgs_ctx* ctx = mgs_compat::Contexts::get(gpus.front());
    TimeDurations::Get()->Tic("sort_phase");
    if (n > 0) mgs_compat::check(mgs_sort_host(ctx, mgs_compat::DType<T>::value, elements.data(), n), "sort");
    TimeDurations::Get()->Toc("sort_phase");
  } else if (algorithm == "gnu_parallel") {
    omp_set_num_threads(threads);
    TimeDurations::Get()->Tic("sort_phase");
    __gnu_parallel::sort(elements.begin(), elements.end());
    TimeDurations::Get()->Toc("sort_phase");
  } else if (algorithm == "std") {
    TimeDurations::Get()->Tic("sort_phase");
    std::sort(elements.begin(), elements.end());
    TimeDurations::Get()->Toc("sort_phase");
  } else {
    std::cout << "Error: algorithm '" << algorithm << "' is not available in this build\n";
    std::exit(1);
  }

  std::cout << n << ",\"" << algorithm << "\",\"";
  for (size_t i = 0; i < gpus.size(); ++i) std::cout << gpus[i] << (i + 1 < gpus.size() ? "," : "\"");
  std::cout << ",\"" << data_type << "\",\"" << dist << "\"," << seed << "," << threads << "," << chunk_size << ","
            << merge_group_size << "," << num_buffers << ",";
  std::cout << std::fixed << std::setprecision(9);
  auto& d = TimeDurations::Get()->durations;
  std::cout << d["memory_allocation"].count() << "," << d["sort_phase"].count() << ","
            << d["memory_deallocation"].count() << "," << TimeDurations::Get()->TotalExecutionTime().count() << "\n";
  return std::is_sorted(elements.begin(), elements.end());
}

}  // namespace

int main(int argc, char* argv[]) {
  const std::vector<std::string> args(argv + 1, argv + argc);
  if (args.empty() || args.size() % 2 == 0 || std::find(args.begin(), args.end(), "--help") != args.end()) Usage();
  std::string v;
  size_t n = 0;
  if (!ArgumentLimits::ParseNumElements(args.front(), &n)) Fail("Invalid <num_elements> = " + args.front());
  std::string algorithm = ArgumentLimits::GetDefaultAlgorithm();
  if (Option(args, "--algorithm", &v) && !ArgumentLimits::ParseAlgorithm(v, &algorithm)) Fail("Invalid <algorithm> = " + v);
  std::vector<int> gpus = ArgumentLimits::GetDefaultGpus();
  if (Option(args, "--gpus", &v) && !ArgumentLimits::ParseGpus(v, &gpus)) Fail("Invalid <gpus> = " + v);
  int chunks = static_cast<int>(gpus.size());
  if (Option(args, "--chunks", &v)) {
    if (!ArgumentLimits::IsDigits(v) || std::stoi(v) < 1 || (std::stoi(v) & (std::stoi(v) - 1)) != 0)
      Fail("Invalid <chunks> = " + v);
    chunks = std::stoi(v);
  }
  std::string data_type = ArgumentLimits::GetDefaultDataType();
  if (Option(args, "--data_type", &v) && !ArgumentLimits::ParseDataType(v, &data_type)) Fail("Invalid <data_type> = " + v);
  std::string dist = ArgumentLimits::GetDefaultDistributionType();
  if (Option(args, "--distribution_type", &v) && !ArgumentLimits::ParseDistributionType(v, &dist))
    Fail("Invalid <distribution_type> = " + v);
  uint32_t seed = ArgumentLimits::GetDefaultDistributionSeed();
  if (Option(args, "--distribution_seed", &v) && !ArgumentLimits::ParseDistributionSeed(v, &seed))
    Fail("Invalid <distribution_seed> = " + v);
  int threads = ArgumentLimits::GetDefaultNumThreads();
  if (Option(args, "--num_threads", &v) && !ArgumentLimits::ParseNumThreads(v, &threads))
    Fail("Invalid <num_threads> = " + v);
  size_t chunk_size = ArgumentLimits::GetDefaultChunkSize();
  if (Option(args, "--chunk_size", &v) && !ArgumentLimits::ParseChunkSize(v, &chunk_size))
    Fail("Invalid <chunk_size> = " + v);
  size_t merge_group_size = ArgumentLimits::GetDefaultMergeGroupSize();
  if (Option(args, "--merge_group_size", &v) && !ArgumentLimits::ParseMergeGroupSize(v, &merge_group_size))
    Fail("Invalid <merge_group_size> = " + v);
  size_t num_buffers = ArgumentLimits::GetDefaultNumBuffers();
  if (Option(args, "--num_buffers", &v) && !ArgumentLimits::ParseNumBuffers(v, &num_buffers))
    Fail("Invalid <num_buffers> = " + v);

  bool ok = false;
  if (data_type == "int") {
    ok = Run<int>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size, num_buffers);
  } else if (data_type == "long") {
    ok = Run<long>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size, num_buffers);
  } else if (data_type == "float") {
    ok = Run<float>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size, num_buffers);
  } else if (data_type == "double") {
    ok = Run<double>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size, num_buffers);
  } else if (data_type == "uint32") {
    ok = Run<unsigned>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size,
                       num_buffers);
  } else {
    ok = Run<unsigned long>(n, algorithm, gpus, chunks, data_type, dist, seed, threads, chunk_size, merge_group_size,
                            num_buffers);
  }
  if (!ok) std::cout << "Error: Invalid sort order.\n";
  return 0;
}
