// Generic device primitives (scans, radix sorts) on the instance's stream.
// Scans and sorts are CUB's device-wide algorithms, run in the instance's
// preallocated temporary storage so that nothing is allocated per step.
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <algorithm>

#include "fsb_kernels.cuh"

namespace fsb {

void exclusive_scan_int(Ctx& c, const int* in, int* out, size_t n) {
  size_t bytes = c.cub_tmp_bytes;
  cub::DeviceScan::ExclusiveSum(c.cub_tmp, bytes, in, out, (int)n, c.stream);
  c.count_launch(2);
}

// modulo 2^32 (for sums whose terms cancel in pairs)
void exclusive_scan_u32(Ctx& c, const unsigned* in, unsigned* out, size_t n) {
  size_t bytes = c.cub_tmp_bytes;
  cub::DeviceScan::ExclusiveSum(c.cub_tmp, bytes, in, out, (int)n, c.stream);
  c.count_launch(2);
}

void inclusive_scan_int(Ctx& c, const int* in, int* out, size_t n) {
  size_t bytes = c.cub_tmp_bytes;
  cub::DeviceScan::InclusiveSum(c.cub_tmp, bytes, in, out, (int)n, c.stream);
  c.count_launch(2);
}

void sort_pairs_u32(Ctx& c, const unsigned* kin, unsigned* kout, const int* vin, int* vout, size_t n,
                    int end_bit) {
  size_t bytes = c.cub_tmp_bytes;
  cub::DeviceRadixSort::SortPairs(c.cub_tmp, bytes, kin, kout, vin, vout, (int)n, 0, end_bit, c.stream);
  c.count_launch(1 + (end_bit + 7) / 8);
}

void sort_pairs_u64(Ctx& c, const unsigned long long* kin, unsigned long long* kout, const int* vin,
                    int* vout, size_t n) {
  size_t bytes = c.cub_tmp_bytes;
  cub::DeviceRadixSort::SortPairs(c.cub_tmp, bytes, kin, kout, vin, vout, (int)n, 0, 64, c.stream);
  c.count_launch(9);
}

size_t cub_temp_bytes_needed(size_t nn, size_t nconn) {
  size_t mx = 0, b = 0;
  const size_t ns = std::max(nn + 1, nconn + 2);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const int*)nullptr, (int*)nullptr, (int)ns);
  mx = std::max(mx, b);
  cub::DeviceScan::InclusiveSum(nullptr, b, (const int*)nullptr, (int*)nullptr, (int)ns);
  mx = std::max(mx, b);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr, (int)ns);
  mx = std::max(mx, b);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned*)nullptr, (unsigned*)nullptr,
                                  (const int*)nullptr, (int*)nullptr, (int)std::max(nconn, nn), 0, 32);
  mx = std::max(mx, b);
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned long long*)nullptr,
                                  (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr,
                                  (int)nn, 0, 64);
  mx = std::max(mx, b);
  return mx + 256;
}

void fetch_counters(Ctx& c, int n) {
  cudaMemcpyAsync(c.h_cnt, c.d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream);
  cudaStreamSynchronize(c.stream);
}

}  // namespace fsb
