// peak.cu — measured issue rates of the integer multiply pipe and of the
// library's own 256-bit Montgomery product: the denominators of the rooflines
// the benchmark reports for the multiply-bound kernels (MSM bucket
// accumulation, NTT passes).
//
// Three loops, each over independent chains so that the pipe, not latency,
// bounds them, in blocks of 256 threads:
//   mad.lo.u32     a = a * m + c, 8 chains per thread
//   mad.wide.u32   A = x * y + A (32 x 32 -> 64 bits), 8 chains per thread
//   Montgomery     x = x * y mod q over BN254's base field (fe_mul, inline),
//                  4 chains per thread
// Each launch is one wave: as many 256-thread blocks per SM as fit at once
// (the occupancy query), so every block of an SM runs beside the others for
// the whole loop. Each block reads the SM's cycle counter around its loop, so
// a rate comes out per SM per clock, independent of the clock the GPU ran at;
// the CUDA-event time of the launch gives the same rate per second and,
// divided into the cycles, the SM clock under that load.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "field.cuh"

namespace zkb {

static constexpr int kPeakThreads = 256;

__global__ void __launch_bounds__(kPeakThreads) k_peak_madlo(uint32_t m, uint32_t c, int iters,
                                                             uint32_t* sink, long long* cycles) {
  uint32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = threadIdx.x + 977u * k + blockIdx.x;
  __syncthreads();
  const long long t0 = clock64();
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
  }
  __syncthreads();
  const long long t1 = clock64();
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s ^= a[k];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_madwide(uint32_t y, int iters, uint32_t* sink,
                                                               long long* cycles) {
  uint64_t a[8];
  uint32_t x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    a[k] = threadIdx.x + 131ull * k;
    x[k] = threadIdx.x * 2654435761u + (uint32_t)k;
  }
  __syncthreads();
  const long long t0 = clock64();
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(a[k]) : "r"(x[k]), "r"(y));
  }
  __syncthreads();
  const long long t1 = clock64();
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s ^= a[k];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = (uint32_t)s ^ (uint32_t)(s >> 32);
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_montmul(int iters, uint32_t* sink, long long* cycles) {
  FqP f;
  uint32_t x[4][8], y[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) y[j] = f.one(j) ^ (j == 0 ? 12345u : 0u);
  y[7] &= 0x0fffffffu;  // below q
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 0; j < 8; ++j) x[k][j] = j < 7 ? threadIdx.x * 7919u + 31u * k + j : 1u;
  __syncthreads();
  const long long t0 = clock64();
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 4; ++k) fe_mul(x[k], x[k], y, f);
  }
  __syncthreads();
  const long long t1 = clock64();
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int j = 0; j < 8; ++j) s ^= x[k][j];
  sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
}

// Median of the per-block cycle counts (blocks on one SM run side by side, so
// each spans about the whole loop of its SM).
static double median_cycles(std::vector<long long>& v) {
  std::sort(v.begin(), v.end());
  return v.empty() ? 0.0 : (double)v[v.size() / 2];
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_measure_int_peaks(zkb_int_peaks* out, void* stream) {
  set_error("%s", "");
  if (!out) return fail(ZKB_EINVAL, "null output");
  std::memset(out, 0, sizeof *out);
  cudaStream_t s = as_stream(stream);
  int device = 0, sms = 0;
  ZKB_TRY(check_cuda(cudaGetDevice(&device), "cudaGetDevice"));
  ZKB_TRY(check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count"));
  // the largest one-wave grid of the three kernels sizes the buffers
  int occ[3] = {0, 0, 0};
  ZKB_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_peak_madlo, kPeakThreads, 0),
                     "occupancy"));
  ZKB_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_peak_madwide, kPeakThreads, 0),
                     "occupancy"));
  ZKB_TRY(check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_peak_montmul, kPeakThreads, 0),
                     "occupancy"));
  for (int k = 0; k < 3; ++k)
    if (occ[k] < 1) return fail(ZKB_ECUDA, "integer peak probe %d does not fit an SM", k);
  const int max_blocks = sms * *std::max_element(occ, occ + 3);
  const size_t threads_total = (size_t)max_blocks * kPeakThreads;
  uint32_t* sink = nullptr;
  long long* cycles = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = check_cuda(cudaMalloc(&sink, threads_total * 4), "peak probe buffer");
  if (rc == ZKB_OK) rc = check_cuda(cudaMalloc(&cycles, (size_t)max_blocks * 8), "peak probe cycles");
  if (rc == ZKB_OK) rc = check_cuda(cudaEventCreate(&e0), "event");
  if (rc == ZKB_OK) rc = check_cuda(cudaEventCreate(&e1), "event");
  // one probe: warm-up launch, timed launch, per-SM-clock rate and per-second rate
  auto probe = [&](int which, int iters, double ops_per_iter, double* per_clk, double* per_s,
                   double* mhz) -> int {
    const int per_sm = occ[which], blocks = sms * per_sm;
    std::vector<long long> host(blocks);
    for (int rep = 0; rep < 2; ++rep) {
      if (rep == 1) ZKB_TRY(check_cuda(cudaEventRecord(e0, s), "event record"));
      if (which == 0) {
        k_peak_madlo<<<blocks, kPeakThreads, 0, s>>>(0x9e3779b9u, 0x7f4a7c15u, iters, sink, cycles);
      } else if (which == 1) {
        k_peak_madwide<<<blocks, kPeakThreads, 0, s>>>(0x85ebca6bu, iters, sink, cycles);
      } else {
        k_peak_montmul<<<blocks, kPeakThreads, 0, s>>>(iters, sink, cycles);
      }
      ZKB_TRY(check_launch("integer peak probe"));
      if (rep == 1) ZKB_TRY(check_cuda(cudaEventRecord(e1, s), "event record"));
    }
    ZKB_TRY(check_cuda(cudaEventSynchronize(e1), "peak probe"));
    float ms = 0.f;
    ZKB_TRY(check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event time"));
    ZKB_TRY(check_cuda(cudaMemcpy(host.data(), cycles, (size_t)blocks * 8, cudaMemcpyDeviceToHost),
                       "peak probe cycles copy"));
    const double cyc = median_cycles(host);
    const double ops_per_sm = ops_per_iter * iters * kPeakThreads * per_sm;
    *per_clk = cyc > 0 ? ops_per_sm / cyc : 0.0;
    *per_s = ms > 0 ? ops_per_sm * sms / (ms * 1e-3) : 0.0;
    *mhz = ms > 0 ? cyc / (ms * 1e-3) / 1e6 : 0.0;
    return ZKB_OK;
  };
  if (rc == ZKB_OK) {
    rc = probe(0, 1 << 15, 8.0, &out->madlo_per_clk_sm, &out->madlo_per_s, &out->madlo_mhz);
  }
  if (rc == ZKB_OK) {
    rc = probe(1, 1 << 14, 8.0, &out->madwide_per_clk_sm, &out->madwide_per_s, &out->madwide_mhz);
  }
  if (rc == ZKB_OK) {
    rc = probe(2, 1 << 8, 4.0, &out->montmul_per_clk_sm, &out->montmul_per_s, &out->montmul_mhz);
  }
  out->sms = sms;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  if (cycles) cudaFree(cycles);
  return rc;
}

}  // extern "C"
