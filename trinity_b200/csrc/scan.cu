/*
 * scan.cu — ordered prefix sums and stream compaction.
 *
 * Replaces the reference's per-thread task heaps + reduceTasks/prefixSum
 * (sync.cpp:24-86). Order matters: the reference, run on one thread, lists
 * candidates in ascending id and numbers new vertices/elements in that order,
 * so every compaction here is stable.
 *
 * Three launches: tile sums (2048 items per 256-thread block, staged through
 * shared memory so global loads stay coalesced), a one-block scan of the tile
 * sums, and a tile-local scan that adds the tile offset and writes.
 */
#include "trn_internal.h"
#include <tuple>
#include <mutex>
#include <map>

#include <cstdio>

namespace trn {

static constexpr int kItems = 8;
static constexpr int kTile = TRN_THREADS * kItems;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* warp_sums, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = (lane < (TRN_THREADS / 32)) ? warp_sums[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (TRN_THREADS / 32)) warp_sums[lane] = w;
  }
  __syncthreads();
  T prefix = (warp > 0 ? warp_sums[warp - 1] : T(0)) + x - v;
  if (total) *total = warp_sums[TRN_THREADS / 32 - 1];
  return prefix;
}

__global__ void k_tile_sum_i64(const long long* __restrict__ in, int n, const int* dn,
                               long long* tile) {
  if (dn) n = *dn;
  __shared__ long long sm[kTile];
  __shared__ long long ws[TRN_THREADS / 32];
  const long long base = (long long) blockIdx.x * kTile;
  for (int k = threadIdx.x; k < kTile; k += TRN_THREADS) {
    long long i = base + k;
    sm[k] = (i < n) ? in[i] : 0;
  }
  __syncthreads();
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) s += sm[threadIdx.x * kItems + k];
  long long tot;
  block_exclusive_scan<long long>(s, ws, &tot);
  if (threadIdx.x == 0) tile[blockIdx.x] = tot;
}

__global__ void k_tile_count_u8(const uint8_t* __restrict__ flags, int n, long long* tile) {
  __shared__ long long ws[TRN_THREADS / 32];
  const long long base = (long long) blockIdx.x * kTile;
  long long c = 0;
  for (int k = threadIdx.x; k < kTile; k += TRN_THREADS) {
    long long i = base + k;
    if (i < n && flags[i]) ++c;
  }
  long long tot;
  block_exclusive_scan<long long>(c, ws, &tot);
  if (threadIdx.x == 0) tile[blockIdx.x] = tot;
}

/* one block: exclusive scan of the tile sums in place, grand total out */
__global__ void k_scan_tiles(long long* tile, int ntiles, long long* total64, int* total32) {
  __shared__ long long ws[TRN_THREADS / 32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b = 0; b < ntiles; b += TRN_THREADS) {
    int i = b + threadIdx.x;
    long long v = (i < ntiles) ? tile[i] : 0;
    long long tot;
    long long ex = block_exclusive_scan<long long>(v, ws, &tot);
    if (i < ntiles) tile[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (total64) *total64 = carry;
    if (total32) *total32 = (int) carry;
  }
}

__global__ void k_tile_scan_i64(const long long* __restrict__ in, long long* __restrict__ out,
                                int n, const int* dn, const long long* tile) {
  if (dn) n = *dn;
  __shared__ long long sm[kTile];
  __shared__ long long ws[TRN_THREADS / 32];
  const long long base = (long long) blockIdx.x * kTile;
  for (int k = threadIdx.x; k < kTile; k += TRN_THREADS) {
    long long i = base + k;
    sm[k] = (i < n) ? in[i] : 0;
  }
  __syncthreads();
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) s += sm[threadIdx.x * kItems + k];
  long long ex = block_exclusive_scan<long long>(s, ws, nullptr) + tile[blockIdx.x];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    long long v = sm[threadIdx.x * kItems + k];
    sm[threadIdx.x * kItems + k] = ex;
    ex += v;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kTile; k += TRN_THREADS) {
    long long i = base + k;
    if (i < n) out[i] = sm[k];
  }
}

__global__ void k_tile_compact_u8(const uint8_t* __restrict__ flags, int n, int* __restrict__ list,
                                  const long long* tile) {
  __shared__ uint8_t sf[kTile];
  __shared__ long long ws[TRN_THREADS / 32];
  const long long base = (long long) blockIdx.x * kTile;
  for (int k = threadIdx.x; k < kTile; k += TRN_THREADS) {
    long long i = base + k;
    sf[k] = (i < n && flags[i]) ? 1 : 0;
  }
  __syncthreads();
  long long c = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) c += sf[threadIdx.x * kItems + k];
  long long pos = block_exclusive_scan<long long>(c, ws, nullptr) + tile[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kItems; ++k)
    if (sf[threadIdx.x * kItems + k]) list[pos++] = (int) (base + threadIdx.x * kItems + k);
}

void scan_ws_alloc(ScanWs* ws, long long max_n) {
  ws->max_tiles = (int) ((max_n + kTile - 1) / kTile) + 1;
  cudaMalloc(&ws->tile, sizeof(long long) * ws->max_tiles);
  cudaMalloc(&ws->count, sizeof(int) * 4);
  cudaMalloc(&ws->total, sizeof(long long) * 2);
}

void scan_ws_free(ScanWs* ws) {
  cudaFree(ws->tile);
  cudaFree(ws->count);
  cudaFree(ws->total);
  *ws = ScanWs();
}

void scan_i64(const long long* in, long long* out, int n, ScanWs& ws, cudaStream_t s, const int* dn) {
  int ntiles = (n + kTile - 1) / kTile;
  if (ntiles == 0) {
    cudaMemsetAsync(ws.total, 0, sizeof(long long), s);
    return;
  }
  ProfScope ps("scan", s, (double) n * 16);
  k_tile_sum_i64<<<ntiles, TRN_THREADS, 0, s>>>(in, n, dn, ws.tile);
  note_launch();
  k_scan_tiles<<<1, TRN_THREADS, 0, s>>>(ws.tile, ntiles, ws.total, nullptr);
  note_launch();
  k_tile_scan_i64<<<ntiles, TRN_THREADS, 0, s>>>(in, out, n, dn, ws.tile);
  note_launch();
}

void compact_u8(const uint8_t* flags, int n, int* list, ScanWs& ws, cudaStream_t s) {
  int ntiles = (n + kTile - 1) / kTile;
  if (ntiles == 0) {
    cudaMemsetAsync(ws.count, 0, sizeof(int), s);
    return;
  }
  ProfScope ps("compact", s, (double) n * 2);
  k_tile_count_u8<<<ntiles, TRN_THREADS, 0, s>>>(flags, n, ws.tile);
  note_launch();
  k_scan_tiles<<<1, TRN_THREADS, 0, s>>>(ws.tile, ntiles, nullptr, ws.count);
  note_launch();
  k_tile_compact_u8<<<ntiles, TRN_THREADS, 0, s>>>(flags, n, list, ws.tile);
  note_launch();
}

static const Tune kDefaultTune;
static thread_local const Tune* t_tune = nullptr;
const Tune& tune() { return t_tune ? *t_tune : kDefaultTune; }
void set_thread_tune(const Tune* t) { t_tune = t; }

int grid_bounded(long long bound, long long cap, int threads) {
  return grid_for(bound < 0 ? cap : (bound < cap ? bound : cap), threads);
}

/* at most as many blocks as are resident at once on the device (one wave:
 * a grid-stride kernel whose blocks hold more registers than grid_for's
 * 8 a SM assumes would otherwise end on a partial wave) */
int grid_resident(const void* kernel, int threads, int grid, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t>, int> cache;
  static const int sms = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(kernel, threads, smem);
    auto it = cache.find(key);
    if (it != cache.end()) {
      per_sm = it->second;
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
      }
      cache[key] = per_sm;
    }
  }
  if (per_sm <= 0) return grid;
  const int cap = per_sm * sms;
  return grid < cap ? grid : cap;
}

int grid_for(long long n, int threads) {
  static const int sms = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  long long blocks = (n + threads - 1) / threads;
  long long cap = (long long) sms * 8;  /* 8 resident 256-thread blocks per SM */
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int) blocks;
}

void check_launch(const char* what) {
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) std::fprintf(stderr, "trinity_b200: launch %s: %s\n", what, cudaGetErrorString(e));
}

}  // namespace trn
