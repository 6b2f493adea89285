// Error state and twiddle tables shared by all operators.
#include "common.cuh"

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace ht {

namespace {
thread_local std::string g_last_error;
std::mutex g_tw_mutex;
std::map<std::pair<int, int>, float2*> g_tw;  // (device, N) -> table
const int kSizes[] = {18, 24, 32, 36, 48, 64, 96, 128, 192, 256, 384, 512,
                      768, 1024, 1536, 2048, 3072, 4096};
}  // namespace

std::atomic<long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {
std::mutex g_attr_mutex;
std::map<std::pair<int, const void*>, int> g_attr;  // (device, kernel) -> bytes allowed
}  // namespace

bool smem_attr_done(const void* kernel, int bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  auto it = g_attr.find(std::make_pair(dev, kernel));
  return it != g_attr.end() && it->second >= bytes;
}

void smem_attr_mark(const void* kernel, int bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  int& b = g_attr[std::make_pair(dev, kernel)];
  if (bytes > b) b = bytes;
}

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

bool fft_size_supported(int N) {
  for (int s : kSizes)
    if (s == N) return true;
  return false;
}

const float2* twiddle_table(int N, int device) {
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  auto key = std::make_pair(device, N);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) return it->second;
  const int M = 4 * N;
  std::vector<float2> h(M);
  for (int m = 0; m < M; ++m) {
    // exp(-2 pi i m / M), argument reduced exactly in integers first
    const double a = -2.0 * M_PI * (double)m / (double)M;
    h[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  float2* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(float2) * M);
  if (e != cudaSuccess) {
    set_error(std::string("twiddle table allocation: ") + cudaGetErrorString(e));
    return nullptr;
  }
  e = cudaMemcpy(d, h.data(), sizeof(float2) * M, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    set_error(std::string("twiddle table upload: ") + cudaGetErrorString(e));
    return nullptr;
  }
  g_tw[key] = d;
  return d;
}

}  // namespace ht
