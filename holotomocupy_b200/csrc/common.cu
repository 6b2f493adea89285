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

// ------------------------------------------------------------- timers
namespace {
struct TimerState {
  bool armed = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  double units = 0.0;
};
std::mutex g_timer_mutex;
std::map<std::string, TimerState> g_timers;
std::vector<std::pair<std::string, size_t>> g_timer_slots;  // slot -> (name, pair index)
}  // namespace

KTimer::KTimer(const char* name, cudaStream_t stream, double units) : st(stream) {
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  auto it = g_timers.find(name);
  if (it == g_timers.end() || !it->second.armed) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess) return;
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return;
  }
  cudaEventRecord(a, stream);
  it->second.ev.emplace_back(a, b);
  it->second.units += units;
  g_timer_slots.emplace_back(name, it->second.ev.size() - 1);
  slot = (int)g_timer_slots.size() - 1;
}

KTimer::~KTimer() {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  const auto& s = g_timer_slots[slot];
  cudaEventRecord(g_timers[s.first].ev[s.second].second, st);
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

extern "C" int ht_ktimer_arm(const char* name, int on) {
  using namespace ht;
  HT_REQUIRE(name, "ht_ktimer_arm: null name");
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  TimerState& t = g_timers[name];
  for (auto& p : t.ev) {
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  t.ev.clear();
  t.units = 0.0;
  g_timer_slots.clear();
  t.armed = on != 0;
  return kOk;
}

extern "C" int ht_ktimer_read(const char* name, double* total_ms, long* launches, double* units) {
  using namespace ht;
  HT_REQUIRE(name && total_ms && launches && units, "ht_ktimer_read: null pointer");
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  double tot = 0.0;
  long n = 0;
  auto it = g_timers.find(name);
  *units = it != g_timers.end() ? it->second.units : 0.0;
  if (it != g_timers.end())
    for (auto& p : it->second.ev) {
      HT_CHECK_CUDA(cudaEventSynchronize(p.second));
      float ms = 0.f;
      HT_CHECK_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
      tot += ms;
      ++n;
    }
  *total_ms = tot;
  *launches = n;
  return kOk;
}
