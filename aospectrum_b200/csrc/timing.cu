// CUDA-event timing of selected kernel launches (see timing.h).
#include "timing.h"

#include <mutex>
#include <vector>

namespace aosb {
namespace {

struct Category {
  std::vector<cudaEvent_t> events;  // start, stop pairs
  double flops = 0.0, bytes = 0.0;
  int64_t launches = 0;
};

struct Timer {
  std::mutex mu;
  bool on = false;
  Category cat[kTimedCount];
};

Timer& timer() {
  static Timer t;
  return t;
}

}  // namespace

bool timing_begin(cudaStream_t st, cudaEvent_t (&ev)[2]) {
  ev[0] = ev[1] = nullptr;
  Timer& t = timer();
  {
    std::lock_guard<std::mutex> lock(t.mu);
    if (!t.on) return false;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return false;
  if (cudaEventCreate(&ev[0]) != cudaSuccess) return false;
  if (cudaEventCreate(&ev[1]) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    ev[0] = nullptr;
    return false;
  }
  cudaEventRecord(ev[0], st);
  return true;
}

void timing_end(int cat, cudaStream_t st, cudaEvent_t (&ev)[2], double flops, double bytes) {
  if (ev[0] == nullptr || cat < 0 || cat >= kTimedCount) return;
  cudaEventRecord(ev[1], st);
  Timer& t = timer();
  std::lock_guard<std::mutex> lock(t.mu);
  Category& c = t.cat[cat];
  c.events.push_back(ev[0]);
  c.events.push_back(ev[1]);
  c.flops += flops;
  c.bytes += bytes;
  c.launches += 1;
}

}  // namespace aosb

extern "C" int aosb_kernel_timing(int32_t enable) {
  aosb::Timer& t = aosb::timer();
  std::lock_guard<std::mutex> lock(t.mu);
  for (auto& c : t.cat) {
    for (cudaEvent_t e : c.events) cudaEventDestroy(e);
    c.events.clear();
    c.flops = c.bytes = 0.0;
    c.launches = 0;
  }
  t.on = enable != 0;
  return 0;
}

extern "C" int aosb_kernel_timing_read_category(int32_t category, double* total_ms, double* flops,
                                                double* bytes, int64_t* launches) {
  if (category < 0 || category >= aosb::kTimedCount) return AOSB_ERR_ARGUMENT;
  aosb::Timer& t = aosb::timer();
  std::lock_guard<std::mutex> lock(t.mu);
  const aosb::Category& c = t.cat[category];
  double ms = 0.0;
  for (size_t i = 0; i + 1 < c.events.size(); i += 2) {
    if (cudaEventSynchronize(c.events[i + 1]) != cudaSuccess) return AOSB_ERR_CUDA;
    float one = 0.0f;
    if (cudaEventElapsedTime(&one, c.events[i], c.events[i + 1]) != cudaSuccess) return AOSB_ERR_CUDA;
    ms += one;
  }
  if (total_ms) *total_ms = ms;
  if (flops) *flops = c.flops;
  if (bytes) *bytes = c.bytes;
  if (launches) *launches = c.launches;
  return 0;
}

extern "C" int aosb_kernel_timing_read(double* total_ms, double* flops, double* bytes,
                                       int64_t* launches) {
  return aosb_kernel_timing_read_category(aosb::kTimedSchur, total_ms, flops, bytes, launches);
}
