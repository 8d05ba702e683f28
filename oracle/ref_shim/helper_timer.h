/* Minimal stand-in for the CUDA-samples timer header that the reference's
 * refine.h includes (GPU_Refine/refine.h:5).  Only the five calls that
 * refine.cu makes are provided; timing uses std::chrono.  This file is part
 * of the test oracle build recipe and is never linked into the product. */
#pragma once
#include <chrono>

struct StopWatchInterface {
  std::chrono::steady_clock::time_point t0;
  double acc_ms = 0.0;
  bool running = false;
};

inline bool sdkCreateTimer(StopWatchInterface **t) { *t = new StopWatchInterface(); return true; }
inline bool sdkStartTimer(StopWatchInterface **t) { (*t)->t0 = std::chrono::steady_clock::now(); (*t)->running = true; return true; }
inline bool sdkStopTimer(StopWatchInterface **t) {
  if ((*t)->running) {
    (*t)->acc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - (*t)->t0).count();
    (*t)->running = false;
  }
  return true;
}
inline bool sdkResetTimer(StopWatchInterface **t) { (*t)->acc_ms = 0.0; (*t)->running = false; return true; }
inline float sdkGetTimerValue(StopWatchInterface **t) { return (float)(*t)->acc_ms; }
