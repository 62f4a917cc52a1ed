// Status strings, error text and version of the C ABI.
#include <stdarg.h>

#include <atomic>

#include "common.cuh"

namespace igm {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

}  // namespace igm

extern "C" long long igm_launch_count(void) { return igm::g_launches.load(std::memory_order_relaxed); }

extern "C" const char* igm_status_string(int status) {
  switch (status) {
    case IGM_OK: return "IGM_OK";
    case IGM_ERR_BAD_SHAPE: return "IGM_ERR_BAD_SHAPE";
    case IGM_ERR_BAD_ARGUMENT: return "IGM_ERR_BAD_ARGUMENT";
    case IGM_ERR_NAN_DETECTED: return "IGM_ERR_NAN_DETECTED";
    case IGM_ERR_NOT_CONVERGED: return "IGM_ERR_NOT_CONVERGED";
    case IGM_ERR_CUDA: return "IGM_ERR_CUDA";
    case IGM_ERR_UNSUPPORTED: return "IGM_ERR_UNSUPPORTED";
    case IGM_ERR_WORKSPACE: return "IGM_ERR_WORKSPACE";
    default: return "IGM_ERR_UNKNOWN";
  }
}

extern "C" const char* igm_last_error(void) { return igm::g_last_error; }

extern "C" int igm_version(void) { return 100; }
