// Debug support: the guard regions of the guard build (see DevBuf) and the
// query of their violation count, present in every build.
#include <atomic>
#include <cstdio>
#include <vector>

#include "pls_internal.hpp"

namespace pls {

#ifdef PLS_DEBUG_GUARDS
namespace {
std::atomic<int64_t> g_guard_violations{0};
}  // namespace

// The fill is synchronous: the library's kernels run on non-blocking streams
// that do not wait for the legacy stream a plain cudaMemset uses.
void guard_arm(void *end) {
  PLS_CUDA(cudaMemset(end, 0xFF, kGuardBytes));
  PLS_CUDA(cudaDeviceSynchronize());
}

// Called from destructors: reports through the counter and stderr, never
// throws. The device is synchronised first, so the kernels that used the
// buffer have finished.
void guard_check(const void *end) noexcept {
  std::vector<unsigned char> h(kGuardBytes);
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(h.data(), end, kGuardBytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  for (size_t i = 0; i < kGuardBytes; ++i)
    if (h[i] != 0xFF) {
      g_guard_violations.fetch_add(1);
      std::fprintf(stderr, "plsparse_b200: a write past a device buffer's end, byte %zu of the guard\n", i);
      return;
    }
}
#endif

}  // namespace pls

extern "C" int64_t perflibs_b200_debug_guard_violations(void) {
#ifdef PLS_DEBUG_GUARDS
  return pls::g_guard_violations.load();
#else
  return -1;
#endif
}
