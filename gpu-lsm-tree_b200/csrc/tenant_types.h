// Plain data shared by the multi-tenant host engine and its kernels.
#pragma once

#include <cstdint>

namespace gpulsm {
namespace tenants {

constexpr uint32_t kMaxFenceLevels = 8;

// Per-tenant placement and state (device resident).
struct TenantMeta {
  unsigned long long cap;        // rows per run buffer
  unsigned long long main_off;   // arena offset of main buffer 0 (buffer 1 follows at +cap)
  unsigned long long delta_off;  // arena offset of delta buffer 0
  unsigned long long fence_off;  // fence arena offset (main fences, then delta fences)
  unsigned long long fence_cap;  // fence entries reserved per run
  uint32_t main_n, delta_n;
  uint32_t main_cur, delta_cur;  // which buffer holds the live run
};

struct Arena {
  uint32_t *keys;
  uint32_t *vals;
  uint32_t *fences;
};

}  // namespace tenants
}  // namespace gpulsm
