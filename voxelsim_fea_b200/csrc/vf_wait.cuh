// Bounded waits on shared-memory mbarriers (TMA pipelines).
//
// A wait polls mbarrier.try_wait.parity with a suspend-time hint of
// kPollHintNs nanoseconds (the PTX operand is in ns: the thread may sleep up
// to that long per poll when the phase is not yet complete) and gives up
// after kWaitLimitNs of %globaltimer time or kMaxPolls polls, whichever comes
// first.  The poll cap alone bounds the wait: kMaxPolls x kPollHintNs <= 1 s.
// On expiry the caller raises the kernel's error flag, drains its own copies
// in flight (again bounded) and returns; the host turns the flag into a
// status.
#pragma once

#include <stdint.h>

namespace vf {

constexpr unsigned kPollHintNs = 2000u;                  // 2 us per poll at most
constexpr unsigned long long kWaitLimitNs = 1000000000ull;   // 1 s of wall time
constexpr unsigned kMaxPolls = 500000u;
static_assert((unsigned long long)kMaxPolls * kPollHintNs <= kWaitLimitNs,
              "polls x hint must stay within the 1 s wait limit");

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"((unsigned)__cvta_generic_to_shared(bar)), "r"(parity), "r"(kPollHintNs)
      : "memory");
  return ok != 0;
}

// true: the phase with this parity completed; false: the wait expired.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait_hint(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned i = 1; i < kMaxPolls; ++i) {
    if (mbar_try_wait_hint(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
  return false;
}

}  // namespace vf
