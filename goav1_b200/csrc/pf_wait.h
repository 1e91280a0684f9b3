// pf_wait.h - bounded waits for the library's synchronous calls.
//
// A call that returns only when its device work is done (pf_sync, a host
// frame's pf_frame_apply, the searches) waits on a CUDA stream or event.  A
// context created with pf_config.wait_timeout_us > 0 polls instead of
// blocking and gives up at the deadline with PF_ERR_TIMEOUT, so a caller on a
// real-time thread (a decoder that must present a frame) regains control
// when the device stalls.  The work stays queued: a later pf_sync (or
// pf_destroy) waits for it.
//
// wait_until is plain host code over a readiness query, so it is exercised
// on the CPU with a query that stalls (tests/test_wait.py).
#pragma once

#include <stdint.h>

#include <chrono>
#include <thread>

namespace pf {

enum WaitQuery { kWaitReady = 0, kWaitPending = 1, kWaitFailed = 2 };
enum WaitResult { kWaitDone = 0, kWaitTimedOut = 1, kWaitError = 2 };

// Polls query() until it reports kWaitReady (kWaitDone) or kWaitFailed
// (kWaitError), or until timeout_us microseconds have passed since the call
// (kWaitTimedOut); the query is polled at least once.  Polls back off from
// yielding to sleeps of up to 50 us, so a long wait costs little CPU.
template <class Query>
int wait_until(Query query, int64_t timeout_us) {
  using clock = std::chrono::steady_clock;
  const clock::time_point deadline = clock::now() + std::chrono::microseconds(timeout_us);
  for (int polls = 0;; polls++) {
    const int q = query();
    if (q == kWaitReady) return kWaitDone;
    if (q == kWaitFailed) return kWaitError;
    if (clock::now() >= deadline) return kWaitTimedOut;
    if (polls < 64)
      std::this_thread::yield();
    else
      std::this_thread::sleep_for(std::chrono::microseconds(polls < 256 ? 5 : 50));
  }
}

}  // namespace pf
