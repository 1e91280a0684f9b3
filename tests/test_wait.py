"""The bounded wait behind pf_config.wait_timeout_us (goav1_b200/csrc/pf_wait.h)
on the CPU: a readiness query that stalls makes the deadline run out
(kWaitTimedOut after the deadline, not before), one that becomes ready ends
the wait, one that fails reports the failure.  The header is compiled into a
small host program with the system C++ compiler; no device is involved."""

import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <chrono>
#include <cstdio>
#include "pf_wait.h"
int main() {
  using namespace pf;
  using clock = std::chrono::steady_clock;
  int n = 0;
  const int r1 = wait_until([&]() { return ++n >= 10 ? (int)kWaitReady : (int)kWaitPending; }, 1000000);
  int polls = 0;
  const clock::time_point t0 = clock::now();
  const int r2 = wait_until([&]() { polls++; return (int)kWaitPending; }, 20000);  // a stall: never ready
  const double ms = std::chrono::duration<double, std::milli>(clock::now() - t0).count();
  const int r3 = wait_until([&]() { return (int)kWaitFailed; }, 1000);
  int once = 0;
  const int r4 = wait_until([&]() { once++; return (int)kWaitReady; }, 0);
  std::printf("%d %d %d %d %d %d %d %.3f\n", r1, n, r2, polls, r3, r4, once, ms);
  return 0;
}
"""


@pytest.fixture(scope="module")
def results():
    cxx = os.environ.get("CXX", "g++")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "wait.cpp"), os.path.join(d, "wait")
        with open(src, "w") as f:
            f.write(HARNESS)
        subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "goav1_b200", "csrc"), src, "-o", exe,
                        "-lpthread"], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(v) for v in out[:7]] + [float(out[7])]


def test_ready_query_ends_the_wait(results):
    r1, n = results[0], results[1]
    assert (r1, n) == (0, 10)


def test_stalled_query_times_out_at_the_deadline(results):
    r2, polls, ms = results[2], results[3], results[7]
    assert r2 == 1  # kWaitTimedOut
    assert ms >= 20.0 and ms < 2000.0, ms
    assert polls > 1


def test_failed_query_and_zero_deadline(results):
    r3, r4, once = results[4], results[5], results[6]
    assert r3 == 2  # kWaitError
    assert (r4, once) == (0, 1)  # a zero deadline still polls once
