"""Per-device bookkeeping of the library's device-side state (per_device.h).

The __constant__ spherical-harmonics tables, the tcgen05 GEMM's status word
and the addresses of the static scratch arrays exist once per device. Their
host-side tables are PerDevice<T>, keyed by the device ordinal that is
current when the state is needed. Only one GPU is available to the tests, so
the two-device case is checked here on the host: the header is plain C++
and is compiled with g++ into a small program that drives two ordinals.
"""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "librascal_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <stdexcept>
#include "per_device.h"

#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d: %s\n", __LINE__, #c); return 1; } } while (0)

int main() {
  using rgpu::PerDevice;
  static PerDevice<int *> status;  // stands in for a per-device status word
  int on0 = 0, on1 = 0;
  int inits = 0;
  // device 0 first, then device 1: each gets its own slot, set up once
  int * p0 = status.once(0, [&](int *& p) { p = &on0; ++inits; });
  int * p1 = status.once(1, [&](int *& p) { p = &on1; ++inits; });
  CHECK(p0 == &on0 && p1 == &on1 && inits == 2);
  CHECK(status.once(0, [&](int *& p) { p = nullptr; ++inits; }) == &on0);  // no second set-up
  CHECK(status.once(1, [&](int *& p) { p = nullptr; ++inits; }) == &on1);
  CHECK(inits == 2);
  CHECK(status.ready(0) && status.ready(1) && !status.ready(2));
  // a set-up that fails leaves the slot unready, so the next call retries
  static PerDevice<char> filled;
  bool threw = false;
  try {
    filled.once(3, [](char &) { throw std::runtime_error("cudaMemcpyToSymbol failed"); });
  } catch (const std::runtime_error &) { threw = true; }
  CHECK(threw && !filled.ready(3));
  int calls = 0;
  filled.once(3, [&](char & c) { c = 1; ++calls; });
  CHECK(calls == 1 && filled.ready(3) && filled.at(3) == 1 && filled.at(0) == 0);
  // ordinals outside the table are errors, not out-of-bounds writes
  bool oob = false;
  try { status.at(rgpu::kMaxDevices); } catch (const std::out_of_range &) { oob = true; }
  CHECK(oob);
  oob = false;
  try { status.at(-1); } catch (const std::out_of_range &) { oob = true; }
  CHECK(oob);
  std::printf("ok\n");
  return 0;
}
"""


def test_per_device_tables_keep_devices_apart():
    gxx = "g++"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "per_device_test.cpp")
        exe = os.path.join(d, "per_device_test")
        with open(src, "w") as f:
            f.write(PROGRAM)
        try:
            subprocess.run([gxx, "-std=c++17", "-O1", "-I" + CSRC, src, "-o", exe, "-pthread"], check=True,
                           capture_output=True, text=True)
        except FileNotFoundError:
            pytest.skip("no host C++ compiler")
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.strip() == "ok"


def test_device_state_uses_per_device_tables():
    """Every once-per-device set-up in the CUDA sources goes through a
    PerDevice table: no process-wide 'done' flag or cached device pointer."""
    import re
    offenders = []
    for name in os.listdir(CSRC):
        if not name.endswith((".cu", ".cuh", ".h")):
            continue
        text = open(os.path.join(CSRC, name)).read()
        for m in re.finditer(r"static\s+(bool|int|\w+\s*\*)\s+\w+\s*=\s*(false|nullptr|0)\s*;", text):
            offenders.append("%s: %s" % (name, m.group(0)))
        # device buffers kept across calls belong to a device
        for m in re.finditer(r"static\s+(thread_local\s+)?DevBuf\b[^;]*;", text):
            offenders.append("%s: %s" % (name, m.group(0)))
    assert not offenders, offenders
    common = open(os.path.join(CSRC, "common.cuh")).read()
    assert "PerDevice<char> g_sph_filled" in common
    assert "PerDevice<TcStatus *>" in open(os.path.join(CSRC, "gemm_tc.cu")).read()
    assert "PerDevice<DevicePointers>" in open(os.path.join(CSRC, "noalloc.cu")).read()
