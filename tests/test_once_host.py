"""PerDeviceOnce (csrc/once.h): the per-device, thread-safe one-time set-up
that guards cudaFuncSetAttribute at every launch site.  A host-only C++
program (g++, no CUDA) drives it from several threads over several device
ordinals and checks that each device's set-up ran exactly once, that a
second device is not skipped because the first one is done, that a failed
set-up is retried, and that ordinals past the tracked range run every time."""
import subprocess
import textwrap
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

PROGRAM = textwrap.dedent(r"""
    #include <atomic>
    #include <cstdio>
    #include <stdexcept>
    #include <thread>
    #include <vector>
    #include "once.h"

    int main() {
      fdb::PerDeviceOnce once;
      std::atomic<int> runs[8];
      for (auto& r : runs) r = 0;
      std::vector<std::thread> ts;
      for (int t = 0; t < 16; ++t)
        ts.emplace_back([&, t] {
          for (int rep = 0; rep < 1000; ++rep) {
            const int dev = (t + rep) % 8;
            once(dev, [&] { runs[dev]++; });
          }
        });
      for (auto& th : ts) th.join();
      for (int d = 0; d < 8; ++d)
        if (runs[d] != 1 || !once.done(d)) { std::printf("device %d ran %d times\n", d, (int)runs[d]); return 1; }
      if (once.done(8)) { std::printf("device 8 marked done\n"); return 2; }

      // A set-up that throws leaves its device not done, and the next call retries.
      fdb::PerDeviceOnce again;
      int tries = 0;
      try { again(3, [&] { ++tries; throw std::runtime_error("x"); }); } catch (const std::runtime_error&) {}
      if (again.done(3)) return 3;
      again(3, [&] { ++tries; });
      again(3, [&] { ++tries; });
      if (tries != 2 || !again.done(3)) { std::printf("retry: %d\n", tries); return 4; }

      // Ordinals outside the tracked range are never remembered: set-up runs each time.
      int wide = 0;
      for (int i = 0; i < 3; ++i) again(fdb::PerDeviceOnce::kTracked + 1, [&] { ++wide; });
      again(-1, [&] { ++wide; });
      if (wide != 4) { std::printf("untracked: %d\n", wide); return 5; }
      std::puts("ok");
      return 0;
    }
""")


def test_per_device_once(tmp_path):
    src = tmp_path / "once_test.cpp"
    exe = tmp_path / "once_test"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", str(ROOT / "falcondb_b200" / "csrc"),
                    str(src), "-o", str(exe)], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
