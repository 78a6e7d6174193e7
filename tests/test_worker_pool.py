"""The persistent host worker pool of the batched solves
(pyqcm_b200/csrc/worker_pool.hpp): every index of every batch runs exactly once,
with the pool reused across batches, its size changing between calls, and batch
calls arriving from several host threads at once. Host code, compiled here."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pyqcm_b200", "csrc")

DRIVER = r"""
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>
#include "worker_pool.hpp"
int main() {
  // like the library's pools: never destroyed, its detached threads live until exit
  qed::WorkerPool &pool = *new qed::WorkerPool;
  int bad = 0;
  auto batch = [&](int n, int extra) {
    std::vector<std::atomic<int>> hits(n);
    for (auto &h : hits) h = 0;
    std::atomic<int> next{0};
    pool.run(extra, [&] { for (int i = next++; i < n; i = next++) hits[i]++; });
    int b = 0;
    for (auto &h : hits) if (h.load() != 1) ++b;
    return b;
  };
  for (int r = 0; r < 300; ++r) bad += batch(1 + (r * 37) % 2000, r % 17);
  std::vector<std::thread> callers;
  std::atomic<int> bad2{0};
  for (int c = 0; c < 4; ++c)
    callers.emplace_back([&, c] { for (int r = 0; r < 50; ++r) bad2 += batch(500 + c, (r + c) % 9); });
  for (auto &t : callers) t.join();
  printf("%d %d\n", bad, bad2.load());
  fflush(stdout);
  return (bad || bad2) ? 1 : 0;
}
"""


def test_worker_pool_runs_every_index_once():
    d = tempfile.mkdtemp(prefix="worker_pool_")
    src = os.path.join(d, "drv.cpp")
    exe = os.path.join(d, "drv")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, src, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["0", "0"]
