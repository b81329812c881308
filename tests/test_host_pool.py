"""The host thread pool behind host_parallel (this_studio_b200/csrc/common.cuh,
HostPool): every index of every job is run exactly once with several callers
submitting at once and jobs submitted from inside a chunk, and a child made
by fork() while the parent's workers are busy completes its own jobs.  Host
code only: compiled with nvcc and run without a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

PROGRAM = r"""
#include "common.cuh"
#include <sys/wait.h>
#include <unistd.h>
using namespace demsph;

static long once(long n, bool nested) {
    std::vector<int> hit(n, 0);
    std::atomic<long> bad{0};
    host_parallel(n, [&](long a, long b) {
        for (long i = a; i < b; i++) hit[i]++;
        if (nested) {
            std::vector<int> h2(70000, 0);
            host_parallel(70000, [&](long x, long y) { for (long i = x; i < y; i++) h2[i]++; });
            for (int v : h2) bad += v != 1;
        }
    });
    for (int v : hit) bad += v != 1;
    return bad;
}

int main() {
    std::atomic<long> bad{0};
    std::vector<std::thread> callers;
    for (int c = 0; c < 6; c++)
        callers.emplace_back([&, c] {
            for (int rep = 0; rep < 200; rep++) bad += once(100000 + 7919 * ((13 * rep + c) % 50), rep % 8 == 0);
        });
    for (auto& t : callers) t.join();
    std::atomic<bool> stop{false};
    std::thread busy([&] { while (!stop) bad += once(300000, false); });
    for (int k = 0; k < 10; k++) {
        pid_t pid = fork();
        if (pid == 0) _exit(once(400000, false) + once(200000, true) == 0 ? 0 : 1);
        int st = 0;
        waitpid(pid, &st, 0);
        if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad++;
    }
    stop = true;
    busy.join();
    std::printf("bad %ld\n", bad.load());
    return bad.load() != 0;
}
"""


@pytest.mark.skipif(not shutil.which(NVCC) and not os.path.exists(NVCC), reason="nvcc not found")
def test_host_pool_runs_every_chunk_once(tmp_path):
    src = tmp_path / "pool.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "pool"
    cmd = [NVCC, "-O2", "-std=c++17", "-Xcompiler", "-pthread", "-I" + os.path.join(ROOT, "this_studio_b200", "csrc"),
           str(src), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "bad 0" in r.stdout, r.stdout + r.stderr
