"""The host copy pool behind pageable callers' staging copies (csrc/copy_pool.hpp).

Compiled with g++ into a small driver and run on the CPU: copies of many sizes
and misaligned offsets, several groups in flight at once, a group waited for by
its scope guard, and worker counts from none to eight must each give a byte-exact
copy and leave no slice running after wait() returns; parallel_for must visit
every index exactly once."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpgpu-binary-automaton-synchronizing-algorithms_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "copy_pool.hpp"
using sbfs::CopyPool;
static int check(const std::vector<char> &a, const std::vector<char> &b, size_t off, size_t n) {
    for (size_t i = 0; i < n; ++i) if (a[off + i] != b[off + i]) return 1;
    return 0;
}
int main() {
    std::mt19937_64 rng(7);
    const size_t sizes[] = {0, 1, 63, 1000, (256u << 10) - 1, 256u << 10, (3u << 20) + 13, (24u << 20) + 5};
    int bad = 0;
    for (int workers : {0, 1, 3, 8}) {
        CopyPool pool(workers);
        for (size_t n : sizes) {
            for (size_t off : {size_t(0), size_t(5)}) {
                std::vector<char> src(n + off + 8), dst(n + off + 8, 0);
                for (auto &c : src) c = (char)rng();
                CopyPool::Group g;
                pool.copy(dst.data() + off, src.data() + off, n, g);
                pool.wait(g);
                bad += check(src, dst, off, n);
                for (size_t i = 0; i < off; ++i) bad += dst[i] != 0;       // nothing before
                for (size_t i = off + n; i < dst.size(); ++i) bad += dst[i] != 0;   // nothing after
            }
        }
        // three groups in flight, waited for in reverse order
        const size_t n = (5u << 20) + 77;
        std::vector<char> s[3], d[3];
        CopyPool::Group g[3];
        for (int i = 0; i < 3; ++i) {
            s[i].resize(n); d[i].assign(n, 0);
            for (auto &c : s[i]) c = (char)rng();
            pool.copy(d[i].data(), s[i].data(), n, g[i]);
        }
        for (int i = 2; i >= 0; --i) { pool.wait(g[i]); bad += check(s[i], d[i], 0, n); }
        // the scope guard waits on leaving the block
        std::vector<char> s2((7u << 20) + 3), d2(s2.size(), 0);
        for (auto &c : s2) c = (char)rng();
        {
            CopyPool::Group g2;
            CopyPool::Scope guard{&pool, g2};
            pool.copy(d2.data(), s2.data(), s2.size(), g2);
        }
        bad += check(s2, d2, 0, s2.size());
        // parallel_for visits every index exactly once, in disjoint parts
        for (size_t n : {size_t(0), size_t(1), size_t(100), size_t(12345), size_t(1) << 20}) {
            std::vector<int> hit(n, 0);
            pool.parallel_for(n, 1000, [&](size_t a, size_t b) { for (size_t i = a; i < b; ++i) hit[i] += 1; });
            for (size_t i = 0; i < n; ++i) bad += hit[i] != 1;
        }
    }
    std::printf("default_workers=%d bad=%d\n", CopyPool::default_workers(), bad);
    return bad ? 1 : 0;
}
"""


def test_copy_pool_copies_exactly(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    cc = subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    if cc.returncode != 0 and "not found" in cc.stderr:
        pytest.skip("no g++")
    assert cc.returncode == 0, cc.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "bad=0" in run.stdout
