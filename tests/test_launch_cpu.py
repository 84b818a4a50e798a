"""The fused pass's thread layouts and grid rule (csrc/hj_launch.h) on the CPU.

A driver compiled with g++ evaluates track_grid_size over bunch sizes up to
1e10 particles, every layout and bin count. For each it counts the particles
block 0 deposits per turn: block 0 takes the most groups (the groups of PPT
particles b·T + t + k·g·T), plus the n mod PPT tail. The test checks that
count stays within the packed cell counter's bound (kMaxBlockParticles), that
the grid is positive, and that below one wave of blocks the grid is no
larger than one block per B/2 particles."""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "haissinskijulia_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "hj_launch.h"
int main() {
  long long n; int B, sms, bps, cfg;
  printf("%lld\n", (long long)hj::kMaxBlockParticles);
  while (scanf("%lld %d %d %d %d", &n, &B, &sms, &bps, &cfg) == 5) {
    if (!hj::pass_cfg_valid(cfg)) { printf("invalid\n"); continue; }
    const int g = hj::track_grid_size(n, B, sms, bps, cfg);
    const long long T = hj::pass_cfg_threads(cfg), P = hj::pass_cfg_ppt(cfg);
    const long long ng = n / P, gt = (long long)g * T;
    long long groups0 = 0;
    for (long long t = 0; t < T && t < ng; ++t) groups0 += (ng - t + gt - 1) / gt;
    printf("%d %lld\n", g, groups0 * P + (n - ng * P));
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("launch")
    src = d / "launch.cpp"
    src.write_text(DRIVER)
    exe = d / "launch"
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return str(exe)


def _run(exe, cases):
    text = "".join(f"{n} {B} {s} {b} {c}\n" for n, B, s, b, c in cases)
    out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True)
    lines = out.stdout.splitlines()
    return int(lines[0]), lines[1:]


def test_block_deposits_stay_within_the_cell_counter(driver):
    rng = random.Random(5)
    sizes = [1, 2, 3, 4, 5, 31, 33, 1000, 4096, 10**5, 10**6, 10**8, 148 * 2**20,
             2 * 10**9, 2**32 + 65_538, 2**33 + 7, 10**10]
    sizes += [rng.randrange(1, 2 * 10**10) for _ in range(300)]
    layouts = [0, 1, 2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 16, 21, 24, 29]
    cases = [(n, B, 148, bps, c) for n in sizes for B in (64, 4096, 16384)
             for bps in (1, 2) for c in layouts]
    kmax, lines = _run(driver, cases)
    assert kmax == 2**20 - 8
    for (n, B, sms, bps, c), line in zip(cases, lines):
        g, per_block = (int(v) for v in line.split())
        assert g >= 1
        assert per_block <= kmax, (n, B, bps, c, g, per_block)
        if g < sms * bps:                     # below one wave: >= B/2 particles a block
            assert g <= max(1, -(-n // max(B // 2, 1))), (n, B, c, g)


def test_invalid_layouts(driver):
    _, lines = _run(driver, [(1000, 64, 148, 1, c) for c in (-2, 6, 7, 14, 15, 22, 23, 32)])
    assert lines == ["invalid"] * 8
