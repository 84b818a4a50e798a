"""The batch pool's range allocator (csrc/hj_ranges.h) on the CPU.

A small driver compiled with g++ replays a random admit/retire sequence like
serving's churn. After every step: the free ranges are sorted, disjoint and
never adjacent; they and the live bunches tile the pool exactly; every
admission takes the first free range that fits, rounded to a multiple of 4;
and a refusal happens only when no free range fits."""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "haissinskijulia_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "hj_ranges.h"
int main() {
  long long pool;
  if (scanf("%lld", &pool) != 1) return 1;
  hj_ranges::Ranges fr{{0, (int64_t)pool}};
  char op;
  long long a, b;
  while (scanf(" %c %lld %lld", &op, &a, &b) == 3) {
    if (op == 't') {
      int64_t s = -1, c = 0;
      bool ok = hj_ranges::take(fr, a, &s, &c);
      printf("%d %lld %lld", ok ? 1 : 0, (long long)s, (long long)c);
    } else {
      hj_ranges::give(fr, a, b);
      printf("g");
    }
    printf(" | %lld", (long long)hj_ranges::largest(fr));
    for (auto& r : fr) printf(" %lld:%lld", (long long)r.first, (long long)r.second);
    printf("\n");
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("ranges")
    src = d / "ranges.cpp"
    src.write_text(DRIVER)
    exe = d / "ranges"
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    return str(exe)


def _run(exe, pool, ops):
    text = f"{pool}\n" + "".join(f"{o} {a} {b}\n" for o, a, b in ops)
    out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True)
    return out.stdout.splitlines()


def _parse(line):
    head, tail = line.split(" | ")
    parts = tail.split()
    largest = int(parts[0])
    free = [tuple(int(v) for v in p.split(":")) for p in parts[1:]]
    return head.split(), largest, free


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_admit_and_retire(driver, seed):
    rng = random.Random(seed)
    pool = 4000
    live = {}                       # start -> cap
    ops, expect = [], []
    # build the op list on a Python model, then replay it in the driver
    free = [(0, pool)]
    for _ in range(600):
        if live and (rng.random() < 0.45 or len(live) > 40):
            s = rng.choice(sorted(live))
            c = live.pop(s)
            ops.append(("g", s, c))
            free.append((s, c))
            free.sort()
            merged = []
            for r in free:
                if merged and merged[-1][0] + merged[-1][1] == r[0]:
                    merged[-1] = (merged[-1][0], merged[-1][1] + r[1])
                else:
                    merged.append(r)
            free = merged
            expect.append(None)
        else:
            n = rng.choice([1, 3, 4, 5, 17, 64, 250, 999])
            need = max((n + 3) // 4 * 4, 4)
            fit = next((r for r in free if r[1] >= need), None)
            ops.append(("t", n, 0))
            if fit is None:
                expect.append((0, None, None))
            else:
                i = free.index(fit)
                live[fit[0]] = need
                free[i] = (fit[0] + need, fit[1] - need)
                if free[i][1] == 0:
                    free.pop(i)
                expect.append((1, fit[0], need))
    lines = _run(driver, pool, ops)
    assert len(lines) == len(ops)
    live = {}
    for (op, a, b), want, line in zip(ops, expect, lines):
        head, largest, fr = _parse(line)
        if op == "t":
            ok, s, c = int(head[0]), int(head[1]), int(head[2])
            assert ok == want[0]
            if ok:
                assert (s, c) == (want[1], want[2]) and s % 4 == 0
                live[s] = c
            else:                   # refused only when nothing fits
                need = max((a + 3) // 4 * 4, 4)
                assert all(length < need for _, length in fr)
        else:
            del live[a]
        # sorted, disjoint, never adjacent; free + live tile the pool
        for (s0, l0), (s1, _) in zip(fr, fr[1:]):
            assert s0 + l0 < s1
        assert largest == max((length for _, length in fr), default=0)
        pieces = sorted(fr + list(live.items()))
        pos = 0
        for s, length in pieces:
            assert s == pos and length > 0
            pos += length
        assert pos == pool
