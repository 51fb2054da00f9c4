"""The learned-start outcome monitor (csrc/unet_guard.h), on the CPU.

The policy header is CUDA-free; it is compiled here with g++ into a small
shared library and driven with synthetic sequences of solves: a network that
wins clearly (probes become rare, it stays on), one that loses (switched off
after K consecutive losses, retried with back-off), and one that recovers
(switched back on by a winning retry).
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "hydrocode_astro1_b200", "csrc")

DRIVER = r"""
#include "unet_guard.h"
static hc::UnetGuard g;
extern "C" void reset(int K) { g = hc::UnetGuard(); g.K = K; }
extern "C" int allows() { return hc::unet_guard_allows(g) ? 1 : 0; }
extern "C" void record(int predicted, int iters) { hc::unet_guard_record(g, predicted != 0, iters); }
extern "C" void stats(long long *o) {
    o[0] = g.probes; o[1] = g.wins; o[2] = g.loss_total; o[3] = g.switch_offs; o[4] = g.off;
}
"""


@pytest.fixture(scope="module")
def guard(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("guard")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    so = d / "libguard.so"
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I", HDR, str(src), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.stats.argtypes = [C.POINTER(C.c_longlong)]
    return L


def stats(L):
    o = (C.c_longlong * 5)()
    L.stats(o)
    return dict(zip(("probes", "wins", "losses", "switch_offs", "off"), o))


def run(L, K, n, cost):
    """n solves; cost(predicted, solve_index) -> SOR iterations.  A solve
    that is allowed a prediction takes it (always accepted here)."""
    L.reset(K)
    kinds = []
    for t in range(n):
        pred = bool(L.allows())
        L.record(int(pred), cost(pred, t))
        kinds.append(pred)
    return kinds


def test_monitor_off_changes_nothing(guard):
    kinds = run(guard, 0, 50, lambda p, t: 100)
    assert all(kinds) and stats(guard)["probes"] == 0


def test_clear_win_probes_rarely(guard):
    # the prediction needs 8% of the plain iterations (the 256^3 explosion)
    kinds = run(guard, 3, 2000, lambda p, t: 90 if p else 1100)
    st = stats(guard)
    assert st["off"] == 0 and st["switch_offs"] == 0
    plain = [t for t, k in enumerate(kinds) if not k]
    assert plain[0] == 2                  # the first probe right after the first prediction
    assert 3 <= len(plain) <= 6, plain    # then after 64, 128, 256, ... predicted solves
    assert all(kinds[3:66])               # none in the steps after a short warm-up


def test_losing_network_switches_off_and_backs_off(guard):
    # accepted predictions that cost 9% more than the previous potential
    kinds = run(guard, 3, 200, lambda p, t: 545 if p else 500)
    st = stats(guard)
    assert st["switch_offs"] == 1 and st["off"] == 1
    first_off = next(t for t in range(3, 200) if not any(kinds[t:t + 10]))
    assert first_off <= 8, kinds[:12]
    # retries after 16, 32, 64, ... plain solves: few predicted solves overall
    assert sum(kinds) <= 9, sum(kinds)


def test_recovering_network_comes_back(guard):
    # loses for the first 40 solves, then wins clearly
    kinds = run(guard, 2, 300, lambda p, t: (600 if t < 40 else 50) if p else 500)
    st = stats(guard)
    assert st["switch_offs"] >= 1 and st["off"] == 0
    assert all(kinds[150:250])
