"""The slab decomposition of the hydro step (hydrocode_astro1_b200/slab.py)
on the CPU: slabs backed by the oracle, in one process and as gloo ranks of a
process group, step bit for bit as the oracle's single grid (state and every
dt) -- the decomposition reproduces the reference's step exactly, since each
slab's planes see the same neighbours and the same dt."""
import os
import socket

import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim

torch = pytest.importorskip("torch")
from hydrocode_astro1_b200 import slab  # noqa: E402
from slab_oracle import OracleSlab, gloo_worker  # noqa: E402

BC = (1, 2, 2, 1, 1, 2)   # reflective and outflow faces, no periodic x


def single(shape, steps):
    q0 = ics.smooth_random(shape, seed=21)
    o = OracleSim(*shape, cfl=0.35, bc=BC)
    o.set_state(q0)
    d, _, _ = o.step(steps)
    return o.state(), d


def test_plan_partitions_the_planes():
    for nx, parts in ((10, 1), (10, 3), (64, 4), (23, 7)):
        p = slab.plan(nx, parts)
        assert p[0]["own"][0] == 0 and p[-1]["own"][1] == nx
        for a, b in zip(p[:-1], p[1:]):
            assert a["own"][1] == b["own"][0]
            assert a["local"][1] == a["own"][1] + 1 and b["local"][0] == b["own"][0] - 1
        assert all(e["local"][1] - e["local"][0] >= 3 for e in p)
    with pytest.raises(ValueError):
        slab.plan(8, 3)


@pytest.mark.parametrize("parts", [2, 3])
def test_local_slabs_match_single_grid(parts):
    shape, steps = (21, 9, 11), 8
    ref, dts = single(shape, steps)
    q0 = ics.smooth_random(shape, seed=21)
    slabs = [OracleSlab(shape, e, cfl=0.35, bc=BC) for e in slab.plan(shape[0], parts)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    got_dt = [comm.step() for _ in range(steps)]
    assert np.array_equal(np.array(got_dt), dts)
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    assert np.array_equal(got, ref)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_single_grid(world, tmp_path):
    shape, steps = (19, 8, 10), 6
    ref, dts = single(shape, steps)
    torch.multiprocessing.spawn(gloo_worker, args=(world, free_port(), shape, steps, BC, str(tmp_path)),
                                nprocs=world, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)], axis=1)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"dt{r}.npy"), dts)
    assert np.array_equal(got, ref)
