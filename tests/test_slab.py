"""The slab decomposition of the step (hydrocode_astro1_b200/slab.py) on the
CPU: slabs backed by the oracle, in one process and as gloo ranks of a
process group, step bit for bit as the oracle's single grid (state and every
dt; with self-gravity also the potential, the SOR iteration count and the
final update norm) -- the decomposition reproduces the reference's step
exactly, since each slab's planes see the same neighbours and the same dt,
the moment sums run in the reference's cell order across the slabs, and the
red-black half sweeps see the same neighbour values."""
import os
import socket

import numpy as np
import pytest

import ics
from oracle.oracle import OracleSim

torch = pytest.importorskip("torch")
from hydrocode_astro1_b200 import slab  # noqa: E402
from slab_oracle import OracleSlab, TreeOracleSlab, gloo_worker  # noqa: E402

BC = (1, 2, 2, 1, 1, 2)   # reflective and outflow faces, no periodic x
GRAV = dict(G=1.0, gamma=2.0, cfl=0.3, omega=1.7, tol=1e-7, max_iter=3000)
GBC = (2, 2, 2, 2, 2, 2)


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


def single_gravity(shape, steps):
    q0 = ics.gravity_blob(shape)
    o = OracleSim(*shape, bc=GBC, **GRAV)
    o.set_state(q0)
    d, its, res = o.step(steps)
    return o.state(), o.phi.copy(), d, its, res


@pytest.mark.parametrize("parts", [2, 3])
def test_local_slabs_with_gravity_match_single_grid(parts):
    """Three self-gravitating steps (the first solve from a zero potential,
    the later ones warm-started); 17 planes in 3 slabs puts odd global
    offsets on two of them."""
    shape, steps = (17, 12, 14), 3
    ref, phi, dts, its, res = single_gravity(shape, steps)
    assert its.min() > 10   # every solve iterates
    q0 = ics.gravity_blob(shape)
    slabs = [OracleSlab(shape, e, bc=GBC, **GRAV) for e in slab.plan(shape[0], parts)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    got_dt = [comm.step() for _ in range(steps)]
    assert np.array_equal(np.array(got_dt), dts)
    assert np.array_equal(np.concatenate([s.own_state() for s in slabs], axis=1), ref)
    assert np.array_equal(np.concatenate([s.own_phi() for s in slabs], axis=0), phi)
    for s in slabs:
        assert s.o.g.last_iter == its[-1] and s.o.g.last_res == res[-1]


def test_gravity_solve_stops_at_max_iter_like_single_grid():
    """A solve capped below convergence: every slab reports the cap and the
    last iteration's norm, and the step keeps the previous acceleration."""
    shape, steps = (15, 11, 12), 2
    kw = dict(GRAV, max_iter=6)
    q0 = ics.gravity_blob(shape)
    o = OracleSim(*shape, bc=GBC, **kw)
    o.set_state(q0)
    d, its, res = o.step(steps)
    slabs = [OracleSlab(shape, e, bc=GBC, **kw) for e in slab.plan(shape[0], 2)]
    for s in slabs:
        s.set_state(q0)
    comm = slab.LocalComm(slabs)
    got_dt = [comm.step() for _ in range(steps)]
    assert np.array_equal(np.array(got_dt), d)
    assert np.array_equal(np.concatenate([s.own_state() for s in slabs], axis=1), o.state())
    assert all(s.o.g.last_iter == 6 == its[-1] and s.o.g.last_res == res[-1] for s in slabs)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_with_gravity_match_single_grid(world, tmp_path):
    shape, steps = (16, 10, 12), 2
    ref, phi, dts, its, res = single_gravity(shape, steps)
    torch.multiprocessing.spawn(gloo_worker,
                                args=(world, free_port(), shape, steps, GBC, str(tmp_path), GRAV),
                                nprocs=world, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)], axis=1)
    got_phi = np.concatenate([np.load(tmp_path / f"phi{r}.npy") for r in range(world)], axis=0)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"dt{r}.npy"), dts)
        it, rr = np.load(tmp_path / f"it{r}.npy")
        assert it == its[-1] and rr == res[-1]
    assert np.array_equal(got, ref)
    assert np.array_equal(got_phi, phi)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_tree_moments_match_one_slab(world, tmp_path):
    """The tree form of the moment protocol (per-plane partials, gathered in
    plane order with ProcessGroupComm.gather's padded all-gather, added in
    plane order) as 2 and 3 gloo ranks against the same order on one slab
    of the whole grid: state, potential, dt, iterations and final norm bit
    for bit."""
    shape, steps = (16, 10, 12), 2
    q0 = ics.gravity_blob(shape)
    one = TreeOracleSlab(shape, slab.plan(shape[0], 1)[0], bc=GBC, **GRAV)
    one.set_state(q0)
    comm = slab.LocalComm([one])
    dts = [comm.step() for _ in range(steps)]
    torch.multiprocessing.spawn(gloo_worker,
                                args=(world, free_port(), shape, steps, GBC, str(tmp_path), GRAV, True),
                                nprocs=world, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{r}.npy") for r in range(world)], axis=1)
    got_phi = np.concatenate([np.load(tmp_path / f"phi{r}.npy") for r in range(world)], axis=0)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"dt{r}.npy"), np.array(dts))
        it, rr = np.load(tmp_path / f"it{r}.npy")
        assert it == one.o.g.last_iter and rr == one.o.g.last_res
    assert np.array_equal(got, one.own_state())
    assert np.array_equal(got_phi, one.own_phi())
