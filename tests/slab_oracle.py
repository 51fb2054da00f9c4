"""A slab of the decomposition (hydrocode_astro1_b200/slab.py) backed by the
CPU oracle: test infrastructure, so that the decomposition protocol -- the
signal-speed maximum over slabs, the Poisson solve across slabs (moment
chain, half sweeps with ghost exchanges, the norm maximum), the step with
the whole grid's dt, the ghost plane exchange -- runs as gloo ranks on the
CPU and is compared with the oracle's single-grid step."""
import ctypes as C

import numpy as np
import torch

from oracle.oracle import OracleSim, _ptr


class OracleSlab:
    def __init__(self, shape, entry, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), **kw):
        nx, ny, nz = shape
        d = [(hi[t] - lo[t]) / shape[t] for t in range(3)]
        l0, l1 = entry["local"]
        a, b = entry["own"]
        self.entry = entry
        self.ny, self.nz = ny, nz
        self.nx_l = l1 - l0
        self.gnx = nx
        self.ioff = l0
        self.olo, self.ohi = a - l0, b - l0
        self.own_planes = b - a
        # the whole grid's bounds and cell sizes, bit for bit
        self.o = OracleSim(self.nx_l, ny, nz, lo=lo, hi=hi, **kw)
        self.o.g.dx, self.o.g.dy, self.o.g.dz = d
        self.gravity = kw.get("G", 0.0) > 0.0
        self.max_iter, self.tol = self.o.g.max_iter, self.o.g.tol
        self.cfl = kw.get("cfl", 0.4)
        self.smax = None
        self.mom = np.zeros(13)
        self.com = np.zeros(3)
        self._r0 = self._norm = 0.0

    def set_state(self, q_global):
        l0, l1 = self.entry["local"]
        self.o.set_state(q_global[:, l0:l1])

    def signal_speed(self):
        return self.o.lib.hco_signal_max(C.byref(self.o.g))

    def set_signal_speed(self, v):
        self.smax = v

    def step(self):
        g = self.o.g
        s = self.smax
        dt = self.cfl * min(g.dx / s, min(g.dy / s, g.dz / s))   # compute_dt_3d's arithmetic
        if self.gravity:
            self.o.lib.hco_step_ext(C.byref(g), dt)
        else:
            self.o.lib.hco_step_dt(C.byref(g), dt)
        return dt

    def get_planes(self, i0, count):
        return torch.from_numpy(np.ascontiguousarray(self.o.q[:, i0:i0 + count]))

    def set_planes(self, i0, t):
        self.o.q[:, i0:i0 + t.shape[1]] = t.numpy()

    # gravity: the reference's sequential moments, chained slab to slab
    def moment_layout(self, p):
        return True, (4 if p == 0 else 9)

    def moments(self, p, acc):
        acc = np.ascontiguousarray(acc, dtype=np.float64)
        self.o.lib.hco_moments_acc(C.byref(self.o.g), _ptr(self.o.q[0]), p, self.olo, self.ohi, self.ioff,
                                   _ptr(self.com), _ptr(acc))
        return acc

    def set_moments(self, p, acc, nplanes):
        acc = np.ascontiguousarray(acc, dtype=np.float64)
        if p == 0:
            self.o.lib.hco_moments_com(C.byref(self.o.g), _ptr(acc), _ptr(self.com))
            self.mom[0] = acc[0]
            self.mom[1:4] = self.com
        else:
            self.mom[4:] = acc

    def sor_begin(self):
        pass

    def sor_sweep(self, it, colour):
        r = self.o.lib.hco_sor_half(C.byref(self.o.g), _ptr(self.o.q[0]), colour ^ (self.ioff & 1))
        if colour == 0:
            self._r0 = r
        else:   # the reference's res = mx(mx(0, r_red), r_black)
            t = 0.0 if 0.0 > self._r0 else self._r0
            self._norm = t if t > r else r

    def sor_boundary(self):
        self.o.lib.hco_boundary_mom(C.byref(self.o.g), _ptr(self.mom), self.ioff, self.gnx, self.olo, self.ohi)

    def sor_norm(self, it):
        return self._norm

    def sor_end(self, used, res, conv):
        self.o.g.last_iter = used
        self.o.g.last_res = res
        if conv:
            self.o.lib.hco_gravity_acceleration(C.byref(self.o.g))

    def get_phi_planes(self, i0, count):
        return torch.from_numpy(np.ascontiguousarray(self.o.phi[i0:i0 + count]))

    def set_phi_planes(self, i0, t):
        self.o.phi[i0:i0 + t.shape[0]] = t.numpy()

    def own_state(self):
        return self.o.state()[:, self.olo:self.ohi]

    def own_phi(self):
        return self.o.phi[self.olo:self.ohi].copy()


class TreeOracleSlab(OracleSlab):
    """The oracle slab with the tree form of the moment protocol: one
    partial per own plane (the reference's sums over that plane alone),
    gathered from all slabs in plane order and added in plane order -- a
    fixed order that any split of the planes reproduces."""

    def moment_layout(self, p):
        return False, (4 if p == 0 else 9)

    def moments(self, p, buf):
        w = 4 if p == 0 else 9
        out = np.zeros((self.ohi - self.olo, w))
        for i in range(self.olo, self.ohi):
            acc = np.zeros(w)
            self.o.lib.hco_moments_acc(C.byref(self.o.g), _ptr(self.o.q[0]), p, i, i + 1, self.ioff,
                                       _ptr(self.com), _ptr(acc))
            out[i - self.olo] = acc
        return out.reshape(-1)

    def set_moments(self, p, data, nplanes):
        w = 4 if p == 0 else 9
        parts = np.asarray(data, dtype=np.float64).reshape(nplanes, w)
        acc = [0.0] * w
        for row in parts:
            for q in range(w):
                acc[q] += float(row[q])
        super().set_moments(p, np.array(acc), nplanes)


def gloo_worker(rank, world, port, shape, steps, bc, out_dir, gravity=None, tree=False):
    """One rank of a gloo process group: its oracle slab of the smooth random
    flow (or, with gravity = dict of solver keywords, the polytrope-like
    self-gravitating blob) takes `steps` steps through ProcessGroupComm, then
    writes its own planes, potential and the time steps to out_dir."""
    import datetime
    import os
    import sys

    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import ics
    from hydrocode_astro1_b200 import slab

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        entry = slab.plan(shape[0], world)[rank]
        if gravity:
            q0 = ics.gravity_blob(shape)
            sl = (TreeOracleSlab if tree else OracleSlab)(shape, entry, bc=bc, **gravity)
        else:
            q0 = ics.smooth_random(shape, seed=21)
            sl = OracleSlab(shape, entry, cfl=0.35, bc=bc)
        sl.set_state(q0)
        comm = slab.ProcessGroupComm(sl, dist, rank, world)
        dts = [comm.step() for _ in range(steps)]
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), sl.own_state())
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array(dts))
        if gravity:
            np.save(os.path.join(out_dir, f"phi{rank}.npy"), sl.own_phi())
            np.save(os.path.join(out_dir, f"it{rank}.npy"), np.array([sl.o.g.last_iter, sl.o.g.last_res]))
    finally:
        dist.destroy_process_group()
