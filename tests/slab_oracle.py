"""A slab of the decomposition (hydrocode_astro1_b200/slab.py) backed by the
CPU oracle: test infrastructure, so that the decomposition protocol -- the
signal-speed maximum over slabs, the step with the whole grid's dt, the ghost
plane exchange -- runs as gloo ranks on the CPU and is compared with the
oracle's single-grid step."""
import ctypes as C

import numpy as np
import torch

from oracle.oracle import OracleSim


class OracleSlab:
    def __init__(self, shape, entry, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), **kw):
        nx, ny, nz = shape
        d = [(hi[t] - lo[t]) / shape[t] for t in range(3)]
        l0, l1 = entry["local"]
        self.entry = entry
        self.ny, self.nz = ny, nz
        self.nx_l = l1 - l0
        self.o = OracleSim(self.nx_l, ny, nz, lo=(lo[0] + l0 * d[0], lo[1], lo[2]),
                           hi=(lo[0] + l1 * d[0], hi[1], hi[2]), **kw)
        # the whole grid's cell sizes, bit for bit
        self.o.g.dx, self.o.g.dy, self.o.g.dz = d
        self.cfl = kw.get("cfl", 0.4)
        self.smax = None

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
        self.o.lib.hco_step_dt(C.byref(g), dt)
        return dt

    def get_planes(self, i0, count):
        return torch.from_numpy(np.ascontiguousarray(self.o.q[:, i0:i0 + count]))

    def set_planes(self, i0, t):
        self.o.q[:, i0:i0 + t.shape[1]] = t.numpy()

    def own_state(self):
        a, b = self.entry["own"]
        l0 = self.entry["local"][0]
        return self.o.state()[:, a - l0:b - l0]


def gloo_worker(rank, world, port, shape, steps, bc, out_dir):
    """One rank of a gloo process group: its oracle slab of the smooth random
    flow takes `steps` steps through ProcessGroupComm, then writes its own
    planes and the time steps to out_dir."""
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
        q0 = ics.smooth_random(shape, seed=21)
        entry = slab.plan(shape[0], world)[rank]
        sl = OracleSlab(shape, entry, cfl=0.35, bc=bc)
        sl.set_state(q0)
        comm = slab.ProcessGroupComm(sl, dist, rank, world)
        dts = [comm.step() for _ in range(steps)]
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), sl.own_state())
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array(dts))
    finally:
        dist.destroy_process_group()
