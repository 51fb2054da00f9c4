"""One grid split along i into slabs, stepped as the whole grid.

The reference steps one grid in one process (hydro_solver_3d.c:637-811).
Here the grid's planes 0..nx-1 are cut into contiguous slabs; each slab is a
context of its own planes plus one ghost plane on each side that has a
neighbour (a copy of the neighbour's edge plane).  One hydro step of the
whole grid is then, per slab:

  1. the CFL signal speed max(|u_d| + c) that the step's dt is formed from
     (hydro_solver_3d.c:422-450) is replaced by its maximum over all slabs
     -- dt = cfl min(d/s) is monotone in s, so every slab takes the whole
     grid's dt bit for bit;
  2. the slab steps: its own planes are updated from its own and ghost
     planes exactly as the whole grid updates them (the interior update reads
     one plane on each side, :654-771); boundary conditions act on the
     global faces it holds, and on its ghost faces, whose values step 3
     replaces;
  3. every ghost plane receives the neighbour's updated edge plane.

The signal speed each slab forms after its step covers its own cells and its
ghost planes after the boundary conditions (copies or reflections of its own
edge cells), so the maximum over slabs is the whole grid's.  Hydro only: a
self-gravitating grid (G > 0) is not decomposed (its Poisson solve needs
the slabs' ghost planes exchanged after every colour sweep and the update
norm reduced per iteration, which this driver does not do).  Periodic x
boundaries are not decomposed either.

Transport: `ProcessGroupComm` -- one slab per rank of a torch.distributed
process group (NCCL between GPUs, gloo on the CPU): an all-reduce of the
signal speed and paired sends/receives of plane buffers; `LocalComm` -- all
slabs in one process (several contexts on one device), planes copied
directly.
"""
from __future__ import annotations

import numpy as np


def plan(nx, parts):
    """Own planes [a, b) of each slab (a partition of 0..nx-1, sizes as
    equal as possible) and its local planes [lo, hi): one ghost plane on each
    side with a neighbour."""
    if parts < 1 or nx < 3 * parts:
        raise ValueError(f"{nx} planes cannot be split into {parts} slabs of at least 3 planes")
    base, extra = divmod(nx, parts)
    out, a = [], 0
    for r in range(parts):
        b = a + base + (1 if r < extra else 0)
        lo = a - 1 if r > 0 else a
        hi = b + 1 if r < parts - 1 else b
        out.append(dict(own=(a, b), local=(lo, hi)))
        a = b
    return out


class GpuSlab:
    """A slab as a context of this library (FP64 or FP32), its state in
    device memory; planes move through torch CUDA tensors."""

    def __init__(self, shape, entry, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), device=0, **kw):
        import torch

        import hydrocode_astro1_b200 as hc
        if kw.get("G", 0.0) > 0.0:
            raise ValueError("slab decomposition: hydro only (G = 0)")
        nx, ny, nz = shape
        d = [(hi[t] - lo[t]) / shape[t] for t in range(3)]
        l0, l1 = entry["local"]
        self.entry = entry
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.ny, self.nz = ny, nz
        self.nx_l = l1 - l0
        self.dtype = torch.float64 if kw.get("precision", hc.FP64) == hc.FP64 else torch.float32
        slo = (lo[0] + l0 * d[0], lo[1], lo[2])
        shi = (lo[0] + l1 * d[0], hi[1], hi[2])
        self.s = hc.HydroSolver3D((self.nx_l, ny, nz), lo=slo, hi=shi, dx=d[0], dy=d[1], dz=d[2], device=device,
                                  **kw)

    def set_state(self, q_global):
        l0, l1 = self.entry["local"]
        self.s.set_state(np.ascontiguousarray(q_global[:, l0:l1]))

    def signal_speed(self):
        return self.s.signal_speed()

    def set_signal_speed(self, v):
        self.s.set_signal_speed(v)

    def step(self):
        return float(self.s.step(1)[0])

    def get_planes(self, i0, count):
        t = self.torch.empty((5, count, self.ny, self.nz), dtype=self.dtype, device=self.dev)
        self.s.copy_planes(i0, count, t.data_ptr(), False)
        return t

    def set_planes(self, i0, t):
        t = t.contiguous()
        self.s.copy_planes(i0, t.shape[1], t.data_ptr(), True)

    def own_state(self):
        """The slab's own planes (5, b - a, ny, nz) as numpy FP64."""
        a, b = self.entry["own"]
        l0 = self.entry["local"][0]
        return self.s.state()[:, a - l0:b - l0]

    def close(self):
        self.s.close()


class LocalComm:
    """All slabs in this process."""

    def __init__(self, slabs):
        self.slabs = slabs

    def step(self):
        s = max(sl.signal_speed() for sl in self.slabs)
        for sl in self.slabs:
            sl.set_signal_speed(s)
        dts = [sl.step() for sl in self.slabs]
        if any(dt != dts[0] for dt in dts):
            raise RuntimeError(f"slabs took different time steps: {dts}")
        for left, right in zip(self.slabs[:-1], self.slabs[1:]):
            up = left.get_planes(left.nx_l - 2, 1)
            down = right.get_planes(1, 1)
            right.set_planes(0, up)
            left.set_planes(left.nx_l - 1, down)
        return dts[0]


class ProcessGroupComm:
    """One slab per rank of a torch.distributed process group."""

    def __init__(self, slab, dist, rank, world, device="cpu"):
        self.slab, self.dist, self.rank, self.world = slab, dist, rank, world
        self.device = device

    def allreduce_max(self, v):
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def exchange(self):
        import torch
        sl, r, n = self.slab, self.rank, self.world
        ops, recv = [], {}
        if r > 0:
            ops.append(self.dist.P2POp(self.dist.isend, sl.get_planes(1, 1), r - 1))
            recv["lo"] = torch.empty_like(sl.get_planes(0, 1))
            ops.append(self.dist.P2POp(self.dist.irecv, recv["lo"], r - 1))
        if r < n - 1:
            ops.append(self.dist.P2POp(self.dist.isend, sl.get_planes(sl.nx_l - 2, 1), r + 1))
            recv["hi"] = torch.empty_like(sl.get_planes(sl.nx_l - 1, 1))
            ops.append(self.dist.P2POp(self.dist.irecv, recv["hi"], r + 1))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        if "lo" in recv:
            sl.set_planes(0, recv["lo"])
        if "hi" in recv:
            sl.set_planes(sl.nx_l - 1, recv["hi"])

    def step(self):
        s = self.allreduce_max(self.slab.signal_speed())
        self.slab.set_signal_speed(s)
        dt = self.slab.step()
        self.exchange()
        return dt
