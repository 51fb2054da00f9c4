"""One grid split along i into slabs, stepped as the whole grid.

The reference steps one grid in one process (hydro_solver_3d.c:637-811).
Here the grid's planes 0..nx-1 are cut into contiguous slabs; each slab is a
context of its own planes plus one ghost plane on each side that has a
neighbour (a copy of the neighbour's edge plane).  One step of the whole
grid is then, per slab:

  1. the CFL signal speed max(|u_d| + c) that the step's dt is formed from
     (hydro_solver_3d.c:422-450) is replaced by its maximum over all slabs
     -- dt = cfl min(d/s) is monotone in s, so every slab takes the whole
     grid's dt bit for bit;
  2. with self-gravity, the Poisson solve of the whole grid runs across the
     slabs (gravity_solver_3d.c:510-747, `solve_gravity`):
       - the multipole moments of the density: the reference's sequential
         sums chained slab to slab in plane order, or per-plane partials
         gathered in plane order and added in the single grid's tree order;
       - red-black SOR: every half sweep updates each slab's own cells of
         one colour, then every ghost plane receives the neighbour's plane
         (the other colour's cells a sweep reads are the neighbour's final
         values, as in the single grid); the boundary values after the first
         iteration, on the global faces each slab holds;
       - the stop test on the maximum of the slabs' update norms (a maximum
         is exact in any order), so every slab stops at the same iteration;
  3. the slab steps: its own planes are updated from its own and ghost
     planes exactly as the whole grid updates them (the interior update and
     the gravity source read one plane on each side, :654-771); boundary
     conditions act on the global faces it holds, and on its ghost faces,
     whose values step 4 replaces;
  4. every ghost plane receives the neighbour's updated edge plane.

The signal speed each slab forms after its step covers its own cells and its
ghost planes after the boundary conditions (copies or reflections of its own
edge cells), so the maximum over slabs is the whole grid's.  Periodic x
boundaries are not decomposed; self-gravity needs FP64 slabs with the
isolated boundary.

Transport: `ProcessGroupComm` -- one slab per rank of a torch.distributed
process group (NCCL between GPUs, gloo on the CPU): all-reduces of the
signal speed and the update norm, the moment chain as paired sends and
receives plus a broadcast, an all-gather of the moment partials, and paired
sends/receives of plane buffers; `LocalComm` -- all slabs in one process
(several contexts on one device), everything copied directly.

A slab object (`GpuSlab`, or the oracle's slab in the tests) provides:
signal_speed/set_signal_speed/step, get_planes/set_planes (state),
and with gravity: moment_layout, moments, set_moments, sor_begin,
sor_sweep, sor_boundary, sor_norm, sor_end, get_phi_planes/set_phi_planes,
and the attributes gravity, gnx, own_planes, max_iter, tol, nx_l.
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


def solve_gravity(comm):
    """The whole grid's Poisson solve across the slabs of comm; returns
    (converged, iterations, residual) -- the single grid's, bit for bit."""
    for p in (0, 1):
        sequential, width = comm.layout(p)
        data = comm.chain(p, np.zeros(width)) if sequential else comm.gather(p, width)
        comm.each(lambda sl: sl.set_moments(p, data, sl.gnx))
    comm.each(lambda sl: sl.sor_begin())
    max_iter, tol = comm.params()
    res, used, conv = 0.0, max(max_iter, 0), False
    for it in range(max_iter):
        for colour in (0, 1):
            comm.each(lambda sl: sl.sor_sweep(it, colour))
            comm.exchange_phi()
        if it == 0:
            comm.each(lambda sl: sl.sor_boundary())
            comm.exchange_phi()
        res = comm.max(lambda sl: sl.sor_norm(it))
        if res < tol:
            used, conv = it + 1, True
            break
    comm.each(lambda sl: sl.sor_end(used, res, conv))
    return conv, used, res


class GpuSlab:
    """A slab as a context of this library (FP64 or FP32; FP64 with
    self-gravity), its state in device memory; planes move through torch
    CUDA tensors."""

    def __init__(self, shape, entry, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), device=0, **kw):
        import torch

        import hydrocode_astro1_b200 as hc
        nx, ny, nz = shape
        d = [(hi[t] - lo[t]) / shape[t] for t in range(3)]
        l0, l1 = entry["local"]
        a, b = entry["own"]
        self.entry = entry
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.ny, self.nz = ny, nz
        self.nx_l = l1 - l0
        self.gnx = nx
        self.own_planes = b - a
        self.gravity = kw.get("G", 0.0) > 0.0
        self.dtype = torch.float64 if kw.get("precision", hc.FP64) == hc.FP64 else torch.float32
        # the whole grid's bounds and cell sizes; the context holds planes [l0, l1)
        self.s = hc.HydroSolver3D((self.nx_l, ny, nz), lo=lo, hi=hi, dx=d[0], dy=d[1], dz=d[2], device=device,
                                  **kw)
        self.s.set_slab(nx, l0)
        self.max_iter, self.tol = self.s.cfg.max_iter, self.s.cfg.tol

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

    # gravity ----------------------------------------------------------------
    def moment_layout(self, p):
        return self.s.slab_moment_layout(p)

    def moments(self, p, buf):
        return self.s.slab_moments(p, np.ascontiguousarray(buf, dtype=np.float64))

    def set_moments(self, p, data, nplanes):
        self.s.slab_set_moments(p, data, nplanes)

    def sor_begin(self):
        self.s.slab_sor_begin()

    def sor_sweep(self, it, colour):
        self.s.slab_sor_sweep(it, colour)

    def sor_boundary(self):
        self.s.slab_sor_boundary()

    def sor_norm(self, it):
        return self.s.slab_sor_norm(it)

    def sor_end(self, used, res, conv):
        self.s.slab_sor_end(used, res, conv)

    def get_phi_planes(self, i0, count):
        # [2][count][ny (nz+1)/2], indexed by the whole grid's colour
        t = self.torch.empty((2, count, self.ny * ((self.nz + 1) // 2)), dtype=self.torch.float64, device=self.dev)
        self.s.slab_phi_planes(i0, count, t.data_ptr(), False)
        return t

    def set_phi_planes(self, i0, t):
        t = t.contiguous()
        self.s.slab_phi_planes(i0, t.shape[1], t.data_ptr(), True)

    def own_state(self):
        """The slab's own planes (5, b - a, ny, nz) as numpy FP64."""
        a, b = self.entry["own"]
        l0 = self.entry["local"][0]
        return self.s.state()[:, a - l0:b - l0]

    def close(self):
        self.s.close()


class _Comm:
    """The step of the whole grid over the transport's collectives."""

    def step(self):
        s = self.max(lambda sl: sl.signal_speed())
        self.each(lambda sl: sl.set_signal_speed(s))
        if self.gravity:
            solve_gravity(self)
        dt = self.step_slabs()
        self.exchange_state()
        return dt


class LocalComm(_Comm):
    """All slabs in this process."""

    def __init__(self, slabs):
        self.slabs = slabs
        self.gravity = slabs[0].gravity

    def each(self, fn):
        return [fn(sl) for sl in self.slabs]

    def max(self, fn):
        return max(fn(sl) for sl in self.slabs)

    def params(self):
        return self.slabs[0].max_iter, self.slabs[0].tol

    def layout(self, p):
        return self.slabs[0].moment_layout(p)

    def chain(self, p, acc):
        for sl in self.slabs:
            acc = sl.moments(p, acc.copy())
        return acc

    def gather(self, p, width):
        return np.concatenate([sl.moments(p, np.zeros(sl.own_planes * width)) for sl in self.slabs])

    def step_slabs(self):
        dts = [sl.step() for sl in self.slabs]
        if any(dt != dts[0] for dt in dts):
            raise RuntimeError(f"slabs took different time steps: {dts}")
        return dts[0]

    def _exchange(self, get, put):
        for left, right in zip(self.slabs[:-1], self.slabs[1:]):
            up = get(left, left.nx_l - 2)
            down = get(right, 1)
            put(right, 0, up)
            put(left, left.nx_l - 1, down)

    def exchange_state(self):
        self._exchange(lambda sl, i: sl.get_planes(i, 1), lambda sl, i, t: sl.set_planes(i, t))

    def exchange_phi(self):
        self._exchange(lambda sl, i: sl.get_phi_planes(i, 1), lambda sl, i, t: sl.set_phi_planes(i, t))


class ProcessGroupComm(_Comm):
    """One slab per rank of a torch.distributed process group; `device` is
    where the collectives' tensors live ("cpu" for gloo, "cuda" for NCCL)."""

    def __init__(self, slab, dist, rank, world, device="cpu"):
        self.slab, self.dist, self.rank, self.world = slab, dist, rank, world
        self.device = device
        self.gravity = slab.gravity

    def each(self, fn):
        return fn(self.slab)

    def max(self, fn):
        import torch
        t = torch.tensor([fn(self.slab)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def allreduce_max(self, v):
        return self.max(lambda sl: v)

    def params(self):
        return self.slab.max_iter, self.slab.tol

    def layout(self, p):
        return self.slab.moment_layout(p)

    def chain(self, p, acc):
        """Sums continued rank by rank in plane order; every rank gets the
        last rank's."""
        import torch
        r, n = self.rank, self.world
        t = torch.zeros(len(acc), dtype=torch.float64, device=self.device)
        if r > 0:
            self.dist.recv(t, r - 1)
        out = self.slab.moments(p, t.cpu().numpy().copy())
        t = torch.from_numpy(out).to(self.device)
        if r < n - 1:
            self.dist.send(t, r + 1)
        self.dist.broadcast(t, n - 1)
        return t.cpu().numpy().copy()

    def gather(self, p, width):
        """Every rank's per-plane partials, concatenated in rank (plane)
        order."""
        import torch
        sizes = torch.tensor([self.slab.own_planes * width], dtype=torch.int64, device=self.device)
        all_sizes = [torch.zeros_like(sizes) for _ in range(self.world)]
        self.dist.all_gather(all_sizes, sizes)
        all_sizes = [int(s.item()) for s in all_sizes]
        m = max(all_sizes)
        mine = self.slab.moments(p, np.zeros(self.slab.own_planes * width))
        t = torch.zeros(m, dtype=torch.float64, device=self.device)
        t[:len(mine)] = torch.from_numpy(mine).to(self.device)
        bufs = [torch.zeros_like(t) for _ in range(self.world)]
        self.dist.all_gather(bufs, t)
        return np.concatenate([b[:k].cpu().numpy() for b, k in zip(bufs, all_sizes)])

    def step_slabs(self):
        return self.slab.step()

    def _exchange(self, get, put):
        import torch
        sl, r, n = self.slab, self.rank, self.world
        ops, recv = [], {}
        if r > 0:
            ops.append(self.dist.P2POp(self.dist.isend, get(1), r - 1))
            recv["lo"] = torch.empty_like(get(0))
            ops.append(self.dist.P2POp(self.dist.irecv, recv["lo"], r - 1))
        if r < n - 1:
            ops.append(self.dist.P2POp(self.dist.isend, get(sl.nx_l - 2), r + 1))
            recv["hi"] = torch.empty_like(get(sl.nx_l - 1))
            ops.append(self.dist.P2POp(self.dist.irecv, recv["hi"], r + 1))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        if "lo" in recv:
            put(0, recv["lo"])
        if "hi" in recv:
            put(sl.nx_l - 1, recv["hi"])

    def exchange(self):
        self.exchange_state()

    def exchange_state(self):
        self._exchange(lambda i: self.slab.get_planes(i, 1), lambda i, t: self.slab.set_planes(i, t))

    def exchange_phi(self):
        self._exchange(lambda i: self.slab.get_phi_planes(i, 1), lambda i, t: self.slab.set_phi_planes(i, t))
