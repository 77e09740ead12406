"""One realization's PM force and particles split over ranks by x slabs.

The reference runs one realization on many MPI ranks: comm_init gives each
rank a slab of mesh planes and its left and right neighbours
(comm.c:35-111), FFTW-MPI transposes the spectrum between x slabs and kz
slabs inside the transforms (pm.c:282-355), particles within one cell of a
slab's upper edge act on the next slab as buffer particles whose forces come
back to their owners (send_buffer_positions / add_buffer_forces,
pm.c:416-532), and move_particles2 sends particles that left a slab to the
rank that owns their new position (move.c:15-175).

Here a rank is one GPU (one process, ``torch.distributed`` over NCCL) or,
for tests, one of several ranks held by one process (``LocalComm``).  The
per-rank compute is the library's (``cg_sim_slab_*``, wrapped by
``GpuRank``); this module does the exchanges:

  1. buffer positions to the right neighbour (shifted by -L across the
     periodic face), received from the left;
  2. ``density``: the rank's particles and the received copies into its
     planes, r2c along z (the density sums add up to check_total_density's);
  3. half spectrum: x slabs -> kz slabs (all-to-all of blocks);
  4. ``kspace``: x, Green and inverse x passes of the rank's kz planes;
  5. three force spectra: kz slabs -> x slabs;
  6. ``c2r`` of the rank's planes, ``interp`` of its particles and copies;
  7. buffer forces back to the left neighbour, added to the owners'
     forces (after their own, in add_buffer_forces' order).

A rank object provides: ``N``, ``L``, ``n`` (particles held), device
tensors ``positions()`` and ``forces()`` (3 x n, float32, writable),
``spectrum(which)`` ((N/2+1) x N x N x 2 float32, which 0 the density, 1..3
the force components), ``density(x0, nx, bx)`` (returns the slab's density
sum), ``kspace(kz0, nkz)``, ``c2r(x0, nx)``, ``interp(x0, nx, bx, bf)``,
``get_particles()`` / ``set_particles(rows)`` (n x 14 float32 rows of the
reference Particle, 56 bytes each) and ``sync()``.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def slab_ranges(n, size):
    """(start, count) of `size` contiguous, balanced ranges over n items."""
    base, extra = divmod(n, size)
    out, s = [], 0
    for r in range(size):
        c = base + (1 if r < extra else 0)
        out.append((s, c))
        s += c
    return out


class LocalComm:
    """All ranks in this process: an exchange is a copy between them."""

    def __init__(self, size):
        self.size = size
        self.ranks = list(range(size))

    def exchange(self, send, recv_shapes, device, dtype=torch.float32):
        """send[i][s]: tensor from local rank i to rank s (or None);
        returns recv[i][s] (None where nothing came)."""
        return [[send[s][r].clone() if send[s][r] is not None else None
                 for s in range(self.size)] for r in self.ranks]

    def allreduce(self, values):
        return [float(sum(values))] * len(values)


class TorchComm:
    """One rank per process over torch.distributed (NCCL between GPUs, gloo
    between CPU processes): exchanges are point-to-point sends and receives
    posted together."""

    def __init__(self, group=None, device="cpu"):
        """device: where the process group's tensors live ("cuda" for NCCL,
        "cpu" for gloo)."""
        import torch.distributed as td
        self.td = td
        self.group = group
        self.device = device
        self.size = td.get_world_size(group)
        self.ranks = [td.get_rank(group)]

    def exchange(self, send, recv_shapes, device, dtype=torch.float32):
        me = self.ranks[0]
        recv = [None] * self.size
        ops = []
        for s in range(self.size):
            if s == me:
                recv[s] = send[0][s].clone() if send[0][s] is not None else None
                continue
            if send[0][s] is not None:
                ops.append(self.td.P2POp(self.td.isend, send[0][s].contiguous(), s, self.group))
            if recv_shapes[0][s] is not None:
                recv[s] = torch.empty(recv_shapes[0][s], dtype=dtype, device=device)
                ops.append(self.td.P2POp(self.td.irecv, recv[s], s, self.group))
        if ops:
            for req in self.td.batch_isend_irecv(ops):
                req.wait()
        return [recv]

    def allreduce(self, values):
        t = torch.tensor([float(values[0])], dtype=torch.float64, device=self.device)
        self.td.all_reduce(t, group=self.group)
        return [float(t.item())]


def _counts_exchange(comm, counts, device):
    """counts[i][s]: ints from local rank i to rank s; returns the received
    counts recv[i][s]."""
    send = [[torch.tensor([float(c)], dtype=torch.float64, device=device) for c in row]
            for row in counts]
    shapes = [[(1,)] * comm.size for _ in comm.ranks]
    recv = comm.exchange(send, shapes, device, torch.float64)
    return [[int(t.item()) for t in row] for row in recv]


class SlabPM:
    """The slab-decomposed force of one realization.  `ranks` holds the
    rank objects of the ranks this process runs (all of them for
    LocalComm, one for TorchComm), in comm.ranks order."""

    def __init__(self, ranks, comm, device):
        self.ranks, self.comm, self.device = ranks, comm, device
        r0 = ranks[0]
        self.N, self.L = r0.N, r0.L
        self.size = comm.size
        self.xs = slab_ranges(self.N, self.size)
        self.ks = slab_ranges(self.N // 2 + 1, self.size)
        self.density_sum = None

    # -- geometry (float32 as pm.c:422-434 and comm.c:121-130 form them)
    def x_right(self, r):
        x0, nx = self.xs[r]
        L, N = np.float32(self.L), np.float32(self.N)
        eps = L / N
        return np.float32(L / N * np.float32(x0 + nx) - eps)

    def x_bounds(self, r):
        x0, nx = self.xs[r]
        L = np.float32(self.L)
        return (np.float32(L * np.float32(x0) / np.float32(self.N)),
                np.float32(L * np.float32(x0 + nx) / np.float32(self.N)))

    # -- the force
    def forces(self):
        P, N, dev = self.size, self.N, self.device
        me = self.comm.ranks
        # 1. buffer positions to the right neighbour
        sel, sends = [], []
        for i, r in enumerate(me):
            x = self.ranks[i].positions()
            idx = torch.nonzero(x[0] > float(self.x_right(r))).flatten()
            bx = x[:, idx].clone()
            if self.xs[r][0] + self.xs[r][1] == N:         # across the periodic face
                bx[0] = bx[0] + np.float32(-self.L)
            sel.append(idx)
            row = [None] * P
            row[(r + 1) % P] = bx
            sends.append(row)
        counts = [[0 if t is None else t.shape[1] for t in row] for row in sends]
        rc = _counts_exchange(self.comm, counts, dev)
        shapes = [[(3, rc[i][s]) if s == (r - 1) % P else None for s in range(P)]
                  for i, r in enumerate(me)]
        got = self.comm.exchange(sends, shapes, dev)
        bufs = [got[i][(r - 1) % P] for i, r in enumerate(me)]
        # 2. density and r2c along z of each rank's planes
        sums = []
        for i, r in enumerate(me):
            x0, nx = self.xs[r]
            sums.append(self.ranks[i].density(x0, nx, bufs[i]))
        self.density_sum = self.comm.allreduce(sums)[0]
        # 3-5. spectrum to kz slabs, k-space passes, force spectra back
        self._transpose(0, to_kz=True)
        for i, r in enumerate(me):
            k0, nk = self.ks[r]
            self.ranks[i].kspace(k0, nk)
        for a in (1, 2, 3):
            self._transpose(a, to_kz=False)
        # 6. z c2r and interpolation of each rank's particles and copies
        bfs = []
        for i, r in enumerate(me):
            x0, nx = self.xs[r]
            self.ranks[i].c2r(x0, nx)
            bf = torch.zeros_like(bufs[i])
            self.ranks[i].interp(x0, nx, bufs[i], bf)
            bfs.append(bf)
        # 7. buffer forces back to their owners
        sends = []
        for i, r in enumerate(me):
            row = [None] * P
            row[(r - 1) % P] = bfs[i]
            sends.append(row)
        shapes = [[(3, sel[i].numel()) if s == (r + 1) % P else None for s in range(P)]
                  for i, r in enumerate(me)]
        got = self.comm.exchange(sends, shapes, dev)
        for i, r in enumerate(me):
            fb = got[i][(r + 1) % P]
            f = self.ranks[i].forces()
            f[:, sel[i]] = f[:, sel[i]] + fb
            self.ranks[i].sync()
        return self.density_sum

    def _transpose(self, which, to_kz):
        """Blocks [kz slab of s] x [x slab of r] of spectrum `which` from
        rank r to rank s (to_kz), or the reverse."""
        P, N, dev = self.size, self.N, self.device
        me = self.comm.ranks
        sends, shapes, specs = [], [], []
        for i, r in enumerate(me):
            t = self.ranks[i].spectrum(which)
            specs.append(t)
            row, srow = [], []
            for s in range(P):
                if to_kz:      # my x slab, s's kz slab
                    (x0, nx), (k0, nk) = self.xs[r], self.ks[s]
                    (rx0, rnx), (rk0, rnk) = self.xs[s], self.ks[r]
                else:          # my kz slab, s's x slab
                    (x0, nx), (k0, nk) = self.xs[s], self.ks[r]
                    (rx0, rnx), (rk0, rnk) = self.xs[r], self.ks[s]
                if s == r:     # the block a rank keeps is already in place
                    row.append(None)
                    srow.append(None)
                    continue
                row.append(t[k0:k0 + nk, x0:x0 + nx].contiguous())
                srow.append((rnk, rnx, N, 2))
            sends.append(row)
            shapes.append(srow)
        got = self.comm.exchange(sends, shapes, dev)
        for i, r in enumerate(me):
            t = specs[i]
            for s in range(P):
                if to_kz:
                    (rx0, rnx), (rk0, rnk) = self.xs[s], self.ks[r]
                else:
                    (rx0, rnx), (rk0, rnk) = self.xs[r], self.ks[s]
                if s != r:
                    t[rk0:rk0 + rnk, rx0:rx0 + rnx] = got[i][s]
            self.ranks[i].sync()

    # -- particles to the rank of their slab (move.c:15-175, after the wrap)
    def exchange_particles(self):
        P, dev = self.size, self.device
        me = self.comm.ranks
        if P == 1:
            return [self.ranks[0].n]
        bounds = [self.x_bounds(s) for s in range(P)]
        edges = torch.tensor([float(b[0]) for b in bounds[1:]], dtype=torch.float32, device=dev)
        sends, keep = [], []
        for i, r in enumerate(me):
            rows = self.ranks[i].get_particles()
            owner = torch.bucketize(rows[:, 0].contiguous(), edges, right=True)
            row = []
            for s in range(P):
                row.append(rows[owner == s].T.contiguous())     # 14 x m
            sends.append(row)
        counts = [[t.shape[1] for t in row] for row in sends]
        rc = _counts_exchange(self.comm, counts, dev)
        shapes = [[(14, rc[i][s]) for s in range(P)] for i in range(len(me))]
        got = self.comm.exchange(sends, shapes, dev)
        for i, r in enumerate(me):
            rows = torch.cat([g.T for g in got[i]], dim=0).contiguous()
            self.ranks[i].set_particles(rows)
        return [self.ranks[i].n for i in range(len(me))]


class _DevArray:
    """A device buffer as __cuda_array_interface__, for torch.as_tensor."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


class GpuRank:
    """A rank of SlabPM on this process's GPU: one cg_sim handle (through a
    Simulation) with its slab stages.  The cell-order sort stays off, so the
    handle's arrays are in the order the particles were given."""

    def __init__(self, sim):
        self.sim, self.lib = sim, sim.lib
        self.N, self.L = sim.ngrid, sim.boxsize
        _lib.check(self.lib.cg_sim_set_sort_interval(sim.h, 0), "cg_sim_set_sort_interval")

    @property
    def n(self):
        return int(self.lib.cg_sim_np(self.sim.h))

    def sync(self):
        torch.cuda.synchronize()
        _lib.check(self.lib.cg_sim_sync(self.sim.h), "cg_sim_sync")

    def _ptrs(self):
        x = (ctypes.c_void_p * 3)()
        f = (ctypes.c_void_p * 3)()
        _lib.check(self.lib.cg_sim_state_ptrs(self.sim.h, x, f), "cg_sim_state_ptrs")
        return x, f

    def _soa(self, ptrs):
        n = self.n
        cols = [torch.as_tensor(_DevArray(ptrs[a], (n,)), device="cuda") for a in range(3)]
        return cols

    def positions(self):
        x, _ = self._ptrs()
        return torch.stack(self._soa(x))

    def forces(self):
        """3 x n view whose writes reach the handle (column assignment
        through the three per-component arrays)."""
        return _Forces(self._soa(self._ptrs()[1]))

    def spectrum(self, which):
        p = ctypes.c_void_p()
        _lib.check(self.lib.cg_sim_spectrum_ptr(self.sim.h, which, ctypes.byref(p)),
                   "cg_sim_spectrum_ptr")
        N = self.N
        return torch.as_tensor(_DevArray(p.value, (N // 2 + 1, N, N, 2)), device="cuda")

    def density(self, x0, nx, bx):
        self.sync()
        b = bx.contiguous()
        s = ctypes.c_double()
        _lib.check(self.lib.cg_sim_slab_density(self.sim.h, x0, nx, b.data_ptr() if b.numel() else None,
                                                b.shape[1], ctypes.byref(s)), "cg_sim_slab_density")
        return s.value

    def kspace(self, kz0, nkz):
        self.sync()
        _lib.check(self.lib.cg_sim_slab_kspace(self.sim.h, kz0, nkz), "cg_sim_slab_kspace")
        self.sync()

    def c2r(self, x0, nx):
        self.sync()
        _lib.check(self.lib.cg_sim_slab_c2r(self.sim.h, x0, nx), "cg_sim_slab_c2r")

    def interp(self, x0, nx, bx, bf):
        b = bx.contiguous()
        self.sync()
        _lib.check(self.lib.cg_sim_slab_interp(self.sim.h, x0, nx,
                                               b.data_ptr() if b.numel() else None, b.shape[1],
                                               bf.data_ptr() if bf.numel() else None),
                   "cg_sim_slab_interp")
        self.sync()

    def get_particles(self):
        n = self.n
        out = torch.empty((n, 14), dtype=torch.float32, device="cuda")
        if n:
            self.sync()
            _lib.check(self.lib.cg_sim_get_particles(self.sim.h, out.data_ptr()),
                       "cg_sim_get_particles")
        return out

    def set_particles(self, rows):
        a_x, a_v = self.sim.times()
        rows = rows.contiguous()
        self.sync()
        _lib.check(self.lib.cg_sim_set_particles(self.sim.h, rows.data_ptr() if rows.numel() else None,
                                                 rows.shape[0], a_x, a_v), "cg_sim_set_particles")
        self.sync()


class _Forces:
    """The handle's three force arrays behind a 3 x n tensor-like view."""

    def __init__(self, cols):
        self.cols = cols

    def __getitem__(self, key):
        _, idx = key
        return torch.stack([c[idx] for c in self.cols])

    def __setitem__(self, key, value):
        _, idx = key
        for a in range(3):
            self.cols[a][idx] = value[a]
