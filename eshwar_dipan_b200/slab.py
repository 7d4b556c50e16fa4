"""One grid split into slabs along x over ranks (one process per GPU).

The reference's MPI variant splits the grid over processes and swaps ghost
layers after every pass (mpiinfo_xyz.h:739-787 of
Grand_potential_Finite_difference_2D_MPI).  Here each rank holds its own rows
[x0, x1) of the global grid plus HALO rows below and above them, and steps that
local grid whole with the single-GPU engine.  A step reads no further than two
rows from a cell, so after a step the rank's own rows are exactly what a step of
the whole grid gives, and one exchange per step (each rank sends the rows its
neighbours hold as halo) makes the halos exact again.

Halo rows that lie outside the global grid (a periodic edge, or a Neumann edge
of a field whose other field is periodic there) hold what the reference's
ghost copy puts there (assign_buffer_points_conditions,
utility_functions.h:471-654): row remap(v) of the field's own boundary types.
A non-periodic edge has no halo; the local grid keeps the global boundary type
there.

The plan is host logic only.  A rank drives it with a stepper (step, smooth,
pack, unpack, stats) and a transport: torch.distributed point-to-point
messages (NCCL between GPUs, gloo between CPU processes), or in-process copies
between several steppers.
"""
import ctypes

import numpy as np

from ._abi import Params

__all__ = ["HALO", "remap", "SlabPlan", "SlabRunner", "GpuSlab", "reduce_stats"]

HALO = 3
NEUMANN, PERIODIC = 1, 3


def remap(v, m, tlo, thi):
    """Interior row v in [-3, m+2] -> the interior row its ghost copy holds
    (Neumann mirrors about the boundary cell, periodic wraps with period m-1);
    the same map as the step kernels' boundary reads."""
    g, r = v + 3, m + 6
    src = g
    if g < 3:
        j = 2 - g
        src = 4 + j if tlo == NEUMANN else r - 5 - j
    elif g >= r - 3:
        j = g - (r - 3)
        src = r - 5 - j if thi == NEUMANN else 4 + j
    return src - 3


class _Message:
    """Rows one rank sends another in each exchange: item i moves row
    src_rows[i] of field fields[i] of the sender's local grid into row
    dst_rows[i] of the receiver's."""

    def __init__(self, src, dst):
        self.src, self.dst = src, dst
        self.fields, self.src_rows, self.dst_rows = [], [], []

    def __len__(self):
        return len(self.fields)


class SlabPlan:
    """Rows of every rank and the exchange between them, for a grid of
    `params` split over `nranks` ranks (this one is `rank`)."""

    def __init__(self, params, nranks, rank, halo=HALO):
        mx = int(params.mesh_x)
        if nranks < 1 or not 0 <= rank < nranks:
            raise ValueError("rank %d of %d" % (rank, nranks))
        if mx < nranks * (halo + 1):
            raise ValueError("MESH_X=%d is too small for %d slabs of at least %d rows" % (mx, nranks, halo + 1))
        if params.shift:
            raise ValueError("the moving frame needs the whole grid on one GPU")
        self.params, self.nranks, self.rank, self.halo = params, nranks, rank, halo
        self.mx, self.my = mx, int(params.mesh_y)
        self.N, self.K = int(params.numphases), int(params.numcomponents) - 1
        # boundary types along x per field kind (0: phi, 1: mu): [low, high]
        self.bcx = [(int(params.bc_type[f][0]), int(params.bc_type[f][1])) for f in (0, 1)]
        per_lo = any(b[0] == PERIODIC for b in self.bcx)
        per_hi = any(b[1] == PERIODIC for b in self.bcx)
        self.bounds = [mx * r // nranks for r in range(nranks + 1)]
        self.hlo = [halo if (r > 0 or per_lo) else 0 for r in range(nranks)]
        self.hhi = [halo if (r < nranks - 1 or per_hi) else 0 for r in range(nranks)]
        self.x0, self.x1 = self.bounds[rank], self.bounds[rank + 1]
        self.messages = self._messages()
        self.sends = [m for m in self.messages if m.src == rank and m.dst != rank]
        self.recvs = [m for m in self.messages if m.dst == rank and m.src != rank]
        self.local_copies = [m for m in self.messages if m.src == rank and m.dst == rank]

    # ---- rows
    def local_rows(self, r=None):
        """global rows [x0 - halo below, x1 + halo above) of rank r's grid"""
        r = self.rank if r is None else r
        return range(self.bounds[r] - self.hlo[r], self.bounds[r + 1] + self.hhi[r])

    def nlocal(self, r=None):
        r = self.rank if r is None else r
        return self.bounds[r + 1] - self.bounds[r] + self.hlo[r] + self.hhi[r]

    def own(self, r=None):
        """rank r's own rows as local rows [a, b)"""
        r = self.rank if r is None else r
        return self.hlo[r], self.hlo[r] + self.bounds[r + 1] - self.bounds[r]

    def source(self, v, field):
        """the global row whose values global row v (possibly a ghost row)
        holds for state field `field` (0..N-1 phi, then mu)"""
        if 0 <= v < self.mx:
            return v
        lo, hi = self.bcx[0 if field < self.N else 1]
        return remap(v, self.mx, lo, hi)

    def owner(self, row):
        for r in range(self.nranks):
            if self.bounds[r] <= row < self.bounds[r + 1]:
                return r
        raise ValueError("row %d outside the grid" % row)

    def _messages(self):
        msgs = {}
        for dst in range(self.nranks):
            rows = list(self.local_rows(dst))
            a, b = self.own(dst)
            halo_rows = list(range(0, a)) + list(range(b, len(rows)))
            for lr in halo_rows:
                v = rows[lr]
                for f in range(self.N + self.K):
                    s = self.source(v, f)
                    src = self.owner(s)
                    m = msgs.setdefault((src, dst), _Message(src, dst))
                    m.fields.append(f)
                    m.src_rows.append(s - (self.bounds[src] - self.hlo[src]))
                    m.dst_rows.append(lr)
        return [msgs[k] for k in sorted(msgs)]

    # ---- parameters and state of the local grid
    def local_params(self):
        """gp_params of this rank's grid: MESH_X rows; an edge with a halo
        gets Neumann (its rows are replaced after every step), the others keep
        the global types"""
        q = Params()
        ctypes.memmove(ctypes.byref(q), ctypes.byref(self.params), ctypes.sizeof(self.params))
        q.mesh_x = self.nlocal()
        for f in range(3):
            if self.hlo[self.rank]:
                q.bc_type[f][0] = q.bc_proxy_type[f][0] = NEUMANN
            if self.hhi[self.rank]:
                q.bc_type[f][1] = q.bc_proxy_type[f][1] = NEUMANN
        return q

    def local_state(self, phi, mu):
        """this rank's local phi [N][rows][MESH_Y] and mu from the global
        interior fields"""
        rows = list(self.local_rows())
        lp = np.stack([phi[a][[self.source(v, a) for v in rows]] for a in range(self.N)])
        lm = np.stack([mu[k][[self.source(v, self.N + k) for v in rows]] for k in range(self.K)])
        return np.ascontiguousarray(lp), np.ascontiguousarray(lm)

    def own_part(self, local):
        """the rank's own rows of a local [F][rows][MESH_Y] array"""
        a, b = self.own()
        return local[:, a:b]


def reduce_stats(st, allreduce):
    """Progress statistics of the whole grid from each rank's statistics of
    its own rows: extremes by max/min, the sums by addition.  allreduce(array,
    op) with op in ("max", "min", "sum") reduces a float64 array over ranks."""
    out = dict(st)
    for k in ("phi_max", "mu_max"):
        out[k] = allreduce(np.asarray(st[k], dtype=np.float64), "max")
    for k in ("phi_min", "mu_min"):
        out[k] = allreduce(np.asarray(st[k], dtype=np.float64), "min")
    for k in ("rel_change_phi", "rel_change_mu", "phi_sum", "comp_sum"):
        out[k] = allreduce(np.asarray(st[k], dtype=np.float64), "sum")
    out["nonfinite"] = int(allreduce(np.asarray([st["nonfinite"]], dtype=np.float64), "sum")[0])
    return out


class SlabRunner:
    """Steps one rank's slab: after every step (and smoothing sweep) the
    halo exchange of the plan.  `stepper` is this rank's grid; `transport`
    moves the packed rows of the plan's messages (see TorchTransport)."""

    def __init__(self, plan, stepper, transport):
        self.plan, self.stepper, self.transport = plan, stepper, transport

    def exchange(self):
        p, s = self.plan, self.stepper
        for m in p.local_copies:
            s.unpack(m.fields, m.dst_rows, s.pack(m.fields, m.src_rows))
        if not p.sends and not p.recvs:
            return
        out = [(m, s.pack(m.fields, m.src_rows)) for m in p.sends]
        got = self.transport.exchange(out, [(m, s.empty(len(m))) for m in p.recvs])
        for m, buf in got:
            s.unpack(m.fields, m.dst_rows, buf)

    def smooth(self, n):
        for _ in range(int(n)):
            self.stepper.smooth(1)
            self.exchange()

    def step(self, n):
        for _ in range(int(n)):
            self.stepper.step(1)
            self.exchange()


class TorchTransport:
    """Point-to-point messages over torch.distributed: every send and receive
    of an exchange in one batch (NCCL groups them, so no order of the ranks'
    calls can deadlock).  Under NCCL the buffers are CUDA tensors and `stream`
    (a torch.cuda stream: the context's own) orders the messages after the
    packs and before the unpacks."""

    def __init__(self, dist, stream=None):
        self.dist, self.stream = dist, stream

    def exchange(self, sends, recvs):
        d = self.dist
        ops = [d.P2POp(d.isend, buf, m.dst) for m, buf in sends]
        ops += [d.P2POp(d.irecv, buf, m.src) for m, buf in recvs]
        if not ops:
            return recvs
        if self.stream is not None:
            import torch
            with torch.cuda.stream(self.stream):
                for w in d.batch_isend_irecv(ops):
                    w.wait()
        else:
            for w in d.batch_isend_irecv(ops):
                w.wait()
        return recvs


class GpuSlab:
    """This rank's grid on its GPU: a Simulation of the local rows whose
    statistics cover its own rows; rows move through CUDA tensors on the
    context's stream (gp_rows_pack / gp_rows_unpack)."""

    def __init__(self, plan, phi, mu, precision=None):
        import torch

        from . import GP_FP64, Simulation, check, lib
        precision = GP_FP64 if precision is None else precision
        self._check, self._lib = check, lib
        self.plan = plan
        lp, lm = plan.local_state(phi, mu)
        self.sim = Simulation(plan.local_params(), lp, lm, precision=precision)
        a, b = plan.own()
        check(lib().gp_set_stat_rows(self.sim._h, a, b), self.sim._h)
        self.stream = torch.cuda.ExternalStream(lib().gp_stream(self.sim._h))
        self.dtype = torch.float64 if precision == GP_FP64 else torch.float32
        self._torch = torch
        self._tables = {}

    def _table(self, fields, rows):
        key = (tuple(fields), tuple(rows))
        t = self._tables.get(key)
        if t is None:
            t = (np.ascontiguousarray(fields, dtype=np.int32), np.ascontiguousarray(rows, dtype=np.int32))
            self._tables[key] = t
        return t

    def empty(self, n):
        with self._torch.cuda.stream(self.stream):
            return self._torch.empty((n, self.plan.my), dtype=self.dtype, device="cuda")

    def pack(self, fields, rows):
        f, r = self._table(fields, rows)
        buf = self.empty(len(f))
        self._check(self._lib().gp_rows_pack(self.sim._h, len(f), f.ctypes.data, r.ctypes.data, buf.data_ptr()),
                    self.sim._h)
        return buf

    def unpack(self, fields, rows, buf):
        f, r = self._table(fields, rows)
        self._check(self._lib().gp_rows_unpack(self.sim._h, len(f), f.ctypes.data, r.ctypes.data, buf.data_ptr()),
                    self.sim._h)

    def step(self, n):
        self.sim.step(n, stats=False)

    def smooth(self, n):
        self.sim.smooth(n)

    def stats(self):
        """statistics of the own rows after a step that took them (step_stats)"""
        return self.sim.stats()

    def step_stats(self, n):
        """n steps, the last with the statistics of the own rows"""
        return self.sim.step(n)

    def get(self):
        """the own rows of phi and mu"""
        ph, m = self.sim.get()
        return self.plan.own_part(ph), self.plan.own_part(m)

    def close(self):
        self._torch.cuda.synchronize()
        self.sim.close()
