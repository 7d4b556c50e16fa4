"""One grid split into slabs along x (eshwar_dipan_b200.slab) on CPU: the
plan's messages rebuild every halo row from its owner, and ranks that step
their slabs with the oracle and swap halos over gloo after every step hold
the whole-grid oracle's rows bit for bit (two and three ranks; Neumann,
periodic and mixed boundary types along x)."""
import os
import socket
import sys

import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from eshwar_dipan_b200.slab import SlabPlan, SlabRunner, TorchTransport, reduce_stats, remap
from gp_cases import PARITY_CASES, write_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = {
    "neumann": (PARITY_CASES["bin_iso_antitrap"]["kw"], PARITY_CASES["bin_iso_antitrap"]["seeds"]),
    "periodic": (PARITY_CASES["bin_aniso_periodic"]["kw"], PARITY_CASES["bin_aniso_periodic"]["seeds"]),
    # phi periodic along x, mu Neumann: the edge ranks hold halos whose mu rows mirror their own
    "mixed": (dict(N=3, K=2, mesh=(40, 36), dab=0.02, bc_phi=(3, 3, 1, 1), bc_mu=(1, 1, 1, 1), A_off=0.25),
              [(0, 2, 18, 6.0), (1, 20, 10, 6.0), (0, 37, 30, 5.0)]),
}


def _deck(tmpdir, name):
    kw, seeds = CASES[name]
    ip, fp = write_case(str(tmpdir), name, dict(kw), seeds=seeds)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    return ip, fp, p, phi, mu


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_plan_messages_rebuild_every_halo(tmp_path, name, nranks):
    _, _, p, phi, mu = _deck(tmp_path, name)
    rng = np.random.default_rng(nranks)
    phi = phi + rng.standard_normal(phi.shape)
    mu = mu + rng.standard_normal(mu.shape)
    plans = [SlabPlan(p, nranks, r) for r in range(nranks)]
    full = [pl.local_state(phi, mu) for pl in plans]
    # every rank's halo rows wiped, then filled by the messages from the owners' own rows
    loc = []
    for pl, (lp, lm) in zip(plans, full):
        a, b = pl.own()
        st = np.concatenate([lp, lm]).copy()
        st[:, :a] = np.nan
        st[:, b:] = np.nan
        loc.append(st)
    for m in plans[0].messages:
        for f, s, d in zip(m.fields, m.src_rows, m.dst_rows):
            a, b = plans[m.src].own()
            assert a <= s < b, "a message reads a halo row"
            loc[m.dst][f, d] = loc[m.src][f, s]
    for pl, (lp, lm), st in zip(plans, full, loc):
        np.testing.assert_array_equal(st, np.concatenate([lp, lm]))
        own = pl.own_part(st)
        np.testing.assert_array_equal(own, np.concatenate([phi, mu])[:, pl.x0:pl.x1])
    # the plan of each rank names the same messages
    for pl in plans[1:]:
        assert [(m.src, m.dst, m.fields, m.src_rows, m.dst_rows) for m in pl.messages] == \
               [(m.src, m.dst, m.fields, m.src_rows, m.dst_rows) for m in plans[0].messages]


def test_remap_is_the_kernels_boundary_map():
    # Neumann mirrors about the boundary cell; periodic wraps with period m-1
    assert [remap(v, 10, 1, 1) for v in (-3, -2, -1, 10, 11, 12)] == [3, 2, 1, 8, 7, 6]
    assert [remap(v, 10, 3, 3) for v in (-3, -2, -1, 10, 11, 12)] == [6, 7, 8, 1, 2, 3]


def test_reduce_stats():
    st = {"phi_max": [1.0, 0.5], "phi_min": [0.0, -0.1], "mu_max": [2.0], "mu_min": [0.3],
          "rel_change_phi": [1e-3, 2e-3], "rel_change_mu": [4e-3], "phi_sum": [10.0, 20.0], "comp_sum": [3.0],
          "nonfinite": 1, "steps_done": 7}

    def two_ranks(a, op):   # the other rank holds twice the values
        b = 2 * a
        return {"max": np.maximum, "min": np.minimum, "sum": np.add}[op](a, b)
    r = reduce_stats(st, two_ranks)
    assert list(r["phi_max"]) == [2.0, 1.0] and list(r["phi_min"]) == [0.0, -0.2]
    assert list(r["phi_sum"]) == [30.0, 60.0] and r["nonfinite"] == 3 and r["steps_done"] == 7


class OracleSlab:
    """A rank's slab stepped by the CPU oracle (test infrastructure), rows
    moved through CPU tensors."""

    def __init__(self, plan, phi, mu):
        from oracle_py import Oracle
        self.plan = plan
        lp, lm = plan.local_state(phi, mu)
        self.o = Oracle(plan.local_params(), recip_div=1)
        self.o.set(lp, lm)

    def _state(self):
        ph, m = self.o.get()
        return np.concatenate([ph, m])

    def empty(self, n):
        import torch
        return torch.empty((n, self.plan.my), dtype=torch.float64)

    def pack(self, fields, rows):
        import torch
        st = self._state()
        return torch.from_numpy(np.ascontiguousarray(st[fields, rows]))

    def unpack(self, fields, rows, buf):
        st = self._state()
        st[fields, rows] = buf.numpy()
        self.o.set(st[:self.plan.N], st[self.plan.N:])

    def step(self, n):
        self.o.step(n)

    def smooth(self, n):
        self.o.smooth(n)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, tmpdir, name, nsmooth, nsteps, out):
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        _, _, p, phi, mu = _deck(os.path.join(tmpdir, "r%d" % rank), name)
        plan = SlabPlan(p, world, rank)
        run = SlabRunner(plan, OracleSlab(plan, phi, mu), TorchTransport(dist))
        run.smooth(nsmooth)
        run.step(nsteps)
        own = plan.own_part(run.stepper._state())
        # gather the own rows (objects: the slabs differ in size)
        got = [None] * world
        dist.all_gather_object(got, (plan.x0, plan.x1, own))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("neumann", 2), ("periodic", 2), ("mixed", 3)])
def test_gloo_ranks_match_whole_grid(tmp_path, name, world):
    import torch.multiprocessing as mp
    from oracle_py import Oracle, bits_equal, mismatch_report
    nsmooth, nsteps = 3, 12
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(tmp_path), name, nsmooth, nsteps, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    got = q.get(timeout=300)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    _, _, p, phi, mu = _deck(tmp_path / "whole", name)
    o = Oracle(p, recip_div=1)
    o.set(phi, mu)
    o.smooth(nsmooth)
    o.step(nsteps)
    ph, m = o.get()
    whole = np.concatenate([ph, m])
    stitched = np.concatenate([own for _, _, own in sorted(got, key=lambda g: g[0])], axis=1)
    assert [g[0] for g in sorted(got, key=lambda g: g[0])] == SlabPlan(p, world, 0).bounds[:-1]
    assert bits_equal(stitched, whole), mismatch_report(stitched, whole)
    assert not np.all((ph == 0) | (ph == 1))   # an interface crosses the grid
