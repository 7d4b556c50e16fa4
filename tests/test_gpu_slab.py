"""Slabs on the GPU: a grid split along x into slab contexts (gp_set_stat_rows,
gp_rows_pack / gp_rows_unpack through CUDA tensors), the halo rows swapped
after every step, gives the whole-grid context's fields bit for bit and, with
the statistics of each slab's own rows reduced over the slabs, its progress
record (extremes exactly, sums to rounding).  The slabs run as contexts of one
process on one GPU, one after another, so that nothing waits on another
launch; between GPUs the same messages go through NCCL (TorchTransport)."""
import numpy as np
import pytest

import eshwar_dipan_b200 as gp
from eshwar_dipan_b200.slab import GpuSlab, SlabPlan, reduce_stats
from eshwar_dipan_b200.workloads import workload
from oracle_py import bits_equal, mismatch_report

pytestmark = pytest.mark.gpu


class InProcess:
    """The slabs' exchange inside one process: every pack first, then a
    device-wide wait, then every unpack."""

    def __init__(self, plans, slabs):
        self.plans, self.slabs = plans, slabs

    def exchange(self):
        import torch
        moved = []
        for m in self.plans[0].messages:
            moved.append((m, self.slabs[m.src].pack(m.fields, m.src_rows)))
        torch.cuda.synchronize()
        for m, buf in moved:
            self.slabs[m.dst].unpack(m.fields, m.dst_rows, buf)
        torch.cuda.synchronize()


def _allreduce_over(values):
    def red(_, op):
        a = np.stack(values.pop(0))
        return {"max": a.max(axis=0), "min": a.min(axis=0), "sum": a.sum(axis=0)}[op]
    return red


@pytest.mark.parametrize("name,scale,nslabs", [("cfg4", 8, 4), ("cfg2", 8, 3), ("cfg1", 1, 2)])
def test_slabs_match_whole_grid(tmp_path, name, scale, nslabs):
    import torch
    it, ft, desc, _ = workload(name, scale)
    ip, fp = str(tmp_path / "i.in"), str(tmp_path / "f.in")
    open(ip, "w").write(it)
    open(fp, "w").write(ft)
    p = gp.load_params(ip)
    phi, mu = gp.fill(p, fp)
    plans = [SlabPlan(p, nslabs, r) for r in range(nslabs)]
    slabs = [GpuSlab(pl, phi, mu) for pl in plans]
    ex = InProcess(plans, slabs)
    try:
        with gp.Simulation(p, phi, mu) as whole:
            whole.smooth(p.nsmooth - 1)
            for _ in range(p.nsmooth - 1):
                for s in slabs:
                    s.smooth(1)
                ex.exchange()
            done = 0
            for n in (1, 30, 69):
                for k in range(n):
                    last = k == n - 1
                    for s in slabs:
                        if last:
                            s.step_stats(1)
                        else:
                            s.step(1)
                    ex.exchange()
                st = whole.step(n)
                done += n
                a_phi, a_mu = whole.get()
                parts = [s.get() for s in slabs]
                b_phi = np.concatenate([q[0] for q in parts], axis=1)
                b_mu = np.concatenate([q[1] for q in parts], axis=1)
                assert bits_equal(b_phi, a_phi), "%s phi after %d steps: %s" % (desc, done, mismatch_report(b_phi, a_phi))
                assert bits_equal(b_mu, a_mu), "%s mu after %d steps: %s" % (desc, done, mismatch_report(b_mu, a_mu))
                sts = [s.stats() for s in slabs]
                keys = ("phi_max", "mu_max", "phi_min", "mu_min", "rel_change_phi", "rel_change_mu", "phi_sum",
                        "comp_sum")
                vals = [[np.asarray(x[k], dtype=np.float64) for x in sts] for k in keys]
                vals.append([np.asarray([x["nonfinite"]], dtype=np.float64) for x in sts])
                r = reduce_stats(sts[0], _allreduce_over(vals))
                for k in ("phi_max", "phi_min", "mu_max", "mu_min"):
                    np.testing.assert_array_equal(r[k], st[k], err_msg=k)
                for k in ("rel_change_phi", "rel_change_mu", "phi_sum", "comp_sum"):
                    np.testing.assert_allclose(r[k], st[k], rtol=1e-10, atol=1e-300, err_msg=k)
                assert r["nonfinite"] == st["nonfinite"] == 0
            assert not np.all((a_phi == 0) | (a_phi == 1))
    finally:
        for s in slabs:
            s.close()
        torch.cuda.synchronize()
