"""Parity cases for the tests: small grids the CPU oracle finishes in seconds."""
import os

from eshwar_dipan_b200.workloads import filling_text, input_text, random_seeds, write_case  # noqa: F401

# Parity cases: small grids the CPU oracle finishes in seconds.  Each covers a
# branch of the reference step (see the `covers` text).
PARITY_CASES = {
    "bin_aniso_neumann": dict(
        covers="binary 2-phase, 4-fold anisotropy, obstacle, Neumann, dx=2 (power of two)",
        kw=dict(N=2, K=1, mesh=(48, 40), dx=2.0, dt=0.08, eps=8.0, dab=0.04, d_solid=1.0, T=0.96),
        seeds=[(0, 24, 20, 9.0)]),
    "bin_iso_antitrap": dict(
        covers="binary, isotropic, anti-trapping on (D_solid=0), seed touching the X- wall",
        kw=dict(N=2, K=1, mesh=(40, 44), aniso=False, dab=0.0, d_solid=0.0, dt=0.02),
        seeds=[(0, 20, 22, 8.0), (0, 2, 10, 5.0)]),
    "bin_aniso_periodic": dict(
        covers="binary anisotropic, periodic in x and y (period MESH-1), seeds across the wrap",
        kw=dict(N=2, K=1, mesh=(40, 36), bc_phi=(3, 3, 3, 3), dab=0.05),
        seeds=[(0, 1, 18, 6.0), (0, 30, 34, 5.0), (0, 20, 10, 4.5)]),
    "three_phase_rot45": dict(
        covers="3 phases, binary solute, anisotropy with a 45 degree rotated pair, Gamma_abc, mixed BCs",
        kw=dict(N=3, K=1, mesh=(44, 40), dab=[0.0, 0.02, 0.02], rot={(1, 2): 45.0}, bc_phi=(3, 3, 1, 1)),
        seeds=[(0, 14, 18, 8.0), (1, 30, 22, 7.0), (1, 20, 36, 5.0)]),
    "ternary3_aniso_periodic": dict(
        covers="3 phases, ternary (TERNARY closed-form 2x2 inverse), anisotropy, periodic",
        kw=dict(N=3, K=2, mesh=(40, 40), dab=0.02, bc_phi=(3, 3, 3, 3), A_off=0.25),
        seeds=[(0, 12, 12, 6.0), (1, 28, 26, 6.5), (0, 38, 2, 4.0)]),
    "four_phase_ternary_iso": dict(
        covers="4 phases, ternary, isotropic, periodic x / Neumann y",
        kw=dict(N=4, K=2, mesh=(36, 44), aniso=False, dab=0.0, bc_phi=(3, 3, 1, 1)),
        seeds=[(0, 10, 12, 6.0), (1, 26, 14, 6.0), (2, 18, 32, 6.0)]),
    "well_aniso": dict(
        covers="well potential (Function_W=2), anisotropy, binary",
        kw=dict(N=2, K=1, mesh=(40, 40), well=True, dab=0.03),
        seeds=[(0, 20, 20, 9.0)]),
    "dilute_three_phase": dict(
        covers="DILUTE inversion, K=2, 3 phases, dx=1.5 (true divisions)",
        kw=dict(N=3, K=2, mesh=(36, 36), mode="dilute", dx=1.5, dt=0.04, aniso=False, dab=0.0),
        seeds=[(0, 12, 12, 6.0), (1, 24, 24, 6.0)]),
    "dirsolid_binary": dict(
        covers="non-isothermal: a temperature gradient moving along y (Tempgrady), solid at the bottom, "
               "anisotropic, periodic x / Neumann y; T-dependent c(mu), Mu, B and C per cell",
        kw=dict(N=2, K=1, mesh=(40, 64), dab=0.03, bc_phi=(3, 3, 1, 1), d_solid=0.0, T=1.0, Teq=1.0,
                tempgrady=(0.97, 0.06, 60.0, 20.0, 0.5)),
        cubes=[(0, 0, 0, 39, 18)], seeds=[(0, 10, 19, 3.0), (0, 27, 19, 4.0)]),
    "dirsolid_ternary3": dict(
        covers="non-isothermal ternary 3-phase (TERNARY inversion), two solids growing from the bottom",
        kw=dict(N=3, K=2, mesh=(36, 56), dab=0.02, bc_phi=(3, 3, 1, 1), A_off=0.25, T=1.0, Teq=1.0,
                tempgrady=(0.97, 0.06, 60.0, 20.0, 0.5)),
        cubes=[(0, 0, 0, 17, 14), (1, 18, 0, 35, 14)], seeds=[(0, 9, 15, 3.0)]),
    "bin_mixed_bc": dict(
        covers="phi periodic in y, mu Neumann everywhere; different copy tables per field",
        kw=dict(N=2, K=1, mesh=(40, 40), bc_phi=(1, 1, 3, 3), bc_mu=(1, 1, 1, 1)),
        seeds=[(0, 20, 1, 7.0), (0, 10, 30, 5.0)]),
}


def build_case(tmpdir, name, ntimesteps=None):
    c = PARITY_CASES[name]
    kw = dict(c["kw"])
    if ntimesteps is not None:
        kw["ntimesteps"] = ntimesteps
    return write_case(str(tmpdir), name, kw, seeds=c.get("seeds", ()), cubes=c.get("cubes", ()))
