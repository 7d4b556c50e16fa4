"""Input.in / Filling.in generators (synthetic MicroSim input decks).

The text follows the reference's key = value; format (Input.in of the serial
solver), so the same files drive the product parser, the oracle and the
reference itself.  Numbers are written with repr() of short decimals so every
program parses identical doubles.
"""
import math
import os

PHASE_NAMES = ["alpha", "beta", "gamma", "delta", "eps", "zeta"]
COMP_NAMES = ["Al", "Cu", "Ni", "Zn", "Mg"]


def _fmt(v):
    if isinstance(v, int):
        return str(v)
    s = repr(float(v))
    return s


def input_text(N=2, K=1, mesh=(48, 40), dx=1.0, dy=None, dt=0.02, eps=4.0, tau_ab=0.28, tau=1.31,
               gamma=1.0, gamma_abc=10.0, aniso=True, dab=0.02, rot=None, well=False,
               bc_phi=(1, 1, 1, 1), bc_mu=None, mode=None, T=0.97, Teq=1.0,
               d_liquid=None, d_solid=0.0, A_off=0.0, nsmooth=10, ntimesteps=100, ascii=True,
               writecomposition=0, liquid_c=None, extra="", tempgrady=None, shift=False, shiftj=30,
               bc_T=None):
    """Reference-format Input.in for N phases (the last one liquid) and K solutes.

    bc_* = (X+, X-, Y+, Y-) in the reference's BOUNDARY tuple order.
    mode: 'binary' | 'ternary' | 'dilute' | 'none' (default: binary for K=1,
    ternary for K=2).
    tempgrady: None (isothermal), or (base temperature, DeltaT, Distance,
    OFFSET, velocity): ISOTHERMAL = 0 with that moving temperature gradient
    along y (directional solidification).  shift: the moving frame, which
    follows the interface once it passes column shiftj.
    """
    dy = dx if dy is None else dy
    bc_mu = bc_phi if bc_mu is None else bc_mu
    if mode is None:
        mode = "binary" if K == 1 else "ternary"
    L = N - 1
    pairs = [(a, b) for a in range(N) for b in range(a + 1, N)]
    triples = [(a, b, c) for a in range(N) for b in range(a + 1, N) for c in range(b + 1, N)]
    lines = []
    add = lines.append
    add("DIMENSION = 2;")
    add("MESH_X = %d;" % mesh[0])
    add("MESH_Y = %d;" % mesh[1])
    add("MESH_Z = 1;")
    add("DELTA_X = %s;" % _fmt(dx))
    add("DELTA_Y = %s;" % _fmt(dy))
    add("DELTA_Z = %s;" % _fmt(dx))
    add("DELTA_t = %s;" % _fmt(dt))
    add("NUMPHASES = %d;" % N)
    add("NUMCOMPONENTS = %d;" % (K + 1))
    add("NTIMESTEPS = %d;" % ntimesteps)
    add("NSMOOTH = %d;" % nsmooth)
    add("SAVET = %d;" % ntimesteps)
    add("STARTTIME = 0;")
    add("RESTART = 0;")
    add("COMPONENTS = {%s};" % ", ".join(COMP_NAMES[: K + 1]))
    add("PHASES = {%s};" % ", ".join(PHASE_NAMES[: N - 1] + ["liquid"]))
    add("GAMMA = {%s};" % ", ".join(_fmt(gamma) for _ in pairs))
    dl = d_liquid if d_liquid is not None else [1.0, 0.5, 0.75][:K]
    for a in range(N):
        vals = dl if a == L else [d_solid] * K
        add("DIFFUSIVITY = {1, %d, %s};" % (a, ", ".join(_fmt(v) for v in vals)))
    add("R = 1.0;")
    add("V = 1.0;")
    bc_T = bc_mu if bc_T is None else bc_T
    for f, bc in (("phi", bc_phi), ("mu", bc_mu), ("c", bc_mu), ("T", bc_T)):
        add("BOUNDARY = {%s, %d, %d, %d, %d, 0, 0};" % ((f,) + tuple(bc)))
    for f in ("phi", "mu", "c", "T"):
        add("BOUNDARY_VALUE = {%s, 0, 0, 0, 0, 0, 0};" % f)
    add("ISOTHERMAL = %d;" % (0 if tempgrady else 1))
    if mode == "binary":
        add("BINARY = 1;")
    elif mode == "ternary":
        add("TERNARY = 1;")
    elif mode == "dilute":
        add("DILUTE = 1;")
    add("T = %s;" % _fmt(T))
    add("WRITEFORMAT = %s;" % ("ASCII" if ascii else "BINARY"))
    add("TRACK_PROGRESS = 10;")
    add("epsilon = %s;" % _fmt(eps))
    add("tau = %s;" % _fmt(tau))
    add("Tau = {%s};" % ", ".join(_fmt(tau_ab) for _ in pairs))
    add("Function_anisotropy = %d;" % (1 if aniso else 0))
    add("Anisotropy_type = 4;")
    dabv = dab if isinstance(dab, (list, tuple)) else [dab] * len(pairs)
    add("dab = {%s};" % ", ".join(_fmt(v) for v in dabv))
    rot = rot or {}
    for (a, b) in pairs:
        add("Rotation_matrix = {%d, %d, 0, 0, %s};" % (a, b, _fmt(rot.get((a, b), 0.0))))
    add("Function_W = %d;" % (2 if well else 1))
    add("Gamma_abc = {%s};" % ", ".join(_fmt(gamma_abc) for _ in triples))
    add("Shift = %d;" % (1 if shift else 0))
    add("Shiftj = %d;" % shiftj)
    add("Writecomposition = %d;" % writecomposition)
    add("Noise_phasefield = 0;")
    add("Amp_Noise_Phase = 0.0;")
    add("Equilibrium_temperature = %s;" % _fmt(Teq))
    add("Filling_temperature = 1.0;")
    tg = tempgrady if tempgrady else (0.96, 0.06, 800.0, 0, 0.016)
    add("Tempgrady = {%s};" % ", ".join(_fmt(v) for v in tg))
    add("Function_F = 1;")
    for a in range(N):
        if K == 1:
            add("A = {%d, 1.0};" % a)
        else:
            add("A = {%d, %s, %s};" % (a, ", ".join("1.0" for _ in range(K)),
                                       ", ".join(_fmt(A_off) for _ in range(K * (K - 1) // 2))))
    # equilibrium compositions: solids pulled towards one solute each, liquid in the middle
    def c_solid(a):
        if K == 1:
            return [0.2 if a % 2 == 0 else 0.8]
        base = [0.15] * K
        if a < K:
            base[a] = 0.7
        return base
    c_liq = [0.5] if K == 1 else [0.33] * K
    c_fill = liquid_c if liquid_c is not None else ([0.45] if K == 1 else [0.3] * K)
    for key in ("ceq", "cfill"):
        for a in range(L):
            cs = c_solid(a)
            add("%s = {%d, %d, %s};" % (key, a, a, ", ".join(_fmt(v) for v in cs)))
            add("%s = {%d, %d, %s};" % (key, a, L, ", ".join(_fmt(v) for v in c_liq)))
            add("%s = {%d, %d, %s};" % (key, L, a, ", ".join(_fmt(v) for v in c_liq)))
        cl = c_liq if key == "ceq" else c_fill
        add("%s = {%d, %d, %s};" % (key, L, L, ", ".join(_fmt(v) for v in cl)))
    for a in range(L):
        sl = [0.45 if (a % 2 == 0) else -0.45] + [0.1] * (K - 1)
        for (p1, p2) in ((a, a), (a, L), (L, a)):
            add("slopes = {%d, %d, %s};" % (p1, p2, ", ".join(_fmt(v) for v in sl)))
    add("slopes = {%d, %d, %s};" % (L, L, ", ".join("0.45" for _ in range(K))))
    if extra:
        lines.extend(extra.strip().splitlines())
    return "\n".join(lines) + "\n"


def filling_text(seeds=(), cubes=()):
    """seeds: (phase, x, y, r) cylinders; cubes: (phase, x0, y0, x1, y1)."""
    out = []
    for (ph, x0, y0, x1, y1) in cubes:
        out.append("FILLCUBE = {%d, %d, %d, 0, %d, %d, 0};" % (ph, x0, y0, x1, y1))
    for (ph, x, y, r) in seeds:
        out.append("FILLCYLINDER = {%d, %d, %d, 0, 0, %s};" % (ph, x, y, _fmt(r)))
    return "\n".join(out) + "\n"


def write_case(dirpath, name, input_kwargs, seeds=(), cubes=()):
    os.makedirs(dirpath, exist_ok=True)
    ip = os.path.join(dirpath, name + ".in")
    fp = os.path.join(dirpath, name + "_fill.in")
    with open(ip, "w") as f:
        f.write(input_text(**input_kwargs))
    with open(fp, "w") as f:
        f.write(filling_text(seeds, cubes))
    return ip, fp


class SplitMix64:
    """Deterministic PRNG for synthetic seed layouts (splitmix64)."""

    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    def uniform(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def random_seeds(n, mesh, rmin, rmax, nsolid, seed=0):
    """n cylinders with uniform centres, r ~ U[rmin, rmax] (rounded to 0.5), random solid phase."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(n):
        x = int(rng.uniform() * mesh[0])
        y = int(rng.uniform() * mesh[1])
        r = round((rmin + (rmax - rmin) * rng.uniform()) * 2) / 2.0
        ph = int(rng.uniform() * nsolid) % nsolid
        out.append((ph, x, y, r))
    return out


def ensemble(n=256, seed=0, side_min=128, side_max=1024, shrink=1):
    """Batched-ensemble decks: n independent binary 2-phase simulations, side
    32*round(logU[side_min, side_max]/32) (divided by shrink, at least 32),
    liquid composition c0 ~ U[0.40, 0.48], anisotropy strength delta ~ U[0, 0.05],
    1..8 solid seeds with uniform centres and r ~ U[4, 12].  Returns a list of
    (input kwargs, seeds)."""
    rng = SplitMix64(seed)
    out = []
    lo, hi = math.log(side_min), math.log(side_max)
    for s in range(n):
        side = 32 * int(round(math.exp(lo + (hi - lo) * rng.uniform()) / 32.0))
        side = max(32, side // shrink // 32 * 32 if shrink > 1 else side)
        c0 = round(0.40 + 0.08 * rng.uniform(), 6)
        delta = round(0.05 * rng.uniform(), 6)
        nseeds = 1 + int(8 * rng.uniform()) % 8
        kw = dict(N=2, K=1, mesh=(side, side), aniso=True, dab=delta, d_solid=0.0, d_liquid=[1.0], dt=0.02,
                  eps=4.0, T=1.0, liquid_c=[c0])
        out.append((kw, random_seeds(nseeds, (side, side), 4.0, 12.0, 1, seed=seed * 1000003 + s + 1)))
    return out


def workload(name, scale=1):
    """(Input.in text, Filling.in text, description, input kwargs) of a
    benchmark configuration:
      cfg1  256^2 binary 2-phase, isotropic, Neumann, one supercritical seed r=40
      cfg2  2048^2 ternary 3-phase, 4-fold anisotropy 0.02, periodic, 64 seeds
      cfg3  member 0 of the batched ensemble (see ensemble())
      cfg4  4096^2 ternary 3-phase, isotropic, Neumann, 256 seeds
      cfg5  512^2 binary 2-phase dendrite, anisotropy 0.04, one seed r=12
    scale > 1 shrinks the grid by that factor per axis with the same seed
    density (at least one seed)."""
    if name == "cfg2":
        m = 2048 // scale
        nseeds = max(1, 64 // (scale * scale))
        kw = dict(N=3, K=2, mesh=(m, m), dab=0.02, bc_phi=(3, 3, 3, 3), d_liquid=[1.0, 0.5], d_solid=0.0,
                  A_off=0.0, dt=0.02, eps=4.0, T=0.97)
        seeds = random_seeds(nseeds, (m, m), 4.0, 12.0, 2, seed=0)
        desc = "%dx%d ternary 3-phase FP64, aniso 0.02, periodic, %d seeds r~U[4,12]" % (m, m, nseeds)
    elif name == "cfg4":
        m = 4096 // scale
        nseeds = max(1, 256 // (scale * scale))
        kw = dict(N=3, K=2, mesh=(m, m), dab=0.0, aniso=False, bc_phi=(1, 1, 1, 1), d_liquid=[1.0, 0.5],
                  d_solid=0.0, dt=0.02, eps=4.0, T=0.97)
        seeds = random_seeds(nseeds, (m, m), 4.0, 12.0, 2, seed=0)
        desc = "%dx%d ternary 3-phase FP64, isotropic, Neumann, %d seeds" % (m, m, nseeds)
    elif name == "cfg3":
        kw, seeds = ensemble(shrink=scale)[0]
        kw = dict(kw)
        m = kw["mesh"][0]
        desc = ("ensemble member 0: %dx%d binary 2-phase, delta %.4f, c0 %.4f, %d seeds"
                % (m, m, kw["dab"], kw["liquid_c"][0], len(seeds)))
    elif name == "cfg5":
        m = 512 // scale
        kw = dict(N=2, K=1, mesh=(m, m), aniso=True, dab=0.04, d_solid=0.0, d_liquid=[1.0], dt=0.02, eps=4.0,
                  T=1.0, liquid_c=[0.42])
        seeds = [(0, m // 2, m // 2, 12.0 / scale)]
        desc = "%dx%d binary 2-phase dendrite FP64, aniso 0.04, Neumann, one seed r=12" % (m, m)
    elif name == "cfg1":
        m = 256 // scale
        kw = dict(N=2, K=1, mesh=(m, m), aniso=False, dab=0.0, d_solid=0.0, d_liquid=[1.0], dt=0.02, eps=4.0,
                  T=1.0, liquid_c=[0.45])
        seeds = [(0, m // 2, m // 2, 40.0 / scale)]
        desc = "%dx%d binary 2-phase FP64, isotropic, Neumann, one supercritical seed r=40" % (m, m)
    else:
        raise ValueError("unknown workload " + name)
    return input_text(**kw), filling_text(seeds), desc, kw


def write_workload(d, name, scale=1):
    """workload() written to d/<name>.in and d/<name>_fill.in: (paths, description, kwargs)."""
    it, ft, desc, kw = workload(name, scale)
    ip, fp = os.path.join(d, name + ".in"), os.path.join(d, name + "_fill.in")
    open(ip, "w").write(it)
    open(fp, "w").write(ft)
    return ip, fp, desc, kw
