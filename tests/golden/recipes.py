"""Inputs that reproduce the reference's shipped result files (DATA/*.vtk of the
serial grand-potential solver), as found by running the reference built from
source: the example Input.in of the solver (100x100, dx=2, dt=0.08, 2 phases,
binary, epsilon=8, obstacle, NSMOOTH=10, D_solid = D_liquid = 1) with

  output.out_1000.vtk      : T=0.96, Function_anisotropy=1, dab=0.04, 1000 steps
  Output_iso_<t>.vtk       : T=0.98, Function_anisotropy=0, t = 1000..10000
  output.out_0.vtk         : the t=0 state of either

and Filling.in = FILLCYLINDER = {0, 50, 50, 0, 0, 20}.  golden_vtk.npz holds the
files' values (make_golden.py).
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FILLING = "FILLCYLINDER = {0, 50, 50, 0, 0, 20};\n"

GOLDEN = {
    # key in golden_vtk.npz: (kind, steps, {field name in file: (field kind, index)})
    "output_out_0": ("aniso", 0, {"alpha": ("phi", 0), "beta": ("phi", 1), "Mu_C1": ("mu", 0)}),
    "output_out_1000": ("aniso", 1000, {"alpha": ("phi", 0), "beta": ("phi", 1), "Mu_Al": ("mu", 0)}),
}
for _t in range(1000, 10001, 1000):
    GOLDEN["Output_iso_%d" % _t] = ("iso", _t, {"alpha": ("phi", 0), "beta": ("phi", 1), "Mu_Al": ("mu", 0)})


def golden_input(kind, nsteps=1000):
    aniso = kind == "aniso"
    return "\n".join([
        "DIMENSION = 2;", "MESH_X = 100;", "MESH_Y = 100;", "MESH_Z = 1;",
        "DELTA_X = 2.0;", "DELTA_Y = 2.0;", "DELTA_Z = 2.0;", "DELTA_t = 0.08;",
        "NUMPHASES = 2;", "NUMCOMPONENTS = 2;",
        "NTIMESTEPS = %d;" % nsteps, "NSMOOTH = 10;", "SAVET = 1000;", "STARTTIME = 0;", "RESTART = 0;",
        "COMPONENTS = {Al, Cu};", "PHASES = {alpha, beta};",
        "GAMMA = {1.0};",
        "DIFFUSIVITY = {1, 0, 1};", "DIFFUSIVITY = {1, 1, 1};",
        "R = 1.0;", "V = 1.0;",
        "BOUNDARY = {phi, 1, 1, 1, 1, 0, 0};", "BOUNDARY = {mu, 1, 1, 1, 1, 0, 0};",
        "BOUNDARY = {c, 1, 1, 1, 1, 0, 0};", "BOUNDARY = {T, 1, 1, 1, 1, 0, 0};",
        "BOUNDARY_VALUE = {phi, 0, 0, 0, 0, 0, 0};", "BOUNDARY_VALUE = {mu, 0, 0, 0, 0, 0, 0};",
        "BOUNDARY_VALUE = {c, 0, 0, 0, 0, 0, 0};", "BOUNDARY_VALUE = {T, 0, 0, 0, 0, 0, 0};",
        "ISOTHERMAL = 1;", "BINARY = 1;", "DILUTE = 0;",
        "T = %s;" % ("0.96" if aniso else "0.98"),
        "WRITEFORMAT = ASCII;", "TRACK_PROGRESS = 1000;",
        "epsilon = 8.0;", "tau = 1.31;", "Tau = {0.28};",
        "Function_anisotropy = %d;" % (1 if aniso else 0),
        "Anisotropy_type = 4;", "dab = {0.04};", "Rotation_matrix = {0, 1, 0, 0, 0};",
        "Function_W = 1;", "Gamma_abc = {};",
        "Shift = 0;", "Shiftj = 30;", "Writecomposition = 0;",
        "Noise_phasefield = 0;", "Amp_Noise_Phase = 0.001;",
        "Equilibrium_temperature = 1.0;", "Filling_temperature = 1.0;",
        "Tempgrady = {0.96, 0.06, 800.0, 0, 0.016};",
        "Function_F = 1;",
        "A = {0, 1};", "A = {1, 1};",
        "ceq = {0, 0, 0.78125};", "ceq = {0, 1, 0.5};", "ceq = {1, 1, 0.5};", "ceq = {1, 0, 0.5};",
        "cfill = {0, 0, 0.78125};", "cfill = {0, 1, 0.5};", "cfill = {1, 1, 0.5};", "cfill = {1, 0, 0.5};",
        "slopes = {0, 0, 0.45};", "slopes = {0, 1, 0.45};", "slopes = {1, 0, 0.45};", "slopes = {1, 1, 0.45};",
    ]) + "\n"


def write_golden_case(dirpath, kind):
    ip = os.path.join(str(dirpath), "golden_%s.in" % kind)
    fp = os.path.join(str(dirpath), "golden_fill.in")
    with open(ip, "w") as f:
        f.write(golden_input(kind))
    with open(fp, "w") as f:
        f.write(FILLING)
    return ip, fp


def load_golden():
    return np.load(os.path.join(HERE, "golden_vtk.npz"))


def golden_text(npz, key, name):
    """The file's '%le' strings of one field, rebuilt from mantissa/exponent."""
    man = npz["%s__%s__man" % (key, name)]
    ex = npz["%s__%s__exp" % (key, name)]
    out = []
    for m, e in zip(man.tolist(), ex.tolist()):
        s = "-" if m < 0 else ""
        d = "%07d" % abs(m)
        out.append("%s%s.%se%+03d" % (s, d[0], d[1:], e))
    return out


def as_le(values):
    """Format like C's "%le" (glibc rounds correctly, as Python does)."""
    return ["%.6e" % v for v in np.asarray(values).ravel().tolist()]
