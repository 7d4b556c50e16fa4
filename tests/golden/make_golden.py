"""Extract the reference's shipped result files into a test fixture.

Reads Grand_potential_Finite_difference_2D_serial/DATA/*.vtk of the reference
(ASCII legacy VTK, '%le' values, 100x100, 2 phases, 1 solute) and stores every
value as its decimal mantissa (int32, 7 digits) and exponent (int8), which is
exact for '%le' text, in golden_vtk.npz next to this script.

    python tests/golden/make_golden.py /path/to/reference

The recipes that reproduce these files (edits to the reference's Input.in,
Filling.in = one FILLCYLINDER = {0, 50, 50, 0, 0, 20}) are in recipes.json.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_vtk(path):
    lines = open(path).read().split("\n")
    out = {}
    i = 0
    while i < len(lines):
        if lines[i].startswith("SCALARS"):
            name = lines[i].split()[1]
            vals = []
            j = i + 2
            while j < len(lines) and lines[j].strip() and not lines[j].startswith("SCALARS"):
                vals.append(lines[j].strip())
                j += 1
            out[name] = vals
            i = j
        else:
            i += 1
    return out


def encode(vals):
    man = np.zeros(len(vals), dtype=np.int32)
    ex = np.zeros(len(vals), dtype=np.int8)
    for n, v in enumerate(vals):
        m = re.fullmatch(r"(-?)(\d)\.(\d{6})e([+-]\d+)", v)
        assert m, v
        sign = -1 if m.group(1) else 1
        man[n] = sign * int(m.group(2) + m.group(3))
        ex[n] = int(m.group(4))
    return man, ex


def main(ref):
    data_dir = os.path.join(ref, "Grand_potential_Finite_difference_2D_serial", "DATA")
    arrays = {}
    for fn in sorted(os.listdir(data_dir)):
        if not fn.endswith(".vtk"):
            continue
        fields = parse_vtk(os.path.join(data_dir, fn))
        key = fn[:-4].replace(".", "_")
        for name, vals in fields.items():
            man, ex = encode(vals)
            arrays["%s__%s__man" % (key, name)] = man
            arrays["%s__%s__exp" % (key, name)] = ex
    np.savez_compressed(os.path.join(HERE, "golden_vtk.npz"), **arrays)
    print("wrote", len(arrays) // 2, "fields")


def decode(npz, key, name):
    man = npz["%s__%s__man" % (key, name)].astype(np.float64)
    ex = npz["%s__%s__exp" % (key, name)].astype(np.float64)
    return man * 10.0 ** (ex - 6)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
