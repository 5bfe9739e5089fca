"""Shared test helpers."""
import glob
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def rel_err(a, b):
    """max |a - b| / max |b| (max-norm relative error of a field)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / den


def golden_physics(g):
    """(gamma_gas, Kpoly, S0) of a golden case; the standard disk (diskmain.cpp:28-29) when
    the fixture does not carry them."""
    return (float(g["gamma_gas"]) if "gamma_gas" in g else 2.0, float(g["Kpoly"]) if "Kpoly" in g else 0.25,
            float(g["S0"]) if "S0" in g else 0.372)


def golden_cases():
    out = {}
    for f in sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))):
        name = os.path.basename(f)[4:-4]
        z = np.load(f)
        out[name] = {k: z[k] for k in z.files}
    return out


def parse_header_symbols(path=os.path.join(ROOT, "include", "diskgpu.h")):
    """Function names declared in a C header (lines of the form `type name(`)."""
    import re
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dg_[a-z0-9_]+)\s*\(", txt)))
