"""Regenerate the golden fixtures in this directory from the reference itself.

Runs the reference's own sources (diskfft/src/hydro.hpp, kalnajs.hpp, diskmain.cpp,
test_kalnajs.cpp), compiled unmodified against the project's FFTW shim by
`make -C oracle ref` into oracle/_ref/, and stores their outputs:

  ref_<case>.npz        fields from oracle/_ref/refdump: the standard-disk initial state,
                        its potential and forces, the dt sequence, and the state after
                        n steps of timestep -> potential -> forces -> step
  test_kalnajs_ref.txt  stdout of the reference's known-answer test (FFT vs direct sum)
  diskdisk_ref_<case>/  modes table + stdout of a short unmodified `diskdisk` run

Needs the reference tree (only present where the fixtures are generated); the tests
read only the committed outputs.  Usage: python tests/golden/make_golden.py
"""
import argparse
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# name: (Nu, Nphi, eps, selfgrav, amp, nsteps)
CASES = {
    "32x32_sg": (32, 32, 0.02, 1, 1e-3, 20),
    "48x40_sg": (48, 40, 0.01, 1, 5e-2, 15),
    "16x24_nosg": (16, 24, 0.02, 0, 5e-2, 30),
    "64x64_strong": (64, 64, 0.005, 1, 0.2, 40),
    "8x12_sg": (8, 12, 0.04, 1, 0.1, 25),
    "24x27_odd": (24, 27, 0.02, 1, 0.1, 12),
    # general-Gamma disks of the sweep law (hydro.hpp:45-46 with Gamma != 2): the physics
    # of two sweep points, as dg_params_physical maps (Q_min, M_d/M_*, softening/r, Gamma)
    # (1.1, 0.3, 0.15, 1.5) and (1.6, 0.8, 0.07, 1.75); the second has its K capped
    "40x48_g1.5": (40, 48, 0.0225, 1, 5e-2, 20),
    "32x40_g1.75": (32, 40, 0.0049, 1, 0.1, 20),
}

# name: (gamma_gas, Kpoly, S0) for the cases whose physics differs from diskmain.cpp:28-29
PHYSICS = {
    "40x48_g1.5": (1.5, 0.08770103346609004, 0.16741633318186389),
    "32x40_g1.75": (1.75, 0.1975331689842986, 0.44644355515163703),
}
STANDARD_PHYSICS = (2.0, 0.25, 0.372)

DISKDISK = {
    # name: argv of diskdisk (Nu Nphi eps tlim selfgrav amp nthreads)
    "64_t1": ["64", "64", "0.01", "1.0", "1", "1e-3", "1"],
    # the growth-rate-versus-softening runs of diskfft/README.md:25-27 (128^2, to t = 9)
    "128_e0.02_t9": ["128", "128", "0.02", "9", "1", "1e-3", "8"],
    "128_e0.005_t9": ["128", "128", "0.005", "9", "1", "1e-3", "8"],
    "128_e0.0025_t9": ["128", "128", "0.0025", "9", "1", "1e-3", "8"],
    # through saturation (README.md:41-42 quotes |C2|/|C0| = 0.24, Omega_p 1.46 -> 1.34)
    "256_e0.005_t20": ["256", "256", "0.005", "20", "1", "1e-3", "8"],
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", help="regenerate only these fixtures (names above)")
    a = ap.parse_args()
    want = (lambda n: True) if not a.only else (lambda n: n in a.only)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref"], check=True)
    ref = os.path.join(ROOT, "oracle", "_ref")
    tmp = os.path.join(HERE, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    for name, (Nu, Nphi, eps, sg, amp, n) in CASES.items():
        if not want(name):
            continue
        out = os.path.join(tmp, name + ".bin")
        phys = PHYSICS.get(name, STANDARD_PHYSICS)
        extra = ["1"] + [repr(x) for x in phys] if name in PHYSICS else []
        subprocess.run([os.path.join(ref, "refdump"), str(Nu), str(Nphi), repr(eps), str(sg),
                        repr(amp), str(n), out] + extra, check=True)
        r = O.read_refdump(out)
        r["gamma_gas"], r["Kpoly"], r["S0"] = phys
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **{k: np.asarray(v) for k, v in r.items()})
    if want("test_kalnajs_ref"):
        res = subprocess.run([os.path.join(ref, "test_kalnajs_ref")], capture_output=True, text=True)
        with open(os.path.join(HERE, "test_kalnajs_ref.txt"), "w") as f:
            f.write(res.stdout)
            f.write(f"exit={res.returncode}\n")
    for name, argv in DISKDISK.items():
        if not want(name):
            continue
        d = os.path.join(HERE, f"diskdisk_ref_{name}")
        os.makedirs(d, exist_ok=True)
        res = subprocess.run([os.path.join(ref, "diskdisk_ref")] + argv, capture_output=True, text=True,
                             cwd=d, check=True)
        with open(os.path.join(d, "stdout.txt"), "w") as f:
            f.write(res.stdout)
        with open(os.path.join(d, "argv.txt"), "w") as f:
            f.write(" ".join(argv) + "\n")
    shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
