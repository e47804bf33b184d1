#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden from the reference itself.

The dumps are written by the reference's own generator (test/gen_dump.py) with
the seeds and sizes the reference's end-to-end suite uses (test/test_sqcalc.py
sections 1, 2, 2b, 5, 9b), and the S(q) tables by the reference's own numpy
direct sum (test/ref_sq.py).  Both scripts run here unchanged; this file only
drives them.  Run from the repository root with the reference checked out:

    python tests/golden/make_golden.py <path of the sqcalc checkout>

It rewrites tests/golden/*.dump, *.dat and cases.json.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# name -> gen_dump.py arguments (test/test_sqcalc.py:179-306, :817-819)
DUMPS = {
    "gas": dict(natoms=250, length=20, frames=4, seed=7),
    "tri": dict(natoms=150, length=18, frames=3, seed=11, tilt="1.5 0.5 -2.0",
                columns="id xu yu zu type"),
    "lattice": dict(natoms=125, length=20, frames=3, seed=3, mode="lattice", fractions="1.0"),
    "ka": dict(natoms=400, length=16, frames=3, seed=5, fractions="0.8,0.2"),
}

# ref_sq.py runs: (case name, dump, mapping, weight, norm, qmin, qmax, nq)
CASES = [
    ("gas_unit_self", "gas", "1:Si,2:O", "unit", "self", 0.0, 6.0, 120),
    ("gas_neutron_mean", "gas", "1:Si,2:O", "neutron", "mean", 0.0, 6.0, 120),
    ("gas_xray_mean", "gas", "1:Si,2:O", "xray", "mean", 0.0, 6.0, 120),
    ("gas_ion_xray_mean", "gas", "1:Si4+,2:O2-", "xray", "mean", 0.0, 6.0, 120),
    ("gas_unit_n_window", "gas", "1:Si,2:O", "unit", "n", 0.5, 5.9, 27),
    ("tri_unit_self", "tri", "1:Si,2:O", "unit", "self", 0.0, 6.0, 120),
    ("lattice_unit_self", "lattice", "1:Si", "unit", "self", 0.0, 6.0, 120),
    ("ka_unit_mean", "ka", "1:Si,2:O", "unit", "mean", 0.0, 6.0, 120),
]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the sqcalc checkout>")
    ref = sys.argv[1]
    gen = os.path.join(ref, "test", "gen_dump.py")
    refsq = os.path.join(ref, "test", "ref_sq.py")
    for name, kw in DUMPS.items():
        cmd = [sys.executable, gen, "--output", os.path.join(HERE, name + ".dump")]
        for key, value in kw.items():
            flag = "--" + key.replace("_", "-")
            cmd += [flag] + str(value).split() if key == "tilt" else [flag, str(value)]
        subprocess.run(cmd, check=True)
    meta = []
    for case, dump, mapping, weight, norm, qmin, qmax, nq in CASES:
        out = os.path.join(HERE, case + ".dat")
        subprocess.run([sys.executable, refsq, "--input", os.path.join(HERE, dump + ".dump"),
                        "--mapping", mapping, "--weight", weight, "--norm", norm,
                        "--qmin", str(qmin), "--qmax", str(qmax), "--nq", str(nq),
                        "--output", out], check=True)
        meta.append(dict(case=case, dump=dump + ".dump", mapping=mapping, weight=weight,
                         norm=norm, qmin=qmin, qmax=qmax, nq=nq, table=case + ".dat"))
    with open(os.path.join(HERE, "cases.json"), "w") as fh:
        json.dump(dict(generator="test/gen_dump.py + test/ref_sq.py of thatstar/sqcalc",
                       dumps=DUMPS, cases=meta), fh, indent=1)
    print("wrote", len(meta), "golden tables")


if __name__ == "__main__":
    main()
