"""Generates cie_tables.json from the reference's colour-matching data.

The film of the reference integrates spectra against the CIE colour-matching
functions and converts RGB inputs with a BT.709 spectral basis; both tables
are read at start-up from lib/numli/data/ (cg.hpp:329-337):

  xyz_{x,y,z}.csv                     "λ,value" rows, 390-830 nm at 5 nm
  cie1931-basis-bt709-380+5+780.csv   "r,g,b" rows, 380-780 nm at 5 nm

The device film must use the same tables for its images to match, and the
reference tree is not available where this library runs, so this script
records the table entries verbatim (as the decimal strings of the files, so
that parsing them with strtof reproduces the reference's floats bit for
bit).  Run it where the reference is mounted:

    python lambda_b200/data/gen_cie_tables.py /path/to/reference
"""
import json
import os
import sys


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LAMBDA_REFERENCE", "")
    if not ref:
        sys.exit("usage: gen_cie_tables.py <reference source tree> (or set LAMBDA_REFERENCE)")
    d = os.path.join(ref, "lib", "numli", "data")
    out = {"source": "lib/numli/data of the reference (CIE colour-matching "
                     "functions and BT.709 spectral basis)"}
    for axis in "xyz":
        rows = []
        with open(os.path.join(d, f"xyz_{axis}.csv")) as f:
            for line in f:
                line = line.strip()
                if not line:
                    continue
                lam, val = line.split(",")[:2]
                rows.append([lam.strip(), val.strip()])
        out[f"cmf_{axis}"] = rows
    basis = []
    with open(os.path.join(d, "cie1931-basis-bt709-380+5+780.csv")) as f:
        for line in f:
            line = line.strip()
            if line:
                basis.append([c.strip() for c in line.split(",")[:3]])
    out["bt709_basis"] = {"lambda_min": 380.0, "lambda_step": 5.0,
                          "rows": basis}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "cie_tables.json"), "w") as f:
        json.dump(out, f, indent=0)


if __name__ == "__main__":
    main()
