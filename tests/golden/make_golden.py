# SPDX-License-Identifier: MIT
"""Regenerate tests/golden/avbd_core_vectors.json.

Compiles gen_core_vectors.cpp against the reference checkout (its C++ mirror
of constraint_math.slang and its block fixtures) and stores the output. Run
in a checkout that has the reference:  python tests/golden/make_golden.py
[--ref /path/to/parallel-mater]. The GPU box never runs this script; it only
reads the committed JSON.
"""
import argparse
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PMB_REFERENCE_ROOT", "/root/reference"))
    args = ap.parse_args()
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "gen")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                        f"-I{args.ref}/src", f"-I{args.ref}/tests/solver",
                        os.path.join(HERE, "gen_core_vectors.cpp"), "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    data = json.loads(out)
    with open(os.path.join(HERE, "avbd_core_vectors.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print({k: len(v) for k, v in data.items() if isinstance(v, list)})


if __name__ == "__main__":
    main()
