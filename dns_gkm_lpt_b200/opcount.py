"""Regenerate dns_gkm_lpt_b200/opcount.json, the algorithmic FP64 operation
count of one cell update used as the roofline numerator by bench.py.

    python -m dns_gkm_lpt_b200.opcount

Compiles csrc/opcount.cpp (the device numerics instantiated on the host with
an operation-counting scalar) with g++ and runs it.
"""
import json
import os
import subprocess
import tempfile

PKG = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(PKG, "opcount.json")


def generate() -> dict:
    exe = os.path.join(tempfile.mkdtemp(), "opcount")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(PKG, "csrc"),
                    os.path.join(PKG, "csrc", "opcount.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    data = json.loads(out)
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
    return data


def load() -> dict:
    with open(OUT) as f:
        return json.load(f)


if __name__ == "__main__":
    d = generate()
    print(d["flops_per_cell_update"], "flops per cell update ->", OUT)
