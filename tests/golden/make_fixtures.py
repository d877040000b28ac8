"""Copy the reference's shipped collapse tables into tests/golden/ as fixtures.

The tables are data produced by the reference's ellipsoidal-collapse solver (50x20x20
Float32 zvir(log10 F, e, p/e) in the HomelTab binary layout: 3 x Int32 + 6 x Float32
header, then the column-major table).  They are inputs to the radial-shell collapse and
to the Fortran golden-vector test (test/test_radialshell_fortran.jl), and must travel
with the repository because the reference tree is not available where the GPU tests and
the benchmark run.  Run this once in a container that has the reference checkout:

    python tests/golden/make_fixtures.py /path/to/Huntian.jl

It copies test/data/HomelTab_fortran.dat and test/data/HomelTab_julia.dat byte for byte
and writes their SHA-256 digests to tables.sha256.
"""
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = ["HomelTab_fortran.dat", "HomelTab_julia.dat"]


def main(ref_root: str) -> None:
    lines = []
    for name in TABLES:
        src = os.path.join(ref_root, "test", "data", name)
        dst = os.path.join(HERE, name)
        shutil.copyfile(src, dst)
        digest = hashlib.sha256(open(dst, "rb").read()).hexdigest()
        lines.append(f"{digest}  {name}\n")
    with open(os.path.join(HERE, "tables.sha256"), "w") as f:
        f.writelines(lines)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path of the Huntian.jl checkout>")
    main(sys.argv[1])
