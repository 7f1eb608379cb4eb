"""Builds the CPU oracle (oracle.c -> oracle/liboracle.so) and, when the
reference sources are present, the reference library (build_ref.sh ->
oracle/_ref/libcuhc.so). Test infrastructure only.

    python oracle/build.py
"""

import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
SOURCE = HERE / "oracle.c"
LIBRARY = HERE / "liboracle.so"


def build_oracle(force=False):
    if not force and LIBRARY.exists() and LIBRARY.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIBRARY
    # -ffp-contract=off: the compiler fuses no multiply-add on its own; every
    # fmaf in the source is the only fused operation, as in the reference.
    cmd = ["gcc", "-O3", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
           "-fPIC", "-shared", str(SOURCE), "-o", str(LIBRARY) + ".tmp", "-lm"]
    subprocess.run(cmd, check=True)
    pathlib.Path(str(LIBRARY) + ".tmp").replace(LIBRARY)
    return LIBRARY


def build_reference():
    """Reference libcuhc.so for sm_100a; a no-op when the sources are absent."""
    subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True)
    return HERE / "_ref" / "libcuhc.so"


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference())
