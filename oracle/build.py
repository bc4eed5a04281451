"""Build recipe of the CPU oracle (test infrastructure).

Compiles oracle/bqcd_oracle.c (+ the flat C API and the command-line driver)
with gcc into oracle/lib/liboracle.so and oracle/lib/oracle.  The flags keep
Fortran complex arithmetic rules and disable FMA contraction so the restated
arithmetic follows the reference's evaluation order.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib")
CFLAGS = ["-std=gnu11", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fcx-fortran-rules", "-fopenmp",
          "-fPIC", "-Wall"]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False):
    os.makedirs(LIB, exist_ok=True)
    core = [os.path.join(HERE, f) for f in ("bqcd_oracle.c", "bqcd_oracle.h")]
    so = os.path.join(LIB, "liboracle.so")
    exe = os.path.join(LIB, "oracle")
    capi = os.path.join(HERE, "oracle_capi.c")
    main = os.path.join(HERE, "oracle_main.c")
    cmds = []
    if _stale(so, core + [capi]):
        cmds.append(["gcc", *CFLAGS, "-shared", core[0], capi, "-o", so, "-lm"])
    if _stale(exe, core + [main]):
        cmds.append(["gcc", *CFLAGS, core[0], main, "-o", exe, "-lm"])
    for c in cmds:
        if verbose:
            print(" ".join(c))
        subprocess.run(c, check=True)
    return so, exe


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
