"""Build libuassa.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False, debug=True):
    """libuassa.so and (debug=True) the bounds-checked libuassa_debug.so."""
    for target in (["all", "debug"] if debug else ["all"]):
        cmd = ["make", "-C", os.path.join(HERE, "csrc"), "-j8", target]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or out.returncode != 0:
            sys.stdout.write(out.stdout)
            sys.stderr.write(out.stderr)
        if out.returncode != 0:
            raise RuntimeError(f"libuassa build failed ({target})")
    return os.path.join(HERE, "libuassa.so")


if __name__ == "__main__":
    print(build(verbose=True))
