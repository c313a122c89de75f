"""Build the sm_100a library in place (magpackage_b200/libmagasm.so)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose: bool = False) -> str:
    out = subprocess.run(["make", "-C", os.path.join(HERE, "csrc")], capture_output=True, text=True)
    if verbose:
        print(out.stdout, out.stderr)
    if out.returncode != 0:
        raise RuntimeError("libmagasm build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    return os.path.join(HERE, "libmagasm.so")


if __name__ == "__main__":
    print(build(verbose=True))
