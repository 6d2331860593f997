"""Build step of the package: compiles libplc.so for sm_100a in-tree.

``build()`` runs the Makefile in ``csrc/`` (nvcc with
``-gencode arch=compute_100a,code=sm_100a``); the library lands in
``powerllel_channel_sycl_b200/lib/libplc.so`` so it travels with the source
tree.  nvcc cross-compiles, so this works on hosts without a GPU.
"""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 4, verbose: bool = False) -> str:
    cmd = ["make", f"-j{jobs}", "-C", os.path.join(_HERE, "csrc")]
    if not verbose:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)
    path = os.path.join(_HERE, "lib", "libplc.so")
    if not os.path.exists(path):
        raise RuntimeError("libplc.so was not produced")
    return path


if __name__ == "__main__":
    print(build(verbose=True))
