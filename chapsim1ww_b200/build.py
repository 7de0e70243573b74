"""In-tree build of libchapsim.so (sm_100a) and of the CPU oracle checker."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build_library(verbose=False):
    out = subprocess.run(["make", "-j8", "-C", os.path.join(HERE, "csrc")], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libchapsim build failed:\n" + out.stdout + out.stderr)
    if verbose:
        print(out.stdout)
    return os.path.join(HERE, "libchapsim.so")


def build_oracle(verbose=False):
    out = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if verbose:
        print(out.stdout)
    return os.path.join(ROOT, "oracle", "liboracle.so")
