"""Builds the CPU checkers under oracle/ -- test infrastructure, never the
product: liboracle.so (the C restatement) always; where the reference tree is
present, oracle/_ref/libmcref.so (the reference compiled from its sources)
and, once the library is built, oracle/_ref/front_driver (the reference's
flow driver over the C++ front).  The reference tree is read where it lies:
MC_REFERENCE_TREE, or /root/reference.  Built files travel with the
repository; a machine without the tree keeps the ones built before.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_TREE = os.environ.get("MC_REFERENCE_TREE", "/root/reference")


def _make(*targets):
    cmd = ["make", "-s", "-C", HERE]
    if os.path.isdir(os.path.join(REFERENCE_TREE, "include", "flow")):
        cmd.append(f"REF={REFERENCE_TREE}")
    subprocess.run(cmd + list(targets), check=True, stdout=subprocess.DEVNULL)


def build(front=False):
    _make("all")
    if front:
        _make("front")


if __name__ == "__main__":
    build(front=True)
