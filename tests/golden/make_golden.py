"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own CPU FlowSolver (compiled from its sources by
oracle/Makefile into oracle/_ref/libmcref.so, against single-rank MPI/PETSc
shims) on seeded inputs and stores its outputs:

  ref_box6x3x3.npz      6x3x3 cells on a 0.06 x 0.03 x 0.03 m box: mesh arrays,
                        face geometry, and all 13 fields (u, v, w, p, the
                        pressure correction, k, epsilon, turbulent production,
                        T, mixture fraction, progress variable and the two
                        variances) plus face mass fluxes after each of 4 SIMPLE
                        passes; CSR pattern of the momentum and
                        pressure-correction matrices.
  ref_cfg1_10passes.npz 40x20x20 = 16,000 cells on the 0.2 x 0.1 x 0.1 m box:
                        all 13 fields after 10 SIMPLE passes (the parity gate).

Both start from the reference's initial state with u, v, w, p, T replaced by
the inlet state plus seeded uniform noise (+-1%, numpy PCG64, seed 0), and use
the shim's linear-solver tolerance 1e-13.  Usage (in the container that has the
reference tree):  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from checkers import Reference, noisy_initial_fields, ref_available  # noqa: E402

BASE = {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}
FIELDS = ("U", "V", "W", "P", "TEM")
ALL_FIELDS = ("U", "V", "W", "P", "PP", "TE", "ED", "TP", "TEM", "FUL", "PRO", "VARF", "VARP")


def seeded_reference(ex, ey, ez, lx, ly, lz, seed=0):
    ref = Reference(ex, ey, ez, lx, ly, lz, delta=1.0e-5, bcgs_rtol=1e-13, cg_rtol=1e-13)
    init = noisy_initial_fields(ref.N, BASE, seed)
    for name, vals in init.items():
        a = ref.field(name)
        a[:ref.N] = vals
        ref.set_field(name, a)
    return ref, init


def make_small():
    ex, ey, ez, L = 6, 3, 3, (0.06, 0.03, 0.03)
    ref, init = seeded_reference(ex, ey, ez, *L)
    m = ref.mesh()
    out = {"dims": np.array([ex, ey, ez]), "lengths": np.array(L),
           "points": m.points, "cells": m.cells, "faces": m.faces, "cell_faces": m.cell_faces,
           "cell_neighbours": m.cell_neighbours, "cell_centers": m.cell_centers,
           "boundary_types": m.boundary_types,
           "face_area": ref.face_array(1), "face_lambda": ref.face_array(2), "face_rlencos": ref.face_array(3),
           "face_normal": ref.face_array(5), "face_center": ref.face_array(6), "cell_volume": ref.cell_array(6),
           "inlet_effective_viscosity": np.array(ref.inlet_effective_viscosity())}
    for name in FIELDS:
        out[f"init_{name}"] = init[name]
    for p in range(4):
        ref.step()
        for name in ALL_FIELDS:
            out[f"pass{p + 1}_{name}"] = ref.field(name)
        out[f"pass{p + 1}_mdot"] = ref.face_array(0)
        if p == 0:
            rp, col, val = ref.csr(1)
            out["pressure_rowptr"], out["pressure_col"], out["pressure_val_pass1"] = rp, col, val
            rp, col, _ = ref.csr(0)
            out["matrix_rowptr"], out["matrix_col"] = rp, col
    np.savez_compressed(os.path.join(HERE, "ref_box6x3x3.npz"), **out)


def make_cfg1():
    ex, ey, ez, L = 40, 20, 20, (0.2, 0.1, 0.1)
    ref, _ = seeded_reference(ex, ey, ez, *L)
    for _ in range(10):
        ref.step()
    out = {"dims": np.array([ex, ey, ez]), "lengths": np.array(L), "passes": np.array(10)}
    for name in ALL_FIELDS:
        out[name] = ref.field(name)
    rp, col, _ = ref.csr(1)
    out["pressure_rowptr"], out["pressure_col"] = rp, col
    np.savez_compressed(os.path.join(HERE, "ref_cfg1_10passes.npz"), **out)


if __name__ == "__main__":
    if not ref_available():
        sys.exit("oracle/_ref/libmcref.so not built (run make -C oracle with the reference tree present)")
    make_small()
    make_cfg1()
    print("wrote", os.listdir(HERE))
