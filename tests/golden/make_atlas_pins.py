"""Extracts the reference-generated data that pins two host-side pieces of
this library to outputs of the reference itself, into
tests/golden/atlas_pins.npz:

* the longitudinal form factors |<a| exp(i q z) |b>|^2 of the reference's
  PzP-tail basis (docs/src/assets/physics/data/form_factors.csv, written by
  examples/10_physics_atlas.jl:284-310 from the basis envelopes of
  basis_envelopes.csv), against kernel_build.lo_form_factors;
* one bordered periodic Poisson solve (hartree.csv, written by
  examples/10_physics_atlas.jl:256-282 with solve_periodic_poisson,
  numerics/reference/poisson.jl:41-65), against outer.solve_periodic_poisson.

The CSVs are output of the reference's Julia code (12 significant digits);
they are read from the reference checkout, which only this script needs:

    python tests/golden/make_atlas_pins.py [path-to-reference]
"""
import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def rows(path):
    with open(path) as f:
        return list(csv.DictReader(f))


def main(ref):
    data = os.path.join(ref, "docs", "src", "assets", "physics", "data")
    env = [r for r in rows(os.path.join(data, "basis_envelopes.csv")) if r["method"] == "pzp_tails"]
    states = sorted({int(r["state"]) for r in env})
    a, b = states[0], states[0] + 1  # form_factors.csv: the first central column and the next
    def psi(s):
        rs = [r for r in env if int(r["state"]) == s]
        return (np.array([float(r["z_nm"]) for r in rs]),
                np.array([float(r["real_psi_per_sqrt_nm"]) + 1j * float(r["imag_psi_per_sqrt_nm"]) for r in rs]))
    z, pa = psi(a)
    z2, pb = psi(b)
    assert np.array_equal(z, z2)
    ff = rows(os.path.join(data, "form_factors.csv"))
    par = {r["name"]: float(r["value"]) for r in rows(os.path.join(data, "parameters.csv"))}
    har = rows(os.path.join(data, "hartree.csv"))
    np.savez_compressed(
        os.path.join(HERE, "atlas_pins.npz"),
        z_nm=z, psi_a=pa, psi_b=pb,
        q_per_nm=np.array([float(r["q_per_nm"]) for r in ff]),
        diagonal_F2=np.array([float(r["diagonal_F2"]) for r in ff]),
        transition_F2=np.array([float(r["transition_F2"]) for r in ff]),
        period_nm=par["period"], points_per_period=par["spatial_points_per_period"],
        hartree_z_nm=np.array([float(r["z_nm"]) for r in har]),
        donors_m3=np.array([float(r["donors_m3"]) for r in har]),
        electrons_m3=np.array([float(r["electrons_m3"]) for r in har]),
        hartree_meV=np.array([float(r["hartree_meV"]) for r in har]),
    )


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
