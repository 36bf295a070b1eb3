"""Extracts the reference-generated data that pins two host-side pieces of
this library to outputs of the reference itself, into
tests/golden/atlas_pins.npz:

* the longitudinal form factors |<a| exp(i q z) |b>|^2 of the reference's
  PzP-tail basis (docs/src/assets/physics/data/form_factors.csv, written by
  examples/10_physics_atlas.jl:284-310 from the basis envelopes of
  basis_envelopes.csv), against kernel_build.lo_form_factors;
* one bordered periodic Poisson solve (hartree.csv, written by
  examples/10_physics_atlas.jl:256-282 with solve_periodic_poisson,
  numerics/reference/poisson.jl:41-65), against outer.solve_periodic_poisson;
* the non-interacting resolvent of the projected PzP-tail Hamiltonian
  (basis_operators.csv, method pzp_tails: the 25 x 25 H of
  examples/10_physics_atlas.jl:128-131), its eigen-energies (method energy,
  the diagonal of C' H C), the central-period weight of each eigenstate
  (basis_metrics.csv, method energy: 1 - outside_central_weight) and the
  local density of states on the central rows (spectral_population.csv,
  atlas lines 224-247: eta = 2 meV, 181 energies), summed over z, against
  the Dyson solve G^R = ((E + i eta) I - H)^-1;
* the occupied part of that density of states (the same CSV's
  occupied_per_meV_nm: the Fermi function at the chemical potential and
  lattice temperature of optical_parameters.csv times the density of
  states), against the equilibrium Keldysh function of the seed,
  G^< = -f (G^R - G^A) (_seed_green_production, seed.jl:151-197).

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
    ops = rows(os.path.join(data, "basis_operators.csv"))
    nb = max(int(r["a"]) for r in ops if r["method"] == "pzp_tails")
    H = np.zeros((nb, nb), dtype=complex)
    for r in ops:
        if r["method"] == "pzp_tails":
            H[int(r["a"]) - 1, int(r["b"]) - 1] = float(r["H_real_meV"]) + 1j * float(r["H_imag_meV"])
    levels = np.array(sorted(float(r["H_real_meV"]) for r in ops if r["method"] == "energy" and r["a"] == r["b"]))
    met = sorted((r for r in rows(os.path.join(data, "basis_metrics.csv")) if r["method"] == "energy"),
                 key=lambda r: int(r["state"]))
    central_weight = np.array([1.0 - float(r["outside_central_weight"]) for r in met])
    spec = rows(os.path.join(data, "spectral_population.csv"))
    E = sorted({float(r["energy_meV"]) for r in spec})
    dz = float(par["period"]) / float(par["spatial_points_per_period"])
    ldos = {e: 0.0 for e in E}
    occ = {e: 0.0 for e in E}
    for r in spec:
        ldos[float(r["energy_meV"])] += float(r["ldos_per_meV_nm"]) * dz
        occ[float(r["energy_meV"])] += float(r["occupied_per_meV_nm"]) * dz
    opt = rows(os.path.join(data, "optical_parameters.csv"))[0]
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
        H_pzp_meV=H, levels_meV=levels, central_weight=central_weight, eta_meV=2.0,
        spectral_E_meV=np.array(E), central_dos_per_meV=np.array([ldos[e] for e in E]),
        central_occupied_per_meV=np.array([occ[e] for e in E]),
        mu_meV=float(opt["chemical_potential_meV"]), temperature_K=float(opt["temperature_K"]),
    )


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
