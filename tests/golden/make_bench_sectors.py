"""Generates tests/golden/bench_sectors_L24_M512.json (committed; needs a GPU).  Run from the
repository root:

    python tests/golden/make_bench_sectors.py [--L 24] [--M 512] [--sweeps 2] [--seed 0]

The bench's H_eff workload is the two-site problem at the middle bond of an MPS whose bond sectors
are those of a converged DMRG state: the synthetic ab-initio Hamiltonian (seed 0) at L orbitals,
N = L electrons, TwoU1 Sz = 0, two-site sweeps at bond dimension M from the const initial state
(init_bond_dimension 64).  This script runs those sweeps on the device and records, for every bond
0 .. L, the sectors (N_up, N_down, size) of the MPS.  The bench then fills site tensors over these
sectors with seeded random values, the same in both of its arms, so that both build the same problem
without running a sweep.
"""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=24)
    ap.add_argument("--M", type=int, default=512)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.fcidump import synthetic_integrals
    from qcmaquis_b200.heff import Context, parse_mps_tensor
    from qcmaquis_b200.mpo import MPO
    h, V, e = synthetic_integrals(a.L, a.seed)
    ctx = Context(0)
    d = DMRG(ctx, MPO.qc(h, V), a.L // 2, a.L // 2, a.M, 64)
    energies = [float(d.sweep()[0].min()) for _ in range(a.sweeps)]
    sites = [parse_mps_tensor(b) for b in d.export_mps()]
    bonds = [[list(map(int, s)) for s in sites[0]["left"]]] + [[list(map(int, s)) for s in st["right"]] for st in sites]
    for i, st in enumerate(sites):
        assert [list(map(int, s)) for s in st["left"]] == bonds[i]
    out = {"L": a.L, "N": a.L, "M": a.M, "seed": a.seed, "sweeps": a.sweeps, "init_bond_dimension": 64,
           "energies_min_per_sweep": energies, "phys": [list(map(int, s)) for s in sites[0]["phys"]], "bonds": bonds}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"bench_sectors_L{a.L}_M{a.M}.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print(path, [sum(s[2] for s in b) for b in bonds])


if __name__ == "__main__":
    main()
