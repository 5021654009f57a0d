"""Generates tests/golden/golden.json (committed).  Run from the repository root:

    python tests/golden/make_golden.py [path-to-reference-tree]

* hubbard_ladder_6x2_reference: the two-site TwoU1 energy asserted by the
  reference's own regression test (regression/applications/dmrg/
  test_fermiladder_ts.py:65), read from that file when the reference tree is
  given, otherwise the committed value is kept.
* *_fci: exact diagonalisation (oracle/fci.py); config 1 uses the dense
  4900 x 4900 eigensolver.
* hubbard_ladder_6x2_local_density_{up,down}_reference: the per-site densities
  the same reference test asserts (reference_value('Local density up'/'down'),
  tolerance 1e-3), read from that file like the energy;
  hubbard_ladder_6x2_fci_local_density: gamma_ii / 2 of the exact ground state
  (N_up = N_down, so each spin carries half the spin-summed density).
* config1_oracle_sweep_energies: per-sweep energies (min over the sweep's
  steps, results_collector.h:147) of the oracle's two-site DMRG for config 1
  (L=8, N=8, TwoU1 Sz=0, M=64, 4 sweeps, tol 1e-10, maxiter 8, const init).
"""
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from qcmaquis_b200.fcidump import hubbard_ladder_integrals, synthetic_integrals  # noqa: E402
from qcmaquis_b200.mpo import MPO  # noqa: E402
from oracle.fci import FCI, fci_energy  # noqa: E402
from oracle.oracle import OracleDMRG  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def main():
    old = json.load(open(OUT)) if os.path.exists(OUT) else {}
    g = {}
    ref = old.get("hubbard_ladder_6x2_reference")
    if len(sys.argv) > 1:
        txt = open(os.path.join(sys.argv[1], "dmrg/regression/applications/dmrg/test_fermiladder_ts.py")).read()
        ref = float(re.search(r"Energy\D*?([0-9]+\.[0-9]+)", txt).group(1))
    g["hubbard_ladder_6x2_reference"] = ref
    for spin in ("up", "down"):
        key = f"hubbard_ladder_6x2_local_density_{spin}_reference"
        g[key] = old.get(key)
        if len(sys.argv) > 1:
            m = re.search(r"reference_value\('Local density " + spin + r"',\s*value=\[([^\]]*)\]", txt)
            g[key] = [float(v) for v in m.group(1).split(",")]
    h, V, e = hubbard_ladder_integrals(6)
    g["hubbard_ladder_6x2_fci"] = fci_energy(h, V, e, 10, 10)
    f = FCI(h, V, e, 10, 10)
    E0, c0 = f.ground_state()
    g["hubbard_ladder_6x2_fci_local_density"] = [float(x) / 2 for x in np.diag(f.one_rdm(c0))]
    h, V, e = synthetic_integrals(8, 0)
    g["config1_fci"] = float(np.linalg.eigvalsh(FCI(h, V, e, 4, 4).dense())[0])
    m = MPO.qc(h, V)
    d = OracleDMRG(m.blob(), 8, 4, 4, 64)
    g["config1_oracle_sweep_energies"] = [float(d.sweep(s)[0].min()) for s in range(4)]
    g["config1_h00"] = float(h[0, 0])
    g["config1_V0000"] = float(V[0, 0, 0, 0])
    json.dump(g, open(OUT, "w"), indent=1)
    print(json.dumps(g, indent=1))


if __name__ == "__main__":
    main()
