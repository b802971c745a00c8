"""Generate the FP64 oracle fixtures of the large workloads (committed; read by tests and bench.py).

The oracle (oracle/, a CPU restatement of the reference mqvector kernels and adjoint driver, in
complex128) is run once on the host for workloads too large to re-run inside a test or a
benchmark, and its results are stored next to this script:

* ``hea26_oracle.json``: the headline workload, HEA 26 qubits x 12 layers (RY, RZ on every qubit,
  CNOT ladder), 624 parameters, 51-term ZZ + X Hamiltonian, seed 0: <H> and the 624-entry gradient
  of parameter set 0 of the benchmark's batch of 8 (the Hamiltonian's coefficients are drawn after
  the angles, so they depend on the batch size), plus the first parameters and Hamiltonian
  coefficients as a check that the workload is the same.
* ``hea22_oracle.json``: HEA 22 qubits x 6 layers, batch 2, seed 0, parameter sets 0 and 1.

Run from the repository root (8 host threads: about five minutes for the 26-qubit case):

    python tests/golden/make_oracle_fixtures.py [hea26] [hea22]

``--check-reference`` instead compares the committed fixtures with the reference's own CPU
simulator built from its sources (oracle/_ref, ``make -C oracle ref``), complex128, and prints the
largest differences (the 22-qubit one also runs in tests/test_reference_binary.py):

    python tests/golden/make_oracle_fixtures.py --check-reference [hea26] [hea22]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _hea_fixture(n, layers, batch, samples, name):
    from mindquantum_b200 import workloads
    from oracle import oracle as O

    circ, ham, params = workloads.hea(n, layers, batch, seed=0, encoder=True)
    rows = []
    for s in samples:
        t0 = time.time()
        ref = O.get_expectation_with_grad(n, [ham], circ, params[s:s + 1], np.zeros(0), circ.params_name, [],
                                          np.complex128)
        dt = time.time() - t0
        rows.append({"sample": s, "f": float(ref[0, 0, 0].real), "f_imag": float(ref[0, 0, 0].imag),
                     "grad": [float(x) for x in ref[0, 0, 1:].real], "oracle_seconds": dt,
                     "params_head": [float(x) for x in params[s, :8]]})
        print(f"{name}: sample {s}: f = {ref[0, 0, 0].real:.15f} in {dt:.1f} s", flush=True)
    out = {"workload": f"hea({n}, {layers}, {batch}, seed=0, encoder=True)", "n_qubits": n, "layers": layers,
           "batch": batch, "ham_coeff_head": [float(c) for _, c in ham.ham_termlist[:6]],
           "n_params": len(circ.params_name), "precision": "complex128 (oracle)", "threads": O.num_threads(),
           "samples": rows}
    with open(os.path.join(HERE, f"{name}_oracle.json"), 'w', encoding='utf8') as f:
        json.dump(out, f, indent=1)
        f.write('\n')


def _check_reference(name):
    from mindquantum_b200 import workloads
    from oracle import refbin as R

    with open(os.path.join(HERE, f"{name}_oracle.json"), encoding='utf8') as f:
        fx = json.load(f)
    circ, ham, params = workloads.hea(fx['n_qubits'], fx['layers'], fx['batch'], seed=0, encoder=True)
    for row in fx['samples']:
        s = row['sample']
        t0 = time.time()
        ref = R.grad(fx['n_qubits'], circ, ham, params[s:s + 1])[0]
        print(f"{name}: sample {s}: |f - f_ref| = {abs(ref[0].real - row['f']):.3e}, max |g - g_ref| = "
              f"{np.max(np.abs(ref[1:].real - np.array(row['grad']))):.3e} (reference {time.time() - t0:.1f} s)",
              flush=True)


def main(argv):
    if '--check-reference' in argv:
        for name in [a for a in argv if a != '--check-reference'] or ['hea22', 'hea26']:
            _check_reference(name)
        return
    which = argv or ['hea26', 'hea22']
    if 'hea22' in which:
        _hea_fixture(22, 6, 2, [0, 1], 'hea22')
    if 'hea26' in which:
        _hea_fixture(26, 12, 8, [0], 'hea26')


if __name__ == '__main__':
    main(sys.argv[1:])
