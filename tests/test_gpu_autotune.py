"""The autotuner on the device: it times every candidate tile shape, sets the
fastest, and results under every shape stay those of the oracle / default."""

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import random_problem

pytestmark = pytest.mark.gpu


def test_tune_gates_and_results_unchanged(cuda, tmp_path, monkeypatch):
    import qforte_b200 as qb
    from qforte_b200 import autotune
    from qforte_b200.device import gates_config
    from qforte_b200.workloads import layered_random_circuit
    monkeypatch.setenv("QFB_TUNE_CACHE", str(tmp_path / "t.json"))
    circ, spec = layered_random_circuit(15, 6, 2)
    try:
        shape, timings = autotune.tune_gates(circ, 15, reps=1)
        assert len(timings) >= 5 and ",".join(map(str, shape)) in timings
        qc = qb.Computer(15)
        qc.apply_circuit(circ)
        st = O.State(15)
        st.apply_gates([O.make_gate(k, t, c, p) for k, t, c, p in spec])
        assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < 1e-12
        assert autotune.apply_cached(nqubit=15)["gates"] == shape
    finally:
        gates_config(0, 3)


def test_tune_evaluator_full_space_windows(cuda, tmp_path, monkeypatch):
    from qforte_b200 import autotune
    from qforte_b200.ucc import DUCC, evaluator_config
    from qforte_b200._lib import lib
    monkeypatch.setenv("QFB_TUNE_CACHE", str(tmp_path / "t.json"))
    mol, pool = random_problem(6, 8)
    tops = list(range(len(pool)))
    rng = np.random.default_rng(1)
    P = rng.uniform(-0.1, 0.1, (3, len(tops)))
    eng0 = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    E0, G0 = eng0.energy_grad(P)
    evaluator_config(False)
    try:
        eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
        shape, timings = autotune.tune_evaluator(eng, 3, reps=1)
        assert shape is not None and len(timings) == len(autotune.WINDOW_CANDIDATES)
        E, G = eng.energy_grad(P)
        assert np.max(np.abs(E - E0)) < 1e-12 and np.max(np.abs(G - G0)) < 1e-11
        for cand in autotune.WINDOW_CANDIDATES:  # every shape gives the same numbers
            lib().qfb_ucc_tiles(*cand)
            e2 = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
            E2, G2 = e2.energy_grad(P)
            assert np.max(np.abs(E2 - E0)) < 1e-12 and np.max(np.abs(G2 - G0)) < 1e-11
    finally:
        evaluator_config(True)
        lib().qfb_ucc_tiles(12, 11, 3)
    # the compact path has nothing to tune
    assert autotune.tune_evaluator(eng0, 3)[0] is None
