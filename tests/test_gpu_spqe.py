"""SPQE on the device against the reference's own SPQE runs.

The cases of the host replay in test_spqe_host.py on the fused engine: the
selection step's U, exp(i dt H) and U^dagger as fused Pauli-exponential passes,
the micro-iterations' residuals and energies from the evaluator's residual
run.  Golden values: tests/golden/spqe_norb3_seed11.npz, written by the
reference's SPQE (ucc/spqe.py).  Pins: the H4 run reaches FCI within 5e-11
(tests/test_spqe.py:11-39); every selection picks the reference's operators
with the same counts per macro-iteration; per-iteration energies 1e-10 where
the selection order matches the reference's (mirror-image determinants tie in
H4's first selection, so rounding may swap their order: test_spqe_host.py).
"""

import numpy as np
import pytest

from test_spqe_host import check_spqe

pytestmark = pytest.mark.gpu


def test_spqe_on_device_matches_reference(cuda):
    from qforte_b200 import ucc
    check_spqe(ucc, "fused", strict=False)


def test_scipy_solver_matches_jacobi_on_device(cuda):
    from qforte_b200 import ucc
    from test_spqe_host import check_scipy_matches_jacobi
    check_scipy_matches_jacobi(ucc, "fused")


def test_sampled_spqe_on_device_matches_oracle_sampler(cuda, monkeypatch):
    """Sampled SPQE with seeded device draws (qfb_state_sample) selects what
    the oracle's restatement of the sampler selects from the host replay's
    state, and reaches the same energies (1e-10)."""
    from qforte_b200 import ucc
    from test_qite_host import HostComputer
    from test_spqe_host import run_sampled
    dev = run_sampled(ucc, "fused")
    monkeypatch.setattr(ucc, "Computer", HostComputer)
    host = run_sampled(ucc, "percall")
    assert list(dev._tops) == list(host._tops)
    assert np.max(np.abs(np.array(dev._energies) - np.array(host._energies))) < 1e-10


def test_moment_corrections_on_device(cuda):
    from qforte_b200 import ucc
    from test_spqe_host import check_moments
    check_moments(ucc, "fused", strict=False)
