"""SRQK, NTSRQK and MRSQK on the device against the reference's own runs.

The cases of the host replay in test_krylov_host.py with the Krylov basis in
HBM: every basis state's Trotter circuit through Computer.apply_circuit, H on
it by qfb_sum_apply, the matrix elements as device inner products.  Golden
values: tests/golden/srqk_norb3_seed11.npz, written by the reference's SRQK
(qkd/srqk.py); the H4 run also meets the reference test's bar of 1e-4 from FCI
(tests/test_fast_qk.py:407-411).  Tolerances are those of the host replay:
matrix elements 1e-10; the lowest eigenvalue, which rounding of the matrices
moves (overlap condition numbers 2.7e12 and 1e6), 1e-5 (H4) and 1e-8 (random
system) from the reference's.
"""

import pytest

from conftest import golden
from test_krylov_host import MRSQK_EIG_TOL, check_mrsqk, check_ntsrqk, check_srqk

pytestmark = pytest.mark.gpu


def test_srqk_on_device_matches_reference(cuda):
    from qforte_b200 import krylov
    check_srqk(krylov, golden("srqk_norb3_seed11.npz"))


def test_ntsrqk_on_device_matches_reference(cuda):
    """Exact time evolution by the device Taylor series (qfb_sum_apply, qfb_axpy)
    against the reference's expm_multiply basis: matrix elements 1e-10."""
    from qforte_b200 import krylov
    check_ntsrqk(krylov, golden("srqk_norb3_seed11.npz"))


def test_mrsqk_on_device_matches_reference(cuda):
    """Reference selection from the device SRQK basis, the CI of the candidate
    determinants and the multireference basis on the device: the reference's
    selections and spin-adapted references, lowest eigenvalues within 1e-7 and
    H4 within 1e-6 of FCI (tests/test_fast_qk.py:401-405)."""
    from qforte_b200 import krylov
    check_mrsqk(krylov, golden("mrsqk_norb3_seed11.npz"), MRSQK_EIG_TOL)
