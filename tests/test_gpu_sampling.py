"""Measurement draws on the device (Computer::measure_circuit /
measure_readouts / measure_z_readouts_fast, computer.cc:135-315): the seeded
sampler gives the oracle's indices bit for bit, and the measurements give the
reference's expectation values within their statistical error (the
reference's own generator is unseeded)."""

import ctypes

import numpy as np
import pytest

import qforte_b200 as qb
from oracle import oracle as O
from qforte_b200._lib import check, lib, ptr
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _state(psi):
    qc = qb.Computer(int(np.log2(len(psi))))
    qc.set_coeff_vec(psi)
    return qc


@pytest.mark.parametrize("n,shots", [(3, 500), (6, 2000), (13, 4000), (17, 30000)])
def test_samples_equal_the_oracle_bit_for_bit(cuda, n, shots):
    rng = np.random.default_rng(n)
    psi = rng.normal(size=2 ** n) + 1j * rng.normal(size=2 ** n)
    psi /= np.linalg.norm(psi)
    qc = _state(psi)
    for seed in (1, 2 ** 63 + 12345):
        got = qc.sample(shots, seed=seed)
        want = O.sample_indices(psi, seed, shots)
        assert np.array_equal(got, want)


def test_sparse_states_draw_only_their_support(cuda):
    """Whole 4,096-amplitude blocks and 64-amplitude sub-blocks of zero
    weight, a basis state, and tiny amplitudes below the 2^-56 weight unit."""
    n = 15
    psi = np.zeros(2 ** n, dtype=np.complex128)
    support = [5, 4097, 9000, 2 ** n - 1]
    psi[support] = [0.5, 0.5j, -0.5, 0.5]
    psi[123] = 1e-10  # |c|^2 = 1e-20 < 2^-56: weight 0
    qc = _state(psi)
    got = qc.sample(5000, seed=7)
    assert set(got.tolist()) <= set(support)
    assert np.array_equal(got, O.sample_indices(psi, 7, 5000))
    one = np.zeros(2 ** n, dtype=np.complex128)
    one[2 ** n - 1] = 1.0
    assert set(_state(one).sample(100, seed=3).tolist()) == {2 ** n - 1}


def test_unnormalised_and_zero_states_are_refused(cuda):
    psi = np.full(64, 0.25, dtype=np.complex128)  # squared norm 4
    with pytest.raises(ValueError):
        _state(psi).sample(10, seed=1)
    with pytest.raises(ValueError):
        _state(np.zeros(64, dtype=np.complex128)).sample(10, seed=1)


def test_batch_slot_through_the_c_abi(cuda):
    h = ctypes.c_void_p()
    check(lib().qfb_state_create(10, 3, ctypes.byref(h)))
    try:
        rng = np.random.default_rng(4)
        psi = rng.normal(size=1024) + 1j * rng.normal(size=1024)
        psi /= np.linalg.norm(psi)
        check(lib().qfb_state_upload(h, 2, ptr(psi), 1024))
        out = np.empty(777, dtype=np.uint64)
        check(lib().qfb_state_sample(h, 2, 99, 777, ptr(out)))
        assert np.array_equal(out, O.sample_indices(psi, 99, 777))
        assert lib().qfb_state_sample(h, 3, 99, 10, ptr(out)) != 0
    finally:
        lib().qfb_state_destroy(h)


def test_measurements_match_the_reference_expectation(cuda):
    """measure_circuit on the reference's 6-qubit golden state: the mean of
    the +-1 outcomes of X_0 Y_2 Z_4 is the reference's
    perfect_measure_circuit value within 5 standard errors."""
    z = golden("gates_n6.npz")
    qc = _state(z["psi"])
    qb.computer.set_sampling_seed(2024)
    circ = qb.build_circuit("X_0 Y_2 Z_4")
    shots = 200000
    vals = np.array(qc.measure_circuit(circ, shots))
    exact = float(z["perfect_measure"])
    assert abs(qc.perfect_measure_circuit(circ) - exact) < 1e-12
    se = np.sqrt(max(1.0 - exact ** 2, 1e-12) / shots)
    assert abs(vals.mean() - exact) < 5 * se
    # the state is left as it was, and readouts agree with the values
    assert np.max(np.abs(qc.get_coeff_array() - z["psi"])) < 1e-15
    qb.computer.set_sampling_seed(2024)
    reads = qc.measure_readouts(circ, 1000)
    v2 = [(-1) ** (sum(r) % 2) for r in reads]
    assert np.array_equal(np.array(v2, dtype=float), vals[:1000])
    zr = qc.measure_z_readouts_fast(1, 3, 10)
    assert len(zr) == 10 and all(len(r) == 3 for r in zr)
