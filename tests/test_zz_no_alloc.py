"""The allocation-free expectation-value entry point.

qfb_sum_expval_noalloc computes what qfb_sum_expval computes, for callers that
must not allocate device memory while they run (a request loop holding a
fixed HBM budget, or code running while other work may hold every free byte).
Its scratch is a fixed array inside the library, so the test calls it twice in
a row (the second call sees the first call's leftovers) and checks both calls
against the allocating entry point, at the energy tolerance of the parity
tests.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-10


def _expvals(lib, ds, bra, ket, n):
    a = np.zeros(n, dtype=np.complex128)
    b = np.zeros(n, dtype=np.complex128)
    from qforte_b200._lib import check, ptr
    check(lib.qfb_sum_expval(ds.h, bra, ket, ptr(a)), "qfb_sum_expval")
    check(lib.qfb_sum_expval_noalloc(ds.h, bra, ket, ptr(b)), "qfb_sum_expval_noalloc")
    return a, b


def test_noalloc_expval_matches_allocating_entry_point(cuda):
    import qforte_b200 as qb
    from qforte_b200._lib import check, lib, ptr
    from qforte_b200.device import sum_from_terms
    L = lib()

    # a Hamiltonian's energy on a random 10-qubit state
    mol = qb.random_molecule(5, 5, seed=3)
    rng = np.random.default_rng(1)
    psi = rng.normal(size=1024) + 1j * rng.normal(size=1024)
    psi /= np.linalg.norm(psi)
    qc = qb.Computer(10)
    qc.set_coeff_vec(psi)
    ham = sum_from_terms(mol.hamiltonian._pauli_terms())
    for _ in range(2):
        a, b = _expvals(L, ham, qc._h, qc._h, 1)
        assert abs(a[0] - b[0]) < E_TOL

    # a pool of operators (one result per operator) between two different
    # states of a batch of three, twice in a row
    pool = qb.SQOpPool()
    pool.set_orb_spaces(mol.hf_reference)
    pool.fill_pool("GSD")
    terms, seg = [], []
    for k, (c, op) in enumerate(pool):
        s = qb.SQOperator()
        s.add_op(op)
        pt = s.jw_transform()._pauli_terms()
        terms += pt
        seg += [k] * len(pt)
    psum = sum_from_terms(terms, seg, len(pool))
    bra, ket = ctypes.c_void_p(), ctypes.c_void_p()
    check(L.qfb_state_create(10, 3, ctypes.byref(bra)))
    check(L.qfb_state_create(10, 3, ctypes.byref(ket)))
    try:
        for b in range(3):
            v = rng.normal(size=1024) + 1j * rng.normal(size=1024)
            w = rng.normal(size=1024) + 1j * rng.normal(size=1024)
            check(L.qfb_state_upload(bra, b, ptr(v), 1024))
            check(L.qfb_state_upload(ket, b, ptr(w), 1024))
        for _ in range(2):
            a, b = _expvals(L, psum, bra, ket, 3 * len(pool))
            assert np.max(np.abs(a - b)) < E_TOL
    finally:
        L.qfb_state_destroy(bra)
        L.qfb_state_destroy(ket)


def _dense_expvals(psi, terms, segments, nsegment):
    """out[g] = sum over segment g's terms of c <psi| P(x, z) |psi>, with
    P(x, z)|i> = i^{|x & z|} (-1)^{|i & z|} |i ^ x>."""
    idx = np.arange(psi.size, dtype=np.uint64)
    out = np.zeros(nsegment, dtype=np.complex128)
    for (c, x, z), g in zip(terms, segments):
        x, z = np.uint64(x), np.uint64(z)
        sign = 1 - 2 * (np.bitwise_count(idx & z).astype(np.int64) & 1)
        v = np.zeros_like(psi)
        v[idx ^ x] = (1j ** int(np.bitwise_count(x & z))) * sign * psi
        out[g] += c * np.vdot(psi, v)
    return out


def test_noalloc_multi_chunk_rows_and_clamped_chunks(cuda):
    """The two layouts the 10-qubit cases above never reach, each checked
    against the allocating entry point and the dense sums of the state read
    back, twice, alternating, so every call follows one that left different
    contents in the shared scratch.

    * 22 qubits, 64,500 results of which two are non-empty, three x-groups:
      rows + results = 64,503 leave room for 345 partials per row, fewer than
      the 395 that would fill 148 SMs eight times over, so the chunk count is
      clamped to what fits.
    * 16 qubits, four x-groups in three results: 32 chunks per (state,
      group) row, so every result sums several partials of each group."""
    import qforte_b200 as qb
    from qforte_b200._lib import lib
    from qforte_b200.device import sum_from_terms
    L = lib()
    rng = np.random.default_rng(5)

    def random_state(n):
        qc = qb.Computer(n)
        v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        qc.set_coeff_vec(v / np.linalg.norm(v))
        return qc

    big = random_state(22)
    nseg = 64500
    xm = (1 << 3) | (1 << 17) | (1 << 21)
    t_big = [(complex(rng.normal(), rng.normal()), 0, int(z))
             for z in rng.integers(0, 1 << 22, 50)]
    t_big += [(complex(rng.normal(), rng.normal()), xm, int(z))
              for z in rng.integers(0, 1 << 22, 20)]
    t_big += [(0.75 + 0.0j, 0, (1 << 21) | 5)]
    s_big = [0] * 70 + [nseg - 1]
    clamped = sum_from_terms(t_big, s_big, nseg)
    small = random_state(16)
    op = qb.build_operator("0.5, X_0 Z_2 Y_15; 0.25, Y_1 X_9; -0.3, Z_3 Z_12; 0.7, X_0 Y_2 Y_15; "
                           "-0.2j, Z_5 X_9 Y_1")
    t_small, s_small = op._pauli_terms(), [0, 1, 0, 1, 2]
    multi = sum_from_terms(t_small, s_small, 3)
    want_big = _dense_expvals(big.get_coeff_array(), t_big, s_big, nseg)
    want_small = _dense_expvals(small.get_coeff_array(), t_small, s_small, 3)
    for _ in range(2):
        a, b = _expvals(L, clamped, big._h, big._h, nseg)
        assert np.max(np.abs(a - b)) < E_TOL
        assert np.max(np.abs(b - want_big)) < E_TOL
        a, b = _expvals(L, multi, small._h, small._h, 3)
        assert np.max(np.abs(a - b)) < E_TOL
        assert np.max(np.abs(b - want_small)) < E_TOL


def test_noalloc_refuses_work_beyond_its_fixed_scratch(cuda):
    import qforte_b200 as qb
    from qforte_b200._lib import QFB_EINVAL, last_error, lib, ptr
    from qforte_b200.device import sum_from_terms
    L = lib()
    op = qb.build_operator("0.5, X_0 Z_2; 0.25, Y_1; -0.3, Z_3")
    ds = sum_from_terms(op._pauli_terms())  # 3 x-groups
    st = ctypes.c_void_p()
    assert L.qfb_state_create(4, 30000, ctypes.byref(st)) == 0
    try:
        out = np.zeros(30000, dtype=np.complex128)
        rc = L.qfb_sum_expval_noalloc(ds.h, st, st, ptr(out))
        assert rc == QFB_EINVAL
        assert "fixed scratch" in last_error()
    finally:
        L.qfb_state_destroy(st)
