"""Host-side planning of gate runs (no GPU): how many shared-memory tile runs
and one-gate passes a circuit becomes, and the bytes those passes move."""

import numpy as np
import pytest

import qforte_b200 as qb
from qforte_b200.device import gate_plan, gates_config
from qforte_b200.workloads import layered_random_circuit


@pytest.fixture(autouse=True)
def _default_tiles():
    yield
    gates_config(0, 3)


def test_small_state_is_one_run():
    circ, _ = layered_random_circuit(8, 10, 1)
    w, s, b = gate_plan(circ.gates(), 8)
    assert (w, s, b) == (1, 0, 32.0 * 2 ** 8)


def test_one_pass_per_gate_counts_touched_amplitudes():
    gates_config(-1, 4)
    g = [qb.gate("H", 0, 0), qb.gate("T", 1, 1), qb.gate("Z", 2, 2), qb.gate("cX", 0, 3),
         qb.gate("cZ", 1, 2), qb.gate("SWAP", 0, 1), qb.gate("I", 3, 3)]
    w, s, b = gate_plan(g, 4)
    full = 32.0 * 16
    # H full; T and Z one diagonal entry != 1: half; cX controlled: half;
    # cZ controlled diagonal with one entry != 1: a quarter; SWAP generic: full;
    # identity: nothing
    assert (w, s) == (0, 7)
    assert b == full * (1 + 0.5 + 0.5 + 0.5 + 0.25 + 1 + 0)


def test_sweep_runs_fuse_layers():
    circ, spec = layered_random_circuit(24, 20, 2)
    w, s, b = gate_plan(circ.gates(), 24)
    assert 0 < w + s < len(spec) / 4
    gates_config(12, 4)
    w12, s12, _ = gate_plan(circ.gates(), 24)
    assert w12 + s12 <= w + s


def test_plan_rejects_gates_beyond_the_state():
    with pytest.raises(ValueError):
        gate_plan([qb.gate("X", 5, 5)], 4)
    with pytest.raises(ValueError):
        gates_config(20, 4)


@pytest.mark.parametrize("tile,low", [(2, 0), (4, 1), (6, 3), (9, 4), (10, 3), (11, 3), (12, 3),
                                      (12, 6)])
@pytest.mark.parametrize("n", [3, 4, 5, 8, 14])
def test_every_gate_is_planned_once(tile, low, n):
    """Planning ends for every tile shape (including tiles too narrow for some
    2-qubit gates); tile runs carry at most the gates not given their own pass
    (exchanges and SWAPs on register bits become relabelings, identities
    nothing)."""
    from qforte_b200.device import gate_phases
    rng = np.random.default_rng(n * 100 + tile)
    gates = []
    for _ in range(150):
        if rng.random() < 0.5:
            t = int(rng.integers(n))
            gates.append(qb.gate(["H", "T", "Rx", "Y"][int(rng.integers(4))], t, t, 0.3))
        elif n > 1:
            t, c = (int(v) for v in rng.choice(n, 2, replace=False))
            gates.append(qb.gate(["cX", "cZ", "SWAP", "A"][int(rng.integers(4))], t, c, 0.7))
    gates_config(tile, low)
    w, s, _ = gate_plan(gates, n)
    phases, ops = gate_phases(gates, n)
    assert ops + s <= len(gates)
    assert (w == 0) == (phases == 0)
    assert w <= phases


def test_dense_block_planning():
    """Dense mode: runs on at most k qubits (one pass each, however many gates
    they hold); states under 10 qubits keep the tile runs; k is 0, 5 or 6."""
    circ, spec = layered_random_circuit(24, 20, 2)
    gates_config(0, 3, 0, 6)
    w6, s6, b6 = gate_plan(circ.gates(), 24)
    assert w6 > 0 and w6 + s6 < len(spec)
    gates_config(0, 3, 0, 5)
    w5, s5, _ = gate_plan(circ.gates(), 24)
    assert w5 + s5 >= w6 + s6
    deep = [qb.gate("H", q, q) for q in (1, 4, 7, 11, 14)] * 40
    deep += [qb.gate("cX", 4, 11), qb.gate("SWAP", 1, 14), qb.gate("cZ", 7, 4)] * 20
    assert gate_plan(deep, 15)[:2] == (1, 0)
    small = circ.gates()[:40]
    small = [g for g in small if g.target() < 8 and g.control() < 8]
    tiles_dense = gate_plan(small, 8)
    gates_config(0, 3, 0, 0)
    assert tiles_dense == gate_plan(small, 8)
    with pytest.raises(ValueError):
        gates_config(0, 3, 0, 7)


@pytest.mark.parametrize("tile,low", [(8, 3), (9, 4), (10, 3), (11, 3), (11, 6)])
@pytest.mark.parametrize("complex64", [False, True])
def test_fused_plans_are_consistent(tile, low, complex64):
    """The fused form of the tile phases, planned on the host for tiles of 8
    to 11 qubits (1 to 8 warps of amplitude vectors), random, control-heavy
    and layered circuits: every thread table a permutation of the thread-bit
    assignments with offsets inside the tile, every segment's variant bits on
    thread bits and shared by the 8 vectors of each n-block (as the tensor-core
    products need), every matrix inside the phase's range."""
    from test_gpu_parity import _control_heavy_circuit, _rand_circuit
    from qforte_b200.device import gate_fused_plan, gates_config
    from qforte_b200.workloads import layered_random_circuit
    gates_config(tile, low)
    try:
        for n, seed in ((12, 1), (14, 2), (16, 3)):
            for circ in (_rand_circuit(n, 400, seed)[0], _control_heavy_circuit(n, seed)[0],
                         layered_random_circuit(n, 10, seed)[0]):
                phases, segments, entries = gate_fused_plan(circ.gates(), n, complex64)
                assert phases > 0 and segments > 0 and entries >= 64 * segments
    finally:
        gates_config()
