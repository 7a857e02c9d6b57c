"""One state split over ranks (qforte_b200.sharded), on CPU with gloo ranks.

The sharding logic -- the qubit map, the half-shard exchanges that swap a
qubit between a rank bit and a local bit, runs of local gates with renamed
qubits, expectation values across ranks with their phases and one all-reduce
-- runs unchanged; the local shard is a host state driven by the oracle (the
device shard is qforte_b200.Computer, covered by the GPU tests).  The gathered
state and the expectation values must equal the oracle's single-state
results (1e-12, 1e-10) for every gate kind, on 2 and 4 ranks.
"""

import math
import os
import socket

import numpy as np
import pytest

ONE = ["X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I"]
TWO = ["A", "cX", "acX", "cY", "cZ", "cR", "cV", "cRz", "SWAP", "CNOT", "aCNOT"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class HostShard:
    """A local shard on the host (test stand-in for the device Computer)."""

    def __init__(self, n):
        import torch
        self.n = n
        self.t = torch.zeros(1 << n, dtype=torch.complex128)

    def reset(self):
        self.t.zero_()
        self.t[0] = 1.0

    def null_state(self):
        self.t.zero_()

    def tensor(self):
        return self.t

    def apply_circuit(self, circ):
        from oracle import oracle as O
        st = O.State(self.n, self.t.numpy())
        st.apply_gates([(g.target(), g.control(), g.matrix()) for g in circ.gates()])
        self.t.copy_(__import__("torch").from_numpy(st.psi))

    def expval_between(self, terms, ket):
        bra = self.t.numpy()
        k = bra if ket is None else ket.t.numpy()
        idx = np.arange(bra.size, dtype=np.uint64)
        tot = 0j
        for c, x, z in terms:
            x, z = np.uint64(x), np.uint64(z)
            sign = 1 - 2 * (np.bitwise_count(idx & z).astype(np.int64) & 1)
            v = np.zeros_like(k)
            v[idx ^ x] = (1j ** int(np.bitwise_count(x & z))) * sign * k
            tot += c * np.vdot(bra, v)
        return tot


def _circuit(n, ngates, seed):
    import qforte_b200 as qb
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    circ, ora = qb.Circuit(), []
    for _ in range(ngates):
        if rng.random() < 0.5:
            k, t = ONE[rng.integers(len(ONE))], int(rng.integers(n))
            c = t
        else:
            k = TWO[rng.integers(len(TWO))]
            t, c = (int(v) for v in rng.choice(n, 2, replace=False))
        p = float(rng.uniform(0, 4 * math.pi))
        circ.add(qb.gate(k, t, c, p))
        ora.append(O.make_gate(k, t, c, p))
    return circ, ora


def _terms(n, nterms, seed):
    rng = np.random.default_rng(seed)
    return [(complex(rng.normal(), rng.normal()), int(rng.integers(0, 1 << n)),
             int(rng.integers(0, 1 << n))) for _ in range(nterms)]


def _rank(rank, world, port, n, out):
    import sys
    from datetime import timedelta

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    from qforte_b200.sharded import ShardedComputer
    from test_sharded_gloo import HostShard, _circuit, _terms

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        sc = ShardedComputer(n, local_factory=HostShard, chunk_bytes=256)
        circ, _ = _circuit(n, 160, 7 + world)
        sc.apply_circuit(circ)
        full = sc.gather()
        ev = sc.expval_terms(_terms(n, 40, 3))
        # a second circuit after the map has moved, then the state again
        circ2, _ = _circuit(n, 60, 9)
        sc.apply_circuit(circ2)
        full2 = sc.gather()
        ev2 = sc.expval_terms(_terms(n, 25, 4))
        out.put((rank, full, ev, full2, ev2, sc.exchanges, list(sc.pos)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_state_equals_one_state(world):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    from test_sharded_gloo import HostShard, _circuit, _terms  # noqa: F401
    n = 7
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        r, *rest = q.get(timeout=300)
        got[r] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full, ev, full2, ev2, nex, pos = got[0]
    # the oracle on one state
    st = O.State(n)
    st.apply_gates(_circuit(n, 160, 7 + world)[1])
    assert np.max(np.abs(full - st.psi)) < 1e-12
    ref = HostShard(n)
    ref.t.copy_(__import__("torch").from_numpy(st.psi))
    assert abs(ev - ref.expval_between(_terms(n, 40, 3), None)) < 1e-10
    st.apply_gates(_circuit(n, 60, 9)[1])
    assert np.max(np.abs(full2 - st.psi)) < 1e-12
    ref.t.copy_(__import__("torch").from_numpy(st.psi))
    assert abs(ev2 - ref.expval_between(_terms(n, 25, 4), None)) < 1e-10
    # qubits moved between rank bits and local bits, identically on every rank
    assert nex > 0 and sorted(pos) == list(range(n))
    for r in range(1, world):
        assert got[r][0] is None and got[r][4] == nex and got[r][5] == pos
        assert got[r][1] == ev and got[r][3] == ev2


def test_sharded_state_rejects_bad_shapes(monkeypatch):
    from qforte_b200.sharded import ShardedComputer

    class FakeDist:
        @staticmethod
        def get_world_size(group=None):
            return 3

        @staticmethod
        def get_rank(group=None):
            return 0

    import torch.distributed
    monkeypatch.setattr(torch.distributed, "get_world_size", FakeDist.get_world_size)
    monkeypatch.setattr(torch.distributed, "get_rank", FakeDist.get_rank)
    with pytest.raises(ValueError, match="power-of-two"):
        ShardedComputer(6, local_factory=HostShard)
    monkeypatch.setattr(torch.distributed, "get_world_size", lambda group=None: 8)
    with pytest.raises(ValueError, match="fewer than 2 local"):
        ShardedComputer(4, local_factory=HostShard)
