"""The sharded state on the device path: qforte_b200.sharded.ShardedComputer
with its default local shard (the device Computer) in an NCCL group of one
rank.  With one GPU per run here, no rank exchanges are possible; the gate
runs with renamed qubits, the expectation values and the all-reduce go
through the product path and must equal the oracle's (1e-12, 1e-10).  The
exchanges themselves are covered on 2 and 4 gloo ranks (test_sharded_gloo.py).
"""

import socket

import numpy as np
import pytest

from test_sharded_gloo import HostShard, _circuit, _terms

pytestmark = pytest.mark.gpu


def test_sharded_state_on_one_gpu(cuda):
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from qforte_b200.sharded import ShardedComputer
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        n = 12
        sc = ShardedComputer(n)
        circ, ora = _circuit(n, 300, 21)
        sc.apply_circuit(circ)
        st = O.State(n)
        st.apply_gates(ora)
        assert np.max(np.abs(sc.local().get_coeff_array() - st.psi)) < 1e-12
        assert np.max(np.abs(sc.gather() - st.psi)) < 1e-12
        terms = _terms(n, 50, 5)
        ref = HostShard(n)
        ref.t.copy_(torch.from_numpy(st.psi))
        assert abs(sc.expval_terms(terms) - ref.expval_between(terms, None)) < 1e-10
        assert sc.exchanges == 0
    finally:
        dist.destroy_process_group()
