"""Host-side checks of the serving loop that need no GPU."""

import types

import numpy as np
import pytest

from qforte_b200.serving import Server


def _fake(nqubit, nparam):
    return types.SimpleNamespace(nqubit=nqubit, nparam=nparam)


def test_batch_width_cap_follows_the_budget():
    s = Server(hbm_budget=150e9, max_batch=256)
    assert s._bucket_cap(_fake(10, 50)) == 256
    # 26 qubits: 2 GiB of psi and sigma per row, half the budget for one run
    assert s._bucket_cap(_fake(26, 2478)) == 32
    small = Server(hbm_budget=1e9)
    with pytest.raises(ValueError):
        small._bucket_cap(_fake(26, 10))


def test_submit_checks_problem_and_parameters():
    s = Server()
    s.register("a", _fake(4, 3))
    with pytest.raises(KeyError):
        s.submit("b", np.zeros(3))
    with pytest.raises(ValueError):
        s.submit("a", np.zeros(4))
    with pytest.raises(ValueError):
        s.register("a", _fake(4, 3))
    f = s.submit("a", np.zeros(3))  # queued until the loop starts
    assert not f.done()
