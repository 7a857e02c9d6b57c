"""The serving loop: continuous batching of many drivers' requests, with
admission against an HBM budget.  Every result must equal the problem's
single-call result, and a request's result must be the same alone and in a
mix of concurrent requests of other problems and kinds."""

import threading
import time

import numpy as np
import pytest

from tests.helpers import random_problem

pytestmark = pytest.mark.gpu

E_TOL = 1e-10
G_TOL = 1e-8


def _problems():
    from qforte_b200.ucc import DUCC
    out = {}
    for norb, seed in ((4, 1), (5, 2), (6, 3)):
        mol, pool = random_problem(norb, seed)
        out[f"norb{norb}"] = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
    return out


def test_results_same_alone_and_in_the_mix(cuda):
    from qforte_b200.serving import Server
    probs = _problems()
    rng = np.random.default_rng(0)
    key = "norb5"
    tp = rng.uniform(-0.1, 0.1, probs[key].nparam)
    with Server(hbm_budget=8e9, streams=3) as srv:
        for k, d in probs.items():
            srv.register(k, d)
        e_alone, g_alone = srv.submit(key, tp, True).result(timeout=120)

    subs, lock = [], threading.Lock()
    with Server(hbm_budget=8e9, streams=3) as srv:
        for k, d in probs.items():
            srv.register(k, d)

        def client(seed):
            r = np.random.default_rng(seed)
            for i in range(40):
                k = sorted(probs)[r.integers(3)]
                p = r.uniform(-0.1, 0.1, probs[k].nparam)
                wg = bool(r.integers(2))
                f = srv.submit(k, p, wg)
                with lock:
                    subs.append((k, p, wg, f))
                if i == 20 and seed == 1:
                    with lock:
                        subs.append((key, tp, True, srv.submit(key, tp, True)))
                time.sleep(r.exponential(2e-4))

        ts = [threading.Thread(target=client, args=(s,)) for s in (1, 2, 3)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        results = [(k, p, wg, f.result(timeout=300)) for k, p, wg, f in subs]
        st = srv.stats()
    assert st["completed"] == len(subs) + 0 and st["batches"] < len(subs)
    assert st["latency_ms"]["p99"] >= st["latency_ms"]["p50"] > 0
    found = False
    for k, p, wg, (e, g) in results:
        e1, g1 = probs[k].energy_grad(p)
        assert abs(e - e1) < E_TOL
        if wg:
            assert np.max(np.abs(g - g1)) < G_TOL
        else:
            assert g is None
        if k == key and p is tp:
            found = True
            assert abs(e - e_alone) < 1e-12 and np.max(np.abs(g - g_alone)) < 1e-12
    assert found


def test_admission_keeps_within_the_budget(cuda):
    from qforte_b200.serving import Server
    probs = _problems()
    d = probs["norb6"]
    # room for one 8-row evaluator of the 12-qubit problem at a time
    one_row = 2 * 16 * (1 << d.nqubit)
    budget = 20 * one_row
    rng = np.random.default_rng(4)
    with Server(hbm_budget=budget, max_batch=8, streams=4) as srv:
        for k, p in probs.items():
            srv.register(k, p)
        futs = [(k, p, srv.submit(k, p, True)) for k, p in
                ((sorted(probs)[i % 3], rng.uniform(-0.1, 0.1, probs[sorted(probs)[i % 3]].nparam))
                 for i in range(48))]
        res = [(k, p, f.result(timeout=300)) for k, p, f in futs]
        st = srv.stats()
    assert st["peak_device_bytes"] <= budget
    for k, p, (e, g) in res:
        e1, g1 = probs[k].energy_grad(p)
        assert abs(e - e1) < E_TOL and np.max(np.abs(g - g1)) < G_TOL
