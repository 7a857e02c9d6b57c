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
    with Server(hbm_budget=budget, max_batch=8, streams=4, pack=False) as srv:
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


def _pack_problems():
    from qforte_b200.ucc import DUCC
    out = []
    for norb, seed, pt in ((4, 1, "SD"), (5, 2, "SD"), (6, 3, "SD"), (5, 9, "GSD"), (8, 4, "SD")):
        mol, pool = random_problem(norb, seed, pt)
        tops = list(range(0, len(pool), 1 if len(pool) < 400 else 3))
        out.append(DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pt))
    return out


def test_pack_evaluates_every_problem_in_one_launch(cuda):
    """Items of five problems (8 to 16 qubits, SD and GSD pools), energies
    and gradients mixed, in one launch: each equals its problem's evaluator
    result, and an item's result is bitwise the same alone."""
    from qforte_b200.ucc import Pack
    duccs = _pack_problems()
    pk = Pack(duccs, capacity=64)
    rng = np.random.default_rng(7)
    members = [int(v) for v in rng.integers(len(duccs), size=40)]
    params = [rng.uniform(-0.1, 0.1, duccs[k].nparam) for k in members]
    wg = [bool(v) for v in rng.integers(2, size=40)]
    e, g = pk.run(members, params, wg)
    for i, k in enumerate(members):
        e1, g1 = duccs[k].energy_grad(params[i])
        assert abs(e[i] - e1) < E_TOL
        if wg[i]:
            assert np.max(np.abs(g[i] - g1)) < G_TOL
        else:
            assert g[i] is None
    ea, ga = pk.run([members[5]], [params[5]], [True])
    assert ea[0] == e[5]
    if wg[5]:
        assert np.array_equal(ga[0], g[5])


def test_pack_rejects_what_it_cannot_pack(cuda):
    from qforte_b200.ucc import DUCC, Pack, evaluator_config
    mol, pool = random_problem(10, 5)
    big = DUCC(mol.hamiltonian, pool, list(range(0, len(pool), 25)), mol.hf_reference)
    small = _pack_problems()[0]
    with pytest.raises(ValueError, match="shared memory"):
        Pack([small, big])
    mol, pool = random_problem(4, 6)
    evaluator_config("complex")
    try:
        cplx = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
        cplx.evaluator(1)
    finally:
        evaluator_config(True)
    with pytest.raises(ValueError, match="mix real and complex"):
        Pack([small, cplx])


def test_pack_item_naming_no_member_gets_nan(cuda):
    """Items written straight into the device blocks: one naming no member
    is refused by the kernel's bound check (NaN energy), the others run."""
    import torch
    from qforte_b200._lib import check, lib
    from qforte_b200.ucc import Pack
    duccs = _pack_problems()[:2]
    pk = Pack(duccs, capacity=8)
    d_items, d_par, d_en, d_gr = pk.tensors()
    rng = np.random.default_rng(3)
    p0 = rng.uniform(-0.1, 0.1, duccs[0].nparam)
    d_items[:3] = torch.tensor([[0, 1], [7, 1], [-1, 0]], dtype=torch.int32)
    d_par[0, :p0.size] = torch.from_numpy(p0)
    check(lib().qfb_set_stream(torch.cuda.current_stream().cuda_stream))
    pk.launch(3)
    torch.cuda.synchronize()
    en = d_en[:3].cpu().numpy()
    assert np.isnan(en[1]) and np.isnan(en[2])
    e1, g1 = duccs[0].energy_grad(p0)
    assert abs(en[0] - e1) < E_TOL
    assert np.max(np.abs(d_gr[0, :p0.size].cpu().numpy() - g1)) < G_TOL


def test_server_packs_small_problems_together(cuda):
    """With packing on, requests of all three small problems share launches:
    far fewer launches than requests, results as each problem's evaluator
    gives them, the same alone and in the mix."""
    from qforte_b200.serving import Server
    probs = _problems()
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(120):
        k = sorted(probs)[i % 3]
        reqs.append((k, rng.uniform(-0.1, 0.1, probs[k].nparam), bool(i % 2)))
    with Server(hbm_budget=8e9, streams=2, pack=True) as srv:
        for k, d in probs.items():
            srv.register(k, d)
        futs = [srv.submit(k, p, wg) for k, p, wg in reqs]
        res = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["batches"] < len(reqs) / 4
    for (k, p, wg), (e, g) in zip(reqs, res):
        e1, g1 = probs[k].energy_grad(p)
        assert abs(e - e1) < E_TOL
        assert (g is None) == (not wg)
        if wg:
            assert np.max(np.abs(g - g1)) < G_TOL
    with Server(hbm_budget=8e9, streams=2, pack=True) as srv:
        for k, d in probs.items():
            srv.register(k, d)
        k, p, wg = reqs[7]
        e, g = srv.submit(k, p, wg).result(timeout=120)
    assert e == res[7][0] and np.array_equal(g, res[7][1])

