"""Autotuning of the tile shapes that decide how many operations one pass
over the state fuses.

* Gate runs (``tune_gates``): ``tile_bits`` qubits per shared-memory tile, the
  ``low_bits`` lowest qubits every tile keeps (contiguous rows) and the
  ``reg_bits`` register bits each thread holds, for a circuit on a given
  qubit count.
* Full-space evaluator windows (``tune_evaluator``): the forward and gradient
  tile sizes and the low bits, for a dUCC problem and batch width.  (The
  compact sector path holds whole states in shared memory and has no tile.)

Each candidate is timed on the device with CUDA events after a warm-up run,
the fastest one is set process-wide and the choice is cached in a JSON file
(``$QFB_TUNE_CACHE`` or ``~/.cache/qforte_b200/tuning.json``) under a key
naming the workload, so ``apply_cached`` restores it in a later process.
"""

import json
import os

import numpy as np

from .device import gate_plan, gates_config

__all__ = ["tune_gates", "tune_evaluator", "apply_cached", "cache_path",
           "GATE_CANDIDATES", "WINDOW_CANDIDATES"]

# (tile_bits, low_bits, reg_bits, dense): register-blocked tiles, and dense
# 5- and 6-qubit blocks on the FP64 tensor cores
GATE_CANDIDATES = ((10, 3, 3, 0), (10, 4, 3, 0), (11, 3, 3, 0), (11, 4, 3, 0), (9, 3, 3, 0),
                   (12, 3, 4, 0), (0, 3, 0, 5), (0, 3, 0, 6))
WINDOW_CANDIDATES = ((12, 11, 3), (11, 11, 3), (13, 11, 3), (12, 10, 3), (12, 12, 3),
                     (12, 11, 4))


def cache_path():
    p = os.environ.get("QFB_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "qforte_b200", "tuning.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key, value):
    d = _load()
    d[key] = value
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _time(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def gate_key(nqubit):
    return f"gates:n={int(nqubit)}"


def tune_gates(circuit, nqubit, candidates=GATE_CANDIDATES, reps=2, store=True):
    """Time ``circuit`` on a fresh ``nqubit`` state under each (tile_bits,
    low_bits, reg_bits, dense); set and return the fastest with every timing
    (ms)."""
    from .computer import Computer
    qc = Computer(int(nqubit))
    timings = {}
    for cand in candidates:
        tile, low, regs, dense = (tuple(cand) + (0,))[:4]
        first = tuple(cand) == tuple(candidates[0])
        if not first and (tile > nqubit or (dense and nqubit < 10)):
            continue
        gates_config(tile, low, regs, dense)
        runs, singles, _ = gate_plan(circuit.gates(), nqubit)
        ms = _time(lambda: qc.apply_circuit(circuit), reps)
        timings[f"{tile},{low},{regs},{dense}"] = {"ms": ms, "passes": runs + singles}
    best = min(timings, key=lambda k: timings[k]["ms"])
    shape = tuple(int(v) for v in best.split(","))
    gates_config(*shape)
    if store:
        _store(gate_key(nqubit), list(shape))
    return shape, timings


def evaluator_key(ducc, nbatch):
    return f"ucc:n={ducc.nqubit}:nparam={ducc.nparam}:batch={int(nbatch)}"


def _ucc_tiles(fwd, grad, low):
    from ._lib import check, lib
    check(lib().qfb_ucc_tiles(int(fwd), int(grad), int(low)), "qfb_ucc_tiles")


def tune_evaluator(ducc, nbatch, candidates=WINDOW_CANDIDATES, reps=2, store=True, seed=0):
    """Time one energy+gradient run of ``ducc``'s full-space evaluator at
    ``nbatch`` rows under each (fwd_bits, grad_bits, low_bits); set and return
    the fastest with every timing (ms).  Returns None when the problem takes
    the compact sector path (no tile to choose)."""
    from .ucc import Evaluator
    rng = np.random.default_rng(seed)
    P = rng.uniform(-0.1, 0.1, (int(nbatch), ducc.nparam))
    timings = {}
    for fwd, grad, low in candidates:
        _ucc_tiles(fwd, grad, low)
        ev = Evaluator(ducc, int(nbatch))
        if ev.path == 2:
            _ucc_tiles(*candidates[0])
            return None, {}
        d_par, _, _ = ev.tensors()
        import torch
        d_par.copy_(torch.from_numpy(P))
        timings[f"{fwd},{grad},{low}"] = {"ms": _time(lambda: ev.run(True), reps)}
        del ev
    best = min(timings, key=lambda k: timings[k]["ms"])
    shape = tuple(int(v) for v in best.split(","))
    _ucc_tiles(*shape)
    ducc._evals.clear()  # evaluators made from now on use the chosen shape
    if store:
        _store(evaluator_key(ducc, nbatch), list(shape))
    return shape, timings


def apply_cached(nqubit=None, ducc=None, nbatch=None):
    """Set the cached tile shapes for a gate workload on ``nqubit`` qubits and /
    or a dUCC problem at ``nbatch`` rows; returns what was applied."""
    d = _load()
    out = {}
    if nqubit is not None and gate_key(nqubit) in d:
        shape = tuple(d[gate_key(nqubit)])
        gates_config(*shape)
        out["gates"] = shape
    if ducc is not None and nbatch is not None and evaluator_key(ducc, nbatch) in d:
        shape = tuple(d[evaluator_key(ducc, nbatch)])
        _ucc_tiles(*shape)
        out["windows"] = shape
    return out
