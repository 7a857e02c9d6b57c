"""Benchmark: batched dUCCSD energy + adjoint-gradient evaluations on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

(K defaults to 40 for the default workload, 5 for the others; W to 3.)

Workload (one step): 256 parameter sets of the 16-qubit dUCCSD problem
(8 spatial orbitals, 8 electrons, 360 SD parameters, seeded random integrals,
5,793 Hamiltonian terms); each evaluation is the energy <U^dag H U> and its full
adjoint gradient.  Metric: evaluations per second (whole job).

* ``value``    device-timed (CUDA events, max over ranks): parameters already in
               HBM, one graph-captured run per step; consecutive steps rotate
               over four evaluators on four streams (``--streams``), so one
               step's kernels use the SMs the others leave idle (the forward
               program fills 128 SMs of 148, the sweep's latency-bound CTAs
               leave issue slots free).
* ``e2e``      the same through the public API with host buffers: the step's
               parameters copied from pinned host memory and its energies and
               gradients read back, inside the timed region (a step's copies
               overlap the other stream's kernels).
* ``roofline`` the dominant kernel, timed stage by stage with CUDA events.
* ``cpu_baseline`` the compiled reference (``oracle/_ref``) on a bounded sample
               of the same workload, on this host's cores (rank 0, N = 1 only).

N > 1 runs N independent replicas (one process per GPU, no collective on the
data path): weak scaling.  ``--impl reference`` times the reference's own CPU
path on the same workload and prints the same metric.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "UCC energy+grad evals/s"

# The compact-sector kernels of the default workload (16 qubits, 256 sets), from
# one ncu capture of that workload (--set full --clock-control none,
# -k regex:k_sector_(forward|h|sweep), 3 launches): DRAM bytes read + written
# per launch, and the L1 / shared-memory pipe and issue activity that bind them.
NCU_SECTOR_UCC16_B256 = {
    "k_sector_forward": {"dram_bytes": 1.497e6, "l1_shared_pipe_pct": 50.7, "issue_active_pct": 39.8,
                         "warps_active_pct": 42.9},
    "k_sector_h": {"dram_bytes": 31.35e6, "l1_shared_pipe_pct": 88.6, "issue_active_pct": 34.6,
                   "warps_active_pct": 49.9},
    "k_sector_sweep": {"dram_bytes": 21.58e6, "l1_shared_pipe_pct": 47.8, "issue_active_pct": 35.5,
                       "warps_active_pct": 21.7},
}
UNIT = "evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 40 for the default workload, whose steps "
                         "rotate over --streams evaluators, else 5)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--norb", type=int, default=8)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--streams", type=int, default=4,
                    help="default workload: consecutive steps alternate between this many "
                         "evaluators, each on its own stream, so their kernels and copies overlap")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the gate-sweep, Pauli-exponential and serving numbers of the "
                         "default run")
    ap.add_argument("--full-space", action="store_true",
                    help="keep full-space states (no compact sector evaluator)")
    ap.add_argument("--one-set", action="store_true",
                    help="one parameter set per CTA in the compact forward program "
                         "(default: two real sets per CTA)")
    ap.add_argument("--workload", default="ucc",
                    choices=["ucc", "gates", "grad", "adapt", "serve", "pexp", "pqe", "sample"],
                    help="ucc: batched dUCCSD energy+gradient (default); gates: the gate sweep; "
                         "grad: differentiable energy, forward+backward against forward alone; "
                         "adapt: every ADAPT pool gradient of a 12-operator state in one launch; "
                         "pexp: Pauli-exponential passes on one large state; "
                         "pqe: batched PQE residual vectors; sample: measurement draws")
    ap.add_argument("--pexp-n", type=int, default=28, help="pexp: qubits")
    ap.add_argument("--pexp-strings", type=int, default=64,
                    help="pexp: random Pauli strings, and dUCC operators, per program")
    ap.add_argument("--adapt-norb", type=int, default=10, help="adapt workload: orbitals")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: mean requests per second")
    ap.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals")
    ap.add_argument("--norb-range", default="5,13", help="serve: orbital counts lo,hi")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM budget")
    ap.add_argument("--norbs", default="8,10", help="grad workload: orbital counts")
    ap.add_argument("--nqubits", default="20,24,28",
                    help="gate sweep: comma-separated qubit counts")
    ap.add_argument("--layers", type=int, default=100, help="gate sweep: layers per circuit")
    ap.add_argument("--tile", type=int, default=0,
                    help="gate sweep: tile bits of gate runs (0 default, -1 one pass per gate)")
    ap.add_argument("--low-bits", type=int, default=3,
                    help="gate sweep: lowest qubits every tile keeps")
    ap.add_argument("--reg-bits", type=int, default=0,
                    help="gate sweep: register bits per thread of a tile (0: default)")
    ap.add_argument("--dense", type=int, default=0,
                    help="gate sweep: fuse runs into dense 5- or 6-qubit blocks on the FP64 "
                         "tensor cores (0: tile runs)")
    ap.add_argument("--phase-form", choices=["auto", "fused", "ops"], default="auto",
                    help="gate sweep: tile phases as fused 8 x 8 matrices on the FP64 tensor "
                         "cores, gate by gate, or fused for states larger than L2 (default)")
    ap.add_argument("--complex64", action="store_true",
                    help="gate sweep: the complex64 throughput variant (FP32 arithmetic)")
    ap.add_argument("--autotune", action="store_true",
                    help="gate sweep: pick the tile shape per qubit count with the autotuner")
    a = ap.parse_args()
    if a.steps is None:
        a.steps = 40 if a.workload == "ucc" else 5
    return a


def problem(norb, seed):
    import qforte_b200 as qb
    mol = qb.random_molecule(norb, norb, seed)
    pool = qb.SQOpPool()
    pool.set_orb_spaces(mol.hf_reference)
    pool.fill_pool("SD")
    return mol, pool


def replica_parameters(seed, rank, batch, nparam):
    """One replica's parameter rows: amplitudes U(-0.1, 0.1), seeded per rank so
    every replica evaluates its own batch."""
    return np.random.default_rng(seed + 1 + rank).uniform(-0.1, 0.1, (batch, nparam))


def max_over_ranks(x, world, device):
    """The largest of every rank's x (a device-timed duration): the job ends
    when its slowest replica does.  One all-reduce, taken by every rank."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, batch, ms_max):
    """Evaluations per second over all replicas: each rank evaluates `batch`
    sets per step and the step lasts as long as the slowest rank's."""
    return world * batch / (ms_max / 1000.0)


def workload_config(a, nterms, nparam):
    return {"workload": f"batched dUCCSD energy + adjoint gradient, {2 * a.norb} qubits "
                        f"({a.norb} orbitals, {a.norb} electrons), {nparam} SD parameters, "
                        f"{nterms} Hamiltonian terms, {a.batch} parameter sets per step",
            "nqubit": 2 * a.norb, "batch": a.batch, "nparam": nparam, "hamiltonian_terms": nterms,
            "l2": f"inputs larger than L2: {2 * a.batch} states x {16 << (2 * a.norb)} B "
                  "resident per step",
            "parallelism": f"replicas x{a.gpus}",
            "streams": f"consecutive steps on {max(1, a.streams)} evaluator(s), one stream each"}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(a, mol, pool, rows, rounds=1):
    """The compiled reference (serial shipped build) on a bounded sample of the
    workload, one evaluation per host core at once (the batch's evaluations
    are independent).  Each worker times U(t) in full, H on a tenth of its
    terms and 12 reverse-sweep steps, scaled to one whole evaluation."""
    from oracle import oracle as O
    from qforte_b200.pauli import letters
    O.load_reference_engine()  # fail here, in the parent, if it is not built

    def terms(qo):
        return [(complex(c), letters(*circ._pauli_masks()[:2])) for c, circ in qo.terms()]

    import qforte_b200 as qb
    kf, kg = [], []
    for _, op in pool:
        s = qb.SQOperator()
        s.add_op(op)
        q = s.jw_transform()
        kg.append(terms(q))
        q.simplify()
        q.order_terms()
        kf.append(terms(q))
    ht = terms(mol.hamiltonian)
    h_sample = max(1, len(ht) // 10)
    m_sample = 12
    workers = max(1, min(O.host_cores(), 128))
    per, walls, parts = [], [], None
    for _ in range(max(1, rounds)):
        rate, t, wall, parts = O.ref_eval_parallel(2 * a.norb, mol.hf_reference, kf, kg, rows, ht,
                                                   h_sample, m_sample, workers)
        per += t
        walls.append(wall)
    t_eval = statistics.median(per)
    return {"value": workers / t_eval, "unit": UNIT, "cores": workers, "kind": "reference",
            "sample": f"per evaluation: U(t) as gates in full, apply_operator(H) on {h_sample} "
                      f"of {len(ht)} terms scaled x{len(ht) / h_sample:.1f} (twice: energy and "
                      f"sigma), {m_sample} of {len(kf)} reverse-sweep steps scaled; one "
                      f"evaluation per core on {workers} cores at once, {max(1, rounds)} "
                      "round(s), median seconds per evaluation; serial shipped build "
                      "(USE_OpenMP off) in each worker",
            "extrapolated": True, "cpu_model": cpu_model(),
            "seconds_per_eval": t_eval, "sample_wall_s": statistics.median(walls),
            "parts": parts[0] if parts else None}


def run_reference(a, rank, world):
    """--impl reference: the reference's CPU path on the same workload."""
    mol, pool = problem(a.norb, a.seed)
    rng = np.random.default_rng(a.seed + 1)
    P = rng.uniform(-0.1, 0.1, (a.batch, len(pool)))
    if rank != 0:
        return None
    try:
        from oracle import oracle as O
        O.load_reference_engine()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference module not built: {e}"}))
        return None
    # each step is one bounded sample round on every host core; the rounds of
    # the whole run stay within a few minutes
    rounds = max(1, min(a.steps, 8))
    cb = cpu_baseline(a, mol, pool, P, rounds=rounds)
    v = cb["value"]
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": rounds,
            "warmup": 0, "ms_per_step": 1000.0 * cb["sample_wall_s"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex128 states)",
            "data": "synthetic",
            "config": workload_config(a, len(mol.hamiltonian), len(pool)), "impl": "reference",
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                "extrapolated", "cpu_model")},
            "timing": "ms_per_step is the wall time of one sample round (one sampled "
                      "evaluation per core); value extrapolates the sampled parts of each "
                      "evaluation to the whole evaluation",
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line))
    return line


GATE_METRIC = "gate-sweep pass GB/s"


def gate_cpu_baseline(n, spec, seconds=12.0):
    """The compiled reference's apply_circuit on the first gates of the sweep
    circuit: seconds per gate, GB/s at the reference's own bytes per gate."""
    from oracle import oracle as O
    qf = O.load_reference_engine()
    t1 = O.ref_gate_sample(qf, n, spec, 4)
    ngates = int(max(4, min(len(spec), seconds / max(t1, 1e-9))))
    t = O.ref_gate_sample(qf, n, spec, ngates)
    return t, ngates


def run_gates(a, rank, world, local, emit=True):
    """Gate sweep: layered random circuits applied with Computer.apply_circuit."""
    import torch
    import qforte_b200 as qb
    from qforte_b200._lib import launch_count
    from qforte_b200.device import gate_phases, gate_plan, gates_config
    from qforte_b200.workloads import layered_random_circuit
    torch.cuda.set_device(local)
    gates_config(a.tile, a.low_bits, a.reg_bits, getattr(a, "dense", 0),
                 {"auto": None, "fused": True, "ops": False}[getattr(a, "phase_form", "auto")])
    peak, src = peaks()
    ns = [int(v) for v in a.nqubits.split(",") if v]
    rows = []
    clocks = Clocks(local)
    for n in ns:
        circ, spec = layered_random_circuit(n, a.layers, a.seed + n)
        tuned = None
        if a.autotune:
            from qforte_b200.autotune import tune_gates
            tuned, _ = tune_gates(circ, n, reps=1, store=False)
        nw, nsingle, pass_bytes = gate_plan(circ.gates(), n)
        nphase, _ = gate_phases(circ.gates(), n)
        c64 = getattr(a, "complex64", False)
        if c64:
            pass_bytes /= 2.0  # 8-byte amplitudes
        qc = qb.ComputerC64(n) if c64 else qb.Computer(n)
        for _ in range(max(a.warmup, 3) if n < 28 else 1):
            qc.apply_circuit(circ)
        steps = a.steps if n < 28 else 1
        torch.cuda.synchronize()
        if n == ns[-1]:
            clocks.start()
        l0 = launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            qc.apply_circuit(circ)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        launches = (launch_count() - l0) // steps
        ck = clocks.stop() if n == ns[-1] else None
        gbs = pass_bytes / (ms * 1e-3) / 1e9
        rows.append({"nqubit": n, "gates": len(spec), "passes": nw + nsingle, "tile_runs": nw,
                     "register_phases": nphase, "one_gate_passes": nsingle,
                     "ms_per_circuit": ms, "pass_gbs": gbs,
                     "frac_of_hbm": gbs / peak,
                     "effective_gate_gbs": len(spec) * (16.0 if c64 else 32.0) * 2 ** n /
                                           (ms * 1e-3) / 1e9,
                     "gpu_launches": launches,
                     "tile": list(tuned) if tuned else a.tile})
        del qc
    last = rows[-1]
    line = {"metric": GATE_METRIC, "value": last["pass_gbs"], "unit": "GB/s", "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": last["ms_per_circuit"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 (throughput only)" if getattr(a, "complex64", False) else "c128",
            "data": "synthetic",
            "config": {"workload": f"layered random circuits, {a.layers} layers, "
                                   f"{','.join(map(str, ns))} qubits, from |0...0>",
                       "tile_bits": a.tile, "low_bits": a.low_bits, "reg_bits": a.reg_bits,
                       "dense_block_qubits": getattr(a, "dense", 0),
                       "phase_form": getattr(a, "phase_form", "auto"),
                       "l2": "state larger than L2 from 23 qubits"},
            "sweep": rows,
            "roofline": {"bound": "hbm",
                         "kernel": ("k_dense_block" if getattr(a, "dense", 0) else
                                    "k_gate2 / k_gate4" if a.tile == -1 else "k_gate_tile"),
                         "achieved": last["pass_gbs"],
                         "peak": peak, "peak_source": src, "unit": "GB/s",
                         "frac": last["pass_gbs"] / peak, "traffic": None},
            "gpu_launches": last["gpu_launches"], "clocks": ck}
    if not a.no_cpu_baseline:
        try:
            n0 = min(ns)
            _, spec0 = layered_random_circuit(n0, a.layers, a.seed + n0)
            t, ng = gate_cpu_baseline(n0, spec0)
            bpg = 32.0 * 2 ** n0
            line["cpu_baseline"] = {"value": bpg / t / 1e9, "unit": "GB/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"apply_circuit of the first {ng} gates of the "
                                              f"{n0}-qubit sweep circuit, 32 * 2^n bytes per gate, "
                                              "serial shipped build",
                                    "seconds_per_gate": t}
        except Exception as e:
            line["cpu_baseline"] = {"unavailable": str(e)}
    if emit:
        print(json.dumps(line))
    return line


PEXP_METRIC = "Pauli-exponential pass GB/s"


def run_pexp(a, local, emit=True, ducc_part=True):
    """Pauli-exponential passes on one n-qubit state (default 28 qubits, 4 GiB).

    * ``strings``: exp(i phi P) for random Pauli strings with distinct x-masks,
      one streaming pass each (pairs j, j ^ x; phase from popcount(j & z)),
      32 * 2^n bytes per pass.  Applied as U^dagger (one pass per string),
      then U, and the state must come back to |0...0>.
    * ``ducc``: the ansatz strings of seeded SD operators of the half-filled
      (n/2)-orbital problem; U applied with windows (several exponentials per
      pass over the state) and U^dagger one Givens step per pass (each step
      touches only its active pairs)."""
    import ctypes
    import torch
    import qforte_b200 as qb
    from qforte_b200._lib import check, launch_count, lib
    from qforte_b200.device import DeviceProg
    from qforte_b200.ucc import ansatz_strings
    torch.cuda.set_device(local)
    n, K = a.pexp_n, a.pexp_strings
    N = 1 << n
    peak, src = peaks()
    rng = np.random.default_rng(a.seed + n)
    xs, seen = [], set()
    while len(xs) < K:
        x = int(rng.integers(1, N))
        if x not in seen:
            seen.add(x)
            xs.append(x)
    zs = [int(rng.integers(0, N)) for _ in range(K)]
    prog = DeviceProg(np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64),
                      np.ones(K), np.arange(K, dtype=np.int32), K)
    params = rng.uniform(-np.pi, np.pi, K)
    h = ctypes.c_void_p()
    check(lib().qfb_state_create(n, 1, ctypes.byref(h)), "qfb_state_create")
    L = lib()
    P = params.ctypes.data_as(ctypes.c_void_p)

    def apply(pr, par, sign):
        check(L.qfb_prog_apply(pr.h, h, par, 1, sign), "qfb_prog_apply")

    def timed(fn, reps):
        for _ in range(max(a.warmup, 3) if n < 28 else 1):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = launch_count()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, (launch_count() - l0) // reps

    clocks = Clocks(local)
    clocks.start()
    ms_s, launches = timed(lambda: apply(prog, P, -1), max(1, a.steps))
    ck = clocks.stop()
    # round trip: U (one pass per string) after U^dagger gives |0...0> back
    check(L.qfb_state_reset(h), "reset")
    apply(prog, P, 1)
    apply(prog, P, -1)
    out = (ctypes.c_double * 2)()
    check(L.qfb_state_get_amp(h, 0, 0, out), "qfb_state_get_amp")
    roundtrip_err = abs(complex(out[0], out[1]) - 1.0)
    gbs = K * 32.0 * N / (ms_s * 1e-3) / 1e9
    if not ducc_part:
        check(L.qfb_state_destroy(h), "destroy")
        return {"pass_gbs": gbs, "frac_of_hbm": gbs / peak, "peak": peak, "peak_source": src,
                "nqubit": n, "strings": K, "ms_per_program": ms_s,
                "gpu_launches": int(launches), "roundtrip_abs_err": roundtrip_err}

    # dUCC ansatz program of the (n/2)-orbital half-filled problem
    norb = n // 2
    pool = qb.SQOpPool()
    pool.set_orb_spaces([1] * norb + [0] * norb)
    pool.fill_pool("SD")
    tops = sorted(int(t) for t in rng.choice(len(pool), min(K, len(pool)), replace=False))
    X, Z, S, PP = ansatz_strings(pool, tops)
    dp = DeviceProg(np.array(X, dtype=np.uint64), np.array(Z, dtype=np.uint64), np.array(S),
                    np.array(PP, dtype=np.int32), len(tops))
    amps = rng.uniform(-0.1, 0.1, len(tops))
    PA = amps.ctypes.data_as(ctypes.c_void_p)
    check(L.qfb_state_reset(h), "reset")
    ms_w, l_w = timed(lambda: apply(dp, PA, 1), max(1, a.steps))
    ms_g, l_g = timed(lambda: apply(dp, PA, -1), max(1, a.steps))
    check(L.qfb_state_reset(h), "reset")
    apply(dp, PA, 1)
    apply(dp, PA, -1)
    check(L.qfb_state_get_amp(h, 0, 0, out), "qfb_state_get_amp")
    ducc_err = abs(complex(out[0], out[1]) - 1.0)
    check(L.qfb_state_destroy(h), "destroy")
    ducc = {"operators": len(tops), "strings": len(X), "steps": int(dp.nsteps),
            "windowed_ms": ms_w, "windowed_launches": int(l_w),
            "windowed_pass_gbs": l_w * 32.0 * N / (ms_w * 1e-3) / 1e9,
            "per_step_ms": ms_g, "per_step_launches": int(l_g),
            "effective_step_gbs": int(dp.nsteps) * 32.0 * N / (ms_g * 1e-3) / 1e9,
            "roundtrip_abs_err": ducc_err}
    line = {"metric": PEXP_METRIC, "value": gbs, "unit": "GB/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"{K} exponentials of random Pauli strings (distinct x-masks) "
                                   f"on one {n}-qubit state, one streaming pass each",
                       "nqubit": n, "l2": f"state {16 * N} B, larger than L2"},
            "roofline": {"bound": "hbm", "kernel": "k_prog_step", "achieved": gbs, "peak": peak,
                         "peak_source": src, "unit": "GB/s", "frac": gbs / peak,
                         "algorithmic_bytes_per_launch": 32.0 * N,
                         "avg_launch_ms": ms_s / max(1, launches), "traffic": None},
            "roundtrip_abs_err": roundtrip_err, "ducc": ducc,
            "gpu_launches": int(launches), "clocks": ck}
    if emit:
        print(json.dumps(line))
    return line


def run_pqe(a, local):
    """PQE residual vectors (UCCNPQE.get_residual_vector) for a batch of
    parameter sets of the dUCCSD problem: psi, H psi, U^dagger on sigma and
    the projections on the excited determinants in one graph launch, against
    the reference's recipe through the Computer API call for call and the
    compiled reference on the host."""
    import time
    import torch
    from qforte_b200._lib import launch_count
    from qforte_b200.ucc import DUCC, UCCNPQE, excited_determinants
    torch.cuda.set_device(local)
    mol, pool = problem(a.norb, a.seed)
    tops = list(range(len(pool)))
    M = len(tops)
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    rng = np.random.default_rng(a.seed + 3)
    P = rng.uniform(-0.1, 0.1, (a.batch, M))
    dets = excited_determinants(pool, tops, mol.hf_reference)
    E, R = eng.residuals(P, dets)
    ev = eng.evaluator(a.batch)
    d_params = ev.tensors()[0]
    d_params.copy_(torch.from_numpy(P))
    for _ in range(max(a.warmup, 3)):
        ev.run(4)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        ev.run(4)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    launches = (launch_count() - l0) // a.steps
    t_end = time.perf_counter() + max(0.0, 0.8 - a.steps * ms / 1000.0)
    while time.perf_counter() < t_end:
        ev.run(4)
        torch.cuda.synchronize()
    ck = clocks.stop()
    # end to end: host parameters in, residuals out, every step
    hP = torch.from_numpy(P).pin_memory()
    hR = torch.empty((a.batch, len(dets)), dtype=torch.float64).pin_memory()

    def view(addr, shape):
        class _I:
            __cuda_array_interface__ = {"shape": shape, "typestr": "<f8",
                                        "data": (int(addr), False), "version": 2}
        return torch.as_tensor(_I(), device="cuda")

    d_res = view(ev.d_res, (a.batch, len(dets)))
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        d_params.copy_(hP, non_blocking=True)
        ev.run(4)
        hR.copy_(d_res, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / a.steps
    assert np.max(np.abs(hR.numpy() - R)) < 1e-12
    # plain per-call path: the reference's recipe through the Computer API
    drv = UCCNPQE(mol, engine="percall")
    drv._pool_obj = pool
    drv._tops, drv._tamps = tops, list(P[0])
    drv._excited_dets = dets
    drv._noise_factor = 0.0
    drv._res_vec_evals = drv._res_m_evals = 0
    drv.get_residual_vector(P[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r_plain = np.array(drv.get_residual_vector(P[0]))
    t_plain = time.perf_counter() - t0
    line = {"metric": "PQE residual vectors/s", "value": 1000.0 * a.batch / ms, "unit": "vectors/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"PQE residuals of the dUCCSD problem, {2 * a.norb} qubits "
                                   f"({a.norb} orbitals), {M} residuals, {a.batch} parameter "
                                   "sets per step"},
            "e2e": {"value": 1000.0 * a.batch / ms_e2e, "unit": "vectors/s",
                    "h2d_bytes_per_step": int(P.nbytes), "d2h_bytes_per_step": int(hR.numel() * 8)},
            "evaluator_path": ev.path, "gpu_launches": int(launches), "clocks": ck,
            "plain_per_call": {"value": 1.0 / t_plain, "unit": "vectors/s",
                               "max_abs_diff_vs_batched": float(np.max(np.abs(r_plain - R[0])))},
            "batched_vs_plain": (1000.0 * a.batch / ms) * t_plain}
    if not a.no_cpu_baseline:
        try:
            from oracle import oracle as O
            from qforte_b200.pauli import letters
            import qforte_b200 as qb

            def terms(qo):
                return [(complex(c), letters(*circ._pauli_masks()[:2])) for c, circ in qo.terms()]

            qf = O.load_reference_engine()
            kf = []
            for _, op in pool:
                sq = qb.SQOperator()
                sq.add_op(op)
                q = sq.jw_transform()
                q.simplify()
                q.order_terms()
                kf.append(terms(q))
            ht = terms(mol.hamiltonian)
            hs = max(1, len(ht) // 10)
            t, parts = O.ref_pqe_sample(qf, 2 * a.norb, mol.hf_reference, kf, list(P[0]), ht, hs)
            line["cpu_baseline"] = {"value": 1.0 / t, "unit": "vectors/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"one get_residual_vector: U and U^dagger as gates in "
                                              f"full, apply_operator(H) on {hs} of {len(ht)} "
                                              "terms scaled; serial shipped build",
                                    "parts_s": parts}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    print(json.dumps(line))
    return line


def run_sample(a, local):
    """Measurement draws (Computer::measure_z_readouts_fast's sampling,
    computer.cc:185-211): 10^6 seeded basis-state draws from one n-qubit
    state (default 28 qubits) per step, host indices out."""
    import time
    import torch
    import qforte_b200 as qb
    from qforte_b200._lib import check, launch_count, lib, ptr
    torch.cuda.set_device(local)
    n, shots = a.pexp_n, 1_000_000
    qc = qb.Computer(n)
    t = qc.tensor()
    g = torch.Generator(device="cuda").manual_seed(a.seed)
    t.copy_(torch.complex(torch.randn(t.shape, dtype=torch.float64, device="cuda", generator=g),
                          torch.randn(t.shape, dtype=torch.float64, device="cuda", generator=g)))
    t.div_(torch.linalg.vector_norm(t))
    out = np.empty(shots, dtype=np.uint64)
    for k in range(max(a.warmup, 3)):
        check(lib().qfb_state_sample(qc._h, 0, k, shots, ptr(out)))
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(a.steps):
        check(lib().qfb_state_sample(qc._h, 0, 100 + k, shots, ptr(out)))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    launches = (launch_count() - l0) // a.steps
    ck = clocks.stop()
    peak, src = peaks()
    state_gbs = 16.0 * 2 ** n / (ms * 1e-3) / 1e9
    line = {"metric": "measurement draws/s", "value": shots / (ms * 1e-3), "unit": "draws/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"{shots} seeded draws from one random {n}-qubit state per "
                                   "step, indices copied to the host",
                       "nqubit": n},
            "roofline": {"bound": "hbm", "kernel": "k_samp_weights + k_samp_draw",
                         "achieved": state_gbs, "peak": peak, "peak_source": src, "unit": "GB/s",
                         "frac": state_gbs / peak, "algorithmic_bytes_per_launch": 16.0 * 2 ** n,
                         "note": "one read of the state per step; the whole call is timed",
                         "traffic": None},
            "gpu_launches": int(launches), "clocks": ck}
    if not a.no_cpu_baseline:
        try:
            from oracle import oracle as O
            qf = O.load_reference_engine()
            nr = 20
            rc = qf.Computer(nr)
            rng = np.random.default_rng(1)
            v = rng.normal(size=2 ** nr) + 1j * rng.normal(size=2 ** nr)
            v /= np.linalg.norm(v)
            rc.set_coeff_vec(list(v))
            rs = 100_000
            t0 = time.perf_counter()
            rc.measure_z_readouts_fast(0, 0, rs)
            tc = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": rs / tc, "unit": "draws/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"measure_z_readouts_fast(0, 0, {rs}) on a random "
                                              f"{nr}-qubit state (the 28-qubit state does not fit "
                                              "the bounded sample), serial shipped build"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    print(json.dumps(line))
    return line


def run_grad(a, local):
    """Differentiable dUCCSD energy: forward (energy) and forward+backward
    (energy and the adjoint gradient through torch.autograd) per parameter
    set, at each orbital count (half filling, SD pool)."""
    import torch
    from qforte_b200.autograd import ucc_energy
    from qforte_b200.ucc import DUCC
    torch.cuda.set_device(local)
    rows = []
    for norb in [int(v) for v in a.norbs.split(",") if v]:
        mol, pool = problem(norb, a.seed)
        eng = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
        M = len(pool)
        rng = np.random.default_rng(a.seed + norb)
        res = {"nqubit": 2 * norb, "nparam": M, "hamiltonian_terms": len(mol.hamiltonian)}
        for B in (1, a.batch):
            t = torch.tensor(rng.uniform(-0.1, 0.1, (B, M)), device="cuda", requires_grad=True)
            for _ in range(max(a.warmup, 3)):
                ucc_energy(t, eng).sum().backward()
                with torch.no_grad():
                    ucc_energy(t, eng)
            times = {}
            for mode in ("forward", "forward+backward"):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for _ in range(a.steps):
                    if mode == "forward":
                        with torch.no_grad():
                            ucc_energy(t, eng)
                    else:
                        t.grad = None
                        ucc_energy(t, eng).sum().backward()
                e1.record()
                torch.cuda.synchronize()
                times[mode] = e0.elapsed_time(e1) / a.steps
            res[f"batch{B}"] = {"forward_ms": times["forward"],
                                "forward_backward_ms": times["forward+backward"],
                                "ratio": times["forward+backward"] / times["forward"]}
        rows.append(res)
        del eng
    big = rows[-1][f"batch{a.batch}"]
    line = {"metric": "dUCCSD energy+gradient evals/s (autograd)",
            "value": 1000.0 * a.batch / big["forward_backward_ms"], "unit": "evals/s",
            "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": big["forward_backward_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "torch.autograd over the adjoint sweep, SD pool, half filling, "
                                   f"orbitals {a.norbs}, batches 1 and {a.batch}"},
            "sizes": rows}
    print(json.dumps(line))
    return line


def run_adapt(a, local):
    """ADAPT pool gradients 2 Re <H psi|A_k psi> of every generalized
    spin-conserving single and double (GSD pool) at a 12-operator dUCC state,
    against the plain per-call path (UCCVQE.measure_gradient3 through the
    Computer API, call for call, timed on a sample of operators)."""
    import time
    import torch
    import qforte_b200 as qb
    from qforte_b200._lib import launch_count
    from qforte_b200.ucc import ADAPTVQE, DUCC
    torch.cuda.set_device(local)
    norb = a.adapt_norb
    mol = qb.random_molecule(norb, norb, a.seed)
    pool = qb.SQOpPool()
    pool.set_orb_spaces(mol.hf_reference)
    pool.fill_pool("GSD")
    rng = np.random.default_rng(a.seed + 7)
    tops = [int(v) for v in rng.choice(len(pool), 12, replace=False)]
    amps = rng.uniform(-0.1, 0.1, 12)
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    t0 = time.perf_counter()
    eng._pool_program()
    compile_s = time.perf_counter() - t0
    for _ in range(max(a.warmup, 3)):
        g = eng.pool_gradients(amps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    e0.record()
    for _ in range(a.steps):
        g = eng.pool_gradients(amps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    launches = (launch_count() - l0) // a.steps
    # plain per-call path (measure_gradient3, call for call) on a sample of operators
    drv = ADAPTVQE(mol, engine="percall")
    drv._pool_obj = pool
    drv._tops, drv._tamps = tops, list(amps)
    # the sample: the 20 largest gradients and 20 operators drawn at random
    top = [int(v) for v in np.argsort(-np.abs(g))[:20]]
    rest = [int(v) for v in rng.choice(len(pool), 40, replace=False) if int(v) not in top]
    idx = top + rest[:20]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    qc_psi = qb.Computer(2 * norb)
    qc_psi.apply_circuit(drv.build_Uvqc())
    qc_sig = qb.Computer(qc_psi)
    qc_sig.apply_operator(mol.hamiltonian)
    torch.cuda.synchronize()
    t_state = time.perf_counter() - t0
    t1 = time.perf_counter()
    g_plain = []
    for k in idx:
        coeff, operator = pool[k]
        qc_temp = qb.Computer(qc_psi)
        op = qb.SQOperator()
        op.add_op(operator)
        K = op.jw_transform()
        K.mult_coeffs(coeff)
        qc_temp.apply_operator(K)
        g_plain.append(2.0 * np.real(np.vdot(qc_sig.get_coeff_vec(), qc_temp.get_coeff_vec())))
    t_ops = (time.perf_counter() - t1) / len(idx)
    plain_s = t_state + t_ops * len(pool)
    err = float(np.max(np.abs(np.array(g_plain) - g[idx])))
    line = {"metric": "ADAPT pool gradients per second", "value": len(pool) / (ms * 1e-3),
            "unit": "gradients/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"GSD pool gradients, {2 * norb} qubits ({norb} orbitals, "
                                   f"{norb} electrons), 12-operator dUCC state",
                       "pool_ops": len(pool), "pool_strings": int(eng._pool_program().nstrings),
                       "evaluator_path": eng.evaluator(1).path,
                       "hamiltonian_terms": len(mol.hamiltonian)},
            "gpu_launches": launches, "pool_compile_s": compile_s,
            "max_abs_gradient": float(np.max(np.abs(g))),
            "gradients_above_1e-10": int(np.sum(np.abs(g) > 1e-10)),
            "plain_per_call": {"seconds": plain_s, "unit": "s per full pool",
                               "sample": f"state + H psi once, then {len(idx)} of {len(pool)} "
                                         "operators (the 20 largest gradients and 20 at random) "
                                         "through Computer copies, apply_operator and "
                                         "get_coeff_vec, scaled",
                               "max_abs_diff_vs_batched": err},
            "batched_vs_plain": plain_s / (ms * 1e-3)}
    print(json.dumps(line))
    return line


def serve_trace(a, problems):
    """Poisson arrivals over ``duration`` seconds: (t, key, params, with_grad)."""
    rng = np.random.default_rng(a.seed + 99)
    keys = sorted(problems)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / a.rate)
        if t > a.duration:
            return out
        k = keys[rng.integers(len(keys))]
        out.append((t, k, rng.uniform(-0.1, 0.1, problems[k].nparam), bool(rng.integers(2))))


def replay(server, trace):
    """Submit the trace at its arrival times (open loop); wait for every result."""
    import time
    t0 = time.perf_counter()
    futs = []
    for t, k, p, wg in trace:
        dt = t - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        futs.append((k, server.submit(k, p, wg), time.perf_counter()))
    res = [(k, f.result(), ts) for k, f, ts in futs]
    return res, time.perf_counter() - t0


def run_serve(a, local):
    """Serving: Poisson stream of mixed energy / energy+gradient requests of
    random-integral dUCCSD problems, orbital counts U{lo..hi}, half filling."""
    import torch
    import qforte_b200 as qb
    from qforte_b200.serving import Server
    from qforte_b200.ucc import DUCC
    torch.cuda.set_device(local)
    lo, hi = (int(v) for v in a.norb_range.split(","))
    problems = {}
    for norb in range(lo, hi + 1):
        mol, pool = problem(norb, a.seed + norb)
        problems[f"norb{norb}"] = DUCC(mol.hamiltonian, pool, list(range(len(pool))),
                                       mol.hf_reference)
    trace = serve_trace(a, problems)
    budget = a.budget_gb * 1e9

    def served(max_batch, streams, tr):
        srv = Server(hbm_budget=budget, max_batch=max_batch, streams=streams, device=local)
        for k, d in problems.items():
            srv.register(k, d)
        with srv:
            # warm: one request of each problem and kind (captures the graphs)
            for k, d in problems.items():
                for wg in (False, True):
                    srv.submit(k, np.zeros(d.nparam), wg).result()
            srv.reset_stats()
            res, wall = replay(srv, tr)
            st = srv.stats()
        return st, res, wall

    st, res, wall = served(256, 4, trace)
    by = {}
    for k, (e, g), ts in res:
        by.setdefault(k, 0)
        by[k] += 1
    # per-problem latency: the client-side submit time to the future's completion
    # is not kept per request by the server, so report the server's overall
    # percentiles and the requests per problem
    # sequential baseline: the same requests one at a time (batch 1, one stream)
    nseq = min(len(trace), max(8, len(trace) // 4))
    st1, _, wall1 = served(1, 1, trace[:nseq])
    line = {"metric": "served dUCC requests/s", "value": len(res) / wall, "unit": "requests/s",
            "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": 1000.0 * wall,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"Poisson arrivals at {a.rate}/s for {a.duration} s, "
                                   f"dUCCSD problems of {lo}..{hi} orbitals (half filling, SD "
                                   "pool), half energy and half energy+gradient requests",
                       "requests": len(trace), "per_problem": by, "hbm_budget_gb": a.budget_gb},
            "latency_ms": st.get("latency_ms"), "server": st,
            "sequential": {"requests": nseq, "requests_per_s": nseq / wall1,
                           "latency_ms": st1.get("latency_ms"),
                           "sample": "the first requests of the same trace served one at a time "
                                     "(batch 1, one stream, same evaluator kernels)"}}
    print(json.dumps(line))
    return line


def serve_saturating(a, local, rate=50000.0, duration=0.4, norbs=(5, 6, 7, 8)):
    """Serving at an arrival rate far above what one request at a time can
    take: a Poisson stream of mixed energy / energy+gradient requests of the
    10-16-qubit dUCCSD problems, served with packed launches (every problem's
    requests together, ucc.Pack), against the same trace served one request at
    a time (each problem's own evaluator, batch 1, one stream, no packing) over
    its first requests."""
    import torch
    from qforte_b200.serving import Server
    from qforte_b200.ucc import DUCC
    torch.cuda.set_device(local)
    problems = {}
    for norb in norbs:
        mol, pool = problem(norb, a.seed + norb)
        problems[f"norb{norb}"] = DUCC(mol.hamiltonian, pool, list(range(len(pool))),
                                       mol.hf_reference)
    t = argparse.Namespace(seed=a.seed, rate=rate, duration=duration)
    trace = serve_trace(t, problems)
    t.seed = a.seed + 1000
    t.duration = 0.3
    warm = serve_trace(t, problems)

    def served(max_batch, streams, tr, warm_tr, pack):
        srv = Server(hbm_budget=a.budget_gb * 1e9, max_batch=max_batch, streams=streams,
                     device=local, pack=pack)
        for k, d in problems.items():
            srv.register(k, d)
        with srv:
            replay(srv, warm_tr)
            srv.reset_stats()
            res, wall = replay(srv, tr)
            st = srv.stats()
        return st, len(res), wall

    st, n, wall = served(256, 4, trace, warm, True)
    nseq = min(len(trace), 400)
    st1, n1, wall1 = served(1, 1, trace[:nseq], warm[:64], False)
    return {"workload": f"Poisson arrivals at {rate:.0f}/s for {duration} s, dUCCSD problems of "
                        f"{norbs[0]}..{norbs[-1]} orbitals (half filling, SD pool), half energy "
                        "and half energy+gradient requests",
            "requests": n, "served_requests_per_s": n / wall,
            "served_latency_ms": st.get("latency_ms"),
            "served_batches": st.get("batches"), "served_mean_batch_rows": st.get("mean_batch_rows"),
            "one_at_a_time": {"requests": n1, "requests_per_s": n1 / wall1,
                              "latency_ms": st1.get("latency_ms"),
                              "sample": "the first requests of the same trace, each problem's "
                                        "own evaluator, batch 1, one stream, no packing"},
            "served_vs_one_at_a_time": (n / wall) / (n1 / wall1)}


def secondary(a, local):
    """The metric's other numbers, timed in the same process after the
    headline: gate-sweep passes at 28 qubits (register-blocked tile runs and
    one pass per gate) and at 32 qubits (tile runs, one 64 GiB state),
    Pauli-exponential passes at 28 qubits, and serving latency at a
    saturating arrival rate."""
    from qforte_b200.device import gates_config
    out = {}
    g = argparse.Namespace(**vars(a))
    g.steps, g.warmup, g.no_cpu_baseline, g.autotune = 1, 1, True, False

    def gates(name, n, tile, layers):
        g.nqubits, g.tile, g.layers = str(n), tile, layers
        try:
            r = run_gates(g, 0, 1, local, emit=False)["sweep"][-1]
        finally:
            gates_config(0, 3, 0)
        out[name] = {"layers": layers, "gates": r["gates"], "passes": r["passes"],
                     "ms_per_circuit": r["ms_per_circuit"], "pass_gbs": r["pass_gbs"],
                     "frac_of_hbm": r["frac_of_hbm"],
                     "effective_gate_gbs": r["effective_gate_gbs"],
                     "gpu_launches": r["gpu_launches"], "state_bytes": 16 << n}

    def soft(name, fn):
        # a part that cannot run here (for instance 64 GiB not free) is
        # recorded with its reason; the headline line stands without it
        try:
            fn()
        except Exception as e:  # noqa: BLE001
            out[name] = {"unavailable": f"{type(e).__name__}: {e}"}

    soft("gates28_tile_runs", lambda: gates("gates28_tile_runs", 28, 0, 100))
    soft("gates28_one_pass_per_gate", lambda: gates("gates28_one_pass_per_gate", 28, -1, 20))
    soft("gates32_tile_runs", lambda: gates("gates32_tile_runs", 32, 0, 10))
    p = argparse.Namespace(**vars(a))
    p.pexp_n, p.pexp_strings, p.steps, p.warmup = 28, 64, 3, 1
    soft("pauli_exp28", lambda: out.__setitem__(
        "pauli_exp28", run_pexp(p, local, emit=False, ducc_part=False)))
    soft("serving", lambda: out.__setitem__("serving", serve_saturating(a, local)))
    out["peak_gbs"], out["peak_source"] = peaks()
    return out


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    if a.workload == "gates":
        if rank == 0:
            run_gates(a, rank, world, local)
        return
    if a.workload == "grad":
        if rank == 0:
            run_grad(a, local)
        return
    if a.workload == "adapt":
        if rank == 0:
            run_adapt(a, local)
        return
    if a.workload == "serve":
        if rank == 0:
            run_serve(a, local)
        return
    if a.workload == "pexp":
        if rank == 0:
            run_pexp(a, local)
        return
    if a.workload == "pqe":
        if rank == 0:
            run_pqe(a, local)
        return
    if a.workload == "sample":
        if rank == 0:
            run_sample(a, local)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import qforte_b200 as qb
    from qforte_b200 import _lib
    from qforte_b200.ucc import DUCC

    _lib.check(_lib.lib().qfb_set_stream(_lib.ctypes.c_void_p(
        torch.cuda.current_stream().cuda_stream)))
    mol, pool = problem(a.norb, a.seed)
    tops = list(range(len(pool)))
    M = len(tops)
    if a.full_space or a.one_set:
        from qforte_b200.ucc import evaluator_config
        evaluator_config(False if a.full_space else "one-set")
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    P = replica_parameters(a.seed, rank, a.batch, M)
    # consecutive steps alternate between S evaluators, each on its own stream
    S = max(1, a.streams)
    evs = [eng.evaluator(a.batch)]
    for _ in range(1, S):
        from qforte_b200.ucc import Evaluator
        evs.append(Evaluator(eng, a.batch))
    ev = evs[0]
    stream = torch.cuda.current_stream()
    streams = [stream] + [torch.cuda.Stream() for _ in range(1, S)]
    bufs = [e.tensors() for e in evs]
    for b in bufs:
        b[0].copy_(torch.from_numpy(P))
    d_params, d_energy, d_grad = bufs[0]

    def on(k):
        """Make stream k the library's stream (torch's current one too)."""
        _lib.check(_lib.lib().qfb_set_stream(_lib.ctypes.c_void_p(streams[k].cuda_stream)))
        return torch.cuda.stream(streams[k])

    def fork(ev0):
        # every stream starts after the timed region's opening event
        for st in streams[1:]:
            st.wait_event(ev0)

    def join(ev1):
        for st in streams[1:]:
            e = torch.cuda.Event()
            e.record(st)
            stream.wait_event(e)
        ev1.record(stream)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-resident throughput ----------------------------------------
    for _ in range(max(a.warmup, 3)):
        for k in range(S):
            with on(k):
                evs[k].run(True)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = _lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fork(e0)
    for i in range(a.steps):
        with on(i % S):
            evs[i % S].run(True)
    join(e1)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - l0
    ms = e0.elapsed_time(e1) / a.steps
    # a timed region shorter than the sampler's period is followed by untimed
    # steps of the same workload until the clock record spans 0.8 s
    import time as _time
    t_end = _time.perf_counter() + max(0.0, 0.8 - a.steps * ms / 1000.0)
    while _time.perf_counter() < t_end:
        for k in range(S):
            with on(k):
                evs[k].run(True)
        torch.cuda.synchronize()
    barrier()
    ck = clocks.stop()
    if ck is not None:
        ck["window"] = "timed region plus untimed steps of the same workload to 0.8 s"
    ms_all = max_over_ranks(ms, world, "cuda")
    value = whole_job_rate(world, a.batch, ms_all)

    # ---- end to end through the public API with host buffers ---------------
    # every step copies its parameters from pinned host memory and reads its
    # energies and gradients back; with S streams a step's copies overlap the
    # other streams' kernels, and a stream's host buffers are reused only
    # after its previous step's read-back completed
    hP = torch.from_numpy(P).pin_memory()
    hE = [torch.empty(a.batch, dtype=torch.float64).pin_memory() for _ in range(S)]
    hG = [torch.empty((a.batch, M), dtype=torch.float64).pin_memory() for _ in range(S)]
    done = [None] * S
    for k in range(S):
        with on(k):
            evs[k].eval(P, True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    fork(e0)
    for i in range(a.steps):
        k = i % S
        if done[k] is not None:
            done[k].synchronize()  # the host holds step i - S's results
        with on(k):
            bufs[k][0].copy_(hP, non_blocking=True)
            evs[k].run(True)
            hE[k].copy_(bufs[k][1], non_blocking=True)
            hG[k].copy_(bufs[k][2], non_blocking=True)
            done[k] = torch.cuda.Event()
            done[k].record(streams[k])
    for d in done:
        if d is not None:
            d.synchronize()
    join(e1)
    torch.cuda.synchronize()
    _lib.check(_lib.lib().qfb_set_stream(_lib.ctypes.c_void_p(stream.cuda_stream)))
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / a.steps, world, "cuda")
    e2e = whole_job_rate(world, a.batch, ms_e2e)
    # the numbers coming back are the evaluator's
    for k in range(S):
        assert np.all(np.isfinite(hE[k].numpy())) and np.all(np.isfinite(hG[k].numpy()))

    # ---- the plain per-call GPU path: the reference's drivers call for call --
    plain = None
    if rank == 0 and not a.no_cpu_baseline:
        import time
        from qforte_b200.ucc import UCCNVQE
        drv = UCCNVQE(mol, engine="percall")
        drv._pool_obj = pool
        drv._tops, drv._tamps = tops, list(P[0])
        drv.energy_feval(P[0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E_p = drv.energy_feval(P[0])
        g_p = drv.measure_gradient(P[0])
        torch.cuda.synchronize()
        t_p = time.perf_counter() - t0
        e_b, g_b = ev.eval(P, True)
        plain = {"value": 1.0 / t_p, "unit": UNIT,
                 "sample": "one energy + gradient of parameter row 0 through the Computer API "
                           "call for call (UCCNVQE engine='percall': the ansatz circuit built and "
                           "applied, direct_op_exp_val, then the reverse sweep of "
                           "measure_gradient with Computer copies, apply_operator and "
                           "get_coeff_vec readbacks)",
                 "wall_s": t_p,
                 "energy_abs_diff": abs(E_p - float(e_b[0])),
                 "gradient_max_abs_diff": float(np.max(np.abs(np.asarray(g_p) - g_b[0])))}

    # ---- roofline of the dominant kernel -------------------------------------
    import ctypes
    st_ms = (ctypes.c_double * 4)()
    st_n = (ctypes.c_int64 * 4)()
    _lib.check(_lib.lib().qfb_ucc_profile(ev.h, 1, max(2, min(a.steps, 5)), st_ms, st_n))
    stages = ["reference", "U(t) program", "H psi + energy", "gradient sweep"]
    N = 1 << (2 * a.norb)
    compact = ev.path == 2
    if ev.path == 3:
        # slot-minor compact states in global memory: a step record reads and
        # writes the pairs it touches; stage totals are reported, per launch
        # the mean over the stage's launches
        nsec, nnz = ev.sector_size, ev.h_rows
        per_launch_bytes = {1: 32 * nsec * a.batch, 2: (12 * nnz / max(1, a.batch) + 32 * nsec) * a.batch,
                            3: 64 * nsec * a.batch}
    elif compact:
        # one CTA per parameter set, states in shared memory: the HBM bytes
        # each kernel must move per launch are the save buffer it writes /
        # reads (8 bytes an amplitude with real states, else 16) and, for H,
        # the H rows once (12 bytes an entry); every parameter set then
        # streams the rows again from L2, reported beside it
        nsec, nnz = ev.sector_size, ev.h_rows
        elem = 8 if ev.real_states else 16
        per_launch_bytes = {1: elem * nsec * a.batch,
                            2: 12 * nnz + 2 * elem * nsec * a.batch,
                            3: 2 * elem * nsec * a.batch}
        l2_stream = {2: 12 * nnz * a.batch}
    else:
        state_bytes = 16 * N * a.batch
        # algorithmic bytes per launch of each stage's main kernel
        per_launch_bytes = {1: 2 * state_bytes,          # exp pass: read + write psi
                            2: 2 * state_bytes,          # H psi: read psi (gathered) + write sigma
                            3: 4 * state_bytes}          # gradient step: RMW psi and sigma
    dom = max((1, 2, 3), key=lambda k: st_ms[k])
    # launches of each stage's main kernel (stage 2 also holds the two small
    # energy-reduction kernels, stage 3 the gradient finalisation)
    main_launches = {1: st_n[1], 2: 1, 3: max(1, st_n[3] - 1)}
    nl = max(1, main_launches[dom])
    avg_ms = st_ms[dom] / nl
    hbm, src = peaks()
    achieved = per_launch_bytes[dom] / (avg_ms / 1000.0) / 1e9
    if ev.path == 3:
        kernel = {1: "k_cg_step (forward)", 2: "k_cg_h_rows", 3: "k_cg_step (sweep)"}[dom]
    elif compact:
        kernel = {1: "k_sector_forward", 2: "k_sector_h", 3: "k_sector_sweep"}[dom]
    else:
        kernel = {1: "k_window<1>", 2: "k_sum_apply_sector" if ev.sector_size else "k_sum_apply_tiled",
                  3: "k_window<2>"}[dom]
    roof = {"bound": "hbm", "kernel": kernel, "stage": stages[dom], "achieved": achieved,
            "peak": hbm, "peak_source": src, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": None, "algorithmic_bytes_per_launch": per_launch_bytes[dom],
            "avg_launch_ms": avg_ms,
            "stages_ms": {stages[k]: st_ms[k] for k in range(4)},
            "stages_launches": {stages[k]: int(st_n[k]) for k in range(4)},
            "evaluator_path": {0: "full space", 1: "full space, sigma on the sector",
                               2: "compact sector in shared memory",
                               3: "compact sector in global memory"}[ev.path]}
    if ev.path in (2, 3):
        roof["sector_amplitudes"] = ev.sector_size
        roof["h_row_entries"] = ev.h_rows
    if compact:
        roof["real_states"] = ev.real_states
        roof["bound"] = "l1/shared"
        roof["bound_note"] = ("states live in shared memory, so HBM carries only the save "
                              "buffer and the step lists; frac is the HBM fraction, the binding "
                              "unit is the L1 / shared-memory pipe (ncu figures in "
                              "binding_unit)")
        ncu = NCU_SECTOR_UCC16_B256.get(kernel)
        if ncu is not None and a.norb == 8 and a.batch == 256:
            roof["traffic"] = ncu["dram_bytes"]
            roof["binding_unit"] = dict(ncu)
        if dom in l2_stream:
            roof["l2_stream_bytes_per_launch"] = l2_stream[dom]
            roof["l2_stream_gbs"] = l2_stream[dom] / (avg_ms / 1000.0) / 1e9

    dtype = "f64 (real sector states; complex128 API)" if compact and ev.real_states else "c128"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": max(a.warmup, 3), "ms_per_step": ms_all, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": workload_config(a, len(mol.hamiltonian), M),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(P.nbytes),
                    "d2h_bytes_per_step": int(hE[0].numel() * 8 + hG[0].numel() * 8)},
            "roofline": roof, "gpu_launches": int(launches), "clocks": ck}
    if plain is not None:
        # the same evaluation through the per-call C ABI with the host work
        # hoisted (state preparation, H psi, one device gradient call): the
        # plain path's device time, beside the Python drivers' wall time above
        import time
        eng.energy_grad_percall(P[0])
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        c0.record(stream)
        E_c, g_c = eng.energy_grad_percall(P[0])
        c1.record(stream)
        torch.cuda.synchronize()
        t_c = time.perf_counter() - t0
        line["plain_per_call"] = plain
        line["batched_vs_plain"] = value / plain["value"]
        line["per_call_cabi"] = {"value": 1000.0 / c0.elapsed_time(c1), "unit": UNIT,
                                 "device_ms": c0.elapsed_time(c1), "wall_s": t_c,
                                 "sample": "one energy + gradient of parameter row 0, full-space "
                                           "states, through the per-call C ABI (reference prep, "
                                           "U(t), H psi, <psi|H psi>, one device gradient call)",
                                 "energy_abs_diff": abs(E_c - float(e_b[0])),
                                 "gradient_max_abs_diff": float(np.max(np.abs(g_c - g_b[0])))}
        line["batched_vs_per_call_cabi"] = value / line["per_call_cabi"]["value"]
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cb = cpu_baseline(a, mol, pool, P)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                       "extrapolated", "cpu_model")}
            line["cpu_baseline"]["parts_s"] = cb["parts"]
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if rank == 0 and world == 1 and not a.no_secondary:
        line["secondary"] = secondary(a, local)
    if rank == 0:
        print(json.dumps(line))
    del ev, eng
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
