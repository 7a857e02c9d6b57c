"""Record the engine calls of the reference's own drivers (fixture generator).

The reference package is imported unmodified -- its Python drivers and its
compiled C++ ``Computer`` (``make -C oracle ref``), sources read where they lie
($QFORTE_REF_SRC, default /root/reference/src/qforte) -- with ``qforte.Computer``
(and the two module functions that take or make Computers) replaced by a
recording wrapper around the real one.  The reference's tests are then run as
written there:

* tests/test_uccsd.py:13-29: UCCNVQE, He/cc-pVDZ, SD pool, analytic gradient,
  at FCI within 1e-10;
* tests/test_adapt_vqe.py:12-40: ADAPTVQE, H4/STO-6G, SDTQ pool, at FCI
  within 5e-11.

Every Computer call -- constructor, copy, apply_circuit, apply_operator,
direct_op_exp_val, get_coeff_vec, ... -- is written to
tests/golden/dropin_trace_<name>.npz with its operands (circuits as gate
label, target, control and parameter; operators as terms) and the reference's
result (numbers exactly; a state vector as its norm and its inner products
with three seeded random vectors).  tests/test_dropin_trace_host.py replays a
trace on the oracle and tests/test_gpu_dropin_replay.py on the device
Computer, call for call.

Run from the repository root:  python tests/golden/make_dropin_trace.py
"""

import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
warnings.filterwarnings("ignore")

from oracle import oracle as O  # noqa: E402

# call codes (the replay side reads the same table from tests/dropin_trace.py)
sys.path.insert(0, os.path.join(ROOT, "tests"))
from dropin_trace import OPS, projections  # noqa: E402


class Recorder:
    """Tables of one trace: gates, circuits, operators, pools, vectors, calls."""

    def __init__(self):
        self.labels, self.lab_idx = [], {}
        self.gates, self.gate_idx = [], {}
        self.circ_gates, self.circ_ptr, self.circ_idx = [], [0], {}
        self.term_coef, self.term_circ, self.op_ptr, self.op_idx = [], [], [0], {}
        self.pool_coef, self.pool_op, self.pool_ptr = [], [], [0]
        self.vec, self.vec_ptr = [], [0]
        self.idx, self.idx_ptr = [], [0]
        self.calls, self.res, self.res_ptr = [], [], [0]

    def gate(self, g):
        lab = g.gate_id()
        if lab not in self.lab_idx:
            self.lab_idx[lab] = len(self.labels)
            self.labels.append(lab)
        p = g.parameter() if g.has_parameter() else None
        key = (lab, g.target(), g.control(), p)
        if key not in self.gate_idx:
            self.gate_idx[key] = len(self.gates)
            self.gates.append((self.lab_idx[lab], g.target(), g.control(),
                               0 if p is None else 1, 0.0 if p is None else float(p)))
        return self.gate_idx[key]

    def circuit(self, circ):
        key = tuple(self.gate(g) for g in circ.gates())
        if key not in self.circ_idx:
            self.circ_idx[key] = len(self.circ_ptr) - 1
            self.circ_gates.extend(key)
            self.circ_ptr.append(len(self.circ_gates))
        return self.circ_idx[key]

    def operator(self, qo):
        key = tuple((complex(c), self.circuit(circ)) for c, circ in qo.terms())
        if key not in self.op_idx:
            self.op_idx[key] = len(self.op_ptr) - 1
            for c, k in key:
                self.term_coef.append(c)
                self.term_circ.append(k)
            self.op_ptr.append(len(self.term_coef))
        return self.op_idx[key]

    def pool(self, pool):
        for c, op in pool.terms():
            self.pool_coef.append(complex(c))
            self.pool_op.append(self.operator(op))
        self.pool_ptr.append(len(self.pool_coef))
        return len(self.pool_ptr) - 2

    def vector(self, v):
        self.vec.extend(complex(x) for x in v)
        self.vec_ptr.append(len(self.vec))
        return len(self.vec_ptr) - 2

    def indices(self, idxs):
        self.idx.extend(int(i) for i in idxs)
        self.idx_ptr.append(len(self.idx))
        return len(self.idx_ptr) - 2

    def call(self, cid, op, a=-1, b=-1, result=()):
        self.calls.append((cid, OPS[op], a, b))
        self.res.extend(complex(x) for x in result)
        self.res_ptr.append(len(self.res))

    def save(self, path, meta):
        arr = lambda x, t: np.array(x, dtype=t)  # noqa: E731
        g = np.array(self.gates, dtype=np.float64).reshape(-1, 5)
        np.savez_compressed(
            path, labels=np.array(self.labels), gate_lab=g[:, 0].astype(np.int32),
            gate_t=g[:, 1].astype(np.int32), gate_c=g[:, 2].astype(np.int32),
            gate_hp=g[:, 3].astype(np.int8), gate_p=g[:, 4],
            circ_gates=arr(self.circ_gates, np.int32), circ_ptr=arr(self.circ_ptr, np.int64),
            term_coef=arr(self.term_coef, np.complex128), term_circ=arr(self.term_circ, np.int32),
            op_ptr=arr(self.op_ptr, np.int64), pool_coef=arr(self.pool_coef, np.complex128),
            pool_op=arr(self.pool_op, np.int32), pool_ptr=arr(self.pool_ptr, np.int64),
            vec=arr(self.vec, np.complex128), vec_ptr=arr(self.vec_ptr, np.int64),
            idx=arr(self.idx, np.int64), idx_ptr=arr(self.idx_ptr, np.int64),
            calls=arr(self.calls, np.int32).reshape(-1, 4), res=arr(self.res, np.complex128),
            res_ptr=arr(self.res_ptr, np.int64), **meta)


def install(qf, rec):
    """Replace qforte.Computer and the functions that take or make Computers."""
    Real = qf.Computer
    real_inner, real_prepare = qf.inner_product, qf.prepare_computer_from_circuit
    count = [0]

    class RecComputer:
        def __init__(self, arg):
            self.cid = count[0]
            count[0] += 1
            if isinstance(arg, RecComputer):
                self.c = Real(arg.c)
                rec.call(self.cid, "copy", arg.cid)
            else:
                self.c = Real(int(arg))
                rec.call(self.cid, "new", int(arg))

        def apply_circuit(self, circ):
            rec.call(self.cid, "apply_circuit", rec.circuit(circ))
            return self.c.apply_circuit(circ)

        def apply_operator(self, qo):
            rec.call(self.cid, "apply_operator", rec.operator(qo))
            return self.c.apply_operator(qo)

        def apply_gate(self, g):
            c = qf.Circuit()
            c.add(g)
            rec.call(self.cid, "apply_circuit", rec.circuit(c))
            return self.c.apply_gate(g)

        def apply_constant(self, a):
            rec.call(self.cid, "apply_constant", rec.vector([a]))
            return self.c.apply_constant(a)

        def direct_op_exp_val(self, qo):
            v = self.c.direct_op_exp_val(qo)
            rec.call(self.cid, "direct_op_exp_val", rec.operator(qo), result=[v])
            return v

        def get_coeff_vec(self):
            v = self.c.get_coeff_vec()
            rec.call(self.cid, "get_coeff_vec", result=projections(np.asarray(v)))
            return v

        def set_coeff_vec(self, v):
            rec.call(self.cid, "set_coeff_vec", rec.vector(v))
            return self.c.set_coeff_vec(v)

        def get_nqubit(self):
            n = self.c.get_nqubit()
            rec.call(self.cid, "get_nqubit", result=[n])
            return n

        def direct_oppl_exp_val(self, pool):
            v = self.c.direct_oppl_exp_val(pool)
            rec.call(self.cid, "direct_oppl_exp_val", rec.pool(pool), result=v)
            return v

        def direct_idxd_oppl_exp_val(self, pool, idxs):
            v = self.c.direct_idxd_oppl_exp_val(pool, idxs)
            rec.call(self.cid, "direct_idxd_oppl_exp_val", rec.pool(pool), rec.indices(idxs), result=v)
            return v

        def __getattr__(self, name):
            raise AttributeError(f"the recorder does not wrap Computer.{name}")

    def inner_product(a, b):
        v = real_inner(a.c, b.c)
        rec.call(a.cid, "inner_product", b.cid, result=[v])
        return v

    def prepare(n, circ):
        qc = RecComputer(n)
        qc.apply_circuit(circ)
        return qc

    qf.Computer = RecComputer
    qf.inner_product = inner_product
    qf.prepare_computer_from_circuit = prepare
    return lambda: setattr(qf, "Computer", Real) or setattr(qf, "inner_product", real_inner) or \
        setattr(qf, "prepare_computer_from_circuit", real_prepare)


def main():
    ref_src = os.environ.get("QFORTE_REF_SRC", "/root/reference/src/qforte")
    qf = O.load_reference(ref_src)
    data = os.path.join(os.path.dirname(os.path.dirname(ref_src.rstrip("/"))), "tests")
    runs = {
        "uccnvqe_he": (lambda: (lambda mol: (lambda alg: (alg.run(pool_type="SD", use_analytic_grad=True), alg)[1])(
            qf.UCCNVQE(mol)))(qf.system_factory(system_type="molecule", build_type="external",
                                                basis="cc-pvdz", filename=os.path.join(data, "He-ccpvdz.json"))),
                       -2.887594831090938, 1.0e-10),
        "adaptvqe_h4": (lambda: (lambda mol: (lambda alg: (alg.run(adapt_maxiter=20, avqe_thresh=1.0e-4,
                                                                   opt_thresh=1.0e-5, use_analytic_grad=True,
                                                                   pool_type="SDTQ"), alg)[1])(
            qf.ADAPTVQE(mol, print_summary_file=False)))(
            qf.system_factory(stytem_type="molecule", build_type="external", basis="sto-6g",
                              filename=os.path.join(data, "H4-sto6g-075a.json"))),
                        -2.1628978832666865, 5.0e-11),
    }
    only = sys.argv[1:] or list(runs)
    for name in only:
        fn, e_fci, tol = runs[name]
        rec = Recorder()
        restore = install(qf, rec)
        try:
            alg = fn()
        finally:
            restore()
        e = alg.get_gs_energy()
        assert abs(e - e_fci) < tol, (name, e, e_fci)
        path = os.path.join(HERE, f"dropin_trace_{name}.npz")
        rec.save(path, dict(name=name, energy=e, e_fci=e_fci, tol=tol))
        print(f"{name}: {len(rec.calls)} calls, {len(rec.gates)} gates, {len(rec.circ_ptr) - 1} circuits, "
              f"{len(rec.op_ptr) - 1} operators, energy {e:.12f}, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
