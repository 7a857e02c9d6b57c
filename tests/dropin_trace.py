"""Replay of a recorded reference-driver trace (tests/golden/dropin_trace_*.npz).

A trace holds every Computer call the reference's own drivers made, with the
operands and the reference's results (tests/golden/make_dropin_trace.py).
``replay(trace, make, check)`` rebuilds the operands with this package's
Gate, Circuit and QubitOperator, makes the calls on Computers from
``make(n)`` / ``make(src)`` and hands every recorded result and the replayed
one to ``check``.  State vectors are compared through ``projections``: the
norm and the inner products with three seeded random unit vectors.
"""

import numpy as np

OPS = {name: i for i, name in enumerate((
    "new", "copy", "apply_circuit", "apply_operator", "apply_constant", "direct_op_exp_val",
    "get_coeff_vec", "set_coeff_vec", "get_nqubit", "direct_oppl_exp_val",
    "direct_idxd_oppl_exp_val", "inner_product"))}
NAMES = {i: name for name, i in OPS.items()}


def projections(v):
    """[norm, <r_0|v>, <r_1|v>, <r_2|v>] with r_k seeded random unit vectors."""
    v = np.asarray(v, dtype=np.complex128)
    rng = np.random.default_rng(1000 + v.size)
    out = [np.linalg.norm(v)]
    for _ in range(3):
        r = rng.normal(size=v.size) + 1j * rng.normal(size=v.size)
        out.append(np.vdot(r / np.linalg.norm(r), v))
    return np.array(out, dtype=np.complex128)


class Trace:
    """A loaded trace with this package's objects built on demand."""

    def __init__(self, z):
        self.z = z if isinstance(z, dict) else {k: z[k] for k in z.files}  # read each array once
        self.labels = [str(s) for s in z["labels"]]
        self._circ, self._op = {}, {}

    def circuit(self, k):
        import qforte_b200 as qb
        if k not in self._circ:
            z = self.z
            c = qb.Circuit()
            for gi in z["circ_gates"][z["circ_ptr"][k]:z["circ_ptr"][k + 1]]:
                lab = self.labels[z["gate_lab"][gi]]
                t, ctl = int(z["gate_t"][gi]), int(z["gate_c"][gi])
                if z["gate_hp"][gi]:
                    c.add(qb.gate(lab, t, ctl, float(z["gate_p"][gi])))
                else:
                    c.add(qb.gate(lab, t, ctl))
            self._circ[k] = c
        return self._circ[k]

    def operator(self, k):
        import qforte_b200 as qb
        if k not in self._op:
            z = self.z
            qo = qb.QubitOperator()
            for j in range(z["op_ptr"][k], z["op_ptr"][k + 1]):
                qo.add(complex(z["term_coef"][j]), self.circuit(int(z["term_circ"][j])))
            self._op[k] = qo
        return self._op[k]

    def pool(self, k):
        import qforte_b200 as qb
        z = self.z
        pool = qb.QubitOpPool()
        for j in range(z["pool_ptr"][k], z["pool_ptr"][k + 1]):
            pool.add(complex(z["pool_coef"][j]), self.operator(int(z["pool_op"][j])))
        return pool

    def vector(self, k):
        z = self.z
        return z["vec"][z["vec_ptr"][k]:z["vec_ptr"][k + 1]]

    def indices(self, k):
        z = self.z
        return [int(i) for i in z["idx"][z["idx_ptr"][k]:z["idx_ptr"][k + 1]]]


def replay(z, make, check, inner=None, limit=None):
    """Make the recorded calls (the first ``limit`` of them, or all); check(i,
    name, recorded, replayed) for each call with a result.  make(n) or
    make(src_computer) builds a Computer; inner(a, b) is the module-level
    inner product.  Returns the number of calls made."""
    tr = Trace(z)
    z = tr.z
    comps = {}
    res, rp = z["res"], z["res_ptr"]
    calls = z["calls"] if limit is None else z["calls"][:limit]
    for i, (cid, op, a, b) in enumerate(calls):
        name = NAMES[int(op)]
        rec = res[rp[i]:rp[i + 1]]
        if name == "new":
            comps[int(cid)] = make(int(a))
            continue
        if name == "copy":
            comps[int(cid)] = make(comps[int(a)])
            continue
        qc = comps[int(cid)]
        if name == "apply_circuit":
            qc.apply_circuit(tr.circuit(int(a)))
        elif name == "apply_operator":
            qc.apply_operator(tr.operator(int(a)))
        elif name == "apply_constant":
            qc.apply_constant(complex(tr.vector(int(a))[0]))
        elif name == "set_coeff_vec":
            qc.set_coeff_vec(list(tr.vector(int(a))))
        elif name == "direct_op_exp_val":
            check(i, name, rec, np.array([qc.direct_op_exp_val(tr.operator(int(a)))]))
        elif name == "get_coeff_vec":
            check(i, name, rec, projections(qc.get_coeff_vec()))
        elif name == "get_nqubit":
            check(i, name, rec, np.array([qc.get_nqubit()]))
        elif name == "direct_oppl_exp_val":
            check(i, name, rec, np.array(qc.direct_oppl_exp_val(tr.pool(int(a)))))
        elif name == "direct_idxd_oppl_exp_val":
            check(i, name, rec, np.array(qc.direct_idxd_oppl_exp_val(tr.pool(int(a)), tr.indices(int(b)))))
        elif name == "inner_product":
            check(i, name, rec, np.array([inner(qc, comps[int(a)])]))
        else:
            raise ValueError(f"unknown call {name}")
    return len(calls)
