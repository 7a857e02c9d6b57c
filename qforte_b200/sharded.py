"""One state vector of n qubits split over the ranks of a process group.

A state too large for one GPU (33 qubits and up: 128 GiB of complex128 and
more) is held as 2^g shards of 2^(n-g) amplitudes, one per rank of a group of
2^g ranks (one process per GPU).  Physical slot s < L = n - g of an amplitude
index is bit s of the rank's local index; slot L + k is bit k of the rank.
Logical qubit q sits in slot ``pos[q]`` (initially q).

* Gates (Computer.apply_circuit, computer.cc:93-114): a run of consecutive
  gates whose qubits all sit in local slots is applied to the local shard as
  one call of the device gate path (tile runs, one pass per gate, dense
  blocks), with the gates' qubits renamed to their slots.  A gate on a qubit
  in a rank slot first swaps that qubit with a local slot: every rank sends
  the half of its shard whose local bit differs from its rank bit to the
  partner rank (rank ^ 2^k) and receives the partner's half in its place
  (pairwise send / receive, NCCL over NVLink; in chunks, so the extra device
  memory is bounded).  The logical state is unchanged, only the qubit map.
* Expectation values of Pauli sums (direct_op_exp_val,
  computer.cc:753-771): a term P(x, z) with x's rank bits xg pairs every rank
  r' with the rank r = r' ^ xg.  For each distinct xg (at most 2^g - 1 besides
  0) the ranks exchange whole shards, each rank computes
  <psi_r'| P(x_local, z_local) |psi_r> on the device with the coefficient
  i^{|xg & zg|} (-1)^{|r & zg|}, and one all-reduce sums the ranks.

No kernel here waits on another rank: every exchange is a host-ordered
collective step of torch.distributed, taken by all ranks in the same order.
The local shard is a ``qforte_b200.Computer``; tests on CPU substitute a
host stand-in through ``local_factory``.
"""

import math

import numpy as np

__all__ = ["ShardedComputer"]


def _bits(v):
    out, k = [], 0
    while v:
        if v & 1:
            out.append(k)
        v >>= 1
        k += 1
    return out


class ShardedComputer:
    """An n-qubit complex128 state over the 2^g ranks of ``group`` (|0...0>).

    ``local_factory(nqubit)`` makes the local shard (default: the device
    Computer); ``chunk_bytes`` bounds the buffers of one exchange.
    """

    def __init__(self, nqubit, group=None, local_factory=None, chunk_bytes=1 << 30):
        import torch.distributed as dist
        self._dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        g = int(round(math.log2(self.world)))
        if 1 << g != self.world:
            raise ValueError(f"a sharded state needs a power-of-two number of ranks, not {self.world}")
        if nqubit - g < 2:
            raise ValueError(f"{nqubit} qubits over {self.world} ranks leave fewer than 2 local qubits")
        self.nqubit, self.g, self.L = int(nqubit), g, int(nqubit) - g
        if local_factory is None:
            from .computer import Computer
            local_factory = Computer
        self._factory = local_factory
        self._local = local_factory(self.L)
        self._chunk = max(16, int(chunk_bytes) // 16)  # amplitudes per exchange chunk
        self.pos = list(range(self.nqubit))   # logical qubit -> slot
        self.slot = list(range(self.nqubit))  # slot -> logical qubit
        self._clock = [0] * self.nqubit       # last use of each logical qubit
        self._t = 0
        self.exchanges = 0
        self.reset()

    # ---- state ---------------------------------------------------------------
    def get_nqubit(self):
        return self.nqubit

    def reset(self):
        """|0...0>: amplitude 1 at index 0, which lives on rank 0."""
        if self.rank == 0:
            self._local.reset()
        else:
            self._local.null_state()

    def local(self):
        return self._local

    def _tensor(self):
        return self._local.tensor()

    def gather(self, dst=0):
        """The whole state in logical qubit order on rank ``dst`` (numpy; for
        tests at sizes a host holds), None elsewhere."""
        import torch
        t = torch.view_as_real(self._tensor().contiguous())
        parts = [torch.empty_like(t) for _ in range(self.world)] if self.rank == dst else None
        self._dist.gather(t, parts, dst=self._peer(dst), group=self.group)
        if self.rank != dst:
            return None
        phys = np.concatenate([torch.view_as_complex(p).cpu().numpy() for p in parts])
        # physical index -> logical index: bit pos[q] of the physical index is qubit q
        n = self.nqubit
        idx = np.arange(1 << n, dtype=np.int64)
        logical = np.zeros_like(idx)
        for q in range(n):
            logical |= ((idx >> self.pos[q]) & 1) << q
        out = np.empty_like(phys)
        out[logical] = phys
        return out

    # ---- qubit map -------------------------------------------------------------
    def _swap_in(self, q, keep):
        """Bring logical qubit q from its rank slot into a local slot, evicting
        the local qubit used least recently that is not in ``keep``."""
        G = self.pos[q]
        k = G - self.L
        cand = [s for s in range(self.L) if self.slot[s] not in keep]
        j = min(cand, key=lambda s: (self._clock[self.slot[s]], -s))
        self._exchange_half(j, k)
        q_out = self.slot[j]
        self.pos[q], self.pos[q_out] = j, G
        self.slot[j], self.slot[G] = q, q_out
        self.exchanges += 1

    def _exchange_half(self, j, k):
        """Swap the roles of local bit j and rank bit k: send the half of the
        shard whose bit j differs from this rank's bit k to the partner and
        take the partner's half in its place, chunk by chunk."""
        import torch
        dist = self._dist
        b = (self.rank >> k) & 1
        partner = self.rank ^ (1 << k)
        t = self._tensor()
        half = t.view(-1, 2, 1 << j)[:, 1 - b, :]  # [2^(L-1-j), 2^j] strided
        flat_rows, width = half.shape
        rows_per = max(1, self._chunk // width)
        for r0 in range(0, flat_rows, rows_per):
            part = half[r0:r0 + rows_per]
            send = torch.view_as_real(part.contiguous())  # (re, im) pairs on the wire
            recv = torch.empty_like(send)
            self._sendrecv(send, recv, partner)
            part.copy_(torch.view_as_complex(recv))

    def _sendrecv(self, send, recv, partner):
        dist = self._dist
        ops = [dist.P2POp(dist.isend, send, self._peer(partner), group=self.group),
               dist.P2POp(dist.irecv, recv, self._peer(partner), group=self.group)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()

    def _peer(self, r):
        """Group rank -> global rank (batch_isend_irecv takes global ranks)."""
        if self.group is None:
            return r
        return self._dist.get_global_rank(self.group, r)

    # ---- gates ---------------------------------------------------------------
    def apply_circuit(self, circ):
        self.apply_gates(circ.gates())

    def apply_gate(self, gate):
        self.apply_gates([gate])

    def apply_gates(self, gates):
        from .circuit import Circuit
        from .computer import _as_gate
        from .gate import Gate
        gates = [_as_gate(g) for g in gates]
        run = []

        def flush():
            if run:
                c = Circuit()
                for g in run:
                    c.add(g)
                self._local.apply_circuit(c)
                run.clear()

        for g in gates:
            t, c = g.target(), g.control()
            if t >= self.nqubit or c >= self.nqubit:
                raise ValueError(f"gate on qubit {max(t, c)} of a {self.nqubit}-qubit state")
            need = {t, c}
            if any(self.pos[q] >= self.L for q in need):
                flush()
                for q in need:
                    if self.pos[q] >= self.L:
                        self._swap_in(q, need)
            self._t += 1
            for q in need:
                self._clock[q] = self._t
            # the same gate (label, matrix, parameter) on the qubits' slots
            run.append(Gate(g.gate_id(), self.pos[t], self.pos[c], g._mat, g._param))
        flush()

    # ---- expectation values ------------------------------------------------------
    def _phys(self, m):
        out = 0
        for q in _bits(m):
            out |= 1 << self.pos[q]
        return out

    def expval_terms(self, terms):
        """<psi| sum_k c_k P(x_k, z_k) |psi> for logical masks [(c, x, z)]."""
        import torch
        dist = self._dist
        Lmask = (1 << self.L) - 1
        groups = {}
        for c, x, z in terms:
            xp, zp = self._phys(int(x)), self._phys(int(z))
            groups.setdefault(xp >> self.L, []).append((complex(c), xp & Lmask, zp & Lmask,
                                                        zp >> self.L))
        total = 0j
        for xg in sorted(groups):
            partner = self.rank ^ xg
            if xg == 0:
                ket = None
            else:
                ket = self._factory(self.L)
                src = torch.view_as_real(self._tensor().contiguous())
                recv = torch.empty_like(src)
                self._sendrecv(src, recv, partner)
                ket.tensor().copy_(torch.view_as_complex(recv))
            local = []
            for c, xl, zl, zg in groups[xg]:
                ph = (1j ** bin(xg & zg).count("1")) * (-1) ** bin(partner & zg).count("1")
                local.append((c * ph, xl, zl))
            total += self._local_expval(local, ket)
            del ket
        dev = self._tensor().device
        v = torch.tensor([total.real, total.imag], dtype=torch.float64, device=dev)
        dist.all_reduce(v, group=self.group)
        return complex(v[0].item(), v[1].item())

    def _local_expval(self, terms, ket):
        """sum_k c_k <local| P(x_k, z_k) |ket> (ket None: the local shard)."""
        if hasattr(self._local, "expval_between"):
            return self._local.expval_between(terms, ket)
        from ._lib import check, lib, ptr
        from .device import sum_from_terms
        ds = sum_from_terms(terms)
        out = np.zeros(1, dtype=np.complex128)
        k = self._local if ket is None else ket
        check(lib().qfb_sum_expval(ds.h, self._local._h, k._h, ptr(out)), "expectation value")
        return complex(out[0])

    def direct_op_exp_val(self, qo):
        terms = qo._pauli_terms(applied=True)
        if terms is None:
            raise ValueError("a sharded state takes expectation values of Pauli sums only")
        return self.expval_terms(terms)
