/*
 * qfb.h -- C ABI of the B200 state-vector engine (libqfb.so).
 *
 * Drop-in boundary for QForte's `Computer` (src/qforte/computer.h:22-185) and
 * the pybind11 surface that exposes it (src/qforte/bindings.cc:149-191).  Every
 * entry point takes plain pointers and sizes, returns an int status (QFB_OK = 0)
 * and never throws; qfb_last_error() gives the message of the calling thread's
 * last failure.  The reference maps std::invalid_argument to ValueError and
 * std::runtime_error to RuntimeError; here QFB_EINVAL plays the first role and
 * every other non-zero status the second.
 *
 * Memory: the library owns the device buffers of states and compiled tables;
 * callers own host arrays, which are copied before the call returns.  All work
 * is enqueued on the calling thread's stream (qfb_set_stream, default: the
 * legacy default stream); results that come back to the host (energies, inner
 * products, amplitudes) synchronise that stream.
 *
 * Layout: a state of n qubits is 2^n complex128 amplitudes, interleaved
 * (re, im), basis index i <-> qubit k is bit k of i (qubit_basis.h:27-45).
 */
#ifndef QFB_H
#define QFB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QFB_API __attribute__((visibility("default")))
#else
#define QFB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    QFB_OK = 0,
    QFB_EINVAL = 22,     /* bad argument (reference: std::invalid_argument)  */
    QFB_ENOMEM = 12,     /* device allocation refused                          */
    QFB_EDEVICE = 5,     /* CUDA error                                         */
    QFB_ETIMEDOUT = 110, /* a bounded device wait gave up                      */
    QFB_ENOSYS = 38      /* not supported in this build                        */
};

typedef struct { double re, im; } qfb_complex;

/* Gate kinds. Matrices follow make_gate.cc:18-235; the kind is informational,
 * the kernels act on the matrix exactly as Computer::apply_gate does. */
typedef struct {
    int32_t target;
    int32_t control; /* == target for 1-qubit gates                          */
    qfb_complex mat[4][4]; /* row/col index (control_bit << 1) | target_bit  */
} qfb_gate;

/* One Pauli string in mask form: X on bits of xmask & ~zmask, Z on zmask &
 * ~xmask, Y where both are set.  P|j> = i^ny (-1)^popcount(j & zmask) |j ^ xmask>
 * with ny = popcount(xmask & zmask). */
typedef struct {
    uint64_t xmask;
    uint64_t zmask;
} qfb_pauli;

typedef struct qfb_state_s *qfb_state; /* one (or a batch of) state vector(s) */
typedef struct qfb_sum_s *qfb_sum;     /* device-resident grouped Pauli sum   */
typedef struct qfb_prog_s *qfb_prog;   /* device-resident Pauli-exponential program */

/* ---- library ------------------------------------------------------------ */
QFB_API int qfb_version(void);
QFB_API int qfb_last_error(char *buf, size_t len);
/* Make `stream` (a cudaStream_t) the calling thread's stream; NULL = default. */
QFB_API int qfb_set_stream(void *stream);
QFB_API int qfb_sync(void);
/* Count of kernels this library launched in this process (evidence counter). */
QFB_API int qfb_launch_count(uint64_t *out);
/* How long a gate tile waits for its bulk load copies before it gives up,
 * flags the failure and leaves its tile unwritten (reported as QFB_ETIMEDOUT
 * by the next qfb_sync or state download).  Default 2 s; at most 60 s; 0
 * gives up without waiting, which lets a test exercise that path with no
 * fault.  No counterpart in the reference (its CPU loops never wait). */
QFB_API int qfb_set_tile_wait_limit(uint64_t ns);

/* ---- states: Computer::Computer / copy ctor / reset / null_state ----------
 * computer.cc:28-54, computer.h:28.  nbatch > 1 holds nbatch independent
 * states of the same size back to back (batched evaluation). */
QFB_API int qfb_state_create(int nqubit, int nbatch, qfb_state *out);
QFB_API int qfb_state_destroy(qfb_state s);
QFB_API int qfb_state_info(qfb_state s, int *nqubit, int *nbatch);
QFB_API void *qfb_state_device_ptr(qfb_state s);
/* dst <- src (same shape).  Computer(const Computer&). */
QFB_API int qfb_state_copy(qfb_state dst, qfb_state src);
/* batch slot `dst_b` of dst <- slot `src_b` of src. */
QFB_API int qfb_state_copy_slot(qfb_state dst, int dst_b, qfb_state src, int src_b);
/* |0...0> in every slot (Computer::reset, computer.cc:51-54). */
QFB_API int qfb_state_reset(qfb_state s);
/* all zero (Computer::null_state, computer.cc:49). */
QFB_API int qfb_state_null(qfb_state s);
/* zero, then amplitude `value` at each listed basis index, slot b
 * (Computer::set_state, computer.cc:42-47). */
QFB_API int qfb_state_set_basis(qfb_state s, int b, const uint64_t *index, const qfb_complex *value,
                        int64_t n);
/* host <-> device copies of slot b (set_coeff_vec / get_coeff_vec,
 * computer.h:112,132; bindings.cc:176-182). */
QFB_API int qfb_state_upload(qfb_state s, int b, const qfb_complex *host, uint64_t n);
QFB_API int qfb_state_download(qfb_state s, int b, qfb_complex *host, uint64_t n);
QFB_API int qfb_state_get_amp(qfb_state s, int b, uint64_t index, qfb_complex *out);

/* nshots basis indices sampled from |c_i|^2 of slot b (the draws of
 * Computer::measure_circuit / measure_readouts / measure_z_readouts_fast,
 * computer.cc:135-315, which use an unseeded std::discrete_distribution).
 * Seeded and reproducible: weights trunc(|c_i|^2 2^56) with |c_i|^2 = re*re +
 * im*im rounded as written, draw k = the smallest i whose inclusive weight
 * prefix exceeds floor(u_k T / 2^64), T the weight total and u_k the k-th
 * output of SplitMix64 seeded with `seed`; equal seeds give equal indices on
 * any device and in a CPU restatement.  The squared norm must be below 1.5
 * (QFB_EINVAL otherwise); amplitudes with |c|^2 < 2^-56 are never drawn. */
QFB_API int qfb_state_sample(qfb_state s, int b, uint64_t seed, int64_t nshots, uint64_t *out);

/* ---- gates: Computer::apply_circuit / apply_gate ---------------------------
 * computer.cc:93-114, :340-751.  The result is that of applying the gates one
 * by one in list order.  Runs of gates whose qubits fit in one set of
 * tile_bits qubits are applied together to shared-memory tiles of the state
 * (one read and one write of the state per run); gates on disjoint qubits may
 * move between runs, which reorders only commuting operations. */
QFB_API int qfb_apply_gates(qfb_state s, const qfb_gate *gates, int64_t ngates);
/* Tile shape of the gate runs, process-wide: tile_bits qubits per tile (0: the
 * default of 10; at most 12; -1: one full-state pass per gate, as the
 * reference does), always including the lowest max(low_bits, 3) qubits
 * (default 3).  Within a tile, each thread holds 2^R amplitudes in registers
 * (R between 2 and 4, qfb_gates_regs) and the run is applied in phases that
 * each fix R mixing qubits.  No counterpart in the reference; set by the
 * autotuner. */
QFB_API int qfb_gates_config(int tile_bits, int low_bits);
/* ---- complex64 states: throughput only -------------------------------------
 * A state of 2^n complex64 amplitudes (interleaved float re, im) for the
 * complex64 variant of the gate sweep.  Gates are applied as for complex128
 * states (the same planning, register-blocked tile runs and one-gate passes)
 * with FP32 arithmetic; never used for parity with the reference, whose
 * Computer is complex128 only.  No counterpart in the reference. */
typedef struct qfb_state_c64_s *qfb_state_c64;
QFB_API int qfb_c64_create(int nqubit, qfb_state_c64 *out); /* |0...0> */
QFB_API int qfb_c64_destroy(qfb_state_c64 s);
QFB_API int qfb_c64_reset(qfb_state_c64 s);
QFB_API int qfb_c64_upload(qfb_state_c64 s, const float *host, uint64_t n);
QFB_API int qfb_c64_download(qfb_state_c64 s, float *host, uint64_t n);
QFB_API int qfb_c64_apply_gates(qfb_state_c64 s, const qfb_gate *gates, int64_t ngates);
/* sum of |amplitude|^2, accumulated in FP64 */
QFB_API int qfb_c64_norm2(qfb_state_c64 s, double *out);

/* Dense blocks on the FP64 tensor cores, process-wide: k = 5 or 6 makes
 * qfb_apply_gates fuse each run of gates on at most k qubits into one 2^k x 2^k
 * unitary (the product of the gates as Computer::apply_gate applies them,
 * computer.cc:340-751) and apply it in one pass with mma.sync FP64; 0 (the
 * default) keeps the register-blocked tile runs.  States of fewer than 10
 * qubits always take the tile runs.  Replaces dense runs of apply_1qubit_gate
 * / apply_2qubit_gate (computer.cc:340-425, :458-751); set by the autotuner. */
QFB_API int qfb_gates_dense(int k);
/* Register bits R per thread of the gate tiles, process-wide (0: the default
 * of 3; always clamped so a tile has at most 256 threads and at least 4).  No
 * counterpart in the reference; set by the autotuner. */
QFB_API int qfb_gates_regs(int reg_bits);
/* Form of the tile phases, process-wide: 1 applies each phase (of 3 register
 * bits, in tiles of 256 amplitudes and more) as a few 8 x 8 matrices on the
 * FP64 tensor cores (mma.sync), the product of its gates, one per assignment
 * of the thread bits its controls test, and one factor per amplitude vector
 * (complex64 states widened to FP64 for the products); 0 applies the phase's
 * gates one by one; 2 (the default) is 1 for states of 128 MiB and more
 * (larger than L2) and 0 below.
 * Both forms give the result of the gates in list order (up to the rounding
 * of the fused products).  No counterpart in the reference; set by the
 * autotuner. */
QFB_API int qfb_gates_fused(int mode);
/* Host only: the fused form of the tile runs qfb_apply_gates would apply to
 * one nqubit state (complex64 != 0: a complex64 state) under the current tile
 * shape, each phase checked as the device reads it (thread tables: every
 * thread-bit assignment once, offsets in the tile; segments: variant bits on
 * thread bits, shared by the 8 vectors of each n-block; matrices in range).
 * Returns QFB_EINVAL on a failed check; else the fused phases, their
 * segments and matrix entries.  No counterpart in the reference. */
QFB_API int qfb_gates_fused_plan(const qfb_gate *gates, int64_t ngates, int nqubit, int complex64,
                                 int64_t *phases, int64_t *segments, int64_t *entries);
/* Host only: how qfb_apply_gates would apply these gates to one nqubit state
 * under the current tile shape: the number of tile runs, of one-gate passes,
 * and the bytes those passes read and write (a run 32 * 2^n; a one-gate pass
 * only the amplitudes its case touches).  No counterpart in the reference. */
QFB_API int qfb_gates_plan(const qfb_gate *gates, int64_t ngates, int nqubit, int64_t *windows,
                           int64_t *single_passes, double *pass_bytes);
/* Host only: the register phases of those tile runs (shared-memory round
 * trips of the tile) and the gate operations they hold.  No counterpart in
 * the reference. */
QFB_API int qfb_gates_phases(const qfb_gate *gates, int64_t ngates, int nqubit, int64_t *phases,
                             int64_t *ops);

/* ---- scalars and inner products -------------------------------------------
 * apply_constant computer.cc:130-133; dot computer.cc:975-980. */
QFB_API int qfb_scale(qfb_state s, qfb_complex a);
/* out[b] = <a_b | b_b> for every slot. */
QFB_API int qfb_vdot(qfb_state a, qfb_state b, qfb_complex *out);
/* y <- y + alpha * x (same shape). */
QFB_API int qfb_axpy(qfb_state y, qfb_complex alpha, qfb_state x);

/* ---- grouped Pauli sums (QubitOperator of Pauli circuits) ------------------
 * Terms are grouped by xmask on the device so one read of the (j, j^x) pairs
 * serves every term of a group.  `segment` gives, per term, the index of the
 * result it contributes to (0 for a plain operator; the pool index for a
 * pool of operators); nsegment results come back from qfb_sum_expval. */
QFB_API int qfb_sum_create(const qfb_pauli *paulis, const qfb_complex *coeffs, const int32_t *segment,
                   int64_t nterms, int32_t nsegment, qfb_sum *out);
QFB_API int qfb_sum_destroy(qfb_sum h);
QFB_API int qfb_sum_info(qfb_sum h, int64_t *nterms, int64_t *ngroups, int32_t *nsegment);
/* out[b * nsegment + g] = <bra_b | O_g | ket_b>.  bra may equal ket
 * (direct_op_exp_val computer.cc:753-771, direct_oppl_exp_val :773-782). */
QFB_API int qfb_sum_expval(qfb_sum h, qfb_state bra, qfb_state ket, qfb_complex *out);
/* The same expectation values as qfb_sum_expval, computed without allocating
 * any device memory.  No counterpart in the reference.  It serves callers that
 * must not allocate on the device while they run: a request loop that admits
 * work against a fixed HBM budget and has to keep its footprint constant from
 * call to call, or code running where every free byte may be held by other
 * work, so that an allocation could fail or stall.  Its reduction scratch is a
 * fixed 65,536-entry complex128 array (1 MiB) inside the library, held by every
 * GPU that loads the library until the process exits; the first call on each
 * device looks up that array's device address.  Limit: nbatch * (number of
 * x-groups) + nbatch * nsegment <= 65,536, otherwise QFB_EINVAL.  All calls
 * share the array, so calls whose kernels overlap on the GPU (different
 * streams or host threads at the same time) race on it; the caller orders
 * them.  Results are copied to `out` and the calling thread's stream is
 * synchronised. */
QFB_API int qfb_sum_expval_noalloc(qfb_sum h, qfb_state bra, qfb_state ket, qfb_complex *out);
/* dst <- O src, all segments summed (apply_operator computer.cc:80-91). */
QFB_API int qfb_sum_apply(qfb_sum h, qfb_state dst, qfb_state src);

/* ---- Pauli-exponential programs (dUCC / ADAPT ansatz) ----------------------
 * The program is the ordered list of exp(i phi_k P_k); phi_k =
 * scale[k] * params[param[k]] (so one compiled program serves every
 * amplitude vector).  Consecutive strings sharing an xmask run in one pass.
 * Replaces exponentiate_pauli_string + trotterize (utils/exponentiate.py:9-87,
 * utils/trotterization.py:10-57) followed by Computer::apply_circuit. */
QFB_API int qfb_prog_create(const qfb_pauli *paulis, const double *scale, const int32_t *param,
                    int64_t nstrings, int32_t nparam, qfb_prog *out);
QFB_API int qfb_prog_destroy(qfb_prog p);
QFB_API int qfb_prog_info(qfb_prog p, int64_t *nstrings, int64_t *nsteps, int32_t *nparam);
/* Apply the program to every slot; params is [nbatch][nparam] (a single row
 * is broadcast when nrows == 1).  sign = +1 applies U, -1 applies U^dagger
 * (the strings in reverse order with negated angles). */
QFB_API int qfb_prog_apply(qfb_prog p, qfb_state s, const double *params, int32_t nrows, int32_t sign);

/* ---- adjoint dUCC gradient (UCCVQE.measure_gradient, uccvqeabc.py:122-251) --
 * psi holds U(t)|ref>, sigma holds H psi.  `kprog` lists, per parameter mu,
 * the strings of K_mu with scale = the imaginary parts of K_mu's JW
 * coefficients (param[k] = mu); grad[b][mu] = 2 Re <sigma|K_mu|psi_mu>.
 * `uprog` is the program whose parameter-mu strings, reversed with negated
 * angles, un-apply U_mu between steps: K itself for particle-hole pools
 * (uccvqeabc.py:228-230), the forward ansatz program for spin-adapted ones,
 * whose U_mu is the product of its component excitations (:208-224).  psi
 * and sigma are consumed (un-rotated back towards the reference). */
QFB_API int qfb_ucc_gradient(qfb_prog kprog, qfb_prog uprog, qfb_state psi, qfb_state sigma,
                             const double *params, int32_t nrows, double *grad);

/* ---- compiled dUCC evaluator (batched, CUDA-graph captured) ----------------
 * One object per (ansatz, Hamiltonian, batch size): it owns nbatch psi and
 * sigma states, a device parameter block [nbatch][nparam], device outputs
 * energy[nbatch] and grad[nbatch][nparam], and every scratch buffer its
 * reductions need, so a run allocates nothing and synchronises nothing and
 * can be captured once into a CUDA graph and replayed.  A run computes, per
 * slot b: psi_b = U(t_b)|ref>, sigma_b = H psi_b, energy[b] = <psi_b|sigma_b>
 * and (with_grad) the adjoint gradient of UCCVQE.measure_gradient
 * (uccvqeabc.py:122-251) with kprog / uprog as for qfb_ucc_gradient.  kprog
 * and uprog may be NULL when no gradient is wanted. */
typedef struct qfb_ucc_s *qfb_ucc;
QFB_API int qfb_ucc_create(qfb_prog fprog, qfb_prog kprog, qfb_prog uprog, qfb_sum ham,
                           int nqubit, uint64_t ref_index, int nbatch, qfb_ucc *out);
QFB_API int qfb_ucc_destroy(qfb_ucc u);
/* Size of the particle-number sector the evaluator works in (0: the full
 * space).  When every step of every program keeps the reference's numbers of
 * alpha (even) and beta (odd) bits, psi stays in that sector and sigma = H psi
 * is formed on its indices only (sigma is zero elsewhere); the energy and
 * gradient equal the full-space ones.  No counterpart in the reference, whose
 * Computer::apply_operator (computer.cc:80-91) always runs over all 2^n
 * amplitudes. */
QFB_API int qfb_ucc_sector(qfb_ucc u, int64_t *nsec);
/* How the evaluator runs: 0 full space; 1 full-space states with sigma formed
 * on the sector; 2 compact sector states, one CTA per parameter set holding
 * psi and sigma in shared memory (sectors up to 6,400 amplitudes); 3 compact
 * sector states in global memory, slot-minor (larger sectors; sigma from
 * stored H rows up to 24 GB of them, else from the grouped terms).  Paths 2
 * and 3 need every program step in Givens form.  No counterpart in the
 * reference. */
QFB_API int qfb_ucc_path(qfb_ucc u, int32_t *path);
/* 1 when the evaluator's compact states are stored as real doubles (see
 * qfb_ucc_config), else 0.  No counterpart in the reference. */
QFB_API int qfb_ucc_real_states(qfb_ucc u, int32_t *real);
/* Parameter sets one CTA of the compact shared-memory forward program holds:
 * 2 with real states (two sets in one 16-byte slot per amplitude), 1
 * otherwise, 0 off the compact shared-memory path.  No counterpart in the
 * reference. */
QFB_API int qfb_ucc_sets_per_cta(qfb_ucc u, int32_t *sets);
/* Entries of the H rows the compact path streams for each parameter set (0
 * on the other paths).  No counterpart in the reference. */
QFB_API int qfb_ucc_rows(qfb_ucc u, int64_t *nnz);
/* Process-wide: whether evaluators created from now on may use the compact
 * sector paths (1, the default: shared memory when the sector fits, else
 * global memory), only the global-memory one (2), only the global-memory one
 * with sigma formed from the grouped terms instead of stored H rows (3; the
 * rows are over 24 GB beyond ~24 qubits, where this happens by itself), 1
 * or 2 with complex state storage (4, 5), 1 with one real parameter set per
 * CTA in the shared-memory forward program instead of two (6), or neither (0).  Otherwise a
 * compact evaluator whose H and step coefficients are all real keeps psi and
 * sigma as real doubles (half the memory and traffic).  No counterpart in the
 * reference. */
QFB_API int qfb_ucc_config(int compact);
/* Process-wide tile shape of the full-space windows of evaluators created
 * from now on: fwd_bits qubits per forward tile (default 12, at most 13),
 * grad_bits per two-state gradient tile (default 11, at most 12), always
 * including the lowest low_bits qubits (default 3).  Set by the autotuner.
 * No counterpart in the reference. */
QFB_API int qfb_ucc_tiles(int fwd_bits, int grad_bits, int low_bits);
/* Device bytes the evaluator holds (states, parameter and output blocks,
 * scratch); a request loop admits work against its HBM budget with this.  No
 * counterpart in the reference. */
QFB_API int qfb_ucc_memory(qfb_ucc u, uint64_t *bytes);
/* ADAPT pool gradients (UCCVQE.measure_gradient3, uccvqeabc.py:253-283): give
 * the evaluator a pool program (the pool operators' K strings, one parameter
 * per operator, as for kprog); a run of mode 3 then computes psi, sigma, the
 * energy and 2 Re <sigma|K_k|psi> for every pool operator k of every slot into
 * a device block [nbatch][npool] (qfb_ucc_pool_buffer), in one graph launch
 * when captured.  The pool's steps must be in Givens form. */
QFB_API int qfb_ucc_set_pool(qfb_ucc u, qfb_prog pool);
QFB_API int qfb_ucc_pool_buffer(qfb_ucc u, double **d_pool_grad);
/* Host convenience: params in, energies and pool gradients out, synchronous. */
QFB_API int qfb_ucc_eval_pool(qfb_ucc u, const double *params, double *energy, double *pool_grad);
/* PQE residuals (UCCNPQE.get_residual_vector, uccnpqe.py:249-292): give the
 * evaluator n excited determinants I_k (full-space basis indices) and their
 * phase factors (uccnpqe.py:193-247); a run of mode 4 then computes psi,
 * sigma = H psi, the energy and res[b][k] = Re(<I_k|U^dagger H U|ref> *
 * phase_k) into a device block [nbatch][n] (qfb_ucc_residual_buffer), in one
 * graph launch when captured.  U^dagger is the ansatz program in reverse with
 * negated angles, applied to sigma (which the run consumes). */
QFB_API int qfb_ucc_set_residuals(qfb_ucc u, const uint64_t *dets, const qfb_complex *phases,
                                  int32_t n);
QFB_API int qfb_ucc_residual_buffer(qfb_ucc u, double **d_res);
/* Host convenience: params in, energies and residuals out, synchronous. */
QFB_API int qfb_ucc_eval_residuals(qfb_ucc u, const double *params, double *energy, double *res);
/* Device addresses of the parameter block and the outputs. */
QFB_API int qfb_ucc_buffers(qfb_ucc u, double **d_params, double **d_energy, double **d_grad);
/* Enqueue one evaluation on the calling thread's stream (replays the
 * captured graph when one exists for this mode).  with_grad: 0 energy only;
 * 1 energy and gradient; 2 the gradient sweep alone, on the psi and sigma a
 * preceding with_grad = 0 run left (the sweep un-rotates them in place, so a
 * second mode-2 run needs a new mode-0 run first); 3 energy and the pool
 * gradients (qfb_ucc_set_pool); 4 energy and the PQE residuals
 * (qfb_ucc_set_residuals). */
QFB_API int qfb_ucc_run(qfb_ucc u, int with_grad);
/* Capture one evaluation of the given mode into a CUDA graph (replayed by
 * later runs). */
QFB_API int qfb_ucc_capture(qfb_ucc u, int with_grad);
/* Host convenience: params in, energies (and gradients) out, synchronous. */
QFB_API int qfb_ucc_eval(qfb_ucc u, const double *params, double *energy, double *grad);
/* Instrumented runs: `reps` evaluations enqueued stage by stage with CUDA
 * events between the stages; returns the mean milliseconds and the kernel
 * launches of each stage: [0] reference state, [1] U(t) program, [2] H psi and
 * energy, [3] gradient sweep. */
QFB_API int qfb_ucc_profile(qfb_ucc u, int with_grad, int reps, double *stage_ms,
                            int64_t *stage_launches);

/* ---- packed evaluations of several problems (serving) ---------------------
 * A pack gathers the compact-sector evaluators of several dUCC problems (each
 * qfb_ucc_path == 2: states of up to ~16 qubits held in shared memory, all
 * with the same state storage, qfb_ucc_real_states) so that parameter sets of
 * different problems run in ONE launch: item i evaluates params[i][0..nparam)
 * of member items[i].member, energy into energy[i] and, when items[i].grad is
 * set, the adjoint gradient into grad[i][0..nparam) (row stride maxparam).
 * One CTA per item runs the whole evaluation in shared memory: the forward
 * program, sigma = H psi, the energy, the reverse sweep and the per-parameter
 * sums (energy_feval / measure_gradient, algorithm.py:458-474,
 * uccvqeabc.py:122-251).  The members must outlive the pack.  No counterpart
 * in the reference (its Computer evaluates one problem per call). */
typedef struct qfb_pack_s *qfb_pack;
QFB_API int qfb_pack_create(const qfb_ucc *members, int nmembers, int capacity, qfb_pack *out);
QFB_API int qfb_pack_destroy(qfb_pack p);
QFB_API int qfb_pack_info(qfb_pack p, int32_t *capacity, int32_t *maxparam, uint64_t *bytes);
/* Device blocks: items [capacity][2] int32 (member, grad), params and grad
 * [capacity][maxparam], energy [capacity]. */
QFB_API int qfb_pack_buffers(qfb_pack p, int32_t **items, double **params, double **energy,
                             double **grad);
/* Enqueue the first nitems items of the device blocks on the calling thread's
 * stream (an item naming no member gets a NaN energy). */
QFB_API int qfb_pack_launch(qfb_pack p, int nitems);
/* Host arrays in and out, synchronising: member[i], with_grad[i] (may be
 * NULL: energies only), params [nitems][maxparam], energy [nitems], grad
 * [nitems][maxparam] (may be NULL when no item asks for a gradient). */
QFB_API int qfb_pack_run(qfb_pack p, const int32_t *member, const int32_t *with_grad, int nitems,
                         const double *params, double *energy, double *grad);


#ifdef __cplusplus
}
#endif

#endif /* QFB_H */
