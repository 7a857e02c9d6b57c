// Gate runs on register-blocked shared-memory tiles (Computer::apply_circuit,
// computer.cc:93-114, with the per-gate case analysis of computer.cc:340-751).
//
// A run is a list of gates whose qubits all lie in one set Q of b qubits (Q
// always holds qubits 0..2, so a tile is 2^(b-3) chunks of 8 contiguous
// amplitudes = 128 bytes).  One CTA owns one tile of 2^b amplitudes:
//
//   1. the tile's chunks are copied from HBM into shared memory by the bulk
//      copy engine (cp.async.bulk, completion on an mbarrier);
//   2. the run is split on the host into phases.  A phase fixes R "register
//      bits" of the tile; each thread loads the 2^R amplitudes that differ in
//      those bits into registers, applies every gate of the phase there, and
//      writes them back.  A gate needs its mixing bits (the target of a
//      non-diagonal 2x2 block, both bits of a 4x4 matrix) among the register
//      bits; diagonal factors and controls may sit on any tile bit, the
//      thread's own bits decide them;
//   3. the tile goes back to HBM by bulk copies.
//
// Shared-memory layout: element l of the tile sits at tpad(l) = l + (l>>3) +
// (l>>6) + (l>>9) + (l>>12) (16-byte units).  tpad is additive over disjoint
// bit sets, keeps each 8-element chunk contiguous (one bulk copy), and gives
// tile bit p the bank step 2^(p mod 3) (in 16-byte bank groups): a quarter warp
// of 128-bit accesses is conflict-free when the three lowest thread bits come
// from the three residue classes of p mod 3, which the host arranges.
#pragma once

#include "qfb_common.cuh"

namespace qfbt {

constexpr int kMaxTileBits = 12;
constexpr int kMaxThreadBits = 8;  // up to 256 threads per tile
constexpr int kMaxRegBits = 4;

enum : int32_t {
    OP_DENSE = 0,  // complex 2x2 on register bit t
    OP_REAL,       // 2x2 with real entries
    OP_RXI,        // real diagonal, imaginary off-diagonal
    OP_PSWAP,      // exchange of the pair (the reference's op_0_1 == op_1_0 case)
    OP_ANTI,       // anti-diagonal b, c
    OP_DIAG,       // diagonal factors a (bit 0) / d (bit 1) where dset says
    OP_GEN4,       // generic 4x4 on register bits t (low) and c (high index bit)
    OP_BSWAP       // SWAP of register bits t and c
};

constexpr uint32_t OPC_DIAG = 20, OPC_DIAG_THREAD = 32, OPC_GEN4 = 33, OPC_BSWAP = 49;

// One gate operation of a phase.  `opc` selects the arithmetic and the
// register position of its bit(s) at once (one jump table):
//    0..19  2x2 kinds DENSE, REAL, RXI, PSWAP, ANTI on register bit t: 4 * kind + t
//   20..31  OP_DIAG on register bit t: 20 + 4 * (dset - 1) + t
//       32  OP_DIAG on a thread bit (tbit)
//   33..48  OP_GEN4 on register bits t, c: 33 + 4 * t + c
//   49..64  OP_BSWAP of register bits t, c: 49 + 4 * t + c
// dset: bit0 factor a where the bit is 0, bit1 factor d where it is 1 (entries
// equal to 1 are skipped).
struct TOp {
    uint32_t opc;
    uint32_t tctl;  // tile bits of the thread part that must be 1 (control)
    uint32_t tbit;  // OP_DIAG on a thread bit: that tile bit's mask
    uint32_t aux;   // 2x2 kinds and OP_DIAG: cm | cv << 16, a control on register
                    // bits (registers k with k & cm == cv); OP_DIAG on a thread bit:
                    // the same | dset << 8; OP_GEN4: first of its 16 matrix entries
    double2 m[4];   // a, b, c, d
};
static_assert(sizeof(TOp) == 80, "TOp layout");

struct TPhase {
    uint32_t roff[1 << kMaxRegBits];  // load: tpad offset of register k's tile bits
    uint32_t soff[1 << kMaxRegBits];  // store: the same after the phase's relabelings
    int32_t o0, no;                   // ops of this phase
    int32_t th0;                      // this phase's entries of the thread table
    int32_t nm;                       // fused form: matrix entries of its segments
    int32_t s0, ns;                   // fused form: segments of this phase
    int32_t sc;                       // fused form: per-thread factor table (-1: none)
    int32_t m0;                       // fused form: first matrix entry of its segments
};
static_assert(sizeof(TPhase) == 160, "TPhase layout");

// The fused form of a phase (tiles with R = 3 and at least 32 threads; the
// products in FP64 also for complex64 tiles): the phase's ops, in order,
// become a few segments, each one 8 x 8 matrix on the 8 register amplitudes,
// applied on the FP64 tensor cores.
//  * Vector t of the phase (the 8 amplitudes at tile offsets base(t) +
//    roff[k], base from entry t of the thread table) is processed by warp
//    t / 32 as column t % 8 of n-block (t / 8) % 4: per n-block the warp
//    computes Y = M X with mma.sync.m8n8k4 FP64 (k-blocks of registers 0-3
//    and 4-7; real and imaginary parts as four real products), B fragments
//    read straight from the tile, D fragments stored straight back.
//  * The matrix of a segment depends on the vector only through its variant
//    bits (the tile bits of the thread part that its ops test: controls on
//    thread bits, the bit of a diagonal on a thread bit that is also
//    controlled by register bits), at most kMaxVarBits of them; the host
//    builds one matrix per assignment of those bits and orders the thread
//    table so that the phase's variant bits are vector-index bits 3 and up:
//    all 8 columns of an n-block share one matrix.
//  * Diagonal factors that depend on thread bits alone (a diagonal on a
//    thread bit, controlled by thread bits or not at all) scale all 8
//    amplitudes of a vector alike and commute with everything else in the
//    phase: their product, per vector, is one table entry (applied on load).
// Variant index: bit j is tile bit (dsel >> 4j) & 15 of the vector; matrix of
// variant x at m0 + 64 x, in A-fragment order: entry 32 kb + lane holds
// (Re, Im) of M[lane / 4][4 kb + lane % 4].
// A warp reads its A fragments straight from the matrix pool (each lane its
// own entry: one coalesced 512-byte load per fragment, L1-resident across the
// tiles of a run); a phase's thread table is copied into one of two
// shared-memory buffers before the barrier that precedes the phase.  The host
// splits a phase whose segments hold more than kStage matrix entries into
// phases on the same registers.
constexpr int kMaxVarBits = 3;
constexpr int kStage = 512;  // matrix entries of one phase
struct TSeg {
    uint32_t m0;    // first entry of this segment's matrices
    uint32_t dsel;  // variant bits: tile bit positions, 4 bits each
    uint32_t mm;    // register bits the matrix mixes (host statistics)
    uint32_t nd;    // number of variant bits
};
static_assert(sizeof(TSeg) == 16, "TSeg layout");
// thread table entry of thread tid in a phase: tl | tpad(tl) << 16, with tl
// the thread's tile bits (the phase's non-register bits set from tid)

struct TRun {
    uint64_t qmask;  // qubits of the tile (tile bit i = the i-th lowest)
    int32_t b;       // tile bits
    int32_t ch0;     // first entry of this run's chunk table
    int32_t p0, np;  // phases
};
// chunk table entry c of a run: the global offset of the tile's chunk c
// (8 amplitudes on qubits 0..2), i.e. c's bits placed on the tile's qubits
// above 2

__host__ __device__ __forceinline__ uint32_t tpad(uint32_t l) {
    return l + (l >> 3) + (l >> 6) + (l >> 9) + (l >> 12);
}

// Elements (16 bytes) a padded tile of 2^b amplitudes occupies.
__host__ __device__ __forceinline__ uint32_t tpad_size(int b) { return tpad((1u << b) - 1u) + 1u; }

// The same layout for 8-byte (complex64) elements: two elements of padding
// where complex128 has one, so every 8-element chunk still starts on a
// 16-byte boundary (the bulk copies need it) and stays contiguous.
__host__ __device__ __forceinline__ uint32_t tpad8(uint32_t l) { return 2u * tpad(l) - l; }
__host__ __device__ __forceinline__ uint32_t tpad8_size(int b) { return tpad8((1u << b) - 1u) + 2u; }

// ---- PTX helpers: mbarrier and bulk copies ---------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of the mbarrier, giving up after `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit_and_wait() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16-byte asynchronous global -> shared copy (L2 only) and its group waits.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ---- gate arithmetic on the registers --------------------------------------
// Register positions are template parameters, so every register index below
// is a compile-time constant and the amplitudes stay in registers; the host
// encodes (position, control) pairs and one switch picks the instantiation.

// f(x0, x1) on every pair (k, k | 2^T) of registers with k & cm == cv (a
// control on register bits, uniform across the CTA; cm = 0: every pair).
template <int R, int T, class F, class A>
__device__ __forceinline__ void for_pairs(A (&v)[1 << R], uint32_t cm, uint32_t cv, const F &f) {
    if constexpr (T < R) {
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
            if (k & (1 << T)) continue;
            if (((uint32_t)k & cm) == cv) f(v[k], v[k | (1 << T)]);
        }
    }
}

template <class A>
struct FDense {  // complex 2x2
    A a, b, c, d;
    __device__ __forceinline__ void operator()(A &x0, A &x1) const {
        const A y0 = c_add(c_mul(a, x0), c_mul(b, x1));
        x1 = c_add(c_mul(c, x0), c_mul(d, x1));
        x0 = y0;
    }
};
template <class A>
struct FReal {  // real 2x2
    typename AmpT<A>::S a, b, c, d;
    __device__ __forceinline__ void operator()(A &x0, A &x1) const {
        const A y0 = AmpT<A>::make(a * x0.x + b * x1.x, a * x0.y + b * x1.y);
        x1 = AmpT<A>::make(c * x0.x + d * x1.x, c * x0.y + d * x1.y);
        x0 = y0;
    }
};
template <class A>
struct FRxi {  // a, d real; b = i bi, c = i ci
    typename AmpT<A>::S a, bi, ci, d;
    __device__ __forceinline__ void operator()(A &x0, A &x1) const {
        const A y0 = AmpT<A>::make(a * x0.x - bi * x1.y, a * x0.y + bi * x1.x);
        x1 = AmpT<A>::make(d * x1.x - ci * x0.y, d * x1.y + ci * x0.x);
        x0 = y0;
    }
};
struct FPswap {
    template <class A>
    __device__ __forceinline__ void operator()(A &x0, A &x1) const {
        const A t = x0;
        x0 = x1;
        x1 = t;
    }
};
template <class A>
struct FAnti {
    A b, c;
    __device__ __forceinline__ void operator()(A &x0, A &x1) const {
        const A t = x0;
        x0 = c_mul(b, x1);
        x1 = c_mul(c, t);
    }
};

// diagonal on register bit T: a where the bit is 0 (DS & 1), d where it is 1
// (DS & 2), on the registers with k & cm == cv
template <int R, int T, int DS, class A>
__device__ __forceinline__ void ap_diag(A (&v)[1 << R], uint32_t cm, uint32_t cv, A a, A d) {
    if constexpr (T < R) {
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
            if (((uint32_t)k & cm) != cv) continue;
            if (k & (1 << T)) {
                if constexpr ((DS & 2) != 0) v[k] = c_mul(d, v[k]);
            } else {
                if constexpr ((DS & 1) != 0) v[k] = c_mul(a, v[k]);
            }
        }
    }
}

// one factor on the registers with k & cm == cv
template <int R, class A>
__device__ __forceinline__ void ap_scale(A (&v)[1 << R], uint32_t cm, uint32_t cv, A f) {
#pragma unroll
    for (int k = 0; k < (1 << R); ++k)
        if (((uint32_t)k & cm) == cv) v[k] = c_mul(f, v[k]);
}

// A read-only load the compiler keeps in place (not hoisted out of the
// unrolled loops below, where 16 hoisted complex entries would spill).
__device__ __forceinline__ double2 ld_entry(const double2 *p) {
    double2 r;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
    return r;
}

// Matrix index (bit C << 1) | bit T; each output is the sum over the inputs
// in column order.  The host zeroes the entries the reference skips (|m| <=
// 1e-16, computer.cc:721-750), so their products add exact zeros.
template <int R, int T, int C, class A>
__device__ __forceinline__ void ap_gen4(A (&v)[1 << R], const double2 *__restrict__ m) {
    if constexpr (T < R && C < R && T != C) {
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
            if (k & ((1 << T) | (1 << C))) continue;
            const int i0 = k, i1 = k | (1 << T), i2 = k | (1 << C), i3 = k | (1 << T) | (1 << C);
            A y[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const A m0 = AmpT<A>::cvt(ld_entry(m + 4 * i)),
                        m1 = AmpT<A>::cvt(ld_entry(m + 4 * i + 1)),
                        m2 = AmpT<A>::cvt(ld_entry(m + 4 * i + 2)),
                        m3 = AmpT<A>::cvt(ld_entry(m + 4 * i + 3));
                y[i] = c_add(c_add(c_add(c_mul(m0, v[i0]), c_mul(m1, v[i1])), c_mul(m2, v[i2])),
                             c_mul(m3, v[i3]));
            }
            v[i0] = y[0];
            v[i1] = y[1];
            v[i2] = y[2];
            v[i3] = y[3];
        }
    }
}

// SWAP of register bits T and C
template <int R, int T, int C, class A>
__device__ __forceinline__ void ap_bswap(A (&v)[1 << R]) {
    if constexpr (T < R && C < R && T != C) {
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
            if ((k & (1 << T)) && !(k & (1 << C))) {
                const int k2 = k ^ (1 << T) ^ (1 << C);
                const A x = v[k];
                v[k] = v[k2];
                v[k2] = x;
            }
        }
    }
}

// case lists: (opcode, t) / (opcode, t, c)
#define QFBT_T4(B, X) X(B + 0, 0) X(B + 1, 1) X(B + 2, 2) X(B + 3, 3)
#define QFBT_TT16(B, X) X(B + 0, 0, 0) X(B + 1, 0, 1) X(B + 2, 0, 2) X(B + 3, 0, 3) X(B + 4, 1, 0) X(B + 5, 1, 1) X(B + 6, 1, 2) X(B + 7, 1, 3) X(B + 8, 2, 0) X(B + 9, 2, 1) X(B + 10, 2, 2) X(B + 11, 2, 3) X(B + 12, 3, 0) X(B + 13, 3, 1) X(B + 14, 3, 2) X(B + 15, 3, 3)

template <int R, class A>
__device__ __forceinline__ void apply_op(A (&v)[1 << R], const TOp *__restrict__ op, uint32_t tl,
                                         const double2 *__restrict__ m4) {
    using S = typename AmpT<A>::S;
    auto cv_ = [](double2 z) { return AmpT<A>::cvt(z); };
    const uint4 hdr = __ldg(reinterpret_cast<const uint4 *>(op));
    if ((tl & hdr.y) != hdr.y) return;  // a control on one of the thread's bits is 0
    const uint32_t cm = hdr.w & 0xffu, cv = (hdr.w >> 16) & 0xffu;
    switch (hdr.x) {
#define X(N, T)                                                                            \
    case N:                                                                                \
        for_pairs<R, T>(v, cm, cv,                                                         \
                        FDense<A>{cv_(__ldg(&op->m[0])), cv_(__ldg(&op->m[1])),            \
                                  cv_(__ldg(&op->m[2])), cv_(__ldg(&op->m[3]))});          \
        break;
        QFBT_T4(0, X)
#undef X
#define X(N, T)                                                                            \
    case N:                                                                                \
        for_pairs<R, T>(v, cm, cv,                                                         \
                        FReal<A>{(S)__ldg(&op->m[0].x), (S)__ldg(&op->m[1].x),             \
                                 (S)__ldg(&op->m[2].x), (S)__ldg(&op->m[3].x)});           \
        break;
        QFBT_T4(4, X)
#undef X
#define X(N, T)                                                                            \
    case N:                                                                                \
        for_pairs<R, T>(v, cm, cv,                                                         \
                        FRxi<A>{(S)__ldg(&op->m[0].x), (S)__ldg(&op->m[1].y),              \
                                (S)__ldg(&op->m[2].y), (S)__ldg(&op->m[3].x)});            \
        break;
        QFBT_T4(8, X)
#undef X
#define X(N, T) case N: for_pairs<R, T>(v, cm, cv, FPswap{}); break;
        QFBT_T4(12, X)
#undef X
#define X(N, T) case N: for_pairs<R, T>(v, cm, cv, FAnti<A>{cv_(__ldg(&op->m[1])), cv_(__ldg(&op->m[2]))}); break;
        QFBT_T4(16, X)
#undef X
#define X(N, T) case N: ap_diag<R, T, 1>(v, cm, cv, cv_(__ldg(&op->m[0])), cv_(__ldg(&op->m[3]))); break;
        QFBT_T4(20, X)
#undef X
#define X(N, T) case N: ap_diag<R, T, 2>(v, cm, cv, cv_(__ldg(&op->m[0])), cv_(__ldg(&op->m[3]))); break;
        QFBT_T4(24, X)
#undef X
#define X(N, T) case N: ap_diag<R, T, 3>(v, cm, cv, cv_(__ldg(&op->m[0])), cv_(__ldg(&op->m[3]))); break;
        QFBT_T4(28, X)
#undef X
        case OPC_DIAG_THREAD: {
            // the diagonal bit is one of this thread's bits: one factor for all registers
            const bool one = (tl & hdr.z) != 0;
            if ((hdr.w >> 8) & (one ? 2u : 1u)) ap_scale<R>(v, cm, cv, cv_(__ldg(&op->m[one ? 3 : 0])));
            break;
        }
#define X(N, T, C) case N: ap_gen4<R, T, C>(v, m4 + (int)hdr.w); break;
        QFBT_TT16(33, X)
#undef X
#define X(N, T, C) case N: ap_bswap<R, T, C>(v); break;
        QFBT_TT16(49, X)
#undef X
        default:
            break;
    }
}

// ---- the fused form ---------------------------------------------------------

// D += A B on one 8x8x4 FP64 block (register operands only).
__device__ __forceinline__ void tmma(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// Variant of a vector with tile bits tl for a segment with header h.
__device__ __forceinline__ uint32_t seg_variant(uint32_t tl, const uint4 &h) {
    uint32_t var = 0;
    for (uint32_t j = 0; j < h.w; ++j) var |= ((tl >> ((h.y >> (4 * j)) & 15u)) & 1u) << j;
    return var;
}

// One fused phase on this warp's 32 vectors: its segments in order (each
// reads the vectors at roff and writes them back, the last one at soff).  A:
// the tile's amplitudes (complex128, or complex64 widened to FP64 for the
// products and rounded back on store).
template <class A>
__device__ __forceinline__ void fused_phase(const TPhase *__restrict__ ph, const TSeg *__restrict__ segs,
                                            const double2 *__restrict__ fm, const uint32_t *thr, A *tile) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    const int s0 = __ldg(&ph->s0), ns = __ldg(&ph->ns), sc = __ldg(&ph->sc);
    if (ns == 0) {  // relabelings only: each thread moves its own vector
        A *t0 = tile + (thr[threadIdx.x] >> 16);
        A v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = t0[__ldg(&ph->roff[k])];
        if (sc >= 0) {
            const double2 f = __ldg(fm + sc + threadIdx.x);
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = AmpT<A>::cvt(c_mul(f, AmpT<A>::wide(v[k])));
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) t0[__ldg(&ph->soff[k])] = v[k];
        return;
    }
    const uint32_t ri0 = __ldg(&ph->roff[q]), ri1 = __ldg(&ph->roff[4 + q]);
    const uint32_t ro_mid = __ldg(&ph->roff[g]), ro_last = __ldg(&ph->soff[g]);
    for (int si = 0; si < ns; ++si) {
        const uint4 h = __ldg(reinterpret_cast<const uint4 *>(segs + s0 + si));
        const uint32_t ro = si + 1 == ns ? ro_last : ro_mid;
        const bool scale = si == 0 && sc >= 0;
        const double2 *mseg = fm + h.x;
        double2 a0[2], a1[2];
        // two n-blocks at a time: all their B loads, then 16 mma in four
        // independent chains, then their D stores (n-blocks hold disjoint
        // vectors, so the loads may all precede the stores)
#pragma unroll
        for (int np = 0; np < 4; np += 2) {
            double2 x0[2], x1[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int tv = warp * 32 + (np + u) * 8;  // first vector of the n-block
                if (np + u == 0 || h.w != 0) {
                    const double2 *mv = mseg + 64u * seg_variant(thr[tv] & 0xffffu, h);
                    a0[u] = __ldg(mv + lane);
                    a1[u] = __ldg(mv + 32 + lane);
                } else {
                    a0[u] = a0[0];
                    a1[u] = a1[0];
                }
                // B fragments: registers 4 kb + q of vector tv + g
                const uint32_t bb = thr[tv + g] >> 16;
                x0[u] = AmpT<A>::wide(tile[bb + ri0]);
                x1[u] = AmpT<A>::wide(tile[bb + ri1]);
                if (scale) {
                    const double2 f = __ldg(fm + sc + tv + g);
                    x0[u] = c_mul(f, x0[u]);
                    x1[u] = c_mul(f, x1[u]);
                }
            }
            double dr[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, di[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                tmma(dr[u][0], dr[u][1], a0[u].x, x0[u].x);
                tmma(di[u][0], di[u][1], a0[u].x, x0[u].y);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                tmma(dr[u][0], dr[u][1], a0[u].y, -x0[u].y);
                tmma(di[u][0], di[u][1], a0[u].y, x0[u].x);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                tmma(dr[u][0], dr[u][1], a1[u].x, x1[u].x);
                tmma(di[u][0], di[u][1], a1[u].x, x1[u].y);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                tmma(dr[u][0], dr[u][1], a1[u].y, -x1[u].y);
                tmma(di[u][0], di[u][1], a1[u].y, x1[u].x);
            }
            // D fragments: register g of vectors tv + 2q and tv + 2q + 1 (every
            // lane's B loads completed before the warp-wide mma)
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int tv = warp * 32 + (np + u) * 8;
                tile[(thr[tv + 2 * q] >> 16) + ro] = AmpT<A>::cvt(make_double2(dr[u][0], di[u][0]));
                tile[(thr[tv + 2 * q + 1] >> 16) + ro] = AmpT<A>::cvt(make_double2(dr[u][1], di[u][1]));
            }
        }
        if (si + 1 < ns) __syncwarp();  // the next segment reads what this one wrote
    }
}

// v with a zero bit inserted at every set bit of m (ascending): the bits of
// v placed on the complement of m.
__device__ __forceinline__ uint64_t spread_around(uint64_t v, uint64_t m) {
    while (m) {
        const int p = __ffsll((long long)m) - 1;
        v = insert0(v, p);
        m &= m - 1;
    }
    return v;
}

// Device word set when a bounded wait gave up (read and cleared by the host;
// this header belongs to the one translation unit that launches the kernel).
static __device__ int g_tile_wait_err = 0;

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// How long a tile waits for its load copies before it gives up (default
// kWaitLimitNs; 0: give up without waiting, so a test can make the wait run
// out without any fault).  Only the first wait reads it: the wait that keeps
// the copies in flight from landing after the CTA exits always allows
// kWaitLimitNs.
static __device__ uint64_t g_tile_wait_limit_ns = kWaitLimitNs;

// Offsets in the padded tile for amplitudes of A (the host's tables use the
// same function).
template <class A>
__host__ __device__ __forceinline__ uint32_t tpad_of(uint32_t l) {
    return sizeof(A) == 16 ? tpad(l) : tpad8(l);
}
template <class A>
__host__ __device__ __forceinline__ uint32_t tpad_size_of(int b) {
    return sizeof(A) == 16 ? tpad_size(b) : tpad8_size(b);
}

// One CTA per tile (blockIdx.x: tile position over the qubits outside Q;
// blockIdx.y: batch slot); 2^(b-R) threads, 2^R amplitudes each.  A: double2
// (complex128) or float2 (the complex64 throughput variant, arithmetic in
// FP32); a chunk is 8 amplitudes either way (128 or 64 bytes).
// F: the phases' fused form (segments and per-thread factors in segs / fm)
// instead of their op lists.
template <int R, class A = double2, bool F = false>
__global__ void __launch_bounds__(256, F ? 4 : R == 4 ? 1 : 3)
    k_gate_tile(A *__restrict__ psi, uint64_t nbasis, TRun run,
                const TPhase *__restrict__ phases, const TOp *__restrict__ ops,
                const double2 *__restrict__ m4, const uint64_t *__restrict__ chunks,
                const uint32_t *__restrict__ threads, const TSeg *__restrict__ segs,
                const double2 *__restrict__ fm) {
    extern __shared__ __align__(128) unsigned char t_smem[];
    constexpr uint32_t kChunk = 8u * sizeof(A);
    A *tile = reinterpret_cast<A *>(t_smem);
    const int b = run.b;
    uint64_t *bar = reinterpret_cast<uint64_t *>(tile + tpad_size_of<A>(b));
    const uint32_t bar_a = smem_u32(bar);
    const int tid = threadIdx.x, nth = blockDim.x;
    const int nch = 1 << (b - 3);
    __shared__ uint64_t s_base;
    // fused form: two buffers of a phase's thread table after the barrier word
    constexpr bool kF = F && R == 3;
    uint32_t *sthr = reinterpret_cast<uint32_t *>(
        t_smem + ((sizeof(A) * tpad_size_of<A>(b) + 16 + 15) & ~(size_t)15));
    auto stage = [&](int p) {
        if constexpr (kF)
            sthr[(p & 1) * (1 << kMaxThreadBits) + tid] =
                __ldg(&threads[__ldg(&phases[run.p0 + p].th0) + tid]);
    };

    if (tid == 0) {
        if constexpr (!kF) {
            mbar_init(bar_a, 1);
            mbar_expect_tx(bar_a, (uint32_t)nch * kChunk);
        }
        // tile origin: blockIdx.x's bits on the qubits outside Q, plus the slot
        s_base = (uint64_t)blockIdx.y * nbasis + spread_around(blockIdx.x, run.qmask);
    }
    __syncthreads();
    A *s = psi + s_base;
    const uint64_t *ch = chunks + run.ch0;
    if constexpr (kF) {
        // 16-byte asynchronous copies, PPC consecutive threads per chunk
        constexpr int PPC = (int)kChunk / 16;
        for (int i = tid; i < PPC * nch; i += nth) {
            const int c = i / PPC, e = i % PPC;
            cp_async16(smem_u32(reinterpret_cast<unsigned char *>(tile + tpad_of<A>((uint32_t)c << 3)) + 16 * e),
                       reinterpret_cast<const unsigned char *>(s + __ldg(&ch[c])) + 16 * e);
        }
        cp_async_commit();
        if (run.np > 0) stage(0);
        cp_async_wait_all();
        __syncthreads();  // the tile and phase 0's thread table
        for (int p = 0; p < run.np; ++p) {
            fused_phase<A>(phases + run.p0 + p, segs, fm, sthr + (p & 1) * (1 << kMaxThreadBits), tile);
            if (p + 1 < run.np) stage(p + 1);
            __syncthreads();
        }
        for (int i = tid; i < PPC * nch; i += nth) {
            const int c = i / PPC, e = i % PPC;
            *reinterpret_cast<uint4 *>(reinterpret_cast<unsigned char *>(s + __ldg(&ch[c])) + 16 * e) =
                *reinterpret_cast<const uint4 *>(
                    reinterpret_cast<const unsigned char *>(tile + tpad_of<A>((uint32_t)c << 3)) + 16 * e);
        }
    } else {
        for (int c = tid; c < nch; c += nth)
            bulk_g2s(smem_u32(tile + tpad_of<A>((uint32_t)c << 3)), s + __ldg(&ch[c]), kChunk, bar_a);
        const uint64_t limit = g_tile_wait_limit_ns;
        if (limit == 0 || !mbar_wait_bounded(bar_a, 0, limit)) {
            // the copies did not complete in time: flag it, give them a second
            // bounded wait so none lands after this CTA's shared memory is
            // released, and leave the tile unwritten
            if (tid == 0) atomicExch(&g_tile_wait_err, 1);
            mbar_wait_bounded(bar_a, 0, kWaitLimitNs);
            return;
        }

        for (int p = 0; p < run.np; ++p) {
            const TPhase *ph = phases + run.p0 + p;
            const uint32_t tw = __ldg(&threads[__ldg(&ph->th0) + tid]);
            const uint32_t tl = tw & 0xffffu;
            A *t0 = tile + (tw >> 16);
            A v[1 << R];
#pragma unroll
            for (int k = 0; k < (1 << R); ++k) v[k] = t0[__ldg(&ph->roff[k])];
            const int o0 = __ldg(&ph->o0), o1 = o0 + __ldg(&ph->no);
            for (int o = o0; o < o1; ++o) apply_op<R, A>(v, ops + o, tl, m4);
#pragma unroll
            for (int k = 0; k < (1 << R); ++k) t0[__ldg(&ph->soff[k])] = v[k];
            if (p + 1 < run.np) __syncthreads();
        }
        fence_async_smem();
        __syncthreads();
        for (int c = tid; c < nch; c += nth)
            bulk_s2g(s + __ldg(&ch[c]), smem_u32(tile + tpad_of<A>((uint32_t)c << 3)), kChunk);
        bulk_commit_and_wait();
    }
}

}  // namespace qfbt
