// Compact particle-number sector evaluator.
//
// When every step of a dUCC evaluator's programs keeps the reference's
// numbers of alpha (even) and beta (odd) electrons, psi = U(t)|ref> and
// sigma = H psi live in the sector of those numbers.  That sector is stored
// compactly: index i = ra * nbeta + rb for the alpha string of rank ra and
// the beta string of rank rb (ranks in ascending order of the strings' bits).
// A 16-qubit, 8-electron sector is 4,900 amplitudes, so one CTA holds psi and
// sigma of one parameter set in shared memory and runs the whole evaluation
// there: the forward program, sigma = H psi from a sparse row list of H built
// once per evaluator, the energy, and the adjoint reverse sweep, with one
// barrier per program step and no global traffic besides the H rows, the
// steps' pair lists (read-only, L2-resident, shared by every CTA) and one save
// of psi and sigma between the kernels.
//
// When every step's pair coefficients and H are real (particle-hole and
// generalised pools of real excitations, real integrals), psi and sigma stay
// real and are stored as doubles (V = double): half the shared memory and
// half the shared-memory traffic of complex storage (V = double2).
//
// Each step is one of the Givens-form steps of the full-space program: the
// pairs (j0, j1 = j0 ^ x) with j0's bits on the step's pattern positions equal
// to one of its active patterns (bit h of x clear).  Restricted to the sector,
// such a j0 factors into an alpha string and a beta string matching the
// pattern's alpha and beta bits, so the pairs of one pattern are the product
// of an alpha list and a beta list, each entry holding a string's rank, its
// partner's rank (string ^ x) and its share of the sign
// sigma(j0) = (-1)^popcount(j0 & zbase).  The global-memory path
// (qfb_csec.cuh) reads those lists (records of RHead / RPat / SEntry); the
// shared-memory kernels here read the product expanded on the host into one
// word pair per amplitude pair (PHead / PStream), ordered so that each half
// warp (quarter warp for complex amplitudes) touches distinct banks.  The
// arithmetic on each pair is that of the full-space kernels (givens_pair and
// the gradient inner product).
#pragma once

#include <cstdint>

namespace qfbs {

struct SEntry {  // one string of an alpha or beta list
    uint16_t r0, r1;  // rank, partner's rank
    uint32_t s;       // parity of string & zbase
};

// A step record: the 16-byte header, the patterns, then the entries of their
// lists, contiguous in one stream of 16-byte words.  Records run in the order
// a kernel executes them.
struct RHead {
    int32_t npf;   // patterns | flags << 8
    int32_t row;   // partial row of an inner product
    double gamma;
};
struct RPat {
    uint16_t a0, na, b0, nb;  // lists: entries [a0, a0 + na) and [b0, b0 + nb) of the record
    uint32_t inv;             // ceil(2^32 / nb), 0 when nb == 1
    uint32_t pad;
    double2 gn, hn;
};
enum : int { R_ROT = 1, R_IP = 2, R_TWO = 4 };

struct SStream {          // one kernel's records
    const uint4 *rec;     // records, 16-byte words
    const int2 *span;     // per record: first word, words
    const int32_t *param; // per record: parameter of its angle
    int n;
    int maxw;             // longest record (words)
};

// A step record on the pair list, used by the shared-memory kernels: the
// pairs of the step's patterns as explicit sector index pairs, ordered on the
// host so that the lanes of a warp reach distinct shared-memory banks, and the
// step's constants.  A stream's headers, pairs and pattern coefficients are
// three arrays.
struct PHead {
    int32_t p0;     // first pair
    int32_t np;     // pairs
    int32_t fl;     // flags (R_ROT | R_IP | R_TWO) | patterns << 8
    int32_t row;    // partial row of an inner product
    double gamma;
    int32_t c0;     // first pattern's (gn, hn) in coef
    int32_t param;  // parameter of the record's angle
};
static_assert(sizeof(PHead) == 32, "PHead is two 16-byte words");

// A pair word: i0 (bits 0-13) | i1 << 14 | neg << 28 | pattern << 29 (a
// Givens-form step has at most 8 active patterns).
constexpr int kPairIdxBits = 14;  // sector indices below 16384
constexpr int kSweepRing = 2;     // register sets of pair words in the sweep (2 or 4)
constexpr int kStepThreads = 512;   // block of the forward and residual kernels
constexpr int kSweepThreads = 256;  // block of the sweep (more pairs per thread per record)
constexpr int kPairPatterns = 8;
struct PStream {
    const PHead *hd;
    const uint32_t *pair;
    const double2 *coef;  // per pattern: gn, hn
    int n;
};

struct SLaunch {
    int nsec, nbeta, ref_i, nparam;
    PStream fwd, sweep;
    const int32_t *rowptr;     // H rows
    const uint32_t *col;
    const double *val_r;       // real H (val_c == nullptr) ...
    const double2 *val_c;      // ... or complex
    const double *params;      // [B][nparam]
    double *energy;            // [B]
    double2 *partial;          // [K steps][B][warps]
    void *save;                // V [B][2][nsec]: psi after the forward program, sigma
};

__device__ __forceinline__ double2 s_cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 s_cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 s_cjmul(double2 a, double2 b) {  // conj(a) b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Amplitude arithmetic for both storage types (complex double2, real double).
__device__ __forceinline__ double2 v_zero(double2) { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double v_zero(double) { return 0.0; }
__device__ __forceinline__ void v_one(double2 &v) { v = make_double2(1.0, 0.0); }
__device__ __forceinline__ void v_one(double &v) { v = 1.0; }
template <class V>
__device__ __forceinline__ V v_one_of() {
    V v;
    v_one(v);
    return v;
}
// coefficient g times amplitude x (real storage: g is real)
__device__ __forceinline__ double2 v_mul(double2 g, double2 x) { return s_cmul(g, x); }
__device__ __forceinline__ double v_mul(double2 g, double x) { return g.x * x; }
__device__ __forceinline__ double v_mul(double g, double x) { return g * x; }
// c x + s y
__device__ __forceinline__ double2 v_lin(double c, double2 x, double s, double2 y) {
    return make_double2(c * x.x + s * y.x, c * x.y + s * y.y);
}
__device__ __forceinline__ double v_lin(double c, double x, double s, double y) { return c * x + s * y; }
// conj(a) b as a complex number
__device__ __forceinline__ double2 v_cj(double2 a, double2 b) { return s_cjmul(a, b); }
__device__ __forceinline__ double2 v_cj(double a, double b) { return make_double2(a * b, 0.0); }
// acc += f x (f a real matrix entry)
__device__ __forceinline__ void v_acc(double2 &acc, double f, double2 x) {
    acc.x += f * x.x;
    acc.y += f * x.y;
}
__device__ __forceinline__ void v_acc(double &acc, double f, double x) { acc += f * x; }
__device__ __forceinline__ double2 v_add(double2 a, double2 b) { return s_cadd(a, b); }
__device__ __forceinline__ double v_add(double a, double b) { return a + b; }
__device__ __forceinline__ double v_shfl_down(double v, int o) {
    return __shfl_down_sync(0xffffffffu, v, o);
}
__device__ __forceinline__ double2 v_shfl_down(double2 v, int o) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, o), __shfl_down_sync(0xffffffffu, v.y, o));
}

// new0 = c v0 + s hn v1, new1 = c v1 + s gn v0 (as givens_pair)
template <class V, class K>
__device__ __forceinline__ void s_givens(V &v0, V &v1, double c, double s, K gn, K hn) {
    const V a = v_mul(hn, v1), b = v_mul(gn, v0);
    const V n0 = v_lin(c, v0, s, a);
    v1 = v_lin(c, v1, s, b);
    v0 = n0;
}

// A pair's share of <w|K|v>: conj(w0) hn v1 + conj(w1) gn v0
__device__ __forceinline__ double v_ip(double w0, double w1, double v0, double v1, double gn,
                                       double hn) {
    return w0 * (hn * v1) + w1 * (gn * v0);
}
__device__ __forceinline__ double2 v_ip(double2 w0, double2 w1, double2 v0, double2 v1, double2 gn,
                                        double2 hn) {
    return s_cadd(s_cjmul(w0, s_cmul(hn, v1)), s_cjmul(w1, s_cmul(gn, v0)));
}
__device__ __forceinline__ double2 v_as2(double x) { return make_double2(x, 0.0); }
__device__ __forceinline__ double2 v_as2(double2 x) { return x; }

__device__ __forceinline__ PHead p_head(const PHead *p) {
    const int4 a = __ldg(reinterpret_cast<const int4 *>(p));
    const int4 b = __ldg(reinterpret_cast<const int4 *>(p) + 1);
    PHead h;
    h.p0 = a.x;
    h.np = a.y;
    h.fl = a.z;
    h.row = a.w;
    h.gamma = __hiloint2double(b.y, b.x);
    h.c0 = b.z;
    h.param = b.w;
    return h;
}

// Pair words of a record held per thread: three for real amplitudes, two
// for complex ones (whose pairs need twice the registers).
template <class V>
__host__ __device__ constexpr int pair_slots() {
    return sizeof(V) == sizeof(double) ? 3 : 2;
}

// Words past a stream's last pair (zeros), so that the prefetch below loads
// without a bound check (a selected value would wait for its load at once).
constexpr int kPairPad = 4 * 1024;

// This thread's first KP pair words of record h (pairs tid, tid + nth, ...);
// words past the record are loaded but never used (p_record checks np).
template <int KP>
__device__ __forceinline__ void p_words(const PStream &S, const PHead &h, uint32_t (&pw)[KP]) {
#pragma unroll
    for (int j = 0; j < KP; ++j) pw[j] = __ldg(S.pair + h.p0 + threadIdx.x + j * blockDim.x);
}


// One pair: the share of <w|K|v> into acc and / or the rotation of v (and w
// when TWO) by the angle whose cos / sin is (c, s).
template <bool ROT, bool IP, bool TWO, class V>
__device__ __forceinline__ void p_pair(uint32_t pw, double c, double s, double gamma, V gn, V hn, V *v,
                                       V *w, V &acc) {
    constexpr uint32_t M = (1u << kPairIdxBits) - 1u;
    const int i0 = (int)(pw & M), i1 = (int)((pw >> kPairIdxBits) & M);
    const bool neg = (pw >> (2 * kPairIdxBits)) & 1u;
    V v0 = v[i0], v1 = v[i1];
    V w0 = v_zero(V()), w1 = w0;
    if (IP || TWO) {
        w0 = w[i0];
        w1 = w[i1];
    }
    if (IP) v_acc(acc, neg ? -gamma : gamma, v_ip(w0, w1, v0, v1, gn, hn));
    if (ROT) {
        const double ss = neg ? -s : s;
        s_givens(v0, v1, c, ss, gn, hn);
        v[i0] = v0;
        v[i1] = v1;
        if (TWO) {
            s_givens(w0, w1, c, ss, gn, hn);
            w[i0] = w0;
            w[i1] = w1;
        }
    }
}

// One record on the compact states: this thread's pairs (the prefetched
// words first, then any beyond KP per thread).  The pairs of one record touch
// distinct amplitudes, so threads need no ordering within it.
// The coefficients (gn, hn) of pattern k of a stream: real parts only for
// real amplitudes.
__device__ __forceinline__ void p_ldcoef(const PStream &S, int k, double &gn, double &hn) {
    gn = __ldg(reinterpret_cast<const double *>(S.coef + 2 * k));
    hn = __ldg(reinterpret_cast<const double *>(S.coef + 2 * k + 1));
}
__device__ __forceinline__ void p_ldcoef(const PStream &S, int k, double2 &gn, double2 &hn) {
    gn = __ldg(S.coef + 2 * k);
    hn = __ldg(S.coef + 2 * k + 1);
}

// gn, hn: the coefficients of a single-pattern record (p_coef); records of
// several patterns load each pair's from its pattern number.
template <bool ROT, bool IP, bool TWO, class V, int KP>
__device__ __forceinline__ void p_record(const PStream &S, const PHead &h, const uint32_t (&pw)[KP],
                                         double2 csn, V gn, V hn, V *v, V *w, V &acc) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const bool one = (h.fl >> 8) == 1;
    auto run = [&](uint32_t p) {
        if (!one) p_ldcoef(S, h.c0 + (int)(p >> (2 * kPairIdxBits + 1)), gn, hn);
        p_pair<ROT, IP, TWO, V>(p, csn.x, csn.y, h.gamma, gn, hn, v, w, acc);
    };
#pragma unroll
    for (int j = 0; j < KP; ++j)
        if (tid + j * nth < h.np) run(pw[j]);
    for (int k = tid + KP * nth; k < h.np; k += nth) run(__ldg(S.pair + h.p0 + k));
}

// The coefficients of record h when it has a single pattern (else zeros)
template <class V>
__device__ __forceinline__ void p_coef(const PStream &S, const PHead &h, V &gn, V &hn) {
    gn = hn = v_zero(V());
    if ((h.fl >> 8) == 1) p_ldcoef(S, h.c0, gn, hn);
}

// A record as the kernels keep it in shared memory: its header, the cos / sin
// of its angle for this CTA's parameter set and, for a single-pattern record,
// its coefficients.
template <class V>
struct PSmem {
    PHead h;
    double2 cs;
    V gn, hn;
};
static_assert(sizeof(PSmem<double>) == 64 && sizeof(PSmem<double2>) == 80, "PSmem layout");

// Every record's header, coefficients and cos / sin of sign * gamma * theta
// into s_pr
template <class V>
__device__ __forceinline__ void p_angles(const PStream &S, const double *par, int sign,
                                         PSmem<V> *s_pr) {
    for (int r = threadIdx.x; r < S.n; r += blockDim.x) {
        const PHead h = p_head(S.hd + r);
        double sn, cs;
        sincos((double)sign * h.gamma * par[h.param], &sn, &cs);
        V gn, hn;
        p_coef(S, h, gn, hn);
        s_pr[r].h = h;
        s_pr[r].cs = make_double2(cs, sn);
        s_pr[r].gn = gn;
        s_pr[r].hn = hn;
    }
}

__device__ __forceinline__ double v_shfl_xor(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double2 v_shfl_xor(double2 v, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

// Warp sums of two values at once: a's into lane 0, b's into lane 16 (the
// first exchange halves the work of two separate reductions).
template <class V>
__device__ __forceinline__ V p_sum2(V a, V b) {
    const bool hi = threadIdx.x & 16;
    V k = v_add(hi ? b : a, v_shfl_xor(hi ? a : b, 16));
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) k = v_add(k, v_shfl_down(k, o));
    return k;
}
template <class V>
__device__ __forceinline__ V p_sum1(V a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a = v_add(a, v_shfl_down(a, o));
    return a;
}

// Apply record rec with this thread's prefetched words; returns this
// thread's share of the record's inner product (SWEEP records carry flags:
// rotation of both states, inner product or both).
template <bool SWEEP, class V, int KP>
__device__ __forceinline__ V p_step(const PStream &S, const PSmem<V> &rec, const uint32_t (&pw)[KP],
                                    V *v, V *w) {
    const PHead h = rec.h;
    const double2 csn = rec.cs;
    const V gn = rec.gn, hn = rec.hn;
    const int fl = h.fl & 255;
    V acc = v_zero(V());
    if (!SWEEP) {
        p_record<true, false, false, V, KP>(S, h, pw, csn, gn, hn, v, w, acc);
    } else if (fl == (R_ROT | R_IP | R_TWO)) {
        p_record<true, true, true, V, KP>(S, h, pw, csn, gn, hn, v, w, acc);
    } else if (fl == R_IP) {
        p_record<false, true, false, V, KP>(S, h, pw, csn, gn, hn, v, w, acc);
    } else {
        p_record<true, false, true, V, KP>(S, h, pw, csn, gn, hn, v, w, acc);
    }
    return acc;
}

// The warp partials of the inner products of records a and b (b < 0: none):
// one per warp and record at partial[row][slot][warp] (nslot slots), zero
// from warps that hold no pair of the record, two records reduced together
// where both have one.
template <class V>
__device__ __forceinline__ void p_partials(const PSmem<V> *s_pr, int a, V acca, int b, V accb,
                                           double2 *partial, int nslot, int slot) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const PHead ha = s_pr[a].h;
    const bool ipa = ha.fl & R_IP;
    bool ipb = false;
    PHead hb = ha;
    if (b >= 0) {
        hb = s_pr[b].h;
        ipb = hb.fl & R_IP;
    }
    if (!ipa && !ipb) return;
    const bool ida = 32 * warp >= ha.np, idb = 32 * warp >= hb.np;  // warp holds no pair
    auto put = [&](const PHead &h, V x) {
        partial[((size_t)h.row * nslot + slot) * nw + warp] = v_as2(x);
    };
    if (ipa && ipb && !ida && !idb) {
        const V k = p_sum2(acca, accb);
        if (lane == 0) put(ha, k);
        if (lane == 16) put(hb, k);
        return;
    }
    if (ipa) {
        const V k = ida ? v_zero(V()) : p_sum1(acca);
        if (lane == 0) put(ha, k);
    }
    if (ipb) {
        const V k = idb ? v_zero(V()) : p_sum1(accb);
        if (lane == 0) put(hb, k);
    }
}

// Run a stream, one barrier per record.  RING register sets rotate: while
// record r is applied from one, the pair words of the next RING - 1 records
// are in flight in the others (each set is refilled right after its record
// ran), so a record's words have had RING - 1 records' time to arrive from
// L2.  SWEEP: the inner products of records (r, r + 1) are reduced together.
template <bool SWEEP, class V>
__device__ __forceinline__ void p_run(const PStream &S, const PSmem<V> *s_pr, V *v, V *w,
                                      double2 *partial, int nslot, int slot) {
    constexpr int KP = pair_slots<V>();
    constexpr int RING = SWEEP ? kSweepRing : 4;
    const int n = S.n;
    uint32_t w0[KP], w1[KP], w2[KP], w3[KP];
    if (n > 0) p_words(S, s_pr[0].h, w0);
    if (n > 1) p_words(S, s_pr[1].h, w1);
    if (RING == 4 && n > 2) p_words(S, s_pr[2].h, w2);
    for (int r = 0; r < n; r += RING) {
        if (RING == 4 && r + 3 < n) p_words(S, s_pr[r + 3].h, w3);
        const V a0 = p_step<SWEEP, V, KP>(S, s_pr[r], w0, v, w);
        __syncthreads();
        if (r + 1 >= n) {
            if (SWEEP) p_partials(s_pr, r, a0, -1, a0, partial, nslot, slot);
            break;
        }
        if (r + RING < n) p_words(S, s_pr[r + RING].h, w0);
        const V a1 = p_step<SWEEP, V, KP>(S, s_pr[r + 1], w1, v, w);
        if (SWEEP) p_partials(s_pr, r, a0, r + 1, a1, partial, nslot, slot);
        __syncthreads();
        if (RING == 2) {
            if (r + 3 < n) p_words(S, s_pr[r + 3].h, w1);
            continue;
        }
        if (r + 2 >= n) break;
        if (r + 5 < n) p_words(S, s_pr[r + 5].h, w1);
        const V a2 = p_step<SWEEP, V, KP>(S, s_pr[r + 2], w2, v, w);
        __syncthreads();
        if (r + 3 >= n) {
            if (SWEEP) p_partials(s_pr, r + 2, a2, -1, a2, partial, nslot, slot);
            break;
        }
        if (r + 6 < n) p_words(S, s_pr[r + 6].h, w2);
        const V a3 = p_step<SWEEP, V, KP>(S, s_pr[r + 3], w3, v, w);
        if (SWEEP) p_partials(s_pr, r + 2, a2, r + 3, a3, partial, nslot, slot);
        __syncthreads();
    }
}

// The evaluation runs as three kernels: the forward program (one CTA per
// parameter set, psi in shared memory), sigma = H psi with the energy (a few
// parameter sets and a slice of the rows per CTA, sigma rows straight to the
// save buffer), and the reverse sweep (one CTA per parameter set, psi and
// sigma in shared memory).  Shared memory of the forward and sweep kernels:
// the states, then every record's header with the cos / sin of its angle
// (PSmem).

template <class V>
__global__ void __launch_bounds__(kStepThreads, 1024 / kStepThreads) k_sector_forward(SLaunch L) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw);
    PSmem<V> *s_pr = reinterpret_cast<PSmem<V> *>(s_raw + ((sizeof(V) * L.nsec + 15) & ~(size_t)15));
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    for (int i = tid; i < L.nsec; i += nth) psi[i] = i == L.ref_i ? v_one_of<V>() : v_zero(V());
    p_angles(L.fwd, par, 1, s_pr);
    __syncthreads();
    p_run<false, V>(L.fwd, s_pr, psi, (V *)nullptr, nullptr, 1, 0);
    V *sv = reinterpret_cast<V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < L.nsec; i += nth) sv[i] = psi[i];
}

// sigma = H psi and the energy, P parameter sets per CTA.  CTA x works on
// group g = x / Q (sets g P .. g P + P - 1) and row slice q = x % Q: it loads
// the group's psi into shared memory, streams the slice's H rows once for all
// P sets (one warp per row, U entries in flight per lane, each entry's column
// gathered from every set), writes the sigma rows to the save
// buffer and one partial energy per set to epart[set][q].  The CTA that
// completes a group last (a ticket on count[g], which it resets) sums the
// group's partials in q order into energy, so the sum's order is fixed.
template <bool REAL, class V, int P, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_sector_h(
    SLaunch L, int nbatch, int Q, double *__restrict__ epart, unsigned *__restrict__ count) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ double s_red[NT / 32][P];
    __shared__ unsigned s_ticket;
    // real states of an even number of sets sit in pairs, [P / 2][nsec] of
    // double2 (sets 2h, 2h + 1): one 16-byte gather reads two sets
    constexpr bool PAIR = REAL && sizeof(V) == sizeof(double) && P % 2 == 0;
    V *psi = reinterpret_cast<V *>(s_raw);  // [P][nsec] unless PAIR
    double2 *ps2 = reinterpret_cast<double2 *>(s_raw);
    const int g = blockIdx.x / Q, q = blockIdx.x - g * Q, tid = threadIdx.x;
    const int b0 = g * P, nb = min(P, nbatch - b0), n = L.nsec;
    V *save = reinterpret_cast<V *>(L.save);
    if constexpr (PAIR) {
        const double *sd = reinterpret_cast<const double *>(L.save);
#pragma unroll
        for (int h = 0; h < P / 2; ++h) {
            const double *s0 = sd + (size_t)(b0 + (2 * h < nb ? 2 * h : 0)) * 2 * n;
            const double *s1 = sd + (size_t)(b0 + (2 * h + 1 < nb ? 2 * h + 1 : 0)) * 2 * n;
            for (int i = tid; i < n; i += NT) ps2[h * n + i] = make_double2(s0[i], s1[i]);
        }
    } else {
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const V *sv = save + (size_t)(b0 + (p < nb ? p : 0)) * 2 * n;
            for (int i = tid; i < n; i += NT) psi[p * n + i] = sv[i];
        }
    }
    __syncthreads();
    const int r0 = (int)((int64_t)q * n / Q), r1 = (int)((int64_t)(q + 1) * n / Q);
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int U = P >= 2 ? 4 : 8;  // H row entries in flight per lane
    // after a row's reduction, lane GL p holds set p's sum (GL lanes per set)
    constexpr int GL = 32 / P;
    const int lp = lane / GL;
    double en = 0.0;  // energy share of set lp (lanes lane % GL == 0)
    for (int i = r0 + warp; i < r1; i += NT / 32) {
        V acc[P];
#pragma unroll
        for (int p = 0; p < P; ++p) acc[p] = v_zero(V());
        const int e1 = L.rowptr[i + 1];
        for (int e0 = L.rowptr[i] + lane; e0 < e1; e0 += 32 * U) {
            uint32_t c[U];
            double fr[REAL ? U : 1];
            double2 fc[REAL ? 1 : U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + 32 * u;
                c[u] = (e < e1) ? __ldg(&L.col[e]) : 0u;
                if (REAL) fr[u] = (e < e1) ? __ldg(&L.val_r[e]) : 0.0;
                else fc[REAL ? 0 : u] = (e < e1) ? __ldg(&L.val_c[e]) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if constexpr (PAIR) {
#pragma unroll
                    for (int h = 0; h < P / 2; ++h) {
                        const double2 x = ps2[h * n + (int)c[u]];
                        v_acc(acc[2 * h], fr[u], x.x);
                        v_acc(acc[2 * h + 1], fr[u], x.y);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < P; ++p) {
                        const V x = psi[p * n + (int)c[u]];
                        if constexpr (REAL) {
                            v_acc(acc[p], fr[u], x);
                        } else {
                            acc[p] = v_add(acc[p], v_mul(fc[REAL ? 0 : u], x));
                        }
                    }
                }
            }
        }
        // reduce-scatter: each exchange halves the values a lane carries
        V m;
        if constexpr (P == 4) {
            const bool b4 = lane & 16, b3 = lane & 8;
            const V k0 = v_add(b4 ? acc[2] : acc[0], v_shfl_xor(b4 ? acc[0] : acc[2], 16));
            const V k1 = v_add(b4 ? acc[3] : acc[1], v_shfl_xor(b4 ? acc[1] : acc[3], 16));
            m = v_add(b3 ? k1 : k0, v_shfl_xor(b3 ? k0 : k1, 8));
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) m = v_add(m, v_shfl_down(m, o));
        } else if constexpr (P == 2) {
            const bool b4 = lane & 16;
            m = v_add(b4 ? acc[1] : acc[0], v_shfl_xor(b4 ? acc[0] : acc[1], 16));
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) m = v_add(m, v_shfl_down(m, o));
        } else {
            m = acc[0];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = v_add(m, v_shfl_down(m, o));
        }
        if ((lane & (GL - 1)) == 0) {
            if (lp < nb) save[(size_t)(b0 + lp) * 2 * n + n + i] = m;
            V pv;
            if constexpr (PAIR) {
                const double2 x = ps2[(lp >> 1) * n + i];
                pv = (lp & 1) ? x.y : x.x;
            } else {
                pv = psi[lp * n + i];
            }
            en += v_cj(pv, m).x;
        }
    }
    if ((lane & (GL - 1)) == 0) s_red[warp][lp] = en;
    __syncthreads();
    if (tid == 0) {
        for (int p = 0; p < nb; ++p) {
            double t = 0.0;
            for (int k = 0; k < NT / 32; ++k) t += s_red[k][p];
            epart[(size_t)(b0 + p) * Q + q] = t;
        }
        __threadfence();
        s_ticket = atomicAdd(&count[g], 1u);
    }
    __syncthreads();
    if (s_ticket == (unsigned)Q - 1u) {  // every slice of the group is in
        __threadfence();
        if (tid < nb) {
            double t = 0.0;
            for (int k = 0; k < Q; ++k) t += __ldcg(&epart[(size_t)(b0 + tid) * Q + k]);
            L.energy[b0 + tid] = t;
        }
        if (tid == 0) count[g] = 0u;
    }
}

template <class V>
__global__ void __launch_bounds__(kSweepThreads, 1024 / kSweepThreads) k_sector_sweep(SLaunch L) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw), *sig = psi + L.nsec;
    PSmem<V> *s_pr = reinterpret_cast<PSmem<V> *>(s_raw + ((sizeof(V) * 2 * L.nsec + 15) & ~(size_t)15));
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < 2 * L.nsec; i += nth) psi[i] = sv[i];
    p_angles(L.sweep, par, -1, s_pr);
    __syncthreads();
    p_run<true, V>(L.sweep, s_pr, psi, sig, L.partial, gridDim.x, blockIdx.x);
}

// PQE residuals on the compact states: sigma of slot blockIdx.x from the save
// buffer, U^dagger applied to it in shared memory (stream R: the forward
// records in reverse order, angles negated), then
// res[b][k] = Re(sigma[idx[k]] * phase[k]) (0 where idx[k] < 0).
template <class V>
__global__ void __launch_bounds__(kStepThreads, 1024 / kStepThreads) k_sector_resid(SLaunch L, PStream R,
                                                         const int64_t *__restrict__ idx,
                                                         const double2 *__restrict__ phase,
                                                         int nres, double *__restrict__ res) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *sig = reinterpret_cast<V *>(s_raw);
    PSmem<V> *s_pr = reinterpret_cast<PSmem<V> *>(s_raw + ((sizeof(V) * L.nsec + 15) & ~(size_t)15));
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec + L.nsec;
    for (int i = tid; i < L.nsec; i += nth) sig[i] = sv[i];
    p_angles(R, par, -1, s_pr);
    __syncthreads();
    p_run<false, V>(R, s_pr, sig, (V *)nullptr, nullptr, 1, 0);
    for (int k = tid; k < nres; k += nth) {
        const int64_t i = idx[k];
        double r = 0.0;
        if (i >= 0) {
            const double2 v = v_cj(v_one_of<V>(), sig[i]), ph = phase[k];
            r = v.x * ph.x - v.y * ph.y;
        }
        res[(size_t)b * nres + k] = r;
    }
}

// Pool inner products on the compact states: each CTA loads psi and sigma of
// slot blockIdx.y and runs the inner-product records r = blockIdx.x,
// blockIdx.x + gridDim.x, ... of the pool stream.  The records leave the
// states unchanged, so they need no barrier between them.
template <class V>
__global__ void __launch_bounds__(512, 2) k_sector_pool(SLaunch L, PStream P) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw), *sig = psi + L.nsec;
    const int b = blockIdx.y, tid = threadIdx.x, nth = blockDim.x, nw = nth >> 5;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < 2 * L.nsec; i += nth) psi[i] = sv[i];
    __syncthreads();
    for (int r = blockIdx.x; r < P.n; r += gridDim.x) {
        constexpr int KP = pair_slots<V>();
        const PHead h = p_head(P.hd + r);
        uint32_t pw[KP];
        p_words(P, h, pw);
        V gn, hn;
        p_coef(P, h, gn, hn);
        V acc = v_zero(V());
        p_record<false, true, false, V, KP>(P, h, pw, make_double2(1.0, 0.0), gn, hn, psi, sig, acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc = v_add(acc, v_shfl_down(acc, o));
        if ((tid & 31) == 0) L.partial[((size_t)h.row * gridDim.y + b) * nw + (tid >> 5)] = v_as2(acc);
    }
}

// ---------------------------------------------------------------------------
// Two real parameter sets per CTA (forward program)
// ---------------------------------------------------------------------------
// With real states, sets 2g and 2g + 1 share one CTA of the forward program:
// amplitude slot i holds both sets' values as one double2 (.x set 2g, .y set
// 2g + 1), so every pair word, record header, shared-memory load / store and
// barrier serves both sets, while each set keeps its own angle (cos / sin per
// set in the record).  The arithmetic on each set is that of k_sector_forward.
// (The reverse sweep stays one set per CTA: paired, its shared memory of two
// states for two sets leaves half the warps per set to hide latency, and it
// ran slower at 256 sets on 148 SMs.)

struct PSmemPR {
    PHead h;
    double2 c, s;   // cos / sin of the record's angle: .x first set, .y second
    double gn, hn;  // single-pattern records: the coefficients
};
static_assert(sizeof(PSmemPR) == 80, "PSmemPR layout");

__device__ __forceinline__ void p_angles_pr(const PStream &S, const double *parA, const double *parB,
                                            int sign, PSmemPR *s_pr) {
    for (int r = threadIdx.x; r < S.n; r += blockDim.x) {
        const PHead h = p_head(S.hd + r);
        double sa, ca, sb, cb;
        sincos((double)sign * h.gamma * parA[h.param], &sa, &ca);
        sincos((double)sign * h.gamma * parB[h.param], &sb, &cb);
        double gn, hn;
        p_coef(S, h, gn, hn);
        s_pr[r].h = h;
        s_pr[r].c = make_double2(ca, cb);
        s_pr[r].s = make_double2(sa, sb);
        s_pr[r].gn = gn;
        s_pr[r].hn = hn;
    }
}

// One pair of a forward record on both sets (p_pair's rotation per set).
__device__ __forceinline__ void pr_pair(uint32_t pw, double2 c, double2 s, double gn, double hn,
                                        double2 *v) {
    constexpr uint32_t M = (1u << kPairIdxBits) - 1u;
    const int i0 = (int)(pw & M), i1 = (int)((pw >> kPairIdxBits) & M);
    const bool neg = (pw >> (2 * kPairIdxBits)) & 1u;
    const double2 a0 = v[i0], a1 = v[i1];
    const double sx = neg ? -s.x : s.x, sy = neg ? -s.y : s.y;
    v[i0] = make_double2(c.x * a0.x + sx * (hn * a1.x), c.y * a0.y + sy * (hn * a1.y));
    v[i1] = make_double2(c.x * a1.x + sx * (gn * a0.x), c.y * a1.y + sy * (gn * a0.y));
}

template <int KP>
__device__ __forceinline__ void pr_record(const PStream &S, const PSmemPR &rec, const uint32_t (&pw)[KP],
                                          double2 *v) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const PHead &h = rec.h;
    const bool one = (h.fl >> 8) == 1;
    double gn = rec.gn, hn = rec.hn;
    auto run = [&](uint32_t p) {
        if (!one) p_ldcoef(S, h.c0 + (int)(p >> (2 * kPairIdxBits + 1)), gn, hn);
        pr_pair(p, rec.c, rec.s, gn, hn, v);
    };
#pragma unroll
    for (int j = 0; j < KP; ++j)
        if (tid + j * nth < h.np) run(pw[j]);
    for (int k = tid + KP * nth; k < h.np; k += nth) run(__ldg(S.pair + h.p0 + k));
}

// p_run's forward program for two real sets: the same ring of four
// prefetched sets of pair words, one barrier per record.
__device__ __forceinline__ void pr_run(const PStream &S, const PSmemPR *s_pr, double2 *v) {
    constexpr int KP = 2;
    const int n = S.n;
    uint32_t w0[KP], w1[KP], w2[KP], w3[KP];
    if (n > 0) p_words(S, s_pr[0].h, w0);
    if (n > 1) p_words(S, s_pr[1].h, w1);
    if (n > 2) p_words(S, s_pr[2].h, w2);
    for (int r = 0; r < n; r += 4) {
        if (r + 3 < n) p_words(S, s_pr[r + 3].h, w3);
        pr_record<KP>(S, s_pr[r], w0, v);
        __syncthreads();
        if (r + 1 >= n) break;
        if (r + 4 < n) p_words(S, s_pr[r + 4].h, w0);
        pr_record<KP>(S, s_pr[r + 1], w1, v);
        __syncthreads();
        if (r + 2 >= n) break;
        if (r + 5 < n) p_words(S, s_pr[r + 5].h, w1);
        pr_record<KP>(S, s_pr[r + 2], w2, v);
        __syncthreads();
        if (r + 3 >= n) break;
        if (r + 6 < n) p_words(S, s_pr[r + 6].h, w2);
        pr_record<KP>(S, s_pr[r + 3], w3, v);
        __syncthreads();
    }
}

// Forward program of sets 2g, 2g + 1 (g = blockIdx.x; a last odd set runs
// alone, its twin a copy that is not saved); psi of both into the save buffer.
__global__ void __launch_bounds__(kStepThreads, 1) k_sector_forward_pr(SLaunch L, int nbatch) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    double2 *psi = reinterpret_cast<double2 *>(s_raw);
    PSmemPR *s_pr = reinterpret_cast<PSmemPR *>(s_raw + ((16 * (size_t)L.nsec + 15) & ~(size_t)15));
    const int b0 = 2 * blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const bool two = b0 + 1 < nbatch;
    const double *parA = L.params + (size_t)b0 * L.nparam;
    const double *parB = two ? parA + L.nparam : parA;
    for (int i = tid; i < L.nsec; i += nth)
        psi[i] = i == L.ref_i ? make_double2(1.0, 1.0) : make_double2(0.0, 0.0);
    p_angles_pr(L.fwd, parA, parB, 1, s_pr);
    __syncthreads();
    pr_run(L.fwd, s_pr, psi);
    double *sv = reinterpret_cast<double *>(L.save) + (size_t)b0 * 2 * L.nsec;
    for (int i = tid; i < L.nsec; i += nth) {
        const double2 x = psi[i];
        sv[i] = x.x;
        if (two) sv[2 * (size_t)L.nsec + i] = x.y;
    }
}

// ---------------------------------------------------------------------------
// Packed evaluations of several problems in one launch
// ---------------------------------------------------------------------------

// One problem of a packed launch: the compact evaluator data of one dUCC
// problem (its sector, forward and sweep pair lists, H rows on the sector and
// the sweep record rows of each parameter).
struct PackMember {
    int nsec, ref_i, nparam, pad;
    PStream fwd, sweep;
    const int32_t *rowptr;
    const uint32_t *col;
    const double *val_r;   // real H (val_c == nullptr) ...
    const double2 *val_c;  // ... or complex
    const int2 *psteps;    // per parameter: its rows of the sweep partials
};

constexpr int kPackThreads = 256;

// sigma = H psi on one CTA's state (a warp per row, the lanes over the row's
// entries) and this CTA's energy <psi|H|psi>, summed in a fixed order.
template <class V>
__device__ __forceinline__ double p_hpsi(const PackMember &m, const V *psi, V *sig, double *s_red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int U = 4;  // row entries in flight per lane
    double en = 0.0;
    for (int i = warp; i < m.nsec; i += nw) {
        V acc = v_zero(V());
        const int e1 = m.rowptr[i + 1];
        for (int e0 = m.rowptr[i] + lane; e0 < e1; e0 += 32 * U) {
            uint32_t c[U];
            double fr[U];
            double2 fc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + 32 * u;
                const bool in = e < e1;
                c[u] = in ? __ldg(&m.col[e]) : 0u;
                if (sizeof(V) == sizeof(double2) && m.val_c) {
                    fc[u] = in ? __ldg(&m.val_c[e]) : make_double2(0.0, 0.0);
                    fr[u] = 0.0;
                } else {
                    fr[u] = in ? __ldg(&m.val_r[e]) : 0.0;
                    fc[u] = make_double2(0.0, 0.0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const V x = psi[c[u]];
                if constexpr (sizeof(V) == sizeof(double2)) {
                    if (m.val_c) acc = v_add(acc, v_mul(fc[u], x));
                    else v_acc(acc, fr[u], x);
                } else {
                    v_acc(acc, fr[u], x);
                }
            }
        }
        acc = p_sum1(acc);
        if (lane == 0) {
            sig[i] = acc;
            en += v_cj(psi[i], acc).x;
        }
    }
    if (lane == 0) s_red[warp] = en;
    __syncthreads();
    double t = 0.0;
    for (int k = 0; k < nw; ++k) t += s_red[k];
    return t;
}

// CTA x evaluates item x: parameter set params[x][0 .. nparam) of problem
// items[x].x, with its gradient when items[x].y != 0.  Energy into energy[x],
// gradient into grad[x][0 .. nparam); partial[x] holds the sweep's warp
// partials ([max_rows][warps] per item).  The whole evaluation stays in
// this CTA's shared memory: psi = U(t)|ref> (forward pair lists), sigma = H psi
// from the H rows, the energy, the reverse sweep and the per-parameter sums,
// so one launch serves parameter sets of different problems side by side.
template <class V>
__global__ void __launch_bounds__(kPackThreads, 2) k_sector_pack(
    const PackMember *__restrict__ members, const int2 *__restrict__ items, int maxparam,
    const double *__restrict__ params, double *__restrict__ energy, double *__restrict__ grad,
    double2 *__restrict__ partial, int max_rows, int nmem) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ double s_red[kPackThreads / 32];
    const int2 it = items[blockIdx.x];
    if ((unsigned)it.x >= (unsigned)nmem) {  // no such problem: NaN energy, nothing else
        if (threadIdx.x == 0) energy[blockIdx.x] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    const PackMember m = members[it.x];
    const int tid = threadIdx.x, nth = blockDim.x, nw = nth >> 5;
    V *psi = reinterpret_cast<V *>(s_raw), *sig = psi + m.nsec;
    PSmem<V> *s_pr = reinterpret_cast<PSmem<V> *>(s_raw + ((sizeof(V) * 2 * m.nsec + 15) & ~(size_t)15));
    const double *par = params + (size_t)blockIdx.x * maxparam;
    for (int i = tid; i < m.nsec; i += nth) psi[i] = i == m.ref_i ? v_one_of<V>() : v_zero(V());
    p_angles(m.fwd, par, 1, s_pr);
    __syncthreads();
    p_run<false, V>(m.fwd, s_pr, psi, (V *)nullptr, nullptr, 1, 0);
    __syncthreads();
    const double e = p_hpsi<V>(m, psi, sig, s_red);
    if (tid == 0) energy[blockIdx.x] = e;
    if (!it.y || m.nparam == 0) return;
    __syncthreads();  // every thread is done with the forward angles and sigma
    p_angles(m.sweep, par, -1, s_pr);
    __syncthreads();
    double2 *pp = partial + (size_t)blockIdx.x * max_rows * nw;
    p_run<true, V>(m.sweep, s_pr, psi, sig, pp, 1, 0);
    __syncthreads();  // this CTA's partials are visible to all its threads
    double *g = grad + (size_t)blockIdx.x * maxparam;
    for (int mu = tid; mu < m.nparam; mu += nth) {
        const int2 r = m.psteps[mu];
        double acc = 0.0;
        for (int s = r.x; s < r.y; ++s)
            for (int c = 0; c < nw; ++c) acc += pp[(size_t)s * nw + c].x;
        g[mu] = 2.0 * acc;
    }
}

// Shared-memory bytes of the kernels for a sector of nsec amplitudes:
// states, then the record angles, then the record ring.
inline size_t sector_smem_states(size_t nstates, size_t nsec, bool real) {
    return ((nstates * nsec * (real ? 8 : 16)) + 15) & ~(size_t)15;
}

}  // namespace qfbs
