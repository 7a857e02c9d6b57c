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
// barrier per program step and no global traffic besides the H rows and one
// save of psi and sigma between the kernels.
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
// sigma(j0) = (-1)^popcount(j0 & zbase).  The arithmetic on each pair is that
// of the full-space kernels (givens_pair and the gradient inner product).
#pragma once

#include <cstdint>

namespace qfbs {

struct SEntry {  // one string of an alpha or beta list
    uint16_t r0, r1;  // rank, partner's rank
    uint32_t s;       // parity of string & zbase
};

// A step record: the 16-byte header, the patterns, then the entries of their
// lists, contiguous so that one cooperative copy brings a whole step into
// shared memory.  Records run in the order a kernel executes them.
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
    int maxw;             // longest record (words), <= block size
};

struct SLaunch {
    int nsec, nbeta, ref_i, nparam;
    SStream fwd, sweep;
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
template <class V>
__device__ __forceinline__ void s_givens(V &v0, V &v1, double c, double s, double2 gn, double2 hn) {
    const V a = v_mul(hn, v1), b = v_mul(gn, v0);
    const V n0 = v_lin(c, v0, s, a);
    v1 = v_lin(c, v1, s, b);
    v0 = n0;
}

// One record on the compact states: rotation of v (and w when TWO) by the
// angle whose cos / sin is csn, and / or the inner product <w|K|v> of the
// step's generator into acc.  rec is the record in shared memory.
template <bool ROT, bool IP, bool TWO, class V>
__device__ __forceinline__ void s_record(const uint4 *rec, int nbeta, double2 csn, V *v, V *w,
                                         double2 &acc) {
    const RHead hd = *reinterpret_cast<const RHead *>(rec);
    const RPat *pats = reinterpret_cast<const RPat *>(rec + 1);
    const SEntry *ents = reinterpret_cast<const SEntry *>(rec);
    const int np = hd.npf & 255;
    const double cs = csn.x, sn = csn.y;
    for (int p = 0; p < np; ++p) {
        const RPat pt = pats[p];
        const int total = (int)pt.na * (int)pt.nb;
        for (int q = threadIdx.x; q < total; q += blockDim.x) {
            const int ai = pt.inv ? (int)__umulhi((uint32_t)q, pt.inv) : q;
            const int bi = q - ai * (int)pt.nb;
            const SEntry ea = ents[pt.a0 + ai], eb = ents[pt.b0 + bi];
            const int i0 = (int)ea.r0 * nbeta + (int)eb.r0, i1 = (int)ea.r1 * nbeta + (int)eb.r1;
            const bool neg = (ea.s ^ eb.s) & 1u;
            V v0 = v[i0], v1 = v[i1];
            if (IP) {
                const V w0 = w[i0], w1 = w[i1];
                const double2 t = s_cadd(v_cj(w0, v_mul(pt.hn, v1)), v_cj(w1, v_mul(pt.gn, v0)));
                const double gs = neg ? -hd.gamma : hd.gamma;
                acc.x += gs * t.x;
                acc.y += gs * t.y;
            }
            if (ROT) {
                const double ss = neg ? -sn : sn;
                s_givens(v0, v1, cs, ss, pt.gn, pt.hn);
                v[i0] = v0;
                v[i1] = v1;
                if (TWO) {
                    V w0 = w[i0], w1 = w[i1];
                    s_givens(w0, w1, cs, ss, pt.gn, pt.hn);
                    w[i0] = w0;
                    w[i1] = w1;
                }
            }
        }
    }
}

__device__ __forceinline__ double2 s_warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// cos and sin of sign * gamma * theta of every record of a stream, into s_cs
__device__ __forceinline__ void s_angles(const SStream &S, const double *par, int sign,
                                         double2 *s_cs) {
    for (int r = threadIdx.x; r < S.n; r += blockDim.x) {
        const RHead hd = *reinterpret_cast<const RHead *>(S.rec + S.span[r].x);
        double sn, cs;
        sincos((double)sign * hd.gamma * par[S.param[r]], &sn, &cs);
        s_cs[r] = make_double2(cs, sn);
    }
}

// Run a stream: record r + 2 is copied from global memory into registers
// while record r is applied from shared memory (three buffers of maxw words
// at s_rec), and stored after it; one barrier per record.
template <bool SWEEP, class V>
__device__ __forceinline__ void s_run(const SLaunch &L, const SStream &S, const double2 *s_cs,
                                      uint4 *s_rec, V *v, V *w) {
    const int tid = threadIdx.x, nw = blockDim.x >> 5;
    for (int r = 0; r < 2 && r < S.n; ++r) {
        const int2 sp = S.span[r];
        if (tid < sp.y) s_rec[r * S.maxw + tid] = S.rec[sp.x + tid];
    }
    __syncthreads();
    for (int r = 0; r < S.n; ++r) {
        uint4 nxt = make_uint4(0, 0, 0, 0);
        bool have = false;
        if (r + 2 < S.n) {
            const int2 sp = S.span[r + 2];
            have = tid < sp.y;
            if (have) nxt = S.rec[sp.x + tid];
        }
        const uint4 *rec = s_rec + (r % 3) * S.maxw;
        const int npf = reinterpret_cast<const RHead *>(rec)->npf;
        const int fl = npf >> 8;
        double2 acc = make_double2(0.0, 0.0);
        if (!SWEEP) {
            s_record<true, false, false, V>(rec, L.nbeta, s_cs[r], v, nullptr, acc);
        } else if (fl == (R_ROT | R_IP | R_TWO)) {
            s_record<true, true, true, V>(rec, L.nbeta, s_cs[r], v, w, acc);
        } else if (fl == R_IP) {
            s_record<false, true, false, V>(rec, L.nbeta, s_cs[r], v, w, acc);
        } else {
            s_record<true, false, true, V>(rec, L.nbeta, s_cs[r], v, w, acc);
        }
        if (SWEEP && (fl & R_IP)) {
            acc = s_warp_sum(acc);
            const int row = reinterpret_cast<const RHead *>(rec)->row;
            if ((tid & 31) == 0)
                L.partial[((size_t)row * gridDim.x + blockIdx.x) * nw + (tid >> 5)] = acc;
        }
        if (have) s_rec[((r + 2) % 3) * S.maxw + tid] = nxt;
        __syncthreads();
    }
}

constexpr int kRowUnroll = 8;  // H row entries in flight per lane

// The evaluation runs as three kernels, one CTA per parameter set
// (blockIdx.x) each: the forward program (psi in shared memory), sigma = H psi
// with the energy (psi in shared memory, sigma rows straight to the save
// buffer), and the reverse sweep (psi and sigma in shared memory).  The
// first two hold one state and fit two CTAs per SM.  Shared memory: the
// states, then the cos / sin of every record's angle, then the record ring.

template <class V>
__global__ void __launch_bounds__(512, 2) k_sector_forward(SLaunch L) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw);
    double2 *s_cs = reinterpret_cast<double2 *>(s_raw + ((sizeof(V) * L.nsec + 15) & ~(size_t)15));
    uint4 *s_rec = reinterpret_cast<uint4 *>(s_cs + L.fwd.n);
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    for (int i = tid; i < L.nsec; i += nth) psi[i] = v_zero(V());
    s_angles(L.fwd, par, 1, s_cs);
    __syncthreads();
    if (tid == 0) v_one(psi[L.ref_i]);
    s_run<false, V>(L, L.fwd, s_cs, s_rec, psi, (V *)nullptr);
    V *sv = reinterpret_cast<V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < L.nsec; i += nth) sv[i] = psi[i];
}

template <bool REAL, class V>
__global__ void __launch_bounds__(512, 2) k_sector_h(SLaunch L) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ double2 s_red[32];
    V *psi = reinterpret_cast<V *>(s_raw);
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    V *sv = reinterpret_cast<V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < L.nsec; i += nth) psi[i] = sv[i];
    __syncthreads();
    // one warp per row, kRowUnroll entries in flight per lane
    const int lane = tid & 31, nw = nth >> 5;
    double2 en = make_double2(0.0, 0.0);
    for (int i = tid >> 5; i < L.nsec; i += nw) {
        V acc = v_zero(V());
        const int e1 = L.rowptr[i + 1];
        for (int e0 = L.rowptr[i] + lane; e0 < e1; e0 += 32 * kRowUnroll) {
            uint32_t c[kRowUnroll];
            double fr[REAL ? kRowUnroll : 1];
            double2 fc[REAL ? 1 : kRowUnroll];
#pragma unroll
            for (int u = 0; u < kRowUnroll; ++u) {
                const int e = e0 + 32 * u;
                c[u] = (e < e1) ? __ldg(&L.col[e]) : 0u;
                if (REAL) fr[u] = (e < e1) ? __ldg(&L.val_r[e]) : 0.0;
                else fc[REAL ? 0 : u] = (e < e1) ? __ldg(&L.val_c[e]) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < kRowUnroll; ++u) {
                const V x = psi[c[u]];
                if constexpr (REAL) {
                    v_acc(acc, fr[u], x);
                } else {
                    acc = v_add(acc, v_mul(fc[REAL ? 0 : u], x));
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc = v_add(acc, v_shfl_down(acc, o));
        if (lane == 0) {
            sv[L.nsec + i] = acc;
            en = s_cadd(en, v_cj(psi[i], acc));
        }
    }
    if (lane == 0) s_red[tid >> 5] = en;
    __syncthreads();
    if (tid == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int k = 0; k < nw; ++k) t = s_cadd(t, s_red[k]);
        L.energy[b] = t.x;
    }
}

template <class V>
__global__ void __launch_bounds__(512, 2) k_sector_sweep(SLaunch L) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw), *sig = psi + L.nsec;
    double2 *s_cs = reinterpret_cast<double2 *>(s_raw + ((sizeof(V) * 2 * L.nsec + 15) & ~(size_t)15));
    uint4 *s_rec = reinterpret_cast<uint4 *>(s_cs + L.sweep.n);
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < 2 * L.nsec; i += nth) psi[i] = sv[i];
    s_angles(L.sweep, par, -1, s_cs);
    __syncthreads();
    s_run<true, V>(L, L.sweep, s_cs, s_rec, psi, sig);
}

// PQE residuals on the compact states: sigma of slot blockIdx.x from the save
// buffer, U^dagger applied to it in shared memory (stream R: the forward
// records in reverse order, angles negated), then
// res[b][k] = Re(sigma[idx[k]] * phase[k]) (0 where idx[k] < 0).
template <class V>
__global__ void __launch_bounds__(512, 2) k_sector_resid(SLaunch L, SStream R,
                                                         const int64_t *__restrict__ idx,
                                                         const double2 *__restrict__ phase,
                                                         int nres, double *__restrict__ res) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *sig = reinterpret_cast<V *>(s_raw);
    double2 *s_cs = reinterpret_cast<double2 *>(s_raw + ((sizeof(V) * L.nsec + 15) & ~(size_t)15));
    uint4 *s_rec = reinterpret_cast<uint4 *>(s_cs + R.n);
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec + L.nsec;
    for (int i = tid; i < L.nsec; i += nth) sig[i] = sv[i];
    s_angles(R, par, -1, s_cs);
    __syncthreads();
    s_run<false, V>(L, R, s_cs, s_rec, sig, (V *)nullptr);
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
// blockIdx.x + gridDim.x, ... of the pool stream (records leave the states
// unchanged, so CTAs share none).
template <class V>
__global__ void __launch_bounds__(512, 2) k_sector_pool(SLaunch L, SStream P) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *psi = reinterpret_cast<V *>(s_raw), *sig = psi + L.nsec;
    uint4 *s_rec = reinterpret_cast<uint4 *>(s_raw + ((sizeof(V) * 2 * L.nsec + 15) & ~(size_t)15));
    const int b = blockIdx.y, tid = threadIdx.x, nth = blockDim.x, nw = nth >> 5;
    const V *sv = reinterpret_cast<const V *>(L.save) + (size_t)b * 2 * L.nsec;
    for (int i = tid; i < 2 * L.nsec; i += nth) psi[i] = sv[i];
    for (int r = blockIdx.x; r < P.n; r += gridDim.x) {
        const int2 sp = P.span[r];
        if (tid < sp.y) s_rec[tid] = P.rec[sp.x + tid];
        __syncthreads();
        double2 acc = make_double2(0.0, 0.0);
        s_record<false, true, false, V>(s_rec, L.nbeta, make_double2(1.0, 0.0), psi, sig, acc);
        acc = s_warp_sum(acc);
        const int row = reinterpret_cast<const RHead *>(s_rec)->row;
        if ((tid & 31) == 0)
            L.partial[((size_t)row * gridDim.y + b) * nw + (tid >> 5)] = acc;
        __syncthreads();
    }
}

// Shared-memory bytes of the kernels for a sector of nsec amplitudes:
// states, then the record angles, then the record ring.
inline size_t sector_smem_states(size_t nstates, size_t nsec, bool real) {
    return ((nstates * nsec * (real ? 8 : 16)) + 15) & ~(size_t)15;
}

}  // namespace qfbs
