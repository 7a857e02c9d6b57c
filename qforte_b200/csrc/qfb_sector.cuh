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
// barrier per program step and no global traffic besides the H rows.
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

struct SPat {  // the pairs of one active pattern of a step
    int32_t a0, na;  // alpha list entries [a0, a0 + na)
    int32_t b0, nb;  // beta list entries [b0, b0 + nb)
    double2 gn, hn;
};

struct SStep {
    int32_t p0, np;  // patterns [p0, p0 + np)
    int32_t param;
    int32_t pad;
    double gamma;
};

struct SLaunch {
    int nsec, nbeta, ref_i, nparam;
    int nf, fused, nmu, mode;  // mode bit 0: forward + H (else load), bit 1: sweep, bit 2: save
    const SStep *fsteps;       // forward program
    const SStep *ksteps;       // K program (inner products); partial row = K step index
    const SStep *usteps;       // U program (un-rotation)
    const int2 *kmu, *umu;     // steps of each parameter in the K and U programs
    const SPat *pats;
    const SEntry *ents;
    const int32_t *rowptr;     // H rows
    const uint32_t *col;
    const double *val_r;       // real H (val_c == nullptr) ...
    const double2 *val_c;      // ... or complex
    const double *params;      // [B][nparam]
    double *energy;            // [B]
    double2 *partial;          // [K steps][B][warps]
    double2 *save;             // [B][2][nsec]: psi, sigma after H
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

// new0 = c v0 + s hn v1, new1 = c v1 + s gn v0 (as givens_pair)
__device__ __forceinline__ void s_givens(double2 &v0, double2 &v1, double c, double s, double2 gn,
                                         double2 hn) {
    const double2 a = s_cmul(hn, v1), b = s_cmul(gn, v0);
    const double2 n0 = make_double2(c * v0.x + s * a.x, c * v0.y + s * a.y);
    v1 = make_double2(c * v1.x + s * b.x, c * v1.y + s * b.y);
    v0 = n0;
}

// One step on the compact states: rotation by sign * gamma * theta (rot),
// and / or the inner product <w|K|v> of the step's generator (acc).
template <bool ROT, bool IP, bool TWO>
__device__ __forceinline__ void s_step(const SLaunch &L, const SStep &st, double theta, int sign,
                                       double2 *v, double2 *w, double2 &acc) {
    double sn = 0.0, cs = 1.0;
    if (ROT) sincos((double)sign * st.gamma * theta, &sn, &cs);
    const int nb = L.nbeta;
    for (int p = st.p0; p < st.p0 + st.np; ++p) {
        const SPat pt = L.pats[p];
        const int total = pt.na * pt.nb;
        for (int q = threadIdx.x; q < total; q += blockDim.x) {
            const int ai = q / pt.nb, bi = q - ai * pt.nb;
            const SEntry ea = L.ents[pt.a0 + ai], eb = L.ents[pt.b0 + bi];
            const int i0 = (int)ea.r0 * nb + (int)eb.r0, i1 = (int)ea.r1 * nb + (int)eb.r1;
            const bool neg = (ea.s ^ eb.s) & 1u;
            double2 v0 = v[i0], v1 = v[i1];
            if (IP) {
                const double2 w0 = w[i0], w1 = w[i1];
                const double2 t = s_cadd(s_cjmul(w0, s_cmul(pt.hn, v1)), s_cjmul(w1, s_cmul(pt.gn, v0)));
                const double gs = neg ? -st.gamma : st.gamma;
                acc.x += gs * t.x;
                acc.y += gs * t.y;
            }
            if (ROT) {
                const double ss = neg ? -sn : sn;
                s_givens(v0, v1, cs, ss, pt.gn, pt.hn);
                v[i0] = v0;
                v[i1] = v1;
                if (TWO) {
                    double2 w0 = w[i0], w1 = w[i1];
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

// Per-warp share of an inner product, written to partial[row][b][warp].
__device__ __forceinline__ void s_flush(const SLaunch &L, int row, double2 acc) {
    acc = s_warp_sum(acc);
    const int nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0)
        L.partial[((size_t)row * gridDim.x + blockIdx.x) * nw + (threadIdx.x >> 5)] = acc;
}

// One CTA per parameter set (blockIdx.x); psi and sigma in shared memory.
__global__ void __launch_bounds__(512) k_sector_eval(SLaunch L) {
    extern __shared__ double2 s_mem[];
    __shared__ double2 s_red[32];
    double2 *psi = s_mem, *sig = s_mem + L.nsec;
    const int b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const double *par = L.params + (size_t)b * L.nparam;
    double2 *sv = L.save + (size_t)b * 2 * L.nsec;
    double2 dummy = make_double2(0.0, 0.0);
    if (L.mode & 1) {
        for (int i = tid; i < L.nsec; i += nth) psi[i] = make_double2(0.0, 0.0);
        __syncthreads();
        if (tid == 0) psi[L.ref_i] = make_double2(1.0, 0.0);
        __syncthreads();
        for (int s = 0; s < L.nf; ++s) {
            const SStep st = L.fsteps[s];
            s_step<true, false, false>(L, st, par[st.param], 1, psi, nullptr, dummy);
            __syncthreads();
        }
        // sigma = H psi: one warp per row
        const int lane = tid & 31, nw = nth >> 5;
        for (int i = tid >> 5; i < L.nsec; i += nw) {
            double2 acc = make_double2(0.0, 0.0);
            const int e1 = L.rowptr[i + 1];
            if (L.val_c) {
                for (int e = L.rowptr[i] + lane; e < e1; e += 32)
                    acc = s_cadd(acc, s_cmul(__ldg(&L.val_c[e]), psi[__ldg(&L.col[e])]));
            } else {
                for (int e = L.rowptr[i] + lane; e < e1; e += 32) {
                    const double f = __ldg(&L.val_r[e]);
                    const double2 x = psi[__ldg(&L.col[e])];
                    acc.x += f * x.x;
                    acc.y += f * x.y;
                }
            }
            acc = s_warp_sum(acc);
            if (lane == 0) sig[i] = acc;
        }
        __syncthreads();
        double2 e = make_double2(0.0, 0.0);
        for (int i = tid; i < L.nsec; i += nth) e = s_cadd(e, s_cjmul(psi[i], sig[i]));
        e = s_warp_sum(e);
        if ((tid & 31) == 0) s_red[tid >> 5] = e;
        __syncthreads();
        if (tid == 0) {
            double2 t = make_double2(0.0, 0.0);
            for (int k = 0; k < (nth >> 5); ++k) t = s_cadd(t, s_red[k]);
            L.energy[b] = t.x;
        }
        if (L.mode & 4)
            for (int i = tid; i < 2 * L.nsec; i += nth) sv[i] = s_mem[i];
    } else {
        for (int i = tid; i < 2 * L.nsec; i += nth) s_mem[i] = sv[i];
    }
    __syncthreads();
    if (!(L.mode & 2)) return;
    for (int mu = L.nmu - 1; mu >= 0; --mu) {
        const double th = par[mu];
        const int2 kr = L.kmu[mu];
        if (L.fused) {
            double2 acc = make_double2(0.0, 0.0);
            const SStep st = L.ksteps[kr.x];
            if (mu > 0)
                s_step<true, true, true>(L, st, th, -1, psi, sig, acc);
            else
                s_step<false, true, false>(L, st, th, -1, psi, sig, acc);
            s_flush(L, kr.x, acc);
            __syncthreads();
            continue;
        }
        for (int s = kr.x; s < kr.y; ++s) {
            double2 acc = make_double2(0.0, 0.0);
            s_step<false, true, false>(L, L.ksteps[s], th, -1, psi, sig, acc);
            s_flush(L, s, acc);
        }
        __syncthreads();
        if (mu == 0) break;
        const int2 ur = L.umu[mu];
        for (int s = ur.x; s < ur.y; ++s) {
            const SStep st = L.usteps[s];
            s_step<true, false, true>(L, st, par[st.param], -1, psi, sig, dummy);
            __syncthreads();
        }
    }
}

}  // namespace qfbs
