// Compact particle-number sector evaluator with the states in global memory.
//
// For sectors too large for one CTA's shared memory (18-26 qubits at half
// filling: 15,876 to 2.9 M amplitudes) psi and sigma of all B parameter sets
// are stored state-minor, amplitude i of slot s at [i * B + s], so the B
// slots of one amplitude are contiguous and every access below is coalesced
// across slots.  A program step is one launch over (pair, slot): the pairs
// are the alpha-list x beta-list products of the step's record (the same
// records as the shared-memory path, qfb_sector.cuh), read from global
// memory.  sigma = H psi runs one warp per output amplitude with the lanes
// over slots, from the sector's H rows, or (rows over their budget) one
// x-group of H per launch from pair records.  When H and every step are real
// the states are stored as doubles (V = double), else as complex (double2).
#pragma once

#include <cstdint>

#include "qfb_sector.cuh"

namespace qfbg {

using qfbs::RHead;
using qfbs::RPat;
using qfbs::SEntry;

struct GLaunch {
    int nsec, nbeta, B;
    int spw;                   // slots per warp: min(32, B rounded up to a power of two)
    void *psi, *sig;           // V [nsec][B]
    const double *params;      // [B][nparam]
    int nparam;
};

__device__ __forceinline__ double2 g_cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 g_cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 g_cjmul(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

using qfbs::v_add;
using qfbs::v_cj;
using qfbs::v_lin;
using qfbs::v_mul;
using qfbs::v_zero;

// One step record over (pair, slot): lane l of a warp takes slot
// group * spw + l % spw and pair sub-index l / spw.  ROT rotates psi (and
// sigma when TWO) by sign * gamma * theta_slot; IP accumulates <sigma|K|psi>
// per slot into partial[(row * B + s) * gridDim.x + blockIdx.x].
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization waits here for the grid before it in the stream (and its
// memory), then lets the grid after it begin launching, so at most two grids
// of a chain of launches are resident and the next launch's latency hides
// behind this grid's run.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void g_pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <bool ROT, bool IP, bool TWO, class V>
__global__ void __launch_bounds__(256) k_cg_step(GLaunch L, const uint4 *__restrict__ rec,
                                                 int param, int sign, int row,
                                                 double2 *__restrict__ partial) {
    g_pdl_enter();
    V *psi = reinterpret_cast<V *>(L.psi), *sig = reinterpret_cast<V *>(L.sig);
    __shared__ double2 s_acc[8][32];
    const RHead hd = *reinterpret_cast<const RHead *>(rec);
    const RPat *pats = reinterpret_cast<const RPat *>(rec + 1);
    const SEntry *ents = reinterpret_cast<const SEntry *>(rec);
    const int np = hd.npf & 255;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int per = 32 / L.spw;  // pairs per warp at a time
    const int s = blockIdx.y * L.spw + (lane % L.spw);
    const bool live = s < L.B;
    double cs = 1.0, sn = 0.0;
    if (ROT && live) sincos((double)sign * hd.gamma * L.params[(size_t)s * L.nparam + param], &sn, &cs);
    double2 acc = make_double2(0.0, 0.0);
    const int sub = lane / L.spw;
    const int stride = gridDim.x * nwarp * per;
    for (int p = 0; p < np; ++p) {
        const RPat pt = pats[p];
        const int total = (int)pt.na * (int)pt.nb;
        for (int q = (blockIdx.x * nwarp + warp) * per + sub; q < total; q += stride) {
            const int ai = pt.inv ? (int)__umulhi((uint32_t)q, pt.inv) : q;
            const int bi = q - ai * (int)pt.nb;
            const SEntry ea = ents[pt.a0 + ai], eb = ents[pt.b0 + bi];
            if (!live) continue;
            const size_t i0 = ((size_t)ea.r0 * L.nbeta + eb.r0) * L.B + s;
            const size_t i1 = ((size_t)ea.r1 * L.nbeta + eb.r1) * L.B + s;
            const bool neg = (ea.s ^ eb.s) & 1u;
            const V v0 = psi[i0], v1 = psi[i1];
            if (IP) {
                const V w0 = sig[i0], w1 = sig[i1];
                const double2 t = g_cadd(v_cj(w0, v_mul(pt.hn, v1)), v_cj(w1, v_mul(pt.gn, v0)));
                const double gs = neg ? -hd.gamma : hd.gamma;
                acc.x += gs * t.x;
                acc.y += gs * t.y;
            }
            if (ROT) {
                const double ss = neg ? -sn : sn;
                psi[i0] = v_lin(cs, v0, ss, v_mul(pt.hn, v1));
                psi[i1] = v_lin(cs, v1, ss, v_mul(pt.gn, v0));
                if (TWO) {
                    const V w0 = sig[i0], w1 = sig[i1];
                    sig[i0] = v_lin(cs, w0, ss, v_mul(pt.hn, w1));
                    sig[i1] = v_lin(cs, w1, ss, v_mul(pt.gn, w0));
                }
            }
        }
    }
    if (!IP) return;
    // lanes of one slot: l % spw equal; sum over the pair sub-index, then warps
    for (int o = L.spw; o < 32; o <<= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane < L.spw) s_acc[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < L.spw) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nwarp; ++w) t = g_cadd(t, s_acc[w][threadIdx.x]);
        const int ss = blockIdx.y * L.spw + threadIdx.x;
        if (ss < L.B) partial[((size_t)row * L.B + ss) * gridDim.x + blockIdx.x] = t;
    }
}

// Inner products of many independent records in one launch (blockIdx.z =
// record; ADAPT pool operators): partial[(row * B + s) * gridDim.x + blockIdx.x].
template <class V>
__global__ void __launch_bounds__(256) k_cg_ip_many(GLaunch L, const uint4 *__restrict__ recs,
                                                    const int2 *__restrict__ span,
                                                    double2 *__restrict__ partial) {
    const V *psi = reinterpret_cast<const V *>(L.psi), *sig = reinterpret_cast<const V *>(L.sig);
    __shared__ double2 s_acc[8][32];
    const uint4 *rec = recs + span[blockIdx.z].x;
    const RHead hd = *reinterpret_cast<const RHead *>(rec);
    const RPat *pats = reinterpret_cast<const RPat *>(rec + 1);
    const SEntry *ents = reinterpret_cast<const SEntry *>(rec);
    const int np = hd.npf & 255;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int per = 32 / L.spw, sub = lane / L.spw;
    const int s = blockIdx.y * L.spw + (lane % L.spw);
    const bool live = s < L.B;
    const int stride = gridDim.x * nwarp * per;
    double2 acc = make_double2(0.0, 0.0);
    for (int p = 0; p < np; ++p) {
        const RPat pt = pats[p];
        const int total = (int)pt.na * (int)pt.nb;
        for (int q = (blockIdx.x * nwarp + warp) * per + sub; q < total; q += stride) {
            const int ai = pt.inv ? (int)__umulhi((uint32_t)q, pt.inv) : q;
            const int bi = q - ai * (int)pt.nb;
            const SEntry ea = ents[pt.a0 + ai], eb = ents[pt.b0 + bi];
            if (!live) continue;
            const size_t i0 = ((size_t)ea.r0 * L.nbeta + eb.r0) * L.B + s;
            const size_t i1 = ((size_t)ea.r1 * L.nbeta + eb.r1) * L.B + s;
            const V v0 = psi[i0], v1 = psi[i1], w0 = sig[i0], w1 = sig[i1];
            const double2 t = g_cadd(v_cj(w0, v_mul(pt.hn, v1)), v_cj(w1, v_mul(pt.gn, v0)));
            const double gs = ((ea.s ^ eb.s) & 1u) ? -hd.gamma : hd.gamma;
            acc.x += gs * t.x;
            acc.y += gs * t.y;
        }
    }
    for (int o = L.spw; o < 32; o <<= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane < L.spw) s_acc[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < L.spw) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nwarp; ++w) t = g_cadd(t, s_acc[w][threadIdx.x]);
        const int ss = blockIdx.y * L.spw + threadIdx.x;
        if (ss < L.B) partial[((size_t)hd.row * L.B + ss) * gridDim.x + blockIdx.x] = t;
    }
}

// psi = |ref> in every slot (psi zeroed beforehand).
template <class V>
__global__ void k_cg_ref(GLaunch L, int ref_i) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < L.B) qfbs::v_one(reinterpret_cast<V *>(L.psi)[(size_t)ref_i * L.B + s]);
}

// sigma = H psi from the sector's H rows: one warp per output row i, lanes
// over (slot, entry sub-index) as in k_cg_step; energy partials per slot.
// epart[s * gridDim.x + blockIdx.x] = sum over this block's rows of conj(psi) sigma.
template <bool REAL, class V>
__global__ void __launch_bounds__(256) k_cg_h_rows(GLaunch L, const int32_t *__restrict__ rowptr,
                                                   const uint32_t *__restrict__ col,
                                                   const double *__restrict__ val_r,
                                                   const double2 *__restrict__ val_c,
                                                   double2 *__restrict__ epart) {
    const V *psi = reinterpret_cast<const V *>(L.psi);
    V *sig = reinterpret_cast<V *>(L.sig);
    __shared__ double2 s_e[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int per = 32 / L.spw, sub = lane / L.spw;
    const int s = blockIdx.y * L.spw + (lane % L.spw);
    const bool live = s < L.B;
    double2 en = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * nwarp + warp; i < L.nsec; i += gridDim.x * nwarp) {
        V acc = v_zero(V());
        const int e1 = rowptr[i + 1];
        for (int e = rowptr[i] + sub; e < e1; e += per) {
            const uint32_t c = __ldg(&col[e]);
            const V x = live ? psi[(size_t)c * L.B + s] : v_zero(V());
            if constexpr (REAL) {
                qfbs::v_acc(acc, __ldg(&val_r[e]), x);
            } else {
                acc = v_add(acc, v_mul(__ldg(&val_c[e]), x));
            }
        }
        for (int o = L.spw; o < 32; o <<= 1) acc = v_add(acc, qfbs::v_shfl_down(acc, o));
        if (sub == 0 && live) {
            sig[(size_t)i * L.B + s] = acc;
            en = g_cadd(en, v_cj(psi[(size_t)i * L.B + s], acc));
        }
    }
    if (lane < L.spw) s_e[warp][lane] = en;
    __syncthreads();
    if (threadIdx.x < L.spw) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nwarp; ++w) t = g_cadd(t, s_e[w][threadIdx.x]);
        const int ss = blockIdx.y * L.spw + threadIdx.x;
        if (ss < L.B) epart[(size_t)ss * gridDim.x + blockIdx.x] = t;
    }
}

// Bits 0, 2, 4, ... (odd = 0) or 1, 3, 5, ... (odd = 1) of v, packed.
__device__ __forceinline__ uint32_t g_pext_parity(uint64_t v, int odd) {
    uint64_t x = (v >> odd) & 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x >> 4)) & 0x00ff00ff00ff00ffull;
    x = (x | (x >> 8)) & 0x0000ffff0000ffffull;
    x = (x | (x >> 16)) & 0x00000000ffffffffull;
    return (uint32_t)x;
}

struct GGroup {  // one x-group of H restricted to the sector (layout of SecGroup)
    uint64_t x;
    int32_t begin, end, real;
    int32_t halves;
};

struct GTerm {  // one term of a grouped sum (layout of TermDev)
    uint64_t z;
    double2 c;
};

// ---- H psi without stored rows: H as one pair record per x-group ----------
//
// Within one x-group of H (terms c_t P_t sharing x), the sector indices the
// group connects come in pairs (i0, i1 = i0 ^ x on the determinants), i0 the
// one with x's highest bit clear, and each sector index is in at most one
// pair.  The group's record lists them as alpha list x beta list per
// pattern of the determinant's bits at the group's pattern positions; the
// kernels below add H_g psi into sigma one group per launch, so no two
// threads of a launch touch one sigma entry (groups launched concurrently add
// into separate sigma copies, summed afterwards).

// sigma = f psi per row, f = sum_t c_t (-1)^popcount(det & z_t) over the
// diagonal group's terms [t0, t1) (one warp per row, terms over the lanes);
// every slot of the row.  This is the first H kernel: it writes sigma.
template <class V>
__global__ void __launch_bounds__(256) k_cg_h_diag(GLaunch L, const uint64_t *__restrict__ det,
                                                   const GTerm *__restrict__ terms,
                                                   const double2 *__restrict__ rterms, int t0,
                                                   int t1, int real) {
    const V *psi = reinterpret_cast<const V *>(L.psi);
    V *sig = reinterpret_cast<V *>(L.sig);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int i = blockIdx.x * nwarp + warp; i < L.nsec; i += gridDim.x * nwarp) {
        const uint64_t k = det[i];
        double2 f = make_double2(0.0, 0.0);
        if (real) {
            for (int t = t0 + lane; t < t1; t += 32) {
                const double2 zc = __ldg(&rterms[t]);
                f.x += (__popcll(k & (uint64_t)__double_as_longlong(zc.x)) & 1) ? -zc.y : zc.y;
            }
        } else {
            for (int t = t0 + lane; t < t1; t += 32) {
                const double2 c = __ldg(&terms[t].c);
                if (__popcll(k & __ldg(&terms[t].z)) & 1) { f.x -= c.x; f.y -= c.y; }
                else { f.x += c.x; f.y += c.y; }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            f.x += __shfl_xor_sync(0xffffffffu, f.x, o);
            f.y += __shfl_xor_sync(0xffffffffu, f.y, o);
        }
        for (int s = lane; s < L.B; s += 32)
            sig[(size_t)i * L.B + s] = v_mul(f, psi[(size_t)i * L.B + s]);
    }
}

// sig[i] += sum over c < ncopies of copies[c * n + i] (in copy order)
template <class V>
__global__ void __launch_bounds__(256) k_cg_add_copies(V *__restrict__ sig, const V *__restrict__ copies,
                                                       size_t n, int ncopies) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        V t = sig[i];
        for (int c = 0; c < ncopies; ++c) t = v_add(t, copies[(size_t)c * n + i]);
        sig[i] = t;
    }
}

// sigma += H_g psi for one x-group.  TABLE: per pattern, sigma[i1] +=
// sgn gn psi[i0] and sigma[i0] += sgn hn psi[i1] with sgn = (-1)^(ea.s ^ eb.s)
// (the sign of the group's first z-mask on i0's determinant).  Otherwise the
// two matrix elements are summed per pair from the group's terms [t0, t1):
// H[i1][i0] = sum_t c_t (-1)^popcount(j0 & z_t), H[i0][i1] the same at
// j1 = j0 ^ x.  Lanes over (pair, slot) as in k_cg_step.
template <bool TABLE, class V>
__global__ void __launch_bounds__(256) k_cg_h_group(GLaunch L, const uint4 *__restrict__ rec,
                                                    const uint64_t *__restrict__ det,
                                                    const GTerm *__restrict__ terms,
                                                    const double2 *__restrict__ rterms, int t0,
                                                    int t1, int real, uint64_t x) {
    g_pdl_enter();
    const V *psi = reinterpret_cast<const V *>(L.psi);
    V *sig = reinterpret_cast<V *>(L.sig);
    const RHead hd = *reinterpret_cast<const RHead *>(rec);
    const RPat *pats = reinterpret_cast<const RPat *>(rec + 1);
    const SEntry *ents = reinterpret_cast<const SEntry *>(rec);
    const int np = hd.npf & 255;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int per = 32 / L.spw;
    const int s = blockIdx.y * L.spw + (lane % L.spw);
    const bool live = s < L.B;
    const int sub = lane / L.spw;
    const int stride = gridDim.x * nwarp * per;
    for (int p = 0; p < np; ++p) {
        const RPat pt = pats[p];
        const int total = (int)pt.na * (int)pt.nb;
        for (int q = (blockIdx.x * nwarp + warp) * per + sub; q < total; q += stride) {
            const int ai = pt.inv ? (int)__umulhi((uint32_t)q, pt.inv) : q;
            const int bi = q - ai * (int)pt.nb;
            const SEntry ea = ents[pt.a0 + ai], eb = ents[pt.b0 + bi];
            if (!live) continue;
            const size_t c0 = (size_t)ea.r0 * L.nbeta + eb.r0, c1 = (size_t)ea.r1 * L.nbeta + eb.r1;
            double2 k10, k01;
            if (TABLE) {
                const bool neg = (ea.s ^ eb.s) & 1u;
                k10 = neg ? make_double2(-pt.gn.x, -pt.gn.y) : pt.gn;
                k01 = neg ? make_double2(-pt.hn.x, -pt.hn.y) : pt.hn;
            } else {
                const uint64_t j0 = det[c0], j1 = j0 ^ x;
                k10 = make_double2(0.0, 0.0);
                k01 = make_double2(0.0, 0.0);
                if (real) {
                    for (int t = t0; t < t1; ++t) {
                        const double2 zc = __ldg(&rterms[t]);
                        const uint64_t z = (uint64_t)__double_as_longlong(zc.x);
                        k10.x += (__popcll(j0 & z) & 1) ? -zc.y : zc.y;
                        k01.x += (__popcll(j1 & z) & 1) ? -zc.y : zc.y;
                    }
                } else {
                    for (int t = t0; t < t1; ++t) {
                        const double2 c = __ldg(&terms[t].c);
                        const uint64_t z = __ldg(&terms[t].z);
                        if (__popcll(j0 & z) & 1) { k10.x -= c.x; k10.y -= c.y; }
                        else { k10.x += c.x; k10.y += c.y; }
                        if (__popcll(j1 & z) & 1) { k01.x -= c.x; k01.y -= c.y; }
                        else { k01.x += c.x; k01.y += c.y; }
                    }
                }
            }
            const size_t i0 = c0 * L.B + s, i1 = c1 * L.B + s;
            const V v0 = psi[i0], v1 = psi[i1];
            sig[i1] = v_add(sig[i1], v_mul(k10, v0));
            sig[i0] = v_add(sig[i0], v_mul(k01, v1));
        }
    }
}

// epart[s * gridDim.x + blockIdx.x] = this block's share of <psi_s|sigma_s>.
template <class V>
__global__ void __launch_bounds__(256) k_cg_dot(GLaunch L, double2 *__restrict__ epart) {
    const V *psi = reinterpret_cast<const V *>(L.psi), *sig = reinterpret_cast<const V *>(L.sig);
    __shared__ double2 s_e[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int per = 32 / L.spw, sub = lane / L.spw;
    const int s = blockIdx.y * L.spw + (lane % L.spw);
    double2 acc = make_double2(0.0, 0.0);
    if (s < L.B)
        for (int i = (blockIdx.x * nwarp + warp) * per + sub; i < L.nsec; i += gridDim.x * nwarp * per)
            acc = g_cadd(acc, v_cj(psi[(size_t)i * L.B + s], sig[(size_t)i * L.B + s]));
    for (int o = L.spw; o < 32; o <<= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane < L.spw) s_e[warp][lane] = acc;
    __syncthreads();
    if (threadIdx.x < L.spw) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nwarp; ++w) t = g_cadd(t, s_e[w][threadIdx.x]);
        const int ss = blockIdx.y * L.spw + threadIdx.x;
        if (ss < L.B) epart[(size_t)ss * gridDim.x + blockIdx.x] = t;
    }
}

// energy[s] = Re sum_k epart[s * n + k]  (one warp per slot, fixed order)
__global__ void k_cg_energy(const double2 *__restrict__ epart, int n, int B,
                            double *__restrict__ energy) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= B) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = lane; k < n; k += 32) acc = g_cadd(acc, epart[(size_t)s * n + k]);
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane == 0) energy[s] = acc.x;
}

}  // namespace qfbg
