// libqfb.so: grouped Pauli sums and Pauli-exponential programs.
//
// Pauli algebra on basis states (mask form, qfb.h):
//   P|j> = i^ny (-1)^popcount(j & z) |j ^ x>,   ny = popcount(x & z).
//
// Grouped sums (qfb_sum_*).  The reference evaluates sum_t c_t P_t one term at a
// time: a state copy, the term's gates, a scale and an accumulation per term
// (Computer::apply_operator, computer.cc:80-91; direct_op_exp_val :753-771).
// Here the terms are grouped by x on the host; within a group all terms pair
// amplitude j with j ^ x, so for each pair one read of the two amplitudes
// serves every term of the group:
//   f_x(j) = sum_{t in x} c_t i^ny_t (-1)^popcount(j & z_t)
//   <bra|O|ket> = sum_x sum_j conj(bra[j ^ x]) f_x(j) ket[j]
//   (O ket)[k]  = sum_x f_x(k ^ x) ket[k ^ x]
// f_x(j ^ x) differs from f_x(j) only by (-1)^popcount(x & z_t) per term, so a
// pair costs one parity per term.  Groups whose coefficients c_t i^ny_t are all
// real (every Hamiltonian built from real integrals) take a real-arithmetic path.
//
// Programs (qfb_prog_*).  exp(i phi P) acts on each pair (j, j ^ x) as
//   new_j     = cos(phi) psi_j     + i sin(phi) ph(j ^ x) psi_{j^x}
//   new_{j^x} = cos(phi) psi_{j^x} + i sin(phi) ph(j)     psi_j
// with ph(j) = i^ny (-1)^popcount(j & z) (a diagonal phase when x = 0).  This
// is the unitary that utils/exponentiate.py:9-87 builds out of 2w + 1 gates
// (basis change, CNOT ladder, Rz(-2 Im c), uncompute); here it is one pass.
// Consecutive strings sharing x map the same pairs onto themselves, so a run
// of them (all strings of one dUCC excitation) is applied in one pass with
// the rotations chained in registers.
//
// Adjoint gradient (qfb_ucc_gradient) follows UCCVQE.measure_gradient
// (uccvqeabc.py:122-251): g_mu = 2 Re <sigma_mu|K_mu|psi_mu>, then
// psi_{mu-1} = U_mu^dagger psi_mu and sigma_{mu-1} = U_mu^dagger sigma_mu.  When
// K_mu is one x-group the inner product and both un-rotations share one pass
// over (psi, sigma); no intermediate state is stored.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "qfb_common.cuh"
#include "qfb_csec.cuh"
#include "qfb_sector.cuh"
#include "qfb_window.cuh"

using namespace qfb;

namespace {

struct TermDev {  // one term of a grouped sum
    uint64_t z;
    double2 c;  // c_t * i^ny_t
};

struct GroupDev {
    uint64_t x;
    int32_t h;      // highest set bit of x, -1 when x == 0
    int32_t begin;  // first term
    int32_t end;    // one past the last term
    int32_t real;   // all term coefficients real
};

struct StrDev {  // one Pauli string of a program
    uint64_t z;
    int32_t ny;     // popcount(x & z) mod 4
    int32_t param;  // parameter index
    double scale;   // phi = scale * params[param]
};

struct StepDev {  // run of consecutive strings sharing one x (and one parameter)
    uint64_t x;
    int32_t h;
    int32_t s0;  // first string
    int32_t ns;  // number of strings
    int32_t param;
    // Givens form (tab >= 0): the strings commute and their sum K restricted
    // to each pair (j, j ^ x) is sigma(j) * [[0, gamma hn], [gamma gn, 0]]
    // with sigma(j) = (-1)^popcount(j & zbase) and (gn, hn) read from the
    // table at the pattern of j's bits at the nd positions in dpos (6 bits
    // each); exp(t K) is then a rotation by t * gamma on every active pair.
    int32_t tab;   // offset of the (gn, hn) table, in double2 entries; -1: none
    int32_t nd;
    uint64_t dpos;
    uint64_t zbase;
    double gamma;
    // Active pairs only: the na <= kMaxActive patterns with a non-zero entry,
    // as table index and bit mask; j0 = (free-bit counter with zeros inserted
    // at the nd + 1 sorted positions in zpos, 6 bits each) | patbits[a].
    int32_t na;    // -1: enumerate every pair and test the pattern
    uint8_t patidx[8];
    uint64_t zpos;
    uint64_t patbits[8];
};
constexpr int kMaxActive = 8;

constexpr int kMaxStepStrings = 64;   // strings per fused step (longer runs are split)
constexpr int kTermTile = 256;        // terms staged in shared memory at a time

int highest_bit(uint64_t x) { return x ? 63 - __builtin_clzll(x) : -1; }

// ---------------------------------------------------------------------------
// grouped sums
// ---------------------------------------------------------------------------

// partial[((b * G) + g) * gridDim.x + blockIdx.x] = this block's share of
// <bra_b | O_g | ket_b>.  grid = (chunks, G, nbatch).
__global__ void __launch_bounds__(256) k_sum_expval(
    const double2 *__restrict__ bra, const double2 *__restrict__ ket, uint64_t nbasis,
    const GroupDev *__restrict__ groups, const TermDev *__restrict__ terms, int32_t ngroups,
    double2 *__restrict__ partial) {
    __shared__ TermDev s_t[kTermTile];
    const int g = blockIdx.y;
    const uint64_t off = (uint64_t)blockIdx.z * nbasis;
    const GroupDev gr = groups[g];
    const uint64_t npair = nbasis >> 1;
    const uint64_t chunk = (npair + gridDim.x - 1) / gridDim.x;
    const uint64_t p0 = (uint64_t)blockIdx.x * chunk;
    const uint64_t p1 = min(npair, p0 + chunk);
    double2 acc = make_double2(0.0, 0.0);
    for (int tb = gr.begin; tb < gr.end; tb += kTermTile) {
        const int nt = min(kTermTile, gr.end - tb);
        __syncthreads();
        for (int i = threadIdx.x; i < nt; i += blockDim.x) s_t[i] = terms[tb + i];
        __syncthreads();
        for (uint64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            uint64_t j0, j1;
            if (gr.h >= 0) {
                j0 = insert0(p, gr.h);
                j1 = j0 ^ gr.x;
            } else {
                j0 = p << 1;
                j1 = j0 | 1ull;
            }
            const double2 a0 = ket[off + j0], a1 = ket[off + j1];
            const double2 b0 = bra[off + j0], b1 = bra[off + j1];
            if (gr.real) {
                double f0 = 0.0, f1 = 0.0;
                for (int t = 0; t < nt; ++t) {
                    const double c = s_t[t].c.x;
                    f0 += parity64(j0 & s_t[t].z) ? -c : c;
                    f1 += parity64(j1 & s_t[t].z) ? -c : c;
                }
                // x != 0: conj(b1) f0 a0 + conj(b0) f1 a1 ; x == 0: conj(b0) f0 a0 + conj(b1) f1 a1
                const double2 u = (gr.h >= 0) ? c_cjmul(b1, a0) : c_cjmul(b0, a0);
                const double2 v = (gr.h >= 0) ? c_cjmul(b0, a1) : c_cjmul(b1, a1);
                acc.x += f0 * u.x + f1 * v.x;
                acc.y += f0 * u.y + f1 * v.y;
            } else {
                double2 f0 = make_double2(0.0, 0.0), f1 = make_double2(0.0, 0.0);
                for (int t = 0; t < nt; ++t) {
                    const double2 c = s_t[t].c;
                    if (parity64(j0 & s_t[t].z)) { f0.x -= c.x; f0.y -= c.y; }
                    else { f0.x += c.x; f0.y += c.y; }
                    if (parity64(j1 & s_t[t].z)) { f1.x -= c.x; f1.y -= c.y; }
                    else { f1.x += c.x; f1.y += c.y; }
                }
                const double2 u = (gr.h >= 0) ? c_cjmul(b1, a0) : c_cjmul(b0, a0);
                const double2 v = (gr.h >= 0) ? c_cjmul(b0, a1) : c_cjmul(b1, a1);
                acc = c_add(acc, c_add(c_mul(f0, u), c_mul(f1, v)));
            }
        }
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0)
        partial[((uint64_t)blockIdx.z * ngroups + g) * gridDim.x + blockIdx.x] = acc;
}

// out[b * nseg + s] = sum of partial rows [row0[s], row0[s+1]) of batch b, each
// row `chunks` long.  grid = (nseg, nbatch).
__global__ void k_seg_sum(const double2 *__restrict__ partial, const int32_t *__restrict__ seg_g0,
                          int32_t ngroups, int32_t chunks, double2 *__restrict__ out) {
    const int s = blockIdx.x, b = blockIdx.y;
    const uint64_t r0 = ((uint64_t)b * ngroups + seg_g0[s]) * chunks;
    const uint64_t r1 = ((uint64_t)b * ngroups + seg_g0[s + 1]) * chunks;
    double2 acc = make_double2(0.0, 0.0);
    for (uint64_t k = r0 + threadIdx.x; k < r1; k += blockDim.x) acc = c_add(acc, partial[k]);
    acc = block_sum(acc);
    if (threadIdx.x == 0) out[(uint64_t)b * gridDim.x + s] = acc;
}

// dst[k] = sum_g f_g(k ^ x_g) src[k ^ x_g]; one output per thread, written once.
__global__ void __launch_bounds__(256) k_sum_apply(
    double2 *__restrict__ dst, const double2 *__restrict__ src, uint64_t nbasis,
    const GroupDev *__restrict__ groups, const TermDev *__restrict__ terms, int32_t ngroups) {
    const uint64_t off = (uint64_t)blockIdx.y * nbasis;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nbasis;
         k += (uint64_t)gridDim.x * blockDim.x) {
        double2 acc = make_double2(0.0, 0.0);
        for (int g = 0; g < ngroups; ++g) {
            const GroupDev gr = groups[g];
            const uint64_t j = k ^ gr.x;
            const double2 a = src[off + j];
            if (gr.real) {
                double f = 0.0;
                for (int t = gr.begin; t < gr.end; ++t) {
                    const double c = __ldg(&terms[t].c.x);
                    f += parity64(j & __ldg(&terms[t].z)) ? -c : c;
                }
                acc.x += f * a.x;
                acc.y += f * a.y;
            } else {
                double2 f = make_double2(0.0, 0.0);
                for (int t = gr.begin; t < gr.end; ++t) {
                    const double2 c = terms[t].c;
                    if (parity64(j & terms[t].z)) { f.x -= c.x; f.y -= c.y; }
                    else { f.x += c.x; f.y += c.y; }
                }
                acc = c_add(acc, c_mul(f, a));
            }
        }
        dst[off + k] = acc;
    }
}

// dst = O src with four outputs per thread: k = k0 | d, d = 0..3.  For a
// group x the four inputs j_d = (k0 ^ x) ^ d form one aligned quad, and
// popcount(j_d & z) = popcount((k0 ^ x) & z) + popcount(d & z): one parity per
// term serves all four outputs.  Terms are read in the real form (z, Re c)
// when the group is real.
__global__ void __launch_bounds__(256) k_sum_apply4(
    double2 *__restrict__ dst, const double2 *__restrict__ src, uint64_t nbasis,
    const GroupDev *__restrict__ groups, const TermDev *__restrict__ terms,
    const double2 *__restrict__ rterms, int32_t ngroups) {
    const uint64_t off = (uint64_t)blockIdx.y * nbasis;
    const uint64_t nquad = nbasis >> 2;
    for (uint64_t qd = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; qd < nquad;
         qd += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k0 = qd << 2;
        double2 acc0 = make_double2(0.0, 0.0), acc1 = acc0, acc2 = acc0, acc3 = acc0;
        for (int g = 0; g < ngroups; ++g) {
            const uint64_t x = __ldg(&groups[g].x);
            const int tb = __ldg(&groups[g].begin), te = __ldg(&groups[g].end);
            const int real = __ldg(&groups[g].real);
            const uint64_t base = k0 ^ x;
            const uint64_t qb = base & ~3ull;
            // a[e] = src[qb | e]; input of output d is a[d ^ (x & 3)]
            double2 a0 = src[off + qb], a1 = src[off + qb + 1];
            double2 a2 = src[off + qb + 2], a3 = src[off + qb + 3];
            if (x & 1) {
                double2 t = a0; a0 = a1; a1 = t;
                t = a2; a2 = a3; a3 = t;
            }
            if (x & 2) {
                double2 t = a0; a0 = a2; a2 = t;
                t = a1; a1 = a3; a3 = t;
            }
            if (real) {
                double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
                for (int t = tb; t < te; ++t) {
                    const double2 zc = __ldg(&rterms[t]);  // (z bits, Re c)
                    const uint64_t z = (uint64_t)__double_as_longlong(zc.x);
                    const double c = parity64(base & z) ? -zc.y : zc.y;
                    const double c1 = (z & 1) ? -c : c;
                    f0 += c;
                    f1 += c1;
                    f2 += (z & 2) ? -c : c;
                    f3 += (z & 2) ? -c1 : c1;
                }
                acc0.x += f0 * a0.x; acc0.y += f0 * a0.y;
                acc1.x += f1 * a1.x; acc1.y += f1 * a1.y;
                acc2.x += f2 * a2.x; acc2.y += f2 * a2.y;
                acc3.x += f3 * a3.x; acc3.y += f3 * a3.y;
            } else {
                double2 f0 = make_double2(0.0, 0.0), f1 = f0, f2 = f0, f3 = f0;
                for (int t = tb; t < te; ++t) {
                    const uint64_t z = __ldg(&terms[t].z);
                    double2 c = terms[t].c;
                    if (parity64(base & z)) c = make_double2(-c.x, -c.y);
                    const double2 c1 = (z & 1) ? make_double2(-c.x, -c.y) : c;
                    const double2 c2 = (z & 2) ? make_double2(-c.x, -c.y) : c;
                    const double2 c3 = (z & 2) ? make_double2(-c1.x, -c1.y) : c1;
                    f0 = c_add(f0, c); f1 = c_add(f1, c1); f2 = c_add(f2, c2); f3 = c_add(f3, c3);
                }
                acc0 = c_add(acc0, c_mul(f0, a0));
                acc1 = c_add(acc1, c_mul(f1, a1));
                acc2 = c_add(acc2, c_mul(f2, a2));
                acc3 = c_add(acc3, c_mul(f3, a3));
            }
        }
        dst[off + k0] = acc0;
        dst[off + k0 + 1] = acc1;
        dst[off + k0 + 2] = acc2;
        dst[off + k0 + 3] = acc3;
    }
}

// dst = O src over output tiles in shared memory, several states per block.
// Block (t, c) owns outputs k = t * 2^m + tid (one per thread) of states
// c * NB .. c * NB + NB - 1.  Groups are visited ordered by their high part
// x >> m: for each distinct high part the block stages the partner tile
// (the 2^m inputs k ^ x of its outputs for every x with that high part) of
// its NB states once, then every group of that high part reads its inputs
// from shared memory.  f_x(k ^ x) depends on k and x only, so it is computed
// once and applied to all NB states.
constexpr int kApplyTileBits = 8;
constexpr int kApplyStates = 16;

// IDX = uint32_t when the state has at most 32 qubits (one popcount per term).
template <typename IDX>
__global__ void __launch_bounds__(1 << kApplyTileBits, 2) k_sum_apply_tiled(
    double2 *__restrict__ dst, const double2 *__restrict__ src, uint64_t nbasis, int nbatch,
    int m, const GroupDev *__restrict__ groups, const int32_t *__restrict__ hi_g0,
    const uint64_t *__restrict__ hi_val, int nhi, const TermDev *__restrict__ terms,
    const double2 *__restrict__ rterms) {
    extern __shared__ double2 apply_smem[];
    double2(*tile)[1 << kApplyTileBits] = reinterpret_cast<double2(*)[1 << kApplyTileBits]>(apply_smem);
    const int T = 1 << m;
    const int tid = threadIdx.x;
    const uint64_t kbase = (uint64_t)blockIdx.x << m;
    const int s0 = blockIdx.y * kApplyStates;
    const int ns = min(kApplyStates, nbatch - s0);
    const IDX k = (IDX)(kbase + tid);
    double2 acc[kApplyStates];
#pragma unroll
    for (int s = 0; s < kApplyStates; ++s) acc[s] = make_double2(0.0, 0.0);
    for (int r = 0; r < nhi; ++r) {
        const uint64_t jbase = kbase ^ (hi_val[r] << m);
        __syncthreads();
        for (int s = 0; s < ns; ++s)
            for (int l = tid; l < T; l += blockDim.x)
                tile[s][l] = src[(uint64_t)(s0 + s) * nbasis + jbase + l];
        __syncthreads();
        if (tid >= T) continue;
        for (int g = hi_g0[r]; g < hi_g0[r + 1]; ++g) {
            const GroupDev gr = groups[g];
            const IDX j = k ^ (IDX)gr.x;
            const int lj = (int)(j & (IDX)(T - 1));
            if (gr.real) {
                double f = 0.0;
#pragma unroll 4
                for (int t = gr.begin; t < gr.end; ++t) {
                    const double2 zc = __ldg(&rterms[t]);
                    const IDX z = (IDX)__double_as_longlong(zc.x);
                    const int odd = (sizeof(IDX) == 4) ? (__popc((uint32_t)(j & z)) & 1)
                                                       : parity64((uint64_t)(j & z));
                    f += odd ? -zc.y : zc.y;
                }
#pragma unroll
                for (int s = 0; s < kApplyStates; ++s) {
                    if (s < ns) {
                        const double2 a = tile[s][lj];
                        acc[s].x += f * a.x;
                        acc[s].y += f * a.y;
                    }
                }
            } else {
                double2 f = make_double2(0.0, 0.0);
                for (int t = gr.begin; t < gr.end; ++t) {
                    const double2 c = terms[t].c;
                    if (parity64((uint64_t)j & __ldg(&terms[t].z))) { f.x -= c.x; f.y -= c.y; }
                    else { f.x += c.x; f.y += c.y; }
                }
#pragma unroll
                for (int s = 0; s < kApplyStates; ++s)
                    if (s < ns) acc[s] = c_add(acc[s], c_mul(f, tile[s][lj]));
            }
        }
    }
    if (tid < T) {
#pragma unroll
        for (int s = 0; s < kApplyStates; ++s)
            if (s < ns) dst[(uint64_t)(s0 + s) * nbasis + (uint64_t)k] = acc[s];
    }
}

constexpr size_t kApplySmem = sizeof(double2) * kApplyStates * (1 << kApplyTileBits);

// One x-group of a Hamiltonian restricted to a particle-number sector: an
// output index k of the sector reaches k ^ x inside the sector exactly when k
// holds half of x's alpha (even) bits and half of its beta (odd) bits.
struct SecGroup {
    uint64_t x;
    int32_t begin, end, real;
    int32_t halves;  // popcount(x & alpha) / 2 | (popcount(x & beta) / 2) << 8
};

template <typename IDX>
__device__ __forceinline__ int popc_t(IDX v) {
    return (sizeof(IDX) == 4) ? __popc((uint32_t)v) : __popcll((uint64_t)v);
}

// sigma = H psi on the amplitudes of one sector (states whose amplitudes lie
// in that sector; the caller zeroes sigma elsewhere).  One warp per output
// index k of the sector and one lane per state: the group scan and the
// coefficient sums f_x(k ^ x) are uniform across the warp, and each lane
// gathers psi[state][k ^ x] once per group that connects k inside the sector.
template <typename IDX>
__global__ void __launch_bounds__(256) k_sum_apply_sector(
    double2 *__restrict__ dst, const double2 *__restrict__ src, uint64_t nbasis, int nbatch,
    const IDX *__restrict__ sec, int64_t nsec, const SecGroup *__restrict__ groups, int ngroups,
    const TermDev *__restrict__ terms, const double2 *__restrict__ rterms) {
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= nsec) return;
    const int s = blockIdx.y * 32 + lane;
    const bool live = s < nbatch;
    const IDX k = sec[i];
    const double2 *row = src + (uint64_t)(live ? s : 0) * nbasis;
    const IDX A = (IDX)0x5555555555555555ull;
    double2 acc = make_double2(0.0, 0.0);
    for (int g = 0; g < ngroups; ++g) {
        const uint64_t gx = __ldg(&groups[g].x);
        const IDX x = (IDX)gx;
        const IDX kx = k & x;
        if ((popc_t<IDX>(kx & A) | popc_t<IDX>(kx & ~A) << 8) != __ldg(&groups[g].halves)) continue;
        const IDX j = k ^ x;
        const double2 v = live ? __ldg(&row[j]) : make_double2(0.0, 0.0);
        const int t0 = __ldg(&groups[g].begin), t1 = __ldg(&groups[g].end);
        if (__ldg(&groups[g].real)) {
            double f = 0.0;
#pragma unroll 4
            for (int t = t0; t < t1; ++t) {
                const double2 zc = __ldg(&rterms[t]);
                const IDX z = (IDX)__double_as_longlong(zc.x);
                f += (popc_t<IDX>(j & z) & 1) ? -zc.y : zc.y;
            }
            acc.x += f * v.x;
            acc.y += f * v.y;
        } else {
            double2 f = make_double2(0.0, 0.0);
            for (int t = t0; t < t1; ++t) {
                const double2 c = terms[t].c;
                if (parity64((uint64_t)j & __ldg(&terms[t].z))) { f.x -= c.x; f.y -= c.y; }
                else { f.x += c.x; f.y += c.y; }
            }
            acc = c_add(acc, c_mul(f, v));
        }
    }
    if (live) dst[(uint64_t)s * nbasis + (uint64_t)k] = acc;
}

// The same for small batches: one thread per output index k of the sector and
// NS states per thread, so a warp's lanes are 32 different outputs (each
// lane skips the groups that do not connect its k inside the sector).
template <typename IDX, int NS>
__global__ void __launch_bounds__(256) k_sum_apply_sector_k(
    double2 *__restrict__ dst, const double2 *__restrict__ src, uint64_t nbasis, int nbatch,
    const IDX *__restrict__ sec, int64_t nsec, const SecGroup *__restrict__ groups, int ngroups,
    const TermDev *__restrict__ terms, const double2 *__restrict__ rterms) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsec) return;
    const int s0 = blockIdx.y * NS;
    const IDX k = sec[i];
    const IDX A = (IDX)0x5555555555555555ull;
    double2 acc[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] = make_double2(0.0, 0.0);
    for (int g = 0; g < ngroups; ++g) {
        const IDX x = (IDX)__ldg(&groups[g].x);
        const IDX kx = k & x;
        if ((popc_t<IDX>(kx & A) | popc_t<IDX>(kx & ~A) << 8) != __ldg(&groups[g].halves)) continue;
        const IDX j = k ^ x;
        const int t0 = __ldg(&groups[g].begin), t1 = __ldg(&groups[g].end);
        double2 f = make_double2(0.0, 0.0);
        if (__ldg(&groups[g].real)) {
            for (int t = t0; t < t1; ++t) {
                const double2 zc = __ldg(&rterms[t]);
                const IDX z = (IDX)__double_as_longlong(zc.x);
                f.x += (popc_t<IDX>(j & z) & 1) ? -zc.y : zc.y;
            }
        } else {
            for (int t = t0; t < t1; ++t) {
                const double2 c = terms[t].c;
                if (parity64((uint64_t)j & __ldg(&terms[t].z))) { f.x -= c.x; f.y -= c.y; }
                else { f.x += c.x; f.y += c.y; }
            }
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (s0 + s < nbatch) {
                const double2 v = __ldg(&src[(uint64_t)(s0 + s) * nbasis + j]);
                acc[s] = c_add(acc[s], c_mul(f, v));
            }
        }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if (s0 + s < nbatch) dst[(uint64_t)(s0 + s) * nbasis + (uint64_t)k] = acc[s];
}

template <typename IDX>
static void launch_sector_apply(double2 *dst, const double2 *src, uint64_t nbasis, int B,
                                const IDX *sec, int64_t nsec, const SecGroup *groups, int ngroups,
                                const TermDev *terms, const double2 *rterms) {
    if (B >= 24) {
        const dim3 grid((unsigned)((nsec + 7) / 8), (unsigned)((B + 31) / 32));
        k_sum_apply_sector<IDX><<<grid, 256, 0, t_stream>>>(dst, src, nbasis, B, sec, nsec, groups,
                                                           ngroups, terms, rterms);
        return;
    }
    const unsigned gx = (unsigned)((nsec + 255) / 256);
#define QFB_SECTOR_K(NS)                                                                        \
    k_sum_apply_sector_k<IDX, NS><<<dim3(gx, (unsigned)((B + NS - 1) / NS)), 256, 0, t_stream>>>( \
        dst, src, nbasis, B, sec, nsec, groups, ngroups, terms, rterms)
    if (B == 1) QFB_SECTOR_K(1);
    else if (B == 2) QFB_SECTOR_K(2);
    else if (B <= 4) QFB_SECTOR_K(4);
    else if (B <= 8) QFB_SECTOR_K(8);
    else QFB_SECTOR_K(12);
#undef QFB_SECTOR_K
}

// ---------------------------------------------------------------------------
// programs
// ---------------------------------------------------------------------------

struct StepParams {
    const StrDev *strs;
    const double *params;  // [nrows][nparam]
    const double2 *tab;    // Givens tables of the program
    int32_t nparam;
    int32_t bcast;    // single parameter row for every slot
    int32_t sign;     // +1: U, -1: negated angles
    int32_t reverse;  // strings of a step in reverse order (exact U^dagger)
};

__device__ __forceinline__ double step_param(const StepParams &sp, int b, int param) {
    return sp.params[(sp.bcast ? 0 : (size_t)b) * sp.nparam + param];
}

// Pattern of j's bits at the step's table positions.
__device__ __forceinline__ int step_pattern(uint64_t j, int nd, uint64_t dpos) {
    int pat = 0;
    for (int i = 0; i < nd; ++i) pat |= (int)((j >> ((dpos >> (6 * i)) & 63)) & 1ull) << i;
    return pat;
}

// Free-bit counter f with zeros inserted at the step's nd + 1 sorted
// positions (the pattern bits and h): the f-th pair of one active pattern.
__device__ __forceinline__ uint64_t active_pair(uint64_t f, const StepDev &st) {
    for (int i = 0; i <= st.nd; ++i) f = insert0(f, (int)((st.zpos >> (6 * i)) & 63));
    return f;
}

// Stage this step's strings (in application order) with cos/sin of their
// angles for slot b into shared memory.
__device__ __forceinline__ void stage_step(const StepDev &st, const StepParams &sp, int b,
                                           uint64_t *s_z, int *s_q, double2 *s_cs,
                                           double *s_scale) {
    for (int i = threadIdx.x; i < st.ns; i += blockDim.x) {
        const int k = st.s0 + (sp.reverse ? st.ns - 1 - i : i);
        const StrDev sd = sp.strs[k];
        const double phi = (double)sp.sign * sd.scale * step_param(sp, b, sd.param);
        double s, c;
        sincos(phi, &s, &c);
        s_z[i] = sd.z;
        s_q[i] = sd.ny;
        s_cs[i] = make_double2(c, s);
        if (s_scale) s_scale[i] = sd.scale;
    }
    __syncthreads();
}

// exp(i phi P) on the pair (v0 at j0, v1 at j1 = j0 ^ x); for x == 0 call with
// j1 == j0 on each amplitude separately (v1 is then ignored).
__device__ __forceinline__ void rotate_pair(double2 &v0, double2 &v1, uint64_t j0, uint64_t j1,
                                            uint64_t z, int ny, double2 cs, bool diag) {
    const int q0 = (ny + 1 + 2 * parity64(j0 & z)) & 3;  // i * ph(j0)
    if (diag) {
        const double2 r = c_ipow(v0, q0);
        v0 = make_double2(cs.x * v0.x + cs.y * r.x, cs.x * v0.y + cs.y * r.y);
        return;
    }
    const int q1 = (ny + 1 + 2 * parity64(j1 & z)) & 3;  // i * ph(j1)
    const double2 r1 = c_ipow(v1, q1), r0 = c_ipow(v0, q0);
    const double2 n0 = make_double2(cs.x * v0.x + cs.y * r1.x, cs.x * v0.y + cs.y * r1.y);
    const double2 n1 = make_double2(cs.x * v1.x + cs.y * r0.x, cs.x * v1.y + cs.y * r0.y);
    v0 = n0;
    v1 = n1;
}

// Givens rotation of one active pair: new0 = c v0 + s hn v1, new1 = c v1 + s gn v0
// (s already carries sigma(j)).
__device__ __forceinline__ void givens_pair(double2 &v0, double2 &v1, double c, double s,
                                            double2 gn, double2 hn) {
    const double2 a = c_mul(hn, v1), b = c_mul(gn, v0);
    const double2 n0 = make_double2(c * v0.x + s * a.x, c * v0.y + s * a.y);
    v1 = make_double2(c * v1.x + s * b.x, c * v1.y + s * b.y);
    v0 = n0;
}

__global__ void __launch_bounds__(256) k_prog_step(double2 *__restrict__ psi, uint64_t nbasis,
                                                   StepDev st, StepParams sp) {
    __shared__ uint64_t s_z[kMaxStepStrings];
    __shared__ int s_q[kMaxStepStrings];
    __shared__ double2 s_cs[kMaxStepStrings];
    const int b = blockIdx.y;
    double2 *s = psi + (uint64_t)b * nbasis;
    const uint64_t npair = nbasis >> 1;
    if (st.tab >= 0) {
        double sn, cs;
        sincos((double)sp.sign * st.gamma * step_param(sp, b, st.param), &sn, &cs);
        const double2 *tab = sp.tab + st.tab;
        const bool act = st.na > 0;
        const int fb = act ? (63 - __clzll(nbasis) - 1 - st.nd) : 0;
        const uint64_t total = act ? ((uint64_t)st.na << fb) : npair;
        for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
             q += (uint64_t)gridDim.x * blockDim.x) {
            uint64_t j0;
            int pat;
            if (act) {
                const int ai = (int)(q >> fb);
                j0 = active_pair(q & ((1ull << fb) - 1ull), st) | st.patbits[ai];
                pat = st.patidx[ai];
            } else {
                j0 = insert0(q, st.h);
                pat = step_pattern(j0, st.nd, st.dpos);
            }
            const double2 gn = __ldg(&tab[2 * pat]), hn = __ldg(&tab[2 * pat + 1]);
            if (!act && gn.x == 0.0 && gn.y == 0.0 && hn.x == 0.0 && hn.y == 0.0) continue;
            const uint64_t j1 = j0 ^ st.x;
            const double ss = parity64(j0 & st.zbase) ? -sn : sn;
            double2 v0 = s[j0], v1 = s[j1];
            givens_pair(v0, v1, cs, ss, gn, hn);
            s[j0] = v0;
            s[j1] = v1;
        }
        return;
    }
    stage_step(st, sp, b, s_z, s_q, s_cs, nullptr);
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npair;
         p += (uint64_t)gridDim.x * blockDim.x) {
        if (st.h >= 0) {
            const uint64_t j0 = insert0(p, st.h), j1 = j0 ^ st.x;
            double2 v0 = s[j0], v1 = s[j1];
            for (int i = 0; i < st.ns; ++i) rotate_pair(v0, v1, j0, j1, s_z[i], s_q[i], s_cs[i], false);
            s[j0] = v0;
            s[j1] = v1;
        } else {
            const uint64_t j0 = p << 1, j1 = j0 | 1ull;
            double2 v0 = s[j0], v1 = s[j1], dummy;
            for (int i = 0; i < st.ns; ++i) {
                rotate_pair(v0, dummy, j0, j0, s_z[i], s_q[i], s_cs[i], true);
                rotate_pair(v1, dummy, j1, j1, s_z[i], s_q[i], s_cs[i], true);
            }
            s[j0] = v0;
            s[j1] = v1;
        }
    }
}

// One gradient step: accumulate <sigma|K|psi> for K = sum_i (i scale_i) P_i over
// this step's strings, then (when `rotate`) apply the step's rotation with the
// angles of `sp` (negated: U^dagger) to both states.
// partial[((row * nbatch) + b) * gridDim.x + blockIdx.x].
__global__ void __launch_bounds__(256) k_grad_step(double2 *__restrict__ psi,
                                                   double2 *__restrict__ sig, uint64_t nbasis,
                                                   StepDev st, StepParams sp, int rotate, int row,
                                                   double2 *__restrict__ partial) {
    __shared__ uint64_t s_z[kMaxStepStrings];
    __shared__ int s_q[kMaxStepStrings];
    __shared__ double2 s_cs[kMaxStepStrings];
    __shared__ double s_scale[kMaxStepStrings];
    const int b = blockIdx.y;
    double2 *ps = psi + (uint64_t)b * nbasis;
    double2 *sg = sig + (uint64_t)b * nbasis;
    const uint64_t npair = nbasis >> 1;
    double2 acc = make_double2(0.0, 0.0);
    if (st.tab >= 0) {
        double sn, cs;
        sincos((double)sp.sign * st.gamma * step_param(sp, b, st.param), &sn, &cs);
        const double2 *tab = sp.tab + st.tab;
        const bool act = st.na > 0;
        const int fb = act ? (63 - __clzll(nbasis) - 1 - st.nd) : 0;
        const uint64_t total = act ? ((uint64_t)st.na << fb) : npair;
        for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
             q += (uint64_t)gridDim.x * blockDim.x) {
            uint64_t j0;
            int pat;
            if (act) {
                const int ai = (int)(q >> fb);
                j0 = active_pair(q & ((1ull << fb) - 1ull), st) | st.patbits[ai];
                pat = st.patidx[ai];
            } else {
                j0 = insert0(q, st.h);
                pat = step_pattern(j0, st.nd, st.dpos);
            }
            const double2 gn = __ldg(&tab[2 * pat]), hn = __ldg(&tab[2 * pat + 1]);
            if (!act && gn.x == 0.0 && gn.y == 0.0 && hn.x == 0.0 && hn.y == 0.0) continue;
            const uint64_t j1 = j0 ^ st.x;
            const bool neg = parity64(j0 & st.zbase);
            double2 v0 = ps[j0], v1 = ps[j1], w0 = sg[j0], w1 = sg[j1];
            // <sigma|K|psi> on the pair: sigma(j) gamma (conj(w0) hn v1 + conj(w1) gn v0)
            const double2 t = c_add(c_cjmul(w0, c_mul(hn, v1)), c_cjmul(w1, c_mul(gn, v0)));
            const double gs = neg ? -st.gamma : st.gamma;
            acc.x += gs * t.x;
            acc.y += gs * t.y;
            if (rotate) {
                const double ss = neg ? -sn : sn;
                givens_pair(v0, v1, cs, ss, gn, hn);
                givens_pair(w0, w1, cs, ss, gn, hn);
                ps[j0] = v0;
                ps[j1] = v1;
                sg[j0] = w0;
                sg[j1] = w1;
            }
        }
    } else {
        stage_step(st, sp, b, s_z, s_q, s_cs, s_scale);
        const bool diag = st.h < 0;
        for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npair;
             p += (uint64_t)gridDim.x * blockDim.x) {
            const uint64_t j0 = diag ? (p << 1) : insert0(p, st.h);
            const uint64_t j1 = diag ? (j0 | 1ull) : (j0 ^ st.x);
            double2 v0 = ps[j0], v1 = ps[j1], w0 = sg[j0], w1 = sg[j1];
            // (K psi)_j = sum_i scale_i * (i ph_i(j ^ x)) psi_{j ^ x}
            double2 k0 = make_double2(0.0, 0.0), k1 = make_double2(0.0, 0.0);
            for (int i = 0; i < st.ns; ++i) {
                const int qa = (s_q[i] + 1 + 2 * parity64(j0 & s_z[i])) & 3;
                const int qb = (s_q[i] + 1 + 2 * parity64(j1 & s_z[i])) & 3;
                const double sc = s_scale[i];
                if (diag) {
                    const double2 r0 = c_ipow(v0, qa), r1 = c_ipow(v1, qb);
                    k0.x += sc * r0.x; k0.y += sc * r0.y;
                    k1.x += sc * r1.x; k1.y += sc * r1.y;
                } else {
                    const double2 r1 = c_ipow(v1, qb), r0 = c_ipow(v0, qa);
                    k0.x += sc * r1.x; k0.y += sc * r1.y;
                    k1.x += sc * r0.x; k1.y += sc * r0.y;
                }
            }
            acc = c_add(acc, c_add(c_cjmul(w0, k0), c_cjmul(w1, k1)));
            if (rotate) {
                double2 dummy;
                for (int i = 0; i < st.ns; ++i) {
                    if (diag) {
                        rotate_pair(v0, dummy, j0, j0, s_z[i], s_q[i], s_cs[i], true);
                        rotate_pair(v1, dummy, j1, j1, s_z[i], s_q[i], s_cs[i], true);
                        rotate_pair(w0, dummy, j0, j0, s_z[i], s_q[i], s_cs[i], true);
                        rotate_pair(w1, dummy, j1, j1, s_z[i], s_q[i], s_cs[i], true);
                    } else {
                        rotate_pair(v0, v1, j0, j1, s_z[i], s_q[i], s_cs[i], false);
                        rotate_pair(w0, w1, j0, j1, s_z[i], s_q[i], s_cs[i], false);
                    }
                }
                ps[j0] = v0;
                ps[j1] = v1;
                sg[j0] = w0;
                sg[j1] = w1;
            }
        }
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0)
        partial[((uint64_t)row * gridDim.y + b) * gridDim.x + blockIdx.x] = acc;
}

// per-slot partial sums of conj(a) b: partial[b * gridDim.x + blockIdx.x]
__global__ void k_vdot_rows(const double2 *__restrict__ a, const double2 *__restrict__ b,
                            uint64_t nbasis, double2 *__restrict__ partial) {
    const uint64_t off = (uint64_t)blockIdx.y * nbasis;
    double2 acc = make_double2(0.0, 0.0);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nbasis;
         i += (uint64_t)gridDim.x * blockDim.x)
        acc = c_add(acc, c_cjmul(a[off + i], b[off + i]));
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(uint64_t)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// energy[b] = Re sum_k partial[b * n + k]   (one block per slot)
__global__ void k_energy_final(const double2 *__restrict__ partial, int n,
                               double *__restrict__ energy) {
    double2 acc = make_double2(0.0, 0.0);
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        acc = c_add(acc, partial[(uint64_t)blockIdx.x * n + k]);
    acc = block_sum(acc);
    if (threadIdx.x == 0) energy[blockIdx.x] = acc.x;
}

// Pool inner products <sigma|K_s|psi> of Givens-form steps read from a device
// array (one step per blockIdx.y, slot blockIdx.z, chunk blockIdx.x), states
// untouched: every ADAPT pool operator in one launch.
// partial[((s * B) + b) * chunks + c].
__global__ void __launch_bounds__(256) k_pool_ip(const double2 *__restrict__ psi,
                                                 const double2 *__restrict__ sig, uint64_t nbasis,
                                                 const StepDev *__restrict__ steps,
                                                 const double2 *__restrict__ tab,
                                                 double2 *__restrict__ partial) {
    const int s = blockIdx.y, b = blockIdx.z, B = gridDim.z;
    const StepDev &st = steps[s];
    const double2 *ps = psi + (uint64_t)b * nbasis;
    const double2 *sg = sig + (uint64_t)b * nbasis;
    const double2 *tb = tab + st.tab;
    const int fb = 63 - __clzll(nbasis) - 1 - st.nd;
    const uint64_t total = (uint64_t)st.na << fb;
    double2 acc = make_double2(0.0, 0.0);
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const int ai = (int)(q >> fb);
        const uint64_t j0 = active_pair(q & ((1ull << fb) - 1ull), st) | st.patbits[ai];
        const int pat = st.patidx[ai];
        const double2 gn = __ldg(&tb[2 * pat]), hn = __ldg(&tb[2 * pat + 1]);
        const uint64_t j1 = j0 ^ st.x;
        const double2 v0 = ps[j0], v1 = ps[j1], w0 = sg[j0], w1 = sg[j1];
        const double2 t = c_add(c_cjmul(w0, c_mul(hn, v1)), c_cjmul(w1, c_mul(gn, v0)));
        const double gs = parity64(j0 & st.zbase) ? -st.gamma : st.gamma;
        acc.x += gs * t.x;
        acc.y += gs * t.y;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[((uint64_t)s * B + b) * gridDim.x + blockIdx.x] = acc;
}

// grad[b * M + mu] = 2 Re sum over mu's steps s and chunks c of
// partial[((s * B) + b) * chunks + c].  grid = (M, B).
// res[b][k] = Re(st[idx[k] * s_i + b * s_b] * phase[k]) (0 where idx[k] < 0)
template <class V>
__global__ void k_resid_gather(const V *__restrict__ st, const int64_t *__restrict__ idx,
                               uint64_t s_i, uint64_t s_b, const double2 *__restrict__ phase,
                               int nres, int B, double *__restrict__ res) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nres * B) return;
    const int b = (int)(t / nres), k = (int)(t % nres);
    const int64_t i = idx[k];
    double r = 0.0;
    if (i >= 0) {
        const double2 v = qfbs::v_cj(qfbs::v_one_of<V>(), st[(uint64_t)i * s_i + (uint64_t)b * s_b]);
        const double2 ph = phase[k];
        r = v.x * ph.x - v.y * ph.y;
    }
    res[(size_t)b * nres + k] = r;
}

__global__ void k_grad_final(const double2 *__restrict__ partial, const int2 *__restrict__ psteps,
                             int chunks, double *__restrict__ grad) {
    const int mu = blockIdx.x, b = blockIdx.y, B = gridDim.y, M = gridDim.x;
    const int2 r = psteps[mu];
    double2 acc = make_double2(0.0, 0.0);
    for (int s = r.x; s < r.y; ++s)
        for (int c = threadIdx.x; c < chunks; c += blockDim.x)
            acc = c_add(acc, partial[((uint64_t)s * B + b) * chunks + c]);
    acc = block_sum(acc);
    if (threadIdx.x == 0) grad[(uint64_t)b * M + mu] = 2.0 * acc.x;
}

// The same for few partials per step row (chunks <= 32): one thread per
// gradient entry, parameters fastest (coalesced writes), the partials summed
// in row and chunk order.
__global__ void k_grad_final_few(const double2 *__restrict__ partial, const int2 *__restrict__ psteps,
                                 int chunks, int M, int B, double *__restrict__ grad) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)M * B) return;
    const int mu = (int)(t % M), b = (int)(t / M);
    const int2 r = psteps[mu];
    double acc = 0.0;
    for (int s = r.x; s < r.y; ++s) {
        const double2 *p = partial + ((uint64_t)s * B + b) * chunks;
        for (int c = 0; c < chunks; ++c) acc += p[c].x;
    }
    grad[(uint64_t)b * M + mu] = 2.0 * acc;
}

__global__ void k_set_ref(double2 *__restrict__ psi, uint64_t nbasis, uint64_t ref, int nbatch) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbatch) psi[(uint64_t)b * nbasis + ref] = make_double2(1.0, 0.0);
}

}  // namespace

// ===========================================================================
// host objects
// ===========================================================================

// Groups ordered by their high part x >> m, for k_sum_apply_tiled.
struct TiledView {
    int m = 0, nhi = 0;
    void *blob = nullptr;
    GroupDev *d_groups = nullptr;
    int32_t *d_hi0 = nullptr;
    uint64_t *d_hival = nullptr;
};

// H rows on a particle-number sector and compact plans (defined with the
// compact evaluator below); cached on the Hamiltonian and on the forward
// program so that every evaluator of one problem shares them.
struct SectorRows;
struct SectorPlan;
static std::atomic<uint64_t> g_prog_uid{1};

struct qfb_sum_s {
    int64_t nterms = 0;
    int32_t ngroups = 0;
    int32_t nsegment = 0;
    TiledView *tiled[kApplyTileBits + 1] = {nullptr};
    ~qfb_sum_s() {
        for (auto *t : tiled)
            if (t) {
                dev_free(t->blob);
                delete t;
            }
    }
    void *blob = nullptr;  // device: groups, terms, segment starts
    GroupDev *d_groups = nullptr;
    TermDev *d_terms = nullptr;
    double2 *d_rterms = nullptr;  // (z bits, Re c) per term, for real groups
    int32_t *d_seg_g0 = nullptr;
    std::vector<GroupDev> h_groups;
    std::vector<TermDev> h_terms;  // host copy of the terms (H records of the sector)
    std::vector<int32_t> h_seg_g0;
    // (nqubit, alpha count, beta count, bank-interleaved) -> rows
    std::map<std::tuple<int, int, int, int>, std::shared_ptr<SectorRows>> rows_cache;
};

// A window plan of a program for one qubit count (qfb_window.cuh).
struct WinPlan {
    int b = 0, L = 0, nqubit = 0, nt = 1;
    std::vector<qfbw::Window> wins;
    std::vector<qfbw::WStep> steps;
    std::vector<qfbw::WStr> strs;
    std::vector<double2> tabs;
    void *blob = nullptr;
    qfbw::WStep *d_steps = nullptr;
    qfbw::WStr *d_strs = nullptr;
    double2 *d_tabs = nullptr;
    size_t smem_max = 0;
    int ntiles() const { return 1 << (nqubit - b); }
};

struct qfb_prog_s {
    uint64_t uid = g_prog_uid.fetch_add(1);  // identity for caches keyed on other programs
    // (K uid, U uid, nqubit, alpha count, beta count, shared) -> plan (null: none)
    std::map<std::tuple<uint64_t, uint64_t, int, int, int, int>, std::shared_ptr<SectorPlan>>
        sector_plans;
    int64_t nstrings = 0;
    int32_t nparam = 0;
    void *blob = nullptr;
    StrDev *d_strs = nullptr;
    double2 *d_tab = nullptr;       // Givens tables (StepDev::tab)
    std::vector<double2> h_tab;
    std::vector<StrDev> h_strs;
    std::vector<StepDev> h_steps;
    std::vector<int32_t> p_step0, p_step1;  // steps of each parameter (gradient)
    bool params_contiguous = true;
    WinPlan *fwd_plan[41] = {nullptr};   // by qubit count
    WinPlan *grad_plan[41] = {nullptr};  // gradient sweep with K = this program ...
    const qfb_prog_s *grad_plan_u[41] = {nullptr};  // ... and U_mu from this one
    // plans replaced while the program lives (a new tile shape or U program):
    // captured evaluator graphs may still read them, so they go with the program
    std::vector<WinPlan *> retired;
    ~qfb_prog_s() {
        for (auto *v : {&fwd_plan, &grad_plan})
            for (auto *pl : *v)
                if (pl) {
                    dev_free(pl->blob);
                    delete pl;
                }
        for (auto *pl : retired) {
            dev_free(pl->blob);
            delete pl;
        }
    }
};

namespace {

// Tile size (qubits) of the forward and gradient windows: a forward tile of
// 2^12 amplitudes is 64 KB; a gradient window holds psi and sigma, 2 x 32 KB.
constexpr int kFwdTileBits = 12;
constexpr int kGradTileBits = 11;
constexpr int kLowBits = 3;
// process-wide tile shape of new window plans (qfb_ucc_tiles)
int g_win_fwd = kFwdTileBits, g_win_grad = kGradTileBits, g_win_low = kLowBits;

static qfbw::Window make_window(uint64_t U, int n, int b, int L) {
    qfbw::Window w{};
    const uint64_t all = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
    uint64_t q = U | ((1ull << L) - 1ull);
    for (int k = 0; k < n && __builtin_popcountll(q) < b; ++k) q |= 1ull << k;
    w.qmask = q & all;
    w.cmask = all & ~w.qmask;
    w.b = b;
    w.global_step = -1;
    w.global_mu = -1;
    return w;
}

static void push_strings(WinPlan *pl, const qfb_prog_s *p, const StepDev &st, uint64_t qmask,
                         int sign, bool reversed) {
    for (int i = 0; i < st.ns; ++i) {
        const int k = st.s0 + (reversed ? st.ns - 1 - i : i);
        const StrDev &sd = p->h_strs[k];
        qfbw::WStr w;
        w.zl = qfbw::pext_h(sd.z, qmask);
        w.zc = sd.z & ~qmask;
        w.ny = sd.ny;
        w.param = sd.param;
        w.rscale = sign * sd.scale;
        w.scale = sd.scale;
        pl->strs.push_back(w);
    }
}

static void push_step(WinPlan *pl, const qfbw::Window &win, const qfb_prog_s *p,
                      const StepDev &st, int rotate, int ip_row, int sign) {
    qfbw::WStep w{};
    w.xl = qfbw::pext_h(st.x, win.qmask);
    w.hl = w.xl ? 63 - __builtin_clzll(w.xl) : -1;
    w.s0 = (int32_t)pl->strs.size() - win.sr0;
    w.ns = st.ns;
    w.rotate = rotate;
    w.ip_row = ip_row;
    w.tab = -1;
    w.param = st.param;
    w.sign = sign;
    bool inside = st.tab >= 0;
    for (int i = 0; inside && i < st.nd; ++i)
        inside = (win.qmask >> ((st.dpos >> (6 * i)) & 63)) & 1ull;
    if (inside) {
        // pattern positions in tile coordinates
        w.nd = st.nd;
        w.dpos = 0;
        for (int i = 0; i < st.nd; ++i) {
            const int q = (int)((st.dpos >> (6 * i)) & 63);
            const int lp = __builtin_popcountll(win.qmask & ((1ull << q) - 1ull));
            w.dpos |= (uint64_t)lp << (6 * i);
        }
        w.zb_l = qfbw::pext_h(st.zbase, win.qmask);
        w.zb_c = st.zbase & ~win.qmask;
        w.gamma = st.gamma;
        w.na = st.na;
        if (st.na > 0) {
            for (int a = 0; a < st.na; ++a) {
                w.patidx[a] = st.patidx[a];
                w.patbits[a] = (uint32_t)qfbw::pext_h(st.patbits[a], win.qmask);
            }
            int zp[7], nz = 0;
            for (int i = 0; i < st.nd; ++i) zp[nz++] = (int)((w.dpos >> (6 * i)) & 63);
            zp[nz++] = w.hl;
            std::sort(zp, zp + nz);
            w.zpos = 0;
            for (int i = 0; i < nz; ++i) w.zpos |= (uint32_t)zp[i] << (4 * i);
        }
        w.tab = (int32_t)pl->tabs.size() - win.tr0;
        const int n = 2 << st.nd;
        pl->tabs.insert(pl->tabs.end(), p->h_tab.begin() + st.tab, p->h_tab.begin() + st.tab + n);
    }
    pl->steps.push_back(w);
}

static int upload_plan(WinPlan *pl) {
    const size_t sb = sizeof(qfbw::WStep) * std::max<size_t>(1, pl->steps.size());
    const size_t sbal = (sb + 255) & ~(size_t)255;
    const size_t rb = sizeof(qfbw::WStr) * std::max<size_t>(1, pl->strs.size());
    const size_t rbal = (rb + 255) & ~(size_t)255;
    const size_t tb = sizeof(double2) * std::max<size_t>(1, pl->tabs.size());
    int rc = dev_alloc(&pl->blob, sbal + rbal + tb);
    if (rc) return rc;
    pl->d_steps = (qfbw::WStep *)pl->blob;
    pl->d_strs = (qfbw::WStr *)((char *)pl->blob + sbal);
    pl->d_tabs = (double2 *)((char *)pl->blob + sbal + rbal);
    if (!pl->tabs.empty())
        QFB_CUDA(cudaMemcpyAsync(pl->d_tabs, pl->tabs.data(), sizeof(double2) * pl->tabs.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    if (!pl->steps.empty())
        QFB_CUDA(cudaMemcpyAsync(pl->d_steps, pl->steps.data(), sb, cudaMemcpyHostToDevice,
                                 t_stream));
    if (!pl->strs.empty())
        QFB_CUDA(cudaMemcpyAsync(pl->d_strs, pl->strs.data(), rb, cudaMemcpyHostToDevice,
                                 t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    for (auto &w : pl->wins) {
        if (w.global_step >= 0 || w.global_mu >= 0) continue;
        w.needs_strings = 0;
        for (int32_t k = w.st0; k < w.st1; ++k)
            if (pl->steps[k].tab < 0) w.needs_strings = 1;
        pl->smem_max = std::max(
            pl->smem_max, qfbw::win_smem_bytes(w.b, pl->L, w.needs_strings ? w.sr1 - w.sr0 : 0,
                                               w.st1 - w.st0, pl->nt, w.tr1 - w.tr0));
    }
    return QFB_OK;
}

// Forward windows: consecutive steps whose x-supports fit in the tile.
static int build_fwd_plan(qfb_prog_s *p, int n, WinPlan **out) {
    WinPlan *pl = new WinPlan;
    pl->nqubit = n;
    pl->b = std::min(g_win_fwd, n);
    pl->L = std::min(g_win_low, pl->b);
    pl->nt = 1;
    const uint64_t low = (1ull << pl->L) - 1ull;
    const int room = pl->b - pl->L;
    const size_t K = p->h_steps.size();
    size_t i = 0;
    while (i < K) {
        const StepDev &s0 = p->h_steps[i];
        if (__builtin_popcountll(s0.x & ~low) > room || s0.ns > qfbw::kWinMaxStr) {
            qfbw::Window w{};
            w.global_step = (int32_t)i;
            w.global_mu = -1;
            pl->wins.push_back(w);
            ++i;
            continue;
        }
        auto ntab = [](const StepDev &st) { return st.tab >= 0 ? (2 << st.nd) : 0; };
        uint64_t U = s0.x;
        size_t j = i + 1;
        int nstr = s0.ns, nt = ntab(s0);
        while (j < K) {
            const StepDev &sj = p->h_steps[j];
            const uint64_t U2 = U | sj.x;
            if (__builtin_popcountll(U2 & ~low) > room || nstr + sj.ns > qfbw::kWinMaxStr ||
                (int)(j - i) + 1 > qfbw::kWinMaxSteps || nt + ntab(sj) > qfbw::kWinMaxTab)
                break;
            U = U2;
            nstr += sj.ns;
            nt += ntab(sj);
            ++j;
        }
        qfbw::Window w = make_window(U & ~low, n, pl->b, pl->L);
        w.st0 = (int32_t)pl->steps.size();
        w.sr0 = (int32_t)pl->strs.size();
        w.tr0 = (int32_t)pl->tabs.size();
        for (size_t k = i; k < j; ++k) {
            push_step(pl, w, p, p->h_steps[k], 1, -1, +1);
            push_strings(pl, p, p->h_steps[k], w.qmask, +1, false);
        }
        w.st1 = (int32_t)pl->steps.size();
        w.sr1 = (int32_t)pl->strs.size();
        w.tr1 = (int32_t)pl->tabs.size();
        pl->wins.push_back(w);
        i = j;
    }
    int rc = upload_plan(pl);
    if (rc) {
        delete pl;
        return rc;
    }
    *out = pl;
    return QFB_OK;
}

// Gradient windows: the reverse sweep over parameters; per parameter the
// inner product(s) <sigma|K_mu|psi> on kp's strings, then (except for the
// first parameter) U_mu^dagger from up's strings in reverse.  When kp and up
// are one program and the parameter is one x-group, both share one pass.
static int build_grad_plan(qfb_prog_s *kp, const qfb_prog_s *up, int n, WinPlan **out) {
    WinPlan *pl = new WinPlan;
    pl->nqubit = n;
    pl->b = std::min(g_win_grad, n);
    pl->L = std::min(g_win_low, pl->b);
    pl->nt = 2;
    const uint64_t low = (1ull << pl->L) - 1ull;
    const int room = pl->b - pl->L;
    const int M = kp->nparam;
    auto steps_of = [](const qfb_prog_s *p, int m, int32_t &a0, int32_t &a1) {
        a0 = p->p_step0[m];
        a1 = p->p_step1[m];
        if (a0 < 0) a0 = a1 = 0;
    };
    auto supp = [&](int m) {
        uint64_t u = 0;
        int32_t a0, a1;
        steps_of(kp, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s) u |= kp->h_steps[s].x;
        steps_of(up, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s) u |= up->h_steps[s].x;
        return u;
    };
    auto nstr_of = [&](int m) {
        int c = 0;
        int32_t a0, a1;
        steps_of(kp, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s) c += kp->h_steps[s].ns;
        steps_of(up, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s) c += up->h_steps[s].ns;
        return c;
    };
    auto empty = [&](int m) { return kp->p_step0[m] < 0 && up->p_step0[m] < 0; };
    // steps and table entries a parameter adds to a window (upper bounds)
    auto nst_of = [&](int m) {
        int32_t a0, a1, b0, b1;
        steps_of(kp, m, a0, a1);
        steps_of(up, m, b0, b1);
        return (a1 - a0) + (b1 - b0);
    };
    auto ntab_of = [&](int m) {
        int c = 0;
        int32_t a0, a1;
        steps_of(kp, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s)
            if (kp->h_steps[s].tab >= 0) c += 2 << kp->h_steps[s].nd;
        steps_of(up, m, a0, a1);
        for (int32_t s = a0; s < a1; ++s)
            if (up->h_steps[s].tab >= 0) c += 2 << up->h_steps[s].nd;
        return c;
    };
    int mu = M - 1;
    while (mu >= 0) {
        if (empty(mu)) {
            --mu;
            continue;
        }
        if (__builtin_popcountll(supp(mu) & ~low) > room || nstr_of(mu) > qfbw::kWinMaxStr ||
            nst_of(mu) > qfbw::kWinMaxSteps || ntab_of(mu) > qfbw::kWinMaxTab) {
            qfbw::Window w{};
            w.global_step = -1;
            w.global_mu = mu;
            pl->wins.push_back(w);
            --mu;
            continue;
        }
        uint64_t U = supp(mu);
        int nstr = nstr_of(mu), nst = nst_of(mu), ntb = ntab_of(mu);
        int lo = mu;
        while (lo - 1 >= 0) {
            const int m = lo - 1;
            if (empty(m)) {
                --lo;
                continue;
            }
            const uint64_t U2 = U | supp(m);
            if (__builtin_popcountll(U2 & ~low) > room || nstr + nstr_of(m) > qfbw::kWinMaxStr ||
                nst + nst_of(m) > qfbw::kWinMaxSteps || ntb + ntab_of(m) > qfbw::kWinMaxTab)
                break;
            U = U2;
            nstr += nstr_of(m);
            nst += nst_of(m);
            ntb += ntab_of(m);
            --lo;
        }
        qfbw::Window w = make_window(U & ~low, n, pl->b, pl->L);
        w.st0 = (int32_t)pl->steps.size();
        w.sr0 = (int32_t)pl->strs.size();
        w.tr0 = (int32_t)pl->tabs.size();
        for (int m = mu; m >= lo; --m) {
            const int rot = (m > 0) ? 1 : 0;
            int32_t k0, k1, u0, u1;
            steps_of(kp, m, k0, k1);
            steps_of(up, m, u0, u1);
            if (kp == up && k1 - k0 == 1) {
                // U^dagger exactly: strings reversed, angles negated
                push_step(pl, w, kp, kp->h_steps[k0], rot, k0, -1);
                push_strings(pl, kp, kp->h_steps[k0], w.qmask, -1, true);
                continue;
            }
            for (int32_t s = k0; s < k1; ++s) {
                push_step(pl, w, kp, kp->h_steps[s], 0, s, -1);
                push_strings(pl, kp, kp->h_steps[s], w.qmask, -1, true);
            }
            // up's strings in forward order with negated angles, as the
            // reference's Trotter product of -t K_mu (uccvqeabc.py:208-238)
            if (rot)
                for (int32_t s = u0; s < u1; ++s) {
                    push_step(pl, w, up, up->h_steps[s], 1, -1, -1);
                    push_strings(pl, up, up->h_steps[s], w.qmask, -1, false);
                }
        }
        w.st1 = (int32_t)pl->steps.size();
        w.sr1 = (int32_t)pl->strs.size();
        w.tr1 = (int32_t)pl->tabs.size();
        pl->wins.push_back(w);
        mu = lo - 1;
    }
    int rc = upload_plan(pl);
    if (rc) {
        delete pl;
        return rc;
    }
    *out = pl;
    return QFB_OK;
}

static bool plan_shape_is(const WinPlan *pl, int bits, int n) {
    const int b = std::min(bits, n);
    return pl->b == b && pl->L == std::min(g_win_low, b);
}

static int ensure_plans(qfb_prog_s *p, int n, bool fwd, const qfb_prog_s *up = nullptr) {
    if (n < 1 || n > 40) return fail(QFB_EINVAL, "window plan: bad qubit count %d", n);
    int rc = QFB_OK;
    if (fwd && p->fwd_plan[n] && !plan_shape_is(p->fwd_plan[n], g_win_fwd, n)) {
        p->retired.push_back(p->fwd_plan[n]);
        p->fwd_plan[n] = nullptr;
    }
    if (fwd && !p->fwd_plan[n]) rc = build_fwd_plan(p, n, &p->fwd_plan[n]);
    if (rc == QFB_OK && up &&
        (p->grad_plan_u[n] != up ||
         (p->grad_plan[n] && !plan_shape_is(p->grad_plan[n], g_win_grad, n)))) {
        if (p->grad_plan[n]) {
            p->retired.push_back(p->grad_plan[n]);
            p->grad_plan[n] = nullptr;
        }
        rc = build_grad_plan(p, up, n, &p->grad_plan[n]);
        p->grad_plan_u[n] = (rc == QFB_OK) ? up : nullptr;
    }
    return rc;
}

static int set_win_smem(size_t bytes, int nt) {
    static size_t done[3] = {0, 0, 0};
    if (bytes <= done[nt]) return QFB_OK;
    if (bytes > 227 * 1024)
        return fail(QFB_ENOSYS, "window of %zu bytes of shared memory", bytes);
    if (nt == 1)
        QFB_CUDA(cudaFuncSetAttribute(qfbw::k_window<1>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    else
        QFB_CUDA(cudaFuncSetAttribute(qfbw::k_window<2>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[nt] = bytes;
    return QFB_OK;
}

static int launch_window(const WinPlan *pl, const qfbw::Window &w, double2 *psi, double2 *sig,
                         uint64_t nbasis, int B, const double *d_par, int nparam, int bcast,
                         double2 *partial) {
    qfbw::WinLaunch a;
    a.qmask = w.qmask;
    a.cmask = w.cmask;
    a.b = w.b;
    a.L = pl->L;
    a.nsteps = w.st1 - w.st0;
    a.nstr = w.sr1 - w.sr0;
    a.steps = pl->d_steps + w.st0;
    a.strs = pl->d_strs + w.sr0;
    if (!w.needs_strings) a.nstr = 0;  // every step has its Givens table
    a.tab = pl->d_tabs + w.tr0;
    a.ntab = w.tr1 - w.tr0;
    a.params = d_par;
    a.nparam = nparam;
    a.bcast = bcast;
    a.partial = partial;
    a.ntiles = pl->ntiles();
    const size_t smem = qfbw::win_smem_bytes(w.b, pl->L, a.nstr, a.nsteps, pl->nt, a.ntab);
    if (smem > pl->smem_max) return fail(QFB_EDEVICE, "window shared memory %zu > %zu", smem, pl->smem_max);
    const dim3 grid((unsigned)a.ntiles, (unsigned)B);
    if (pl->nt == 1)
        qfbw::k_window<1><<<grid, qfbw::kWinThreads, smem, t_stream>>>(psi, nullptr, nbasis, a);
    else
        qfbw::k_window<2><<<grid, qfbw::kWinThreads, smem, t_stream>>>(psi, sig, nbasis, a);
    QFB_LAUNCHED();
    return QFB_OK;
}

int upload_params(const double *params, int32_t nrows, int32_t nparam, double **d_out) {
    *d_out = nullptr;
    const size_t n = (size_t)std::max(nrows, 1) * std::max(nparam, 1);
    int rc = dev_alloc((void **)d_out, n * sizeof(double));
    if (rc) return rc;
    if (nparam > 0)
        QFB_CUDA(cudaMemcpyAsync(*d_out, params, (size_t)nrows * nparam * sizeof(double),
                                 cudaMemcpyHostToDevice, t_stream));
    return QFB_OK;
}

unsigned chunks_for(uint64_t npair, int nbatch, int nrows_of_work) {
    // enough blocks to fill every SM several times over, at least 1024 pairs each
    const uint64_t target = (uint64_t)sm_count() * 8;
    uint64_t per = (uint64_t)nbatch * std::max(nrows_of_work, 1);
    uint64_t c = (target + per - 1) / per;
    const uint64_t cap = std::max<uint64_t>(1, npair / 1024);
    if (c > cap) c = cap;
    if (c < 1) c = 1;
    if (c > 65535) c = 65535;
    return (unsigned)c;
}

}  // namespace

// Givens form of a step (StepDev): the strings must commute, their z-masks
// may differ from the first one's only at <= 6 positions (other than h), and
// -(k01 k10) on every active pattern must be one real gamma^2.
static void make_table(qfb_prog_s *p, StepDev &st) {
    st.tab = -1;
    st.nd = 0;
    st.dpos = 0;
    st.zbase = 0;
    st.gamma = 0.0;
    st.na = -1;
    if (st.x == 0 || st.ns < 1) return;
    const StrDev *S = &p->h_strs[st.s0];
    for (int a = 0; a < st.ns; ++a)
        for (int b = a + 1; b < st.ns; ++b)
            if (__builtin_popcountll(st.x & (S[a].z ^ S[b].z)) & 1) return;  // not commuting
    const uint64_t zb = S[0].z;
    uint64_t D = 0;
    for (int a = 0; a < st.ns; ++a) D |= S[a].z ^ zb;
    D &= ~(1ull << st.h);
    const int nd = __builtin_popcountll(D);
    if (nd > 6) return;
    int dp[6];
    {
        uint64_t m = D;
        for (int i = 0; i < nd; ++i) {
            dp[i] = __builtin_ctzll(m);
            m &= m - 1;
        }
    }
    const int npat = 1 << nd;
    std::vector<std::complex<double>> g(npat), hh(npat);
    double scale_norm = 0.0;
    for (int a = 0; a < st.ns; ++a) scale_norm += std::fabs(S[a].scale);
    static const std::complex<double> ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    for (int pat = 0; pat < npat; ++pat) {
        uint64_t jd = 0;
        for (int i = 0; i < nd; ++i)
            if (pat >> i & 1) jd |= 1ull << dp[i];
        std::complex<double> gg = 0.0, hv = 0.0;
        for (int a = 0; a < st.ns; ++a) {
            const int par = __builtin_popcountll(jd & (S[a].z ^ zb)) & 1;
            const std::complex<double> term = S[a].scale * ipow[(S[a].ny + 1) & 3] * (par ? -1.0 : 1.0);
            gg += term;
            hv += (S[a].ny & 1) ? -term : term;
        }
        g[pat] = gg;
        hh[pat] = hv;
    }
    const double tol = 1e-12 * std::max(scale_norm, 1e-300);
    double gamma2 = -1.0;
    for (int pat = 0; pat < npat; ++pat) {
        const bool active = std::abs(g[pat]) > tol || std::abs(hh[pat]) > tol;
        if (!active) {
            g[pat] = hh[pat] = 0.0;
            continue;
        }
        const std::complex<double> pr = -(g[pat] * hh[pat]);
        if (std::fabs(pr.imag()) > tol * scale_norm || pr.real() <= 0.0) return;
        if (gamma2 < 0.0)
            gamma2 = pr.real();
        else if (std::fabs(pr.real() - gamma2) > 1e-12 * gamma2)
            return;
    }
    const double gamma = gamma2 > 0.0 ? std::sqrt(gamma2) : 1.0;
    st.tab = (int32_t)p->h_tab.size();
    st.nd = nd;
    for (int i = 0; i < nd; ++i) st.dpos |= (uint64_t)dp[i] << (6 * i);
    {
        int na = 0;
        for (int pat = 0; pat < npat; ++pat)
            if (g[pat] != 0.0 || hh[pat] != 0.0) {
                if (na < kMaxActive) {
                    st.patidx[na] = (uint8_t)pat;
                    uint64_t bits = 0;
                    for (int i = 0; i < nd; ++i)
                        if (pat >> i & 1) bits |= 1ull << dp[i];
                    st.patbits[na] = bits;
                }
                ++na;
            }
        st.na = (na <= kMaxActive) ? na : -1;
        // sorted positions of the pattern bits and h
        int zp[7], nz = 0;
        for (int i = 0; i < nd; ++i) zp[nz++] = dp[i];
        zp[nz++] = st.h;
        std::sort(zp, zp + nz);
        st.zpos = 0;
        for (int i = 0; i < nz; ++i) st.zpos |= (uint64_t)zp[i] << (6 * i);
    }
    st.zbase = zb;
    st.gamma = gamma2 > 0.0 ? gamma : 0.0;
    for (int pat = 0; pat < npat; ++pat) {
        const std::complex<double> gn = g[pat] / gamma, hn = hh[pat] / gamma;
        p->h_tab.push_back(make_double2(gn.real(), gn.imag()));
        p->h_tab.push_back(make_double2(hn.real(), hn.imag()));
    }
}

extern "C" {

static int enqueue_sum_apply(const qfb_sum_s *h, double2 *dst, const double2 *src,
                             uint64_t nbasis, int B);
static int ensure_tiled(qfb_sum_s *h, int nqubit);

int qfb_sum_create(const qfb_pauli *paulis, const qfb_complex *coeffs, const int32_t *segment,
                   int64_t nterms, int32_t nsegment, qfb_sum *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_sum_create: null output");
    *out = nullptr;
    if (nterms < 0 || (nterms > 0 && (!paulis || !coeffs)))
        return fail(QFB_EINVAL, "qfb_sum_create: bad term arrays");
    if (nsegment < 1) return fail(QFB_EINVAL, "qfb_sum_create: nsegment = %d < 1", nsegment);
    if (nterms > INT32_MAX) return fail(QFB_EINVAL, "qfb_sum_create: too many terms");
    for (int64_t t = 0; t < nterms; ++t) {
        const int32_t sg = segment ? segment[t] : 0;
        if (sg < 0 || sg >= nsegment)
            return fail(QFB_EINVAL, "qfb_sum_create: term %lld has segment %d outside [0, %d)",
                        (long long)t, sg, nsegment);
    }
    // group by (segment, x) in order of first appearance within each segment
    std::vector<std::vector<int64_t>> seg_order(nsegment);
    std::vector<std::unordered_map<uint64_t, size_t>> seg_map(nsegment);
    std::vector<std::vector<std::vector<int64_t>>> seg_groups(nsegment);
    for (int64_t t = 0; t < nterms; ++t) {
        const int32_t sg = segment ? segment[t] : 0;
        auto &m = seg_map[sg];
        auto it = m.find(paulis[t].xmask);
        if (it == m.end()) {
            m.emplace(paulis[t].xmask, seg_groups[sg].size());
            seg_groups[sg].push_back({t});
        } else {
            seg_groups[sg][it->second].push_back(t);
        }
    }
    qfb_sum h = new qfb_sum_s;
    h->nterms = nterms;
    h->nsegment = nsegment;
    std::vector<TermDev> terms;
    terms.reserve(nterms);
    h->h_seg_g0.push_back(0);
    for (int32_t sg = 0; sg < nsegment; ++sg) {
        for (auto &grp : seg_groups[sg]) {
            GroupDev gd;
            gd.x = paulis[grp[0]].xmask;
            gd.h = highest_bit(gd.x);
            gd.begin = (int32_t)terms.size();
            bool real = true;
            for (int64_t t : grp) {
                const uint64_t x = paulis[t].xmask, z = paulis[t].zmask;
                const int ny = __builtin_popcountll(x & z) & 3;
                // c * i^ny (exact)
                double re = coeffs[t].re, im = coeffs[t].im, r2, i2;
                switch (ny) {
                    case 0: r2 = re; i2 = im; break;
                    case 1: r2 = -im; i2 = re; break;
                    case 2: r2 = -re; i2 = -im; break;
                    default: r2 = im; i2 = -re; break;
                }
                TermDev td;
                td.z = z;
                td.c = make_double2(r2, i2);
                if (i2 != 0.0) real = false;
                terms.push_back(td);
            }
            gd.end = (int32_t)terms.size();
            gd.real = real ? 1 : 0;
            h->h_groups.push_back(gd);
        }
        h->h_seg_g0.push_back((int32_t)h->h_groups.size());
    }
    h->ngroups = (int32_t)h->h_groups.size();
    h->h_terms = terms;
    // each sub-array starts on a 256-byte boundary (TermDev holds a double2)
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t gbytes = al(sizeof(GroupDev) * std::max<size_t>(1, h->h_groups.size()));
    const size_t tbytes = al(sizeof(TermDev) * std::max<size_t>(1, terms.size()));
    const size_t rbytes = al(sizeof(double2) * std::max<size_t>(1, terms.size()));
    const size_t sbytes = sizeof(int32_t) * h->h_seg_g0.size();
    std::vector<double2> rterms(terms.size());
    for (size_t t = 0; t < terms.size(); ++t) {
        double zb;
        std::memcpy(&zb, &terms[t].z, sizeof(double));
        rterms[t] = make_double2(zb, terms[t].c.x);
    }
    int rc = dev_alloc(&h->blob, gbytes + tbytes + rbytes + sbytes);
    if (rc) {
        delete h;
        return rc;
    }
    h->d_groups = (GroupDev *)h->blob;
    h->d_terms = (TermDev *)((char *)h->blob + gbytes);
    h->d_rterms = (double2 *)((char *)h->blob + gbytes + tbytes);
    h->d_seg_g0 = (int32_t *)((char *)h->blob + gbytes + tbytes + rbytes);
    cudaError_t e = cudaSuccess;
    if (!h->h_groups.empty())
        e = cudaMemcpyAsync(h->d_groups, h->h_groups.data(), sizeof(GroupDev) * h->h_groups.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !terms.empty())
        e = cudaMemcpyAsync(h->d_terms, terms.data(), sizeof(TermDev) * terms.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !rterms.empty())
        e = cudaMemcpyAsync(h->d_rterms, rterms.data(), sizeof(double2) * rterms.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->d_seg_g0, h->h_seg_g0.data(), sbytes, cudaMemcpyHostToDevice,
                            t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);  // host vectors may go away
    if (e != cudaSuccess) {
        dev_free(h->blob);
        delete h;
        return cuda_fail(e, "qfb_sum_create upload");
    }
    *out = h;
    return QFB_OK;
}

int qfb_sum_destroy(qfb_sum h) {
    if (!h) return QFB_OK;
    dev_free(h->blob);
    delete h;
    return QFB_OK;
}

int qfb_sum_info(qfb_sum h, int64_t *nterms, int64_t *ngroups, int32_t *nsegment) {
    if (!h) return fail(QFB_EINVAL, "qfb_sum_info: null sum");
    if (nterms) *nterms = h->nterms;
    if (ngroups) *ngroups = h->ngroups;
    if (nsegment) *nsegment = h->nsegment;
    return QFB_OK;
}

int qfb_sum_expval(qfb_sum h, qfb_state bra, qfb_state ket, qfb_complex *out) {
    if (!h || !bra || !ket || !out) return fail(QFB_EINVAL, "qfb_sum_expval: null argument");
    if (bra->nqubit != ket->nqubit || bra->nbatch != ket->nbatch)
        return fail(QFB_EINVAL, "qfb_sum_expval: bra and ket shapes differ");
    for (const auto &g : h->h_groups)
        if (g.h >= bra->nqubit)
            return fail(QFB_EINVAL, "qfb_sum_expval: operator acts on qubit %d of a %d-qubit state",
                        g.h, bra->nqubit);
    const int B = bra->nbatch;
    const size_t nout = (size_t)B * h->nsegment;
    if (h->ngroups == 0) {
        for (size_t i = 0; i < nout; ++i) out[i] = qfb_complex{0.0, 0.0};
        return QFB_OK;
    }
    const uint64_t npair = bra->nbasis >> 1;
    const unsigned chunks = chunks_for(npair, B, h->ngroups);
    const size_t nparts = (size_t)B * h->ngroups * chunks;
    void *buf = nullptr;
    int rc = dev_alloc(&buf, sizeof(double2) * (nparts + nout));
    if (rc) return rc;
    double2 *partial = (double2 *)buf;
    double2 *res = partial + nparts;
    for (int32_t g0 = 0; g0 < h->ngroups; g0 += 65535) {
        // grid.y is limited to 65535 groups per launch
        const int32_t ng = std::min<int32_t>(65535, h->ngroups - g0);
        if (g0 == 0 && ng == h->ngroups) {
            k_sum_expval<<<dim3(chunks, ng, B), 256, 0, t_stream>>>(
                bra->d, ket->d, bra->nbasis, h->d_groups, h->d_terms, h->ngroups, partial);
            QFB_LAUNCHED();
        } else {
            dev_free(buf);
            return fail(QFB_ENOSYS, "qfb_sum_expval: more than 65535 x-groups");
        }
    }
    k_seg_sum<<<dim3(h->nsegment, B), 256, 0, t_stream>>>(partial, h->d_seg_g0, h->ngroups,
                                                          chunks, res);
    QFB_LAUNCHED();
    QFB_CUDA(cudaMemcpyAsync(out, res, sizeof(double2) * nout, cudaMemcpyDeviceToHost, t_stream));
    dev_free(buf);
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_sum_apply(qfb_sum h, qfb_state dst, qfb_state src) {
    if (!h || !dst || !src) return fail(QFB_EINVAL, "qfb_sum_apply: null argument");
    if (dst == src) return fail(QFB_EINVAL, "qfb_sum_apply: dst and src must differ");
    if (dst->nqubit != src->nqubit || dst->nbatch != src->nbatch)
        return fail(QFB_EINVAL, "qfb_sum_apply: dst and src shapes differ");
    for (const auto &g : h->h_groups)
        if (g.h >= src->nqubit)
            return fail(QFB_EINVAL, "qfb_sum_apply: operator acts on qubit %d of a %d-qubit state",
                        g.h, src->nqubit);
    int rc = ensure_tiled(h, src->nqubit);
    if (rc) return rc;
    return enqueue_sum_apply(h, dst->d, src->d, src->nbasis, src->nbatch);
}

int qfb_prog_create(const qfb_pauli *paulis, const double *scale, const int32_t *param,
                    int64_t nstrings, int32_t nparam, qfb_prog *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_prog_create: null output");
    *out = nullptr;
    if (nstrings < 0 || (nstrings > 0 && (!paulis || !scale || !param)))
        return fail(QFB_EINVAL, "qfb_prog_create: bad arrays");
    if (nparam < 0) return fail(QFB_EINVAL, "qfb_prog_create: nparam < 0");
    for (int64_t k = 0; k < nstrings; ++k)
        if (param[k] < 0 || param[k] >= nparam)
            return fail(QFB_EINVAL, "qfb_prog_create: string %lld uses parameter %d of %d",
                        (long long)k, param[k], nparam);
    qfb_prog p = new qfb_prog_s;
    p->nstrings = nstrings;
    p->nparam = nparam;
    p->p_step0.assign(nparam, -1);
    p->p_step1.assign(nparam, -1);
    for (int64_t k = 0; k < nstrings; ++k) {
        StrDev sd;
        sd.z = paulis[k].zmask;
        sd.ny = __builtin_popcountll(paulis[k].xmask & paulis[k].zmask) & 3;
        sd.param = param[k];
        sd.scale = scale[k];
        p->h_strs.push_back(sd);
        const bool extend = !p->h_steps.empty() && p->h_steps.back().x == paulis[k].xmask &&
                            p->h_steps.back().param == param[k] &&
                            p->h_steps.back().ns < kMaxStepStrings;
        if (extend) {
            p->h_steps.back().ns += 1;
        } else {
            StepDev st;
            st.x = paulis[k].xmask;
            st.h = highest_bit(st.x);
            st.s0 = (int32_t)k;
            st.ns = 1;
            st.param = param[k];
            st.tab = -1;
            st.nd = 0;
            st.dpos = 0;
            st.zbase = 0;
            st.gamma = 0.0;
            st.na = -1;
            st.zpos = 0;
            for (int a = 0; a < kMaxActive; ++a) {
                st.patidx[a] = 0;
                st.patbits[a] = 0;
            }
            p->h_steps.push_back(st);
        }
    }
    // steps of each parameter must be contiguous for the reverse gradient sweep
    for (size_t s = 0; s < p->h_steps.size(); ++s) {
        const int32_t mu = p->h_steps[s].param;
        if (p->p_step0[mu] < 0) {
            p->p_step0[mu] = (int32_t)s;
        } else if (p->p_step1[mu] != (int32_t)s) {
            p->params_contiguous = false;
        }
        p->p_step1[mu] = (int32_t)s + 1;
    }
    for (auto &st : p->h_steps) make_table(p, st);
    const size_t sb = (sizeof(StrDev) * std::max<size_t>(1, p->h_strs.size()) + 255) & ~(size_t)255;
    const size_t tb = sizeof(double2) * std::max<size_t>(1, p->h_tab.size());
    int rc = dev_alloc(&p->blob, sb + tb);
    if (rc) {
        delete p;
        return rc;
    }
    p->d_strs = (StrDev *)p->blob;
    p->d_tab = (double2 *)((char *)p->blob + sb);
    cudaError_t e = cudaSuccess;
    if (!p->h_strs.empty())
        e = cudaMemcpyAsync(p->d_strs, p->h_strs.data(), sizeof(StrDev) * p->h_strs.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !p->h_tab.empty())
        e = cudaMemcpyAsync(p->d_tab, p->h_tab.data(), sizeof(double2) * p->h_tab.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e != cudaSuccess) {
        dev_free(p->blob);
        delete p;
        return cuda_fail(e, "qfb_prog_create upload");
    }
    *out = p;
    return QFB_OK;
}

int qfb_prog_destroy(qfb_prog p) {
    if (!p) return QFB_OK;
    dev_free(p->blob);
    delete p;
    return QFB_OK;
}

int qfb_prog_info(qfb_prog p, int64_t *nstrings, int64_t *nsteps, int32_t *nparam) {
    if (!p) return fail(QFB_EINVAL, "qfb_prog_info: null program");
    if (nstrings) *nstrings = p->nstrings;
    if (nsteps) *nsteps = (int64_t)p->h_steps.size();
    if (nparam) *nparam = p->nparam;
    return QFB_OK;
}

static int check_prog_state(qfb_prog p, qfb_state s, int32_t nrows, const char *who) {
    if (nrows != 1 && nrows != s->nbatch)
        return fail(QFB_EINVAL, "%s: %d parameter rows for %d slots", who, nrows, s->nbatch);
    for (const auto &st : p->h_steps)
        if (st.h >= s->nqubit)
            return fail(QFB_EINVAL, "%s: program acts on qubit %d of a %d-qubit state", who, st.h,
                        s->nqubit);
    for (const auto &sd : p->h_strs)
        if (sd.z >> s->nqubit)
            return fail(QFB_EINVAL, "%s: program acts on a qubit beyond %d", who, s->nqubit);
    return QFB_OK;
}

// ---- enqueue helpers: kernels only, no allocation, no host synchronisation --

static int enqueue_step(const qfb_prog_s *p, const StepDev &st, double2 *psi, uint64_t nbasis,
                        int B, const double *d_par, int bcast, int sign, int reverse) {
    StepParams sp{p->d_strs, d_par, p->d_tab, p->nparam, bcast, sign, reverse};
    const dim3 grid(grid_for(nbasis >> 1, 256, 4), B);
    k_prog_step<<<grid, 256, 0, t_stream>>>(psi, nbasis, st, sp);
    QFB_LAUNCHED();
    return QFB_OK;
}

// U (sign +1) or U^dagger (sign -1).  Forward application runs the window
// plan of this qubit count when one has been built (ensure_plans).
static int enqueue_prog(const qfb_prog_s *p, double2 *psi, int nqubit, int B,
                        const double *d_par, int bcast, int sign) {
    const uint64_t nbasis = 1ull << nqubit;
    const WinPlan *pl = (sign > 0) ? p->fwd_plan[nqubit] : nullptr;
    if (pl) {
        int rc = set_win_smem(pl->smem_max, 1);
        if (rc) return rc;
        for (const auto &w : pl->wins) {
            rc = (w.global_step >= 0)
                     ? enqueue_step(p, p->h_steps[w.global_step], psi, nbasis, B, d_par, bcast, 1,
                                    0)
                     : launch_window(pl, w, psi, nullptr, nbasis, B, d_par, p->nparam, bcast,
                                     nullptr);
            if (rc) return rc;
        }
        return QFB_OK;
    }
    const int64_t ns = (int64_t)p->h_steps.size();
    for (int64_t k = 0; k < ns; ++k) {
        int rc = enqueue_step(p, p->h_steps[sign > 0 ? k : ns - 1 - k], psi, nbasis, B, d_par,
                              bcast, sign, sign > 0 ? 0 : 1);
        if (rc) return rc;
    }
    return QFB_OK;
}

static int tile_bits_for(int nqubit) { return std::min(kApplyTileBits, nqubit); }

static int ensure_tiled(qfb_sum_s *h, int nqubit) {
    const int m = tile_bits_for(nqubit);
    if (h->tiled[m]) return QFB_OK;
    static std::once_flag smem_once;
    static cudaError_t smem_err = cudaSuccess;
    std::call_once(smem_once, [] {
        smem_err = cudaFuncSetAttribute(k_sum_apply_tiled<uint32_t>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kApplySmem);
        if (smem_err == cudaSuccess)
            smem_err = cudaFuncSetAttribute(k_sum_apply_tiled<uint64_t>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kApplySmem);
    });
    if (smem_err != cudaSuccess) return cuda_fail(smem_err, "tiled apply shared memory");
    std::vector<int32_t> order(h->h_groups.size());
    for (size_t g = 0; g < order.size(); ++g) order[g] = (int32_t)g;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return (h->h_groups[a].x >> m) < (h->h_groups[b].x >> m);
    });
    std::vector<GroupDev> gs;
    std::vector<int32_t> hi0;
    std::vector<uint64_t> hiv;
    for (size_t i = 0; i < order.size(); ++i) {
        const GroupDev &g = h->h_groups[order[i]];
        const uint64_t hi = g.x >> m;
        if (hiv.empty() || hiv.back() != hi) {
            hiv.push_back(hi);
            hi0.push_back((int32_t)i);
        }
        gs.push_back(g);
    }
    hi0.push_back((int32_t)gs.size());
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t gb = al(sizeof(GroupDev) * std::max<size_t>(1, gs.size()));
    const size_t hb = al(sizeof(int32_t) * hi0.size());
    const size_t vb = sizeof(uint64_t) * std::max<size_t>(1, hiv.size());
    TiledView *tv = new TiledView;
    tv->m = m;
    tv->nhi = (int)hiv.size();
    int rc = dev_alloc(&tv->blob, gb + hb + vb);
    if (rc) {
        delete tv;
        return rc;
    }
    tv->d_groups = (GroupDev *)tv->blob;
    tv->d_hi0 = (int32_t *)((char *)tv->blob + gb);
    tv->d_hival = (uint64_t *)((char *)tv->blob + gb + hb);
    cudaError_t e = cudaSuccess;
    if (!gs.empty())
        e = cudaMemcpyAsync(tv->d_groups, gs.data(), sizeof(GroupDev) * gs.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(tv->d_hi0, hi0.data(), sizeof(int32_t) * hi0.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !hiv.empty())
        e = cudaMemcpyAsync(tv->d_hival, hiv.data(), sizeof(uint64_t) * hiv.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e != cudaSuccess) {
        dev_free(tv->blob);
        delete tv;
        return cuda_fail(e, "tiled group view upload");
    }
    h->tiled[m] = tv;
    return QFB_OK;
}

static int enqueue_sum_apply(const qfb_sum_s *h, double2 *dst, const double2 *src,
                             uint64_t nbasis, int B) {
    const int nq = 63 - __builtin_clzll(nbasis);
    const TiledView *tv = h->tiled[tile_bits_for(nq)];
    if (tv && h->ngroups > 0) {
        const dim3 grid((unsigned)(nbasis >> tv->m), (unsigned)((B + kApplyStates - 1) / kApplyStates));
        if (nq <= 32)
            k_sum_apply_tiled<uint32_t><<<grid, 1 << kApplyTileBits, kApplySmem, t_stream>>>(
                dst, src, nbasis, B, tv->m, tv->d_groups, tv->d_hi0, tv->d_hival, tv->nhi,
                h->d_terms, h->d_rterms);
        else
            k_sum_apply_tiled<uint64_t><<<grid, 1 << kApplyTileBits, kApplySmem, t_stream>>>(
                dst, src, nbasis, B, tv->m, tv->d_groups, tv->d_hi0, tv->d_hival, tv->nhi,
                h->d_terms, h->d_rterms);
        QFB_LAUNCHED();
        return QFB_OK;
    }
    if (nbasis >= 4) {
        const dim3 grid(grid_for(nbasis >> 2, 256), B);
        k_sum_apply4<<<grid, 256, 0, t_stream>>>(dst, src, nbasis, h->d_groups, h->d_terms,
                                                 h->d_rterms, h->ngroups);
    } else {
        const dim3 grid(grid_for(nbasis, 256), B);
        k_sum_apply<<<grid, 256, 0, t_stream>>>(dst, src, nbasis, h->d_groups, h->d_terms,
                                                h->ngroups);
    }
    QFB_LAUNCHED();
    return QFB_OK;
}

// The reverse sweep of one parameter with the per-step kernels; partial
// rows are laid out [step][slot][chunks].
static int enqueue_grad_mu(const qfb_prog_s *kp, const qfb_prog_s *up, int mu, double2 *psi,
                           double2 *sig, uint64_t nbasis, int B, const double *d_par, int bcast,
                           double2 *partial, unsigned chunks) {
    // fused step: U^dagger exactly (strings reversed, angles negated); separate
    // un-rotation: up's strings in forward order with negated angles, as the
    // reference's Trotter product of -t K does (uccvqeabc.py:208-238)
    StepParams kpar{kp->d_strs, d_par, kp->d_tab, kp->nparam, bcast, -1, 1};
    StepParams upar{up->d_strs, d_par, up->d_tab, up->nparam, bcast, -1, 0};
    const dim3 grid(chunks, B);
    const int32_t s0 = kp->p_step0[mu], s1 = kp->p_step1[mu];
    const bool last = (mu == 0);
    if (kp == up && s0 >= 0 && s1 - s0 == 1) {
        k_grad_step<<<grid, 256, 0, t_stream>>>(psi, sig, nbasis, kp->h_steps[s0], kpar,
                                                last ? 0 : 1, s0, partial);
        QFB_LAUNCHED();
        return QFB_OK;
    }
    // first every inner product on (psi_mu, sigma_mu) ...
    for (int32_t s = s0; s >= 0 && s < s1; ++s) {
        k_grad_step<<<grid, 256, 0, t_stream>>>(psi, sig, nbasis, kp->h_steps[s], kpar, 0, s,
                                                partial);
        QFB_LAUNCHED();
    }
    if (last) return QFB_OK;
    // ... then U_mu^dagger on both states, steps in reverse order
    const dim3 g2(grid_for(nbasis >> 1, 256, 4), B);
    const int32_t u0 = up->p_step0[mu], u1 = up->p_step1[mu];
    for (int32_t s = u0; u0 >= 0 && s < u1; ++s) {
        k_prog_step<<<g2, 256, 0, t_stream>>>(psi, nbasis, up->h_steps[s], upar);
        QFB_LAUNCHED();
        k_prog_step<<<g2, 256, 0, t_stream>>>(sig, nbasis, up->h_steps[s], upar);
        QFB_LAUNCHED();
    }
    return QFB_OK;
}

// Partial-row chunks of the gradient sweep for this program and qubit count.
static unsigned grad_chunks(const qfb_prog_s *kp, int nqubit, int B) {
    const WinPlan *pl = kp->grad_plan[nqubit];
    return pl ? (unsigned)pl->ntiles() : chunks_for((1ull << nqubit) >> 1, B, 1);
}

// Reverse sweep of the adjoint gradient.  partial holds nsteps(kp) * B *
// chunks entries (chunks = grad_chunks); row (s * B + b) receives step s's
// share of <sigma|K_mu|psi>.
static int enqueue_gradient(const qfb_prog_s *kp, const qfb_prog_s *up, double2 *psi,
                            double2 *sig, int nqubit, int B, const double *d_par, int bcast,
                            double2 *partial) {
    const uint64_t nbasis = 1ull << nqubit;
    const unsigned chunks = grad_chunks(kp, nqubit, B);
    const WinPlan *pl = (kp->grad_plan_u[nqubit] == up) ? kp->grad_plan[nqubit] : nullptr;
    if (pl) {
        int rc = set_win_smem(pl->smem_max, 2);
        if (rc) return rc;
        for (const auto &w : pl->wins) {
            rc = (w.global_mu >= 0)
                     ? enqueue_grad_mu(kp, up, w.global_mu, psi, sig, nbasis, B, d_par, bcast,
                                       partial, chunks)
                     : launch_window(pl, w, psi, sig, nbasis, B, d_par, kp->nparam, bcast,
                                     partial);
            if (rc) return rc;
        }
        return QFB_OK;
    }
    for (int mu = kp->nparam - 1; mu >= 0; --mu) {
        int rc = enqueue_grad_mu(kp, up, mu, psi, sig, nbasis, B, d_par, bcast, partial, chunks);
        if (rc) return rc;
    }
    return QFB_OK;
}

int qfb_prog_apply(qfb_prog p, qfb_state s, const double *params, int32_t nrows, int32_t sign) {
    if (!p || !s) return fail(QFB_EINVAL, "qfb_prog_apply: null argument");
    if (p->nparam > 0 && !params) return fail(QFB_EINVAL, "qfb_prog_apply: null parameters");
    if (sign != 1 && sign != -1) return fail(QFB_EINVAL, "qfb_prog_apply: sign must be +1 or -1");
    int rc = check_prog_state(p, s, nrows, "qfb_prog_apply");
    if (rc) return rc;
    if (p->h_steps.empty()) return QFB_OK;
    if (sign > 0) {
        rc = ensure_plans(p, s->nqubit, true);
        if (rc) return rc;
    }
    double *d_par = nullptr;
    rc = upload_params(params, nrows, p->nparam, &d_par);
    if (rc) return rc;
    rc = enqueue_prog(p, s->d, s->nqubit, s->nbatch, d_par, nrows == 1 ? 1 : 0, sign);
    dev_free(d_par);
    return rc;
}

int qfb_ucc_gradient(qfb_prog kp, qfb_prog up, qfb_state psi, qfb_state sig,
                     const double *params, int32_t nrows, double *grad) {
    if (!kp || !up || !psi || !sig || !grad)
        return fail(QFB_EINVAL, "qfb_ucc_gradient: null argument");
    if (kp->nparam > 0 && !params) return fail(QFB_EINVAL, "qfb_ucc_gradient: null parameters");
    if (psi->nqubit != sig->nqubit || psi->nbatch != sig->nbatch)
        return fail(QFB_EINVAL, "qfb_ucc_gradient: psi and sigma shapes differ");
    if (psi == sig) return fail(QFB_EINVAL, "qfb_ucc_gradient: psi and sigma must differ");
    if (up->nparam != kp->nparam)
        return fail(QFB_EINVAL, "qfb_ucc_gradient: K and U programs have %d and %d parameters",
                    kp->nparam, up->nparam);
    if (!kp->params_contiguous || !up->params_contiguous)
        return fail(QFB_EINVAL, "qfb_ucc_gradient: each parameter's strings must be contiguous");
    int rc = check_prog_state(kp, psi, nrows, "qfb_ucc_gradient");
    if (rc == QFB_OK) rc = check_prog_state(up, psi, nrows, "qfb_ucc_gradient");
    if (rc) return rc;
    const int M = kp->nparam, B = psi->nbatch;
    if (M == 0) return QFB_OK;
    rc = ensure_plans(kp, psi->nqubit, false, up);
    if (rc) return rc;
    double *d_par = nullptr;
    rc = upload_params(params, nrows, M, &d_par);
    if (rc) return rc;
    const unsigned chunks = grad_chunks(kp, psi->nqubit, B);
    const size_t nrow = (size_t)std::max<size_t>(kp->h_steps.size(), 1) * B;
    void *buf = nullptr;
    rc = dev_alloc(&buf, sizeof(double2) * nrow * chunks + sizeof(double) * (size_t)B * M +
                             sizeof(int2) * M);
    if (rc) {
        dev_free(d_par);
        return rc;
    }
    double2 *partial = (double2 *)buf;
    double *d_grad = (double *)(partial + nrow * chunks);
    int2 *d_ps = (int2 *)(d_grad + (size_t)B * M);
    std::vector<int2> ps(M);
    for (int mu = 0; mu < M; ++mu)
        ps[mu] = make_int2(std::max(kp->p_step0[mu], 0), std::max(kp->p_step1[mu], 0));
    QFB_CUDA(cudaMemcpyAsync(d_ps, ps.data(), sizeof(int2) * M, cudaMemcpyHostToDevice, t_stream));
    rc = enqueue_gradient(kp, up, psi->d, sig->d, psi->nqubit, B, d_par, nrows == 1 ? 1 : 0,
                          partial);
    if (rc == QFB_OK) {
        k_grad_final<<<dim3(M, B), 128, 0, t_stream>>>(partial, d_ps, chunks, d_grad);
        QFB_LAUNCHED();
        QFB_CUDA(cudaMemcpyAsync(grad, d_grad, sizeof(double) * (size_t)B * M,
                                 cudaMemcpyDeviceToHost, t_stream));
    }
    dev_free(buf);
    dev_free(d_par);
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return rc;
}

}  // extern "C"

// ===========================================================================
// compiled dUCC evaluator
// ===========================================================================

// True when K = sum_a scale_a P_a over strings sharing the x-mask x maps |j>
// to |j ^ x> only where j and j ^ x hold equal numbers of alpha (even) and of
// beta (odd) bits.  Patterns run over the bits where K's coefficient can
// change (the strings' differing z bits and x); more than 16 such bits report
// false.
static bool strings_conserve(const StrDev *S, int ns, uint64_t x) {
    if (x == 0 || ns == 0) return true;
    const uint64_t A = 0x5555555555555555ull;
    const int hxa = __builtin_popcountll(x & A), hxb = __builtin_popcountll(x & ~A);
    if ((hxa | hxb) & 1) return false;
    uint64_t P = x;
    for (int a = 0; a < ns; ++a) P |= S[a].z ^ S[0].z;
    const int np = __builtin_popcountll(P);
    if (np > 16) return false;
    int pos[16];
    for (int i = 0; i < np; ++i) {
        pos[i] = __builtin_ctzll(P);
        P &= P - 1;
    }
    double norm = 0.0;
    for (int a = 0; a < ns; ++a) norm += std::fabs(S[a].scale);
    const double tol = 1e-13 * norm;
    static const std::complex<double> ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    for (int pat = 0; pat < (1 << np); ++pat) {
        uint64_t j = 0;
        for (int i = 0; i < np; ++i)
            if (pat >> i & 1) j |= 1ull << pos[i];
        std::complex<double> c = 0.0;
        for (int a = 0; a < ns; ++a) {
            const int par = __builtin_popcountll(j & (S[a].z ^ S[0].z)) & 1;
            c += S[a].scale * ipow[S[a].ny & 3] * (par ? -1.0 : 1.0);
        }
        if (std::abs(c) <= tol) continue;
        if (2 * __builtin_popcountll(j & x & A) != hxa || 2 * __builtin_popcountll(j & x & ~A) != hxb)
            return false;
    }
    return true;
}

// A step is exponentiated as a whole: its strings must commute (the product
// of their exponentials is then exp(theta K)) and K must keep every sector.
static bool step_conserves(const qfb_prog_s *p, const StepDev &st) {
    if (st.x == 0) return true;
    const StrDev *S = &p->h_strs[st.s0];
    for (int a = 0; a < st.ns; ++a)
        for (int b = a + 1; b < st.ns; ++b)
            if (__builtin_popcountll(st.x & (S[a].z ^ S[b].z)) & 1) return false;
    return strings_conserve(S, st.ns, st.x);
}

// A program used only for inner products <sigma|K_mu|psi> needs each
// parameter's whole operator K_mu to keep every sector: its strings are
// checked x-mask by x-mask, wherever they sit in the program.
static bool prog_sum_conserves(const qfb_prog_s *p) {
    std::unordered_map<uint64_t, std::vector<StrDev>> by_x;
    int cur = -1;
    auto flush = [&]() {
        for (auto &kv : by_x)
            if (!strings_conserve(kv.second.data(), (int)kv.second.size(), kv.first)) return false;
        by_x.clear();
        return true;
    };
    std::vector<const StepDev *> order;
    for (const auto &st : p->h_steps) order.push_back(&st);
    std::stable_sort(order.begin(), order.end(),
                     [](const StepDev *a, const StepDev *b) { return a->param < b->param; });
    for (const StepDev *st : order) {
        if (st->param != cur) {
            if (!flush()) return false;
            cur = st->param;
        }
        auto &v = by_x[st->x];
        v.insert(v.end(), p->h_strs.begin() + st->s0, p->h_strs.begin() + st->s0 + st->ns);
    }
    return flush();
}

static bool prog_conserves(const qfb_prog_s *p) {
    for (const auto &st : p->h_steps)
        if (!step_conserves(p, st)) return false;
    return true;
}

// Every index of n qubits with the reference's numbers of alpha (even) and
// beta (odd) bits, ascending; empty when the sector has 2^31 or more entries.
static std::vector<uint64_t> sector_indices(int n, uint64_t ref) {
    const uint64_t A = 0x5555555555555555ull;
    const uint64_t all = (n >= 64) ? ~0ull : (1ull << n) - 1ull;
    const int na = (n + 1) / 2, nb = n / 2;
    const int ka = __builtin_popcountll(ref & A & all), kb = __builtin_popcountll(ref & ~A & all);
    auto combos = [](int m, int k, int offset) {
        std::vector<uint64_t> out;
        if (k > m) return out;
        if (k == 0) {
            out.push_back(0);
            return out;
        }
        uint64_t c = (1ull << k) - 1ull;
        while (c < (1ull << m)) {
            uint64_t d = 0, w = c;
            while (w) {
                const int b = __builtin_ctzll(w);
                d |= 1ull << (2 * b + offset);
                w &= w - 1;
            }
            out.push_back(d);
            const uint64_t t = c | (c - 1);  // next combination (Gosper)
            c = (t + 1) | (((~t & -~t) - 1) >> (__builtin_ctzll(c) + 1));
        }
        return out;
    };
    const std::vector<uint64_t> ca = combos(na, ka, 0), cb = combos(nb, kb, 1);
    std::vector<uint64_t> sec;
    if ((double)ca.size() * (double)cb.size() >= 2147483648.0) return sec;
    sec.reserve(ca.size() * cb.size());
    for (uint64_t b : cb)
        for (uint64_t a : ca) sec.push_back(a | b);
    std::sort(sec.begin(), sec.end());
    return sec;
}

// ---------------------------------------------------------------------------
// compact sector evaluator (qfb_sector.cuh): host plan
// ---------------------------------------------------------------------------

constexpr size_t kSectorSmemMax = 200 * 1024;  // psi + sigma of one parameter set
constexpr int kSectorThreads = 512;
constexpr int kSectorHSlicesMax = 64;  // row slices of k_sector_h
constexpr int kHChains = 4;            // concurrent x-group chains of H without rows
static int g_ucc_compact = 1;  // process-wide: use the compact evaluator when it applies
// qfb_ucc_config 4 and 5: complex state storage even where every coefficient is real
static bool ucc_complex_states() { return g_ucc_compact == 4 || g_ucc_compact == 5; }

// Rows of H on the compact sector: row i (the sector index of det[i]) holds,
// for every group x connecting det[i] to j = det[i] ^ x inside the sector,
// the column of j and f_x(j) = sum_t c_t (-1)^popcount(j & z_t).  Pass 1
// (col == nullptr) counts the entries of each row.
__global__ void k_sector_rows(const uint64_t *__restrict__ det, int nsec,
                              const SecGroup *__restrict__ groups, int ngroups,
                              const TermDev *__restrict__ terms, const double2 *__restrict__ rterms,
                              const int32_t *__restrict__ arank, const int32_t *__restrict__ brank,
                              int nbeta, int nqubit, const int32_t *__restrict__ rowptr,
                              int32_t *__restrict__ count, uint32_t *__restrict__ col,
                              double *__restrict__ val_r, double2 *__restrict__ val_c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsec) return;
    const uint64_t k = det[i];
    const uint64_t A = 0x5555555555555555ull;
    int e = rowptr ? rowptr[i] : 0, c = 0;
    for (int g = 0; g < ngroups; ++g) {
        const SecGroup gr = groups[g];
        const uint64_t kx = k & gr.x;
        if ((__popcll(kx & A) | __popcll(kx & ~A) << 8) != gr.halves) continue;
        if (!col) {
            ++c;
            continue;
        }
        const uint64_t j = k ^ gr.x;
        double2 f = make_double2(0.0, 0.0);
        if (gr.real) {
            for (int t = gr.begin; t < gr.end; ++t) {
                const double2 zc = rterms[t];
                f.x += parity64(j & (uint64_t)__double_as_longlong(zc.x)) ? -zc.y : zc.y;
            }
        } else {
            for (int t = gr.begin; t < gr.end; ++t) {
                const double2 cc = terms[t].c;
                if (parity64(j & terms[t].z)) { f.x -= cc.x; f.y -= cc.y; }
                else { f.x += cc.x; f.y += cc.y; }
            }
        }
        uint32_t ca = 0, cb = 0;
        for (int q = 0, ia = 0, ib = 0; q < nqubit; ++q) {
            if (q & 1) cb |= (uint32_t)((j >> q) & 1ull) << ib++;
            else ca |= (uint32_t)((j >> q) & 1ull) << ia++;
        }
        col[e] = (uint32_t)(arank[ca] * nbeta + brank[cb]);
        if (val_c) val_c[e] = f;
        else val_r[e] = f.x;
        ++e;
    }
    if (!col) count[i] = c;
}

// One kernel's records (qfbs::SStream) on the host.
struct StreamHost {
    std::vector<uint4> rec;
    std::vector<int2> span;
    std::vector<int32_t> param;
    int maxw = 0;
};

// A step of a program in compact form: its patterns with their alpha and
// beta lists (entries of the lists follow in `ents`).
struct CStep {
    int32_t param = 0;
    double gamma = 0.0;
    struct Pat {
        std::vector<qfbs::SEntry> a, b;
        double2 gn, hn;
    };
    std::vector<Pat> pats;
};

// Device copies of a plan's record streams (shared by its evaluators).
struct SectorPlanDev {
    void *blob = nullptr;
    size_t bytes = 0;
    const uint4 *frec = nullptr, *srec = nullptr;
    const int2 *fspan = nullptr, *sspan = nullptr;
    const int32_t *fparam = nullptr, *sparam = nullptr;
    ~SectorPlanDev() { dev_free(blob); }
};

// Device copies of a plan's pair-list streams (qfbs::PStream) for one bank
// slot width, uploaded once and shared by the plan's evaluators.
struct PairPlanDev {
    void *blob = nullptr;
    size_t bytes = 0;
    qfbs::PStream fwd{}, sweep{};
    std::vector<qfbs::PHead> fwd_hd;  // host copy (residual streams run it in reverse)
    ~PairPlanDev() { dev_free(blob); }
};

struct SectorPlan {
    int na_orb = 0, nb_orb = 0, nalpha = 0, nbeta = 0, nsec = 0, ref_i = 0;
    int ka = 0, kb = 0;  // alpha and beta electrons of the sector
    std::shared_ptr<SectorPlanDev> dev;
    std::shared_ptr<PairPlanDev> pdev[2];  // pair lists ordered for 8 / 16 bank slots
    std::vector<uint64_t> adet, bdet;
    std::vector<int32_t> arank, brank;
    std::vector<CStep> fsteps, ksteps, usteps;
    std::vector<int2> kmu, umu;
    int fused = 0;
    StreamHost fwd, sweep;
    struct SweepItem {
        int unrot;  // step of usteps (1) or ksteps (0)
        int step, flags, row;
    };
    std::vector<SweepItem> sweep_items;  // the sweep stream's records, in order
};

static uint32_t pext_parity_bits(uint64_t v, int odd, int n) {
    uint32_t r = 0;
    for (int q = odd, k = 0; q < n; q += 2, ++k) r |= (uint32_t)((v >> q) & 1ull) << k;
    return r;
}

// Strings of one spin (odd = 0 alpha on even qubits, 1 beta on odd qubits)
// whose bits on P equal want's, with their partner ranks and sign bits.
// false: a partner leaves the sector.
static bool sector_list(const SectorPlan &sp, int odd, int n, uint64_t P, uint64_t want,
                        uint64_t x, uint64_t zb, std::vector<qfbs::SEntry> &out) {
    const uint64_t M = odd ? 0xAAAAAAAAAAAAAAAAull : 0x5555555555555555ull;
    const std::vector<uint64_t> &det = odd ? sp.bdet : sp.adet;
    const std::vector<int32_t> &rank = odd ? sp.brank : sp.arank;
    out.clear();
    for (size_t r = 0; r < det.size(); ++r) {
        if ((det[r] & P & M) != (want & P & M)) continue;
        const int32_t pr = rank[pext_parity_bits(det[r] ^ (x & M), odd, n)];
        if (pr < 0) return false;
        qfbs::SEntry e;
        e.r0 = (uint16_t)r;
        e.r1 = (uint16_t)pr;
        e.s = (uint32_t)(__builtin_popcountll(det[r] & zb & M) & 1);
        out.push_back(e);
    }
    return true;
}

static bool sector_steps(const SectorPlan &sp, const qfb_prog_s *p, int n,
                         std::vector<CStep> &out) {
    for (const StepDev &st : p->h_steps) {
        if (st.tab < 0 || st.na <= 0 || st.x == 0) return false;
        uint64_t P = 1ull << st.h;
        for (int i = 0; i < st.nd; ++i) P |= 1ull << ((st.dpos >> (6 * i)) & 63);
        CStep cs;
        cs.param = st.param;
        cs.gamma = st.gamma;
        for (int a = 0; a < st.na; ++a) {
            CStep::Pat pt;
            if (!sector_list(sp, 0, n, P, st.patbits[a], st.x, st.zbase, pt.a)) return false;
            if (!sector_list(sp, 1, n, P, st.patbits[a], st.x, st.zbase, pt.b)) return false;
            if (pt.a.empty() || pt.b.empty()) continue;
            pt.gn = p->h_tab[st.tab + 2 * st.patidx[a]];
            pt.hn = p->h_tab[st.tab + 2 * st.patidx[a] + 1];
            cs.pats.push_back(std::move(pt));
        }
        out.push_back(std::move(cs));
    }
    return true;
}

// Append one record (header, patterns, their lists) to a stream; false when
// it outgrows one 16-byte word per thread or 16-bit list offsets.
static bool push_record(StreamHost &S, const CStep &cs, int flags, int row,
                        int max_words = kSectorThreads) {
    const int np = (int)cs.pats.size();
    if (np > 255) return false;
    size_t nent = 0;
    for (const auto &pt : cs.pats) nent += pt.a.size() + pt.b.size();
    const size_t bytes = sizeof(qfbs::RHead) + np * sizeof(qfbs::RPat) + nent * sizeof(qfbs::SEntry);
    const int words = (int)((bytes + 15) / 16);
    if (words > max_words) return false;
    std::vector<uint4> w((size_t)words, make_uint4(0, 0, 0, 0));
    char *base = (char *)w.data();
    qfbs::RHead hd;
    hd.npf = np | (flags << 8);
    hd.row = row;
    hd.gamma = cs.gamma;
    std::memcpy(base, &hd, sizeof(hd));
    size_t e = (sizeof(qfbs::RHead) + np * sizeof(qfbs::RPat)) / sizeof(qfbs::SEntry);
    for (int k = 0; k < np; ++k) {
        const auto &pt = cs.pats[k];
        qfbs::RPat rp{};
        rp.a0 = (uint16_t)e;
        rp.na = (uint16_t)pt.a.size();
        std::memcpy(base + e * sizeof(qfbs::SEntry), pt.a.data(), pt.a.size() * sizeof(qfbs::SEntry));
        e += pt.a.size();
        rp.b0 = (uint16_t)e;
        rp.nb = (uint16_t)pt.b.size();
        std::memcpy(base + e * sizeof(qfbs::SEntry), pt.b.data(), pt.b.size() * sizeof(qfbs::SEntry));
        e += pt.b.size();
        if (e > 65535) return false;
        rp.inv = (pt.b.size() == 1) ? 0u
                                    : (uint32_t)(((1ull << 32) + pt.b.size() - 1) / pt.b.size());
        rp.gn = pt.gn;
        rp.hn = pt.hn;
        std::memcpy(base + sizeof(qfbs::RHead) + k * sizeof(qfbs::RPat), &rp, sizeof(rp));
    }
    S.span.push_back(make_int2((int)S.rec.size(), words));
    S.param.push_back(cs.param);
    S.rec.insert(S.rec.end(), w.begin(), w.end());
    S.maxw = std::max(S.maxw, words);
    return true;
}

// The compact plan of an evaluator, or false when it does not apply (a step
// outside the Givens form, a sector too large for shared memory, ranks that
// do not fit 16 bits, a step record larger than the block).
static bool build_sector_plan(SectorPlan &sp, const qfb_prog_s *fp, const qfb_prog_s *kp,
                              const qfb_prog_s *up, int n, uint64_t ref, bool shared = true) {
    const int mw = 1 << 30;  // records of any size (the shared path reads pair lists)
    const uint64_t A = 0x5555555555555555ull;
    const uint64_t all = (1ull << n) - 1ull;
    sp.na_orb = (n + 1) / 2;
    sp.nb_orb = n / 2;
    if (sp.na_orb > 20) return false;
    const int ka = __builtin_popcountll(ref & A & all), kb = __builtin_popcountll(ref & ~A & all);
    sp.ka = ka;
    sp.kb = kb;
    auto strings = [&](int m, int k, int odd, std::vector<uint64_t> &det, std::vector<int32_t> &rank) {
        rank.assign((size_t)1 << m, -1);
        if (k > m) return;
        uint64_t c = (k == 0) ? 0 : ((1ull << k) - 1ull);
        while (true) {
            uint64_t d = 0;
            for (int b = 0; b < m; ++b)
                if (c >> b & 1ull) d |= 1ull << (2 * b + odd);
            rank[c] = (int32_t)det.size();
            det.push_back(d);
            if (k == 0) break;
            const uint64_t t = c | (c - 1);
            c = (t + 1) | (((~t & -~t) - 1) >> (__builtin_ctzll(c) + 1));
            if (c >= (1ull << m)) break;
        }
    };
    strings(sp.na_orb, ka, 0, sp.adet, sp.arank);
    strings(sp.nb_orb, kb, 1, sp.bdet, sp.brank);
    sp.nalpha = (int)sp.adet.size();
    sp.nbeta = (int)sp.bdet.size();
    if (sp.nalpha == 0 || sp.nbeta == 0 || sp.nalpha > 65535 || sp.nbeta > 65535) return false;
    const size_t nsec = (size_t)sp.nalpha * sp.nbeta;
    if (shared && nsec * 2 * sizeof(double2) > kSectorSmemMax) return false;
    if (shared && nsec > (1u << qfbs::kPairIdxBits)) return false;  // pair words hold 14-bit indices
    if (nsec >= (1ull << 31)) return false;
    sp.nsec = (int)nsec;
    sp.ref_i = sp.arank[pext_parity_bits(ref, 0, n)] * sp.nbeta + sp.brank[pext_parity_bits(ref, 1, n)];
    if (!sector_steps(sp, fp, n, sp.fsteps)) return false;
    for (const CStep &cs : sp.fsteps)
        if (!push_record(sp.fwd, cs, qfbs::R_ROT, -1, mw)) return false;
    if (kp) {
        if (!sector_steps(sp, kp, n, sp.ksteps)) return false;
        if (!sector_steps(sp, up, n, sp.usteps)) return false;
        const int M = kp->nparam;
        sp.fused = (kp == up) ? 1 : 0;
        for (int mu = 0; mu < M; ++mu)
            if (kp->p_step0[mu] < 0 || kp->p_step1[mu] - kp->p_step0[mu] != 1) sp.fused = 0;
        // the reverse sweep in execution order (uccvqeabc.py:122-251): for mu
        // from last to first, <sigma|K_mu|psi> on each K step, then (mu > 0)
        // U_mu^dagger on both states; a single step that is both K and U does
        // the two at once
        auto sweep_rec = [&](int unrot, int s, int fl, int row) {
            sp.sweep_items.push_back(SectorPlan::SweepItem{unrot, s, fl, row});
            return push_record(sp.sweep, unrot ? sp.usteps[s] : sp.ksteps[s], fl, row, mw);
        };
        for (int mu = M - 1; mu >= 0; --mu) {
            const int s0 = kp->p_step0[mu], s1 = kp->p_step1[mu];
            if (sp.fused) {
                const int fl = mu > 0 ? (qfbs::R_ROT | qfbs::R_IP | qfbs::R_TWO) : qfbs::R_IP;
                if (!sweep_rec(0, s0, fl, s0)) return false;
                continue;
            }
            for (int s = s0; s >= 0 && s < s1; ++s)
                if (!sweep_rec(0, s, qfbs::R_IP, s)) return false;
            if (mu == 0) break;
            const int u0 = up->p_step0[mu], u1 = up->p_step1[mu];
            for (int s = u0; u0 >= 0 && s < u1; ++s)
                if (!sweep_rec(1, s, qfbs::R_ROT | qfbs::R_TWO, -1)) return false;
        }
    }
    if (!shared) return true;
    const size_t ang = sizeof(qfbs::PSmem<double2>) * std::max(sp.fwd.span.size(), sp.sweep.span.size());
    if (nsec * 2 * sizeof(double2) + ang > kSectorSmemMax) return false;
    return true;
}

// One kernel's pair-list records (qfbs::PStream) on the host.
struct PairHost {
    std::vector<qfbs::PHead> hd;
    std::vector<uint32_t> pair;
    std::vector<double2> coef;  // per pattern: gn, hn
};

constexpr uint32_t kPairIdxMask = (1u << qfbs::kPairIdxBits) - 1u;
static inline uint32_t pair_i0(uint32_t w) { return w & kPairIdxMask; }
static inline uint32_t pair_i1(uint32_t w) { return (w >> qfbs::kPairIdxBits) & kPairIdxMask; }

// Order the pairs of one record so that each run of S consecutive pairs (the
// lanes of a half warp reading 8-byte amplitudes, S = 16, or of a quarter warp
// reading 16-byte amplitudes, S = 8) reads S distinct bank slots (index mod S)
// at i0 and S distinct slots at i1 as far as the record allows.  Each run is a
// maximum matching between i0 slots and i1 slots over the pairs left (Kuhn's
// augmenting paths, fullest slots tried first), topped up from the fullest
// (i0 slot, i1 slot) buckets.  Only the order in which threads take the
// record's pairs changes; the pairs of a record touch distinct amplitudes.
static void order_pairs(uint32_t *p, size_t n, int S) {
    if (n <= 1) return;
    std::vector<std::vector<uint32_t>> bk((size_t)S * S);
    for (size_t k = 0; k < n; ++k) {
        const uint32_t a = pair_i0(p[k]) % (uint32_t)S, b = pair_i1(p[k]) % (uint32_t)S;
        bk[(size_t)a * S + b].push_back(p[k]);
    }
    std::vector<int> d0(S), d1(S), m1(S), ord0(S), ord1(S);
    size_t out = 0;
    std::function<bool(int, uint32_t &)> augment = [&](int a, uint32_t &seen) -> bool {
        for (int b : ord1) {
            if (bk[(size_t)a * S + b].empty() || (seen >> b & 1u)) continue;
            seen |= 1u << b;
            if (m1[b] < 0 || augment(m1[b], seen)) {
                m1[b] = a;
                return true;
            }
        }
        return false;
    };
    while (out < n) {
        std::fill(d0.begin(), d0.end(), 0);
        std::fill(d1.begin(), d1.end(), 0);
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) {
                const int c = (int)bk[(size_t)a * S + b].size();
                d0[a] += c;
                d1[b] += c;
            }
        for (int k = 0; k < S; ++k) ord0[k] = ord1[k] = k;
        std::stable_sort(ord0.begin(), ord0.end(), [&](int x, int y) { return d0[x] > d0[y]; });
        std::stable_sort(ord1.begin(), ord1.end(), [&](int x, int y) { return d1[x] > d1[y]; });
        std::fill(m1.begin(), m1.end(), -1);
        for (int a : ord0) {
            if (!d0[a]) continue;
            uint32_t seen = 0;
            augment(a, seen);
        }
        const size_t want = std::min<size_t>((size_t)S, n - out), first = out;
        for (int b = 0; b < S; ++b)
            if (m1[b] >= 0) {
                auto &v = bk[(size_t)m1[b] * S + b];
                p[out++] = v.back();
                v.pop_back();
            }
        while (out - first < want) {  // fewer distinct slots than lanes left
            size_t best = 0;
            for (size_t k = 1; k < bk.size(); ++k)
                if (bk[k].size() > bk[best].size()) best = k;
            p[out++] = bk[best].back();
            bk[best].pop_back();
        }
    }
}

// Append one step as a pair-list record: every pair (i0, i1) of its patterns
// with the sign bit of (-1)^popcount(j0 & zbase) and the pattern's number,
// ordered for the banks.
static bool push_pairs(PairHost &P, const SectorPlan &sp, const CStep &cs, int flags, int row, int S) {
    const int npat = (int)cs.pats.size();
    if (npat > qfbs::kPairPatterns || sp.nsec > (1 << qfbs::kPairIdxBits)) return false;
    qfbs::PHead h{};
    h.p0 = (int32_t)P.pair.size();
    h.c0 = (int32_t)(P.coef.size() / 2);
    h.fl = flags | npat << 8;
    h.row = row;
    h.gamma = cs.gamma;
    h.param = cs.param;
    for (int k = 0; k < npat; ++k) {
        const auto &pt = cs.pats[k];
        P.coef.push_back(pt.gn);
        P.coef.push_back(pt.hn);
        const uint32_t pat = (uint32_t)k << (2 * qfbs::kPairIdxBits + 1);
        for (const qfbs::SEntry &ea : pt.a)
            for (const qfbs::SEntry &eb : pt.b) {
                const uint32_t i0 = (uint32_t)ea.r0 * (uint32_t)sp.nbeta + eb.r0;
                const uint32_t i1 = (uint32_t)ea.r1 * (uint32_t)sp.nbeta + eb.r1;
                const uint32_t neg = ((ea.s ^ eb.s) & 1u) << (2 * qfbs::kPairIdxBits);
                P.pair.push_back(i0 | i1 << qfbs::kPairIdxBits | neg | pat);
            }
    }
    if (P.pair.size() >= (1ull << 31)) return false;
    h.np = (int32_t)(P.pair.size() - (size_t)h.p0);
    order_pairs(P.pair.data() + h.p0, (size_t)h.np, S);
    P.hd.push_back(h);
    return true;
}

// Device bytes of one stream (headers, pair words, coefficients, each piece
// 256-byte aligned), and its upload to base.
static size_t pair_bytes(const PairHost &P) {
    auto al = [](size_t x) { return (std::max<size_t>(x, 16) + 255) & ~(size_t)255; };
    return al(sizeof(qfbs::PHead) * P.hd.size()) +
           al(sizeof(uint32_t) * (P.pair.size() + qfbs::kPairPad)) + al(sizeof(double2) * P.coef.size());
}
static int pair_upload(const PairHost &P, char *base, qfbs::PStream &out) {
    auto al = [](size_t x) { return (std::max<size_t>(x, 16) + 255) & ~(size_t)255; };
    char *hd = base, *pr = hd + al(sizeof(qfbs::PHead) * P.hd.size());
    char *cf = pr + al(sizeof(uint32_t) * (P.pair.size() + qfbs::kPairPad));
    if (!P.hd.empty())
        QFB_CUDA(cudaMemcpyAsync(hd, P.hd.data(), sizeof(qfbs::PHead) * P.hd.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    if (!P.pair.empty())
        QFB_CUDA(cudaMemcpyAsync(pr, P.pair.data(), sizeof(uint32_t) * P.pair.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaMemsetAsync(pr + sizeof(uint32_t) * P.pair.size(), 0,
                             sizeof(uint32_t) * qfbs::kPairPad, t_stream));

    if (!P.coef.empty())
        QFB_CUDA(cudaMemcpyAsync(cf, P.coef.data(), sizeof(double2) * P.coef.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    out.hd = (const qfbs::PHead *)hd;
    out.pair = (const uint32_t *)pr;
    out.coef = (const double2 *)cf;
    out.n = (int)P.hd.size();
    return QFB_OK;
}

// The plan's forward and sweep streams as pair lists ordered for S bank slots.
static int pair_plan(SectorPlan &sp, int S, std::shared_ptr<PairPlanDev> *out) {
    std::shared_ptr<PairPlanDev> &slot = sp.pdev[S == 16 ? 1 : 0];
    if (slot) {
        *out = slot;
        return QFB_OK;
    }
    PairHost F, W;
    for (const CStep &cs : sp.fsteps)
        if (!push_pairs(F, sp, cs, qfbs::R_ROT, -1, S))
            return fail(QFB_ENOSYS, "compact sector: forward step outside the pair-list limits");
    for (const auto &it : sp.sweep_items)
        if (!push_pairs(W, sp, it.unrot ? sp.usteps[it.step] : sp.ksteps[it.step], it.flags, it.row, S))
            return fail(QFB_ENOSYS, "compact sector: sweep step outside the pair-list limits");
    auto d = std::make_shared<PairPlanDev>();
    const size_t bf = pair_bytes(F), bw = pair_bytes(W);
    int rc = dev_alloc(&d->blob, bf + bw);
    if (rc) return rc;
    d->bytes = bf + bw;
    rc = pair_upload(F, (char *)d->blob, d->fwd);
    if (!rc) rc = pair_upload(W, (char *)d->blob + bf, d->sweep);
    if (!rc) QFB_CUDA(cudaStreamSynchronize(t_stream));
    if (rc) return rc;
    d->fwd_hd = F.hd;
    slot = d;
    *out = d;
    return QFB_OK;
}

struct qfb_ucc_s {
    qfb_prog_s *fwd = nullptr;
    qfb_prog_s *grad = nullptr;   // K_mu (inner products)
    qfb_prog_s *unrot = nullptr;  // U_mu (un-rotation)
    const qfb_sum_s *ham = nullptr;
    int nqubit = 0, nbatch = 0, nparam = 0;
    uint64_t nbasis = 0, ref = 0;
    unsigned vchunks = 1, gchunks = 1;
    void *blob = nullptr;
    double2 *psi = nullptr, *sig = nullptr;
    double *params = nullptr, *energy = nullptr, *gradv = nullptr;
    double2 *vpart = nullptr, *gpart = nullptr;
    int2 *psteps = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // by run mode
    uint64_t graph_kernels[5] = {0, 0, 0, 0, 0};
    // particle-number sector of the state (every program conserves it):
    // H psi is formed on these indices only; nsec == 0 means the full space
    int64_t nsec = 0;
    size_t bytes = 0;     // device bytes held (blobs)
    int compact = 0;      // compact sector evaluator (qfb_sector.cuh)
    int sreal = 0;        // compact: real states (every coefficient and H real)
    int greal = 0;        // compact in global memory: real states
    int64_t nnz = 0;      // entries of the H rows on the compact sector
    std::shared_ptr<SectorRows> rows;  // compact paths: H rows on the sector
    // compact, shared memory: k_sector_h shape (parameter sets per CTA, block
    // size, row slices), partial energies [B][slices] and group tickets
    int h_sets = 1, h_threads = kSectorThreads, h_slices = 1;
    double *h_epart = nullptr;
    unsigned *h_count = nullptr;
    qfbs::SLaunch SL{};
    void *sec = nullptr;  // uint32_t (nqubit <= 32) or uint64_t indices
    SecGroup *sgroups = nullptr;
    int nsgroups = 0;
    std::shared_ptr<SectorPlan> splan;  // compact paths: strings, ranks and step records
    // compact sector in global memory (qfb_csec.cuh)
    int gsec = 0;
    qfbg::GLaunch GL{};
    const uint4 *g_frec = nullptr, *g_srec = nullptr;  // device copies of the record streams
    unsigned g_sgrid = 1, g_hgrid = 1, g_ygrid = 1;
    double2 *g_epart = nullptr;
    // H without rows: the x-groups' launches run on kHChains concurrent
    // chains, chain k adding into its own sigma copy (k = 0: GL.sig)
    void *hblob = nullptr;  // sigma copies of chains 1..
    cudaStream_t hside[kHChains - 1] = {};
    cudaEvent_t hfork = nullptr, hjoin[kHChains - 1] = {};
    const int32_t *g_rowptr = nullptr;
    const uint32_t *g_col = nullptr;
    const double *g_vr = nullptr;
    const double2 *g_vc = nullptr;
    // ADAPT pool (qfb_ucc_set_pool): 2 Re <sigma|K_k|psi> for every pool operator k
    const qfb_prog_s *pool = nullptr;
    int npool = 0;
    void *pblob = nullptr;
    double *pgrad = nullptr;   // [B][npool]
    double2 *ppart = nullptr;  // [pool steps][B][pchunks]
    int2 *pranges = nullptr;   // pool steps of each operator
    StepDev *pool_steps = nullptr;  // full space: the pool's steps on the device
    unsigned pchunks = 1;
    qfbs::SStream pstream{};   // global-memory sector: the pool's inner-product records
    qfbs::PStream ppairs{};    // shared-memory sector: the pool's pair lists
    // PQE residuals (qfb_ucc_set_residuals): Re(<I_k|U^dagger H U|ref> phase_k)
    int nres = 0;
    void *rblob = nullptr;
    size_t rbytes = 0;
    double *res = nullptr;            // [B][nres]
    const int64_t *ridx = nullptr;    // full-space index, or compact index (-1: outside)
    const double2 *rphase = nullptr;  // [nres]
    qfbs::PStream rstream{};          // compact: forward pair lists in reverse order
    std::shared_ptr<PairPlanDev> pairs;  // compact: the plan's pair lists in use
    int64_t nprows = 1;                  // rows of the gradient partials (gradient steps)
    // compact, real states: two parameter sets per CTA in the forward kernel
    // (k_sector_forward_pr), with pair lists ordered for 16-byte slots
    int paired = 0;
    std::shared_ptr<PairPlanDev> pairs16b;
    qfbs::SLaunch SLp{};
};

// Whether every pattern of every record of a stream has real coefficients.
static bool stream_is_real(const StreamHost &S) {
    for (const int2 &sp : S.span) {
        const char *rec = (const char *)&S.rec[sp.x];
        qfbs::RHead hd;
        std::memcpy(&hd, rec, sizeof(hd));
        for (int p = 0; p < (hd.npf & 255); ++p) {
            qfbs::RPat pt;
            std::memcpy(&pt, rec + sizeof(qfbs::RHead) + p * sizeof(qfbs::RPat), sizeof(pt));
            if (pt.gn.y != 0.0 || pt.hn.y != 0.0) return false;
        }
    }
    return true;
}

// Reorder the entries of every H row so that each run of S consecutive
// entries gathers psi from S different bank slots as far as the row allows:
// S = 8 for complex states (the 8 lanes of a quarter warp in k_sector_h read
// 16-byte amplitudes, slot = column mod 8), S = 16 for real states (a half
// warp reads 8-byte amplitudes, slot = column mod 16).  Entries are bucketed
// by slot and dealt out one bucket after the other, fullest bucket first.
// Only the order of the row's sum changes.
static int sector_rows_interleave(const std::vector<int32_t> &rowptr, int64_t nnz, uint32_t *d_col,
                                  void *d_val, size_t vbytes, int S) {
    if (nnz == 0) return QFB_OK;
    std::vector<uint32_t> col((size_t)nnz), col2((size_t)nnz);
    std::vector<char> val((size_t)nnz * vbytes), val2((size_t)nnz * vbytes);
    QFB_CUDA(cudaMemcpyAsync(col.data(), d_col, sizeof(uint32_t) * nnz, cudaMemcpyDeviceToHost,
                             t_stream));
    QFB_CUDA(cudaMemcpyAsync(val.data(), d_val, vbytes * nnz, cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    std::vector<std::vector<int64_t>> bucket((size_t)S);
    std::vector<size_t> next((size_t)S);
    std::vector<int> order((size_t)S);
    const size_t nrow = rowptr.size() - 1;
    for (size_t i = 0; i < nrow; ++i) {
        for (auto &b : bucket) b.clear();
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) bucket[col[e] % (uint32_t)S].push_back(e);
        std::fill(next.begin(), next.end(), 0);
        int64_t out = rowptr[i];
        auto left = [&](int r) { return bucket[r].size() - next[r]; };
        auto emit = [&](int r) {
            const int64_t e = bucket[r][next[r]++];
            col2[out] = col[e];
            std::memcpy(&val2[(size_t)out * vbytes], &val[(size_t)e * vbytes], vbytes);
            ++out;
        };
        while (out < rowptr[i + 1]) {  // one group of (up to) S positions
            const int64_t n = std::min<int64_t>(S, rowptr[i + 1] - out);
            for (int r = 0; r < S; ++r) order[r] = r;
            std::sort(order.begin(), order.end(), [&](int a, int b) { return left(a) > left(b); });
            int64_t taken = 0;
            for (int k = 0; k < S && taken < n; ++k)
                if (left(order[k]) > 0) {
                    emit(order[k]);
                    ++taken;
                }
            while (taken < n) {  // fewer distinct slots than positions left
                int best = 0;
                for (int r = 1; r < S; ++r)
                    if (left(r) > left(best)) best = r;
                emit(best);
                ++taken;
            }
        }
    }
    QFB_CUDA(cudaMemcpyAsync(d_col, col2.data(), sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice,
                             t_stream));
    QFB_CUDA(cudaMemcpyAsync(d_val, val2.data(), vbytes * nnz, cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

constexpr double kRowsBudget = 24e9;  // bytes of H rows a global-memory sector path may hold

static_assert(sizeof(qfbg::GGroup) == sizeof(SecGroup), "GGroup mirrors SecGroup");
static_assert(sizeof(qfbg::GTerm) == sizeof(TermDev), "GTerm mirrors TermDev");

struct SectorRows {
    void *blob = nullptr;
    size_t bytes = 0;
    // the sector's dets in compact order, the rank tables and the groups
    // (kept for sigma without rows when the rows are over budget)
    void *tblob = nullptr;
    size_t tbytes = 0;
    const uint64_t *det = nullptr;
    const int32_t *arank = nullptr, *brank = nullptr;
    const SecGroup *groups = nullptr;
    int ngroups = 0;
    const int32_t *rowptr = nullptr;
    const uint32_t *col = nullptr;
    const double *vr = nullptr;    // real H ...
    const double2 *vc = nullptr;   // ... or complex
    int64_t nnz = 0;
    bool too_big = false;          // over kRowsBudget: no rows held
    // too_big: H as pair records, one or more per x-group (build_h_records)
    struct HRec {
        int2 span;       // words of the record in hrec
        int table;       // 1: (gn, hn) per pattern; 0: matrix elements from the terms
        int t0, t1, real;
        uint64_t x;
        int64_t pairs;
    };
    std::vector<HRec> hrecs;
    void *hblob = nullptr;
    const uint4 *d_hrec = nullptr;
    int diag_t0 = 0, diag_t1 = 0, diag_real = 1;  // the x = 0 group (t0 == t1: none)
    ~SectorRows() {
        dev_free(blob);
        dev_free(tblob);
        dev_free(hblob);
    }
};

// The device copies of a plan's record streams, uploaded once.
static int plan_upload(SectorPlan &sp) {
    if (sp.dev) return QFB_OK;
    auto d = std::make_shared<SectorPlanDev>();
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_fr = take(sizeof(uint4) * sp.fwd.rec.size());
    const size_t o_fs = take(sizeof(int2) * sp.fwd.span.size());
    const size_t o_fp = take(sizeof(int32_t) * sp.fwd.param.size());
    const size_t o_sr = take(sizeof(uint4) * sp.sweep.rec.size());
    const size_t o_ss = take(sizeof(int2) * sp.sweep.span.size());
    const size_t o_sp = take(sizeof(int32_t) * sp.sweep.param.size());
    int rc = dev_alloc(&d->blob, off);
    if (rc) return rc;
    d->bytes = off;
    char *base = (char *)d->blob;
    struct Up { size_t o; const void *p; size_t n; };
    const Up ups[] = {{o_fr, sp.fwd.rec.data(), sizeof(uint4) * sp.fwd.rec.size()},
                      {o_fs, sp.fwd.span.data(), sizeof(int2) * sp.fwd.span.size()},
                      {o_fp, sp.fwd.param.data(), sizeof(int32_t) * sp.fwd.param.size()},
                      {o_sr, sp.sweep.rec.data(), sizeof(uint4) * sp.sweep.rec.size()},
                      {o_ss, sp.sweep.span.data(), sizeof(int2) * sp.sweep.span.size()},
                      {o_sp, sp.sweep.param.data(), sizeof(int32_t) * sp.sweep.param.size()}};
    for (const Up &x : ups)
        if (x.n) QFB_CUDA(cudaMemcpyAsync(base + x.o, x.p, x.n, cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    d->frec = (const uint4 *)(base + o_fr);
    d->fspan = (const int2 *)(base + o_fs);
    d->fparam = (const int32_t *)(base + o_fp);
    d->srec = (const uint4 *)(base + o_sr);
    d->sspan = (const int2 *)(base + o_ss);
    d->sparam = (const int32_t *)(base + o_sp);
    sp.dev = d;
    return QFB_OK;
}

// H of `ham` on the plan's sector as pair records (sigma without stored
// rows): per x-group, the patterns of j0's bits (x's highest bit clear) at
// the group's pattern positions -- the bits where its z-masks differ and x's
// other bits -- that keep the alpha and beta counts, each with its alpha and
// beta lists.  Up to kHTableBits pattern bits the record holds each
// pattern's two matrix elements (gn = H[i1][i0], hn = H[i0][i1], divided by
// the sign of the first z-mask on j0); beyond that its patterns cover x's
// bits only and the kernel sums the terms per pair.  The x = 0 group is kept
// as a term range.
constexpr int kHTableBits = 7;
constexpr size_t kHRecEntries = 60000;  // SEntry offsets of a record are 16-bit

static int build_h_records(const qfb_sum_s *ham, const SectorPlan &sp,
                           const std::vector<SecGroup> &sg, int n, SectorRows &rows) {
    const uint64_t A = 0x5555555555555555ull;
    StreamHost S;
    for (const SecGroup &g : sg) {
        const TermDev *T = ham->h_terms.data() + g.begin;
        const int nt = g.end - g.begin;
        if (g.x == 0) {
            rows.diag_t0 = g.begin;
            rows.diag_t1 = g.end;
            rows.diag_real = g.real;
            continue;
        }
        const int h = highest_bit(g.x);
        const uint64_t hb = 1ull << h, zb = T[0].z;
        uint64_t D = 0;
        for (int t = 0; t < nt; ++t) D |= T[t].z ^ zb;
        const uint64_t PBt = (D | g.x) & ~hb;
        const bool table = __builtin_popcountll(PBt) <= kHTableBits;
        const uint64_t PB = table ? PBt : (g.x & ~hb);
        int pos[64], npb = 0;
        for (uint64_t m = PB; m; m &= m - 1) pos[npb++] = __builtin_ctzll(m);
        const int ka = __builtin_popcountll(g.x & A) / 2, kb = __builtin_popcountll(g.x & ~A) / 2;
        CStep cs;
        size_t nent = 0;
        int64_t pairs = 0;
        auto flush = [&]() -> int {
            if (cs.pats.empty()) return QFB_OK;
            if (!push_record(S, cs, 0, 0, 1 << 30))
                return fail(QFB_ENOSYS, "H record of an x-group too large");
            SectorRows::HRec r{};
            r.span = S.span.back();
            r.table = table ? 1 : 0;
            r.t0 = g.begin;
            r.t1 = g.end;
            r.real = g.real;
            r.x = g.x;
            r.pairs = pairs;
            rows.hrecs.push_back(r);
            cs.pats.clear();
            nent = 0;
            pairs = 0;
            return QFB_OK;
        };
        for (uint64_t pat = 0; pat < (1ull << npb); ++pat) {
            uint64_t jd = 0;
            for (int i = 0; i < npb; ++i)
                if (pat >> i & 1) jd |= 1ull << pos[i];
            if (__builtin_popcountll(jd & g.x & A) != ka || __builtin_popcountll(jd & g.x & ~A) != kb)
                continue;  // the pair would leave the sector
            CStep::Pat pt;
            if (table) {
                std::complex<double> gn = 0.0, hn = 0.0;
                for (int t = 0; t < nt; ++t) {
                    const std::complex<double> c(T[t].c.x, T[t].c.y);
                    const double sg0 = (__builtin_popcountll(jd & (T[t].z ^ zb)) & 1) ? -1.0 : 1.0;
                    const double sx = (__builtin_popcountll(g.x & T[t].z) & 1) ? -1.0 : 1.0;
                    gn += c * sg0;
                    hn += c * (sg0 * sx);
                }
                if (gn == 0.0 && hn == 0.0) continue;
                pt.gn = make_double2(gn.real(), gn.imag());
                pt.hn = make_double2(hn.real(), hn.imag());
            } else {
                pt.gn = pt.hn = make_double2(0.0, 0.0);
            }
            const uint64_t zl = table ? zb : 0;
            if (!sector_list(sp, 0, n, PB | hb, jd, g.x, zl, pt.a) ||
                !sector_list(sp, 1, n, PB | hb, jd, g.x, zl, pt.b))
                return fail(QFB_EDEVICE, "H record: a pair leaves the sector");
            if (pt.a.empty() || pt.b.empty()) continue;
            if (nent + pt.a.size() + pt.b.size() > kHRecEntries || cs.pats.size() >= 255) {
                const int rc = flush();
                if (rc) return rc;
            }
            nent += pt.a.size() + pt.b.size();
            pairs += (int64_t)pt.a.size() * (int64_t)pt.b.size();
            cs.pats.push_back(std::move(pt));
        }
        const int rc = flush();
        if (rc) return rc;
    }
    if (!S.rec.empty()) {
        const int rc = dev_alloc(&rows.hblob, sizeof(uint4) * S.rec.size());
        if (rc) return rc;
        QFB_CUDA(cudaMemcpyAsync(rows.hblob, S.rec.data(), sizeof(uint4) * S.rec.size(),
                                 cudaMemcpyHostToDevice, t_stream));
        rows.d_hrec = (const uint4 *)rows.hblob;
        rows.tbytes += sizeof(uint4) * S.rec.size();
    }
    return QFB_OK;
}

// H rows of `ham` on the plan's sector (compact order), built on the device
// once per (qubits, electrons, layout) and cached on the Hamiltonian.  With
// `global`, rows over kRowsBudget are refused (QFB_ENOMEM) and the refusal
// is cached too; `interleave` orders each row's entries for k_sector_h.
static int get_sector_rows(qfb_sum_s *ham, const SectorPlan &sp, const std::vector<SecGroup> &sg,
                           int n, int interleave, bool global, std::shared_ptr<SectorRows> *out) {
    // interleave: 0 none, else the bank slots of one gather group (8 or 16)
    const int layout = interleave == 8 ? 1 : interleave == 16 ? 3 : (global && g_ucc_compact == 3) ? 2 : 0;
    const auto key = std::make_tuple(n, sp.ka, sp.kb, layout);
    auto it = ham->rows_cache.find(key);
    if (it != ham->rows_cache.end()) {
        if (!global && it->second->too_big)
            return fail(QFB_ENOMEM, "sector H rows exceed their budget");
        *out = it->second;
        return QFB_OK;
    }
    const int nsec = sp.nsec;
    bool real = true;
    for (const SecGroup &g : sg) real = real && g.real;
    const double entry_bytes = real ? 12.0 : 20.0;
    auto rows = std::make_shared<SectorRows>();
    // persistent tables: dets in compact order, ranks, groups, row counts
    std::vector<uint64_t> det((size_t)nsec);
    for (int ra = 0; ra < sp.nalpha; ++ra)
        for (int rb = 0; rb < sp.nbeta; ++rb) det[(size_t)ra * sp.nbeta + rb] = sp.adet[ra] | sp.bdet[rb];
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_det = take(sizeof(uint64_t) * det.size());
    const size_t o_ar = take(sizeof(int32_t) * sp.arank.size());
    const size_t o_br = take(sizeof(int32_t) * sp.brank.size());
    const size_t o_g = take(sizeof(SecGroup) * sg.size());
    const size_t o_cnt = take(sizeof(int32_t) * (size_t)(nsec + 1));
    int rc = dev_alloc(&rows->tblob, off);
    if (rc) return rc;
    rows->tbytes = off;
    char *base = (char *)rows->tblob;
    QFB_CUDA(cudaMemcpyAsync(base + o_det, det.data(), sizeof(uint64_t) * det.size(),
                             cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaMemcpyAsync(base + o_ar, sp.arank.data(), sizeof(int32_t) * sp.arank.size(),
                             cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaMemcpyAsync(base + o_br, sp.brank.data(), sizeof(int32_t) * sp.brank.size(),
                             cudaMemcpyHostToDevice, t_stream));
    if (!sg.empty())
        QFB_CUDA(cudaMemcpyAsync(base + o_g, sg.data(), sizeof(SecGroup) * sg.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    int32_t *d_cnt = (int32_t *)(base + o_cnt);
    rows->det = (const uint64_t *)(base + o_det);
    rows->arank = (const int32_t *)(base + o_ar);
    rows->brank = (const int32_t *)(base + o_br);
    rows->groups = (const SecGroup *)(base + o_g);
    rows->ngroups = (int)sg.size();
    auto over_budget = [&]() -> int {  // rows kept without entries: sigma from the groups
        rows->too_big = true;
        if (global) {
            const int hrc = build_h_records(ham, sp, sg, n, *rows);
            if (hrc) return hrc;
        }
        QFB_CUDA(cudaStreamSynchronize(t_stream));
        ham->rows_cache[key] = rows;
        if (!global) return fail(QFB_ENOMEM, "sector H rows exceed their budget");
        *out = rows;
        return QFB_OK;
    };
    if (global && g_ucc_compact == 3) return over_budget();  // rows switched off
    {   // estimate from the reference row before counting every row
        const uint64_t A = 0x5555555555555555ull;
        const uint64_t k = sp.adet[sp.ref_i / sp.nbeta] | sp.bdet[sp.ref_i % sp.nbeta];
        int64_t c = 0;
        for (const SecGroup &g : sg) {
            const uint64_t kx = k & g.x;
            if ((__builtin_popcountll(kx & A) | __builtin_popcountll(kx & ~A) << 8) == g.halves) ++c;
        }
        if ((double)c * nsec * entry_bytes > 1.5 * kRowsBudget) return over_budget();
    }
    const unsigned nb = (unsigned)((nsec + 127) / 128);
    k_sector_rows<<<nb, 128, 0, t_stream>>>(rows->det, nsec, rows->groups, (int)sg.size(),
                                            ham->d_terms, ham->d_rterms, rows->arank, rows->brank,
                                            sp.nbeta, n, nullptr, d_cnt, nullptr, nullptr, nullptr);
    QFB_LAUNCHED();
    std::vector<int32_t> cnt((size_t)nsec);
    QFB_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int32_t) * nsec, cudaMemcpyDeviceToHost,
                             t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    std::vector<int32_t> rowptr((size_t)nsec + 1, 0);
    int64_t nnz = 0;
    for (int i = 0; i < nsec; ++i) {
        rowptr[i] = (int32_t)nnz;
        nnz += cnt[i];
        if (nnz >= ((int64_t)1 << 31)) return over_budget();
    }
    rowptr[nsec] = (int32_t)nnz;
    if ((double)nnz * entry_bytes > kRowsBudget) return over_budget();
    size_t coff = ((sizeof(int32_t) * (nsec + 1)) + 255) & ~(size_t)255;
    const size_t o_col = coff;
    coff += ((sizeof(uint32_t) * std::max<int64_t>(nnz, 1)) + 255) & ~(size_t)255;
    const size_t o_val = coff;
    coff += (real ? sizeof(double) : sizeof(double2)) * std::max<int64_t>(nnz, 1);
    rc = dev_alloc(&rows->blob, coff);
    if (rc) return rc;
    rows->bytes = coff;
    rows->nnz = nnz;
    char *cb = (char *)rows->blob;
    QFB_CUDA(cudaMemcpyAsync(cb, rowptr.data(), sizeof(int32_t) * (nsec + 1), cudaMemcpyHostToDevice,
                             t_stream));
    int32_t *d_rp = (int32_t *)cb;
    uint32_t *d_col = (uint32_t *)(cb + o_col);
    double *d_vr = real ? (double *)(cb + o_val) : nullptr;
    double2 *d_vc = real ? nullptr : (double2 *)(cb + o_val);
    k_sector_rows<<<nb, 128, 0, t_stream>>>(rows->det, nsec, rows->groups, (int)sg.size(),
                                            ham->d_terms, ham->d_rterms, rows->arank, rows->brank,
                                            sp.nbeta, n, d_rp, nullptr, d_col, d_vr, d_vc);
    QFB_LAUNCHED();
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    if (interleave) {
        rc = sector_rows_interleave(rowptr, nnz, d_col, real ? (void *)d_vr : (void *)d_vc,
                                    real ? sizeof(double) : sizeof(double2), interleave);
        if (rc) return rc;
    }
    rows->rowptr = d_rp;
    rows->col = d_col;
    rows->vr = d_vr;
    rows->vc = d_vc;
    ham->rows_cache[key] = rows;
    *out = rows;
    return QFB_OK;
}

// The shape of k_sector_h for an evaluator: P parameter sets per CTA (as
// many as shared memory holds, up to 4 real or 2 complex: each H row entry
// loaded serves P gathers), the block size (1024 threads for the shapes whose
// shared memory leaves one CTA per SM) and the row slices Q per group that minimise the estimated makespan
// ceil(G Q / slots) (1 / Q + c) over G = ceil(B / P) groups, c being a CTA's
// fixed cost (loading the group's psi) relative to a whole group's rows.
static void sector_h_shape(qfb_ucc u, int nsec) {
    const size_t elem = u->sreal ? sizeof(double) : sizeof(double2);
    const int B = u->nbatch;
    int P = u->sreal ? 4 : 2;
    while (P > 1 && ((size_t)P * nsec * elem > kSectorSmemMax || P > B)) P >>= 1;
    const size_t smem = qfbs::sector_smem_states((size_t)P, (size_t)nsec, u->sreal);
    // 1024 threads for the shapes that hold one CTA per SM (launched so)
    const int NT = (P == 4 || (P == 2 && !u->sreal)) ? 1024 : kSectorThreads;
    const int cps = std::max(1, std::min(2048 / NT, (int)((227 * 1024) / (smem + 1024))));
    const int slots = sm_count() * cps, G = (B + P - 1) / P;
    const int qmax = std::max(1, std::min(kSectorHSlicesMax, nsec / 64));
    int best = 1;
    double bcost = 1e300;
    for (int Q = 1; Q <= qmax; ++Q) {
        const double waves = std::ceil((double)G * Q / slots);
        const double cost = waves * (1.0 / Q + 0.01);
        if (cost < bcost - 1e-12) {
            bcost = cost;
            best = Q;
        }
    }
    u->h_sets = P;
    u->h_threads = NT;
    u->h_slices = best;
}

// Attach a compact plan and its H rows to an evaluator (shared memory or,
// with `global`, global memory states).
static int sector_attach(qfb_ucc u, qfb_sum_s *ham, const std::shared_ptr<SectorPlan> &plan,
                         const std::vector<SecGroup> &sg, bool global) {
    SectorPlan &sp = *plan;
    int rc = plan_upload(sp);
    if (rc) return rc;
    std::shared_ptr<SectorRows> rows;
    const bool real_steps = !ucc_complex_states() && stream_is_real(sp.fwd) && stream_is_real(sp.sweep);
    bool h_real = true;
    for (const SecGroup &g : sg) h_real = h_real && g.real;
    int interleave = 0;
    if (!global) {
        // real states: real H rows and real pair coefficients in both streams
        u->sreal = (real_steps && h_real) ? 1 : 0;
        sector_h_shape(u, sp.nsec);
        // the H kernel gathers 16-byte words (complex amplitudes, or two real
        // sets at once) by quarter warps: 8 bank slots; single real sets 16
        interleave = (u->sreal && u->h_sets == 1) ? 16 : 8;
    }
    rc = get_sector_rows(ham, sp, sg, u->nqubit, interleave, global, &rows);
    if (rc) return rc;
    std::shared_ptr<PairPlanDev> pairs;
    if (!global) {
        if (u->sreal != ((real_steps && rows->vc == nullptr) ? 1 : 0))
            return fail(QFB_EINVAL, "compact sector: H rows' type differs from their groups'");
        rc = pair_plan(sp, u->sreal ? 16 : 8, &pairs);
        if (rc) return rc;
        u->pairs = pairs;
        u->bytes += pairs->bytes;
        // two real sets per CTA in the forward program where its shared memory fits
        const size_t fwd_b = ((16 * (size_t)sp.nsec + 15) & ~(size_t)15) +
                             sizeof(qfbs::PSmemPR) * (size_t)pairs->fwd.n;
        if (u->sreal && g_ucc_compact != 6 && u->nbatch >= 2 && fwd_b <= kSectorSmemMax) {
            rc = pair_plan(sp, 8, &u->pairs16b);
            if (rc) return rc;
            if (u->pairs16b != pairs) u->bytes += u->pairs16b->bytes;
            u->paired = 1;
        }
    }
    u->splan = plan;
    u->rows = rows;
    u->nnz = rows->nnz;
    u->bytes += sp.dev->bytes + rows->bytes + rows->tbytes;
    const SectorPlanDev &d = *sp.dev;
    if (global && rows->too_big) {
        // sigma copies and streams of the concurrent x-group chains
        const size_t sb = (u->greal ? sizeof(double) : sizeof(double2)) * (size_t)sp.nsec * u->nbatch;
        rc = dev_alloc(&u->hblob, sb * (kHChains - 1));
        if (rc) return rc;
        u->bytes += sb * (kHChains - 1);
        cudaError_t e = cudaEventCreateWithFlags(&u->hfork, cudaEventDisableTiming);
        for (int k = 0; k < kHChains - 1 && e == cudaSuccess; ++k) {
            e = cudaStreamCreateWithFlags(&u->hside[k], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&u->hjoin[k], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) return cuda_fail(e, "sector H chains");
    }
    if (global) {
        u->g_frec = d.frec;
        u->g_srec = d.srec;
        u->g_rowptr = rows->rowptr;
        u->g_col = rows->col;
        u->g_vr = rows->vr;
        u->g_vc = rows->vc;
        return QFB_OK;
    }
    qfbs::SLaunch &L = u->SL;
    L.nsec = sp.nsec;
    L.nbeta = sp.nbeta;
    L.ref_i = sp.ref_i;
    L.nparam = u->nparam;
    L.fwd = pairs->fwd;
    L.sweep = pairs->sweep;
    L.rowptr = rows->rowptr;
    L.col = rows->col;
    L.val_r = rows->vr;
    L.val_c = rows->vc;
    L.params = u->params;
    L.energy = u->energy;
    L.partial = u->gpart;
    if (u->paired) {
        u->SLp = L;
        u->SLp.fwd = u->pairs16b->fwd;
    }
    return QFB_OK;
}

template <class V>
static cudaError_t sector_smem_attr_v() {
    const int m = (int)kSectorSmemMax;
    cudaError_t err = cudaFuncSetAttribute(qfbs::k_sector_forward<V>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    auto attr = [&](const void *f) {
        if (err == cudaSuccess) err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    };
    if constexpr (sizeof(V) == sizeof(double)) {
        attr((const void *)qfbs::k_sector_h<true, V, 4, 1024>);
        attr((const void *)qfbs::k_sector_h<true, V, 2, 512>);
        attr((const void *)qfbs::k_sector_h<true, V, 1, 512>);
    } else {
        attr((const void *)qfbs::k_sector_h<true, V, 2, 1024>);
        attr((const void *)qfbs::k_sector_h<true, V, 1, 512>);
        attr((const void *)qfbs::k_sector_h<false, V, 2, 1024>);
        attr((const void *)qfbs::k_sector_h<false, V, 1, 512>);
    }
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(qfbs::k_sector_sweep<V>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(qfbs::k_sector_resid<V>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(qfbs::k_sector_pool<V>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(qfbs::k_sector_pack<V>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    if constexpr (sizeof(V) == sizeof(double)) {
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(qfbs::k_sector_forward_pr,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, m);
    }
    return err;
}

static int sector_smem_attr() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        err = sector_smem_attr_v<double2>();
        if (err == cudaSuccess) err = sector_smem_attr_v<double>();
    });
    return err == cudaSuccess ? QFB_OK : cuda_fail(err, "sector evaluator shared memory");
}

template <class V>
static int ucc_stage_compact_v(qfb_ucc u, int stage, int with_grad) {
    const qfbs::SLaunch &L = u->SL;
    const size_t n = (size_t)L.nsec;
    const bool real = sizeof(V) == sizeof(double);
    switch (stage) {
        case 1:
            if constexpr (sizeof(V) == sizeof(double)) {
                if (u->paired) {
                    const qfbs::SLaunch &LP = u->SLp;
                    qfbs::k_sector_forward_pr<<<(u->nbatch + 1) / 2, qfbs::kStepThreads,
                                                ((16 * n + 15) & ~(size_t)15) +
                                                    sizeof(qfbs::PSmemPR) * (size_t)LP.fwd.n,
                                                t_stream>>>(LP, u->nbatch);
                    QFB_LAUNCHED();
                    break;
                }
            }
            qfbs::k_sector_forward<V><<<u->nbatch, qfbs::kStepThreads,
                                        qfbs::sector_smem_states(1, n, real) +
                                            sizeof(qfbs::PSmem<V>) * (size_t)L.fwd.n,
                                        t_stream>>>(L);
            QFB_LAUNCHED();
            break;
        case 2: {
            const int P = u->h_sets, Q = u->h_slices, B = u->nbatch;
            const unsigned grid = (unsigned)(((B + P - 1) / P) * Q);
            const size_t smem = qfbs::sector_smem_states((size_t)P, n, real);
#define QFB_SECTOR_H(RE, PP, NT)                                                              \
    qfbs::k_sector_h<RE, V, PP, NT><<<grid, NT, smem, t_stream>>>(L, B, Q, u->h_epart, u->h_count)
            if constexpr (sizeof(V) == sizeof(double)) {
                if (P == 4) QFB_SECTOR_H(true, 4, 1024);
                else if (P == 2) QFB_SECTOR_H(true, 2, 512);
                else QFB_SECTOR_H(true, 1, 512);
            } else if (L.val_c) {
                if (P == 2) QFB_SECTOR_H(false, 2, 1024);
                else QFB_SECTOR_H(false, 1, 512);
            } else {
                if (P == 2) QFB_SECTOR_H(true, 2, 1024);
                else QFB_SECTOR_H(true, 1, 512);
            }
#undef QFB_SECTOR_H
            QFB_LAUNCHED();
            break;
        }
        case 3:
            if (!(with_grad && u->grad && u->nparam > 0)) break;
            qfbs::k_sector_sweep<V><<<u->nbatch, qfbs::kSweepThreads,
                                      qfbs::sector_smem_states(2, n, real) +
                                          sizeof(qfbs::PSmem<V>) * (size_t)L.sweep.n,
                                      t_stream>>>(L);
            QFB_LAUNCHED();
            {
                const int64_t n = (int64_t)u->nparam * u->nbatch;
                k_grad_final_few<<<(unsigned)((n + 255) / 256), 256, 0, t_stream>>>(
                    u->gpart, u->psteps, (int)u->gchunks, u->nparam, u->nbatch, u->gradv);
            }
            QFB_LAUNCHED();
            break;
        default:
            break;
    }
    return QFB_OK;
}

// Compact evaluator: stage 1 the forward program, stage 2 sigma = H psi and
// the energy, stage 3 the reverse sweep (psi and sigma pass through the save
// buffer between them); real states when every coefficient is real.
static int ucc_stage_compact(qfb_ucc u, int stage, int with_grad) {
    return u->sreal ? ucc_stage_compact_v<double>(u, stage, with_grad)
                    : ucc_stage_compact_v<double2>(u, stage, with_grad);
}

// Pairs of the largest record of a stream (grid sizing of the global path).
static int64_t stream_max_pairs(const StreamHost &S) {
    int64_t most = 1;
    for (const int2 &sp : S.span) {
        const char *rec = (const char *)&S.rec[sp.x];
        qfbs::RHead hd;
        std::memcpy(&hd, rec, sizeof(hd));
        int64_t pairs = 0;
        for (int p = 0; p < (hd.npf & 255); ++p) {
            qfbs::RPat pt;
            std::memcpy(&pt, rec + sizeof(qfbs::RHead) + p * sizeof(qfbs::RPat), sizeof(pt));
            pairs += (int64_t)pt.na * pt.nb;
        }
        most = std::max(most, pairs);
    }
    return most;
}

static unsigned global_grid(int64_t pairs, int spw) {
    const int64_t per_block = 8 * (32 / spw);  // pairs one block covers per sweep of its warps
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(2048, (pairs + 2 * per_block - 1) /
                                                                     (2 * per_block)));
}

// Launch with programmatic stream serialization (the kernel opens with
// g_pdl_enter): chains of short dependent launches overlap each launch's
// latency with the previous grid's run.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// Compact sector in global memory: stage 0 the reference, 1 the forward
// records, 2 sigma = H psi and the energy, 3 the sweep records.
template <class V>
static int ucc_stage_global_v(qfb_ucc u, int stage, int with_grad) {
    const qfbg::GLaunch &L = u->GL;
    const SectorPlan &sp = *u->splan;
    const dim3 grid(u->g_sgrid, u->g_ygrid);
    switch (stage) {
        case 0:
            QFB_CUDA(cudaMemsetAsync(L.psi, 0, sizeof(V) * (size_t)L.nsec * L.B, t_stream));
            qfbg::k_cg_ref<V><<<(L.B + 127) / 128, 128, 0, t_stream>>>(L, sp.ref_i);
            QFB_LAUNCHED();
            break;
        case 1:
            for (size_t r = 0; r < sp.fwd.span.size(); ++r) {
                QFB_CUDA(launch_pdl(qfbg::k_cg_step<true, false, false, V>, grid, dim3(256), t_stream, L,
                                    u->g_frec + sp.fwd.span[r].x, sp.fwd.param[r], 1, -1,
                                    (double2 *)nullptr));
                QFB_LAUNCHED();
            }
            break;
        case 2: {
            const dim3 hg(u->g_hgrid, u->g_ygrid);
            if (u->rows->too_big) {
                const SectorRows &R = *u->rows;
                const qfbg::GTerm *gt = (const qfbg::GTerm *)u->ham->d_terms;
                const size_t ns = (size_t)L.nsec * L.B;
                if (R.diag_t1 > R.diag_t0) {
                    qfbg::k_cg_h_diag<V><<<u->g_hgrid, 256, 0, t_stream>>>(
                        L, R.det, gt, u->ham->d_rterms, R.diag_t0, R.diag_t1, R.diag_real);
                    QFB_LAUNCHED();
                } else {
                    QFB_CUDA(cudaMemsetAsync(L.sig, 0, sizeof(V) * ns, t_stream));
                }
                // chain k takes groups k, k + kHChains, ... into its own sigma
                // copy (no two launches in flight touch one copy); the copies
                // are added into sigma in chain order afterwards
                V *extra = reinterpret_cast<V *>(u->hblob);
                QFB_CUDA(cudaMemsetAsync(extra, 0, sizeof(V) * ns * (kHChains - 1), t_stream));
                QFB_CUDA(cudaEventRecord(u->hfork, t_stream));
                qfbg::GLaunch Lk[kHChains];
                cudaStream_t sk[kHChains];
                for (int k = 0; k < kHChains; ++k) {
                    Lk[k] = L;
                    if (k > 0) {
                        Lk[k].sig = extra + ns * (k - 1);
                        QFB_CUDA(cudaStreamWaitEvent(u->hside[k - 1], u->hfork, 0));
                    }
                    sk[k] = k ? u->hside[k - 1] : t_stream;
                }
                for (size_t i = 0; i < R.hrecs.size(); ++i) {
                    const auto &r = R.hrecs[i];
                    const int k = (int)(i % kHChains);
                    const dim3 rg(global_grid(r.pairs, L.spw), u->g_ygrid);
                    const uint4 *rec = R.d_hrec + r.span.x;
                    if (r.table)
                        QFB_CUDA(launch_pdl(qfbg::k_cg_h_group<true, V>, rg, dim3(256), sk[k], Lk[k], rec,
                                            R.det, gt, u->ham->d_rterms, r.t0, r.t1, r.real, r.x));
                    else
                        QFB_CUDA(launch_pdl(qfbg::k_cg_h_group<false, V>, rg, dim3(256), sk[k], Lk[k], rec,
                                            R.det, gt, u->ham->d_rterms, r.t0, r.t1, r.real, r.x));
                    QFB_LAUNCHED();
                }
                for (int k = 1; k < kHChains; ++k) {
                    QFB_CUDA(cudaEventRecord(u->hjoin[k - 1], u->hside[k - 1]));
                    QFB_CUDA(cudaStreamWaitEvent(t_stream, u->hjoin[k - 1], 0));
                }
                qfbg::k_cg_add_copies<V><<<(unsigned)std::min<size_t>((ns + 255) / 256, 8192), 256, 0,
                                           t_stream>>>(reinterpret_cast<V *>(L.sig), extra, ns,
                                                       kHChains - 1);
                QFB_LAUNCHED();
                qfbg::k_cg_dot<V><<<hg, 256, 0, t_stream>>>(L, u->g_epart);
            }
            else if (u->g_vc) {
                if constexpr (sizeof(V) == sizeof(double2))
                    qfbg::k_cg_h_rows<false, V><<<hg, 256, 0, t_stream>>>(L, u->g_rowptr, u->g_col,
                                                                         nullptr, u->g_vc, u->g_epart);
            } else {
                qfbg::k_cg_h_rows<true, V><<<hg, 256, 0, t_stream>>>(L, u->g_rowptr, u->g_col, u->g_vr,
                                                                    nullptr, u->g_epart);
            }
            QFB_LAUNCHED();
            qfbg::k_cg_energy<<<(L.B + 7) / 8, 256, 0, t_stream>>>(u->g_epart, (int)u->g_hgrid, L.B,
                                                                  u->energy);
            QFB_LAUNCHED();
            break;
        }
        default: {
            if (!(with_grad && u->grad && u->nparam > 0)) break;
            for (size_t r = 0; r < sp.sweep.span.size(); ++r) {
                qfbs::RHead hd;
                std::memcpy(&hd, &sp.sweep.rec[sp.sweep.span[r].x], sizeof(hd));
                const int fl = hd.npf >> 8;
                const uint4 *rec = u->g_srec + sp.sweep.span[r].x;
                const int par = sp.sweep.param[r];
                if (fl == (qfbs::R_ROT | qfbs::R_IP | qfbs::R_TWO))
                    QFB_CUDA(launch_pdl(qfbg::k_cg_step<true, true, true, V>, grid, dim3(256), t_stream, L,
                                        rec, par, -1, (int)hd.row, u->gpart));
                else if (fl == qfbs::R_IP)
                    QFB_CUDA(launch_pdl(qfbg::k_cg_step<false, true, false, V>, grid, dim3(256), t_stream,
                                        L, rec, par, -1, (int)hd.row, u->gpart));
                else
                    QFB_CUDA(launch_pdl(qfbg::k_cg_step<true, false, true, V>, grid, dim3(256), t_stream, L,
                                        rec, par, -1, -1, (double2 *)nullptr));
                QFB_LAUNCHED();
            }
            k_grad_final<<<dim3(u->nparam, L.B), 128, 0, t_stream>>>(u->gpart, u->psteps, u->gchunks,
                                                                   u->gradv);
            QFB_LAUNCHED();
            break;
        }
    }
    return QFB_OK;
}

// Compact sector in global memory, real or complex state storage.
static int ucc_stage_global(qfb_ucc u, int stage, int with_grad) {
    return u->greal ? ucc_stage_global_v<double>(u, stage, with_grad)
                    : ucc_stage_global_v<double2>(u, stage, with_grad);
}

static int ucc_stage(qfb_ucc u, int stage, int with_grad) {
    if (u->compact) return ucc_stage_compact(u, stage, with_grad);
    if (u->gsec) return ucc_stage_global(u, stage, with_grad);
    const int B = u->nbatch;
    int rc = QFB_OK;
    switch (stage) {
        case 0:
            QFB_CUDA(cudaMemsetAsync(u->psi, 0, sizeof(double2) * u->nbasis * B, t_stream));
            k_set_ref<<<(B + 127) / 128, 128, 0, t_stream>>>(u->psi, u->nbasis, u->ref, B);
            QFB_LAUNCHED();
            break;
        case 1:
            rc = enqueue_prog(u->fwd, u->psi, u->nqubit, B, u->params, 0, 1);
            break;
        case 2:
            if (u->nsec > 0) {
                QFB_CUDA(cudaMemsetAsync(u->sig, 0, sizeof(double2) * u->nbasis * B, t_stream));
                if (u->nqubit <= 32)
                    launch_sector_apply(u->sig, u->psi, u->nbasis, B, (const uint32_t *)u->sec,
                                        u->nsec, u->sgroups, u->nsgroups, u->ham->d_terms,
                                        u->ham->d_rterms);
                else
                    launch_sector_apply(u->sig, u->psi, u->nbasis, B, (const uint64_t *)u->sec,
                                        u->nsec, u->sgroups, u->nsgroups, u->ham->d_terms,
                                        u->ham->d_rterms);
                QFB_LAUNCHED();
            } else {
                rc = enqueue_sum_apply(u->ham, u->sig, u->psi, u->nbasis, B);
            }
            if (rc) return rc;
            k_vdot_rows<<<dim3(u->vchunks, B), 256, 0, t_stream>>>(u->psi, u->sig, u->nbasis,
                                                                 u->vpart);
            QFB_LAUNCHED();
            k_energy_final<<<B, 128, 0, t_stream>>>(u->vpart, u->vchunks, u->energy);
            QFB_LAUNCHED();
            break;
        default:
            if (with_grad && u->grad && u->nparam > 0) {
                rc = enqueue_gradient(u->grad, u->unrot, u->psi, u->sig, u->nqubit, B,
                                      u->params, 0, u->gpart);
                if (rc) return rc;
                k_grad_final<<<dim3(u->nparam, B), 128, 0, t_stream>>>(u->gpart, u->psteps,
                                                                     u->gchunks, u->gradv);
                QFB_LAUNCHED();
            }
            break;
    }
    return rc;
}

// Stage 4: the pool's inner products on psi and sigma (qfb_ucc_set_pool).
static int ucc_pool_stage(qfb_ucc u) {
    if (!u->pool) return fail(QFB_EINVAL, "qfb_ucc_run: no pool set (qfb_ucc_set_pool)");
    const int B = u->nbatch;
    unsigned chunks = u->pchunks;
    if (u->gsec) {
        const dim3 grid(u->pchunks, u->g_ygrid, (unsigned)u->pstream.n);
        if (u->greal)
            qfbg::k_cg_ip_many<double><<<grid, 256, 0, t_stream>>>(u->GL, u->pstream.rec,
                                                                   u->pstream.span, u->ppart);
        else
            qfbg::k_cg_ip_many<double2><<<grid, 256, 0, t_stream>>>(u->GL, u->pstream.rec,
                                                                    u->pstream.span, u->ppart);
        QFB_LAUNCHED();
    } else if (u->compact) {
        qfbs::SLaunch L = u->SL;
        L.partial = u->ppart;
        const int sm = sm_count();
        const int G = std::max(1, std::min(u->ppairs.n, (2 * sm + B - 1) / B));
        const size_t smem = qfbs::sector_smem_states(2, (size_t)L.nsec, u->sreal);
        if (u->sreal)
            qfbs::k_sector_pool<double><<<dim3(G, B), kSectorThreads, smem, t_stream>>>(L, u->ppairs);
        else
            qfbs::k_sector_pool<double2><<<dim3(G, B), kSectorThreads, smem, t_stream>>>(L, u->ppairs);
        QFB_LAUNCHED();
        chunks = kSectorThreads / 32;
    } else {
        const dim3 grid(u->pchunks, (unsigned)u->pool->h_steps.size(), B);
        k_pool_ip<<<grid, 256, 0, t_stream>>>(u->psi, u->sig, u->nbasis, u->pool_steps,
                                              u->pool->d_tab, u->ppart);
        QFB_LAUNCHED();
    }
    if (chunks <= 32)
        k_grad_final_few<<<(unsigned)(((int64_t)u->npool * B + 255) / 256), 256, 0, t_stream>>>(
            u->ppart, u->pranges, (int)chunks, u->npool, B, u->pgrad);
    else
        k_grad_final<<<dim3(u->npool, B), 128, 0, t_stream>>>(u->ppart, u->pranges, chunks, u->pgrad);
    QFB_LAUNCHED();
    return QFB_OK;
}

// Residual stage (qfb_ucc_set_residuals): U^dagger on sigma, then the
// residual entries.  Sigma is consumed.
static int ucc_resid_stage(qfb_ucc u) {
    if (!u->rblob) return fail(QFB_EINVAL, "qfb_ucc_run: no residuals set (qfb_ucc_set_residuals)");
    const int B = u->nbatch;
    const unsigned gg = (unsigned)(((int64_t)u->nres * B + 255) / 256);
    if (u->compact) {
        const qfbs::SLaunch &L = u->SL;
        const size_t smem = qfbs::sector_smem_states(1, (size_t)L.nsec, u->sreal) +
                            (u->sreal ? sizeof(qfbs::PSmem<double>) : sizeof(qfbs::PSmem<double2>)) *
                                (size_t)u->rstream.n;
        if (u->sreal)
            qfbs::k_sector_resid<double><<<B, qfbs::kStepThreads, smem, t_stream>>>(
                L, u->rstream, u->ridx, u->rphase, u->nres, u->res);
        else
            qfbs::k_sector_resid<double2><<<B, qfbs::kStepThreads, smem, t_stream>>>(
                L, u->rstream, u->ridx, u->rphase, u->nres, u->res);
        QFB_LAUNCHED();
        return QFB_OK;
    }
    if (u->gsec) {
        qfbg::GLaunch Ls = u->GL;  // rotate sigma: the step kernel rotates L.psi
        Ls.psi = u->GL.sig;
        const SectorPlan &sp = *u->splan;
        const dim3 grid(u->g_sgrid, u->g_ygrid);
        for (size_t r = sp.fwd.span.size(); r-- > 0;) {
            if (u->greal)
                qfbg::k_cg_step<true, false, false, double><<<grid, 256, 0, t_stream>>>(
                    Ls, u->g_frec + sp.fwd.span[r].x, sp.fwd.param[r], -1, -1, nullptr);
            else
                qfbg::k_cg_step<true, false, false, double2><<<grid, 256, 0, t_stream>>>(
                    Ls, u->g_frec + sp.fwd.span[r].x, sp.fwd.param[r], -1, -1, nullptr);
            QFB_LAUNCHED();
        }
        if (u->greal)
            k_resid_gather<double><<<gg, 256, 0, t_stream>>>((const double *)u->GL.sig, u->ridx,
                                                             (uint64_t)B, 1, u->rphase, u->nres, B,
                                                             u->res);
        else
            k_resid_gather<double2><<<gg, 256, 0, t_stream>>>((const double2 *)u->GL.sig, u->ridx,
                                                              (uint64_t)B, 1, u->rphase, u->nres, B,
                                                              u->res);
        QFB_LAUNCHED();
        return QFB_OK;
    }
    int rc = enqueue_prog(u->fwd, u->sig, u->nqubit, B, u->params, 0, -1);
    if (rc) return rc;
    k_resid_gather<double2><<<gg, 256, 0, t_stream>>>(u->sig, u->ridx, 1, u->nbasis, u->rphase,
                                                      u->nres, B, u->res);
    QFB_LAUNCHED();
    return QFB_OK;
}

// mode 0: energy (stages 0-2); 1: energy and gradient (0-3); 2: the gradient
// sweep alone (stage 3) on psi and sigma as a mode-0 run left them; 3: energy
// and the pool's gradients (stages 0-2, then the pool stage); 4: energy and
// the PQE residuals (stages 0-2, then the residual stage).
static int ucc_enqueue(qfb_ucc u, int mode) {
    const int last = (mode == 3 || mode == 4) ? 2 : 3;
    for (int st = (mode == 2 ? 3 : 0); st <= last; ++st) {
        int rc = ucc_stage(u, st, mode == 1 || mode == 2);
        if (rc) return rc;
    }
    if (mode == 3) return ucc_pool_stage(u);
    if (mode == 4) return ucc_resid_stage(u);
    return QFB_OK;
}

extern "C" {

static int ucc_create_impl(qfb_prog fprog, qfb_prog gprog, qfb_prog uprog, qfb_sum ham,
                           int nqubit, uint64_t ref_index, int nbatch, qfb_ucc *out,
                           bool allow_sector);

int qfb_ucc_create(qfb_prog fprog, qfb_prog gprog, qfb_prog uprog, qfb_sum ham, int nqubit,
                   uint64_t ref_index, int nbatch, qfb_ucc *out) {
    // plans, window plans and sector rows are cached on the shared program and
    // Hamiltonian objects: one creation at a time
    static std::mutex create_mu;
    std::lock_guard<std::mutex> lk(create_mu);
    int rc = ucc_create_impl(fprog, gprog, uprog, ham, nqubit, ref_index, nbatch, out, true);
    if (rc == QFB_ENOMEM && out && !*out)  // no room for the sector's tables: full space
        rc = ucc_create_impl(fprog, gprog, uprog, ham, nqubit, ref_index, nbatch, out, false);
    return rc;
}

static int ucc_create_impl(qfb_prog fprog, qfb_prog gprog, qfb_prog uprog, qfb_sum ham,
                           int nqubit, uint64_t ref_index, int nbatch, qfb_ucc *out,
                           bool allow_sector) {
    if (!out) return fail(QFB_EINVAL, "qfb_ucc_create: null output");
    *out = nullptr;
    if (!fprog || !ham) return fail(QFB_EINVAL, "qfb_ucc_create: null program or Hamiltonian");
    if (nqubit < 1 || nqubit > 40 || nbatch < 1)
        return fail(QFB_EINVAL, "qfb_ucc_create: nqubit = %d, nbatch = %d", nqubit, nbatch);
    if (ref_index >> nqubit) return fail(QFB_EINVAL, "qfb_ucc_create: reference index too large");
    if ((gprog == nullptr) != (uprog == nullptr))
        return fail(QFB_EINVAL, "qfb_ucc_create: give both gradient programs or neither");
    if (gprog && (gprog->nparam != fprog->nparam || !gprog->params_contiguous ||
                  uprog->nparam != fprog->nparam || !uprog->params_contiguous))
        return fail(QFB_EINVAL, "qfb_ucc_create: gradient programs do not match the ansatz");
    for (const auto &g : ham->h_groups)
        if (g.h >= nqubit) return fail(QFB_EINVAL, "qfb_ucc_create: H acts beyond qubit %d", nqubit);
    for (const qfb_prog_s *p : {static_cast<const qfb_prog_s *>(fprog),
                                static_cast<const qfb_prog_s *>(gprog),
                                static_cast<const qfb_prog_s *>(uprog)}) {
        if (!p) continue;
        for (const auto &st : p->h_steps)
            if (st.h >= nqubit) return fail(QFB_EINVAL, "qfb_ucc_create: program beyond qubit");
        for (const auto &sd : p->h_strs)
            if (sd.z >> nqubit) return fail(QFB_EINVAL, "qfb_ucc_create: program beyond qubit");
    }
    int prc = ensure_tiled(ham, nqubit);
    if (prc == QFB_OK) prc = ensure_plans(fprog, nqubit, true);
    if (prc == QFB_OK && gprog) prc = ensure_plans(gprog, nqubit, false, uprog);
    if (prc) return prc;
    std::vector<uint64_t> sector;
    std::vector<SecGroup> sgroups;
    if (prog_conserves(fprog) && (!gprog || (prog_sum_conserves(gprog) && prog_conserves(uprog)))) {
        sector = sector_indices(nqubit, ref_index);
        const uint64_t A = 0x5555555555555555ull;
        for (const auto &g : ham->h_groups) {
            const int ha = __builtin_popcountll(g.x & A), hb = __builtin_popcountll(g.x & ~A);
            if ((ha | hb) & 1) continue;  // never connects two indices of one sector
            sgroups.push_back(SecGroup{g.x, g.begin, g.end, g.real, ha / 2 | (hb / 2) << 8});
        }
        if (sgroups.empty()) sector.clear();
    }
    std::shared_ptr<SectorPlan> plan;
    bool compact = false, gsec = false;
    if (g_ucc_compact && allow_sector && !sector.empty()) {
        const uint64_t A = 0x5555555555555555ull, all = (1ull << nqubit) - 1ull;
        const int ka = __builtin_popcountll(ref_index & A & all);
        const int kb = __builtin_popcountll(ref_index & ~A & all);
        auto get_plan = [&](bool shared) {
            const auto key = std::make_tuple(gprog ? gprog->uid : 0, uprog ? uprog->uid : 0, nqubit,
                                             ka, kb, shared ? 1 : 0);
            auto it = fprog->sector_plans.find(key);
            if (it != fprog->sector_plans.end()) return it->second;
            auto sp = std::make_shared<SectorPlan>();
            std::shared_ptr<SectorPlan> r;
            if (build_sector_plan(*sp, fprog, gprog, uprog, nqubit, ref_index, shared)) r = sp;
            fprog->sector_plans[key] = r;
            return r;
        };
        if (g_ucc_compact == 1 || g_ucc_compact == 4 || g_ucc_compact == 6) {  // 2, 3: global memory only (3: sigma without stored rows)
            plan = get_plan(true);
            compact = plan != nullptr;
        }
        if (!compact) {
            plan = get_plan(false);
            gsec = plan != nullptr;
        }
    }
    static const SectorPlan no_plan;
    const SectorPlan &splan = plan ? *plan : no_plan;
    if (compact) {
        int src = sector_smem_attr();
        if (src) return src;
    }
    if (compact || gsec) sector.clear();
    const int spw = gsec ? (int)std::min<int64_t>(32, 1ll << (int)std::ceil(std::log2((double)nbatch))) : 32;
    const unsigned sgrid = gsec ? global_grid(std::max(stream_max_pairs(splan.fwd),
                                                       stream_max_pairs(splan.sweep)), spw)
                                : 1;
    const unsigned hgrid = gsec ? (unsigned)std::min<int64_t>(1024, (splan.nsec + 7) / 8) : 1;
    qfb_ucc u = new qfb_ucc_s;
    u->compact = compact ? 1 : 0;
    u->gsec = gsec ? 1 : 0;
    u->fwd = fprog;
    u->grad = gprog;
    u->unrot = uprog;
    u->ham = ham;
    u->nqubit = nqubit;
    u->nbatch = nbatch;
    u->nparam = fprog->nparam;
    u->nbasis = 1ull << nqubit;
    u->ref = ref_index;
    u->vchunks = grid_for(u->nbasis, 256, 2);
    if (u->vchunks * (unsigned)nbatch > 65535u) u->vchunks = std::max(1u, 65535u / nbatch);
    u->gchunks = compact ? qfbs::kSweepThreads / 32
                         : gsec ? sgrid : (gprog ? grad_chunks(gprog, nqubit, nbatch) : 1);
    const size_t B = nbatch, M = std::max(u->nparam, 1);
    const size_t nsteps = gprog ? std::max<size_t>(gprog->h_steps.size(), 1) : 1;
    const size_t b_state = (compact || gsec) ? 16 : sizeof(double2) * u->nbasis * B;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_psi = take(b_state), o_sig = take(b_state);
    const size_t o_par = take(sizeof(double) * B * M), o_en = take(sizeof(double) * B);
    const size_t o_gr = take(sizeof(double) * B * M);
    const size_t o_vp = take(sizeof(double2) * B * u->vchunks);
    const size_t o_gp = take(gprog ? sizeof(double2) * nsteps * B * u->gchunks : 16);
    const size_t o_ps = take(sizeof(int2) * M);
    const size_t idx_bytes = nqubit <= 32 ? sizeof(uint32_t) : sizeof(uint64_t);
    const size_t o_sec = take(idx_bytes * std::max<size_t>(sector.size(), 1));
    const size_t o_sg = take(sizeof(SecGroup) * std::max<size_t>(sgroups.size(), 1));
    const size_t o_save = take(compact ? sizeof(double2) * 2 * (size_t)splan.nsec * B : 16);
    const size_t o_hep = take(compact ? sizeof(double) * B * kSectorHSlicesMax : 16);
    const size_t o_hcnt = take(compact ? sizeof(unsigned) * B : 16);
    // global-memory compact states are real doubles when H and every step are real
    bool greal = gsec && !ucc_complex_states() && stream_is_real(splan.fwd) && stream_is_real(splan.sweep);
    for (const SecGroup &g : sgroups) greal = greal && g.real;
    const size_t b_cstate = gsec ? (greal ? sizeof(double) : sizeof(double2)) * (size_t)splan.nsec * B : 16;
    const size_t o_cpsi = take(b_cstate), o_csig = take(b_cstate);
    const size_t o_epart = take(gsec ? sizeof(double2) * B * hgrid : 16);
    int rc = dev_alloc(&u->blob, off);
    if (rc) {
        delete u;
        return rc;
    }
    u->bytes = off;
    char *base = (char *)u->blob;
    u->psi = (double2 *)(base + o_psi);
    u->sig = (double2 *)(base + o_sig);
    u->params = (double *)(base + o_par);
    u->energy = (double *)(base + o_en);
    u->gradv = (double *)(base + o_gr);
    u->vpart = (double2 *)(base + o_vp);
    u->gpart = (double2 *)(base + o_gp);
    u->psteps = (int2 *)(base + o_ps);
    u->nprows = (int64_t)nsteps;
    u->nsec = compact ? (int64_t)splan.nsec : (int64_t)sector.size();
    u->SL.save = (double2 *)(base + o_save);
    u->h_epart = (double *)(base + o_hep);
    u->h_count = (unsigned *)(base + o_hcnt);
    if (gsec) {
        u->nsec = splan.nsec;
        u->GL.nsec = splan.nsec;
        u->GL.nbeta = splan.nbeta;
        u->GL.B = nbatch;
        u->GL.spw = spw;
        u->GL.psi = base + o_cpsi;
        u->GL.sig = base + o_csig;
        u->greal = greal ? 1 : 0;
        u->GL.params = u->params;
        u->GL.nparam = u->nparam;
        u->g_sgrid = sgrid;
        u->g_hgrid = hgrid;
        u->g_ygrid = (unsigned)((nbatch + spw - 1) / spw);
        u->g_epart = (double2 *)(base + o_epart);
    }
    u->sec = base + o_sec;
    u->sgroups = (SecGroup *)(base + o_sg);
    u->nsgroups = (int)sgroups.size();
    std::vector<uint32_t> sec32;
    if (nqubit <= 32) sec32.assign(sector.begin(), sector.end());
    std::vector<int2> ps(M, make_int2(0, 0));
    if (gprog)
        for (int mu = 0; mu < gprog->nparam; ++mu)
            ps[mu] = make_int2(std::max(gprog->p_step0[mu], 0), std::max(gprog->p_step1[mu], 0));
    cudaError_t e = cudaMemsetAsync(u->blob, 0, off, t_stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(u->psteps, ps.data(), sizeof(int2) * M, cudaMemcpyHostToDevice,
                            t_stream);
    if (e == cudaSuccess && !sector.empty())
        e = cudaMemcpyAsync(u->sec, nqubit <= 32 ? (const void *)sec32.data() : (const void *)sector.data(),
                            idx_bytes * sector.size(), cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !sgroups.empty())
        e = cudaMemcpyAsync(u->sgroups, sgroups.data(), sizeof(SecGroup) * sgroups.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&u->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        dev_free(u->blob);
        delete u;
        return cuda_fail(e, "qfb_ucc_create");
    }
    if (compact || gsec) {
        rc = sector_attach(u, ham, plan, sgroups, gsec);
        if (rc) {
            qfb_ucc_destroy(u);
            return rc;
        }
    }
    *out = u;
    return QFB_OK;
}

int qfb_ucc_tiles(int fwd_bits, int grad_bits, int low_bits) {
    if (low_bits < 0 || low_bits > 6 || fwd_bits < low_bits + 2 || fwd_bits > 13 ||
        grad_bits < low_bits + 2 || grad_bits > 12)
        return fail(QFB_EINVAL, "qfb_ucc_tiles: (%d, %d, %d) outside fwd in [low+2, 13], "
                    "grad in [low+2, 12], low in [0, 6]", fwd_bits, grad_bits, low_bits);
    g_win_fwd = fwd_bits;
    g_win_grad = grad_bits;
    g_win_low = low_bits;
    return QFB_OK;
}

int qfb_ucc_config(int compact) {
    if (compact < 0 || compact > 6) return fail(QFB_EINVAL, "qfb_ucc_config: compact = %d", compact);
    g_ucc_compact = compact;
    return QFB_OK;
}

int qfb_ucc_real_states(qfb_ucc u, int32_t *real) {
    if (!u || !real) return fail(QFB_EINVAL, "qfb_ucc_real_states: null argument");
    *real = u->sreal | u->greal;
    return QFB_OK;
}

int qfb_ucc_sets_per_cta(qfb_ucc u, int32_t *sets) {
    if (!u || !sets) return fail(QFB_EINVAL, "qfb_ucc_sets_per_cta: null argument");
    *sets = u->compact ? (u->paired ? 2 : 1) : 0;
    return QFB_OK;
}

int qfb_ucc_rows(qfb_ucc u, int64_t *nnz) {
    if (!u || !nnz) return fail(QFB_EINVAL, "qfb_ucc_rows: null argument");
    *nnz = u->nnz;
    return QFB_OK;
}

int qfb_ucc_path(qfb_ucc u, int32_t *path) {
    if (!u || !path) return fail(QFB_EINVAL, "qfb_ucc_path: null argument");
    *path = u->gsec ? 3 : u->compact ? 2 : (u->nsec > 0 ? 1 : 0);
    return QFB_OK;
}

int qfb_ucc_sector(qfb_ucc u, int64_t *nsec) {
    if (!u || !nsec) return fail(QFB_EINVAL, "qfb_ucc_sector: null argument");
    *nsec = u->nsec;
    return QFB_OK;
}

int qfb_ucc_destroy(qfb_ucc u) {
    if (!u) return QFB_OK;
    dev_free(u->pblob);
    dev_free(u->rblob);
    for (auto &x : u->exec)
        if (x) cudaGraphExecDestroy(x);
    if (u->cap_stream) cudaStreamDestroy(u->cap_stream);
    for (auto &x : u->hside)
        if (x) cudaStreamDestroy(x);
    for (auto &x : u->hjoin)
        if (x) cudaEventDestroy(x);
    if (u->hfork) cudaEventDestroy(u->hfork);
    dev_free(u->hblob);
    dev_free(u->blob);
    delete u;
    return QFB_OK;
}

int qfb_ucc_set_pool(qfb_ucc u, qfb_prog pool) {
    if (!u || !pool) return fail(QFB_EINVAL, "qfb_ucc_set_pool: null argument");
    if (!pool->params_contiguous || pool->nparam < 1)
        return fail(QFB_EINVAL, "qfb_ucc_set_pool: the pool program needs one parameter per operator");
    for (const auto &st : pool->h_steps)
        if (st.h >= u->nqubit) return fail(QFB_EINVAL, "qfb_ucc_set_pool: pool acts beyond qubit");
    const int B = u->nbatch, M = pool->nparam;
    const size_t nst = pool->h_steps.size();
    if (nst == 0 || nst > 65535) return fail(QFB_ENOSYS, "qfb_ucc_set_pool: %zu pool steps", nst);
    qfbs::SStream ps{};
    StreamHost sh;
    PairHost ph;  // shared-memory sector: the pool as pair lists
    unsigned chunks = 1;
    if (u->compact || u->gsec) {
        std::vector<CStep> cs;
        if (!sector_steps(*u->splan, pool, u->nqubit, cs))
            return fail(QFB_ENOSYS, "qfb_ucc_set_pool: pool outside the Givens form on the sector");
        for (size_t k = 0; k < cs.size(); ++k) {
            if (u->gsec && !push_record(sh, cs[k], qfbs::R_IP, (int)k, 1 << 30))
                return fail(QFB_ENOSYS, "qfb_ucc_set_pool: pool step too large");
            if (u->compact && !push_pairs(ph, *u->splan, cs[k], qfbs::R_IP, (int)k, u->sreal ? 16 : 8))
                return fail(QFB_ENOSYS, "qfb_ucc_set_pool: pool step too large");
        }
        bool real = true;
        for (const double2 &c : ph.coef) real = real && c.y == 0.0;
        if ((u->sreal && !real) || (u->greal && !stream_is_real(sh)))
            return fail(QFB_ENOSYS, "qfb_ucc_set_pool: complex pool coefficients on an evaluator "
                                    "with real states (create it with qfb_ucc_config(4))");
        chunks = u->compact ? kSectorThreads / 32 : global_grid(stream_max_pairs(sh), u->GL.spw);
    } else {
        uint64_t most = 1;
        for (const auto &st : pool->h_steps) {
            if (st.tab < 0 || st.na <= 0 || st.x == 0)
                return fail(QFB_ENOSYS, "qfb_ucc_set_pool: pool step outside the Givens form");
            const int fb = u->nqubit - 1 - st.nd;
            if (fb < 0) return fail(QFB_ENOSYS, "qfb_ucc_set_pool: pool step wider than the state");
            most = std::max<uint64_t>(most, (uint64_t)st.na << fb);
        }
        chunks = (unsigned)std::min<uint64_t>(256, std::max<uint64_t>(1, most / (256 * 8)));
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_pg = take(sizeof(double) * (size_t)B * M);
    const size_t o_pp = take(sizeof(double2) * nst * B * chunks);
    const size_t o_pr = take(sizeof(int2) * M);
    const size_t o_ps = take((u->compact || u->gsec) ? 16 : sizeof(StepDev) * nst);
    const size_t o_rec = take(sizeof(uint4) * sh.rec.size());
    const size_t o_sp = take(sizeof(int2) * sh.span.size());
    const size_t o_pl = take(u->compact ? pair_bytes(ph) : 16);
    void *blob = nullptr;
    int rc = dev_alloc(&blob, off);
    if (rc) return rc;
    char *base = (char *)blob;
    std::vector<int2> pr(M);
    for (int k = 0; k < M; ++k)
        pr[k] = pool->p_step0[k] >= 0 ? make_int2(pool->p_step0[k], pool->p_step1[k]) : make_int2(0, 0);
    cudaError_t e = cudaMemsetAsync(blob, 0, off, t_stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + o_pr, pr.data(), sizeof(int2) * M, cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !u->compact && !u->gsec)
        e = cudaMemcpyAsync(base + o_ps, pool->h_steps.data(), sizeof(StepDev) * nst,
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !sh.rec.empty())
        e = cudaMemcpyAsync(base + o_rec, sh.rec.data(), sizeof(uint4) * sh.rec.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess && !sh.span.empty())
        e = cudaMemcpyAsync(base + o_sp, sh.span.data(), sizeof(int2) * sh.span.size(),
                            cudaMemcpyHostToDevice, t_stream);
    qfbs::PStream pp{};
    if (e == cudaSuccess && u->compact && pair_upload(ph, base + o_pl, pp)) e = cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e != cudaSuccess) {
        dev_free(blob);
        return cuda_fail(e, "qfb_ucc_set_pool");
    }
    dev_free(u->pblob);
    if (u->exec[3]) {
        cudaGraphExecDestroy(u->exec[3]);
        u->exec[3] = nullptr;
    }
    u->pblob = blob;
    u->pool = pool;
    u->npool = M;
    u->pgrad = (double *)(base + o_pg);
    u->ppart = (double2 *)(base + o_pp);
    u->pranges = (int2 *)(base + o_pr);
    u->pool_steps = (StepDev *)(base + o_ps);
    u->pchunks = chunks;
    ps.rec = (const uint4 *)(base + o_rec);
    ps.span = (const int2 *)(base + o_sp);
    ps.param = nullptr;
    ps.n = (int)sh.span.size();
    ps.maxw = std::max(sh.maxw, 1);
    u->pstream = ps;
    u->ppairs = pp;
    return QFB_OK;
}

int qfb_ucc_set_residuals(qfb_ucc u, const uint64_t *dets, const qfb_complex *phases, int32_t n) {
    if (!u || n < 1 || !dets || !phases)
        return fail(QFB_EINVAL, "qfb_ucc_set_residuals: bad arguments");
    for (int32_t k = 0; k < n; ++k)
        if (dets[k] >> u->nqubit)
            return fail(QFB_EINVAL, "qfb_ucc_set_residuals: determinant %d beyond qubit %d", k,
                        u->nqubit);
    std::vector<int64_t> idx((size_t)n);
    for (int32_t k = 0; k < n; ++k) {
        if (u->compact || u->gsec) {
            const SectorPlan &sp = *u->splan;
            const int32_t ra = sp.arank[pext_parity_bits(dets[k], 0, u->nqubit)];
            const int32_t rb = sp.brank[pext_parity_bits(dets[k], 1, u->nqubit)];
            idx[k] = (ra < 0 || rb < 0) ? -1 : (int64_t)ra * sp.nbeta + rb;
        } else {
            idx[k] = (int64_t)dets[k];
        }
    }
    // compact, shared memory: the forward pair-list headers in reverse order
    std::vector<qfbs::PHead> rhd;
    if (u->compact) rhd.assign(u->pairs->fwd_hd.rbegin(), u->pairs->fwd_hd.rend());
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const int B = u->nbatch;
    const size_t o_res = 0, o_idx = al(sizeof(double) * (size_t)B * n),
                 o_ph = o_idx + al(sizeof(int64_t) * n), o_sp = o_ph + al(sizeof(double2) * n),
                 total = o_sp + sizeof(qfbs::PHead) * std::max<size_t>(1, rhd.size());
    void *blob = nullptr;
    int rc = dev_alloc(&blob, total);
    if (rc) return rc;
    char *bp = (char *)blob;
    std::vector<double2> ph((size_t)n);
    for (int32_t k = 0; k < n; ++k) ph[k] = make_double2(phases[k].re, phases[k].im);
    QFB_CUDA(cudaMemcpyAsync(bp + o_idx, idx.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice,
                             t_stream));
    QFB_CUDA(cudaMemcpyAsync(bp + o_ph, ph.data(), sizeof(double2) * n, cudaMemcpyHostToDevice,
                             t_stream));
    if (!rhd.empty())
        QFB_CUDA(cudaMemcpyAsync(bp + o_sp, rhd.data(), sizeof(qfbs::PHead) * rhd.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaMemsetAsync(bp + o_res, 0, sizeof(double) * (size_t)B * n, t_stream));
    if (u->exec[4]) {  // a captured residual run refers to the old buffers
        cudaGraphExecDestroy(u->exec[4]);
        u->exec[4] = nullptr;
    }
    if (u->rblob) {
        u->bytes -= u->rbytes;
        dev_free(u->rblob);
    }
    u->rblob = blob;
    u->rbytes = total;
    u->bytes += total;
    u->nres = n;
    u->res = (double *)(bp + o_res);
    u->ridx = (const int64_t *)(bp + o_idx);
    u->rphase = (const double2 *)(bp + o_ph);
    if (u->compact) {
        u->rstream = u->SL.fwd;
        u->rstream.hd = (const qfbs::PHead *)(bp + o_sp);
    }
    return QFB_OK;
}

int qfb_ucc_residual_buffer(qfb_ucc u, double **d_res) {
    if (!u || !d_res) return fail(QFB_EINVAL, "qfb_ucc_residual_buffer: null argument");
    if (!u->rblob) return fail(QFB_EINVAL, "qfb_ucc_residual_buffer: no residuals set");
    *d_res = u->res;
    return QFB_OK;
}

int qfb_ucc_eval_residuals(qfb_ucc u, const double *params, double *energy, double *res) {
    if (!u || !energy || !res) return fail(QFB_EINVAL, "qfb_ucc_eval_residuals: null argument");
    if (!u->rblob) return fail(QFB_EINVAL, "qfb_ucc_eval_residuals: no residuals set");
    if (u->nparam > 0 && !params) return fail(QFB_EINVAL, "qfb_ucc_eval_residuals: null parameters");
    const size_t np = (size_t)u->nbatch * u->nparam;
    if (np) QFB_CUDA(cudaMemcpyAsync(u->params, params, sizeof(double) * np,
                                     cudaMemcpyHostToDevice, t_stream));
    int rc = qfb_ucc_run(u, 4);
    if (rc) return rc;
    QFB_CUDA(cudaMemcpyAsync(energy, u->energy, sizeof(double) * u->nbatch,
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaMemcpyAsync(res, u->res, sizeof(double) * u->nbatch * u->nres,
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_ucc_eval_pool(qfb_ucc u, const double *params, double *energy, double *pool_grad) {
    if (!u || !energy || !pool_grad) return fail(QFB_EINVAL, "qfb_ucc_eval_pool: null argument");
    if (!u->pool) return fail(QFB_EINVAL, "qfb_ucc_eval_pool: no pool set");
    if (u->nparam > 0 && !params) return fail(QFB_EINVAL, "qfb_ucc_eval_pool: null parameters");
    const size_t np = (size_t)u->nbatch * u->nparam;
    if (np) QFB_CUDA(cudaMemcpyAsync(u->params, params, sizeof(double) * np,
                                     cudaMemcpyHostToDevice, t_stream));
    int rc = qfb_ucc_run(u, 3);
    if (rc) return rc;
    QFB_CUDA(cudaMemcpyAsync(energy, u->energy, sizeof(double) * u->nbatch,
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaMemcpyAsync(pool_grad, u->pgrad, sizeof(double) * u->nbatch * u->npool,
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_ucc_pool_buffer(qfb_ucc u, double **d_pool_grad) {
    if (!u || !d_pool_grad) return fail(QFB_EINVAL, "qfb_ucc_pool_buffer: null argument");
    if (!u->pool) return fail(QFB_EINVAL, "qfb_ucc_pool_buffer: no pool set");
    *d_pool_grad = u->pgrad;
    return QFB_OK;
}

int qfb_ucc_memory(qfb_ucc u, uint64_t *bytes) {
    if (!u || !bytes) return fail(QFB_EINVAL, "qfb_ucc_memory: null argument");
    *bytes = u->bytes;
    return QFB_OK;
}

int qfb_ucc_buffers(qfb_ucc u, double **d_params, double **d_energy, double **d_grad) {
    if (!u) return fail(QFB_EINVAL, "qfb_ucc_buffers: null evaluator");
    if (d_params) *d_params = u->params;
    if (d_energy) *d_energy = u->energy;
    if (d_grad) *d_grad = u->gradv;
    return QFB_OK;
}

int qfb_ucc_run(qfb_ucc u, int with_grad) {
    if (!u) return fail(QFB_EINVAL, "qfb_ucc_run: null evaluator");
    if (with_grad < 0 || with_grad > 4) return fail(QFB_EINVAL, "qfb_ucc_run: mode %d", with_grad);
    const int k = with_grad;
    if (u->exec[k]) {
        QFB_CUDA(cudaGraphLaunch(u->exec[k], t_stream));
        g_launches.fetch_add(u->graph_kernels[k], std::memory_order_relaxed);
        return QFB_OK;
    }
    return ucc_enqueue(u, with_grad);
}

int qfb_ucc_capture(qfb_ucc u, int with_grad) {
    if (!u) return fail(QFB_EINVAL, "qfb_ucc_capture: null evaluator");
    if (with_grad < 0 || with_grad > 4)
        return fail(QFB_EINVAL, "qfb_ucc_capture: mode %d", with_grad);
    const int k = with_grad;
    if (u->exec[k]) return QFB_OK;
    cudaStream_t saved = t_stream;
    t_stream = u->cap_stream;
    const uint64_t n0 = g_launches.load();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(u->cap_stream, cudaStreamCaptureModeThreadLocal);
    int rc = (e == cudaSuccess) ? ucc_enqueue(u, with_grad) : cuda_fail(e, "begin capture");
    cudaError_t e2 = cudaStreamEndCapture(u->cap_stream, &graph);
    t_stream = saved;
    const uint64_t nk = g_launches.load() - n0;
    g_launches.fetch_sub(nk, std::memory_order_relaxed);  // counted when replayed
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "end capture");
    e = cudaGraphInstantiate(&u->exec[k], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        u->exec[k] = nullptr;
        return cuda_fail(e, "graph instantiate");
    }
    u->graph_kernels[k] = nk;
    return QFB_OK;
}

int qfb_ucc_eval(qfb_ucc u, const double *params, double *energy, double *grad) {
    if (!u || !energy) return fail(QFB_EINVAL, "qfb_ucc_eval: null argument");
    if (u->nparam > 0 && !params) return fail(QFB_EINVAL, "qfb_ucc_eval: null parameters");
    const size_t np = (size_t)u->nbatch * u->nparam;
    if (np) QFB_CUDA(cudaMemcpyAsync(u->params, params, sizeof(double) * np,
                                     cudaMemcpyHostToDevice, t_stream));
    int rc = qfb_ucc_run(u, grad ? 1 : 0);
    if (rc) return rc;
    QFB_CUDA(cudaMemcpyAsync(energy, u->energy, sizeof(double) * u->nbatch,
                             cudaMemcpyDeviceToHost, t_stream));
    if (grad && np)
        QFB_CUDA(cudaMemcpyAsync(grad, u->gradv, sizeof(double) * np, cudaMemcpyDeviceToHost,
                                 t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_ucc_profile(qfb_ucc u, int with_grad, int reps, double *stage_ms,
                    int64_t *stage_launches) {
    if (!u || !stage_ms || reps < 1) return fail(QFB_EINVAL, "qfb_ucc_profile: bad argument");
    cudaEvent_t ev[5];
    for (auto &e : ev) QFB_CUDA(cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    int64_t nl[4] = {0, 0, 0, 0};
    int rc = QFB_OK;
    for (int r = 0; r < reps && rc == QFB_OK; ++r) {
        QFB_CUDA(cudaEventRecord(ev[0], t_stream));
        for (int st = 0; st < 4 && rc == QFB_OK; ++st) {
            const uint64_t l0 = g_launches.load();
            rc = ucc_stage(u, st, with_grad);
            nl[st] = (int64_t)(g_launches.load() - l0);
            QFB_CUDA(cudaEventRecord(ev[st + 1], t_stream));
        }
        QFB_CUDA(cudaEventSynchronize(ev[4]));
        for (int st = 0; st < 4; ++st) {
            float ms = 0.f;
            QFB_CUDA(cudaEventElapsedTime(&ms, ev[st], ev[st + 1]));
            acc[st] += ms;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int st = 0; st < 4; ++st) {
        stage_ms[st] = acc[st] / reps;
        if (stage_launches) stage_launches[st] = nl[st];
    }
    return rc;
}

}  // extern "C"

// ===========================================================================
// packed evaluations: parameter sets of several problems in one launch
// ===========================================================================

struct qfb_pack_s {
    int nmem = 0, cap = 0, maxparam = 1, max_rows = 1, sreal = 0;
    size_t smem = 0, bytes = 0;
    void *blob = nullptr;
    qfbs::PackMember *d_mem = nullptr;
    int2 *items = nullptr;
    double *params = nullptr, *energy = nullptr, *grad = nullptr;
    double2 *partial = nullptr;
};

extern "C" int qfb_pack_create(const qfb_ucc *members, int nmembers, int capacity, qfb_pack *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_pack_create: null output");
    *out = nullptr;
    if (!members || nmembers < 1 || capacity < 1 || capacity > 65535)
        return fail(QFB_EINVAL, "qfb_pack_create: need members and a capacity in [1, 65535]");
    int rc = sector_smem_attr();
    if (rc) return rc;
    auto p = std::make_unique<qfb_pack_s>();
    p->nmem = nmembers;
    p->cap = capacity;
    std::vector<qfbs::PackMember> hm((size_t)nmembers);
    for (int k = 0; k < nmembers; ++k) {
        const qfb_ucc u = members[k];
        if (!u) return fail(QFB_EINVAL, "qfb_pack_create: member %d is null", k);
        if (!u->compact || u->gsec)
            return fail(QFB_EINVAL,
                        "qfb_pack_create: member %d does not keep its states in shared memory "
                        "(only compact-sector evaluators of up to ~16 qubits can be packed)", k);
        if (u->nparam > 0 && !u->grad)
            return fail(QFB_EINVAL, "qfb_pack_create: member %d has no gradient program", k);
        if (k == 0) p->sreal = u->sreal;
        if (u->sreal != p->sreal)
            return fail(QFB_EINVAL, "qfb_pack_create: members mix real and complex state storage");
        const qfbs::SLaunch &L = u->SL;
        const size_t es = u->sreal ? sizeof(qfbs::PSmem<double>) : sizeof(qfbs::PSmem<double2>);
        const size_t need = qfbs::sector_smem_states(2, (size_t)L.nsec, u->sreal) +
                            es * (size_t)std::max(L.fwd.n, L.sweep.n);
        if (need > kSectorSmemMax)
            return fail(QFB_EINVAL, "qfb_pack_create: member %d needs %zu bytes of shared memory",
                        k, need);
        p->smem = std::max(p->smem, need);
        p->maxparam = std::max(p->maxparam, u->nparam);
        p->max_rows = std::max(p->max_rows, (int)u->nprows);
        qfbs::PackMember &m = hm[(size_t)k];
        m.nsec = L.nsec;
        m.ref_i = L.ref_i;
        m.nparam = u->nparam;
        m.pad = 0;
        m.fwd = L.fwd;
        m.sweep = L.sweep;
        m.rowptr = L.rowptr;
        m.col = L.col;
        m.val_r = L.val_r;
        m.val_c = L.val_c;
        m.psteps = u->psteps;
    }
    const size_t C = (size_t)capacity, MP = (size_t)p->maxparam;
    const size_t nw = qfbs::kPackThreads / 32;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_mem = take(sizeof(qfbs::PackMember) * (size_t)nmembers);
    const size_t o_it = take(sizeof(int2) * C), o_par = take(sizeof(double) * C * MP);
    const size_t o_en = take(sizeof(double) * C), o_gr = take(sizeof(double) * C * MP);
    const size_t o_pt = take(sizeof(double2) * C * (size_t)p->max_rows * nw);
    rc = dev_alloc(&p->blob, off);
    if (rc) return rc;
    p->bytes = off;
    char *base = (char *)p->blob;
    p->d_mem = (qfbs::PackMember *)(base + o_mem);
    p->items = (int2 *)(base + o_it);
    p->params = (double *)(base + o_par);
    p->energy = (double *)(base + o_en);
    p->grad = (double *)(base + o_gr);
    p->partial = (double2 *)(base + o_pt);
    cudaError_t e = cudaMemsetAsync(p->blob, 0, off, t_stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_mem, hm.data(), sizeof(qfbs::PackMember) * hm.size(),
                            cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e != cudaSuccess) {
        dev_free(p->blob);
        return cuda_fail(e, "qfb_pack_create");
    }
    *out = p.release();
    return QFB_OK;
}

extern "C" int qfb_pack_destroy(qfb_pack p) {
    if (!p) return QFB_OK;
    dev_free(p->blob);
    delete p;
    return QFB_OK;
}

extern "C" int qfb_pack_info(qfb_pack p, int32_t *capacity, int32_t *maxparam, uint64_t *bytes) {
    if (!p) return fail(QFB_EINVAL, "qfb_pack_info: null pack");
    if (capacity) *capacity = p->cap;
    if (maxparam) *maxparam = p->maxparam;
    if (bytes) *bytes = p->bytes;
    return QFB_OK;
}

extern "C" int qfb_pack_buffers(qfb_pack p, int32_t **items, double **params, double **energy,
                                double **grad) {
    if (!p) return fail(QFB_EINVAL, "qfb_pack_buffers: null pack");
    if (items) *items = (int32_t *)p->items;
    if (params) *params = p->params;
    if (energy) *energy = p->energy;
    if (grad) *grad = p->grad;
    return QFB_OK;
}

extern "C" int qfb_pack_launch(qfb_pack p, int nitems) {
    if (!p) return fail(QFB_EINVAL, "qfb_pack_launch: null pack");
    if (nitems < 0 || nitems > p->cap)
        return fail(QFB_EINVAL, "qfb_pack_launch: %d items for a capacity of %d", nitems, p->cap);
    if (nitems == 0) return QFB_OK;
    if (p->sreal)
        qfbs::k_sector_pack<double><<<nitems, qfbs::kPackThreads, p->smem, t_stream>>>(
            p->d_mem, p->items, p->maxparam, p->params, p->energy, p->grad, p->partial, p->max_rows,
            p->nmem);
    else
        qfbs::k_sector_pack<double2><<<nitems, qfbs::kPackThreads, p->smem, t_stream>>>(
            p->d_mem, p->items, p->maxparam, p->params, p->energy, p->grad, p->partial, p->max_rows,
            p->nmem);
    QFB_LAUNCHED();
    return QFB_OK;
}

extern "C" int qfb_pack_run(qfb_pack p, const int32_t *member, const int32_t *with_grad, int nitems,
                            const double *params, double *energy, double *grad) {
    if (!p) return fail(QFB_EINVAL, "qfb_pack_run: null pack");
    if (nitems < 0 || nitems > p->cap)
        return fail(QFB_EINVAL, "qfb_pack_run: %d items for a capacity of %d", nitems, p->cap);
    if (nitems == 0) return QFB_OK;
    if (!member || !params || !energy)
        return fail(QFB_EINVAL, "qfb_pack_run: null argument");
    std::vector<int2> it((size_t)nitems);
    bool any_grad = false;
    for (int i = 0; i < nitems; ++i) {
        if (member[i] < 0 || member[i] >= p->nmem)
            return fail(QFB_EINVAL, "qfb_pack_run: item %d names member %d of %d", i, member[i],
                        p->nmem);
        it[(size_t)i] = make_int2(member[i], with_grad && with_grad[i] ? 1 : 0);
        any_grad = any_grad || it[(size_t)i].y;
    }
    if (any_grad && !grad) return fail(QFB_EINVAL, "qfb_pack_run: gradients asked for, no buffer");
    const size_t MP = (size_t)p->maxparam;
    QFB_CUDA(cudaMemcpyAsync(p->items, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice,
                             t_stream));
    QFB_CUDA(cudaMemcpyAsync(p->params, params, sizeof(double) * MP * nitems,
                             cudaMemcpyHostToDevice, t_stream));
    int rc = qfb_pack_launch(p, nitems);
    if (rc) return rc;
    QFB_CUDA(cudaMemcpyAsync(energy, p->energy, sizeof(double) * nitems, cudaMemcpyDeviceToHost,
                             t_stream));
    if (grad)
        QFB_CUDA(cudaMemcpyAsync(grad, p->grad, sizeof(double) * MP * nitems,
                                 cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

// ===========================================================================
// expectation values without device allocation
// ===========================================================================

// Scratch of qfb_sum_expval_noalloc: the per-block partial sums and the
// per-segment results live in this fixed array of the library's device image
// instead of a fresh allocation.  Every GPU that loads the library holds it
// (1 MiB) until the process exits.
constexpr size_t kNoAllocEntries = 65536;  // double2 entries
static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocEntries];

static std::mutex g_noalloc_mu;
static double2 *g_noalloc_addr[64];  // device address of the array, per device

// The array's device address on the current device, looked up once per
// device (with that device current) on the first call that needs it.
static int noalloc_scratch(double2 **out) {
    int dev = 0;
    QFB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(QFB_ENOSYS, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_addr[dev] = (double2 *)p;
    }
    *out = g_noalloc_addr[dev];
    return QFB_OK;
}

extern "C" int qfb_sum_expval_noalloc(qfb_sum h, qfb_state bra, qfb_state ket,
                                      qfb_complex *out) {
    if (!h || !bra || !ket || !out)
        return fail(QFB_EINVAL, "qfb_sum_expval_noalloc: null argument");
    if (bra->nqubit != ket->nqubit || bra->nbatch != ket->nbatch)
        return fail(QFB_EINVAL, "qfb_sum_expval_noalloc: bra and ket shapes differ");
    for (const auto &g : h->h_groups)
        if (g.h >= bra->nqubit)
            return fail(QFB_EINVAL,
                        "qfb_sum_expval_noalloc: operator acts on qubit %d of a %d-qubit state",
                        g.h, bra->nqubit);
    const int B = bra->nbatch;
    const size_t nout = (size_t)B * h->nsegment;
    if (h->ngroups == 0) {
        for (size_t i = 0; i < nout; ++i) out[i] = qfb_complex{0.0, 0.0};
        return QFB_OK;
    }
    if (h->ngroups > 65535)
        return fail(QFB_ENOSYS, "qfb_sum_expval_noalloc: more than 65535 x-groups");
    // one partial per (slot, group, chunk) plus one result per (slot, segment)
    const size_t rows = (size_t)B * h->ngroups;
    if (rows + nout > kNoAllocEntries)
        return fail(QFB_EINVAL,
                    "qfb_sum_expval_noalloc: %d states x %d x-groups + %zu results need more than "
                    "the %zu entries of the fixed scratch; use qfb_sum_expval",
                    B, h->ngroups, nout, kNoAllocEntries);
    unsigned chunks = chunks_for(bra->nbasis >> 1, B, h->ngroups);
    const size_t fit = (kNoAllocEntries - nout) / rows;
    if (chunks > fit) chunks = (unsigned)fit;
    double2 *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // every partial is written by exactly one block before it is read, so
    // the previous call's contents need no clearing
    double2 *partial = scratch;
    double2 *res = scratch + rows * chunks;
    k_sum_expval<<<dim3(chunks, h->ngroups, B), 256, 0, t_stream>>>(
        bra->d, ket->d, bra->nbasis, h->d_groups, h->d_terms, h->ngroups, partial);
    QFB_LAUNCHED();
    k_seg_sum<<<dim3(h->nsegment, B), 256, 0, t_stream>>>(partial, h->d_seg_g0, h->ngroups,
                                                          chunks, res);
    QFB_LAUNCHED();
    QFB_CUDA(cudaMemcpyAsync(out, res, sizeof(double2) * nout, cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}
