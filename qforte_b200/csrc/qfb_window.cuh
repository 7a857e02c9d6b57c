// Windowed Pauli-exponential passes over shared-memory tiles.
//
// exp(i phi P) couples amplitude j only with j ^ x (x = P's X/Y support), and
// its phase (-1)^popcount(j & z) splits into the bits of j inside any qubit
// set Q and a sign that is constant over the rest.  So if every step of a
// run of consecutive exponentials has its x inside one set Q of b qubits, the
// state splits into 2^(n-b) independent tiles (the indices that agree outside
// Q), and the whole run can be applied to each tile in shared memory: one
// read and one write of the state per run instead of per exponential.
//
// The planner walks a program (forward: strings in order; gradient: the
// reverse sweep of UCCVQE.measure_gradient, uccvqeabc.py:122-251) and cuts it
// into windows whose x-supports fit in b qubits.  Q always holds the lowest L
// qubits, so a tile is gathered in contiguous runs of 2^L amplitudes (128 B
// for L = 3), and is padded with the lowest unused qubits up to b.  Each
// window is one launch over (tile, slot); in gradient windows a step can
// also accumulate its share of <sigma|K_mu|psi> (one partial per tile).
//
// The arithmetic per pair is the per-step kernel's, step for step, so a
// windowed program produces the same amplitudes as the unwindowed one.
#pragma once

#include <vector>

namespace qfbw {

struct WStep {       // one step of a window, masks in tile coordinates
    uint64_t xl;     // x compressed into the tile's bits
    int32_t hl;      // highest bit of xl, -1 when xl == 0 (diagonal)
    int32_t s0;      // first string (window-relative)
    int32_t ns;      // strings
    int32_t rotate;  // apply the rotation
    int32_t ip_row;  // >= 0: add this step's <sigma|K|psi> share to that row
    // Givens form (StepDev of qfb_pauli.cu) in tile coordinates; tab < 0: none
    int32_t tab;     // offset into the plan's tables (double2 entries)
    int32_t nd;
    int32_t param;
    int32_t sign;    // angle sign of the rotation
    int32_t pad;
    uint64_t dpos;   // 6-bit tile positions of the pattern bits
    uint64_t zb_l;   // zbase inside the tile ...
    uint64_t zb_c;   // ... and outside it (a per-tile sign)
    double gamma;
    // active pairs only (na > 0): zeros inserted at the nd + 1 sorted tile
    // positions in zpos (4 bits each), then patbits[a] or-ed in
    int32_t na;
    uint32_t zpos;
    uint32_t patbits[8];
    uint8_t patidx[8];
};

struct WStr {
    uint64_t zl;    // z compressed into the tile's bits
    uint64_t zc;    // z outside the tile (per-tile constant sign)
    int32_t ny;     // popcount(x & z) mod 4
    int32_t param;  // parameter index
    double rscale;  // rotation angle = rscale * params[param] (sign included)
    double scale;   // K coefficient is i * scale (inner products)
};

struct Window {
    uint64_t qmask, cmask;
    int32_t b;
    int32_t st0, st1;        // steps [st0, st1) of the plan
    int32_t sr0, sr1;        // strings [sr0, sr1) of the plan
    int32_t tr0, tr1;        // Givens table entries [tr0, tr1) of the plan
    int32_t global_step;     // >= 0: not windowed, run this program step globally
    int32_t global_mu;       // >= 0: not windowed, run parameter mu's gradient globally
    int32_t needs_strings;   // a step without a Givens table: stage the strings
};

constexpr int kWinMaxStr = 512;
constexpr int kWinMaxSteps = 128;
constexpr int kWinMaxTab = 1024;  // double2 table entries staged per window
constexpr int kWinThreads = 256;
constexpr int kWinWarps = kWinThreads / 32;

inline uint64_t pext_h(uint64_t v, uint64_t m) {
    uint64_t r = 0;
    int k = 0;
    while (m) {
        const uint64_t low = m & (~m + 1);
        if (v & low) r |= 1ull << k;
        ++k;
        m &= m - 1;
    }
    return r;
}

__device__ __forceinline__ uint64_t pdep_d(uint64_t v, uint64_t m) {
    uint64_t r = 0;
    while (m) {
        const uint64_t low = m & (~m + 1);
        if (v & 1ull) r |= low;
        v >>= 1;
        m &= m - 1;
    }
    return r;
}

struct WinLaunch {
    uint64_t qmask, cmask;
    int b, L;
    int nsteps, nstr;
    const WStep *steps;  // this window's steps
    const WStr *strs;    // this window's strings
    const double2 *tab;  // this window's Givens tables (WStep::tab is relative)
    int ntab;
    const double *params;
    int nparam, bcast;
    double2 *partial;  // [rows][nbatch][ntiles]
    int ntiles;
};

// Shared-memory layout of a window, ordered by alignment: the 16-byte
// arrays (tiles, per-step and per-string cos/sin) first, then the 8-byte
// ones, then the ints; the spread table starts on a 16-byte boundary.
struct WinSmem {
    size_t cs_step, cs_str, gtab, ipw, steps, g_step, sc_str, zl_str, q_str, tab, total;
};

__host__ __device__ inline WinSmem win_smem_layout(int b, int L, int nstr, int nsteps, int nt,
                                                   int ntab) {
    WinSmem m;
    const size_t T = (size_t)1 << b;
    size_t o = (size_t)nt * T * 16;
    m.cs_step = o;
    o += (size_t)nsteps * 16;
    m.cs_str = o;
    o += (size_t)nstr * 16;
    m.gtab = o;
    o += (size_t)ntab * 16;
    m.ipw = o;
    o += (size_t)2 * kWinWarps * 16;
    m.steps = o;
    o += (size_t)nsteps * sizeof(WStep);
    m.g_step = o;
    o += (size_t)nsteps * 8;
    m.sc_str = o;
    o += (size_t)nstr * 8;
    m.zl_str = o;
    o += (size_t)nstr * 8;
    m.q_str = o;
    o += (size_t)nstr * 4;
    o = (o + 15) & ~(size_t)15;
    m.tab = o;
    o += ((size_t)1 << (b - L)) * 8;
    m.total = o;
    return m;
}

__host__ __device__ inline size_t win_smem_bytes(int b, int L, int nstr, int nsteps, int nt,
                                                 int ntab) {
    return win_smem_layout(b, L, nstr, nsteps, nt, ntab).total;
}

__device__ __forceinline__ int tile_pattern(uint32_t l, int nd, uint64_t dpos) {
    int pat = 0;
    for (int i = 0; i < nd; ++i) pat |= (int)((l >> ((dpos >> (6 * i)) & 63)) & 1u) << i;
    return pat;
}

template <int NT>
__global__ void __launch_bounds__(kWinThreads, 3) k_window(double2 *__restrict__ psi,
                                                        double2 *__restrict__ sig,
                                                        uint64_t nbasis, WinLaunch a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = 1 << a.b;
    const WinSmem lay = win_smem_layout(a.b, a.L, a.nstr, a.nsteps, NT, a.ntab);
    double2 *t0 = reinterpret_cast<double2 *>(smem);
    double2 *t1 = t0 + T;
    double2 *s_stcs = reinterpret_cast<double2 *>(smem + lay.cs_step);  // (cos, sin * tile sign)
    double2 *s_cs = reinterpret_cast<double2 *>(smem + lay.cs_str);
    double *s_stg = reinterpret_cast<double *>(smem + lay.g_step);  // gamma * tile sign
    double *s_sc = reinterpret_cast<double *>(smem + lay.sc_str);
    uint64_t *s_zl = reinterpret_cast<uint64_t *>(smem + lay.zl_str);
    int *s_q = reinterpret_cast<int *>(smem + lay.q_str);
    uint64_t *s_tab = reinterpret_cast<uint64_t *>(smem + lay.tab);
    double2 *s_gtab = reinterpret_cast<double2 *>(smem + lay.gtab);
    double2 *s_ipw = reinterpret_cast<double2 *>(smem + lay.ipw);  // [2][warps]
    WStep *s_steps = reinterpret_cast<WStep *>(smem + lay.steps);

    const int slot = blockIdx.y, tile = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const uint64_t base = pdep_d((uint64_t)tile, a.cmask);
    for (int h = tid; h < (T >> a.L); h += nth) s_tab[h] = pdep_d((uint64_t)h << a.L, a.qmask);
    const double *par = a.params + (a.bcast ? 0 : (size_t)slot * a.nparam);
    for (int i = tid; i < a.nstr; i += nth) {
        const WStr w = a.strs[i];
        double s, c;
        sincos(w.rscale * par[w.param], &s, &c);
        s_cs[i] = make_double2(c, s);
        s_sc[i] = w.scale;
        s_zl[i] = w.zl;
        s_q[i] = (w.ny + 1 + 2 * parity64(base & w.zc)) & 3;
    }
    for (int i = tid; i < a.ntab; i += nth) s_gtab[i] = a.tab[i];
    for (int st = tid; st < a.nsteps; st += nth) {
        const WStep w = a.steps[st];
        s_steps[st] = w;
        if (w.tab < 0) continue;
        const double ts = parity64(base & w.zb_c) ? -1.0 : 1.0;
        double s, c;
        sincos((double)w.sign * w.gamma * par[w.param], &s, &c);
        s_stcs[st] = make_double2(c, s * ts);
        s_stg[st] = w.gamma * ts;
    }
    __syncthreads();
    const uint64_t lowm = (1ull << a.L) - 1ull;
    double2 *P = psi + (uint64_t)slot * nbasis;
    double2 *S = (NT == 2) ? sig + (uint64_t)slot * nbasis : nullptr;
    for (int l = tid; l < T; l += nth) {
        const uint64_t g = base | s_tab[l >> a.L] | ((uint64_t)l & lowm);
        t0[l] = P[g];
        if (NT == 2) t1[l] = S[g];
    }
    __syncthreads();

    // Inner products: each warp reduces its share and publishes it in one of
    // two buffers; after the step's barrier, warp 0 of the next step adds the
    // warps' shares and writes the tile's partial.  One barrier per step.
    const int lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    int pend_row = -1;
    for (int st = 0; st < a.nsteps; ++st) {
        const WStep &w = s_steps[st];
        if (pend_row >= 0 && warp == 0) {
            double2 v = (lane < nwarps) ? s_ipw[((st - 1) & 1) * kWinWarps + lane]
                                        : make_double2(0.0, 0.0);
            v = warp_sum(v);
            if (lane == 0)
                a.partial[((uint64_t)pend_row * gridDim.y + slot) * a.ntiles + tile] = v;
        }
        pend_row = -1;
        double2 ip = make_double2(0.0, 0.0);
        const bool want_ip = (NT == 2) && (w.ip_row >= 0);
        if (w.tab >= 0) {
            const double c = s_stcs[st].x, sn = s_stcs[st].y, gam = s_stg[st];
            const double2 *tb = s_gtab + w.tab;
            const uint32_t xl = (uint32_t)w.xl, zb = (uint32_t)w.zb_l;
            const int nd = w.nd, hl = w.hl;
            const bool act = w.na > 0;
            const int fb = act ? (a.b - 1 - nd) : 0;
            const int total = act ? (w.na << fb) : (T >> 1);
            const uint32_t zpos = w.zpos;
            for (int q = tid; q < total; q += nth) {
                uint32_t l0;
                int pat;
                if (act) {
                    // the q-th active pair: free bits with zeros at D and h
                    const int ai = q >> fb;
                    uint32_t f = (uint32_t)q & ((1u << fb) - 1u);
                    for (int i = 0; i <= nd; ++i) {
                        const int ps = (int)((zpos >> (4 * i)) & 15u);
                        f = ((f >> ps) << (ps + 1)) | (f & ((1u << ps) - 1u));
                    }
                    l0 = f | w.patbits[ai];
                    pat = w.patidx[ai];
                } else {
                    l0 = (uint32_t)insert0((uint64_t)q, hl);
                    pat = tile_pattern(l0, nd, w.dpos);
                }
                const double2 gn = tb[2 * pat], hn = tb[2 * pat + 1];
                if (!act && gn.x == 0.0 && gn.y == 0.0 && hn.x == 0.0 && hn.y == 0.0) continue;
                const uint32_t l1 = l0 ^ xl;
                const bool neg = __popc(l0 & zb) & 1;
                double2 v0 = t0[l0], v1 = t0[l1];
                double2 w0 = make_double2(0.0, 0.0), w1 = w0;
                if (NT == 2) {
                    w0 = t1[l0];
                    w1 = t1[l1];
                }
                if (want_ip) {
                    const double2 t = c_add(c_cjmul(w0, c_mul(hn, v1)), c_cjmul(w1, c_mul(gn, v0)));
                    const double g = neg ? -gam : gam;
                    ip.x += g * t.x;
                    ip.y += g * t.y;
                }
                if (w.rotate) {
                    const double ss = neg ? -sn : sn;
                    {
                        const double2 ra = c_mul(hn, v1), rb = c_mul(gn, v0);
                        const double2 n0 = make_double2(c * v0.x + ss * ra.x, c * v0.y + ss * ra.y);
                        v1 = make_double2(c * v1.x + ss * rb.x, c * v1.y + ss * rb.y);
                        v0 = n0;
                    }
                    t0[l0] = v0;
                    t0[l1] = v1;
                    if (NT == 2) {
                        const double2 ra = c_mul(hn, w1), rb = c_mul(gn, w0);
                        const double2 n0 = make_double2(c * w0.x + ss * ra.x, c * w0.y + ss * ra.y);
                        w1 = make_double2(c * w1.x + ss * rb.x, c * w1.y + ss * rb.y);
                        w0 = n0;
                        t1[l0] = w0;
                        t1[l1] = w1;
                    }
                }
            }
        } else if (w.hl >= 0) {
            for (int p = tid; p < (T >> 1); p += nth) {
                const uint64_t l0 = insert0((uint64_t)p, w.hl), l1 = l0 ^ w.xl;
                double2 v0 = t0[l0], v1 = t0[l1];
                double2 w0 = make_double2(0.0, 0.0), w1 = w0;
                if (NT == 2) {
                    w0 = t1[l0];
                    w1 = t1[l1];
                }
                if (want_ip) {
                    double2 k0 = make_double2(0.0, 0.0), k1 = k0;
                    for (int i = w.s0; i < w.s0 + w.ns; ++i) {
                        const int qa = (s_q[i] + 2 * parity64(l0 & s_zl[i])) & 3;
                        const int qb = (s_q[i] + 2 * parity64(l1 & s_zl[i])) & 3;
                        const double sc = s_sc[i];
                        const double2 r1 = c_ipow(v1, qb), r0 = c_ipow(v0, qa);
                        k0.x += sc * r1.x;
                        k0.y += sc * r1.y;
                        k1.x += sc * r0.x;
                        k1.y += sc * r0.y;
                    }
                    ip = c_add(ip, c_add(c_cjmul(w0, k0), c_cjmul(w1, k1)));
                }
                if (w.rotate) {
                    for (int i = w.s0; i < w.s0 + w.ns; ++i) {
                        const int q0 = (s_q[i] + 2 * parity64(l0 & s_zl[i])) & 3;
                        const int q1 = (s_q[i] + 2 * parity64(l1 & s_zl[i])) & 3;
                        const double2 cs = s_cs[i];
                        {
                            const double2 r1 = c_ipow(v1, q1), r0 = c_ipow(v0, q0);
                            const double2 n0 = make_double2(cs.x * v0.x + cs.y * r1.x,
                                                            cs.x * v0.y + cs.y * r1.y);
                            v1 = make_double2(cs.x * v1.x + cs.y * r0.x, cs.x * v1.y + cs.y * r0.y);
                            v0 = n0;
                        }
                        if (NT == 2) {
                            const double2 r1 = c_ipow(w1, q1), r0 = c_ipow(w0, q0);
                            const double2 n0 = make_double2(cs.x * w0.x + cs.y * r1.x,
                                                            cs.x * w0.y + cs.y * r1.y);
                            w1 = make_double2(cs.x * w1.x + cs.y * r0.x, cs.x * w1.y + cs.y * r0.y);
                            w0 = n0;
                        }
                    }
                    t0[l0] = v0;
                    t0[l1] = v1;
                    if (NT == 2) {
                        t1[l0] = w0;
                        t1[l1] = w1;
                    }
                }
            }
        } else {
            for (int l = tid; l < T; l += nth) {
                double2 v = t0[l];
                double2 wv = (NT == 2) ? t1[l] : make_double2(0.0, 0.0);
                if (want_ip) {
                    double2 k = make_double2(0.0, 0.0);
                    for (int i = w.s0; i < w.s0 + w.ns; ++i) {
                        const int q = (s_q[i] + 2 * parity64((uint64_t)l & s_zl[i])) & 3;
                        const double2 r = c_ipow(v, q);
                        k.x += s_sc[i] * r.x;
                        k.y += s_sc[i] * r.y;
                    }
                    ip = c_add(ip, c_cjmul(wv, k));
                }
                if (w.rotate) {
                    for (int i = w.s0; i < w.s0 + w.ns; ++i) {
                        const int q = (s_q[i] + 2 * parity64((uint64_t)l & s_zl[i])) & 3;
                        const double2 cs = s_cs[i];
                        const double2 r = c_ipow(v, q);
                        v = make_double2(cs.x * v.x + cs.y * r.x, cs.x * v.y + cs.y * r.y);
                        if (NT == 2) {
                            const double2 rw = c_ipow(wv, q);
                            wv = make_double2(cs.x * wv.x + cs.y * rw.x, cs.x * wv.y + cs.y * rw.y);
                        }
                    }
                    t0[l] = v;
                    if (NT == 2) t1[l] = wv;
                }
            }
        }
        if (want_ip) {
            ip = warp_sum(ip);
            if (lane == 0) s_ipw[(st & 1) * kWinWarps + warp] = ip;
            pend_row = w.ip_row;
        }
        __syncthreads();
    }
    if (pend_row >= 0 && warp == 0) {
        double2 v = (lane < nwarps) ? s_ipw[((a.nsteps - 1) & 1) * kWinWarps + lane]
                                    : make_double2(0.0, 0.0);
        v = warp_sum(v);
        if (lane == 0) a.partial[((uint64_t)pend_row * gridDim.y + slot) * a.ntiles + tile] = v;
    }

    for (int l = tid; l < T; l += nth) {
        const uint64_t g = base | s_tab[l >> a.L] | ((uint64_t)l & lowm);
        P[g] = t0[l];
        if (NT == 2) S[g] = t1[l];
    }
}

}  // namespace qfbw
