// libqfb.so core: library plumbing, state lifecycle, gate application,
// scale / axpy / inner products.
//
// Gate semantics follow Computer::apply_1qubit_gate (computer.cc:340-425) and
// Computer::apply_2qubit_gate (computer.cc:458-751) case by case, including
// the reference's quirks, so a circuit gives the reference's amplitudes:
//   * a 2x2 block with only off-diagonal entries that compare equal is applied
//     as X (`op_0_1 == op_1_0 == 1.0`, computer.cc:398, :548, :669);
//   * a 2-qubit matrix with m00 == m11 == 1 and |m01| + |m10| < 1e-16 is
//     applied as a controlled 2x2 block on the control = 1 half, ignoring any
//     other entry outside that block (computer.cc:469-719);
//   * any other 2-qubit matrix is applied in full, each output accumulated
//     over the 4 inputs in column order, entries with |m| <= 1e-16 skipped
//     (computer.cc:721-750).
// The classification is made once per gate on the host; each kernel then
// touches only the amplitudes its case changes (a diagonal gate with one
// entry equal to 1 reads and writes half the state, a controlled gate a
// quarter or half).
#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "qfb_common.cuh"
#include "qfb_dense.cuh"
#include "qfb_gatetile.cuh"

namespace qfb {

thread_local std::string t_last_error;
thread_local cudaStream_t t_stream = nullptr;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(e == cudaErrorMemoryAllocation ? QFB_ENOMEM : QFB_EDEVICE, "%s: %s (%s)", what,
                cudaGetErrorString(e), cudaGetErrorName(e));
}

static std::mutex g_pool_mu;
static bool g_pool_ready[64];

static void pool_init(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= 64 || g_pool_ready[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;  // keep freed blocks cached in this process
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_pool_ready[dev] = true;
}

int dev_alloc(void **p, size_t bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    pool_init(dev);
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, t_stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(QFB_ENOMEM, "device allocation of %zu bytes failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    return QFB_OK;
}

void dev_free(void *p) {
    if (p) cudaFreeAsync(p, t_stream);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (dev >= 0 && dev < 64) cached[dev] = n;
    return n;
}

}  // namespace qfb

using namespace qfb;

// ===========================================================================
// kernels
// ===========================================================================

namespace {

enum : int { K_DENSE = 0, K_DIAG = 1, K_SWAP = 2, K_ANTI = 3 };

struct Gate2 {  // a 2x2 block acting on target bit t, optionally where bit c == 1
    int kind;
    int t;
    int c;         // -1: no control
    int diag_set;  // K_DIAG: bit0 -> a != 1, bit1 -> d != 1
    double2 a, b, cc, d;
};

struct Gate4 {  // generic 2-qubit matrix
    int t, c;
    uint32_t nz;  // bit (4*i + j) set when |m[i][j]| > 1e-16
    double2 m[16];
};

template <class A = double2>
__global__ void k_gate2(A *__restrict__ psi, uint64_t nbasis, Gate2 g) {
    A *s = psi + (uint64_t)blockIdx.y * nbasis;
    const A ga = AmpT<A>::cvt(g.a), gb = AmpT<A>::cvt(g.b), gc = AmpT<A>::cvt(g.cc),
            gd = AmpT<A>::cvt(g.d);
    const uint64_t tbit = 1ull << g.t;
    const uint64_t npair = (g.c < 0) ? (nbasis >> 1) : (nbasis >> 2);
    const int lo = (g.c < 0) ? g.t : min(g.t, g.c);
    const int hi = (g.c < 0) ? -1 : max(g.t, g.c);
    const uint64_t cbit = (g.c < 0) ? 0ull : (1ull << g.c);
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npair;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i0 = insert0(p, lo);
        if (hi >= 0) i0 = insert0(i0, hi) | cbit;
        const uint64_t i1 = i0 | tbit;
        if (g.kind == K_DENSE) {
            const A x0 = s[i0], x1 = s[i1];
            s[i0] = c_add(c_mul(ga, x0), c_mul(gb, x1));
            s[i1] = c_add(c_mul(gc, x0), c_mul(gd, x1));
        } else if (g.kind == K_DIAG) {
            if (g.diag_set & 1) s[i0] = c_mul(ga, s[i0]);
            if (g.diag_set & 2) s[i1] = c_mul(gd, s[i1]);
        } else if (g.kind == K_SWAP) {
            const A x0 = s[i0], x1 = s[i1];
            s[i0] = x1;
            s[i1] = x0;
        } else {
            const A x0 = s[i0], x1 = s[i1];
            s[i0] = c_mul(gb, x1);
            s[i1] = c_mul(gc, x0);
        }
    }
}

template <class A = double2>
__global__ void k_gate4(A *__restrict__ psi, uint64_t nbasis, Gate4 g) {
    A *s = psi + (uint64_t)blockIdx.y * nbasis;
    const uint64_t tbit = 1ull << g.t, cbit = 1ull << g.c;
    const int lo = min(g.t, g.c), hi = max(g.t, g.c);
    const uint64_t nquad = nbasis >> 2;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nquad;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = insert0(insert0(p, lo), hi);
        uint64_t idx[4];
        idx[0] = base;
        idx[1] = base | tbit;
        idx[2] = base | cbit;
        idx[3] = base | cbit | tbit;
        A x[4], y[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) x[j] = s[idx[j]];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            A acc = AmpT<A>::make(0, 0);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (g.nz & (1u << (4 * i + j)))
                    acc = c_add(acc, c_mul(AmpT<A>::cvt(g.m[4 * i + j]), x[j]));
            y[i] = acc;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) s[idx[i]] = y[i];
    }
}

// ---------------------------------------------------------------------------
// Gate runs: a run of gates whose qubits all lie in one set Q of b qubits
// (always holding the lowest L >= 3 qubits) is applied to 2^b-amplitude tiles
// by k_gate_tile (qfb_gatetile.cuh): one read and one write of the state for
// the whole run.  WGate is a run's gate in tile coordinates, as the planner
// hands it to the phase planner.
// ---------------------------------------------------------------------------
enum : int { K_GEN = 4 };

struct WGate {
    int32_t kind;  // K_DENSE..K_ANTI: 2x2 block on t (where bit c is set, c >= 0); K_GEN: 4x4
    int32_t t, c;  // bit positions inside the tile
    int32_t diag_set;
    uint32_t nz;
    int32_t pad;
    double2 m[16];  // 2x2 kinds: a, b, c, d in m[0..3]
};

struct GWin {
    uint64_t qmask, cmask;
    int b, L, g0, ng;
};

__global__ void k_scale(double2 *__restrict__ psi, uint64_t n, double2 a) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        psi[i] = c_mul(psi[i], a);
}

__global__ void k_axpy(double2 *__restrict__ y, const double2 *__restrict__ x, uint64_t n,
                       double2 a) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = c_add(y[i], c_mul(a, x[i]));
}

__global__ void k_set_first(double2 *__restrict__ psi, uint64_t nbasis, int nbatch) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbatch) psi[(uint64_t)b * nbasis] = make_double2(1.0, 0.0);
}

__global__ void k_scatter(double2 *__restrict__ psi, const uint64_t *__restrict__ idx,
                          const double2 *__restrict__ val, int64_t n) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) psi[idx[k]] = val[k];
}

// partial[b * gridDim.x + blockIdx.x] = sum over this block's indices of conj(a) b
__global__ void k_vdot_partial(const double2 *__restrict__ a, const double2 *__restrict__ b,
                               uint64_t nbasis, double2 *__restrict__ partial) {
    const uint64_t off = (uint64_t)blockIdx.y * nbasis;
    double2 acc = make_double2(0.0, 0.0);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nbasis;
         i += (uint64_t)gridDim.x * blockDim.x)
        acc = c_add(acc, c_cjmul(a[off + i], b[off + i]));
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(uint64_t)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// out[r] = sum_{k < n} partial[r * n + k]  (one block per row, fixed order)
__global__ void k_rows_sum(const double2 *__restrict__ partial, int64_t n,
                           double2 *__restrict__ out) {
    const double2 *row = partial + (uint64_t)blockIdx.x * n;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) acc = c_add(acc, row[k]);
    acc = block_sum(acc);
    if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

// ---------------------------------------------------------------------------
// Sampling of basis states (Computer::measure_circuit / measure_readouts /
// measure_z_readouts_fast, computer.cc:135-315), seeded and reproducible:
//   weight w_i = trunc(|c_i|^2 * 2^56), |c_i|^2 = re*re + im*im rounded as
//     written (no fused multiply-add), so any implementation gets the same w;
//   T = sum of the weights (exact integer sums, any order);
//   draw k: u = mix64(seed + (k + 1) * 0x9E3779B97F4A7C15) (the SplitMix64
//     generator of Steele, Lea and Flood, finaliser constants of Vigna),
//     r = floor(u * T / 2^64);
//   sample = the smallest i whose inclusive prefix sum of weights exceeds r.
// Blocks of 4096 amplitudes, sub-blocks of 64: k_samp_weights forms each
// block's inclusive sub-block prefixes and total, k_samp_scan the inclusive
// prefixes of the block totals, k_samp_draw searches block, sub-block, then
// at most 64 amplitudes.
// ---------------------------------------------------------------------------
constexpr int kSampBlock = 4096, kSampSub = 64;

__device__ __forceinline__ uint64_t samp_weight(double2 c) {
    const double p = __dadd_rn(__dmul_rn(c.x, c.x), __dmul_rn(c.y, c.y));
    return (uint64_t)__double2ull_rz(__dmul_rn(p, 72057594037927936.0));  // 2^56
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// grid: blocks of 4096 amplitudes; 256 threads (8 warps), each warp sums 8 of
// the block's 64-amplitude sub-blocks with coalesced reads (two amplitudes a
// lane).  sub_incl[blk * 64 + j]: inclusive prefix of the block's sub-block
// sums; blk_tot[blk]: its total; blk_p[blk]: its sum of |c|^2 in double (the
// norm check).
__global__ void __launch_bounds__(256) k_samp_weights(const double2 *__restrict__ s, uint64_t n,
                                                      uint64_t *__restrict__ sub_incl,
                                                      uint64_t *__restrict__ blk_tot,
                                                      double *__restrict__ blk_p) {
    __shared__ uint64_t s_sub[kSampSub];
    __shared__ double s_p[kSampSub];
    const uint64_t base = (uint64_t)blockIdx.x * kSampBlock;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double2 c[2 * (kSampSub / 8)];
#pragma unroll
    for (int k = 0; k < kSampSub / 8; ++k) {  // all loads in flight first
        const uint64_t i0 = base + (uint64_t)(wid * (kSampSub / 8) + k) * kSampSub + lane;
        c[2 * k] = i0 < n ? s[i0] : make_double2(0.0, 0.0);
        c[2 * k + 1] = i0 + 32 < n ? s[i0 + 32] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int k = 0; k < kSampSub / 8; ++k) {
        uint64_t w = samp_weight(c[2 * k]) + samp_weight(c[2 * k + 1]);
        double pd = c[2 * k].x * c[2 * k].x + c[2 * k].y * c[2 * k].y + c[2 * k + 1].x * c[2 * k + 1].x +
                    c[2 * k + 1].y * c[2 * k + 1].y;
        for (int o = 16; o > 0; o >>= 1) {
            w += __shfl_down_sync(0xffffffffu, w, o);
            pd += __shfl_down_sync(0xffffffffu, pd, o);
        }
        if (lane == 0) {
            s_sub[wid * (kSampSub / 8) + k] = w;
            s_p[wid * (kSampSub / 8) + k] = pd;
        }
    }
    __syncthreads();
    if (tid == 0) {
        uint64_t acc = 0;
        double pa = 0.0;
        for (int j = 0; j < kSampSub; ++j) {
            acc += s_sub[j];
            pa += s_p[j];
            sub_incl[(uint64_t)blockIdx.x * kSampSub + j] = acc;
        }
        blk_tot[blockIdx.x] = acc;
        blk_p[blockIdx.x] = pa;
    }
}

// One CTA of 1024 threads: blk_incl = inclusive prefix of the block totals,
// *total = T, *bad = 1 when the sum of |c|^2 is 1.5 or more (weights could
// overflow 64 bits) or T is 0.
__global__ void __launch_bounds__(1024) k_samp_scan(const uint64_t *__restrict__ blk_tot,
                                                    const double *__restrict__ blk_p, int64_t nblk,
                                                    uint64_t *__restrict__ blk_incl,
                                                    uint64_t *__restrict__ total, int *__restrict__ bad) {
    __shared__ uint64_t s_w[32];
    __shared__ double s_d[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t per = (nblk + 1023) / 1024, b0 = (int64_t)tid * per,
                  b1 = b0 + per < nblk ? b0 + per : nblk;
    uint64_t mine = 0;
    double pd = 0.0;
    for (int64_t k = b0; k < b1; ++k) {
        mine += blk_tot[k];
        pd += blk_p[k];
    }
    // exclusive scan of the 1024 thread sums
    uint64_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    for (int o = 16; o > 0; o >>= 1) pd += __shfl_down_sync(0xffffffffu, pd, o);
    if (lane == 31) s_w[wid] = incl;
    if (lane == 0) s_d[wid] = pd;
    __syncthreads();
    if (wid == 0) {
        uint64_t x = s_w[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        s_w[lane] = x;  // inclusive over warps
    }
    __syncthreads();
    uint64_t acc = incl - mine + (wid > 0 ? s_w[wid - 1] : 0ull);
    for (int64_t k = b0; k < b1; ++k) {
        acc += blk_tot[k];
        blk_incl[k] = acc;
    }
    if (tid == 0) {
        double ps = 0.0;
        for (int k = 0; k < 32; ++k) ps += s_d[k];
        const uint64_t T = s_w[31];
        *total = T;
        *bad = (!(ps < 1.5) || T == 0) ? 1 : 0;
    }
}

// One thread per draw.
__global__ void k_samp_draw(const double2 *__restrict__ s, uint64_t n,
                            const uint64_t *__restrict__ sub_incl,
                            const uint64_t *__restrict__ blk_incl, int64_t nblk,
                            const uint64_t *__restrict__ total, const int *__restrict__ bad,
                            uint64_t seed, int64_t nshots, uint64_t *__restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nshots || *bad) return;
    const uint64_t T = *total;
    const uint64_t u = mix64(seed + (uint64_t)(k + 1) * 0x9E3779B97F4A7C15ull);
    uint64_t r = __umul64hi(u, T);
    // smallest block whose inclusive prefix exceeds r
    int64_t lo = 0, hi = nblk - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (blk_incl[mid] > r) hi = mid; else lo = mid + 1;
    }
    if (lo > 0) r -= blk_incl[lo - 1];
    const uint64_t *sub = sub_incl + (uint64_t)lo * kSampSub;
    int a = 0, c = kSampSub - 1;
    while (a < c) {
        const int mid = (a + c) >> 1;
        if (sub[mid] > r) c = mid; else a = mid + 1;
    }
    if (a > 0) r -= sub[a - 1];
    uint64_t i = (uint64_t)lo * kSampBlock + (uint64_t)a * kSampSub;
    const uint64_t iend = i + kSampSub < n ? i + kSampSub : n;
    uint64_t acc = 0;
    for (; i + 1 < iend; ++i) {
        acc += samp_weight(s[i]);
        if (acc > r) break;
    }
    out[k] = i;
}

inline double2 d2(const qfb_complex &c) { return make_double2(c.re, c.im); }
inline bool is_one(const qfb_complex &c) { return c.re == 1.0 && c.im == 0.0; }
inline bool ceq(const qfb_complex &a, const qfb_complex &b) {
    return a.re == b.re && a.im == b.im;
}
inline double cabs_h(const qfb_complex &c) { return std::hypot(c.re, c.im); }

constexpr double kThr = 1.0e-16;  // Computer::compute_threshold_ (computer.h:172)

// Classify a 2x2 block as computer.cc:353-423 does.
Gate2 classify2(const qfb_complex &a, const qfb_complex &b, const qfb_complex &c,
                const qfb_complex &d, int t, int ctrl) {
    Gate2 g;
    g.t = t;
    g.c = ctrl;
    g.a = d2(a);
    g.b = d2(b);
    g.cc = d2(c);
    g.d = d2(d);
    g.diag_set = 0;
    const bool has_diag = cabs_h(a) + cabs_h(d) > kThr;
    const bool has_off = cabs_h(b) + cabs_h(c) > kThr;
    if (has_diag && has_off) {
        g.kind = K_DENSE;
    } else if (has_diag) {
        g.kind = K_DIAG;
        g.diag_set = (is_one(a) ? 0 : 1) | (is_one(d) ? 0 : 2);
    } else {
        g.kind = ceq(b, c) ? K_SWAP : K_ANTI;
    }
    return g;
}

// One gate as the kernels apply it (classified once on the host).
struct HGate {
    int form;  // 0: Gate2 (1-qubit or controlled), 1: Gate4
    Gate2 g2;
    Gate4 g4;
    uint64_t qubits;
};

HGate classify_gate(const qfb_gate &g) {
    HGate h{};
    const auto &m = g.mat;
    h.qubits = (1ull << g.target) | (1ull << g.control);
    if (g.target == g.control) {
        h.form = 0;
        h.g2 = classify2(m[0][0], m[0][1], m[1][0], m[1][1], g.target, -1);
        return h;
    }
    const bool controlled =
        (cabs_h(m[0][1]) + cabs_h(m[1][0]) < kThr) && is_one(m[0][0]) && is_one(m[1][1]);
    if (controlled) {
        h.form = 0;
        h.g2 = classify2(m[2][2], m[2][3], m[3][2], m[3][3], g.target, g.control);
        return h;
    }
    h.form = 1;
    h.g4.t = g.target;
    h.g4.c = g.control;
    h.g4.nz = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            h.g4.m[4 * i + j] = d2(m[i][j]);
            if (cabs_h(m[i][j]) > kThr) h.g4.nz |= 1u << (4 * i + j);
        }
    return h;
}

// One full-state pass for one gate, on nbatch states of nbasis amplitudes.
template <class A>
int launch_single_t(A *d, uint64_t nbasis, int nbatch, const HGate &h) {
    const dim3 block(256);
    if (h.form == 0) {
        const uint64_t n = (h.g2.c < 0) ? (nbasis >> 1) : (nbasis >> 2);
        k_gate2<A><<<dim3(grid_for(n, 256), nbatch), block, 0, t_stream>>>(d, nbasis, h.g2);
    } else {
        k_gate4<A><<<dim3(grid_for(nbasis >> 2, 256), nbatch), block, 0, t_stream>>>(d, nbasis,
                                                                                      h.g4);
    }
    QFB_LAUNCHED();
    return QFB_OK;
}

int launch_single(qfb_state s, const HGate &h) { return launch_single_t(s->d, s->nbasis, s->nbatch, h); }

constexpr int kGateTileDefault = 10;  // 2^10 amplitudes = 18 KB of shared memory per tile
constexpr int kGateTileMax = 12;
int g_gate_tile_bits = 0;  // 0: kGateTileDefault; -1: one pass per gate
int g_gate_low_bits = 3;

int g_gate_reg_bits = 0;  // 0: default
// Form of the tile phases: 0 gate by gate; 1 fused (8 x 8 matrices on the
// FP64 tensor cores) where it applies; 2 (default) fused for states of at
// least kFusedMinBytes (larger than L2: below it the gate-by-gate form is
// faster, the tile traffic being L2-resident).
int g_gate_fused = 2;
constexpr uint64_t kFusedMinBytes = 1ull << 27;

// Register bits R of a tile of b qubits: 2^(b-R) threads (<= 256) hold 2^R
// amplitudes each.  Default 3 (8 amplitudes, 80 registers a thread, three
// CTAs an SM); qfb_gates_regs may ask for another value, clamped to the tile.
inline int tile_reg_bits(int b) {
    const int lo = std::max(2, b - 8), hi = std::min(qfbt::kMaxRegBits, std::max(2, b - 2));
    const int want = g_gate_reg_bits > 0 ? g_gate_reg_bits : 3;
    return std::min(hi, std::max(lo, want));
}

// Tile shape for an n-qubit state: false when every gate takes its own pass
// (tile_bits -1, or a state smaller than two 128-byte chunks).
bool gate_tile_shape(int n, int &b, int &L) {
    b = g_gate_tile_bits == 0 ? kGateTileDefault : g_gate_tile_bits;
    if (b < 0 || n < 4) return false;
    L = std::max(3, std::min(g_gate_low_bits, n));
    b = std::max(4, std::min(b, n));
    b = std::max(b, std::min(n, L + 2));  // room for any 2-qubit gate beside the low qubits
    return true;
}

// Shared memory of the fused-form tile kernel: the tile and barrier word
// (`plain` bytes), aligned to 16, then two thread-table buffers.
inline int fused_bytes(int plain) {
    return ((plain + 15) & ~15) + 2 * (1 << qfbt::kMaxThreadBits) * (int)sizeof(uint32_t);
}

int gate_tile_smem() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        auto bytes = [](int b) { return (int)(sizeof(double2) * qfbt::tpad_size(b) + 16); };
        auto bytes8 = [](int b) { return (int)(sizeof(float2) * qfbt::tpad8_size(b) + 16); };
        auto attr = [&](const void *f, int n) {
            if (err == cudaSuccess)
                err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, n);
        };
        attr((const void *)qfbt::k_gate_tile<2>, bytes(10));
        attr((const void *)qfbt::k_gate_tile<3>, bytes(11));
        attr((const void *)qfbt::k_gate_tile<4>, bytes(kGateTileMax));
        attr((const void *)qfbt::k_gate_tile<2, float2>, bytes8(10));
        attr((const void *)qfbt::k_gate_tile<3, float2>, bytes8(11));
        attr((const void *)qfbt::k_gate_tile<4, float2>, bytes8(kGateTileMax));
        attr((const void *)qfbt::k_gate_tile<3, double2, true>, fused_bytes(bytes(11)));
        attr((const void *)qfbt::k_gate_tile<3, float2, true>, fused_bytes(bytes8(11)));
    });
    return err == cudaSuccess ? QFB_OK : cuda_fail(err, "gate tile shared memory");
}

struct GatePlanWin {
    GWin w;
    int64_t single;  // >= 0: a window of one gate, applied by its own pass
};

// Greedy windows: scanning the unapplied gates in order, a gate joins the
// current window when no earlier unapplied gate shares one of its qubits
// (gates on disjoint qubits commute) and its qubits fit in the window's b
// qubits together with those already chosen; a gate that cannot join blocks
// its qubits for the rest of the scan.  The window's qubits always include
// the lowest L, and are filled up to b with the lowest unused ones.
void plan_gate_windows(const std::vector<HGate> &hg, int n, int b, int L,
                       std::vector<GatePlanWin> &wins, std::vector<WGate> &wg) {
    const int64_t N = (int64_t)hg.size();
    const uint64_t all = (n >= 64) ? ~0ull : (1ull << n) - 1ull;
    const uint64_t low = (1ull << L) - 1ull;
    std::vector<char> done((size_t)N, 0);
    int64_t first = 0;
    std::vector<int64_t> sel;
    while (first < N) {
        uint64_t Q = low, blocked = 0;
        sel.clear();
        int64_t scanned = 0;
        for (int64_t i = first; i < N && blocked != all && scanned < 16384; ++i) {
            if (done[i]) continue;
            ++scanned;
            const uint64_t gm = hg[i].qubits;
            if (gm & blocked) {
                blocked |= gm;
                continue;
            }
            const uint64_t nq = Q | gm;
            if (__builtin_popcountll(nq) <= b) {
                Q = nq;
                sel.push_back(i);
                done[i] = 1;
            } else {
                blocked |= gm;
            }
        }
        if (sel.empty()) {
            // the first unapplied gate fits no tile of this shape: its own pass
            sel.push_back(first);
            done[first] = 1;
        }
        while (first < N && done[first]) ++first;
        GatePlanWin pw{};
        if (sel.size() == 1) {
            pw.single = sel[0];
            wins.push_back(pw);
            continue;
        }
        for (int q = 0; q < n && __builtin_popcountll(Q) < b; ++q) Q |= 1ull << q;
        auto loc = [&](int q) { return __builtin_popcountll(Q & ((1ull << q) - 1ull)); };
        pw.single = -1;
        pw.w.qmask = Q;
        pw.w.cmask = all & ~Q;
        pw.w.b = b;
        pw.w.L = L;
        pw.w.g0 = (int)wg.size();
        pw.w.ng = (int)sel.size();
        for (int64_t i : sel) {
            const HGate &h = hg[i];
            WGate w{};
            if (h.form == 0) {
                w.kind = h.g2.kind;
                w.t = loc(h.g2.t);
                w.c = h.g2.c < 0 ? -1 : loc(h.g2.c);
                w.diag_set = h.g2.diag_set;
                w.m[0] = h.g2.a;
                w.m[1] = h.g2.b;
                w.m[2] = h.g2.cc;
                w.m[3] = h.g2.d;
            } else {
                w.kind = K_GEN;
                w.t = loc(h.g4.t);
                w.c = loc(h.g4.c);
                w.nz = h.g4.nz;
                for (int k = 0; k < 16; ++k) w.m[k] = h.g4.m[k];
            }
            wg.push_back(w);
        }
        wins.push_back(pw);
    }
}

struct TilePlan {
    std::vector<qfbt::TPhase> ph;
    std::vector<qfbt::TOp> ops;
    std::vector<double2> m4;
    std::vector<uint64_t> chunks;   // per run: global offset of each 8-amplitude chunk
    std::vector<uint32_t> threads;  // per phase: tl | tpad(tl) << 16 of each thread
    std::vector<qfbt::TSeg> segs;   // fused form: segments of the phases
    std::vector<double2> fm;        // fused form: segment matrices, per-thread factors
};

// The bits of v, lowest first, placed on the set bits of m.
uint64_t deposit_host(uint64_t v, uint64_t m) {
    uint64_t r = 0;
    for (; m; m &= m - 1, v >>= 1)
        if (v & 1ull) r |= m & (~m + 1);
    return r;
}

// The 4x4 matrix of SWAP exactly (unit entries at (0,0), (1,2), (2,1), (3,3)).
bool is_swap4(const WGate &g) {
    const uint32_t want = (1u << 0) | (1u << 6) | (1u << 9) | (1u << 15);
    if (g.nz != want) return false;
    for (int e : {0, 6, 9, 15})
        if (g.m[e].x != 1.0 || g.m[e].y != 0.0) return false;
    return true;
}

// ---- the fused form of a phase ----------------------------------------------

inline double2 cmul_h(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
inline double2 cadd_h(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// One op of a phase on the 2^R registers of the thread with tile bits tl,
// exactly as qfbt::apply_op applies it.
void top_apply_host(const qfbt::TOp &o, const double2 *m4, uint32_t tl, int R, double2 *v) {
    if ((tl & o.tctl) != o.tctl) return;
    const uint32_t NR = 1u << R, cm = o.aux & 0xffu, cv = (o.aux >> 16) & 0xffu;
    const uint32_t opc = o.opc;
    if (opc < qfbt::OPC_DIAG) {
        const uint32_t kind = opc / 4, tb = 1u << (opc % 4);
        for (uint32_t k = 0; k < NR; ++k) {
            if ((k & tb) || (k & cm) != cv) continue;
            const double2 x0 = v[k], x1 = v[k | tb];
            if (kind == qfbt::OP_PSWAP) {
                v[k] = x1;
                v[k | tb] = x0;
            } else if (kind == qfbt::OP_ANTI) {
                v[k] = cmul_h(o.m[1], x1);
                v[k | tb] = cmul_h(o.m[2], x0);
            } else {
                v[k] = cadd_h(cmul_h(o.m[0], x0), cmul_h(o.m[1], x1));
                v[k | tb] = cadd_h(cmul_h(o.m[2], x0), cmul_h(o.m[3], x1));
            }
        }
    } else if (opc < qfbt::OPC_DIAG_THREAD) {
        const uint32_t dset = (opc - qfbt::OPC_DIAG) / 4 + 1, tb = 1u << ((opc - qfbt::OPC_DIAG) % 4);
        for (uint32_t k = 0; k < NR; ++k) {
            if ((k & cm) != cv) continue;
            if (k & tb) {
                if (dset & 2u) v[k] = cmul_h(o.m[3], v[k]);
            } else if (dset & 1u) {
                v[k] = cmul_h(o.m[0], v[k]);
            }
        }
    } else if (opc == qfbt::OPC_DIAG_THREAD) {
        const bool one = (tl & o.tbit) != 0;
        if (!(((o.aux >> 8) & 3u) & (one ? 2u : 1u))) return;
        const double2 f = o.m[one ? 3 : 0];
        for (uint32_t k = 0; k < NR; ++k)
            if ((k & cm) == cv) v[k] = cmul_h(f, v[k]);
    } else if (opc < qfbt::OPC_BSWAP) {
        const uint32_t tb = 1u << ((opc - qfbt::OPC_GEN4) / 4), cb = 1u << ((opc - qfbt::OPC_GEN4) % 4);
        const double2 *m = m4 + o.aux;
        for (uint32_t k = 0; k < NR; ++k) {
            if (k & (tb | cb)) continue;
            const uint32_t idx[4] = {k, k | tb, k | cb, k | tb | cb};
            double2 y[4];
            for (int i = 0; i < 4; ++i) {
                double2 acc = make_double2(0.0, 0.0);
                for (int j = 0; j < 4; ++j) acc = cadd_h(acc, cmul_h(m[4 * i + j], v[idx[j]]));
                y[i] = acc;
            }
            for (int i = 0; i < 4; ++i) v[idx[i]] = y[i];
        }
    } else {
        const uint32_t tb = 1u << ((opc - qfbt::OPC_BSWAP) / 4), cb = 1u << ((opc - qfbt::OPC_BSWAP) % 4);
        for (uint32_t k = 0; k < NR; ++k)
            if ((k & tb) && !(k & cb)) std::swap(v[k], v[k ^ tb ^ cb]);
    }
}

// The fused form of phase ph (R = 3, 2^(b-3) >= 32 threads; its
// ops already in tp.ops), appended to tp.ph: segments of consecutive ops with
// at most kMaxVarBits variant bits, each an 8 x 8 matrix per variant in
// A-fragment order, and the per-vector product of the factors that depend on
// thread bits alone.  Consecutive segments share a phase while the union of
// their variant bits fits in the vector-index bits above the three lowest
// (n-block and warp bits) and their matrices in one staging buffer (kStage
// entries); otherwise the phase is split into phases on the same registers,
// each with its own thread table: all but the last store to the load
// offsets, the next loads them again.
void fuse_phase(TilePlan &tp, const qfbt::TPhase &ph, int b, bool c64) {
    constexpr int R = 3;
    auto toff = [c64](uint32_t l) { return c64 ? qfbt::tpad8(l) : qfbt::tpad(l); };
    constexpr uint32_t NR = 8;
    const uint32_t nth = 1u << (b - R);
    const int nvb = b - R - 3;  // vector-index bits above the n-block columns
    // a segment's variant bits must all fit there (8-qubit tiles have 2)
    const int maxv = std::min(qfbt::kMaxVarBits, nvb);
    // the register bits' tile bits (loads): register position j <-> roff[1 << j]
    int rbit[R];
    uint32_t S = 0;
    for (int j = 0; j < R; ++j) {
        rbit[j] = 0;
        for (int p = 0; p < b; ++p)
            if (toff(1u << p) == ph.roff[1 << j]) rbit[j] = p;
        S |= 1u << rbit[j];
    }
    const uint32_t T = ((1u << b) - 1u) & ~S;  // thread bits
    std::vector<int> run_ops;
    std::vector<qfbt::TOp> fac_ops;
    std::vector<double2> col(NR), mat;
    struct Seg {
        uint32_t D;  // variant bits
        qfbt::TSeg h;
    };
    std::vector<Seg> segs;
    std::vector<double2> mats;
    auto flush = [&](uint32_t D) {
        if (run_ops.empty()) return;
        std::vector<int> dbits;
        for (int p = 0; p < 16; ++p)
            if (D >> p & 1u) dbits.push_back(p);
        const uint32_t nvar = 1u << dbits.size();
        Seg sg{};
        sg.D = D;
        sg.h.m0 = (uint32_t)mats.size();
        sg.h.nd = (uint32_t)dbits.size();
        for (size_t j = 0; j < dbits.size(); ++j) sg.h.dsel |= (uint32_t)dbits[j] << (4 * j);
        mat.assign((size_t)NR * NR, make_double2(0.0, 0.0));
        for (uint32_t x = 0; x < nvar; ++x) {
            uint32_t tl = 0;
            for (size_t j = 0; j < dbits.size(); ++j)
                if (x >> j & 1u) tl |= 1u << dbits[j];
            for (uint32_t c = 0; c < NR; ++c) {
                std::fill(col.begin(), col.end(), make_double2(0.0, 0.0));
                col[c] = make_double2(1.0, 0.0);
                for (int oi : run_ops) top_apply_host(tp.ops[oi], tp.m4.data(), tl, R, col.data());
                for (uint32_t r = 0; r < NR; ++r) {
                    mat[r * NR + c] = col[r];
                    if (col[r].x != 0.0 || col[r].y != 0.0) sg.h.mm |= r ^ c;
                }
            }
            for (uint32_t kb = 0; kb < 2; ++kb)
                for (uint32_t lane = 0; lane < 32; ++lane)
                    mats.push_back(mat[(lane >> 2) * NR + 4 * kb + (lane & 3)]);

        }
        segs.push_back(sg);
        run_ops.clear();
    };
    uint32_t D = 0;
    for (int oi = ph.o0; oi < ph.o0 + ph.no; ++oi) {
        const qfbt::TOp &o = tp.ops[oi];
        if (o.opc == qfbt::OPC_DIAG_THREAD && (o.aux & 0xffu) == 0) {  // thread bits alone
            fac_ops.push_back(o);
            continue;
        }
        const uint32_t need = o.tctl | (o.opc == qfbt::OPC_DIAG_THREAD ? o.tbit : 0u);
        if (__builtin_popcount(D | need) > maxv) {
            flush(D);
            D = 0;
        }
        D |= need;
        run_ops.push_back(oi);
    }
    flush(D);
    // thread table of a phase with variant bits Dv: vector-index bits 0-2 from
    // the other thread bits, chosen by residue class (tile bit mod 3) so the
    // quarter-warp accesses of the B and D fragments spread over the banks;
    // then Dv; then the rest
    auto table = [&](uint32_t Dv) {
        const int c0 = rbit[0] % 3, c1 = rbit[1] % 3, c2 = 3 - c0 - c1;
        const int want[3] = {c2 >= 0 && c2 < 3 && c2 != c0 && c2 != c1 ? c2 : -1, c1, c2};
        uint32_t free_bits = T & ~Dv;
        std::vector<int> tb;
        for (int w : want) {
            int pick = -1;
            for (int p = 0; p < b && pick < 0; ++p)
                if ((free_bits >> p & 1u) && (w < 0 || p % 3 == w)) pick = p;
            for (int p = 0; p < b && pick < 0; ++p)
                if (free_bits >> p & 1u) pick = p;
            tb.push_back(pick);
            free_bits &= ~(1u << pick);
        }
        for (int p = 0; p < b; ++p)
            if (Dv >> p & 1u) tb.push_back(p);
        for (int p = 0; p < b; ++p)
            if (free_bits >> p & 1u) tb.push_back(p);
        const int th0 = (int)tp.threads.size();
        for (uint32_t t = 0; t < nth; ++t) {
            uint32_t tl = 0;
            for (size_t j = 0; j < tb.size(); ++j)
                if (t >> j & 1u) tl |= 1u << tb[j];
            tp.threads.push_back(tl | (toff(tl) << 16));
        }
        return th0;
    };
    // group the segments into phases
    size_t i = 0;
    bool first = true;
    do {
        qfbt::TPhase q = ph;
        uint32_t Dv = 0;
        size_t j = i;
        const uint32_t base = i < segs.size() ? segs[i].h.m0 : 0u;
        while (j < segs.size()) {
            const uint32_t end = j + 1 < segs.size() ? segs[j + 1].h.m0 : (uint32_t)mats.size();
            if (j > i && (end - base > (uint32_t)qfbt::kStage ||
                          __builtin_popcount(Dv | segs[j].D) > nvb))
                break;
            Dv |= segs[j].D;
            ++j;
        }
        q.th0 = table(Dv);
        q.s0 = (int)tp.segs.size();
        q.m0 = (int)tp.fm.size();
        for (size_t k = i; k < j; ++k) {
            qfbt::TSeg h = segs[k].h;
            h.m0 = (uint32_t)q.m0 + (h.m0 - base);
            tp.segs.push_back(h);
        }
        const uint32_t end = j < segs.size() ? segs[j].h.m0 : (uint32_t)mats.size();
        tp.fm.insert(tp.fm.end(), mats.begin() + base, mats.begin() + end);
        q.ns = (int)(j - i);
        q.nm = (int)(end - base);
        q.sc = -1;
        if (first && !fac_ops.empty()) {
            q.sc = (int)tp.fm.size();
            for (uint32_t t = 0; t < nth; ++t) {
                double2 f = make_double2(1.0, 0.0);
                const uint32_t tl = tp.threads[q.th0 + t] & 0xffffu;
                for (const qfbt::TOp &o : fac_ops) top_apply_host(o, tp.m4.data(), tl, 0, &f);
                tp.fm.push_back(f);
            }
        }
        if (j < segs.size())  // more segments follow on the same registers
            std::memcpy(q.soff, q.roff, sizeof(q.roff));
        tp.ph.push_back(q);
        i = j;
        first = false;
    } while (i < segs.size());
}

// Split a run's gates (tile coordinates) into phases of R register bits.
// Scanning the unplaced gates in order, a gate joins the current phase when
// no earlier unplaced gate shares one of its tile bits and its mixing bits
// fit in the phase's R register bits together with those already chosen; a
// gate that cannot join blocks its bits for the rest of the scan, so only
// gates on disjoint qubits change order.
// c64: shared offsets in the complex64 tile layout (qfbt::tpad8).
// fused: the phases' fused form where it applies (R = 3, at least 32
// threads).
void plan_tile_phases(const WGate *g, int ng, int b, int R, qfbt::TRun &run, TilePlan &tp,
                      bool c64 = false, bool fused = false) {
    auto toff = [c64](uint32_t l) { return c64 ? qfbt::tpad8(l) : qfbt::tpad(l); };
    std::vector<uint32_t> mix((size_t)ng), qm((size_t)ng);
    for (int i = 0; i < ng; ++i) {
        const WGate &w = g[i];
        if (w.kind == K_GEN) {
            qm[i] = mix[i] = (1u << w.t) | (1u << w.c);
        } else {
            qm[i] = (1u << w.t) | (w.c >= 0 ? 1u << w.c : 0u);
            mix[i] = (w.kind == K_DIAG) ? 0u : (1u << w.t);
        }
    }
    const uint32_t all = (1u << b) - 1u;
    std::vector<char> done((size_t)ng, 0);
    std::vector<int> sel;
    int first = 0;
    run.p0 = (int)tp.ph.size();
    while (first < ng) {
        uint32_t S = 0, blocked = 0;
        sel.clear();
        for (int i = first; i < ng; ++i) {
            if (done[i]) continue;
            if (qm[i] & blocked) {
                blocked |= qm[i];
                continue;
            }
            if (__builtin_popcount(S | mix[i]) <= R) {
                S |= mix[i];
                sel.push_back(i);
                done[i] = 1;
            } else {
                blocked |= qm[i];
            }
        }
        while (first < ng && done[first]) ++first;
        // complete S to R bits, each filler from the residue class (tile bit
        // mod 3) that keeps the most bits among the thread bits
        while (__builtin_popcount(S) < R) {
            int best = -1, bestn = -1;
            for (int p = b - 1; p >= 0; --p) {
                if (S >> p & 1u) continue;
                int cnt = 0;
                for (int q = 0; q < b; ++q)
                    if (!(S >> q & 1u) && q % 3 == p % 3) ++cnt;
                if (cnt > bestn) {
                    bestn = cnt;
                    best = p;
                }
            }
            S |= 1u << best;
        }
        // thread bits; the three lowest (a quarter warp) from distinct classes
        const uint32_t T = all & ~S;
        std::vector<int> tb;
        for (int cls = 0; cls < 3; ++cls)
            for (int p = 0; p < b; ++p)
                if ((T >> p & 1u) && p % 3 == cls) {
                    tb.push_back(p);
                    break;
                }
        for (int p = 0; p < b; ++p)
            if ((T >> p & 1u) && std::find(tb.begin(), tb.end(), p) == tb.end()) tb.push_back(p);
        qfbt::TPhase ph{};
        // physical register position of each tile bit in S, and whether its
        // register bit holds the complement of the tile bit: uncontrolled
        // exchanges on a register bit (X) and SWAPs of two register bits are
        // relabelings, applied here instead of on the device
        int pos[32], flip[32];
        for (int p = 0, k = 0; p < b; ++p) {
            pos[p] = (S >> p & 1u) ? k++ : -1;
            flip[p] = 0;
        }
        for (int k = 0; k < (1 << R); ++k) {
            uint32_t l = 0;
            for (int p = 0; p < b; ++p)
                if (pos[p] >= 0 && (k >> pos[p] & 1)) l |= 1u << p;
            ph.roff[k] = toff(l);
        }
        ph.th0 = (int)tp.threads.size();
        for (uint32_t tid = 0; tid < (1u << (b - R)); ++tid) {
            uint32_t tl = 0;
            for (size_t j = 0; j < tb.size(); ++j)
                if (tid >> j & 1u) tl |= 1u << tb[j];
            tp.threads.push_back(tl | (toff(tl) << 16));
        }
        ph.o0 = (int)tp.ops.size();
        auto swap2 = [](double2 &x, double2 &y) {
            const double2 t = x;
            x = y;
            y = t;
        };
        for (int i : sel) {
            const WGate &w = g[i];
            if (w.kind == K_GEN && is_swap4(w)) {
                std::swap(pos[w.t], pos[w.c]);
                std::swap(flip[w.t], flip[w.c]);
                continue;
            }
            if (w.kind == K_SWAP && w.c < 0) {
                flip[w.t] ^= 1;
                continue;
            }
            qfbt::TOp o{};
            uint32_t opc = 0;
            if (w.kind == K_GEN) {
                opc = qfbt::OPC_GEN4 + (uint32_t)(4 * pos[w.t] + pos[w.c]);
                const int fm = flip[w.t] | (flip[w.c] << 1);
                o.aux = (uint32_t)tp.m4.size();
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c) {
                        const int k = 4 * (r ^ fm) + (c ^ fm);
                        tp.m4.push_back((w.nz >> k & 1u) ? w.m[k] : make_double2(0.0, 0.0));
                    }
            } else {
                uint32_t cm = 0, cv = 0;
                if (w.c >= 0) {
                    if (S >> w.c & 1u) {  // control on a register bit
                        cm = 1u << pos[w.c];
                        cv = flip[w.c] ? 0u : cm;
                    } else {  // control on one of the thread's bits
                        o.tctl = 1u << w.c;
                    }
                }
                double2 a = w.m[0], bb = w.m[1], cc = w.m[2], d = w.m[3];
                const bool fl = (S >> w.t & 1u) && flip[w.t];
                if (fl) {  // the register bit holds the complement: conjugate by X
                    swap2(a, d);
                    swap2(bb, cc);
                }
                o.m[0] = a;
                o.m[1] = bb;
                o.m[2] = cc;
                o.m[3] = d;
                if (w.kind == K_DIAG) {
                    uint32_t dset = (uint32_t)w.diag_set;
                    if (fl) dset = ((dset & 1u) << 1) | ((dset >> 1) & 1u);
                    if (dset == 0) continue;  // identity: no arithmetic
                    if (S >> w.t & 1u) {
                        opc = qfbt::OPC_DIAG + 4u * (dset - 1u) + (uint32_t)pos[w.t];
                        o.aux = cm | (cv << 16);
                    } else {
                        opc = qfbt::OPC_DIAG_THREAD;
                        o.tbit = 1u << w.t;
                        o.aux = cm | (dset << 8) | (cv << 16);
                    }
                } else {
                    uint32_t kind;
                    if (w.kind == K_SWAP)
                        kind = qfbt::OP_PSWAP;
                    else if (w.kind == K_ANTI)
                        kind = qfbt::OP_ANTI;
                    else if (a.y == 0.0 && bb.y == 0.0 && cc.y == 0.0 && d.y == 0.0)
                        kind = qfbt::OP_REAL;
                    else if (a.y == 0.0 && d.y == 0.0 && bb.x == 0.0 && cc.x == 0.0)
                        kind = qfbt::OP_RXI;
                    else
                        kind = qfbt::OP_DENSE;
                    opc = 4u * kind + (uint32_t)pos[w.t];
                    o.aux = cm | (cv << 16);
                }
            }
            o.opc = opc;
            tp.ops.push_back(o);
        }
        // store offsets: physical register k holds, for each tile bit p of S,
        // the value (bit pos[p] of k) ^ flip[p]
        for (int k = 0; k < (1 << R); ++k) {
            uint32_t l = 0;
            for (int p = 0; p < b; ++p)
                if (pos[p] >= 0 && (((k >> pos[p]) & 1) ^ flip[p])) l |= 1u << p;
            ph.soff[k] = toff(l);
        }
        ph.no = (int)tp.ops.size() - ph.o0;
        if (fused && R == 3 && b - R >= 5)
            fuse_phase(tp, ph, b, c64);
        else
            tp.ph.push_back(ph);
    }
    run.np = (int)tp.ph.size() - run.p0;
    run.b = b;
}

// ---------------------------------------------------------------------------
// Dense blocks (FP64 tensor cores): runs of gates on at most K qubits fused
// into one 2^K x 2^K unitary each.
// ---------------------------------------------------------------------------

int g_gate_dense = 0;  // 0: off; 5 or 6: runs of gates become dense K-qubit blocks

// A gate (tile coordinates) on one vector of 2^K amplitudes, as k_gate2 /
// k_gate4 apply it (the case analysis of computer.cc:340-751).
void wgate_apply_host(const WGate &w, double2 *v, int K) {
    auto mul = [](double2 a, double2 b) {
        return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    };
    auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
    const uint32_t R = 1u << K, tb = 1u << w.t;
    if (w.kind == K_GEN) {
        const uint32_t cb = 1u << w.c;
        for (uint32_t i = 0; i < R; ++i) {
            if (i & (tb | cb)) continue;
            const uint32_t idx[4] = {i, i | tb, i | cb, i | cb | tb};
            double2 x[4], y[4];
            for (int j = 0; j < 4; ++j) x[j] = v[idx[j]];
            for (int r = 0; r < 4; ++r) {
                double2 acc = make_double2(0.0, 0.0);
                for (int j = 0; j < 4; ++j)
                    if (w.nz & (1u << (4 * r + j))) acc = add(acc, mul(w.m[4 * r + j], x[j]));
                y[r] = acc;
            }
            for (int r = 0; r < 4; ++r) v[idx[r]] = y[r];
        }
        return;
    }
    const uint32_t cb = w.c < 0 ? 0u : (1u << w.c);
    for (uint32_t i = 0; i < R; ++i) {
        if ((i & tb) || (i & cb) != cb) continue;
        const uint32_t i1 = i | tb;
        const double2 x0 = v[i], x1 = v[i1];
        switch (w.kind) {
            case K_DENSE:
                v[i] = add(mul(w.m[0], x0), mul(w.m[1], x1));
                v[i1] = add(mul(w.m[2], x0), mul(w.m[3], x1));
                break;
            case K_DIAG:
                if (w.diag_set & 1) v[i] = mul(w.m[0], x0);
                if (w.diag_set & 2) v[i1] = mul(w.m[3], x1);
                break;
            case K_SWAP:
                v[i] = x1;
                v[i1] = x0;
                break;
            default:
                v[i] = mul(w.m[1], x1);
                v[i1] = mul(w.m[2], x0);
                break;
        }
    }
}

// The run's unitary, appended to `out` as a real plane then an imaginary
// plane, row-major (row r, column s: the amplitude of block index r that
// block index s becomes): each gate applied in order to every column of the
// identity.
void dense_unitary(const WGate *g, int ng, int K, std::vector<double> &out) {
    const size_t R = (size_t)1 << K;
    std::vector<double2> col(R);
    const size_t o = out.size();
    out.resize(o + 2 * R * R);
    for (size_t s = 0; s < R; ++s) {
        std::fill(col.begin(), col.end(), make_double2(0.0, 0.0));
        col[s] = make_double2(1.0, 0.0);
        for (int i = 0; i < ng; ++i) wgate_apply_host(g[i], col.data(), K);
        for (size_t r = 0; r < R; ++r) {
            out[o + r * R + s] = col[r].x;
            out[o + R * R + r * R + s] = col[r].y;
        }
    }
}

// The dense pass of a window on block qubits S (|S| = K): tiles over S and
// the lowest 10 - K other qubits.
qfbd::DRun dense_run(uint64_t smask, int n) {
    uint64_t q = smask;
    for (int b = 0; b < n && __builtin_popcountll(q) < qfbd::kTileBits; ++b) q |= 1ull << b;
    qfbd::DRun r{};
    r.qmask = q;
    uint32_t k = 0;
    for (uint64_t m = q; m; m &= m - 1, ++k)
        if (smask & (m & (~m + 1ull))) r.sbits |= 1u << k;
    r.ntiles = (1ull << n) >> qfbd::kTileBits;
    return r;
}

// Resident CTAs of the dense kernel for block size K, times the SMs.
int dense_grid(int K, unsigned &grid) {
    static std::once_flag once;
    static int per_sm[2] = {0, 0};
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm[0], qfbd::k_dense_block<5>, qfbd::Shape<5>::THREADS,
            2 * sizeof(double2) * qfbd::Shape<5>::BUF);
        if (err == cudaSuccess)
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm[1], qfbd::k_dense_block<6>, qfbd::Shape<6>::THREADS,
                2 * sizeof(double2) * qfbd::Shape<6>::BUF);
    });
    if (err != cudaSuccess) return cuda_fail(err, "dense block occupancy");
    grid = (unsigned)std::max(1, per_sm[K - 5]) * (unsigned)sm_count();
    return QFB_OK;
}

// Apply a gate list with dense blocks: windows of at most K qubits (the
// greedy scan of plan_gate_windows, no forced low qubits) fused into one
// unitary each; a window of one gate takes its own one-gate pass.
int apply_gates_dense(qfb_state s, const std::vector<HGate> &hg, int K) {
    const int n = s->nqubit;
    std::vector<GatePlanWin> wins;
    std::vector<WGate> wg;
    plan_gate_windows(hg, n, K, 0, wins, wg);
    std::vector<double> us;
    for (const GatePlanWin &pw : wins)
        if (pw.single < 0) dense_unitary(wg.data() + pw.w.g0, pw.w.ng, K, us);
    void *buf = nullptr;
    if (!us.empty()) {
        int rc = dev_alloc(&buf, sizeof(double) * us.size());
        if (rc) return rc;
        QFB_CUDA(cudaMemcpyAsync(buf, us.data(), sizeof(double) * us.size(),
                                 cudaMemcpyHostToDevice, t_stream));
    }
    unsigned cap = 0;
    int rc = dense_grid(K, cap);
    const size_t per_u = (size_t)2 << (2 * K);
    size_t ui = 0;
    for (size_t i = 0; i < wins.size() && rc == QFB_OK; ++i) {
        const GatePlanWin &pw = wins[i];
        if (pw.single >= 0) {
            rc = launch_single(s, hg[pw.single]);
            continue;
        }
        const qfbd::DRun run = dense_run(pw.w.qmask, n);
        const double *U = (const double *)buf + per_u * ui++;
        const uint64_t total = run.ntiles * (uint64_t)s->nbatch;
        const unsigned grid = (unsigned)std::min<uint64_t>(total, cap);
        if (K == 5) {
            qfbd::k_dense_block<5><<<grid, qfbd::Shape<5>::THREADS,
                                     2 * sizeof(double2) * qfbd::Shape<5>::BUF, t_stream>>>(
                s->d, s->nbasis, s->nbatch, run, U);
        } else {
            qfbd::k_dense_block<6><<<grid, qfbd::Shape<6>::THREADS,
                                     2 * sizeof(double2) * qfbd::Shape<6>::BUF, t_stream>>>(
                s->d, s->nbasis, s->nbatch, run, U);
        }
        rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    }
    if (buf) dev_free(buf);
    return rc;
}

// Runs of a gate list and the phases of each run.
void plan_gate_tiles(const std::vector<HGate> &hg, int n, int b, int L,
                     std::vector<GatePlanWin> &wins, TilePlan &tp, std::vector<qfbt::TRun> &runs,
                     bool c64 = false, bool fused = false) {
    std::vector<WGate> wg;
    plan_gate_windows(hg, n, b, L, wins, wg);
    runs.assign(wins.size(), qfbt::TRun{});
    for (size_t i = 0; i < wins.size(); ++i) {
        const GatePlanWin &pw = wins[i];
        if (pw.single >= 0) continue;
        qfbt::TRun &r = runs[i];
        r.qmask = pw.w.qmask;
        r.ch0 = (int)tp.chunks.size();
        for (uint64_t c = 0; c < (1ull << (pw.w.b - 3)); ++c)
            tp.chunks.push_back(deposit_host(c, pw.w.qmask & ~7ull));
        plan_tile_phases(wg.data() + pw.w.g0, pw.w.ng, pw.w.b, tile_reg_bits(pw.w.b), r, tp, c64,
                         fused);
    }
}

// Bounds-check and classify a gate list for an nqubit state.
int classify_gates(const qfb_gate *gates, int64_t ngates, int nqubit, const char *fn,
                   std::vector<HGate> &hg) {
    if (ngates < 0 || (ngates > 0 && !gates)) return fail(QFB_EINVAL, "%s: bad gate array", fn);
    for (int64_t k = 0; k < ngates; ++k) {
        const qfb_gate &g = gates[k];
        if (g.target < 0 || g.target >= nqubit || g.control < 0 || g.control >= nqubit)
            return fail(QFB_EINVAL, "%s: gate %lld acts on qubit (%d, %d) of a %d-qubit state", fn,
                        (long long)k, g.target, g.control, nqubit);
    }
    hg.resize((size_t)ngates);
    for (int64_t k = 0; k < ngates; ++k) hg[(size_t)k] = classify_gate(gates[k]);
    return QFB_OK;
}

// Apply classified gates to nbatch states of 2^n amplitudes of A (double2, or
// float2 for the complex64 variant): register-blocked tile runs, one pass per
// gate where a gate joins no run (or the tile shape says so).
template <class A>
int apply_gates_tiles(A *d, int n, int nbatch, const std::vector<HGate> &hg) {
    const uint64_t nbasis = 1ull << n;
    int b = 0, L = 0;
    if (!gate_tile_shape(n, b, L) || hg.size() == 1) {
        for (const HGate &h : hg) {
            const int rc = launch_single_t(d, nbasis, nbatch, h);
            if (rc) return rc;
        }
        return QFB_OK;
    }
    constexpr bool c64 = sizeof(A) == sizeof(float2);
    std::vector<GatePlanWin> wins;
    TilePlan tp;
    std::vector<qfbt::TRun> runs;
    const bool fused = g_gate_fused == 1 ||
                       (g_gate_fused == 2 && sizeof(A) * nbasis * (uint64_t)nbatch >= kFusedMinBytes);
    plan_gate_tiles(hg, n, b, L, wins, tp, runs, c64, fused);
    // one upload of phases, ops, 4x4 matrices, chunk and thread tables and
    // the fused form
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t bp = al(sizeof(qfbt::TPhase) * tp.ph.size());
    const size_t bo = al(sizeof(qfbt::TOp) * tp.ops.size());
    const size_t bm = al(sizeof(double2) * tp.m4.size());
    const size_t bc = al(sizeof(uint64_t) * tp.chunks.size());
    const size_t bt = al(sizeof(uint32_t) * tp.threads.size());
    const size_t bs = al(sizeof(qfbt::TSeg) * tp.segs.size());
    const size_t bf = sizeof(double2) * tp.fm.size();
    void *buf = nullptr;
    if (!tp.ph.empty()) {
        std::vector<unsigned char> host(bp + bo + bm + bc + bt + bs + bf);
        auto put = [&](size_t off, const void *src, size_t sz) {
            if (sz) std::memcpy(host.data() + off, src, sz);
        };
        put(0, tp.ph.data(), sizeof(qfbt::TPhase) * tp.ph.size());
        put(bp, tp.ops.data(), sizeof(qfbt::TOp) * tp.ops.size());
        put(bp + bo, tp.m4.data(), sizeof(double2) * tp.m4.size());
        put(bp + bo + bm, tp.chunks.data(), sizeof(uint64_t) * tp.chunks.size());
        put(bp + bo + bm + bc, tp.threads.data(), sizeof(uint32_t) * tp.threads.size());
        put(bp + bo + bm + bc + bt, tp.segs.data(), sizeof(qfbt::TSeg) * tp.segs.size());
        put(bp + bo + bm + bc + bt + bs, tp.fm.data(), bf);
        int rc = dev_alloc(&buf, host.size());
        if (rc) return rc;
        QFB_CUDA(cudaMemcpyAsync(buf, host.data(), host.size(), cudaMemcpyHostToDevice, t_stream));
    }
    unsigned char *ub = (unsigned char *)buf;
    const qfbt::TPhase *d_ph = (const qfbt::TPhase *)ub;
    const qfbt::TOp *d_ops = (const qfbt::TOp *)(ub + bp);
    const double2 *d_m4 = (const double2 *)(ub + bp + bo);
    const uint64_t *d_ch = (const uint64_t *)(ub + bp + bo + bm);
    const uint32_t *d_th = (const uint32_t *)(ub + bp + bo + bm + bc);
    const qfbt::TSeg *d_sg = (const qfbt::TSeg *)(ub + bp + bo + bm + bc + bt);
    const double2 *d_fm = (const double2 *)(ub + bp + bo + bm + bc + bt + bs);
    int rc = gate_tile_smem();
    for (size_t i = 0; i < wins.size() && rc == QFB_OK; ++i) {
        const GatePlanWin &pw = wins[i];
        if (pw.single >= 0) {
            rc = launch_single_t(d, nbasis, nbatch, hg[pw.single]);
            continue;
        }
        const int tb = pw.w.b, R = tile_reg_bits(tb);
        const size_t smem0 = sizeof(A) * qfbt::tpad_size_of<A>(tb) + 16;
        const bool fz = fused && R == 3 && tb - R >= 5;
        const size_t smem = fz ? (size_t)fused_bytes((int)smem0) : smem0;
        const dim3 grid((unsigned)(nbasis >> tb), nbatch), block(1u << (tb - R));
#define QFB_TILE(RR, FF)                                                                        \
    qfbt::k_gate_tile<RR, A, FF><<<grid, block, smem, t_stream>>>(d, nbasis, runs[i], d_ph, d_ops, \
                                                                  d_m4, d_ch, d_th, d_sg, d_fm)
        if (R == 2)
            QFB_TILE(2, false);
        else if (R == 3 && fz)
            QFB_TILE(3, true);
        else if (R == 3)
            QFB_TILE(3, false);
        else
            QFB_TILE(4, false);
#undef QFB_TILE
        rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    }
    dev_free(buf);
    return rc;
}

// Sum of |amplitude|^2 of a complex64 state, accumulated in FP64.
__global__ void k_norm2_c64(const float2 *__restrict__ psi, uint64_t n, double2 *__restrict__ part) {
    double acc = 0.0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float2 v = psi[i];
        acc += (double)v.x * v.x + (double)v.y * v.y;
    }
    const double2 t = block_sum(make_double2(acc, 0.0));
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int qfb_version(void) { return 10000; }

int qfb_last_error(char *buf, size_t len) {
    if (!buf || !len) return QFB_EINVAL;
    std::strncpy(buf, t_last_error.c_str(), len - 1);
    buf[len - 1] = '\0';
    return QFB_OK;
}

int qfb_set_stream(void *stream) {
    t_stream = (cudaStream_t)stream;
    return QFB_OK;
}

// After a stream synchronisation: report (and clear) a bounded device wait
// that gave up since the last check.
static int check_device_waits() {
    int v = 0;
    QFB_CUDA(cudaMemcpyFromSymbolAsync(&v, qfbt::g_tile_wait_err, sizeof(int), 0,
                                       cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    if (v == 0) return QFB_OK;
    const int zero = 0;
    QFB_CUDA(cudaMemcpyToSymbolAsync(qfbt::g_tile_wait_err, &zero, sizeof(int), 0,
                                     cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return fail(QFB_ETIMEDOUT, "a gate tile's bulk copies did not complete within the wait "
                               "limit; the state is not valid");
}

int qfb_sync(void) {
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return check_device_waits();
}

int qfb_set_tile_wait_limit(uint64_t ns) {
    if (ns > 60000000000ull)
        return fail(QFB_EINVAL, "qfb_set_tile_wait_limit: %llu ns is above the 60 s bound",
                    (unsigned long long)ns);
    QFB_CUDA(cudaMemcpyToSymbolAsync(qfbt::g_tile_wait_limit_ns, &ns, sizeof(ns), 0,
                                     cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_launch_count(uint64_t *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_launch_count: null output");
    *out = g_launches.load();
    return QFB_OK;
}

int qfb_state_create(int nqubit, int nbatch, qfb_state *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_state_create: null output");
    *out = nullptr;
    if (nqubit < 1 || nqubit > 40)
        return fail(QFB_EINVAL, "qfb_state_create: nqubit = %d outside [1, 40]", nqubit);
    if (nbatch < 1) return fail(QFB_EINVAL, "qfb_state_create: nbatch = %d < 1", nbatch);
    qfb_state s = new qfb_state_s;
    s->nqubit = nqubit;
    s->nbatch = nbatch;
    s->nbasis = 1ull << nqubit;
    s->d = nullptr;
    int rc = dev_alloc((void **)&s->d, s->nbasis * (uint64_t)nbatch * sizeof(double2));
    if (rc) {
        delete s;
        return rc;
    }
    rc = qfb_state_reset(s);
    if (rc) {
        qfb_state_destroy(s);
        return rc;
    }
    *out = s;
    return QFB_OK;
}

int qfb_state_destroy(qfb_state s) {
    if (!s) return QFB_OK;
    dev_free(s->d);
    delete s;
    return QFB_OK;
}

int qfb_state_info(qfb_state s, int *nqubit, int *nbatch) {
    if (!s) return fail(QFB_EINVAL, "qfb_state_info: null state");
    if (nqubit) *nqubit = s->nqubit;
    if (nbatch) *nbatch = s->nbatch;
    return QFB_OK;
}

void *qfb_state_device_ptr(qfb_state s) { return s ? (void *)s->d : nullptr; }

int qfb_state_copy(qfb_state dst, qfb_state src) {
    if (!dst || !src) return fail(QFB_EINVAL, "qfb_state_copy: null state");
    if (dst->nqubit != src->nqubit || dst->nbatch != src->nbatch)
        return fail(QFB_EINVAL, "qfb_state_copy: shape mismatch (%d q x %d vs %d q x %d)",
                    dst->nqubit, dst->nbatch, src->nqubit, src->nbatch);
    if (dst == src) return QFB_OK;
    QFB_CUDA(cudaMemcpyAsync(dst->d, src->d, src->nbasis * src->nbatch * sizeof(double2),
                             cudaMemcpyDeviceToDevice, t_stream));
    return QFB_OK;
}

int qfb_state_copy_slot(qfb_state dst, int db, qfb_state src, int sb) {
    if (!dst || !src) return fail(QFB_EINVAL, "qfb_state_copy_slot: null state");
    if (dst->nqubit != src->nqubit)
        return fail(QFB_EINVAL, "qfb_state_copy_slot: qubit counts differ (%d vs %d)",
                    dst->nqubit, src->nqubit);
    if (db < 0 || db >= dst->nbatch || sb < 0 || sb >= src->nbatch)
        return fail(QFB_EINVAL, "qfb_state_copy_slot: slot out of range");
    QFB_CUDA(cudaMemcpyAsync(dst->d + (uint64_t)db * dst->nbasis,
                             src->d + (uint64_t)sb * src->nbasis, src->nbasis * sizeof(double2),
                             cudaMemcpyDeviceToDevice, t_stream));
    return QFB_OK;
}

int qfb_state_null(qfb_state s) {
    if (!s) return fail(QFB_EINVAL, "qfb_state_null: null state");
    QFB_CUDA(cudaMemsetAsync(s->d, 0, s->nbasis * s->nbatch * sizeof(double2), t_stream));
    return QFB_OK;
}

int qfb_state_reset(qfb_state s) {
    int rc = qfb_state_null(s);
    if (rc) return rc;
    k_set_first<<<(s->nbatch + 127) / 128, 128, 0, t_stream>>>(s->d, s->nbasis, s->nbatch);
    QFB_LAUNCHED();
    return QFB_OK;
}

int qfb_state_set_basis(qfb_state s, int b, const uint64_t *index, const qfb_complex *value,
                        int64_t n) {
    if (!s) return fail(QFB_EINVAL, "qfb_state_set_basis: null state");
    if (b < 0 || b >= s->nbatch) return fail(QFB_EINVAL, "qfb_state_set_basis: bad slot %d", b);
    if (n < 0 || (n > 0 && (!index || !value)))
        return fail(QFB_EINVAL, "qfb_state_set_basis: bad arrays");
    for (int64_t k = 0; k < n; ++k)
        if (index[k] >= s->nbasis)
            return fail(QFB_EINVAL, "qfb_state_set_basis: index %llu outside the %d-qubit basis",
                        (unsigned long long)index[k], s->nqubit);
    double2 *slot = s->d + (uint64_t)b * s->nbasis;
    QFB_CUDA(cudaMemsetAsync(slot, 0, s->nbasis * sizeof(double2), t_stream));
    if (n == 0) return QFB_OK;
    // a repeated index keeps its last value, as the reference's loop does
    std::vector<uint64_t> uidx;
    std::vector<double2> uval;
    {
        std::unordered_map<uint64_t, size_t> pos;
        for (int64_t k = 0; k < n; ++k) {
            auto it = pos.find(index[k]);
            if (it == pos.end()) {
                pos.emplace(index[k], uidx.size());
                uidx.push_back(index[k]);
                uval.push_back(d2(value[k]));
            } else {
                uval[it->second] = d2(value[k]);
            }
        }
    }
    const int64_t cnt = (int64_t)uidx.size();
    void *buf = nullptr;
    // the value array starts on a 256-byte boundary (double2 needs 16)
    const size_t ibytes = ((size_t)cnt * sizeof(uint64_t) + 255) & ~(size_t)255;
    int rc = dev_alloc(&buf, ibytes + (size_t)cnt * sizeof(double2));
    if (rc) return rc;
    uint64_t *d_idx = (uint64_t *)buf;
    double2 *d_val = (double2 *)((char *)buf + ibytes);
    QFB_CUDA(cudaMemcpyAsync(d_idx, uidx.data(), cnt * sizeof(uint64_t), cudaMemcpyHostToDevice,
                             t_stream));
    QFB_CUDA(cudaMemcpyAsync(d_val, uval.data(), cnt * sizeof(double2), cudaMemcpyHostToDevice,
                             t_stream));
    k_scatter<<<(unsigned)((cnt + 255) / 256), 256, 0, t_stream>>>(slot, d_idx, d_val, cnt);
    QFB_LAUNCHED();
    dev_free(buf);
    return QFB_OK;
}

int qfb_state_upload(qfb_state s, int b, const qfb_complex *host, uint64_t n) {
    if (!s || !host) return fail(QFB_EINVAL, "qfb_state_upload: null argument");
    if (b < 0 || b >= s->nbatch) return fail(QFB_EINVAL, "qfb_state_upload: bad slot %d", b);
    if (n != s->nbasis)
        return fail(QFB_EINVAL, "qfb_state_upload: %llu amplitudes given, state holds %llu",
                    (unsigned long long)n, (unsigned long long)s->nbasis);
    QFB_CUDA(cudaMemcpyAsync(s->d + (uint64_t)b * s->nbasis, host, n * sizeof(double2),
                             cudaMemcpyHostToDevice, t_stream));
    return QFB_OK;
}

int qfb_state_download(qfb_state s, int b, qfb_complex *host, uint64_t n) {
    if (!s || !host) return fail(QFB_EINVAL, "qfb_state_download: null argument");
    if (b < 0 || b >= s->nbatch) return fail(QFB_EINVAL, "qfb_state_download: bad slot %d", b);
    if (n != s->nbasis)
        return fail(QFB_EINVAL, "qfb_state_download: buffer of %llu for a state of %llu",
                    (unsigned long long)n, (unsigned long long)s->nbasis);
    QFB_CUDA(cudaMemcpyAsync(host, s->d + (uint64_t)b * s->nbasis, n * sizeof(double2),
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return check_device_waits();
}

int qfb_state_get_amp(qfb_state s, int b, uint64_t index, qfb_complex *out) {
    if (!s || !out) return fail(QFB_EINVAL, "qfb_state_get_amp: null argument");
    if (b < 0 || b >= s->nbatch || index >= s->nbasis)
        return fail(QFB_EINVAL, "qfb_state_get_amp: index out of range");
    QFB_CUDA(cudaMemcpyAsync(out, s->d + (uint64_t)b * s->nbasis + index, sizeof(double2),
                             cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_gates_config(int tile_bits, int low_bits) {
    if (low_bits < 0 || low_bits > 6)
        return fail(QFB_EINVAL, "qfb_gates_config: low_bits = %d outside [0, 6]", low_bits);
    if (tile_bits != -1 && tile_bits != 0 && (tile_bits < low_bits + 2 || tile_bits > kGateTileMax))
        return fail(QFB_EINVAL, "qfb_gates_config: tile_bits = %d outside [%d, %d]", tile_bits,
                    low_bits + 2, kGateTileMax);
    g_gate_tile_bits = tile_bits;
    g_gate_low_bits = low_bits;
    return QFB_OK;
}

int qfb_gates_dense(int k) {
    if (k != 0 && k != 5 && k != 6)
        return fail(QFB_EINVAL, "qfb_gates_dense: k = %d is not 0, 5 or 6", k);
    g_gate_dense = k;
    return QFB_OK;
}

int qfb_gates_fused(int mode) {
    if (mode < 0 || mode > 2) return fail(QFB_EINVAL, "qfb_gates_fused: %d is not 0, 1 or 2", mode);
    g_gate_fused = mode;
    return QFB_OK;
}

int qfb_gates_regs(int reg_bits) {
    if (reg_bits < 0 || reg_bits > qfbt::kMaxRegBits)
        return fail(QFB_EINVAL, "qfb_gates_regs: reg_bits = %d outside [0, %d]", reg_bits,
                    qfbt::kMaxRegBits);
    g_gate_reg_bits = reg_bits;
    return QFB_OK;
}

int qfb_gates_plan(const qfb_gate *gates, int64_t ngates, int nqubit, int64_t *windows,
                   int64_t *single_passes, double *pass_bytes) {
    if (ngates < 0 || (ngates > 0 && !gates) || nqubit < 1 || nqubit > 40)
        return fail(QFB_EINVAL, "qfb_gates_plan: bad arguments");
    std::vector<HGate> hg((size_t)ngates);
    for (int64_t k = 0; k < ngates; ++k) {
        const qfb_gate &g = gates[k];
        if (g.target < 0 || g.target >= nqubit || g.control < 0 || g.control >= nqubit)
            return fail(QFB_EINVAL, "qfb_gates_plan: gate %lld acts beyond qubit %d",
                        (long long)k, nqubit);
        hg[k] = classify_gate(g);
    }
    const double full = 32.0 * (double)(1ull << nqubit);
    // amplitudes a one-gate pass reads and writes (16 bytes each way)
    auto single_bytes = [&](const HGate &h) {
        if (h.form == 1) return full;
        double f = (h.g2.c < 0) ? 1.0 : 0.5;
        if (h.g2.kind == K_DIAG && h.g2.diag_set != 3) f *= (h.g2.diag_set == 0) ? 0.0 : 0.5;
        return f * full;
    };
    int64_t nw = 0, ns = 0;
    double bytes = 0.0;
    int b = 0, L = 0;
    const bool dense = g_gate_dense > 0 && nqubit >= qfbd::kTileBits && ngates > 1;
    if (!dense && (!gate_tile_shape(nqubit, b, L) || ngates == 1)) {
        for (const HGate &h : hg) bytes += single_bytes(h);
        ns = ngates;
    } else {
        std::vector<GatePlanWin> wins;
        std::vector<WGate> wg;
        if (dense)
            plan_gate_windows(hg, nqubit, g_gate_dense, 0, wins, wg);
        else
            plan_gate_windows(hg, nqubit, b, L, wins, wg);
        for (const GatePlanWin &pw : wins) {
            if (pw.single >= 0) {
                ++ns;
                bytes += single_bytes(hg[pw.single]);
            } else {
                ++nw;
                bytes += full;
            }
        }
    }
    if (windows) *windows = nw;
    if (single_passes) *single_passes = ns;
    if (pass_bytes) *pass_bytes = bytes;
    return QFB_OK;
}

int qfb_gates_phases(const qfb_gate *gates, int64_t ngates, int nqubit, int64_t *phases,
                     int64_t *ops) {
    if (ngates < 0 || (ngates > 0 && !gates) || nqubit < 1 || nqubit > 40)
        return fail(QFB_EINVAL, "qfb_gates_phases: bad arguments");
    std::vector<HGate> hg((size_t)ngates);
    for (int64_t k = 0; k < ngates; ++k) {
        const qfb_gate &g = gates[k];
        if (g.target < 0 || g.target >= nqubit || g.control < 0 || g.control >= nqubit)
            return fail(QFB_EINVAL, "qfb_gates_phases: gate %lld acts beyond qubit %d",
                        (long long)k, nqubit);
        hg[k] = classify_gate(g);
    }
    int b = 0, L = 0;
    int64_t np = 0, no = 0;
    if (gate_tile_shape(nqubit, b, L) && ngates > 1) {
        std::vector<GatePlanWin> wins;
        TilePlan tp;
        std::vector<qfbt::TRun> runs;
        plan_gate_tiles(hg, nqubit, b, L, wins, tp, runs);
        np = (int64_t)tp.ph.size();
        no = (int64_t)tp.ops.size();
    }
    if (phases) *phases = np;
    if (ops) *ops = no;
    return QFB_OK;
}

int qfb_gates_fused_plan(const qfb_gate *gates, int64_t ngates, int nqubit, int complex64,
                         int64_t *phases, int64_t *segments, int64_t *entries) {
    if (ngates < 0 || (ngates > 0 && !gates) || nqubit < 1 || nqubit > 40)
        return fail(QFB_EINVAL, "qfb_gates_fused_plan: bad arguments");
    std::vector<HGate> hg((size_t)ngates);
    for (int64_t k = 0; k < ngates; ++k) {
        const qfb_gate &g = gates[k];
        if (g.target < 0 || g.target >= nqubit || g.control < 0 || g.control >= nqubit)
            return fail(QFB_EINVAL, "qfb_gates_fused_plan: gate %lld acts beyond qubit %d",
                        (long long)k, nqubit);
        hg[k] = classify_gate(g);
    }
    int b = 0, L = 0;
    int64_t np = 0, ns = 0, ne = 0;
    const bool c64 = complex64 != 0;
    auto toff = [c64](uint32_t l) { return c64 ? qfbt::tpad8(l) : qfbt::tpad(l); };
    if (gate_tile_shape(nqubit, b, L) && ngates > 1) {
        std::vector<GatePlanWin> wins;
        TilePlan tp;
        std::vector<qfbt::TRun> runs;
        plan_gate_tiles(hg, nqubit, b, L, wins, tp, runs, c64, true);
        for (size_t w = 0; w < wins.size(); ++w) {
            if (wins[w].single >= 0) continue;
            const qfbt::TRun &r = runs[w];
            const int R = tile_reg_bits(r.b);
            if (!(R == 3 && r.b - R >= 5)) continue;  // this run keeps the gate-by-gate form
            const uint32_t nth = 1u << (r.b - R), all = (1u << r.b) - 1u;
            for (int p = r.p0; p < r.p0 + r.np; ++p) {
                const qfbt::TPhase &ph = tp.ph[(size_t)p];
                uint32_t S = 0;  // the register bits
                for (int k = 1; k < 8; k <<= 1)
                    for (int q = 0; q < r.b; ++q)
                        if (toff(1u << q) == ph.roff[k]) S |= 1u << q;
                // the thread table: a permutation of the thread-bit assignments
                std::vector<char> seen((size_t)1 << r.b, 0);
                for (uint32_t t = 0; t < nth; ++t) {
                    const uint32_t e = tp.threads[(size_t)ph.th0 + t], tl = e & 0xffffu;
                    if ((tl & ~(all & ~S)) || (e >> 16) != toff(tl) || seen[tl])
                        return fail(QFB_EINVAL, "qfb_gates_fused_plan: bad thread table (phase %d)", p);
                    seen[tl] = 1;
                }
                if (ph.nm > qfbt::kStage || ph.m0 < 0 || (size_t)ph.m0 + (size_t)ph.nm > tp.fm.size() ||
                    (ph.sc >= 0 && (size_t)ph.sc + nth > tp.fm.size()))
                    return fail(QFB_EINVAL, "qfb_gates_fused_plan: matrices out of range (phase %d)", p);
                for (int s = ph.s0; s < ph.s0 + ph.ns; ++s) {
                    const qfbt::TSeg &sg = tp.segs[(size_t)s];
                    uint32_t vm = 0;
                    for (uint32_t j = 0; j < sg.nd; ++j) vm |= 1u << ((sg.dsel >> (4 * j)) & 15u);
                    if ((vm & ~(all & ~S)) || sg.nd > (uint32_t)qfbt::kMaxVarBits ||
                        (int64_t)sg.m0 < ph.m0 || (size_t)sg.m0 + 64u * (1u << sg.nd) > (size_t)ph.m0 + ph.nm)
                        return fail(QFB_EINVAL, "qfb_gates_fused_plan: bad segment %d", s);
                    // the 8 vectors of an n-block share the variant bits
                    for (uint32_t t = 0; t < nth; ++t)
                        if (((tp.threads[(size_t)ph.th0 + t] ^ tp.threads[(size_t)ph.th0 + (t & ~7u)]) & vm) != 0)
                            return fail(QFB_EINVAL, "qfb_gates_fused_plan: variant splits an n-block (segment %d)", s);
                }
                ++np;
                ns += ph.ns;
                ne += ph.nm;
            }
        }
    }
    if (phases) *phases = np;
    if (segments) *segments = ns;
    if (entries) *entries = ne;
    return QFB_OK;
}

int qfb_apply_gates(qfb_state s, const qfb_gate *gates, int64_t ngates) {
    if (!s) return fail(QFB_EINVAL, "qfb_apply_gates: null state");
    std::vector<HGate> hg;
    int rc = classify_gates(gates, ngates, s->nqubit, "qfb_apply_gates", hg);
    if (rc || ngates == 0) return rc;
    const int n = s->nqubit;
    if (g_gate_dense > 0 && n >= qfbd::kTileBits && ngates > 1)
        return apply_gates_dense(s, hg, g_gate_dense);
    return apply_gates_tiles<double2>(s->d, n, s->nbatch, hg);
}

// ---- complex64 states: the throughput-only variant of the gate path ---------

struct qfb_state_c64_s {
    int nqubit;
    uint64_t nbasis;
    float2 *d;
};

int qfb_c64_create(int nqubit, qfb_state_c64 *out) {
    if (!out) return fail(QFB_EINVAL, "qfb_c64_create: null output");
    *out = nullptr;
    if (nqubit < 1 || nqubit > 40)
        return fail(QFB_EINVAL, "qfb_c64_create: nqubit = %d outside [1, 40]", nqubit);
    auto s = std::make_unique<qfb_state_c64_s>();
    s->nqubit = nqubit;
    s->nbasis = 1ull << nqubit;
    s->d = nullptr;
    int rc = dev_alloc((void **)&s->d, s->nbasis * sizeof(float2));
    if (rc) return rc;
    qfb_state_c64 h = s.release();
    rc = qfb_c64_reset(h);
    if (rc) {
        qfb_c64_destroy(h);
        return rc;
    }
    *out = h;
    return QFB_OK;
}

int qfb_c64_destroy(qfb_state_c64 s) {
    if (!s) return QFB_OK;
    dev_free(s->d);
    delete s;
    return QFB_OK;
}

int qfb_c64_reset(qfb_state_c64 s) {
    if (!s) return fail(QFB_EINVAL, "qfb_c64_reset: null state");
    static const float one[2] = {1.0f, 0.0f};
    QFB_CUDA(cudaMemsetAsync(s->d, 0, s->nbasis * sizeof(float2), t_stream));
    QFB_CUDA(cudaMemcpyAsync(s->d, one, sizeof(float2), cudaMemcpyHostToDevice, t_stream));
    return QFB_OK;
}

int qfb_c64_upload(qfb_state_c64 s, const float *host, uint64_t n) {
    if (!s || !host) return fail(QFB_EINVAL, "qfb_c64_upload: null argument");
    if (n != s->nbasis)
        return fail(QFB_EINVAL, "qfb_c64_upload: %llu amplitudes for a state of %llu",
                    (unsigned long long)n, (unsigned long long)s->nbasis);
    QFB_CUDA(cudaMemcpyAsync(s->d, host, n * sizeof(float2), cudaMemcpyHostToDevice, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

int qfb_c64_download(qfb_state_c64 s, float *host, uint64_t n) {
    if (!s || !host) return fail(QFB_EINVAL, "qfb_c64_download: null argument");
    if (n != s->nbasis)
        return fail(QFB_EINVAL, "qfb_c64_download: buffer of %llu for a state of %llu",
                    (unsigned long long)n, (unsigned long long)s->nbasis);
    QFB_CUDA(cudaMemcpyAsync(host, s->d, n * sizeof(float2), cudaMemcpyDeviceToHost, t_stream));
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return check_device_waits();
}

int qfb_c64_apply_gates(qfb_state_c64 s, const qfb_gate *gates, int64_t ngates) {
    if (!s) return fail(QFB_EINVAL, "qfb_c64_apply_gates: null state");
    std::vector<HGate> hg;
    int rc = classify_gates(gates, ngates, s->nqubit, "qfb_c64_apply_gates", hg);
    if (rc || ngates == 0) return rc;
    return apply_gates_tiles<float2>(s->d, s->nqubit, 1, hg);
}

int qfb_c64_norm2(qfb_state_c64 s, double *out) {
    if (!s || !out) return fail(QFB_EINVAL, "qfb_c64_norm2: null argument");
    const unsigned nblk = grid_for(s->nbasis, 256, 2);
    void *buf = nullptr;
    int rc = dev_alloc(&buf, sizeof(double2) * ((size_t)nblk + 1));
    if (rc) return rc;
    double2 *part = (double2 *)buf, *res = part + nblk;
    k_norm2_c64<<<nblk, 256, 0, t_stream>>>(s->d, s->nbasis, part);
    rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    if (rc == QFB_OK) {
        k_rows_sum<<<1, 256, 0, t_stream>>>(part, nblk, res);
        rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    }
    double2 h = make_double2(0.0, 0.0);
    if (rc == QFB_OK) {
        const cudaError_t e = cudaMemcpyAsync(&h, res, sizeof(double2), cudaMemcpyDeviceToHost,
                                              t_stream);
        rc = e == cudaSuccess ? QFB_OK : cuda_fail(e, "qfb_c64_norm2");
    }
    if (rc == QFB_OK) {
        const cudaError_t e = cudaStreamSynchronize(t_stream);
        rc = e == cudaSuccess ? QFB_OK : cuda_fail(e, "qfb_c64_norm2");
    }
    dev_free(buf);
    if (rc == QFB_OK) *out = h.x;
    return rc;
}

int qfb_scale(qfb_state s, qfb_complex a) {
    if (!s) return fail(QFB_EINVAL, "qfb_scale: null state");
    const uint64_t n = s->nbasis * s->nbatch;
    k_scale<<<grid_for(n, 256), 256, 0, t_stream>>>(s->d, n, d2(a));
    QFB_LAUNCHED();
    return QFB_OK;
}

int qfb_axpy(qfb_state y, qfb_complex alpha, qfb_state x) {
    if (!y || !x) return fail(QFB_EINVAL, "qfb_axpy: null state");
    if (y->nqubit != x->nqubit || y->nbatch != x->nbatch)
        return fail(QFB_EINVAL, "qfb_axpy: shape mismatch");
    const uint64_t n = y->nbasis * y->nbatch;
    k_axpy<<<grid_for(n, 256), 256, 0, t_stream>>>(y->d, x->d, n, d2(alpha));
    QFB_LAUNCHED();
    return QFB_OK;
}

int qfb_state_sample(qfb_state s, int b, uint64_t seed, int64_t nshots, uint64_t *out) {
    if (!s || (nshots > 0 && !out)) return fail(QFB_EINVAL, "qfb_state_sample: null argument");
    if (b < 0 || b >= s->nbatch) return fail(QFB_EINVAL, "qfb_state_sample: bad slot %d", b);
    if (nshots < 0) return fail(QFB_EINVAL, "qfb_state_sample: nshots = %lld", (long long)nshots);
    if (nshots == 0) return QFB_OK;
    const uint64_t n = s->nbasis;
    const int64_t nblk = (int64_t)((n + kSampBlock - 1) / kSampBlock);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_sub = 0, o_tot = al(sizeof(uint64_t) * nblk * kSampSub),
                 o_p = o_tot + al(sizeof(uint64_t) * nblk), o_inc = o_p + al(sizeof(double) * nblk),
                 o_T = o_inc + al(sizeof(uint64_t) * nblk), o_bad = o_T + 256,
                 o_out = o_bad + 256, bytes = o_out + sizeof(uint64_t) * (size_t)nshots;
    void *buf = nullptr;
    int rc = dev_alloc(&buf, bytes);
    if (rc) return rc;
    char *p = (char *)buf;
    const double2 *st = s->d + (uint64_t)b * n;
    k_samp_weights<<<(unsigned)nblk, 256, 0, t_stream>>>(st, n, (uint64_t *)(p + o_sub),
                                                        (uint64_t *)(p + o_tot), (double *)(p + o_p));
    rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    if (rc == QFB_OK) {
        k_samp_scan<<<1, 1024, 0, t_stream>>>((const uint64_t *)(p + o_tot), (const double *)(p + o_p),
                                              nblk, (uint64_t *)(p + o_inc), (uint64_t *)(p + o_T),
                                              (int *)(p + o_bad));
        rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    }
    if (rc == QFB_OK) {
        k_samp_draw<<<(unsigned)((nshots + 255) / 256), 256, 0, t_stream>>>(
            st, n, (const uint64_t *)(p + o_sub), (const uint64_t *)(p + o_inc), nblk,
            (const uint64_t *)(p + o_T), (const int *)(p + o_bad), seed, nshots,
            (uint64_t *)(p + o_out));
        rc = [&]() -> int { QFB_LAUNCHED(); return QFB_OK; }();
    }
    int bad = 0;
    if (rc == QFB_OK) {
        cudaError_t e = cudaMemcpyAsync(&bad, p + o_bad, sizeof(int), cudaMemcpyDeviceToHost, t_stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out, p + o_out, sizeof(uint64_t) * (size_t)nshots,
                                cudaMemcpyDeviceToHost, t_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "qfb_state_sample");
    }
    dev_free(buf);
    if (rc) return rc;
    if (bad)
        return fail(QFB_EINVAL, "qfb_state_sample: the state's squared norm is 0 or 1.5 or more; "
                                "normalise it before sampling");
    return QFB_OK;
}

int qfb_vdot(qfb_state a, qfb_state b, qfb_complex *out) {
    if (!a || !b || !out) return fail(QFB_EINVAL, "qfb_vdot: null argument");
    if (a->nqubit != b->nqubit || a->nbatch != b->nbatch)
        return fail(QFB_EINVAL, "qfb_vdot: shape mismatch");
    const unsigned nblk = grid_for(a->nbasis, 256, 2);
    void *buf = nullptr;
    int rc = dev_alloc(&buf, sizeof(double2) * ((size_t)nblk + 1) * a->nbatch);
    if (rc) return rc;
    double2 *partial = (double2 *)buf;
    double2 *res = partial + (size_t)nblk * a->nbatch;
    k_vdot_partial<<<dim3(nblk, a->nbatch), 256, 0, t_stream>>>(a->d, b->d, a->nbasis, partial);
    QFB_LAUNCHED();
    k_rows_sum<<<a->nbatch, 256, 0, t_stream>>>(partial, nblk, res);
    QFB_LAUNCHED();
    QFB_CUDA(cudaMemcpyAsync(out, res, sizeof(double2) * a->nbatch, cudaMemcpyDeviceToHost,
                             t_stream));
    dev_free(buf);
    QFB_CUDA(cudaStreamSynchronize(t_stream));
    return QFB_OK;
}

}  // extern "C"
