// Dense fused-gate blocks on the FP64 tensor cores.
//
// A run of gates whose qubits all lie in a set S of K qubits (K = 5 or 6) is
// one 2^K x 2^K unitary U, formed on the host as the product of the gates'
// matrices (each as Computer::apply_gate applies it, computer.cc:340-751).
// One pass over the state applies U: the state is cut into tiles of 2^10
// amplitudes over the qubits Q = S + the lowest 10 - K other qubits; a tile is
// a 2^K x 2^(10-K) matrix T (row: the bits of S, column: the other bits of Q)
// and the pass computes T <- U T.  The complex product is four real products
// on mma.sync.m8n8k4 with FP64 operands (the only FP64 tensor-core form on
// sm_100a: tcgen05 has no FP64 kind):
//   Re T' = Re U Re T - Im U Im T,    Im T' = Re U Im T + Im U Re T.
// Each warp owns 8 rows of U, held as A fragments in registers for the whole
// (persistent) kernel; the B fragments come from the tile in shared memory.
// Tiles are staged with cp.async and double-buffered, so the next tile's
// loads are in flight while the current one is multiplied.
//
// Per amplitude a pass moves 32 bytes (read + write) and does 2^K complex
// multiply-adds (8 * 2^K flops): K = 5 is about balanced between HBM and the
// FP64 tensor pipe on B200, K = 6 is tensor-bound.
#pragma once

#include <cstdint>

namespace qfbd {

constexpr int kTileBits = 10;  // 2^10 amplitudes a tile

template <int K>
struct Shape {
    static constexpr int M = kTileBits - K;   // column bits
    static constexpr int ROWS = 1 << K;
    static constexpr int COLS = 1 << M;
    // row pitch in double2: +2 spreads the rows a quarter warp reads for one B
    // fragment (4 rows x 2 columns) over the 8 16-byte bank slots
    static constexpr int W = COLS + 2;
    static constexpr int THREADS = 4 * ROWS;  // ROWS / 8 warps of 8 rows each
    static constexpr int KSTEPS = ROWS / 4;   // k = 4 per mma
    static constexpr int CB = COLS / 8;       // 8-column blocks per tile
    static constexpr int BUF = ROWS * W;      // double2 per tile buffer
    static constexpr int PER = (1 << kTileBits) / THREADS;  // amplitudes a thread moves
};

// One dense pass: the tile's qubits Q, which of Q's 10 bits (in ascending
// order) are the block's, and the tiles per state.
struct DRun {
    uint64_t qmask;
    uint32_t sbits;
    uint32_t pad;
    uint64_t ntiles;
};

// D += A B on one 8x8x4 FP64 block (pure register arithmetic: no volatile, so
// the compiler may interleave independent accumulators).
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t d_smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The bits of v, lowest first, placed on the set bits of m.
__device__ __forceinline__ uint64_t d_deposit(uint64_t v, uint64_t m) {
    uint64_t r = 0;
    for (; m; m &= m - 1, v >>= 1)
        if (v & 1ull) r |= m & (~m + 1ull);
    return r;
}

// The bits of v at the set bits of m, packed lowest first.
__device__ __forceinline__ uint32_t d_extract(uint32_t v, uint32_t m) {
    uint32_t r = 0;
    for (int k = 0; m; m &= m - 1, ++k)
        if (v & m & (~m + 1u)) r |= 1u << k;
    return r;
}

// v with a zero bit inserted at every set bit of m (ascending).
__device__ __forceinline__ uint64_t d_spread(uint64_t v, uint64_t m) {
    while (m) {
        const int p = __ffsll((long long)m) - 1;
        const uint64_t lo = v & ((1ull << p) - 1ull);
        v = ((v >> p) << (p + 1)) | lo;
        m &= m - 1;
    }
    return v;
}

// U: [2][ROWS][ROWS] doubles, the real plane then the imaginary one (row r,
// column s: the amplitude of block index r after the run from block index s).
// Tile index l has its bits on Q's qubits in ascending order: its amplitude
// sits deposit(l, Q) past the tile's origin, and in shared memory at row
// (l's block bits) and column (l's other bits).  Grid: persistent CTAs over
// ntiles * nbatch tiles.
template <int K>
__global__ void __launch_bounds__(Shape<K>::THREADS) k_dense_block(
    double2 *__restrict__ psi, uint64_t nbasis, int nbatch, DRun run, const double *__restrict__ U) {
    using S = Shape<K>;
    extern __shared__ __align__(16) unsigned char d_raw[];
    double2 *buf0 = reinterpret_cast<double2 *>(d_raw);
    double2 *buf1 = buf0 + S::BUF;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q = lane & 3;

    // A fragments of this warp's 8 rows of U: row 8 warp + g, column 4 j + q
    double ar[S::KSTEPS], ai[S::KSTEPS];
    const double *ur = U + (size_t)(8 * warp + g) * S::ROWS + q;
#pragma unroll
    for (int j = 0; j < S::KSTEPS; ++j) {
        ar[j] = __ldg(ur + 4 * j);
        ai[j] = __ldg(ur + S::ROWS * S::ROWS + 4 * j);
    }
    uint64_t go[S::PER];
    uint32_t so[S::PER];
    const uint32_t cbits = ((1u << kTileBits) - 1u) & ~run.sbits;
#pragma unroll
    for (int p = 0; p < S::PER; ++p) {
        const uint32_t l = (uint32_t)(tid + p * S::THREADS);
        go[p] = d_deposit(l, run.qmask);
        so[p] = d_extract(l, run.sbits) * S::W + d_extract(l, cbits);
    }

    const uint64_t total = run.ntiles * (uint64_t)nbatch;
    auto origin = [&](uint64_t T) {
        const uint64_t slot = T / run.ntiles, t = T - slot * run.ntiles;
        return psi + slot * nbasis + d_spread(t, run.qmask);
    };
    auto load = [&](uint64_t T, double2 *b) {
        const double2 *src = origin(T);
#pragma unroll
        for (int p = 0; p < S::PER; ++p) cp16(d_smem_u32(b + so[p]), src + go[p]);
        cp_commit();
    };

    uint64_t T = blockIdx.x;
    if (T < total) load(T, buf0);
    int cur = 0;
    for (; T < total; T += gridDim.x) {
        double2 *b = cur ? buf1 : buf0;
        const uint64_t Tn = T + gridDim.x;
        if (Tn < total) {
            load(Tn, cur ? buf0 : buf1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();

        double dr[S::CB][2], di[S::CB][2];
#pragma unroll
        for (int c = 0; c < S::CB; ++c) dr[c][0] = dr[c][1] = di[c][0] = di[c][1] = 0.0;
#pragma unroll
        for (int j = 0; j < S::KSTEPS; ++j) {
#pragma unroll
            for (int c = 0; c < S::CB; ++c) {
                // B fragment: tile row 4 j + q, column 8 c + g
                const double2 x = b[(4 * j + q) * S::W + 8 * c + g];
                dmma(dr[c][0], dr[c][1], ar[j], x.x);
                dmma(dr[c][0], dr[c][1], ai[j], -x.y);
                dmma(di[c][0], di[c][1], ar[j], x.y);
                dmma(di[c][0], di[c][1], ai[j], x.x);
            }
        }
        __syncthreads();  // every warp has read the whole tile
        // D fragment: row 8 warp + g, columns 8 c + 2 q and + 1
#pragma unroll
        for (int c = 0; c < S::CB; ++c) {
            double2 *o = b + (8 * warp + g) * S::W + 8 * c + 2 * q;
            o[0] = make_double2(dr[c][0], di[c][0]);
            o[1] = make_double2(dr[c][1], di[c][1]);
        }
        __syncthreads();
        double2 *dst = origin(T);
#pragma unroll
        for (int p = 0; p < S::PER; ++p) dst[go[p]] = b[so[p]];
        __syncthreads();  // this buffer is refilled by the next iteration's prefetch
        cur ^= 1;
    }
}

}  // namespace qfbd
