/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the state-vector engine.
 *
 * Plain-C restatement of QForte's `Computer` gate kernels, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * Nothing in the product links or calls this file.
 *
 * State layout: interleaved complex128, psi[2*i] = Re, psi[2*i+1] = Im, basis
 * index i with qubit k <-> bit k (qubit_basis.h:27-45).
 * Gate matrices: 4x4 complex, row-major, interleaved (mat[2*(4*r+c)+{0,1}]);
 * 1-qubit gates use the top-left 2x2 block; 2-qubit row/column index is
 * (control_bit << 1) | target_bit (gate.cc:7-8, :75).
 *
 * Each branch follows the case analysis of the reference:
 *   apply_1qubit_gate    computer.cc:340-425
 *   apply_2qubit_gate    computer.cc:458-751  (controlled fast path :469-719,
 *                                               generic accumulation :721-750)
 *   apply_operator       computer.cc:80-91
 *   apply_constant       computer.cc:130-133
 *   dot / inner_product  computer.cc:975-980, :763-765
 * including the reference's quirks (a gate whose off-diagonals compare equal
 * is treated as X, `op_0_1 == op_1_0 == 1.0` at :398/:548/:669; the
 * controlled path ignores matrix entries outside the control=1 block).
 * Parity status: pinned against the compiled reference (tests/golden).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define THR 1.0e-16 /* Computer::compute_threshold_ (computer.h:172) */

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx cadd(cplx a, cplx b) {
    cplx r = {a.re + b.re, a.im + b.im};
    return r;
}
static inline double cabs_(cplx a) { return hypot(a.re, a.im); }
static inline int ceq(cplx a, cplx b) { return a.re == b.re && a.im == b.im; }
static inline int cis1(cplx a) { return a.re == 1.0 && a.im == 0.0; }

static inline cplx mat_at(const double *mat, int r, int c) {
    cplx v = {mat[2 * (4 * r + c)], mat[2 * (4 * r + c) + 1]};
    return v;
}

/* Apply the 2x2 block [[a, b], [c, d]] to every pair (i0, i0 | tbit) where i0
 * has bit `t` clear and (when cmask != 0) all bits of cmask set.  The four
 * cases mirror computer.cc:353-423 (and the controlled copies :479-595). */
static void apply_block(cplx *psi, uint64_t nbasis, int t, uint64_t cmask, cplx a, cplx b, cplx c,
                        cplx d) {
    const uint64_t tbit = (uint64_t)1 << t;
    const int has_diag = (cabs_(a) + cabs_(d) > THR);
    const int has_off = (cabs_(b) + cabs_(c) > THR);
    for (uint64_t i0 = 0; i0 < nbasis; ++i0) {
        if (i0 & tbit) continue;
        if ((i0 & cmask) != cmask) continue;
        const uint64_t i1 = i0 | tbit;
        const cplx x0 = psi[i0], x1 = psi[i1];
        if (has_diag && has_off) {
            psi[i0] = cadd(cmul(a, x0), cmul(b, x1));
            psi[i1] = cadd(cmul(c, x0), cmul(d, x1));
        } else if (has_diag) {
            if (!cis1(a)) psi[i0] = cmul(a, x0);
            if (!cis1(d)) psi[i1] = cmul(d, x1);
        } else {
            /* (op_0_1 == op_1_0) == 1.0 : any equal off-diagonal pair acts as X */
            if (ceq(b, c)) {
                psi[i0] = x1;
                psi[i1] = x0;
            } else {
                psi[i0] = cmul(b, x1);
                psi[i1] = cmul(c, x0);
            }
        }
    }
}

void ora_apply_gate(double *psi_, int nqubit, int target, int control, const double *mat) {
    cplx *psi = (cplx *)psi_;
    const uint64_t nbasis = (uint64_t)1 << nqubit;
    if (target == control) {
        apply_block(psi, nbasis, target, 0, mat_at(mat, 0, 0), mat_at(mat, 0, 1), mat_at(mat, 1, 0),
                    mat_at(mat, 1, 1));
        return;
    }
    const cplx m00 = mat_at(mat, 0, 0), m01 = mat_at(mat, 0, 1), m10 = mat_at(mat, 1, 0),
               m11 = mat_at(mat, 1, 1);
    if ((cabs_(m01) + cabs_(m10) < THR) && cis1(m00) && cis1(m11)) {
        /* controlled unitary: act on the control = 1 half only */
        apply_block(psi, nbasis, target, (uint64_t)1 << control, mat_at(mat, 2, 2),
                    mat_at(mat, 2, 3), mat_at(mat, 3, 2), mat_at(mat, 3, 3));
        return;
    }
    /* generic path: new[I] = sum_j m[i][j] psi[J] over the 2-qubit sub-basis,
     * accumulated in (i, j) order exactly as computer.cc:725-749 does. */
    const uint64_t tbit = (uint64_t)1 << target, cbit = (uint64_t)1 << control;
    cplx *out = (cplx *)calloc(nbasis, sizeof(cplx));
    for (int i = 0; i < 4; ++i) {
        const int ic = i >> 1, it = i & 1;
        for (int j = 0; j < 4; ++j) {
            const int jc = j >> 1, jt = j & 1;
            const cplx m = mat_at(mat, i, j);
            if (!(cabs_(m) > THR)) continue;
            for (uint64_t J = 0; J < nbasis; ++J) {
                if ((int)((J & cbit) != 0) != jc || (int)((J & tbit) != 0) != jt) continue;
                uint64_t I = J;
                I = ic ? (I | cbit) : (I & ~cbit);
                I = it ? (I | tbit) : (I & ~tbit);
                out[I] = cadd(out[I], cmul(m, psi[J]));
            }
        }
    }
    memcpy(psi, out, nbasis * sizeof(cplx));
    free(out);
}

/* Computer::apply_circuit (computer.cc:93-97): gates in list order. */
void ora_apply_gates(double *psi, int nqubit, int64_t ngates, const int32_t *targets,
                     const int32_t *controls, const double *mats) {
    for (int64_t g = 0; g < ngates; ++g)
        ora_apply_gate(psi, nqubit, targets[g], controls[g], mats + 32 * g);
}

/* Computer::apply_constant (computer.cc:130-133). */
void ora_scale(double *psi_, int nqubit, double re, double im) {
    cplx *psi = (cplx *)psi_;
    const uint64_t nbasis = (uint64_t)1 << nqubit;
    const cplx a = {re, im};
    for (uint64_t i = 0; i < nbasis; ++i) psi[i] = cmul(psi[i], a);
}

/* <a|b> = sum_i conj(a_i) b_i in index order (computer.cc:975-980). */
void ora_dot(const double *a_, const double *b_, int nqubit, double *out) {
    const cplx *a = (const cplx *)a_, *b = (const cplx *)b_;
    const uint64_t nbasis = (uint64_t)1 << nqubit;
    cplx acc = {0.0, 0.0};
    for (uint64_t i = 0; i < nbasis; ++i) {
        const cplx ca = {a[i].re, -a[i].im};
        acc = cadd(acc, cmul(ca, b[i]));
    }
    out[0] = acc.re;
    out[1] = acc.im;
}

/* Computer::apply_operator (computer.cc:80-91): for each term, copy the state,
 * apply the term's circuit, scale by its coefficient, accumulate.
 * Term k's gates are [offsets[k], offsets[k+1]) of the flat gate arrays. */
void ora_apply_operator(double *psi_, int nqubit, int64_t nterms, const double *coeffs,
                        const int64_t *offsets, const int32_t *targets, const int32_t *controls,
                        const double *mats) {
    cplx *psi = (cplx *)psi_;
    const uint64_t nbasis = (uint64_t)1 << nqubit;
    cplx *old = (cplx *)malloc(nbasis * sizeof(cplx));
    cplx *result = (cplx *)calloc(nbasis, sizeof(cplx));
    memcpy(old, psi, nbasis * sizeof(cplx));
    for (int64_t k = 0; k < nterms; ++k) {
        const int64_t g0 = offsets[k], g1 = offsets[k + 1];
        ora_apply_gates(psi_, nqubit, g1 - g0, targets + g0, controls + g0, mats + 32 * g0);
        ora_scale(psi_, nqubit, coeffs[2 * k], coeffs[2 * k + 1]);
        for (uint64_t i = 0; i < nbasis; ++i) result[i] = cadd(result[i], psi[i]);
        memcpy(psi, old, nbasis * sizeof(cplx));
    }
    memcpy(psi, result, nbasis * sizeof(cplx));
    free(old);
    free(result);
}
