/*
 * h2oracle.c -- CPU oracle of the H2 matrix-vector product.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain C restatement of H2Factory.jl's CPU matvec
 * (traversal, orientation rules, leaf products, level transfers, dense/diagonal/Toeplitz
 * couplings, near product), used by the tests, by the benchmark's CPU baseline and by the
 * reference arm of the benchmark. The product (the CUDA library) never calls it.
 *
 * It consumes the same flattened map descriptor as the CUDA library (include/h2b200.h), so
 * both compute the same map. The reference itself (Julia) cannot run on this machine; the
 * oracle is pinned against the closed-form known-answer tests that the reference's own test
 * suite and documentation use (tests/golden, tests/test_oracle_golden.py).
 *
 * Per-level loops are parallel over nodes with OpenMP, the same decomposition as the
 * reference's OhMyThreads @tasks over node chunks (src/farinteractions/aggregation.jl:108,
 * src/farinteractions/disaggregation.jl:168).
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/h2b200.h"

static __thread char oracle_err[512];

static void oracle_set_error(const char *msg) {
    strncpy(oracle_err, msg, sizeof(oracle_err) - 1);
    oracle_err[sizeof(oracle_err) - 1] = 0;
}

const char *oracle_last_error(void) { return oracle_err; }

/* ---- real instantiation ---- */
#define SC double
#define CONJ(z) (z)
#define SFX(n) n##_r
#define MKIMAG(v)
#define TAKEREAL(z) creal(z)
#include "h2oracle_impl.h"
#undef SC
#undef CONJ
#undef SFX
#undef MKIMAG
#undef TAKEREAL

/* ---- complex instantiation ---- */
#define SC double _Complex
#define CONJ(z) conj(z)
#define SFX(n) n##_c
#define MKIMAG(v) +(v) * I
#define TAKEREAL(z) (z)
#include "h2oracle_impl.h"
#undef SC
#undef CONJ
#undef SFX
#undef MKIMAG
#undef TAKEREAL

static int check_args(const h2b_map_desc *d, int mode, int nrhs, const double *alpha, const double *beta) {
    if (!d) { oracle_set_error("null descriptor"); return H2B_ERR_INVALID; }
    if (mode < 0 || mode > 2) { oracle_set_error("mode must be 0, 1 or 2"); return H2B_ERR_INVALID; }
    if (nrhs < 1) { oracle_set_error("nrhs must be >= 1"); return H2B_ERR_INVALID; }
    if ((alpha == NULL) != (beta == NULL)) { oracle_set_error("alpha and beta must both be given or both be NULL"); return H2B_ERR_INVALID; }
    if (d->field == H2B_REAL && alpha && (alpha[1] != 0.0 || beta[1] != 0.0)) {
        oracle_set_error("complex alpha/beta on a real map");
        return H2B_ERR_INVALID;
    }
    if (d->near_on_device) { oracle_set_error("the oracle needs host near blocks"); return H2B_ERR_INVALID; }
    return H2B_OK;
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* farmul!(y, op(A), x[, α, β]) (src/farinteractions/farmul.jl:8-70) */
int oracle_farmul(const h2b_map_desc *d, int mode, int nrhs, const double *x, int64_t ldx, double *y,
                  int64_t ldy, const double *alpha, const double *beta, int nthreads) {
    int st = check_args(d, mode, nrhs, alpha, beta);
    if (st) return st;
    set_threads(nthreads);
    const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
    const int threearg = (alpha == NULL);
    const int64_t ny = (mode == H2B_FORWARD) ? d->test.ndofs : d->trial.ndofs;
    if (d->field == H2B_REAL) {
        if (threearg)
            for (int r = 0; r < nrhs; ++r) memset(y + (int64_t)r * ldy, 0, sizeof(double) * (size_t)ny);
        return farmul_r(d, mode, nrhs, x, ldx, y, ldy, threearg ? one : alpha, threearg ? zero : beta);
    }
    if (threearg)
        for (int r = 0; r < nrhs; ++r) memset(y + 2 * (int64_t)r * ldy, 0, 2 * sizeof(double) * (size_t)ny);
    return farmul_c(d, mode, nrhs, (const double _Complex *)x, ldx, (double _Complex *)y, ldy,
                    threearg ? one : alpha, threearg ? zero : beta);
}

/* nearmul!(y, op(A), x[, α, β]) (src/nearinteractions/nearmul.jl:8-14) */
int oracle_nearmul(const h2b_map_desc *d, int mode, int nrhs, const double *x, int64_t ldx, double *y,
                   int64_t ldy, const double *alpha, const double *beta, int nthreads) {
    int st = check_args(d, mode, nrhs, alpha, beta);
    if (st) return st;
    set_threads(nthreads);
    const double a0 = alpha ? alpha[0] : 1.0, a1 = alpha ? alpha[1] : 0.0;
    const double b0 = beta ? beta[0] : 0.0, b1 = beta ? beta[1] : 0.0;
    if (d->field == H2B_REAL) return nearmul_r(d, mode, nrhs, x, ldx, y, ldy, a0, b0);
    return nearmul_c(d, mode, nrhs, (const double _Complex *)x, ldx, (double _Complex *)y, ldy,
                     a0 + a1 * I, b0 + b1 * I);
}

/* mul!(y, op(A), x[, α, β]): near with (α, β), then far with (α, 1)
 * (src/maps/abstracth2map.jl:54-86). */
int oracle_matvec(const h2b_map_desc *d, int mode, int nrhs, const double *x, int64_t ldx, double *y,
                  int64_t ldy, const double *alpha, const double *beta, int nthreads) {
    int st = oracle_nearmul(d, mode, nrhs, x, ldx, y, ldy, alpha, beta, nthreads);
    if (st) return st;
    const double one[2] = {1.0, 0.0};
    return oracle_farmul(d, mode, nrhs, x, ldx, y, ldy, alpha ? alpha : one, one, nthreads);
}

/* Standalone Toeplitz operator of ext/H2Toeplitz/H2Toeplitz.jl:19-47: y = T x with T the
 * multilevel Toeplitz matrix of the FFT'd wrap-around kernel `khat` (complex, prod(2s-1)),
 * adjoint != 0 gives T' x. Used to pin the FFT conventions against the dense oracle. */
int oracle_toeplitz_apply(const int *s, const double *khat, const double *x, double *y, int adjoint) {
    int ts[3] = {2 * s[0] - 1, 2 * s[1] - 1, 2 * s[2] - 1};
    const int64_t nt = (int64_t)ts[0] * ts[1] * ts[2];
    double _Complex *buf = (double _Complex *)calloc((size_t)nt, sizeof(double _Complex));
    if (!buf) return H2B_ERR_NOMEM;
    const double _Complex *xx = (const double _Complex *)x;
    const double _Complex *K = (const double _Complex *)khat;
    for (int i3 = 0; i3 < s[2]; ++i3)
        for (int i2 = 0; i2 < s[1]; ++i2)
            for (int i1 = 0; i1 < s[0]; ++i1) {
                double _Complex v = xx[i1 + s[0] * ((int64_t)i2 + s[1] * i3)];
                buf[i1 + ts[0] * ((int64_t)i2 + ts[1] * i3)] = adjoint ? conj(v) : v;
            }
    /* forward: ifft(K .* fft(x)); adjoint: conj(fft(K .* ifft(conj x))) */
    dft_axes_c(buf, ts, adjoint);
    for (int64_t e = 0; e < nt; ++e) buf[e] *= K[e];
    dft_axes_c(buf, ts, !adjoint);
    double _Complex *yy = (double _Complex *)y;
    for (int i3 = 0; i3 < s[2]; ++i3)
        for (int i2 = 0; i2 < s[1]; ++i2)
            for (int i1 = 0; i1 < s[0]; ++i1) {
                double _Complex v = buf[i1 + ts[0] * ((int64_t)i2 + ts[1] * i3)];
                yy[i1 + s[0] * ((int64_t)i2 + s[1] * i3)] = adjoint ? conj(v) : v;
            }
    free(buf);
    return H2B_OK;
}

/* fft (inverse = 0) or ifft (inverse = 1) of a complex column-major array with extents n[3],
 * AbstractFFTs conventions. Exposed so tests can build Toeplitz couplings with the same
 * transform the oracle applies. */
int oracle_dft(double *a, const int *n, int inverse) {
    dft_axes_c((double _Complex *)a, n, inverse);
    return H2B_OK;
}
