/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the CSR SpGEMM hot path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs may load this library.  The product path
 * (gpuspgemm_b200) never calls it: it is the checker, not the thing measured.
 *
 * What it restates.  The reference has no CPU SpGEMM.  Its method computes
 *     C(i,:) = sum over k in A(i,:) of A(i,k) * B(k,:)
 * in three GPU phases (src/libproposal/include/proposal/):
 *   - NIP per row  = sum_{k in A(i,:)} len(B(k,:))        setup.cuh:29-95
 *   - exact nnz per row = number of distinct column keys   sym1.cuh:77-94
 *   - sorted column list per row                           sym2.cuh:104-120
 *   - c_ij += a_ik * b_kj, every structural product kept,  num.cuh:104-116
 *     no dropping of entries whose value cancels to zero
 * This file computes the same C with a row-wise Gustavson SpGEMM: a dense
 * marker + accumulator per thread, columns emitted in ascending order,
 * products summed in A-row order (k ascending within the row as stored).
 * Each product a*b is rounded before it is added (compiled with
 * -ffp-contract=off), as in the reference, whose atomicAdd of a*b cannot
 * fuse the multiply into the add (num.cuh:113).
 *
 * The total-NIP routine restates utils::get_nip (src/libutils/include/utils/nip.cuh:19-78),
 * and the .csr equality tolerance restates operator== (csr.cuh:218-239).
 *
 * Threads: OpenMP over rows, schedule(dynamic, 64).  The caller chooses the
 * thread count (oracle_set_threads).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_OK 0
#define ORACLE_ERR_ALLOC 1
#define ORACLE_ERR_OVERFLOW 2
#define ORACLE_ERR_ARG 3

int oracle_version(void) { return 1; }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* NIP per row (int64) and total NIP; restates setup.cuh:29-95 / nip.cuh:19-49. */
int64_t oracle_nip(int32_t m, const int32_t* a_rpt, const int32_t* a_col,
                   const int32_t* b_rpt, int64_t* nip_per_row /* may be NULL */) {
    int64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int32_t i = 0; i < m; i++) {
        int64_t s = 0;
        for (int32_t p = a_rpt[i]; p < a_rpt[i + 1]; p++) {
            const int32_t k = a_col[p];
            s += (int64_t)(b_rpt[k + 1] - b_rpt[k]);
        }
        if (nip_per_row) nip_per_row[i] = s;
        total += s;
    }
    return total;
}

/* Insertion sort for short lists, else qsort. */
static int cmp_i32(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}
static void sort_i32(int32_t* v, int32_t n) {
    if (n < 32) {
        for (int32_t i = 1; i < n; i++) {
            int32_t x = v[i], j = i - 1;
            while (j >= 0 && v[j] > x) { v[j + 1] = v[j]; j--; }
            v[j + 1] = x;
        }
    } else {
        qsort(v, (size_t)n, sizeof(int32_t), cmp_i32);
    }
}

/*
 * Symbolic: exact distinct-column count of every row of C = A*B, written as a
 * row pointer (exclusive scan, c_rpt[m] = nnz(C)).  Returns ORACLE_ERR_OVERFLOW
 * when nnz(C) does not fit int32 (the reference's CSR uses int32 nnz, csr.cuh:25).
 */
int oracle_symbolic(int32_t m, int32_t n, const int32_t* a_rpt, const int32_t* a_col,
                    const int32_t* b_rpt, const int32_t* b_col, int32_t* c_rpt) {
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    if (!cnt) return ORACLE_ERR_ALLOC;
    int err = 0;
#pragma omp parallel
    {
        int32_t* mark = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        if (!mark) {
#pragma omp atomic write
            err = 1;
        } else {
            for (int32_t j = 0; j < n; j++) mark[j] = -1;
#pragma omp for schedule(dynamic, 64)
            for (int32_t i = 0; i < m; i++) {
                int64_t c = 0;
                for (int32_t p = a_rpt[i]; p < a_rpt[i + 1]; p++) {
                    const int32_t k = a_col[p];
                    for (int32_t q = b_rpt[k]; q < b_rpt[k + 1]; q++) {
                        const int32_t j = b_col[q];
                        if (mark[j] != i) { mark[j] = i; c++; }
                    }
                }
                cnt[i] = c;
            }
            free(mark);
        }
    }
    if (err) { free(cnt); return ORACLE_ERR_ALLOC; }
    int64_t acc = 0;
    for (int32_t i = 0; i < m; i++) {
        c_rpt[i] = (int32_t)acc;
        acc += cnt[i];
        if (acc > INT32_MAX) { free(cnt); return ORACLE_ERR_OVERFLOW; }
    }
    c_rpt[m] = (int32_t)acc;
    free(cnt);
    return ORACLE_OK;
}

/* Numeric fill, FP64 accumulate.  c_rpt comes from oracle_symbolic. */
int oracle_numeric_f64(int32_t m, int32_t n, const int32_t* a_rpt, const int32_t* a_col,
                       const double* a_val, const int32_t* b_rpt, const int32_t* b_col,
                       const double* b_val, const int32_t* c_rpt, int32_t* c_col,
                       double* c_val) {
    int err = 0;
#pragma omp parallel
    {
        int32_t* mark = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        double* acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        if (!mark || !acc) {
#pragma omp atomic write
            err = 1;
        } else {
            for (int32_t j = 0; j < n; j++) mark[j] = -1;
#pragma omp for schedule(dynamic, 64)
            for (int32_t i = 0; i < m; i++) {
                int32_t* cols = c_col + c_rpt[i];
                int32_t len = 0;
                for (int32_t p = a_rpt[i]; p < a_rpt[i + 1]; p++) {
                    const int32_t k = a_col[p];
                    const double a = a_val[p];
                    for (int32_t q = b_rpt[k]; q < b_rpt[k + 1]; q++) {
                        const int32_t j = b_col[q];
                        const double prod = a * b_val[q];
                        if (mark[j] != i) {
                            mark[j] = i;
                            acc[j] = 0.0;
                            cols[len++] = j;
                        }
                        acc[j] += prod;
                    }
                }
                sort_i32(cols, len);
                for (int32_t t = 0; t < len; t++) c_val[c_rpt[i] + t] = acc[cols[t]];
            }
        }
        free(mark);
        free(acc);
    }
    return err ? ORACLE_ERR_ALLOC : ORACLE_OK;
}

/* Numeric fill, FP32 values accumulated in FP32 (the f32 build of the reference). */
int oracle_numeric_f32(int32_t m, int32_t n, const int32_t* a_rpt, const int32_t* a_col,
                       const float* a_val, const int32_t* b_rpt, const int32_t* b_col,
                       const float* b_val, const int32_t* c_rpt, int32_t* c_col,
                       float* c_val) {
    int err = 0;
#pragma omp parallel
    {
        int32_t* mark = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
        float* acc = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
        if (!mark || !acc) {
#pragma omp atomic write
            err = 1;
        } else {
            for (int32_t j = 0; j < n; j++) mark[j] = -1;
#pragma omp for schedule(dynamic, 64)
            for (int32_t i = 0; i < m; i++) {
                int32_t* cols = c_col + c_rpt[i];
                int32_t len = 0;
                for (int32_t p = a_rpt[i]; p < a_rpt[i + 1]; p++) {
                    const int32_t k = a_col[p];
                    const float a = a_val[p];
                    for (int32_t q = b_rpt[k]; q < b_rpt[k + 1]; q++) {
                        const int32_t j = b_col[q];
                        const float prod = a * b_val[q];
                        if (mark[j] != i) {
                            mark[j] = i;
                            acc[j] = 0.0f;
                            cols[len++] = j;
                        }
                        acc[j] += prod;
                    }
                }
                sort_i32(cols, len);
                for (int32_t t = 0; t < len; t++) c_val[c_rpt[i] + t] = acc[cols[t]];
            }
        }
        free(mark);
        free(acc);
    }
    return err ? ORACLE_ERR_ALLOC : ORACLE_OK;
}

/*
 * Per-entry condition bound sum_k |a_ik| |b_kj| (FP64), used by the tests to
 * state a cancellation-aware error: |c_gpu - c_ref| / bound.
 */
int oracle_abs_bound_f64(int32_t m, int32_t n, const int32_t* a_rpt, const int32_t* a_col,
                         const double* a_val, const int32_t* b_rpt, const int32_t* b_col,
                         const double* b_val, const int32_t* c_rpt, const int32_t* c_col,
                         double* bound) {
    int err = 0;
#pragma omp parallel
    {
        double* acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        if (!acc) {
#pragma omp atomic write
            err = 1;
        } else {
#pragma omp for schedule(dynamic, 64)
            for (int32_t i = 0; i < m; i++) {
                for (int32_t t = c_rpt[i]; t < c_rpt[i + 1]; t++) acc[c_col[t]] = 0.0;
                for (int32_t p = a_rpt[i]; p < a_rpt[i + 1]; p++) {
                    const int32_t k = a_col[p];
                    const double a = fabs(a_val[p]);
                    for (int32_t q = b_rpt[k]; q < b_rpt[k + 1]; q++)
                        acc[b_col[q]] += a * fabs(b_val[q]);
                }
                for (int32_t t = c_rpt[i]; t < c_rpt[i + 1]; t++) bound[t] = acc[c_col[t]];
            }
        }
        free(acc);
    }
    return err ? ORACLE_ERR_ALLOC : ORACLE_OK;
}

/*
 * The reference's value tolerance, operator== in csr.cuh:218-239:
 * equal, or |l - r| <= 1e-8 + 1e-5 * max(|l|, |r|).  Returns the number of
 * entries that fail it.
 */
int64_t oracle_count_reference_mismatch_f64(int64_t nnz, const double* l, const double* r) {
    int64_t bad = 0;
    for (int64_t t = 0; t < nnz; t++) {
        const double x = l[t], y = r[t];
        if (x == y) continue;
        const double ax = fabs(x), ay = fabs(y);
        if (!(fabs(x - y) <= 1e-8 + 1e-5 * (ax > ay ? ax : ay))) bad++;
    }
    return bad;
}
