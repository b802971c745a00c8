/*
 * CPU oracle for the MindQuantum state-vector hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is a plain-C restatement of the reference `mqvector` CPU policy
 * (OpenMP loops over amplitude pairs / quads).  It exists so the tests, the
 * smoke check and the CPU baseline leg of the benchmark can check / time the
 * B200 kernels against the reference algorithm.  Nothing in the product links
 * or calls it.
 *
 * Conventions (all from the reference):
 *   - the state is 2^n interleaved complex numbers, little endian: amplitude
 *     index bit q <-> qubit q;
 *   - a k-qubit matrix acting on objs[0..k-1] is indexed by
 *     sum_b bit(objs[b]) << b  (ApplyTwoQubitsMatrix / ApplyNQubitsMatrix,
 *     ccsrc/lib/simulator/vector/detail/cpu_common/cpu_vector_core_matrix_gate.cpp:29-149);
 *   - a control mask restricts the update to indices with all control bits set;
 *   - reductions accumulate in the state's own real type, as the reference's
 *     `calc_type` accumulators do (float for complex64).
 *
 * Every function exists in two precisions: suffix _d (complex128) and _f (complex64).
 * Matrices are always passed as interleaved double (re, im) row-major; for the
 * float build they are rounded to float first, as the reference does with
 * `to_vector<py_qs_data_t>(m)`.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t idx_t;

/* POLAR table: i^k, ccsrc/lib/mq_base/utils.cc:22 */
static const double POLAR_RE[4] = {1, 0, -1, 0};
static const double POLAR_IM[4] = {0, 1, 0, -1};

static inline idx_t insert_zero(idx_t l, int q) {
    /* ((l & high) << 1) + (l & low) as in SingleQubitGateMask, ccsrc/lib/simulator/utils.cpp:42-52 */
    idx_t low = (((idx_t)1) << q) - 1;
    return ((l & ~low) << 1) | (l & low);
}

static inline idx_t insert_zero2(idx_t l, int qa, int qb) {
    /* SHIFT_BIT_TWO, ccsrc/include/simulator/utils.h:53-58 (qa < qb) */
    idx_t i = insert_zero(l, qa);
    return insert_zero(i, qb);
}

#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#define OMP_RED _Pragma("omp parallel for schedule(static) reduction(+ : acc_re, acc_im)")

#define DEFINE_ORACLE(T, SUF)                                                                                    \
    typedef T _Complex c##SUF;                                                                                   \
    static inline c##SUF mk##SUF(double re, double im) { return (T)re + (T)im * (c##SUF)I; }                   \
                                                                                                                 \
    /* ApplySingleQubitMatrix: cpu_common/cpu_vector_core_matrix_gate.cpp:151-200 (generic), AVX variant       \
     * cpu_avx_double/cpu_vector_core_matrix_gate.cpp:23-70.  m: 2x2 row-major interleaved. */                \
    void orc_apply_single_matrix_##SUF(T *qs_, int n, int q, idx_t ctrl, const double *m) {                    \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        c##SUF m00 = mk##SUF(m[0], m[1]), m01 = mk##SUF(m[2], m[3]);                                            \
        c##SUF m10 = mk##SUF(m[4], m[5]), m11 = mk##SUF(m[6], m[7]);                                            \
        idx_t half = ((idx_t)1) << (n - 1), om = ((idx_t)1) << q;                                              \
        OMP_FOR for (idx_t l = 0; l < half; l++) {                                                               \
            idx_t i = insert_zero(l, q);                                                                         \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t j = i | om;                                                                                    \
            c##SUF a = qs[i], b = qs[j];                                                                         \
            qs[i] = m00 * a + m01 * b;                                                                           \
            qs[j] = m10 * a + m11 * b;                                                                           \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyTwoQubitsMatrix: cpu_vector_core_matrix_gate.cpp:83-149.  basis index = b(objs0) + 2 b(objs1). */  \
    void orc_apply_two_matrix_##SUF(T *qs_, int n, int q0, int q1, idx_t ctrl, const double *m) {              \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        c##SUF g[16];                                                                                            \
        for (int t = 0; t < 16; t++) g[t] = mk##SUF(m[2 * t], m[2 * t + 1]);                                     \
        int qa = q0 < q1 ? q0 : q1, qb = q0 < q1 ? q1 : q0;                                                      \
        idx_t quarter = ((idx_t)1) << (n - 2), m1 = ((idx_t)1) << q0, m2 = ((idx_t)1) << q1;                   \
        OMP_FOR for (idx_t l = 0; l < quarter; l++) {                                                            \
            idx_t i = insert_zero2(l, qa, qb);                                                                   \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t id[4] = {i, i + m1, i + m2, i + m1 + m2};                                                      \
            c##SUF v[4] = {qs[id[0]], qs[id[1]], qs[id[2]], qs[id[3]]};                                          \
            for (int r = 0; r < 4; r++)                                                                          \
                qs[id[r]] = g[4 * r] * v[0] + g[4 * r + 1] * v[1] + g[4 * r + 2] * v[2] + g[4 * r + 3] * v[3];  \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyNQubitsMatrix: cpu_vector_core_matrix_gate.cpp:29-81 (any k, loop over base indices). */           \
    void orc_apply_n_matrix_##SUF(T *qs_, int n, const int *objs, int k, idx_t ctrl, const double *m) {        \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        int md = 1 << k;                                                                                         \
        idx_t *om = (idx_t *)malloc(sizeof(idx_t) * md);                                                         \
        c##SUF *g = (c##SUF *)malloc(sizeof(c##SUF) * md * md);                                                  \
        for (int a = 0; a < md; a++) {                                                                           \
            idx_t mk = 0;                                                                                        \
            for (int b = 0; b < k; b++)                                                                          \
                if (a >> b & 1) mk |= ((idx_t)1) << objs[b];                                                     \
            om[a] = mk;                                                                                          \
        }                                                                                                        \
        for (int t = 0; t < md * md; t++) g[t] = mk##SUF(m[2 * t], m[2 * t + 1]);                                \
        idx_t all = om[md - 1], dim = ((idx_t)1) << n;                                                           \
        OMP_FOR for (idx_t l = 0; l < dim; l++) {                                                                \
            if ((l & ctrl) != ctrl || (l & all) != 0) continue;                                                  \
            c##SUF v[64], r[64];                                                                                 \
            for (int a = 0; a < md; a++) v[a] = qs[om[a] | l];                                                   \
            for (int a = 0; a < md; a++) {                                                                       \
                c##SUF t = 0;                                                                                    \
                for (int b = 0; b < md; b++) t += g[a * md + b] * v[b];                                          \
                r[a] = t;                                                                                        \
            }                                                                                                    \
            for (int a = 0; a < md; a++) qs[om[a] | l] = r[a];                                                   \
        }                                                                                                        \
        free(om);                                                                                                \
        free(g);                                                                                                 \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyXLike: cpu_vector_core_x_like.cpp:29-57.  X: v1=v2=1, Y: v1=-i, v2=i. */                           \
    void orc_apply_xlike_##SUF(T *qs_, int n, int q, idx_t ctrl, double v1r, double v1i, double v2r,           \
                               double v2i) {                                                                     \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        c##SUF v1 = mk##SUF(v1r, v1i), v2 = mk##SUF(v2r, v2i);                                                  \
        idx_t half = ((idx_t)1) << (n - 1), om = ((idx_t)1) << q;                                              \
        OMP_FOR for (idx_t l = 0; l < half; l++) {                                                               \
            idx_t i = insert_zero(l, q);                                                                         \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t j = i | om;                                                                                    \
            c##SUF tmp = qs[i];                                                                                  \
            qs[i] = qs[j] * v1;                                                                                  \
            qs[j] = tmp * v2;                                                                                    \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyZLike: cpu_vector_core_z_like.cpp:29-52 (phase on the |1> half). */                                 \
    void orc_apply_zlike_##SUF(T *qs_, int n, int q, idx_t ctrl, double vr, double vi) {                       \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        c##SUF v = mk##SUF(vr, vi);                                                                              \
        idx_t half = ((idx_t)1) << (n - 1), om = ((idx_t)1) << q;                                              \
        OMP_FOR for (idx_t l = 0; l < half; l++) {                                                               \
            idx_t i = insert_zero(l, q) | om;                                                                    \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            qs[i] *= v;                                                                                          \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyRzz: cpu_vector_core_rot_pauli.cpp:380-428 (diag me, e, e, me). */                                  \
    void orc_apply_rzz_##SUF(T *qs_, int n, int q0, int q1, idx_t ctrl, double val) {                          \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        T c = (T)cos(val / 2), s = (T)sin(val / 2);                                                              \
        c##SUF e = c + s * (c##SUF)I, me = c - s * (c##SUF)I;                                                    \
        int qa = q0 < q1 ? q0 : q1, qb = q0 < q1 ? q1 : q0;                                                      \
        idx_t quarter = ((idx_t)1) << (n - 2), m1 = ((idx_t)1) << q0, m2 = ((idx_t)1) << q1;                   \
        OMP_FOR for (idx_t l = 0; l < quarter; l++) {                                                            \
            idx_t i = insert_zero2(l, qa, qb);                                                                   \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            qs[i] *= me;                                                                                         \
            qs[i + m1] *= e;                                                                                     \
            qs[i + m2] *= e;                                                                                     \
            qs[i + m1 + m2] *= me;                                                                               \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyRPS: cpu_vector_core_rot_pauli.cpp:466-524, exp(-i val/2 P) for a Pauli string P. */                \
    void orc_apply_rps_##SUF(T *qs_, int n, idx_t mx, idx_t my, idx_t mz, int num_y, idx_t ctrl, double val) { \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        T a = (T)cos(val / 2), b = (T)sin(val / 2);                                                              \
        idx_t mf = mx | my, dim = ((idx_t)1) << n;                                                               \
        OMP_FOR for (idx_t i = 0; i < dim; i++) {                                                                \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t j = i ^ mf;                                                                                    \
            if (i > j) continue;                                                                                 \
            int p = (num_y + 2 * __builtin_popcountll(i & my) + 2 * __builtin_popcountll(i & mz)) & 3;          \
            c##SUF c = mk##SUF(POLAR_RE[p], POLAR_IM[p]);                                                        \
            if (i == j) {                                                                                        \
                qs[i] *= (a - (c##SUF)I * b * c);                                                                \
            } else {                                                                                             \
                c##SUF qi = qs[i], qj = qs[j];                                                                   \
                qs[i] = qi * a - (c##SUF)I * qj * b / c;                                                         \
                qs[j] = qj * a - (c##SUF)I * qi * b * c;                                                         \
            }                                                                                                    \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyPauliString: cpu_vector_core_policy.cpp:163-210. */                                                \
    void orc_apply_pauli_string_##SUF(T *qs_, int n, idx_t mx, idx_t my, idx_t mz, int num_y, idx_t ctrl) {    \
        c##SUF *qs = (c##SUF *)qs_;                                                                              \
        idx_t mf = mx | my, dim = ((idx_t)1) << n;                                                               \
        OMP_FOR for (idx_t i = 0; i < dim; i++) {                                                                \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t j = i ^ mf;                                                                                    \
            if (i > j) continue;                                                                                 \
            int p = (num_y + 2 * __builtin_popcountll(i & my) + 2 * __builtin_popcountll(i & mz)) & 3;          \
            c##SUF c = mk##SUF(POLAR_RE[p], POLAR_IM[p]);                                                        \
            if (i == j) {                                                                                        \
                qs[i] = qs[i] * c;                                                                               \
            } else {                                                                                             \
                c##SUF tmp = qs[j];                                                                              \
                qs[j] = qs[i] * c;                                                                               \
                qs[i] = tmp / c;                                                                                 \
            }                                                                                                    \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ApplyTerms: cpu_vector_core_policy.cpp:133-161; out = H qs (out must be zeroed by the caller). */        \
    void orc_apply_terms_##SUF(const T *qs_, T *out_, int n, int nt, const idx_t *mx, const idx_t *my,         \
                               const idx_t *mz, const int *ny, const double *coeff) {                           \
        const c##SUF *qs = (const c##SUF *)qs_;                                                                  \
        c##SUF *out = (c##SUF *)out_;                                                                            \
        idx_t dim = ((idx_t)1) << n;                                                                             \
        for (int t = 0; t < nt; t++) {                                                                           \
            idx_t mf = mx[t] | my[t];                                                                            \
            T coef = (T)coeff[t];                                                                                  \
            OMP_FOR for (idx_t i = 0; i < dim; i++) {                                                            \
                idx_t j = i ^ mf;                                                                                \
                if (i > j) continue;                                                                             \
                int p = (ny[t] + 2 * __builtin_popcountll(i & my[t]) + 2 * __builtin_popcountll(i & mz[t])) & 3; \
                c##SUF c = mk##SUF(POLAR_RE[p], POLAR_IM[p]);                                                    \
                out[j] += qs[i] * coef * c;                                                                        \
                if (i != j) out[i] += qs[j] * coef / c;                                                            \
            }                                                                                                    \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ExpectationOfTerms: cpu_vector_core_policy.cpp:212-261 (one reduction pass per term). */                \
    void orc_expectation_of_terms_##SUF(const T *bra_, const T *ket_, int n, int nt, const idx_t *mx,          \
                                        const idx_t *my, const idx_t *mz, const int *ny, const double *coeff,   \
                                        double *out) {                                                           \
        const c##SUF *bra = (const c##SUF *)bra_, *ket = (const c##SUF *)ket_;                                   \
        idx_t dim = ((idx_t)1) << n;                                                                             \
        double tot_re = 0, tot_im = 0;                                                                           \
        for (int t = 0; t < nt; t++) {                                                                           \
            idx_t mf = mx[t] | my[t];                                                                            \
            T coef = (T)coeff[t];                                                                                  \
            T acc_re = 0, acc_im = 0;                                                                            \
            OMP_RED for (idx_t i = 0; i < dim; i++) {                                                            \
                idx_t j = i ^ mf;                                                                                \
                if (i > j) continue;                                                                             \
                int p = (ny[t] + 2 * __builtin_popcountll(i & my[t]) + 2 * __builtin_popcountll(i & mz[t])) & 3; \
                c##SUF c = mk##SUF(POLAR_RE[p], POLAR_IM[p]);                                                    \
                c##SUF tmp = conj(bra[j]) * ket[i] * coef * c;                                                     \
                if (i != j) tmp += conj(bra[i]) * ket[j] * coef / c;                                               \
                acc_re += creal(tmp);                                                                            \
                acc_im += cimag(tmp);                                                                            \
            }                                                                                                    \
            tot_re += acc_re;                                                                                    \
            tot_im += acc_im;                                                                                    \
        }                                                                                                        \
        out[0] = tot_re;                                                                                         \
        out[1] = tot_im;                                                                                         \
    }                                                                                                            \
                                                                                                                 \
    /* Vdot: cpu_vector_core_dot_like.cpp:33-53, <bra|ket>. */                                                 \
    void orc_vdot_##SUF(const T *bra_, const T *ket_, int n, double *out) {                                    \
        const c##SUF *bra = (const c##SUF *)bra_, *ket = (const c##SUF *)ket_;                                   \
        idx_t dim = ((idx_t)1) << n;                                                                             \
        T acc_re = 0, acc_im = 0;                                                                                \
        OMP_RED for (idx_t i = 0; i < dim; i++) {                                                                \
            c##SUF t = conj(bra[i]) * ket[i];                                                                    \
            acc_re += creal(t);                                                                                  \
            acc_im += cimag(t);                                                                                  \
        }                                                                                                        \
        out[0] = acc_re;                                                                                         \
        out[1] = acc_im;                                                                                         \
    }                                                                                                            \
                                                                                                                 \
    /* ExpectDiffSingleQubitMatrix / ExpectDiffTwoQubitsMatrix / ExpectDiffNQubitsMatrix:                      \
     * cpu_vector_core_gate_expect.cpp:244-375 and 128-240: sum over groups of conj(bra) * (m ket). */          \
    void orc_expect_diff_matrix_##SUF(const T *bra_, const T *ket_, int n, const int *objs, int k, idx_t ctrl, \
                                      const double *m, double *out) {                                            \
        const c##SUF *bra = (const c##SUF *)bra_, *ket = (const c##SUF *)ket_;                                   \
        int md = 1 << k;                                                                                         \
        idx_t om[64];                                                                                            \
        c##SUF g[64 * 64];                                                                                       \
        for (int a = 0; a < md; a++) {                                                                           \
            idx_t mk = 0;                                                                                        \
            for (int b = 0; b < k; b++)                                                                          \
                if (a >> b & 1) mk |= ((idx_t)1) << objs[b];                                                     \
            om[a] = mk;                                                                                          \
        }                                                                                                        \
        for (int t = 0; t < md * md; t++) g[t] = mk##SUF(m[2 * t], m[2 * t + 1]);                                \
        idx_t all = om[md - 1], dim = ((idx_t)1) << n;                                                           \
        T acc_re = 0, acc_im = 0;                                                                                \
        OMP_RED for (idx_t l = 0; l < dim; l++) {                                                                \
            if ((l & ctrl) != ctrl || (l & all) != 0) continue;                                                  \
            c##SUF v[64];                                                                                        \
            for (int a = 0; a < md; a++) v[a] = ket[om[a] | l];                                                  \
            c##SUF res = 0;                                                                                      \
            for (int a = 0; a < md; a++) {                                                                       \
                c##SUF t = 0;                                                                                    \
                for (int b = 0; b < md; b++) t += g[a * md + b] * v[b];                                          \
                res += conj(bra[om[a] | l]) * t;                                                                 \
            }                                                                                                    \
            acc_re += creal(res);                                                                                \
            acc_im += cimag(res);                                                                                \
        }                                                                                                        \
        out[0] = acc_re;                                                                                         \
        out[1] = acc_im;                                                                                         \
    }                                                                                                            \
                                                                                                                 \
    /* ExpectDiffRPS: cpu_vector_core_gate_expect.cpp:32-126 -> <bra| d/dval exp(-i val/2 P) |ket>. */          \
    void orc_expect_diff_rps_##SUF(const T *bra_, const T *ket_, int n, idx_t mx, idx_t my, idx_t mz,          \
                                   int num_y, idx_t ctrl, double val, double *out) {                            \
        const c##SUF *bra = (const c##SUF *)bra_, *ket = (const c##SUF *)ket_;                                   \
        T a = (T)(-sin(val / 2) / 2), b = (T)(cos(val / 2) / 2);                                                 \
        idx_t mf = mx | my, dim = ((idx_t)1) << n;                                                               \
        T acc_re = 0, acc_im = 0;                                                                                \
        OMP_RED for (idx_t i = 0; i < dim; i++) {                                                                \
            if ((i & ctrl) != ctrl) continue;                                                                    \
            idx_t j = i ^ mf;                                                                                    \
            if (i > j) continue;                                                                                 \
            int p = (num_y + 2 * __builtin_popcountll(i & my) + 2 * __builtin_popcountll(i & mz)) & 3;          \
            c##SUF c = mk##SUF(POLAR_RE[p], POLAR_IM[p]);                                                        \
            c##SUF res;                                                                                          \
            if (i == j) {                                                                                        \
                res = conj(bra[i]) * ket[i] * (a - (c##SUF)I * b * c);                                           \
            } else {                                                                                             \
                res = conj(bra[i]) * (ket[i] * a - (c##SUF)I * ket[j] * b / c);                                  \
                res += conj(bra[j]) * (ket[j] * a - (c##SUF)I * ket[i] * b * c);                                 \
            }                                                                                                    \
            acc_re += creal(res);                                                                                \
            acc_im += cimag(res);                                                                                \
        }                                                                                                        \
        out[0] = acc_re;                                                                                         \
        out[1] = acc_im;                                                                                         \
    }                                                                                                            \
                                                                                                                 \
    /* GetCumulativeProbs: cpu_vector_core_policy.cpp:293-312 (serial prefix sum, last entry forced to 1). */  \
    void orc_cumulative_probs_##SUF(const T *qs_, int n, T *prob) {                                            \
        const c##SUF *qs = (const c##SUF *)qs_;                                                                  \
        idx_t dim = ((idx_t)1) << n;                                                                             \
        prob[0] = creal(qs[0]) * creal(qs[0]) + cimag(qs[0]) * cimag(qs[0]);                                     \
        for (idx_t i = 1; i < dim; i++)                                                                          \
            prob[i] = creal(qs[i]) * creal(qs[i]) + cimag(qs[i]) * cimag(qs[i]) + prob[i - 1];                   \
        prob[dim - 1] = 1.0;                                                                                     \
    }                                                                                                            \
                                                                                                                 \
    /* Csr_Dot_Vec (ccsrc/include/core/sparse/algo.h:160-176): out = A vec, row sums in T. */                 \
    void orc_csr_dot_vec_##SUF(const int64_t *indptr, const int64_t *indices, const T *data_, idx_t dim,      \
                               const T *vec_, T *out_) {                                                         \
        const c##SUF *data = (const c##SUF *)data_, *vec = (const c##SUF *)vec_;                                 \
        c##SUF *out = (c##SUF *)out_;                                                                            \
        OMP_FOR for (idx_t i = 0; i < dim; i++) {                                                                \
            c##SUF sum = mk##SUF(0, 0);                                                                          \
            for (int64_t j = indptr[i]; j < indptr[i + 1]; j++) sum += data[j] * vec[indices[j]];               \
            out[i] = sum;                                                                                        \
        }                                                                                                        \
    }                                                                                                            \
                                                                                                                 \
    /* ExpectationOfCsr (algo.h:178-200): sum_i conj(bra_i) (A ket)_i. */                                      \
    void orc_expectation_of_csr_##SUF(const int64_t *indptr, const int64_t *indices, const T *data_, idx_t dim, \
                                      const T *bra_, const T *ket_, double *out) {                              \
        const c##SUF *data = (const c##SUF *)data_, *bra = (const c##SUF *)bra_, *ket = (const c##SUF *)ket_;   \
        T acc_re = 0, acc_im = 0;                                                                                \
        OMP_RED for (idx_t i = 0; i < dim; i++) {                                                                \
            c##SUF sum = mk##SUF(0, 0);                                                                          \
            for (int64_t j = indptr[i]; j < indptr[i + 1]; j++) sum += data[j] * ket[indices[j]];               \
            c##SUF t = conj(bra[i]) * sum;                                                                       \
            acc_re += creal(t);                                                                                  \
            acc_im += cimag(t);                                                                                  \
        }                                                                                                        \
        out[0] = acc_re;                                                                                         \
        out[1] = acc_im;                                                                                         \
    }                                                                                                            \
                                                                                                                 \
    /* LowerBound: cpu_vector_core_policy.cpp:315-332 (merge of sorted uniforms into the cdf). */              \
    void orc_lower_bound_##SUF(const T *cum, idx_t dim, const T *sampled, idx_t ns, uint32_t *out) {          \
        idx_t s = 0, d = 0;                                                                                      \
        while (s < ns) {                                                                                         \
            if (sampled[s] < cum[d]) {                                                                           \
                out[s] = (uint32_t)d;                                                                            \
                s++;                                                                                             \
            } else {                                                                                             \
                d++;                                                                                             \
            }                                                                                                    \
        }                                                                                                        \
    }

DEFINE_ORACLE(double, d)
DEFINE_ORACLE(float, f)

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
