// Register-op dispatch of the precompiled fused tile kernels (sm_100a).
//
// Inside a register stage every thread holds the 2^RB amplitudes of the tile whose tile-local
// indices differ in the stage's RB register bits.  A gate of the stage is resolved on the host
// into one register code (RegCode in mqb_internal.h) naming its structure and the register
// positions it touches: target position P (Q for a second target), the position C of a single
// control among the register bits.  The device code below has one switch case per code, so in
// every case the register indices, the control pattern and the gradient angles are compile-time
// constants: the amplitude loops carry no runtime predicate, select or branch.  Ops the codes do
// not specialise (several register controls, controlled two-qubit gates) take generic cases
// whose control mask is tested at run time.
//
// Math per amplitude (FP32 for complex64, FP64 for complex128): dense 2x2 8 FMA-class
// instructions, real 2x2 and RX-like 4, diagonal 4, X 0 (register moves), dense 4x4 16.
#ifndef MQB_REGOPS_CUH_
#define MQB_REGOPS_CUH_

#include <cuda_runtime.h>

#include "kernels.cuh"

#include "regmath.cuh"

namespace mqb {
namespace reg {

// Bit of an off-register diagonal target: src 1 thread (tile-local bit of Lt), 2 outside (global
// qubit of base), 3 absent (0).  src 0 (register position) only occurs in generic ops.
__device__ __forceinline__ int off_bit(int src, int val, uint32_t Lt, uint64_t base) {
    if (src == 1) return int((Lt >> val) & 1u);
    if (src == 2) return int((base >> val) & 1u);
    return 0;
}
__device__ __forceinline__ int any_bit(int src, int val, int j, uint32_t Lt, uint64_t base) {
    if (src == 0) return (j >> val) & 1;
    return off_bit(src, val, Lt, base);
}
// Diagonal entry index of a gate whose targets are all off the registers.
__device__ __forceinline__ int scale_index(const StageOp &so, uint32_t Lt, uint64_t base) {
    return off_bit(so.dsrc[0], so.dval[0], Lt, base) | (off_bit(so.dsrc[1], so.dval[1], Lt, base) << 1);
}

// ================================================================= forward (U psi)
// Interpreter forms: matrices read from the pass's matrix table M; C = single register control
// position (-1: none).
__host__ __device__ constexpr unsigned cmask(int c) { return c < 0 ? 0u : (1u << c); }

template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_dense1(V (&v)[1 << RB], const V *M) {
    j_dense1<V, RB, P, cmask(C)>(v, M[0], M[1], M[2], M[3]);
}
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_real1(V (&v)[1 << RB], const V *M) {
    j_real1<V, RB, P, cmask(C)>(v, M[0].x, M[1].x, M[2].x, M[3].x);
}
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_rxl1(V (&v)[1 << RB], const V *M) {
    j_rxl1<V, RB, P, cmask(C)>(v, M[0].x, M[1].y);
}
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_x1(V (&v)[1 << RB]) {
    j_x1<V, RB, P, cmask(C)>(v);
}
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_diag1(V (&v)[1 << RB], V d0, V d1) {
    j_diag1<V, RB, P, cmask(C)>(v, d0, d1);
}
template <typename V, int RB, int C>
__device__ __forceinline__ void f_scale(V (&v)[1 << RB], V d) {
    j_scale<V, RB, cmask(C)>(v, d);
}
template <typename V, int RB, int P, int Q>
__device__ __forceinline__ void f_diag2(V (&v)[1 << RB], const V *M) {
    j_diag2<V, RB, P, Q, 0u>(v, M[0], M[1], M[2], M[3]);
}

// dense 4x4 with a runtime register control mask (GEN) or none
template <typename V, int RB, int P, int Q, bool GEN>
__device__ __forceinline__ void f_dense2(V (&v)[1 << RB], const V *M, unsigned mask) {
    if constexpr (!GEN) {
        j_dense2<V, RB, P, Q, 0u>(v, M);
    } else {
#pragma unroll
        for (int j = 0; j < (1 << RB); ++j) {
            if (((j >> P) & 1) || ((j >> Q) & 1)) continue;
            if ((unsigned(j) & mask) != mask) continue;
            const int id[4] = {j, j | (1 << P), j | (1 << Q), j | (1 << P) | (1 << Q)};
            V x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) x[r] = v[id[r]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V s = cmul(M[r * 4], x[0]);
#pragma unroll
                for (int c = 1; c < 4; ++c) s = cmadd(M[r * 4 + c], x[c], s);
                v[id[r]] = s;
            }
        }
    }
}

// generic dense 2x2 with a register control mask
template <typename V, int RB, int P>
__device__ __forceinline__ void g_dense1(V (&v)[1 << RB], const V *M, uint32_t mask) {
    const V m00 = M[0], m01 = M[1], m10 = M[2], m11 = M[3];
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (((j >> P) & 1) || (uint32_t(j) & mask) != mask) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = cmadd(m00, a, cmul(m01, b));
        v[j | (1 << P)] = cmadd(m10, a, cmul(m11, b));
    }
}

// generic diagonal (1 or 2 targets anywhere, register control mask)
template <typename V, int RB>
__device__ __forceinline__ void g_diag(V (&v)[1 << RB], const V *M, const StageOp &so, uint32_t Lt, uint64_t base) {
    const uint32_t mask = so.rctrl;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((uint32_t(j) & mask) != mask) continue;
        const int r = any_bit(so.dsrc[0], so.dval[0], j, Lt, base) | (any_bit(so.dsrc[1], so.dval[1], j, Lt, base) << 1);
        v[j] = cmul(v[j], M[r]);
    }
}

#define MQB_P5(X, B) X(B + 0, 0) X(B + 1, 1) X(B + 2, 2) X(B + 3, 3) X(B + 4, 4)
#define MQB_PQ5(X, B, P) X(B + 0, P, 0) X(B + 1, P, 1) X(B + 2, P, 2) X(B + 3, P, 3) X(B + 4, P, 4)
#define MQB_PQ25(X, B) MQB_PQ5(X, B, 0) MQB_PQ5(X, B + 5, 1) MQB_PQ5(X, B + 10, 2) MQB_PQ5(X, B + 15, 3) \
    MQB_PQ5(X, B + 20, 4)

// One gate of a forward stage; the code says which register kernel applies.
template <typename V, int RB>
__device__ __forceinline__ void fwd_op(int code, V (&v)[1 << RB], const V *M, const StageOp &so, uint32_t Lt,
                                       uint64_t base) {
    switch (code) {
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) f_dense1<V, RB, P, -1>(v, M); \
        break;
        MQB_P5(X1, RC_DENSE1)
#undef X1
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) f_real1<V, RB, P, -1>(v, M); \
        break;
        MQB_P5(X1, RC_REAL1)
#undef X1
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) f_rxl1<V, RB, P, -1>(v, M); \
        break;
        MQB_P5(X1, RC_RXL1)
#undef X1
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) f_x1<V, RB, P, -1>(v); \
        break;
        MQB_P5(X1, RC_X1)
#undef X1
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) f_diag1<V, RB, P, -1>(v, M[0], M[1]); \
        break;
        MQB_P5(X1, RC_DIAG1)
#undef X1
        case RC_SCALE:
            f_scale<V, RB, -1>(v, M[scale_index(so, Lt, base)]);
            break;
#define X2(cd, P, C) \
    case cd:         \
        if constexpr (P < RB && C < RB && P != C) f_dense1<V, RB, P, C>(v, M); \
        break;
        MQB_PQ25(X2, RC_DENSE1C)
#undef X2
#define X2(cd, P, C) \
    case cd:         \
        if constexpr (P < RB && C < RB && P != C) f_x1<V, RB, P, C>(v); \
        break;
        MQB_PQ25(X2, RC_X1C)
#undef X2
#define X2(cd, P, C) \
    case cd:         \
        if constexpr (P < RB && C < RB && P != C) f_diag1<V, RB, P, C>(v, M[0], M[1]); \
        break;
        MQB_PQ25(X2, RC_DIAG1C)
#undef X2
#define X1(cd, C) \
    case cd:      \
        if constexpr (C < RB) f_scale<V, RB, C>(v, M[scale_index(so, Lt, base)]); \
        break;
        MQB_P5(X1, RC_SCALEC)
#undef X1
#define X2(cd, P, Q) \
    case cd:         \
        if constexpr (P < RB && Q < RB && P != Q) f_diag2<V, RB, P, Q>(v, M); \
        break;
        MQB_PQ25(X2, RC_DIAG2)
#undef X2
#define X2(cd, K, P)                                                                 \
    case cd:                                                                         \
        if constexpr (K < 2 && P < RB) {                                             \
            const int b = off_bit(so.dsrc[1 - K], so.dval[1 - K], Lt, base);         \
            if (K == 0) f_diag1<V, RB, P, -1>(v, M[b << 1], M[1 | (b << 1)]);        \
            else f_diag1<V, RB, P, -1>(v, M[b], M[2 | b]);                           \
        }                                                                            \
        break;
        MQB_PQ5(X2, RC_DIAG2S, 0) MQB_PQ5(X2, RC_DIAG2S + 5, 1)
#undef X2
#define X2(cd, P, Q) \
    case cd:         \
        if constexpr (P < RB && Q < RB && P != Q) f_dense2<V, RB, P, Q, false>(v, M, 0u); \
        break;
        MQB_PQ25(X2, RC_DENSE2)
#undef X2
#define X1(cd, P) \
    case cd:      \
        if constexpr (P < RB) g_dense1<V, RB, P>(v, M, so.rctrl); \
        break;
        MQB_P5(X1, RC_GDENSE1)
#undef X1
        case RC_GDIAG:
            g_diag<V, RB>(v, M, so, Lt, base);
            break;
#define X2(cd, P, Q) \
    case cd:         \
        if constexpr (P < RB && Q < RB && P != Q) f_dense2<V, RB, P, Q, true>(v, M, so.rctrl); \
        break;
        MQB_PQ25(X2, RC_GDENSE2)
#undef X2
        default:
            break;
    }
}

// ============================================== backward (psi <- U^dag psi, gradients, lambda)
// Interpreter forms over the register math of regmath.cuh: U and dU_a = M + (1 + a) size(M)
// read from the matrix table.  C = -2 marks a runtime register control mask, G = -1 a runtime
// gradient mask (the generic codes).

template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_dense1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, int gm, uint32_t mask,
                                         decltype(V::x) (&acc)[3][NH]) {
    const V a00 = cconj(M[0]), a01 = cconj(M[2]), a10 = cconj(M[1]), a11 = cconj(M[3]);
    if constexpr (C >= -1 && G >= 0) {
        V d[3][4];
#pragma unroll
        for (int an = 0; an < 3; ++an)
#pragma unroll
            for (int e = 0; e < 4; ++e) d[an][e] = ((G >> an) & 1) ? M[4 + an * 4 + e] : cval<V>(0, 0);
        jb_dense1<V, RB, NH, P, cmask(C), G>(v, l, a00, a01, a10, a11, d, acc);
    } else {
#pragma unroll
        for (int j = 0; j < (1 << RB); ++j) {
            if (((j >> P) & 1) || (uint32_t(j) & mask) != mask) continue;
            constexpr int bit = 1 << P;
            const V w0 = cmadd(a00, v[j], cmul(a01, v[j | bit])), w1 = cmadd(a10, v[j], cmul(a11, v[j | bit]));
            v[j] = w0;
            v[j | bit] = w1;
#pragma unroll
            for (int an = 0; an < 3; ++an) {
                if (!((gm >> an) & 1)) continue;
                const V *d = M + 4 + an * 4;
                const V y0 = cmadd(d[0], w0, cmul(d[1], w1)), y1 = cmadd(d[2], w0, cmul(d[3], w1));
#pragma unroll
                for (int h = 0; h < NH; ++h) acc[an][h] += redot(l[h][j], y0) + redot(l[h][j | bit], y1);
            }
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const V x0 = l[h][j], x1 = l[h][j | bit];
                l[h][j] = cmadd(a00, x0, cmul(a01, x1));
                l[h][j | bit] = cmadd(a10, x0, cmul(a11, x1));
            }
        }
    }
}

template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_real1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                        decltype(V::x) (&acc)[3][NH]) {
    using R = decltype(V::x);
    const R z = 0;
    jb_real1<V, RB, NH, P, cmask(C), G>(v, l, M[0].x, M[2].x, M[1].x, M[3].x, (G & 1) ? M[4].x : z,
                                        (G & 1) ? M[5].x : z, (G & 1) ? M[6].x : z, (G & 1) ? M[7].x : z, acc);
}

template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_rxl1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                       decltype(V::x) (&acc)[3][NH]) {
    using R = decltype(V::x);
    const R z = 0;
    jb_rxl1<V, RB, NH, P, cmask(C), G>(v, l, M[0].x, -M[1].y, (G & 1) ? M[4].x : z, (G & 1) ? M[5].y : z, acc);
}

template <typename V, int RB, int NH, int P, int C>
__device__ __forceinline__ void b_x1(V (&v)[1 << RB], V (&l)[NH][1 << RB]) {
    jb_x1<V, RB, NH, P, cmask(C)>(v, l);
}

// diagonal with target on register P: entries (d0, d1), derivative entries (e0, e1)
template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_diag1(V (&v)[1 << RB], V (&l)[NH][1 << RB], V d0, V d1, V e0, V e1,
                                        decltype(V::x) (&acc)[3][NH]) {
    jb_diag1<V, RB, NH, P, cmask(C), G>(v, l, cconj(d0), cconj(d1), e0, e1, acc);
}

template <typename V, int RB, int NH, int C, int G>
__device__ __forceinline__ void b_scale(V (&v)[1 << RB], V (&l)[NH][1 << RB], V d, V e,
                                        decltype(V::x) (&acc)[3][NH]) {
    jb_scale<V, RB, NH, cmask(C), G>(v, l, cconj(d), e, acc);
}

template <typename V, int RB, int NH, int P, int Q, int G>
__device__ __forceinline__ void b_diag2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                        decltype(V::x) (&acc)[3][NH]) {
    const V c[4] = {cconj(M[0]), cconj(M[1]), cconj(M[2]), cconj(M[3])};
    const V e[4] = {(G & 1) ? M[4] : c[0], (G & 1) ? M[5] : c[0], (G & 1) ? M[6] : c[0], (G & 1) ? M[7] : c[0]};
    jb_diag2<V, RB, NH, P, Q, 0u, G>(v, l, c, e, acc);
}

template <typename V, int RB, int NH, int P, int Q, int G, bool GEN>
__device__ __forceinline__ void b_dense2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, int gm, uint32_t mask,
                                         decltype(V::x) (&acc)[3][NH]) {
    const int gmask = G >= 0 ? G : gm;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (((j >> P) & 1) || ((j >> Q) & 1)) continue;
        if (GEN && (uint32_t(j) & mask) != mask) continue;
        const int id[4] = {j, j | (1 << P), j | (1 << Q), j | (1 << P) | (1 << Q)};
        V w[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            V s = cmul(cconj(M[r]), v[id[0]]);
#pragma unroll
            for (int c = 1; c < 4; ++c) s = cmadd(cconj(M[c * 4 + r]), v[id[c]], s);
            w[r] = s;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) v[id[r]] = w[r];
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!((gmask >> an) & 1)) continue;
            const V *d = M + 16 + an * 16;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V y = cmul(d[r * 4], w[0]);
#pragma unroll
                for (int c = 1; c < 4; ++c) y = cmadd(d[r * 4 + c], w[c], y);
#pragma unroll
                for (int h = 0; h < NH; ++h) acc[an][h] += redot(l[h][id[r]], y);
            }
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            V x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) x[r] = l[h][id[r]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V s = cmul(cconj(M[r]), x[0]);
#pragma unroll
                for (int c = 1; c < 4; ++c) s = cmadd(cconj(M[c * 4 + r]), x[c], s);
                l[h][id[r]] = s;
            }
        }
    }
}

// generic diagonal (targets anywhere, register control mask, runtime gradient mask)
template <typename V, int RB, int NH>
__device__ __forceinline__ void gb_diag(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, const StageOp &so,
                                        uint32_t Lt, uint64_t base, int gm, decltype(V::x) (&acc)[3][NH]) {
    const uint32_t mask = so.rctrl;
    const int ms = so.mat_size;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((uint32_t(j) & mask) != mask) continue;
        const int r = any_bit(so.dsrc[0], so.dval[0], j, Lt, base) | (any_bit(so.dsrc[1], so.dval[1], j, Lt, base) << 1);
        const V c = cconj(M[r]);
        const V w = cmul(v[j], c);
        v[j] = w;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!((gm >> an) & 1)) continue;
            const V y = cmul(M[(1 + an) * ms + r], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[an][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c);
    }
}

// Backward op code: register code * 4 + gradient selector (0: none, 1: angle 0, 2: angles 0-2,
// 3: runtime mask).
template <typename V, int RB, int NH>
__device__ __forceinline__ void bwd_op(int bcode, V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                       const StageOp &so, uint32_t Lt, uint64_t base, int gm,
                                       decltype(V::x) (&acc)[3][NH]) {
    switch (bcode) {
#define B1(cd, P)                                                                                        \
    case (cd) * 4 + 0:                                                                                   \
        if constexpr (P < RB) b_dense1<V, RB, NH, P, -1, 0>(v, l, M, 0, 0u, acc);                        \
        break;                                                                                           \
    case (cd) * 4 + 1:                                                                                   \
        if constexpr (P < RB) b_dense1<V, RB, NH, P, -1, 1>(v, l, M, 0, 0u, acc);                        \
        break;                                                                                           \
    case (cd) * 4 + 2:                                                                                   \
        if constexpr (P < RB) b_dense1<V, RB, NH, P, -1, 7>(v, l, M, 0, 0u, acc);                        \
        break;                                                                                           \
    case (cd) * 4 + 3:                                                                                   \
        if constexpr (P < RB) b_dense1<V, RB, NH, P, -1, -1>(v, l, M, gm, 0u, acc);                      \
        break;
        MQB_P5(B1, RC_DENSE1)
#undef B1
#define B1(cd, P)                                                        \
    case (cd) * 4 + 0:                                                   \
        if constexpr (P < RB) b_real1<V, RB, NH, P, -1, 0>(v, l, M, acc); \
        break;                                                           \
    case (cd) * 4 + 1:                                                   \
        if constexpr (P < RB) b_real1<V, RB, NH, P, -1, 1>(v, l, M, acc); \
        break;
        MQB_P5(B1, RC_REAL1)
#undef B1
#define B1(cd, P)                                                       \
    case (cd) * 4 + 0:                                                  \
        if constexpr (P < RB) b_rxl1<V, RB, NH, P, -1, 0>(v, l, M, acc); \
        break;                                                          \
    case (cd) * 4 + 1:                                                  \
        if constexpr (P < RB) b_rxl1<V, RB, NH, P, -1, 1>(v, l, M, acc); \
        break;
        MQB_P5(B1, RC_RXL1)
#undef B1
#define B1(cd, P)                                      \
    case (cd) * 4 + 0:                                 \
        if constexpr (P < RB) b_x1<V, RB, NH, P, -1>(v, l); \
        break;
        MQB_P5(B1, RC_X1)
#undef B1
#define B1(cd, P)                                                                                \
    case (cd) * 4 + 0:                                                                           \
        if constexpr (P < RB) b_diag1<V, RB, NH, P, -1, 0>(v, l, M[0], M[1], M[0], M[0], acc);   \
        break;                                                                                   \
    case (cd) * 4 + 1:                                                                           \
        if constexpr (P < RB) b_diag1<V, RB, NH, P, -1, 1>(v, l, M[0], M[1], M[2], M[3], acc);   \
        break;
        MQB_P5(B1, RC_DIAG1)
#undef B1
        case RC_SCALE * 4 + 0: {
            const int r = scale_index(so, Lt, base);
            b_scale<V, RB, NH, -1, 0>(v, l, M[r], M[r], acc);
        } break;
        case RC_SCALE * 4 + 1: {
            const int r = scale_index(so, Lt, base);
            b_scale<V, RB, NH, -1, 1>(v, l, M[r], M[so.mat_size + r], acc);
        } break;
#define B2(cd, P, C)                                                                                      \
    case (cd) * 4 + 0:                                                                                    \
        if constexpr (P < RB && C < RB && P != C) b_dense1<V, RB, NH, P, C, 0>(v, l, M, 0, 0u, acc);       \
        break;                                                                                            \
    case (cd) * 4 + 1:                                                                                    \
        if constexpr (P < RB && C < RB && P != C) b_dense1<V, RB, NH, P, C, 1>(v, l, M, 0, 0u, acc);       \
        break;
        MQB_PQ25(B2, RC_DENSE1C)
#undef B2
#define B2(cd, P, C)                                                         \
    case (cd) * 4 + 0:                                                       \
        if constexpr (P < RB && C < RB && P != C) b_x1<V, RB, NH, P, C>(v, l); \
        break;
        MQB_PQ25(B2, RC_X1C)
#undef B2
#define B2(cd, P, C)                                                                                          \
    case (cd) * 4 + 0:                                                                                        \
        if constexpr (P < RB && C < RB && P != C) b_diag1<V, RB, NH, P, C, 0>(v, l, M[0], M[1], M[0], M[0], acc); \
        break;                                                                                                \
    case (cd) * 4 + 1:                                                                                        \
        if constexpr (P < RB && C < RB && P != C) b_diag1<V, RB, NH, P, C, 1>(v, l, M[0], M[1], M[2], M[3], acc); \
        break;
        MQB_PQ25(B2, RC_DIAG1C)
#undef B2
#define B1(cd, C)                                                                       \
    case (cd) * 4 + 0:                                                                  \
        if constexpr (C < RB) {                                                         \
            const int r = scale_index(so, Lt, base);                                    \
            b_scale<V, RB, NH, C, 0>(v, l, M[r], M[r], acc);                            \
        }                                                                               \
        break;                                                                          \
    case (cd) * 4 + 1:                                                                  \
        if constexpr (C < RB) {                                                         \
            const int r = scale_index(so, Lt, base);                                    \
            b_scale<V, RB, NH, C, 1>(v, l, M[r], M[so.mat_size + r], acc);              \
        }                                                                               \
        break;
        MQB_P5(B1, RC_SCALEC)
#undef B1
#define B2(cd, P, Q)                                                                           \
    case (cd) * 4 + 0:                                                                         \
        if constexpr (P < RB && Q < RB && P != Q) b_diag2<V, RB, NH, P, Q, 0>(v, l, M, acc);   \
        break;                                                                                 \
    case (cd) * 4 + 1:                                                                         \
        if constexpr (P < RB && Q < RB && P != Q) b_diag2<V, RB, NH, P, Q, 1>(v, l, M, acc);   \
        break;
        MQB_PQ25(B2, RC_DIAG2)
#undef B2
#define B2(cd, K, P)                                                                               \
    case (cd) * 4 + 0:                                                                             \
        if constexpr (K < 2 && P < RB) {                                                           \
            const int b = off_bit(so.dsrc[1 - K], so.dval[1 - K], Lt, base);                       \
            const int i0 = K == 0 ? (b << 1) : b, i1 = K == 0 ? (1 | (b << 1)) : (2 | b);          \
            b_diag1<V, RB, NH, P, -1, 0>(v, l, M[i0], M[i1], M[i0], M[i1], acc);                   \
        }                                                                                          \
        break;                                                                                     \
    case (cd) * 4 + 1:                                                                             \
        if constexpr (K < 2 && P < RB) {                                                           \
            const int b = off_bit(so.dsrc[1 - K], so.dval[1 - K], Lt, base);                       \
            const int i0 = K == 0 ? (b << 1) : b, i1 = K == 0 ? (1 | (b << 1)) : (2 | b);          \
            b_diag1<V, RB, NH, P, -1, 1>(v, l, M[i0], M[i1], M[4 + i0], M[4 + i1], acc);           \
        }                                                                                          \
        break;
        MQB_PQ5(B2, RC_DIAG2S, 0) MQB_PQ5(B2, RC_DIAG2S + 5, 1)
#undef B2
#define B2(cd, P, Q)                                                                                              \
    case (cd) * 4 + 0:                                                                                            \
        if constexpr (P < RB && Q < RB && P != Q) b_dense2<V, RB, NH, P, Q, 0, false>(v, l, M, 0, 0u, acc);       \
        break;                                                                                                    \
    case (cd) * 4 + 1:                                                                                            \
        if constexpr (P < RB && Q < RB && P != Q) b_dense2<V, RB, NH, P, Q, 1, false>(v, l, M, 0, 0u, acc);       \
        break;                                                                                                    \
    case (cd) * 4 + 3:                                                                                            \
        if constexpr (P < RB && Q < RB && P != Q) b_dense2<V, RB, NH, P, Q, -1, false>(v, l, M, gm, 0u, acc);     \
        break;
        MQB_PQ25(B2, RC_DENSE2)
#undef B2
#define B1(cd, P)                                                                      \
    case (cd) * 4 + 3:                                                                 \
        if constexpr (P < RB) b_dense1<V, RB, NH, P, -2, -1>(v, l, M, gm, so.rctrl, acc); \
        break;
        MQB_P5(B1, RC_GDENSE1)
#undef B1
        case RC_GDIAG * 4 + 3:
            gb_diag<V, RB, NH>(v, l, M, so, Lt, base, gm, acc);
            break;
#define B2(cd, P, Q)                                                                                              \
    case (cd) * 4 + 3:                                                                                            \
        if constexpr (P < RB && Q < RB && P != Q) b_dense2<V, RB, NH, P, Q, -1, true>(v, l, M, gm, so.rctrl, acc); \
        break;
        MQB_PQ25(B2, RC_GDENSE2)
#undef B2
        default:
            break;
    }
}

#undef MQB_P5
#undef MQB_PQ5
#undef MQB_PQ25

}  // namespace reg
}  // namespace mqb

#endif
