// Register kernels of the fused tile passes (sm_100a).
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

namespace mqb {
namespace reg {

template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename V>
__device__ __forceinline__ V cmadd(V a, V b, V c) {  // a * b + c
    V r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
    r.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
    return r;
}
template <typename V>
__device__ __forceinline__ V cconj(V a) {
    a.y = -a.y;
    return a;
}
template <typename V, typename R>
__device__ __forceinline__ V rlin(R a, V x, R b, V y) {  // a x + b y, a and b real
    V r;
    r.x = fma(a, x.x, b * y.x);
    r.y = fma(a, x.y, b * y.y);
    return r;
}
template <typename V, typename R>
__device__ __forceinline__ V rxl(R a, V x, R b, V y) {  // a x + i b y, a and b real
    V r;
    r.x = fma(a, x.x, -b * y.y);
    r.y = fma(a, x.y, b * y.x);
    return r;
}
template <typename V>
__device__ __forceinline__ decltype(V::x) redot(V l, V y) {  // Re(conj(l) y)
    return fma(l.x, y.x, l.y * y.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Register index j takes part in a gate on position P with single control position C (C < 0: none).
template <int P, int C>
__device__ __forceinline__ constexpr bool active(int j) {
    return !((j >> P) & 1) && (C < 0 || ((j >> (C < 0 ? 0 : C)) & 1));
}
template <int C>
__device__ __forceinline__ constexpr bool ctl_on(int j) {
    return C < 0 || ((j >> (C < 0 ? 0 : C)) & 1);
}

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

// ============================================================================ forward (U psi)

template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_dense1(V (&v)[1 << RB], const V *M) {
    const V m00 = M[0], m01 = M[1], m10 = M[2], m11 = M[3];
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = cmadd(m00, a, cmul(m01, b));
        v[j | (1 << P)] = cmadd(m10, a, cmul(m11, b));
    }
}

template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_real1(V (&v)[1 << RB], const V *M) {
    const auto m00 = M[0].x, m01 = M[1].x, m10 = M[2].x, m11 = M[3].x;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = rlin(m00, a, m01, b);
        v[j | (1 << P)] = rlin(m10, a, m11, b);
    }
}

// [[a, i b], [i b, a]] with a, b real (RX)
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_rxl1(V (&v)[1 << RB], const V *M) {
    const auto a = M[0].x, b = M[1].y;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        const V x0 = v[j], x1 = v[j | (1 << P)];
        v[j] = rxl(a, x0, b, x1);
        v[j | (1 << P)] = rxl(a, x1, b, x0);
    }
}

template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_x1(V (&v)[1 << RB]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        const V a = v[j];
        v[j] = v[j | (1 << P)];
        v[j | (1 << P)] = a;
    }
}

template <typename V, int RB, int P, int C>
__device__ __forceinline__ void f_diag1(V (&v)[1 << RB], V d0, V d1) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<C>(j)) continue;
        v[j] = cmul(v[j], ((j >> P) & 1) ? d1 : d0);
    }
}

template <typename V, int RB, int C>
__device__ __forceinline__ void f_scale(V (&v)[1 << RB], V d) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<C>(j)) continue;
        v[j] = cmul(v[j], d);
    }
}

// diagonal on two register positions: P carries matrix bit 0, Q matrix bit 1
template <typename V, int RB, int P, int Q>
__device__ __forceinline__ void f_diag2(V (&v)[1 << RB], const V *M) {
    const V d0 = M[0], d1 = M[1], d2 = M[2], d3 = M[3];
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        const int r = ((j >> P) & 1) | (((j >> Q) & 1) << 1);
        v[j] = cmul(v[j], r == 0 ? d0 : r == 1 ? d1 : r == 2 ? d2 : d3);
    }
}

// dense 4x4: P carries matrix bit 0, Q matrix bit 1; MASK (runtime) = register controls
template <typename V, int RB, int P, int Q, bool GEN>
__device__ __forceinline__ void f_dense2(V (&v)[1 << RB], const V *M, uint32_t mask) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (((j >> P) & 1) || ((j >> Q) & 1)) continue;
        if (GEN && (uint32_t(j) & mask) != mask) continue;
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
// acc[a][h] += Re<lambda_h | dU/d angle_a | psi'> over the thread's amplitudes, psi' = U^dag psi,
// lambda_h taken before its own uncompute.  G: gradient-angle mask (compile time), or -1 for the
// runtime mask gm.  Derivative matrices follow M in the table: dM_a = M + (1 + a) * size(M).

template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_dense1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, int gm, uint32_t mask,
                                         decltype(V::x) (&acc)[3][NH]) {
    const V a00 = cconj(M[0]), a01 = cconj(M[2]), a10 = cconj(M[1]), a11 = cconj(M[3]);
    const int gmask = G >= 0 ? G : gm;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        if (C == -2 && (uint32_t(j) & mask) != mask) continue;   // generic: runtime control mask
        constexpr int bit = 1 << P;
        const V w0 = cmadd(a00, v[j], cmul(a01, v[j | bit])), w1 = cmadd(a10, v[j], cmul(a11, v[j | bit]));
        v[j] = w0;
        v[j | bit] = w1;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!((gmask >> an) & 1)) continue;
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

template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_real1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                        decltype(V::x) (&acc)[3][NH]) {
    const auto a00 = M[0].x, a01 = M[2].x, a10 = M[1].x, a11 = M[3].x;   // U^dag = U^T
    decltype(V::x) d00 = 0, d01 = 0, d10 = 0, d11 = 0;
    if (G & 1) {
        d00 = M[4].x;
        d01 = M[5].x;
        d10 = M[6].x;
        d11 = M[7].x;
    }
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        constexpr int bit = 1 << P;
        const V w0 = rlin(a00, v[j], a01, v[j | bit]), w1 = rlin(a10, v[j], a11, v[j | bit]);
        v[j] = w0;
        v[j | bit] = w1;
        if (G & 1) {
            const V y0 = rlin(d00, w0, d01, w1), y1 = rlin(d10, w0, d11, w1);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y0) + redot(l[h][j | bit], y1);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V x0 = l[h][j], x1 = l[h][j | bit];
            l[h][j] = rlin(a00, x0, a01, x1);
            l[h][j | bit] = rlin(a10, x0, a11, x1);
        }
    }
}

// U = [[a, i b], [i b, a]]: U^dag = [[a, -i b], [-i b, a]]; dU has the same form
template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_rxl1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                       decltype(V::x) (&acc)[3][NH]) {
    const auto a = M[0].x, nb = -M[1].y;
    decltype(V::x) da = 0, db = 0;
    if (G & 1) {
        da = M[4].x;
        db = M[5].y;
    }
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!active<P, C>(j)) continue;
        constexpr int bit = 1 << P;
        const V x0 = v[j], x1 = v[j | bit];
        const V w0 = rxl(a, x0, nb, x1), w1 = rxl(a, x1, nb, x0);
        v[j] = w0;
        v[j | bit] = w1;
        if (G & 1) {
            const V y0 = rxl(da, w0, db, w1), y1 = rxl(da, w1, db, w0);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y0) + redot(l[h][j | bit], y1);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V z0 = l[h][j], z1 = l[h][j | bit];
            l[h][j] = rxl(a, z0, nb, z1);
            l[h][j | bit] = rxl(a, z1, nb, z0);
        }
    }
}

template <typename V, int RB, int NH, int P, int C>
__device__ __forceinline__ void b_x1(V (&v)[1 << RB], V (&l)[NH][1 << RB]) {
    f_x1<V, RB, P, C>(v);
#pragma unroll
    for (int h = 0; h < NH; ++h) f_x1<V, RB, P, C>(l[h]);
}

// diagonal with target on register P: entries (d0, d1), derivative entries (e0, e1)
template <typename V, int RB, int NH, int P, int C, int G>
__device__ __forceinline__ void b_diag1(V (&v)[1 << RB], V (&l)[NH][1 << RB], V d0, V d1, V e0, V e1,
                                        decltype(V::x) (&acc)[3][NH]) {
    const V c0 = cconj(d0), c1 = cconj(d1);
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<C>(j)) continue;
        const bool hi = (j >> P) & 1;
        const V w = cmul(v[j], hi ? c1 : c0);
        v[j] = w;
        if (G & 1) {
            const V y = cmul(hi ? e1 : e0, w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], hi ? c1 : c0);
    }
}

template <typename V, int RB, int NH, int C, int G>
__device__ __forceinline__ void b_scale(V (&v)[1 << RB], V (&l)[NH][1 << RB], V d, V e,
                                        decltype(V::x) (&acc)[3][NH]) {
    const V c = cconj(d);
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<C>(j)) continue;
        const V w = cmul(v[j], c);
        v[j] = w;
        if (G & 1) {
            const V y = cmul(e, w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c);
    }
}

template <typename V, int RB, int NH, int P, int Q, int G>
__device__ __forceinline__ void b_diag2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                        decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        const int r = ((j >> P) & 1) | (((j >> Q) & 1) << 1);
        const V c = cconj(M[r]);
        const V w = cmul(v[j], c);
        v[j] = w;
        if (G & 1) {
            const V y = cmul(M[4 + r], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c);
    }
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
