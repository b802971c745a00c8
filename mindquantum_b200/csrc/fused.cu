// Fused tile passes with register stages (sm_100a).
//
// A fused pass owns K "tile" qubits; every block processes 2^K-amplitude tiles of the state.  A
// tile is staged through shared memory once per pass (coalesced 16-byte global accesses), then
// processed in register stages: each of the 2^TB threads holds the 2^RB amplitudes whose
// tile-local index differs in the stage's RB register bits, and applies all gates of the stage on
// those registers with compile-time register indices (gate targets are register positions
// chosen by the host scheduler).  Between stages the tile is exchanged through shared memory in
// an XOR-swizzled layout, so a pass costs one HBM read + write of the state plus
// (stages + 1) shared-memory round trips, instead of one per gate.
//
// The backward kernel runs the adjoint sweep of a pass on the psi and lambda_h tiles: per gate,
// psi <- U^dag psi, Re<lambda_h| dU/dangle |psi> accumulated in FP64 (warp shuffles into
// per-warp shared slots, one atomicAdd per block and slot), lambda_h <- U^dag lambda_h.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace mqb {

namespace {

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
template <typename V>
__device__ __forceinline__ double redot(V l, V y) {  // Re(conj(l) * y) in FP64
    return double(l.x) * double(y.x) + double(l.y) * double(y.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <typename V>
__device__ __forceinline__ uint32_t swz(uint32_t L) {
    if (sizeof(V) == 8) return L ^ ((L >> 4) & 15u) ^ ((L >> 8) & 15u) ^ ((L >> 12) & 15u);
    return L ^ ((L >> 3) & 7u) ^ ((L >> 6) & 7u) ^ ((L >> 9) & 7u) ^ ((L >> 12) & 7u);
}

__device__ __forceinline__ uint64_t tile_base(const TileGeom &g, uint64_t t) {
    uint64_t base = 0;
    for (int i = 0; i < g.n_out; ++i)
        if (t >> i & 1) base |= uint64_t(1) << g.outside[i];
    return base;
}

__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__device__ __forceinline__ void build_table(uint64_t *tab, const TileGeom &g) {
    const int nh = 1 << (g.K - g.c);
    for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        uint64_t off = 0;
        for (int i = 0; i < g.K - g.c; ++i)
            if (h >> i & 1) off |= uint64_t(1) << g.qbits[g.c + i];
        tab[h] = off;
    }
}

// global (coalesced 16-byte vectors) -> swizzled shared tile.  Every thread moves NV vectors;
// all of its global loads are issued before the first shared store so their latencies overlap.
template <typename V, int NV>
__device__ __forceinline__ void stage_in(V *tile, const V *src, uint64_t base, const uint64_t *tab, int c) {
    constexpr int APV = 16 / sizeof(V);
    constexpr int CH = NV < 8 ? NV : 8;   // vectors in flight per thread (bounded register use)
    const uint32_t lowmask = (1u << c) - 1u;
#pragma unroll
    for (int i0 = 0; i0 < NV; i0 += CH) {
        uint4 buf[CH];
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const uint32_t L = (threadIdx.x + uint32_t(i0 + i) * blockDim.x) * APV;
            const uint64_t gi = base + tab[L >> c] + (L & lowmask);
            buf[i] = __ldcs(reinterpret_cast<const uint4 *>(src + gi));
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const uint32_t L = (threadIdx.x + uint32_t(i0 + i) * blockDim.x) * APV;
            if (APV == 2) {
                const V *pv = reinterpret_cast<const V *>(&buf[i]);
                tile[swz<V>(L)] = pv[0];
                tile[swz<V>(L + 1)] = pv[1];
            } else {
                *reinterpret_cast<uint4 *>(&tile[swz<V>(L)]) = buf[i];
            }
        }
    }
}

template <typename V>
__device__ __forceinline__ void stage_zero(V *tile, uint64_t base, int K) {
    for (int L = threadIdx.x; L < (1 << K); L += blockDim.x) {
        V v;
        v.x = (base == 0 && L == 0) ? 1 : 0;
        v.y = 0;
        tile[swz<V>(L)] = v;
    }
}

template <typename V, int NV>
__device__ __forceinline__ void stage_out(const V *tile, V *dst, uint64_t base, const uint64_t *tab, int c) {
    constexpr int APV = 16 / sizeof(V);
    const uint32_t lowmask = (1u << c) - 1u;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const uint32_t L = (threadIdx.x + uint32_t(i) * blockDim.x) * APV;
        const uint64_t gi = base + tab[L >> c] + (L & lowmask);
        uint4 raw;
        if (APV == 2) {
            V *pv = reinterpret_cast<V *>(&raw);
            pv[0] = tile[swz<V>(L)];
            pv[1] = tile[swz<V>(L + 1)];
        } else {
            raw = *reinterpret_cast<const uint4 *>(&tile[swz<V>(L)]);
        }
        __stcs(reinterpret_cast<uint4 *>(dst + gi), raw);
    }
}

// ----------------------------------------------------------------------------------- register ops
// All register kernels index the thread's amplitude array with compile-time indices; the gate's
// register position P is a template parameter reached through a switch.  CTRL selects the path
// with controls among the register bits (rctrl != 0); the uncontrolled path has no predicates.
template <typename V>
__device__ __forceinline__ V rmul(float a, V x) {  // real scalar (float) times complex
    V r;
    r.x = a * x.x;
    r.y = a * x.y;
    return r;
}
template <typename V>
__device__ __forceinline__ V rmul(double a, V x) {
    V r;
    r.x = a * x.x;
    r.y = a * x.y;
    return r;
}
template <typename V>
__device__ __forceinline__ V rmadd(decltype(V::x) a, V x, V c) {  // a x + c, a real
    V r;
    r.x = fma(a, x.x, c.x);
    r.y = fma(a, x.y, c.y);
    return r;
}

// Matrix entries (row-major 2x2) of U or U^dag.
template <typename V, bool ADJ>
__device__ __forceinline__ void mat2(const V *M, V &m00, V &m01, V &m10, V &m11) {
    if (ADJ) {
        m00 = cconj(M[0]);
        m01 = cconj(M[2]);
        m10 = cconj(M[1]);
        m11 = cconj(M[3]);
    } else {
        m00 = M[0];
        m01 = M[1];
        m10 = M[2];
        m11 = M[3];
    }
}

template <typename V, int RB, int P, bool CTRL>
__device__ __forceinline__ void fw_dense1(V (&v)[1 << RB], V m00, V m01, V m10, V m11, uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        constexpr int bit = 1 << P;
        const V a = v[j], b = v[j | bit];
        v[j] = cmadd(m00, a, cmul(m01, b));
        v[j | bit] = cmadd(m10, a, cmul(m11, b));
    }
}

template <typename V, int RB, int P, bool CTRL>
__device__ __forceinline__ void fw_real1(V (&v)[1 << RB], decltype(V::x) m00, decltype(V::x) m01,
                                         decltype(V::x) m10, decltype(V::x) m11, uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        constexpr int bit = 1 << P;
        const V a = v[j], b = v[j | bit];
        v[j] = rmadd(m00, a, rmul(m01, b));
        v[j | bit] = rmadd(m10, a, rmul(m11, b));
    }
}

template <typename V, int RB, int P, bool CTRL>
__device__ __forceinline__ void fw_perm1(V (&v)[1 << RB], V m01, V m10, bool unit, uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        constexpr int bit = 1 << P;
        const V a = v[j], b = v[j | bit];
        if (unit) {
            v[j] = b;
            v[j | bit] = a;
        } else {
            v[j] = cmul(m01, b);
            v[j | bit] = cmul(m10, a);
        }
    }
}

// X on register position P controlled by register position C (CNOT inside the registers): a
// compile-time permutation of the thread's registers, i.e. register renaming.
template <typename V, int RB, int P, int C>
__device__ __forceinline__ void fw_cswap(V (&v)[1 << RB]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((j >> P & 1) || !(j >> C & 1)) continue;
        const V a = v[j];
        v[j] = v[j | (1 << P)];
        v[j | (1 << P)] = a;
    }
}

template <typename V, int RB>
__device__ __forceinline__ void dispatch_cswap(V (&v)[1 << RB], int p, int c) {
#define MQB_CS(P, C)                                                   \
    case (P * 8 + C):                                                  \
        if constexpr (RB > P && RB > C) fw_cswap<V, RB, P, C>(v);     \
        break;
    switch (p * 8 + c) {
        MQB_CS(0, 1) MQB_CS(0, 2) MQB_CS(0, 3) MQB_CS(0, 4) MQB_CS(1, 0) MQB_CS(1, 2) MQB_CS(1, 3) MQB_CS(1, 4)
        MQB_CS(2, 0) MQB_CS(2, 1) MQB_CS(2, 3) MQB_CS(2, 4) MQB_CS(3, 0) MQB_CS(3, 1) MQB_CS(3, 2) MQB_CS(3, 4)
        MQB_CS(4, 0) MQB_CS(4, 1) MQB_CS(4, 2) MQB_CS(4, 3)
        default: break;
    }
#undef MQB_CS
}

template <typename V, int RB, int P, bool CTRL>
__device__ __forceinline__ void fw_diag1(V (&v)[1 << RB], V d0, V d1, uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        v[j] = cmul(v[j], (j >> P & 1) ? d1 : d0);
    }
}

template <typename V, int RB, bool CTRL>
__device__ __forceinline__ void fw_scale(V (&v)[1 << RB], V d, uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        v[j] = cmul(v[j], d);
    }
}

// Dense two-qubit gate on register positions P0 < P1 (matrix already in position order).
template <typename V, int RB, int P0, int P1, bool ADJ>
__device__ __forceinline__ void reg_dense2(V (&v)[1 << RB], const V (&m)[16], uint32_t rctrl) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((j >> P0 & 1) || (j >> P1 & 1)) continue;
        if ((uint32_t(j) & rctrl) != rctrl) continue;
        const int id[4] = {j, j | (1 << P0), j | (1 << P1), j | (1 << P0) | (1 << P1)};
        V x[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) x[r] = v[id[r]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            V s;
            s.x = 0;
            s.y = 0;
#pragma unroll
            for (int col = 0; col < 4; ++col) s = cmadd(ADJ ? cconj(m[col * 4 + r]) : m[r * 4 + col], x[col], s);
            v[id[r]] = s;
        }
    }
}

// Load a 4x4 matrix with its index bits in register-position order (swap bits 0/1 if needed).
template <typename V>
__device__ __forceinline__ void load_mat4(V (&m)[16], const V *M, bool swap) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int rr = swap ? (((r & 1) << 1) | (r >> 1)) : r;
            const int cc = swap ? (((c & 1) << 1) | (c >> 1)) : c;
            m[r * 4 + c] = M[rr * 4 + cc];
        }
}

template <typename V>
__device__ __forceinline__ int diag_bit(int src, int val, int j, uint32_t Lt, uint64_t base) {
    if (src == 0) return (j >> val) & 1;
    if (src == 1) return int((Lt >> val) & 1u);
    return int((base >> val) & 1u);
}

// Diagonal gate with two targets (generic).
template <typename V, int RB, bool ADJ>
__device__ __forceinline__ void reg_diag2(V (&v)[1 << RB], const StageOp &so, const V *D, uint32_t Lt, uint64_t base) {
    V d[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) d[r] = ADJ ? cconj(D[r]) : D[r];
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((uint32_t(j) & so.rctrl) != so.rctrl) continue;
        const int b0 = diag_bit<V>(so.dsrc[0], so.dval[0], j, Lt, base);
        const int b1 = diag_bit<V>(so.dsrc[1], so.dval[1], j, Lt, base);
        const V dd = b1 ? (b0 ? d[3] : d[2]) : (b0 ? d[1] : d[0]);
        v[j] = cmul(v[j], dd);
    }
}

#define MQB_POS_SWITCH(p, CALL5)  \
    switch (p) {                  \
        case 0: CALL5(0); break;  \
        case 1: CALL5(1); break;  \
        case 2: CALL5(2); break;  \
        case 3: CALL5(3); break;  \
        case 4: CALL5(4); break;  \
        default: break;           \
    }

// One gate of a forward stage.
template <typename V, int RB, bool ADJ>
__device__ __forceinline__ void fwd_gate(V (&v)[1 << RB], const StageOp &so, const V *M, uint32_t Lt, uint64_t base) {
    using R = decltype(V::x);
    const bool ctrl = so.rctrl != 0;
    switch (so.kind) {
        case SK_DENSE1: {
            V m00, m01, m10, m11;
            mat2<V, ADJ>(M, m00, m01, m10, m11);
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) fw_dense1<V, RB, P, true>(v, m00, m01, m10, m11, so.rctrl);                       \
        else fw_dense1<V, RB, P, false>(v, m00, m01, m10, m11, so.rctrl);                           \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_REAL1: {
            const R m00 = M[0].x, m11 = M[3].x;
            const R m01 = ADJ ? M[2].x : M[1].x, m10 = ADJ ? M[1].x : M[2].x;
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) fw_real1<V, RB, P, true>(v, m00, m01, m10, m11, so.rctrl);                        \
        else fw_real1<V, RB, P, false>(v, m00, m01, m10, m11, so.rctrl);                            \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_PERM1:
        case SK_SWAP1: {
            if (so.kind == SK_SWAP1 && so.rc1 >= 0) {   // one control among the register bits
                dispatch_cswap<V, RB>(v, so.p0, so.rc1);
                break;
            }
            const bool unit = so.kind == SK_SWAP1;
            const V m01 = ADJ ? cconj(M[2]) : M[1], m10 = ADJ ? cconj(M[1]) : M[2];
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) fw_perm1<V, RB, P, true>(v, m01, m10, unit, so.rctrl);                            \
        else fw_perm1<V, RB, P, false>(v, m01, m10, unit, so.rctrl);                                \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_DIAG1: {
            const V d0 = ADJ ? cconj(M[0]) : M[0], d1 = ADJ ? cconj(M[1]) : M[1];
            if (so.dsrc[0] == 0) {
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) fw_diag1<V, RB, P, true>(v, d0, d1, so.rctrl);                                    \
        else fw_diag1<V, RB, P, false>(v, d0, d1, so.rctrl);                                        \
    }
                MQB_POS_SWITCH(so.dval[0], MQB_C)
#undef MQB_C
            } else {
                const V d = diag_bit<V>(so.dsrc[0], so.dval[0], 0, Lt, base) ? d1 : d0;
                if (ctrl)
                    fw_scale<V, RB, true>(v, d, so.rctrl);
                else
                    fw_scale<V, RB, false>(v, d, so.rctrl);
            }
        } break;
        case SK_DIAG2:
            reg_diag2<V, RB, ADJ>(v, so, M, Lt, base);
            break;
        case SK_DENSE2: {
            const bool swap = so.p0 > so.p1;
            const int lo = swap ? so.p1 : so.p0, hi = swap ? so.p0 : so.p1;
            V m[16];
            load_mat4(m, M, swap);
#define MQB_D2(A, B)                                                      \
    case (A * 8 + B):                                                     \
        if constexpr (RB > B) reg_dense2<V, RB, A, B, ADJ>(v, m, so.rctrl); \
        break;
            switch (lo * 8 + hi) {
                MQB_D2(0, 1) MQB_D2(0, 2) MQB_D2(0, 3) MQB_D2(0, 4) MQB_D2(1, 2) MQB_D2(1, 3) MQB_D2(1, 4)
                MQB_D2(2, 3) MQB_D2(2, 4) MQB_D2(3, 4)
                default: break;
            }
#undef MQB_D2
        } break;
        default:
            break;
    }
}

// ------------------------------------------------------------------- adjoint step with gradients
// psi <- U^dag psi, partial[a][h] += Re<lambda_h| dU_a |psi>, lambda_h <- U^dag lambda_h; the
// partials of one gate accumulate in the state's precision over the thread's amplitudes and are
// reduced in FP64 across threads.
template <typename V, int RB, int NH, int P, bool CTRL>
__device__ __forceinline__ void bw_dense1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, const V *dM, int gm,
                                          uint32_t rctrl, decltype(V::x) (&acc)[3][NH]) {
    V a00, a01, a10, a11;
    mat2<V, true>(M, a00, a01, a10, a11);
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        constexpr int bit = 1 << P;
        const V w0 = cmadd(a00, v[j], cmul(a01, v[j | bit])), w1 = cmadd(a10, v[j], cmul(a11, v[j | bit]));
        v[j] = w0;
        v[j | bit] = w1;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(gm >> an & 1)) continue;
            const V *d = dM + an * 4;
            const V y0 = cmadd(d[0], w0, cmul(d[1], w1)), y1 = cmadd(d[2], w0, cmul(d[3], w1));
#pragma unroll
            for (int h = 0; h < NH; ++h)
                acc[an][h] += l[h][j].x * y0.x + l[h][j].y * y0.y + l[h][j | bit].x * y1.x + l[h][j | bit].y * y1.y;
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V x0 = l[h][j], x1 = l[h][j | bit];
            l[h][j] = cmadd(a00, x0, cmul(a01, x1));
            l[h][j | bit] = cmadd(a10, x0, cmul(a11, x1));
        }
    }
}

template <typename V, int RB, int NH, int P, bool CTRL>
__device__ __forceinline__ void bw_real1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, const V *dM, int gm,
                                         uint32_t rctrl, decltype(V::x) (&acc)[3][NH]) {
    using R = decltype(V::x);
    const R a00 = M[0].x, a01 = M[2].x, a10 = M[1].x, a11 = M[3].x;   // U^dag = U^T
    R d00 = 0, d01 = 0, d10 = 0, d11 = 0;
    if (gm & 1) {
        d00 = dM[0].x;
        d01 = dM[1].x;
        d10 = dM[2].x;
        d11 = dM[3].x;
    }
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        constexpr int bit = 1 << P;
        const V w0 = rmadd(a00, v[j], rmul(a01, v[j | bit])), w1 = rmadd(a10, v[j], rmul(a11, v[j | bit]));
        v[j] = w0;
        v[j | bit] = w1;
        if (gm & 1) {
            const V y0 = rmadd(d00, w0, rmul(d01, w1)), y1 = rmadd(d10, w0, rmul(d11, w1));
#pragma unroll
            for (int h = 0; h < NH; ++h)
                acc[0][h] += l[h][j].x * y0.x + l[h][j].y * y0.y + l[h][j | bit].x * y1.x + l[h][j | bit].y * y1.y;
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V x0 = l[h][j], x1 = l[h][j | bit];
            l[h][j] = rmadd(a00, x0, rmul(a01, x1));
            l[h][j | bit] = rmadd(a10, x0, rmul(a11, x1));
        }
    }
}

template <typename V, int RB, int NH, int P, bool CTRL>
__device__ __forceinline__ void bw_diag1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, const V *dM, int gm,
                                         uint32_t rctrl, decltype(V::x) (&acc)[3][NH]) {
    const V c0 = cconj(M[0]), c1 = cconj(M[1]);
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        const int b = j >> P & 1;
        const V w = cmul(v[j], b ? c1 : c0);
        v[j] = w;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(gm >> an & 1)) continue;
            const V y = cmul(dM[an * 2 + b], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[an][h] += l[h][j].x * y.x + l[h][j].y * y.y;
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], b ? c1 : c0);
    }
}

// diagonal gate whose target is constant over the thread's registers (thread or outside bit)
template <typename V, int RB, int NH, bool CTRL>
__device__ __forceinline__ void bw_scale(V (&v)[1 << RB], V (&l)[NH][1 << RB], V c, const V *dMb, int nd, int gm,
                                         uint32_t rctrl, decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (CTRL && (uint32_t(j) & rctrl) != rctrl) continue;
        const V w = cmul(v[j], c);
        v[j] = w;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(gm >> an & 1)) continue;
            const V y = cmul(dMb[an * nd], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[an][h] += l[h][j].x * y.x + l[h][j].y * y.y;
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c);
    }
}

template <typename V, int RB, int NH, int P0, int P1>
__device__ __forceinline__ void bw_dense2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V (&m)[16], const V *dMbase,
                                          bool swap, int gm, uint32_t rctrl, decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((j >> P0 & 1) || (j >> P1 & 1)) continue;
        if ((uint32_t(j) & rctrl) != rctrl) continue;
        const int id[4] = {j, j | (1 << P0), j | (1 << P1), j | (1 << P0) | (1 << P1)};
        V w[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            V s;
            s.x = 0;
            s.y = 0;
#pragma unroll
            for (int c = 0; c < 4; ++c) s = cmadd(cconj(m[c * 4 + r]), v[id[c]], s);
            w[r] = s;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) v[id[r]] = w[r];
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(gm >> an & 1)) continue;
            V dm[16];
            load_mat4(dm, dMbase + an * 16, swap);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V y;
                y.x = 0;
                y.y = 0;
#pragma unroll
                for (int c = 0; c < 4; ++c) y = cmadd(dm[r * 4 + c], w[c], y);
#pragma unroll
                for (int h = 0; h < NH; ++h) acc[an][h] += l[h][id[r]].x * y.x + l[h][id[r]].y * y.y;
            }
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            V x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) x[r] = l[h][id[r]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V s;
                s.x = 0;
                s.y = 0;
#pragma unroll
                for (int c = 0; c < 4; ++c) s = cmadd(cconj(m[c * 4 + r]), x[c], s);
                l[h][id[r]] = s;
            }
        }
    }
}

template <typename V, int RB, int NH>
__device__ __forceinline__ void bw_diag2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const StageOp &so, const V *D,
                                         const V *dM, int gm, uint32_t Lt, uint64_t base,
                                         decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((uint32_t(j) & so.rctrl) != so.rctrl) continue;
        const int b0 = diag_bit<V>(so.dsrc[0], so.dval[0], j, Lt, base);
        const int b1 = diag_bit<V>(so.dsrc[1], so.dval[1], j, Lt, base);
        const int r = b0 | (b1 << 1);
        const V dc = cconj(D[r]);
        const V w = cmul(dc, v[j]);
        v[j] = w;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(gm >> an & 1)) continue;
            const V y = cmul(dM[an * 4 + r], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[an][h] += l[h][j].x * y.x + l[h][j].y * y.y;
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(dc, l[h][j]);
    }
}

template <typename V, int RB, int NH>
__device__ __forceinline__ void bwd_gate(V (&v)[1 << RB], V (&l)[NH][1 << RB], const StageOp &so, const V *M,
                                         uint32_t Lt, uint64_t base, decltype(V::x) (&acc)[3][NH]) {
    const V *dM = M + so.mat_size;
    const int gm = so.n_angles ? so.grad_mask : 0;
    const bool ctrl = so.rctrl != 0;
    switch (so.kind) {
        case SK_DENSE1: {
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) bw_dense1<V, RB, NH, P, true>(v, l, M, dM, gm, so.rctrl, acc);                    \
        else bw_dense1<V, RB, NH, P, false>(v, l, M, dM, gm, so.rctrl, acc);                        \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_REAL1: {
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) bw_real1<V, RB, NH, P, true>(v, l, M, dM, gm, so.rctrl, acc);                     \
        else bw_real1<V, RB, NH, P, false>(v, l, M, dM, gm, so.rctrl, acc);                         \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_PERM1:
        case SK_SWAP1: {
            // constant gates: no gradient, uncompute psi and every lambda
            if (so.kind == SK_SWAP1 && so.rc1 >= 0) {   // self-inverse register permutation
                dispatch_cswap<V, RB>(v, so.p0, so.rc1);
#pragma unroll
                for (int h = 0; h < NH; ++h) dispatch_cswap<V, RB>(l[h], so.p0, so.rc1);
                break;
            }
            const bool unit = so.kind == SK_SWAP1;
            const V m01 = cconj(M[2]), m10 = cconj(M[1]);
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) {                                                                                 \
            fw_perm1<V, RB, P, true>(v, m01, m10, unit, so.rctrl);                                  \
            _Pragma("unroll") for (int h = 0; h < NH; ++h) fw_perm1<V, RB, P, true>(l[h], m01, m10, unit, so.rctrl); \
        } else {                                                                                    \
            fw_perm1<V, RB, P, false>(v, m01, m10, unit, so.rctrl);                                 \
            _Pragma("unroll") for (int h = 0; h < NH; ++h) fw_perm1<V, RB, P, false>(l[h], m01, m10, unit, so.rctrl); \
        }                                                                                           \
    }
            MQB_POS_SWITCH(so.p0, MQB_C)
#undef MQB_C
        } break;
        case SK_DIAG1: {
            if (so.dsrc[0] == 0) {
#define MQB_C(P)                                                                                    \
    if constexpr (RB > P) {                                                                         \
        if (ctrl) bw_diag1<V, RB, NH, P, true>(v, l, M, dM, gm, so.rctrl, acc);                     \
        else bw_diag1<V, RB, NH, P, false>(v, l, M, dM, gm, so.rctrl, acc);                         \
    }
                MQB_POS_SWITCH(so.dval[0], MQB_C)
#undef MQB_C
            } else {
                const int b = diag_bit<V>(so.dsrc[0], so.dval[0], 0, Lt, base);
                const V c = cconj(M[b]);
                if (ctrl)
                    bw_scale<V, RB, NH, true>(v, l, c, dM + b, 2, gm, so.rctrl, acc);
                else
                    bw_scale<V, RB, NH, false>(v, l, c, dM + b, 2, gm, so.rctrl, acc);
            }
        } break;
        case SK_DIAG2:
            bw_diag2<V, RB, NH>(v, l, so, M, dM, gm, Lt, base, acc);
            break;
        case SK_DENSE2: {
            const bool swap = so.p0 > so.p1;
            const int lo = swap ? so.p1 : so.p0, hi = swap ? so.p0 : so.p1;
            V m[16];
            load_mat4(m, M, swap);
#define MQB_B2(A, B)                                                                          \
    case (A * 8 + B):                                                                         \
        if constexpr (RB > B) bw_dense2<V, RB, NH, A, B>(v, l, m, dM, swap, gm, so.rctrl, acc); \
        break;
            switch (lo * 8 + hi) {
                MQB_B2(0, 1) MQB_B2(0, 2) MQB_B2(0, 3) MQB_B2(0, 4) MQB_B2(1, 2) MQB_B2(1, 3) MQB_B2(1, 4)
                MQB_B2(2, 3) MQB_B2(2, 4) MQB_B2(3, 4)
                default: break;
            }
#undef MQB_B2
        } break;
        default:
            break;
    }
}

// Copy the matrices (and derivative matrices) of every gate of the pass into shared memory.
template <typename V>
__device__ __forceinline__ void load_mtab(V *mtab, const StageOp *sops, int n_ops, const V *mb, const V *cpool) {
    // one warp per gate: the loads of different gates are in flight together
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int k = threadIdx.x >> 5; k < n_ops; k += nw) {
        const StageOp &so = sops[k];
        const V *src = (so.msrc_ps ? mb : cpool) + so.msrc;
        for (int e = lane; e < so.mcount; e += 32) mtab[so.moff + e] = src[e];
    }
}

template <int RB>
__device__ __forceinline__ uint32_t reg_offset(int j, const uint32_t (&pr)[RB]) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < RB; ++i)
        if (j >> i & 1) o ^= pr[i];
    return o;
}

}  // namespace

size_t fused2_smem(const TileGeom &g, int n_tiles_in_smem, int n_stages, int n_stage_ops, int n_local_slots,
                   int n_hams, int elem_bytes, int threads, int mtab_entries) {
    size_t s = (size_t(1) << g.K) * elem_bytes * n_tiles_in_smem;
    s = (s + 15) & ~size_t(15);
    s += size_t(mtab_entries) * elem_bytes;
    s = (s + 15) & ~size_t(15);
    s += (size_t(1) << (g.K - g.c)) * sizeof(uint64_t);
    s = (s + 15) & ~size_t(15);
    s += size_t(n_stages) * sizeof(StageDesc);
    s = (s + 15) & ~size_t(15);
    s += size_t(n_stage_ops) * sizeof(StageOp);
    s = (s + 15) & ~size_t(15);
    if (n_hams > 0) s += size_t(threads / 32) * std::max(1, n_local_slots) * n_hams * sizeof(double);
    return s;
}

template <typename R, int RB>
__global__ void __launch_bounds__(256, 2) fused_fwd2_kernel(const Fwd2Args<R> a) {
    using V = cplx<R>;
    constexpr int NR = 1 << RB;
    constexpr int NV = NR / (16 / int(sizeof(V)));   // 16-byte vectors per thread per tile
    extern __shared__ __align__(16) unsigned char smem[];
    const TileGeom &g = a.g;
    const int K = g.K, c = g.c;
    const int TB = K - RB;
    V *tile = reinterpret_cast<V *>(smem);
    size_t o = align16((size_t(1) << K) * sizeof(V));
    V *mtab = reinterpret_cast<V *>(smem + o);
    o = align16(o + size_t(a.mtab_entries) * sizeof(V));
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + o);
    o = align16(o + (size_t(1) << (K - c)) * sizeof(uint64_t));
    StageDesc *sst = reinterpret_cast<StageDesc *>(smem + o);
    o = align16(o + size_t(a.n_stages) * sizeof(StageDesc));
    StageOp *sops = reinterpret_cast<StageOp *>(smem + o);
    build_table(tab, g);
    for (int i = threadIdx.x; i < a.n_stages; i += blockDim.x) sst[i] = a.stages[i];
    for (int i = threadIdx.x; i < a.n_ops; i += blockDim.x) sops[i] = a.sops[i];
    __syncthreads();
    const int64_t n_tiles = int64_t(1) << g.n_out;
    const int64_t dim = int64_t(1) << g.n;
    const int tid = threadIdx.x;
    int64_t cached_b = -1;
    for (int64_t w = blockIdx.x; w < a.batch * n_tiles; w += gridDim.x) {
        const int64_t b = w >> g.n_out;
        const uint64_t t = uint64_t(w) & uint64_t(n_tiles - 1);
        const uint64_t base = tile_base(g, t);
        if (b != cached_b) {
            load_mtab(mtab, sops, a.n_ops, a.mats + b * a.mats_stride, a.cpool);
            cached_b = b;
        }
        if (a.src)
            stage_in<V, NV>(tile, a.src + b * a.src_batch_stride, base, tab, c);
        else
            stage_zero(tile, base, K);
        __syncthreads();
        for (int s = 0; s < a.n_stages; ++s) {
            const StageDesc &sd = sst[s];
            uint32_t Lt = 0;
            for (int i = 0; i < TB; ++i)
                if (tid >> i & 1) Lt |= 1u << sd.tbits[i];
            const uint32_t pLt = swz<V>(Lt);
            uint32_t pr[RB];
#pragma unroll
            for (int i = 0; i < RB; ++i) pr[i] = swz<V>(1u << sd.rbits[i]);
            V v[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) v[j] = tile[pLt ^ reg_offset<RB>(j, pr)];
            for (int k = sd.op_begin; k < sd.op_end; ++k) {
                const StageOp &so = sops[k];
                if ((base & so.octrl) != so.octrl) continue;
                if ((Lt & so.tctrl) != so.tctrl) continue;
                fwd_gate<V, RB, false>(v, so, mtab + so.moff, Lt, base);
            }
#pragma unroll
            for (int j = 0; j < NR; ++j) tile[pLt ^ reg_offset<RB>(j, pr)] = v[j];
            __syncthreads();
        }
        stage_out<V, NV>(tile, a.dst + b * dim, base, tab, c);
        __syncthreads();
    }
}

template <typename R, int RB, int NH>
__global__ void __launch_bounds__(256, 2) fused_bwd2_kernel(const Bwd2Args<R> a) {
    using V = cplx<R>;
    constexpr int NR = 1 << RB;
    constexpr int NV = NR / (16 / int(sizeof(V)));   // 16-byte vectors per thread per tile
    extern __shared__ __align__(16) unsigned char smem[];
    const TileGeom &g = a.g;
    const int K = g.K, c = g.c;
    const int TB = K - RB;
    const int TS = 1 << K;
    V *psi = reinterpret_cast<V *>(smem);
    V *lam = psi + TS;
    size_t o = align16(size_t(TS) * sizeof(V) * (1 + NH));
    V *mtab = reinterpret_cast<V *>(smem + o);
    o = align16(o + size_t(a.mtab_entries) * sizeof(V));
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + o);
    o = align16(o + (size_t(1) << (K - c)) * sizeof(uint64_t));
    StageDesc *sst = reinterpret_cast<StageDesc *>(smem + o);
    o = align16(o + size_t(a.n_stages) * sizeof(StageDesc));
    StageOp *sops = reinterpret_cast<StageOp *>(smem + o);
    o = align16(o + size_t(a.n_ops) * sizeof(StageOp));
    double *wacc = reinterpret_cast<double *>(smem + o);   // [warps][n_local_slots][NH]
    const int nw = blockDim.x / 32;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int nls = a.n_local_slots;
    build_table(tab, g);
    for (int i = threadIdx.x; i < a.n_stages; i += blockDim.x) sst[i] = a.stages[i];
    for (int i = threadIdx.x; i < a.n_ops; i += blockDim.x) sops[i] = a.sops[i];
    for (int i = threadIdx.x; i < nw * nls * NH; i += blockDim.x) wacc[i] = 0;
    __syncthreads();
    const int64_t n_tiles = int64_t(1) << g.n_out;
    const int64_t dim = int64_t(1) << g.n;
    const int64_t total = a.batch * n_tiles;
    const int tid = threadIdx.x;
    int64_t cached_b = -1;
    for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
        const int64_t b = w >> g.n_out;
        const uint64_t t = uint64_t(w) & uint64_t(n_tiles - 1);
        const uint64_t base = tile_base(g, t);
        if (b != cached_b) {
            load_mtab(mtab, sops, a.n_ops, a.mats + b * a.mats_stride, a.cpool);
            cached_b = b;
        }
        stage_in<V, NV>(psi, a.psi_src + b * dim, base, tab, c);
#pragma unroll
        for (int h = 0; h < NH; ++h) stage_in<V, NV>(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, c);
        __syncthreads();
        for (int s = a.n_stages - 1; s >= 0; --s) {
            const StageDesc &sd = sst[s];
            uint32_t Lt = 0;
            for (int i = 0; i < TB; ++i)
                if (tid >> i & 1) Lt |= 1u << sd.tbits[i];
            const uint32_t pLt = swz<V>(Lt);
            uint32_t pr[RB];
#pragma unroll
            for (int i = 0; i < RB; ++i) pr[i] = swz<V>(1u << sd.rbits[i]);
            V v[NR];
            V l[NH][NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) {
                const uint32_t ad = pLt ^ reg_offset<RB>(j, pr);
                v[j] = psi[ad];
#pragma unroll
                for (int h = 0; h < NH; ++h) l[h][j] = lam[h * TS + ad];
            }
            for (int k = sd.op_end - 1; k >= sd.op_begin; --k) {
                const StageOp &so = sops[k];
                if ((base & so.octrl) != so.octrl) continue;   // uniform over the block
                R acc[3][NH];
#pragma unroll
                for (int an = 0; an < 3; ++an)
#pragma unroll
                    for (int h = 0; h < NH; ++h) acc[an][h] = 0;
                if ((Lt & so.tctrl) == so.tctrl) bwd_gate<V, RB, NH>(v, l, so, mtab + so.moff, Lt, base, acc);
                if (so.lslot >= 0) {
                    int r = 0;
                    for (int an = 0; an < so.n_angles; ++an) {
                        if (!(so.grad_mask >> an & 1)) continue;
#pragma unroll
                        for (int h = 0; h < NH; ++h) {
                            double x = 0;
#pragma unroll
                            for (int q = 0; q < 3; ++q)
                                if (q == an) x = double(acc[q][h]);
                            x = warp_sum(x);
                            if (lane == 0) wacc[(warp * nls + so.lslot + r) * NH + h] += x;
                        }
                        ++r;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < NR; ++j) {
                const uint32_t ad = pLt ^ reg_offset<RB>(j, pr);
                psi[ad] = v[j];
#pragma unroll
                for (int h = 0; h < NH; ++h) lam[h * TS + ad] = l[h][j];
            }
            __syncthreads();
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) stage_out<V, NV>(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, c);
        if (a.psi_dst) stage_out<V, NV>(psi, a.psi_dst + b * dim, base, tab, c);
        const int64_t nxt = w + gridDim.x;
        const bool flush = (nxt >= total) || ((nxt >> g.n_out) != b);
        __syncthreads();
        if (flush) {
            for (int i = threadIdx.x; i < nls * NH; i += blockDim.x) {
                double sum = 0;
                for (int ww = 0; ww < nw; ++ww) {
                    sum += wacc[ww * nls * NH + i];
                    wacc[ww * nls * NH + i] = 0;
                }
                const int ls = i / NH, h = i % NH;
                if (sum != 0) atomicAdd(&a.gslots[(b * a.n_slots + a.slot_map[ls]) * a.n_hams + h], sum);
            }
            __syncthreads();
        }
    }
}

template <typename KernelT>
static int blocks_for2(KernelT kern, int threads, size_t smem, int sm_count, int64_t work) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = int64_t(sm_count) * per_sm;
    return int(std::max<int64_t>(1, std::min<int64_t>(want, work)));
}

template <typename R>
cudaError_t launch_fused_fwd2(const Fwd2Args<R> &a, int sm_count, cudaStream_t s) {
    const int RB = a.reg_bits;
    const int TB = a.g.K - RB;
    if (a.g.c < 1 || a.g.K > kMaxTileBits || RB < 1 || RB > kMaxRegBits || TB < 5 || TB > kMaxThreadBits)
        return cudaErrorInvalidValue;
    const int threads = 1 << TB;
    const size_t smem = fused2_smem(a.g, 1, a.n_stages, a.n_ops, 0, 0, sizeof(cplx<R>), threads, a.mtab_entries);
    const int64_t work = a.batch << a.g.n_out;
#define MQB_F2(RBV)                                                                                         \
    case RBV: {                                                                                             \
        auto kern = fused_fwd2_kernel<R, RBV>;                                                              \
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); \
        if (e != cudaSuccess) return e;                                                                     \
        kern<<<blocks_for2(kern, threads, smem, sm_count, work), threads, smem, s>>>(a);                    \
        return cudaGetLastError();                                                                          \
    }
    // register bits used by the scheduler: apply passes 5 (complex64) / 4 (complex128); the forward
    // passes of a gradient run with the backward layout (4, 3 / 3, 2)
    switch (RB) {
        MQB_F2(sizeof(R) == 4 ? 5 : 4)
        MQB_F2(sizeof(R) == 4 ? 4 : 3)
        MQB_F2(sizeof(R) == 4 ? 3 : 2)
        default:
            return cudaErrorInvalidValue;
    }
#undef MQB_F2
}

template <typename R>
cudaError_t launch_fused_bwd2(const Bwd2Args<R> &a, int sm_count, cudaStream_t s) {
    const int RB = a.reg_bits;
    const int TB = a.g.K - RB;
    if (a.g.c < 1 || a.g.K > kMaxTileBits || RB < 1 || RB > 4 || TB < 5 || TB > kMaxThreadBits || a.n_hams < 1 ||
        a.n_hams > 4)
        return cudaErrorInvalidValue;
    const int threads = 1 << TB;
    const size_t smem =
        fused2_smem(a.g, 1 + a.n_hams, a.n_stages, a.n_ops, a.n_local_slots, a.n_hams, sizeof(cplx<R>), threads,
                    a.mtab_entries);
    const int64_t work = a.batch << a.g.n_out;
#define MQB_B2K(RBV, NHV)                                                                                   \
    case RBV * 8 + NHV: {                                                                                   \
        auto kern = fused_bwd2_kernel<R, RBV, NHV>;                                                         \
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); \
        if (e != cudaSuccess) return e;                                                                     \
        kern<<<blocks_for2(kern, threads, smem, sm_count, work), threads, smem, s>>>(a);                    \
        return cudaGetLastError();                                                                          \
    }
    // register bits used by the scheduler: one lambda 4 (complex64) / 3 (complex128), more lambdas 3 / 2
    constexpr int RB1 = sizeof(R) == 4 ? 4 : 3, RBN = sizeof(R) == 4 ? 3 : 2;
    switch (RB * 8 + a.n_hams) {
        MQB_B2K(RB1, 1) MQB_B2K(RBN, 2) MQB_B2K(RBN, 3) MQB_B2K(RBN, 4)
        default:
            return cudaErrorInvalidValue;
    }
#undef MQB_B2K
}

template cudaError_t launch_fused_fwd2<float>(const Fwd2Args<float> &, int, cudaStream_t);
template cudaError_t launch_fused_fwd2<double>(const Fwd2Args<double> &, int, cudaStream_t);
template cudaError_t launch_fused_bwd2<float>(const Bwd2Args<float> &, int, cudaStream_t);
template cudaError_t launch_fused_bwd2<double>(const Bwd2Args<double> &, int, cudaStream_t);

}  // namespace mqb
