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

// global (coalesced 16-byte vectors) -> swizzled shared tile
template <typename V>
__device__ __forceinline__ void stage_in(V *tile, const V *src, uint64_t base, const uint64_t *tab, int K, int c) {
    constexpr int APV = 16 / sizeof(V);
    const int nvec = (1 << K) / APV;
    const uint32_t lowmask = (1u << c) - 1u;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const uint32_t L = uint32_t(v) * APV;
        const uint64_t gi = base + tab[L >> c] + (L & lowmask);
        const uint4 raw = __ldg(reinterpret_cast<const uint4 *>(src + gi));
        if (APV == 2) {
            const V *pv = reinterpret_cast<const V *>(&raw);
            tile[swz<V>(L)] = pv[0];
            tile[swz<V>(L + 1)] = pv[1];
        } else {
            *reinterpret_cast<uint4 *>(&tile[swz<V>(L)]) = raw;
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

template <typename V>
__device__ __forceinline__ void stage_out(const V *tile, V *dst, uint64_t base, const uint64_t *tab, int K, int c) {
    constexpr int APV = 16 / sizeof(V);
    const int nvec = (1 << K) / APV;
    const uint32_t lowmask = (1u << c) - 1u;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const uint32_t L = uint32_t(v) * APV;
        const uint64_t gi = base + tab[L >> c] + (L & lowmask);
        uint4 raw;
        if (APV == 2) {
            V *pv = reinterpret_cast<V *>(&raw);
            pv[0] = tile[swz<V>(L)];
            pv[1] = tile[swz<V>(L + 1)];
        } else {
            raw = *reinterpret_cast<const uint4 *>(&tile[swz<V>(L)]);
        }
        *reinterpret_cast<uint4 *>(dst + gi) = raw;
    }
}

// ----------------------------------------------------------------------------------- register ops
// Forward / adjoint dense single-qubit gate on register position P.
template <typename V, int RB, int P, bool ADJ>
__device__ __forceinline__ void reg_dense1(V (&v)[1 << RB], const V *M, uint32_t rctrl, bool on) {
    V m00 = M[0], m01 = M[1], m10 = M[2], m11 = M[3];
    if (ADJ) {
        const V t01 = m01;
        m00 = cconj(m00);
        m01 = cconj(m10);
        m10 = cconj(t01);
        m11 = cconj(m11);
    }
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        constexpr int bit = 1 << P;
        const bool act = on && ((uint32_t(j) & rctrl) == rctrl);
        const V a = v[j], b = v[j | bit];
        const V na = cmadd(m00, a, cmul(m01, b)), nb = cmadd(m10, a, cmul(m11, b));
        v[j] = act ? na : a;
        v[j | bit] = act ? nb : b;
    }
}

// Dense two-qubit gate on register positions P0 < P1; matrix index bit 0 <-> position of `lo_is_bit0`.
template <typename V, int RB, int P0, int P1, bool ADJ>
__device__ __forceinline__ void reg_dense2(V (&v)[1 << RB], const V (&m)[16], uint32_t rctrl, bool on) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((j >> P0 & 1) || (j >> P1 & 1)) continue;
        const bool act = on && ((uint32_t(j) & rctrl) == rctrl);
        const int id[4] = {j, j | (1 << P0), j | (1 << P1), j | (1 << P0) | (1 << P1)};
        V x[4], y[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) x[r] = v[id[r]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            V s;
            s.x = 0;
            s.y = 0;
#pragma unroll
            for (int col = 0; col < 4; ++col) s = cmadd(ADJ ? cconj(m[col * 4 + r]) : m[r * 4 + col], x[col], s);
            y[r] = s;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) v[id[r]] = act ? y[r] : x[r];
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

template <typename V, int RB, bool ADJ>
__device__ __forceinline__ void dispatch_dense1(V (&v)[1 << RB], int p, const V *M, uint32_t rctrl, bool on) {
    switch (p) {
        case 0: reg_dense1<V, RB, 0, ADJ>(v, M, rctrl, on); break;
        case 1: if constexpr (RB > 1) reg_dense1<V, RB, 1, ADJ>(v, M, rctrl, on); break;
        case 2: if constexpr (RB > 2) reg_dense1<V, RB, 2, ADJ>(v, M, rctrl, on); break;
        case 3: if constexpr (RB > 3) reg_dense1<V, RB, 3, ADJ>(v, M, rctrl, on); break;
        case 4: if constexpr (RB > 4) reg_dense1<V, RB, 4, ADJ>(v, M, rctrl, on); break;
        default: break;
    }
}

template <typename V, int RB, bool ADJ>
__device__ __forceinline__ void dispatch_dense2(V (&v)[1 << RB], int lo, int hi, const V (&m)[16], uint32_t rctrl,
                                                bool on) {
#define MQB_D2(A, B)                                                  \
    case (A * 8 + B):                                                 \
        if constexpr (RB > B) reg_dense2<V, RB, A, B, ADJ>(v, m, rctrl, on); \
        break;
    switch (lo * 8 + hi) {
        MQB_D2(0, 1) MQB_D2(0, 2) MQB_D2(0, 3) MQB_D2(0, 4) MQB_D2(1, 2) MQB_D2(1, 3) MQB_D2(1, 4) MQB_D2(2, 3)
        MQB_D2(2, 4) MQB_D2(3, 4)
        default: break;
    }
#undef MQB_D2
}

template <typename V>
__device__ __forceinline__ int diag_bit(int src, int val, int j, uint32_t Lt, uint64_t base) {
    if (src == 0) return (j >> val) & 1;
    if (src == 1) return int((Lt >> val) & 1u);
    return int((base >> val) & 1u);
}

// Diagonal gate (one or two targets): v[j] *= d[index bits of j]
template <typename V, int RB, bool ADJ>
__device__ __forceinline__ void reg_diag(V (&v)[1 << RB], const StageOp &so, const V *D, uint32_t Lt, uint64_t base,
                                         bool on) {
    const bool two = so.kind == SK_DIAG2;
    V d0 = D[0], d1 = D[1], d2 = d0, d3 = d1;
    if (two) {
        d2 = D[2];
        d3 = D[3];
    }
    if (ADJ) {
        d0 = cconj(d0);
        d1 = cconj(d1);
        d2 = cconj(d2);
        d3 = cconj(d3);
    }
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        const bool act = on && ((uint32_t(j) & so.rctrl) == so.rctrl);
        const int b0 = diag_bit<V>(so.dsrc[0], so.dval[0], j, Lt, base);
        const int b1 = two ? diag_bit<V>(so.dsrc[1], so.dval[1], j, Lt, base) : 0;
        const V d = b1 ? (b0 ? d3 : d2) : (b0 ? d1 : d0);
        const V r = cmul(v[j], d);
        v[j] = act ? r : v[j];
    }
}

// Adjoint step of one gate on psi and lambda registers with FP64 gradient partials.
template <typename V, int RB, int NH, int P>
__device__ __forceinline__ void bwd_dense1(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M, const V *dM, int na,
                                           int gmask, uint32_t rctrl, bool on, double (&acc)[3][NH]) {
    const V a00 = cconj(M[0]), a01 = cconj(M[2]), a10 = cconj(M[1]), a11 = cconj(M[3]);
    V d[3][4];
#pragma unroll
    for (int an = 0; an < 3; ++an)
        if (an < na && (gmask >> an & 1))
#pragma unroll
            for (int e = 0; e < 4; ++e) d[an][e] = dM[an * 4 + e];
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (j >> P & 1) continue;
        constexpr int bit = 1 << P;
        const bool act = on && ((uint32_t(j) & rctrl) == rctrl);
        if (!act) continue;
        const V w0 = cmadd(a00, v[j], cmul(a01, v[j | bit])), w1 = cmadd(a10, v[j], cmul(a11, v[j | bit]));
        v[j] = w0;
        v[j | bit] = w1;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(an < na && (gmask >> an & 1))) continue;
            const V y0 = cmadd(d[an][0], w0, cmul(d[an][1], w1)), y1 = cmadd(d[an][2], w0, cmul(d[an][3], w1));
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

template <typename V, int RB, int NH, int P0, int P1>
__device__ __forceinline__ void bwd_dense2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V (&m)[16], const V *dMbase,
                                           bool swap, int na, int gmask, uint32_t rctrl, bool on,
                                           double (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if ((j >> P0 & 1) || (j >> P1 & 1)) continue;
        const bool act = on && ((uint32_t(j) & rctrl) == rctrl);
        if (!act) continue;
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
            if (!(an < na && (gmask >> an & 1))) continue;
            V dm[16];
            load_mat4(dm, dMbase + an * 16, swap);
            V y[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                V s;
                s.x = 0;
                s.y = 0;
#pragma unroll
                for (int c = 0; c < 4; ++c) s = cmadd(dm[r * 4 + c], w[c], s);
                y[r] = s;
            }
#pragma unroll
            for (int h = 0; h < NH; ++h)
#pragma unroll
                for (int r = 0; r < 4; ++r) acc[an][h] += redot(l[h][id[r]], y[r]);
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
__device__ __forceinline__ void bwd_diag(V (&v)[1 << RB], V (&l)[NH][1 << RB], const StageOp &so, const V *D,
                                         const V *dM, int na, int gmask, uint32_t Lt, uint64_t base, bool on,
                                         double (&acc)[3][NH]) {
    const bool two = so.kind == SK_DIAG2;
    const int nd = two ? 4 : 2;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        const bool act = on && ((uint32_t(j) & so.rctrl) == so.rctrl);
        if (!act) continue;
        const int b0 = diag_bit<V>(so.dsrc[0], so.dval[0], j, Lt, base);
        const int b1 = two ? diag_bit<V>(so.dsrc[1], so.dval[1], j, Lt, base) : 0;
        const int r = b0 | (b1 << 1);
        const V dc = cconj(D[r]);
        const V w = cmul(dc, v[j]);
        v[j] = w;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!(an < na && (gmask >> an & 1))) continue;
            const V y = cmul(dM[an * nd + r], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[an][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(dc, l[h][j]);
    }
}

template <typename V, int RB, int NH>
__device__ __forceinline__ void bwd_dispatch1(V (&v)[1 << RB], V (&l)[NH][1 << RB], int p, const V *M, const V *dM,
                                              int na, int gmask, uint32_t rctrl, bool on, double (&acc)[3][NH]) {
    switch (p) {
        case 0: bwd_dense1<V, RB, NH, 0>(v, l, M, dM, na, gmask, rctrl, on, acc); break;
        case 1: if constexpr (RB > 1) bwd_dense1<V, RB, NH, 1>(v, l, M, dM, na, gmask, rctrl, on, acc); break;
        case 2: if constexpr (RB > 2) bwd_dense1<V, RB, NH, 2>(v, l, M, dM, na, gmask, rctrl, on, acc); break;
        case 3: if constexpr (RB > 3) bwd_dense1<V, RB, NH, 3>(v, l, M, dM, na, gmask, rctrl, on, acc); break;
        case 4: if constexpr (RB > 4) bwd_dense1<V, RB, NH, 4>(v, l, M, dM, na, gmask, rctrl, on, acc); break;
        default: break;
    }
}

template <typename V, int RB, int NH>
__device__ __forceinline__ void bwd_dispatch2(V (&v)[1 << RB], V (&l)[NH][1 << RB], int lo, int hi, const V (&m)[16],
                                              const V *dM, bool swap, int na, int gmask, uint32_t rctrl, bool on,
                                              double (&acc)[3][NH]) {
#define MQB_B2(A, B)                                                                                \
    case (A * 8 + B):                                                                               \
        if constexpr (RB > B) bwd_dense2<V, RB, NH, A, B>(v, l, m, dM, swap, na, gmask, rctrl, on, acc); \
        break;
    switch (lo * 8 + hi) {
        MQB_B2(0, 1) MQB_B2(0, 2) MQB_B2(0, 3) MQB_B2(0, 4) MQB_B2(1, 2) MQB_B2(1, 3) MQB_B2(1, 4) MQB_B2(2, 3)
        MQB_B2(2, 4) MQB_B2(3, 4)
        default: break;
    }
#undef MQB_B2
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
__global__ void __launch_bounds__(256) fused_fwd2_kernel(const Fwd2Args<R> a) {
    using V = cplx<R>;
    constexpr int NR = 1 << RB;
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
            stage_in(tile, a.src + b * a.src_batch_stride, base, tab, K, c);
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
                const bool on = (Lt & so.tctrl) == so.tctrl;
                const V *M = mtab + so.moff;
                if (so.kind == SK_DENSE1) {
                    dispatch_dense1<V, RB, false>(v, so.p0, M, so.rctrl, on);
                } else if (so.kind == SK_DENSE2) {
                    const bool swap = so.p0 > so.p1;
                    V m[16];
                    load_mat4(m, M, swap);
                    dispatch_dense2<V, RB, false>(v, swap ? so.p1 : so.p0, swap ? so.p0 : so.p1, m, so.rctrl, on);
                } else {
                    reg_diag<V, RB, false>(v, so, M, Lt, base, on);
                }
            }
#pragma unroll
            for (int j = 0; j < NR; ++j) tile[pLt ^ reg_offset<RB>(j, pr)] = v[j];
            __syncthreads();
        }
        stage_out(tile, a.dst + b * dim, base, tab, K, c);
        __syncthreads();
    }
}

template <typename R, int RB, int NH>
__global__ void __launch_bounds__(256) fused_bwd2_kernel(const Bwd2Args<R> a) {
    using V = cplx<R>;
    constexpr int NR = 1 << RB;
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
        stage_in(psi, a.psi_src + b * dim, base, tab, K, c);
#pragma unroll
        for (int h = 0; h < NH; ++h) stage_in(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, K, c);
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
                const bool on = (Lt & so.tctrl) == so.tctrl;
                const V *M = mtab + so.moff;
                const V *dM = M + so.mat_size;
                const int na = so.n_angles;
                double acc[3][NH];
#pragma unroll
                for (int an = 0; an < 3; ++an)
#pragma unroll
                    for (int h = 0; h < NH; ++h) acc[an][h] = 0;
                if (so.kind == SK_DENSE1) {
                    bwd_dispatch1<V, RB, NH>(v, l, so.p0, M, dM, na, so.grad_mask, so.rctrl, on, acc);
                } else if (so.kind == SK_DENSE2) {
                    const bool swap = so.p0 > so.p1;
                    V m[16];
                    load_mat4(m, M, swap);
                    bwd_dispatch2<V, RB, NH>(v, l, swap ? so.p1 : so.p0, swap ? so.p0 : so.p1, m, dM, swap, na,
                                             so.grad_mask, so.rctrl, on, acc);
                } else {
                    bwd_diag<V, RB, NH>(v, l, so, M, dM, na, so.grad_mask, Lt, base, on, acc);
                }
                if (so.lslot >= 0) {
                    int r = 0;
                    for (int an = 0; an < so.n_angles; ++an) {
                        if (!(so.grad_mask >> an & 1)) continue;
#pragma unroll
                        for (int h = 0; h < NH; ++h) {
                            double x = 0;
#pragma unroll
                            for (int q = 0; q < 3; ++q)
                                if (q == an) x = acc[q][h];
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
        for (int h = 0; h < NH; ++h) stage_out(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, K, c);
        if (a.psi_dst) stage_out(psi, a.psi_dst + b * dim, base, tab, K, c);
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
    switch (RB) {
        MQB_F2(1) MQB_F2(2) MQB_F2(3) MQB_F2(4) MQB_F2(5)
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
    switch (RB * 8 + a.n_hams) {
        MQB_B2K(1, 1) MQB_B2K(2, 1) MQB_B2K(3, 1) MQB_B2K(4, 1)
        MQB_B2K(1, 2) MQB_B2K(2, 2) MQB_B2K(3, 2) MQB_B2K(4, 2)
        MQB_B2K(1, 3) MQB_B2K(2, 3) MQB_B2K(3, 3)
        MQB_B2K(1, 4) MQB_B2K(2, 4) MQB_B2K(3, 4)
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
