// Tile staging of the fused passes (sm_100a): global memory <-> XOR-swizzled shared tiles.
// Shared by the precompiled tile kernels and the pass kernels generated at run time (compiled
// by NVRTC, so only built-in types are used).
#ifndef MQB_TILE_CUH_
#define MQB_TILE_CUH_

#include "jit_abi.h"

namespace mqb {
namespace tile {

typedef unsigned long long u64;

// Shared-memory index of tile-local amplitude L: the high index bits are XOR-folded into the low
// 4 (complex64) / 3 (complex128) bits.  The map is linear over GF(2) and a bijection, so
// swz(a ^ b) = swz(a) ^ swz(b) and bank conflicts of a stage exchange depend only on which tile
// bits are thread bits.
template <typename V>
__device__ __forceinline__ unsigned swz(unsigned L) {
    if (sizeof(V) == 8) return L ^ ((L >> 4) & 15u) ^ ((L >> 8) & 15u) ^ ((L >> 12) & 15u);
    return L ^ ((L >> 3) & 7u) ^ ((L >> 6) & 7u) ^ ((L >> 9) & 7u) ^ ((L >> 12) & 7u);
}

__device__ __forceinline__ u64 tile_base(const TileGeom &g, u64 t) {
    u64 base = 0;
    for (int i = 0; i < g.n_out; ++i)
        if (t >> i & 1) base |= u64(1) << g.outside[i];
    return base;
}

__device__ __forceinline__ u64 align16(u64 x) { return (x + 15) & ~u64(15); }

__device__ __forceinline__ void build_table(u64 *tab, const TileGeom &g) {
    const int nh = 1 << (g.K - g.c);
    for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        u64 off = 0;
        for (int i = 0; i < g.K - g.c; ++i)
            if (h >> i & 1) off |= u64(1) << g.qbits[g.c + i];
        tab[h] = off;
    }
}

// global (coalesced 16-byte vectors) -> swizzled shared tile.  Every thread moves NV vectors;
// all of its global loads are issued before the first shared store so their latencies overlap.
template <typename V, int NV>
__device__ __forceinline__ void stage_in(V *tile, const V *src, u64 base, const u64 *tab, int c) {
    constexpr int APV = 16 / sizeof(V);
    constexpr int CH = NV < 8 ? NV : 8;   // vectors in flight per thread (bounded register use)
    const unsigned lowmask = (1u << c) - 1u;
#pragma unroll
    for (int i0 = 0; i0 < NV; i0 += CH) {
        uint4 buf[CH];
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const unsigned L = (threadIdx.x + unsigned(i0 + i) * blockDim.x) * APV;
            const u64 gi = base + tab[L >> c] + (L & lowmask);
            buf[i] = __ldcs(reinterpret_cast<const uint4 *>(src + gi));
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const unsigned L = (threadIdx.x + unsigned(i0 + i) * blockDim.x) * APV;
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
__device__ __forceinline__ void stage_zero(V *tile, u64 base, int K) {
    for (int L = threadIdx.x; L < (1 << K); L += blockDim.x) {
        V v;
        v.x = (base == 0 && L == 0) ? 1 : 0;
        v.y = 0;
        tile[swz<V>(L)] = v;
    }
}

template <typename V, int NV>
__device__ __forceinline__ void stage_out(const V *tile, V *dst, u64 base, const u64 *tab, int c) {
    constexpr int APV = 16 / sizeof(V);
    const unsigned lowmask = (1u << c) - 1u;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const unsigned L = (threadIdx.x + unsigned(i) * blockDim.x) * APV;
        const u64 gi = base + tab[L >> c] + (L & lowmask);
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

// Copy the matrices (and derivative matrices) of every op of a pass into shared memory: one
// warp per op, so the loads of different ops are in flight together.
template <typename V>
__device__ __forceinline__ void load_mtab(V *mtab, const JitMtab *mt, int n, const V *mb, const V *cpool) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int k = threadIdx.x >> 5; k < n; k += nw) {
        const JitMtab e = mt[k];
        const V *src = (e.msrc_ps ? mb : cpool) + e.msrc;
        for (int i = lane; i < e.mcount; i += 32) mtab[e.moff + i] = src[i];
    }
}

}  // namespace tile
}  // namespace mqb

#endif
