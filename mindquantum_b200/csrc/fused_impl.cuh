// Fused tile passes with register stages (sm_100a): kernels and launchers.  Each of
// fused_{fwd,bwd}_{c64,c128}.cu instantiates one direction at one precision, so the four compile
// in parallel.
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
#ifndef MQB_FUSED_IMPL_CUH_
#define MQB_FUSED_IMPL_CUH_

#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.cuh"
#include "regops.cuh"
#include "tile.cuh"

namespace mqb {

namespace {

using reg::warp_sum;
using reg::warp_sum_acc;

using mqb::tile::swz;
using mqb::tile::tile_base;
using mqb::tile::align16;
using mqb::tile::build_table;
using mqb::tile::stage_in;
using mqb::tile::stage_zero;
using mqb::tile::stage_out;

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
    mqb::tile::u64 *tab = reinterpret_cast<mqb::tile::u64 *>(smem + o);
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
                if (so.cflags && ((base & so.octrl) != so.octrl || (Lt & so.tctrl) != so.tctrl)) continue;
                reg::fwd_op<V, RB>(so.code, v, mtab + so.moff, so, Lt, base);
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
    mqb::tile::u64 *tab = reinterpret_cast<mqb::tile::u64 *>(smem + o);
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
                if ((Lt & so.tctrl) == so.tctrl)
                    reg::bwd_op<V, RB, NH>(so.bcode, v, l, mtab + so.moff, so, Lt, base,
                                           so.n_angles ? so.grad_mask : 0, acc);
                if (so.lslot >= 0) {
                    int r = 0;
                    for (int an = 0; an < so.n_angles; ++an) {
                        if (!(so.grad_mask >> an & 1)) continue;
#pragma unroll
                        for (int h = 0; h < NH; ++h) {
                            R xr = 0;
#pragma unroll
                            for (int q = 0; q < 3; ++q)
                                if (q == an) xr = acc[q][h];
                            const double x = double(warp_sum_acc(xr));   // FP32 across the warp for complex64
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

}  // namespace mqb

#endif
