// Asynchronous tile movement of the generated pass kernels (sm_100a): TMA tensor copies between
// global memory and shared-memory tile buffers, completed on mbarriers, and the bounded waits
// around them.  Compiled by NVRTC together with the generated kernels, so only built-in types
// and inline PTX are used.
//
// No copy here uses cluster multicast: every tensor map covers this GPU's own memory and every
// copy lands in the issuing CTA's own shared memory.
#ifndef MQB_PIPE_CUH_
#define MQB_PIPE_CUH_

#include "jit_abi.h"

namespace mqb {
namespace pipe {

typedef unsigned long long u64;

// A CUtensorMap (128 opaque bytes, 64-byte aligned), passed to the kernels as a __grid_constant__.
struct __align__(64) TMap {
    u64 w[16];
};

__device__ __forceinline__ unsigned saddr(const void *p) {
    u64 a;
    asm("cvta.to.shared.u64 %0, %1;" : "=l"(a) : "l"(p));
    return static_cast<unsigned>(a);
}

__device__ __forceinline__ u64 now_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Limit of every wait on an mbarrier: far above any tile's load or compute time (microseconds),
// so only a broken pipeline reaches it; the kernel then reports MQB_DEV_ERR_TIMEOUT and returns.
constexpr u64 kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ void mbar_init(u64 *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(u64 *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(u64 *bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(u64 *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of `parity` to complete; false when kWaitLimitNs passed first.
__device__ __forceinline__ bool mbar_wait(u64 *bar, unsigned parity) {
    if (mbar_test(bar, parity)) return true;
    const u64 t0 = now_ns();
    while (!mbar_test(bar, parity))
        if (now_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// Wait until a buffer's ticket names tile k (the tile whose copies were last started into it);
// false when kWaitLimitNs passed first.  A buffer's mbarrier tells phases apart by parity only, so
// a consumer may test it only once the buffer's previous tile has been handed over: the issuer
// writes the ticket after it has finished with that previous tile.
__device__ __forceinline__ bool wait_ticket(const volatile long long *slot, long long k) {
    if (*slot == k) return true;
    const u64 t0 = now_ns();
    while (*slot != k)
        if (now_ns() - t0 > kWaitLimitNs) return false;
    return true;
}

// Named barrier `id` (1 + consumer group; 0 is __syncthreads) among the n threads of a group.
__device__ __forceinline__ void consumers_sync(int id, int n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Named barrier `id` among the n threads of a consumer group, returning whether q holds on every
// one of them: a group takes every wait's outcome together, so no thread leaves the tile loop
// alone and none is left waiting at a later barrier.
__device__ __forceinline__ bool consumers_and(int id, int n, bool q) {
    unsigned r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred p, %2, %3, q;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(r)
        : "r"(static_cast<unsigned>(q)), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// The matrices of a pass's ops into shared memory, by the nt consumer threads (one warp per op).
template <typename V>
__device__ __forceinline__ void load_mtab(V *mtab, const JitMtab *mt, int n, const V *mb, const V *cpool, unsigned tid,
                                          unsigned nt) {
    const unsigned lane = tid & 31u, nw = nt >> 5;
    for (int k = static_cast<int>(tid >> 5); k < n; k += static_cast<int>(nw)) {
        const JitMtab e = mt[k];
        const V *src = (e.msrc_ps ? mb : cpool) + e.msrc;
        for (int i = static_cast<int>(lane); i < e.mcount; i += 32) mtab[e.moff + i] = src[i];
    }
}

// Make this thread's generic-proxy writes to shared memory visible to the TMA (async proxy).
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tensor copy global -> shared of one box at coordinates c[0..nd), completing on `bar`.
__device__ __forceinline__ void tma_load(void *dst, const TMap *m, int nd, const int *c, u64 *bar) {
    const unsigned d = saddr(dst), b = saddr(bar);
    const u64 mp = reinterpret_cast<u64>(m);
    switch (nd) {
        case 1:
            asm volatile(
                "cp.async.bulk.tensor.1d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];" ::"r"(d),
                "l"(mp), "r"(c[0]), "r"(b)
                : "memory");
            break;
        case 2:
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(d),
                "l"(mp), "r"(c[0]), "r"(c[1]), "r"(b)
                : "memory");
            break;
        case 3:
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(d),
                "l"(mp), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(b)
                : "memory");
            break;
        case 4:
            asm volatile(
                "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(d),
                "l"(mp), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(b)
                : "memory");
            break;
        default:
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(d),
                "l"(mp), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b)
                : "memory");
            break;
    }
}

// Tensor copy shared -> global of one box (bulk-group completion).
__device__ __forceinline__ void tma_store(const TMap *m, int nd, const int *c, const void *src) {
    const unsigned s = saddr(src);
    const u64 mp = reinterpret_cast<u64>(m);
    switch (nd) {
        case 1:
            asm volatile("cp.async.bulk.tensor.1d.global.shared::cta.bulk_group [%0, {%1}], [%2];" ::"l"(mp), "r"(c[0]), "r"(s)
                         : "memory");
            break;
        case 2:
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(mp), "r"(c[0]),
                         "r"(c[1]), "r"(s)
                         : "memory");
            break;
        case 3:
            asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(mp), "r"(c[0]),
                         "r"(c[1]), "r"(c[2]), "r"(s)
                         : "memory");
            break;
        case 4:
            asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(mp),
                         "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(s)
                         : "memory");
            break;
        default:
            asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(mp),
                         "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(s)
                         : "memory");
            break;
    }
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The shared-memory sources of every committed store have been read.
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Every committed store is complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Coordinates of the box with loop value v of the tile whose first global element index is `base`
// (batch index included above the state's qubits).
__device__ __forceinline__ void box_coords(const TmaGeom &t, u64 base, int v, int *c) {
    for (int k = 0; k < t.n_loop; ++k)
        if (v >> k & 1) base |= u64(1) << t.loop_q[k];
    for (int j = 0; j < t.nd; ++j) {
        u64 x = base >> t.shift[j];
        if (j + 1 < t.nd) x &= (u64(1) << (t.shift[j + 1] - t.shift[j])) - 1;
        if (j == 0) x *= u64(t.epa);
        c[j] = static_cast<int>(x);
    }
}

// Issue the loads of one tile of `map` into `dst` (2^n_loop boxes of box_bytes each).
__device__ __forceinline__ void load_tile(const TMap *m, const TmaGeom &t, u64 base, unsigned char *dst, u64 *bar) {
    int c[5];
    for (int v = 0; v < (1 << t.n_loop); ++v) {
        box_coords(t, base, v, c);
        tma_load(dst + static_cast<u64>(v) * t.box_bytes, m, t.nd, c, bar);
    }
}

__device__ __forceinline__ void store_tile(const TMap *m, const TmaGeom &t, u64 base, const unsigned char *src) {
    int c[5];
    for (int v = 0; v < (1 << t.n_loop); ++v) {
        box_coords(t, base, v, c);
        tma_store(m, t.nd, c, src + static_cast<u64>(v) * t.box_bytes);
    }
}

__device__ __forceinline__ void report(int *err, int code) {
    if (err) atomicCAS(err, 0, code);
}

}  // namespace pipe
}  // namespace mqb

#endif
