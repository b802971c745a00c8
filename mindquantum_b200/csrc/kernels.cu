// CUDA kernels of the mqb200 state-vector engine (sm_100a).
//
//   matgen      : per (sample, gate) gate matrices and their angle derivatives from the
//                 parameter vector (the reference evaluates ParameterResolver::Combination and
//                 builds a matrix per gate per call on the host, vector_state.tpp:236-343).
//   (the fused tile passes live in fused.cu)
//   ham         : lambda = H psi and/or <bra|H|ket> for a group of Pauli terms whose flip masks fit
//                 in one tile; terms with a common flip mask share one partner read
//                 (replaces ApplyTerms / ExpectationOfTerms' pass per term, cpu_vector_core_policy.cpp:133-261).
//   plain_*     : one kernel per gate over the whole state (the unfused schedule of the reference).
//   sampling    : chunked |psi|^2 sums, prefix, per-shot search (GetCumulativeProbs + LowerBound).
//
// Every reduction accumulates in FP64 (per-thread partials, warp shuffles, per-warp shared
// slots, one atomicAdd per block per slot).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "kernels.cuh"
#include "pipe.cuh"

namespace mqb {

// ------------------------------------------------------------------------------------------ helpers
template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename V>
__device__ __forceinline__ V cadd(V a, V b) {
    V r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
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
__device__ __forceinline__ V czero() {
    V r;
    r.x = 0;
    r.y = 0;
    return r;
}
template <typename V, typename W>
__device__ __forceinline__ V cvt(W a) {
    V r;
    r.x = a.x;
    r.y = a.y;
    return r;
}
__device__ __forceinline__ double dmk_re(double2 a) { return a.x; }

__device__ __forceinline__ uint32_t ins0(uint32_t x, int b) {
    const uint32_t lo = x & ((1u << b) - 1u);
    return ((x >> b) << (b + 1)) | lo;
}
__device__ __forceinline__ uint64_t ins0_64(uint64_t x, int b) {
    const uint64_t lo = x & ((uint64_t(1) << b) - 1);
    return ((x >> b) << (b + 1)) | lo;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint64_t tile_base(const TileGeom &g, uint64_t t) {
    uint64_t base = 0;
    for (int i = 0; i < g.n_out; ++i)
        if (t >> i & 1) base |= uint64_t(1) << g.outside[i];
    return base;
}

__device__ __forceinline__ void build_table(uint64_t *tab, const TileGeom &g) {
    const int nh = 1 << (g.K - g.c);
    for (int h = threadIdx.x; h < nh; h += blockDim.x) {
        uint64_t off = 0;
        for (int i = 0; i < g.K - g.c; ++i)
            if (h >> i & 1) off |= uint64_t(1) << g.qbits[g.c + i];
        tab[h] = off;
    }
}

template <typename V>
__device__ __forceinline__ void load_tile(V *tile, const V *src, uint64_t base, const uint64_t *tab, int K, int c) {
    constexpr int APV = 16 / sizeof(V);
    const int nvec = (1 << K) / APV;
    const uint32_t lowmask = (1u << c) - 1u;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const uint32_t L = uint32_t(v) * APV;
        const uint64_t gi = base + tab[L >> c] + (L & lowmask);
        *reinterpret_cast<uint4 *>(&tile[L]) = __ldg(reinterpret_cast<const uint4 *>(src + gi));
    }
}

template <typename V>
__device__ __forceinline__ void store_tile(const V *tile, V *dst, uint64_t base, const uint64_t *tab, int K, int c) {
    constexpr int APV = 16 / sizeof(V);
    const int nvec = (1 << K) / APV;
    const uint32_t lowmask = (1u << c) - 1u;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        const uint32_t L = uint32_t(v) * APV;
        const uint64_t gi = base + tab[L >> c] + (L & lowmask);
        *reinterpret_cast<uint4 *>(dst + gi) = *reinterpret_cast<const uint4 *>(&tile[L]);
    }
}

template <typename V>
__device__ __forceinline__ void zero_tile(V *tile, uint64_t base, int K) {
    for (int L = threadIdx.x; L < (1 << K); L += blockDim.x) {
        V v = czero<V>();
        if (base == 0 && L == 0) v.x = 1;
        tile[L] = v;
    }
}

__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// ------------------------------------------------------------------------------------------ matgen
// Gate matrices in double precision; index bit b <-> object qubit b.  Dense matrices are
// row-major 2^m x 2^m, diagonal gates store the diagonal only.
struct GateMats {
    double2 M[16];
    double2 D[3][16];
};

__device__ __forceinline__ double2 z2(double x, double y) { return make_double2(x, y); }

__device__ void pauli2(int p, double2 out[4]) {  // 0 I, 1 X, 2 Y, 3 Z
    out[0] = out[1] = out[2] = out[3] = z2(0, 0);
    if (p == 0) {
        out[0] = out[3] = z2(1, 0);
    } else if (p == 1) {
        out[1] = out[2] = z2(1, 0);
    } else if (p == 2) {
        out[1] = z2(0, -1);
        out[2] = z2(0, 1);
    } else {
        out[0] = z2(1, 0);
        out[3] = z2(-1, 0);
    }
}

// exp(-i t/2 P0 (x) P1) and its t-derivative, P0 on object qubit 0 (index bit 0)
__device__ void two_qubit_rotation(int p0, int p1, double t, double2 *M, double2 *D) {
    double2 a[4], b[4];
    pauli2(p0, a);
    pauli2(p1, b);
    const double c = cos(t / 2), s = sin(t / 2);
    for (int r = 0; r < 4; ++r) {
        for (int col = 0; col < 4; ++col) {
            const double2 pa = a[(r & 1) * 2 + (col & 1)];
            const double2 pb = b[(r >> 1) * 2 + (col >> 1)];
            const double2 p = z2(pa.x * pb.x - pa.y * pb.y, pa.x * pb.y + pa.y * pb.x);
            const double id = (r == col) ? 1.0 : 0.0;
            // M = c I - i s P ; D = 0.5 (-s I - i c P)
            M[r * 4 + col] = z2(c * id + s * p.y, -s * p.x);
            D[r * 4 + col] = z2(0.5 * (-s * id + c * p.y), -0.5 * c * p.x);
        }
    }
}

__device__ void gate_mats(int gid, const double *t, GateMats &g) {
    for (int i = 0; i < 16; ++i) {
        g.M[i] = z2(0, 0);
        g.D[0][i] = g.D[1][i] = g.D[2][i] = z2(0, 0);
    }
    switch (gid) {
        case GID_RX: {
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            g.M[0] = z2(c, 0), g.M[1] = z2(0, -s), g.M[2] = z2(0, -s), g.M[3] = z2(c, 0);
            g.D[0][0] = z2(-s / 2, 0), g.D[0][1] = z2(0, -c / 2), g.D[0][2] = z2(0, -c / 2), g.D[0][3] = z2(-s / 2, 0);
        } break;
        case GID_RY: {
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            g.M[0] = z2(c, 0), g.M[1] = z2(-s, 0), g.M[2] = z2(s, 0), g.M[3] = z2(c, 0);
            g.D[0][0] = z2(-s / 2, 0), g.D[0][1] = z2(-c / 2, 0), g.D[0][2] = z2(c / 2, 0), g.D[0][3] = z2(-s / 2, 0);
        } break;
        case GID_RZ: {  // diagonal
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            g.M[0] = z2(c, -s), g.M[1] = z2(c, s);
            g.D[0][0] = z2(-s / 2, -c / 2), g.D[0][1] = z2(-s / 2, c / 2);
        } break;
        case GID_PS: {  // diagonal
            const double c = cos(t[0]), s = sin(t[0]);
            g.M[0] = z2(1, 0), g.M[1] = z2(c, s);
            g.D[0][0] = z2(0, 0), g.D[0][1] = z2(-s, c);
        } break;
        case GID_GP: {  // diagonal
            const double c = cos(t[0]), s = sin(t[0]);
            g.M[0] = g.M[1] = z2(c, -s);
            g.D[0][0] = g.D[0][1] = z2(-s, -c);
        } break;
        case GID_RZZ: {  // diagonal
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            for (int r = 0; r < 4; ++r) {
                const double z = (r == 0 || r == 3) ? 1.0 : -1.0;
                g.M[r] = z2(c, -s * z);
                g.D[0][r] = z2(-s / 2, -c / 2 * z);
            }
        } break;
        case GID_RXX: two_qubit_rotation(1, 1, t[0], g.M, g.D[0]); break;
        case GID_RYY: two_qubit_rotation(2, 2, t[0], g.M, g.D[0]); break;
        case GID_RXY: two_qubit_rotation(1, 2, t[0], g.M, g.D[0]); break;
        case GID_RXZ: two_qubit_rotation(1, 3, t[0], g.M, g.D[0]); break;
        case GID_RYZ: two_qubit_rotation(2, 3, t[0], g.M, g.D[0]); break;
        case GID_GIVENS: {
            const double c = cos(t[0]), s = sin(t[0]);
            g.M[0] = z2(1, 0), g.M[5] = z2(c, 0), g.M[6] = z2(-s, 0), g.M[9] = z2(s, 0), g.M[10] = z2(c, 0);
            g.M[15] = z2(1, 0);
            g.D[0][5] = z2(-s, 0), g.D[0][6] = z2(-c, 0), g.D[0][9] = z2(c, 0), g.D[0][10] = z2(-s, 0);
        } break;
        case GID_SWAPALPHA: {
            const double c = cos(M_PI * t[0]), s = sin(M_PI * t[0]);
            const double2 a = z2((1 + c) / 2, s / 2), b = z2((1 - c) / 2, -s / 2);
            g.M[0] = z2(1, 0), g.M[5] = a, g.M[6] = b, g.M[9] = b, g.M[10] = a, g.M[15] = z2(1, 0);
            const double2 de = z2(-M_PI / 2 * s, M_PI / 2 * c);
            g.D[0][5] = de, g.D[0][6] = z2(-de.x, -de.y), g.D[0][9] = z2(-de.x, -de.y), g.D[0][10] = de;
        } break;
        case GID_U3: {
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            const double2 el = z2(cos(t[2]), sin(t[2])), ep = z2(cos(t[1]), sin(t[1]));
            const double2 elp = z2(el.x * ep.x - el.y * ep.y, el.x * ep.y + el.y * ep.x);
            g.M[0] = z2(c, 0), g.M[1] = z2(-el.x * s, -el.y * s), g.M[2] = z2(ep.x * s, ep.y * s);
            g.M[3] = z2(elp.x * c, elp.y * c);
            g.D[0][0] = z2(-s / 2, 0), g.D[0][1] = z2(-el.x * c / 2, -el.y * c / 2);
            g.D[0][2] = z2(ep.x * c / 2, ep.y * c / 2), g.D[0][3] = z2(-elp.x * s / 2, -elp.y * s / 2);
            // d/dphi: i * (lower row)
            g.D[1][2] = z2(-ep.y * s, ep.x * s), g.D[1][3] = z2(-elp.y * c, elp.x * c);
            // d/dlambda: i * (right column)
            g.D[2][1] = z2(el.y * s, -el.x * s), g.D[2][3] = z2(-elp.y * c, elp.x * c);
        } break;
        case GID_RN: {
            const double a = t[0], b = t[1], cc = t[2];
            const double f = sqrt(a * a + b * b + cc * cc);
            if (f == 0) {
                g.M[0] = g.M[3] = z2(1, 0);
                break;
            }
            const double co = cos(f / 2), si = sin(f / 2);
            // M = cos(f/2) I - i sin(f/2) (a X + b Y + c Z) / f
            g.M[0] = z2(co, -si * cc / f);
            g.M[1] = z2(-si * b / f, -si * a / f);
            g.M[2] = z2(si * b / f, -si * a / f);
            g.M[3] = z2(co, si * cc / f);
            // dM/dk = -(k/f)(si/2) I - i h (k/f)(co/(2f) - si/f^2) - i sigma_k si/f, h = aX + bY + cZ
            const double comp[3] = {a, b, cc};
            for (int k = 0; k < 3; ++k) {
                const double fk = comp[k] / f;
                const double w = fk * (co / (2 * f) - si / (f * f));
                double2 h[4] = {z2(cc, 0), z2(a, -b), z2(a, b), z2(-cc, 0)};
                double2 sg[4];
                pauli2(k + 1, sg);
                for (int e = 0; e < 4; ++e) {
                    const double idd = (e == 0 || e == 3) ? 1.0 : 0.0;
                    // -i * h * w  -> (h.y * w, -h.x * w);  -i * sg * si/f -> (sg.y*si/f, -sg.x*si/f)
                    g.D[k][e] = z2(-fk * si / 2 * idd + h[e].y * w + sg[e].y * si / f, -h[e].x * w - sg[e].x * si / f);
                }
            }
        } break;
        case GID_FSIM: {
            const double c = cos(t[0]), s = sin(t[0]);
            g.M[0] = z2(1, 0), g.M[5] = z2(c, 0), g.M[6] = z2(0, -s), g.M[9] = z2(0, -s), g.M[10] = z2(c, 0);
            g.M[15] = z2(cos(t[1]), -sin(t[1]));
            g.D[0][5] = z2(-s, 0), g.D[0][6] = z2(0, -c), g.D[0][9] = z2(0, -c), g.D[0][10] = z2(-s, 0);
            g.D[1][15] = z2(-sin(t[1]), -cos(t[1]));
        } break;
        case GID_RPS: {
            const double c = cos(t[0] / 2), s = sin(t[0] / 2);
            g.M[0] = z2(c, s);
            g.D[0][0] = z2(-s / 2, c / 2);
        } break;
        default:
            break;
    }
}

template <typename R>
__global__ void matgen_kernel(MatgenArgs a) {
    using V = cplx<R>;
    const int64_t total = a.batch * a.n_ops;
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < total; w += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = w / a.n_ops;
        const int k = int(w % a.n_ops);
        const DevOp &op = a.ops[k];
        if (!op.per_sample) continue;
        V *out = reinterpret_cast<V *>(a.mats) + b * a.mats_stride;
        if (op.gate_id == GID_CUSTOM) {
            const double2 *src = reinterpret_cast<const double2 *>(a.custom) + b * a.custom_stride + op.custom_off;
            for (int e = 0; e < op.mat_size; ++e) out[op.mat_off + e] = cvt<V>(src[e]);
            if (op.grad_mask)
                for (int e = 0; e < op.mat_size; ++e) out[op.dmat_off + e] = cvt<V>(src[op.mat_size + e]);
            continue;
        }
        const mqb_gate_desc &d = a.descs[k];
        double t[3] = {0, 0, 0};
        const double *p = a.params + b * a.param_stride;
        for (int an = 0; an < d.n_angles; ++an) {
            double v = d.angle_const[an];
            for (int q = d.term_begin[an]; q < d.term_begin[an] + d.term_count[an]; ++q)
                v += a.terms[q].coeff * p[a.terms[q].param];
            t[an] = v;
        }
        GateMats gm;
        gate_mats(op.gate_id, t, gm);
        for (int e = 0; e < op.mat_size; ++e) out[op.mat_off + e] = cvt<V>(gm.M[e]);
        if (op.grad_mask)
            for (int an = 0; an < op.n_angles; ++an)
                for (int e = 0; e < op.mat_size; ++e)
                    out[op.dmat_off + an * op.mat_size + e] = cvt<V>(gm.D[an][e]);
    }
}

template <typename R>
cudaError_t launch_matgen(const MatgenArgs &a, cudaStream_t s) {
    const int64_t total = a.batch * a.n_ops;
    if (total == 0) return cudaSuccess;
    const int threads = 128;
    const int blocks = int(std::min<int64_t>((total + threads - 1) / threads, 4096));
    matgen_kernel<R><<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename KernelT>
static int blocks_for(KernelT kern, size_t smem, int sm_count, int64_t work) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t want = int64_t(sm_count) * per_sm;
    return int(std::max<int64_t>(1, std::min<int64_t>(want, work)));
}

// ------------------------------------------------------------------------------------------ Hamiltonian
size_t ham_smem(const TileGeom &g, int elem_bytes) {
    size_t s = (size_t(1) << g.K) * elem_bytes;
    s = (s + 15) & ~size_t(15);
    s += (size_t(1) << (g.K - g.c)) * sizeof(uint64_t);
    s = (s + 15) & ~size_t(15);
    s += size_t(kThreads / 32) * 2 * sizeof(double);
    return s;
}

template <typename R>
__global__ void __launch_bounds__(kThreads) ham_kernel(const HamArgs<R> a) {
    using V = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem[];
    const TileGeom &g = a.g;
    const int K = g.K, c = g.c;
    const int TS = 1 << K;
    V *ket = reinterpret_cast<V *>(smem);
    size_t o = align16(size_t(TS) * sizeof(V));
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + o);
    o = align16(o + (size_t(1) << (K - c)) * sizeof(uint64_t));
    double *wf = reinterpret_cast<double *>(smem + o);  // [warps][2]
    const int nw = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    build_table(tab, g);
    for (int i = threadIdx.x; i < nw * 2; i += blockDim.x) wf[i] = 0;
    __syncthreads();
    const int64_t n_tiles = int64_t(1) << g.n_out;
    const int64_t dim = int64_t(1) << g.n;
    const int64_t total = a.batch * n_tiles;
    const uint32_t lowmask = (1u << c) - 1u;
    for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
        const int64_t b = w >> g.n_out;
        const uint64_t t = uint64_t(w) & uint64_t(n_tiles - 1);
        const uint64_t base = tile_base(g, t);
        load_tile(ket, a.ket + b * dim, base, tab, K, c);
        __syncthreads();
        double fr = 0, fi = 0;
        for (int L = threadIdx.x; L < TS; L += blockDim.x) {
            double ar = 0, ai = 0;   // (H ket)_L in FP64
            for (int k = 0; k < a.n_classes; ++k) {
                const HamClass &hc = a.classes[k];
                const uint32_t i = uint32_t(L) ^ hc.lflip;
                const uint64_t gi = base + tab[i >> c] + (i & lowmask);
                double wr = 0, wi = 0;   // sum_t coeff_t * phase_t(gi)
                for (int q = hc.term_begin; q < hc.term_begin + hc.term_count; ++q) {
                    const HamTerm &ht = a.terms[q];
                    const int ph = (ht.ny + 2 * __popcll(gi & ht.my_mz)) & 3;
                    // POLAR: 1, i, -1, -i
                    wr += (ph == 0) ? ht.coeff : (ph == 2 ? -ht.coeff : 0.0);
                    wi += (ph == 1) ? ht.coeff : (ph == 3 ? -ht.coeff : 0.0);
                }
                const V kv = ket[i];
                ar += wr * double(kv.x) - wi * double(kv.y);
                ai += wr * double(kv.y) + wi * double(kv.x);
            }
            const uint64_t gL = base + tab[uint32_t(L) >> c] + (uint32_t(L) & lowmask);
            if (a.fout) {
                const V bv = a.bra[b * dim + gL];
                fr += double(bv.x) * ar + double(bv.y) * ai;
                fi += double(bv.x) * ai - double(bv.y) * ar;
            }
            if (a.out) {
                V *op = a.out + b * a.out_batch_stride + gL;
                V r;
                if (a.accumulate) {
                    const V old = *op;
                    r.x = old.x + ar;
                    r.y = old.y + ai;
                } else {
                    r.x = ar;
                    r.y = ai;
                }
                *op = r;
            }
        }
        if (a.fout) {
            fr = warp_sum(fr);
            fi = warp_sum(fi);
            if (lane == 0) {
                wf[warp * 2] += fr;
                wf[warp * 2 + 1] += fi;
            }
        }
        const int64_t nxt = w + gridDim.x;
        const bool flush = (nxt >= total) || ((nxt >> g.n_out) != b);
        __syncthreads();
        if (flush && a.fout) {
            if (threadIdx.x < 2) {
                double s = 0;
                for (int ww = 0; ww < nw; ++ww) {
                    s += wf[ww * 2 + threadIdx.x];
                    wf[ww * 2 + threadIdx.x] = 0;
                }
                atomicAdd(&a.fout[b * a.f_stride + threadIdx.x], s);
            }
            __syncthreads();
        }
    }
}

// The weighted partner sums of one tile for one thread: for every flip class k of the group,
// out[r] += W_k(L_r) * ket[L_r ^ flip_k] over the thread's NR = 2^NRB amplitudes L_r = tid + T r.
// `at(r, f)` is the shared-memory index of the amplitude L_r ^ f, sflip[k] class k's flip in the
// same index space.  W_k comes from the terms' signs, split into the thread part popc(tid & m) and
// the register part popc((r << hi_shift) & m): a Walsh-Hadamard transform over r of per-bin sums
// when the class has more than two terms.
template <typename R, int NRB, typename At>
__device__ __forceinline__ void ham_classes(const cplx<R> *ket, At at, const HamClass *cls, const uint32_t *sflip,
                                            int n_classes, int term_begin, const uint32_t *tmask,
                                            const cplx<R> *tcoef, int hi_shift, R (&ar)[1 << NRB],
                                            R (&ai)[1 << NRB]) {
    using V = cplx<R>;
    constexpr int NR = 1 << NRB;
    const int tid = threadIdx.x;
    for (int k = 0; k < n_classes; ++k) {
        const HamClass &hc = cls[k];
        const int tb = hc.term_begin - term_begin;
        R wr[NR], wi[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) wr[r] = wi[r] = 0;
        uint32_t any_mask = 0;
        if (hc.term_count <= 2)
            for (int q = tb; q < tb + hc.term_count; ++q) any_mask |= tmask[q];
        if (hc.term_count <= 2 && any_mask == 0) {
            // no sign on the tile's bits (X-type terms): one weight for every amplitude
            R cr = 0, ci = 0;
            for (int q = tb; q < tb + hc.term_count; ++q) {
                cr += tcoef[q].x;
                ci += tcoef[q].y;
            }
            const uint32_t f = sflip[k];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const V kv = ket[at(r, f)];
                ar[r] = fma(cr, kv.x, fma(-ci, kv.y, ar[r]));
                ai[r] = fma(cr, kv.y, fma(ci, kv.x, ai[r]));
            }
            continue;
        }
        if (hc.term_count <= 2) {
            for (int q = tb; q < tb + hc.term_count; ++q) {
                const uint32_t m = tmask[q];
                const V cq = tcoef[q];
                const uint32_t pt = __popc(uint32_t(tid) & m);
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const bool neg = (pt + __popc((uint32_t(r) << hi_shift) & m)) & 1;
                    wr[r] += neg ? -cq.x : cq.x;
                    wi[r] += neg ? -cq.y : cq.y;
                }
            }
        } else {
#pragma unroll
            for (int bn = 0; bn < NR; ++bn) {
                for (int q = tb + hc.bins[bn]; q < tb + hc.bins[bn + 1]; ++q) {
                    const V cq = tcoef[q];
                    const bool neg = __popc(uint32_t(tid) & tmask[q]) & 1;
                    wr[bn] += neg ? -cq.x : cq.x;
                    wi[bn] += neg ? -cq.y : cq.y;
                }
            }
#pragma unroll
            for (int sb = 0; sb < NRB; ++sb)
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    if (r >> sb & 1) continue;
                    const int r2 = r | (1 << sb);
                    const R xr = wr[r], xi = wi[r];
                    wr[r] = xr + wr[r2];
                    wi[r] = xi + wi[r2];
                    wr[r2] = xr - wr[r2];
                    wi[r2] = xi - wi[r2];
                }
        }
        const uint32_t f = sflip[k];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const V kv = ket[at(r, f)];
            ar[r] = fma(wr[r], kv.x, fma(-wi[r], kv.y, ar[r]));
            ai[r] = fma(wr[r], kv.y, fma(wi[r], kv.x, ai[r]));
        }
    }
}

// Register-binned Hamiltonian pass.  Every thread owns the NR = 2^NRB amplitudes L = tid + T r of
// a tile (T = 2^(K - NRB) threads), so the sign (-1)^popc(L & m) of a Pauli term splits into a
// per-thread part popc(tid & m) and a per-register part popc(r & m_hi).  A class's weight
// W(L) = sum_t c_t (-1)^popc(L & m_t) is then, for the thread's amplitudes, the Walsh-Hadamard
// transform over r of bins B[m_hi] = sum_t c_t (-1)^popc(tid & m_t): one signed add per term and
// NRB * NR butterflies per thread instead of one popcount per term and amplitude.  The outside
// qubits' signs are folded into the terms' coefficients once per tile.
template <typename R, int NRB>
__global__ void __launch_bounds__(sizeof(R) == 4 ? 512 : 256) ham2_kernel(const HamArgs<R> a) {
    using V = cplx<R>;
    constexpr int NR = 1 << NRB;
    extern __shared__ __align__(16) unsigned char smem[];
    const TileGeom &g = a.g;
    const int K = g.K, c = g.c;
    const int TS = 1 << K;
    const int T = blockDim.x, tid = threadIdx.x;
    const int nt = a.n_terms;
    V *ket = reinterpret_cast<V *>(smem);
    size_t o = align16(size_t(TS) * sizeof(V));
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + o);
    o = align16(o + (size_t(1) << (K - c)) * sizeof(uint64_t));
    double *wf = reinterpret_cast<double *>(smem + o);
    o = align16(o + size_t(T / 32) * 2 * sizeof(double));
    HamClass *cls = reinterpret_cast<HamClass *>(smem + o);
    o = align16(o + size_t(a.n_classes) * sizeof(HamClass));
    V *tcoef = reinterpret_cast<V *>(smem + o);
    o = align16(o + size_t(nt) * sizeof(V));
    uint32_t *tmask = reinterpret_cast<uint32_t *>(smem + o);
    o = align16(o + size_t(nt) * sizeof(uint32_t));
    uint32_t *sflip = reinterpret_cast<uint32_t *>(smem + o);
    o = align16(o + size_t(a.n_classes) * sizeof(uint32_t));
    // groups after the first add to the output: their previous sum is staged with the tile
    V *prev = nullptr;
    if (a.accumulate && a.out) prev = reinterpret_cast<V *>(smem + o);
    const int nw = T / 32, warp = tid / 32, lane = tid % 32;
    build_table(tab, g);
    for (int i = tid; i < nw * 2; i += T) wf[i] = 0;
    for (int i = tid; i < a.n_classes; i += T) {
        cls[i] = a.classes[i];
        sflip[i] = a.classes[i].lflip;
    }
    for (int i = tid; i < nt; i += T) tmask[i] = a.terms[a.term_begin + i].lmask;
    __syncthreads();
    const int64_t n_tiles = int64_t(1) << g.n_out;
    const int64_t dim = int64_t(1) << g.n;
    const int64_t total = a.batch * n_tiles;
    const uint32_t lowmask = (1u << c) - 1u;
    const int hi_shift = K - NRB;
    const bool bra_is_ket = a.bra == a.ket;
    for (int64_t w = blockIdx.x; w < total; w += gridDim.x) {
        const int64_t b = w >> g.n_out;
        const uint64_t t = uint64_t(w) & uint64_t(n_tiles - 1);
        const uint64_t base = tile_base(g, t);
        load_tile(ket, a.ket + b * dim, base, tab, K, c);
        if (prev) load_tile(prev, a.out + b * a.out_batch_stride, base, tab, K, c);
        for (int q = tid; q < nt; q += T) {
            const HamTerm &ht = a.terms[a.term_begin + q];
            const bool neg = __popcll(base & ht.omask) & 1;
            V cq;
            cq.x = R(neg ? -ht.cb_re : ht.cb_re);
            cq.y = R(neg ? -ht.cb_im : ht.cb_im);
            tcoef[q] = cq;
        }
        __syncthreads();
        R ar[NR], ai[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) ar[r] = ai[r] = 0;
        ham_classes<R, NRB>(
            ket, [&](int r, uint32_t f) { return uint32_t(tid + T * r) ^ f; }, cls, sflip, a.n_classes, a.term_begin,
            tmask, tcoef, hi_shift, ar, ai);
        double fr = 0, fi = 0;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const uint32_t L = uint32_t(tid + T * r);
            const uint64_t gL = base + tab[L >> c] + (L & lowmask);
            if (a.fout) {
                // <psi|H psi> (bra == ket): the bra amplitudes are the staged tile's
                const V bv = bra_is_ket ? ket[L] : a.bra[b * dim + gL];
                fr += double(bv.x) * double(ar[r]) + double(bv.y) * double(ai[r]);
                fi += double(bv.x) * double(ai[r]) - double(bv.y) * double(ar[r]);
            }
            if (a.out) {
                V *op = a.out + b * a.out_batch_stride + gL;
                V v;
                v.x = ar[r];
                v.y = ai[r];
                if (a.accumulate) {
                    const V old = prev[L];
                    v.x += old.x;
                    v.y += old.y;
                }
                *op = v;
            }
        }
        if (a.fout) {
            fr = warp_sum(fr);
            fi = warp_sum(fi);
            if (lane == 0) {
                wf[warp * 2] += fr;
                wf[warp * 2 + 1] += fi;
            }
        }
        const int64_t nxt = w + gridDim.x;
        const bool flush = (nxt >= total) || ((nxt >> g.n_out) != b);
        __syncthreads();
        if (flush && a.fout) {
            if (tid < 2) {
                double s2 = 0;
                for (int ww = 0; ww < nw; ++ww) {
                    s2 += wf[ww * 2 + tid];
                    wf[ww * 2 + tid] = 0;
                }
                atomicAdd(&a.fout[b * a.f_stride + tid], s2);
            }
            __syncthreads();
        }
    }
}

// The register-binned pass with its tiles moved by the TMA.  NB shared buffers per operand (the
// tile, and the previous groups' sum when the group adds to the output) are filled by tensor
// copies (cp.async.bulk.tensor, no multicast) that complete on one mbarrier per buffer.  The
// block's tiles are w = blockIdx.x + i gridDim.x; thread 0 starts tile i + NB into buffer i % NB
// once the whole block has finished tile i, so the copies of the next tiles run under the current
// tile's classes.  A tile lies in shared memory in the copies' landing order (tile bit j at
// position land[j]); the index map is a bit permutation, so a flip is an XOR there too.  Every
// wait is bounded: a timeout sets the error word and ends the block after its copies drained.
template <typename R, int NRB>
__global__ void __launch_bounds__(256) ham_ring_kernel(const HamArgs<R> a, const HamRingGeom rg,
                                                       const __grid_constant__ pipe::TMap mk,
                                                       const __grid_constant__ pipe::TMap mo) {
    using V = cplx<R>;
    constexpr int NR = 1 << NRB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // tile buffers on 128-byte boundaries (the launch adds 128 bytes for this)
    unsigned char *smem = smem_raw + ((128u - (pipe::saddr(smem_raw) & 127u)) & 127u);
    const TileGeom &g = a.g;
    const int K = g.K, c = g.c;
    const int TS = 1 << K;
    const int T = blockDim.x, tid = threadIdx.x;
    const int nt = a.n_terms, NB = rg.nb;
    const bool staged = a.accumulate && a.out && rg.stage_prev;
    const size_t tile_bytes = size_t(TS) * sizeof(V);
    V *ring = reinterpret_cast<V *>(smem);
    V *pring = reinterpret_cast<V *>(smem + size_t(NB) * tile_bytes);
    size_t o = size_t(staged ? 2 : 1) * NB * tile_bytes;
    pipe::u64 *full = reinterpret_cast<pipe::u64 *>(smem + o);
    o = align16(o + size_t(NB) * sizeof(pipe::u64));
    uint64_t *tab = reinterpret_cast<uint64_t *>(smem + o);
    o = align16(o + (size_t(1) << (K - c)) * sizeof(uint64_t));
    double *wf = reinterpret_cast<double *>(smem + o);
    o = align16(o + size_t(T / 32) * 2 * sizeof(double));
    HamClass *cls = reinterpret_cast<HamClass *>(smem + o);
    o = align16(o + size_t(a.n_classes) * sizeof(HamClass));
    V *tcoef = reinterpret_cast<V *>(smem + o);
    o = align16(o + size_t(nt) * sizeof(V));
    uint32_t *tmask = reinterpret_cast<uint32_t *>(smem + o);
    o = align16(o + size_t(nt) * sizeof(uint32_t));
    uint32_t *sflip = reinterpret_cast<uint32_t *>(smem + o);
    const int nw = T / 32, warp = tid / 32, lane = tid % 32;
    auto land = [&](uint32_t L) {
        uint32_t x = 0;
        for (int j = 0; j < K; ++j)
            if (L >> j & 1) x |= 1u << rg.land[j];
        return x;
    };
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) pipe::mbar_init(&full[b], 1);
        pipe::fence_mbar_init();
    }
    build_table(tab, g);
    for (int i = tid; i < nw * 2; i += T) wf[i] = 0;
    for (int i = tid; i < a.n_classes; i += T) {
        cls[i] = a.classes[i];
        sflip[i] = land(a.classes[i].lflip);
    }
    for (int i = tid; i < nt; i += T) tmask[i] = a.terms[a.term_begin + i].lmask;
    const int hi_shift = K - NRB;
    const uint32_t lt = land(uint32_t(tid));
    uint32_t lr[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) lr[r] = land(uint32_t(r) << hi_shift);
    __syncthreads();
    const int64_t n_tiles = int64_t(1) << g.n_out;
    const int64_t dim = int64_t(1) << g.n;
    const int64_t total = a.batch * n_tiles;
    const int64_t first = blockIdx.x, step = gridDim.x;
    const int64_t count = first < total ? (total - first + step - 1) / step : 0;
    const uint32_t lowmask = (1u << c) - 1u;
    const bool bra_is_ket = a.bra == a.ket;
    const unsigned tx = unsigned(tile_bytes) * (staged ? 2u : 1u);
    auto issue = [&](int64_t i) {   // thread 0: the copies of the block's tile i into buffer i % NB
        const int64_t w = first + i * step;
        const uint64_t gb = (uint64_t(w >> g.n_out) << g.n) | tile_base(g, uint64_t(w) & uint64_t(n_tiles - 1));
        const int buf = int(i % NB);
        pipe::mbar_expect_tx(&full[buf], tx);
        pipe::load_tile(&mk, rg.tg, gb, reinterpret_cast<unsigned char *>(ring + size_t(buf) * TS), &full[buf]);
        if (staged)
            pipe::load_tile(&mo, rg.tg, gb, reinterpret_cast<unsigned char *>(pring + size_t(buf) * TS), &full[buf]);
    };
    if (tid == 0)
        for (int64_t i = 0; i < NB && i < count; ++i) issue(i);
    int64_t i = 0;
    bool failed = false;
    for (; i < count; ++i) {
        const int buf = int(i % NB);
        if (!__syncthreads_and(pipe::mbar_wait(&full[buf], unsigned(i / NB) & 1u))) {
            failed = true;
            break;
        }
        const int64_t w = first + i * step;
        const int64_t b = w >> g.n_out;
        const uint64_t base = tile_base(g, uint64_t(w) & uint64_t(n_tiles - 1));
        const V *ket = ring + size_t(buf) * TS;
        const V *prev = pring + size_t(buf) * TS;
        for (int q = tid; q < nt; q += T) {
            const HamTerm &ht = a.terms[a.term_begin + q];
            const bool neg = __popcll(base & ht.omask) & 1;
            V cq;
            cq.x = R(neg ? -ht.cb_re : ht.cb_re);
            cq.y = R(neg ? -ht.cb_im : ht.cb_im);
            tcoef[q] = cq;
        }
        __syncthreads();
        R ar[NR], ai[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) ar[r] = ai[r] = 0;
        ham_classes<R, NRB>(
            ket, [&](int r, uint32_t f) { return (lt | lr[r]) ^ f; }, cls, sflip, a.n_classes, a.term_begin, tmask,
            tcoef, hi_shift, ar, ai);
        double fr = 0, fi = 0;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const uint32_t L = uint32_t(tid + T * r);
            const uint64_t gL = base + tab[L >> c] + (L & lowmask);
            if (a.fout) {
                const V bv = bra_is_ket ? ket[lt | lr[r]] : a.bra[b * dim + gL];
                fr += double(bv.x) * double(ar[r]) + double(bv.y) * double(ai[r]);
                fi += double(bv.x) * double(ai[r]) - double(bv.y) * double(ar[r]);
            }
            if (a.out) {
                V v;
                v.x = ar[r];
                v.y = ai[r];
                if (a.accumulate) {
                    const V old = staged ? prev[lt | lr[r]] : a.out[b * a.out_batch_stride + gL];
                    v.x += old.x;
                    v.y += old.y;
                }
                a.out[b * a.out_batch_stride + gL] = v;
            }
        }
        if (a.fout) {
            fr = warp_sum(fr);
            fi = warp_sum(fi);
            if (lane == 0) {
                wf[warp * 2] += fr;
                wf[warp * 2 + 1] += fi;
            }
        }
        const int64_t nxt = w + step;
        const bool flush = (nxt >= total) || ((nxt >> g.n_out) != b);
        __syncthreads();   // the block is done with buffer buf
        if (tid == 0 && i + NB < count) issue(i + NB);
        if (flush && a.fout) {
            if (tid < 2) {
                double s2 = 0;
                for (int ww = 0; ww < nw; ++ww) {
                    s2 += wf[ww * 2 + tid];
                    wf[ww * 2 + tid] = 0;
                }
                atomicAdd(&a.fout[b * a.f_stride + tid], s2);
            }
            __syncthreads();
        }
    }
    if (failed && tid == 0) {
        pipe::report(rg.err, MQB_DEV_ERR_TIMEOUT);
        // copies already started still write into this block's shared memory: let them land
        for (int64_t j = i; j < count && j < i + NB; ++j) pipe::mbar_wait(&full[j % NB], unsigned(j / NB) & 1u);
    }
}

static size_t align_up16(size_t x) { return (x + 15) & ~size_t(15); }

size_t ham_ring_smem(const TileGeom &g, int elem_bytes, int threads, int n_classes, int n_terms, bool staged, int nb) {
    size_t s = 128 + size_t(staged ? 2 : 1) * nb * ((size_t(1) << g.K) * elem_bytes);   // 128: base alignment
    s = align_up16(s + size_t(nb) * sizeof(uint64_t));
    s = align_up16(s + (size_t(1) << (g.K - g.c)) * sizeof(uint64_t));
    s = align_up16(s + size_t(threads / 32) * 2 * sizeof(double));
    s = align_up16(s + size_t(n_classes) * sizeof(HamClass));
    s = align_up16(s + size_t(n_terms) * elem_bytes);
    s = align_up16(s + size_t(n_terms) * sizeof(uint32_t));
    return s + size_t(n_classes) * sizeof(uint32_t);
}

template <typename R>
cudaError_t launch_ham_ring(const HamArgs<R> &a, const HamRingGeom &rg, const void *map_ket, const void *map_prev,
                            int sm_count, cudaStream_t s) {
    const int threads = 1 << (a.g.K - kHamRegBits);
    const size_t smem = ham_ring_smem(a.g, int(sizeof(cplx<R>)), threads, a.n_classes, a.n_terms,
                                      a.accumulate && a.out && rg.stage_prev, rg.nb);
    auto kern = ham_ring_kernel<R, kHamRegBits>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t work = a.batch << a.g.n_out;
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(sm_count) * per_sm, work)));
    pipe::TMap mk, mo;
    std::memcpy(&mk, map_ket, sizeof(mk));
    std::memcpy(&mo, map_prev, sizeof(mo));
    kern<<<blocks, threads, smem, s>>>(a, rg, mk, mo);
    return cudaGetLastError();
}

static size_t ham2_smem(const TileGeom &g, int elem_bytes, int threads, int n_classes, int n_terms, bool staged_out) {
    size_t s = align_up16((size_t(1) << g.K) * elem_bytes);
    s = align_up16(s + (size_t(1) << (g.K - g.c)) * sizeof(uint64_t));
    s = align_up16(s + size_t(threads / 32) * 2 * sizeof(double));
    s = align_up16(s + size_t(n_classes) * sizeof(HamClass));
    s = align_up16(s + size_t(n_terms) * elem_bytes);
    s = align_up16(s + size_t(n_terms) * sizeof(uint32_t));
    s = align_up16(s + size_t(n_classes) * sizeof(uint32_t));
    if (staged_out) s += (size_t(1) << g.K) * elem_bytes;   // the previous groups' sum
    return s;
}

template <typename R>
cudaError_t launch_ham(const HamArgs<R> &a, int sm_count, cudaStream_t s) {
    if (a.g.c < 1 || a.g.K > kMaxTileBits || a.g.K < 1) return cudaErrorInvalidValue;  // 16-byte tile accesses need a contiguous low qubit
    if (a.g.K >= 5 + kHamRegBits && (a.g.K - kHamRegBits) <= (sizeof(R) == 4 ? 9 : 8)) {
        const int threads = 1 << (a.g.K - kHamRegBits);
        const size_t smem2 = ham2_smem(a.g, int(sizeof(cplx<R>)), threads, a.n_classes, a.n_terms,
                                       a.accumulate && a.out);
        if (smem2 <= 160 * 1024) {
            auto kern = ham2_kernel<R, kHamRegBits>;
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem2));
            if (e != cudaSuccess) return e;
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem2) != cudaSuccess || per_sm < 1)
                per_sm = 1;
            const int64_t work = a.batch << a.g.n_out;
            const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(sm_count) * per_sm, work)));
            kern<<<blocks, threads, smem2, s>>>(a);
            return cudaGetLastError();
        }
    }
    const size_t smem = ham_smem(a.g, sizeof(cplx<R>));
    auto kern = ham_kernel<R>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    const int64_t work = a.batch << a.g.n_out;
    kern<<<blocks_for(kern, smem, sm_count, work), kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ plain (per gate)
struct PlainOp {
    int32_t kind, m;
    int32_t tq[MQB_MAX_OBJ];
    int32_t sorted[MQB_MAX_OBJ];
    uint64_t ctrl;
    uint64_t px, py, pz;
    int32_t pny;
    int32_t hb;   // RPS: highest flip bit (-1 if no flip)
};

static PlainOp make_plain(const DevOp &op) {
    PlainOp p{};
    p.kind = op.kind;
    p.m = op.m;
    for (int k = 0; k < op.m; ++k) p.tq[k] = p.sorted[k] = op.tq[k];
    for (int i = 1; i < op.m; ++i)
        for (int j = i; j > 0 && p.sorted[j - 1] > p.sorted[j]; --j) std::swap(p.sorted[j], p.sorted[j - 1]);
    p.ctrl = op.ctrl;
    p.px = op.px;
    p.py = op.py;
    p.pz = op.pz;
    p.pny = op.pny;
    const uint64_t f = op.px | op.py;
    p.hb = f ? 63 - __builtin_clzll(f) : -1;
    return p;
}

// RPS pair update: qi' = a qi - i b qj / c(i),  qj' = a qj - i b qi c(i)   (ApplyRPS)
template <typename V>
__device__ __forceinline__ void rps_pair(V &qi, V &qj, double a, double b, int ph, bool same) {
    // c = i^ph ; 1/c = i^{-ph}
    const double cr[4] = {1, 0, -1, 0}, ci[4] = {0, 1, 0, -1};
    const double c_r = cr[ph & 3], c_i = ci[ph & 3];
    const double ic_r = cr[(4 - ph) & 3], ic_i = ci[(4 - ph) & 3];
    if (same) {
        // qi *= (a - i b c)
        const double fr = a + b * c_i, fi = -b * c_r;
        const double xr = qi.x, xi = qi.y;
        qi.x = fr * xr - fi * xi;
        qi.y = fr * xi + fi * xr;
        return;
    }
    const double ir = qi.x, ii = qi.y, jr = qj.x, ji = qj.y;
    // -i b (qj / c) = -i b (qj * ic)
    const double t1r = jr * ic_r - ji * ic_i, t1i = jr * ic_i + ji * ic_r;
    const double t2r = ir * c_r - ii * c_i, t2i = ir * c_i + ii * c_r;
    qi.x = a * ir + b * t1i;
    qi.y = a * ii - b * t1r;
    qj.x = a * jr + b * t2i;
    qj.y = a * ji - b * t2r;
}

template <typename R, bool ADJ>
__global__ void plain_apply_kernel(cplx<R> *st, int n, int64_t batch, const PlainOp op, const cplx<R> *mats,
                                   int64_t mats_stride, int64_t mat_off) {
    using V = cplx<R>;
    const int64_t dim = int64_t(1) << n;
    if (op.kind == KIND_RPS) {
        const bool noflip = op.hb < 0;
        const int64_t groups = noflip ? dim : dim / 2;
        const uint64_t mf = op.px | op.py;
        for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < batch * groups;
             w += int64_t(gridDim.x) * blockDim.x) {
            const int64_t b = w / groups;
            const uint64_t gr = uint64_t(w % groups);
            const uint64_t i = noflip ? gr : ins0_64(gr, op.hb);
            if ((i & op.ctrl) != op.ctrl) continue;
            const V ab = mats[b * mats_stride + mat_off];
            const double a = ab.x, bb = ADJ ? -double(ab.y) : double(ab.y);
            const int ph = (op.pny + 2 * __popcll(i & op.py) + 2 * __popcll(i & op.pz)) & 3;
            V *s = st + b * dim;
            const uint64_t j = i ^ mf;
            V qi = s[i], qj = noflip ? qi : s[j];
            rps_pair(qi, qj, a, bb, ph, noflip);
            s[i] = qi;
            if (!noflip) s[j] = qj;
        }
        return;
    }
    if (op.kind == KIND_DIAG) {
        for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < batch * dim;
             w += int64_t(gridDim.x) * blockDim.x) {
            const int64_t b = w >> n;
            const uint64_t i = uint64_t(w) & uint64_t(dim - 1);
            if ((i & op.ctrl) != op.ctrl) continue;
            int r = 0;
            for (int k = 0; k < op.m; ++k) r |= int((i >> op.tq[k]) & 1) << k;
            V d = mats[b * mats_stride + mat_off + r];
            if (ADJ) d = cconj(d);
            st[b * dim + i] = cmul(st[b * dim + i], d);
        }
        return;
    }
    const int m = op.m, nd = 1 << m;
    const int64_t groups = dim >> m;
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < batch * groups;
         w += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = w / groups;
        uint64_t i0 = uint64_t(w % groups);
        for (int k = 0; k < m; ++k) i0 = ins0_64(i0, op.sorted[k]);
        if ((i0 & op.ctrl) != op.ctrl) continue;
        const V *M = mats + b * mats_stride + mat_off;
        V *s = st + b * dim;
        V v[1 << MQB_MAX_OBJ];
        uint64_t off[1 << MQB_MAX_OBJ];
        for (int r = 0; r < nd; ++r) {
            uint64_t o = 0;
            for (int k = 0; k < m; ++k)
                if (r >> k & 1) o |= uint64_t(1) << op.tq[k];
            off[r] = o;
            v[r] = s[i0 | o];
        }
        for (int r = 0; r < nd; ++r) {
            V acc = czero<V>();
            for (int col = 0; col < nd; ++col) acc = cmadd(ADJ ? cconj(M[col * nd + r]) : M[r * nd + col], v[col], acc);
            s[i0 | off[r]] = acc;
        }
    }
}

template <typename R>
cudaError_t launch_plain_apply(cplx<R> *st, int n, int64_t batch, const DevOp &op, const cplx<R> *mats,
                               int64_t mats_stride, const cplx<R> *cpool, bool adjoint, int sm_count, cudaStream_t s) {
    const PlainOp p = make_plain(op);
    const cplx<R> *base = op.per_sample ? mats : cpool;
    const int64_t stride = op.per_sample ? mats_stride : 0;
    const int threads = 256;
    const int blocks = sm_count * 8;
    if (adjoint)
        plain_apply_kernel<R, true><<<blocks, threads, 0, s>>>(st, n, batch, p, base, stride, op.mat_off);
    else
        plain_apply_kernel<R, false><<<blocks, threads, 0, s>>>(st, n, batch, p, base, stride, op.mat_off);
    return cudaGetLastError();
}

// <lam_h| dM |psi> real parts for every gradient angle of one gate, accumulated into gslots.
template <typename R>
__global__ void plain_grad_kernel(const cplx<R> *psi, const cplx<R> *lam, int n, int64_t batch, int n_hams,
                                  const PlainOp op, int n_angles, int grad_mask, int slot0, const cplx<R> *mats,
                                  int64_t mats_stride, int64_t dmat_off, int mat_size, double *gslots, int n_slots) {
    using V = cplx<R>;
    __shared__ double red[32];
    const int64_t dim = int64_t(1) << n;
    // one (sample, angle, ham) combination per blockIdx.y
    const int combos = n_angles * n_hams;
    const int64_t b = blockIdx.y / combos;
    const int an = (blockIdx.y % combos) / n_hams;
    const int h = blockIdx.y % n_hams;
    if (!(grad_mask >> an & 1)) return;
    int slot = slot0;
    for (int q = 0; q < an; ++q)
        if (grad_mask >> q & 1) ++slot;
    const V *D = mats + b * mats_stride + dmat_off + an * mat_size;
    const V *p = psi + b * dim;
    const V *l = lam + (int64_t(h) * batch + b) * dim;
    double acc = 0;
    if (op.kind == KIND_RPS) {
        const bool noflip = op.hb < 0;
        const int64_t groups = noflip ? dim : dim / 2;
        const uint64_t mf = op.px | op.py;
        const double da = D[0].x, db = D[0].y;
        for (int64_t gr = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gr < groups;
             gr += int64_t(gridDim.x) * blockDim.x) {
            const uint64_t i = noflip ? uint64_t(gr) : ins0_64(uint64_t(gr), op.hb);
            if ((i & op.ctrl) != op.ctrl) continue;
            const int ph = (op.pny + 2 * __popcll(i & op.py) + 2 * __popcll(i & op.pz)) & 3;
            const uint64_t j = i ^ mf;
            V qi = p[i], qj = noflip ? qi : p[j];
            rps_pair(qi, qj, da, db, ph, noflip);
            acc += double(l[i].x) * qi.x + double(l[i].y) * qi.y;
            if (!noflip) acc += double(l[j].x) * qj.x + double(l[j].y) * qj.y;
        }
    } else if (op.kind == KIND_DIAG) {
        for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x) {
            if ((uint64_t(i) & op.ctrl) != op.ctrl) continue;
            int r = 0;
            for (int k = 0; k < op.m; ++k) r |= int((uint64_t(i) >> op.tq[k]) & 1) << k;
            const V y = cmul(D[r], p[i]);
            acc += double(l[i].x) * y.x + double(l[i].y) * y.y;
        }
    } else {
        const int m = op.m, nd = 1 << m;
        const int64_t groups = dim >> m;
        for (int64_t gr = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gr < groups;
             gr += int64_t(gridDim.x) * blockDim.x) {
            uint64_t i0 = uint64_t(gr);
            for (int k = 0; k < m; ++k) i0 = ins0_64(i0, op.sorted[k]);
            if ((i0 & op.ctrl) != op.ctrl) continue;
            uint64_t off[1 << MQB_MAX_OBJ];
            V v[1 << MQB_MAX_OBJ];
            for (int r = 0; r < nd; ++r) {
                uint64_t o = 0;
                for (int k = 0; k < m; ++k)
                    if (r >> k & 1) o |= uint64_t(1) << op.tq[k];
                off[r] = o;
                v[r] = p[i0 | o];
            }
            for (int r = 0; r < nd; ++r) {
                V y = czero<V>();
                for (int col = 0; col < nd; ++col) y = cmadd(D[r * nd + col], v[col], y);
                const V lv = l[i0 | off[r]];
                acc += double(lv.x) * y.x + double(lv.y) * y.y;
            }
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0 && v != 0) atomicAdd(&gslots[(b * n_slots + slot) * n_hams + h], v);
    }
}

template <typename R>
cudaError_t launch_plain_grad(const cplx<R> *psi, const cplx<R> *lam, int n, int64_t batch, int n_hams,
                              const DevOp &op, const cplx<R> *mats, int64_t mats_stride, double *gslots,
                              int n_slots, int sm_count, cudaStream_t s) {
    if (!op.grad_mask) return cudaSuccess;
    const PlainOp p = make_plain(op);
    const int64_t dim = int64_t(1) << n;
    const int threads = 256;
    const int bx = int(std::max<int64_t>(1, std::min<int64_t>((dim + threads - 1) / threads, sm_count * 4)));
    const int64_t by = batch * op.n_angles * n_hams;
    if (by > 65535) return cudaErrorInvalidValue;
    dim3 grid(bx, unsigned(by));
    plain_grad_kernel<R><<<grid, threads, 0, s>>>(psi, lam, n, batch, n_hams, p, op.n_angles, op.grad_mask, op.slot0,
                                                  mats, mats_stride, op.dmat_off, op.mat_size, gslots, n_slots);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ reductions
template <typename R>
__global__ void vdot_kernel(const cplx<R> *a, const cplx<R> *b, int n, double *out) {
    __shared__ double red[2][32];
    const int64_t dim = int64_t(1) << n;
    const int64_t s = blockIdx.y;
    const cplx<R> *pa = a + s * dim, *pb = b + s * dim;
    double re = 0, im = 0;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x) {
        const cplx<R> x = pa[i], y = pb[i];
        re += double(x.x) * y.x + double(x.y) * y.y;
        im += double(x.x) * y.y - double(x.y) * y.x;
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = re;
        red[1][threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool ok = threadIdx.x < (blockDim.x >> 5);
        re = warp_sum(ok ? red[0][threadIdx.x] : 0.0);
        im = warp_sum(ok ? red[1][threadIdx.x] : 0.0);
        if (threadIdx.x == 0) {
            atomicAdd(&out[2 * s], re);
            atomicAdd(&out[2 * s + 1], im);
        }
    }
}

template <typename R>
cudaError_t launch_vdot(const cplx<R> *a, const cplx<R> *b, int n, int64_t batch, double *out, int sm_count,
                        cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * 2 * batch, s);
    if (e != cudaSuccess) return e;
    const int64_t dim = int64_t(1) << n;
    const int threads = 256;
    const int bx = int(std::max<int64_t>(1, std::min<int64_t>((dim + threads - 1) / threads, sm_count * 4)));
    if (batch > 65535) return cudaErrorInvalidValue;
    vdot_kernel<R><<<dim3(bx, unsigned(batch)), threads, 0, s>>>(a, b, n, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ sparse (CSR) Hamiltonians
// out[b] = A ket[b] and fout[b] += <bra[b]|A ket[b]> (Csr_Dot_Vec / ExpectationOfCsr,
// ccsrc/include/core/sparse/algo.h:160-200) with A kept as slices of 32 rows: entry k of the
// slice's row `lane` sits at slice_ptr[s] + 32 k + lane, rows padded to the slice's longest row
// (padding: column = the row itself, value 0).  One warp per slice, one thread per row, so the
// matrix reads of a warp are 128-byte (columns) and 256/512-byte (values) runs, and for a matrix
// built from Pauli strings (columns r ^ f) the state gathers of a warp land in one aligned block.
// One pass over the matrix serves up to kCsrStates states.  Row sums are in the state precision
// like the reference's; the expectation is accumulated in FP64.
constexpr int kCsrStates = 4;

template <typename R>
__global__ void __launch_bounds__(256) sell_kernel(CsrArgs<R> a, int64_t b0) {
    __shared__ double red[2 * kCsrStates][8];
    const int nb = int(a.batch - b0 < kCsrStates ? a.batch - b0 : kCsrStates);
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t n_warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int64_t n_slices = (a.dim + 31) >> 5;
    double fre[kCsrStates], fim[kCsrStates];
#pragma unroll
    for (int k = 0; k < kCsrStates; ++k) fre[k] = fim[k] = 0;
    for (int64_t sl = warp; sl < n_slices; sl += n_warps) {
        const int64_t row = (sl << 5) + lane;
        const bool valid = row < a.dim;
        const int64_t beg = a.slice_ptr[sl];
        const int len = a.slice_len[sl];
        R ar[kCsrStates], ai[kCsrStates];
#pragma unroll
        for (int k = 0; k < kCsrStates; ++k) ar[k] = ai[k] = 0;
        if (valid) {
            for (int e = 0; e < len; ++e) {
                const int64_t at = beg + (int64_t(e) << 5) + lane;
                const int64_t col = a.cols[at];
                const cplx<R> d = a.vals[at];
#pragma unroll
                for (int k = 0; k < kCsrStates; ++k) {
                    if (k < nb) {
                        const cplx<R> x = a.ket[(b0 + k) * a.dim + col];
                        ar[k] += d.x * x.x - d.y * x.y;
                        ai[k] += d.x * x.y + d.y * x.x;
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kCsrStates; ++k) {
                if (k < nb) {
                    const int64_t at = (b0 + k) * a.dim + row;
                    if (a.out) a.out[at] = cplx<R>{ar[k], ai[k]};
                    if (a.fout) {
                        const cplx<R> bv = a.bra[at];
                        fre[k] += double(bv.x) * ar[k] + double(bv.y) * ai[k];
                        fim[k] += double(bv.x) * ai[k] - double(bv.y) * ar[k];
                    }
                }
            }
        }
    }
    if (!a.fout) return;
#pragma unroll
    for (int k = 0; k < kCsrStates; ++k) {
        const double r = warp_sum(fre[k]), i = warp_sum(fim[k]);
        if (lane == 0) {
            red[2 * k][threadIdx.x >> 5] = r;
            red[2 * k + 1][threadIdx.x >> 5] = i;
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const bool ok = threadIdx.x < (blockDim.x >> 5);
        for (int k = 0; k < nb; ++k) {
            const double r = warp_sum(ok ? red[2 * k][threadIdx.x] : 0.0);
            const double i = warp_sum(ok ? red[2 * k + 1][threadIdx.x] : 0.0);
            if (threadIdx.x == 0) {
                atomicAdd(&a.fout[(b0 + k) * a.f_stride], r);
                atomicAdd(&a.fout[(b0 + k) * a.f_stride + 1], i);
            }
        }
    }
}

template <typename R>
cudaError_t launch_csr(const CsrArgs<R> &a, int sm_count, cudaStream_t s) {
    const int threads = 256;
    const int64_t n_slices = (a.dim + 31) >> 5;
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>((n_slices + 7) / 8, int64_t(sm_count) * 8)));
    for (int64_t b0 = 0; b0 < a.batch; b0 += kCsrStates) {
        sell_kernel<R><<<blocks, threads, 0, s>>>(a, b0);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// One 2x2 matrix (unitary or not) on `qubit` of `batch` states where every control bit is set:
// the single sweep of ApplySingleQubitMatrix (cpu_vector_core_matrix_gate.cpp:151), used for the
// operators a noise channel picks (X, Y, Z, diag(a, b), [[0, a], [b, 0]], a global factor).
template <typename R>
__global__ void matrix1_kernel(cplx<R> *st, int n, int qubit, uint64_t ctrl, int64_t batch, Mat1 m) {
    const int64_t half = int64_t(1) << (n - 1), dim = int64_t(1) << n;
    const int64_t low = (int64_t(1) << qubit) - 1;
    const R m0r = R(m.v[0]), m0i = R(m.v[1]), m1r = R(m.v[2]), m1i = R(m.v[3]);
    const R m2r = R(m.v[4]), m2i = R(m.v[5]), m3r = R(m.v[6]), m3i = R(m.v[7]);
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < batch * half;
         w += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = w / half, l = w % half;
        const int64_t i = ((l & ~low) << 1) | (l & low), j = i | (int64_t(1) << qubit);
        if ((uint64_t(i) & ctrl) != ctrl) continue;
        cplx<R> *p = st + b * dim;
        const cplx<R> a = p[i], c = p[j];
        p[i] = cplx<R>{m0r * a.x - m0i * a.y + m1r * c.x - m1i * c.y, m0r * a.y + m0i * a.x + m1r * c.y + m1i * c.x};
        p[j] = cplx<R>{m2r * a.x - m2i * a.y + m3r * c.x - m3i * c.y, m2r * a.y + m2i * a.x + m3r * c.y + m3i * c.x};
    }
}

template <typename R>
cudaError_t launch_matrix1(cplx<R> *st, int n, int qubit, uint64_t ctrl, int64_t batch, const Mat1 &m, int sm_count,
                           cudaStream_t s) {
    const int64_t work = batch * (int64_t(1) << (n - 1));
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, int64_t(sm_count) * 8)));
    matrix1_kernel<R><<<blocks, 256, 0, s>>>(st, n, qubit, ctrl, batch, m);
    return cudaGetLastError();
}

// Request blockIdx.y of `ops` over its pairs (amplitudes with bit q = 0 and 1), blocks in x
// striding the pairs, four pairs per thread in flight (all loads before the first store).
// Amplitudes a matrix column does not use are not read (a projector reads half the state), except
// where the controls are unset and the norm needs them as they are.
template <typename R, bool NORM>
__global__ void row_ops_kernel(cplx<R> *st, int n, const __grid_constant__ RowOps ops, double *norm_out) {
    constexpr int U = 4;
    const int r = blockIdx.y;
    const int q = ops.qubit[r];
    const uint64_t ctrl = ops.ctrl[r];
    const int64_t half = int64_t(1) << (n - 1);
    cplx<R> *p = st + ops.row[r] * (int64_t(1) << n);
    const double *mv = ops.m[r];
    const R m0r = R(mv[0]), m0i = R(mv[1]), m1r = R(mv[2]), m1i = R(mv[3]);
    const R m2r = R(mv[4]), m2i = R(mv[5]), m3r = R(mv[6]), m3i = R(mv[7]);
    const bool use0 = mv[0] != 0 || mv[1] != 0 || mv[4] != 0 || mv[5] != 0;
    const bool use1 = mv[2] != 0 || mv[3] != 0 || mv[6] != 0 || mv[7] != 0;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    double acc = 0;
    for (int64_t l0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; l0 < half; l0 += stride * U) {
        uint64_t i[U];
        bool in[U], on[U];
        cplx<R> a[U], c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t l = l0 + u * stride;
            in[u] = l < half;
            i[u] = in[u] ? ins0_64(uint64_t(l), q) : 0;
            on[u] = in[u] && (i[u] & ctrl) == ctrl;
            const bool raw = NORM && in[u] && !on[u];   // outside the controls the norm takes psi as it is
            a[u] = (on[u] && use0) || raw ? p[i[u]] : cplx<R>{0, 0};
            c[u] = (on[u] && use1) || raw ? p[i[u] | (uint64_t(1) << q)] : cplx<R>{0, 0};
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!in[u]) continue;
            if (!on[u]) {
                if (NORM)
                    acc += double(a[u].x) * a[u].x + double(a[u].y) * a[u].y + double(c[u].x) * c[u].x +
                           double(c[u].y) * c[u].y;
                continue;
            }
            const cplx<R> x{m0r * a[u].x - m0i * a[u].y + m1r * c[u].x - m1i * c[u].y,
                            m0r * a[u].y + m0i * a[u].x + m1r * c[u].y + m1i * c[u].x};
            const cplx<R> y{m2r * a[u].x - m2i * a[u].y + m3r * c[u].x - m3i * c[u].y,
                            m2r * a[u].y + m2i * a[u].x + m3r * c[u].y + m3i * c[u].x};
            if (NORM) {
                acc += double(x.x) * x.x + double(x.y) * x.y + double(y.x) * y.x + double(y.y) * y.y;
            } else {
                p[i[u]] = x;
                p[i[u] | (uint64_t(1) << q)] = y;
            }
        }
    }
    if (NORM) {
        __shared__ double red[32];
        acc = warp_sum(acc);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
            v = warp_sum(v);
            if (threadIdx.x == 0) atomicAdd(norm_out + r, v);
        }
    }
}

template <typename R>
cudaError_t launch_row_ops(cplx<R> *st, int n, const RowOps &ops, double *norm_out, int sm_count, cudaStream_t s) {
    if (ops.count <= 0) return cudaSuccess;
    const int threads = 256;
    const int64_t half = int64_t(1) << (n - 1);
    const int64_t per_state = std::max<int64_t>(1, (half + 4 * threads - 1) / (4 * threads));
    const int64_t want = std::max<int64_t>(1, (int64_t(sm_count) * 8 + ops.count - 1) / ops.count);
    const dim3 grid(unsigned(std::min(per_state, want)), unsigned(ops.count));
    if (norm_out) {
        cudaError_t e = cudaMemsetAsync(norm_out, 0, sizeof(double) * ops.count, s);
        if (e != cudaSuccess) return e;
        row_ops_kernel<R, true><<<grid, threads, 0, s>>>(st, n, ops, norm_out);
    } else {
        row_ops_kernel<R, false><<<grid, threads, 0, s>>>(st, n, ops, nullptr);
    }
    return cudaGetLastError();
}

template <typename R>
__global__ void copy_kernel(cplx<R> *dst, const cplx<R> *src, int n, int64_t batch, int64_t src_stride) {
    const int64_t dim = int64_t(1) << n;
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < batch * dim; w += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = w >> n, i = w & (dim - 1);
        cplx<R> v;
        if (src) {
            v = src[b * src_stride + i];
        } else {
            v.x = (i == 0) ? 1 : 0;
            v.y = 0;
        }
        dst[w] = v;
    }
}

template <typename R>
cudaError_t launch_copy_or_zero(cplx<R> *dst, const cplx<R> *src, int n, int64_t batch, int64_t src_stride,
                                cudaStream_t s) {
    copy_kernel<R><<<2048, 256, 0, s>>>(dst, src, n, batch, src_stride);
    return cudaGetLastError();
}

__global__ void grad_scatter_kernel(const double *gslots, int64_t batch, int n_slots, int n_hams,
                                    const int32_t *csr_ptr, const int32_t *csr_slot, const double *csr_coeff,
                                    int n_params, double scale, double *grad) {
    const int64_t total = batch * n_hams * int64_t(n_params);
    for (int64_t w = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; w < total; w += int64_t(gridDim.x) * blockDim.x) {
        const int p = int(w % n_params);
        const int h = int((w / n_params) % n_hams);
        const int64_t b = w / (int64_t(n_params) * n_hams);
        double s = 0;
        for (int e = csr_ptr[p]; e < csr_ptr[p + 1]; ++e)
            s += csr_coeff[e] * gslots[(b * n_slots + csr_slot[e]) * n_hams + h];
        grad[w] = scale * s;   // scale 2: GradRealDouble, g + conj(g) = 2 Re g
    }
}

cudaError_t launch_grad_scatter(const double *gslots, int64_t batch, int n_slots, int n_hams, const int32_t *csr_ptr,
                                const int32_t *csr_slot, const double *csr_coeff, int n_params, double scale, double *grad,
                                cudaStream_t s) {
    const int64_t total = batch * n_hams * int64_t(n_params);
    if (total == 0) return cudaSuccess;
    const int blocks = int(std::min<int64_t>((total + 255) / 256, 4096));
    grad_scatter_kernel<<<blocks, 256, 0, s>>>(gslots, batch, n_slots, n_hams, csr_ptr, csr_slot, csr_coeff, n_params,
                                                scale, grad);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ sampling
template <typename R>
__global__ void chunk_probs_kernel(const cplx<R> *st, int n, int chunk_bits, double *sums) {
    __shared__ double red[32];
    const int64_t chunk = blockIdx.x;
    const int64_t len = int64_t(1) << chunk_bits;
    double acc = 0;
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
        const cplx<R> v = st[chunk * len + i];
        acc += double(v.x) * v.x + double(v.y) * v.y;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) sums[chunk] = v;
    }
}

template <typename R>
cudaError_t launch_chunk_probs(const cplx<R> *st, int n, int chunk_bits, double *sums, cudaStream_t s) {
    const int64_t n_chunks = int64_t(1) << (n - chunk_bits);
    chunk_probs_kernel<R><<<unsigned(n_chunks), 256, 0, s>>>(st, n, chunk_bits, sums);
    return cudaGetLastError();
}

// in-place exclusive prefix of sums[0..n) into sums[0..n], sums[n] = total (single block)
__global__ void prefix_kernel(double *sums, int64_t n) {
    __shared__ double part[1024];
    const int T = blockDim.x;
    const int64_t per = (n + T - 1) / T;
    const int64_t lo = threadIdx.x * per, hi = (lo + per < n) ? lo + per : n;
    double s = 0;
    for (int64_t i = lo; i < hi; ++i) s += sums[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double run = 0;
        for (int i = 0; i < T; ++i) {
            const double v = part[i];
            part[i] = run;
            run += v;
        }
        sums[n] = run;
    }
    __syncthreads();
    double run = part[threadIdx.x];
    for (int64_t i = lo; i < hi; ++i) {
        const double v = sums[i];
        sums[i] = run;
        run += v;
    }
}

cudaError_t launch_prefix(double *sums, int64_t n, cudaStream_t s) {
    prefix_kernel<<<1, 1024, 0, s>>>(sums, n);
    return cudaGetLastError();
}

// one warp per shot: find the chunk by binary search on the prefix, then scan the chunk
template <typename R>
__global__ void sample_search_kernel(const cplx<R> *st, int n, int chunk_bits, const double *prefix, const double *u,
                                     int64_t shots, int64_t *out) {
    const int lane = threadIdx.x & 31;
    const int64_t n_chunks = int64_t(1) << (n - chunk_bits);
    const int64_t dim = int64_t(1) << n;
    for (int64_t shot = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; shot < shots;
         shot += (int64_t(gridDim.x) * blockDim.x) >> 5) {
        const double x = u[shot];
        // largest chunk k with prefix[k] <= x
        int64_t lo = 0, hi = n_chunks - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= x)
                lo = mid;
            else
                hi = mid - 1;
        }
        double run = prefix[lo];
        int64_t found = -1;
        const int64_t start = lo << chunk_bits, len = int64_t(1) << chunk_bits;
        for (int64_t off = 0; off < len && found < 0; off += 32) {
            double p = 0;
            if (off + lane < len) {
                const cplx<R> v = st[start + off + lane];
                p = double(v.x) * v.x + double(v.y) * v.y;
            }
            // inclusive warp scan
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const double y = __shfl_up_sync(0xffffffffu, p, d);
                if (lane >= d) p += y;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, x < run + p);
            if (hit) {
                found = start + off + __ffs(hit) - 1;
            } else {
                run += __shfl_sync(0xffffffffu, p, 31);
            }
        }
        if (found < 0) {
            // x beyond the accumulated mass of this chunk (rounding): the next non-empty index, or the last one
            found = (start + len < dim - 1) ? start + len : dim - 1;
        }
        if (lane == 0) out[shot] = found;
    }
}

template <typename R>
cudaError_t launch_sample_search(const cplx<R> *st, int n, int chunk_bits, const double *prefix, const double *u,
                                 int64_t shots, int64_t *out, cudaStream_t s) {
    if (shots == 0) return cudaSuccess;
    const int threads = 256;
    const int64_t warps = shots;
    const int blocks = int(std::min<int64_t>((warps * 32 + threads - 1) / threads, 8192));
    sample_search_kernel<R><<<blocks, threads, 0, s>>>(st, n, chunk_bits, prefix, u, shots, out);
    return cudaGetLastError();
}

template <typename R>
__global__ void one_prob_kernel(const cplx<R> *st, int n, int q, double *out) {
    __shared__ double red[32];
    const int64_t half = int64_t(1) << (n - 1);
    double acc = 0;
    for (int64_t l = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; l < half; l += int64_t(gridDim.x) * blockDim.x) {
        const uint64_t i = ins0_64(uint64_t(l), q) | (uint64_t(1) << q);
        const cplx<R> v = st[i];
        acc += double(v.x) * v.x + double(v.y) * v.y;
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) atomicAdd(out, v);
    }
}

template <typename R>
cudaError_t launch_one_prob(const cplx<R> *st, int n, int q, double *out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
    if (e != cudaSuccess) return e;
    one_prob_kernel<R><<<512, 256, 0, s>>>(st, n, q, out);
    return cudaGetLastError();
}

template <typename R>
__global__ void collapse_kernel(cplx<R> *st, int n, int q, int outcome, double scale) {
    const int64_t dim = int64_t(1) << n;
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x) {
        cplx<R> v = st[i];
        if (int((i >> q) & 1) == outcome) {
            v.x = R(v.x * scale);
            v.y = R(v.y * scale);
        } else {
            v.x = 0;
            v.y = 0;
        }
        st[i] = v;
    }
}

template <typename R>
cudaError_t launch_collapse(cplx<R> *st, int n, int q, int outcome, double scale, cudaStream_t s) {
    collapse_kernel<R><<<1024, 256, 0, s>>>(st, n, q, outcome, scale);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------ instantiations
#define MQB_INSTANTIATE(R)                                                                                         \
    template cudaError_t launch_matgen<R>(const MatgenArgs &, cudaStream_t);                                       \
    template cudaError_t launch_ham<R>(const HamArgs<R> &, int, cudaStream_t);                                     \
    template cudaError_t launch_ham_ring<R>(const HamArgs<R> &, const HamRingGeom &, const void *, const void *,   \
                                            int, cudaStream_t);                                                    \
    template cudaError_t launch_plain_apply<R>(cplx<R> *, int, int64_t, const DevOp &, const cplx<R> *, int64_t,   \
                                               const cplx<R> *, bool, int, cudaStream_t);                          \
    template cudaError_t launch_plain_grad<R>(const cplx<R> *, const cplx<R> *, int, int64_t, int, const DevOp &,  \
                                              const cplx<R> *, int64_t, double *, int, int, cudaStream_t);         \
    template cudaError_t launch_vdot<R>(const cplx<R> *, const cplx<R> *, int, int64_t, double *, int,             \
                                        cudaStream_t);                                                             \
    template cudaError_t launch_copy_or_zero<R>(cplx<R> *, const cplx<R> *, int, int64_t, int64_t, cudaStream_t);  \
    template cudaError_t launch_csr<R>(const CsrArgs<R> &, int, cudaStream_t);                                      \
    template cudaError_t launch_matrix1<R>(cplx<R> *, int, int, uint64_t, int64_t, const Mat1 &, int, cudaStream_t); \
    template cudaError_t launch_chunk_probs<R>(const cplx<R> *, int, int, double *, cudaStream_t);                 \
    template cudaError_t launch_sample_search<R>(const cplx<R> *, int, int, const double *, const double *,       \
                                                 int64_t, int64_t *, cudaStream_t);                                \
    template cudaError_t launch_one_prob<R>(const cplx<R> *, int, int, double *, cudaStream_t);                    \
    template cudaError_t launch_row_ops<R>(cplx<R> *, int, const RowOps &, double *, int, cudaStream_t);          \
    template cudaError_t launch_collapse<R>(cplx<R> *, int, int, int, double, cudaStream_t);

MQB_INSTANTIATE(float)
MQB_INSTANTIATE(double)

}  // namespace mqb
