// Register math of the fused tile passes (sm_100a), shared by the precompiled tile kernels and
// the pass kernels generated at run time (this header is also compiled by NVRTC, so it uses no
// host headers).
//
// Inside a register stage every thread holds the 2^RB amplitudes of a tile whose tile-local
// indices differ in the stage's register bits.  The gate kernels below update that array in
// place with compile-time indices: P (Q) is the register position of matrix bit 0 (1), CM the
// mask of register positions that control the gate.  Matrix entries are passed as values, so a
// caller can substitute the identity for threads whose controls on thread or tile bits are not
// set (no branch, the code stays straight-line).
//
// Math per amplitude: dense 2x2 8 FMA-class instructions, real 2x2 and RX-like 4 (a real 2x2 in
// complex64 on sm_100: 2 packed FP32 instructions), diagonal 4, X 0 (register renaming), dense
// 4x4 16.
#ifndef MQB_REGMATH_CUH_
#define MQB_REGMATH_CUH_

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
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// complex64 on sm_100: a real 2x2 row as two packed FP32 instructions (FMUL2, FFMA2) instead of
// four scalar ones; per component the same rounding as the scalar form above.
__device__ __forceinline__ float2 rlin(float a, float2 x, float b, float2 y) {
    return __ffma2_rn(make_float2(a, a), x, __fmul2_rn(make_float2(b, b), y));
}
#endif

// Accumulator of Re(conj(l) x) terms: complex64 keeps the (l.x x.x, l.y x.y) sums apart in one
// packed register (one FFMA2 per term on sm_100), complex128 one FP64 sum (two FMAs per term).
template <typename V>
struct ReAcc;
template <>
struct ReAcc<float2> {
    typedef float2 type;
};
template <>
struct ReAcc<double2> {
    typedef double type;
};
__device__ __forceinline__ float2 ra_zero(float2) { return make_float2(0.f, 0.f); }
__device__ __forceinline__ double ra_zero(double) { return 0.0; }
__device__ __forceinline__ float2 ra_add(float2 a, float2 l, float2 x) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    return __ffma2_rn(l, x, a);
#else
    return make_float2(fmaf(l.x, x.x, a.x), fmaf(l.y, x.y, a.y));
#endif
}
__device__ __forceinline__ double ra_add(double a, double2 l, double2 x) { return fma(l.x, x.x, fma(l.y, x.y, a)); }
__device__ __forceinline__ float ra_sum(float2 a) { return a.x + a.y; }
__device__ __forceinline__ double ra_sum(double a) { return a; }

template <typename V>
__device__ __forceinline__ decltype(V::x) redot(V l, V y) {  // Re(conj(l) y)
    return fma(l.x, y.x, l.y * y.y);
}
template <typename V>
__device__ __forceinline__ V cval(decltype(V::x) re, decltype(V::x) im) {
    V r;
    r.x = re;
    r.y = im;
    return r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum over a warp in the accumulator's own precision: one 32-bit shuffle per step for
// complex64 partials (each already a sum of at most 32 products), FP64 from the warp partial up.
__device__ __forceinline__ float warp_sum_acc(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_acc(double v) { return warp_sum(v); }

// Register index j takes part in a gate on position P controlled by the positions in CM.
template <int P, unsigned CM>
__device__ __forceinline__ constexpr bool pair_on(int j) {
    return !((j >> P) & 1) && ((unsigned(j) & CM) == CM);
}
template <unsigned CM>
__device__ __forceinline__ constexpr bool ctl_on(int j) {
    return (unsigned(j) & CM) == CM;
}

// =============================================================================== forward
template <typename V, int RB, int P, unsigned CM>
__device__ __forceinline__ void j_dense1(V (&v)[1 << RB], V m00, V m01, V m10, V m11) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = cmadd(m00, a, cmul(m01, b));
        v[j | (1 << P)] = cmadd(m10, a, cmul(m11, b));
    }
}

template <typename V, int RB, int P, unsigned CM, typename R>
__device__ __forceinline__ void j_real1(V (&v)[1 << RB], R m00, R m01, R m10, R m11) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = rlin(m00, a, m01, b);
        v[j | (1 << P)] = rlin(m10, a, m11, b);
    }
}

// [[a, i b], [i b, a]] with a, b real (RX)
template <typename V, int RB, int P, unsigned CM, typename R>
__device__ __forceinline__ void j_rxl1(V (&v)[1 << RB], R a, R b) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        const V x0 = v[j], x1 = v[j | (1 << P)];
        v[j] = rxl(a, x0, b, x1);
        v[j | (1 << P)] = rxl(a, x1, b, x0);
    }
}

template <typename V, int RB, int P, unsigned CM>
__device__ __forceinline__ void j_x1(V (&v)[1 << RB]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        const V a = v[j];
        v[j] = v[j | (1 << P)];
        v[j | (1 << P)] = a;
    }
}

// X whose thread-level controls are given by `on`: two selects per amplitude, no branch
template <typename V, int RB, int P, unsigned CM>
__device__ __forceinline__ void j_x1sel(V (&v)[1 << RB], bool on) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        const V a = v[j], b = v[j | (1 << P)];
        v[j] = on ? b : a;
        v[j | (1 << P)] = on ? a : b;
    }
}

template <typename V, int RB, int P, unsigned CM>
__device__ __forceinline__ void j_diag1(V (&v)[1 << RB], V d0, V d1) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        v[j] = cmul(v[j], ((j >> P) & 1) ? d1 : d0);
    }
}

template <typename V, int RB, unsigned CM>
__device__ __forceinline__ void j_scale(V (&v)[1 << RB], V d) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        v[j] = cmul(v[j], d);
    }
}

// diagonal on two register positions: P carries matrix bit 0, Q matrix bit 1
template <typename V, int RB, int P, int Q, unsigned CM>
__device__ __forceinline__ void j_diag2(V (&v)[1 << RB], V d0, V d1, V d2, V d3) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        const int r = ((j >> P) & 1) | (((j >> Q) & 1) << 1);
        v[j] = cmul(v[j], r == 0 ? d0 : r == 1 ? d1 : r == 2 ? d2 : d3);
    }
}

// dense 4x4 (row-major M), P carries matrix bit 0, Q matrix bit 1
template <typename V, int RB, int P, int Q, unsigned CM>
__device__ __forceinline__ void j_dense2(V (&v)[1 << RB], const V *M) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (((j >> P) & 1) || ((j >> Q) & 1) || !ctl_on<CM>(j)) continue;
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

// ============================================= backward (psi <- U^dag psi, gradients, lambda)
// The adjoint step of a gate: psi' = U^dag psi, acc[a][h] += Re<lambda_h| dU_a |psi'> over the
// thread's amplitudes, then lambda_h <- U^dag lambda_h.  G is the mask of gradient angles.
// Every kernel takes U^dag's entries (a..) and the derivative entries (d..) as values: a thread
// whose thread-level controls are off passes the identity and zero derivatives.

template <typename V, int RB, int NH, int P, unsigned CM, int G>
__device__ __forceinline__ void jb_dense1(V (&v)[1 << RB], V (&l)[NH][1 << RB], V a00, V a01, V a10, V a11,
                                          const V (&d)[3][4], decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        constexpr int bit = 1 << P;
        const V w0 = cmadd(a00, v[j], cmul(a01, v[j | bit])), w1 = cmadd(a10, v[j], cmul(a11, v[j | bit]));
        v[j] = w0;
        v[j | bit] = w1;
#pragma unroll
        for (int an = 0; an < 3; ++an) {
            if (!((G >> an) & 1)) continue;
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

// U real: U^dag = U^T (a.. are U^T's entries), real derivative
template <typename V, int RB, int NH, int P, unsigned CM, int G, typename R>
__device__ __forceinline__ void jb_real1(V (&v)[1 << RB], V (&l)[NH][1 << RB], R a00, R a01, R a10, R a11, R d00,
                                         R d01, R d10, R d11, R (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
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

// U = [[a, i b], [i b, a]]: U^dag = [[a, i nb], [i nb, a]] with nb = -b; dU = [[da, i db], [i db, da]]
template <typename V, int RB, int NH, int P, unsigned CM, int G, typename R>
__device__ __forceinline__ void jb_rxl1(V (&v)[1 << RB], V (&l)[NH][1 << RB], R a, R nb, R da, R db,
                                        R (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
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

template <typename V, int RB, int NH, int P, unsigned CM>
__device__ __forceinline__ void jb_x1(V (&v)[1 << RB], V (&l)[NH][1 << RB]) {
    j_x1<V, RB, P, CM>(v);
#pragma unroll
    for (int h = 0; h < NH; ++h) j_x1<V, RB, P, CM>(l[h]);
}

template <typename V, int RB, int NH, int P, unsigned CM>
__device__ __forceinline__ void jb_x1sel(V (&v)[1 << RB], V (&l)[NH][1 << RB], bool on) {
    j_x1sel<V, RB, P, CM>(v, on);
#pragma unroll
    for (int h = 0; h < NH; ++h) j_x1sel<V, RB, P, CM>(l[h], on);
}

// diagonal on register P: c0, c1 = conj of the entries, e0, e1 = derivative entries
template <typename V, int RB, int NH, int P, unsigned CM, int G>
__device__ __forceinline__ void jb_diag1(V (&v)[1 << RB], V (&l)[NH][1 << RB], V c0, V c1, V e0, V e1,
                                         decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
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

template <typename V, int RB, int NH, unsigned CM, int G>
__device__ __forceinline__ void jb_scale(V (&v)[1 << RB], V (&l)[NH][1 << RB], V c, V e,
                                         decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
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

template <typename V, int RB, int NH, int P, int Q, unsigned CM, int G>
__device__ __forceinline__ void jb_diag2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V (&c)[4], const V (&e)[4],
                                         decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        const int r = ((j >> P) & 1) | (((j >> Q) & 1) << 1);
        const V w = cmul(v[j], c[r]);
        v[j] = w;
        if (G & 1) {
            const V y = cmul(e[r], w);
#pragma unroll
            for (int h = 0; h < NH; ++h) acc[0][h] += redot(l[h][j], y);
        }
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c[r]);
    }
}

// ---- gradients from the generator.  For U(t) = exp(-i t/2 G) with G a Pauli product (and for
// the phase gates), dU/dt = -i/2 G U, so Re<lambda| dU |psi'> = Re<lambda| -i/2 G |psi> with psi
// the state before the uncompute: the derivative costs two FMA per amplitude instead of a matrix
// product and a dot product.  gs scales the accumulated sum (1/2, or 0 for threads whose
// thread-level controls are off).

template <typename R, typename V>
__device__ __forceinline__ R re_acc(V l, V x, R acc) {  // acc + Re(conj(l) x)
    return fma(l.x, x.x, fma(l.y, x.y, acc));
}
template <typename R, typename V>
__device__ __forceinline__ R im_acc(V l, V x, R acc) {  // acc + Im(conj(l) x)
    return fma(l.x, x.y, fma(-l.y, x.x, acc));
}

// RY-like: G = Y, Re<l| -i/2 Y |x> = (Re(conj(l1) x0) - Re(conj(l0) x1)) / 2; U^dag = U^T given
template <typename V, int RB, int NH, int P, unsigned CM, typename R>
__device__ __forceinline__ void jbg_ry(V (&v)[1 << RB], V (&l)[NH][1 << RB], R a00, R a01, R a10, R a11, R gs,
                                       R (&acc)[3][NH]) {
    typedef typename ReAcc<V>::type A;
    A gp[NH], gm[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) gp[h] = gm[h] = ra_zero(A());
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        constexpr int bit = 1 << P;
        const V x0 = v[j], x1 = v[j | bit];
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            gp[h] = ra_add(gp[h], l[h][j | bit], x0);
            gm[h] = ra_add(gm[h], l[h][j], x1);
        }
        v[j] = rlin(a00, x0, a01, x1);
        v[j | bit] = rlin(a10, x0, a11, x1);
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V z0 = l[h][j], z1 = l[h][j | bit];
            l[h][j] = rlin(a00, z0, a01, z1);
            l[h][j | bit] = rlin(a10, z0, a11, z1);
        }
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) acc[0][h] += gs * (ra_sum(gp[h]) - ra_sum(gm[h]));
}

// U3(theta, phi, lam) = P(phi) RY'(theta) P(lam), P(x) = diag(1, e^{ix}), with its three gradients
// in generator form (z = U^dag l is lambda on the gate's input side, w = U^dag v psi there):
//   d/dphi = diag(0, i) U:  Re<l|diag(0,i)|v> = -Im(conj(l1) v1)
//   d/dlam = U diag(0, i):  Re<z|diag(0,i)|w> = -Im(conj(z1) w1)
//   d/dtheta = U G, G = [[0, -e^{i lam}], [e^{-i lam}, 0]] / 2:
//                            Re(-e^{i lam} A + e^{-i lam} B) / 2, A = sum conj(z0) w1, B = sum conj(z1) w0
// 12 FMAs per pair for all three instead of a derivative matrix applied per angle; `el` = e^{i lam},
// gw = 1 (0 for a thread whose controls are off).
template <typename V, int RB, int NH, int P, unsigned CM, int G, typename R>
__device__ __forceinline__ void jbg_u3(V (&v)[1 << RB], V (&l)[NH][1 << RB], V a00, V a01, V a10, V a11, V el, R gw,
                                       R (&acc)[3][NH]) {
    R gphi[NH], glam[NH], ar[NH], ai[NH], br[NH], bi[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) gphi[h] = glam[h] = ar[h] = ai[h] = br[h] = bi[h] = 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        constexpr int bit = 1 << P;
        const V x0 = v[j], x1 = v[j | bit];
        const V w0 = cmadd(a00, x0, cmul(a01, x1)), w1 = cmadd(a10, x0, cmul(a11, x1));
        v[j] = w0;
        v[j | bit] = w1;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V l0 = l[h][j], l1 = l[h][j | bit];
            if (G & 2) gphi[h] = im_acc(l1, x1, gphi[h]);
            const V z0 = cmadd(a00, l0, cmul(a01, l1)), z1 = cmadd(a10, l0, cmul(a11, l1));
            if (G & 4) glam[h] = im_acc(z1, w1, glam[h]);
            if (G & 1) {
                ar[h] = re_acc(z0, w1, ar[h]);
                ai[h] = im_acc(z0, w1, ai[h]);
                br[h] = re_acc(z1, w0, br[h]);
                bi[h] = im_acc(z1, w0, bi[h]);
            }
            l[h][j] = z0;
            l[h][j | bit] = z1;
        }
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) {
        // Re(-el A + conj(el) B) / 2
        if (G & 1) acc[0][h] += gw * R(0.5) * (-(el.x * ar[h] - el.y * ai[h]) + (el.x * br[h] + el.y * bi[h]));
        if (G & 2) acc[1][h] -= gw * gphi[h];
        if (G & 4) acc[2][h] -= gw * glam[h];
    }
}

// e^{i lam} of a U3 from its matrix m (row-major) and its theta derivative d: -m01 / s with
// s = sin(theta/2) = -2 Re d00 when |s| >= |c|, else -2 d01 / c with c = cos(theta/2) = Re m00.
template <typename V>
__device__ __forceinline__ V u3_phase(V m00, V m01, V d00, V d01) {
    typedef decltype(V::x) R;
    const R s = R(-2) * d00.x, c = m00.x;
    V e;
    if (fabs(s) >= fabs(c)) {
        e.x = -m01.x / s;
        e.y = -m01.y / s;
    } else {
        e.x = R(-2) * d01.x / c;
        e.y = R(-2) * d01.y / c;
    }
    return e;
}

// RX-like: G = X, Re<l| -i/2 X |x> = (Im(conj(l0) x1) + Im(conj(l1) x0)) / 2; U^dag = [[a, i nb], [i nb, a]]
template <typename V, int RB, int NH, int P, unsigned CM, typename R>
__device__ __forceinline__ void jbg_rx(V (&v)[1 << RB], V (&l)[NH][1 << RB], R a, R nb, R gs, R (&acc)[3][NH]) {
    R g[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) g[h] = 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!pair_on<P, CM>(j)) continue;
        constexpr int bit = 1 << P;
        const V x0 = v[j], x1 = v[j | bit];
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            g[h] = im_acc(l[h][j], x1, g[h]);
            g[h] = im_acc(l[h][j | bit], x0, g[h]);
        }
        v[j] = rxl(a, x0, nb, x1);
        v[j | bit] = rxl(a, x1, nb, x0);
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            const V z0 = l[h][j], z1 = l[h][j | bit];
            l[h][j] = rxl(a, z0, nb, z1);
            l[h][j | bit] = rxl(a, z1, nb, z0);
        }
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) acc[0][h] += gs * g[h];
}

// Diagonal phase gates (RZ, RZZ, PS, GP): dU/dt = -i W U with W diagonal and real, so the
// gradient is sum_j w_j Im(conj(l_j) x_j).  One target on register P: weights (w0, w1) by bit P;
// c0, c1 = conj of the entries for the uncompute.
template <typename V, int RB, int NH, int P, unsigned CM, typename R>
__device__ __forceinline__ void jbg_diag1(V (&v)[1 << RB], V (&l)[NH][1 << RB], V c0, V c1, R w0, R w1,
                                          R (&acc)[3][NH]) {
    R g0[NH], g1[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) g0[h] = g1[h] = 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        const bool hi = (j >> P) & 1;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
            if (hi) g1[h] = im_acc(l[h][j], v[j], g1[h]);
            else g0[h] = im_acc(l[h][j], v[j], g0[h]);
        }
        v[j] = cmul(v[j], hi ? c1 : c0);
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], hi ? c1 : c0);
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) acc[0][h] += w0 * g0[h] + w1 * g1[h];
}

// two targets on registers P (matrix bit 0) and Q (matrix bit 1): weights w[r], r = b0 | b1 << 1
template <typename V, int RB, int NH, int P, int Q, unsigned CM, typename R>
__device__ __forceinline__ void jbg_diag2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V (&c)[4], const R (&w)[4],
                                          R (&acc)[3][NH]) {
    R g[4][NH];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int h = 0; h < NH; ++h) g[r][h] = 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
        const int r = ((j >> P) & 1) | (((j >> Q) & 1) << 1);
#pragma unroll
        for (int h = 0; h < NH; ++h) g[r][h] = im_acc(l[h][j], v[j], g[r][h]);
        v[j] = cmul(v[j], c[r]);
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c[r]);
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) acc[0][h] += w[0] * g[0][h] + w[1] * g[1][h] + w[2] * g[2][h] + w[3] * g[3][h];
}

// targets off the registers: one entry c and one weight w per thread
template <typename V, int RB, int NH, unsigned CM, typename R>
__device__ __forceinline__ void jbg_scale(V (&v)[1 << RB], V (&l)[NH][1 << RB], V c, R w, R (&acc)[3][NH]) {
    R g[NH];
#pragma unroll
    for (int h = 0; h < NH; ++h) g[h] = 0;
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (!ctl_on<CM>(j)) continue;
#pragma unroll
        for (int h = 0; h < NH; ++h) g[h] = im_acc(l[h][j], v[j], g[h]);
        v[j] = cmul(v[j], c);
#pragma unroll
        for (int h = 0; h < NH; ++h) l[h][j] = cmul(l[h][j], c);
    }
#pragma unroll
    for (int h = 0; h < NH; ++h) acc[0][h] += w * g[h];
}

// dense 4x4 from the matrix table: M = U (row-major), dM_a = M + 16 (1 + a)
template <typename V, int RB, int NH, int P, int Q, unsigned CM, int G>
__device__ __forceinline__ void jb_dense2(V (&v)[1 << RB], V (&l)[NH][1 << RB], const V *M,
                                          decltype(V::x) (&acc)[3][NH]) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) {
        if (((j >> P) & 1) || ((j >> Q) & 1) || !ctl_on<CM>(j)) continue;
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
            if (!((G >> an) & 1)) continue;
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

}  // namespace reg
}  // namespace mqb

#endif
