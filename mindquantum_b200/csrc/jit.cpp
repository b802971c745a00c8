// Pass kernels generated at run time (see jit.h).
//
// The precompiled tile kernels dispatch every gate through a switch inside the stage loop; at
// the switch's join the register array must sit in the same registers on every path, which
// costs register moves and keeps runtime control tests in the loop.  A generated pass kernel is
// straight-line code per stage instead: register indices, control masks (register controls as
// template masks, thread and outside controls as a per-thread `on` that swaps in the identity),
// matrix-table offsets and gradient slots are literals, and no branch or join remains between
// the gates of a stage.
#include "jit.h"

#include <cuda_runtime.h>
#include <nvrtc.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace mqb {

// Header texts for NVRTC, embedded at build time from regmath.cuh, tile.cuh and jit_abi.h.
extern const char *const kJitRegmath;
extern const char *const kJitTile;
extern const char *const kJitAbi;

namespace {

struct Entry {
    std::string src;
    std::vector<char> cubin;
    std::string log;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    bool done = false;
};

std::mutex g_mu;
std::unordered_map<std::string, std::shared_ptr<Entry>> g_cache;

const char *vname(int precision) { return precision == MQB_PREC_C64 ? "float2" : "double2"; }
const char *rname(int precision) { return precision == MQB_PREC_C64 ? "float" : "double"; }
int elem_bytes(int precision) { return precision == MQB_PREC_C64 ? 8 : 16; }
size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

// Thread-local tile bit pattern Lt of a stage, as an expression of threadIdx.x.
std::string lt_expr(const StageDesc &sd, int TB) {
    std::ostringstream o;
    o << "(0u";
    for (int i = 0; i < TB; ++i) o << " | (((tid >> " << i << ") & 1u) << " << int(sd.tbits[i]) << ")";
    o << ")";
    return o.str();
}

// Swizzled shared-memory offsets of the thread's register amplitudes (XOR with swz(Lt)).
std::vector<uint32_t> reg_offsets(const StageDesc &sd, int RB, int precision) {
    std::vector<uint32_t> off(size_t(1) << RB);
    for (int j = 0; j < (1 << RB); ++j) {
        uint32_t L = 0;
        for (int i = 0; i < RB; ++i)
            if (j >> i & 1) L |= 1u << sd.rbits[i];
        off[j] = smem_swizzle(L, precision);
    }
    return off;
}

std::string off_bit_expr(int src, int val) {
    std::ostringstream o;
    if (src == 1) o << "int((Lt >> " << val << ") & 1u)";
    else if (src == 2) o << "int((base >> " << val << ") & 1ull)";
    else o << "0";
    return o.str();
}

// `on` of an op whose controls include thread bits or outside qubits ("" when it has none).
std::string on_expr(const StageOp &so) {
    std::ostringstream o;
    bool any = false;
    if (so.tctrl) {
        o << "((Lt & " << so.tctrl << "u) == " << so.tctrl << "u)";
        any = true;
    }
    if (so.octrl) {
        if (any) o << " && ";
        o << "((base & " << so.octrl << "ull) == " << so.octrl << "ull)";
        any = true;
    }
    return any ? o.str() : std::string();
}

std::string mt(int i) { return "mt[" + std::to_string(i) + "]"; }

// ------------------------------------------------------------------------------ forward ops
void emit_forward_op(std::ostringstream &o, const StageOp &so) {
    const std::string on = on_expr(so);
    const bool cond = !on.empty();
    const int M = so.moff;
    const std::string CM = std::to_string(so.rctrl) + "u";
    o << "    {\n";
    if (cond) o << "      const bool on = " << on << ";\n";
    auto sel = [&](const std::string &val, const std::string &id) { return cond ? "(on ? " + val + " : " + id + ")" : val; };
    const std::string one = "cval<V>(1, 0)", zero = "cval<V>(0, 0)";
    switch (so.kind) {
        case SK_DENSE1:
        case SK_PERM1:
            o << "      j_dense1<V, RB, " << so.p0 << ", " << CM << ">(v, " << sel(mt(M), one) << ", "
              << sel(mt(M + 1), zero) << ", " << sel(mt(M + 2), zero) << ", " << sel(mt(M + 3), one) << ");\n";
            break;
        case SK_REAL1:
            o << "      j_real1<V, RB, " << so.p0 << ", " << CM << ">(v, " << sel(mt(M) + ".x", "R(1)") << ", "
              << sel(mt(M + 1) + ".x", "R(0)") << ", " << sel(mt(M + 2) + ".x", "R(0)") << ", "
              << sel(mt(M + 3) + ".x", "R(1)") << ");\n";
            break;
        case SK_RXL1:
            o << "      j_rxl1<V, RB, " << so.p0 << ", " << CM << ">(v, " << sel(mt(M) + ".x", "R(1)") << ", "
              << sel(mt(M + 1) + ".y", "R(0)") << ");\n";
            break;
        case SK_SWAP1:
            if (cond) o << "      j_x1sel<V, RB, " << so.p0 << ", " << CM << ">(v, on);\n";
            else o << "      j_x1<V, RB, " << so.p0 << ", " << CM << ">(v);\n";
            break;
        case SK_DIAG1:
            if (so.dsrc[0] == 0) {
                o << "      j_diag1<V, RB, " << so.dval[0] << ", " << CM << ">(v, " << sel(mt(M), one) << ", "
                  << sel(mt(M + 1), one) << ");\n";
            } else {
                o << "      const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << ";\n";
                o << "      j_scale<V, RB, " << CM << ">(v, " << sel("mt[" + std::to_string(M) + " + r]", one) << ");\n";
            }
            break;
        case SK_DIAG2: {
            const bool in0 = so.dsrc[0] == 0, in1 = so.dsrc[1] == 0;
            if (in0 && in1) {
                o << "      j_diag2<V, RB, " << so.dval[0] << ", " << so.dval[1] << ", " << CM << ">(v, "
                  << sel(mt(M), one) << ", " << sel(mt(M + 1), one) << ", " << sel(mt(M + 2), one) << ", "
                  << sel(mt(M + 3), one) << ");\n";
            } else if (in0 || in1) {
                const int k = in0 ? 0 : 1;
                o << "      const int b = " << off_bit_expr(so.dsrc[1 - k], so.dval[1 - k]) << ";\n";
                if (k == 0) o << "      const int i0 = b << 1, i1 = 1 | (b << 1);\n";
                else o << "      const int i0 = b, i1 = 2 | b;\n";
                o << "      j_diag1<V, RB, " << so.dval[k] << ", " << CM << ">(v, "
                  << sel("mt[" + std::to_string(M) + " + i0]", one) << ", "
                  << sel("mt[" + std::to_string(M) + " + i1]", one) << ");\n";
            } else {
                o << "      const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << " | ("
                  << off_bit_expr(so.dsrc[1], so.dval[1]) << " << 1);\n";
                o << "      j_scale<V, RB, " << CM << ">(v, " << sel("mt[" + std::to_string(M) + " + r]", one) << ");\n";
            }
        } break;
        case SK_DENSE2:
            if (cond) o << "      if (on)";
            o << "      j_dense2<V, RB, " << so.p0 << ", " << so.p1 << ", " << CM << ">(v, mt + " << M << ");\n";
            break;
        default:
            throw std::runtime_error("generated pass kernel: unknown stage op kind");
    }
    o << "    }\n";
}

// ------------------------------------------------------------------------------ backward ops
// Generator weights of the diagonal phase gates (dU/dt = -i W U, W real diagonal); empty when the
// gate's gradient goes through its derivative matrix instead.
std::vector<double> phase_weights(int gid) {
    switch (gid) {
        case GID_RZ: return {0.5, -0.5};
        case GID_PS: return {0.0, -1.0};
        case GID_GP: return {1.0, 1.0};
        case GID_RZZ: return {0.5, -0.5, -0.5, 0.5};
        default: return {};
    }
}

std::string lit(double x) {
    std::ostringstream o;
    o.precision(17);
    o << "R(" << x << ")";
    return o.str();
}

void emit_backward_op(std::ostringstream &o, const StageOp &so, int NH, int gid) {
    const std::string on = on_expr(so);
    const bool cond = !on.empty();
    const int M = so.moff;
    const int G = so.n_angles ? so.grad_mask : 0;
    const int ms = so.mat_size;
    const std::string CM = std::to_string(so.rctrl) + "u";
    const std::string NHs = std::to_string(NH);
    o << "    {\n";
    if (cond) o << "      const bool on = " << on << ";\n";
    if (G) o << "      R acc[3][NH] = {};\n";
    else o << "      R acc[3][NH];\n";
    auto sel = [&](const std::string &val, const std::string &id) { return cond ? "(on ? " + val + " : " + id + ")" : val; };
    const std::string one = "cval<V>(1, 0)", zero = "cval<V>(0, 0)";
    auto dm = [&](int a, int e) { return mt(M + ms * (1 + a) + e); };
    const std::vector<double> pw = (G == 1) ? phase_weights(gid) : std::vector<double>();
    const bool gen_ry = G == 1 && gid == GID_RY && so.kind == SK_REAL1;
    const bool gen_rx = G == 1 && gid == GID_RX && so.kind == SK_RXL1;
    const bool gen_diag = !pw.empty() && (so.kind == SK_DIAG1 || so.kind == SK_DIAG2);
    auto wsel = [&](const std::string &w) { return cond ? "(on ? " + w + " : R(0))" : w; };
    if (gen_ry) {
        o << "      jbg_ry<V, RB, NH, " << so.p0 << ", " << CM << ">(v, l, " << sel(mt(M) + ".x", "R(1)") << ", "
          << sel(mt(M + 2) + ".x", "R(0)") << ", " << sel(mt(M + 1) + ".x", "R(0)") << ", "
          << sel(mt(M + 3) + ".x", "R(1)") << ", " << wsel("R(0.5)") << ", acc);\n";
    } else if (gen_rx) {
        o << "      jbg_rx<V, RB, NH, " << so.p0 << ", " << CM << ">(v, l, " << sel(mt(M) + ".x", "R(1)") << ", "
          << sel("-" + mt(M + 1) + ".y", "R(0)") << ", " << wsel("R(0.5)") << ", acc);\n";
    } else if (gen_diag) {
        const bool two = so.kind == SK_DIAG2;
        const bool in0 = so.dsrc[0] == 0, in1 = two && so.dsrc[1] == 0;
        auto c = [&](const std::string &idx) { return sel("cconj(mt[" + std::to_string(M) + " + " + idx + "])", one); };
        if (!two && in0) {
            o << "      jbg_diag1<V, RB, NH, " << so.dval[0] << ", " << CM << ">(v, l, " << c("0") << ", " << c("1")
              << ", " << wsel(lit(pw[0])) << ", " << wsel(lit(pw[1])) << ", acc);\n";
        } else if (two && in0 && in1) {
            o << "      const V c[4] = {" << c("0") << ", " << c("1") << ", " << c("2") << ", " << c("3") << "};\n";
            o << "      const R w[4] = {" << wsel(lit(pw[0])) << ", " << wsel(lit(pw[1])) << ", " << wsel(lit(pw[2]))
              << ", " << wsel(lit(pw[3])) << "};\n";
            o << "      jbg_diag2<V, RB, NH, " << so.dval[0] << ", " << so.dval[1] << ", " << CM << ">(v, l, c, w, acc);\n";
        } else if (two && (in0 || in1)) {
            const int k = in0 ? 0 : 1;
            o << "      const int b = " << off_bit_expr(so.dsrc[1 - k], so.dval[1 - k]) << ";\n";
            if (k == 0) o << "      const int i0 = b << 1, i1 = 1 | (b << 1);\n";
            else o << "      const int i0 = b, i1 = 2 | b;\n";
            // weights of the register bit's two values, picked by the other target's bit (selects, no indexing)
            const std::string w_lo = k == 0 ? "(b ? " + lit(pw[2]) + " : " + lit(pw[0]) + ")" : "(b ? " + lit(pw[1]) + " : " + lit(pw[0]) + ")";
            const std::string w_hi = k == 0 ? "(b ? " + lit(pw[3]) + " : " + lit(pw[1]) + ")" : "(b ? " + lit(pw[3]) + " : " + lit(pw[2]) + ")";
            o << "      jbg_diag1<V, RB, NH, " << so.dval[k] << ", " << CM << ">(v, l, " << c("i0") << ", " << c("i1")
              << ", " << wsel(w_lo) << ", " << wsel(w_hi) << ", acc);\n";
        } else {
            o << "      const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << " | ("
              << off_bit_expr(two ? so.dsrc[1] : 3, so.dval[1]) << " << 1);\n";
            const std::string w_r = pw.size() > 2 ? "(r == 0 ? " + lit(pw[0]) + " : r == 1 ? " + lit(pw[1]) + " : r == 2 ? " +
                                                        lit(pw[2]) + " : " + lit(pw[3]) + ")"
                                                  : "(r ? " + lit(pw[1]) + " : " + lit(pw[0]) + ")";
            o << "      jbg_scale<V, RB, NH, " << CM << ">(v, l, " << c("r") << ", " << wsel(w_r) << ", acc);\n";
        }
    } else
    switch (so.kind) {
        case SK_DENSE1:
        case SK_PERM1: {
            o << "      V d[3][4];\n";
            for (int a = 0; a < 3; ++a)
                for (int e = 0; e < 4; ++e)
                    o << "      d[" << a << "][" << e << "] = " << (((G >> a) & 1) ? sel(dm(a, e), zero) : zero) << ";\n";
            o << "      jb_dense1<V, RB, NH, " << so.p0 << ", " << CM << ", " << G << ">(v, l, "
              << sel("cconj(" + mt(M) + ")", one) << ", " << sel("cconj(" + mt(M + 2) + ")", zero) << ", "
              << sel("cconj(" + mt(M + 1) + ")", zero) << ", " << sel("cconj(" + mt(M + 3) + ")", one) << ", d, acc);\n";
        } break;
        case SK_REAL1: {
            auto d = [&](int e) { return (G & 1) ? sel(dm(0, e) + ".x", "R(0)") : std::string("R(0)"); };
            o << "      jb_real1<V, RB, NH, " << so.p0 << ", " << CM << ", " << G << ">(v, l, "
              << sel(mt(M) + ".x", "R(1)") << ", " << sel(mt(M + 2) + ".x", "R(0)") << ", "
              << sel(mt(M + 1) + ".x", "R(0)") << ", " << sel(mt(M + 3) + ".x", "R(1)") << ", " << d(0) << ", "
              << d(1) << ", " << d(2) << ", " << d(3) << ", acc);\n";
        } break;
        case SK_RXL1: {
            o << "      jb_rxl1<V, RB, NH, " << so.p0 << ", " << CM << ", " << G << ">(v, l, "
              << sel(mt(M) + ".x", "R(1)") << ", " << sel("-" + mt(M + 1) + ".y", "R(0)") << ", "
              << ((G & 1) ? sel(dm(0, 0) + ".x", "R(0)") : "R(0)") << ", "
              << ((G & 1) ? sel(dm(0, 1) + ".y", "R(0)") : "R(0)") << ", acc);\n";
        } break;
        case SK_SWAP1:
            if (cond) o << "      jb_x1sel<V, RB, NH, " << so.p0 << ", " << CM << ">(v, l, on);\n";
            else o << "      jb_x1<V, RB, NH, " << so.p0 << ", " << CM << ">(v, l);\n";
            break;
        case SK_DIAG1:
        case SK_DIAG2: {
            const bool two = so.kind == SK_DIAG2;
            const bool in0 = so.dsrc[0] == 0, in1 = two && so.dsrc[1] == 0;
            auto c = [&](const std::string &idx) { return sel("cconj(mt[" + std::to_string(M) + " + " + idx + "])", one); };
            auto e = [&](const std::string &idx) {
                return (G & 1) ? sel("mt[" + std::to_string(M + ms) + " + " + idx + "]", zero) : zero;
            };
            if (!two && in0) {
                o << "      jb_diag1<V, RB, NH, " << so.dval[0] << ", " << CM << ", " << G << ">(v, l, " << c("0")
                  << ", " << c("1") << ", " << e("0") << ", " << e("1") << ", acc);\n";
            } else if (two && in0 && in1) {
                o << "      const V c[4] = {" << c("0") << ", " << c("1") << ", " << c("2") << ", " << c("3") << "};\n";
                o << "      const V e[4] = {" << e("0") << ", " << e("1") << ", " << e("2") << ", " << e("3") << "};\n";
                o << "      jb_diag2<V, RB, NH, " << so.dval[0] << ", " << so.dval[1] << ", " << CM << ", " << G
                  << ">(v, l, c, e, acc);\n";
            } else if (two && (in0 || in1)) {
                const int k = in0 ? 0 : 1;
                o << "      const int b = " << off_bit_expr(so.dsrc[1 - k], so.dval[1 - k]) << ";\n";
                if (k == 0) o << "      const int i0 = b << 1, i1 = 1 | (b << 1);\n";
                else o << "      const int i0 = b, i1 = 2 | b;\n";
                o << "      jb_diag1<V, RB, NH, " << so.dval[k] << ", " << CM << ", " << G << ">(v, l, " << c("i0")
                  << ", " << c("i1") << ", " << e("i0") << ", " << e("i1") << ", acc);\n";
            } else {
                o << "      const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << " | ("
                  << off_bit_expr(two ? so.dsrc[1] : 3, so.dval[1]) << " << 1);\n";
                o << "      jb_scale<V, RB, NH, " << CM << ", " << G << ">(v, l, " << c("r") << ", " << e("r")
                  << ", acc);\n";
            }
        } break;
        case SK_DENSE2:
            if (G & ~7) throw std::runtime_error("generated pass kernel: gradient mask out of range");
            if (cond) o << "      if (on)";
            o << "      jb_dense2<V, RB, NH, " << so.p0 << ", " << so.p1 << ", " << CM << ", " << G
              << ">(v, l, mt + " << M << ", acc);\n";
            break;
        default:
            throw std::runtime_error("generated pass kernel: unknown stage op kind");
    }
    if (G && so.lslot >= 0) {
        int r = 0;
        for (int a = 0; a < 3; ++a) {
            if (!((G >> a) & 1)) continue;
            o << "      for (int h = 0; h < NH; ++h) {\n"
              << "        const double x = double(warp_sum_acc(acc[" << a << "][h]));\n"
              << "        if (lane == 0) wacc[(warp * NLS + " << (so.lslot + r) << ") * NH + h] += x;\n"
              << "      }\n";
            ++r;
        }
    }
    o << "    }\n";
}

// ------------------------------------------------------------------ runs of diagonal gates
// Consecutive diagonal gates of a stage commute; their product is applied as one per-amplitude
// factor.  Factors of targets off the registers are one scalar per thread, single-target factors
// on register P are a pair (d0, d1) per thread, so a per-thread table over the register bits
// carrying such factors costs about two complex products per amplitude for the whole run,
// after which the run is one complex product per amplitude.  Two-target and register-controlled
// factors are multiplied in per amplitude.  In the adjoint, Im(conj(lambda) psi) is the same at
// every point of the run (a common unit-modulus diagonal cancels), so all gradients of the run
// come from sums of it over the thread's amplitudes, split by the bits their weights depend on.

bool diag_op(const StageOp &so) { return so.kind == SK_DIAG1 || so.kind == SK_DIAG2; }

// Gates a run may hold in the adjoint: no gradient, or a generator-form gradient.
bool run_ok_backward(const StageOp &so, int gid) {
    if (!diag_op(so)) return false;
    const int G = so.n_angles ? so.grad_mask : 0;
    return G == 0 || (G == 1 && !phase_weights(gid).empty());
}

struct RunPlan {
    std::vector<int> bits;   // register positions carrying per-thread factor pairs
};

enum DiagShape { DS_OFF, DS_REG1, DS_REGOFF, DS_OTHER };
DiagShape diag_shape(const StageOp &so) {
    const bool two = so.kind == SK_DIAG2;
    const bool in0 = so.dsrc[0] == 0, in1 = two && so.dsrc[1] == 0;
    if (so.rctrl) return DS_OTHER;
    if (!in0 && !in1) return DS_OFF;
    if (!two) return DS_REG1;
    if (in0 != in1) return DS_REGOFF;
    return DS_OTHER;
}
int diag_reg_bit(const StageOp &so) { return so.dsrc[0] == 0 ? so.dval[0] : so.dval[1]; }

// Per-thread factors of a run: sc (scalar) and f0_P / f1_P (pairs); `conj` for U^dag.
RunPlan emit_run_factors(std::ostringstream &o, const std::vector<const StageOp *> &run, bool conj) {
    RunPlan plan;
    const std::string one = "cval<V>(1, 0)";
    auto ent = [&](int M, const std::string &idx) {
        const std::string e = "mt[" + std::to_string(M) + " + " + idx + "]";
        return conj ? "cconj(" + e + ")" : e;
    };
    o << "      V sc = cval<V>(1, 0);\n";
    for (int P = 0; P < kMaxRegBits; ++P) {
        bool used = false;
        for (const StageOp *so : run)
            if ((diag_shape(*so) == DS_REG1 || diag_shape(*so) == DS_REGOFF) && diag_reg_bit(*so) == P) used = true;
        if (used) {
            plan.bits.push_back(P);
            o << "      V f0_" << P << " = cval<V>(1, 0), f1_" << P << " = cval<V>(1, 0);\n";
        }
    }
    for (const StageOp *sp : run) {
        const StageOp &so = *sp;
        const std::string on = on_expr(so);
        auto sel = [&](const std::string &v) { return on.empty() ? v : "((" + on + ") ? " + v + " : " + one + ")"; };
        const DiagShape sh = diag_shape(so);
        const int M = so.moff;
        if (sh == DS_OFF) {
            const bool two = so.kind == SK_DIAG2;
            o << "      { const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << " | ("
              << off_bit_expr(two ? so.dsrc[1] : 3, so.dval[1]) << " << 1); sc = cmul(sc, " << sel(ent(M, "r")) << "); }\n";
        } else if (sh == DS_REG1) {
            const int P = so.dval[0];
            o << "      f0_" << P << " = cmul(f0_" << P << ", " << sel(ent(M, "0")) << "); f1_" << P << " = cmul(f1_" << P
              << ", " << sel(ent(M, "1")) << ");\n";
        } else if (sh == DS_REGOFF) {
            const int k = so.dsrc[0] == 0 ? 0 : 1;
            const int P = so.dval[k];
            o << "      { const int b = " << off_bit_expr(so.dsrc[1 - k], so.dval[1 - k]) << ";\n";
            if (k == 0) o << "        const int i0 = b << 1, i1 = 1 | (b << 1);\n";
            else o << "        const int i0 = b, i1 = 2 | b;\n";
            o << "        f0_" << P << " = cmul(f0_" << P << ", " << sel(ent(M, "i0")) << "); f1_" << P << " = cmul(f1_" << P
              << ", " << sel(ent(M, "i1")) << "); }\n";
        }
    }
    // table over the factor bits
    const int nb = int(plan.bits.size());
    o << "      V T[" << (1 << nb) << "];\n      T[0] = sc;\n";
    for (int k = 0; k < nb; ++k) {
        const int P = plan.bits[k];
        for (int idx = 0; idx < (1 << k); ++idx) {
            o << "      T[" << (idx | (1 << k)) << "] = cmul(T[" << idx << "], f1_" << P << "); T[" << idx << "] = cmul(T["
              << idx << "], f0_" << P << ");\n";
        }
    }
    return plan;
}

// The factor of amplitude j: table entry times the per-amplitude factors of the run's other gates.
std::string run_factor_expr(std::ostringstream &o, const RunPlan &plan, const std::vector<const StageOp *> &run, int j,
                            bool conj) {
    int idx = 0;
    for (size_t k = 0; k < plan.bits.size(); ++k)
        if (j >> plan.bits[k] & 1) idx |= 1 << k;
    std::string d = "T[" + std::to_string(idx) + "]";
    const std::string one = "cval<V>(1, 0)";
    for (const StageOp *sp : run) {
        const StageOp &so = *sp;
        const DiagShape sh = diag_shape(so);
        if (sh != DS_OTHER) continue;
        if ((uint32_t(j) & so.rctrl) != so.rctrl) continue;   // register controls not satisfied: identity
        const std::string on = on_expr(so);
        // entry index from the targets' bits (register bits are literals here)
        std::string r;
        auto bit = [&](int k) -> std::string {
            if (so.dsrc[k] == 0) return std::to_string((j >> so.dval[k]) & 1);
            return "(" + off_bit_expr(so.dsrc[k], so.dval[k]) + ")";
        };
        if (so.kind == SK_DIAG1) r = bit(0);
        else r = bit(0) + " | (" + bit(1) + " << 1)";
        std::string e = "mt[" + std::to_string(so.moff) + " + (" + r + ")]";
        if (conj) e = "cconj(" + e + ")";
        if (!on.empty()) e = "((" + on + ") ? " + e + " : " + one + ")";
        d = "cmul(" + d + ", " + e + ")";
    }
    (void)o;
    return d;
}

void emit_forward_run(std::ostringstream &o, const std::vector<const StageOp *> &run, int RB) {
    o << "    {   // run of " << run.size() << " diagonal gates\n";
    const RunPlan plan = emit_run_factors(o, run, false);
    for (int j = 0; j < (1 << RB); ++j)
        o << "      v[" << j << "] = cmul(v[" << j << "], " << run_factor_expr(o, plan, run, j, false) << ");\n";
    o << "    }\n";
}

void emit_backward_run(std::ostringstream &o, const std::vector<const StageOp *> &run, const std::vector<int> &gids,
                       int RB, int NH) {
    o << "    {   // run of " << run.size() << " diagonal gates\n";
    // gradient sums of p_j = Im(conj(lambda_j) psi_j): all, per register bit, per special gate
    bool any_grad = false;
    std::vector<int> need_bits;
    for (size_t k = 0; k < run.size(); ++k) {
        const StageOp &so = *run[k];
        const int G = so.n_angles ? so.grad_mask : 0;
        if (!G) continue;
        any_grad = true;
        const DiagShape sh = diag_shape(so);
        if (sh == DS_REG1 || sh == DS_REGOFF) {
            const int P = diag_reg_bit(so);
            if (std::find(need_bits.begin(), need_bits.end(), P) == need_bits.end()) need_bits.push_back(P);
        }
    }
    if (any_grad) {
        o << "      R S[NH] = {};\n";
        for (int P : need_bits) o << "      R SB" << P << "[NH] = {};\n";
        for (size_t k = 0; k < run.size(); ++k) {
            const StageOp &so = *run[k];
            if ((so.n_angles ? so.grad_mask : 0) && diag_shape(so) == DS_OTHER)
                o << "      R SX" << k << "[4][NH] = {};\n";
        }
        for (int j = 0; j < (1 << RB); ++j) {
            o << "      for (int h = 0; h < NH; ++h) {\n        const R pj = fma(l[h][" << j << "].x, v[" << j << "].y, -l[h]["
              << j << "].y * v[" << j << "].x);\n        S[h] += pj;";
            for (int P : need_bits)
                if (j >> P & 1) o << " SB" << P << "[h] += pj;";
            for (size_t k = 0; k < run.size(); ++k) {
                const StageOp &so = *run[k];
                if (!((so.n_angles ? so.grad_mask : 0) && diag_shape(so) == DS_OTHER)) continue;
                if ((uint32_t(j) & so.rctrl) != so.rctrl) continue;
                // class of j by the gate's register targets (off-register target bits enter the weight)
                int cls = 0;
                if (so.dsrc[0] == 0) cls |= (j >> so.dval[0]) & 1;
                if (so.kind == SK_DIAG2 && so.dsrc[1] == 0) cls |= ((j >> so.dval[1]) & 1) << 1;
                o << " SX" << k << "[" << cls << "][h] += pj;";
            }
            o << "\n      }\n";
        }
        for (size_t k = 0; k < run.size(); ++k) {
            const StageOp &so = *run[k];
            const int G = so.n_angles ? so.grad_mask : 0;
            if (!G) continue;
            const std::vector<double> pw = phase_weights(gids[k]);
            const std::string on = on_expr(so);
            auto onw = [&](const std::string &w) { return on.empty() ? w : "((" + on + ") ? " + w + " : R(0))"; };
            auto wsel4 = [&](const std::string &r) {
                return pw.size() > 2 ? "(" + r + " == 0 ? " + lit(pw[0]) + " : " + r + " == 1 ? " + lit(pw[1]) + " : " + r +
                                           " == 2 ? " + lit(pw[2]) + " : " + lit(pw[3]) + ")"
                                     : "(" + r + " ? " + lit(pw[1]) + " : " + lit(pw[0]) + ")";
            };
            o << "      {\n        R acc[3][NH];\n";
            const DiagShape sh = diag_shape(so);
            if (sh == DS_OFF) {
                const bool two = so.kind == SK_DIAG2;
                o << "        const int r = " << off_bit_expr(so.dsrc[0], so.dval[0]) << " | ("
                  << off_bit_expr(two ? so.dsrc[1] : 3, so.dval[1]) << " << 1);\n";
                o << "        for (int h = 0; h < NH; ++h) acc[0][h] = " << onw(wsel4("r")) << " * S[h];\n";
            } else if (sh == DS_REG1) {
                const int P = so.dval[0];
                o << "        for (int h = 0; h < NH; ++h) acc[0][h] = " << onw(lit(pw[0])) << " * (S[h] - SB" << P << "[h]) + "
                  << onw(lit(pw[1])) << " * SB" << P << "[h];\n";
            } else if (sh == DS_REGOFF) {
                const int kk = so.dsrc[0] == 0 ? 0 : 1;
                const int P = so.dval[kk];
                o << "        const int b = " << off_bit_expr(so.dsrc[1 - kk], so.dval[1 - kk]) << ";\n";
                const std::string w_lo = kk == 0 ? "(b ? " + lit(pw[2]) + " : " + lit(pw[0]) + ")" : "(b ? " + lit(pw[1]) + " : " + lit(pw[0]) + ")";
                const std::string w_hi = kk == 0 ? "(b ? " + lit(pw[3]) + " : " + lit(pw[1]) + ")" : "(b ? " + lit(pw[3]) + " : " + lit(pw[2]) + ")";
                o << "        for (int h = 0; h < NH; ++h) acc[0][h] = " << onw(w_lo) << " * (S[h] - SB" << P << "[h]) + "
                  << onw(w_hi) << " * SB" << P << "[h];\n";
            } else {
                // class c of SX: register target bits; off-register target bits pick the weight per thread
                o << "        for (int h = 0; h < NH; ++h) acc[0][h] = R(0);\n";
                for (int cls = 0; cls < 4; ++cls) {
                    std::string r0 = so.dsrc[0] == 0 ? std::to_string(cls & 1) : "(" + off_bit_expr(so.dsrc[0], so.dval[0]) + ")";
                    std::string r1 = "0";
                    if (so.kind == SK_DIAG2)
                        r1 = so.dsrc[1] == 0 ? std::to_string((cls >> 1) & 1) : "(" + off_bit_expr(so.dsrc[1], so.dval[1]) + ")";
                    if (so.dsrc[0] != 0 && (cls & 1)) continue;
                    if ((so.kind != SK_DIAG2 || so.dsrc[1] != 0) && (cls & 2)) continue;
                    o << "        { const int r = " << r0 << " | (" << r1 << " << 1);\n"
                      << "          for (int h = 0; h < NH; ++h) acc[0][h] += " << onw(wsel4("r")) << " * SX" << k << "[" << cls
                      << "][h]; }\n";
                }
            }
            if (so.lslot >= 0)
                o << "        for (int h = 0; h < NH; ++h) {\n          const double x = double(warp_sum_acc(acc[0][h]));\n"
                  << "          if (lane == 0) wacc[(warp * NLS + " << so.lslot << ") * NH + h] += x;\n        }\n";
            o << "      }\n";
        }
    }
    const RunPlan plan = emit_run_factors(o, run, true);
    for (int j = 0; j < (1 << RB); ++j) {
        o << "      { const V d = " << run_factor_expr(o, plan, run, j, true) << "; v[" << j << "] = cmul(v[" << j
          << "], d); for (int h = 0; h < NH; ++h) l[h][" << j << "] = cmul(l[h][" << j << "], d); }\n";
    }
    o << "    }\n";
}

// Blocks per SM the register budget is sized for: 512 threads per SM at 128 registers each.
int min_blocks(int TB) { return std::max(1, 512 >> TB); }

void emit_header(std::ostringstream &o, int precision) {
    o << "#include \"regmath.cuh\"\n#include \"tile.cuh\"\n"
      << "using namespace mqb;\nusing namespace mqb::reg;\n"
      << "typedef " << vname(precision) << " V;\ntypedef " << rname(precision) << " R;\n";
}

void emit_stage_load(std::ostringstream &o, const StageDesc &sd, int RB, int TB, int precision, int NH) {
    const auto off = reg_offsets(sd, RB, precision);
    o << "   {\n    const unsigned Lt = " << lt_expr(sd, TB) << ";\n"
      << "    const unsigned pLt = tile::swz<V>(Lt);\n    V v[NR];\n";
    if (NH) o << "    V l[NH][NR];\n";
    for (int j = 0; j < (1 << RB); ++j) {
        if (NH) {
            o << "    v[" << j << "] = psi[pLt ^ " << off[j] << "u];";
            o << " for (int h = 0; h < NH; ++h) l[h][" << j << "] = lam[h * TS + (pLt ^ " << off[j] << "u)];\n";
        } else {
            o << "    v[" << j << "] = tl[pLt ^ " << off[j] << "u];\n";
        }
    }
}

void emit_stage_store(std::ostringstream &o, const StageDesc &sd, int RB, int precision, int NH) {
    const auto off = reg_offsets(sd, RB, precision);
    for (int j = 0; j < (1 << RB); ++j) {
        if (NH) {
            o << "    psi[pLt ^ " << off[j] << "u] = v[" << j << "];";
            o << " for (int h = 0; h < NH; ++h) lam[h * TS + (pLt ^ " << off[j] << "u)] = l[h][" << j << "];\n";
        } else {
            o << "    tl[pLt ^ " << off[j] << "u] = v[" << j << "];\n";
        }
    }
    o << "    __syncthreads();\n   }\n";
}

std::string forward_source(const Schedule &s, const Pass &p, int precision) {
    const int RB = p.f_reg_bits, K = p.K, TB = K - RB;
    std::ostringstream o;
    emit_header(o, precision);
    o << "extern \"C\" __global__ void __launch_bounds__(" << (1 << TB) << ", " << min_blocks(TB)
      << ") mqb_fwd_pass(const JitFwdArgs<V> a) {\n"
      << "  constexpr int RB = " << RB << ", NR = 1 << RB, K = " << K << ", C = " << p.c << ";\n"
      << "  constexpr int NV = NR / (16 / int(sizeof(V)));\n"
      << "  extern __shared__ __align__(16) unsigned char smem[];\n"
      << "  V *tl = reinterpret_cast<V *>(smem);\n"
      << "  tile::u64 o = tile::align16((tile::u64(1) << K) * sizeof(V));\n"
      << "  V *mt = reinterpret_cast<V *>(smem + o);\n"
      << "  o = tile::align16(o + tile::u64(a.mtab_entries) * sizeof(V));\n"
      << "  tile::u64 *tab = reinterpret_cast<tile::u64 *>(smem + o);\n"
      << "  tile::build_table(tab, a.g);\n  __syncthreads();\n"
      << "  const unsigned tid = threadIdx.x;\n"
      << "  const long long n_tiles = 1ll << a.g.n_out, dim = 1ll << a.g.n;\n"
      << "  long long cached_b = -1;\n"
      << "  for (long long w = blockIdx.x; w < a.batch * n_tiles; w += gridDim.x) {\n"
      << "   const long long b = w >> a.g.n_out;\n"
      << "   const tile::u64 base = tile::tile_base(a.g, tile::u64(w) & tile::u64(n_tiles - 1));\n"
      << "   if (b != cached_b) {\n    tile::load_mtab(mt, a.mt, a.n_mt, a.mats + b * a.mats_stride, a.cpool);\n"
      << "    cached_b = b;\n   }\n"
      << "   if (a.src) tile::stage_in<V, NV>(tl, a.src + b * a.src_batch_stride, base, tab, C);\n"
      << "   else tile::stage_zero(tl, base, K);\n   __syncthreads();\n";
    for (int si = 0; si < p.f_n_stages; ++si) {
        const StageDesc &sd = s.f_stages[p.f_stage_begin + si];
        emit_stage_load(o, sd, RB, TB, precision, 0);
        for (int k = sd.op_begin; k < sd.op_end;) {
            std::vector<const StageOp *> run;
            int e = k;
            while (e < sd.op_end && diag_op(s.f_stage_ops[p.f_sop_begin + e])) run.push_back(&s.f_stage_ops[p.f_sop_begin + e++]);
            if (run.size() >= 2) {
                emit_forward_run(o, run, RB);
                k = e;
            } else {
                emit_forward_op(o, s.f_stage_ops[p.f_sop_begin + k]);
                ++k;
            }
        }
        emit_stage_store(o, sd, RB, precision, 0);
    }
    o << "   tile::stage_out<V, NV>(tl, a.dst + b * dim, base, tab, C);\n   __syncthreads();\n  }\n}\n";
    return o.str();
}

std::string backward_source(const Schedule &s, const Pass &p, int precision, int NH, const std::vector<DevOp> &ops) {
    const int RB = p.reg_bits, K = p.K, TB = K - RB;
    const int NLS = std::max(1, p.n_slots);
    std::ostringstream o;
    emit_header(o, precision);
    o << "extern \"C\" __global__ void __launch_bounds__(" << (1 << TB) << ", " << min_blocks(TB)
      << ") mqb_adj_pass(const JitBwdArgs<V> a) {\n"
      << "  constexpr int RB = " << RB << ", NR = 1 << RB, K = " << K << ", C = " << p.c << ", NH = " << NH
      << ", NLS = " << NLS << ", TS = 1 << K;\n"
      << "  constexpr int NV = NR / (16 / int(sizeof(V)));\n"
      << "  extern __shared__ __align__(16) unsigned char smem[];\n"
      << "  V *psi = reinterpret_cast<V *>(smem);\n  V *lam = psi + TS;\n"
      << "  tile::u64 o = tile::align16(tile::u64(TS) * sizeof(V) * (1 + NH));\n"
      << "  V *mt = reinterpret_cast<V *>(smem + o);\n"
      << "  o = tile::align16(o + tile::u64(a.mtab_entries) * sizeof(V));\n"
      << "  tile::u64 *tab = reinterpret_cast<tile::u64 *>(smem + o);\n"
      << "  o = tile::align16(o + (tile::u64(1) << (K - C)) * sizeof(tile::u64));\n"
      << "  double *wacc = reinterpret_cast<double *>(smem + o);\n"
      << "  const int nw = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;\n"
      << "  tile::build_table(tab, a.g);\n"
      << "  for (int i = threadIdx.x; i < nw * NLS * NH; i += blockDim.x) wacc[i] = 0;\n  __syncthreads();\n"
      << "  const unsigned tid = threadIdx.x;\n"
      << "  const long long n_tiles = 1ll << a.g.n_out, dim = 1ll << a.g.n, total = a.batch * n_tiles;\n"
      << "  long long cached_b = -1;\n"
      << "  for (long long w = blockIdx.x; w < total; w += gridDim.x) {\n"
      << "   const long long b = w >> a.g.n_out;\n"
      << "   const tile::u64 base = tile::tile_base(a.g, tile::u64(w) & tile::u64(n_tiles - 1));\n"
      << "   if (b != cached_b) {\n    tile::load_mtab(mt, a.mt, a.n_mt, a.mats + b * a.mats_stride, a.cpool);\n"
      << "    cached_b = b;\n   }\n"
      << "   tile::stage_in<V, NV>(psi, a.psi_src + b * dim, base, tab, C);\n"
      << "   for (int h = 0; h < NH; ++h) tile::stage_in<V, NV>(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, C);\n"
      << "   __syncthreads();\n";
    for (int si = p.n_stages - 1; si >= 0; --si) {
        const StageDesc &sd = s.stages[p.stage_begin + si];
        emit_stage_load(o, sd, RB, TB, precision, NH);
        for (int k = sd.op_end - 1; k >= sd.op_begin;) {
            std::vector<const StageOp *> run;
            std::vector<int> gids;
            int e = k;
            while (e >= sd.op_begin) {
                const StageOp &so = s.stage_ops[p.sop_begin + e];
                if (!run_ok_backward(so, ops[so.op].gate_id)) break;
                run.push_back(&so);
                gids.push_back(ops[so.op].gate_id);
                --e;
            }
            if (run.size() >= 2) {
                emit_backward_run(o, run, gids, RB, NH);
                k = e;
            } else {
                const StageOp &so = s.stage_ops[p.sop_begin + k];
                emit_backward_op(o, so, NH, ops[so.op].gate_id);
                --k;
            }
        }
        emit_stage_store(o, sd, RB, precision, NH);
    }
    o << "   for (int h = 0; h < NH; ++h) tile::stage_out<V, NV>(lam + h * TS, a.lam + (h * a.batch + b) * dim, base, tab, C);\n"
      << "   if (a.psi_dst) tile::stage_out<V, NV>(psi, a.psi_dst + b * dim, base, tab, C);\n"
      << "   const long long nxt = w + gridDim.x;\n"
      << "   const bool flush = (nxt >= total) || ((nxt >> a.g.n_out) != b);\n"
      << "   __syncthreads();\n"
      << "   if (flush) {\n"
      << "    for (int i = threadIdx.x; i < a.n_local_slots * NH; i += blockDim.x) {\n"
      << "     double sum = 0;\n"
      << "     for (int ww = 0; ww < nw; ++ww) {\n"
      << "      sum += wacc[ww * NLS * NH + i];\n      wacc[ww * NLS * NH + i] = 0;\n     }\n"
      << "     const int ls = i / NH, h = i % NH;\n"
      << "     if (sum != 0) atomicAdd(&a.gslots[(b * a.n_slots + a.slot_map[ls]) * a.n_hams + h], sum);\n"
      << "    }\n    __syncthreads();\n   }\n  }\n}\n";
    return o.str();
}

void compile_entry(Entry &e) {
    nvrtcProgram prog = nullptr;
    const char *hdrs[3] = {kJitRegmath, kJitTile, kJitAbi};
    const char *names[3] = {"regmath.cuh", "tile.cuh", "jit_abi.h"};
    if (nvrtcCreateProgram(&prog, e.src.c_str(), "mqb_pass.cu", 3, hdrs, names) != NVRTC_SUCCESS) {
        e.log = "nvrtcCreateProgram failed";
        return;
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo"};
    const nvrtcResult r = nvrtcCompileProgram(prog, 3, opts);
    size_t log_n = 0;
    nvrtcGetProgramLogSize(prog, &log_n);
    std::string log(log_n, '\0');
    if (log_n) nvrtcGetProgramLog(prog, &log[0]);
    if (r == NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetCUBINSize(prog, &n);
        e.cubin.resize(n);
        nvrtcGetCUBIN(prog, e.cubin.data());
    } else {
        e.log = std::string(nvrtcGetErrorString(r)) + "\n" + log;
    }
    nvrtcDestroyProgram(&prog);
}

// Compile (in parallel) and load every source of `srcs` the cache lacks; returns the kernels.
std::vector<const void *> kernels_for(const std::vector<std::string> &srcs) {
    std::vector<std::shared_ptr<Entry>> entries(srcs.size());
    std::vector<std::shared_ptr<Entry>> todo;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (size_t i = 0; i < srcs.size(); ++i) {
            if (srcs[i].empty()) continue;
            auto &slot = g_cache[srcs[i]];
            if (!slot) {
                slot = std::make_shared<Entry>();
                slot->src = srcs[i];
                todo.push_back(slot);
            }
            entries[i] = slot;
        }
        if (!todo.empty()) {
            std::atomic<size_t> next{0};
            const unsigned nt = std::max(1u, std::min<unsigned>(unsigned(todo.size()), std::thread::hardware_concurrency()));
            std::vector<std::thread> pool;
            for (unsigned t = 0; t < nt; ++t)
                pool.emplace_back([&] {
                    for (size_t k = next++; k < todo.size(); k = next++) compile_entry(*todo[k]);
                });
            for (auto &th : pool) th.join();
            for (auto &e : todo) {
                if (e->cubin.empty()) {
                    const std::string msg = "compiling a generated pass kernel failed: " + e->log;
                    g_cache.erase(e->src);
                    throw std::runtime_error(msg);
                }
                cudaError_t ce = cudaLibraryLoadData(&e->lib, e->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
                const char *name = e->src.find(") mqb_adj_pass(") != std::string::npos ? "mqb_adj_pass" : "mqb_fwd_pass";
                if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&e->kernel, e->lib, name);
                if (ce != cudaSuccess) {
                    g_cache.erase(e->src);
                    throw std::runtime_error(std::string("loading a generated pass kernel: ") + cudaGetErrorString(ce));
                }
                e->done = true;
            }
        }
    }
    std::vector<const void *> out(srcs.size(), nullptr);
    for (size_t i = 0; i < srcs.size(); ++i)
        if (entries[i]) out[i] = reinterpret_cast<const void *>(entries[i]->kernel);
    return out;
}

}  // namespace

std::string jit_forward_source(const Schedule &s, const Pass &p, int precision) {
    return forward_source(s, p, precision);
}
std::string jit_backward_source(const Schedule &s, const Pass &p, int precision, int n_hams,
                                const std::vector<DevOp> &ops) {
    return backward_source(s, p, precision, n_hams, ops);
}

std::vector<const void *> jit_forward_kernels(const Schedule &s, int precision) {
    std::vector<std::string> srcs(s.passes.size());
    for (size_t i = 0; i < s.passes.size(); ++i)
        if (s.passes[i].fused) srcs[i] = forward_source(s, s.passes[i], precision);
    return kernels_for(srcs);
}

std::vector<const void *> jit_backward_kernels(const Schedule &s, int precision, int n_hams,
                                               const std::vector<DevOp> &ops) {
    std::vector<std::string> srcs(s.passes.size());
    for (size_t i = 0; i < s.passes.size(); ++i)
        if (s.passes[i].fused) srcs[i] = backward_source(s, s.passes[i], precision, n_hams, ops);
    return kernels_for(srcs);
}

int jit_compile_check(const Schedule &s, int precision, int n_hams, const std::vector<DevOp> &ops) {
    std::vector<std::string> srcs;
    for (const Pass &p : s.passes) {
        if (!p.fused) continue;
        srcs.push_back(forward_source(s, p, precision));
        if (n_hams > 0) srcs.push_back(backward_source(s, p, precision, n_hams, ops));
    }
    std::sort(srcs.begin(), srcs.end());
    srcs.erase(std::unique(srcs.begin(), srcs.end()), srcs.end());
    std::vector<Entry> es(srcs.size());
    std::atomic<size_t> next{0};
    const unsigned nt = std::max(1u, std::min<unsigned>(unsigned(es.size()), std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t i = 0; i < es.size(); ++i) es[i].src = srcs[i];
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t k = next++; k < es.size(); k = next++) compile_entry(es[k]);
        });
    for (auto &th : pool) th.join();
    for (const Entry &e : es)
        if (e.cubin.empty()) throw std::runtime_error("compiling a generated pass kernel failed: " + e.log);
    return int(es.size());
}

size_t jit_forward_smem(const Pass &p, int precision) {
    const size_t eb = elem_bytes(precision);
    size_t o = a16((size_t(1) << p.K) * eb);
    o = a16(o + size_t(p.f_mtab_entries) * eb);
    return o + (size_t(1) << (p.K - p.c)) * 8;
}

size_t jit_backward_smem(const Pass &p, int precision, int n_hams) {
    const size_t eb = elem_bytes(precision);
    const int threads = 1 << (p.K - p.reg_bits);
    size_t o = a16((size_t(1) << p.K) * eb * (1 + n_hams));
    o = a16(o + size_t(p.mtab_entries) * eb);
    o = a16(o + (size_t(1) << (p.K - p.c)) * 8);
    return o + size_t(threads / 32) * std::max(1, p.n_slots) * n_hams * sizeof(double);
}

cudaError_t jit_launch(const void *kernel, void *args, int threads, size_t smem, int sm_count, long long work,
                       cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const long long blocks = std::max<long long>(1, std::min<long long>((long long)sm_count * per_sm, work));
    void *argv[] = {args};
    e = cudaLaunchKernel(kernel, dim3(unsigned(blocks)), dim3(unsigned(threads)), argv, smem, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace mqb
