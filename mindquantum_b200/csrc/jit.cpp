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

#include <cuda.h>   // CUtensorMap and its enums; the encoder is fetched from the driver at run time
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>

#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace mqb {

// Header texts for NVRTC, embedded at build time from regmath.cuh, tile.cuh, jit_abi.h and pipe.cuh.
extern const char *const kJitRegmath;
extern const char *const kJitTile;
extern const char *const kJitAbi;
extern const char *const kJitPipe;

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
    const bool gen_u3 = G != 0 && gid == GID_U3 && so.kind == SK_DENSE1;
    auto wsel = [&](const std::string &w) { return cond ? "(on ? " + w + " : R(0))" : w; };
    if (gen_u3) {
        // e^{i lam} comes from the theta derivative, which is in the table only when theta has a gradient
        o << "      const V el = " << ((G & 1) ? "u3_phase(" + mt(M) + ", " + mt(M + 1) + ", " + dm(0, 0) + ", " + dm(0, 1) + ")"
                                           : std::string("cval<V>(1, 0)"))
          << ";\n";
        o << "      jbg_u3<V, RB, NH, " << so.p0 << ", " << CM << ", " << G << ">(v, l, "
          << sel("cconj(" + mt(M) + ")", one) << ", " << sel("cconj(" + mt(M + 2) + ")", zero) << ", "
          << sel("cconj(" + mt(M + 1) + ")", zero) << ", " << sel("cconj(" + mt(M + 3) + ")", one) << ", el, "
          << wsel("R(1)") << ", acc);\n";
    } else if (gen_ry) {
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

// ------------------------------------------------------------------------- tile movement (TMA)
// A tile lives in shared memory in one of two layouts: LAY_SWZ, the XOR-swizzled layout of the
// stage exchanges, and LAY_LAND, the order in which the TMA lands a tile and stores it from.
enum { LAY_SWZ = 0, LAY_LAND = 1 };

struct PassPlan {
    TmaGeom tg{};
    int box_lg[5] = {0, 0, 0, 0, 0};   // log2 of each dimension's box, in amplitudes
    std::vector<int> land;             // tile bit -> landing-layout bit
    int precision = MQB_PREC_C64;
};

// A box holds at most 256 elements per dimension (8-byte elements; complex128 takes two).
int max_box_bits(int precision) { return precision == MQB_PREC_C64 ? 8 : 7; }

// The tensor-map geometry of a pass's tile: the tile qubits split into runs of consecutive qubits
// (at most max_box_bits long); the run at qubit 0 and the four longest others become dimensions
// of the tensor map, the qubits of any further runs are fetched as separate boxes.
PassPlan pass_plan(const std::vector<int> &qbits, int precision) {
    PassPlan pl;
    pl.precision = precision;
    const int K = int(qbits.size());
    if (K == 0 || qbits[0] != 0) throw std::runtime_error("generated pass kernel: the tile must hold qubit 0");
    struct Chunk {
        int start, len, first;   // first global qubit, length, tile bit of the first qubit
    };
    std::vector<Chunk> ch;
    const int mb = max_box_bits(precision);
    for (int i = 0; i < K;) {
        int j = i;
        while (j + 1 < K && qbits[j + 1] == qbits[j] + 1) ++j;
        for (int s0 = i; s0 <= j; s0 += mb) ch.push_back({qbits[s0], std::min(mb, j - s0 + 1), s0});
        i = j + 1;
    }
    std::vector<char> keep(ch.size(), 0);
    keep[0] = 1;
    std::vector<int> rest;
    for (size_t k = 1; k < ch.size(); ++k) rest.push_back(int(k));
    std::stable_sort(rest.begin(), rest.end(), [&](int x, int y) { return ch[x].len > ch[y].len; });
    for (size_t k = 0; k < rest.size() && k < 4; ++k) keep[rest[k]] = 1;
    pl.land.assign(K, -1);
    int pos = 0, nd = 0;
    for (size_t k = 0; k < ch.size(); ++k) {
        if (!keep[k]) continue;
        pl.tg.shift[nd] = ch[k].start;
        pl.box_lg[nd] = ch[k].len;
        ++nd;
        for (int b = 0; b < ch[k].len; ++b) pl.land[ch[k].first + b] = pos++;
    }
    const int dim_bits = pos;
    int nl = 0;
    for (size_t k = 0; k < ch.size(); ++k) {
        if (keep[k]) continue;
        for (int b = 0; b < ch[k].len; ++b) {
            pl.tg.loop_q[nl++] = ch[k].start + b;
            pl.land[ch[k].first + b] = pos++;
        }
    }
    pl.tg.nd = nd;
    pl.tg.n_loop = nl;
    pl.tg.epa = precision == MQB_PREC_C64 ? 1 : 2;
    pl.tg.box_bytes = (1 << dim_bits) * elem_bytes(precision);
    return pl;
}

uint32_t lay_index(const PassPlan &pl, int lay, uint32_t L) {
    if (lay == LAY_SWZ) return smem_swizzle(L, pl.precision);
    uint32_t o = 0;
    for (size_t i = 0; i < pl.land.size(); ++i)
        if (L >> i & 1) o |= 1u << pl.land[i];
    return o;
}

// Shared-memory index of the thread's base amplitude Lt under a layout, as an expression.
std::string lay_lt_expr(const PassPlan &pl, int lay, const StageDesc &sd, int TB) {
    if (lay == LAY_SWZ) return "tile::swz<V>(Lt)";
    std::ostringstream o;
    o << "(0u";
    for (int i = 0; i < TB; ++i) o << " | (((tid >> " << i << ") & 1u) << " << pl.land[sd.tbits[i]] << ")";
    o << ")";
    return o.str();
}

// Whether the lanes of one shared-memory wavefront (a half-warp for 8-byte, a quarter-warp for
// 16-byte amplitudes) fall on distinct banks when a stage accesses a layout: the lanes' layout
// offsets must span the low 4 (3) index bits.
bool lay_conflict_free(const PassPlan &pl, int lay, const StageDesc &sd, int TB) {
    const int lanes = pl.precision == MQB_PREC_C64 ? 4 : 3;
    if (TB < lanes) return false;
    uint32_t rows[4] = {0, 0, 0, 0};
    for (int i = 0; i < lanes; ++i) rows[i] = lay_index(pl, lay, 1u << sd.tbits[i]) & ((1u << lanes) - 1u);
    int rank = 0;
    for (int bit = lanes - 1; bit >= 0; --bit) {
        int piv = -1;
        for (int i = rank; i < lanes; ++i)
            if (rows[i] >> bit & 1) {
                piv = i;
                break;
            }
        if (piv < 0) continue;
        std::swap(rows[rank], rows[piv]);
        for (int i = 0; i < lanes; ++i)
            if (i != rank && (rows[i] >> bit & 1)) rows[i] ^= rows[rank];
        ++rank;
    }
    return rank == lanes;
}

// Layouts of the stages of a kernel (in execution order): the first stage reads the landing
// layout and the last one writes it where that is free of bank conflicts; otherwise the tile is
// relaid in place (relayout_in / relayout_out) and the stage uses the swizzled layout.
struct LayPlan {
    std::vector<int> in, out;
    bool relayout_in = false, relayout_out = false;
};

LayPlan plan_layouts(const PassPlan &pl, const std::vector<const StageDesc *> &ex, int TB) {
    LayPlan lp;
    const size_t S = ex.size();
    lp.in.assign(S, LAY_SWZ);
    lp.out.assign(S, LAY_SWZ);
    if (lay_conflict_free(pl, LAY_LAND, *ex[0], TB)) lp.in[0] = LAY_LAND;
    else lp.relayout_in = true;
    if (lay_conflict_free(pl, LAY_LAND, *ex[S - 1], TB)) lp.out[S - 1] = LAY_LAND;
    else lp.relayout_out = true;
    return lp;
}

// In-place relayout of the n_tiles tiles at `tbase` between the landing and the swizzled layout.
// Every consumer thread moves 16-byte vectors (two complex64 or one complex128 amplitude): it reads
// all of its vectors, the consumers meet at a barrier, then it writes them.  Landing slot u holds
// tile amplitudes L(u) = landing^-1(apv u) (and L(u) ^ 1), L is linear in u, and so is the
// swizzled position Q(u) = swz(L(u)); a complex64 pair lands swapped where Q(u) is odd.
void emit_relayout(std::ostringstream &o, const PassPlan &pl, int K, int TB, int n_tiles, bool to_swz) {
    const int apv = pl.precision == MQB_PREC_C64 ? 2 : 1;
    const int sh = apv == 2 ? 1 : 0;
    const int ubits = K - sh, nvec = 1 << (ubits - TB);
    std::vector<int> inv(K);
    for (int i = 0; i < K; ++i) inv[pl.land[i]] = i;
    std::vector<uint32_t> qv(ubits);
    for (int k = 0; k < ubits; ++k) qv[k] = smem_swizzle(1u << inv[k + sh], pl.precision);
    o << "   {   // relayout " << (to_swz ? "landing -> swizzled" : "swizzled -> landing") << "\n";
    o << "    const unsigned qt = 0u";
    for (int k = 0; k < TB; ++k) o << " ^ (((tid >> " << k << ") & 1u) * " << qv[k] << "u)";
    o << ";\n    uint4 rv[" << n_tiles * nvec << "];\n";
    auto qk_of = [&](int k) {
        uint32_t q = 0;
        for (int bit = 0; bit < ubits - TB; ++bit)
            if (k >> bit & 1) q ^= qv[TB + bit];
        return q;
    };
    auto ptr = [&](int r) { return "reinterpret_cast<uint4 *>(tbase + " + std::to_string(r) + " * TS)"; };
    for (int r = 0; r < n_tiles; ++r)
        for (int k = 0; k < nvec; ++k) {
            const int idx = r * nvec + k;
            if (to_swz) o << "    rv[" << idx << "] = " << ptr(r) << "[tid + " << (k << TB) << "u];\n";
            else o << "    rv[" << idx << "] = " << ptr(r) << "[(qt ^ " << qk_of(k) << "u) >> " << sh << "];\n";
        }
    o << "    pipe::consumers_sync(BAR, NT);\n";
    for (int r = 0; r < n_tiles; ++r)
        for (int k = 0; k < nvec; ++k) {
            const int idx = r * nvec + k;
            if (apv == 2)
                o << "    if ((qt ^ " << qk_of(k) << "u) & 1u) rv[" << idx << "] = make_uint4(rv[" << idx << "].z, rv[" << idx
                  << "].w, rv[" << idx << "].x, rv[" << idx << "].y);\n";
            if (to_swz) o << "    " << ptr(r) << "[(qt ^ " << qk_of(k) << "u) >> " << sh << "] = rv[" << idx << "];\n";
            else o << "    " << ptr(r) << "[tid + " << (k << TB) << "u] = rv[" << idx << "];\n";
        }
    o << "    pipe::consumers_sync(BAR, NT);\n   }\n";
}

// Shape of a kernel's tile ring: G consumer groups of 2^(K - RB) threads share one block's ring
// of NB >= G tile buffers and take its tiles in turn (tile i goes to group i mod G and buffer
// i mod NB); each group has its own matrix table (and, in the adjoint, gradient slots).  There is
// no producer warp: a group stores its own tiles and refills their buffers, so a block of 16
// warps keeps 128 registers per thread.  Defaults (measured on the 26-qubit HEA gradient): two
// groups and three buffers for both kernels (forward 76 ms per step against 87 with one group of
// two buffers, 81 with four groups; adjoint 201 ms against 219 with two buffers).  MQB_PIPE_{FWD,BWD}_{GROUPS,BUFFERS} override them (tuning).
int env_int(const char *name, int dflt, int lo, int hi) {
    const char *e = std::getenv(name);
    return e ? std::max(lo, std::min(hi, std::atoi(e))) : dflt;
}

int max_groups(int nt) { return std::max(1, std::min(15, 1024 / nt)); }

int fwd_groups(const Pass &p) {
    const int nt = 1 << (p.K - p.f_reg_bits);
    return std::min(max_groups(nt), env_int("MQB_PIPE_FWD_GROUPS", 2, 1, 15));
}

int fwd_buffers(const Pass &p) { return std::max(fwd_groups(p), env_int("MQB_PIPE_FWD_BUFFERS", 3, 1, 8)); }

size_t fwd_smem(const Pass &p, int precision) {
    const size_t eb = elem_bytes(precision);
    return size_t(fwd_buffers(p)) * ((size_t(1) << p.K) * eb) +
           size_t(fwd_groups(p)) * a16(size_t(p.f_mtab_entries) * eb) + 8 * 16;
}

int bwd_groups(const Pass &p) {
    const int nt = 1 << (p.K - p.reg_bits);
    return std::min(max_groups(nt), env_int("MQB_PIPE_BWD_GROUPS", 2, 1, 15));
}

size_t bwd_fixed_smem(const Pass &p, int precision, int n_hams) {
    const size_t eb = elem_bytes(precision);
    const int nw = (1 << (p.K - p.reg_bits)) / 32;
    return size_t(bwd_groups(p)) *
               (a16(size_t(p.mtab_entries) * eb) + a16(size_t(nw) * std::max(1, p.n_slots) * n_hams * sizeof(double))) +
           8 * 16;
}

// Buffers of the adjoint ring: G + 1 where they fit in 227 KB, else as many as fit (at least G).
int bwd_buffers(const Pass &p, int precision, int n_hams) {
    const size_t buf = (size_t(1) << p.K) * elem_bytes(precision) * (1 + n_hams);
    const size_t fixed = bwd_fixed_smem(p, precision, n_hams);
    const int G = bwd_groups(p);
    int nb = env_int("MQB_PIPE_BWD_BUFFERS", G + 1, 1, 8);
    while (nb > G && nb * buf + fixed > size_t(227) << 10) --nb;
    if (nb * buf + fixed > size_t(227) << 10)
        throw std::runtime_error("generated adjoint pass: the tile ring does not fit in shared memory");
    return nb;
}

void emit_header(std::ostringstream &o, int precision) {
    o << "#include \"regmath.cuh\"\n#include \"tile.cuh\"\n#include \"pipe.cuh\"\n"
      << "using namespace mqb;\nusing namespace mqb::reg;\n"
      << "typedef " << vname(precision) << " V;\ntypedef " << rname(precision) << " R;\n";
}

uint32_t reg_local(const StageDesc &sd, int RB, int j) {
    uint32_t L = 0;
    for (int i = 0; i < RB; ++i)
        if (j >> i & 1) L |= 1u << sd.rbits[i];
    return L;
}

void emit_stage_load(std::ostringstream &o, const PassPlan &pl, const StageDesc &sd, int RB, int TB, int NH, int lay,
                     bool zero_start) {
    o << "   {\n    const unsigned Lt = " << lt_expr(sd, TB) << ";\n"
      << "    const unsigned pLt = " << lay_lt_expr(pl, lay, sd, TB) << ";\n    V v[NR];\n";
    if (NH) o << "    V l[NH][NR];\n";
    if (zero_start) {
        o << "    if (zero) {\n      v[0] = (base == 0 && Lt == 0u) ? cval<V>(1, 0) : cval<V>(0, 0);\n";
        for (int j = 1; j < (1 << RB); ++j) o << "      v[" << j << "] = cval<V>(0, 0);\n";
        o << "    } else {\n";
    }
    for (int j = 0; j < (1 << RB); ++j) {
        const uint32_t off = lay_index(pl, lay, reg_local(sd, RB, j));
        if (NH) {
            o << "    v[" << j << "] = psi[pLt ^ " << off << "u];";
            o << " for (int h = 0; h < NH; ++h) l[h][" << j << "] = lam[h * TS + (pLt ^ " << off << "u)];\n";
        } else {
            o << "    v[" << j << "] = tl[pLt ^ " << off << "u];\n";
        }
    }
    if (zero_start) o << "    }\n";
}

void emit_stage_store(std::ostringstream &o, const PassPlan &pl, const StageDesc &sd, int RB, int TB, int NH, int lay_in,
                      int lay_out, bool barrier_after) {
    if (lay_out != lay_in)
        o << "    pipe::consumers_sync(BAR, NT);\n    const unsigned pLo = " << lay_lt_expr(pl, lay_out, sd, TB) << ";\n";
    else
        o << "    const unsigned pLo = pLt;\n";
    for (int j = 0; j < (1 << RB); ++j) {
        const uint32_t off = lay_index(pl, lay_out, reg_local(sd, RB, j));
        if (NH) {
            o << "    psi[pLo ^ " << off << "u] = v[" << j << "];";
            o << " for (int h = 0; h < NH; ++h) lam[h * TS + (pLo ^ " << off << "u)] = l[h][" << j << "];\n";
        } else {
            o << "    tl[pLo ^ " << off << "u] = v[" << j << "];\n";
        }
    }
    if (barrier_after) o << "    pipe::consumers_sync(BAR, NT);\n";
    o << "   }\n";
}

// The tile ring of a kernel, by its consumer groups (no producer warp).  Tile k of this block (its
// tiles are blockIdx.x + k gridDim.x) goes to group k mod G and buffer k mod NB; the buffer is
// handed over through its `full` mbarrier, with the TMA's transaction bytes, or (forward passes that
// start from |0...0> and load nothing) with a plain arrival.  Thread 0 of block issues the first
// NB tiles; after that the group that finished tile k stores it (thread 0 of the group, after a
// group barrier) and, at the start of its next tile, refills the buffer with tile k + NB once the
// store has read it out.  Before the issuer arms a buffer it writes the tile's index into the
// buffer's ticket; a consumer tests the mbarrier's parity only once the ticket names its tile (the
// parity alone cannot tell a phase from the one two fills later).  A group that gave up a wait
// lets the copies it started into buffers whose ticket still names them land before it exits.
//
// `issue_body` issues the copies of tile k into buffer sb (b: sample, tb: the tile's outside bits);
// `store_body` those of the finished tile from buffer sb.
void emit_ring_prologue(std::ostringstream &o, const std::string &issue_body, bool zero_opt) {
    o << "  const int grp = int(threadIdx.x) / NT, BAR = 1 + grp;\n"
      << "  const unsigned tid = threadIdx.x % NT;\n"
      << "  const long long first = blockIdx.x, cnt = first < total ? (total - 1 - first) / gridDim.x + 1 : 0;\n"
      << "  const int n = a.g.n;\n"
      << "  long long mine[NB];\n"
      << "  for (int k = 0; k < NB; ++k) mine[k] = -1;\n"
      << "  auto issue = [&](long long k) {\n"
      << "   const int sb = int(k % NB);\n"
      << "   const long long w = first + k * gridDim.x, b = w >> a.g.n_out;\n"
      << "   const tile::u64 tb = tile::tile_base(a.g, tile::u64(w) & tile::u64(n_tiles - 1));\n"
      << "   unsigned char *buf = smem + sb * BUFB;\n"
      << "   mine[sb] = k;\n"
      << "   ticket[sb] = k;\n";
    if (zero_opt) o << "   if (zero) {\n    pipe::mbar_arrive(full + sb);\n    return;\n   }\n";
    o << "   pipe::mbar_expect_tx(full + sb, BUFB);\n" << issue_body << "  };\n"
      << "  if (threadIdx.x == 0)\n   for (long long k = 0; k < cnt && k < NB; ++k) issue(k);\n"
      << "  long long prev = -1;   // this group's last tile\n"
      << "  bool failed = false;\n";
}

// Start of a group's tile i: refill the buffer of its previous tile, then wait (together) for tile i.
void emit_ring_wait(std::ostringstream &o) {
    o << "   if (tid == 0u && prev >= 0 && prev + NB < cnt) {\n"
      << "    pipe::bulk_wait_read_all();\n    issue(prev + NB);\n   }\n"
      << "   if (!pipe::consumers_and(BAR, NT, tid != 0u || (pipe::wait_ticket(ticket + sb, i) && pipe::mbar_wait(full + sb, par)))) {\n"
      << "    if (tid == 0u) pipe::report(a.err, MQB_DEV_ERR_TIMEOUT);\n"
      << "    failed = true;\n"
      << "    break;\n"
      << "   }\n"
      << "   pipe::mbar_test(full + sb, par);\n";
}

// End of a group's tile i: every thread's writes made visible to the TMA, then thread 0 stores.
void emit_ring_store(std::ostringstream &o, const std::string &store_body) {
    o << "   pipe::fence_async_smem();\n   pipe::consumers_sync(BAR, NT);\n"
      << "   if (tid == 0u) {\n    const unsigned char *buf = smem + sb * BUFB;\n" << store_body
      << "    pipe::bulk_commit();\n   }\n   prev = i;\n";
}

void emit_ring_exit(std::ostringstream &o) {
    o << "  if (tid == 0u) {\n"
      << "   if (prev >= 0 && prev + NB < cnt) {   // a buffer nobody else refills (only when NB < G)\n"
      << "    pipe::bulk_wait_read_all();\n    issue(prev + NB);\n   }\n"
      << "   // after a timeout, copies this thread started may still be in flight (on the normal path every\n"
      << "   // copy is consumed before its group finishes); a buffer whose ticket moved on was refilled by\n"
      << "   // its consumer, so this thread's copy into it has landed\n"
      << "   if (failed)\n"
      << "    for (int k = 0; k < NB; ++k)\n"
      << "     if (mine[k] >= 0 && ticket[k] == mine[k]) pipe::mbar_wait(full + k, unsigned(mine[k] / NB) & 1u);\n"
      << "   pipe::bulk_wait_all();\n  }\n";
}

std::string forward_source(const Schedule &s, const Pass &p, int precision) {
    const int RB = p.f_reg_bits, K = p.K, TB = K - RB;
    const PassPlan pl = pass_plan(p.qbits, precision);
    const int NB = fwd_buffers(p), G = fwd_groups(p);
    std::vector<const StageDesc *> ex;
    for (int si = 0; si < p.f_n_stages; ++si) ex.push_back(&s.f_stages[p.f_stage_begin + si]);
    const LayPlan lp = plan_layouts(pl, ex, TB);
    // blocks per SM that the shared-memory ring allows: the register budget is sized for them
    const int min_blocks = int(std::max<size_t>(1, std::min<size_t>(3, (size_t(220) << 10) / fwd_smem(p, precision))));
    std::ostringstream o;
    emit_header(o, precision);
    o << "extern \"C\" __global__ void __launch_bounds__(" << G * (1 << TB) << ", " << min_blocks
      << ") mqb_fwd_pass(const JitFwdArgs<V> a, "
      << "const __grid_constant__ pipe::TMap m_src, const __grid_constant__ pipe::TMap m_dst) {\n"
      << "  constexpr int RB = " << RB << ", NR = 1 << RB, K = " << K << ", NT = 1 << (K - RB), NB = " << NB
      << ", G = " << G << ", TS = 1 << K;\n"
      << "  constexpr unsigned BUFB = TS * sizeof(V);\n"
      << "  extern __shared__ __align__(1024) unsigned char smem[];\n"
      << "  const tile::u64 mtb = tile::align16(tile::u64(a.mtab_entries) * sizeof(V));\n"
      << "  pipe::u64 *full = reinterpret_cast<pipe::u64 *>(smem + NB * BUFB + G * mtb);\n"
      << "  volatile long long *ticket = reinterpret_cast<volatile long long *>(full + NB);\n"
      << "  if (threadIdx.x == 0) {\n   for (int k = 0; k < NB; ++k) {\n    pipe::mbar_init(full + k, 1);\n    ticket[k] = -1;\n   }\n"
      << "   pipe::fence_mbar_init();\n  }\n  __syncthreads();\n"
      << "  const long long n_tiles = 1ll << a.g.n_out, total = a.batch * n_tiles;\n"
      << "  const bool zero = a.src == nullptr;\n";
    emit_ring_prologue(o,
                       "   const tile::u64 bs = a.src_batch_stride ? tile::u64(b) : 0;\n"
                       "   pipe::load_tile(&m_src, a.tg, (bs << n) | tb, buf, full + sb);\n",
                       true);
    o << "  V *mt = reinterpret_cast<V *>(smem + NB * BUFB + grp * mtb);\n"
      << "  long long cached_b = -1;\n"
      << "  for (long long i = grp; i < cnt; i += G) {\n"
      << "   const long long w = first + i * gridDim.x, b = w >> a.g.n_out;\n"
      << "   const tile::u64 base = tile::tile_base(a.g, tile::u64(w) & tile::u64(n_tiles - 1));\n"
      << "   const int sb = int(i % NB);\n   const unsigned par = unsigned(i / NB) & 1u;\n"
      << "   V *tl = reinterpret_cast<V *>(smem + sb * BUFB);\n"
      << "   if (b != cached_b) {\n    pipe::consumers_sync(BAR, NT);\n"
      << "    pipe::load_mtab(mt, a.mt, a.n_mt, a.mats + b * a.mats_stride, a.cpool, tid, NT);\n"
      << "    cached_b = b;\n    pipe::consumers_sync(BAR, NT);\n   }\n";
    emit_ring_wait(o);
    if (lp.relayout_in) {
        o << "   if (!zero) {\n    V *tbase = tl;\n";
        emit_relayout(o, pl, K, TB, 1, true);
        o << "   }\n";
    }
    for (size_t si = 0; si < ex.size(); ++si) {
        const StageDesc &sd = *ex[si];
        const bool last = si + 1 == ex.size();
        emit_stage_load(o, pl, sd, RB, TB, 0, lp.in[si], si == 0);
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
        if (last)   // the FP64 norm check of the output, when the launch asks for it
            o << "    if (a.norm) {\n     double ns = 0;\n"
              << "     for (int j = 0; j < NR; ++j) ns += double(v[j].x) * double(v[j].x) + double(v[j].y) * double(v[j].y);\n"
              << "     ns = warp_sum(ns);\n     if ((threadIdx.x & 31u) == 0u) atomicAdd(a.norm + 2 * b, ns);\n    }\n";
        emit_stage_store(o, pl, sd, RB, TB, 0, lp.in[si], lp.out[si], !last || lp.relayout_out);
    }
    if (lp.relayout_out) {
        o << "   {\n    V *tbase = tl;\n";
        emit_relayout(o, pl, K, TB, 1, false);
        o << "   }\n";
    }
    emit_ring_store(o, "    pipe::store_tile(&m_dst, a.tg, (tile::u64(b) << n) | base, buf);\n");
    o << "  }\n";
    emit_ring_exit(o);
    o << "}\n";
    return o.str();
}

std::string backward_source(const Schedule &s, const Pass &p, int precision, int NH, const std::vector<DevOp> &ops) {
    const int RB = p.reg_bits, K = p.K, TB = K - RB;
    const int NLS = std::max(1, p.n_slots);
    const PassPlan pl = pass_plan(p.qbits, precision);
    const int NB = bwd_buffers(p, precision, NH), G = bwd_groups(p);
    std::vector<const StageDesc *> ex;
    for (int si = p.n_stages - 1; si >= 0; --si) ex.push_back(&s.stages[p.stage_begin + si]);
    const LayPlan lp = plan_layouts(pl, ex, TB);
    std::ostringstream o;
    emit_header(o, precision);
    o << "extern \"C\" __global__ void __launch_bounds__(" << G * (1 << TB) << ", 1) mqb_adj_pass(const JitBwdArgs<V> a, "
      << "const __grid_constant__ pipe::TMap m_psi, const __grid_constant__ pipe::TMap m_lam, "
      << "const __grid_constant__ pipe::TMap m_pdst) {\n"
      << "  constexpr int RB = " << RB << ", NR = 1 << RB, K = " << K << ", NH = " << NH << ", NLS = " << NLS
      << ", TS = 1 << K, NT = 1 << (K - RB), NB = " << NB << ", G = " << G << ";\n"
      << "  constexpr unsigned TILEB = TS * sizeof(V), BUFB = TILEB * (1 + NH);\n"
      << "  constexpr int nw = NT / 32, WS = (nw * NLS * NH + 1) / 2 * 2;   // gradient slots of a group\n"
      << "  extern __shared__ __align__(1024) unsigned char smem[];\n"
      << "  const tile::u64 mtb = tile::align16(tile::u64(a.mtab_entries) * sizeof(V));\n"
      << "  double *wacc0 = reinterpret_cast<double *>(smem + NB * BUFB + G * mtb);\n"
      << "  pipe::u64 *full = reinterpret_cast<pipe::u64 *>(wacc0 + G * WS);\n"
      << "  volatile long long *ticket = reinterpret_cast<volatile long long *>(full + NB);\n"
      << "  if (threadIdx.x == 0) {\n   for (int k = 0; k < NB; ++k) {\n    pipe::mbar_init(full + k, 1);\n    ticket[k] = -1;\n   }\n"
      << "   pipe::fence_mbar_init();\n  }\n"
      << "  for (int i = int(threadIdx.x); i < G * WS; i += int(blockDim.x)) wacc0[i] = 0;\n  __syncthreads();\n"
      << "  const long long n_tiles = 1ll << a.g.n_out, total = a.batch * n_tiles;\n";
    emit_ring_prologue(o,
                       "   pipe::load_tile(&m_psi, a.tg, (tile::u64(b) << n) | tb, buf, full + sb);\n"
                       "   for (int h = 0; h < NH; ++h)\n"
                       "    pipe::load_tile(&m_lam, a.tg, (tile::u64(h * a.batch + b) << n) | tb, buf + (1 + h) * TILEB, "
                       "full + sb);\n",
                       false);
    o << "  const int warp = int(tid) / 32, lane = int(tid) % 32;\n"
      << "  V *mt = reinterpret_cast<V *>(smem + NB * BUFB + grp * mtb);\n"
      << "  double *wacc = wacc0 + grp * WS;\n"
      << "  long long cached_b = -1;\n"
      << "  for (long long i = grp; i < cnt; i += G) {\n"
      << "   const long long w = first + i * gridDim.x, b = w >> a.g.n_out;\n"
      << "   const tile::u64 base = tile::tile_base(a.g, tile::u64(w) & tile::u64(n_tiles - 1));\n"
      << "   const int sb = int(i % NB);\n   const unsigned par = unsigned(i / NB) & 1u;\n"
      << "   V *psi = reinterpret_cast<V *>(smem + sb * BUFB);\n   V *lam = psi + TS;\n"
      << "   if (b != cached_b) {\n    pipe::consumers_sync(BAR, NT);\n"
      << "    pipe::load_mtab(mt, a.mt, a.n_mt, a.mats + b * a.mats_stride, a.cpool, tid, NT);\n"
      << "    cached_b = b;\n    pipe::consumers_sync(BAR, NT);\n   }\n";
    emit_ring_wait(o);
    if (lp.relayout_in) {
        o << "   {\n    V *tbase = psi;\n";
        emit_relayout(o, pl, K, TB, 1 + NH, true);
        o << "   }\n";
    }
    for (size_t si = 0; si < ex.size(); ++si) {
        const StageDesc &sd = *ex[si];
        const bool last = si + 1 == ex.size();
        emit_stage_load(o, pl, sd, RB, TB, NH, lp.in[si], false);
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
        emit_stage_store(o, pl, sd, RB, TB, NH, lp.in[si], lp.out[si], !last || lp.relayout_out);
    }
    if (lp.relayout_out) {
        o << "   {\n    V *tbase = psi;\n";
        emit_relayout(o, pl, K, TB, 1 + NH, false);
        o << "   }\n";
    }
    emit_ring_store(o,
                    "    for (int h = 0; h < NH; ++h)\n"
                    "     pipe::store_tile(&m_lam, a.tg, (tile::u64(h * a.batch + b) << n) | base, buf + (1 + h) * TILEB);\n"
                    "    if (a.psi_dst) pipe::store_tile(&m_pdst, a.tg, (tile::u64(b) << n) | base, buf);\n");
    o << "   const long long nxt = i + G;\n"
      << "   if (nxt >= cnt || ((first + nxt * gridDim.x) >> a.g.n_out) != b) {\n"
      << "    pipe::consumers_sync(BAR, NT);\n"
      << "    for (int s2 = int(tid); s2 < a.n_local_slots * NH; s2 += NT) {\n"
      << "     double sum = 0;\n"
      << "     for (int ww = 0; ww < nw; ++ww) {\n"
      << "      sum += wacc[ww * NLS * NH + s2];\n      wacc[ww * NLS * NH + s2] = 0;\n     }\n"
      << "     const int ls = s2 / NH, h = s2 % NH;\n"
      << "     if (sum != 0) atomicAdd(&a.gslots[(b * a.n_slots + a.slot_map[ls]) * a.n_hams + h], sum);\n"
      << "    }\n    pipe::consumers_sync(BAR, NT);\n   }\n  }\n";
    emit_ring_exit(o);
    o << "}\n";
    return o.str();
}

// On-disk cache of the cubins compiled here, so a new process does not compile the same pass
// kernels again: MQB_JIT_CACHE names the directory ("0" disables it; default
// $XDG_CACHE_HOME/mqb200 or ~/.cache/mqb200).  An entry is keyed by a 64-bit hash of everything
// the compile reads (the source, the embedded headers, the options, the NVRTC version) and stores
// that input next to the cubin, which is loaded only when the stored input equals the current
// one.  The cubins are stored and loaded, never inspected.
std::string cache_dir() {
    const char *e = std::getenv("MQB_JIT_CACHE");
    if (e) return std::string(e) == "0" ? std::string() : std::string(e);
    if (const char *x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/mqb200";
    if (const char *h = std::getenv("HOME")) return std::string(h) + "/.cache/mqb200";
    return std::string();
}

std::string compile_input(const Entry &e, const char *const *opts, int n_opts) {
    int major = 0, minor = 0;
    nvrtcVersion(&major, &minor);
    std::string in = "nvrtc " + std::to_string(major) + "." + std::to_string(minor) + "\n";
    for (int i = 0; i < n_opts; ++i) in += std::string(opts[i]) + "\n";
    for (const char *h : {kJitRegmath, kJitTile, kJitAbi, kJitPipe}) in += std::string(h) + "\n";
    return in + e.src;
}

uint64_t fnv1a(const std::string &s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
    return h;
}

bool read_file(const std::string &path, std::string &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::string buf;
    char tmp[65536];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, k);
    std::fclose(f);
    out.swap(buf);
    return true;
}

void write_file_atomic(const std::string &path, const char *data, size_t n) {
    const std::string tmp = path + ".tmp" + std::to_string(std::hash<std::thread::id>()(std::this_thread::get_id()));
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return;
    const bool ok = std::fwrite(data, 1, n, f) == n;
    std::fclose(f);
    if (ok) std::rename(tmp.c_str(), path.c_str());
    else std::remove(tmp.c_str());
}

void compile_entry(Entry &e) {
    // MQB_JIT_DUMP=<directory>: write every generated source there (for reading them)
    if (const char *dir = std::getenv("MQB_JIT_DUMP")) {
        const std::string path = std::string(dir) + "/mqb_pass_" + std::to_string(std::hash<std::string>()(e.src)) + ".cu";
        if (FILE *f = std::fopen(path.c_str(), "w")) {
            std::fwrite(e.src.data(), 1, e.src.size(), f);
            std::fclose(f);
        }
    }
    nvrtcProgram prog = nullptr;
    const char *hdrs[4] = {kJitRegmath, kJitTile, kJitAbi, kJitPipe};
    const char *names[4] = {"regmath.cuh", "tile.cuh", "jit_abi.h", "pipe.cuh"};
    if (nvrtcCreateProgram(&prog, e.src.c_str(), "mqb_pass.cu", 4, hdrs, names) != NVRTC_SUCCESS) {
        e.log = "nvrtcCreateProgram failed";
        return;
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo"};
    const std::string dir = cache_dir();
    std::string input, key_path;
    if (!dir.empty()) {
        input = compile_input(e, opts, 3);
        char hex[17];
        std::snprintf(hex, sizeof(hex), "%016llx", static_cast<unsigned long long>(fnv1a(input)));
        key_path = dir + "/" + hex;
        std::string stored, cubin;
        if (read_file(key_path + ".in", stored) && stored == input && read_file(key_path + ".cubin", cubin) &&
            !cubin.empty()) {
            e.cubin.assign(cubin.begin(), cubin.end());
            nvrtcDestroyProgram(&prog);
            return;
        }
    }
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
        if (!key_path.empty()) {
            std::string cmd = dir;   // create the directory (and parents) if needed
            for (size_t i = 1; i <= cmd.size(); ++i)
                if (i == cmd.size() || cmd[i] == '/') mkdir(cmd.substr(0, i).c_str(), 0755);
            write_file_atomic(key_path + ".cubin", e.cubin.data(), e.cubin.size());
            write_file_atomic(key_path + ".in", input.data(), input.size());
        }
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

size_t jit_forward_smem(const Pass &p, int precision) { return fwd_smem(p, precision); }

size_t jit_backward_smem(const Pass &p, int precision, int n_hams) {
    const size_t buf = (size_t(1) << p.K) * elem_bytes(precision) * (1 + n_hams);
    return size_t(bwd_buffers(p, precision, n_hams)) * buf + bwd_fixed_smem(p, precision, n_hams);
}

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled, taken from the driver through the runtime (the library does not link
// libcuda itself).
EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    });
    if (!fn) throw std::runtime_error("generated pass kernel: cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

// Tensor map of the amplitudes at `base` ([outer][2^n]) for the tiles of plan pl: dimension j
// holds the index bits [shift[j], shift[j+1]) (the last one all bits above, times outer), its box
// the tile qubits at the bottom of that range.
void encode_map(CUtensorMap *m, const void *base, int n, long long outer, const PassPlan &pl) {
    std::memset(m, 0, sizeof(*m));
    if (!base) return;   // a map the kernel never uses (no such buffer in this launch)
    const TmaGeom &t = pl.tg;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], es[5];
    const uint64_t eb = 8;   // tensor elements: 8-byte words
    for (int j = 0; j < t.nd; ++j) {
        const int lo = t.shift[j], hi = j + 1 < t.nd ? t.shift[j + 1] : n;
        uint64_t d = (uint64_t(1) << (hi - lo)) * (j == 0 ? uint64_t(t.epa) : 1);
        if (j + 1 == t.nd) d *= uint64_t(outer);
        if (d > (uint64_t(1) << 32)) throw std::runtime_error("generated pass kernel: tensor dimension above 2^32");
        dims[j] = d;
        box[j] = (1u << pl.box_lg[j]) * (j == 0 ? unsigned(t.epa) : 1u);
        es[j] = 1;
        if (j > 0) strides[j - 1] = (uint64_t(1) << lo) * eb * uint64_t(t.epa);
    }
    const CUresult r = tensor_map_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, cuuint32_t(t.nd), const_cast<void *>(base),
                                            dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw std::runtime_error("generated pass kernel: cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
}

std::mutex g_err_mu;
int *g_err_word[64] = {nullptr};

cudaError_t launch_pipe(const void *kernel, void **argv, int threads, size_t smem, int sm_count, long long work,
                        cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const long long blocks = std::max<long long>(1, std::min<long long>((long long)sm_count * per_sm, work));
    e = cudaLaunchKernel(kernel, dim3(unsigned(blocks)), dim3(unsigned(threads)), argv, smem, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace

void tile_tma_plan(const std::vector<int> &qbits, int precision, TmaGeom *tg, int8_t *land) {
    const PassPlan pl = pass_plan(qbits, precision);
    *tg = pl.tg;
    for (size_t i = 0; i < pl.land.size(); ++i) land[i] = int8_t(pl.land[i]);
}

void tile_tma_map(void *map, const void *base, int n, long long outer, const std::vector<int> &qbits, int precision) {
    encode_map(static_cast<CUtensorMap *>(map), base, n, outer, pass_plan(qbits, precision));
}

int *jit_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) throw std::runtime_error("jit_error_word: no device");
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (!g_err_word[dev]) {
        int *w = nullptr;
        if (cudaMalloc(&w, sizeof(int)) != cudaSuccess || cudaMemset(w, 0, sizeof(int)) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess)
            throw std::runtime_error("jit_error_word: allocating the error word failed");
        g_err_word[dev] = w;
    }
    return g_err_word[dev];
}

template <typename V>
cudaError_t jit_launch_forward(const void *kernel, JitFwdArgs<V> a, const Pass &p, int precision, int sm_count,
                               cudaStream_t st) {
    const PassPlan pl = pass_plan(p.qbits, precision);
    const long long dim = 1ll << a.g.n;
    if (a.src && a.src_batch_stride != 0 && a.src_batch_stride != dim)
        throw std::runtime_error("generated forward pass: source batch stride must be 0 or the state size");
    a.tg = pl.tg;
    a.err = jit_error_word();
    CUtensorMap ms, md;
    encode_map(&ms, a.src, a.g.n, a.src_batch_stride ? a.batch : 1, pl);
    encode_map(&md, a.dst, a.g.n, a.batch, pl);
    void *argv[] = {&a, &ms, &md};
    return launch_pipe(kernel, argv, fwd_groups(p) * (1 << (p.K - p.f_reg_bits)), jit_forward_smem(p, precision), sm_count,
                       a.batch << a.g.n_out, st);
}

template <typename V>
cudaError_t jit_launch_backward(const void *kernel, JitBwdArgs<V> a, const Pass &p, int precision, int n_hams,
                                int sm_count, cudaStream_t st) {
    const PassPlan pl = pass_plan(p.qbits, precision);
    a.tg = pl.tg;
    a.err = jit_error_word();
    CUtensorMap mp, ml, md;
    encode_map(&mp, a.psi_src, a.g.n, a.batch, pl);
    encode_map(&ml, a.lam, a.g.n, a.batch * n_hams, pl);
    encode_map(&md, a.psi_dst, a.g.n, a.batch, pl);
    void *argv[] = {&a, &mp, &ml, &md};
    return launch_pipe(kernel, argv, bwd_groups(p) * (1 << (p.K - p.reg_bits)), jit_backward_smem(p, precision, n_hams),
                       sm_count,
                       a.batch << a.g.n_out, st);
}

template cudaError_t jit_launch_forward<float2>(const void *, JitFwdArgs<float2>, const Pass &, int, int, cudaStream_t);
template cudaError_t jit_launch_forward<double2>(const void *, JitFwdArgs<double2>, const Pass &, int, int, cudaStream_t);
template cudaError_t jit_launch_backward<float2>(const void *, JitBwdArgs<float2>, const Pass &, int, int, int,
                                                 cudaStream_t);
template cudaError_t jit_launch_backward<double2>(const void *, JitBwdArgs<double2>, const Pass &, int, int, int,
                                                  cudaStream_t);

}  // namespace mqb
