// extern "C" entry points of libmqb200: lowering of gate tables, pass execution, the
// checkpointed adjoint-gradient driver, Hamiltonian passes, reductions and sampling.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "jit.h"
#include "kernels.cuh"

namespace {

thread_local std::string g_last_error;

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Fail(code, buf);
}

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) fail(MQB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <typename F>
int guarded(F &&f) {
    try {
        f();
        return MQB_OK;
    } catch (const Fail &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return MQB_ERR_INVALID;
    }
}

int sm_count_cached() {
    static thread_local int dev = -1, count = 0;
    int d = 0;
    ck(cudaGetDevice(&d), "cudaGetDevice");
    if (d != dev) {
        ck(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, d), "cudaDeviceGetAttribute");
        dev = d;
    }
    return count;
}

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// State buffers are read and written as 16-byte vectors: refuse others before any device work.
void require_aligned(const void *ptr, const char *what) {
    if (ptr && (reinterpret_cast<uintptr_t>(ptr) & 15u)) fail(MQB_ERR_INVALID, "%s must be 16-byte aligned", what);
}

// The register arguments of the entry points that take a bare state: 1..40 qubits, a known precision.
void require_register(int n, int precision) {
    if (n < 1 || n > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40], got %d", n);
    if (precision != MQB_PREC_C64 && precision != MQB_PREC_C128) fail(MQB_ERR_INVALID, "bad precision %d", precision);
}

// Device allocations of the library (program and Hamiltonian tables): an out-of-memory error is
// MQB_ERR_ALLOC.  mqb_inject_alloc_failure arms a countdown on the calling thread: after that many
// successful allocations the next one fails as if the device were out of memory (host-side fault
// injection for tests; nothing reaches the device).
thread_local long long t_alloc_countdown = -1;

void dev_alloc(void **ptr, size_t bytes, const char *what) {
    if (t_alloc_countdown == 0) {
        t_alloc_countdown = -1;
        fail(MQB_ERR_ALLOC, "%s: out of device memory (%zu bytes; injected failure)", what, bytes);
    }
    const cudaError_t e = cudaMalloc(ptr, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(MQB_ERR_ALLOC, "%s: out of device memory (%zu bytes)", what, bytes);
    }
    ck(e, what);
    if (t_alloc_countdown > 0) --t_alloc_countdown;
}

template <typename T>
T *upload(const std::vector<T> &v) {
    if (v.empty()) return nullptr;
    T *d = nullptr;
    dev_alloc(reinterpret_cast<void **>(&d), sizeof(T) * v.size(), "cudaMalloc");
    ck(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    return d;
}

bool is_diag_gid(int gid) { return gid == GID_RZ || gid == GID_PS || gid == GID_GP || gid == GID_RZZ; }

// NVTX ranges: one per C-ABI call (named after it) and one around every kernel launch (named after
// its kind), so an NVTX-aware profiler shows each call's pass structure.  With no tool attached a
// range costs two calls through no-op function pointers.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// Optional per-launch timing: CUDA events around every kernel launch of the engine, recorded on the
// launching stream while enabled; mqb_timing_end synchronizes and reports the time per launch kind.
enum TimedKind { TK_FWD = 0, TK_BWD, TK_HAM, TK_MATGEN, TK_PLAIN_APPLY, TK_PLAIN_GRAD, TK_SCATTER, TK_OTHER, TK_ROWS, TK_COUNT };
const char *const kLaunchRange[TK_COUNT] = {"mqb forward pass",    "mqb adjoint pass",     "mqb hamiltonian pass",
                                            "mqb gate matrices",   "mqb per-gate apply",   "mqb per-gate gradient",
                                            "mqb gradient scatter", "mqb other launch",    "mqb row operations"};
struct TimedLaunch {
    int kind;
    cudaEvent_t a, b;
};
bool g_timing = false;
std::vector<TimedLaunch> g_timed;

struct TimeScope {
    Range range;
    TimedLaunch t{};
    cudaStream_t st;
    bool on;
    TimeScope(int kind, cudaStream_t s) : range(kLaunchRange[kind]), st(s), on(g_timing) {
        if (!on) return;
        t.kind = kind;
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        cudaEventRecord(t.a, st);
    }
    ~TimeScope() {
        if (!on) return;
        cudaEventRecord(t.b, st);
        g_timed.push_back(t);
    }
};

}  // namespace

using namespace mqb;

namespace mqb {
void set_last_error(const char *msg) { g_last_error = msg; }
}  // namespace mqb

struct mqb_hamiltonian {
    int n = 0, precision = 0;
    // Pauli terms, grouped for the register-binned kernel
    std::vector<HamGroup> groups;
    std::vector<HamClass> classes;
    HamClass *d_classes = nullptr;
    HamTerm *d_terms = nullptr;
    // or a sparse matrix (csr == true), as slices of 32 rows with column-major entries
    bool csr = false;
    int64_t nnz = 0, entries = 0;
    int64_t *d_slice_ptr = nullptr;
    int32_t *d_slice_len = nullptr;
    int32_t *d_cols = nullptr;
    void *d_vals = nullptr;
    ~mqb_hamiltonian() {
        cudaFree(d_classes);
        cudaFree(d_terms);
        cudaFree(d_slice_ptr);
        cudaFree(d_slice_len);
        cudaFree(d_cols);
        cudaFree(d_vals);
    }
};

struct SchedDev {
    Schedule s;
    JitMtab *d_jmt = nullptr, *d_f_jmt = nullptr;    // matrix-table sources of the generated kernels
    std::mutex jit_mu;
    std::vector<const void *> jit_fwd;                // generated forward kernel of every pass
    std::map<int, std::vector<const void *>> jit_bwd; // generated backward kernels, by lambdas
    ~SchedDev() {
        cudaFree(d_jmt);
        cudaFree(d_f_jmt);
        cudaFree(s.d_pass_ops);
        cudaFree(s.d_slot_map);
        cudaFree(s.d_stages);
        cudaFree(s.d_stage_ops);
        cudaFree(s.d_f_stages);
        cudaFree(s.d_f_stage_ops);
    }
};

struct mqb_program {
    int n = 0, precision = 0, n_params = 0, fuse = 1, tile_bits = 0, jit = 0;
    std::vector<DevOp> ops;
    std::vector<mqb_gate_desc> descs;
    DevOp *d_ops = nullptr;
    mqb_gate_desc *d_descs = nullptr;
    mqb_param_term *d_terms = nullptr;
    void *d_cpool = nullptr;
    int64_t per_sample = 0;    // complex entries per sample
    int64_t custom_entries = 0;
    int n_slots = 0;
    int32_t *d_csr_ptr = nullptr, *d_csr_slot = nullptr;
    double *d_csr_coeff = nullptr;
    std::vector<char> no_fuse;   // per op: MQB_GATE_NONUNITARY
    bool nonunitary = false;
    std::unique_ptr<SchedDev> apply_sched;
    std::map<int, std::unique_ptr<SchedDev>> grad_sched;   // by number of Hamiltonians
    ~mqb_program() {
        cudaFree(d_ops);
        cudaFree(d_descs);
        cudaFree(d_terms);
        cudaFree(d_cpool);
        cudaFree(d_csr_ptr);
        cudaFree(d_csr_slot);
        cudaFree(d_csr_coeff);
    }
    size_t elem() const { return precision == MQB_PREC_C64 ? 8 : 16; }
    // generated pass kernels pay their compile time back from 2^18 amplitudes on
    bool use_jit() const { return jit > 0 || (jit == 0 && n >= 18); }
};

// Calls that promise to allocate nothing (mqb_apply_static) run the precompiled kernels only.
static thread_local bool t_jit_blocked = false;
namespace mqb {
JitBlock::JitBlock() : prev_(t_jit_blocked) { t_jit_blocked = true; }
JitBlock::~JitBlock() { t_jit_blocked = prev_; }
}  // namespace mqb

static std::vector<JitMtab> jit_mtab(const std::vector<StageOp> &v) {
    std::vector<JitMtab> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = JitMtab{v[i].moff, v[i].mcount, (long long)v[i].msrc, v[i].msrc_ps, 0};
    return o;
}

static const std::vector<const void *> *jit_forward(const mqb_program &p, SchedDev &sd) {
    if (!p.use_jit() || t_jit_blocked || sd.s.passes.empty()) return nullptr;
    std::lock_guard<std::mutex> lk(sd.jit_mu);
    if (sd.jit_fwd.empty()) sd.jit_fwd = jit_forward_kernels(sd.s, p.precision);
    return &sd.jit_fwd;
}

static const std::vector<const void *> *jit_backward(const mqb_program &p, SchedDev &sd, int n_hams) {
    if (!p.use_jit() || t_jit_blocked || sd.s.passes.empty()) return nullptr;
    std::lock_guard<std::mutex> lk(sd.jit_mu);
    auto &v = sd.jit_bwd[n_hams];
    if (v.empty()) v = jit_backward_kernels(sd.s, p.precision, n_hams, p.ops);
    return &v;
}

static std::unique_ptr<SchedDev> make_sched(const mqb_program &p, int K, bool fuse, int reg_bits) {
    auto sd = std::make_unique<SchedDev>();
    // the register kernels need 2^5..2^8 threads of 2^reg_bits amplitudes: smaller registers use
    // the per-gate kernels
    if (K < reg_bits + 5) fuse = false;
    sd->s = build_schedule(p.n, K, contiguity_bits(p.precision), p.ops, fuse, &p.no_fuse);
    build_stages(sd->s, p.ops, reg_bits, p.precision, false);
    build_stages(sd->s, p.ops, fwd_reg_bits(p.precision), p.precision, true);
    sd->s.d_pass_ops = upload(sd->s.pass_ops);
    sd->s.d_slot_map = upload(sd->s.slot_map);
    sd->s.d_stages = upload(sd->s.stages);
    sd->s.d_stage_ops = upload(sd->s.stage_ops);
    sd->s.d_f_stages = upload(sd->s.f_stages);
    sd->s.d_f_stage_ops = upload(sd->s.f_stage_ops);
    sd->d_jmt = upload(jit_mtab(sd->s.stage_ops));
    sd->d_f_jmt = upload(jit_mtab(sd->s.f_stage_ops));
    return sd;
}

// Tile size of the fused kernels: 2^RB registers x 2^8 threads, capped by the register size.
static int tile_bits_for(const mqb_program &p, int reg_bits) {
    int K = reg_bits + 8;
    if (p.tile_bits > 0) K = std::min(K, std::max(reg_bits + 5, p.tile_bits));
    return std::min(K, p.n);
}

static SchedDev &grad_schedule(mqb_program &p, int n_hams) {
    const bool fused = p.fuse && n_hams <= 4;
    const int key = fused ? n_hams : 0;
    auto it = p.grad_sched.find(key);
    if (it != p.grad_sched.end()) return *it->second;
    const int rb = bwd_reg_bits(p.precision, n_hams);
    auto sd = make_sched(p, fused ? tile_bits_for(p, rb) : p.n, fused, rb);
    SchedDev &ref = *sd;
    p.grad_sched[key] = std::move(sd);
    return ref;
}

template <typename R>
static TileGeom pass_geom(int n, const Pass &ps) {
    return make_geom(n, ps.qbits);
}

// ---------------------------------------------------------------------------------------------- execution
template <typename R>
static bool run_forward_pass(const mqb_program &p, const SchedDev &sd, size_t pi, const void *jk,
                             const cplx<R> *mats, const cplx<R> *src, int64_t src_stride, cplx<R> *dst, int64_t batch,
                             cudaStream_t st, double *norm = nullptr) {
    // returns whether the pass also added <psi|psi> of its output to norm[b][0] (generated passes)
    const Schedule &s = sd.s;
    const Pass &ps = s.passes[pi];
    const int sm = sm_count_cached();
    const cplx<R> *cpool = static_cast<const cplx<R> *>(p.d_cpool);
    if (ps.fused && jk) {
        JitFwdArgs<cplx<R>> a{};
        a.g = make_geom(p.n, ps.qbits);
        a.mt = sd.d_f_jmt + ps.f_sop_begin;
        a.n_mt = ps.f_n_sops;
        a.mtab_entries = ps.f_mtab_entries;
        a.mats = mats;
        a.mats_stride = p.per_sample;
        a.cpool = cpool;
        a.src = src;
        a.dst = dst;
        a.batch = batch;
        a.src_batch_stride = src_stride;
        a.norm = norm;
        TimeScope ts(TK_FWD, st);
        ck(jit_launch_forward<cplx<R>>(jk, a, ps, p.precision, sm, st), "generated forward pass");
        return norm != nullptr;
    }
    if (ps.fused) {
        Fwd2Args<R> a{};
        a.g = make_geom(p.n, ps.qbits);
        a.stages = s.d_f_stages + ps.f_stage_begin;
        a.n_stages = ps.f_n_stages;
        a.sops = s.d_f_stage_ops + ps.f_sop_begin;
        a.n_ops = ps.f_n_sops;
        a.reg_bits = ps.f_reg_bits;
        a.mtab_entries = ps.f_mtab_entries;
        a.mats = mats;
        a.mats_stride = p.per_sample;
        a.cpool = cpool;
        a.src = src;
        a.dst = dst;
        a.batch = batch;
        a.src_batch_stride = src_stride;
        TimeScope ts(TK_FWD, st);
        ck(launch_fused_fwd2<R>(a, sm, st), "fused forward pass");
        return false;
    }
    if (src != dst) {
        TimeScope ts(TK_OTHER, st);
        ck(launch_copy_or_zero<R>(dst, src, p.n, batch, src_stride, st), "state copy");
    }
    TimeScope ts(TK_PLAIN_APPLY, st);
    ck(launch_plain_apply<R>(dst, p.n, batch, p.ops[ps.op_begin], mats, p.per_sample, cpool, false, sm, st),
       "gate kernel");
    return false;
}

template <typename R>
static void run_matgen(const mqb_program &p, const double *params, int64_t param_stride, const double *custom,
                       int64_t batch, cplx<R> *mats, cudaStream_t st) {
    if (p.per_sample == 0) return;
    MatgenArgs m{};
    m.ops = p.d_ops;
    m.descs = p.d_descs;
    m.terms = p.d_terms;
    m.n_ops = int(p.ops.size());
    m.params = params;
    m.param_stride = param_stride;
    m.custom = custom;
    m.custom_stride = p.custom_entries;
    m.batch = batch;
    m.mats = mats;
    m.mats_stride = p.per_sample;
    TimeScope ts(TK_MATGEN, st);
    ck(launch_matgen<R>(m, st), "matgen");
}

template <typename R>
static void apply_impl(mqb_program &p, void *states, int64_t batch, const double *params, int64_t param_stride,
                       const double *custom, void *ws, size_t ws_bytes, cudaStream_t st) {
    const size_t need = align_up(size_t(batch) * p.per_sample * sizeof(cplx<R>));
    if (p.per_sample && (ws == nullptr || ws_bytes < need)) fail(MQB_ERR_WORKSPACE, "workspace too small");
    cplx<R> *mats = static_cast<cplx<R> *>(ws);
    run_matgen<R>(p, params, param_stride, custom, batch, mats, st);
    cplx<R> *s = static_cast<cplx<R> *>(states);
    SchedDev &sd = *p.apply_sched;
    const auto *jk = jit_forward(p, sd);
    for (size_t i = 0; i < sd.s.passes.size(); ++i)
        run_forward_pass<R>(p, sd, i, jk ? (*jk)[i] : nullptr, mats, s, int64_t(1) << p.n, s, batch, st);
}

// Hamiltonian passes: out = H ket (if out), f += <bra|H ket> (if fout)
// Whether a Hamiltonian group runs as the TMA-ring pass (MQB_HAM_RING=0 keeps the synchronous
// one): 2^(K-4) threads of at least one warp and at most 256, 16-byte-aligned buffers, and at
// least two buffers per operand in shared memory.  Sets rg.nb.
template <typename R>
static bool ham_ring_fits(const HamArgs<R> &a, HamRingGeom &rg) {
    static const bool on = [] {
        const char *e = std::getenv("MQB_HAM_RING");
        return !(e && e[0] == '0');
    }();
    static const int stage = [] {   // MQB_HAM_RING_STAGE=0: read the previous sum instead of staging it
        const char *e = std::getenv("MQB_HAM_RING_STAGE");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    const int threads = 1 << std::max(0, a.g.K - kHamRegBits);
    if (!on || a.g.K < 5 + kHamRegBits || threads > 256 || a.g.qbits[0] != 0) return false;
    if ((reinterpret_cast<uintptr_t>(a.ket) & 15) || (reinterpret_cast<uintptr_t>(a.out) & 15)) return false;
    rg.stage_prev = stage;
    const bool staged = a.accumulate && a.out && stage;
    // MQB_HAM_RING_BUFFERS: buffers per operand (2..4, tuning).  Two by default: the 26-qubit
    // ZZ + X pass took 22.0 ms with two, 22.7 with three (an unstaged group then fits three blocks
    // per SM instead of two)
    static const int nb_max = [] {
        const char *e = std::getenv("MQB_HAM_RING_BUFFERS");
        return e ? std::max(2, std::min(4, std::atoi(e))) : 2;
    }();
    for (int nb = nb_max; nb >= 2; --nb) {
        if (ham_ring_smem(a.g, int(sizeof(cplx<R>)), threads, a.n_classes, a.n_terms, staged, nb) <= 220 * 1024) {
            rg.nb = nb;
            return true;
        }
    }
    return false;
}

template <typename R>
static void ham_impl(const mqb_hamiltonian &h, const cplx<R> *bra, const cplx<R> *ket, cplx<R> *out, double *fout,
                     int64_t f_stride, int64_t batch, cudaStream_t st) {
    const int sm = sm_count_cached();
    const int64_t dim = int64_t(1) << h.n;
    if (h.csr) {
        CsrArgs<R> a{};
        a.slice_ptr = h.d_slice_ptr;
        a.slice_len = h.d_slice_len;
        a.cols = h.d_cols;
        a.vals = static_cast<const cplx<R> *>(h.d_vals);
        a.dim = dim;
        a.bra = bra;
        a.ket = ket;
        a.out = out;
        a.fout = fout;
        a.f_stride = f_stride;
        a.batch = batch;
        TimeScope ts(TK_HAM, st);
        ck(launch_csr<R>(a, sm, st), "sparse hamiltonian");
        return;
    }
    if (h.groups.empty()) {
        // zero Hamiltonian
        if (out) ck(cudaMemsetAsync(out, 0, sizeof(cplx<R>) * dim * batch, st), "memset");
        return;
    }
    for (size_t gi = 0; gi < h.groups.size(); ++gi) {
        const HamGroup &g = h.groups[gi];
        HamArgs<R> a{};
        a.g = g.geom;
        a.classes = h.d_classes + g.class_begin;
        a.n_classes = g.class_count;
        a.term_begin = h.classes[g.class_begin].term_begin;
        a.n_terms = h.classes[g.class_begin + g.class_count - 1].term_begin +
                    h.classes[g.class_begin + g.class_count - 1].term_count - a.term_begin;
        a.terms = h.d_terms;
        a.ket = ket;
        a.bra = bra;
        a.out = out;
        a.accumulate = gi > 0;
        a.fout = fout;
        a.batch = batch;
        a.out_batch_stride = dim;
        a.f_stride = f_stride;
        TimeScope ts(TK_HAM, st);
        HamRingGeom rg{};
        if (ham_ring_fits(a, rg)) {
            std::vector<int> qb(g.geom.qbits, g.geom.qbits + g.geom.K);
            alignas(64) unsigned char mk[128], mo[128];
            tile_tma_plan(qb, h.precision, &rg.tg, rg.land);
            tile_tma_map(mk, ket, h.n, batch, qb, h.precision);
            tile_tma_map(mo, a.accumulate && out && rg.stage_prev ? out : nullptr, h.n, batch, qb, h.precision);
            rg.err = jit_error_word();
            ck(launch_ham_ring<R>(a, rg, mk, mo, sm, st), "hamiltonian pass");
        } else {
            ck(launch_ham<R>(a, sm, st), "hamiltonian pass");
        }
    }
}

struct GradLayout {
    size_t mats = 0, gslots = 0, lam = 0, w = 0, ckpt = 0, norms = 0, total = 0;
    int n_ckpt = 0;
    bool need_w = false;
    std::vector<int> ckpt_index;   // p (1..P) -> checkpoint buffer index or -1
    // FP64 norm checks of the complex64 state: the states after these forward passes, and the
    // states before these passes that the backward rebuilds by reverse application
    std::vector<int> norm_fwd, norm_bwd;
};

static GradLayout grad_layout(const mqb_program &p, const Schedule &s, int64_t batch, int n_hams, int stride) {
    GradLayout L;
    const int P = int(s.passes.size());
    const size_t state = (size_t(1) << p.n) * p.elem() * batch;
    L.ckpt_index.assign(P + 1, -1);
    for (int q = 1; q <= P; ++q) {
        const bool stored = (q == P) || (stride > 0 && q % stride == 0);
        if (stored) L.ckpt_index[q] = L.n_ckpt++;
        else L.need_w = true;
    }
    for (const Pass &ps : s.passes)
        if (!ps.fused) L.need_w = true;
    if (P == 0) L.need_w = true;
    if (p.precision == MQB_PREC_C64 && P > 0) {
        // every ceil(sqrt(P)) passes (and the last state of the forward sweep)
        const int sn = std::max(1, int(std::ceil(std::sqrt(double(P)))));
        for (int q = 1; q <= P; ++q)
            if (q % sn == 0 || q == P) L.norm_fwd.push_back(q);
        for (int q = P - 1; q >= 1; --q)
            if (L.ckpt_index[q] < 0 && q % sn == 0) L.norm_bwd.push_back(q);
    }
    L.mats = align_up(size_t(batch) * p.per_sample * p.elem());
    L.gslots = align_up(size_t(batch) * std::max(1, p.n_slots) * n_hams * sizeof(double));
    L.lam = align_up(state * n_hams);
    L.w = L.need_w ? align_up(state) : 0;
    L.ckpt = align_up(state) * L.n_ckpt;
    L.norms = align_up((L.norm_fwd.size() + L.norm_bwd.size()) * size_t(batch) * 2 * sizeof(double));
    L.total = L.mats + L.gslots + L.lam + L.w + L.ckpt + L.norms;
    return L;
}

// Adjoint gradient.  With Hamiltonians: lambda_h = H_h psi, f_h = <psi|H_h|psi> and
// grad = 2 Re sum <lambda|dU|psi> (GradRealDouble).  With lam_in instead (n_hams = 1, hams and f
// unused): lambda starts from the caller's state and grad = Re sum <lambda|dU|psi> (scale 1).
template <typename R>
static void grad_impl(mqb_program &p, const mqb_hamiltonian *const *hams, int n_hams, const void *init,
                      int init_batched, int64_t batch, const double *params, int64_t param_stride, const double *custom,
                      double *f, double *grad, int stride, void *ws, size_t ws_bytes, cudaStream_t st,
                      const void *lam_in = nullptr, int lam_batched = 0) {
    using V = cplx<R>;
    if (p.nonunitary && stride != 1)
        fail(MQB_ERR_INVALID, "programs with non-unitary operators need checkpoint stride 1 (every pass stored), got %d",
             stride);
    SchedDev &sd = grad_schedule(p, n_hams);
    const Schedule &s = sd.s;
    const GradLayout L = grad_layout(p, s, batch, n_hams, stride);
    if (ws == nullptr || ws_bytes < L.total) fail(MQB_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, L.total);
    unsigned char *base = static_cast<unsigned char *>(ws);
    V *mats = reinterpret_cast<V *>(base);
    double *gslots = reinterpret_cast<double *>(base + L.mats);
    V *lam = reinterpret_cast<V *>(base + L.mats + L.gslots);
    V *W = L.need_w ? reinterpret_cast<V *>(base + L.mats + L.gslots + L.lam) : nullptr;
    unsigned char *ck0 = base + L.mats + L.gslots + L.lam + L.w;
    const int64_t dim = int64_t(1) << p.n;
    const size_t state_bytes = align_up(size_t(dim) * batch * sizeof(V));
    auto ckpt = [&](int q) -> V * { return reinterpret_cast<V *>(ck0 + state_bytes * L.ckpt_index[q]); };
    auto loc = [&](int q) -> V * { return L.ckpt_index[q] >= 0 ? ckpt(q) : W; };
    const int P = int(s.passes.size());
    const int sm = sm_count_cached();
    const V *cpool = static_cast<const V *>(p.d_cpool);

    ck(cudaMemsetAsync(gslots, 0, L.gslots, st), "memset");
    if (f) ck(cudaMemsetAsync(f, 0, sizeof(double) * 2 * n_hams * batch, st), "memset");
    // norm checks: <psi|psi> in FP64 per sample, [check][batch][re, im]
    double *norms = reinterpret_cast<double *>(ck0 + L.ckpt);
    if (L.norms) ck(cudaMemsetAsync(norms, 0, L.norms, st), "memset");
    size_t n_checked = 0;
    auto norm_check = [&](const V *state) {
        TimeScope ts(TK_OTHER, st);
        ck(launch_vdot<R>(state, state, p.n, batch, norms + 2 * batch * n_checked, sm, st), "norm check");
        ++n_checked;
    };
    size_t next_fwd = 0, next_bwd = 0;
    run_matgen<R>(p, params, param_stride, custom, batch, mats, st);

    // forward: psi_{q+1} = pass_q(psi_q), psi_0 = init (or |0...0>)
    const V *init_v = static_cast<const V *>(init);
    const int64_t init_stride = init_batched ? dim : 0;
    const auto *jf = jit_forward(p, sd);
    const auto *jb = jit_backward(p, sd, n_hams);
    for (int q = 0; q < P; ++q) {
        const V *src = (q == 0) ? init_v : loc(q);
        const int64_t sstr = (q == 0) ? init_stride : dim;
        const bool check = next_fwd < L.norm_fwd.size() && L.norm_fwd[next_fwd] == q + 1;
        // a generated pass adds the norm of its output itself; other passes get a separate reduction
        if (run_forward_pass<R>(p, sd, q, jf ? (*jf)[q] : nullptr, mats, src, sstr, loc(q + 1), batch, st,
                                check ? norms + 2 * batch * n_checked : nullptr))
            ++n_checked;
        else if (check)
            norm_check(loc(q + 1));
        if (check) ++next_fwd;
    }
    V *psiP = W;
    if (P > 0) {
        psiP = loc(P);
    } else {
        ck(launch_copy_or_zero<R>(W, init_v, p.n, batch, init_stride, st), "state copy");
    }
    // lambda_h = H_h psi_P ; f_h = <psi_P|lambda_h>   (or lambda from the caller)
    if (lam_in) {
        TimeScope ts(TK_OTHER, st);
        ck(launch_copy_or_zero<R>(lam, static_cast<const V *>(lam_in), p.n, batch, lam_batched ? dim : 0, st),
           "lambda copy");
    } else {
        for (int h = 0; h < n_hams; ++h)
            ham_impl<R>(*hams[h], psiP, psiP, lam + h * batch * dim, f + 2 * h, 2 * n_hams, batch, st);
    }
    // backward
    for (int q = P - 1; q >= 0; --q) {
        const Pass &ps = s.passes[q];
        const bool stored_q = L.ckpt_index[q] >= 0;
        if (ps.fused && jb && (*jb)[q]) {
            JitBwdArgs<V> a{};
            a.g = make_geom(p.n, ps.qbits);
            a.mt = sd.d_jmt + ps.sop_begin;
            a.n_mt = ps.n_sops;
            a.mtab_entries = ps.mtab_entries;
            a.mats = mats;
            a.mats_stride = p.per_sample;
            a.cpool = cpool;
            a.psi_src = loc(q + 1);
            a.psi_dst = (q > 0 && !stored_q) ? W : nullptr;
            a.lam = lam;
            a.gslots = gslots;
            a.slot_map = s.d_slot_map + ps.slot_begin;
            a.n_slots = std::max(1, p.n_slots);
            a.n_hams = n_hams;
            a.n_local_slots = ps.n_slots;
            a.batch = batch;
            TimeScope ts(TK_BWD, st);
            ck(jit_launch_backward<V>((*jb)[q], a, ps, p.precision, n_hams, sm, st), "generated backward pass");
        } else if (ps.fused) {
            Bwd2Args<R> a{};
            a.g = make_geom(p.n, ps.qbits);
            a.stages = s.d_stages + ps.stage_begin;
            a.n_stages = ps.n_stages;
            a.sops = s.d_stage_ops + ps.sop_begin;
            a.n_ops = ps.n_sops;
            a.reg_bits = ps.reg_bits;
            a.mtab_entries = ps.mtab_entries;
            a.mats = mats;
            a.mats_stride = p.per_sample;
            a.cpool = cpool;
            a.psi_src = loc(q + 1);
            a.psi_dst = (q > 0 && !stored_q) ? W : nullptr;
            a.lam = lam;
            a.n_hams = n_hams;
            a.gslots = gslots;
            a.n_slots = std::max(1, p.n_slots);
            a.slot_map = s.d_slot_map + ps.slot_begin;
            a.n_local_slots = ps.n_slots;
            a.batch = batch;
            TimeScope ts(TK_BWD, st);
            ck(launch_fused_bwd2<R>(a, sm, st), "fused backward pass");
        } else {
            const DevOp &op = p.ops[ps.op_begin];
            V *psi_q;
            if (q > 0 && stored_q) {
                psi_q = ckpt(q);
            } else if (q == 0) {
                // the initial state itself (applying the op in reverse would not undo a non-unitary op)
                TimeScope ts(TK_OTHER, st);
                ck(launch_copy_or_zero<R>(W, init_v, p.n, batch, init_stride, st), "state copy");
                psi_q = W;
            } else {
                V *src = loc(q + 1);
                if (src != W) {
                    TimeScope ts(TK_OTHER, st);
                    ck(launch_copy_or_zero<R>(W, src, p.n, batch, dim, st), "state copy");
                }
                TimeScope ts(TK_PLAIN_APPLY, st);
                ck(launch_plain_apply<R>(W, p.n, batch, op, mats, p.per_sample, cpool, true, sm, st), "gate kernel");
                psi_q = W;
            }
            {
                TimeScope ts(TK_PLAIN_GRAD, st);
                ck(launch_plain_grad<R>(psi_q, lam, p.n, batch, n_hams, op, mats, p.per_sample, gslots,
                                        std::max(1, p.n_slots), sm, st),
                   "gradient kernel");
            }
            for (int h = 0; h < n_hams; ++h) {
                TimeScope ts(TK_PLAIN_APPLY, st);
                ck(launch_plain_apply<R>(lam + h * batch * dim, p.n, batch, op, mats, p.per_sample, cpool, true, sm, st),
                   "gate kernel");
            }
        }
        if (next_bwd < L.norm_bwd.size() && L.norm_bwd[next_bwd] == q) {
            norm_check(W);   // psi before pass q, rebuilt by reverse application
            ++next_bwd;
        }
    }
    TimeScope ts(TK_SCATTER, st);
    ck(launch_grad_scatter(gslots, batch, std::max(1, p.n_slots), n_hams, p.d_csr_ptr, p.d_csr_slot, p.d_csr_coeff,
                           p.n_params, lam_in ? 1.0 : 2.0, grad, st),
       "gradient scatter");
}


// Validate one gate record and derive its execution kind, targets and matrix size (no CUDA).
static DevOp basic_op(const mqb_gate_desc &d, int k, int n_qubits, const mqb_param_term *terms, int n_terms,
                      int n_params, const double *const_matrices, int64_t n_const_entries) {
    DevOp op{};
    op.gate_id = d.gate_id;
    op.m = d.n_obj;
    const uint64_t allq = (uint64_t(1) << n_qubits) - 1;
    if (d.gate_id < 0 || d.gate_id >= GID_COUNT) fail(MQB_ERR_INVALID, "gate %d: unknown gate id %d", k, d.gate_id);
    if (d.gate_id != GID_RPS && (d.n_obj < 1 || d.n_obj > MQB_MAX_OBJ))
        fail(MQB_ERR_INVALID, "gate %d: %d object qubits (max %d)", k, d.n_obj, MQB_MAX_OBJ);
    uint64_t objm = 0;
    for (int i = 0; i < d.n_obj && i < MQB_MAX_OBJ; ++i) {
        if (d.obj[i] < 0 || d.obj[i] >= n_qubits) fail(MQB_ERR_INVALID, "gate %d: qubit %d out of range", k, d.obj[i]);
        if (objm >> d.obj[i] & 1) fail(MQB_ERR_INVALID, "gate %d: repeated object qubit %d", k, d.obj[i]);
        objm |= uint64_t(1) << d.obj[i];
        op.tq[i] = d.obj[i];
    }
    if (d.ctrl_mask & ~allq) fail(MQB_ERR_INVALID, "gate %d: control qubit out of range", k);
    if (d.ctrl_mask & objm) fail(MQB_ERR_INVALID, "gate %d: control and object qubits overlap", k);
    op.ctrl = d.ctrl_mask;
    if (d.n_angles < 0 || d.n_angles > MQB_MAX_ANGLES) fail(MQB_ERR_INVALID, "gate %d: bad angle count", k);
    op.n_angles = d.n_angles;
    op.grad_mask = d.grad_angles & ((1 << d.n_angles) - 1);
    if (terms) {
        for (int a = 0; a < d.n_angles; ++a) {
            if (d.term_begin[a] < 0 || d.term_count[a] < 0 || d.term_begin[a] + d.term_count[a] > n_terms)
                fail(MQB_ERR_INVALID, "gate %d: bad parameter term range", k);
            for (int t = d.term_begin[a]; t < d.term_begin[a] + d.term_count[a]; ++t)
                if (terms[t].param < 0 || terms[t].param >= n_params)
                    fail(MQB_ERR_INVALID, "gate %d: parameter index %d out of range", k, terms[t].param);
        }
    }
    if (d.gate_id == GID_MATRIX) {
        const int dimm = 1 << d.n_obj;
        if (!const_matrices || d.matrix_offset < 0 || d.matrix_offset + int64_t(dimm) * dimm > n_const_entries)
            fail(MQB_ERR_INVALID, "gate %d: constant matrix out of range", k);
        const double *m = const_matrices + 2 * d.matrix_offset;
        bool diag = true;
        for (int r = 0; r < dimm && diag; ++r)
            for (int c = 0; c < dimm; ++c)
                if (r != c && (m[2 * (r * dimm + c)] != 0 || m[2 * (r * dimm + c) + 1] != 0)) {
                    diag = false;
                    break;
                }
        op.per_sample = 0;
        op.n_angles = 0;
        op.grad_mask = 0;
        op.kind = diag ? KIND_DIAG : KIND_DENSE;
        op.mat_size = diag ? dimm : dimm * dimm;
        op.sub = SUB_GENERIC;
        if (!diag && dimm == 2) {
            bool real = true;
            for (int e = 0; e < 4; ++e) real = real && m[2 * e + 1] == 0;
            const bool anti = m[0] == 0 && m[1] == 0 && m[6] == 0 && m[7] == 0;
            if (anti && m[2] == 1 && m[3] == 0 && m[4] == 1 && m[5] == 0)
                op.sub = SUB_SWAP;
            else if (anti)
                op.sub = SUB_PERM;
            else if (real)
                op.sub = SUB_REAL;
        }
        return op;
    }
    if (d.gate_id == GID_RPS) {
        op.kind = KIND_RPS;
        op.mat_size = 1;
        op.px = d.pauli_x;
        op.py = d.pauli_y;
        op.pz = d.pauli_z;
        op.pny = d.pauli_ny;
        op.m = 0;
        if ((d.pauli_x | d.pauli_y | d.pauli_z) & ~allq) fail(MQB_ERR_INVALID, "gate %d: Pauli mask out of range", k);
        if ((d.pauli_x | d.pauli_y | d.pauli_z) & d.ctrl_mask)
            fail(MQB_ERR_INVALID, "gate %d: control and object qubits overlap", k);
        return op;
    }
    if (is_diag_gid(d.gate_id)) {
        op.kind = KIND_DIAG;
        op.mat_size = 1 << d.n_obj;
    } else {
        op.kind = KIND_DENSE;
        op.mat_size = 1 << (2 * d.n_obj);
        if (d.gate_id == GID_RY) op.sub = SUB_REAL;   // RY and its derivative are real matrices
        if (d.gate_id == GID_RX) op.sub = SUB_RXL;    // RX: real diagonal, imaginary off-diagonal
    }
    const int expect_obj =
        (d.gate_id == GID_RZZ || (d.gate_id >= GID_RXX && d.gate_id <= GID_SWAPALPHA) || d.gate_id == GID_FSIM) ? 2 : 1;
    if (d.gate_id != GID_CUSTOM && d.n_obj != expect_obj)
        fail(MQB_ERR_INVALID, "gate %d: gate id %d acts on %d qubits, got %d", k, d.gate_id, expect_obj, d.n_obj);
    return op;
}

// ---------------------------------------------------------------------------------------------- C ABI
extern "C" {

const char *mqb_last_error(void) { return g_last_error.c_str(); }

int mqb_version(void) { return 100; }

int mqb_inject_alloc_failure(int after) {
    t_alloc_countdown = after < 0 ? -1 : after;
    return MQB_OK;
}

int mqb_device_error(int *code, int clear) {
    return guarded([&] {
        if (!code) fail(MQB_ERR_INVALID, "mqb_device_error: null output");
        int *w = jit_error_word();
        ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        ck(cudaMemcpy(code, w, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
        if (clear) ck(cudaMemset(w, 0, sizeof(int)), "cudaMemset");
        ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    });
}

int mqb_timing_begin(void) {
    return guarded([&] {
        for (auto &t : g_timed) {
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        g_timed.clear();
        g_timing = true;
    });
}

int mqb_timing_end(double *ms, int64_t *launches, int n_kinds) {
    return guarded([&] {
        g_timing = false;
        for (int k = 0; k < n_kinds; ++k) {
            ms[k] = 0;
            launches[k] = 0;
        }
        for (auto &t : g_timed) {
            ck(cudaEventSynchronize(t.b), "cudaEventSynchronize");
            float e = 0;
            ck(cudaEventElapsedTime(&e, t.a, t.b), "cudaEventElapsedTime");
            if (t.kind < n_kinds) {
                ms[t.kind] += e;
                launches[t.kind] += 1;
            }
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        g_timed.clear();
    });
}

int mqb_device_sm_count(int *out) {
    return guarded([&] { *out = sm_count_cached(); });
}

int mqb_abi_struct_sizes(int64_t *out, int n) {
    return guarded([&] {
        const int64_t v[4] = {int64_t(sizeof(mqb_gate_desc)), int64_t(sizeof(mqb_param_term)),
                              int64_t(sizeof(mqb_program_options)), int64_t(sizeof(mqb_program_info))};
        for (int i = 0; i < n && i < 4; ++i) out[i] = v[i];
    });
}

int mqb_program_create(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates, const mqb_param_term *terms,
                       int n_terms, int n_params, const double *const_matrices, int64_t n_const_entries,
                       const mqb_program_options *options, mqb_program **out) {
    return guarded([&] {
        Range range("mqb_program_create");
        if (!out) fail(MQB_ERR_INVALID, "out is null");
        *out = nullptr;
        if (n_qubits < 1 || n_qubits > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40], got %d", n_qubits);
        if (precision != MQB_PREC_C64 && precision != MQB_PREC_C128) fail(MQB_ERR_INVALID, "bad precision %d", precision);
        if (n_gates < 0 || (n_gates > 0 && !gates)) fail(MQB_ERR_INVALID, "bad gate table");
        auto p = std::make_unique<mqb_program>();
        p->n = n_qubits;
        p->precision = precision;
        p->n_params = n_params;
        p->fuse = options ? options->fuse : 1;
        p->tile_bits = options ? options->tile_bits : 0;
        p->jit = options ? options->jit : 0;
        p->descs.assign(gates, gates + n_gates);
        p->no_fuse.assign(size_t(n_gates), 0);
        for (int k = 0; k < n_gates; ++k)
            if (gates[k].flags & MQB_GATE_NONUNITARY) {
                if (gates[k].gate_id != GID_MATRIX) fail(MQB_ERR_INVALID, "gate %d: only constant matrices can be non-unitary", k);
                p->no_fuse[size_t(k)] = 1;
                p->nonunitary = true;
            }
        std::vector<std::complex<double>> pool;
        std::vector<std::vector<std::pair<int32_t, double>>> csr(std::max(0, n_params));
        int64_t cursor = 0;
        int slots = 0;
        for (int k = 0; k < n_gates; ++k) {
            const mqb_gate_desc &d = gates[k];
            DevOp op = basic_op(d, k, n_qubits, terms, n_terms, n_params, const_matrices, n_const_entries);
            if (d.gate_id == GID_MATRIX) {
                const int dimm = 1 << d.n_obj;
                const double *m = const_matrices + 2 * d.matrix_offset;
                op.mat_off = int64_t(pool.size());
                if (op.kind == KIND_DIAG) {
                    for (int r = 0; r < dimm; ++r) pool.emplace_back(m[2 * (r * dimm + r)], m[2 * (r * dimm + r) + 1]);
                } else {
                    for (int e = 0; e < dimm * dimm; ++e) pool.emplace_back(m[2 * e], m[2 * e + 1]);
                }
            } else {
                op.per_sample = 1;
                op.mat_off = cursor;
                cursor += op.mat_size;
                if (op.grad_mask) {
                    op.dmat_off = int32_t(cursor);
                    cursor += int64_t(op.mat_size) * op.n_angles;
                }
                if (d.gate_id == GID_CUSTOM) {
                    op.custom_off = int32_t(d.matrix_offset);
                    p->custom_entries = std::max<int64_t>(p->custom_entries, d.matrix_offset + 2 * op.mat_size);
                }
            }
            if (op.grad_mask) {
                op.slot0 = slots;
                int r = 0;
                for (int a = 0; a < op.n_angles; ++a) {
                    if (!(op.grad_mask >> a & 1)) continue;
                    for (int t = d.term_begin[a]; t < d.term_begin[a] + d.term_count[a]; ++t)
                        if (terms[t].flags & 1) csr[terms[t].param].emplace_back(slots + r, terms[t].coeff);
                    ++r;
                }
                slots += r;
            }
            p->ops.push_back(op);
        }
        p->per_sample = cursor;
        p->n_slots = slots;
        p->d_ops = upload(p->ops);
        p->d_descs = upload(p->descs);
        p->d_terms = upload(std::vector<mqb_param_term>(terms, terms + n_terms));
        if (!pool.empty()) {
            if (precision == MQB_PREC_C64) {
                std::vector<float2> v;
                for (auto &c : pool) v.push_back(make_float2(float(c.real()), float(c.imag())));
                p->d_cpool = upload(v);
            } else {
                std::vector<double2> v;
                for (auto &c : pool) v.push_back(make_double2(c.real(), c.imag()));
                p->d_cpool = upload(v);
            }
        }
        std::vector<int32_t> ptr(std::max(0, n_params) + 1, 0), slot;
        std::vector<double> coeff;
        for (int q = 0; q < n_params; ++q) {
            for (auto &e : csr[q]) {
                slot.push_back(e.first);
                coeff.push_back(e.second);
            }
            ptr[q + 1] = int32_t(slot.size());
        }
        p->d_csr_ptr = upload(ptr);
        p->d_csr_slot = upload(slot);
        p->d_csr_coeff = upload(coeff);
        const int rb = fwd_reg_bits(precision);
        p->apply_sched = make_sched(*p, tile_bits_for(*p, rb), p->fuse != 0, rb);
        *out = p.release();
    });
}

int mqb_plan_schedule(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates, const double *const_matrices,
                      int64_t n_const_entries, int tile_bits, int fuse, int *n_passes, int32_t *order, int32_t *pass_of,
                      uint64_t *qmask, int32_t *fused, int32_t *n_stages) {
    return guarded([&] {
        if (n_qubits < 1 || n_qubits > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40]");
        std::vector<DevOp> ops;
        for (int k = 0; k < n_gates; ++k)
            ops.push_back(basic_op(gates[k], k, n_qubits, nullptr, 0, 0, const_matrices, n_const_entries));
        const int rb = fwd_reg_bits(precision);
        int K = std::min(n_qubits, rb + 8);
        if (tile_bits > 0) K = std::min(n_qubits, std::max(rb + 5, tile_bits));
        Schedule s = build_schedule(n_qubits, K, contiguity_bits(precision), ops, fuse != 0 && K >= rb + 5);
        build_stages(s, ops, rb, precision, true);
        int pos = 0;
        for (size_t pi = 0; pi < s.passes.size(); ++pi) {
            const Pass &ps = s.passes[pi];
            uint64_t qm = 0;
            for (int q : ps.qbits) qm |= uint64_t(1) << q;
            qmask[pi] = qm;
            fused[pi] = ps.fused;
            if (n_stages) n_stages[pi] = ps.f_n_stages;
            if (ps.fused) {
                for (int i = ps.op_begin; i < ps.op_end; ++i) {
                    order[pos] = s.pass_ops[i].op;
                    pass_of[pos++] = int32_t(pi);
                }
            } else {
                order[pos] = ps.op_begin;
                pass_of[pos++] = int32_t(pi);
            }
        }
        *n_passes = int(s.passes.size());
    });
}

int mqb_jit_check(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates, const double *const_matrices,
                  int64_t n_const_entries, int tile_bits, int n_hams, int *n_kernels) {
    return guarded([&] {
        if (n_qubits < 1 || n_qubits > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40]");
        if (precision != MQB_PREC_C64 && precision != MQB_PREC_C128) fail(MQB_ERR_INVALID, "unknown precision");
        if (n_hams < 0 || n_hams > 4 || !n_kernels) fail(MQB_ERR_INVALID, "invalid argument");
        std::vector<DevOp> ops;
        int slots = 0;
        for (int k = 0; k < n_gates; ++k) {
            DevOp op = basic_op(gates[k], k, n_qubits, nullptr, 0, 0, const_matrices, n_const_entries);
            if (op.grad_mask) {
                op.slot0 = slots;
                for (int a = 0; a < op.n_angles; ++a) slots += (op.grad_mask >> a) & 1;
            }
            ops.push_back(op);
        }
        const int rb = n_hams ? bwd_reg_bits(precision, n_hams) : fwd_reg_bits(precision);
        int K = std::min(n_qubits, rb + 8);
        if (tile_bits > 0) K = std::min(n_qubits, std::max(rb + 5, tile_bits));
        Schedule s = build_schedule(n_qubits, K, contiguity_bits(precision), ops, K >= rb + 5);
        build_stages(s, ops, rb, precision, false);
        build_stages(s, ops, fwd_reg_bits(precision), precision, true);
        *n_kernels = jit_compile_check(s, precision, n_hams, ops);
    });
}

int mqb_program_destroy(mqb_program *prog) {
    return guarded([&] { delete prog; });
}

int mqb_program_get_info(const mqb_program *p, mqb_program_info *info) {
    return guarded([&] {
        if (!p || !info) fail(MQB_ERR_INVALID, "null argument");
        std::memset(info, 0, sizeof(*info));
        info->n_qubits = p->n;
        info->precision = p->precision;
        info->n_ops = int(p->ops.size());
        info->n_params = p->n_params;
        info->n_passes = int(p->apply_sched->s.passes.size());
        info->tile_bits = p->apply_sched->s.K;
        info->n_grad_slots = p->n_slots;
        info->per_sample_entries = int32_t(p->per_sample);
        info->custom_entries = int32_t(p->custom_entries);
    });
}

int mqb_program_grad_passes(mqb_program *p, int n_hams, int *n_passes, int *tile_bits) {
    return guarded([&] {
        if (!p || !n_passes || !tile_bits) fail(MQB_ERR_INVALID, "null argument");
        if (n_hams < 1) fail(MQB_ERR_INVALID, "need at least one Hamiltonian");
        SchedDev &sd = grad_schedule(*p, n_hams);
        *n_passes = int(sd.s.passes.size());
        *tile_bits = sd.s.K;
    });
}

int mqb_apply_workspace_size(const mqb_program *p, int64_t batch, size_t *bytes) {
    return guarded([&] {
        if (!p || !bytes) fail(MQB_ERR_INVALID, "null argument");
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        *bytes = std::max<size_t>(256, align_up(size_t(batch) * p->per_sample * p->elem()));
    });
}

int mqb_apply(mqb_program *p, void *states, int64_t batch, const double *params, int64_t param_stride,
              const double *custom, void *ws, size_t ws_bytes, void *stream) {
    return guarded([&] {
        Range range("mqb_apply");
        if (!p || !states) fail(MQB_ERR_INVALID, "null argument");
        require_aligned(states, "states");
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        if (p->per_sample && !params && p->n_params) fail(MQB_ERR_INVALID, "parameters required");
        if (p->custom_entries && !custom) fail(MQB_ERR_INVALID, "custom gate matrices required");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (p->precision == MQB_PREC_C64)
            apply_impl<float>(*p, states, batch, params, param_stride, custom, ws, ws_bytes, st);
        else
            apply_impl<double>(*p, states, batch, params, param_stride, custom, ws, ws_bytes, st);
    });
}

int mqb_ham_create(int n_qubits, int precision, const uint64_t *mask_x, const uint64_t *mask_y, const uint64_t *mask_z,
                   const int32_t *num_y, const double *coeff, int n_terms, mqb_hamiltonian **out) {
    return guarded([&] {
        Range range("mqb_ham_create");
        if (!out) fail(MQB_ERR_INVALID, "out is null");
        *out = nullptr;
        if (n_qubits < 1 || n_qubits > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40]");
        if (precision != MQB_PREC_C64 && precision != MQB_PREC_C128) fail(MQB_ERR_INVALID, "bad precision %d", precision);
        if (n_terms < 0) fail(MQB_ERR_INVALID, "n_terms must be >= 0, got %d", n_terms);
        if (n_terms > 0 && (!mask_x || !mask_y || !mask_z || !num_y || !coeff))
            fail(MQB_ERR_INVALID, "null term arrays for %d terms", n_terms);
        const uint64_t allq = (uint64_t(1) << n_qubits) - 1;
        std::vector<uint64_t> mx, my, mz;
        std::vector<int> ny;
        std::vector<double> cf;
        for (int t = 0; t < n_terms; ++t) {
            if ((mask_x[t] | mask_y[t] | mask_z[t]) & ~allq) fail(MQB_ERR_INVALID, "term %d acts outside the register", t);
            if ((mask_x[t] & mask_y[t]) || (mask_x[t] & mask_z[t]) || (mask_y[t] & mask_z[t]))
                fail(MQB_ERR_INVALID, "term %d has overlapping Pauli masks", t);
            if (coeff[t] == 0) continue;
            mx.push_back(mask_x[t]);
            my.push_back(mask_y[t]);
            mz.push_back(mask_z[t]);
            ny.push_back(num_y[t]);
            cf.push_back(coeff[t]);
        }
        auto h = std::make_unique<mqb_hamiltonian>();
        h->n = n_qubits;
        h->precision = precision;
        std::vector<HamClass> classes;
        std::vector<HamTerm> hterms;
        // complex64: 2^12-amplitude tiles, 256 threads of 16 registers each, so two blocks
        // (125 registers a thread) share an SM and one's tile loads overlap the other's math
        const int hk = precision == MQB_PREC_C64 ? std::min(12, default_tile_bits(precision, 1))
                                                 : default_tile_bits(precision, 1);
        build_ham_groups(n_qubits, hk, contiguity_bits(precision), mx, my, mz, ny, cf, h->groups, classes, hterms);
        h->classes = classes;
        h->d_classes = upload(classes);
        h->d_terms = upload(hterms);
        *out = h.release();
    });
}

int mqb_ham_create_csr(int n_qubits, int precision, int64_t nnz, const int64_t *indptr, const int64_t *indices,
                       const void *data, mqb_hamiltonian **out) {
    return guarded([&] {
        Range range("mqb_ham_create_csr");
        if (!out) fail(MQB_ERR_INVALID, "out is null");
        *out = nullptr;
        if (n_qubits < 1 || n_qubits > 31) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 31] for a sparse Hamiltonian");
        if (precision != MQB_PREC_C64 && precision != MQB_PREC_C128) fail(MQB_ERR_INVALID, "unknown precision");
        if (nnz < 0 || !indptr || (nnz > 0 && (!indices || !data))) fail(MQB_ERR_INVALID, "null CSR array");
        const int64_t dim = int64_t(1) << n_qubits;
        if (indptr[0] != 0 || indptr[dim] != nnz) fail(MQB_ERR_INVALID, "indptr must run from 0 to nnz");
        for (int64_t r = 0; r < dim; ++r)
            if (indptr[r + 1] < indptr[r]) fail(MQB_ERR_INVALID, "indptr decreases at row %lld", (long long)r);
        for (int64_t j = 0; j < nnz; ++j)
            if (indices[j] < 0 || indices[j] >= dim)
                fail(MQB_ERR_INVALID, "column index %lld out of range at entry %lld", (long long)indices[j], (long long)j);
        // slices of 32 rows, entry k of row `lane` at slice_ptr + 32 k + lane, padded with
        // (column = the row, value 0) up to the slice's longest row
        const int64_t n_slices = (dim + 31) / 32;
        std::vector<int64_t> sptr(static_cast<size_t>(n_slices));
        std::vector<int32_t> slen(static_cast<size_t>(n_slices));
        int64_t entries = 0;
        for (int64_t sl = 0; sl < n_slices; ++sl) {
            int64_t longest = 0;
            for (int64_t r = sl * 32; r < std::min(dim, sl * 32 + 32); ++r) longest = std::max(longest, indptr[r + 1] - indptr[r]);
            if (longest > INT32_MAX) fail(MQB_ERR_INVALID, "row too long");
            sptr[size_t(sl)] = entries;
            slen[size_t(sl)] = int32_t(longest);
            entries += longest * 32;
        }
        const size_t elem = precision == MQB_PREC_C64 ? 8 : 16;
        std::vector<int32_t> cols(static_cast<size_t>(entries));
        std::vector<unsigned char> vals(static_cast<size_t>(entries) * elem, 0);
        const unsigned char *src = static_cast<const unsigned char *>(data);
        for (int64_t sl = 0; sl < n_slices; ++sl) {
            for (int lane = 0; lane < 32; ++lane) {
                const int64_t r = sl * 32 + lane;
                const int64_t row_len = r < dim ? indptr[r + 1] - indptr[r] : 0;
                for (int64_t k = 0; k < slen[size_t(sl)]; ++k) {
                    const size_t at = size_t(sptr[size_t(sl)] + k * 32 + lane);
                    if (k < row_len) {
                        const int64_t j = indptr[r] + k;
                        cols[at] = int32_t(indices[j]);
                        std::memcpy(&vals[at * elem], src + size_t(j) * elem, elem);
                    } else {
                        cols[at] = int32_t(r < dim ? r : 0);
                    }
                }
            }
        }
        auto h = std::make_unique<mqb_hamiltonian>();
        h->n = n_qubits;
        h->precision = precision;
        h->csr = true;
        h->nnz = nnz;
        h->entries = entries;
        h->d_slice_ptr = upload(sptr);
        h->d_slice_len = upload(slen);
        h->d_cols = upload(cols);
        if (entries > 0) {
            dev_alloc(&h->d_vals, vals.size(), "cudaMalloc");
            ck(cudaMemcpy(h->d_vals, vals.data(), vals.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
        }
        *out = h.release();
    });
}

int mqb_ham_destroy(mqb_hamiltonian *h) {
    return guarded([&] { delete h; });
}

int mqb_apply_hamiltonian(const mqb_hamiltonian *h, const void *in, void *out, int64_t batch, void *stream) {
    return guarded([&] {
        Range range("mqb_apply_hamiltonian");
        if (!h || !in || !out) fail(MQB_ERR_INVALID, "null argument");
        require_aligned(in, "in");
        require_aligned(out, "out");
        if (in == out) fail(MQB_ERR_INVALID, "in and out must be different buffers");
        if (batch < 0) fail(MQB_ERR_INVALID, "batch must be >= 0");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (h->precision == MQB_PREC_C64)
            ham_impl<float>(*h, nullptr, static_cast<const float2 *>(in), static_cast<float2 *>(out), nullptr, 2, batch, st);
        else
            ham_impl<double>(*h, nullptr, static_cast<const double2 *>(in), static_cast<double2 *>(out), nullptr, 2, batch,
                             st);
    });
}

int mqb_expectation(const mqb_hamiltonian *h, const void *bra, const void *ket, int64_t batch, double *out, void *stream) {
    return guarded([&] {
        Range range("mqb_expectation");
        if (!h || !bra || !ket || !out) fail(MQB_ERR_INVALID, "null argument");
        if (batch < 0) fail(MQB_ERR_INVALID, "batch must be >= 0");
        require_aligned(bra, "bra");
        require_aligned(ket, "ket");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        ck(cudaMemsetAsync(out, 0, sizeof(double) * 2 * batch, st), "memset");
        if (h->precision == MQB_PREC_C64)
            ham_impl<float>(*h, static_cast<const float2 *>(bra), static_cast<const float2 *>(ket), nullptr, out, 2, batch, st);
        else
            ham_impl<double>(*h, static_cast<const double2 *>(bra), static_cast<const double2 *>(ket), nullptr, out, 2,
                             batch, st);
    });
}

int mqb_apply_matrix1(int n, int precision, void *states, int64_t batch, int qubit, uint64_t ctrl_mask,
                      const double *matrix, void *stream) {
    return guarded([&] {
        Range range("mqb_apply_matrix1");
        if (!states || !matrix) fail(MQB_ERR_INVALID, "null argument");
        if (n < 1 || n > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40]");
        if (qubit < 0 || qubit >= n) fail(MQB_ERR_INVALID, "qubit %d outside the register", qubit);
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        if (n < 64 && (ctrl_mask >> n)) fail(MQB_ERR_INVALID, "control mask outside the register");
        if (ctrl_mask >> qubit & 1) fail(MQB_ERR_INVALID, "the target qubit cannot be a control");
        Mat1 m;
        for (int k = 0; k < 8; ++k) m.v[k] = matrix[k];
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int sm = sm_count_cached();
        TimeScope ts(TK_OTHER, st);
        if (precision == MQB_PREC_C64)
            ck(launch_matrix1<float>(static_cast<float2 *>(states), n, qubit, ctrl_mask, batch, m, sm, st), "matrix");
        else
            ck(launch_matrix1<double>(static_cast<double2 *>(states), n, qubit, ctrl_mask, batch, m, sm, st), "matrix");
    });
}

namespace {
// Host checks and chunked launches shared by mqb_rows_apply_matrix1 / mqb_rows_matrix1_norm.
void rows_matrix1(int n, int precision, void *states, int64_t batch, int64_t count, const int64_t *rows,
                  const int32_t *qubits, const uint64_t *masks, const double *matrices, double *norm_out,
                  cudaStream_t st) {
    if (n < 1 || n > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40]");
    if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
    if (count < 0) fail(MQB_ERR_INVALID, "count must be >= 0");
    if (count == 0) return;
    if (!states || !rows || !qubits || !masks || !matrices) fail(MQB_ERR_INVALID, "null argument");
    require_aligned(states, "states");
    for (int64_t i = 0; i < count; ++i) {
        if (rows[i] < 0 || rows[i] >= batch) fail(MQB_ERR_INVALID, "request %lld: row %lld outside the batch",
                                                  (long long)i, (long long)rows[i]);
        if (qubits[i] < 0 || qubits[i] >= n) fail(MQB_ERR_INVALID, "request %lld: qubit %d outside the register",
                                                  (long long)i, qubits[i]);
        if (n < 64 && (masks[i] >> n)) fail(MQB_ERR_INVALID, "request %lld: control mask outside the register",
                                            (long long)i);
        if (masks[i] >> qubits[i] & 1) fail(MQB_ERR_INVALID, "request %lld: the target qubit cannot be a control",
                                            (long long)i);
    }
    if (!norm_out) {   // in-place updates of one row from two requests would race
        std::vector<int64_t> sorted(rows, rows + count);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            fail(MQB_ERR_INVALID, "rows must be distinct");
    }
    const int sm = sm_count_cached();
    TimeScope ts(TK_ROWS, st);
    RowOps ops;
    for (int64_t a = 0; a < count; a += kRowOpsMax) {
        ops.count = int(std::min<int64_t>(kRowOpsMax, count - a));
        for (int k = 0; k < ops.count; ++k) {
            ops.row[k] = rows[a + k];
            ops.qubit[k] = qubits[a + k];
            ops.ctrl[k] = masks[a + k];
            for (int v = 0; v < 8; ++v) ops.m[k][v] = matrices[8 * (a + k) + v];
        }
        double *o = norm_out ? norm_out + a : nullptr;
        if (precision == MQB_PREC_C64)
            ck(launch_row_ops<float>(static_cast<float2 *>(states), n, ops, o, sm, st), "row ops");
        else
            ck(launch_row_ops<double>(static_cast<double2 *>(states), n, ops, o, sm, st), "row ops");
    }
}
}  // namespace

int mqb_rows_apply_matrix1(int n, int precision, void *states, int64_t batch, int64_t count, const int64_t *rows,
                           const int32_t *qubits, const uint64_t *ctrl_masks, const double *matrices, void *stream) {
    return guarded([&] {
        Range range("mqb_rows_apply_matrix1");
        rows_matrix1(n, precision, states, batch, count, rows, qubits, ctrl_masks, matrices, nullptr,
                     static_cast<cudaStream_t>(stream));
    });
}

int mqb_rows_matrix1_norm(int n, int precision, const void *states, int64_t batch, int64_t count, const int64_t *rows,
                          const int32_t *qubits, const uint64_t *ctrl_masks, const double *matrices, double *out,
                          void *stream) {
    return guarded([&] {
        if (count > 0 && !out) fail(MQB_ERR_INVALID, "null argument");
        rows_matrix1(n, precision, const_cast<void *>(states), batch, count, rows, qubits, ctrl_masks, matrices, out,
                     static_cast<cudaStream_t>(stream));
    });
}

int mqb_vdot(int n, int precision, const void *a, const void *b, int64_t batch, double *out, void *stream) {
    return guarded([&] {
        Range range("mqb_vdot");
        if (!a || !b || !out) fail(MQB_ERR_INVALID, "null argument");
        require_register(n, precision);
        if (batch < 0) fail(MQB_ERR_INVALID, "batch must be >= 0");
        require_aligned(a, "a");
        require_aligned(b, "b");
        const int sm = sm_count_cached();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (precision == MQB_PREC_C64)
            ck(launch_vdot<float>(static_cast<const float2 *>(a), static_cast<const float2 *>(b), n, batch, out, sm, st), "vdot");
        else
            ck(launch_vdot<double>(static_cast<const double2 *>(a), static_cast<const double2 *>(b), n, batch, out, sm, st),
               "vdot");
    });
}

int mqb_grad_workspace_size(const mqb_program *p, int64_t batch, int n_hams, int stride, size_t *bytes) {
    return guarded([&] {
        if (!p || !bytes) fail(MQB_ERR_INVALID, "null argument");
        if (n_hams < 1) fail(MQB_ERR_INVALID, "need at least one Hamiltonian");
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        SchedDev &sd = grad_schedule(const_cast<mqb_program &>(*p), n_hams);
        *bytes = grad_layout(*p, sd.s, batch, n_hams, stride).total;
    });
}

int mqb_grad_norm_checks(mqb_program *p, const void *ws, size_t ws_bytes, int64_t batch, int n_hams, int stride,
                         double *out, int capacity, int *n_checks, void *stream) {
    return guarded([&] {
        Range range("mqb_grad_norm_checks");
        if (!p || !n_checks) fail(MQB_ERR_INVALID, "null argument");
        if (n_hams < 1 || batch < 1) fail(MQB_ERR_INVALID, "invalid batch or number of Hamiltonians");
        SchedDev &sd = grad_schedule(*p, n_hams);
        const GradLayout L = grad_layout(*p, sd.s, batch, n_hams, stride);
        const int n = int(L.norm_fwd.size() + L.norm_bwd.size());
        *n_checks = n;
        if (n == 0 || !out) return;
        if (!ws || ws_bytes < L.total) fail(MQB_ERR_WORKSPACE, "workspace too small (%zu < %zu)", ws_bytes, L.total);
        if (capacity < n) fail(MQB_ERR_INVALID, "capacity %d below the %d checks", capacity, n);
        const unsigned char *base = static_cast<const unsigned char *>(ws) + L.mats + L.gslots + L.lam + L.w + L.ckpt;
        std::vector<double> raw(size_t(n) * batch * 2);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        ck(cudaMemcpyAsync(raw.data(), base, raw.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
        ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        for (size_t i = 0; i < size_t(n) * batch; ++i) out[i] = raw[2 * i];
    });
}

int mqb_expectation_with_grad(mqb_program *p, const mqb_hamiltonian *const *hams, int n_hams, const void *init,
                              int init_batched, int64_t batch, const double *params, int64_t param_stride,
                              const double *custom, double *f, double *grad, int stride, void *ws, size_t ws_bytes,
                              void *stream) {
    return guarded([&] {
        Range range("mqb_expectation_with_grad");
        if (!p || !hams || !f || !grad) fail(MQB_ERR_INVALID, "null argument");
        require_aligned(init, "init_states");
        require_aligned(ws, "workspace");
        if (n_hams < 1) fail(MQB_ERR_INVALID, "need at least one Hamiltonian");
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        for (int h = 0; h < n_hams; ++h) {
            if (!hams[h]) fail(MQB_ERR_INVALID, "Hamiltonian %d is null", h);
            if (hams[h]->n != p->n || hams[h]->precision != p->precision)
                fail(MQB_ERR_INVALID, "Hamiltonian %d does not match the program's qubits / precision", h);
        }
        if (p->custom_entries && !custom) fail(MQB_ERR_INVALID, "custom gate matrices required");
        if (batch > 65535 / 12) fail(MQB_ERR_INVALID, "batch too large for one call");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (p->precision == MQB_PREC_C64)
            grad_impl<float>(*p, hams, n_hams, init, init_batched, batch, params, param_stride, custom, f, grad, stride, ws,
                             ws_bytes, st);
        else
            grad_impl<double>(*p, hams, n_hams, init, init_batched, batch, params, param_stride, custom, f, grad, stride, ws,
                              ws_bytes, st);
    });
}

int mqb_adjoint_with_lambda(mqb_program *p, const void *lam, int lam_batched, const void *init, int init_batched,
                            int64_t batch, const double *params, int64_t param_stride, const double *custom,
                            double *grad, int stride, void *ws, size_t ws_bytes, void *stream) {
    return guarded([&] {
        Range range("mqb_adjoint_with_lambda");
        if (!p || !lam || !grad) fail(MQB_ERR_INVALID, "null argument");
        require_aligned(lam, "lambda");
        require_aligned(init, "init_states");
        require_aligned(ws, "workspace");
        if (batch < 1) fail(MQB_ERR_INVALID, "batch must be >= 1");
        if (p->custom_entries && !custom) fail(MQB_ERR_INVALID, "custom gate matrices required");
        if (batch > 65535 / 12) fail(MQB_ERR_INVALID, "batch too large for one call");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (p->precision == MQB_PREC_C64)
            grad_impl<float>(*p, nullptr, 1, init, init_batched, batch, params, param_stride, custom, nullptr, grad,
                             stride, ws, ws_bytes, st, lam, lam_batched);
        else
            grad_impl<double>(*p, nullptr, 1, init, init_batched, batch, params, param_stride, custom, nullptr, grad,
                              stride, ws, ws_bytes, st, lam, lam_batched);
    });
}

int mqb_sample_scratch_size(int n, size_t *bytes) {
    return guarded([&] {
        if (!bytes) fail(MQB_ERR_INVALID, "null argument");
        if (n < 1 || n > 40) fail(MQB_ERR_INVALID, "n_qubits must be in [1, 40], got %d", n);
        const int cb = std::min(n, 12);
        *bytes = sizeof(double) * ((size_t(1) << (n - cb)) + 1);
    });
}

int mqb_sample_indices(int n, int precision, const void *state, const double *u, int64_t shots, int64_t *out,
                       void *scratch, size_t scratch_bytes, void *stream) {
    return guarded([&] {
        Range range("mqb_sample_indices");
        require_register(n, precision);
        if (shots < 0) fail(MQB_ERR_INVALID, "shots must be >= 0");
        if (!state || (shots > 0 && (!u || !out))) fail(MQB_ERR_INVALID, "null argument");
        const int cb = std::min(n, 12);
        const size_t need = sizeof(double) * ((size_t(1) << (n - cb)) + 1);
        if (!scratch || scratch_bytes < need) fail(MQB_ERR_WORKSPACE, "scratch too small");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        double *sums = static_cast<double *>(scratch);
        const int64_t nch = int64_t(1) << (n - cb);
        if (precision == MQB_PREC_C64) {
            ck(launch_chunk_probs<float>(static_cast<const float2 *>(state), n, cb, sums, st), "chunk probs");
            ck(launch_prefix(sums, nch, st), "prefix");
            ck(launch_sample_search<float>(static_cast<const float2 *>(state), n, cb, sums, u, shots, out, st), "search");
        } else {
            ck(launch_chunk_probs<double>(static_cast<const double2 *>(state), n, cb, sums, st), "chunk probs");
            ck(launch_prefix(sums, nch, st), "prefix");
            ck(launch_sample_search<double>(static_cast<const double2 *>(state), n, cb, sums, u, shots, out, st), "search");
        }
    });
}

int mqb_qubit_one_probability(int n, int precision, const void *state, int q, double *out, void *stream) {
    return guarded([&] {
        Range range("mqb_qubit_one_probability");
        require_register(n, precision);
        if (!state || !out) fail(MQB_ERR_INVALID, "null argument");
        if (q < 0 || q >= n) fail(MQB_ERR_INVALID, "qubit out of range");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (precision == MQB_PREC_C64)
            ck(launch_one_prob<float>(static_cast<const float2 *>(state), n, q, out, st), "probability");
        else
            ck(launch_one_prob<double>(static_cast<const double2 *>(state), n, q, out, st), "probability");
    });
}

int mqb_collapse(int n, int precision, void *state, int q, int outcome, double scale, void *stream) {
    return guarded([&] {
        Range range("mqb_collapse");
        require_register(n, precision);
        if (!state) fail(MQB_ERR_INVALID, "null argument");
        if (q < 0 || q >= n) fail(MQB_ERR_INVALID, "qubit out of range");
        if (outcome != 0 && outcome != 1) fail(MQB_ERR_INVALID, "outcome must be 0 or 1, got %d", outcome);
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        if (precision == MQB_PREC_C64)
            ck(launch_collapse<float>(static_cast<float2 *>(state), n, q, outcome, scale, st), "collapse");
        else
            ck(launch_collapse<double>(static_cast<double2 *>(state), n, q, outcome, scale, st), "collapse");
    });
}

}  // extern "C"
