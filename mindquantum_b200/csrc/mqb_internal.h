// Internal data structures of the mqb200 engine: the lowered op table, the pass schedule
// produced by the host scheduler, and the launch interfaces of the CUDA kernels.
#ifndef MQB_INTERNAL_H_
#define MQB_INTERNAL_H_

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mqb200.h"
#include "jit_abi.h"
#include "mqb_gate_ids.h"

namespace mqb {

constexpr int kMaxFusedM = 2;        // gates with <= 2 targets run inside fused tiles
constexpr int kMaxTileBits = 13;     // upper bound of the tile size 2^K (TileGeom::qbits)
constexpr int kMaxPassOps = 256;     // ops of one fused pass (staged in shared memory)
constexpr int kMaxPassSlots = 96;    // gradient slots of one fused pass (accumulated in shared memory)
constexpr int kMaxGroupClasses = 64; // flip classes of one Hamiltonian pass
constexpr int kMaxClassTerms = 64;   // Pauli terms of one flip class
constexpr int kThreads = 256;        // threads of the tile kernels

enum OpKind : int32_t { KIND_DENSE = 0, KIND_DIAG = 1, KIND_RPS = 2 };

// One lowered gate in execution order.
struct DevOp {
    int32_t kind;
    int32_t m;                   // number of target qubits
    int32_t tq[MQB_MAX_OBJ];     // global target qubits; tq[b] is matrix index bit b
    uint64_t ctrl;               // global control mask
    int32_t gate_id;
    int32_t per_sample;          // 1: matrices live in the per-sample block
    int64_t mat_off;             // complex entries: const pool offset or per-sample offset of M
    int32_t n_angles;
    int32_t grad_mask;           // bit a: angle a has a gradient
    int32_t slot0;               // gradient slot of the first gradient angle (consecutive)
    int32_t dmat_off;            // per-sample offset of dM_0; dM_a = dmat_off + a * mat_size
    int32_t mat_size;            // complex entries of one matrix (4^m dense, 2^m diagonal, 1 RPS)
    int32_t custom_off;          // GID_CUSTOM: offset of M in the caller's per-sample custom block
    uint64_t px, py, pz;         // GID_RPS masks
    int32_t pny;
    int32_t sub;                 // dense single-qubit structure: SUB_GENERIC, SUB_REAL, SUB_PERM, SUB_SWAP, SUB_RXL
};
// Structure of a dense single-qubit matrix, used to pick a cheaper register kernel.
// SUB_RXL: [[a, ib], [ib, a]] with a, b real, and so are its derivatives (RX).
enum DenseSub : int32_t { SUB_GENERIC = 0, SUB_REAL = 1, SUB_PERM = 2, SUB_SWAP = 3, SUB_RXL = 4 };

// An op as seen inside one fused pass (targets remapped to tile-local bits).
struct PassOp {
    int32_t op;        // program op index
    int32_t kind;
    int32_t m;
    int32_t lt[kMaxFusedM];   // local target bit (dense: always >= 0; diag: -1 when outside the tile)
    int32_t gt[kMaxFusedM];   // global target qubit
    uint32_t lctrl;           // control bits inside the tile (local mask)
    int32_t lslot;            // pass-local gradient slot of the first gradient angle (-1: none)
    uint64_t octrl;           // control bits outside the tile (global mask)
};

// A register stage of a fused pass: every thread holds 2^RB amplitudes of the tile in registers,
// those whose tile-local index differs in the stage's register bits; the stage's gates act on
// register bits only (diagonal gates may act on any bit).  Stages exchange data through the
// tile in shared memory.
constexpr int kMaxRegBits = 5;
constexpr int kMaxThreadBits = 8;
struct StageDesc {
    int8_t rbits[kMaxRegBits];     // register position -> tile-local bit
    int8_t tbits[kMaxThreadBits];  // thread-index bit -> tile-local bit
    int8_t pad[3];
    int32_t op_begin, op_end;      // range in Schedule::stage_ops
};
enum StageOpKind : int32_t {
    SK_DENSE1 = 0, SK_DENSE2 = 1, SK_DIAG1 = 2, SK_DIAG2 = 3, SK_REAL1 = 4, SK_PERM1 = 5, SK_SWAP1 = 6, SK_RXL1 = 7
};
// Register codes: the structure of a stage op as the tile kernels resolve it at compile time.
// P / Q: register positions of matrix bits 0 / 1; C: position of the only register control;
// K: matrix bit of the diagonal target that sits on a register.  The backward kernels use
// code * 4 + gradient selector (0 no gradient, 1 angle 0, 2 angles 0..2, 3 runtime mask).
enum RegCode : int32_t {
    RC_DENSE1 = 0,      // + P        dense 2x2, no register control
    RC_REAL1 = 5,       // + P        real 2x2 (RY, H)
    RC_RXL1 = 10,       // + P        [[a, ib], [ib, a]], a and b real (RX)
    RC_X1 = 15,         // + P        X (register swap)
    RC_DIAG1 = 20,      // + P        diagonal on a register
    RC_SCALE = 25,      //            diagonal whose targets are off the registers (one factor per thread)
    RC_DENSE1C = 26,    // + 5P + C   dense 2x2, one register control
    RC_X1C = 51,        // + 5P + C   CNOT inside the registers
    RC_DIAG1C = 76,     // + 5P + C   controlled diagonal (CZ, CRZ, CPS)
    RC_SCALEC = 101,    // + C        SCALE with one register control
    RC_DIAG2 = 106,     // + 5P + Q   two-target diagonal on registers (RZZ)
    RC_DIAG2S = 131,    // + 5K + P   two-target diagonal, one target on register P, the other off
    RC_DENSE2 = 141,    // + 5P + Q   dense 4x4, no register control
    RC_GDENSE1 = 166,   // + P        dense 2x2, register control mask tested at run time
    RC_GDIAG = 171,     //            any diagonal, register control mask tested at run time
    RC_GDENSE2 = 172,   // + 5P + Q   dense 4x4, register control mask tested at run time
    RC_COUNT = 197
};
struct StageOp {
    int32_t op;          // program op index
    int32_t kind;        // StageOpKind
    int32_t p0, p1;      // dense: register positions of matrix bit 0 / bit 1
    int32_t dsrc[2];     // diag target k: 0 register position, 1 thread (local bit), 2 outside (global qubit)
    int32_t dval[2];     // position / local bit / global qubit
    uint32_t rctrl;      // control bits among register positions
    uint32_t tctrl;      // control bits among thread bits (tile-local mask)
    uint64_t octrl;      // control bits outside the tile (global mask)
    int32_t lslot;       // pass-local gradient slot of the first gradient angle (-1: none)
    int32_t n_angles;    // gradient angles of the gate when it has any, else 0
    int32_t grad_mask;
    int32_t mat_size;    // complex entries of one matrix (4 / 16 dense, 2 / 4 diagonal)
    int32_t moff;        // offset of M in the pass's shared-memory matrix table (dM_a follows at moff + (1+a) mat_size)
    int32_t mcount;      // entries copied into the table (M, then dM_0..)
    int64_t msrc;        // source offset: per-sample block (msrc_ps) or constant pool
    int32_t msrc_ps;     // 1: per-sample matrices, 0: constant pool
    int32_t code;        // RegCode of the forward kernels
    int32_t bcode;       // code * 4 + gradient selector, for the backward kernels
    int32_t cflags;      // bit 0: octrl != 0, bit 1: tctrl != 0 (controls checked per thread)
    int32_t pad;
};

// A pass: one sweep over the state(s).
struct Pass {
    int fused = 1;                 // 1: fused tile pass over ops [op_begin, op_end) of pass_ops; 0: single op
    int K = 0;                     // tile bits
    int c = 0;                     // contiguity bits (low qubits always in the tile)
    std::vector<int> qbits;        // local bit -> global qubit (ascending)
    std::vector<int> outside;      // global qubits not in the tile (ascending)
    int op_begin = 0, op_end = 0;  // fused: range in Schedule::pass_ops; single: op index in op_begin
    int prog_op_begin = 0, prog_op_end = 0;  // program ops covered (execution order)
    int slot_begin = 0, n_slots = 0;         // fused: range in Schedule::slot_map (pass-local gradient slots)
    int stage_begin = 0, n_stages = 0;       // fused: range in Schedule::stages
    int sop_begin = 0, n_sops = 0;           // fused: range in Schedule::stage_ops (StageDesc ranges are relative)
    int mtab_entries = 0;                    // fused: complex entries of the pass's shared-memory matrix table
    // the forward kernel's own stage layout of the same pass (more register bits, no lambdas)
    int f_stage_begin = 0, f_n_stages = 0, f_sop_begin = 0, f_n_sops = 0, f_mtab_entries = 0, f_reg_bits = 0;
    int reg_bits = 0, thread_bits = 0;       // fused: registers / threads of the tile kernel
};

struct Schedule {
    int K = 0;
    std::vector<Pass> passes;
    std::vector<PassOp> pass_ops;
    std::vector<int32_t> slot_map;  // pass-local slot -> global gradient slot
    std::vector<StageDesc> stages;      // backward layout
    std::vector<StageOp> stage_ops;
    std::vector<StageDesc> f_stages;    // forward layout
    std::vector<StageOp> f_stage_ops;
    StageDesc *d_f_stages = nullptr;
    StageOp *d_f_stage_ops = nullptr;
    PassOp *d_pass_ops = nullptr;   // device copies
    int32_t *d_slot_map = nullptr;
    StageDesc *d_stages = nullptr;
    StageOp *d_stage_ops = nullptr;
};

// Hamiltonian: terms grouped into passes; every group's flip masks fit in one tile.
constexpr int kHamRegBits = 4;      // amplitudes per thread of the Hamiltonian kernel: 2^4
struct HamTerm {
    double coeff;
    uint64_t my_mz;     // mask_y | mask_z (global), phase sign bits
    int32_t ny;
    uint32_t lmask;     // my_mz on the group's tile-local bits
    uint64_t omask;     // my_mz on the qubits outside the tile
    double cb_re, cb_im;   // coeff * i^ny * (-1)^popc(flip & my_mz): the phase without the index bits
};
struct HamClass {       // terms sharing one flip mask
    uint64_t flip;      // global flip mask (mask_x | mask_y)
    uint32_t lflip;     // the same mask on the group's tile-local bits
    int32_t term_begin, term_count;
    // terms sorted by the bits of lmask on the thread's register bits (the top kHamRegBits local
    // bits): bins[b] .. bins[b + 1] is bin b, relative to term_begin
    int32_t bins[(1 << kHamRegBits) + 1];
};
struct HamGroup {
    TileGeom geom;
    int class_begin, class_count;
};

// While alive, calls on this thread run the precompiled tile kernels only: no pass kernel is
// generated or loaded (callers that promise to allocate nothing).
class JitBlock {
  public:
    JitBlock();
    ~JitBlock();
    JitBlock(const JitBlock &) = delete;
    JitBlock &operator=(const JitBlock &) = delete;

  private:
    bool prev_;
};

// Builders (scheduler.cpp)
// no_fuse (optional, one entry per op): ops that must run in a pass of their own.
Schedule build_schedule(int n, int K, int c, const std::vector<DevOp> &ops, bool fuse,
                        const std::vector<char> *no_fuse = nullptr);
// Split every fused pass of `s` into register stages with `reg_bits` register bits per thread:
// the backward layout (Schedule::stages) or, with `forward`, the forward layout (f_stages).
void build_stages(Schedule &s, const std::vector<DevOp> &ops, int reg_bits, int precision, bool forward = false);
inline uint32_t smem_swizzle(uint32_t L, int precision) {
    // XOR-fold the index into its low 4 (complex64) / 3 (complex128) bits: linear over GF(2) and
    // a bijection, so bank conflicts of the stage exchanges depend only on the thread bits' residues
    if (precision == MQB_PREC_C64) return L ^ ((L >> 4) & 15u) ^ ((L >> 8) & 15u) ^ ((L >> 12) & 15u);
    return L ^ ((L >> 3) & 7u) ^ ((L >> 6) & 7u) ^ ((L >> 9) & 7u) ^ ((L >> 12) & 7u);
}
void build_ham_groups(int n, int K, int c, const std::vector<uint64_t> &mx, const std::vector<uint64_t> &my,
                      const std::vector<uint64_t> &mz, const std::vector<int> &ny, const std::vector<double> &coeff,
                      std::vector<HamGroup> &groups, std::vector<HamClass> &classes, std::vector<HamTerm> &terms);
TileGeom make_geom(int n, const std::vector<int> &qbits);
int contiguity_bits(int precision);
int default_tile_bits(int precision, int n_states_in_tile);
// Register bits of the fused kernels: forward passes, and backward passes with n_hams lambdas.
int fwd_reg_bits(int precision);
int bwd_reg_bits(int precision, int n_hams);

}  // namespace mqb

#endif
