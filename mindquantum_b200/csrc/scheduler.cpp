// Host-side pass scheduler.
//
// The reference applies every gate as its own sweep over the state
// (VectorState::ApplyCircuit, ccsrc/include/simulator/vector/vector_state.tpp:949-960).  Here a
// circuit is cut into passes: a fused pass owns a set Q of K "tile" qubits (always including
// the lowest c qubits, so every tile is made of 128-byte contiguous runs) and applies, in one
// read + write of the state, every gate whose non-diagonal targets lie in Q.  Diagonal gates
// and control qubits may sit anywhere: outside Q their bits are constant over a tile.
//
// The greedy scan keeps the circuit's order of non-commuting gates: a gate that cannot join
// the current pass blocks all its qubits for the rest of the scan, so no later gate sharing a
// qubit with it can overtake it.
#include <algorithm>
#include <cstdlib>
#include <stdexcept>

#include "mqb_internal.h"

namespace mqb {

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }

int contiguity_bits(int precision) { return precision == MQB_PREC_C64 ? 4 : 3; }

// MQB_FWD_REG_BITS (2..5) overrides the complex64 forward register bits (tuning).
int fwd_reg_bits(int precision) {
    if (precision == MQB_PREC_C64)
        if (const char *e = std::getenv("MQB_FWD_REG_BITS")) return std::max(2, std::min(5, std::atoi(e)));
    return precision == MQB_PREC_C64 ? 5 : 4;
}

int bwd_reg_bits(int precision, int n_hams) {
    if (n_hams <= 1) return precision == MQB_PREC_C64 ? 4 : 3;
    return precision == MQB_PREC_C64 ? 3 : 2;
}

int default_tile_bits(int precision, int n_states_in_tile) {
    // keep the shared-memory tiles of all states at <= 64 KB so 2-3 blocks fit per SM
    const size_t amp = precision == MQB_PREC_C64 ? 8 : 16;
    int K = kMaxTileBits;
    while (K > 6 && (size_t(n_states_in_tile) << K) * amp > 65536) --K;
    return K;
}

TileGeom make_geom(int n, const std::vector<int> &qbits) {
    TileGeom g{};
    g.n = n;
    g.K = int(qbits.size());
    g.c = 0;
    while (g.c < g.K && qbits[g.c] == g.c) ++g.c;
    uint64_t qm = 0;
    for (int i = 0; i < g.K; ++i) {
        g.qbits[i] = int8_t(qbits[i]);
        qm |= uint64_t(1) << qbits[i];
    }
    g.n_out = 0;
    for (int q = 0; q < n; ++q)
        if (!(qm >> q & 1)) g.outside[g.n_out++] = int8_t(q);
    return g;
}

static uint64_t dense_targets(const DevOp &op) {
    if (op.kind != KIND_DENSE) return 0;
    uint64_t m = 0;
    for (int k = 0; k < op.m; ++k) m |= uint64_t(1) << op.tq[k];
    return m;
}

static uint64_t touched(const DevOp &op) {
    uint64_t m = op.ctrl;
    for (int k = 0; k < op.m; ++k) m |= uint64_t(1) << op.tq[k];
    if (op.kind == KIND_RPS) m |= op.px | op.py | op.pz;
    return m;
}

static bool fusable(const DevOp &op) { return (op.kind == KIND_DENSE || op.kind == KIND_DIAG) && op.m <= kMaxFusedM; }

Schedule build_schedule(int n, int K, int c, const std::vector<DevOp> &ops, bool fuse, const std::vector<char> *no_fuse) {
    auto fusable_at = [&](int i) { return fusable(ops[i]) && !(no_fuse && (*no_fuse)[i]); };
    Schedule s;
    if (K > n) K = n;
    // leave room for the widest fused gate next to the contiguity bits; keep at least one
    // contiguity bit so 16-byte vector accesses never straddle two tile runs
    if (c > K - kMaxFusedM) c = std::max(1, K - kMaxFusedM);
    if (n > K && K < kMaxFusedM + 1) fuse = false;
    if (K < 6) fuse = false;
    s.K = K;
    const int L = int(ops.size());
    std::vector<char> done(L, 0);
    int n_done = 0;
    int first = 0;
    const uint64_t all = n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << n) - 1);
    while (n_done < L) {
        while (first < L && done[first]) ++first;
        if (!fuse || !fusable_at(first)) {
            Pass p;
            p.fused = 0;
            p.op_begin = first;
            p.op_end = first + 1;
            p.prog_op_begin = first;
            p.prog_op_end = first + 1;
            s.passes.push_back(p);
            done[first] = 1;
            ++n_done;
            continue;
        }
        uint64_t Q = (n <= K) ? all : ((uint64_t(1) << c) - 1);
        uint64_t blocked = 0;
        std::vector<int> members;
        int n_slots = 0;
        for (int i = first; i < L && int(members.size()) < kMaxPassOps; ++i) {
            if (done[i]) continue;
            const DevOp &op = ops[i];
            const uint64_t t = touched(op);
            if (t & blocked) {
                blocked |= t;
                if ((blocked & all) == all) break;
                continue;
            }
            if (!fusable_at(i)) {
                blocked |= t;
                continue;
            }
            const uint64_t need = dense_targets(op) & ~Q;
            const int op_slots = popc(uint64_t(op.grad_mask));
            if (popc(Q | need) <= K && n_slots + op_slots <= kMaxPassSlots) {
                Q |= need;
                n_slots += op_slots;
                members.push_back(i);
            } else {
                blocked |= t;
            }
        }
        if (members.empty()) {
            // the first gate does not fit next to the contiguity bits: run it on its own
            Pass p;
            p.fused = 0;
            p.op_begin = first;
            p.op_end = first + 1;
            p.prog_op_begin = first;
            p.prog_op_end = first + 1;
            s.passes.push_back(p);
            done[first] = 1;
            ++n_done;
            continue;
        }
        // pad the tile to exactly K qubits with the lowest free qubits
        for (int q = 0; q < n && popc(Q) < K; ++q) Q |= uint64_t(1) << q;
        Pass p;
        p.fused = 1;
        p.K = K;
        for (int q = 0; q < n; ++q) {
            if (Q >> q & 1)
                p.qbits.push_back(q);
            else
                p.outside.push_back(q);
        }
        p.c = 0;
        while (p.c < K && p.qbits[p.c] == p.c) ++p.c;
        int local[64];
        for (int i = 0; i < 64; ++i) local[i] = -1;
        for (int i = 0; i < K; ++i) local[p.qbits[i]] = i;
        p.op_begin = int(s.pass_ops.size());
        p.slot_begin = int(s.slot_map.size());
        for (int i : members) {
            const DevOp &op = ops[i];
            PassOp po{};
            po.op = i;
            po.kind = op.kind;
            po.m = op.m;
            for (int k = 0; k < kMaxFusedM; ++k) {
                po.lt[k] = -1;
                po.gt[k] = 0;
            }
            for (int k = 0; k < op.m; ++k) {
                po.gt[k] = op.tq[k];
                po.lt[k] = local[op.tq[k]];
                if (op.kind == KIND_DENSE && po.lt[k] < 0) throw std::logic_error("dense target outside tile");
            }
            po.lctrl = 0;
            po.octrl = 0;
            for (int q = 0; q < n; ++q) {
                if (!(op.ctrl >> q & 1)) continue;
                if (local[q] >= 0)
                    po.lctrl |= 1u << local[q];
                else
                    po.octrl |= uint64_t(1) << q;
            }
            po.lslot = -1;
            if (op.grad_mask) {
                po.lslot = int(s.slot_map.size()) - p.slot_begin;
                for (int a = 0, r = 0; a < op.n_angles; ++a)
                    if (op.grad_mask >> a & 1) s.slot_map.push_back(op.slot0 + r++);
            }
            s.pass_ops.push_back(po);
            done[i] = 1;
            ++n_done;
        }
        p.op_end = int(s.pass_ops.size());
        p.n_slots = int(s.slot_map.size()) - p.slot_begin;
        p.prog_op_begin = members.empty() ? first : members.front();
        p.prog_op_end = members.empty() ? first : members.back() + 1;
        s.passes.push_back(p);
    }
    return s;
}

// Greedy register-stage grouping of one fused pass (same blocking rule as the pass scan, over
// tile-local bits), then padding of the register set and a bank-conflict-aware thread-bit order.
// Register code (forward) and code * 4 + gradient selector (backward) of a stage op; ops whose
// shape or gradient angles have no specialised kernel take the generic codes.
void assign_codes(StageOp &so) {
    const int nrc = popc(so.rctrl);
    const int C = nrc == 1 ? __builtin_ctz(so.rctrl) : -1;
    const int gm = so.n_angles ? so.grad_mask : 0;
    int code = -1, gsel = 0;
    switch (so.kind) {
        case SK_DENSE1:
        case SK_REAL1:
        case SK_RXL1:
        case SK_PERM1:
        case SK_SWAP1: {
            const int P = so.p0;
            if (nrc == 0) {
                if (so.kind == SK_SWAP1) code = RC_X1 + P;
                else if (so.kind == SK_REAL1) code = RC_REAL1 + P;
                else if (so.kind == SK_RXL1) code = RC_RXL1 + P;
                else code = RC_DENSE1 + P;
            } else if (nrc == 1) {
                code = so.kind == SK_SWAP1 ? RC_X1C + 5 * P + C : RC_DENSE1C + 5 * P + C;
            } else {
                code = RC_GDENSE1 + P;
            }
            // gradient selector; what the specialised kernels lack goes generic
            const bool x = code >= RC_X1 && code < RC_X1 + 5;
            const bool xc = code >= RC_X1C && code < RC_X1C + 25;
            if (gm == 0) {
                gsel = code >= RC_GDENSE1 ? 3 : 0;
            } else if ((x || xc) && gm) {
                code = RC_GDENSE1 + P;   // X matrices carry no derivative; never reached by lowered gates
                gsel = 3;
            } else if (code >= RC_GDENSE1) {
                gsel = 3;
            } else if (gm == 1) {
                gsel = 1;
            } else if (code < RC_DENSE1 + 5 && gm == 7) {
                gsel = 2;
            } else if (code < RC_DENSE1 + 5) {
                gsel = 3;
            } else {
                code = RC_GDENSE1 + P;
                gsel = 3;
            }
        } break;
        case SK_DENSE2: {
            const int P = so.p0, Q = so.p1;
            if (nrc == 0) {
                code = RC_DENSE2 + 5 * P + Q;
                gsel = gm == 0 ? 0 : gm == 1 ? 1 : 3;
            } else {
                code = RC_GDENSE2 + 5 * P + Q;
                gsel = 3;
            }
        } break;
        case SK_DIAG1:
        case SK_DIAG2: {
            const bool two = so.kind == SK_DIAG2;
            const bool in0 = so.dsrc[0] == 0, in1 = two && so.dsrc[1] == 0;
            if (gm != 0 && gm != 1) {
                code = RC_GDIAG;
            } else if (!two) {
                if (in0) code = nrc == 0 ? RC_DIAG1 + so.dval[0] : nrc == 1 ? RC_DIAG1C + 5 * so.dval[0] + C : RC_GDIAG;
                else code = nrc == 0 ? RC_SCALE : nrc == 1 ? RC_SCALEC + C : RC_GDIAG;
            } else if (nrc != 0) {
                code = RC_GDIAG;
            } else if (in0 && in1) {
                code = RC_DIAG2 + 5 * so.dval[0] + so.dval[1];
            } else if (in0) {
                code = RC_DIAG2S + so.dval[0];
            } else if (in1) {
                code = RC_DIAG2S + 5 + so.dval[1];
            } else {
                code = RC_SCALE;
            }
            gsel = code == RC_GDIAG ? 3 : gm;
        } break;
        default:
            throw std::runtime_error("stage op of unknown kind");
    }
    so.code = code;
    so.bcode = code * 4 + gsel;
    so.cflags = (so.octrl ? 1 : 0) | (so.tctrl ? 2 : 0);
}

void build_stages(Schedule &s, const std::vector<DevOp> &ops, int reg_bits, int precision, bool forward) {
    std::vector<StageDesc> &stages = forward ? s.f_stages : s.stages;
    std::vector<StageOp> &stage_ops = forward ? s.f_stage_ops : s.stage_ops;
    stages.clear();
    stage_ops.clear();
    const int res_mod = precision == MQB_PREC_C64 ? 4 : 3;
    for (Pass &p : s.passes) {
        if (!p.fused) continue;
        const int K = p.K;
        // 2^TB threads (32..256) holding 2^RB amplitudes each; passes are only fused when K >= reg_bits + 5
        const int RB = std::min(reg_bits, K - 5);
        const int TB = K - RB;
        const int stage_begin = int(stages.size());
        const int sop_begin = int(stage_ops.size());
        int mtab = 0;
        const int npo = p.op_end - p.op_begin;
        std::vector<char> done(npo, 0);
        int n_done = 0;
        while (n_done < npo) {
            uint32_t R = 0, blocked = 0;
            std::vector<int> members;
            for (int i = 0; i < npo; ++i) {
                if (done[i]) continue;
                const PassOp &po = s.pass_ops[p.op_begin + i];
                uint32_t touch = po.lctrl, dense = 0;
                for (int k = 0; k < po.m; ++k)
                    if (po.lt[k] >= 0) touch |= 1u << po.lt[k];
                if (po.kind == KIND_DENSE) dense = touch & ~po.lctrl;
                if (touch & blocked) {
                    blocked |= touch;
                    continue;
                }
                if (popc(R | dense) <= RB) {
                    R |= dense;
                    members.push_back(i);
                } else {
                    blocked |= touch;
                }
            }
            // padding: add local bits so that the thread bits keep one bit of every residue class
            auto thread_residue_count = [&](uint32_t Rm, int r) {
                int cnt = 0;
                for (int b = 0; b < K; ++b)
                    if (!(Rm >> b & 1) && b % res_mod == r) ++cnt;
                return cnt;
            };
            // (ties go to the highest bit: the low contiguous bits stay thread bits, so a stage can
            // read and write the tile in the order the TMA lands it without bank conflicts)
            while (popc(R) < RB) {
                int best = -1, best_score = -1;
                for (int b = K - 1; b >= 0; --b) {
                    if (R >> b & 1) continue;
                    const int score = thread_residue_count(R, b % res_mod);
                    if (score > best_score) {
                        best_score = score;
                        best = b;
                    }
                }
                R |= 1u << best;
            }
            StageDesc sd{};
            std::vector<int> rl;
            for (int b = 0; b < K; ++b)
                if (R >> b & 1) rl.push_back(b);
            // register positions: dense targets first in op order are not needed; ascending is fine
            for (int i = 0; i < RB; ++i) sd.rbits[i] = int8_t(rl[i]);
            std::vector<int> tl;
            for (int b = 0; b < K; ++b)
                if (!(R >> b & 1)) tl.push_back(b);
            // lanes first: one thread bit of each residue class, then the rest ascending
            std::vector<int> order;
            std::vector<char> used(tl.size(), 0);
            for (int r = 0; r < res_mod; ++r)
                for (size_t i = 0; i < tl.size(); ++i)
                    if (!used[i] && tl[i] % res_mod == r) {
                        order.push_back(tl[i]);
                        used[i] = 1;
                        break;
                    }
            for (size_t i = 0; i < tl.size(); ++i)
                if (!used[i]) order.push_back(tl[i]);
            for (int i = 0; i < TB; ++i) sd.tbits[i] = int8_t(order[i]);
            int pos_of[32];
            for (int i = 0; i < 32; ++i) pos_of[i] = -1;
            for (int i = 0; i < RB; ++i) pos_of[rl[i]] = i;
            sd.op_begin = int(stage_ops.size()) - sop_begin;
            for (int i : members) {
                const PassOp &po = s.pass_ops[p.op_begin + i];
                const DevOp &dop = ops[po.op];
                StageOp so{};
                so.op = po.op;
                so.lslot = po.lslot;
                so.grad_mask = dop.grad_mask;
                so.n_angles = dop.grad_mask ? dop.n_angles : 0;
                so.mat_size = dop.mat_size;
                so.moff = mtab;
                so.mcount = dop.mat_size * (1 + so.n_angles);
                so.msrc = dop.mat_off;
                so.msrc_ps = dop.per_sample;
                mtab += so.mcount;
                so.octrl = po.octrl;
                so.rctrl = 0;
                so.tctrl = 0;
                for (int b = 0; b < K; ++b) {
                    if (!(po.lctrl >> b & 1)) continue;
                    if (pos_of[b] >= 0)
                        so.rctrl |= 1u << pos_of[b];
                    else
                        so.tctrl |= 1u << b;
                }
                if (po.kind == KIND_DENSE) {
                    so.kind = po.m == 1 ? SK_DENSE1 : SK_DENSE2;
                    if (po.m == 1 && dop.sub == SUB_REAL) so.kind = SK_REAL1;
                    if (po.m == 1 && dop.sub == SUB_PERM) so.kind = SK_PERM1;
                    if (po.m == 1 && dop.sub == SUB_SWAP) so.kind = SK_SWAP1;
                    if (po.m == 1 && dop.sub == SUB_RXL) so.kind = SK_RXL1;
                    so.p0 = pos_of[po.lt[0]];
                    so.p1 = po.m == 2 ? pos_of[po.lt[1]] : 0;
                } else {
                    so.kind = po.m == 1 ? SK_DIAG1 : SK_DIAG2;
                    so.dsrc[1] = 3;   // absent second target
                    so.dval[1] = 0;
                    for (int k = 0; k < po.m; ++k) {
                        if (po.lt[k] >= 0 && pos_of[po.lt[k]] >= 0) {
                            so.dsrc[k] = 0;
                            so.dval[k] = pos_of[po.lt[k]];
                        } else if (po.lt[k] >= 0) {
                            so.dsrc[k] = 1;
                            so.dval[k] = po.lt[k];
                        } else {
                            so.dsrc[k] = 2;
                            so.dval[k] = po.gt[k];
                        }
                    }
                }
                assign_codes(so);
                stage_ops.push_back(so);
                done[i] = 1;
                ++n_done;
            }
            sd.op_end = int(stage_ops.size()) - sop_begin;
            stages.push_back(sd);
        }
        if (forward) {
            p.f_reg_bits = RB;
            p.f_stage_begin = stage_begin;
            p.f_n_stages = int(stages.size()) - stage_begin;
            p.f_sop_begin = sop_begin;
            p.f_n_sops = int(stage_ops.size()) - sop_begin;
            p.f_mtab_entries = mtab;
        } else {
            p.reg_bits = RB;
            p.thread_bits = TB;
            p.stage_begin = stage_begin;
            p.n_stages = int(stages.size()) - stage_begin;
            p.sop_begin = sop_begin;
            p.n_sops = int(stage_ops.size()) - sop_begin;
            p.mtab_entries = mtab;
        }
    }
}

void build_ham_groups(int n, int K, int c, const std::vector<uint64_t> &mx, const std::vector<uint64_t> &my,
                      const std::vector<uint64_t> &mz, const std::vector<int> &ny, const std::vector<double> &coeff,
                      std::vector<HamGroup> &groups, std::vector<HamClass> &classes, std::vector<HamTerm> &terms) {
    if (K > n) K = n;
    if (c > K) c = K;
    const int T = int(coeff.size());
    // classes: distinct flip masks, in order of first appearance
    std::vector<uint64_t> flips;
    std::vector<std::vector<int>> members;
    for (int t = 0; t < T; ++t) {
        const uint64_t f = mx[t] | my[t];
        auto it = std::find(flips.begin(), flips.end(), f);
        if (it == flips.end()) {
            flips.push_back(f);
            members.push_back({t});
        } else {
            members[it - flips.begin()].push_back(t);
        }
    }
    // split oversized classes
    std::vector<uint64_t> cflip;
    std::vector<std::vector<int>> cmem;
    for (size_t i = 0; i < flips.size(); ++i) {
        for (size_t s = 0; s < members[i].size(); s += kMaxClassTerms) {
            cflip.push_back(flips[i]);
            cmem.emplace_back(members[i].begin() + s,
                              members[i].begin() + std::min(members[i].size(), s + size_t(kMaxClassTerms)));
        }
    }
    const uint64_t all = n >= 64 ? ~uint64_t(0) : ((uint64_t(1) << n) - 1);
    std::vector<char> used(cflip.size(), 0);
    size_t n_used = 0;
    while (n_used < cflip.size()) {
        uint64_t Q = (n <= K) ? all : ((uint64_t(1) << c) - 1);
        std::vector<int> in_group;
        for (size_t i = 0; i < cflip.size() && int(in_group.size()) < kMaxGroupClasses; ++i) {
            if (used[i]) continue;
            if (popc(Q | cflip[i]) <= K) {
                Q |= cflip[i];
                in_group.push_back(int(i));
                used[i] = 1;
                ++n_used;
            }
        }
        if (in_group.empty()) throw std::runtime_error("Pauli term acts on more qubits than a tile holds");
        for (int q = 0; q < n && popc(Q) < K; ++q) Q |= uint64_t(1) << q;
        std::vector<int> qb;
        for (int q = 0; q < n; ++q)
            if (Q >> q & 1) qb.push_back(q);
        HamGroup g{};
        g.geom = make_geom(n, qb);
        g.class_begin = int(classes.size());
        g.class_count = int(in_group.size());
        for (int ci : in_group) {
            HamClass hc{};
            hc.flip = cflip[ci];
            hc.lflip = 0;
            for (int i = 0; i < g.geom.K; ++i)
                if (hc.flip >> g.geom.qbits[i] & 1) hc.lflip |= 1u << i;
            hc.term_begin = int(terms.size());
            hc.term_count = int(cmem[ci].size());
            const int K = g.geom.K;
            const int shift = std::max(0, K - kHamRegBits);
            std::vector<HamTerm> ts;
            for (int t : cmem[ci]) {
                HamTerm ht{};
                ht.coeff = coeff[t];
                ht.my_mz = my[t] | mz[t];
                ht.ny = ny[t];
                ht.lmask = 0;
                for (int i = 0; i < K; ++i)
                    if (ht.my_mz >> g.geom.qbits[i] & 1) ht.lmask |= 1u << i;
                uint64_t tile_q = 0;
                for (int i = 0; i < K; ++i) tile_q |= uint64_t(1) << g.geom.qbits[i];
                ht.omask = ht.my_mz & ~tile_q;
                // i^ny (ny counts the Y factors, each Y contributing i) and the flip's sign
                const int ph = (ny[t] + 2 * popc(hc.flip & ht.my_mz)) & 3;
                ht.cb_re = ph == 0 ? coeff[t] : ph == 2 ? -coeff[t] : 0.0;
                ht.cb_im = ph == 1 ? coeff[t] : ph == 3 ? -coeff[t] : 0.0;
                ts.push_back(ht);
            }
            auto bin_of = [&](const HamTerm &ht) { return int((ht.lmask >> shift) & ((1u << kHamRegBits) - 1)); };
            std::stable_sort(ts.begin(), ts.end(), [&](const HamTerm &x, const HamTerm &y) { return bin_of(x) < bin_of(y); });
            for (int b = 0, q = 0; b <= (1 << kHamRegBits); ++b) {
                while (q < int(ts.size()) && bin_of(ts[q]) < b) ++q;
                hc.bins[b] = q;
            }
            terms.insert(terms.end(), ts.begin(), ts.end());
            classes.push_back(hc);
        }
        groups.push_back(g);
    }
}

}  // namespace mqb
