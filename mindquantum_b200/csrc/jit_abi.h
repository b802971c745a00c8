// Plain structures shared by the host and the tile kernels generated at run time (compiled by
// NVRTC, so only built-in types are used here).
#ifndef MQB_JIT_ABI_H_
#define MQB_JIT_ABI_H_

namespace mqb {

// Tile geometry of a fused pass: K tile qubits qbits[0..K) (the c low ones contiguous in memory)
// and the n - K outside qubits that number the tiles.
struct TileGeom {
    int n;                  // qubits
    int K;                  // tile bits
    int c;                  // contiguity bits
    int n_out;              // outside bits
    signed char qbits[13];
    signed char outside[64];
};

// How the TMA moves one tile: the state (and the batch above it) is seen as a tensor of nd <= 5
// dimensions; dimension j holds the global index bits [shift[j], shift[j+1]) (the last one also
// the batch), and its box covers the tile qubits at the bottom of that range.  Tile qubits that
// got no dimension (n_loop of them, at most when a tile has more than five qubit ranges) are
// fetched as 2^n_loop separate boxes, box v at shared offset v * box_bytes.
struct TmaGeom {
    int nd;
    int n_loop;
    int epa;                // 8-byte tensor elements per amplitude (complex64 1, complex128 2)
    int box_bytes;
    int shift[5];
    int loop_q[13];
};

// Error codes the generated kernels leave in their error word (0: none).
enum { MQB_DEV_ERR_TIMEOUT = 1 };

// Where one op's matrices come from and where they go in the pass's shared-memory table.
struct JitMtab {
    int moff;               // offset in the table (complex entries)
    int mcount;             // entries (M, then dM_0, dM_1, ...)
    long long msrc;         // offset in the per-sample block or the constant pool
    int msrc_ps;            // 1: per-sample matrices, 0: constant pool
    int pad;
};

template <typename V>
struct JitFwdArgs {
    TileGeom g;
    const JitMtab *mt;
    int n_mt;
    int mtab_entries;
    const V *mats;
    long long mats_stride;
    const V *cpool;
    const V *src;           // nullptr: start from |0...0>
    V *dst;
    long long batch;
    long long src_batch_stride;
    TmaGeom tg;
    int *err;               // error word (MQB_DEV_ERR_*), set once
    double *norm;           // nullptr, or [batch][2]: += <psi|psi> of the pass's output in FP64 (re)
};

template <typename V>
struct JitBwdArgs {
    TileGeom g;
    const JitMtab *mt;
    int n_mt;
    int mtab_entries;
    const V *mats;
    long long mats_stride;
    const V *cpool;
    const V *psi_src;       // state after the pass
    V *psi_dst;             // state before the pass (nullptr: not stored)
    V *lam;                 // [n_hams][batch][dim]
    double *gslots;         // [batch][n_slots][n_hams]
    const int *slot_map;    // pass-local slot -> global slot
    int n_slots;
    int n_hams;
    int n_local_slots;
    long long batch;
    TmaGeom tg;
    int *err;
};

}  // namespace mqb

#endif
