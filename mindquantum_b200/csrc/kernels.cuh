// Kernel argument structures and launch wrappers of the mqb200 engine.
#ifndef MQB_KERNELS_CUH_
#define MQB_KERNELS_CUH_

#include "mqb_internal.h"

namespace mqb {

template <typename R>
struct CT;
template <>
struct CT<float> {
    using T = float2;
};
template <>
struct CT<double> {
    using T = double2;
};
template <typename R>
using cplx = typename CT<R>::T;

struct MatgenArgs {
    const DevOp *ops;
    const mqb_gate_desc *descs;
    const mqb_param_term *terms;
    int n_ops;
    const double *params;
    int64_t param_stride;
    const double *custom;      // interleaved complex128, per sample
    int64_t custom_stride;     // complex entries per sample
    int64_t batch;
    void *mats;                // per-sample matrices (cplx<R>)
    int64_t mats_stride;       // complex entries per sample
};

template <typename R>
struct Fwd2Args {
    TileGeom g;
    const StageDesc *stages;
    int n_stages;
    const StageOp *sops;
    int n_ops;
    int reg_bits;
    int mtab_entries;          // complex entries of the shared-memory matrix table
    const cplx<R> *mats;
    int64_t mats_stride;
    const cplx<R> *cpool;
    const cplx<R> *src;        // nullptr: start from |0...0>
    cplx<R> *dst;
    int64_t batch;
    int64_t src_batch_stride;  // 0: every sample starts from the same state
};

template <typename R>
struct Bwd2Args {
    TileGeom g;
    const StageDesc *stages;
    int n_stages;
    const StageOp *sops;
    int n_ops;
    int reg_bits;
    int mtab_entries;          // complex entries of the shared-memory matrix table
    const cplx<R> *mats;
    int64_t mats_stride;
    const cplx<R> *cpool;
    const cplx<R> *psi_src;    // state after the pass
    cplx<R> *psi_dst;          // where to store the state before the pass (nullptr: not needed)
    cplx<R> *lam;              // [n_hams][batch][dim]
    int n_hams;
    double *gslots;            // [batch][n_slots][n_hams]
    int n_slots;
    const int32_t *slot_map;   // pass-local slot -> global slot
    int n_local_slots;
    int64_t batch;
};

template <typename R>
struct HamArgs {
    TileGeom g;
    const HamClass *classes;
    int n_classes;
    const HamTerm *terms;
    int term_begin, n_terms;   // the group's terms: terms[term_begin .. term_begin + n_terms)
    const cplx<R> *ket;
    const cplx<R> *bra;        // used for the expectation accumulation
    cplx<R> *out;              // nullptr: expectation only
    int accumulate;            // out += H ket (else out = H ket)
    double *fout;              // [batch][2] (re, im) accumulators, may be nullptr
    int64_t batch;
    int64_t out_batch_stride;
    int64_t f_stride;          // doubles between samples in fout
};

// launch wrappers (kernels.cu); all return cudaError_t of the launch
template <typename R>
cudaError_t launch_matgen(const MatgenArgs &a, cudaStream_t s);
template <typename R>
cudaError_t launch_fused_fwd2(const Fwd2Args<R> &a, int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_fused_bwd2(const Bwd2Args<R> &a, int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_ham(const HamArgs<R> &a, int sm_count, cudaStream_t s);
// The tile movement of the TMA-ring Hamiltonian pass: how the copies cut a group's tile
// (tensor-map geometry), where tile bit j lands in shared memory, the buffers per operand and the
// error word a bounded wait reports to.
struct HamRingGeom {
    TmaGeom tg;
    int8_t land[kMaxTileBits];
    int nb;
    int stage_prev;   // a group that adds to the output stages the previous sum by TMA too (else reads it)
    int *err;
};
size_t ham_ring_smem(const TileGeom &g, int elem_bytes, int threads, int n_classes, int n_terms, bool staged, int nb);
// map_ket / map_prev: CUtensorMap (128 bytes) of a.ket and of a.out ([batch][2^n] each, the same
// tile geometry); map_prev is used only when the group adds to the output and stages it.
template <typename R>
cudaError_t launch_ham_ring(const HamArgs<R> &a, const HamRingGeom &rg, const void *map_ket, const void *map_prev,
                            int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_plain_apply(cplx<R> *st, int n, int64_t batch, const DevOp &op, const cplx<R> *mats,
                               int64_t mats_stride, const cplx<R> *cpool, bool adjoint, int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_plain_grad(const cplx<R> *psi, const cplx<R> *lam, int n, int64_t batch, int n_hams,
                              const DevOp &op, const cplx<R> *mats, int64_t mats_stride, double *gslots,
                              int n_slots, int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_vdot(const cplx<R> *a, const cplx<R> *b, int n, int64_t batch, double *out, int sm_count,
                        cudaStream_t s);
// A sparse matrix applied to `batch` states (rows = dim = 2^n), kept as slices of 32 rows with
// column-major entries: out[b] = A ket[b] (if out), fout[b * f_stride .. +1] += <bra[b]|A ket[b]>.
template <typename R>
struct CsrArgs {
    const int64_t *slice_ptr;  // [n_slices] first entry of every slice
    const int32_t *slice_len;  // [n_slices] entries per row of the slice (padded)
    const int32_t *cols;       // [entries] column of entry 32 k + lane
    const cplx<R> *vals;       // [entries]
    int64_t dim;
    const cplx<R> *bra;
    const cplx<R> *ket;
    cplx<R> *out;
    double *fout;
    int64_t f_stride;
    int64_t batch;
};
template <typename R>
cudaError_t launch_csr(const CsrArgs<R> &a, int sm_count, cudaStream_t s);
// A 2x2 complex matrix by value, row-major, (re, im) pairs.
struct Mat1 {
    double v[8];
};
template <typename R>
cudaError_t launch_matrix1(cplx<R> *st, int n, int qubit, uint64_t ctrl, int64_t batch, const Mat1 &m, int sm_count,
                           cudaStream_t s);
// One step of many noise trajectories in one launch: request i acts on state row[i] with its own
// 2x2 matrix m[i] on qubit[i] where every bit of ctrl[i] is set.  Passed by value (about 21 KB of
// kernel parameters, within the 32 KB that sm_70 and later accept).
constexpr int kRowOpsMax = 256;
struct RowOps {
    int count;
    int32_t qubit[kRowOpsMax];
    uint64_t ctrl[kRowOpsMax];
    int64_t row[kRowOpsMax];
    double m[kRowOpsMax][8];
};
// norm_out == nullptr: apply every request in place (rows distinct); otherwise norm_out[i] =
// || M_i psi_row[i] ||^2 and the states stay as they are.
template <typename R>
cudaError_t launch_row_ops(cplx<R> *st, int n, const RowOps &ops, double *norm_out, int sm_count, cudaStream_t s);
template <typename R>
cudaError_t launch_copy_or_zero(cplx<R> *dst, const cplx<R> *src, int n, int64_t batch, int64_t src_stride,
                                cudaStream_t s);
cudaError_t launch_grad_scatter(const double *gslots, int64_t batch, int n_slots, int n_hams, const int32_t *csr_ptr,
                                const int32_t *csr_slot, const double *csr_coeff, int n_params, double scale, double *grad,
                                cudaStream_t s);
template <typename R>
cudaError_t launch_chunk_probs(const cplx<R> *st, int n, int chunk_bits, double *sums, cudaStream_t s);
cudaError_t launch_prefix(double *sums, int64_t n, cudaStream_t s);
template <typename R>
cudaError_t launch_sample_search(const cplx<R> *st, int n, int chunk_bits, const double *prefix,
                                 const double *u, int64_t shots, int64_t *out, cudaStream_t s);
template <typename R>
cudaError_t launch_one_prob(const cplx<R> *st, int n, int q, double *out, cudaStream_t s);
template <typename R>
cudaError_t launch_collapse(cplx<R> *st, int n, int q, int outcome, double scale, cudaStream_t s);

size_t fused2_smem(const TileGeom &g, int n_tiles_in_smem, int n_stages, int n_stage_ops, int n_local_slots,
                   int n_hams, int elem_bytes, int threads, int mtab_entries);
size_t ham_smem(const TileGeom &g, int elem_bytes);

}  // namespace mqb
#endif
