/*
 * mqb200: B200 (sm_100a) state-vector engine for MindQuantum's mqvector path.
 *
 * A C ABI (plain pointers and sizes, integer status codes, no C++ or torch types)
 * over hand-written CUDA kernels.  State buffers are owned by the caller (e.g. torch
 * tensors): a batch of `batch` states, each 2^n interleaved complex numbers
 * (complex64 = 2 x float32, complex128 = 2 x float64), little endian
 * (amplitude index bit q <-> qubit q), contiguous with stride 2^n.
 *
 * The entry points replace the method table of the reference's pybind module
 * (`BindSim`, ccsrc/python/simulator/include/python/vector/bind_vec_state.h:47-83)
 * and the state-vector policy it dispatches to:
 *
 *   mqb_program_create / mqb_apply           <- apply_circuit / apply_gate
 *                                               (VectorState::ApplyCircuit, vector_state.tpp:949-960;
 *                                                ApplyGate, vector_state.tpp:166-437)
 *   mqb_ham_create / mqb_apply_hamiltonian   <- apply_hamiltonian (VectorState::ApplyHamiltonian,
 *                                                vector_state.tpp:963-974; ApplyTerms,
 *                                                cpu_vector_core_policy.cpp:133-161)
 *   mqb_expectation                          <- get_expectation (GetExpectation, vector_state.tpp:712-726;
 *                                                ExpectationOfTerms, cpu_vector_core_policy.cpp:212-261)
 *   mqb_expectation_with_grad                <- get_expectation_with_grad_multi_multi
 *                                               (GradientHelper::HermitianAdjointGradient, gradient.h:100-197)
 *   mqb_vdot                                 <- blas.inner_product / Vdot (cpu_vector_core_dot_like.cpp:33-53)
 *   mqb_sample_indices                       <- sampling_measure_ending_without_noise
 *                                               (vector_state.tpp:1326-1373: cumulative probs + lower bound)
 *   mqb_qubit_one_probability / mqb_collapse <- ApplyMeasure (vector_state.tpp:440-462)
 *
 * Every call returns MQB_OK (0) or a negative MQB_ERR_* code; mqb_last_error() returns
 * the message of the last failure on the calling thread.  Device work is enqueued on
 * the given cudaStream_t (passed as void*); calls return without synchronizing unless
 * they say otherwise.
 */
#ifndef MQB200_H_
#define MQB200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MQB_API __attribute__((visibility("default")))
#else
#define MQB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MQB_OK 0
#define MQB_ERR_INVALID (-1)
#define MQB_ERR_CUDA (-2)
#define MQB_ERR_UNSUPPORTED (-3)
#define MQB_ERR_WORKSPACE (-4)
#define MQB_ERR_ALLOC (-5)

#define MQB_PREC_C64 0  /* complex64 state, FP32 gate arithmetic, FP64 reductions */
#define MQB_PREC_C128 1 /* complex128 state, FP64 everywhere */

#define MQB_MAX_OBJ 6      /* max object qubits of one gate */
#define MQB_MAX_ANGLES 3   /* max parameter expressions of one gate (U3 / Rn) */

/* Gate ids: see mindquantum_b200/csrc/mqb_gate_ids.h (shared with the Python lowering). */

/* One lowered gate.  Parameter expressions: angle[a] = angle_const[a] +
 * sum_{t in [term_begin[a], term_begin[a]+term_count[a])} terms[t].coeff * params[terms[t].param]. */
typedef struct mqb_gate_desc {
    int32_t gate_id;
    int32_t n_obj;
    int32_t obj[MQB_MAX_OBJ];
    uint64_t ctrl_mask;
    int32_t n_angles;
    int32_t grad_angles;          /* bit a set: angle a requires a gradient */
    double angle_const[MQB_MAX_ANGLES];
    int32_t term_begin[MQB_MAX_ANGLES];
    int32_t term_count[MQB_MAX_ANGLES];
    int64_t matrix_offset;        /* constant gates: offset (complex entries) into const_matrices;
                                     custom parameterized gates: offset into the per-sample custom block */
    uint64_t pauli_x, pauli_y, pauli_z; /* rotation about a Pauli string (GID_RPS), global masks */
    int32_t pauli_ny;
    int32_t flags;                /* MQB_GATE_NONUNITARY: the constant matrix is not unitary (the
                                     superoperator of a noise channel on a vectorized density matrix):
                                     it runs in a pass of its own, never inside a fused pass, and
                                     gradients through it need checkpoint stride 1 */
} mqb_gate_desc;

#define MQB_GATE_NONUNITARY 1

typedef struct mqb_param_term {
    int32_t param;
    int32_t flags;   /* bit 0: the parameter requires a gradient */
    double coeff;
} mqb_param_term;

typedef struct mqb_program_options {
    int32_t fuse;          /* 1: fused tile passes (default), 0: one kernel per gate (plain path) */
    int32_t tile_bits;     /* 0: automatic */
    int32_t jit;           /* generated pass kernels: 0 automatic (registers of 18 qubits and more),
                              1 always, -1 never (the precompiled tile kernels) */
    int32_t reserved[5];
} mqb_program_options;

typedef struct mqb_program mqb_program;
typedef struct mqb_hamiltonian mqb_hamiltonian;

typedef struct mqb_program_info {
    int32_t n_qubits;
    int32_t precision;
    int32_t n_ops;
    int32_t n_params;
    int32_t n_passes;        /* passes of the apply schedule */
    int32_t tile_bits;
    int32_t n_grad_slots;    /* gradient angles (per sample per Hamiltonian) */
    int32_t per_sample_entries; /* complex entries of per-sample matrices */
    int32_t custom_entries;  /* complex entries the caller uploads per sample for custom parameterized gates */
    int32_t reserved[7];
} mqb_program_info;

MQB_API const char *mqb_last_error(void);
MQB_API int mqb_version(void);
MQB_API int mqb_device_sm_count(int *out);
/* Per-launch timing of the engine's kernels (CUDA events on the launching stream).  Kinds:
 * 0 fused forward pass, 1 fused backward pass, 2 Hamiltonian pass, 3 matrix generation,
 * 4 per-gate apply, 5 per-gate gradient, 6 gradient scatter, 7 copies and single-state sweeps,
 * 8 row-wise trajectory steps (mqb_rows_*).  mqb_timing_end
 * synchronizes, writes total milliseconds and launch counts per kind and stops timing. */
MQB_API int mqb_timing_begin(void);
MQB_API int mqb_timing_end(double *ms, int64_t *launches, int n_kinds);
/* Error word of the generated pass kernels on the current device: *code = 0, or
 * MQB_DEV_ERR_TIMEOUT (1) when a kernel gave up a wait on its tile pipeline (the call's results
 * are then invalid); clear != 0 resets it.  Synchronizes the device.  No reference counterpart:
 * the reference's kernels have no bounded waits. */
MQB_API int mqb_device_error(int *code, int clear);
/* Fault injection for tests, on the calling thread: after `after` more successful device
 * allocations of the library, the next one fails with MQB_ERR_ALLOC as if the device were out of
 * memory; after < 0 disarms it.  No reference counterpart (the reference does not check its
 * allocations: gpu_vector_core_policy.cu:36-49). */
MQB_API int mqb_inject_alloc_failure(int after);
/* sizeof of mqb_gate_desc, mqb_param_term, mqb_program_options, mqb_program_info (ABI check). */
MQB_API int mqb_abi_struct_sizes(int64_t *out, int n);

/* ------------------------------------------------------------------ programs (circuits) */
MQB_API int mqb_program_create(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates,
                       const mqb_param_term *terms, int n_terms, int n_params, const double *const_matrices,
                       int64_t n_const_entries, const mqb_program_options *options, mqb_program **out);
MQB_API int mqb_program_destroy(mqb_program *prog);
MQB_API int mqb_program_get_info(const mqb_program *prog, mqb_program_info *info);
/* Host-only, no CUDA call: the pass schedule the engine builds for a gate table.  Arrays hold
 * n_gates entries: order = gate indices in execution order, pass_of = pass of each executed gate,
 * qmask / fused / n_stages = tile qubit mask, kind (1 fused tile pass, 0 single-gate pass) and
 * register stages of each pass (n_stages may be NULL). */
MQB_API int mqb_plan_schedule(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates,
                              const double *const_matrices, int64_t n_const_entries, int tile_bits, int fuse,
                              int *n_passes, int32_t *order, int32_t *pass_of, uint64_t *qmask, int32_t *fused,
                              int32_t *n_stages);
/* Passes and tile bits of the schedule mqb_expectation_with_grad uses for n_hams Hamiltonians. */
MQB_API int mqb_program_grad_passes(mqb_program *prog, int n_hams, int *n_passes, int *tile_bits);

/* Generate the pass kernels of a circuit (the forward kernels, and the backward kernels for
 * n_hams lambdas when n_hams > 0) and compile them with NVRTC without loading them, so no GPU is
 * needed; *n_kernels receives the number of distinct kernels.  No counterpart in the reference:
 * a build check of the generated kernels. */
MQB_API int mqb_jit_check(int n_qubits, int precision, const mqb_gate_desc *gates, int n_gates,
                          const double *const_matrices, int64_t n_const_entries, int tile_bits, int n_hams,
                          int *n_kernels);

/* Workspace (bytes) that mqb_apply needs for `batch` samples. */
MQB_API int mqb_apply_workspace_size(const mqb_program *prog, int64_t batch, size_t *bytes);

/* The same as mqb_apply, without a workspace argument and without allocating: for callers that
 * cannot allocate device memory while they apply a circuit (a runtime that reserves all device
 * memory in a fixed pool at start-up, a thin language binding that only owns the state buffers it
 * passes in, a real-time loop that must not call into the allocator).  No counterpart in the
 * reference.  The gate matrices go to a fixed 4 MiB array inside the library (held on every GPU
 * that loads it until exit); batches whose matrices need more are rejected with
 * MQB_ERR_WORKSPACE.  The first call on a device looks the array's address up and caches it (this
 * first call should come before any stream capture); a device reset invalidates that cached
 * address, so the entry point must not be used after cudaDeviceReset.  It runs the precompiled
 * tile kernels only (loading a generated kernel would allocate).  All calls share the array, so
 * calls whose work overlaps on the GPU race. */
MQB_API int mqb_apply_static(mqb_program *prog, void *states, int64_t batch, const double *params,
                             int64_t param_stride, const double *custom, void *stream);

/* Apply the program in place to `batch` states.  params: device [batch][n_params] float64
 * (row stride param_stride, 0 = broadcast one row); custom: device [batch][custom_entries]
 * complex128 (NULL if the program has no custom parameterized gate). */
MQB_API int mqb_apply(mqb_program *prog, void *states, int64_t batch, const double *params, int64_t param_stride,
              const double *custom, void *workspace, size_t workspace_bytes, void *stream);

/* ------------------------------------------------------------------ Hamiltonians */
MQB_API int mqb_ham_create(int n_qubits, int precision, const uint64_t *mask_x, const uint64_t *mask_y,
                   const uint64_t *mask_z, const int32_t *num_y, const double *coeff, int n_terms,
                   mqb_hamiltonian **out);
/* A Hamiltonian given as a sparse 2^n x 2^n matrix in CSR form: indptr [2^n + 1] int64 from 0 to
 * nnz, indices [nnz] int64 column indices, data [nnz] complex (complex64 for MQB_PREC_C64, else
 * complex128), all host arrays, copied to the device.  Every call that takes a Hamiltonian
 * (apply, expectation, adjoint gradient) then applies the matrix with the CSR kernel.  Replaces
 * Hamiltonian(csr_matrix) (HowTo FRONTEND, ccsrc/include/ops/hamiltonian.h:47-49) with
 * Csr_Dot_Vec / ExpectationOfCsr (ccsrc/include/core/sparse/algo.h:160-200,
 * cpu_vector_core_dot_like.cpp:132-222). */
MQB_API int mqb_ham_create_csr(int n_qubits, int precision, int64_t nnz, const int64_t *indptr,
                               const int64_t *indices, const void *data, mqb_hamiltonian **out);
MQB_API int mqb_ham_destroy(mqb_hamiltonian *ham);

/* out = H in (separate buffers), `batch` states. */
MQB_API int mqb_apply_hamiltonian(const mqb_hamiltonian *ham, const void *in, void *out, int64_t batch, void *stream);

/* out[b] = <bra_b| H |ket_b> as (re, im) float64 on the device, out has 2*batch doubles. */
MQB_API int mqb_expectation(const mqb_hamiltonian *ham, const void *bra, const void *ket, int64_t batch, double *out,
                    void *stream);

/* One 2x2 complex matrix (any matrix, not only unitaries) on `qubit` of `batch` states, in place,
 * where every bit of ctrl_mask is set.  matrix: host, 8 doubles, row-major (re, im) pairs.
 * The sweep of ApplySingleQubitMatrix (cpu_vector_core_matrix_gate.cpp:151), used for the
 * operators a noise channel picks: ApplyX/Y/Z, ApplyILike, ApplyXLike, QSMulValue
 * (vector_state.tpp:491-709). */
MQB_API int mqb_apply_matrix1(int n_qubits, int precision, void *states, int64_t batch, int qubit,
                              uint64_t ctrl_mask, const double *matrix, void *stream);

/* One channel step of many noise trajectories, one launch per 256 requests.  Request i acts on
 * state rows[i] of `states` ([batch][2^n]) with its own 2x2 matrix (matrices + 8 i: 8 doubles,
 * row-major (re, im) pairs) on qubits[i] where every bit of ctrl_masks[i] is set.  rows, qubits,
 * ctrl_masks and matrices are host arrays of `count` entries.
 *   mqb_rows_apply_matrix1: every request in place; rows must be distinct.
 *   mqb_rows_matrix1_norm:  out[i] (device float64) = || M_i psi_rows[i] ||^2, states unchanged:
 *     the probability of a Kraus operator, and P(qubit = 1) with M = [[0, 0], [0, 1]].
 * Batched forms of the per-trajectory sweeps of ApplyChannel (vector_state.tpp:465-709) and
 * ApplyMeasure (vector_state.tpp:440-462): the operator ApplyPauliChannel / ApplyKraus /
 * ApplyDampingChannel picks for each trajectory, and the norms its draws compare against. */
MQB_API int mqb_rows_apply_matrix1(int n_qubits, int precision, void *states, int64_t batch, int64_t count,
                                   const int64_t *rows, const int32_t *qubits, const uint64_t *ctrl_masks,
                                   const double *matrices, void *stream);
MQB_API int mqb_rows_matrix1_norm(int n_qubits, int precision, const void *states, int64_t batch, int64_t count,
                                  const int64_t *rows, const int32_t *qubits, const uint64_t *ctrl_masks,
                                  const double *matrices, double *out, void *stream);

/* out[b] = <a_b|b_b> as (re, im) float64 on the device. */
MQB_API int mqb_vdot(int n_qubits, int precision, const void *a, const void *b, int64_t batch, double *out, void *stream);

/* ------------------------------------------------------------------ adjoint gradient */
/* Workspace for mqb_expectation_with_grad with `batch` samples, `n_hams` Hamiltonians and a
 * checkpoint stride (passes between stored states; 1 = every pass, larger saves memory). */
MQB_API int mqb_grad_workspace_size(const mqb_program *prog, int64_t batch, int n_hams, int ckpt_stride, size_t *bytes);

/* For every sample b: psi = U(params_b) init (init = |0..0> when init_states is NULL, else
 * init_states[b] when init_batched, else init_states[0]); f[b][h] = <psi|H_h|psi> as (re, im);
 * grad[b][h][p] = d f / d params[p] (real, the reference's 2 Re <psi|H dU|psi>).
 * f: device [batch][n_hams][2] float64, grad: device [batch][n_hams][n_params] float64. */
/* FP64 norm checks of the complex64 state made by the last mqb_expectation_with_grad or
 * mqb_adjoint_with_lambda call that used this workspace (same batch, n_hams, stride): out[k][b] =
 * <psi_b|psi_b> at check k, for *n_checks checks (0 for complex128 programs).  The checks come
 * after every ceil(sqrt(P))-th forward pass and the last one, then (stride 0 or > 1) at every
 * ceil(sqrt(P))-th state the backward sweep rebuilds by applying passes in reverse.  With out ==
 * NULL only *n_checks is set.  Copies to the host and synchronizes the stream.  No reference
 * counterpart: the reference keeps no record of the norm. */
MQB_API int mqb_grad_norm_checks(mqb_program *prog, const void *workspace, size_t workspace_bytes, int64_t batch,
                                 int n_hams, int stride, double *out, int capacity, int *n_checks, void *stream);
MQB_API int mqb_expectation_with_grad(mqb_program *prog, const mqb_hamiltonian *const *hams, int n_hams,
                              const void *init_states, int init_batched, int64_t batch, const double *params,
                              int64_t param_stride, const double *custom, double *f, double *grad,
                              int ckpt_stride, void *workspace, size_t workspace_bytes, void *stream);

/* Adjoint sweep with a caller-given lambda: grad[b][k] = sum over the gates of
 * Re <lambda_g| dU_g/d param_k |psi_{g-1}>, where psi runs forward from init through the program and
 * lambda starts from `lam` at the end of the circuit ([batch][2^n] when lam_batched, else one state)
 * and is uncomputed with psi.  No factor 2 and no Hamiltonian: the building block of the
 * non-Hermitian gradient <phi| U_l^dag H U_r |psi> (imaginary parts from lambda -> i lambda).
 * Replaces the sweeps of GradientHelper::RightSizeGrad / LeftSizeGrad
 * (ccsrc/include/simulator/vector/gradient.h:160-236).  Workspace: mqb_grad_workspace_size with
 * n_hams = 1. */
MQB_API int mqb_adjoint_with_lambda(mqb_program *prog, const void *lam, int lam_batched, const void *init,
                                    int init_batched, int64_t batch, const double *params, int64_t param_stride,
                                    const double *custom, double *grad, int ckpt_stride, void *ws,
                                    size_t ws_bytes, void *stream);

/* ------------------------------------------------------------------ sampling / measurement */
/* Sorted uniforms u[s] (device float64, ascending) -> amplitude indices out[s] (device int64):
 * out[s] = smallest i with cdf(i) > u[s], cdf(i) = sum_{j<=i} |psi_j|^2 and cdf(dim-1) = 1.
 * scratch: device buffer of at least mqb_sample_scratch_size bytes. */
MQB_API int mqb_sample_scratch_size(int n_qubits, size_t *bytes);
MQB_API int mqb_sample_indices(int n_qubits, int precision, const void *state, const double *sorted_u, int64_t shots,
                       int64_t *out, void *scratch, size_t scratch_bytes, void *stream);

/* out (device float64) = sum of |psi_i|^2 over indices with bit `qubit` set. */
MQB_API int mqb_qubit_one_probability(int n_qubits, int precision, const void *state, int qubit, double *out,
                              void *stream);
/* Keep the half with bit `qubit` == outcome, scale it by `scale`, zero the other half. */
MQB_API int mqb_collapse(int n_qubits, int precision, void *state, int qubit, int outcome, double scale, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MQB200_H_ */
