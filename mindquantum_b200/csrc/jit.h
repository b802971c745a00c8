// Pass kernels generated at run time: each fused pass of a schedule gets its own kernel, in
// which the stage layouts and every gate (kind, register positions, control masks, matrix-table
// offsets, gradient slots) are compile-time constants.  The kernels are compiled with NVRTC for
// sm_100a, cached by source text, and launched with the same arguments the precompiled tile
// kernels take.
#ifndef MQB_JIT_H_
#define MQB_JIT_H_

#include <string>
#include <vector>

#include "mqb_internal.h"

namespace mqb {

// Per pass of `s`: the forward kernel (nullptr for unfused passes).  Compiles what the cache
// lacks, in parallel; throws std::runtime_error with the compiler log on failure.
std::vector<const void *> jit_forward_kernels(const Schedule &s, int precision);
// Per pass of `s`: the backward kernel for n_hams lambdas (`ops`: the program's lowered gates).
std::vector<const void *> jit_backward_kernels(const Schedule &s, int precision, int n_hams,
                                               const std::vector<DevOp> &ops);

size_t jit_forward_smem(const Pass &p, int precision);
size_t jit_backward_smem(const Pass &p, int precision, int n_hams);

// Launch the generated kernel of pass p over every tile of the batch: G consumer groups of
// 2^(K - RB) threads, the TMA tensor maps of the launch's buffers encoded here, and the kernel's
// error word filled in (jit_error_word).
template <typename V>
cudaError_t jit_launch_forward(const void *kernel, JitFwdArgs<V> a, const Pass &p, int precision, int sm_count,
                               cudaStream_t st);
template <typename V>
cudaError_t jit_launch_backward(const void *kernel, JitBwdArgs<V> a, const Pass &p, int precision, int n_hams,
                                int sm_count, cudaStream_t st);

// The error word the generated kernels of the current device report to (MQB_DEV_ERR_*; 0: none),
// allocated on first use.
int *jit_error_word();

// TMA movement of a tile with qubits `qbits` (ascending, qbits[0] == 0), as the generated kernels
// do it: the tensor-map geometry and the shared-memory landing bit of every tile bit, and the
// tensor map (a CUtensorMap, 128 bytes) of the amplitudes at `base` ([outer][2^n]).
void tile_tma_plan(const std::vector<int> &qbits, int precision, TmaGeom *tg, int8_t *land);
void tile_tma_map(void *map, const void *base, int n, long long outer, const std::vector<int> &qbits, int precision);

// Generate and compile (without loading: no GPU needed) the kernels of every fused pass, the
// backward ones too when n_hams > 0; returns the number of distinct kernels.
int jit_compile_check(const Schedule &s, int precision, int n_hams, const std::vector<DevOp> &ops);

// Sources of the kernels of one pass (for tests and inspection).
std::string jit_forward_source(const Schedule &s, const Pass &p, int precision);
std::string jit_backward_source(const Schedule &s, const Pass &p, int precision, int n_hams,
                                const std::vector<DevOp> &ops);

}  // namespace mqb

#endif
