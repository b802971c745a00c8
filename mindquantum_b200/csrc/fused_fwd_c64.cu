// Fused tile kernels: the forward pass at complex64 precision.
#include "fused_impl.cuh"

namespace mqb {
template cudaError_t launch_fused_fwd2<float>(const Fwd2Args<float> &, int, cudaStream_t);
}  // namespace mqb

namespace mqb {
size_t fused2_smem(const TileGeom &g, int n_tiles_in_smem, int n_stages, int n_stage_ops, int n_local_slots,
                   int n_hams, int elem_bytes, int threads, int mtab_entries) {
    size_t s = (size_t(1) << g.K) * elem_bytes * n_tiles_in_smem;
    s = (s + 15) & ~size_t(15);
    s += size_t(mtab_entries) * elem_bytes;
    s = (s + 15) & ~size_t(15);
    s += (size_t(1) << (g.K - g.c)) * sizeof(uint64_t);
    s = (s + 15) & ~size_t(15);
    s += size_t(n_stages) * sizeof(StageDesc);
    s = (s + 15) & ~size_t(15);
    s += size_t(n_stage_ops) * sizeof(StageOp);
    s = (s + 15) & ~size_t(15);
    if (n_hams > 0) s += size_t(threads / 32) * std::max(1, n_local_slots) * n_hams * sizeof(double);
    return s;
}
}  // namespace mqb
