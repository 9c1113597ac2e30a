// xmarch.cu -- fused x-march stage kernel (placeholder: not yet enabled).
#include "internal.cuh"

namespace nuosc {

template <typename T>
bool xmarch_supported(const Geom &, bool, XTile) { return false; }
int xmarch_num_vblocks(const Geom &g, XTile t) { return (g.nvs + t.vb - 1) / t.vb; }
template <typename T>
cudaError_t launch_stage_xmarch(const StageArgs<T> &, int, bool, XTile, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t launch_moment_finalize(const double *, double *, Geom, int, cudaStream_t) { return cudaErrorNotSupported; }

template bool xmarch_supported<double>(const Geom &, bool, XTile);
template bool xmarch_supported<float>(const Geom &, bool, XTile);
template cudaError_t launch_stage_xmarch<double>(const StageArgs<double> &, int, bool, XTile, cudaStream_t);
template cudaError_t launch_stage_xmarch<float>(const StageArgs<float> &, int, bool, XTile, cudaStream_t);

XTile autotune_lookup(int, int) { return XTile{16, 64, 32}; }

}  // namespace nuosc
