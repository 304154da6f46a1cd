// rbsor_launch.h -- host-visible launch entry points of the solver kernels.
#pragma once

#include <cuda_runtime.h>

#include "rbsor.cuh"

namespace ptk {

// One tile configuration: sweeps per step S, owned tile height th and width tw.
struct TileConfig {
  int S, th, tw;
};

int tile_config_count();
TileConfig tile_config(int idx);
size_t tile_config_smem(int idx);

// k_tile_count + k_assemble + k_init on the stream.
// any_warm: some system has PT_FLAG_WARM_START (adds the guess-rejection pass)
cudaError_t launch_assembly(const KParams &P, const TileConfig &tc, cudaStream_t stream,
                            bool any_warm = false);
// The persistent solve; *grid receives the block count used.
cudaError_t launch_solve(const KParams &P, int cfg, int sms, cudaStream_t stream, int *grid);
// The same in two halves: set the kernel's attributes and size its grid (not a
// stream operation, so it stays outside a stream capture), then launch.
cudaError_t prepare_solve(const KParams &P, int cfg, int sms, int *grid);
cudaError_t launch_prepared(const KParams &P, int cfg, int grid, cudaStream_t stream);
// k_tile_count alone (interior cells and box per tile; reads only the masks).
cudaError_t launch_tile_count(const KParams &P, const TileConfig &tc, cudaStream_t stream);
// spans[2 ty], spans[2 ty + 1] = the first and last tile column of row band ty
// of image sys0 that hold interior cells, or -1, -1 (the solve reads the
// image only there, one pixel around).
cudaError_t launch_band_flags(const KParams &P, int sys0, int *spans, cudaStream_t stream);
// Interleave one image's channels sys0 .. sys0+C-1 into its output.
cudaError_t launch_emit(const KParams &P, int sys0, const TileConfig &tc, long long npx,
                        cudaStream_t stream);

}  // namespace ptk
