/* Batched transport launches: the compiled variants of the event loop over
 * the lanes of several scenes (counters, dose, shared scanner / phantom,
 * mode). */
#include <cuda_runtime.h>

#include "mcpet_transport.cuh"

namespace mcpet {
using namespace dev;

namespace {

/* Batched transport kernel: counters, dose, shared scanner/phantom, mode
 * (fast, prompt). */
EventKernel batch_event_kernel(bool counters, bool dose, int share, int mode) {
  if (dose)
    return counters ? event_variant<true, kEventBlocks, false, true, false, true, 0, 11>(mode)
                    : event_variant<false, kEventBlocks, false, true, false, true, 0, 11>(mode);
  if (counters) return event_variant<true, kEventBlocks, false, true, false, false, 0, 11>(mode);
  switch (share) {
    case kShareScanner:
      return event_variant<false, kEventBlocks, false, true, false, false, kShareScanner, 11>(mode);
    case kSharePhantom:
      return event_variant<false, kEventBlocks, false, true, false, false, kSharePhantom, 11>(mode);
    case kShareScanner | kSharePhantom:
      return event_variant<false, kEventBlocks, false, true, false, false, kShareScanner | kSharePhantom, 11>(mode);
    default:
      return event_variant<false, kEventBlocks, false, true, false, false, 0, 11>(mode);
  }
}

}  // namespace

cudaError_t transport_batch_occupancy(bool counters, bool dose, int share, int mode, int block, size_t smem,
                                      int* blocks_per_sm) {
  EventKernel k = batch_event_kernel(counters, dose, share, mode);
  if (!k) return cudaErrorNotSupported;
  return occupancy_of(k, block, smem, blocks_per_sm);
}

cudaError_t launch_transport_batch(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                                   const SceneSlot* slots, int n_slots, bool counters, bool dose, int share, int mode,
                                   int grid, int block, size_t smem, bool after_previous, cudaStream_t stream) {
  EventKernel k = batch_event_kernel(counters, dose, share, mode);
  if (!k) return cudaErrorNotSupported;
  /* after_previous: the launch may start placing blocks while the previous
   * launch on the stream drains its last lanes (programmatic dependent
   * launch; the kernel signals it once a block runs out of lanes) */
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = after_previous ? 1 : 0;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k, P, T, O, slots, n_slots);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace mcpet
