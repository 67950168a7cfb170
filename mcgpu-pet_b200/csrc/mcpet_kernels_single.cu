/* Single-scene transport launches: the history loop and the compiled
 * variants of the event loop (plain, uncapped, recording, dose), selected
 * by counters, algorithm and mode. */
#include <cuda_runtime.h>

#include "mcpet_transport.cuh"

namespace mcpet {
using namespace dev;

namespace {

/* Chained single-scene launches of a batched run (plain event kernel). */
EventKernel chained_event_kernel(int mode) {
  switch (mode) {
    case kTransportChained | 0: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 16>;
    case kTransportChained | 1: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 17>;
    case kTransportChained | 8: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 24>;
    case kTransportChained | 9: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 25>;
    case kTransportChained | 2: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 18>;
    case kTransportChained | 3: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 19>;
    case kTransportChained | 10: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 26>;
    case kTransportChained | 11: return transport_events_kernel<false, kEventBlocks, false, false, false, false, 0, 27>;
    default: return nullptr;
  }
}

/* Single-scene transport kernel of a run: algorithm, counters, mode. */
EventKernel single_event_kernel(bool counters, int algorithm, int mode) {
  if (mode & kTransportChained) return (!counters && algorithm == kAlgorithmEvents) ? chained_event_kernel(mode) : nullptr;
  if (algorithm == kAlgorithmEventsDose)
    return counters ? event_variant<true, kEventBlocks, false, false, false, true, 0, 11>(mode)
                    : event_variant<false, kEventBlocks, false, false, false, true, 0, 11>(mode);
  if (algorithm == kAlgorithmEventsRecord)
    return counters ? event_variant<true, kEventBlocks, false, false, true, false, 0, 9>(mode)
                    : event_variant<false, kEventBlocks, false, false, true, false, 0, 9>(mode);
  if (algorithm == kAlgorithmEventsUncapped)
    return counters ? event_variant<true, 1, false, false, false, false, 0, 9>(mode)
                    : event_variant<false, 1, false, false, false, false, 0, 9>(mode);
  return counters ? event_variant<true, kEventBlocks, false, false, false, false, 0, 15>(mode)
                  : event_variant<false, kEventBlocks, false, false, false, false, 0, 15>(mode);
}

template <bool C>
HistoryKernel history_variant(int mode) {
  switch (mode & 7) {   /* the history loop has no sinogram-only variant */
    case 0: return transport_kernel<C, 0>;
    case 1: return transport_kernel<C, 1>;
    case 2: return transport_kernel<C, 2>;
    case 3: return transport_kernel<C, 3>;
    case 4: return transport_kernel<C, 4>;
    case 5: return transport_kernel<C, 5>;
    case 6: return transport_kernel<C, 6>;
    default: return transport_kernel<C, 7>;
  }
}

}  // namespace

cudaError_t transport_occupancy(bool counters, int algorithm, int mode, int block, size_t smem, int* blocks_per_sm) {
  if (algorithm == kAlgorithmHistories)
    return occupancy_of(counters ? history_variant<true>(mode) : history_variant<false>(mode), block, smem,
                        blocks_per_sm);
  EventKernel k = single_event_kernel(counters, algorithm, mode);
  if (!k) return cudaErrorNotSupported;
  return occupancy_of(k, block, smem, blocks_per_sm);
}

cudaError_t launch_transport(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                             bool counters, int algorithm, int mode, int grid, int block, size_t smem,
                             cudaStream_t stream, bool after_previous) {
  if (algorithm == kAlgorithmHistories) {
    if (after_previous) return cudaErrorNotSupported;
    HistoryKernel k = counters ? history_variant<true>(mode) : history_variant<false>(mode);
    k<<<grid, block, smem, stream>>>(P, T, O);
    return cudaGetLastError();
  }
  EventKernel k = single_event_kernel(counters, algorithm, mode);
  if (!k) return cudaErrorNotSupported;
  if (!after_previous) {
    k<<<grid, block, smem, stream>>>(P, T, O, nullptr, 0);
    return cudaGetLastError();
  }
  /* a launch of a batched run after another: it may start placing blocks
   * while the previous one drains (programmatic dependent launch) */
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const SceneSlot* none = nullptr;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k, P, T, O, none, 0);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace mcpet
