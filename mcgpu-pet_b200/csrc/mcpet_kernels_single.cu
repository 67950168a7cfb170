/* Single-scene transport launches: the history loop and the compiled
 * variants of the event loop (plain, uncapped, recording, dose), selected
 * by counters, algorithm and mode. */
#include <cuda_runtime.h>

#include "mcpet_transport.cuh"

namespace mcpet {
using namespace dev;

namespace {

/* Single-scene transport kernel of a run: algorithm, counters, mode. */
EventKernel single_event_kernel(bool counters, int algorithm, int mode) {
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
                             cudaStream_t stream) {
  if (algorithm == kAlgorithmHistories) {
    HistoryKernel k = counters ? history_variant<true>(mode) : history_variant<false>(mode);
    k<<<grid, block, smem, stream>>>(P, T, O);
    return cudaGetLastError();
  }
  EventKernel k = single_event_kernel(counters, algorithm, mode);
  if (!k) return cudaErrorNotSupported;
  k<<<grid, block, smem, stream>>>(P, T, O, nullptr, 0);
  return cudaGetLastError();
}

}  // namespace mcpet
