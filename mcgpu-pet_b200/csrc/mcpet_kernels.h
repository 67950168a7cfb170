/* Launch wrappers of the transport and probe kernels (host side). */
#pragma once
#include <cuda_runtime_api.h>
#include <vector_types.h>
#include <stddef.h>
#include <stdint.h>
#include "mcpet_params.h"

namespace mcpet {

constexpr int kAlgorithmHistories = 1;  /* one lane per thread, history after history */
constexpr int kAlgorithmEvents = 2;     /* warp-regrouped event loop, registers capped for occupancy */
constexpr int kAlgorithmEventsUncapped = 3; /* same loop, registers not capped (MCPET_MINBLOCKS=1) */
constexpr int kAlgorithmEventsRecord = 4;   /* event loop that also records tallied coincidences (gradient) */
constexpr int kAlgorithmEventsDose = 5;     /* event loop with the dose tallies */

/* Transport variants (bits of `mode` in the launchers): single-precision
 * direction rotation and decay clock (balanced lanes), the prompt-gamma
 * emitter, loop caps read from the run parameters. */
constexpr int kTransportFast = 1;
constexpr int kTransportPrompt = 2;
constexpr int kTransportCaps = 4;
constexpr int kTransportSinogramOnly = 8;   /* no PSF tally (and no sinogram-dry PSF replays) */
/* automatic balanced lanes: expected decays spread over this many lanes per
 * resident thread (host plans and device-built plans alike) */
constexpr double kAutoLanesPerThread = 6.0;
constexpr int kTransportChained = 16;       /* single-scene launch of a batched run that may follow another
                                               (programmatic dependent launch; seed read from the batch
                                               slot); plain event kernel, no loop caps */

size_t transport_dynamic_smem(const TransportParams& P, int block, int algorithm);
int transport_block_threads();
cudaError_t transport_occupancy(bool counters, int algorithm, int mode, int block, size_t smem, int* blocks_per_sm);
cudaError_t launch_transport(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                             bool counters, int algorithm, int mode, int grid, int block, size_t smem,
                             cudaStream_t stream, bool after_previous = false);

/* batched runs: several scenes in one launch of the batch event kernel.  share:
 * bit 0 = every scene has the launch's scanner (detector, sinogram, tally
 * settings), bit 1 = every scene has the launch's phantom (grid, voxel keys,
 * palette, tables); those are then read from P and T (non-counting,
 * dose-free launches only) */
size_t transport_batch_dynamic_smem(const TransportParams& P, int block);
constexpr int kBatchShareScanner = 1;
constexpr int kBatchSharePhantom = 2;
cudaError_t transport_batch_occupancy(bool counters, bool dose, int share, int mode, int block, size_t smem,
                                      int* blocks_per_sm);
cudaError_t launch_transport_batch(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                                   const SceneSlot* slots, int n_slots, bool counters, bool dose, int share, int mode,
                                   int grid, int block, size_t smem, bool after_previous, cudaStream_t stream);

/* batched regeneration: advance every slot's RANECU seed by `step` within
 * [1, m1 - 1] (the next replay of a captured batch) */
cudaError_t launch_advance_seeds(SceneSlot* slots, int n_slots, int step, cudaStream_t stream);

/* allocation-free runs: lane plan and work-queue words in a static device array */
constexpr int kNoAllocMaxVoxels = 1 << 20;
cudaError_t launch_transport_noalloc(const TransportParams& P, DeviceTables T, DeviceTallies O,
                                     const float* activity, int lane_mode, int tpb, int hpl, int sm_count,
                                     bool counters, int mode, int grid, int block, size_t smem,
                                     cudaStream_t stream);
/* guard trips of the last allocation-free call on the current device */
cudaError_t noalloc_guard_trips(unsigned long long* trips);

/* gradient of the sinogram log-likelihood: replay of the recorded events */
cudaError_t launch_grad_replay(const TransportParams& P, const DeviceTables& T, const uint32_t* events,
                               unsigned long long n_events, const float* y, const int* trues, const int* scatter,
                               const float* bg, const float* activity, float* grad_a, float* grad_s,
                               unsigned long long* stats, int sm_count, int mode, cudaStream_t stream);
cudaError_t launch_loglik(long long nbins, const float* y, const int* trues, const int* scatter, const float* bg,
                          double* out, int sm_count, cudaStream_t stream);

cudaError_t launch_probe_rng(const TransportParams& P, int n, const int64_t* ids, int ndraw, int2* seeds,
                             float* draws, double* ddraws, cudaStream_t s);
cudaError_t launch_probe_detector(const TransportParams& P, int n, const float* e2, const float* e1,
                                  const float3* p2, const float3* p1, const float3* d2, const float3* d1,
                                  const int8_t* s2, const int8_t* s1, int2* seeds, int* out, cudaStream_t s);
cudaError_t launch_probe_compton(const ComptonTable* tab, int n, float* energy, const int* mat, int2* seeds,
                                 double* costh, cudaStream_t s);
cudaError_t launch_probe_rayleigh(const RayleighRows& R, int n, const float* energy, const int* mat,
                                  const float* pmax, int2* seeds, double* costh, cudaStream_t s);
cudaError_t launch_probe_source(const TransportParams& P, int background, int2* seeds, float3* out,
                                cudaStream_t s);

}  // namespace mcpet
