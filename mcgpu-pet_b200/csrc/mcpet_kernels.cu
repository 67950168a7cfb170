/* Launch wrappers of the transport kernels, and the probe, gradient and
 * allocation-free kernels (sm_100a).  The transport kernels themselves are
 * in mcpet_transport.cuh; their single-scene event-loop variants are compiled
 * in mcpet_kernels_single.cu and the batched ones in mcpet_kernels_batch.cu.
 *
 * transport_kernel is a persistent grid (a multiple of the SM count): every
 * thread repeatedly claims the next lane of the lane plan through a
 * warp-aggregated atomic on a global cursor and runs that lane to the end of
 * the acquisition time (the reference runs one lane per hardware thread of a
 * one-block-per-voxel grid, MCGPU-PET.cu:457-483).  Lanes are ordered by
 * decreasing expected work so the longest start first.  The Compton shell
 * table, the material palette and the energy spectrum live in shared memory;
 * sinogram and image increments are global int32 reductions.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>

#include "mcpet_transport.cuh"

namespace mcpet {
using namespace dev;

namespace {

/* ---------------------------------------------------------- probes */

__global__ void probe_rng_kernel(TransportParams P, int n, const int64_t* ids, int ndraw, int2* seeds,
                                 float* draws, double* ddraws) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rng r = rng_stream(P, (uint64_t)ids[i]);
  seeds[i] = make_int2(r.x, r.y);
  Rng r2 = r;
  for (int d = 0; d < ndraw; ++d) draws[(size_t)i * ndraw + d] = ranecu(r);
  for (int d = 0; d < ndraw; ++d) ddraws[(size_t)i * ndraw + d] = ranecu_double(r2);
}

__global__ void probe_detector_kernel(TransportParams P, DeviceTallies O, int n, const float* e2, const float* e1,
                                      const float3* p2, const float3* p1, const float3* d2, const float3* d1,
                                      const int8_t* s2, const int8_t* s1, int2* seeds, int* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PhotonState b, a;
  b.pos = p2[i]; b.dir = d2[i]; b.energy = e2[i]; b.state = s2[i]; b.travel = 0.f;
  a.pos = p1[i]; a.dir = d1[i]; a.energy = e1[i]; a.state = s1[i]; a.travel = 0.f;
  Rng rng;
  rng.x = seeds[i].x;
  rng.y = seeds[i].y;
  int* o = out + 6 * i;
  o[0] = -1; o[1] = 0; o[2] = -1; o[3] = -1;
  float xb, yb, zb, xa, ya, za;
  to_cylinder(P, b.pos, b.dir, xb, yb, zb);
  float phib = atan2f(yb, xb);
  if (fabsf(zb) < 0.5f * P.height) {
    to_cylinder(P, a.pos, a.dir, xa, ya, za);
    float phia = atan2f(ya, xa);
    if (fabsf(za) < 0.5f * P.height) {
      long long bin = sinogram_bin(P, phib, zb, phia, za);
      if (bin >= 0) {
        float g1 = blur_sinogram(rng);
        float g2 = blur_sinogram(rng);
        float eb = b.energy + (P.e_resol / 2.35f) * b.energy * g1;
        float ea = a.energy + (P.e_resol / 2.35f) * a.energy * g2;
        int ib = __float2int_rd(eb / 1000.0f);
        int ia = __float2int_rd(ea / 1000.0f);
        if ((ib < P.ne) && (ib >= 0)) o[2] = ib;
        if ((ia < P.ne) && (ia >= 0)) o[3] = ia;
        if (eb > P.e_low && eb < P.e_high && ea > P.e_low && ea < P.e_high) {
          o[0] = (int)bin;
          o[1] = (b.state == 0 && a.state == 0) ? 1 : 2;
        }
      }
    }
  }
  o[4] = rng.x;
  o[5] = rng.y;
}

__global__ void probe_compton_kernel(const ComptonTable* tab, int n, float* energy, const int* mat, int2* seeds,
                                     double* costh, int max_shells) {
  __shared__ ComptonTable cmp;
  extern __shared__ float4 dyn_smem[];
  {
    const int* src = reinterpret_cast<const int*>(tab);
    int* dst = reinterpret_cast<int*>(&cmp);
    for (int i = threadIdx.x; i < (int)(sizeof(ComptonTable) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  SharedScratch rn{reinterpret_cast<float*>(dyn_smem) + threadIdx.x, (int)blockDim.x};
  Rng r;
  r.x = seeds[i].x;
  r.y = seeds[i].y;
  float e = energy[i];
  double c = 0.0;
  sample_compton(r, e, mat[i], cmp, rn, c);
  energy[i] = e;
  costh[i] = c;
  seeds[i] = make_int2(r.x, r.y);
}

__global__ void probe_rayleigh_kernel(RayleighRows R, int n, const float* energy, const int* mat, const float* pmax,
                                      int2* seeds, double* costh) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rng r;
  r.x = seeds[i].x;
  r.y = seeds[i].y;
  double c = 0.0;
  sample_rayleigh(r, energy[i], mat[i], pmax[i], R, c);
  costh[i] = c;
  seeds[i] = make_int2(r.x, r.y);
}

template <bool kFast>
__global__ void probe_source_kernel(TransportParams P, int background, int2* seeds, float3* out) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if ((long long)v >= P.n_voxels) return;
  int vx = v % P.nx, vy = (v / P.nx) % P.ny, vz = v / (P.nx * P.ny);
  Rng r;
  r.x = seeds[v].x;
  r.y = seeds[v].y;
  float3 pos, dir, dir2;
  emit_first(r, P, vx, vy, vz, pos, dir);
  emit_second<kFast>(r, background != 0, dir, dir2);
  out[4 * v + 0] = pos;
  out[4 * v + 1] = dir;
  out[4 * v + 2] = pos;
  out[4 * v + 3] = dir2;
  seeds[v] = make_int2(r.x, r.y);
}

/* ------------------------------------------------------ gradient
 *
 * The Poisson log-likelihood of a measured sinogram y under the model
 * lambda = trues + scatter (the forward transport) + background r:
 *   L = sum_b  y_b ln(lambda_b) - lambda_b.
 * Its gradient with respect to the voxel activities and density scales is
 * estimated from the tallied coincidences of the forward run, which recorded
 * for each one the RANECU state at its emission, its voxel and its bin
 * (EventRecord).  With w_b = y_b / lambda_b - 1:
 *   dL/dA_v = sum over events e from voxel v of w_b(e) / A_v
 * (event back-tallying: lambda is linear in A), and
 *   dL/ds_v = sum over events e of w_b(e) * S_v(e)
 * (path-replay score function): S_v(e) sums, over the Woodcock steps of the
 * event's two photons inside voxel v, d ln p(step) / d ln rho_v -- +1 for a
 * real interaction, -p_real/(1-p_real) for a virtual one (the majorant is
 * held fixed; the interaction type and everything after it do not depend on
 * rho_v).  Each history is recomputed from its RNG state instead of being
 * stored; a replay whose photons do not land in the recorded bin is counted
 * and left out of dL/ds (dL/dA needs no replay). */

constexpr int kReplaySteps = 96;   /* voxel runs one replayed pair may visit */

struct ScoreList {
  int vox[kReplaySteps];
  float score[kReplaySteps];
  int n;
  bool overflow;
  __device__ __forceinline__ void operator()(int v, bool real, float prob_virtual) {
    const float sc = real ? 1.0f : (prob_virtual > 0.0f ? -(1.0f - prob_virtual) / prob_virtual : 0.0f);
    if (n > 0 && vox[n - 1] == v) {
      score[n - 1] += sc;
    } else if (n < kReplaySteps) {
      vox[n] = v;
      score[n] = sc;
      ++n;
    } else {
      overflow = true;
    }
  }
};

template <int kMode>
__global__ void __launch_bounds__(kBlock) grad_replay_kernel(TransportParams P, DeviceTables T, const uint32_t* events,
                                                             unsigned long long n_events, const float* y,
                                                             const int* trues, const int* scatter, const float* bg,
                                                             const float* activity, float* grad_a, float* grad_s,
                                                             unsigned long long* stats) {
  __shared__ ComptonTable cmp;
  extern __shared__ float4 dyn_smem[];
  float* scratch = reinterpret_cast<float*>(dyn_smem);
  {
    const int* src = reinterpret_cast<const int*>(T.compton);
    int* dst = reinterpret_cast<int*>(&cmp);
    for (int i = threadIdx.x; i < (int)(sizeof(ComptonTable) / 4); i += blockDim.x) dst[i] = __ldg(&src[i]);
  }
  __syncthreads();
  SharedScratch rn{scratch + threadIdx.x, (int)blockDim.x};
  const bool background = P.background_mode != 0;
  unsigned long long ok_count = 0, bad_count = 0;
  LaneCounters cnt = {};
  ScoreList h;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n_events;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t* r = events + 6 * i;
    Rng rng = {(int)r[0], (int)r[1]};
    const int voxel = (int)r[2];
    const long long bin = (long long)(((unsigned long long)r[5] << 32) | r[4]);
    const float lam = (float)(__ldg(&trues[bin]) + __ldg(&scatter[bin])) + (bg ? __ldg(&bg[bin]) : 0.0f);
    const float w = __ldg(&y[bin]) / lam - 1.0f;
    if (grad_a) atomicAdd(&grad_a[voxel], w / __ldg(&activity[voxel]));
    if (!grad_s) continue;
    h.n = 0;
    h.overflow = false;
    PhotonState a, b;
    emit_first(rng, P, voxel % P.nx, (voxel / P.nx) % P.ny, voxel / (P.nx * P.ny), a.pos, a.dir);
    const float3 origin = a.pos, dir0 = a.dir;
    a.energy = kAnnihilation;
    a.travel = 0.0f;
    a.state = 0;
    const bool esc_a = track_photon<false, kMode>(rng, P, T, T.palette, cmp, rn, a, cnt, &h);
    emit_second<(kMode & kModeFast) != 0>(rng, background, dir0, b.dir);
    b.pos = origin;
    b.energy = kAnnihilation;
    b.travel = 0.0f;
    b.state = 0;
    const bool esc_b = track_photon<false, kMode>(rng, P, T, T.palette, cmp, rn, b, cnt, &h);
    /* the replayed pair must land in the recorded bin (geometry of the
     * sinogram tally, MCGPU-PET_kernel.cu:1645-1791) */
    bool ok = esc_a && esc_b && !h.overflow;
    if (ok) {
      float xb, yb, zb, xa, ya, za;
      to_cylinder(P, b.pos, b.dir, xb, yb, zb);
      const float phib = atan2f(yb, xb);
      to_cylinder(P, a.pos, a.dir, xa, ya, za);
      const float phia = atan2f(ya, xa);
      ok = fabsf(zb) < 0.5f * P.height && fabsf(za) < 0.5f * P.height &&
           sinogram_bin<(kMode & kModeFast) != 0>(P, phib, zb, phia, za) == bin;
    }
    if (!ok) {
      ++bad_count;
      continue;
    }
    ++ok_count;
    for (int k = 0; k < h.n; ++k) atomicAdd(&grad_s[h.vox[k]], w * h.score[k]);
  }
  if (ok_count) atomicAdd(&stats[0], ok_count);
  if (bad_count) atomicAdd(&stats[1], bad_count);
}

/* L = sum_b y_b ln(lambda_b) - lambda_b: FP32 partials per thread and per
 * block, one FP64 atomic per block. */
__global__ void __launch_bounds__(256) loglik_kernel(long long nbins, const float* y, const int* trues,
                                                     const int* scatter, const float* bg, double* out) {
  float acc = 0.0f;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nbins;
       b += (long long)gridDim.x * blockDim.x) {
    const float lam = (float)(trues[b] + scatter[b]) + (bg ? bg[b] : 0.0f);
    const float yb = y[b];
    if (lam > 0.0f) acc += (yb > 0.0f ? yb * logf(lam) : 0.0f) - lam;
  }
  __shared__ float part[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    atomicAdd(out, (double)t);
  }
}

/* ------------------------------------------------ allocation-free runs
 *
 * Scratch of mcpet_run_device_noalloc: the lane plan (built on the device
 * from the caller's activity map) and the work-queue words live in this one
 * file-scope device array instead of library allocations.  Its size is fixed
 * at build time (kNoAllocMaxVoxels emitters of 32 bytes plus a small header,
 * about 32 MiB) and every GPU that loads the library holds it until the
 * process exits.  All calls on a device share it: calls that overlap on the
 * GPU race on it.  Each call rewrites the header and the plan it uses. */

constexpr int kPlanChunk = 4096;                                  /* voxels per plan block */
constexpr int kPlanMaxChunks = kNoAllocMaxVoxels / kPlanChunk;

/* header words */
enum : int {
  kHdrCursor = 0,       /* lane work queue */
  kHdrGuard = 1,        /* guard trips of the call (plan limit + transport guards) */
  kHdrLanes = 2,        /* lanes of the plan (kernel reads [2], [3]) */
  kHdrEmitters = 3,
  kHdrCoinc = 4,        /* coincidence counter when the caller passes none */
  kHdrHpl = 5,          /* decays per balanced lane used by the plan */
};

struct NoAllocScratch {
  unsigned long long header[8];
  unsigned long long chunk_lanes[kPlanMaxChunks];
  unsigned int chunk_emitters[kPlanMaxChunks];
  int chunk_last_voxel[kPlanMaxChunks];    /* highest emitting voxel of the chunk, -1 if none */
  double chunk_activity[kPlanMaxChunks];   /* activity of the chunk's emitting voxels */
  Emitter plan[kNoAllocMaxVoxels];
};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

__device__ __forceinline__ unsigned long long plan_lanes_of(float a, int mode, int tpb, double t_s,
                                                            unsigned long long hpl) {
  if (mode == 0) return (unsigned long long)tpb;
  double L = ceil((double)a * t_s / (double)hpl);
  if (L < 1) L = 1;
  if (L > 1.0e8) L = 1.0e8;
  return (unsigned long long)L;
}

/* per chunk of voxels: emitters, their activity and the last emitting voxel */
__global__ void plan_count_kernel(const float* act, int nvox, NoAllocScratch* S) {
  __shared__ double sa[32];
  __shared__ unsigned int se[32];
  __shared__ int sv[32];
  const int v0 = blockIdx.x * kPlanChunk, v1 = min(v0 + kPlanChunk, nvox);
  unsigned int ne = 0;
  double asum = 0.0;
  int vlast = -1;
  for (int v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
    float a = act[v];
    if (a > 1.0e-7f) {
      ne += 1;
      asum += (double)a;
      vlast = v;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    ne += __shfl_down_sync(0xffffffffu, ne, o);
    asum += __shfl_down_sync(0xffffffffu, asum, o);
    vlast = max(vlast, __shfl_down_sync(0xffffffffu, vlast, o));
  }
  if ((threadIdx.x & 31) == 0) {
    se[threadIdx.x >> 5] = ne;
    sa[threadIdx.x >> 5] = asum;
    sv[threadIdx.x >> 5] = vlast;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int te = 0;
    double ta = 0.0;
    int tv = -1;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      te += se[w];
      ta += sa[w];
      tv = max(tv, sv[w]);
    }
    S->chunk_emitters[blockIdx.x] = te;
    S->chunk_activity[blockIdx.x] = ta;
    S->chunk_last_voxel[blockIdx.x] = tv;
  }
}

/* decays per balanced lane: the caller's value, or the automatic one from
 * the activity map on the device (expected decays over kAutoLanesPerThread
 * lanes per resident thread, clamped to [1, 4096], as on the host) */
__global__ void plan_hpl_kernel(int n_chunks, double t_s, int hpl, double resident_threads, NoAllocScratch* S) {
  if (threadIdx.x != 0) return;
  unsigned long long h = (unsigned long long)(hpl > 0 ? hpl : 1);
  if (hpl <= 0) {
    double A = 0.0;
    for (int c = 0; c < n_chunks; ++c) A += S->chunk_activity[c];
    double x = A * t_s / (resident_threads * kAutoLanesPerThread);
    if (x < 1) x = 1;
    if (x > 4096) x = 4096;
    h = (unsigned long long)(int)x;
  }
  S->header[kHdrHpl] = h;
}

/* per chunk of voxels: lanes */
__global__ void plan_lanes_kernel(const float* act, int nvox, int mode, int tpb, double t_s, NoAllocScratch* S) {
  __shared__ unsigned long long sl[32];
  const unsigned long long hpl = S->header[kHdrHpl];
  const int v0 = blockIdx.x * kPlanChunk, v1 = min(v0 + kPlanChunk, nvox);
  unsigned long long nl = 0;
  for (int v = v0 + threadIdx.x; v < v1; v += blockDim.x) {
    float a = act[v];
    if (a > 1.0e-7f) nl += plan_lanes_of(a, mode, tpb, t_s, hpl);
  }
  for (int o = 16; o > 0; o >>= 1) nl += __shfl_down_sync(0xffffffffu, nl, o);
  if ((threadIdx.x & 31) == 0) sl[threadIdx.x >> 5] = nl;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tl = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tl += sl[w];
    S->chunk_lanes[blockIdx.x] = tl;
  }
}

/* Exclusive prefix over the chunks, totals, and the words that start at
 * zero.  A plan whose RANECU streams reach 2^31 (the reference's 31-bit
 * thread ids; stream = lane index for balanced lanes, voxel *
 * threads_per_block + thread for reference lanes) runs nothing: the call
 * counts a guard trip, in its guard word and, when counters are collected,
 * in counters[9]. */
__global__ void plan_scan_kernel(int n_chunks, int mode, int tpb, NoAllocScratch* S, unsigned long long* counters) {
  if (threadIdx.x != 0) return;
  unsigned long long lanes = 0;
  unsigned int emitters = 0;
  int last = -1;
  for (int c = 0; c < n_chunks; ++c) {
    unsigned long long l = S->chunk_lanes[c];
    unsigned int e = S->chunk_emitters[c];
    S->chunk_lanes[c] = lanes;
    S->chunk_emitters[c] = emitters;
    lanes += l;
    emitters += e;
    last = max(last, S->chunk_last_voxel[c]);
  }
  S->header[kHdrCursor] = 0;
  S->header[kHdrGuard] = 0;
  S->header[kHdrCoinc] = 0;
  const unsigned long long streams =
      (mode == 0) ? (last < 0 ? 0ull : ((unsigned long long)last + 1) * (unsigned long long)tpb) : lanes;
  if (streams >= (1ull << 31)) {
    S->header[kHdrGuard] = 1;
    if (counters) counters[9] += 1;
    lanes = 0;
    emitters = 0;
  }
  S->header[kHdrLanes] = lanes;
  S->header[kHdrEmitters] = emitters;
}

/* emitter records in voxel order (one block per chunk, block-wide scans) */
__global__ void plan_fill_kernel(const float* act, int nvox, int mode, int tpb, double t_s, NoAllocScratch* S) {
  __shared__ unsigned int we[32];
  __shared__ unsigned long long wl[32];
  __shared__ unsigned int run_e;
  __shared__ unsigned long long run_l;
  const unsigned long long hpl = S->header[kHdrHpl];
  if (S->header[kHdrLanes] == 0) return;   /* empty or refused plan */
  const int c = blockIdx.x;
  const int v0 = c * kPlanChunk, v1 = min(v0 + kPlanChunk, nvox);
  if (threadIdx.x == 0) {
    run_e = S->chunk_emitters[c];
    run_l = S->chunk_lanes[c];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = v0; base < v1; base += blockDim.x) {
    const int v = base + threadIdx.x;
    float a = (v < v1) ? act[v] : 0.0f;
    const bool emit = a > 1.0e-7f;
    unsigned int e = emit ? 1u : 0u;
    unsigned long long l = emit ? plan_lanes_of(a, mode, tpb, t_s, hpl) : 0ull;
    /* inclusive warp scans */
    unsigned int ie = e;
    unsigned long long il = l;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned int te = __shfl_up_sync(0xffffffffu, ie, o);
      unsigned long long tl = __shfl_up_sync(0xffffffffu, il, o);
      if (lane >= o) {
        ie += te;
        il += tl;
      }
    }
    if (lane == 31) {
      we[warp] = ie;
      wl[warp] = il;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int acc_e = 0;
      unsigned long long acc_l = 0;
      for (int w = 0; w < nw; ++w) {
        unsigned int te = we[w];
        unsigned long long tl = wl[w];
        we[w] = acc_e;
        wl[w] = acc_l;
        acc_e += te;
        acc_l += tl;
      }
      we[31] = acc_e;           /* tile totals (nw <= 8 < 31) */
      wl[31] = acc_l;
    }
    __syncthreads();
    if (emit) {
      const unsigned int rank = run_e + we[warp] + (ie - e);
      const unsigned long long first = run_l + wl[warp] + (il - l);
      Emitter em;
      em.inv_rate = (double)l / (double)a;
      em.voxel = (uint32_t)v;
      em.n_lanes = (uint32_t)l;
      em.first_lane = first;
      em.stream_base = (mode == 0) ? (uint64_t)v * (uint64_t)tpb : first;
      S->plan[rank] = em;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      run_e += we[31];
      run_l += wl[31];
    }
    __syncthreads();
  }
}

}  // namespace

/* ---------------------------------------------------------- launchers */

/* Dynamic shared memory: spectrum, palette, shell scratch and the event
 * loop's per-thread fields (a single scene uses the fields before kCHist, a
 * batch those before kCBx, a prompt-gamma scene all of them). */
static size_t dynamic_smem(const TransportParams& P, int block, int algorithm, bool batch) {
  size_t s = 0;
  if (P.spectrum_in_shared) s += ((size_t)P.ne * 4 + 15) / 16 * 16;
  if (P.palette_in_shared) s += ((size_t)P.palette_in_shared * sizeof(PaletteEntry) + 15) / 16 * 16;
  s += (size_t)(P.max_shells > 0 ? P.max_shells : 1) * block * sizeof(float);
  if (algorithm != kAlgorithmHistories) {
    const int fields = P.prompt_energy > 0.0f ? kCold : (batch ? kCBx : kColdSingle);
    s += (size_t)fields * block * sizeof(uint32_t);
  }
  return s;
}

size_t transport_dynamic_smem(const TransportParams& P, int block, int algorithm) {
  return dynamic_smem(P, block, algorithm, false);
}

size_t transport_batch_dynamic_smem(const TransportParams& P, int block) {
  return dynamic_smem(P, block, kAlgorithmEvents, true);
}

int transport_block_threads() { return kBlock; }

__global__ void advance_seeds_kernel(SceneSlot* slots, int n_slots, int step) {
  const long long m = (long long)kM1 - 1;   /* seeds stay in [1, m1 - 1] */
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_slots; k += gridDim.x * blockDim.x) {
    const long long s = ((long long)slots[k].P.seed - 1 + step) % m;
    slots[k].P.seed = (int)(s < 0 ? s + m : s) + 1;
  }
}

cudaError_t launch_advance_seeds(SceneSlot* slots, int n_slots, int step, cudaStream_t stream) {
  const int grid = (n_slots + 127) / 128;
  advance_seeds_kernel<<<grid > 0 ? grid : 1, 128, 0, stream>>>(slots, n_slots, step);
  return cudaGetLastError();
}

/* Device address of the scratch array, looked up once per device with that
 * device current (the array's host-side name is only a stand-in).  The
 * address stays valid for the life of the device's primary context; after a
 * cudaDeviceReset the module may be loaded elsewhere and the cached address
 * is stale, so the allocation-free entry point must not be used across a
 * device reset. */
static std::mutex g_scratch_mutex;
static void* g_scratch_ptr[128];

static cudaError_t noalloc_scratch(NoAllocScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = static_cast<NoAllocScratch*>(g_scratch_ptr[dev]);
  return cudaSuccess;
}

cudaError_t launch_transport_noalloc(const TransportParams& P, DeviceTables T, DeviceTallies O,
                                     const float* activity, int lane_mode, int tpb, int hpl, int sm_count,
                                     bool counters, int mode, int grid, int block, size_t smem,
                                     cudaStream_t stream) {
  EventKernel k = counters ? event_variant<true, kEventBlocks, true, false, false, false, 0, 11>(mode)
                           : event_variant<false, kEventBlocks, true, false, false, false, 0, 11>(mode);
  if (!k) return cudaErrorNotSupported;
  NoAllocScratch* S = nullptr;
  cudaError_t e = noalloc_scratch(&S);
  if (e != cudaSuccess) return e;
  const int nvox = (int)P.n_voxels;
  if (nvox <= 0 || nvox > kNoAllocMaxVoxels) return cudaErrorInvalidValue;
  const int n_chunks = (nvox + kPlanChunk - 1) / kPlanChunk;
  const double t_s = (double)P.acq_ps * 1e-12;
  unsigned long long* cnt = counters ? O.counters : nullptr;
  plan_count_kernel<<<n_chunks, 256, 0, stream>>>(activity, nvox, S);
  plan_hpl_kernel<<<1, 32, 0, stream>>>(n_chunks, t_s, hpl, (double)sm_count * 2048.0, S);
  plan_lanes_kernel<<<n_chunks, 256, 0, stream>>>(activity, nvox, lane_mode, tpb, t_s, S);
  plan_scan_kernel<<<1, 32, 0, stream>>>(n_chunks, lane_mode, tpb, S, cnt);
  plan_fill_kernel<<<n_chunks, 256, 0, stream>>>(activity, nvox, lane_mode, tpb, t_s, S);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  T.emitters = S->plan;
  O.lane_cursor = &S->header[kHdrCursor];
  O.guard = &S->header[kHdrGuard];
  O.plan_counts = &S->header[kHdrLanes];
  if (!O.coincidences) O.coincidences = &S->header[kHdrCoinc];
  e = occupancy_smem_attr(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, block, smem, stream>>>(P, T, O, nullptr, 0);
  return cudaGetLastError();
}

/* Guard trips of the last allocation-free call on the current device (a
 * blocking 8-byte read of the scratch header; allocates nothing). */
cudaError_t noalloc_guard_trips(unsigned long long* trips) {
  NoAllocScratch* S = nullptr;
  cudaError_t e = noalloc_scratch(&S);
  if (e != cudaSuccess) return e;
  return cudaMemcpy(trips, &S->header[kHdrGuard], sizeof(unsigned long long), cudaMemcpyDeviceToHost);
}

cudaError_t launch_grad_replay(const TransportParams& P, const DeviceTables& T, const uint32_t* events,
                               unsigned long long n_events, const float* y, const int* trues, const int* scatter,
                               const float* bg, const float* activity, float* grad_a, float* grad_s,
                               unsigned long long* stats, int sm_count, int mode, cudaStream_t stream) {
  /* the replay recomputes histories with the forward run's arithmetic */
  auto kernel = (mode & kModeFast) ? grad_replay_kernel<kModeFast> : grad_replay_kernel<0>;
  const size_t smem = (size_t)(P.max_shells > 0 ? P.max_shells : 1) * kBlock * sizeof(float);
  cudaError_t e = occupancy_smem_attr(kernel, smem);
  if (e != cudaSuccess) return e;
  int bps = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, kBlock, smem);
  if (e != cudaSuccess) return e;
  if (bps < 1) bps = 1;
  unsigned long long need = (n_events + kBlock - 1) / kBlock;
  int grid = (int)std::min<unsigned long long>(need > 0 ? need : 1, (unsigned long long)sm_count * bps);
  kernel<<<grid, kBlock, smem, stream>>>(P, T, events, n_events, y, trues, scatter, bg, activity, grad_a,
                                                     grad_s, stats);
  return cudaGetLastError();
}

cudaError_t launch_loglik(long long nbins, const float* y, const int* trues, const int* scatter, const float* bg,
                          double* out, int sm_count, cudaStream_t stream) {
  long long need = (nbins + 255) / 256;
  int grid = (int)std::min<long long>(need > 0 ? need : 1, (long long)sm_count * 8);
  loglik_kernel<<<grid, 256, 0, stream>>>(nbins, y, trues, scatter, bg, out);
  return cudaGetLastError();
}

cudaError_t launch_probe_rng(const TransportParams& P, int n, const int64_t* ids, int ndraw, int2* seeds,
                             float* draws, double* ddraws, cudaStream_t s) {
  probe_rng_kernel<<<(n + 127) / 128, 128, 0, s>>>(P, n, ids, ndraw, seeds, draws, ddraws);
  return cudaGetLastError();
}

cudaError_t launch_probe_detector(const TransportParams& P, int n, const float* e2, const float* e1,
                                  const float3* p2, const float3* p1, const float3* d2, const float3* d1,
                                  const int8_t* s2, const int8_t* s1, int2* seeds, int* out, cudaStream_t s) {
  DeviceTallies O = {};
  probe_detector_kernel<<<(n + 127) / 128, 128, 0, s>>>(P, O, n, e2, e1, p2, p1, d2, d1, s2, s1, seeds, out);
  return cudaGetLastError();
}

cudaError_t launch_probe_compton(const ComptonTable* tab, int n, float* energy, const int* mat, int2* seeds,
                                 double* costh, cudaStream_t s) {
  size_t smem = (size_t)kMaxShells * 128 * sizeof(float);
  probe_compton_kernel<<<(n + 127) / 128, 128, smem, s>>>(tab, n, energy, mat, seeds, costh, kMaxShells);
  return cudaGetLastError();
}

cudaError_t launch_probe_rayleigh(const RayleighRows& R, int n, const float* energy, const int* mat,
                                  const float* pmax, int2* seeds, double* costh, cudaStream_t s) {
  probe_rayleigh_kernel<<<(n + 127) / 128, 128, 0, s>>>(R, n, energy, mat, pmax, seeds, costh);
  return cudaGetLastError();
}

cudaError_t launch_probe_source(const TransportParams& P, int background, int2* seeds, float3* out,
                                cudaStream_t s) {
  int n = (int)P.n_voxels;
  /* bit 0: background mode; bit 1: the balanced lanes' arithmetic */
  if (background & 2) probe_source_kernel<true><<<(n + 127) / 128, 128, 0, s>>>(P, background & 1, seeds, out);
  else probe_source_kernel<false><<<(n + 127) / 128, 128, 0, s>>>(P, background & 1, seeds, out);
  return cudaGetLastError();
}

}  // namespace mcpet
