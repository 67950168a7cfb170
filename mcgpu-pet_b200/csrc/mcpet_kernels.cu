/* Transport kernels of the photon-transport path (sm_100a) and their launch
 * wrappers.
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
#include "mcpet_device.cuh"
#include "mcpet_kernels.h"

namespace mcpet {
using namespace dev;

namespace {

/* Per-thread scratch for the Compton shell profiles, laid out [shell][thread]
 * in shared memory so the accesses of a warp hit distinct banks. */
struct SharedScratch {
  float* base;
  int stride;
  __device__ __forceinline__ float& operator[](int i) const { return base[i * stride]; }
};

struct LaneCounters {
  unsigned long long steps, refresh, majorant, tallies, photons, compton, rayleigh, photo, lanes, guard;
};

template <bool kCount>
struct Counting;
template <>
struct Counting<false> {
  __device__ __forceinline__ static void add(unsigned long long&, unsigned long long) {}
};
template <>
struct Counting<true> {
  __device__ __forceinline__ static void add(unsigned long long& c, unsigned long long v) { c += v; }
};

__device__ __forceinline__ uint64_t claim_lane(unsigned long long* cursor) {
  unsigned mask = __activemask();
  int lane_id = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane_id == leader) base = atomicAdd(cursor, (unsigned long long)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane_id) - 1u));
}

__device__ __forceinline__ int find_emitter(const Emitter* em, int n, uint64_t lane) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(&em[mid].first_lane) <= lane) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct PhotonState {
  float3 pos, dir;
  float energy;
  float travel;
  int state;    /* 0 unscattered, 1 Compton, 2 Rayleigh, 3 multiple */
};

/* Transport one photon from its emission point until it leaves the voxel box
 * (returns true) or is absorbed (returns false).  Woodcock delta tracking and
 * interaction selection of MCGPU-PET_kernel.cu:298-414. */
template <bool kCount, typename Scratch>
__device__ __forceinline__ bool track_photon(Rng& rng, const TransportParams& P, const DeviceTables& T,
                                             const PaletteEntry* pal, const ComptonTable& C, Scratch rn,
                                             PhotonState& ph, LaneCounters& cnt) {
  float energy = ph.energy;
  int index = __float2int_rd((energy - P.e0) * P.ide);
  float2 w = __ldg(reinterpret_cast<const float2*>(T.woodcock) + index);
  float mfp_w = w.x + energy * w.y;
  Counting<kCount>::add(cnt.majorant, 1);
  int mat_old = -1;
  float4 rec_lo = make_float4(0.f, 0.f, 0.f, 0.f), rec_hi = make_float4(0.f, 0.f, 0.f, 0.f);
  int steps = 0;
  for (;;) {
    int vox = locate(P, ph.pos.x, ph.pos.y, ph.pos.z);
    if (vox < 0) break;
    float prob, randno, mfp_density;
    int mat0;
    do {
      float step = -(mfp_w)*logf(ranecu(rng));
      ph.travel += step;
      ph.pos.x += step * ph.dir.x;
      ph.pos.y += step * ph.dir.y;
      ph.pos.z += step * ph.dir.z;
      vox = locate(P, ph.pos.x, ph.pos.y, ph.pos.z);
      if (vox < 0) break;
      if ((unsigned long long)vox >= (unsigned long long)P.n_voxels || ++steps > kMaxWoodcockSteps) {
        Counting<true>::add(cnt.guard, 1);
        ph.energy = energy;
        return false;
      }
      uint32_t key = T.vox16 ? (uint32_t)__ldg(&T.vox16[vox]) : __ldg(&T.vox32[vox]);
      PaletteEntry pe = pal[key];
      mat0 = pe.mat0;
      Counting<kCount>::add(cnt.steps, 1);
      if (mat0 != mat_old) {
        const float4* r = reinterpret_cast<const float4*>(T.mfp + (size_t)index * kMaxMaterials + mat0);
        rec_lo = __ldg(r);
        rec_hi = __ldg(r + 1);
        mat_old = mat0;
        Counting<kCount>::add(cnt.refresh, 1);
      }
      mfp_density = mfp_w * pe.rho;
      prob = 1.0f - mfp_density * (rec_lo.x + energy * rec_lo.y);
      randno = ranecu(rng);
    } while (randno < prob);
    if (vox < 0) break;

    prob += mfp_density * (rec_lo.z + energy * rec_lo.w);
    if (randno < prob) {
      /* Compton */
      double costh;
      if (!sample_compton(rng, energy, mat0, C, rn, costh)) {
        Counting<true>::add(cnt.guard, 1);
        ph.energy = energy;
        return false;
      }
      rotate(ph.dir, costh, 6.28318530717958647693 * ranecu_double(rng));
      Counting<kCount>::add(cnt.compton, 1);
      index = __float2int_rd((energy - P.e0) * P.ide);
      if (index > -1) {
        w = __ldg(reinterpret_cast<const float2*>(T.woodcock) + index);
        mfp_w = w.x + energy * w.y;
        mat_old = -2;
        ph.state = (ph.state == 0) ? 1 : 3;
        Counting<kCount>::add(cnt.majorant, 1);
      }
    } else {
      prob += mfp_density * (rec_hi.x + energy * rec_hi.y);
      if (randno < prob) {
        /* Rayleigh */
        double costh;
        if (!sample_rayleigh(rng, energy, mat0, rec_hi.z, T.rayleigh, costh)) {
          Counting<true>::add(cnt.guard, 1);
          ph.energy = energy;
          return false;
        }
        rotate(ph.dir, costh, 6.28318530717958647693 * ranecu_double(rng));
        ph.state = (ph.state == 0) ? 2 : 3;
        Counting<kCount>::add(cnt.rayleigh, 1);
      } else {
        /* photoelectric absorption */
        index = -11;
        Counting<kCount>::add(cnt.photo, 1);
      }
    }
    if (index < 0) break;
  }
  ph.energy = energy;
  return index > -1;
}

/* Write one packed 44-byte PSF record (PSF_element_struct, MCGPU-PET.h:235-247)
 * as eleven 32-bit words. */
__device__ __forceinline__ void put_psf_record(uint32_t* psf, long long k, unsigned long long t_emit,
                                               float travel, int voxel, float energy, float z, float phi,
                                               const float3& d, int state) {
  uint32_t* w = psf + 11 * k;
  w[0] = (uint32_t)(t_emit & 0xffffffffull);
  w[1] = (uint32_t)(t_emit >> 32);
  w[2] = __float_as_uint((float)((double)travel * kInvLightSpeed));
  w[3] = (uint32_t)voxel;
  w[4] = __float_as_uint(energy);
  w[5] = __float_as_uint(z);
  w[6] = __float_as_uint(phi);
  w[7] = __float_as_uint(d.x);
  w[8] = __float_as_uint(d.y);
  w[9] = __float_as_uint(d.z);
  w[10] = (uint32_t)(uint16_t)(short)state;   /* index1 = scatter state, index2 = 0 */
}

/* Coincidence processing of one photon pair whose two photons escaped
 * (MCGPU-PET_kernel.cu:417-432): sinogram tally (tally_Sinogram,
 * :1624-1836) and/or phase-space tally (tally_PSF_coincidences, :531-644).
 * "b" = the second photon (tracked last), "a" = the first. */
template <bool kCount>
__device__ __forceinline__ void detect_pair(Rng& rng, const TransportParams& P, const DeviceTallies& O,
                                            int* spec_sh, int voxel, unsigned long long t_left,
                                            const PhotonState& b, const PhotonState& a, LaneCounters& cnt,
                                            unsigned long long& detected) {
  const bool want_sino = (P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 2);
  const bool want_psf = (P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 1);
  if (want_sino) {
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
          if ((ib < P.ne) && (ib >= 0)) {
            if (spec_sh) atomicAdd(&spec_sh[ib], 1);
            else atomicAdd(&O.spectrum[ib], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if ((ia < P.ne) && (ia >= 0)) {
            if (spec_sh) atomicAdd(&spec_sh[ia], 1);
            else atomicAdd(&O.spectrum[ia], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if (eb > P.e_low && eb < P.e_high && ea > P.e_low && ea < P.e_high) {
            if (bin < P.nbins) {
              if (b.state == 0 && a.state == 0) {
                atomicAdd(&O.trues[bin], 1);
                atomicAdd(&O.image_trues[voxel], 1);
              } else {
                atomicAdd(&O.scatter[bin], 1);
                atomicAdd(&O.image_scatter[voxel], 1);
              }
              detected += 1;
              Counting<kCount>::add(cnt.tallies, 2);
            } else {
              Counting<true>::add(cnt.guard, 1);
            }
          }
        }
      }
    }
  }
  if (want_psf) {
    float xb, yb, zb;
    float db = to_cylinder(P, b.pos, b.dir, xb, yb, zb);
    float travel_b = b.travel + db;
    float phib = atan2f(yb, xb);
    if (fabsf(zb) < 0.5f * P.height) {
      float xa, ya, za;
      float da = to_cylinder(P, a.pos, a.dir, xa, ya, za);
      float travel_a = a.travel + da;
      float phia = atan2f(ya, xa);
      float g1 = blur_psf(rng);
      float g2 = blur_psf(rng);
      float eb = b.energy + (P.e_resol * (1.0f / 2.35f)) * b.energy * g1;
      float ea = a.energy + (P.e_resol * (1.0f / 2.35f)) * a.energy * g2;
      if (fabsf(za) < 0.5f * P.height && (eb > P.e_low) && (eb < P.e_high) && (ea > P.e_low) &&
          (ea < P.e_high)) {
        int k = atomicAdd(O.psf_count, 2);
        if (k > 2000000000) *O.psf_count = 2000000000;
        if (k < P.psf_capacity - 1 && O.psf) {
          long long kb = (travel_b < travel_a) ? k : k + 1;
          long long ka = (travel_b < travel_a) ? k + 1 : k;
          unsigned long long t_emit = P.acq_ps - t_left;
          put_psf_record(O.psf, kb, t_emit, travel_b, voxel, eb, zb, phib, b.dir, b.state);
          put_psf_record(O.psf, ka, t_emit, travel_a, voxel, ea, za, phia, a.dir, a.state);
        }
      }
    }
  }
}

constexpr int kBlock = 256;

template <bool kCount>
__global__ void __launch_bounds__(kBlock) transport_kernel(TransportParams P, DeviceTables T, DeviceTallies O) {
  __shared__ ComptonTable cmp;
  extern __shared__ float4 dyn_smem[];
  /* dynamic shared layout: [spectrum ints][palette entries][rn scratch] */
  int* spec_sh = nullptr;
  char* cursor = reinterpret_cast<char*>(dyn_smem);
  if (P.spectrum_in_shared) {
    spec_sh = reinterpret_cast<int*>(cursor);
    cursor += ((P.ne * 4 + 15) / 16) * 16;
  }
  const PaletteEntry* pal = T.palette;
  PaletteEntry* pal_sh = nullptr;
  if (P.palette_in_shared) {
    pal_sh = reinterpret_cast<PaletteEntry*>(cursor);
    cursor += ((P.palette_in_shared * (int)sizeof(PaletteEntry) + 15) / 16) * 16;
    pal = pal_sh;
  }
  SharedScratch rn{reinterpret_cast<float*>(cursor) + threadIdx.x, (int)blockDim.x};

  {
    const int* src = reinterpret_cast<const int*>(T.compton);
    int* dst = reinterpret_cast<int*>(&cmp);
    for (int i = threadIdx.x; i < (int)(sizeof(ComptonTable) / 4); i += blockDim.x) dst[i] = __ldg(&src[i]);
    if (spec_sh)
      for (int i = threadIdx.x; i < P.ne; i += blockDim.x) spec_sh[i] = 0;
    if (pal_sh)
      for (int i = threadIdx.x; i < P.palette_in_shared; i += blockDim.x) pal_sh[i] = T.palette[i];
  }
  __syncthreads();

  LaneCounters cnt = {};
  unsigned long long histories = 0, detected = 0;
  const bool background = P.background_mode != 0;
  for (;;) {
    uint64_t lane = claim_lane(O.lane_cursor);
    if (lane >= P.n_lanes) break;
    const Emitter* em = T.emitters + find_emitter(T.emitters, P.n_emitters, lane);
    const int voxel = (int)__ldg(&em->voxel);
    const uint64_t k = lane - __ldg(&em->first_lane);
    Rng rng = rng_stream(P, __ldg(&em->stream_base) + k);
    double inv_act = __ldg(&em->inv_rate);
    const int vx = voxel % P.nx;
    const int vy = (voxel / P.nx) % P.ny;
    const int vz = voxel / (P.nx * P.ny);
    unsigned long long t_left = P.acq_ps;
    Counting<kCount>::add(cnt.lanes, 1);

    for (;;) {
      /* time to the next decay of this lane (MCGPU-PET_kernel.cu:267-291) */
      double dt = -log(ranecu_double(rng)) * inv_act;
      unsigned long long dt_ps = __double2ull_rn(dt * 1e12);
      if (!(dt_ps < t_left)) break;
      t_left = t_left - dt_ps;
      histories += 2;
      inv_act = inv_act * exp(dt * P.inv_mean_life);

      PhotonState a, b;
      emit_first(rng, P, vx, vy, vz, a.pos, a.dir);
      const float3 origin = a.pos, dir0 = a.dir;
      a.energy = kAnnihilation;
      a.travel = 0.0f;
      a.state = 0;
      Counting<kCount>::add(cnt.photons, 2);
      bool esc_a = track_photon<kCount>(rng, P, T, pal, cmp, rn, a, cnt);

      emit_second(rng, background, dir0, b.dir);
      b.pos = origin;
      b.energy = kAnnihilation;
      b.travel = 0.0f;
      b.state = 0;
      bool esc_b = track_photon<kCount>(rng, P, T, pal, cmp, rn, b, cnt);

      if (esc_a && esc_b) {
        bool pass = (P.tally_type == 0) || (P.tally_type == 1 && b.state == 0 && a.state == 0) ||
                    (P.tally_type == 2 && (b.state != 0 || a.state != 0));
        if (pass) detect_pair<kCount>(rng, P, O, spec_sh, voxel, t_left, b, a, cnt, detected);
      }
    }
  }

  atomicAdd(O.histories, histories);
  if (detected) atomicAdd(O.coincidences, detected);
  if (cnt.guard) atomicAdd(O.guard, cnt.guard);
  if (kCount && O.counters) {
    atomicAdd(&O.counters[0], cnt.steps);
    atomicAdd(&O.counters[1], cnt.refresh);
    atomicAdd(&O.counters[2], cnt.majorant);
    atomicAdd(&O.counters[3], cnt.tallies);
    atomicAdd(&O.counters[4], cnt.photons);
    atomicAdd(&O.counters[5], cnt.compton);
    atomicAdd(&O.counters[6], cnt.rayleigh);
    atomicAdd(&O.counters[7], cnt.photo);
    atomicAdd(&O.counters[8], cnt.lanes);
    atomicAdd(&O.counters[9], cnt.guard);
  }
  __syncthreads();
  if (spec_sh)
    for (int i = threadIdx.x; i < P.ne; i += blockDim.x)
      if (spec_sh[i]) atomicAdd(&O.spectrum[i], spec_sh[i]);
}

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

__global__ void probe_source_kernel(TransportParams P, int background, int2* seeds, float3* out) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if ((long long)v >= P.n_voxels) return;
  int vx = v % P.nx, vy = (v / P.nx) % P.ny, vz = v / (P.nx * P.ny);
  Rng r;
  r.x = seeds[v].x;
  r.y = seeds[v].y;
  float3 pos, dir, dir2;
  emit_first(r, P, vx, vy, vz, pos, dir);
  emit_second(r, background != 0, dir, dir2);
  out[4 * v + 0] = pos;
  out[4 * v + 1] = dir;
  out[4 * v + 2] = pos;
  out[4 * v + 3] = dir2;
  seeds[v] = make_int2(r.x, r.y);
}

}  // namespace

/* ---------------------------------------------------------- launchers */

size_t transport_dynamic_smem(const TransportParams& P, int block) {
  size_t s = 0;
  if (P.spectrum_in_shared) s += ((size_t)P.ne * 4 + 15) / 16 * 16;
  if (P.palette_in_shared) s += ((size_t)P.palette_in_shared * sizeof(PaletteEntry) + 15) / 16 * 16;
  s += (size_t)(P.max_shells > 0 ? P.max_shells : 1) * block * sizeof(float);
  return s;
}

int transport_block_threads() { return kBlock; }

cudaError_t transport_occupancy(bool counters, int block, size_t smem, int* blocks_per_sm) {
  if (counters)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, transport_kernel<true>, block, smem);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, transport_kernel<false>, block, smem);
}

cudaError_t launch_transport(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                             bool counters, int grid, int block, size_t smem, cudaStream_t stream) {
  if (smem > 48 * 1024) {
    cudaError_t e = counters ? cudaFuncSetAttribute(transport_kernel<true>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                             : cudaFuncSetAttribute(transport_kernel<false>,
                                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (counters) transport_kernel<true><<<grid, block, smem, stream>>>(P, T, O);
  else transport_kernel<false><<<grid, block, smem, stream>>>(P, T, O);
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
  probe_source_kernel<<<(n + 127) / 128, 128, 0, s>>>(P, background, seeds, out);
  return cudaGetLastError();
}

}  // namespace mcpet
