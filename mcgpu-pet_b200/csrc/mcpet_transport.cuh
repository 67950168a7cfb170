/* Device code of the transport kernels (sm_100a), shared by the translation
 * units that compile their variants (mcpet_kernels*.cu), and the launch
 * helpers those use.  Everything here has internal linkage: each unit
 * instantiates its own set of variants. */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>

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

/* Compile-time variants of the transport kernels (kMode bits): kModeFast
 * is the arithmetic of balanced lanes (single-precision rotation, decay
 * clock, photon-2 emission, Compton sampling, sinogram indices and energy
 * blur; GCOa's normaliser from the interaction record's bound);
 * kModePrompt compiles the prompt-gamma emitter; kModeCaps reads the loop
 * guards' caps from the run parameters instead of the defaults; kModeSino
 * leaves out the phase-space (PSF) tally of runs that tally the sinogram
 * only; kModeChain makes the single-scene kernel a chained launch of a
 * batched run (programmatic dependent launch, seed from the batch slot).  A
 * variant carries none of the code of the features it leaves out. */
constexpr int kModeFast = kTransportFast, kModePrompt = kTransportPrompt, kModeCaps = kTransportCaps,
              kModeSino = kTransportSinogramOnly, kModeChain = kTransportChained;

template <int kMode>
__device__ __forceinline__ int steps_cap(const TransportParams& P) {
  return (kMode & kModeCaps) ? P.max_steps : kMaxWoodcockSteps;
}
template <int kMode>
__device__ __forceinline__ int rejections_cap(const TransportParams& P) {
  return (kMode & kModeCaps) ? P.max_rejections : kMaxRejections;
}
/* direction change after a real scattering with the next random draw */
template <int kMode>
__device__ __forceinline__ void scatter_direction(Rng& rng, float3& dir, double costh) {
  if (kMode & kModeFast) rotate_fast(dir, (float)costh, ranecu(rng));
  else rotate(dir, costh, 6.28318530717958647693 * ranecu_double(rng));
}

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

/* Dose of one real interaction (MCGPU-PET_kernel.cu:396-410): `loss` is the
 * reference's temporary, E_after - E_before for Compton and -E for
 * photoelectric absorption; energy is deposited when it is below -0.001 eV.
 * Material sums go to `mat` (a block's shared copy, or global memory), the
 * ROI voxel sums to global memory, each term rounded to an integer as the
 * device build of tally_materials_dose / tally_voxel_energy_deposition does
 * (MCGPU-PET_kernel.cu:1593-1650; SCALE_eV = 1). */
struct DoseSink {
  unsigned long long* mat;   /* [15][2] or NULL */
  unsigned long long* vox;   /* [ROI][2] or NULL */
  __device__ __forceinline__ void operator()(const TransportParams& P, float loss, int material,
                                             const float3& pos) const {
    if (!(loss < -0.001f)) return;
    const float edep = -1.0f * loss;
    const unsigned long long e1 = __float2ull_rn(edep), e2 = __float2ull_rn(edep * edep);
    if (mat) {
      atomicAdd(&mat[2 * material], e1);
      atomicAdd(&mat[2 * material + 1], e2);
    }
    if (vox) {
      const int x = __float2int_rd(pos.x * P.inv_vx);
      const int y = __float2int_rd(pos.y * P.inv_vy);
      const int z = __float2int_rd(pos.z * P.inv_vz);
      const int* r = P.dose_roi;
      if (x < r[0] || x > r[1] || y < r[2] || y > r[3] || z < r[4] || z > r[5]) return;
      const int dx = 1 + r[1] - r[0];
      const long long k = (long long)(x - r[0]) + (long long)(y - r[2]) * dx +
                          (long long)(z - r[4]) * dx * (1 + r[3] - r[2]);
      atomicAdd(&vox[2 * k], e1);
      atomicAdd(&vox[2 * k + 1], e2);
    }
  }
};

/* Observer of the Woodcock steps inside the phantom: voxel, whether the
 * step ended in a real interaction, and the probability of a virtual one. */
struct NoStepHook {
  __device__ __forceinline__ void operator()(int, bool, float) {}
};

/* Transport one photon from its emission point until it leaves the voxel box
 * (returns true) or is absorbed (returns false).  Woodcock delta tracking and
 * interaction selection of MCGPU-PET_kernel.cu:298-414. */
template <bool kCount, int kMode, typename Scratch, typename Hook = NoStepHook>
__device__ __forceinline__ bool track_photon(Rng& rng, const TransportParams& P, const DeviceTables& T,
                                             const PaletteEntry* pal, const ComptonTable& C, Scratch rn,
                                             PhotonState& ph, LaneCounters& cnt, Hook* hook = nullptr,
                                             const DoseSink* dose = nullptr) {
  float energy = ph.energy;
  int index = __float2int_rd((energy - P.e0) * P.ide);
  if ((kMode & kModePrompt) && (index < 0 || index >= P.n_e - 1)) {   /* energy outside the tables */
    Counting<true>::add(cnt.guard, 1);
    return false;
  }
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
      if ((unsigned long long)vox >= (unsigned long long)P.n_voxels || ++steps > steps_cap<kMode>(P)) {
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
      if (hook) (*hook)(vox, !(randno < prob), prob);
    } while (randno < prob);
    if (vox < 0) break;

    prob += mfp_density * (rec_lo.z + energy * rec_lo.w);
    if (randno < prob) {
      /* Compton */
      double costh;
      const float e_before = energy;
      if (!sample_compton<(kMode & kModeFast) != 0>(rng, energy, mat0, C, rn, costh,
                                                    (kMode & kModeFast) ? rec_hi.w : -1.0f,
                                                    rejections_cap<kMode>(P))) {
        Counting<true>::add(cnt.guard, 1);
        ph.energy = energy;
        return false;
      }
      scatter_direction<kMode>(rng, ph.dir, costh);
      Counting<kCount>::add(cnt.compton, 1);
      if (dose) (*dose)(P, energy - e_before, mat0, ph.pos);
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
        if (!sample_rayleigh(rng, energy, mat0, rec_hi.z, T.rayleigh, costh, rejections_cap<kMode>(P))) {
          Counting<true>::add(cnt.guard, 1);
          ph.energy = energy;
          return false;
        }
        scatter_direction<kMode>(rng, ph.dir, costh);
        ph.state = (ph.state == 0) ? 2 : 3;
        Counting<kCount>::add(cnt.rayleigh, 1);
      } else {
        /* photoelectric absorption */
        index = -11;
        Counting<kCount>::add(cnt.photo, 1);
        if (dose) (*dose)(P, -energy, mat0, ph.pos);
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
 * "b" = the second photon (tracked last), "a" = the first.  `centre` is the
 * detector centre (P.cx, P.cy, P.cz).  A spurious pair (a prompt gamma with
 * an annihilation photon) is tallied with the scatter whatever the photons'
 * scatter states. */
template <bool kCount, bool kRecord = true, bool kPsf = true, bool kFast = false>
__device__ __forceinline__ void detect_pair(Rng& rng, const TransportParams& P, const float3 centre,
                                            const DeviceTallies& O, int* spec_sh, int voxel,
                                            unsigned long long t_left, const PhotonState& b, const PhotonState& a,
                                            LaneCounters& cnt, unsigned long long& detected, int2 rng_emit,
                                            bool spurious = false) {
  /* !kPsf: a sinogram-only run (REPORT PSF/SINOGRAM 2), so no PSF tally and
   * no sinogram-dry replay */
  const bool want_sino = !kPsf || (P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 2);
  const bool want_psf = kPsf && ((P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 1));
  const bool dry = kPsf && P.sino_dry;
  if (want_sino) {
    float xb, yb, zb, xa, ya, za;
    to_cylinder(P, centre, b.pos, b.dir, xb, yb, zb);
    float phib = atan2f(yb, xb);
    if (fabsf(zb) < 0.5f * P.height) {
      to_cylinder(P, centre, a.pos, a.dir, xa, ya, za);
      float phia = atan2f(ya, xa);
      if (fabsf(za) < 0.5f * P.height) {
        long long bin = sinogram_bin<kFast>(P, phib, zb, phia, za);
        if (bin >= 0) {
          float g1 = blur_sinogram<kFast>(rng);
          float g2 = blur_sinogram<kFast>(rng);
          float eb = b.energy + (P.e_resol / 2.35f) * b.energy * g1;
          float ea = a.energy + (P.e_resol / 2.35f) * a.energy * g2;
          int ib = __float2int_rd(eb / 1000.0f);
          int ia = __float2int_rd(ea / 1000.0f);
          /* sino_dry: the same draws, no sinogram-side writes (a PSF replay) */
          if ((ib < P.ne) && (ib >= 0) && !dry) {
            if (spec_sh) atomicAdd(&spec_sh[ib], 1);
            else atomicAdd(&O.spectrum[ib], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if ((ia < P.ne) && (ia >= 0) && !dry) {
            if (spec_sh) atomicAdd(&spec_sh[ia], 1);
            else atomicAdd(&O.spectrum[ia], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if (eb > P.e_low && eb < P.e_high && ea > P.e_low && ea < P.e_high && !dry) {
            if (bin < P.nbins) {
              if (!spurious && b.state == 0 && a.state == 0) {
                atomicAdd(&O.trues[bin], 1);
                atomicAdd(&O.image_trues[voxel], 1);
              } else {
                atomicAdd(&O.scatter[bin], 1);
                atomicAdd(&O.image_scatter[voxel], 1);
              }
              detected += 1;
              Counting<kCount>::add(cnt.tallies, 2);
              if (kRecord && O.events) {
                /* record for the gradient replay: one counter atomic per
                 * converged group of lanes */
                const unsigned grp = __activemask();
                const int leader = __ffs(grp) - 1;
                const int lane_id = (int)(threadIdx.x & 31);
                unsigned long long base = 0;
                if (lane_id == leader) base = atomicAdd(O.event_count, (unsigned long long)__popc(grp));
                base = __shfl_sync(grp, base, leader);
                const unsigned long long k = base + (unsigned long long)__popc(grp & ((1u << lane_id) - 1u));
                if (k < (unsigned long long)O.event_capacity) {
                  uint4* rec = reinterpret_cast<uint4*>(O.events + 6 * k);
                  uint2* rec2 = reinterpret_cast<uint2*>(O.events + 6 * k + 4);
                  if ((k & 1) == 0) {
                    rec[0] = make_uint4((uint32_t)rng_emit.x, (uint32_t)rng_emit.y, (uint32_t)voxel, 0u);
                    rec2[0] = make_uint2((uint32_t)bin, (uint32_t)((unsigned long long)bin >> 32));
                  } else {
                    uint2* r = reinterpret_cast<uint2*>(O.events + 6 * k);
                    r[0] = make_uint2((uint32_t)rng_emit.x, (uint32_t)rng_emit.y);
                    r[1] = make_uint2((uint32_t)voxel, 0u);
                    r[2] = make_uint2((uint32_t)bin, (uint32_t)((unsigned long long)bin >> 32));
                  }
                }
              }
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
    float db = to_cylinder(P, centre, b.pos, b.dir, xb, yb, zb);
    float travel_b = b.travel + db;
    float phib = atan2f(yb, xb);
    if (fabsf(zb) < 0.5f * P.height) {
      float xa, ya, za;
      float da = to_cylinder(P, centre, a.pos, a.dir, xa, ya, za);
      float travel_a = a.travel + da;
      float phia = atan2f(ya, xa);
      float g1 = blur_psf(rng);
      float g2 = blur_psf(rng);
      float eb = b.energy + (P.e_resol * (1.0f / 2.35f)) * b.energy * g1;
      float ea = a.energy + (P.e_resol * (1.0f / 2.35f)) * a.energy * g2;
      if (fabsf(za) < 0.5f * P.height && (eb > P.e_low) && (eb < P.e_high) && (ea > P.e_low) &&
          (ea < P.e_high)) {
        /* one counter atomic per converged group of lanes, 2 records per lane */
        const unsigned grp = __activemask();
        const int leader = __ffs(grp) - 1;
        const int lane_id = (int)(threadIdx.x & 31);
        int base = 0;
        if (lane_id == leader) base = atomicAdd(O.psf_count, 2 * __popc(grp));
        base = __shfl_sync(grp, base, leader);
        const int k = base + 2 * __popc(grp & ((1u << lane_id) - 1u));
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

template <bool kCount, int kMode>
__global__ void __launch_bounds__(kBlock) transport_kernel(TransportParams P, DeviceTables T, DeviceTallies O) {
  constexpr bool kFastLanes = (kMode & kModeFast) != 0;
  __shared__ ComptonTable cmp;
  __shared__ unsigned long long mdose_sh[2 * kMaxMaterials];
  if (threadIdx.x < 2 * kMaxMaterials) mdose_sh[threadIdx.x] = 0;
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
  const DoseSink dose{O.mat_dose ? mdose_sh : nullptr, O.vox_dose};
  const bool dose_on = O.mat_dose || O.vox_dose;
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
      const unsigned long long dt_ps = decay_interval<(kMode & kModeFast) != 0>(rng, inv_act, P.inv_mean_life);
      if (!(dt_ps < t_left)) break;
      t_left = t_left - dt_ps;
      histories += 2;

      PhotonState a, b;
      const int2 rng_emit = make_int2(rng.x, rng.y);
      emit_first(rng, P, vx, vy, vz, a.pos, a.dir);
      const float3 origin = a.pos, dir0 = a.dir;
      a.energy = kAnnihilation;
      a.travel = 0.0f;
      a.state = 0;
      Counting<kCount>::add(cnt.photons, 2);
      bool esc_a =
          track_photon<kCount, kMode>(rng, P, T, pal, cmp, rn, a, cnt, (NoStepHook*)nullptr, dose_on ? &dose : nullptr);

      emit_second<(kMode & kModeFast) != 0>(rng, background, dir0, b.dir);
      b.pos = origin;
      b.energy = kAnnihilation;
      b.travel = 0.0f;
      b.state = 0;
      bool esc_b =
          track_photon<kCount, kMode>(rng, P, T, pal, cmp, rn, b, cnt, (NoStepHook*)nullptr, dose_on ? &dose : nullptr);

      if (esc_a && esc_b) {
        bool pass = (P.tally_type == 0) || (P.tally_type == 1 && b.state == 0 && a.state == 0) ||
                    (P.tally_type == 2 && (b.state != 0 || a.state != 0));
        if (pass)
          detect_pair<kCount, true, true, kFastLanes>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel,
                                                      t_left, b, a, cnt, detected, rng_emit);
      }
      /* prompt gamma: isotropic from the decay point after the pair, then
       * its pairs with the annihilation photons that escaped (spurious
       * coincidences; not in the trues-only tally) */
      if ((kMode & kModePrompt) && (P.prompt_yield >= 1.0f || ranecu(rng) < P.prompt_yield)) {
        PhotonState g;
        emit_isotropic(rng, g.dir);
        g.pos = origin;
        g.energy = P.prompt_energy;
        g.travel = 0.0f;
        g.state = 0;
        histories += 1;
        Counting<kCount>::add(cnt.photons, 1);
        const bool esc_g = track_photon<kCount, kMode>(rng, P, T, pal, cmp, rn, g, cnt, (NoStepHook*)nullptr,
                                                       dose_on ? &dose : nullptr);
        if (esc_g && P.tally_type != 1) {
          if (esc_a)
            detect_pair<kCount, true, true, kFastLanes>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel,
                                                        t_left, g, a, cnt, detected, rng_emit, true);
          if (esc_b)
            detect_pair<kCount, true, true, kFastLanes>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel,
                                                        t_left, g, b, cnt, detected, rng_emit, true);
        }
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
  if (O.mat_dose && threadIdx.x < 2 * kMaxMaterials && mdose_sh[threadIdx.x])
    atomicAdd(&O.mat_dose[threadIdx.x], mdose_sh[threadIdx.x]);
}

/* ------------------------------------------------------- event kernel
 *
 * transport_events_kernel runs the same per-lane computation as
 * transport_kernel -- every thread draws the same random numbers and performs
 * the same floating-point operations for its lane, so the results are
 * identical -- but schedules it as a state machine regrouped per warp: each
 * round the warp votes on the phase of its 32 photons and executes ONE phase
 * for the threads in it.  Woodcock sub-steps (cheap, frequent) run in batches;
 * Compton sampling (expensive: shell profiles, rejection loops, double
 * precision rotation) runs only when most of the warp needs it, so its
 * instructions execute with nearly all lanes active instead of one or two.
 * Lane-level state that a phase touches once per photon (the pair's emission
 * point and first photon, the decay clock) lives in shared memory, laid out
 * [field][thread]. */

enum : int { kPhDecay = 0, kPhStep = 1, kPhCompton = 2, kPhEnd = 3, kPhDone = 4 };  /* kPhCompton: any real scattering */

/* cold per-thread fields in shared memory */
enum : int {
  kCOx, kCOy, kCOz, kCDx, kCDy, kCDz,            /* emission point and direction of photon 1 */
  kCAx, kCAy, kCAz, kCAu, kCAv, kCAw,            /* photon 1 at exit: position, direction */
  kCAe, kCAt, kCAs,                              /* photon 1 energy (-10 absorbed), travel, state */
  kCInvLo, kCInvHi, kCTLo, kCTHi, kCVox,         /* lane: 1/rate (double), remaining ps (u64), voxel */
  kCRx, kCRy,                                    /* RANECU state right before the pair's emission */
  kCTrial, kCS0,                                 /* pending Compton sampling: trials so far, its s0 */
  kCHist, kCDet,                                 /* batch only: lane photons started, coincidences tallied */
  kCPmax,                                        /* batch only: Rayleigh pmax of the pending interaction */
  kCBx, kCBy, kCBz, kCBu, kCBv, kCBw,            /* prompt gamma only: photon 2 at exit: position, direction, */
  kCBe, kCBt, kCBs,                              /* energy (-10 absorbed), travel, state */
  kCold
};
constexpr int kColdSingle = kCHist;              /* fields a single-scene launch uses (the last ones need no room) */

struct ColdState {
  uint32_t* base;
  int stride;
  __device__ __forceinline__ uint32_t& u(int f) const { return base[f * stride]; }
  __device__ __forceinline__ float f(int k) const { return __uint_as_float(base[k * stride]); }
  __device__ __forceinline__ void setf(int k, float v) const { base[k * stride] = __float_as_uint(v); }
  __device__ __forceinline__ double inv_rate() const {
    return __hiloint2double((int)u(kCInvHi), (int)u(kCInvLo));
  }
  __device__ __forceinline__ void set_inv_rate(double v) const {
    u(kCInvHi) = (uint32_t)__double2hiint(v);
    u(kCInvLo) = (uint32_t)__double2loint(v);
  }
  __device__ __forceinline__ unsigned long long t_left() const {
    return ((unsigned long long)u(kCTHi) << 32) | u(kCTLo);
  }
  __device__ __forceinline__ void set_t_left(unsigned long long v) const {
    u(kCTHi) = (uint32_t)(v >> 32);
    u(kCTLo) = (uint32_t)v;
  }
};


/* Batches whose scenes all have the same scanner (detector, sinogram and
 * tally settings) or the same phantom (grid, voxels, palette, tables) read
 * those from the launch's parameters instead of their slots. */
constexpr int kShareScanner = kBatchShareScanner;
constexpr int kSharePhantom = kBatchSharePhantom;

template <bool kCount, int kMinBlocks = 1, bool kDevicePlan = false, bool kBatch = false, bool kRecord = false,
          bool kDose = false, int kShare = 0, int kMode = 0>
__global__ void __launch_bounds__(kBlock, kMinBlocks) transport_events_kernel(TransportParams P, DeviceTables T,
                                                                              DeviceTallies O,
                                                                              const SceneSlot* __restrict__ slots,
                                                                              int n_slots) {
  /* kBatch: the lanes belong to n_slots scenes.  P, T and O then describe
   * the launch (total lanes, work queue, guard word, counters, the Compton
   * and Rayleigh tables of all scenes' materials; shared staging off); the
   * launch's lanes are the scenes' lanes one scene after the other, and each
   * lane reads its scene's parameters, lane plan, tables and tallies from
   * slots[scene] -- except what kShare marks as the same in every scene
   * (kShareScanner: detector, sinogram and tally settings; kSharePhantom:
   * grid, voxel keys, palette and tables), which comes from P and T as in a
   * single-scene launch.  A batched lane's RANECU start uses P's jump tables
   * (they do not depend on the scene) with its scene's seed; a thread keeps
   * its totals for the current scene in the shared per-thread state and adds
   * them to that scene's when it moves to another.  kRecord: tallied coincidences are also written to
   * O.events for the gradient replay.  kDose: the material and voxel dose
   * tallies are on (O.mat_dose / O.vox_dose, or the slots' in a batch). */
  /* kDevicePlan: the lane plan was built on the device and its size is read
   * from device memory instead of the launch parameters */
  const uint64_t n_lanes = kDevicePlan ? (uint64_t)O.plan_counts[0] : P.n_lanes;
  const int n_emitters = kDevicePlan ? (int)O.plan_counts[1] : P.n_emitters;
  __shared__ unsigned long long mdose_sh[2 * kMaxMaterials];
  __shared__ ComptonTable cmp;
  __shared__ float s0_ann[kMaxMaterials];
  extern __shared__ float4 dyn_smem[];
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
  cursor += (size_t)(P.max_shells > 0 ? P.max_shells : 1) * blockDim.x * sizeof(float);
  const ColdState cold{reinterpret_cast<uint32_t*>(cursor) + threadIdx.x, (int)blockDim.x};
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
  if (threadIdx.x < kMaxMaterials)
    s0_ann[threadIdx.x] = cmp.noscco[threadIdx.x] > 0 ? compton_s0(P.e_annihilation, threadIdx.x, cmp) : 0.0f;
  if (threadIdx.x < 2 * kMaxMaterials) mdose_sh[threadIdx.x] = 0;
  __syncthreads();

  LaneCounters cnt = {};
  /* photons started and coincidences tallied: per thread, added to the
   * run's totals at the end; in a batch per thread and scene, in the shared
   * per-thread state (kCHist, kCDet), added to the scene's totals when the
   * thread moves to another scene and at the end */
  unsigned long long histories = 0, detected = 0;
  const bool background = P.background_mode != 0;
  int scene = 0;            /* scene of the current lane (kBatch) */
  /* dose: a block-shared copy of the material sums (global ones in a batch) */
  const bool dose_on = kDose && (kBatch || O.mat_dose || O.vox_dose);

  /* hot per-thread state */
  Rng rng = {0, 0};
  int phase = kPhDecay;
  bool lane_live = false;
  int which = 1;            /* photon of the pair being tracked */
  bool fresh = false;       /* next step starts a new interaction-loop iteration */
  bool escaped = false;
  bool is_compton = true;   /* pending scattering: Compton (else Rayleigh) */
  PhotonState ph;
  ph.pos = make_float3(0.f, 0.f, 0.f);
  ph.dir = ph.pos;
  ph.energy = 0.f;
  ph.travel = 0.f;
  ph.state = 0;
  int index = 0, mat_old = -1, mat0 = 0, steps = 0;
  float mfp_w = 0.f, cax = 0.f, cbx = 0.f;
  float4 rec_hi = make_float4(0.f, 0.f, 0.f, 0.f);   /* Rayleigh part of the last interaction record */

  /* photon emitted at ph.pos with ph.dir: set up its tracking */
  /* batch: the thread's totals for its current scene, added to that
   * scene's when the thread moves to another scene and at the end */
  if (kBatch) {
    cold.u(kCHist) = 0;
    cold.u(kCDet) = 0;
  }
  cold.u(kCTrial) = 0;
  auto flush_lane = [&]() {
    if (!kBatch) return;
    const unsigned long long h = cold.u(kCHist), c = cold.u(kCDet);
    if (h) atomicAdd(slots[scene].O.histories, h);
    if (c && slots[scene].O.coincidences) atomicAdd(slots[scene].O.coincidences, c);
    cold.u(kCHist) = 0;
    cold.u(kCDet) = 0;
  };

  /* (the scenes of a batch share the energy grid: e0 and ide are P's) */
  auto start_photon = [&](const DeviceTables& TW, float energy) {
    ph.energy = energy;
    ph.travel = 0.0f;
    ph.state = 0;
    index = __float2int_rd((ph.energy - P.e0) * P.ide);
    Counting<kCount>::add(cnt.photons, 1);
    if ((kMode & kModePrompt) && (index < 0 || index >= P.n_e - 1)) {   /* energy outside the tables */
      Counting<true>::add(cnt.guard, 1);
      escaped = false;
      phase = kPhEnd;
      return;
    }
    float2 w = __ldg(reinterpret_cast<const float2*>(TW.woodcock) + index);
    mfp_w = w.x + ph.energy * w.y;
    mat_old = -1;
    steps = 0;
    fresh = true;
    phase = kPhStep;
    Counting<kCount>::add(cnt.majorant, 1);
  };

  for (;;) {
    const unsigned m_dec = __ballot_sync(0xffffffffu, phase == kPhDecay);
    const unsigned m_step = __ballot_sync(0xffffffffu, phase == kPhStep);
    const unsigned m_cmp = __ballot_sync(0xffffffffu, phase == kPhCompton);
    const unsigned m_end = __ballot_sync(0xffffffffu, phase == kPhEnd);
    if (!(m_dec | m_step | m_cmp | m_end)) break;
    const TransportParams& PS = kBatch ? slots[scene].P : P;
    /* phantom (grid, voxels, tables) and scanner (detector, sinogram) of the
     * current lane's scene */
    const TransportParams& PG = (kBatch && !(kShare & kSharePhantom)) ? slots[scene].P : P;
    const DeviceTables& TG = (kBatch && !(kShare & kSharePhantom)) ? slots[scene].T : T;
    const TransportParams& PD = (kBatch && !(kShare & kShareScanner)) ? slots[scene].P : P;
    /* phase of this round: scattering and pair bookkeeping wait until enough
     * lanes need them; Woodcock steps fill the rest */
    const int n_cmp = __popc(m_cmp), n_pair = __popc(m_end | m_dec);
    int sel;
    if (n_cmp >= P.quorum_scatter) sel = 0;
    else if (n_pair >= P.quorum_pair) sel = 1;
    else if (m_step) sel = 2;
    else sel = (n_cmp >= n_pair) ? 0 : 1;

    if (sel == 0) {
      /* ---- real scattering: Compton (MCGPU-PET_kernel.cu:351-373) or
       * Rayleigh (:375-387), then the common direction update.  Rayleigh
       * lanes (GRAa) join a round with Compton lanes only when at least
       * quorum_rayleigh of them wait, so that most rounds run one sampler.
       * The Compton lanes repeat trials of GCOa's first stage until at most
       * an eighth of them are still rejected; those keep their phase and go
       * on in a later round, with the lanes that arrive meanwhile, instead of
       * holding the warp in the rejection loop (each lane draws its random
       * numbers in the same order either way) */
      const unsigned m_ray = __ballot_sync(0xffffffffu, phase == kPhCompton && !is_compton);
      const unsigned m_c = m_cmp & ~m_ray;
      const bool ray_now = (m_cmp == m_ray) || (__popc(m_ray) >= P.quorum_rayleigh);
      if (phase == kPhCompton && (is_compton || ray_now)) {
        double costh = 0.0;
        bool ok = false, pending = false;
        float e = ph.energy;
        if (__builtin_expect(is_compton, 1)) {
          uint32_t trials = cold.u(kCTrial);
          float s0;
          if (kMode & kModeFast) {
            /* balanced lanes: the bin's bound of the normaliser */
            s0 = __ldg(&TG.mfp[(size_t)index * kMaxMaterials + mat0].s0_bound);
          } else if (e == kAnnihilation) {
            s0 = s0_ann[mat0];
          } else if (trials == 0) {
            s0 = compton_s0(e, mat0, cmp);
            cold.setf(kCS0, s0);
          } else {
            s0 = cold.f(kCS0);
          }
          float tau = 0.f, s = 0.f;
          double cdt1 = 0.0;
          bool accepted = false, tripped = false;
          for (;;) {
            if (!accepted && !tripped) {
              if (++trials > (uint32_t)rejections_cap<kMode>(P)) tripped = true;
              else accepted = compton_trial<(kMode & kModeFast) != 0>(rng, e, mat0, cmp, rn, s0, tau, s, cdt1);
            }
            if (8 * __popc(__ballot_sync(m_c, !accepted && !tripped)) <= __popc(m_c)) break;
          }
          if (accepted) {
            cold.u(kCTrial) = 0;
            costh = 1.0 - cdt1;
            ok = compton_doppler<(kMode & kModeFast) != 0>(rng, e, mat0, cmp, rn, tau, s, costh,
                                                           rejections_cap<kMode>(P));
          } else if (tripped) {
            cold.u(kCTrial) = 0;
          } else {
            cold.u(kCTrial) = trials;
            pending = true;
          }
        } else {
          ok = sample_rayleigh(rng, e, mat0, kBatch ? cold.f(kCPmax) : rec_hi.z, T.rayleigh, costh,
                               rejections_cap<kMode>(P));
        }
        if (pending) {
          /* next trial in a later scattering round */
        } else if (__builtin_expect(!ok, 0)) {
          Counting<true>::add(cnt.guard, 1);
          escaped = false;
          phase = kPhEnd;
        } else {
          const float e_before = ph.energy;
          ph.energy = e;
          scatter_direction<kMode>(rng, ph.dir, costh);
          if (is_compton) {
            Counting<kCount>::add(cnt.compton, 1);
            if (dose_on) {
              const DoseSink ds{kBatch ? slots[scene].O.mat_dose : (O.mat_dose ? mdose_sh : nullptr),
                                kBatch ? slots[scene].O.vox_dose : O.vox_dose};
              ds(PS, e - e_before, mat0, ph.pos);
            }
            index = __float2int_rd((e - P.e0) * P.ide);
            if (index > -1) {
              float2 w = __ldg(reinterpret_cast<const float2*>(TG.woodcock) + index);
              mfp_w = w.x + e * w.y;
              mat_old = -2;
              ph.state = (ph.state == 0) ? 1 : 3;
              Counting<kCount>::add(cnt.majorant, 1);
              fresh = true;
              phase = kPhStep;
            } else {
              escaped = false;
              phase = kPhEnd;
            }
          } else {
            ph.state = (ph.state == 0) ? 2 : 3;
            Counting<kCount>::add(cnt.rayleigh, 1);
            fresh = true;
            phase = kPhStep;
          }
        }
      }
    } else if (sel == 1) {
      /* ---- end of a photon: hand over to the second photon, or close the
       * pair (MCGPU-PET_kernel.cu:417-442); then the next decay */
      if (phase == kPhEnd) {
        if (which == 1) {
          if (escaped) {
            cold.setf(kCAx, ph.pos.x); cold.setf(kCAy, ph.pos.y); cold.setf(kCAz, ph.pos.z);
            cold.setf(kCAu, ph.dir.x); cold.setf(kCAv, ph.dir.y); cold.setf(kCAw, ph.dir.z);
            cold.setf(kCAe, ph.energy); cold.setf(kCAt, ph.travel);
            cold.u(kCAs) = (uint32_t)ph.state;
          } else {
            cold.setf(kCAe, -10.0f);
          }
          const float3 d0 = make_float3(cold.f(kCDx), cold.f(kCDy), cold.f(kCDz));
          emit_second<(kMode & kModeFast) != 0>(rng, background, d0, ph.dir);
          ph.pos = make_float3(cold.f(kCOx), cold.f(kCOy), cold.f(kCOz));
          which = 2;
          start_photon(TG, kAnnihilation);
        } else {
          /* end of photon 2: its pair with photon 1; end of a prompt gamma
           * (which == 3): its pairs with photons 1 and 2, spurious */
          const bool prompt = (kMode & kModePrompt) && PS.prompt_energy > 0.0f;
          if (which == 2 && prompt) {
            if (escaped) {
              cold.setf(kCBx, ph.pos.x); cold.setf(kCBy, ph.pos.y); cold.setf(kCBz, ph.pos.z);
              cold.setf(kCBu, ph.dir.x); cold.setf(kCBv, ph.dir.y); cold.setf(kCBw, ph.dir.z);
              cold.setf(kCBe, ph.energy); cold.setf(kCBt, ph.travel);
              cold.u(kCBs) = (uint32_t)ph.state;
            } else {
              cold.setf(kCBe, -10.0f);
            }
          }
          const bool spurious = (kMode & kModePrompt) && which == 3;
          const int partners = spurious ? 2 : 1;
#pragma unroll 1
          for (int k = 0; k < partners; ++k) {
            const int f = k == 0 ? kCAx : kCBx;   /* photon 1 or photon 2: 9 fields in the same order */
            const float ea = cold.f(f + (kCAe - kCAx));
            if (escaped && ea > -0.5f) {
              PhotonState a;
              a.pos = make_float3(cold.f(f), cold.f(f + 1), cold.f(f + 2));
              a.dir = make_float3(cold.f(f + 3), cold.f(f + 4), cold.f(f + 5));
              a.energy = ea;
              a.travel = cold.f(f + (kCAt - kCAx));
              a.state = (int)cold.u(f + (kCAs - kCAx));
              const bool pass = spurious ? (PD.tally_type != 1)
                                         : (PD.tally_type == 0) || (PD.tally_type == 1 && ph.state == 0 && a.state == 0) ||
                                               (PD.tally_type == 2 && (ph.state != 0 || a.state != 0));
              if (pass) {
                unsigned long long det = 0;
                detect_pair<kCount, kRecord, !(kMode & kModeSino), (kMode & kModeFast) != 0>(rng, PD, make_float3(PD.cx, PD.cy, PD.cz),
                                                                  kBatch ? slots[scene].O : O,
                                             spec_sh, (int)cold.u(kCVox),
                                             cold.t_left(), ph, a, cnt, det,
                                             kRecord ? make_int2((int)cold.u(kCRx), (int)cold.u(kCRy))
                                                     : make_int2(0, 0),
                                             spurious);
                if (kBatch) cold.u(kCDet) += (uint32_t)det;
                else detected += det;
              }
            }
          }
          if (which == 2 && prompt && (PS.prompt_yield >= 1.0f || ranecu(rng) < PS.prompt_yield)) {
            /* the prompt gamma: isotropic from the decay point */
            emit_isotropic(rng, ph.dir);
            ph.pos = make_float3(cold.f(kCOx), cold.f(kCOy), cold.f(kCOz));
            which = 3;
            if (kBatch) cold.u(kCHist) += 1;
            else histories += 1;
            start_photon(TG, PS.prompt_energy);
          } else {
            phase = kPhDecay;
          }
        }
      }
      /* ---- next decay of the lane, or the next lane (MCGPU-PET_kernel.cu:259-298) */
      if (phase == kPhDecay) {
        for (;;) {
          if (__builtin_expect(!lane_live, 0)) {   /* rare branches hinted: cold code out of the hot paths */
            const uint64_t lane = claim_lane(O.lane_cursor);
            if (lane >= n_lanes) {
              phase = kPhDone;
              break;
            }
            uint64_t local = lane;
            const Emitter* plan = T.emitters;
            int plan_n = n_emitters;
            if (kBatch) {
              int lo = 0, hi = n_slots - 1;   /* last scene whose first lane is <= lane */
              while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(&slots[mid].first_lane) <= lane) lo = mid;
                else hi = mid - 1;
              }
              if (lo != scene) flush_lane();   /* totals go to a scene when the thread leaves it */
              scene = lo;
              local = lane - __ldg(&slots[scene].first_lane);
              plan = slots[scene].T.emitters;
              plan_n = slots[scene].P.n_emitters;
            }
            const Emitter* em = plan + find_emitter(plan, plan_n, local);
            const TransportParams& PN = kBatch ? slots[scene].P : P;
            /* the jump tables are the same for every scene: the launch's */
            const int seed = (!kBatch && (kMode & kModeChain)) ? __ldg(O.seed_word) : PN.seed;
            rng = rng_stream(P, seed, __ldg(&em->stream_base) + (local - __ldg(&em->first_lane)));
            cold.set_inv_rate(__ldg(&em->inv_rate));
            cold.set_t_left(PN.acq_ps);
            cold.u(kCVox) = __ldg(&em->voxel);
            lane_live = true;
            Counting<kCount>::add(cnt.lanes, 1);
          }
          const TransportParams& PN = kBatch ? slots[scene].P : P;
          double inv_act = cold.inv_rate();
          unsigned long long t_left = cold.t_left();
          const unsigned long long dt_ps = decay_interval<(kMode & kModeFast) != 0>(rng, inv_act, PN.inv_mean_life);
          if (__builtin_expect(!(dt_ps < t_left), 0)) {
            lane_live = false;
            continue;
          }
          cold.set_t_left(t_left - dt_ps);
          if (kBatch) {
            cold.u(kCHist) += 2;
            if (cold.u(kCHist) >= 0x80000000u) flush_lane();   /* keep the 32-bit word from wrapping */
          }
          else histories += 2;
          cold.set_inv_rate(inv_act);
          const int voxel = (int)cold.u(kCVox);
          if (kRecord) {
            cold.u(kCRx) = (uint32_t)rng.x;
            cold.u(kCRy) = (uint32_t)rng.y;
          }
          emit_first(rng, PN, voxel % PN.nx, (voxel / PN.nx) % PN.ny, voxel / (PN.nx * PN.ny), ph.pos, ph.dir);
          cold.setf(kCOx, ph.pos.x); cold.setf(kCOy, ph.pos.y); cold.setf(kCOz, ph.pos.z);
          cold.setf(kCDx, ph.dir.x); cold.setf(kCDy, ph.dir.y); cold.setf(kCDz, ph.dir.z);
          which = 1;
          start_photon((kBatch && !(kShare & kSharePhantom)) ? slots[scene].T : T, kAnnihilation);
          break;
        }
      }
    } else {
      /* ---- Woodcock sub-steps (MCGPU-PET_kernel.cu:313-393), repeated while
       * at least step_keep/8 of the warp's stepping photons still step */
      const int quorum = (__popc(m_step) * P.step_keep + 7) >> 3;
      for (;;) {
        if (phase == kPhStep) {
          const float E = ph.energy;
          bool go = true;
          if (fresh) {
            fresh = false;
            if (locate(PG, ph.pos.x, ph.pos.y, ph.pos.z) < 0) {
              escaped = true;
              phase = kPhEnd;
              go = false;
            }
          }
          if (go) {
            float step = -(mfp_w)*logf(ranecu(rng));
            ph.travel += step;
            ph.pos.x += step * ph.dir.x;
            ph.pos.y += step * ph.dir.y;
            ph.pos.z += step * ph.dir.z;
            const int vox = locate(PG, ph.pos.x, ph.pos.y, ph.pos.z);
            if (vox < 0) {
              escaped = true;
              phase = kPhEnd;
            } else if (__builtin_expect((unsigned long long)vox >= (unsigned long long)PG.n_voxels ||
                                            ++steps > steps_cap<kMode>(P), 0)) {
              Counting<true>::add(cnt.guard, 1);
              escaped = false;
              phase = kPhEnd;
            } else {
              const uint32_t key = TG.vox16 ? (uint32_t)__ldg(&TG.vox16[vox]) : __ldg(&TG.vox32[vox]);
              const PaletteEntry pe = (kBatch && !(kShare & kSharePhantom)) ? TG.palette[key] : pal[key];
              mat0 = pe.mat0;
              Counting<kCount>::add(cnt.steps, 1);
              const float2* rec = reinterpret_cast<const float2*>(TG.mfp + (size_t)index * kMaxMaterials + mat0);
              if (mat0 != mat_old) {
                const float2 ab = __ldg(rec);
                cax = ab.x;
                cbx = ab.y;
                mat_old = mat0;
                Counting<kCount>::add(cnt.refresh, 1);
              }
              const float mfp_density = mfp_w * pe.rho;
              float prob = 1.0f - mfp_density * (cax + E * cbx);
              const float randno = ranecu(rng);
              if (!(randno < prob)) {
                /* real interaction: the record of (energy bin, material) holds
                 * the same values the reference cached at the last change */
                const float2 cc = __ldg(rec + 1);   /* Compton coefficients; the rest only if needed */
                prob += mfp_density * (cc.x + E * cc.y);
                if (__builtin_expect(randno < prob, 1)) {
                  phase = kPhCompton;
                  is_compton = true;
                } else {
                  rec_hi = __ldg(reinterpret_cast<const float4*>(rec) + 1);
                  prob += mfp_density * (rec_hi.x + E * rec_hi.y);
                  if (randno < prob) {
                    phase = kPhCompton;
                    is_compton = false;
                    /* a batch keeps pmax in shared memory (fewer live registers) */
                    if (kBatch) cold.setf(kCPmax, rec_hi.z);
                  } else {
                    index = -11;
                    escaped = false;
                    phase = kPhEnd;
                    Counting<kCount>::add(cnt.photo, 1);
                    if (dose_on) {
                      const DoseSink ds{kBatch ? slots[scene].O.mat_dose : (O.mat_dose ? mdose_sh : nullptr),
                                        kBatch ? slots[scene].O.vox_dose : O.vox_dose};
                      ds(PS, -E, mat0, ph.pos);
                    }
                  }
                }
              }
            }
          }
        }
        if (__popc(__ballot_sync(0xffffffffu, phase == kPhStep)) < quorum) break;
      }
    }
  }

  /* a batched run's next launch may start placing its blocks as this
   * grid's blocks run out of lanes (programmatic dependent launch; no effect
   * on a launch without that dependency) */
  if (kBatch || (kMode & kModeChain)) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (kBatch) {
    flush_lane();
  } else {
    atomicAdd(O.histories, histories);
    if (detected) atomicAdd(O.coincidences, detected);
  }
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
  if (kDose && !kBatch && O.mat_dose && threadIdx.x < 2 * kMaxMaterials && mdose_sh[threadIdx.x])
    atomicAdd(&O.mat_dose[threadIdx.x], mdose_sh[threadIdx.x]);
  /* ... and does not complete before the previous launch has (all of whose
   * blocks are resident or done once this grid runs), so the stream's later
   * work sees every launch of the run finished; a no-op without a
   * programmatic dependency */
  if (kBatch || (kMode & kModeChain)) asm volatile("griddepcontrol.wait;" ::: "memory");
}

/* ---------------------------------------------------------- launch helpers */

/* Shared-memory carveout in percent (MCPET_CARVEOUT, for measurements), or
 * -1 for the largest shared-memory configuration. */
inline int carveout_percent() {
  static const int v = [] {
    const char* e = getenv("MCPET_CARVEOUT");
    if (!e || !*e) return -1;
    const int p = atoi(e);
    return (p >= 0 && p <= 100) ? p : -1;
  }();
  return v;
}

template <typename K>
cudaError_t occupancy_smem_attr(K kernel, size_t smem) {
  /* prefer shared memory over L1 so that the block count is set by registers */
  const int pct = carveout_percent();
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       pct >= 0 ? pct : (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  /* static + dynamic above 48 KB needs the opt-in, so always state the size */
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename K>
cudaError_t occupancy_of(K kernel, int block, size_t smem, int* bps) {
  cudaError_t e = occupancy_smem_attr(kernel, smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, kernel, block, smem);
}

/* The event kernel is compiled with its registers capped so that kEventBlocks
 * blocks of 256 threads stay resident per SM (a few spilled words cost less
 * than the lost warps); kAlgorithmEventsUncapped keeps the uncapped build. */
constexpr int kEventBlocks = 4;

using EventKernel = void (*)(TransportParams, DeviceTables, DeviceTallies, const SceneSlot*, int);
using HistoryKernel = void (*)(TransportParams, DeviceTables, DeviceTallies);

using EventKernel = void (*)(TransportParams, DeviceTables, DeviceTallies, const SceneSlot*, int);
using HistoryKernel = void (*)(TransportParams, DeviceTables, DeviceTallies);

/* One compiled variant of an event-kernel configuration: mode m when the
 * configuration supports it (its bits within kAllowed; the prompt gamma and
 * run-time caps are not combined), else none. */
template <bool C, int B, bool D, bool Bt, bool R, bool Do, int S, int kAllowed, int m>
EventKernel event_mode() {
  constexpr bool ok = (m & ~kAllowed) == 0 && !((m & kModePrompt) && (m & kModeCaps));
  if (!ok) return nullptr;
  return transport_events_kernel<C, B, D, Bt, R, Do, S, (ok ? m : 0)>;
}

template <bool C, int B, bool D, bool Bt, bool R, bool Do, int S, int kAllowed>
EventKernel event_variant(int mode) {
  switch (mode) {
    case 0: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 0>();
    case 1: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 1>();
    case 2: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 2>();
    case 3: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 3>();
    case 4: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 4>();
    case 5: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 5>();
    case 6: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 6>();
    case 7: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 7>();
    case 8: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 8>();
    case 9: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 9>();
    case 10: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 10>();
    case 11: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 11>();
    case 12: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 12>();
    case 13: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 13>();
    case 14: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 14>();
    case 15: return event_mode<C, B, D, Bt, R, Do, S, kAllowed, 15>();
    default: return nullptr;
  }
}

}  // namespace
}  // namespace mcpet
