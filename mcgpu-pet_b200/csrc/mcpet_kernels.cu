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
 * is the single-precision direction rotation and decay clock of balanced
 * lanes; kModePrompt compiles the prompt-gamma emitter; kModeCaps reads the
 * loop guards' caps from the run parameters instead of the defaults.  A
 * variant carries none of the code of the features it leaves out. */
constexpr int kModeFast = kTransportFast, kModePrompt = kTransportPrompt, kModeCaps = kTransportCaps;

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
      if (!sample_compton(rng, energy, mat0, C, rn, costh, nullptr, rejections_cap<kMode>(P))) {
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
template <bool kCount, bool kRecord = true>
__device__ __forceinline__ void detect_pair(Rng& rng, const TransportParams& P, const float3 centre,
                                            const DeviceTallies& O, int* spec_sh, int voxel,
                                            unsigned long long t_left, const PhotonState& b, const PhotonState& a,
                                            LaneCounters& cnt, unsigned long long& detected, int2 rng_emit,
                                            bool spurious = false) {
  const bool want_sino = (P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 2);
  const bool want_psf = (P.tally_psf_sinogram == 0) || (P.tally_psf_sinogram == 1);
  if (want_sino) {
    float xb, yb, zb, xa, ya, za;
    to_cylinder(P, centre, b.pos, b.dir, xb, yb, zb);
    float phib = atan2f(yb, xb);
    if (fabsf(zb) < 0.5f * P.height) {
      to_cylinder(P, centre, a.pos, a.dir, xa, ya, za);
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
          /* sino_dry: the same draws, no sinogram-side writes (a PSF replay) */
          if ((ib < P.ne) && (ib >= 0) && !P.sino_dry) {
            if (spec_sh) atomicAdd(&spec_sh[ib], 1);
            else atomicAdd(&O.spectrum[ib], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if ((ia < P.ne) && (ia >= 0) && !P.sino_dry) {
            if (spec_sh) atomicAdd(&spec_sh[ia], 1);
            else atomicAdd(&O.spectrum[ia], 1);
            Counting<kCount>::add(cnt.tallies, 1);
          }
          if (eb > P.e_low && eb < P.e_high && ea > P.e_low && ea < P.e_high && !P.sino_dry) {
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
          detect_pair<kCount>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel, t_left, b, a, cnt, detected,
                              rng_emit);
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
            detect_pair<kCount>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel, t_left, g, a, cnt,
                                detected, rng_emit, true);
          if (esc_b)
            detect_pair<kCount>(rng, P, make_float3(P.cx, P.cy, P.cz), O, spec_sh, voxel, t_left, g, b, cnt,
                                detected, rng_emit, true);
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
       * quorum_rayleigh of them wait, so that most rounds run one sampler */
      const unsigned m_ray = __ballot_sync(0xffffffffu, phase == kPhCompton && !is_compton);
      const bool ray_now = (m_cmp == m_ray) || (__popc(m_ray) >= P.quorum_rayleigh);
      if (phase == kPhCompton && (is_compton || ray_now)) {
        double costh = 0.0;
        bool ok;
        float e = ph.energy;
        if (is_compton) {
          ok = sample_compton(rng, e, mat0, cmp, rn, costh, s0_ann, rejections_cap<kMode>(P));
        } else {
          ok = sample_rayleigh(rng, e, mat0, kBatch ? cold.f(kCPmax) : rec_hi.z, T.rayleigh, costh,
                               rejections_cap<kMode>(P));
        }
        if (!ok) {
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
                detect_pair<kCount, kRecord>(rng, PD, make_float3(PD.cx, PD.cy, PD.cz), kBatch ? slots[scene].O : O,
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
          if (!lane_live) {
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
            rng = rng_stream(P, PN.seed, __ldg(&em->stream_base) + (local - __ldg(&em->first_lane)));
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
          if (!(dt_ps < t_left)) {
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
            } else if ((unsigned long long)vox >= (unsigned long long)PG.n_voxels || ++steps > steps_cap<kMode>(P)) {
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
                const float4 lo = __ldg(reinterpret_cast<const float4*>(rec));
                rec_hi = __ldg(reinterpret_cast<const float4*>(rec) + 1);
                prob += mfp_density * (lo.z + E * lo.w);
                if (randno < prob) {
                  phase = kPhCompton;
                  is_compton = true;
                } else {
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
           sinogram_bin(P, phib, zb, phia, za) == bin;
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
 * the activity map on the device (expected decays over 3 lanes per
 * resident thread, clamped to [1, 4096]) */
__global__ void plan_hpl_kernel(int n_chunks, double t_s, int hpl, double resident_threads, NoAllocScratch* S) {
  if (threadIdx.x != 0) return;
  unsigned long long h = (unsigned long long)(hpl > 0 ? hpl : 1);
  if (hpl <= 0) {
    double A = 0.0;
    for (int c = 0; c < n_chunks; ++c) A += S->chunk_activity[c];
    double x = A * t_s / (resident_threads * 3.0);
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

/* Shared-memory carveout in percent (MCPET_CARVEOUT, for measurements), or
 * -1 for the largest shared-memory configuration. */
static int carveout_percent() {
  static const int v = [] {
    const char* e = getenv("MCPET_CARVEOUT");
    if (!e || !*e) return -1;
    const int p = atoi(e);
    return (p >= 0 && p <= 100) ? p : -1;
  }();
  return v;
}

template <typename K>
static cudaError_t occupancy_smem_attr(K kernel, size_t smem) {
  /* prefer shared memory over L1 so that the block count is set by registers */
  const int pct = carveout_percent();
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       pct >= 0 ? pct : (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  /* static + dynamic above 48 KB needs the opt-in, so always state the size */
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename K>
static cudaError_t occupancy_of(K kernel, int block, size_t smem, int* bps) {
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

/* The compiled variants of one event-kernel configuration, by mode: every
 * mode below kModes (the modes a configuration supports: 2 = fast only,
 * 4 = fast and prompt, 6 = also the caps, without prompt). */
template <bool C, int B, bool D, bool Bt, bool R, bool Do, int S, int kModes>
static EventKernel event_variant(int mode) {
  switch (mode) {
    case 0: return transport_events_kernel<C, B, D, Bt, R, Do, S, 0>;
    case kModeFast: return transport_events_kernel<C, B, D, Bt, R, Do, S, kModeFast>;
    case kModePrompt:
      if (kModes >= 4) return transport_events_kernel<C, B, D, Bt, R, Do, S, (kModes >= 4 ? kModePrompt : 0)>;
      return nullptr;
    case kModePrompt | kModeFast:
      if (kModes >= 4)
        return transport_events_kernel<C, B, D, Bt, R, Do, S, (kModes >= 4 ? kModePrompt | kModeFast : 0)>;
      return nullptr;
    case kModeCaps:
      if (kModes >= 6) return transport_events_kernel<C, B, D, Bt, R, Do, S, (kModes >= 6 ? kModeCaps : 0)>;
      return nullptr;
    case kModeCaps | kModeFast:
      if (kModes >= 6)
        return transport_events_kernel<C, B, D, Bt, R, Do, S, (kModes >= 6 ? kModeCaps | kModeFast : 0)>;
      return nullptr;
    default: return nullptr;
  }
}

/* Single-scene transport kernel of a run: algorithm, counters, mode. */
static EventKernel single_event_kernel(bool counters, int algorithm, int mode) {
  if (algorithm == kAlgorithmEventsDose)
    return counters ? event_variant<true, kEventBlocks, false, false, false, true, 0, 4>(mode)
                    : event_variant<false, kEventBlocks, false, false, false, true, 0, 4>(mode);
  if (algorithm == kAlgorithmEventsRecord)
    return counters ? event_variant<true, kEventBlocks, false, false, true, false, 0, 2>(mode)
                    : event_variant<false, kEventBlocks, false, false, true, false, 0, 2>(mode);
  if (algorithm == kAlgorithmEventsUncapped)
    return counters ? event_variant<true, 1, false, false, false, false, 0, 2>(mode)
                    : event_variant<false, 1, false, false, false, false, 0, 2>(mode);
  return counters ? event_variant<true, kEventBlocks, false, false, false, false, 0, 6>(mode)
                  : event_variant<false, kEventBlocks, false, false, false, false, 0, 6>(mode);
}

template <bool C>
static HistoryKernel history_variant(int mode) {
  switch (mode & 7) {
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

/* Batched transport kernel: counters, dose, shared scanner/phantom, mode
 * (fast, prompt). */
static EventKernel batch_event_kernel(bool counters, bool dose, int share, int mode) {
  if (dose)
    return counters ? event_variant<true, kEventBlocks, false, true, false, true, 0, 4>(mode)
                    : event_variant<false, kEventBlocks, false, true, false, true, 0, 4>(mode);
  if (counters) return event_variant<true, kEventBlocks, false, true, false, false, 0, 4>(mode);
  switch (share) {
    case kShareScanner:
      return event_variant<false, kEventBlocks, false, true, false, false, kShareScanner, 4>(mode);
    case kSharePhantom:
      return event_variant<false, kEventBlocks, false, true, false, false, kSharePhantom, 4>(mode);
    case kShareScanner | kSharePhantom:
      return event_variant<false, kEventBlocks, false, true, false, false, kShareScanner | kSharePhantom, 4>(mode);
    default:
      return event_variant<false, kEventBlocks, false, true, false, false, 0, 4>(mode);
  }
}

cudaError_t transport_batch_occupancy(bool counters, bool dose, int share, int mode, int block, size_t smem,
                                      int* blocks_per_sm) {
  EventKernel k = batch_event_kernel(counters, dose, share, mode);
  if (!k) return cudaErrorNotSupported;
  return occupancy_of(k, block, smem, blocks_per_sm);
}

cudaError_t launch_transport_batch(const TransportParams& P, const DeviceTables& T, const DeviceTallies& O,
                                   const SceneSlot* slots, int n_slots, bool counters, bool dose, int share, int mode,
                                   int grid, int block, size_t smem, cudaStream_t stream) {
  EventKernel k = batch_event_kernel(counters, dose, share, mode);
  if (!k) return cudaErrorNotSupported;
  k<<<grid, block, smem, stream>>>(P, T, O, slots, n_slots);
  return cudaGetLastError();
}

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
  EventKernel k = counters ? event_variant<true, kEventBlocks, true, false, false, false, 0, 4>(mode)
                           : event_variant<false, kEventBlocks, true, false, false, false, 0, 4>(mode);
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
  probe_source_kernel<<<(n + 127) / 128, 128, 0, s>>>(P, background, seeds, out);
  return cudaGetLastError();
}

}  // namespace mcpet
