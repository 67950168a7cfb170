/* Plain-old-data structures shared by the host library (C++) and the CUDA
 * kernels.  Compiled by both g++ and nvcc. */
#pragma once
#include <stdint.h>

namespace mcpet {

constexpr int kMaxMaterials = 15;     /* MCGPU-PET.h:96 */
constexpr int kMaxShells = 30;        /* MCGPU-PET.h:97 */
constexpr int kNpRayleigh = 128;      /* MCGPU-PET.h:98 */
constexpr int kMaxEnergyBins = 25005; /* MCGPU-PET.h:99 */
constexpr int kLeapHistories = 555555;  /* histories_per_thread of the jump, MCGPU-PET_kernel.cu:252 */
constexpr int kLeapDistance = 256;      /* LEAP_DISTANCE, MCGPU-PET_kernel.cu:898 */
constexpr int kSpectrumSharedMax = 4096; /* spectrum bins privatised in shared memory */

/* Interaction record for one (energy bin, material): the interpolation
 * coefficients of the three inverse mean free paths (total, Compton,
 * Rayleigh; reference mfp_table_a/b, MCGPU-PET.cu:1688-1746) interleaved with
 * the Rayleigh form-factor maximum of the NEXT energy bin (the value GRAa is
 * called with, MCGPU-PET_kernel.cu:379).  32 bytes = one sector, fetched with
 * two 16-byte loads. */
struct alignas(16) MfpRecord {
  float ax, bx, ay, by;
  float az, bz, pmax_next;
  /* An upper bound, over the energies of this bin, of GCOa's rejection
   * normaliser S(E, theta = pi) of the material (its value two bin edges
   * up, times 1 + 1e-5; it grows with E).  Balanced lanes divide by it
   * instead of evaluating S(E, pi) per sampling: a larger constant in a
   * rejection sampler leaves the accepted distribution unchanged. */
  float s0_bound;
};

/* Distinct (material, density) pair of the phantom; voxels store an index. */
struct PaletteEntry {
  int32_t mat0;     /* 0-based material */
  float rho;        /* density g/cm^3 (already scaled by the density factor) */
};

/* Compton shell data (PENELOPE /CGCO/, reference compton_struct). */
struct ComptonTable {
  float fco[kMaxShells * kMaxMaterials];
  float uico[kMaxShells * kMaxMaterials];
  float fj0[kMaxShells * kMaxMaterials];
  int32_t noscco[kMaxMaterials];
};

/* Rayleigh RITA sampling rows (PENELOPE /CGRA/), indexed [mat*128 + i]. */
struct RayleighRows {
  const float* xco;
  const float* pco;
  const float* aco;
  const float* bco;
  const uint8_t* itl;
  const uint8_t* itu;
};

/* One emitting voxel of the lane plan.  Lanes [first_lane, first_lane+n)
 * belong to it; lane k of it uses RANECU stream stream_base + k. */
struct Emitter {
  double inv_rate;        /* lanes/activity  (reference: blockDim.x/activity, MCGPU-PET_kernel.cu:233) */
  uint32_t voxel;         /* linear voxel index (x fastest) */
  uint32_t n_lanes;
  uint64_t first_lane;
  uint64_t stream_base;
};

/* Everything a transport launch needs by value (kernel parameter space). */
struct TransportParams {
  /* voxel grid (voxel_struct, MCGPU-PET.h:262-271) */
  int nx, ny, nz;
  float inv_vx, inv_vy, inv_vz;
  float bbx, bby, bbz;
  long long n_voxels;
  /* energy grid (linear_interp) */
  int n_e;
  float e0, ide;
  /* detector (detector_struct) */
  float cx, cy, cz, radius, height;
  int psf_capacity;
  int tally_psf_sinogram, tally_type;
  /* source */
  unsigned long long acq_ps;
  double inv_mean_life;
  int background_mode;
  /* sinogram and energy window */
  float e_resol, e_low, e_high, fovz;
  int nrows, ncrystals, nangles, nrad, nzs, ne, mrd, span, nsinos;
  long long nbins;
  /* RANECU jump tables: (a^(555555*256))^(2^k) mod m, k = 0..31 */
  int32_t jump1[32];
  int32_t jump2[32];
  int seed;
  /* lane plan */
  uint64_t n_lanes;
  int n_emitters;
  int palette_in_shared;  /* palette size if staged in shared memory, else 0 */
  int spectrum_in_shared; /* 1 when ne <= kSpectrumSharedMax */
  int max_shells;         /* largest noscco over used materials */
  float e_annihilation;   /* 510998.95 eV, passed at run time */
  int quorum_scatter;     /* event loop: lanes needed to run a scattering round */
  int quorum_pair;        /* ... and a pair-bookkeeping (end of photon, next decay) round */
  int step_keep;          /* Woodcock batches continue while step_keep/8 of the stepping lanes step */
  int sino_dry;           /* 1: detector draws as usual but no sinogram, image, spectrum writes */
  int dose_roi[6];        /* voxel dose ROI x0,x1,y0,y1,z0,z1 (0-based, clamped); x1 < 0: off */
  int quorum_rayleigh;    /* event loop: Rayleigh lanes needed to join a round with Compton lanes */
  int max_steps;          /* Woodcock steps per photon before the guard drops it */
  int max_rejections;     /* iterations per sampler rejection loop before the guard drops the photon */
  float prompt_energy;    /* prompt gamma per decay (eV), 0 = none */
  float prompt_yield;     /* its probability per decay (1: no draw) */
};

/* Device pointers of one scene (all read-only during transport). */
struct DeviceTables {
  const uint16_t* vox16;          /* palette index per voxel when n_palette <= 65536 */
  const uint32_t* vox32;          /* palette index per voxel otherwise */
  const PaletteEntry* palette;
  int n_palette;
  const float* woodcock;          /* float2[n_e]: majorant mfp = x + E*y */
  const MfpRecord* mfp;           /* [n_e * 15] */
  const ComptonTable* compton;
  RayleighRows rayleigh;
  const Emitter* emitters;        /* [n_emitters], ordered by decreasing lane work */
};

/* Device pointers of the outputs of one run. */
struct DeviceTallies {
  int* trues;
  int* scatter;
  int* image_trues;
  int* image_scatter;
  int* spectrum;
  uint32_t* psf;                  /* 11 words per packed 44-byte record */
  int* psf_count;
  unsigned long long* histories;
  unsigned long long* coincidences;
  unsigned long long* counters;   /* 10 counters (mcpet_counters order) or NULL */
  unsigned long long* guard;      /* guard trips */
  unsigned long long* lane_cursor;/* lane work queue head */
  const unsigned long long* plan_counts; /* [lanes, emitters] on the device (device-built plans) */
  unsigned long long* mat_dose;   /* [15][2] material dose tally, or NULL */
  unsigned long long* vox_dose;    /* [ROI voxels][2] voxel dose tally, or NULL */
  uint32_t* events;               /* detected-coincidence records (EventRecord) for the gradient, or NULL */
  unsigned long long* event_count;
  long long event_capacity;
  const int* seed_word;           /* RANECU seed on the device (a batch's slot, advanced by graph
                                     replays), or NULL: P.seed */
};

/* One tallied coincidence, enough to replay its history: the lane's RANECU
 * state right before the emission, the emitting voxel and the sinogram bin. */
struct EventRecord {
  int32_t rng_x, rng_y;
  uint32_t voxel;
  uint32_t pad;
  long long bin;
};

/* One scene of a batched launch: its parameters (P.n_lanes, P.n_emitters:
 * its own lane plan T.emitters), tables and outputs, and the first lane of
 * the launch that belongs to it. */
struct SceneSlot {
  TransportParams P;
  DeviceTables T;
  DeviceTallies O;
  unsigned long long first_lane;
};

}  // namespace mcpet
