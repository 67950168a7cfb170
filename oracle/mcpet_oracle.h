/* CPU oracle of the MCGPU-PET photon-transport path -- TEST INFRASTRUCTURE.
 *
 * A plain C restatement of the reference algorithm (MCGPU-PET_kernel.cu),
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * leg as the checker.  It follows the reference's host-compilable arithmetic
 * (the #ifndef USING_CUDA branches and libm) so that it reproduces, bit for
 * bit, the reference kernel compiled for the host (oracle/_ref/libref_cpu.so);
 * that pin is checked by tests/test_oracle_pin.py.  Against the CUDA build the
 * agreement is statistical (libm vs. fast-math intrinsics round differently).
 */
#ifndef MCPET_ORACLE_H_
#define MCPET_ORACLE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_MATERIALS 15
#define ORC_MAX_SHELLS 30
#define ORC_NP_RAYLEIGH 128

typedef struct {
  int nx, ny, nz;
  float inv_vx, inv_vy, inv_vz;
  float bbx, bby, bbz;
  int n_e;
  float e0, ide;
  float cx, cy, cz, radius, height;
  int psf_capacity, tally_psf_sinogram, tally_type;
  unsigned long long acq_ps;
  float mean_life;
  float e_resol, e_low, e_high, fovz;
  int nrows, ncrystals, nangles, nrad, nzs, ne, mrd, span, nsinos;
  long long nbins;
  int tpb, seed, background;
  int dose_roi[6];             /* voxel dose ROI x0,x1,y0,y1,z0,z1 (0-based); x1 < 0: off */
  float prompt_energy;         /* prompt gamma per decay (eV), 0 = none (no reference counterpart) */
  float prompt_yield;          /* its probability per decay (>= 1: no draw) */
} orc_params;

typedef struct {
  const float* woodcock;       /* float2[n_e] */
  const float* mfp_a;          /* float3[n_e*15] */
  const float* mfp_b;          /* float3[n_e*15] */
  const float* pmax;           /* [n_e*15] */
  const float* fco;            /* [30*15], index mat + shell*15 */
  const float* uico;
  const float* fj0;
  const int* noscco;           /* [15] */
  const float* xco;            /* [15*128], index mat*128 + i */
  const float* pco;
  const float* aco;
  const float* bco;
  const unsigned char* itlco;
  const unsigned char* ituco;
} orc_tables;

typedef struct {
  int32_t* trues;
  int32_t* scatter;
  int32_t* image_trues;
  int32_t* image_scatter;
  int32_t* spectrum;
  unsigned char* psf;          /* psf_capacity records of 44 bytes, or NULL */
  int32_t psf_count;
  unsigned long long histories;
  /* event counters: woodcock steps inside the phantom, table refreshes,
   * majorant refreshes, int32 tally increments, photons, compton, rayleigh,
   * photoelectric, lanes */
  unsigned long long counters[9];
  unsigned long long* material_dose;   /* [15][2] or NULL (tally_materials_dose) */
  unsigned long long* voxel_dose;      /* [ROI voxels][2] or NULL (tally_voxel_energy_deposition) */
} orc_outputs;

/* Full transport over the reference lanes (tpb lanes per voxel with
 * activity > 1e-7 Bq, RANECU stream voxel*tpb + lane).  voxel_list (optional)
 * restricts the run to those voxels.  n_threads <= 0: OpenMP default. */
int orc_run(const orc_params* p, const orc_tables* t, const int32_t* mat0, const float* rho,
            const float* activity, const int32_t* voxel_list, long long n_list, int n_threads,
            orc_outputs* out);

/* RANECU stream start (reference jump, bit-serial modular exponentiation) and
 * the first ndraw float / double draws. */
void orc_rng(int seed, const int64_t* stream_ids, int n, int ndraw, int32_t* seeds_out, float* draws,
             double* ddraws);

/* Detector model on a fixed event list (same output layout as
 * mcpet_probe_detector). */
void orc_detector(const orc_params* p, int n, const float* e2, const float* e1, const float* pos2,
                  const float* pos1, const float* dir2, const float* dir1, const int8_t* st2,
                  const int8_t* st1, const int32_t* seeds, int32_t* out);

/* Sinogram bin of a pair of hit points, -1 outside (no energy blur). */
long long orc_sinogram_bin(const orc_params* p, float phi2, float z2, float phi1, float z1);

void orc_compton(const orc_tables* t, int n, const float* energy_in, const int32_t* mat,
                 const int32_t* seeds_in, float* energy_out, double* costh_out, int32_t* seeds_out);
void orc_rayleigh(const orc_tables* t, int n, const float* energy_in, const int32_t* mat,
                  const float* pmax, const int32_t* seeds_in, double* costh_out, int32_t* seeds_out);
void orc_source(int nx, int ny, int nz, const float inv_voxel_size[3], int background,
                const int32_t* seeds_in, float* out, int32_t* seeds_out);

/* NSEG / NSINOS of a sinogram geometry by the reference's running sum
 * (MCGPU-PET.cu:1176-1187). */
void orc_sinogram_sizes(int mrd, int span, int nzs, int* nseg, int* nsinos);

#ifdef __cplusplus
}
#endif
#endif
