/* Host (CPU, OpenMP) build of the REFERENCE's own transport kernel.
 *
 * TEST INFRASTRUCTURE ONLY -- built into oracle/_ref/libref_cpu.so by
 * oracle/ref/Makefile from the reference sources where they lie
 * (MCGPU-PET.h, MCGPU-PET_kernel.cu), with host_shim.h force-included.
 * Used as (1) the timed CPU baseline (kind "reference") and (2) the pin for
 * the C restatement in oracle/mcpet_oracle.c.  The product never links it.
 *
 * The driver reproduces the reference launch (MCGPU-PET.cu:457-483): one
 * "block" per voxel, threads_per_block "threads" per block.  Blocks are
 * distributed over host threads with a dynamic OpenMP schedule; the threads
 * of one block run sequentially (valid because the only __syncthreads in
 * track_particles follow thread 0's shared-memory set-up and precede exit,
 * MCGPU-PET_kernel.cu:248,460).
 */
#include "MCGPU-PET.h"
#include "MCGPU-PET_kernel.cu"

#include <omp.h>
#include <string.h>
#include <stdlib.h>
#include <vector>

thread_local shim_dim3 threadIdx, blockIdx, blockDim, gridDim;
thread_local void* shim_capture[SHIM_MAX_CAPTURE];
thread_local int shim_ncapture;

extern "C" {

/* Flat parameter block (own layout; filled by the Python tests). */
typedef struct {
  int nx, ny, nz;
  float inv_vx, inv_vy, inv_vz;
  float bbx, bby, bbz;
  int n_e;
  float e0, ide;
  float cx, cy, cz, radius, height;
  int psf_size, tally_psf_sino, tally_type;
  unsigned long long acq_ps;
  float mean_life;
  float e_resol, e_low, e_high, fovz;
  int nrows, ncrystals, nangles, nrad, nzs, nbins, res, nvoxs, ne, mrd, span, nsinos;
  int tpb, seed, peta;
} refc_params;

typedef struct {
  const float* fco; const float* uico; const float* fj0; const int* noscco;         /* 450,450,450,15 */
  const float* xco; const float* pco; const float* aco; const float* bco;          /* 1920 each */
  const float* pmax;                                                               /* 25005*15 */
  const unsigned char* itlco; const unsigned char* ituco;                          /* 1920 each */
} refc_tables;

static void fill_tables(const refc_tables* t, compton_struct* c, rayleigh_struct* r) {
  memcpy(c->fco, t->fco, sizeof(c->fco));
  memcpy(c->uico, t->uico, sizeof(c->uico));
  memcpy(c->fj0, t->fj0, sizeof(c->fj0));
  memcpy(c->noscco, t->noscco, sizeof(c->noscco));
  memcpy(r->xco, t->xco, sizeof(r->xco));
  memcpy(r->pco, t->pco, sizeof(r->pco));
  memcpy(r->aco, t->aco, sizeof(r->aco));
  memcpy(r->bco, t->bco, sizeof(r->bco));
  memcpy(r->pmax, t->pmax, sizeof(r->pmax));
  memcpy(r->itlco, t->itlco, sizeof(r->itlco));
  memcpy(r->ituco, t->ituco, sizeof(r->ituco));
}

static void fill_structs(const refc_params* p, detector_struct* d, source_struct* s) {
  memset(d, 0, sizeof(*d));
  memset(s, 0, sizeof(*s));
  d->PSF_center.x = p->cx; d->PSF_center.y = p->cy; d->PSF_center.z = p->cz;
  d->PSF_radius = p->radius; d->PSF_height = p->height;
  d->PSF_size = p->psf_size; d->tally_PSF_SINOGRAM = p->tally_psf_sino; d->tally_TYPE = p->tally_type;
  s->acquisition_time_ps = p->acq_ps; s->mean_life = p->mean_life;
}

static void set_constants(const refc_params* p, const short* roi) {
  voxel_data_CONST.num_voxels.x = p->nx; voxel_data_CONST.num_voxels.y = p->ny; voxel_data_CONST.num_voxels.z = p->nz;
  voxel_data_CONST.inv_voxel_size.x = p->inv_vx; voxel_data_CONST.inv_voxel_size.y = p->inv_vy;
  voxel_data_CONST.inv_voxel_size.z = p->inv_vz;
  voxel_data_CONST.size_bbox.x = p->bbx; voxel_data_CONST.size_bbox.y = p->bby; voxel_data_CONST.size_bbox.z = p->bbz;
  mfp_table_data_CONST.num_values = p->n_e; mfp_table_data_CONST.e0 = p->e0; mfp_table_data_CONST.ide = p->ide;
  if (roi) {
    dose_ROI_x_min_CONST = roi[0]; dose_ROI_x_max_CONST = roi[1];
    dose_ROI_y_min_CONST = roi[2]; dose_ROI_y_max_CONST = roi[3];
    dose_ROI_z_min_CONST = roi[4]; dose_ROI_z_max_CONST = roi[5];
  } else {
    dose_ROI_x_min_CONST = 32500; dose_ROI_x_max_CONST = -32500;
    dose_ROI_y_min_CONST = 32500; dose_ROI_y_max_CONST = -32500;
    dose_ROI_z_min_CONST = 32500; dose_ROI_z_max_CONST = -32500;
  }
  PETA_DEV[0] = (unsigned int)p->peta; PETA_DEV[1] = 0;
}

/* Full transport over all voxel blocks (or the listed subset), with the
 * reference's dose tallies when mat_dose (ulonglong2[15]) / vox_dose
 * (ulonglong2[ROI voxels], roi = x0,x1,y0,y1,z0,z1) are given: its host
 * branch adds to them without atomics, so use n_threads = 1 then.
 * Returns 0 on success. */
int refc_run2(const refc_params* p, const float* voxels /* float3[nvox] */,
              const float* woodcock /* float2[n_e] */, const float* mfp_a, const float* mfp_b,
              const refc_tables* tab,
              int* trues, int* scatter, int* img_t, int* img_s, int* spectrum,
              void* psf, int* index_psf, unsigned long long* total_histories,
              const int* block_list, long long n_block_list, int n_threads,
              unsigned long long* mat_dose, unsigned long long* vox_dose, const short* roi) {
  compton_struct* cmp = (compton_struct*)calloc(1, sizeof(compton_struct));
  rayleigh_struct* ray = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  if (!cmp || !ray) { free(cmp); free(ray); return -1; }
  fill_tables(tab, cmp, ray);
  detector_struct det; source_struct src;
  fill_structs(p, &det, &src);
  set_constants(p, vox_dose ? roi : nullptr);
  const long long nvox = (long long)p->nx * p->ny * p->nz;
  const long long nb = block_list ? n_block_list : nvox;
  unsigned long long hist = 0;
  int idx_psf = 0;
  if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
  {
#pragma omp for schedule(dynamic, 1)
    for (long long ib = 0; ib < nb; ++ib) {
      long long b = block_list ? block_list[ib] : ib;
      gridDim.x = p->nx; gridDim.y = p->ny; gridDim.z = p->nz;
      blockDim.x = p->tpb; blockDim.y = 1; blockDim.z = 1;
      blockIdx.x = (unsigned)(b % p->nx);
      blockIdx.y = (unsigned)((b / p->nx) % p->ny);
      blockIdx.z = (unsigned)(b / ((long long)p->nx * p->ny));
      for (int t = 0; t < p->tpb; ++t) {
        threadIdx.x = t; threadIdx.y = 0; threadIdx.z = 0;
        int seed_copy = p->seed;   /* the kernel's last thread overwrites it (MCGPU-PET_kernel.cu:454) */
        track_particles(&hist, &seed_copy, (PSF_element_struct*)psf, &idx_psf, (ulonglong2*)vox_dose,
                        (float3*)voxels, (float2*)woodcock, (float3*)mfp_a, (float3*)mfp_b,
                        ray, cmp, &det, &src, (ulonglong2*)mat_dose,
                        trues, scatter, img_t, img_s, spectrum,
                        p->e_resol, p->e_low, p->e_high, p->fovz, p->nrows, p->ncrystals,
                        p->nangles, p->nrad, p->nzs, p->nbins, p->res, p->nvoxs, p->ne,
                        p->mrd, p->span, p->nsinos);
      }
    }
  }
  *total_histories = hist;
  *index_psf = idx_psf;
  free(cmp); free(ray);
  return 0;
}

int refc_run(const refc_params* p, const float* voxels, const float* woodcock, const float* mfp_a,
             const float* mfp_b, const refc_tables* tab, int* trues, int* scatter, int* img_t, int* img_s,
             int* spectrum, void* psf, int* index_psf, unsigned long long* total_histories, const int* block_list,
             long long n_block_list, int n_threads) {
  return refc_run2(p, voxels, woodcock, mfp_a, mfp_b, tab, trues, scatter, img_t, img_s, spectrum, psf, index_psf,
                   total_histories, block_list, n_block_list, n_threads, nullptr, nullptr, nullptr);
}

/* RANECU jump-ahead and first draws (MCGPU-PET_kernel.cu:925-1083). */
void refc_prng(int n, int seed_input, const int* thread_ids, int ndraw,
               int* seeds_out /* 2n */, float* draws /* n*ndraw */, double* ddraws /* n*ndraw */) {
  for (int i = 0; i < n; ++i) {
    int2 s;
    init_PRNG(thread_ids[i], 555555, seed_input, &s);
    seeds_out[2 * i] = s.x; seeds_out[2 * i + 1] = s.y;
    int2 s2 = s;
    for (int d = 0; d < ndraw; ++d) draws[(long long)i * ndraw + d] = ranecu(&s);
    for (int d = 0; d < ndraw; ++d) ddraws[(long long)i * ndraw + d] = ranecu_double(&s2);
  }
}

int refc_abmodm(int m, int a, int s) { return abMODm(m, a, s); }

/* Detector model on a fixed event list (tally_Sinogram, MCGPU-PET_kernel.cu:1624-1836).
 * Per event writes: out[0]=sinogram bin or -1, out[1]=class (1 trues, 2 scatter, 0 none),
 * out[2]=spectrum bin of photon 2 or -1, out[3]=spectrum bin of photon 1 or -1,
 * out[4..5]=seed after the call. */
void refc_sinogram_events(const refc_params* p, int n,
                          const float* e2, const float* e1, const float* pos2, const float* pos1,
                          const float* dir2, const float* dir1, const signed char* st2,
                          const signed char* st1, const int* seeds, int* trues, int* scatter,
                          int* img_t, int* img_s, int* spectrum, int* out /* 6n */) {
  detector_struct det; source_struct src;
  fill_structs(p, &det, &src);
  blockIdx.x = blockIdx.y = blockIdx.z = 0;
  gridDim.x = gridDim.y = gridDim.z = 1;
  threadIdx.x = 0; blockDim.x = 1;
  for (int i = 0; i < n; ++i) {
    float E = e2[i], Ef = e1[i];
    float3 P = {pos2[3 * i], pos2[3 * i + 1], pos2[3 * i + 2]};
    float3 Pf = {pos1[3 * i], pos1[3 * i + 1], pos1[3 * i + 2]};
    float3 D = {dir2[3 * i], dir2[3 * i + 1], dir2[3 * i + 2]};
    float3 Df = {dir1[3 * i], dir1[3 * i + 1], dir1[3 * i + 2]};
    signed char s = st2[i], sf = st1[i];
    int2 seed = {seeds[2 * i], seeds[2 * i + 1]};
    unsigned long long acq = p->acq_ps;
    float td = 0.f, tdf = 0.f;
    float E_resol = p->e_resol, E_low = p->e_low, E_high = p->e_high, FOVZ = p->fovz;
    int NROWS = p->nrows, NCRYSTALS = p->ncrystals, NANGLES = p->nangles, NRAD = p->nrad,
        NZS = p->nzs, NBINS = p->nbins, RES = p->res, NVOXS = p->nvoxs, NE = p->ne, MRD = p->mrd,
        SPAN = p->span, NSINOS = p->nsinos;
    shim_ncapture = 0;
    tally_Sinogram(&E, &Ef, &P, &Pf, &D, &Df, &s, &sf, &det, &src, &acq, &td, &tdf, trues, scatter,
                   img_t, img_s, spectrum, &seed, &E_resol, &E_low, &E_high, &FOVZ, &NROWS,
                   &NCRYSTALS, &NANGLES, &NRAD, &NZS, &NBINS, &RES, &NVOXS, &NE, &MRD, &SPAN,
                   &NSINOS);
    int* o = out + 6 * i;
    o[0] = -1; o[1] = 0; o[2] = -1; o[3] = -1;
    int nspec = 0;
    for (int k = 0; k < shim_ncapture; ++k) {
      int* q = (int*)shim_capture[k];
      if (q >= trues && q < trues + p->nbins) { o[0] = (int)(q - trues); o[1] = 1; }
      else if (q >= scatter && q < scatter + p->nbins) { o[0] = (int)(q - scatter); o[1] = 2; }
      else if (q >= spectrum && q < spectrum + p->ne) {
        o[2 + (nspec < 2 ? nspec : 1)] = (int)(q - spectrum);
        nspec++;
      }
    }
    o[4] = seed.x; o[5] = seed.y;
  }
}

/* PENELOPE Compton sampling (GCOa, MCGPU-PET_kernel.cu:1335-1563) at given states. */
void refc_gcoa(int n, const float* energy_in, const int* mat_in, const int* seeds_in,
               const refc_tables* tab, float* energy_out, double* costh_out, int* seeds_out) {
  compton_struct* cmp = (compton_struct*)calloc(1, sizeof(compton_struct));
  rayleigh_struct* ray = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  fill_tables(tab, cmp, ray);
  for (int i = 0; i < n; ++i) {
    float e = energy_in[i]; int m = mat_in[i]; int2 s = {seeds_in[2 * i], seeds_in[2 * i + 1]};
    double c;
    GCOa(&e, &c, &m, &s, cmp);
    energy_out[i] = e; costh_out[i] = c; seeds_out[2 * i] = s.x; seeds_out[2 * i + 1] = s.y;
  }
  free(cmp); free(ray);
}

/* PENELOPE Rayleigh sampling (GRAa, MCGPU-PET_kernel.cu:1231-1296). */
void refc_graa(int n, const float* energy_in, const int* mat_in, const float* pmax_in,
               const int* seeds_in, const refc_tables* tab, double* costh_out, int* seeds_out) {
  compton_struct* cmp = (compton_struct*)calloc(1, sizeof(compton_struct));
  rayleigh_struct* ray = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  fill_tables(tab, cmp, ray);
  for (int i = 0; i < n; ++i) {
    float e = energy_in[i]; int m = mat_in[i]; float pm = pmax_in[i];
    int2 s = {seeds_in[2 * i], seeds_in[2 * i + 1]};
    double c;
    GRAa(&e, &c, &m, &pm, &s, ray);
    costh_out[i] = c; seeds_out[2 * i] = s.x; seeds_out[2 * i + 1] = s.y;
  }
  free(cmp); free(ray);
}

}  /* extern "C" */
