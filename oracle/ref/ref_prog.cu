/* The reference program's host code, wrapped for tests.
 *
 * TEST INFRASTRUCTURE ONLY -- compiled by oracle/ref/Makefile into
 * oracle/_ref/libref_prog.so from MCGPU-PET.cu where it lies (it #includes
 * MCGPU-PET.h and MCGPU-PET_kernel.cu), unmodified, with the reference's
 * flags (-DUSING_CUDA -O3 -use_fast_math, Makefile:44) for sm_100a:
 *
 *   refio_*   the reference's parser and loaders (read_input
 *             MCGPU-PET.cu:866, load_voxels :1381, load_material :1565); host
 *             only, used to pin the product's parser and table builder.
 *   refp_run  the reference's transport run as main() performs it
 *             (MCGPU-PET.cu:228-535: parse, load, init_CUDA_device, zeroed
 *             tallies, one track_particles launch), with the launch bracketed
 *             by CUDA events so the reference kernel time on this GPU is
 *             measured on the device; tallies are returned in memory.
 */
#include "MCGPU-PET.cu"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ refio */
extern "C" {

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
  /* extra parse results */
  int gpu_id, nseg, flag_material_dose;
  float fact_object;
  short roi[6];
  float activity[MAX_MATERIALS];
  float density_max[MAX_MATERIALS];
  float density_nominal[MAX_MATERIALS];
  char voxel_file[250];
  char psf_file[250];
  char dose_file[250];
  char materials[MAX_MATERIALS][250];
} refio_config;

typedef struct {
  refio_config cfg;
  float3* voxels;
  float2* woodcock;
  float3* a;
  float3* b;
  compton_struct* cmp;
  rayleigh_struct* ray;
  PSF_element_struct* psf;
} refio_handle;

/* Parse the input file and load phantom + materials exactly as the reference
 * main() does up to the detector auto-centring (MCGPU-PET.cu:228-322).
 * Relative file names resolve against the current directory, as in the
 * reference.  The reference exit()s on malformed input. */
void* refio_open(const char* in_path) {
  refio_handle* h = (refio_handle*)calloc(1, sizeof(refio_handle));
  h->cmp = (compton_struct*)calloc(1, sizeof(compton_struct));
  h->ray = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  refio_config* c = &h->cfg;
  char arg0[] = "ref", arg1[1024];
  strncpy(arg1, in_path, sizeof(arg1) - 1);
  char* argv[] = {arg0, arg1, nullptr};
  unsigned long long total_histories = 0, psf_bytes = 0;
  int hpt = 0, num_projections = 1, voxels_Edep_bytes = 0;
  detector_struct det; source_struct src; source_energy_struct srce;
  memset(&det, 0, sizeof(det)); memset(&src, 0, sizeof(src)); memset(&srce, 0, sizeof(srce));
  char espc[250];
  double D_angle = -1.0, a0 = 0.0, a1 = 360.0, ia = 0.0, srad = -1.0, vt = 0.0;
  ulonglong2* vedep = nullptr;
  read_input(2, argv, 0, &total_histories, &c->seed, &c->gpu_id, &c->tpb, &hpt, &det, &h->psf,
             &psf_bytes, &src, &srce, c->voxel_file, c->materials, c->psf_file, espc,
             &num_projections, &D_angle, &a0, &a1, &ia, &vedep, &voxels_Edep_bytes, c->dose_file,
             &c->roi[0], &c->roi[1], &c->roi[2], &c->roi[3], &c->roi[4], &c->roi[5], &srad, &vt,
             &c->flag_material_dose, &c->fact_object, &c->e_resol, &c->e_low, &c->e_high, &c->fovz,
             &c->nrows, &c->ncrystals, &c->nangles, &c->nrad, &c->nzs, &c->nbins, &c->res,
             &c->nvoxs, &c->ne, &c->mrd, &c->span, &c->nseg, &c->nsinos);
  free(vedep);
  voxel_struct vd;
  unsigned int vbytes = 0;
  load_voxels(0, c->voxel_file, c->density_max, &c->fact_object, &vd, &h->voxels, &vbytes,
              &c->roi[1], &c->roi[3], &c->roi[5]);
  linear_interp lin;
  int wbytes = 0, tbytes = 0;
  load_material(0, c->materials, c->density_max, c->density_nominal, &lin, &h->woodcock, &wbytes,
                &h->a, &h->b, &tbytes, h->ray, h->cmp);
  if (det.PSF_radius < 0.0f) {   /* auto-centring performed by main(), MCGPU-PET.cu:316-322 */
    det.PSF_center.x = vd.size_bbox.x * 0.5f;
    det.PSF_center.y = vd.size_bbox.y * 0.5f;
    det.PSF_center.z = vd.size_bbox.z * 0.5f;
    det.PSF_radius = -det.PSF_radius;
  }
  c->nx = vd.num_voxels.x; c->ny = vd.num_voxels.y; c->nz = vd.num_voxels.z;
  c->inv_vx = vd.inv_voxel_size.x; c->inv_vy = vd.inv_voxel_size.y; c->inv_vz = vd.inv_voxel_size.z;
  c->bbx = vd.size_bbox.x; c->bby = vd.size_bbox.y; c->bbz = vd.size_bbox.z;
  c->n_e = lin.num_values; c->e0 = lin.e0; c->ide = lin.ide;
  c->cx = det.PSF_center.x; c->cy = det.PSF_center.y; c->cz = det.PSF_center.z;
  c->radius = det.PSF_radius; c->height = det.PSF_height; c->psf_size = det.PSF_size;
  c->tally_psf_sino = det.tally_PSF_SINOGRAM; c->tally_type = det.tally_TYPE;
  c->acq_ps = src.acquisition_time_ps; c->mean_life = src.mean_life;
  memcpy(c->activity, src.activity, sizeof(c->activity));
  c->peta = 1;
  return h;
}

void refio_get_config(void* hp, refio_config* out) { *out = ((refio_handle*)hp)->cfg; }
int refio_sizeof_config(void) { return (int)sizeof(refio_config); }

void refio_get_voxels(void* hp, float* out) {
  refio_handle* h = (refio_handle*)hp;
  memcpy(out, h->voxels, sizeof(float3) * (size_t)h->cfg.nx * h->cfg.ny * h->cfg.nz);
}

/* woodcock: float2[n_e]; a,b: float3[n_e*15]; then the flat Compton/Rayleigh arrays. */
void refio_get_tables(void* hp, float* woodcock, float* a, float* b, float* fco, float* uico,
                      float* fj0, int* noscco, float* xco, float* pco, float* aco, float* bco,
                      float* pmax, unsigned char* itlco, unsigned char* ituco) {
  refio_handle* h = (refio_handle*)hp;
  size_t ne = (size_t)h->cfg.n_e;
  memcpy(woodcock, h->woodcock, sizeof(float2) * ne);
  memcpy(a, h->a, sizeof(float3) * ne * MAX_MATERIALS);
  memcpy(b, h->b, sizeof(float3) * ne * MAX_MATERIALS);
  memcpy(fco, h->cmp->fco, sizeof(h->cmp->fco));
  memcpy(uico, h->cmp->uico, sizeof(h->cmp->uico));
  memcpy(fj0, h->cmp->fj0, sizeof(h->cmp->fj0));
  memcpy(noscco, h->cmp->noscco, sizeof(h->cmp->noscco));
  memcpy(xco, h->ray->xco, sizeof(h->ray->xco));
  memcpy(pco, h->ray->pco, sizeof(h->ray->pco));
  memcpy(aco, h->ray->aco, sizeof(h->ray->aco));
  memcpy(bco, h->ray->bco, sizeof(h->ray->bco));
  memcpy(pmax, h->ray->pmax, sizeof(h->ray->pmax));
  memcpy(itlco, h->ray->itlco, sizeof(h->ray->itlco));
  memcpy(ituco, h->ray->ituco, sizeof(h->ray->ituco));
}

void refio_close(void* hp) {
  refio_handle* h = (refio_handle*)hp;
  if (!h) return;
  free(h->voxels); free(h->woodcock); free(h->a); free(h->b); free(h->psf);
  free(h->cmp); free(h->ray); free(h);
}



}  /* extern "C" */


/* ------------------------------------------------------------------ refp */
extern "C" {

typedef struct {
  int* trues;            /* [nbins] or NULL */
  int* scatter;
  int* image_trues;      /* [nvox] or NULL */
  int* image_scatter;
  int* spectrum;         /* [ne] or NULL */
  void* psf;             /* psf_capacity*44 bytes or NULL */
  long long psf_capacity;
  int psf_count;
  unsigned long long total_histories;
  float kernel_ms;       /* track_particles, CUDA events */
  int nbins, nvox, ne;
  unsigned long long* material_dose;   /* ulonglong2[15] or NULL */
  unsigned long long* voxel_dose;      /* ulonglong2[voxel_dose_capacity] or NULL */
  long long voxel_dose_capacity;
  short roi[6];                        /* the ROI as the reference used it (after load_voxels' clipping) */
  long long n_roi;                     /* voxels of that ROI (0 when the voxel tally is off) */
} refp_outputs;

#define PCHK(x)                                                                        \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "refp: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return (int)e_;                                                                  \
    }                                                                                  \
  } while (0)

/* bg != 0 selects the background (second photon isotropic) mode of the
 * two-argument command line (MCGPU-PET.cu:81-84). */
int refp_run(const char* in_path, int bg, refp_outputs* out) {
  unsigned int peta[2] = {bg ? 0u : 1u, 0u};
  struct voxel_struct voxel_data;
  struct detector_struct detector_data;
  struct source_struct source_data;
  struct source_energy_struct source_energy_data;
  struct linear_interp mfp_table_data;
  struct compton_struct* compton_table = (compton_struct*)calloc(1, sizeof(compton_struct));
  struct rayleigh_struct* rayleigh_table = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  memset(&detector_data, 0, sizeof(detector_data));
  memset(&source_data, 0, sizeof(source_data));
  memset(&source_energy_data, 0, sizeof(source_energy_data));
  float3* voxel_mat_dens = NULL;
  unsigned int voxel_mat_dens_bytes = 0;
  float density_max[MAX_MATERIALS], density_nominal[MAX_MATERIALS];
  PSF_element_struct* PSF = NULL;
  unsigned long long PSF_bytes = 0;
  int mfp_table_bytes = -1, mfp_Woodcock_table_bytes = -1;
  float2* mfp_Woodcock_table = NULL;
  float3 *mfp_table_a = NULL, *mfp_table_b = NULL;
  short int roi[6];
  ulonglong2* voxels_Edep = NULL;
  int voxels_Edep_bytes = 0;
  ulonglong2 materials_dose[MAX_MATERIALS];
  memset(materials_dose, 0, sizeof(materials_dose));
  for (int k = 0; k < MAX_MATERIALS; k++) density_nominal[k] = -1.0f;
  unsigned long long total_histories;
  int histories_per_thread, seed_input, num_threads_per_block, gpu_id, num_projections = 1;
  float fact_object, E_resol, E_low, E_high, FOVZ;
  int NROWS, NCRYSTALS, NANGLES, NRAD, NZS, NBINS, RES, NVOXS, NE, MRD, SPAN, NSEG, NSINOS;
  int flag_material_dose = -2;
  double D_angle = -1.0, a0 = 0.0, a1 = 360.0, ia = 0.0, srad = -1.0, vt = 0.0;
  char file_name_voxels[250], file_name_materials[MAX_MATERIALS][250], file_name_output[250],
      file_dose_output[250], file_name_espc[250];
  char arg0[] = "ref", arg1[1024];
  strncpy(arg1, in_path, sizeof(arg1) - 1);
  arg1[sizeof(arg1) - 1] = 0;
  char* argv[] = {arg0, arg1, nullptr};
  read_input(2, argv, 0, &total_histories, &seed_input, &gpu_id, &num_threads_per_block, &histories_per_thread,
             &detector_data, &PSF, &PSF_bytes, &source_data, &source_energy_data, file_name_voxels,
             file_name_materials, file_name_output, file_name_espc, &num_projections, &D_angle, &a0, &a1, &ia,
             &voxels_Edep, &voxels_Edep_bytes, file_dose_output, &roi[0], &roi[1], &roi[2], &roi[3], &roi[4],
             &roi[5], &srad, &vt, &flag_material_dose, &fact_object, &E_resol, &E_low, &E_high, &FOVZ, &NROWS,
             &NCRYSTALS, &NANGLES, &NRAD, &NZS, &NBINS, &RES, &NVOXS, &NE, &MRD, &SPAN, &NSEG, &NSINOS);
  load_voxels(0, file_name_voxels, density_max, &fact_object, &voxel_data, &voxel_mat_dens, &voxel_mat_dens_bytes,
              &roi[1], &roi[3], &roi[5]);
  load_material(0, file_name_materials, density_max, density_nominal, &mfp_table_data, &mfp_Woodcock_table,
                &mfp_Woodcock_table_bytes, &mfp_table_a, &mfp_table_b, &mfp_table_bytes, rayleigh_table,
                compton_table);
  int NVOX_SIM = voxel_data.num_voxels.x * voxel_data.num_voxels.y * voxel_data.num_voxels.z;
  if (detector_data.PSF_radius < 0.0f) {
    detector_data.PSF_center.x = voxel_data.size_bbox.x * 0.5f;
    detector_data.PSF_center.y = voxel_data.size_bbox.y * 0.5f;
    detector_data.PSF_center.z = voxel_data.size_bbox.z * 0.5f;
    detector_data.PSF_radius = -detector_data.PSF_radius;
  }
  float3* voxel_mat_dens_device = NULL;
  float2* mfp_Woodcock_table_device = NULL;
  float3 *mfp_table_a_device = NULL, *mfp_table_b_device = NULL;
  struct rayleigh_struct* rayleigh_table_device = NULL;
  struct compton_struct* compton_table_device = NULL;
  ulonglong2* voxels_Edep_device = NULL;
  struct detector_struct* detector_data_device = NULL;
  struct source_struct* source_data_device = NULL;
  ulonglong2* materials_dose_device = NULL;
  int* seed_input_device = NULL;
  unsigned long long* total_histories_device = NULL;
  PSF_element_struct* PSF_device = NULL;
  int* index_PSF_device = NULL;
  int *True_dev = NULL, *Scatter_dev = NULL, *Imagen_T_dev = NULL, *Imagen_SC_dev = NULL,
      *Energy_Spectrum_dev = NULL;
  init_CUDA_device(&gpu_id, 0, 1, &voxel_data, &source_data, &source_energy_data, &detector_data,
                   &mfp_table_data, voxel_mat_dens, &voxel_mat_dens_device, voxel_mat_dens_bytes, PSF,
                   &PSF_device, PSF_bytes, &index_PSF_device, mfp_Woodcock_table, &mfp_Woodcock_table_device,
                   mfp_Woodcock_table_bytes, mfp_table_a, mfp_table_b, &mfp_table_a_device, &mfp_table_b_device,
                   mfp_table_bytes, rayleigh_table, &rayleigh_table_device, compton_table, &compton_table_device,
                   &detector_data_device, &source_data_device, voxels_Edep, &voxels_Edep_device,
                   voxels_Edep_bytes, &roi[0], &roi[1], &roi[2], &roi[3], &roi[4], &roi[5], materials_dose,
                   &materials_dose_device, flag_material_dose, &seed_input_device, &seed_input,
                   &total_histories_device, num_projections, NVOX_SIM, &True_dev, &Scatter_dev, &Imagen_T_dev,
                   &Imagen_SC_dev, &Energy_Spectrum_dev, &NBINS, &NE);
  PCHK(cudaMemset(True_dev, 0, (size_t)NBINS * sizeof(int)));
  PCHK(cudaMemset(Scatter_dev, 0, (size_t)NBINS * sizeof(int)));
  PCHK(cudaMemset(Imagen_T_dev, 0, (size_t)NVOX_SIM * sizeof(int)));
  PCHK(cudaMemset(Imagen_SC_dev, 0, (size_t)NVOX_SIM * sizeof(int)));
  PCHK(cudaMemset(Energy_Spectrum_dev, 0, (size_t)NE * sizeof(int)));
  PCHK(cudaMemcpyToSymbol(PETA_DEV, peta, 2 * sizeof(unsigned int), 0, cudaMemcpyHostToDevice));
  dim3 blocks(voxel_data.num_voxels.x, voxel_data.num_voxels.y, voxel_data.num_voxels.z);
  dim3 threads(num_threads_per_block, 1, 1);
  cudaEvent_t e0, e1;
  PCHK(cudaEventCreate(&e0));
  PCHK(cudaEventCreate(&e1));
  PCHK(cudaEventRecord(e0));
  track_particles<<<blocks, threads>>>(total_histories_device, seed_input_device, PSF_device, index_PSF_device,
                                       voxels_Edep_device, voxel_mat_dens_device, mfp_Woodcock_table_device,
                                       mfp_table_a_device, mfp_table_b_device, rayleigh_table_device,
                                       compton_table_device, detector_data_device, source_data_device,
                                       materials_dose_device, True_dev, Scatter_dev, Imagen_T_dev, Imagen_SC_dev,
                                       Energy_Spectrum_dev, E_resol, E_low, E_high, FOVZ, NROWS, NCRYSTALS,
                                       NANGLES, NRAD, NZS, NBINS, RES, NVOXS, NE, MRD, SPAN, NSINOS);
  PCHK(cudaGetLastError());
  PCHK(cudaEventRecord(e1));
  PCHK(cudaEventSynchronize(e1));
  PCHK(cudaEventElapsedTime(&out->kernel_ms, e0, e1));
  int index_PSF = 0;
  PCHK(cudaMemcpy(&out->total_histories, total_histories_device, sizeof(unsigned long long),
                  cudaMemcpyDeviceToHost));
  PCHK(cudaMemcpy(&index_PSF, index_PSF_device, sizeof(int), cudaMemcpyDeviceToHost));
  out->psf_count = index_PSF;
  out->nbins = NBINS;
  out->nvox = NVOX_SIM;
  out->ne = NE;
  if (out->trues) PCHK(cudaMemcpy(out->trues, True_dev, (size_t)NBINS * 4, cudaMemcpyDeviceToHost));
  if (out->scatter) PCHK(cudaMemcpy(out->scatter, Scatter_dev, (size_t)NBINS * 4, cudaMemcpyDeviceToHost));
  if (out->image_trues) PCHK(cudaMemcpy(out->image_trues, Imagen_T_dev, (size_t)NVOX_SIM * 4, cudaMemcpyDeviceToHost));
  if (out->image_scatter)
    PCHK(cudaMemcpy(out->image_scatter, Imagen_SC_dev, (size_t)NVOX_SIM * 4, cudaMemcpyDeviceToHost));
  if (out->spectrum) PCHK(cudaMemcpy(out->spectrum, Energy_Spectrum_dev, (size_t)NE * 4, cudaMemcpyDeviceToHost));
  for (int k = 0; k < 6; ++k) out->roi[k] = roi[k];
  out->n_roi = roi[1] > -1 ? (long long)(roi[1] - roi[0] + 1) * (roi[3] - roi[2] + 1) * (roi[5] - roi[4] + 1) : 0;
  if (out->material_dose && flag_material_dose == 1)
    PCHK(cudaMemcpy(out->material_dose, materials_dose_device, MAX_MATERIALS * sizeof(ulonglong2),
                    cudaMemcpyDeviceToHost));
  if (out->voxel_dose && out->n_roi > 0 && voxels_Edep_device) {
    long long n = out->n_roi < out->voxel_dose_capacity ? out->n_roi : out->voxel_dose_capacity;
    PCHK(cudaMemcpy(out->voxel_dose, voxels_Edep_device, (size_t)n * sizeof(ulonglong2), cudaMemcpyDeviceToHost));
  }
  if (out->psf && out->psf_capacity > 0) {
    long long n = index_PSF < detector_data.PSF_size ? index_PSF : detector_data.PSF_size;
    if (n > out->psf_capacity) n = out->psf_capacity;
    if (n > 0) PCHK(cudaMemcpy(out->psf, PSF_device, (size_t)n * sizeof(PSF_element_struct), cudaMemcpyDeviceToHost));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(voxel_mat_dens_device); cudaFree(PSF_device); cudaFree(index_PSF_device);
  cudaFree(mfp_Woodcock_table_device); cudaFree(mfp_table_a_device); cudaFree(mfp_table_b_device);
  cudaFree(rayleigh_table_device); cudaFree(compton_table_device); cudaFree(detector_data_device);
  cudaFree(source_data_device); cudaFree(seed_input_device); cudaFree(total_histories_device);
  cudaFree(voxels_Edep_device); cudaFree(materials_dose_device);
  cudaFree(True_dev); cudaFree(Scatter_dev); cudaFree(Imagen_T_dev); cudaFree(Imagen_SC_dev);
  cudaFree(Energy_Spectrum_dev);
  free(voxel_mat_dens); free(PSF); free(mfp_Woodcock_table); free(mfp_table_a); free(mfp_table_b);
  free(voxels_Edep); free(compton_table); free(rayleigh_table);
  return 0;
}

}  /* extern "C" */
