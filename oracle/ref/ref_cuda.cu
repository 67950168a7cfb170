/* CUDA build of the REFERENCE's own code, wrapped for tests.
 *
 * TEST INFRASTRUCTURE ONLY -- compiled by oracle/ref/Makefile into
 * oracle/_ref/libref_cuda.so from the reference sources where they lie
 * (MCGPU-PET.cu, which #includes MCGPU-PET.h and MCGPU-PET_kernel.cu), with
 * the reference's own flags (-DUSING_CUDA -O3 -use_fast_math, Makefile:44)
 * retargeted to sm_100a:
 *
 *   refh_*   GPU harnesses that run the reference's device functions
 *            (init_PRNG/ranecu, source, GCOa, GRAa, tally_Sinogram) on a
 *            B200 so the product's kernels can be compared bit for bit on
 *            the same hardware.
 *
 * Every atomicAdd in the reference kernel file is routed through
 * capture_atomic_add, which performs the same add and also records the
 * target address per thread; tally harnesses decode the sinogram bin an
 * event landed in from it.  The product never links this library.
 */
#include <cuda_runtime.h>
#include <stdio.h>

__device__ unsigned long long* g_capture;   /* 8 slots per harness thread */

__device__ __forceinline__ void capture_record(void* p) {
  if (g_capture == nullptr) return;
  unsigned long long t = (unsigned long long)(blockIdx.x + (unsigned long long)gridDim.x *
                                                  (blockIdx.y + (unsigned long long)gridDim.y * blockIdx.z)) *
                             blockDim.x + threadIdx.x;
  unsigned long long* c = g_capture + t * 8;
  unsigned long long k = c[0];
  if (k < 7) { c[1 + k] = (unsigned long long)p; c[0] = k + 1; }
}
__device__ int capture_atomic_add(int* p, int v) { capture_record(p); return atomicAdd(p, v); }
__device__ unsigned long long capture_atomic_add(unsigned long long* p, unsigned long long v) {
  capture_record(p);
  return atomicAdd(p, v);
}
#define atomicAdd capture_atomic_add
#include "MCGPU-PET.cu"
#undef atomicAdd

#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* Parameter block of the harnesses (same leading layout as refc_params in
 * ref_cpu.cpp and refio_config in ref_prog.cu). */
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
} refh_params;
}

/* ------------------------------------------------------------------ refh */
#define HCHK(x)                                                                        \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "refh: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return (int)e_;                                                                  \
    }                                                                                  \
  } while (0)

template <typename T>
static T* dcopy(const T* h, size_t n) {
  T* d = nullptr;
  if (cudaMalloc((void**)&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
  if (h) cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
  else cudaMemset(d, 0, sizeof(T) * (n ? n : 1));
  return d;
}

__global__ void k_prng(int n, int seed_input, const int* tids, int ndraw, int2* seeds_out,
                       float* draws, double* ddraws) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int2 s;
  init_PRNG(tids[i], 555555, seed_input, &s);
  seeds_out[i] = s;
  int2 s2 = s;
  for (int d = 0; d < ndraw; ++d) draws[(size_t)i * ndraw + d] = ranecu(&s);
  for (int d = 0; d < ndraw; ++d) ddraws[(size_t)i * ndraw + d] = ranecu_double(&s2);
}

struct sino_geom {
  float e_resol, e_low, e_high, fovz;
  int nrows, ncrystals, nangles, nrad, nzs, nbins, res, nvoxs, ne, mrd, span, nsinos;
};

__global__ void k_sino(int n, const float* e2, const float* e1, const float3* pos2,
                       const float3* pos1, const float3* dir2, const float3* dir1,
                       const signed char* st2, const signed char* st1, int2* seeds,
                       detector_struct* det, source_struct* src, int* trues, int* scatter,
                       int* img_t, int* img_s, int* spectrum, sino_geom g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float E = e2[i], Ef = e1[i];
  float3 P = pos2[i], Pf = pos1[i], D = dir2[i], Df = dir1[i];
  signed char s = st2[i], sf = st1[i];
  int2 seed = seeds[i];
  unsigned long long acq = src->acquisition_time_ps;
  float td = 0.f, tdf = 0.f;
  tally_Sinogram(&E, &Ef, &P, &Pf, &D, &Df, &s, &sf, det, src, &acq, &td, &tdf, trues, scatter,
                 img_t, img_s, spectrum, &seed, &g.e_resol, &g.e_low, &g.e_high, &g.fovz,
                 &g.nrows, &g.ncrystals, &g.nangles, &g.nrad, &g.nzs, &g.nbins, &g.res, &g.nvoxs,
                 &g.ne, &g.mrd, &g.span, &g.nsinos);
  seeds[i] = seed;
}

__global__ void k_gcoa(int n, float* energy, const int* mat, int2* seeds, double* costh,
                       compton_struct* cmp) {
  __shared__ compton_struct sh;
  if (threadIdx.x == 0) sh = *cmp;
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float e = energy[i]; int m = mat[i]; int2 s = seeds[i]; double c;
  GCOa(&e, &c, &m, &s, &sh);
  energy[i] = e; costh[i] = c; seeds[i] = s;
}

__global__ void k_graa(int n, const float* energy, const int* mat, const float* pmax, int2* seeds,
                       double* costh, rayleigh_struct* ray) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float e = energy[i]; int m = mat[i]; float pm = pmax[i]; int2 s = seeds[i]; double c;
  GRAa(&e, &c, &m, &pm, &s, ray);
  costh[i] = c; seeds[i] = s;
}

/* One thread per voxel block: photon 1 then photon 2 of one pair. */
__global__ void k_source(int2* seeds, float3* out /* 4 per voxel: p1,d1,p2,d2 */) {
  int v = blockIdx.x + blockIdx.y * gridDim.x + blockIdx.z * gridDim.x * gridDim.y;
  int2 s = seeds[v];
  float energy, energyFirst;
  float3 position, direction, position1, direction1;
  direction1.x = 11.0f;
  source(&energy, &position, &direction, &position1, &direction1, &s, nullptr, &energyFirst);
  out[4 * v + 0] = position; out[4 * v + 1] = direction;
  source(&energy, &position, &direction, &position1, &direction1, &s, nullptr, &energyFirst);
  out[4 * v + 2] = position; out[4 * v + 3] = direction;
  seeds[v] = s;
}

extern "C" {

int refh_prng(int n, int seed_input, const int* tids, int ndraw, int* seeds_out, float* draws,
              double* ddraws) {
  int* d_t = dcopy(tids, n);
  int2* d_s = dcopy<int2>(nullptr, n);
  float* d_f = dcopy<float>(nullptr, (size_t)n * ndraw);
  double* d_d = dcopy<double>(nullptr, (size_t)n * ndraw);
  k_prng<<<(n + 127) / 128, 128>>>(n, seed_input, d_t, ndraw, d_s, d_f, d_d);
  HCHK(cudaDeviceSynchronize());
  cudaMemcpy(seeds_out, d_s, sizeof(int2) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(draws, d_f, sizeof(float) * n * ndraw, cudaMemcpyDeviceToHost);
  cudaMemcpy(ddraws, d_d, sizeof(double) * n * ndraw, cudaMemcpyDeviceToHost);
  cudaFree(d_t); cudaFree(d_s); cudaFree(d_f); cudaFree(d_d);
  return 0;
}

/* Same outputs as refc_sinogram_events in ref_cpu.cpp (6 ints per event). */
int refh_sinogram_events(const refh_params* p, int n, const float* e2, const float* e1,
                         const float* pos2, const float* pos1, const float* dir2,
                         const float* dir1, const signed char* st2, const signed char* st1,
                         const int* seeds, int* out) {
  detector_struct det; source_struct src;
  memset(&det, 0, sizeof(det)); memset(&src, 0, sizeof(src));
  det.PSF_center.x = p->cx; det.PSF_center.y = p->cy; det.PSF_center.z = p->cz;
  det.PSF_radius = p->radius; det.PSF_height = p->height;
  src.acquisition_time_ps = p->acq_ps;
  sino_geom g = {p->e_resol, p->e_low, p->e_high, p->fovz, p->nrows, p->ncrystals, p->nangles,
                 p->nrad, p->nzs, p->nbins, p->res, p->nvoxs, p->ne, p->mrd, p->span, p->nsinos};
  float* d_e2 = dcopy(e2, n); float* d_e1 = dcopy(e1, n);
  float3* d_p2 = dcopy((const float3*)pos2, n); float3* d_p1 = dcopy((const float3*)pos1, n);
  float3* d_d2 = dcopy((const float3*)dir2, n); float3* d_d1 = dcopy((const float3*)dir1, n);
  signed char* d_s2 = dcopy(st2, n); signed char* d_s1 = dcopy(st1, n);
  int2* d_seed = dcopy((const int2*)seeds, n);
  detector_struct* d_det = dcopy(&det, 1); source_struct* d_src = dcopy(&src, 1);
  int* d_t = dcopy<int>(nullptr, (size_t)p->nbins);
  int* d_s = dcopy<int>(nullptr, (size_t)p->nbins);
  /* tally_Sinogram indexes the emission image by block id: one slot per block */
  const int nblk = (n + 127) / 128;
  int* d_it = dcopy<int>(nullptr, nblk); int* d_is = dcopy<int>(nullptr, nblk);
  int* d_sp = dcopy<int>(nullptr, (size_t)p->ne);
  unsigned long long* d_cap = dcopy<unsigned long long>(nullptr, (size_t)n * 8);
  HCHK(cudaMemcpyToSymbol(g_capture, &d_cap, sizeof(d_cap)));
  k_sino<<<(n + 127) / 128, 128>>>(n, d_e2, d_e1, d_p2, d_p1, d_d2, d_d1, d_s2, d_s1, d_seed,
                                   d_det, d_src, d_t, d_s, d_it, d_is, d_sp, g);
  HCHK(cudaDeviceSynchronize());
  unsigned long long* cap = (unsigned long long*)malloc(sizeof(unsigned long long) * n * 8);
  int* sd = (int*)malloc(sizeof(int) * 2 * n);
  cudaMemcpy(cap, d_cap, sizeof(unsigned long long) * n * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(sd, d_seed, sizeof(int2) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; ++i) {
    int* o = out + 6 * i;
    o[0] = -1; o[1] = 0; o[2] = -1; o[3] = -1;
    int nspec = 0;
    unsigned long long* c = cap + (size_t)i * 8;
    for (unsigned long long k = 0; k < c[0] && k < 7; ++k) {
      unsigned long long q = c[1 + k];
      unsigned long long bt = (unsigned long long)d_t, bs = (unsigned long long)d_s,
                         bp = (unsigned long long)d_sp;
      if (q >= bt && q < bt + 4ull * p->nbins) { o[0] = (int)((q - bt) / 4); o[1] = 1; }
      else if (q >= bs && q < bs + 4ull * p->nbins) { o[0] = (int)((q - bs) / 4); o[1] = 2; }
      else if (q >= bp && q < bp + 4ull * p->ne) {
        o[2 + (nspec < 2 ? nspec : 1)] = (int)((q - bp) / 4);
        nspec++;
      }
    }
    o[4] = sd[2 * i]; o[5] = sd[2 * i + 1];
  }
  unsigned long long* nullcap = nullptr;
  cudaMemcpyToSymbol(g_capture, &nullcap, sizeof(nullcap));
  free(cap); free(sd);
  cudaFree(d_e2); cudaFree(d_e1); cudaFree(d_p2); cudaFree(d_p1); cudaFree(d_d2); cudaFree(d_d1);
  cudaFree(d_s2); cudaFree(d_s1); cudaFree(d_seed); cudaFree(d_det); cudaFree(d_src);
  cudaFree(d_t); cudaFree(d_s); cudaFree(d_it); cudaFree(d_is); cudaFree(d_sp); cudaFree(d_cap);
  return 0;
}

int refh_gcoa(int n, const float* energy_in, const int* mat_in, const int* seeds_in,
              const float* fco, const float* uico, const float* fj0, const int* noscco,
              float* energy_out, double* costh_out, int* seeds_out) {
  compton_struct c;
  memcpy(c.fco, fco, sizeof(c.fco)); memcpy(c.uico, uico, sizeof(c.uico));
  memcpy(c.fj0, fj0, sizeof(c.fj0)); memcpy(c.noscco, noscco, sizeof(c.noscco));
  compton_struct* d_c = dcopy(&c, 1);
  float* d_e = dcopy(energy_in, n); int* d_m = dcopy(mat_in, n);
  int2* d_s = dcopy((const int2*)seeds_in, n);
  double* d_c2 = dcopy<double>(nullptr, n);
  k_gcoa<<<(n + 127) / 128, 128>>>(n, d_e, d_m, d_s, d_c2, d_c);
  HCHK(cudaDeviceSynchronize());
  cudaMemcpy(energy_out, d_e, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(costh_out, d_c2, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(seeds_out, d_s, sizeof(int2) * n, cudaMemcpyDeviceToHost);
  cudaFree(d_c); cudaFree(d_e); cudaFree(d_m); cudaFree(d_s); cudaFree(d_c2);
  return 0;
}

int refh_graa(int n, const float* energy_in, const int* mat_in, const float* pmax_in,
              const int* seeds_in, const float* xco, const float* pco, const float* aco,
              const float* bco, const unsigned char* itlco, const unsigned char* ituco,
              double* costh_out, int* seeds_out) {
  rayleigh_struct* r = (rayleigh_struct*)calloc(1, sizeof(rayleigh_struct));
  memcpy(r->xco, xco, sizeof(r->xco)); memcpy(r->pco, pco, sizeof(r->pco));
  memcpy(r->aco, aco, sizeof(r->aco)); memcpy(r->bco, bco, sizeof(r->bco));
  memcpy(r->itlco, itlco, sizeof(r->itlco)); memcpy(r->ituco, ituco, sizeof(r->ituco));
  rayleigh_struct* d_r = dcopy(r, 1);
  free(r);
  float* d_e = dcopy(energy_in, n); int* d_m = dcopy(mat_in, n); float* d_p = dcopy(pmax_in, n);
  int2* d_s = dcopy((const int2*)seeds_in, n);
  double* d_c = dcopy<double>(nullptr, n);
  k_graa<<<(n + 127) / 128, 128>>>(n, d_e, d_m, d_p, d_s, d_c, d_r);
  HCHK(cudaDeviceSynchronize());
  cudaMemcpy(costh_out, d_c, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(seeds_out, d_s, sizeof(int2) * n, cudaMemcpyDeviceToHost);
  cudaFree(d_r); cudaFree(d_e); cudaFree(d_m); cudaFree(d_p); cudaFree(d_s); cudaFree(d_c);
  return 0;
}

/* Photon-pair source on a voxel grid; out: 12 floats per voxel (p1,d1,p2,d2). */
int refh_source(int nx, int ny, int nz, float inv_vx, float inv_vy, float inv_vz, int peta,
                const int* seeds_in, float* out, int* seeds_out) {
  voxel_struct vd;
  memset(&vd, 0, sizeof(vd));
  vd.num_voxels.x = nx; vd.num_voxels.y = ny; vd.num_voxels.z = nz;
  vd.inv_voxel_size.x = inv_vx; vd.inv_voxel_size.y = inv_vy; vd.inv_voxel_size.z = inv_vz;
  vd.size_bbox.x = nx / inv_vx; vd.size_bbox.y = ny / inv_vy; vd.size_bbox.z = nz / inv_vz;
  HCHK(cudaMemcpyToSymbol(voxel_data_CONST, &vd, sizeof(vd)));
  unsigned int pe[2] = {(unsigned int)peta, 0u};
  HCHK(cudaMemcpyToSymbol(PETA_DEV, pe, sizeof(pe)));
  size_t nv = (size_t)nx * ny * nz;
  int2* d_s = dcopy((const int2*)seeds_in, nv);
  float3* d_o = dcopy<float3>(nullptr, nv * 4);
  k_source<<<dim3(nx, ny, nz), 1>>>(d_s, d_o);
  HCHK(cudaDeviceSynchronize());
  cudaMemcpy(out, d_o, sizeof(float3) * nv * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(seeds_out, d_s, sizeof(int2) * nv, cudaMemcpyDeviceToHost);
  cudaFree(d_s); cudaFree(d_o);
  return 0;
}

}  /* extern "C" */
