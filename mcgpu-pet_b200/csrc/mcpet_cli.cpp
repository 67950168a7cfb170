/* mcpet.x -- drop-in command line for the transport path.
 *
 *   mcpet.x <input.in>          standard PET pairs
 *   mcpet.x <input.in> <any>    background mode (second photon isotropic),
 *                               the reference's two-argument form
 *                               (MCGPU-PET.cu:81-84)
 *
 * Reads the same input, voxel and material files as the reference and writes
 * the same output files into the current directory.  Environment knobs:
 *   MCPET_LANES=reference|balanced   lane plan (default reference: the
 *                                    reference's lanes and random streams)
 *   MCPET_HISTORIES_PER_LANE=N       balanced-mode lane size
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <chrono>
#include <vector>

#include "mcpet.h"

static int die(mcpet_status s) {
  fprintf(stderr, "\n!!mcpet ERROR!! (status %d) %s\n\n", (int)s, mcpet_last_error());
  return -(int)s;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s <input.in> [background-mode flag]\n", argv[0]);
    return -1;
  }
  const int bg = (argc == 3) ? 1 : 0;
  auto t0 = std::chrono::steady_clock::now();
  printf("\n    -- %s: reading '%s'%s\n", mcpet_version(), argv[1], bg ? " (background mode)" : "");
  mcpet_scene* sc = nullptr;
  mcpet_status s = mcpet_scene_load(argv[1], &sc);
  if (s != MCPET_OK) return die(s);
  mcpet_config cfg;
  mcpet_scene_get_config(sc, &cfg);
  mcpet_scene_info info;
  mcpet_scene_get_info(sc, &info);
  printf("       seed %d, phantom %d x %d x %d voxels (%lld emitting, %.6g Bq), acquisition %.6g s\n", cfg.seed,
         info.nx, info.ny, info.nz, info.n_emitting_voxels, info.total_activity_bq,
         cfg.acquisition_time_ps * 1e-12);
  printf("       detector R=%.5f H=%.5f centre (%.5f,%.5f,%.5f); sinogram %d x %d x %d (%lld bins)\n",
         cfg.detector_radius, cfg.detector_height, cfg.detector_center[0], cfg.detector_center[1],
         cfg.detector_center[2], cfg.n_radial, cfg.n_angles, cfg.n_sinograms, cfg.n_bins);
  if (cfg.tally_material_dose) printf("       Material dose deposition tally ENABLED.\n");
  if (cfg.tally_voxel_dose)
    printf("       3D voxel dose deposition tally ENABLED: ROI X[%d,%d], Y[%d,%d], Z[%d,%d] (%lld voxels)\n",
           cfg.dose_roi[0] + 1, cfg.dose_roi[1] + 1, cfg.dose_roi[2] + 1, cfg.dose_roi[3] + 1, cfg.dose_roi[4] + 1,
           cfg.dose_roi[5] + 1, info.n_dose_voxels);

  mcpet_run_opts opts;
  memset(&opts, 0, sizeof(opts));
  const char* lanes = getenv("MCPET_LANES");
  opts.lane_mode = (lanes && strcmp(lanes, "balanced") == 0) ? MCPET_LANES_BALANCED : MCPET_LANES_REFERENCE;
  const char* hpl = getenv("MCPET_HISTORIES_PER_LANE");
  opts.histories_per_lane = hpl ? atoi(hpl) : 0;
  opts.background_mode = bg;

  const bool sino = cfg.tally_psf_sinogram == 0 || cfg.tally_psf_sinogram == 2;
  const bool psf = cfg.tally_psf_sinogram == 0 || cfg.tally_psf_sinogram == 1;
  std::vector<int32_t> trues, scatter, img_t, img_s, spec(cfg.n_energy_bins > 0 ? cfg.n_energy_bins : 1);
  if (sino) {
    trues.assign((size_t)cfg.n_bins, 0);
    scatter.assign((size_t)cfg.n_bins, 0);
    img_t.assign((size_t)info.n_voxels, 0);
    img_s.assign((size_t)info.n_voxels, 0);
  }
  std::vector<unsigned char> psf_buf;
  if (psf && cfg.psf_size > 0) psf_buf.assign((size_t)cfg.psf_size * MCPET_PSF_RECORD_BYTES, 0);
  int32_t psf_count = 0;
  unsigned long long hist = 0;
  double ms = 0;
  mcpet_tallies t;
  memset(&t, 0, sizeof(t));
  if (sino) {
    t.trues = trues.data();
    t.scatter = scatter.data();
    t.image_trues = img_t.data();
    t.image_scatter = img_s.data();
  }
  t.spectrum = spec.data();
  t.psf = psf_buf.empty() ? nullptr : psf_buf.data();
  t.psf_capacity = psf_buf.empty() ? 0 : cfg.psf_size;
  t.psf_count = &psf_count;
  t.total_histories = &hist;
  t.transport_ms = &ms;
  std::vector<unsigned long long> mdose(2 * MCPET_MAX_MATERIALS, 0), vdose((size_t)(2 * info.n_dose_voxels), 0);
  if (cfg.tally_material_dose) t.material_dose = mdose.data();
  if (info.n_dose_voxels > 0) t.voxel_dose = vdose.data();
  auto t1 = std::chrono::steady_clock::now();
  s = mcpet_run(sc, &opts, &t);
  if (s != MCPET_OK) return die(s);
  auto t2 = std::chrono::steady_clock::now();
  double run_s = std::chrono::duration<double>(t2 - t1).count();
  s = mcpet_write_outputs(sc, &t, nullptr, bg, ms * 1e-3);
  if (s != MCPET_OK) return die(s);
  long long st = 0, ss = 0;
  for (int32_t v : trues) st += v;
  for (int32_t v : scatter) ss += v;
  double total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("\n       Total number of histories simulated = %llu (each annihilation produces 2)\n", hist);
  if (psf) printf("       Elements stored in the PSF = %d (capacity %d)\n", psf_count, cfg.psf_size);
  if (sino) {
    printf("       Trues in the sinogram = %lld, scatter = %lld\n", st, ss);
    printf("       Transport kernel time = %.3f s, run incl. transfers = %.3f s, total = %.3f s\n", ms * 1e-3, run_s,
           total_s);
    if (ms > 0) printf("       Detected coincidences per second (transport) = %.4g\n", (st + ss) / (ms * 1e-3));
  }
  if (cfg.tally_material_dose) {
    /* the materials dose report goes to the standard output, as the reference's */
    FILE* f = fopen("materials_dose.txt", "r");
    if (f) {
      char buf[4096];
      size_t n;
      while ((n = fread(buf, 1, sizeof(buf), f)) > 0) fwrite(buf, 1, n, stdout);
      fclose(f);
    }
  }
  mcpet_scene_free(sc);
  return 0;
}
