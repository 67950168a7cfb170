/* mcpet.h -- C ABI of the B200 (sm_100a) photon-transport path of MCGPU-PET.
 *
 * The reference has no library API: its transport path is reached through the
 * command line program (MCGPU-PET.cu:77-840) and, inside it, through the
 * track_particles kernel contract (MCGPU-PET_kernel.cu:153-187, prototype
 * MCGPU-PET.h:523-524) fed by read_input / load_voxels / load_material /
 * init_CUDA_device.  Each entry point below names the reference code it
 * replaces.  All functions return an mcpet_status and never exit(); the text
 * of the last error on the calling thread is available from mcpet_last_error.
 *
 * Plain C types only.  Host buffers are caller-owned.  Device pointers (the
 * *_device entry points) are caller-owned CUDA allocations on the scene's
 * device; work is ordered on the caller's stream (cudaStream_t passed as
 * void*; NULL = legacy default stream).
 */
#ifndef MCPET_H_
#define MCPET_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCPET_MAX_MATERIALS 15   /* MCGPU-PET.h:96 */
#define MCPET_MAX_SHELLS 30      /* MCGPU-PET.h:97 */
#define MCPET_NP_RAYLEIGH 128    /* MCGPU-PET.h:98 */
#define MCPET_MAX_ENERGY_BINS 25005 /* MCGPU-PET.h:99 (MAX_ENERGYBINS_RAYLEIGH) */
#define MCPET_PSF_RECORD_BYTES 44 /* packed PSF_element_struct, MCGPU-PET.h:235-247 */

typedef enum {
  MCPET_OK = 0,
  MCPET_ERR_ARG = 1,        /* invalid argument or unsupported value */
  MCPET_ERR_IO = 2,         /* file missing / unreadable / unwritable */
  MCPET_ERR_FORMAT = 3,     /* malformed input, voxel or material file */
  MCPET_ERR_CUDA = 4,       /* CUDA runtime error */
  MCPET_ERR_NOMEM = 5,      /* host or device allocation failed */
  MCPET_ERR_LIMIT = 6,      /* a size limit of the format was exceeded */
  MCPET_ERR_DEVICE = 7      /* a device-side guard fired (loop cap, bad index) */
} mcpet_status;

/* Lane decomposition of the emission process. */
typedef enum {
  /* One lane per (emitting voxel, thread) with threads_per_block lanes per
   * voxel and RANECU stream id voxel*threads_per_block+thread: the lane set
   * and random streams of the reference launch (MCGPU-PET.cu:457-483,
   * MCGPU-PET_kernel.cu:251-253).  Histories replay the reference's. */
  MCPET_LANES_REFERENCE = 0,
  /* Lanes per voxel proportional to its expected decays (about
   * histories_per_lane decays each), stream ids = lane index.  Same emission
   * statistics (sum of independent Poisson processes), balanced work. */
  MCPET_LANES_BALANCED = 1
} mcpet_lane_mode;

/* Everything the reference reads from its input file (read_input,
 * MCGPU-PET.cu:866-1280), in the same units.  acquisition_time_ps is
 * (unsigned long long)(seconds*1e12+0.5) as at MCGPU-PET.cu:979. */
typedef struct {
  /* [SECTION SIMULATION CONFIG v.2016-07-05] */
  int seed;                       /* 0 in the file = time-based seed (resolved at parse time) */
  int gpu_id;
  int threads_per_block;
  float density_factor;           /* "fact_object" */
  /* [SECTION SOURCE PET SCAN v.2017-03-14] */
  unsigned long long acquisition_time_ps;
  float mean_life;
  float material_activity[MCPET_MAX_MATERIALS]; /* parsed; unused by the transport (as in the reference) */
  /* [SECTION PHASE SPACE FILE v.2016-07-05] */
  char psf_file[250];
  float detector_center[3];       /* after auto-centring when radius was < 0 */
  float detector_height;
  float detector_radius;
  int psf_size;
  int tally_type;                 /* 0 both, 1 trues only, 2 scatter only */
  int tally_psf_sinogram;         /* 0 both, 1 PSF only, 2 sinogram only */
  int detector_auto_center;       /* 1 when the file gave a negative radius */
  /* [SECTION DOSE DEPOSITION v.2012-12-12] */
  int tally_material_dose;        /* 1 YES, 0 NO */
  int tally_voxel_dose;           /* 1 YES, 0 NO */
  char dose_file[250];
  short dose_roi[6];              /* x_min,x_max,y_min,y_max,z_min,z_max (0-based) */
  /* [SECTION ENERGY PARAMETERS v.2019-04-25] (eV despite the file's label) */
  float energy_resolution;
  float energy_window_low;
  float energy_window_high;
  /* [SECTION SINOGRAM PARAMETERS v.2019-04-25] */
  float fov_z;
  int n_rows, n_crystals, n_angles, n_radial, n_z_slices, image_res, n_energy_bins;
  int max_ring_difference, span;
  int n_segments, n_sinograms;    /* derived as at MCGPU-PET.cu:1176-1187 */
  long long n_bins;               /* n_radial*n_angles*n_sinograms, 64-bit */
  /* [SECTION VOXELIZED GEOMETRY FILE v.2009-11-30] / [SECTION MATERIAL FILE LIST] */
  char voxel_file[250];
  char material_files[MCPET_MAX_MATERIALS][250];
  /* Optional [SECTION PROMPT GAMMA EMISSION v.2026-12-01], placed before the
   * voxel-file section (the reference skips it while it looks for that
   * section, MCGPU-PET.cu:1190-1202): an isotope that also emits a prompt
   * gamma of this energy (eV) with this yield per decay (0 < yield <= 1),
   * e.g. 1157020 eV at 1.0 for 44Sc.  The gamma leaves the decay point
   * isotropically after the annihilation pair; every pair it forms with a
   * detected annihilation photon is a candidate coincidence (spurious,
   * tallied with the scatter).  No counterpart in the reference, which emits
   * only 511 keV photons (MCGPU-PET_kernel.cu:669).  0 = no prompt gamma.
   * Needs material tables that reach above the gamma energy and the
   * sinogram tally only. */
  float prompt_gamma_energy;
  float prompt_gamma_yield;
} mcpet_config;

typedef struct mcpet_scene mcpet_scene;   /* opaque: phantom + tables + device copy */

typedef struct {
  int nx, ny, nz;
  float voxel_size[3];
  float bbox[3];
  long long n_voxels;
  long long n_emitting_voxels;
  double total_activity_bq;
  int n_energy;                   /* rows of the material tables */
  float e0, inv_de;               /* first energy (eV), inverse step (1/eV) */
  int n_materials_used;
  int n_palette;                  /* distinct (material, density) pairs in the phantom */
  float density_max[MCPET_MAX_MATERIALS];
  float density_nominal[MCPET_MAX_MATERIALS];
  long long n_bins;
  int n_energy_spectrum;
  int n_emitters;                 /* lane plan of the last run */
  long long n_lanes;
  long long last_h2d_bytes;       /* bytes copied host->device by the last run */
  long long n_dose_voxels;        /* voxels of the dose ROI (0 when the voxel dose tally is off) */
} mcpet_scene_info;

typedef struct {
  int lane_mode;                  /* mcpet_lane_mode */
  int background_mode;            /* 1 = second photon isotropic (reference's 2-argument CLI, PETA_DEV[0]==0) */
  int histories_per_lane;         /* balanced mode: expected decays per lane (<=0: automatic) */
  int block_threads;              /* CUDA threads per block of the transport kernel (<=0: automatic) */
  int blocks_per_sm;              /* resident blocks per SM for the persistent grid (<=0: automatic) */
  int collect_counters;           /* 1: also fill mcpet_tallies.counters (slower kernel variant) */
  int seed_override;              /* != 0: use this RANECU seed instead of the scene's */
  void* stream;                   /* cudaStream_t; NULL = default stream */
  int algorithm;                  /* 0 automatic, 1 history loop per thread, 2 warp-regrouped event loop
                                     (same results, different schedule) */
  /* Device loop guards.  The reference's Woodcock loop and the rejection
   * loops of GCOa / GRAa are unbounded (MCGPU-PET_kernel.cu:319-342, 1247,
   * 1390-1526); here a photon that takes more Woodcock steps, or more
   * iterations in one rejection loop, than these caps is dropped and counted
   * as a guard trip (the run then returns MCPET_ERR_DEVICE).  <= 0: the
   * defaults, 2^20 steps and 2^16 iterations, which physical input never
   * reaches. */
  int max_woodcock_steps;
  int max_rejections;
} mcpet_run_opts;

/* Event counters (when collect_counters=1). */
typedef struct {
  unsigned long long woodcock_steps_inside;  /* steps that landed inside the phantom */
  unsigned long long table_refreshes;        /* (material, energy) table reloads */
  unsigned long long majorant_refreshes;     /* energy changes (Woodcock table reads) */
  unsigned long long tally_increments;       /* int32 tally increments (sinogram+image+spectrum) */
  unsigned long long photons;                /* photon histories started */
  unsigned long long compton, rayleigh, photoelectric;
  unsigned long long lanes;
  unsigned long long guard_trips;            /* loop caps / index guards that fired */
} mcpet_counters;

/* Output tallies (int32 as in the reference, MCGPU-PET.cu:279-298).
 * Any pointer may be NULL to skip that download / tally. */
typedef struct {
  int32_t* trues;                 /* [n_bins] sinogram of true coincidences */
  int32_t* scatter;               /* [n_bins] sinogram of scatter coincidences */
  int32_t* image_trues;           /* [n_voxels] emission voxel of detected trues */
  int32_t* image_scatter;         /* [n_voxels] emission voxel of detected scatter */
  int32_t* spectrum;              /* [n_energy_spectrum] 1 keV bins, before the window */
  void* psf;                      /* psf_capacity packed 44-byte records */
  long long psf_capacity;         /* elements; the reference's PSF_size */
  int32_t* psf_count;             /* the reference's index_PSF after the run */
  unsigned long long* total_histories;  /* photons (2 per decay), MCGPU-PET_kernel.cu:282 */
  unsigned long long* coincidences;     /* detected pairs = sum(trues) + sum(scatter) */
  mcpet_counters* counters;
  double* transport_ms;           /* device time of the transport kernel(s) */
  /* dose tallies (when the input enables them; tally_materials_dose and
   * tally_voxel_energy_deposition, MCGPU-PET_kernel.cu:396-410, 1593-1650):
   * per pair {sum of Edep in eV (SCALE_eV = 1), sum of Edep^2}, each term
   * rounded to an integer as the reference's device build does */
  unsigned long long* material_dose;    /* [MCPET_MAX_MATERIALS][2] or NULL */
  unsigned long long* voxel_dose;       /* [n_dose_voxels][2] ROI voxels, x fastest, or NULL */
} mcpet_tallies;

/* ---- configuration and scene (host) ---------------------------------- */

/* Parse an input file.  Replaces read_input (MCGPU-PET.cu:866-1280) incl. the
 * NSEG/NSINOS/NBINS derivation (:1176-1189).  Relative paths inside the file
 * are kept as written (resolved against the working directory on load, as the
 * reference does). */
mcpet_status mcpet_config_read(const char* in_path, mcpet_config* cfg);

/* Parse the input file, read the .vox phantom and material tables and build
 * the interpolation tables.  Replaces read_input + load_voxels
 * (MCGPU-PET.cu:1381-1533) + load_material (:1565-1831) + the detector
 * auto-centring in main (:316-322) + the 511 keV coverage check (:344-351). */
mcpet_status mcpet_scene_load(const char* in_path, mcpet_scene** out);

/* Same as mcpet_scene_load but from in-memory voxel arrays (x fastest, then
 * y, then z; material 1-based as in the .vox file; density before the
 * density_factor scale).  Material tables are read from cfg->material_files. */
mcpet_status mcpet_scene_from_arrays(const mcpet_config* cfg, int nx, int ny, int nz,
                                     const float voxel_size_cm[3], const int32_t* material,
                                     const float* density, const float* activity,
                                     mcpet_scene** out);

/* Replace the per-voxel activity (Bq) of an existing scene, same length as the
 * phantom.  The device copy is refreshed lazily on the next run. */
mcpet_status mcpet_scene_set_activity(mcpet_scene* scene, const float* activity);

mcpet_status mcpet_scene_get_config(const mcpet_scene* scene, mcpet_config* cfg);
mcpet_status mcpet_scene_get_info(const mcpet_scene* scene, mcpet_scene_info* info);

/* Export the host tables built by the loader, in the reference layout
 * (MCGPU-PET.h:206-360): woodcock float2[n_e] (x=a, y=b), mfp_a/mfp_b
 * float3[n_e*15], voxels float3[n_voxels] (material+0.0001, density,
 * activity).  Compton/Rayleigh arrays as the struct members.  Any pointer may
 * be NULL.  Used by the parity tests against the reference loaders. */
mcpet_status mcpet_scene_export_tables(const mcpet_scene* scene, float* woodcock, float* mfp_a,
                                       float* mfp_b, float* voxels, float* fco, float* uico,
                                       float* fj0, int32_t* noscco, float* xco, float* pco,
                                       float* aco, float* bco, float* pmax, uint8_t* itlco,
                                       uint8_t* ituco);

void mcpet_scene_free(mcpet_scene* scene);

/* ---- transport on the GPU ---------------------------------------------- */

/* Select the CUDA device (<0: the scene's gpu_id, clamped to the available
 * devices) and upload the scene (palette-compressed voxels, tables, lane
 * plan).  Replaces init_CUDA_device (MCGPU-PET.cu:1842-2146).  Called
 * implicitly by the run functions. */
mcpet_status mcpet_scene_to_device(mcpet_scene* scene, int device);

/* End-to-end run with HOST output buffers: zero the device tallies, run the
 * transport, download the tallies into *out.  Replaces the launch and
 * downloads of main (MCGPU-PET.cu:408-535).  Blocking. */
mcpet_status mcpet_run(mcpet_scene* scene, const mcpet_run_opts* opts, mcpet_tallies* out);

/* Run with DEVICE output buffers (caller-allocated on the scene's device,
 * zeroed by this call), ordered on opts->stream, no host synchronisation
 * except when counters or transport_ms are requested.  psf_count,
 * total_histories and counters must then be device pointers too. */
mcpet_status mcpet_run_device(mcpet_scene* scene, const mcpet_run_opts* opts,
                              mcpet_tallies* device_out);

/* Batched run: the lanes of n_scenes scenes (phantoms of any size, each with
 * its own activity, seed, acquisition time and isotope mean life) in
 * persistent launches of the transport kernel that keep the GPU full through
 * the tail of every scene.  Replaces n_scenes sequential runs of the
 * reference program (MCGPU-PET.cu:77-840, one phantom per process).  Each
 * scene keeps its own lane plan and RANECU streams: its tallies equal those
 * of mcpet_run on that scene alone with the same options (with automatic
 * histories per lane, <= 0, every scene gets its own automatic lanes).  A
 * scene of at least 2e7 decays whose lanes fill the GPU twice over runs as
 * a launch of its own -- the single-scene kernel of a run of it alone, when
 * the batch collects no counters and the scene tallies no dose; the other
 * scenes share one launch of the batch kernel.  The launches follow one another on the stream, each allowed to
 * start placing blocks (programmatic dependent launch) while the previous
 * one drains its last lanes.  The scenes must use the same material files
 * in the same slots (the shared launch reads one Compton and Rayleigh table
 * for all) and sit on one device (scenes not yet on a device are placed on
 * scene 0's).  opts applies to every scene (algorithm 0 or 2 only).
 * outs[k] receives scene k's tallies as in mcpet_run; counters, when
 * requested, are totals of all the launches and go to outs[0], and
 * mcpet_last_run_guard(scenes[0]) reports the launches' guard trips.
 * Blocking. */
mcpet_status mcpet_run_batch(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                             mcpet_tallies* outs);

/* PSF records streamed in bounded chunks instead of one buffer of
 * psf_size * 44 bytes (the reference allocates the whole PSF up front,
 * MCGPU-PET.cu:2094, and writes it at the end, report_PSF
 * MCGPU-PET.cu:3193-3322).  The transport runs as consecutive launches over
 * ranges of lanes -- each lane keeps its RANECU stream, so the set of
 * records and the tallies equal one mcpet_run with an unbounded PSF --
 * and after each launch the sink receives that launch's packed 44-byte
 * records (at most chunk_records of them; order within and across chunks
 * is not specified, as in the reference).  A range whose records overflow
 * the chunk is replayed in halves with its sinogram-side writes suppressed.
 * Returning nonzero from the sink stops the run.  out receives the
 * sinograms/images/spectrum/totals as in mcpet_run (out->psf is ignored;
 * *out->psf_count = records streamed).  Blocking. */
typedef int (*mcpet_psf_sink)(const void* records, long long n_records, void* user);
mcpet_status mcpet_run_psf_stream(mcpet_scene* scene, const mcpet_run_opts* opts, long long chunk_records,
                                  mcpet_psf_sink sink, void* user, mcpet_tallies* out);

/* Gradient of the Poisson log-likelihood of a measured sinogram,
 *   L = sum_b y_b ln(lambda_b) - lambda_b,  lambda = trues + scatter + background,
 * with respect to each voxel's activity and density scale.  No counterpart
 * in the reference (it has no adjoint); the forward model is its transport
 * (mcpet_run_device on device_out, same options and results).  Activity:
 * event back-tallying of w_b = y_b/lambda_b - 1 over the tallied
 * coincidences, divided by the voxel activity.  Density scale s_v (rho_v ->
 * s_v rho_v, majorant held fixed): path-replay score function -- every
 * tallied history is recomputed from the RANECU state recorded at its
 * emission and each Woodcock step inside a voxel adds w_b times
 * d ln p(step)/d ln rho to it.  A replay that does not reproduce the recorded
 * bin is left out of dL/ds and counted in mismatches.  The forward of this
 * call does not produce the dose tallies.  Blocking. */
typedef struct {
  const float* measured;          /* device [n_bins]: y, the measured sinogram (counts) */
  const float* background;        /* device [n_bins]: r, expected background added to the model; NULL = 0 */
  float* grad_activity;           /* device [n_voxels] out: dL/dA_v (per Bq); NULL to skip */
  float* grad_density_scale;      /* device [n_voxels] out: dL/ds_v; NULL to skip */
  void* event_buffer;             /* device scratch, 24 bytes per tallied coincidence; NULL: the scene
                                     keeps one (grown and the forward repeated when too small) */
  long long event_capacity;       /* records event_buffer holds */
  double loglik;                  /* out: L */
  unsigned long long events;      /* out: tallied coincidences of the forward run */
  unsigned long long replayed;    /* out: replays that reproduced their bin */
  unsigned long long mismatches;  /* out: replays that did not (left out) */
  double forward_ms;              /* out: device time of the forward transport (with event records) */
  double gradient_ms;             /* out: device time of the log-likelihood and the replay */
} mcpet_grad_args;

mcpet_status mcpet_grad(mcpet_scene* scene, const mcpet_run_opts* opts, mcpet_tallies* device_out,
                        mcpet_grad_args* args);

/* Batched run into DEVICE tallies (device_outs[k] as in mcpet_run_device),
 * ordered on opts->stream; the merged lane plan is uploaded and released in
 * stream order. */
mcpet_status mcpet_run_batch_device(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                                    mcpet_tallies* device_outs);

/* Lane plan of a run with these settings, as built on the host (no device
 * work): per emitting voxel, in launch order (decreasing work per lane,
 * ties in voxel order), its voxel, lanes, first lane, first RANECU stream
 * and lanes/activity.  The reference launches one block of
 * threads_per_block lanes per voxel (MCGPU-PET.cu:456-458); lane_mode 0
 * reproduces those lanes.  histories_per_lane <= 0: the automatic value.
 * Any output pointer may be NULL.  With capacity below the emitter count
 * only *n_emitters (and *total_lanes) are set and MCPET_ERR_LIMIT is
 * returned. */
mcpet_status mcpet_scene_lane_plan(const mcpet_scene* scene, int lane_mode, int histories_per_lane,
                                   long long capacity, uint32_t* voxel, uint32_t* n_lanes,
                                   unsigned long long* first_lane, unsigned long long* stream_base,
                                   double* inv_rate, long long* n_emitters, unsigned long long* total_lanes);

/* ---- asynchronous host-buffer runs --------------------------------------
 *
 * mcpet_run without the wait: the plan upload, zeroing and transport are
 * enqueued on opts->stream and the downloads into out's host buffers on a
 * stream of the scene's own, and the call returns before any of it has run.
 * The scene alternates between two sets of device tallies, so one run's
 * downloads overlap the next run's transport (two runs of a scene in flight
 * at most: the call for a third waits until the first's downloads are done).
 * out's scalar pointers (total_histories, coincidences, psf_count,
 * counters) are written when the downloads finish; out and its buffers must
 * stay valid until then (use pinned host buffers for copies that overlap).
 * No PSF or dose tallies, no transport_ms.  Runs of a scene are ordered on
 * one stream; until mcpet_run_wait, the scene's other run functions refuse
 * it (MCPET_ERR_ARG), as they share its run words.  mcpet_run_wait blocks
 * until every download of the scene has finished and reports guard trips
 * of those runs as MCPET_ERR_DEVICE.
 * Replaces the reference's blocking launch, synchronisation and downloads
 * (MCGPU-PET.cu:483-535) for callers that run many acquisitions. */
mcpet_status mcpet_run_async(mcpet_scene* scene, const mcpet_run_opts* opts, mcpet_tallies* out);
mcpet_status mcpet_run_wait(mcpet_scene* scene);

/* ---- autotuner ----------------------------------------------------------
 *
 * Picks histories_per_lane (balanced lanes) and block_threads for a workload
 * of one or more scenes by timing candidates on a sample of it: every scene
 * runs with its acquisition time scaled by f and each candidate's histories
 * per lane scaled by f, so the sample has the workload's lanes with f of its
 * decays (f = sample_decays / total decays, raised so that every candidate
 * keeps at least one decay per lane; sample_decays <= 0 means 2e8).
 * Candidates: 1/4, 1/2, 1, 2 and 4 times the automatic histories per lane of
 * the workload (for several scenes: sized from all their decays together)
 * and, for several scenes, the automatic choice itself (every scene its own
 * automatic lanes), at the full block, then smaller blocks at the best of
 * those.  Runs go through mcpet_run_device (one scene) or
 * mcpet_run_batch_device (several) with opts and overwrite device_outs.  The
 * scenes' own settings are restored.  The result goes into
 * opts->histories_per_lane / block_threads of later runs (a batch's
 * histories_per_lane is 0 when the automatic choice won); with reference
 * lanes only the block size is tuned. */
typedef struct {
  int block_threads;              /* chosen threads per block */
  int histories_per_lane;         /* chosen expected decays per lane (0 with reference lanes) */
  double best_ms;                 /* kernel time of the chosen pair on the sample */
  double auto_ms;                 /* kernel time of the automatic choice on the sample */
  double sample_fraction;         /* f */
  int candidates;                 /* pairs timed */
} mcpet_tune_result;

mcpet_status mcpet_autotune(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                            const mcpet_tallies* device_outs, double sample_decays, mcpet_tune_result* out);

/* ---- batched regeneration captured in a CUDA graph --------------------
 *
 * Repeated runs of the same scenes (iterative reconstruction, Monte Carlo
 * averaging over seeds) need new histories every time, not new parameters.
 * mcpet_batch_graph_create builds the batch once, as mcpet_run_batch_device
 * does (the lane plans, the union tables, the launches of the event kernel
 * over every scene's lanes), keeps its own copies of the lane plans and the
 * union tables on the device, and captures into one CUDA graph: the zeroing
 * of device_outs[k], the transport launches, and a step of every scene's
 * seed.
 * Each mcpet_batch_graph_launch then regenerates all histories with one graph
 * launch and no host work: launch r (counted from 0, or from the last
 * mcpet_batch_graph_set_seeds) runs scene k with seed s_k + r*seed_step
 * (kept in [1, 2147483562]) and leaves in device_outs[k] the tallies of
 * mcpet_run_device of scene k alone with that seed and the same options.
 * s_k is opts->seed_override when set, else the scene's own seed.  The
 * scenes must stay alive and on their device while the graph exists; runs of
 * the scenes themselves do not disturb it.  Replaces repeated runs of the
 * reference program, one phantom per process (MCGPU-PET.cu:77-840). */
typedef struct mcpet_batch_graph mcpet_batch_graph;

mcpet_status mcpet_batch_graph_create(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                                      const mcpet_tallies* device_outs, int seed_step, mcpet_batch_graph** out);
/* One replay, ordered on `stream` (a cudaStream_t; NULL = default stream). */
mcpet_status mcpet_batch_graph_launch(mcpet_batch_graph* graph, void* stream);
/* Seeds of the next launch, one per scene (ordered on `stream`, blocking). */
mcpet_status mcpet_batch_graph_set_seeds(mcpet_batch_graph* graph, const int* seeds, void* stream);
/* Guard trips of the last completed launch (blocking read). */
mcpet_status mcpet_batch_graph_guard_trips(mcpet_batch_graph* graph, unsigned long long* trips);
void mcpet_batch_graph_destroy(mcpet_batch_graph* graph);

/* Allocation-free variant of mcpet_run_device, for callers that may not
 * allocate device memory while they run: plugin or custom-call hooks inside a
 * host framework that hands out every device buffer from its own pool, and
 * stream pipelines that cannot afford the device-wide synchronisation that
 * cudaMalloc/cudaFree imply.  No counterpart in the reference (its program
 * allocates everything in init_CUDA_device).
 *
 * The caller passes the per-voxel activity (float, n_voxels, device memory)
 * and the device output buffers of mcpet_tallies.  The scene's tables must
 * already be on the device (mcpet_scene_to_device, done once at set-up, is
 * the call that allocates).  The lane plan and the work-queue words are
 * built in a fixed static device array of the library instead of allocated
 * buffers: it holds plans of up to MCPET_NOALLOC_MAX_VOXELS voxels (about
 * 32 MiB) and every GPU that loads the library reserves it until the process
 * exits.  Larger phantoms are rejected with MCPET_ERR_LIMIT.  All calls on a
 * device share that array and rewrite it, so calls that overlap on the GPU
 * (several streams or threads at once) race; serialise them.  The first call
 * on a device looks up the array's device address; make that first call
 * before any stream capture.  The address is kept for the life of the
 * device's context: do not use this entry point across a cudaDeviceReset.
 * Lanes are laid out in voxel order: with MCPET_LANES_REFERENCE the results
 * equal mcpet_run_device's; with balanced lanes and histories_per_lane <= 0
 * the automatic lane size is computed on the device from activity_device.
 * A plan whose RANECU stream ids would reach 2^31 (the reference's 31-bit
 * thread ids) runs nothing and counts one guard trip.  Guard trips (that
 * one, and the transport's loop caps) are reported in
 * device_out->counters->guard_trips when collect_counters=1, and by
 * mcpet_last_run_guard(scene) after the call (a blocking read of the static
 * array, which allocates nothing). */
#define MCPET_NOALLOC_MAX_VOXELS (1 << 20)
mcpet_status mcpet_run_device_noalloc(mcpet_scene* scene, const float* activity_device,
                                      const mcpet_run_opts* opts, mcpet_tallies* device_out);

/* Device-side guard status of the last run on this scene (blocking read);
 * after mcpet_run_device_noalloc, that call's trips. */
mcpet_status mcpet_last_run_guard(mcpet_scene* scene, unsigned long long* trips);

/* ---- outputs ----------------------------------------------------------- */

/* Write the reference's output files into out_dir (NULL = current
 * directory): sinogram_{Trues,Scatter}.raw.gz and image_{Trues,Scatter}.raw.gz
 * (or sinogram_BG_*.raw.gz / BG_image_*.raw.gz in background mode) when the
 * sinogram is tallied, Energy_Sinogram_Spectrum.dat always, and the PSF text
 * and .raw files when the PSF is tallied.  Replaces MCGPU-PET.cu:503-616 and
 * report_PSF (:3193-3322). */
mcpet_status mcpet_write_outputs(const mcpet_scene* scene, const mcpet_tallies* host,
                                 const char* out_dir, int background_mode, double elapsed_s);

/* ---- verification hooks (the reference's device functions, one call per
 * entry; used by the parity tests against the reference build) ---------- */

/* RANECU lane streams: seed of lane stream id s is the reference init_PRNG
 * jump (s+1)*555555*256 draws ahead (MCGPU-PET_kernel.cu:925-978), computed on
 * the GPU; then ndraw float draws and ndraw double draws (ranecu,
 * ranecu_double :1045-1083) from the same start.  seeds_out[2n]. */
mcpet_status mcpet_probe_rng(int n, int seed_input, const int64_t* stream_ids, int ndraw,
                             int32_t* seeds_out, float* draws, double* ddraws);

/* Detector model on a fixed event list (tally_Sinogram,
 * MCGPU-PET_kernel.cu:1624-1836) on the GPU with the scene's detector and
 * sinogram geometry.  Per event: out[6*i+0]=bin or -1, +1 class (1 true, 2
 * scatter, 0 none), +2/+3 spectrum bins of the two photons or -1, +4/+5
 * seed after the call.  Positions/directions float3, states signed char. */
mcpet_status mcpet_probe_detector(const mcpet_scene* scene, int n, const float* e2,
                                  const float* e1, const float* pos2, const float* pos1,
                                  const float* dir2, const float* dir1, const int8_t* st2,
                                  const int8_t* st1, const int32_t* seeds, int32_t* out);

/* Compton (GCOa :1335-1563) and Rayleigh (GRAa :1231-1296) sampling on the GPU
 * with the scene's tables.  Material 0-based. */
mcpet_status mcpet_probe_compton(const mcpet_scene* scene, int n, const float* energy_in,
                                 const int32_t* mat, const int32_t* seeds_in, float* energy_out,
                                 double* costh_out, int32_t* seeds_out);
mcpet_status mcpet_probe_rayleigh(const mcpet_scene* scene, int n, const float* energy_in,
                                  const int32_t* mat, const float* pmax, const int32_t* seeds_in,
                                  double* costh_out, int32_t* seeds_out);

/* Photon-pair source (source :666-773) for every voxel of an nx*ny*nz grid:
 * out[12*v..] = position1, direction1, position2, direction2.
 * background_mode: 0 or 1 (isotropic second photon), plus 2 for the
 * balanced lanes' photon-2 emission (same distribution, other arithmetic). */
mcpet_status mcpet_probe_source(int nx, int ny, int nz, const float inv_voxel_size[3],
                                int background_mode, const int32_t* seeds_in, float* out,
                                int32_t* seeds_out);

/* ---- misc --------------------------------------------------------------- */

const char* mcpet_last_error(void);
const char* mcpet_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MCPET_H_ */
