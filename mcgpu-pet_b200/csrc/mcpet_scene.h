/* Host-side scene of the transport path: parsed configuration, phantom,
 * interpolation tables in the reference layout, and the device copy. */
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include "mcpet.h"
#include "mcpet_params.h"

struct mcpet_scene {
  mcpet_config cfg;

  /* phantom (load_voxels, MCGPU-PET.cu:1381-1533) */
  int nx = 0, ny = 0, nz = 0;
  float voxel_size[3] = {0, 0, 0};
  float inv_voxel_size[3] = {0, 0, 0};
  float bbox[3] = {0, 0, 0};
  std::vector<int32_t> mat0;      /* 0-based material per voxel */
  std::vector<float> rho;         /* density per voxel, scaled by the density factor */
  std::vector<float> activity;    /* Bq per voxel */
  double emitting_activity = -1;  /* sum of the emitting voxels' activity (Bq); < 0: not yet summed */
  float density_max[mcpet::kMaxMaterials];
  float density_nominal[mcpet::kMaxMaterials];

  /* tables (load_material, MCGPU-PET.cu:1565-1831) in the reference layout */
  int n_e = 0;
  float e0 = 0.f, ide = 0.f;
  double delta_e = 0.0;
  std::vector<float> woodcock;    /* float2[n_e] */
  std::vector<float> mfp_a, mfp_b;/* float3[n_e*15] */
  std::vector<float> pmax;        /* [n_e*15] */
  mcpet::ComptonTable compton;
  std::vector<float> xco, pco, aco, bco;   /* [15*128] */
  std::vector<uint8_t> itl, itu;
  bool material_loaded[mcpet::kMaxMaterials];

  /* palette compression of (material, density) */
  std::vector<mcpet::PaletteEntry> palette;
  std::vector<uint32_t> voxel_key;

  /* device copy */
  struct Device {
    int device = -1;
    bool tables_ready = false;
    bool activity_dirty = true;
    int sm_count = 0;
    void* vox = nullptr;          /* uint16 or uint32 keys */
    bool vox16 = true;
    mcpet::PaletteEntry* palette = nullptr;
    float* woodcock = nullptr;
    mcpet::MfpRecord* mfp = nullptr;
    mcpet::ComptonTable* compton = nullptr;
    float* ray = nullptr;         /* xco|pco|aco|bco contiguous */
    uint8_t* ray8 = nullptr;      /* itl|itu contiguous */
    mcpet::Emitter* emitters = nullptr;
    size_t emitters_cap = 0;
    int n_emitters = 0;
    uint64_t n_lanes = 0;
    double max_lane_decays = 0;   /* expected decays of the plan's longest lane */
    std::string plan_key;
    /* run scratch owned by the scene (host-buffer runs) */
    int* trues = nullptr;
    int* scatter = nullptr;
    int* img_t = nullptr;
    int* img_s = nullptr;
    int* spectrum = nullptr;
    uint32_t* psf = nullptr;
    long long psf_cap = 0;
    unsigned long long* small = nullptr;  /* histories, guard, cursor, psf_count, 10 counters */
    long long nbins_alloc = -1, nvox_alloc = -1;
    int ne_alloc = -1;
    void* ev0 = nullptr;
    void* ev1 = nullptr;
    /* dose tallies: material sums [15][2], ROI voxel sums [n][2] */
    unsigned long long* mdose = nullptr;
    unsigned long long* vdose = nullptr;
    long long vdose_alloc = -1;
    /* gradient (mcpet_grad): event records, device activity, small words */
    uint32_t* events = nullptr;
    long long event_cap = 0;
    float* activity = nullptr;
    unsigned long long* gwords = nullptr;  /* 0 replayed, 1 mismatches, 2 log-likelihood (double) */
    unsigned long long last_guard = 0;
    bool last_run_noalloc = false;   /* mcpet_last_run_guard reads the allocation-free scratch */
    /* asynchronous host-buffer runs (mcpet_run_async): a second set of
     * tallies, snapshots of the run words, a download stream and events */
    int* trues_b = nullptr;
    int* scatter_b = nullptr;
    int* img_t_b = nullptr;
    int* img_s_b = nullptr;
    int* spectrum_b = nullptr;
    long long nbins_b = -1, nvox_b = -1;
    int ne_b = -1;
    unsigned long long* async_words = nullptr;  /* device [2][16] */
    unsigned long long* async_host = nullptr;   /* pinned host [2][16] */
    void* copy_stream = nullptr;
    void* ran[2] = {nullptr, nullptr};          /* transport of set k done */
    void* copied[2] = {nullptr, nullptr};       /* download of set k done */
    bool copied_pending[2] = {false, false};
    int async_next = 0;
    struct AsyncOut {
      const unsigned long long* words;          /* pinned snapshot of this set's run words */
      int32_t* psf_count;
      unsigned long long* total_histories;
      unsigned long long* coincidences;
      mcpet_counters* counters;
      bool counters_on;
      unsigned long long* guard_sum;            /* guard trips of finished asynchronous runs */
    } async_out[2];
    unsigned long long async_guard = 0;
    long long run_h2d = 0;        /* host->device bytes of the run in progress */
    long long last_h2d = 0;       /* ... and of the last completed run */
  } dev;
  /* the autotuner runs scenes on a sample of their decays: the fraction, so
   * that a batch still groups them by their full decays */
  double tune_scale = 1.0;

  ~mcpet_scene();
};

namespace mcpet {

/* thread-local error text */
mcpet_status set_error(mcpet_status s, const char* fmt, ...);

/* mcpet_io.cpp */
mcpet_status parse_input(const char* in_path, mcpet_config* cfg);
mcpet_status load_phantom_file(const char* path, float density_factor, mcpet_scene* sc);
mcpet_status set_phantom_arrays(int nx, int ny, int nz, const float vs[3], const int32_t* material,
                                const float* density, const float* activity, float density_factor,
                                mcpet_scene* sc);
mcpet_status load_materials(mcpet_scene* sc);
mcpet_status finalize_scene(mcpet_scene* sc);
mcpet_status write_outputs(const mcpet_scene* sc, const mcpet_tallies* t, const char* out_dir, int bg,
                           double elapsed_s);
void derive_sinogram_sizes(mcpet_config* cfg);
long long dose_voxels(const mcpet_config& c);
std::string format_materials_dose(const mcpet_scene* sc, const unsigned long long* md, unsigned long long n_hist);

}  // namespace mcpet
