/* C ABI of the transport path: scene life cycle, device upload, lane plan,
 * runs and verification probes. */
#include <cuda_runtime_api.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "mcpet.h"
#include "mcpet_kernels.h"
#include "mcpet_scene.h"

namespace mcpet {
extern thread_local std::string g_error;
}

using namespace mcpet;

namespace {

#define CUDA_TRY(call)                                                                          \
  do {                                                                                          \
    cudaError_t err_ = (call);                                                                  \
    if (err_ != cudaSuccess)                                                                    \
      return set_error(err_ == cudaErrorMemoryAllocation ? MCPET_ERR_NOMEM : MCPET_ERR_CUDA,    \
                       "%s failed: %s", #call, cudaGetErrorString(err_));                      \
  } while (0)

template <typename T>
cudaError_t dmalloc(T** p, size_t bytes) {
  return cudaMalloc((void**)p, bytes);
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

constexpr int kMaxStepsDefault = 1 << 20;       /* Woodcock steps per photon */
constexpr int kMaxRejectionsDefault = 1 << 16;  /* iterations per sampler rejection loop */

/* (a^e) mod m with exact 64-bit arithmetic. */
uint32_t powmod(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1 % m;
  a %= m;
  while (e) {
    if (e & 1) r = (r * a) % m;
    a = (a * a) % m;
    e >>= 1;
  }
  return (uint32_t)r;
}

/* Powers (a^C)^(2^k) mod m for the stream jump, C = 555555*256 draws per
 * stream (the reference init_PRNG leap, MCGPU-PET_kernel.cu:251-253,925-978). */
void jump_tables(int32_t* t1, int32_t* t2) {
  const uint64_t C = (uint64_t)kLeapHistories * kLeapDistance;
  uint64_t p1 = powmod(40014, C, 2147483563ull), p2 = powmod(40692, C, 2147483399ull);
  for (int k = 0; k < 32; ++k) {
    t1[k] = (int32_t)p1;
    t2[k] = (int32_t)p2;
    p1 = (p1 * p1) % 2147483563ull;
    p2 = (p2 * p2) % 2147483399ull;
  }
}

int pick_device(int requested) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return -1;
  if (requested < 0 || requested >= count) return 0;
  return requested;
}

/* Tuning knob from the environment, clamped to [lo, hi]. */
int env_int(const char* name, int def, int lo, int hi) {
  const char* v = getenv(name);
  if (!v || !*v) return def;
  int x = atoi(v);
  return x < lo ? lo : (x > hi ? hi : x);
}

void fill_params(const mcpet_scene* sc, TransportParams& P) {
  memset(&P, 0, sizeof(P));
  const mcpet_config& c = sc->cfg;
  P.nx = sc->nx;
  P.ny = sc->ny;
  P.nz = sc->nz;
  P.inv_vx = sc->inv_voxel_size[0];
  P.inv_vy = sc->inv_voxel_size[1];
  P.inv_vz = sc->inv_voxel_size[2];
  P.bbx = sc->bbox[0];
  P.bby = sc->bbox[1];
  P.bbz = sc->bbox[2];
  P.n_voxels = (long long)sc->mat0.size();
  P.n_e = sc->n_e;
  P.e0 = sc->e0;
  P.ide = sc->ide;
  P.cx = c.detector_center[0];
  P.cy = c.detector_center[1];
  P.cz = c.detector_center[2];
  P.radius = c.detector_radius;
  P.height = c.detector_height;
  P.psf_capacity = c.psf_size;
  P.tally_psf_sinogram = c.tally_psf_sinogram;
  P.tally_type = c.tally_type;
  P.acq_ps = c.acquisition_time_ps;
  P.inv_mean_life = 1.0 / (double)c.mean_life;
  P.e_resol = c.energy_resolution;
  P.e_low = c.energy_window_low;
  P.e_high = c.energy_window_high;
  P.fovz = c.fov_z;
  P.nrows = c.n_rows;
  P.ncrystals = c.n_crystals;
  P.nangles = c.n_angles;
  P.nrad = c.n_radial;
  P.nzs = c.n_z_slices;
  P.ne = c.n_energy_bins;
  P.mrd = c.max_ring_difference;
  P.span = c.span;
  P.nsinos = c.n_sinograms;
  P.nbins = c.n_bins;
  jump_tables(P.jump1, P.jump2);
  P.seed = c.seed;
  int ms = 1;
  for (int m = 0; m < kMaxMaterials; ++m)
    if (sc->material_loaded[m] && sc->compton.noscco[m] > ms) ms = sc->compton.noscco[m];
  P.max_shells = ms;
  P.spectrum_in_shared =
      (c.n_energy_bins > 0 && c.n_energy_bins <= kSpectrumSharedMax && env_int("MCPET_SPECTRUM_SHARED", 1, 0, 1)) ? 1
                                                                                                                : 0;
  P.palette_in_shared =
      (sc->palette.size() <= 2048 && env_int("MCPET_PALETTE_SHARED", 1, 0, 1)) ? (int)sc->palette.size() : 0;
  P.e_annihilation = 510998.95f;
  for (int k = 0; k < 6; ++k) P.dose_roi[k] = c.tally_voxel_dose ? c.dose_roi[k] : (k % 2 ? -1 : 0);
  P.quorum_scatter = env_int("MCPET_QUORUM_SCATTER", 16, 1, 32);
  P.quorum_pair = env_int("MCPET_QUORUM_PAIR", 16, 1, 32);
  P.step_keep = env_int("MCPET_STEP_KEEP", 2, 1, 8);
  P.quorum_rayleigh = env_int("MCPET_QUORUM_RAYLEIGH", 2, 1, 32);
  P.max_steps = kMaxStepsDefault;
  P.max_rejections = kMaxRejectionsDefault;
  P.prompt_energy = c.prompt_gamma_energy > 0.0f ? c.prompt_gamma_energy : 0.0f;
  P.prompt_yield = c.prompt_gamma_energy > 0.0f ? c.prompt_gamma_yield : 0.0f;
}

/* A prompt-gamma scene needs the sinogram tally only and tables that reach
 * above the gamma energy (its energy bin and the next one are read). */
mcpet_status check_prompt(const mcpet_scene* sc) {
  const mcpet_config& c = sc->cfg;
  if (!(c.prompt_gamma_energy > 0.0f)) return MCPET_OK;
  if (c.tally_psf_sinogram != 2)
    return set_error(MCPET_ERR_ARG, "the prompt-gamma emitter supports the sinogram tally only (REPORT PSF/SINOGRAM 2)");
  if (!(c.prompt_gamma_yield > 0.0f && c.prompt_gamma_yield <= 1.0f))
    return set_error(MCPET_ERR_ARG, "prompt gamma yield %g outside (0, 1]", c.prompt_gamma_yield);
  const double top = (double)sc->e0 + (double)(sc->n_e - 2) / (double)sc->ide;
  if (!((double)c.prompt_gamma_energy < top))
    return set_error(MCPET_ERR_ARG,
                     "prompt gamma of %.0f eV above the material tables (last energy bin starts at %.0f eV): "
                     "use tables that reach above it", (double)c.prompt_gamma_energy, top);
  return MCPET_OK;
}

/* loop caps of a run: the options' values, or the defaults */
void apply_caps(const mcpet_run_opts& o, TransportParams& P) {
  P.max_steps = o.max_woodcock_steps > 0 ? o.max_woodcock_steps : kMaxStepsDefault;
  P.max_rejections = o.max_rejections > 0 ? o.max_rejections : kMaxRejectionsDefault;
}

/* GCOa's incoherent scattering function at theta = pi for energy E (eV) and
 * material mat, in double precision: the normaliser of its rejection step
 * (MCGPU-PET_kernel.cu:1366-1391; PENELOPE's analytical one-electron
 * Compton profiles).  Non-decreasing in E: each shell's projected momentum
 * at theta = pi grows with E, and so does its profile integral. */
double compton_s0_host(double E, int mat, const ComptonTable& C) {
  const double mc2 = 510998.918, inv_mc2 = 1.956951306108245e-6, r2 = 1.4142135623731, ir2 = 0.70710678118654502;
  double s0 = 0.0;
  for (int i = 0; i < C.noscco[mat]; ++i) {
    const double u = C.uico[mat + i * kMaxMaterials];
    if (u >= E) continue;
    const double aux = E * (E - u) * 2.0;
    const double pz = C.fj0[mat + i * kMaxMaterials] * (aux - u * mc2) / std::sqrt(aux + aux + u * u) * inv_mc2;
    const double a = pz > 0.0 ? ir2 + pz * r2 : ir2 - pz * r2;
    double t = 0.5 * std::exp(0.5 - a * a);
    if (pz > 0.0) t = 1.0 - t;
    s0 += C.fco[mat + i * kMaxMaterials] * t;
  }
  return s0;
}

mcpet_status upload_tables(mcpet_scene* sc) {
  auto& d = sc->dev;
  if (d.tables_ready) return MCPET_OK;
  const size_t nv = sc->mat0.size();
  d.vox16 = sc->palette.size() <= 65536;
  if (d.vox16) {
    std::vector<uint16_t> k(nv);
    for (size_t i = 0; i < nv; ++i) k[i] = (uint16_t)sc->voxel_key[i];
    CUDA_TRY(dmalloc(&d.vox, nv * 2));
    CUDA_TRY(cudaMemcpy(d.vox, k.data(), nv * 2, cudaMemcpyHostToDevice));
  } else {
    CUDA_TRY(dmalloc(&d.vox, nv * 4));
    CUDA_TRY(cudaMemcpy(d.vox, sc->voxel_key.data(), nv * 4, cudaMemcpyHostToDevice));
  }
  CUDA_TRY(dmalloc(&d.palette, sc->palette.size() * sizeof(PaletteEntry)));
  CUDA_TRY(cudaMemcpy(d.palette, sc->palette.data(), sc->palette.size() * sizeof(PaletteEntry),
                      cudaMemcpyHostToDevice));
  CUDA_TRY(dmalloc(&d.woodcock, sc->woodcock.size() * 4));
  CUDA_TRY(cudaMemcpy(d.woodcock, sc->woodcock.data(), sc->woodcock.size() * 4, cudaMemcpyHostToDevice));
  const size_t nrec = (size_t)sc->n_e * kMaxMaterials;
  std::vector<MfpRecord> rec(nrec);
  for (size_t i = 0; i < nrec; ++i) {
    MfpRecord& r = rec[i];
    r.ax = sc->mfp_a[3 * i + 0];
    r.bx = sc->mfp_b[3 * i + 0];
    r.ay = sc->mfp_a[3 * i + 1];
    r.by = sc->mfp_b[3 * i + 1];
    r.az = sc->mfp_a[3 * i + 2];
    r.bz = sc->mfp_b[3 * i + 2];
    r.pmax_next = (i + kMaxMaterials < nrec) ? sc->pmax[i + kMaxMaterials] : 0.0f;
    r.s0_bound = 0.f;
    const int mat = (int)(i % kMaxMaterials);
    if (sc->compton.noscco[mat] > 0) {
      /* bin k holds the energies with floor((E - e0) * ide) = k: bound them by
       * S at the upper edge of bin k + 1 (a margin for the float index) */
      const double e_hi = (double)sc->e0 + (double)(i / kMaxMaterials + 2) / (double)sc->ide;
      const float b = (float)(compton_s0_host(e_hi, mat, sc->compton) * (1.0 + 1e-5));
      r.s0_bound = std::nextafter(b, 1e30f);
    }
  }
  CUDA_TRY(dmalloc(&d.mfp, nrec * sizeof(MfpRecord)));
  CUDA_TRY(cudaMemcpy(d.mfp, rec.data(), nrec * sizeof(MfpRecord), cudaMemcpyHostToDevice));
  CUDA_TRY(dmalloc(&d.compton, sizeof(ComptonTable)));
  CUDA_TRY(cudaMemcpy(d.compton, &sc->compton, sizeof(ComptonTable), cudaMemcpyHostToDevice));
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  std::vector<float> ray(4 * nr);
  std::copy(sc->xco.begin(), sc->xco.end(), ray.begin());
  std::copy(sc->pco.begin(), sc->pco.end(), ray.begin() + nr);
  std::copy(sc->aco.begin(), sc->aco.end(), ray.begin() + 2 * nr);
  std::copy(sc->bco.begin(), sc->bco.end(), ray.begin() + 3 * nr);
  CUDA_TRY(dmalloc(&d.ray, 4 * nr * 4));
  CUDA_TRY(cudaMemcpy(d.ray, ray.data(), 4 * nr * 4, cudaMemcpyHostToDevice));
  std::vector<uint8_t> r8(2 * nr);
  std::copy(sc->itl.begin(), sc->itl.end(), r8.begin());
  std::copy(sc->itu.begin(), sc->itu.end(), r8.begin() + nr);
  CUDA_TRY(dmalloc(&d.ray8, 2 * nr));
  CUDA_TRY(cudaMemcpy(d.ray8, r8.data(), 2 * nr, cudaMemcpyHostToDevice));
  CUDA_TRY(dmalloc(&d.small, 16 * sizeof(unsigned long long)));
  d.run_h2d += (long long)(nv * (d.vox16 ? 2 : 4) + sc->palette.size() * sizeof(PaletteEntry) +
                           sc->woodcock.size() * 4 + nrec * sizeof(MfpRecord) + sizeof(ComptonTable) + 4 * nr * 4 +
                           2 * nr);
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  d.ev0 = e0;
  d.ev1 = e1;
  d.tables_ready = true;
  return MCPET_OK;
}

DeviceTables device_tables(const mcpet_scene* sc) {
  const auto& d = sc->dev;
  DeviceTables T;
  memset(&T, 0, sizeof(T));
  T.vox16 = d.vox16 ? (const uint16_t*)d.vox : nullptr;
  T.vox32 = d.vox16 ? nullptr : (const uint32_t*)d.vox;
  T.palette = d.palette;
  T.n_palette = (int)sc->palette.size();
  T.woodcock = d.woodcock;
  T.mfp = d.mfp;
  T.compton = d.compton;
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  T.rayleigh.xco = d.ray;
  T.rayleigh.pco = d.ray + nr;
  T.rayleigh.aco = d.ray + 2 * nr;
  T.rayleigh.bco = d.ray + 3 * nr;
  T.rayleigh.itl = d.ray8;
  T.rayleigh.itu = d.ray8 + nr;
  T.emitters = d.emitters;
  return T;
}

/* Lane plan: emitters (voxels with activity > 1e-7 Bq, the reference's
 * threshold at MCGPU-PET_kernel.cu:232) with their lane counts and RANECU
 * streams, ordered by decreasing expected decays per lane. */
/* Lane plan on the host: one emitter per voxel with activity, ordered by
 * decreasing work per lane (ascending 1/rate per lane; ties in voxel order).
 * The voxels are split over host threads, each building and stably sorting
 * 16-byte keys of its range; neighbouring ranges are merged stably, which
 * gives exactly the order of one stable sort over all voxels. */
mcpet_status plan_host(const mcpet_scene* sc, int mode, int tpb, int hpl, std::vector<Emitter>& em,
                       uint64_t& n_lanes) {
  struct Key {
    double inv_rate;
    uint32_t voxel;
    uint32_t n_lanes;
  };
  const auto by_rate = [](const Key& x, const Key& y) { return x.inv_rate < y.inv_rate; };
  const size_t nv = sc->activity.size();
  const double T = (double)sc->cfg.acquisition_time_ps * 1e-12;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int parts = (int)std::max<size_t>(1, std::min<size_t>({(size_t)hw, 16, nv / 65536}));
  std::vector<std::vector<Key>> part((size_t)parts);
  auto build = [&](int t) {
    const size_t v0 = nv * (size_t)t / (size_t)parts, v1 = nv * (size_t)(t + 1) / (size_t)parts;
    std::vector<Key>& out = part[(size_t)t];
    for (size_t v = v0; v < v1; ++v) {
      const float a = sc->activity[v];
      if (!(a > 1.0e-7f)) continue;
      Key e;
      e.voxel = (uint32_t)v;
      if (mode == MCPET_LANES_REFERENCE) {
        e.n_lanes = (uint32_t)tpb;
        e.inv_rate = (tpb / (double)a);
      } else {
        const double expect = (double)a * T;
        double L = ceil(expect / (double)hpl);
        if (L < 1) L = 1;
        if (L > 1.0e8) L = 1.0e8;
        e.n_lanes = (uint32_t)L;
        e.inv_rate = (double)e.n_lanes / (double)a;
      }
      out.push_back(e);
    }
    std::stable_sort(out.begin(), out.end(), by_rate);
  };
  /* fn(ids[0]) here, the others on host threads (here too when a thread
   * cannot be started) */
  auto run = [](const std::vector<int>& ids, const std::function<void(int)>& fn) {
    std::vector<std::thread> th;
    size_t started = 1;
    try {
      for (; started < ids.size(); ++started) th.emplace_back(fn, ids[started]);
    } catch (...) {
    }
    fn(ids[0]);
    for (size_t i = started; i < ids.size(); ++i) fn(ids[i]);
    for (auto& x : th) x.join();
  };
  {
    std::vector<int> ids((size_t)parts);
    std::iota(ids.begin(), ids.end(), 0);
    run(ids, build);
  }
  for (int w = 1; w < parts; w *= 2) {
    auto merge = [&](int t) {
      std::vector<Key> m(part[(size_t)t].size() + part[(size_t)(t + w)].size());
      std::merge(part[(size_t)t].begin(), part[(size_t)t].end(), part[(size_t)(t + w)].begin(),
                 part[(size_t)(t + w)].end(), m.begin(), by_rate);
      part[(size_t)t].swap(m);
      std::vector<Key>().swap(part[(size_t)(t + w)]);
    };
    std::vector<int> ids;
    for (int t = 0; t + w < parts; t += 2 * w) ids.push_back(t);
    run(ids, merge);
  }
  const std::vector<Key>& keys = part[0];
  em.assign(keys.size(), Emitter{});
  uint64_t lanes = 0, max_stream = 0;
  for (size_t i = 0; i < keys.size(); ++i) {
    Emitter& e = em[i];
    e.inv_rate = keys[i].inv_rate;
    e.voxel = keys[i].voxel;
    e.n_lanes = keys[i].n_lanes;
    e.first_lane = lanes;
    e.stream_base = (mode == MCPET_LANES_REFERENCE) ? (uint64_t)e.voxel * (uint64_t)tpb : lanes;
    lanes += e.n_lanes;
    max_stream = std::max<uint64_t>(max_stream, e.stream_base + e.n_lanes);
  }
  if (max_stream >= (1ull << 31))
    return set_error(MCPET_ERR_LIMIT, "lane plan needs %llu RANECU streams (limit 2^31)",
                     (unsigned long long)max_stream);
  n_lanes = lanes;
  return MCPET_OK;
}

/* Lane plan of the scene for these options, rebuilt when the activity or the
 * options changed.  The upload is ordered on st after the work already
 * there (a run still reading the old plan on st finishes first). */
mcpet_status build_lanes(mcpet_scene* sc, int mode, int tpb, int hpl, cudaStream_t st) {
  auto& d = sc->dev;
  char key[128];
  snprintf(key, sizeof(key), "%d/%d/%d", mode, tpb, hpl);
  if (!d.activity_dirty && d.plan_key == key && d.emitters) return MCPET_OK;
  /* a new plan is built on the host from the activity map and uploaded */
  std::vector<Emitter> em;
  uint64_t lanes = 0;
  mcpet_status s = plan_host(sc, mode, tpb, hpl, em, lanes);
  if (s != MCPET_OK) return s;
  if (em.size() > d.emitters_cap) {
    dfree(d.emitters);
    size_t cap = std::max<size_t>(em.size(), 1);
    CUDA_TRY(dmalloc(&d.emitters, cap * sizeof(Emitter)));
    d.emitters_cap = cap;
  }
  /* from pageable memory the copy is staged before the call returns */
  if (!em.empty())
    CUDA_TRY(cudaMemcpyAsync(d.emitters, em.data(), em.size() * sizeof(Emitter), cudaMemcpyHostToDevice, st));
  d.run_h2d += (long long)(em.size() * sizeof(Emitter));
  d.n_emitters = (int)em.size();
  d.n_lanes = lanes;
  d.max_lane_decays = em.empty() ? 0.0 : (double)sc->cfg.acquisition_time_ps * 1e-12 / em[0].inv_rate;
  d.plan_key = key;
  d.activity_dirty = false;
  return MCPET_OK;
}

/* Other runs share the scene's run words and first tally set with the
 * asynchronous runs: they wait for mcpet_run_wait. */
mcpet_status check_no_async(const mcpet_scene* sc) {
  if (sc && (sc->dev.copied_pending[0] || sc->dev.copied_pending[1]))
    return set_error(MCPET_ERR_ARG, "asynchronous runs of this scene are in flight: call mcpet_run_wait first");
  return MCPET_OK;
}

mcpet_status ensure_device(mcpet_scene* sc) {
  if (sc->dev.device < 0) return mcpet_scene_to_device(sc, -1);
  CUDA_TRY(cudaSetDevice(sc->dev.device));
  return MCPET_OK;
}

/* Automatic decays per balanced lane: about kAutoLanesPerThread (6) lanes
 * per resident thread.  Fewer, longer lanes amortise the per-lane start
 * (stream jump, emitter search), more lanes shorten the tail; on the
 * 1e9-decay head workload: 399.2 ms at 1.5 lanes per thread, 384.2 ms at
 * 3, 380.7 ms at 6, 382.5 ms at 12. */
/* Sum of the emitting voxels' activity, cached until the activity changes. */
double emitting_activity(const mcpet_scene* sc) {
  if (sc->emitting_activity < 0) {
    double A = 0;
    for (float a : sc->activity)
      if (a > 1.0e-7f) A += (double)a;
    const_cast<mcpet_scene*>(sc)->emitting_activity = A;
  }
  return sc->emitting_activity;
}

int auto_hpl_of(const std::vector<const mcpet_scene*>& scenes) {
  double D = 0;
  for (const mcpet_scene* sc : scenes) D += emitting_activity(sc) * ((double)sc->cfg.acquisition_time_ps * 1e-12);
  double threads = (double)std::max(scenes[0]->dev.sm_count, 1) * 2048.0;
  double h = D / (threads * kAutoLanesPerThread);
  if (h < 1) h = 1;
  if (h > 4096) h = 4096;
  return (int)h;
}
int auto_hpl(const mcpet_scene* sc) { return auto_hpl_of(std::vector<const mcpet_scene*>(1, sc)); }

mcpet_status validate_opts(const mcpet_scene* sc, const mcpet_run_opts* opts) {
  {
    const mcpet_status ps = check_prompt(sc);
    if (ps != MCPET_OK) return ps;
  }
  int seed = (opts && opts->seed_override != 0) ? opts->seed_override : sc->cfg.seed;
  if (seed <= 0) return set_error(MCPET_ERR_ARG, "RANECU seed must be positive (got %d)", seed);
  if (opts && (opts->lane_mode < 0 || opts->lane_mode > 1))
    return set_error(MCPET_ERR_ARG, "unknown lane mode %d", opts->lane_mode);
  if (opts && (opts->algorithm < 0 || opts->algorithm > 2))
    return set_error(MCPET_ERR_ARG, "unknown algorithm %d", opts->algorithm);
  return MCPET_OK;
}

/* Parameters of one scene's run (host only): everything but the lane plan,
 * the zeroing of the outputs and the launch.  O.coincidences defaults to a
 * scene word. */
mcpet_status prepare_params(mcpet_scene* sc, const mcpet_run_opts& o, DeviceTallies& O, TransportParams& P) {
  {
    const mcpet_status ps = check_prompt(sc);
    if (ps != MCPET_OK) return ps;
  }
  fill_params(sc, P);
  if (o.seed_override != 0) P.seed = o.seed_override;
  if (P.seed <= 0) return set_error(MCPET_ERR_ARG, "RANECU seed must be positive (got %d)", P.seed);
  P.background_mode = o.background_mode ? 1 : 0;
  apply_caps(o, P);
  if (!O.psf) P.psf_capacity = 0;

  const bool sino = sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 2;
  if (sino && (!O.trues || !O.scatter || !O.image_trues || !O.image_scatter || !O.spectrum))
    return set_error(MCPET_ERR_ARG, "sinogram tally requested but a sinogram/image/spectrum buffer is missing");
  if (!O.histories || !O.psf_count) return set_error(MCPET_ERR_ARG, "histories and psf_count are required");
  if (!O.coincidences) O.coincidences = sc->dev.small + 14;
  if (!sc->cfg.tally_material_dose) O.mat_dose = nullptr;
  if (dose_voxels(sc->cfg) == 0) O.vox_dose = nullptr;
  /* the kernel only touches the spectrum when the sinogram is tallied */
  if (!sino) P.spectrum_in_shared = 0;
  return MCPET_OK;
}

/* Zero the outputs of a prepared run, ordered on st. */
mcpet_status zero_outputs(const mcpet_scene* sc, const DeviceTallies& O, cudaStream_t st) {
  const size_t nb = (size_t)sc->cfg.n_bins * 4, nv = sc->mat0.size() * 4;
  if (O.trues) CUDA_TRY(cudaMemsetAsync(O.trues, 0, nb, st));
  if (O.scatter) CUDA_TRY(cudaMemsetAsync(O.scatter, 0, nb, st));
  if (O.image_trues) CUDA_TRY(cudaMemsetAsync(O.image_trues, 0, nv, st));
  if (O.image_scatter) CUDA_TRY(cudaMemsetAsync(O.image_scatter, 0, nv, st));
  if (O.spectrum) CUDA_TRY(cudaMemsetAsync(O.spectrum, 0, (size_t)sc->cfg.n_energy_bins * 4, st));
  CUDA_TRY(cudaMemsetAsync(O.psf_count, 0, 4, st));
  CUDA_TRY(cudaMemsetAsync(O.histories, 0, 8, st));
  CUDA_TRY(cudaMemsetAsync(O.coincidences, 0, 8, st));
  if (O.mat_dose) CUDA_TRY(cudaMemsetAsync(O.mat_dose, 0, 2 * kMaxMaterials * 8, st));
  if (O.vox_dose) CUDA_TRY(cudaMemsetAsync(O.vox_dose, 0, (size_t)dose_voxels(sc->cfg) * 16, st));
  return MCPET_OK;
}

/* Parameters of one scene's run and its zeroed outputs. */
mcpet_status prepare_run(mcpet_scene* sc, const mcpet_run_opts& o, DeviceTallies& O, cudaStream_t st,
                         TransportParams& P) {
  mcpet_status s = prepare_params(sc, o, O, P);
  if (s != MCPET_OK) return s;
  return zero_outputs(sc, O, st);
}

int pick_block(const mcpet_run_opts& o) {
  int block = o.block_threads > 0 ? o.block_threads : transport_block_threads();
  if (block > transport_block_threads()) block = transport_block_threads();
  block = (block / 32) * 32;
  return block < 32 ? 32 : block;
}

mcpet_status launch_planned(mcpet_scene* sc, const mcpet_run_opts& o, TransportParams& P, DeviceTallies& O,
                            cudaStream_t st, double* ms_out);

/* Enqueue one transport run writing into the device tallies O. */
mcpet_status enqueue_run(mcpet_scene* sc, const mcpet_run_opts* opts, DeviceTallies O, cudaStream_t st,
                         double* ms_out) {
  sc->dev.run_h2d = 0;
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  s = ensure_device(sc);
  if (s != MCPET_OK) return s;
  s = upload_tables(sc);
  if (s != MCPET_OK) return s;
  mcpet_run_opts def;
  memset(&def, 0, sizeof(def));
  const mcpet_run_opts& o = opts ? *opts : def;
  int tpb = sc->cfg.threads_per_block > 0 ? sc->cfg.threads_per_block : 32;
  int hpl = o.histories_per_lane > 0 ? o.histories_per_lane : auto_hpl(sc);
  s = build_lanes(sc, o.lane_mode, tpb, hpl, st);
  if (s != MCPET_OK) return s;

  TransportParams P;
  s = prepare_run(sc, o, O, st, P);
  if (s != MCPET_OK) return s;
  P.n_lanes = sc->dev.n_lanes;
  P.n_emitters = sc->dev.n_emitters;

  auto& d = sc->dev;
  d.last_run_noalloc = false;
  unsigned long long* small = d.small;
  O.guard = small + 0;
  O.lane_cursor = small + 1;
  CUDA_TRY(cudaMemsetAsync(small, 0, 2 * sizeof(unsigned long long), st));
  if (O.counters) CUDA_TRY(cudaMemsetAsync(O.counters, 0, 10 * 8, st));

  return launch_planned(sc, o, P, O, st, ms_out);
}

/* Kernel variant of a run: balanced lanes use the single-precision
 * rotation and decay clock (they are held to statistical parity; reference
 * lanes keep the reference's arithmetic for replay), prompt-gamma scenes the
 * emitter, lowered caps the run-time loop guards. */
int run_mode(const mcpet_scene* sc, const mcpet_run_opts& o) {
  int m = 0;
  if (o.lane_mode == MCPET_LANES_BALANCED) m |= kTransportFast;
  if (sc->cfg.prompt_gamma_energy > 0.0f) m |= kTransportPrompt;
  if (o.max_woodcock_steps > 0 || o.max_rejections > 0) m |= kTransportCaps;
  if (sc->cfg.tally_psf_sinogram == 2) m |= kTransportSinogramOnly;
  return m;
}

/* Launch the transport for a prepared run (P, O complete, the work-queue
 * word set), optionally timed. */
mcpet_status launch_planned(mcpet_scene* sc, const mcpet_run_opts& o, TransportParams& P, DeviceTallies& O,
                            cudaStream_t st, double* ms_out) {
  auto& d = sc->dev;
  const bool counters = o.collect_counters && O.counters;
  const int block = pick_block(o);
  const int mode = run_mode(sc, o);
  int algorithm = o.algorithm == kAlgorithmHistories ? kAlgorithmHistories : kAlgorithmEvents;
  if (algorithm == kAlgorithmEvents && env_int("MCPET_MINBLOCKS", 4, 1, 4) == 1 && (mode & ~kTransportFast) == 0)
    algorithm = kAlgorithmEventsUncapped;
  if (O.events && algorithm != kAlgorithmHistories) algorithm = kAlgorithmEventsRecord;
  else if ((O.mat_dose || O.vox_dose) && algorithm != kAlgorithmHistories) algorithm = kAlgorithmEventsDose;
  /* lowered loop caps: the plain event kernel and the history loop read them
   * (the history loop also when the run tallies dose or a prompt gamma) */
  if (mode & kTransportCaps) {
    if (algorithm == kAlgorithmEventsRecord)
      return set_error(MCPET_ERR_ARG, "lowered loop caps are not available for the gradient's recording run");
    if (algorithm != kAlgorithmEvents || (mode & kTransportPrompt)) algorithm = kAlgorithmHistories;
  }
  size_t smem = transport_dynamic_smem(P, block, algorithm);
  int bps = 0;
  CUDA_TRY(transport_occupancy(counters, algorithm, mode, block, smem, &bps));
  if (bps < 1) return set_error(MCPET_ERR_LIMIT, "transport kernel does not fit on an SM (smem %zu)", smem);
  if (o.blocks_per_sm > 0 && o.blocks_per_sm < bps) bps = o.blocks_per_sm;
  int grid = d.sm_count * bps;
  d.last_h2d = d.run_h2d + (long long)sizeof(TransportParams);
  if (P.n_lanes == 0) grid = 1;
  if (ms_out) CUDA_TRY(cudaEventRecord((cudaEvent_t)d.ev0, st));
  CUDA_TRY(launch_transport(P, device_tables(sc), O, counters, algorithm, mode, grid, block, smem, st));
  if (ms_out) {
    CUDA_TRY(cudaEventRecord((cudaEvent_t)d.ev1, st));
    CUDA_TRY(cudaEventSynchronize((cudaEvent_t)d.ev1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, (cudaEvent_t)d.ev0, (cudaEvent_t)d.ev1));
    *ms_out = ms;
  }
  return MCPET_OK;
}

mcpet_status ensure_run_buffers(mcpet_scene* sc, bool want_psf) {
  auto& d = sc->dev;
  long long nb = sc->cfg.n_bins, nv = (long long)sc->mat0.size();
  int ne = sc->cfg.n_energy_bins;
  if (d.nbins_alloc != nb) {
    dfree(d.trues);
    dfree(d.scatter);
    CUDA_TRY(dmalloc(&d.trues, (size_t)nb * 4));
    CUDA_TRY(dmalloc(&d.scatter, (size_t)nb * 4));
    d.nbins_alloc = nb;
  }
  if (d.nvox_alloc != nv) {
    dfree(d.img_t);
    dfree(d.img_s);
    CUDA_TRY(dmalloc(&d.img_t, (size_t)nv * 4));
    CUDA_TRY(dmalloc(&d.img_s, (size_t)nv * 4));
    d.nvox_alloc = nv;
  }
  if (d.ne_alloc != ne) {
    dfree(d.spectrum);
    CUDA_TRY(dmalloc(&d.spectrum, (size_t)std::max(ne, 1) * 4));
    d.ne_alloc = ne;
  }
  if (sc->cfg.tally_material_dose && !d.mdose) CUDA_TRY(dmalloc(&d.mdose, 2 * kMaxMaterials * 8));
  const long long nd = dose_voxels(sc->cfg);
  if (nd != d.vdose_alloc) {
    dfree(d.vdose);
    if (nd > 0) CUDA_TRY(dmalloc(&d.vdose, (size_t)nd * 16));
    d.vdose_alloc = nd;
  }
  long long cap = want_psf ? (long long)std::max(sc->cfg.psf_size, 0) : 0;
  if (cap != d.psf_cap) {
    dfree(d.psf);
    if (cap > 0) CUDA_TRY(dmalloc(&d.psf, (size_t)cap * 44));
    d.psf_cap = cap;
  }
  return MCPET_OK;
}

}  // namespace

mcpet_scene::~mcpet_scene() {
  if (dev.device >= 0) {
    cudaSetDevice(dev.device);
    if (dev.copy_stream) {
      cudaStreamSynchronize((cudaStream_t)dev.copy_stream);   /* outstanding asynchronous downloads */
      cudaStreamDestroy((cudaStream_t)dev.copy_stream);
    }
    for (int k = 0; k < 2; ++k) {
      if (dev.ran[k]) cudaEventDestroy((cudaEvent_t)dev.ran[k]);
      if (dev.copied[k]) cudaEventDestroy((cudaEvent_t)dev.copied[k]);
    }
    if (dev.async_host) cudaFreeHost(dev.async_host);
    dfree(dev.async_words);
    dfree(dev.trues_b);
    dfree(dev.scatter_b);
    dfree(dev.img_t_b);
    dfree(dev.img_s_b);
    dfree(dev.spectrum_b);
    dfree(dev.vox);
    dfree(dev.palette);
    dfree(dev.woodcock);
    dfree(dev.mfp);
    dfree(dev.compton);
    dfree(dev.ray);
    dfree(dev.ray8);
    dfree(dev.emitters);
    dfree(dev.trues);
    dfree(dev.scatter);
    dfree(dev.img_t);
    dfree(dev.img_s);
    dfree(dev.spectrum);
    dfree(dev.psf);
    dfree(dev.small);
    dfree(dev.events);
    dfree(dev.mdose);
    dfree(dev.vdose);
    dfree(dev.activity);
    dfree(dev.gwords);
    if (dev.ev0) cudaEventDestroy((cudaEvent_t)dev.ev0);
    if (dev.ev1) cudaEventDestroy((cudaEvent_t)dev.ev1);
  }
}

/* Copy a finished host-buffer run (scene-owned device buffers) into out. */
mcpet_status download_run(mcpet_scene* sc, const mcpet_run_opts* opts, mcpet_tallies* out, bool want_psf, double ms,
                          cudaStream_t st) {
  auto& d = sc->dev;
  CUDA_TRY(cudaStreamSynchronize(st));
  const size_t nb = (size_t)sc->cfg.n_bins * 4, nv = sc->mat0.size() * 4;
  if (out->trues) CUDA_TRY(cudaMemcpyAsync(out->trues, d.trues, nb, cudaMemcpyDeviceToHost, st));
  if (out->scatter) CUDA_TRY(cudaMemcpyAsync(out->scatter, d.scatter, nb, cudaMemcpyDeviceToHost, st));
  if (out->image_trues) CUDA_TRY(cudaMemcpyAsync(out->image_trues, d.img_t, nv, cudaMemcpyDeviceToHost, st));
  if (out->image_scatter) CUDA_TRY(cudaMemcpyAsync(out->image_scatter, d.img_s, nv, cudaMemcpyDeviceToHost, st));
  if (out->spectrum)
    CUDA_TRY(cudaMemcpyAsync(out->spectrum, d.spectrum, (size_t)sc->cfg.n_energy_bins * 4, cudaMemcpyDeviceToHost,
                             st));
  if (out->material_dose && d.mdose && sc->cfg.tally_material_dose)
    CUDA_TRY(cudaMemcpyAsync(out->material_dose, d.mdose, 2 * kMaxMaterials * 8, cudaMemcpyDeviceToHost, st));
  if (out->voxel_dose && d.vdose && dose_voxels(sc->cfg) > 0)
    CUDA_TRY(cudaMemcpyAsync(out->voxel_dose, d.vdose, (size_t)dose_voxels(sc->cfg) * 16, cudaMemcpyDeviceToHost,
                             st));
  unsigned long long small[16];
  CUDA_TRY(cudaMemcpyAsync(small, d.small, sizeof(small), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  int psf_count = (int)(small[3] & 0xffffffffull);
  if (out->psf_count) *out->psf_count = psf_count;
  if (out->total_histories) *out->total_histories = small[2];
  if (out->coincidences) *out->coincidences = small[14];
  if (want_psf) {
    long long n = std::min<long long>(std::max(psf_count, 0), std::min<long long>(d.psf_cap, out->psf_capacity));
    if (n > 0) CUDA_TRY(cudaMemcpy(out->psf, d.psf, (size_t)n * 44, cudaMemcpyDeviceToHost));
  }
  if (out->counters) {
    memset(out->counters, 0, sizeof(mcpet_counters));
    if (opts && opts->collect_counters) memcpy(out->counters, small + 4, 10 * 8);
    out->counters->guard_trips = small[0];
  }
  if (out->transport_ms) *out->transport_ms = ms;
  d.last_guard = small[0];
  if (small[0] != 0)
    return set_error(MCPET_ERR_DEVICE, "%llu device guard(s) fired (loop cap or out-of-range index)", small[0]);
  return MCPET_OK;
}


/* Compton and Rayleigh data of a batched launch: the union of the material
 * slots loaded by its scenes (a scene loads only the slots its phantom uses,
 * as the reference does). */
struct SharedTables {
  ComptonTable cmp;
  std::vector<float> ray;     /* xco|pco|aco|bco, [15*128] each */
  std::vector<uint8_t> ray8;  /* itl|itu */
};

/* Builds the union; a slot loaded by two scenes must hold the same data. */
mcpet_status merge_shared_tables(mcpet_scene* const* scenes, int n, SharedTables& U) {
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  memset(&U.cmp, 0, sizeof(U.cmp));
  U.ray.assign(4 * nr, 0.f);
  U.ray8.assign(2 * nr, 0);
  bool have[kMaxMaterials] = {false};
  const mcpet_scene* a = scenes[0];
  for (int k = 0; k < n; ++k) {
    const mcpet_scene* b = scenes[k];
    if (b->n_e != a->n_e || b->e0 != a->e0 || b->ide != a->ide)
      return set_error(MCPET_ERR_ARG, "scene %d has another energy grid than scene 0 (first material file)", k);
    for (int m = 0; m < kMaxMaterials; ++m) {
      if (!b->material_loaded[m]) continue;
      const int nsh = b->compton.noscco[m];
      const float* rows[4] = {b->xco.data(), b->pco.data(), b->aco.data(), b->bco.data()};
      const uint8_t* rows8[2] = {b->itl.data(), b->itu.data()};
      if (have[m]) {
        bool same = U.cmp.noscco[m] == nsh;
        for (int i = 0; same && i < nsh; ++i) {
          const int x = m + i * kMaxMaterials;
          same = U.cmp.fco[x] == b->compton.fco[x] && U.cmp.uico[x] == b->compton.uico[x] &&
                 U.cmp.fj0[x] == b->compton.fj0[x];
        }
        for (int r = 0; same && r < 4; ++r)
          same = std::equal(rows[r] + m * kNpRayleigh, rows[r] + (m + 1) * kNpRayleigh,
                            U.ray.begin() + r * nr + m * kNpRayleigh);
        for (int r = 0; same && r < 2; ++r)
          same = std::equal(rows8[r] + m * kNpRayleigh, rows8[r] + (m + 1) * kNpRayleigh,
                            U.ray8.begin() + r * nr + m * kNpRayleigh);
        if (!same)
          return set_error(MCPET_ERR_ARG,
                           "scene %d has other Compton/Rayleigh data in material slot %d than an earlier scene "
                           "(the scenes of a batch must use the same material file in a slot)", k, m + 1);
        continue;
      }
      have[m] = true;
      U.cmp.noscco[m] = nsh;
      for (int i = 0; i < nsh; ++i) {
        const int x = m + i * kMaxMaterials;
        U.cmp.fco[x] = b->compton.fco[x];
        U.cmp.uico[x] = b->compton.uico[x];
        U.cmp.fj0[x] = b->compton.fj0[x];
      }
      for (int r = 0; r < 4; ++r)
        std::copy(rows[r] + m * kNpRayleigh, rows[r] + (m + 1) * kNpRayleigh, U.ray.begin() + r * nr + m * kNpRayleigh);
      for (int r = 0; r < 2; ++r)
        std::copy(rows8[r] + m * kNpRayleigh, rows8[r] + (m + 1) * kNpRayleigh,
                  U.ray8.begin() + r * nr + m * kNpRayleigh);
    }
  }
  return MCPET_OK;
}

/* Host-side checks of a batch (before any device work). */
mcpet_status check_batch(mcpet_scene* const* scenes, int n, const mcpet_run_opts* opts, SharedTables* U) {
  if (!scenes || n < 1) return set_error(MCPET_ERR_ARG, "a batch needs at least one scene");
  if (n >= (1 << 23)) return set_error(MCPET_ERR_LIMIT, "batch of %d scenes (limit 2^23)", n);
  if (opts && opts->algorithm == kAlgorithmHistories)
    return set_error(MCPET_ERR_ARG, "batched runs use the event loop (algorithm 0 or 2)");
  for (int k = 0; k < n; ++k) {
    if (!scenes[k]) return set_error(MCPET_ERR_ARG, "scene %d of the batch is null", k);
    mcpet_status s = validate_opts(scenes[k], opts);
    if (s != MCPET_OK) return s;
    s = check_no_async(scenes[k]);
    if (s != MCPET_OK) return s;
  }
  SharedTables local;
  return merge_shared_tables(scenes, n, U ? *U : local);
}

/* One launch of a batched run: a range of slots, its launch-wide
 * parameters and tables, and its shape.  A scene with enough decays and
 * lanes to fill the GPU by itself is a launch of its own ("solo"): the
 * single-scene kernel of a run of it alone, with its parameters, tables and
 * tallies; the other scenes share one launch of the batch kernel. */
struct BatchGroup {
  int first = 0, count = 0;         /* slots [first, first + count) */
  TransportParams P;                /* launch-wide parameters (the group's lanes) */
  DeviceTables T;
  DeviceTallies O;                  /* solo: the scene's tallies */
  int share = 0;                    /* kBatchShareScanner | kBatchSharePhantom */
  bool solo = false;
  int mode = 0, algorithm = 0;      /* solo: kernel variant of the scene's own run */
  int grid = 1;
  size_t smem = 0;
};

/* Everything one batched run needs, built on the host: the scenes' slots
 * (parameters, tables, tallies, first lane within their launch), the union
 * Compton/Rayleigh tables, and the launches. */
struct BatchLaunch {
  std::vector<SceneSlot> slots;     /* launch order: solo scenes, then the shared launch's (longest lanes first) */
  std::vector<int> scene_of;        /* scene index of each slot */
  std::vector<int> slot_of;         /* slot of each scene */
  std::vector<BatchGroup> groups;
  unsigned long long* counter_words = nullptr;  /* scene 0's counters (totals of the run) */
  SharedTables U;
  uint64_t total = 0;
  bool counters = false, dose = false;
  int mode = 0;                     /* kernel variant (fast arithmetic, prompt gamma, sinogram only) */
  int block = 0;
  /* device blob: slots | Compton table | Rayleigh float rows | Rayleigh byte rows | lane cursors */
  size_t off_cmp = 0, off_ray = 0, off_ray8 = 0, off_cursor = 0, bytes = 0;
};

/* A scene of at least this many decays runs as a launch of its own when its
 * lanes fill the GPU twice over (runs without counters or dose tallies: the
 * chained variant is the plain event kernel). */
constexpr double kSoloDecays = 2.0e7;

/* Decays of a scene's full acquisition (also while the autotuner runs it on
 * a sample). */
double scene_decays(const mcpet_scene* sc) {
  return emitting_activity(sc) * ((double)sc->cfg.acquisition_time_ps * 1e-12) / sc->tune_scale;
}

/* True when scene b has scene a's scanner: detector, sinogram, energy
 * window and tally settings, and the acquisition time of the PSF records
 * (every parameter detect_pair reads). */
bool same_scanner(const TransportParams& a, const TransportParams& b) {
  return a.cx == b.cx && a.cy == b.cy && a.cz == b.cz && a.radius == b.radius && a.height == b.height &&
         a.psf_capacity == b.psf_capacity && a.tally_psf_sinogram == b.tally_psf_sinogram &&
         a.tally_type == b.tally_type && a.background_mode == b.background_mode && a.e_resol == b.e_resol &&
         a.e_low == b.e_low && a.e_high == b.e_high && a.fovz == b.fovz && a.nrows == b.nrows &&
         a.ncrystals == b.ncrystals && a.nangles == b.nangles && a.nrad == b.nrad && a.nzs == b.nzs &&
         a.ne == b.ne && a.mrd == b.mrd && a.span == b.span && a.nsinos == b.nsinos && a.nbins == b.nbins &&
         a.sino_dry == b.sino_dry && a.e_annihilation == b.e_annihilation && a.acq_ps == b.acq_ps;
}

/* True when scene b has scene a's phantom: grid, voxel keys, palette and
 * the Woodcock and interaction tables. */
bool same_phantom(const mcpet_scene* a, const mcpet_scene* b) {
  if (a == b) return true;
  return a->nx == b->nx && a->ny == b->ny && a->nz == b->nz &&
         memcmp(a->voxel_size, b->voxel_size, sizeof(a->voxel_size)) == 0 &&
         memcmp(a->bbox, b->bbox, sizeof(a->bbox)) == 0 && a->dev.vox16 == b->dev.vox16 &&
         a->voxel_key == b->voxel_key && a->palette.size() == b->palette.size() &&
         (a->palette.empty() ||
          memcmp(a->palette.data(), b->palette.data(), a->palette.size() * sizeof(a->palette[0])) == 0) &&
         a->woodcock == b->woodcock && a->mfp_a == b->mfp_a && a->mfp_b == b->mfp_b && a->pmax == b->pmax;
}

/* Lane plans, tables and parameters of a batch (no stream work but the
 * uploads of tables and plans).  outs[k] are scene k's device tallies. */
mcpet_status setup_batch(mcpet_scene* const* scenes, int n, const mcpet_run_opts& o, const DeviceTallies* outs,
                         BatchLaunch& L, cudaStream_t st) {
  mcpet_status cs = check_batch(scenes, n, &o, &L.U);
  if (cs != MCPET_OK) return cs;
  mcpet_scene* s0 = scenes[0];
  L.slots.assign((size_t)n, SceneSlot{});
  int max_shells = 1;
  L.total = 0;
  std::vector<char> solo((size_t)n, 0);
  std::vector<TransportParams> alone((size_t)n);   /* each scene's parameters as in a run of it alone */
  for (int k = 0; k < n; ++k) {
    mcpet_scene* sc = scenes[k];
    sc->dev.run_h2d = 0;
    mcpet_status s = MCPET_OK;
    if (k > 0 && sc->dev.device < 0) s = mcpet_scene_to_device(sc, s0->dev.device);
    else s = ensure_device(sc);
    if (s != MCPET_OK) return s;
    if (sc->dev.device != s0->dev.device)
      return set_error(MCPET_ERR_ARG, "scene %d is on device %d, scene 0 on device %d", k, sc->dev.device,
                       s0->dev.device);
    s = upload_tables(sc);
    if (s != MCPET_OK) return s;
    /* each scene's lanes as in a run of it alone with the same options
     * (automatic: from its own decays), so its tallies equal that run's */
    const int hpl = o.histories_per_lane > 0 ? o.histories_per_lane : auto_hpl(sc);
    const int tpb = sc->cfg.threads_per_block > 0 ? sc->cfg.threads_per_block : 32;
    s = build_lanes(sc, o.lane_mode, tpb, hpl, st);
    if (s != MCPET_OK) return s;
    const double resident = (double)std::max(sc->dev.sm_count, 1) * 2048.0;
    const bool plain = !(o.collect_counters && outs[0].counters) && !outs[k].mat_dose && !outs[k].vox_dose;
    solo[(size_t)k] = plain && scene_decays(sc) >= kSoloDecays && (double)sc->dev.n_lanes >= 2.0 * resident;
    SceneSlot& z = L.slots[(size_t)k];
    memset(&z, 0, sizeof(z));
    z.O = outs[k];
    s = prepare_params(sc, o, z.O, z.P);
    if (s != MCPET_OK) return s;
    alone[(size_t)k] = z.P;
    alone[(size_t)k].n_lanes = sc->dev.n_lanes;
    alone[(size_t)k].n_emitters = sc->dev.n_emitters;
    z.P.spectrum_in_shared = 0;
    z.P.palette_in_shared = 0;
    z.P.n_lanes = sc->dev.n_lanes;
    z.P.n_emitters = sc->dev.n_emitters;
    z.T = device_tables(sc);
    max_shells = std::max(max_shells, z.P.max_shells);
  }
  if (o.max_woodcock_steps > 0 || o.max_rejections > 0)
    return set_error(MCPET_ERR_ARG, "lowered loop caps are available for single-scene runs only");
  CUDA_TRY(cudaSetDevice(s0->dev.device));
  /* launch order: the solo scenes, then the shared launch with longer lanes
   * first, so that no scene's longest lanes start near the end of the
   * launch (each scene's plan is itself ordered longest first); results do
   * not depend on the order */
  L.scene_of.resize((size_t)n);
  for (int k = 0; k < n; ++k) L.scene_of[(size_t)k] = k;
  std::stable_sort(L.scene_of.begin(), L.scene_of.end(), [&](int a, int b) {
    if (solo[(size_t)a] != solo[(size_t)b]) return solo[(size_t)a] > solo[(size_t)b];
    return scenes[a]->dev.max_lane_decays > scenes[b]->dev.max_lane_decays;
  });
  {
    std::vector<SceneSlot> by_scene;
    by_scene.swap(L.slots);
    L.slots.resize((size_t)n);
    L.slot_of.resize((size_t)n);
    for (int j = 0; j < n; ++j) {
      const int k = L.scene_of[(size_t)j];
      L.slots[(size_t)j] = by_scene[(size_t)k];
      L.slot_of[(size_t)k] = j;
    }
  }
  /* the launches: one per solo scene, one for the rest; lanes numbered
   * within a launch */
  L.groups.clear();
  for (int j = 0; j < n;) {
    BatchGroup g;
    g.first = j;
    g.solo = solo[(size_t)L.scene_of[(size_t)j]] != 0;
    g.count = g.solo ? 1 : n - j;
    uint64_t lanes = 0;
    for (int i = j; i < j + g.count; ++i) {
      L.slots[(size_t)i].first_lane = lanes;
      lanes += L.slots[(size_t)i].P.n_lanes;
    }
    L.total += lanes;
    if (g.solo) {
      const int k = L.scene_of[(size_t)j];
      g.P = alone[(size_t)k];
      g.T = L.slots[(size_t)j].T;
      g.O = L.slots[(size_t)j].O;
      g.mode = run_mode(scenes[k], o) | kTransportChained;
      g.algorithm = kAlgorithmEvents;
      L.groups.push_back(g);
      j += g.count;
      continue;
    }
    g.P = L.slots[(size_t)j].P;
    g.P.n_lanes = lanes;
    g.P.n_emitters = 0;
    g.P.max_shells = max_shells;
    /* the launch's shared layout holds the prompt-gamma fields when any of
     * its scenes emits one (each lane reads its own scene's emitter) */
    for (int i = j; i < j + g.count; ++i)
      g.P.prompt_energy = std::max(g.P.prompt_energy, L.slots[(size_t)i].P.prompt_energy);
    g.T = L.slots[(size_t)j].T;
    g.T.emitters = nullptr;
    L.groups.push_back(g);
    j += g.count;
  }

  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  L.off_cmp = ((L.slots.size() * sizeof(SceneSlot) + 255) / 256) * 256;
  L.off_ray = L.off_cmp + ((sizeof(ComptonTable) + 255) / 256) * 256;
  L.off_ray8 = L.off_ray + 4 * nr * sizeof(float);
  L.off_cursor = ((L.off_ray8 + 2 * nr + 255) / 256) * 256;
  L.bytes = L.off_cursor + L.groups.size() * sizeof(unsigned long long);

  L.counters = o.collect_counters && outs[0].counters;
  L.counter_words = L.counters ? outs[0].counters : nullptr;
  L.block = pick_block(o);
  L.dose = false;
  for (const SceneSlot& z : L.slots) L.dose = L.dose || z.O.mat_dose || z.O.vox_dose;
  bool sino_only = true, prompt = false;
  for (const SceneSlot& z : L.slots) {
    sino_only = sino_only && z.P.tally_psf_sinogram == 2;
    prompt = prompt || z.P.prompt_energy > 0.0f;
  }
  L.mode = (o.lane_mode == MCPET_LANES_BALANCED ? kTransportFast : 0) | (prompt ? kTransportPrompt : 0) |
           (sino_only ? kTransportSinogramOnly : 0);
  for (BatchGroup& g : L.groups) {
    if (g.solo) {
      g.smem = transport_dynamic_smem(g.P, L.block, g.algorithm);
      int bps = 0;
      CUDA_TRY(transport_occupancy(L.counters, g.algorithm, g.mode, L.block, g.smem, &bps));
      if (bps < 1) return set_error(MCPET_ERR_LIMIT, "transport kernel does not fit on an SM (smem %zu)", g.smem);
      if (o.blocks_per_sm > 0 && o.blocks_per_sm < bps) bps = o.blocks_per_sm;
      g.grid = g.P.n_lanes == 0 ? 1 : s0->dev.sm_count * bps;
      continue;
    }
    g.share = 0;
    if (!L.counters && !L.dose) {
      bool scanner = true, phantom = true;
      for (int i = g.first + 1; i < g.first + g.count; ++i) {
        scanner = scanner && same_scanner(L.slots[(size_t)g.first].P, L.slots[(size_t)i].P);
        phantom = phantom && same_phantom(scenes[L.scene_of[(size_t)g.first]], scenes[L.scene_of[(size_t)i]]);
      }
      g.share = (scanner ? kBatchShareScanner : 0) | (phantom ? kBatchSharePhantom : 0);
    }
    g.smem = transport_batch_dynamic_smem(g.P, L.block);
    /* a shared phantom's palette is staged in shared memory, as in a single run */
    if (g.share & kBatchSharePhantom) {
      TransportParams one;
      fill_params(scenes[L.scene_of[(size_t)g.first]], one);
      if (one.palette_in_shared) {
        g.P.palette_in_shared = one.palette_in_shared;
        g.smem = transport_batch_dynamic_smem(g.P, L.block);
      }
    }
    int bps = 0;
    CUDA_TRY(transport_batch_occupancy(L.counters, L.dose, g.share, L.mode, L.block, g.smem, &bps));
    if (bps < 1) return set_error(MCPET_ERR_LIMIT, "transport kernel does not fit on an SM (smem %zu)", g.smem);
    if (o.blocks_per_sm > 0 && o.blocks_per_sm < bps) bps = o.blocks_per_sm;
    g.grid = g.P.n_lanes == 0 ? 1 : s0->dev.sm_count * bps;
  }
  return MCPET_OK;
}

/* Host image of the batch's device blob. */
std::vector<unsigned char> batch_blob(const BatchLaunch& L) {
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  std::vector<unsigned char> host(L.bytes, 0);
  memcpy(host.data(), L.slots.data(), L.slots.size() * sizeof(SceneSlot));
  memcpy(host.data() + L.off_cmp, &L.U.cmp, sizeof(ComptonTable));
  memcpy(host.data() + L.off_ray, L.U.ray.data(), 4 * nr * sizeof(float));
  memcpy(host.data() + L.off_ray8, L.U.ray8.data(), 2 * nr);
  return host;
}

/* Point the launch-wide tables of the shared launch at the union tables in
 * the blob on the device (a solo scene's launch reads its own tables). */
void bind_blob(BatchLaunch& L, unsigned char* dbuf) {
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  for (BatchGroup& g : L.groups) {
    if (g.solo) continue;
    g.T.compton = reinterpret_cast<const ComptonTable*>(dbuf + L.off_cmp);
    const float* ray = reinterpret_cast<const float*>(dbuf + L.off_ray);
    g.T.rayleigh.xco = ray;
    g.T.rayleigh.pco = ray + nr;
    g.T.rayleigh.aco = ray + 2 * nr;
    g.T.rayleigh.bco = ray + 3 * nr;
    g.T.rayleigh.itl = dbuf + L.off_ray8;
    g.T.rayleigh.itu = dbuf + L.off_ray8 + nr;
  }
}

/* Stream work of one batched run: zero the scenes' outputs and the run
 * words (guard, counters, one lane cursor per launch in the blob), then the
 * launches, each after the first allowed to start placing blocks while the
 * previous one drains. */
mcpet_status enqueue_batch_launch(mcpet_scene* const* scenes, int n, BatchLaunch& L, unsigned char* dbuf,
                                  unsigned long long* guard, cudaStream_t st, cudaEvent_t ev0 = nullptr,
                                  cudaEvent_t ev1 = nullptr) {
  for (int k = 0; k < n; ++k) {
    mcpet_status s = zero_outputs(scenes[k], L.slots[(size_t)L.slot_of[(size_t)k]].O, st);
    if (s != MCPET_OK) return s;
  }
  unsigned long long* cursors = reinterpret_cast<unsigned long long*>(dbuf + L.off_cursor);
  CUDA_TRY(cudaMemsetAsync(guard, 0, sizeof(unsigned long long), st));
  CUDA_TRY(cudaMemsetAsync(cursors, 0, L.groups.size() * sizeof(unsigned long long), st));
  if (L.counters) CUDA_TRY(cudaMemsetAsync(L.counter_words, 0, 10 * 8, st));
  if (ev0) CUDA_TRY(cudaEventRecord(ev0, st));
  for (size_t i = 0; i < L.groups.size(); ++i) {
    const BatchGroup& g = L.groups[i];
    const SceneSlot* slots = reinterpret_cast<const SceneSlot*>(dbuf) + g.first;
    DeviceTallies O;
    memset(&O, 0, sizeof(O));
    if (g.solo) {
      O = g.O;
      O.seed_word = &slots->P.seed;   /* the slot's seed: graph replays advance it */
    }
    O.guard = guard;
    O.lane_cursor = cursors + i;
    O.counters = L.counter_words;
    if (g.solo)
      CUDA_TRY(launch_transport(g.P, g.T, O, L.counters, g.algorithm, g.mode, g.grid, L.block, g.smem, st, i > 0));
    else
      CUDA_TRY(launch_transport_batch(g.P, g.T, O, slots, g.count, L.counters, L.dose, g.share, L.mode, g.grid,
                                      L.block, g.smem, i > 0, st));
  }
  if (ev1) CUDA_TRY(cudaEventRecord(ev1, st));
  return MCPET_OK;
}

/* Enqueue the launches of the event kernel over the lanes of all scenes.
 * outs[k] are scene k's device tallies.  Each scene keeps its own lane plan
 * (cached on the scene like a single run's), seed and RANECU stream numbers,
 * so its tallies equal those of a run of that scene alone. */
mcpet_status enqueue_batch(mcpet_scene* const* scenes, int n, const mcpet_run_opts* opts, DeviceTallies* outs,
                           cudaStream_t st, double* ms_out) {
  if (!outs) return set_error(MCPET_ERR_ARG, "null argument");
  mcpet_run_opts def;
  memset(&def, 0, sizeof(def));
  const mcpet_run_opts& o = opts ? *opts : def;
  BatchLaunch L;
  mcpet_status s = setup_batch(scenes, n, o, outs, L, st);
  if (s != MCPET_OK) return s;
  for (int k = 0; k < n; ++k) outs[k] = L.slots[(size_t)L.slot_of[(size_t)k]].O;
  mcpet_scene* s0 = scenes[0];
  /* per-call device data: the slots and the union tables, released in stream order */
  const std::vector<unsigned char> host = batch_blob(L);
  unsigned char* dbuf = nullptr;
  CUDA_TRY(cudaMallocAsync((void**)&dbuf, L.bytes, st));
  CUDA_TRY(cudaMemcpyAsync(dbuf, host.data(), L.bytes, cudaMemcpyHostToDevice, st));
  for (int k = 0; k < n; ++k) scenes[k]->dev.last_h2d = scenes[k]->dev.run_h2d;
  s0->dev.last_h2d += (long long)L.bytes;
  bind_blob(L, dbuf);
  auto& d = s0->dev;
  /* the run's guard is scene 0's word */
  for (int k = 0; k < n; ++k) scenes[k]->dev.last_run_noalloc = false;
  for (int k = 1; k < n; ++k) CUDA_TRY(cudaMemsetAsync(scenes[k]->dev.small, 0, sizeof(unsigned long long), st));
  s = enqueue_batch_launch(scenes, n, L, dbuf, d.small + 0, st, ms_out ? (cudaEvent_t)d.ev0 : nullptr,
                           ms_out ? (cudaEvent_t)d.ev1 : nullptr);
  if (s != MCPET_OK) {
    cudaFreeAsync(dbuf, st);
    return s;
  }
  CUDA_TRY(cudaFreeAsync(dbuf, st));
  if (ms_out) {
    CUDA_TRY(cudaEventSynchronize((cudaEvent_t)d.ev1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, (cudaEvent_t)d.ev0, (cudaEvent_t)d.ev1));
    *ms_out = ms;
  }
  return MCPET_OK;
}

DeviceTallies tallies_from(const mcpet_tallies* out) {
  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = out->trues;
  O.scatter = out->scatter;
  O.image_trues = out->image_trues;
  O.image_scatter = out->image_scatter;
  O.spectrum = out->spectrum;
  O.psf = (uint32_t*)out->psf;
  O.psf_count = out->psf_count;
  O.histories = out->total_histories;
  O.coincidences = out->coincidences;
  O.counters = (unsigned long long*)out->counters;
  O.mat_dose = out->material_dose;
  O.vox_dose = out->voxel_dose;
  return O;
}

extern "C" {

const char* mcpet_last_error(void) { return mcpet::g_error.c_str(); }
const char* mcpet_version(void) { return "mcpet-b200 0.1 (sm_100a)"; }

mcpet_status mcpet_config_read(const char* in_path, mcpet_config* cfg) { return parse_input(in_path, cfg); }

static mcpet_status load_common(mcpet_scene* sc) {
  mcpet_status s = load_materials(sc);
  if (s != MCPET_OK) return s;
  return finalize_scene(sc);
}

mcpet_status mcpet_scene_load(const char* in_path, mcpet_scene** out) {
  if (!out) return set_error(MCPET_ERR_ARG, "null output");
  *out = nullptr;
  mcpet_scene* sc = new (std::nothrow) mcpet_scene();
  if (!sc) return set_error(MCPET_ERR_NOMEM, "out of host memory");
  mcpet_status s = parse_input(in_path, &sc->cfg);
  if (s == MCPET_OK) s = load_phantom_file(sc->cfg.voxel_file, sc->cfg.density_factor, sc);
  if (s == MCPET_OK) s = load_common(sc);
  if (s != MCPET_OK) {
    delete sc;
    return s;
  }
  *out = sc;
  return MCPET_OK;
}

mcpet_status mcpet_scene_from_arrays(const mcpet_config* cfg, int nx, int ny, int nz, const float voxel_size_cm[3],
                                     const int32_t* material, const float* density, const float* activity,
                                     mcpet_scene** out) {
  if (!out || !cfg) return set_error(MCPET_ERR_ARG, "null argument");
  *out = nullptr;
  mcpet_scene* sc = new (std::nothrow) mcpet_scene();
  if (!sc) return set_error(MCPET_ERR_NOMEM, "out of host memory");
  sc->cfg = *cfg;
  if (sc->cfg.span <= 0) {
    delete sc;
    return set_error(MCPET_ERR_ARG, "SPAN must be positive");
  }
  derive_sinogram_sizes(&sc->cfg);
  mcpet_status s = set_phantom_arrays(nx, ny, nz, voxel_size_cm, material, density, activity,
                                      sc->cfg.density_factor, sc);
  if (s == MCPET_OK) s = load_common(sc);
  if (s != MCPET_OK) {
    delete sc;
    return s;
  }
  *out = sc;
  return MCPET_OK;
}

mcpet_status mcpet_scene_set_activity(mcpet_scene* sc, const float* activity) {
  if (!sc || !activity) return set_error(MCPET_ERR_ARG, "null argument");
  std::copy(activity, activity + sc->activity.size(), sc->activity.begin());
  sc->dev.activity_dirty = true;
  sc->emitting_activity = -1;
  return MCPET_OK;
}

mcpet_status mcpet_scene_get_config(const mcpet_scene* sc, mcpet_config* cfg) {
  if (!sc || !cfg) return set_error(MCPET_ERR_ARG, "null argument");
  *cfg = sc->cfg;
  return MCPET_OK;
}

mcpet_status mcpet_scene_get_info(const mcpet_scene* sc, mcpet_scene_info* info) {
  if (!sc || !info) return set_error(MCPET_ERR_ARG, "null argument");
  memset(info, 0, sizeof(*info));
  info->nx = sc->nx;
  info->ny = sc->ny;
  info->nz = sc->nz;
  for (int k = 0; k < 3; ++k) {
    info->voxel_size[k] = sc->voxel_size[k];
    info->bbox[k] = sc->bbox[k];
  }
  info->n_voxels = (long long)sc->mat0.size();
  double tot = 0;
  long long ne = 0;
  for (float a : sc->activity)
    if (a > 1.0e-7f) {
      ne++;
      tot += a;
    }
  info->n_emitting_voxels = ne;
  info->total_activity_bq = tot;
  info->n_energy = sc->n_e;
  info->e0 = sc->e0;
  info->inv_de = sc->ide;
  int used = 0;
  for (int m = 0; m < kMaxMaterials; ++m) {
    if (sc->material_loaded[m]) used++;
    info->density_max[m] = sc->density_max[m];
    info->density_nominal[m] = sc->density_nominal[m];
  }
  info->n_materials_used = used;
  info->n_palette = (int)sc->palette.size();
  info->n_bins = sc->cfg.n_bins;
  info->n_energy_spectrum = sc->cfg.n_energy_bins;
  info->n_emitters = sc->dev.n_emitters;
  info->n_lanes = (long long)sc->dev.n_lanes;
  info->last_h2d_bytes = sc->dev.last_h2d;
  info->n_dose_voxels = dose_voxels(sc->cfg);
  return MCPET_OK;
}

mcpet_status mcpet_scene_export_tables(const mcpet_scene* sc, float* woodcock, float* mfp_a, float* mfp_b,
                                       float* voxels, float* fco, float* uico, float* fj0, int32_t* noscco,
                                       float* xco, float* pco, float* aco, float* bco, float* pmax, uint8_t* itlco,
                                       uint8_t* ituco) {
  if (!sc) return set_error(MCPET_ERR_ARG, "null scene");
  if (woodcock) std::copy(sc->woodcock.begin(), sc->woodcock.end(), woodcock);
  if (mfp_a) std::copy(sc->mfp_a.begin(), sc->mfp_a.end(), mfp_a);
  if (mfp_b) std::copy(sc->mfp_b.begin(), sc->mfp_b.end(), mfp_b);
  if (voxels)
    for (size_t i = 0; i < sc->mat0.size(); ++i) {
      voxels[3 * i + 0] = (float)(sc->mat0[i] + 1) + 0.0001f;
      voxels[3 * i + 1] = sc->rho[i];
      voxels[3 * i + 2] = sc->activity[i];
    }
  if (fco) memcpy(fco, sc->compton.fco, sizeof(sc->compton.fco));
  if (uico) memcpy(uico, sc->compton.uico, sizeof(sc->compton.uico));
  if (fj0) memcpy(fj0, sc->compton.fj0, sizeof(sc->compton.fj0));
  if (noscco) memcpy(noscco, sc->compton.noscco, sizeof(sc->compton.noscco));
  if (xco) std::copy(sc->xco.begin(), sc->xco.end(), xco);
  if (pco) std::copy(sc->pco.begin(), sc->pco.end(), pco);
  if (aco) std::copy(sc->aco.begin(), sc->aco.end(), aco);
  if (bco) std::copy(sc->bco.begin(), sc->bco.end(), bco);
  if (pmax) std::copy(sc->pmax.begin(), sc->pmax.end(), pmax);
  if (itlco) std::copy(sc->itl.begin(), sc->itl.end(), itlco);
  if (ituco) std::copy(sc->itu.begin(), sc->itu.end(), ituco);
  return MCPET_OK;
}

void mcpet_scene_free(mcpet_scene* sc) { delete sc; }

mcpet_status mcpet_scene_to_device(mcpet_scene* sc, int device) {
  if (!sc) return set_error(MCPET_ERR_ARG, "null scene");
  int dev = pick_device(device >= 0 ? device : sc->cfg.gpu_id);
  if (dev < 0) return set_error(MCPET_ERR_CUDA, "no CUDA device available");
  if (sc->dev.device >= 0 && sc->dev.device != dev)
    return set_error(MCPET_ERR_ARG, "scene already bound to device %d", sc->dev.device);
  CUDA_TRY(cudaSetDevice(dev));
  sc->dev.device = dev;
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  sc->dev.sm_count = sms;
  return upload_tables(sc);
}

mcpet_status mcpet_run_device(mcpet_scene* sc, const mcpet_run_opts* opts, mcpet_tallies* out) {
  {
    const mcpet_status as_ = check_no_async(sc);
    if (as_ != MCPET_OK) return as_;
  }
  if (!sc || !out) return set_error(MCPET_ERR_ARG, "null argument");
  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = out->trues;
  O.scatter = out->scatter;
  O.image_trues = out->image_trues;
  O.image_scatter = out->image_scatter;
  O.spectrum = out->spectrum;
  O.psf = (uint32_t*)out->psf;
  O.psf_count = out->psf_count;
  O.histories = out->total_histories;
  O.coincidences = out->coincidences;
  O.counters = (unsigned long long*)out->counters;
  O.mat_dose = out->material_dose;
  O.vox_dose = out->voxel_dose;
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  double ms = 0;
  mcpet_status s = enqueue_run(sc, opts, O, st, out->transport_ms ? &ms : nullptr);
  if (s == MCPET_OK && out->transport_ms) *out->transport_ms = ms;
  return s;
}

mcpet_status mcpet_run(mcpet_scene* sc, const mcpet_run_opts* opts, mcpet_tallies* out) {
  {
    const mcpet_status as_ = check_no_async(sc);
    if (as_ != MCPET_OK) return as_;
  }
  if (!sc || !out) return set_error(MCPET_ERR_ARG, "null argument");
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  s = ensure_device(sc);
  if (s != MCPET_OK) return s;
  s = upload_tables(sc);
  if (s != MCPET_OK) return s;
  const bool want_psf = (sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 1) && out->psf;
  s = ensure_run_buffers(sc, want_psf);
  if (s != MCPET_OK) return s;
  auto& d = sc->dev;
  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = d.trues;
  O.scatter = d.scatter;
  O.image_trues = d.img_t;
  O.image_scatter = d.img_s;
  O.spectrum = d.spectrum;
  O.psf = want_psf ? d.psf : nullptr;
  O.histories = d.small + 2;
  O.psf_count = (int*)(d.small + 3);
  O.coincidences = d.small + 14;
  O.counters = (opts && opts->collect_counters) ? d.small + 4 : nullptr;
  O.mat_dose = out->material_dose ? d.mdose : nullptr;
  O.vox_dose = out->voxel_dose ? d.vdose : nullptr;
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  double ms = 0;
  s = enqueue_run(sc, opts, O, st, &ms);
  if (s != MCPET_OK) return s;
  return download_run(sc, opts, out, want_psf, ms, st);
}

}  // extern "C"

namespace {

/* Second set of tallies, word snapshots, download stream and events of the
 * asynchronous runs (allocated on first use). */
mcpet_status ensure_async(mcpet_scene* sc) {
  auto& d = sc->dev;
  const long long nb = sc->cfg.n_bins, nv = (long long)sc->mat0.size();
  const int ne = sc->cfg.n_energy_bins;
  if (d.nbins_b != nb) {
    dfree(d.trues_b);
    dfree(d.scatter_b);
    CUDA_TRY(dmalloc(&d.trues_b, (size_t)nb * 4));
    CUDA_TRY(dmalloc(&d.scatter_b, (size_t)nb * 4));
    d.nbins_b = nb;
  }
  if (d.nvox_b != nv) {
    dfree(d.img_t_b);
    dfree(d.img_s_b);
    CUDA_TRY(dmalloc(&d.img_t_b, (size_t)nv * 4));
    CUDA_TRY(dmalloc(&d.img_s_b, (size_t)nv * 4));
    d.nvox_b = nv;
  }
  if (d.ne_b != ne) {
    dfree(d.spectrum_b);
    CUDA_TRY(dmalloc(&d.spectrum_b, (size_t)std::max(ne, 1) * 4));
    d.ne_b = ne;
  }
  if (!d.async_words) CUDA_TRY(dmalloc(&d.async_words, 2 * 16 * sizeof(unsigned long long)));
  if (!d.async_host) {
    CUDA_TRY(cudaMallocHost((void**)&d.async_host, 2 * 16 * sizeof(unsigned long long)));
    memset(d.async_host, 0, 2 * 16 * sizeof(unsigned long long));
  }
  if (!d.copy_stream) {
    cudaStream_t cs = nullptr;
    CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    d.copy_stream = cs;
  }
  for (int k = 0; k < 2; ++k) {
    if (!d.ran[k]) {
      cudaEvent_t e = nullptr;
      CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      d.ran[k] = e;
    }
    if (!d.copied[k]) {
      cudaEvent_t e = nullptr;
      CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      d.copied[k] = e;
    }
  }
  return MCPET_OK;
}

/* Host function at the end of an asynchronous download: the run's scalars
 * from the pinned snapshot into the caller's variables. */
void CUDART_CB finish_async(void* p) {
  const auto* a = static_cast<const mcpet_scene::Device::AsyncOut*>(p);
  const unsigned long long* w = a->words;
  if (a->psf_count) *a->psf_count = (int32_t)(w[3] & 0xffffffffull);
  if (a->total_histories) *a->total_histories = w[2];
  if (a->coincidences) *a->coincidences = w[14];
  if (a->counters) {
    memset(a->counters, 0, sizeof(mcpet_counters));
    if (a->counters_on) memcpy(a->counters, w + 4, 10 * 8);
    a->counters->guard_trips = w[0];
  }
  if (w[0]) __atomic_fetch_add(a->guard_sum, w[0], __ATOMIC_RELAXED);
}

}  // namespace

extern "C" {

mcpet_status mcpet_scene_lane_plan(const mcpet_scene* sc, int lane_mode, int histories_per_lane,
                                   long long capacity, uint32_t* voxel, uint32_t* n_lanes,
                                   unsigned long long* first_lane, unsigned long long* stream_base,
                                   double* inv_rate, long long* n_emitters, unsigned long long* total_lanes) {
  if (!sc || !n_emitters) return set_error(MCPET_ERR_ARG, "null argument");
  if (lane_mode < 0 || lane_mode > 1) return set_error(MCPET_ERR_ARG, "unknown lane mode %d", lane_mode);
  const int tpb = sc->cfg.threads_per_block > 0 ? sc->cfg.threads_per_block : 32;
  const int hpl = histories_per_lane > 0 ? histories_per_lane : auto_hpl(sc);
  std::vector<Emitter> em;
  uint64_t lanes = 0;
  mcpet_status s = plan_host(sc, lane_mode, tpb, hpl, em, lanes);
  if (s != MCPET_OK) return s;
  *n_emitters = (long long)em.size();
  if (total_lanes) *total_lanes = lanes;
  if (capacity < (long long)em.size())
    return set_error(MCPET_ERR_LIMIT, "lane plan has %zu emitters, capacity %lld", em.size(), capacity);
  for (size_t i = 0; i < em.size(); ++i) {
    if (voxel) voxel[i] = em[i].voxel;
    if (n_lanes) n_lanes[i] = em[i].n_lanes;
    if (first_lane) first_lane[i] = em[i].first_lane;
    if (stream_base) stream_base[i] = em[i].stream_base;
    if (inv_rate) inv_rate[i] = em[i].inv_rate;
  }
  return MCPET_OK;
}

mcpet_status mcpet_run_async(mcpet_scene* sc, const mcpet_run_opts* opts, mcpet_tallies* out) {
  if (!sc || !out) return set_error(MCPET_ERR_ARG, "null argument");
  if (out->psf || out->material_dose || out->voxel_dose)
    return set_error(MCPET_ERR_ARG, "asynchronous runs download no PSF or dose tallies (use mcpet_run)");
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  s = ensure_device(sc);
  if (s != MCPET_OK) return s;
  s = upload_tables(sc);
  if (s != MCPET_OK) return s;
  s = ensure_run_buffers(sc, false);
  if (s != MCPET_OK) return s;
  s = ensure_async(sc);
  if (s != MCPET_OK) return s;
  auto& d = sc->dev;
  const int k = d.async_next;
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  cudaStream_t cs = (cudaStream_t)d.copy_stream;
  /* set k is free again once its previous download finished; the host waits
   * too, because that download's host function still reads async_out[k] */
  if (d.copied_pending[k]) {
    CUDA_TRY(cudaEventSynchronize((cudaEvent_t)d.copied[k]));
    CUDA_TRY(cudaStreamWaitEvent(st, (cudaEvent_t)d.copied[k], 0));
  }
  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = k ? d.trues_b : d.trues;
  O.scatter = k ? d.scatter_b : d.scatter;
  O.image_trues = k ? d.img_t_b : d.img_t;
  O.image_scatter = k ? d.img_s_b : d.img_s;
  O.spectrum = k ? d.spectrum_b : d.spectrum;
  O.histories = d.small + 2;
  O.psf_count = (int*)(d.small + 3);
  O.coincidences = d.small + 14;
  O.counters = (opts && opts->collect_counters) ? d.small + 4 : nullptr;
  s = enqueue_run(sc, opts, O, st, nullptr);
  if (s != MCPET_OK) return s;
  /* the run words are reused by the next run: snapshot them in stream order */
  unsigned long long* words = d.async_words + 16 * k;
  CUDA_TRY(cudaMemcpyAsync(words, d.small, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaEventRecord((cudaEvent_t)d.ran[k], st));
  /* downloads on the scene's copy stream, overlapping the next run */
  CUDA_TRY(cudaStreamWaitEvent(cs, (cudaEvent_t)d.ran[k], 0));
  const size_t nb = (size_t)sc->cfg.n_bins * 4, nv = sc->mat0.size() * 4;
  if (out->trues) CUDA_TRY(cudaMemcpyAsync(out->trues, O.trues, nb, cudaMemcpyDeviceToHost, cs));
  if (out->scatter) CUDA_TRY(cudaMemcpyAsync(out->scatter, O.scatter, nb, cudaMemcpyDeviceToHost, cs));
  if (out->image_trues) CUDA_TRY(cudaMemcpyAsync(out->image_trues, O.image_trues, nv, cudaMemcpyDeviceToHost, cs));
  if (out->image_scatter)
    CUDA_TRY(cudaMemcpyAsync(out->image_scatter, O.image_scatter, nv, cudaMemcpyDeviceToHost, cs));
  if (out->spectrum)
    CUDA_TRY(cudaMemcpyAsync(out->spectrum, O.spectrum, (size_t)sc->cfg.n_energy_bins * 4, cudaMemcpyDeviceToHost,
                             cs));
  unsigned long long* host_words = d.async_host + 16 * k;
  CUDA_TRY(cudaMemcpyAsync(host_words, words, 16 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, cs));
  auto& a = d.async_out[k];
  a.words = host_words;
  a.psf_count = out->psf_count;
  a.total_histories = out->total_histories;
  a.coincidences = out->coincidences;
  a.counters = out->counters;
  a.counters_on = opts && opts->collect_counters;
  a.guard_sum = &d.async_guard;
  CUDA_TRY(cudaLaunchHostFunc(cs, finish_async, &a));
  CUDA_TRY(cudaEventRecord((cudaEvent_t)d.copied[k], cs));
  d.copied_pending[k] = true;
  d.async_next = k ^ 1;
  return MCPET_OK;
}

mcpet_status mcpet_run_wait(mcpet_scene* sc) {
  if (!sc) return set_error(MCPET_ERR_ARG, "null argument");
  auto& d = sc->dev;
  if (!d.copy_stream) return MCPET_OK;
  CUDA_TRY(cudaSetDevice(d.device));
  CUDA_TRY(cudaStreamSynchronize((cudaStream_t)d.copy_stream));
  d.copied_pending[0] = d.copied_pending[1] = false;
  const unsigned long long g = __atomic_exchange_n(&d.async_guard, 0ull, __ATOMIC_RELAXED);
  d.last_guard = g;
  if (g != 0) return set_error(MCPET_ERR_DEVICE, "%llu device guard(s) fired (loop cap or out-of-range index)", g);
  return MCPET_OK;
}

mcpet_status mcpet_run_batch_device(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                                    mcpet_tallies* device_outs) {
  mcpet_status cs = check_batch(scenes, n_scenes, opts, nullptr);
  if (cs != MCPET_OK) return cs;
  if (!device_outs) return set_error(MCPET_ERR_ARG, "null argument");
  std::vector<DeviceTallies> O((size_t)n_scenes);
  for (int k = 0; k < n_scenes; ++k) O[(size_t)k] = tallies_from(&device_outs[k]);
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  double ms = 0;
  mcpet_status s = enqueue_batch(scenes, n_scenes, opts, O.data(), st, device_outs[0].transport_ms ? &ms : nullptr);
  if (s == MCPET_OK && device_outs[0].transport_ms) *device_outs[0].transport_ms = ms;
  return s;
}

}  // extern "C"

/* A captured batched launch that regenerates its histories on every replay. */
struct mcpet_batch_graph {
  int device = -1;
  std::vector<mcpet_scene*> scenes;
  BatchLaunch L;
  unsigned char* dbuf = nullptr;              /* slots + union tables + lane cursors */
  mcpet::Emitter* plans = nullptr;            /* copies of the scenes' lane plans */
  unsigned long long* words = nullptr;        /* guard, (unused), default coincidence words */
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~mcpet_batch_graph() {
    if (device >= 0) cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (dbuf) cudaFree(dbuf);
    if (plans) cudaFree(plans);
    if (words) cudaFree(words);
  }
};

extern "C" {

mcpet_status mcpet_batch_graph_create(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                                      const mcpet_tallies* device_outs, int seed_step, mcpet_batch_graph** out) {
  using namespace mcpet;
  if (!out) return set_error(MCPET_ERR_ARG, "null output");
  *out = nullptr;
  mcpet_status cs = check_batch(scenes, n_scenes, opts, nullptr);
  if (cs != MCPET_OK) return cs;
  if (!device_outs) return set_error(MCPET_ERR_ARG, "null argument");
  if (seed_step < 0) return set_error(MCPET_ERR_ARG, "seed step must be >= 0 (got %d)", seed_step);
  mcpet_run_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  o.stream = nullptr;
  std::unique_ptr<mcpet_batch_graph> g(new (std::nothrow) mcpet_batch_graph());
  if (!g) return set_error(MCPET_ERR_NOMEM, "out of host memory");
  mcpet_status s = scenes[0]->dev.device < 0 ? mcpet_scene_to_device(scenes[0], -1) : ensure_device(scenes[0]);
  if (s != MCPET_OK) return s;
  g->device = scenes[0]->dev.device;
  g->scenes.assign(scenes, scenes + n_scenes);
  CUDA_TRY(cudaMalloc((void**)&g->words, (size_t)(2 + n_scenes) * sizeof(unsigned long long)));
  CUDA_TRY(cudaMemset(g->words, 0, (size_t)(2 + n_scenes) * sizeof(unsigned long long)));
  std::vector<DeviceTallies> outs((size_t)n_scenes);
  for (int k = 0; k < n_scenes; ++k) {
    outs[(size_t)k] = tallies_from(&device_outs[k]);
    if (!outs[(size_t)k].coincidences) outs[(size_t)k].coincidences = g->words + 2 + k;
  }
  BatchLaunch& L = g->L;
  s = setup_batch(scenes, n_scenes, o, outs.data(), L, nullptr);
  if (s != MCPET_OK) return s;
  /* own copies of the lane plans: later runs of the scenes may rebuild theirs */
  size_t n_em = 0;
  for (int k = 0; k < n_scenes; ++k) n_em += (size_t)scenes[k]->dev.n_emitters;
  CUDA_TRY(cudaMalloc((void**)&g->plans, std::max<size_t>(n_em, 1) * sizeof(Emitter)));
  size_t off = 0;
  for (int k = 0; k < n_scenes; ++k) {
    const auto& d = scenes[k]->dev;
    if (d.n_emitters > 0)
      CUDA_TRY(cudaMemcpy(g->plans + off, d.emitters, (size_t)d.n_emitters * sizeof(Emitter),
                          cudaMemcpyDeviceToDevice));
    L.slots[(size_t)L.slot_of[(size_t)k]].T.emitters = g->plans + off;
    off += (size_t)d.n_emitters;
  }
  for (BatchGroup& grp : L.groups)
    if (grp.solo) grp.T.emitters = L.slots[(size_t)grp.first].T.emitters;
  CUDA_TRY(cudaMalloc((void**)&g->dbuf, L.bytes));
  const std::vector<unsigned char> host = batch_blob(L);
  CUDA_TRY(cudaMemcpy(g->dbuf, host.data(), L.bytes, cudaMemcpyHostToDevice));
  bind_blob(L, g->dbuf);

  /* capture: zero the outputs, the launch, then the seeds of the next replay */
  cudaStream_t cap = nullptr;
  CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    s = enqueue_batch_launch(scenes, n_scenes, L, g->dbuf, g->words + 0, cap);
    if (s == MCPET_OK) {
      cudaError_t le = launch_advance_seeds(reinterpret_cast<SceneSlot*>(g->dbuf), n_scenes, seed_step, cap);
      if (le != cudaSuccess) s = set_error(MCPET_ERR_CUDA, "CUDA error: %s", cudaGetErrorString(le));
    }
    e = cudaStreamEndCapture(cap, &g->graph);
  }
  cudaStreamDestroy(cap);
  if (s != MCPET_OK) return s;
  if (e != cudaSuccess) return set_error(MCPET_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  CUDA_TRY(cudaGraphInstantiate(&g->exec, g->graph, 0));
  *out = g.release();
  return MCPET_OK;
}

/* Autotuner: time candidate (histories per lane, threads per block) pairs
 * on a sample of the workload and keep the fastest.  The sample runs every
 * scene with its acquisition time scaled by f and the candidate's histories
 * per lane scaled by the same f, so it has the full workload's lane count and
 * lane order with f of its decays: per-lane work, fill and tail keep their
 * proportions. */
mcpet_status mcpet_autotune(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                            const mcpet_tallies* device_outs, double sample_decays, mcpet_tune_result* out) {
  using namespace mcpet;
  if (!out || !device_outs) return set_error(MCPET_ERR_ARG, "null argument");
  memset(out, 0, sizeof(*out));
  mcpet_run_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (n_scenes > 1) {
    mcpet_status cs = check_batch(scenes, n_scenes, &o, nullptr);
    if (cs != MCPET_OK) return cs;
  } else {
    if (n_scenes != 1 || !scenes || !scenes[0]) return set_error(MCPET_ERR_ARG, "autotune needs at least one scene");
    mcpet_status cs = validate_opts(scenes[0], &o);
    if (cs != MCPET_OK) return cs;
    cs = check_no_async(scenes[0]);
    if (cs != MCPET_OK) return cs;
  }
  o.collect_counters = 0;
  const bool balanced = o.lane_mode == MCPET_LANES_BALANCED;
  for (int k = 0; k < n_scenes; ++k) {
    mcpet_status s = (k > 0 && scenes[k]->dev.device < 0) ? mcpet_scene_to_device(scenes[k], scenes[0]->dev.device)
                                                          : ensure_device(scenes[k]);
    if (s != MCPET_OK) return s;
  }
  /* decays of the workload; the candidates: 1/4 ... 4 times the histories
   * per lane sized from all scenes' decays together and, for a batch, the
   * automatic choice (0: every scene its own automatic lanes).  With
   * reference lanes the plan is fixed and only the block size is tuned. */
  double D = 0;
  for (int k = 0; k < n_scenes; ++k)
    D += emitting_activity(scenes[k]) * ((double)scenes[k]->cfg.acquisition_time_ps * 1e-12);
  const int base = auto_hpl_of(std::vector<const mcpet_scene*>(scenes, scenes + n_scenes));
  const int auto_choice = (balanced && n_scenes == 1) ? base : 0;
  std::vector<int> hpls(1, auto_choice);
  int smallest = 0;
  if (balanced) {
    const int c[5] = {std::max(1, base / 4), std::max(1, base / 2), base, 2 * base, 4 * base};
    smallest = c[0];
    for (int v : c)
      if (std::find(hpls.begin(), hpls.end(), v) == hpls.end()) hpls.push_back(v);
  }
  double f = (sample_decays > 0 ? sample_decays : 2.0e8) / std::max(D, 1.0);
  if (balanced) f = std::max(f, 1.0 / (double)smallest);
  if (f > 1.0) f = 1.0;
  out->sample_fraction = f;

  std::vector<unsigned long long> acq((size_t)n_scenes);
  for (int k = 0; k < n_scenes; ++k) {
    acq[(size_t)k] = scenes[k]->cfg.acquisition_time_ps;
    scenes[k]->cfg.acquisition_time_ps = (unsigned long long)llround((double)acq[(size_t)k] * f);
    scenes[k]->tune_scale = f;   /* a batch groups the scenes by their full decays */
    scenes[k]->dev.activity_dirty = true;
  }
  std::vector<DeviceTallies> outs((size_t)n_scenes);
  cudaStream_t st = (cudaStream_t)o.stream;
  auto time_one = [&](int hpl, int block, double* ms) -> mcpet_status {
    mcpet_run_opts c = o;
    c.histories_per_lane = (balanced && hpl > 0) ? std::max(1, (int)llround(hpl * f)) : 0;
    c.block_threads = block;
    for (int k = 0; k < n_scenes; ++k) outs[(size_t)k] = tallies_from(&device_outs[k]);
    if (n_scenes == 1) return enqueue_run(scenes[0], &c, outs[0], st, ms);
    return enqueue_batch(scenes, n_scenes, &c, outs.data(), st, ms);
  };
  mcpet_status s = MCPET_OK;
  double best = 1e300, ms = 0;
  int best_hpl = hpls[0], best_block = transport_block_threads();
  /* first the histories per lane at the full block, then the block size */
  s = time_one(auto_choice, best_block, &ms);   /* warm-up: clocks, tables, first plan */
  for (size_t i = 0; s == MCPET_OK && i < hpls.size(); ++i) {
    s = time_one(hpls[i], transport_block_threads(), &ms);
    ++out->candidates;
    if (s == MCPET_OK && hpls[i] == auto_choice) out->auto_ms = ms;
    if (s == MCPET_OK && ms < best) {
      best = ms;
      best_hpl = hpls[i];
    }
  }
  const int blocks[2] = {128, 192};
  for (int i = 0; s == MCPET_OK && i < 2; ++i) {
    if (blocks[i] >= transport_block_threads()) continue;
    s = time_one(best_hpl, blocks[i], &ms);
    ++out->candidates;
    if (s == MCPET_OK && ms < best) {
      best = ms;
      best_block = blocks[i];
    }
  }
  for (int k = 0; k < n_scenes; ++k) {
    scenes[k]->cfg.acquisition_time_ps = acq[(size_t)k];
    scenes[k]->tune_scale = 1.0;
    scenes[k]->dev.activity_dirty = true;
  }
  if (s != MCPET_OK) return s;
  out->histories_per_lane = balanced ? best_hpl : 0;   /* 0 for a batch: the automatic choice won */
  out->block_threads = best_block;
  out->best_ms = best;
  return MCPET_OK;
}

mcpet_status mcpet_batch_graph_launch(mcpet_batch_graph* g, void* stream) {
  using namespace mcpet;
  if (!g || !g->exec) return set_error(MCPET_ERR_ARG, "null graph");
  CUDA_TRY(cudaSetDevice(g->device));
  CUDA_TRY(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return MCPET_OK;
}

mcpet_status mcpet_batch_graph_set_seeds(mcpet_batch_graph* g, const int* seeds, void* stream) {
  using namespace mcpet;
  if (!g || !seeds) return set_error(MCPET_ERR_ARG, "null argument");
  const int n = (int)g->scenes.size();
  for (int k = 0; k < n; ++k)
    if (seeds[k] <= 0 || seeds[k] >= (int)2147483563)
      return set_error(MCPET_ERR_ARG, "seed %d of scene %d outside [1, 2147483562]", seeds[k], k);
  CUDA_TRY(cudaSetDevice(g->device));
  for (int k = 0; k < n; ++k) {
    const size_t j = (size_t)g->L.slot_of[(size_t)k];
    g->L.slots[j].P.seed = seeds[k];
    unsigned char* dst = g->dbuf + j * sizeof(SceneSlot) + offsetof(SceneSlot, P) + offsetof(TransportParams, seed);
    CUDA_TRY(cudaMemcpyAsync(dst, &g->L.slots[j].P.seed, sizeof(int), cudaMemcpyHostToDevice,
                             (cudaStream_t)stream));
  }
  CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return MCPET_OK;
}

mcpet_status mcpet_batch_graph_guard_trips(mcpet_batch_graph* g, unsigned long long* trips) {
  using namespace mcpet;
  if (!g || !trips) return set_error(MCPET_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(g->device));
  CUDA_TRY(cudaMemcpy(trips, g->words, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

void mcpet_batch_graph_destroy(mcpet_batch_graph* g) { delete g; }

mcpet_status mcpet_run_batch(mcpet_scene* const* scenes, int n_scenes, const mcpet_run_opts* opts,
                             mcpet_tallies* outs) {
  mcpet_status cs = check_batch(scenes, n_scenes, opts, nullptr);
  if (cs != MCPET_OK) return cs;
  if (!outs) return set_error(MCPET_ERR_ARG, "null argument");
  std::vector<DeviceTallies> O((size_t)n_scenes);
  std::vector<char> want((size_t)n_scenes, 0);
  for (int k = 0; k < n_scenes; ++k) {
    mcpet_scene* sc = scenes[k];
    mcpet_status s = (k > 0 && sc->dev.device < 0) ? mcpet_scene_to_device(sc, scenes[0]->dev.device) : ensure_device(sc);
    if (s != MCPET_OK) return s;
    s = upload_tables(sc);
    if (s != MCPET_OK) return s;
    const bool want_psf = (sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 1) && outs[k].psf;
    want[(size_t)k] = want_psf;
    s = ensure_run_buffers(sc, want_psf);
    if (s != MCPET_OK) return s;
    auto& d = sc->dev;
    DeviceTallies& z = O[(size_t)k];
    memset(&z, 0, sizeof(z));
    z.trues = d.trues;
    z.scatter = d.scatter;
    z.image_trues = d.img_t;
    z.image_scatter = d.img_s;
    z.spectrum = d.spectrum;
    z.psf = want_psf ? d.psf : nullptr;
    z.histories = d.small + 2;
    z.psf_count = (int*)(d.small + 3);
    z.coincidences = d.small + 14;
    z.counters = (k == 0 && opts && opts->collect_counters) ? d.small + 4 : nullptr;
    z.mat_dose = outs[k].material_dose ? d.mdose : nullptr;
    z.vox_dose = outs[k].voxel_dose ? d.vdose : nullptr;
  }
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  double ms = 0;
  mcpet_status s = enqueue_batch(scenes, n_scenes, opts, O.data(), st, &ms);
  if (s != MCPET_OK) return s;
  /* scene 0 holds the launch's guard word and counters */
  mcpet_run_opts rest;
  memset(&rest, 0, sizeof(rest));
  if (opts) rest = *opts;
  rest.collect_counters = 0;
  mcpet_status err = MCPET_OK;
  for (int k = 0; k < n_scenes; ++k) {
    s = download_run(scenes[k], k == 0 ? opts : &rest, &outs[k], want[(size_t)k] != 0, ms, st);
    if (s != MCPET_OK && err == MCPET_OK) err = s;
  }
  return err;
}

mcpet_status mcpet_grad(mcpet_scene* sc, const mcpet_run_opts* opts, mcpet_tallies* device_out,
                        mcpet_grad_args* g) {
  {
    const mcpet_status as_ = check_no_async(sc);
    if (as_ != MCPET_OK) return as_;
  }
  if (!sc || !device_out || !g) return set_error(MCPET_ERR_ARG, "null argument");
  if (!g->measured) return set_error(MCPET_ERR_ARG, "the measured sinogram is required");
  if (!device_out->trues || !device_out->scatter)
    return set_error(MCPET_ERR_ARG, "the gradient needs the trues and scatter sinograms of the forward run");
  if (!(sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 2))
    return set_error(MCPET_ERR_ARG, "the gradient needs the sinogram tally (REPORT PSF/SINOGRAM 0 or 2)");
  if (sc->cfg.prompt_gamma_energy > 0.0f)
    return set_error(MCPET_ERR_ARG, "the gradient replays annihilation pairs only: no prompt-gamma emitter");
  if (g->event_buffer && g->event_capacity <= 0) return set_error(MCPET_ERR_ARG, "event_capacity must be > 0");
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  s = ensure_device(sc);
  if (s != MCPET_OK) return s;
  s = upload_tables(sc);
  if (s != MCPET_OK) return s;
  auto& d = sc->dev;
  cudaStream_t st = opts ? (cudaStream_t)opts->stream : nullptr;
  const long long nv = (long long)sc->mat0.size();
  if (!d.gwords) CUDA_TRY(dmalloc(&d.gwords, 4 * sizeof(unsigned long long)));
  if (!d.activity) CUDA_TRY(dmalloc(&d.activity, (size_t)nv * sizeof(float)));
  CUDA_TRY(cudaMemcpyAsync(d.activity, sc->activity.data(), (size_t)nv * sizeof(float), cudaMemcpyHostToDevice, st));

  /* forward transport with event records; grown and repeated (same seed,
   * same events) if the buffer was too small */
  unsigned long long n_events = 0;
  double fwd_ms = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    uint32_t* ev = (uint32_t*)g->event_buffer;
    long long cap = g->event_capacity;
    if (!ev) {
      if (d.event_cap <= 0) {
        const double expect = emitting_activity(sc) * ((double)sc->cfg.acquisition_time_ps * 1e-12);
        long long want = (long long)std::min(std::max(expect * 0.15, 1.0e6), 2.0e9);
        CUDA_TRY(dmalloc(&d.events, (size_t)want * sizeof(EventRecord)));
        d.event_cap = want;
      }
      ev = d.events;
      cap = d.event_cap;
    }
    DeviceTallies O = tallies_from(device_out);
    O.mat_dose = nullptr;   /* the recording forward does not tally dose */
    O.vox_dose = nullptr;
    O.events = ev;
    O.event_count = d.small + 15;
    O.event_capacity = cap;
    CUDA_TRY(cudaMemsetAsync(O.event_count, 0, sizeof(unsigned long long), st));
    s = enqueue_run(sc, opts, O, st, &fwd_ms);
    if (s != MCPET_OK) return s;
    CUDA_TRY(cudaMemcpyAsync(&n_events, d.small + 15, sizeof(n_events), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (n_events <= (unsigned long long)cap) break;
    if (g->event_buffer || attempt == 1)
      return set_error(MCPET_ERR_LIMIT, "%llu tallied coincidences, event buffer holds %lld", n_events, cap);
    dfree(d.events);
    const long long want = (long long)((double)n_events * 1.1) + 1024;
    CUDA_TRY(dmalloc(&d.events, (size_t)want * sizeof(EventRecord)));
    d.event_cap = want;
  }
  unsigned long long guard = 0;
  CUDA_TRY(cudaMemcpy(&guard, d.small, sizeof(guard), cudaMemcpyDeviceToHost));
  d.last_guard = guard;
  if (guard != 0)
    return set_error(MCPET_ERR_DEVICE, "%llu device guard(s) fired (loop cap or out-of-range index)", guard);

  /* log-likelihood and the replay of the recorded events */
  TransportParams P;
  fill_params(sc, P);
  if (opts && opts->seed_override != 0) P.seed = opts->seed_override;
  P.background_mode = (opts && opts->background_mode) ? 1 : 0;
  DeviceTables T = device_tables(sc);
  CUDA_TRY(cudaMemsetAsync(d.gwords, 0, 4 * sizeof(unsigned long long), st));
  if (g->grad_activity) CUDA_TRY(cudaMemsetAsync(g->grad_activity, 0, (size_t)nv * sizeof(float), st));
  if (g->grad_density_scale) CUDA_TRY(cudaMemsetAsync(g->grad_density_scale, 0, (size_t)nv * sizeof(float), st));
  CUDA_TRY(cudaEventRecord((cudaEvent_t)d.ev0, st));
  CUDA_TRY(launch_loglik(sc->cfg.n_bins, g->measured, device_out->trues, device_out->scatter, g->background,
                         reinterpret_cast<double*>(d.gwords + 2), d.sm_count, st));
  if (n_events > 0 && (g->grad_activity || g->grad_density_scale))
    CUDA_TRY(launch_grad_replay(P, T, g->event_buffer ? (const uint32_t*)g->event_buffer : d.events, n_events,
                                g->measured, device_out->trues, device_out->scatter, g->background, d.activity,
                                g->grad_activity, g->grad_density_scale, d.gwords, d.sm_count,
                                (opts && opts->lane_mode == MCPET_LANES_BALANCED) ? kTransportFast : 0, st));
  CUDA_TRY(cudaEventRecord((cudaEvent_t)d.ev1, st));
  unsigned long long words[4];
  CUDA_TRY(cudaMemcpyAsync(words, d.gwords, sizeof(words), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  float gms = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&gms, (cudaEvent_t)d.ev0, (cudaEvent_t)d.ev1));
  double ll;
  memcpy(&ll, &words[2], sizeof(ll));
  g->loglik = ll;
  g->events = n_events;
  g->replayed = words[0];
  g->mismatches = words[1];
  g->forward_ms = fwd_ms;
  g->gradient_ms = gms;
  return MCPET_OK;
}

mcpet_status mcpet_run_psf_stream(mcpet_scene* sc, const mcpet_run_opts* opts, long long chunk_records,
                                  mcpet_psf_sink sink, void* user, mcpet_tallies* out) {
  {
    const mcpet_status as_ = check_no_async(sc);
    if (as_ != MCPET_OK) return as_;
  }
  if (!sc || !sink || !out) return set_error(MCPET_ERR_ARG, "null argument");
  if (!(sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 1))
    return set_error(MCPET_ERR_ARG, "the scene does not tally a PSF (REPORT PSF/SINOGRAM 0 or 1)");
  if (chunk_records < 2 || chunk_records > 0x7fffffffLL)
    return set_error(MCPET_ERR_ARG, "chunk_records must be in [2, 2^31)");
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  s = ensure_device(sc);
  if (s != MCPET_OK) return s;
  s = upload_tables(sc);
  if (s != MCPET_OK) return s;
  s = ensure_run_buffers(sc, false);
  if (s != MCPET_OK) return s;
  mcpet_run_opts def;
  memset(&def, 0, sizeof(def));
  const mcpet_run_opts& o = opts ? *opts : def;
  const int tpb = sc->cfg.threads_per_block > 0 ? sc->cfg.threads_per_block : 32;
  const int hpl = o.histories_per_lane > 0 ? o.histories_per_lane : auto_hpl(sc);
  sc->dev.run_h2d = 0;
  cudaStream_t st = (cudaStream_t)o.stream;
  s = build_lanes(sc, o.lane_mode, tpb, hpl, st);
  if (s != MCPET_OK) return s;
  auto& d = sc->dev;

  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = d.trues;
  O.scatter = d.scatter;
  O.image_trues = d.img_t;
  O.image_scatter = d.img_s;
  O.spectrum = d.spectrum;
  O.histories = d.small + 2;
  O.psf_count = (int*)(d.small + 3);
  O.coincidences = d.small + 14;
  O.counters = o.collect_counters ? d.small + 4 : nullptr;
  O.mat_dose = out->material_dose ? d.mdose : nullptr;
  O.vox_dose = out->voxel_dose ? d.vdose : nullptr;
  TransportParams P;
  s = prepare_run(sc, o, O, st, P);
  if (s != MCPET_OK) return s;
  O.guard = d.small + 0;
  O.lane_cursor = d.small + 1;
  d.last_run_noalloc = false;
  CUDA_TRY(cudaMemsetAsync(d.small, 0, 2 * sizeof(unsigned long long), st));
  if (O.counters) CUDA_TRY(cudaMemsetAsync(O.counters, 0, 10 * 8, st));
  if (!d.gwords) CUDA_TRY(dmalloc(&d.gwords, 4 * sizeof(unsigned long long)));

  uint32_t* chunk = nullptr;
  CUDA_TRY(dmalloc(&chunk, (size_t)chunk_records * 44));
  std::vector<unsigned char> host((size_t)chunk_records * 44);
  O.psf = chunk;
  P.psf_capacity = (int)chunk_records;
  P.n_emitters = d.n_emitters;
  const uint64_t total = d.n_lanes;
  long long streamed = 0;
  double ms_sum = 0;
  mcpet_status err = MCPET_OK;

  /* one launch over lanes [b, e): dry = replay of a range whose records did
   * not fit (no sinogram-side writes, totals to scratch words) */
  auto run_range = [&](uint64_t b, uint64_t e, bool dry, int& count) -> mcpet_status {
    TransportParams Q = P;
    DeviceTallies R = O;
    Q.n_lanes = e;
    Q.sino_dry = dry ? 1 : 0;
    if (dry) {
      R.histories = d.gwords + 0;
      R.coincidences = d.gwords + 1;
      R.counters = nullptr;
      R.mat_dose = nullptr;
      R.vox_dose = nullptr;
    }
    unsigned long long begin = b;
    CUDA_TRY(cudaMemcpyAsync(O.lane_cursor, &begin, sizeof(begin), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(O.psf_count, 0, 4, st));
    double ms = 0;
    mcpet_status r = launch_planned(sc, o, Q, R, st, &ms);
    if (r != MCPET_OK) return r;
    ms_sum += ms;
    CUDA_TRY(cudaMemcpyAsync(&count, O.psf_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return MCPET_OK;
  };
  auto drain = [&](int count) -> mcpet_status {
    if (count <= 0) return MCPET_OK;
    CUDA_TRY(cudaMemcpy(host.data(), chunk, (size_t)count * 44, cudaMemcpyDeviceToHost));
    streamed += count;
    if (sink(host.data(), count, user) != 0) return set_error(MCPET_ERR_ARG, "the PSF sink stopped the run");
    return MCPET_OK;
  };
  /* ranges whose records overflowed the chunk, replayed in halves */
  std::vector<std::pair<uint64_t, uint64_t>> redo;
  uint64_t b = 0, span = std::max<uint64_t>(1, total / 64);
  while (err == MCPET_OK && b < total) {
    const uint64_t e = std::min<uint64_t>(total, b + span);
    int count = 0;
    err = run_range(b, e, false, count);
    if (err != MCPET_OK) break;
    if (count <= chunk_records) {
      err = drain(count);
      const double per_lane = (double)std::max(count, 1) / (double)(e - b);
      span = std::max<uint64_t>(1, (uint64_t)(0.5 * (double)chunk_records / per_lane));
    } else {
      redo.push_back({b, e});
      span = std::max<uint64_t>(1, (e - b) / 4);
    }
    b = e;
  }
  while (err == MCPET_OK && !redo.empty()) {
    auto r = redo.back();
    redo.pop_back();
    int count = 0;
    err = run_range(r.first, r.second, true, count);
    if (err != MCPET_OK) break;
    if (count <= chunk_records) {
      err = drain(count);
    } else if (r.second - r.first == 1) {
      err = set_error(MCPET_ERR_LIMIT, "one lane produced %d PSF records, more than a chunk of %lld", count,
                      chunk_records);
    } else {
      const uint64_t m = r.first + (r.second - r.first) / 2;
      redo.push_back({m, r.second});
      redo.push_back({r.first, m});
    }
  }
  dfree(chunk);
  if (err != MCPET_OK) return err;
  /* sinograms, images, spectrum and totals as mcpet_run reports them */
  mcpet_tallies t = *out;
  t.psf = nullptr;
  t.psf_capacity = 0;
  int dummy = 0;
  t.psf_count = &dummy;
  s = download_run(sc, opts, &t, false, ms_sum, st);
  if (out->psf_count) *out->psf_count = (int)std::min<long long>(streamed, 0x7fffffff);
  return s;
}

mcpet_status mcpet_run_device_noalloc(mcpet_scene* sc, const float* activity_device, const mcpet_run_opts* opts,
                                      mcpet_tallies* out) {
  {
    const mcpet_status as_ = check_no_async(sc);
    if (as_ != MCPET_OK) return as_;
  }
  if (!sc || !activity_device || !out) return set_error(MCPET_ERR_ARG, "null argument");
  const long long nv = (long long)sc->mat0.size();
  if (nv > MCPET_NOALLOC_MAX_VOXELS || nv > kNoAllocMaxVoxels)
    return set_error(MCPET_ERR_LIMIT,
                     "phantom has %lld voxels; the allocation-free run holds lane plans of at most %d voxels "
                     "(use mcpet_run_device)", nv, (int)kNoAllocMaxVoxels);
  mcpet_status s = validate_opts(sc, opts);
  if (s != MCPET_OK) return s;
  auto& d = sc->dev;
  if (d.device < 0 || !d.tables_ready)
    return set_error(MCPET_ERR_ARG, "the scene is not on a device: call mcpet_scene_to_device first (it allocates)");
  CUDA_TRY(cudaSetDevice(d.device));
  mcpet_run_opts def;
  memset(&def, 0, sizeof(def));
  const mcpet_run_opts& o = opts ? *opts : def;
  const bool sino = sc->cfg.tally_psf_sinogram == 0 || sc->cfg.tally_psf_sinogram == 2;
  if (sino && (!out->trues || !out->scatter || !out->image_trues || !out->image_scatter || !out->spectrum))
    return set_error(MCPET_ERR_ARG, "sinogram tally requested but a sinogram/image/spectrum buffer is missing");
  if (!out->total_histories || !out->psf_count) return set_error(MCPET_ERR_ARG, "histories and psf_count are required");

  s = check_prompt(sc);
  if (s != MCPET_OK) return s;
  TransportParams P;
  fill_params(sc, P);
  if (o.seed_override != 0) P.seed = o.seed_override;
  P.background_mode = o.background_mode ? 1 : 0;
  apply_caps(o, P);
  if (!out->psf) P.psf_capacity = 0;
  else P.psf_capacity = (int)std::min<long long>(out->psf_capacity, 0x7fffffff);
  if (!sino) P.spectrum_in_shared = 0;
  const int tpb = sc->cfg.threads_per_block > 0 ? sc->cfg.threads_per_block : 32;
  /* <= 0: automatic, from the caller's activity map on the device */
  const int hpl = o.histories_per_lane > 0 ? o.histories_per_lane : 0;

  DeviceTallies O;
  memset(&O, 0, sizeof(O));
  O.trues = out->trues;
  O.scatter = out->scatter;
  O.image_trues = out->image_trues;
  O.image_scatter = out->image_scatter;
  O.spectrum = out->spectrum;
  O.psf = (uint32_t*)out->psf;
  O.psf_count = out->psf_count;
  O.histories = out->total_histories;
  O.coincidences = out->coincidences;
  O.counters = (unsigned long long*)out->counters;
  cudaStream_t st = (cudaStream_t)o.stream;
  const size_t nb = (size_t)sc->cfg.n_bins * 4, nvb = (size_t)nv * 4;
  if (O.trues) CUDA_TRY(cudaMemsetAsync(O.trues, 0, nb, st));
  if (O.scatter) CUDA_TRY(cudaMemsetAsync(O.scatter, 0, nb, st));
  if (O.image_trues) CUDA_TRY(cudaMemsetAsync(O.image_trues, 0, nvb, st));
  if (O.image_scatter) CUDA_TRY(cudaMemsetAsync(O.image_scatter, 0, nvb, st));
  if (O.spectrum) CUDA_TRY(cudaMemsetAsync(O.spectrum, 0, (size_t)sc->cfg.n_energy_bins * 4, st));
  CUDA_TRY(cudaMemsetAsync(O.psf_count, 0, 4, st));
  CUDA_TRY(cudaMemsetAsync(O.histories, 0, 8, st));
  if (O.coincidences) CUDA_TRY(cudaMemsetAsync(O.coincidences, 0, 8, st));
  const bool counters = o.collect_counters && O.counters;
  if (O.counters) CUDA_TRY(cudaMemsetAsync(O.counters, 0, 10 * 8, st));

  if (o.max_woodcock_steps > 0 || o.max_rejections > 0)
    return set_error(MCPET_ERR_ARG, "lowered loop caps are not available for the allocation-free run");
  const int mode = run_mode(sc, o);
  int block = transport_block_threads();
  size_t smem = transport_dynamic_smem(P, block, kAlgorithmEvents);
  int bps = 0;
  CUDA_TRY(transport_occupancy(counters, kAlgorithmEvents, mode, block, smem, &bps));
  if (bps < 1) return set_error(MCPET_ERR_LIMIT, "transport kernel does not fit on an SM (smem %zu)", smem);
  if (o.blocks_per_sm > 0 && o.blocks_per_sm < bps) bps = o.blocks_per_sm;
  const int grid = d.sm_count * bps;
  d.last_run_noalloc = true;
  CUDA_TRY(launch_transport_noalloc(P, device_tables(sc), O, activity_device, o.lane_mode, tpb, hpl, d.sm_count,
                                    counters, mode, grid, block, smem, st));
  return MCPET_OK;
}

mcpet_status mcpet_last_run_guard(mcpet_scene* sc, unsigned long long* trips) {
  if (!sc || !trips) return set_error(MCPET_ERR_ARG, "null argument");
  if (sc->dev.device < 0 || !sc->dev.small) {
    *trips = 0;
    return MCPET_OK;
  }
  CUDA_TRY(cudaSetDevice(sc->dev.device));
  if (sc->dev.last_run_noalloc) CUDA_TRY(noalloc_guard_trips(trips));
  else CUDA_TRY(cudaMemcpy(trips, sc->dev.small, 8, cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

mcpet_status mcpet_write_outputs(const mcpet_scene* sc, const mcpet_tallies* host, const char* out_dir,
                                 int background_mode, double elapsed_s) {
  if (!sc || !host) return set_error(MCPET_ERR_ARG, "null argument");
  return write_outputs(sc, host, out_dir, background_mode, elapsed_s);
}

}  // extern "C"

/* ------------------------------------------------------------- probes */

namespace {
template <typename T>
struct DBuf {
  T* p = nullptr;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n, const void* src = nullptr) {
    cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1));
    if (e != cudaSuccess) return e;
    if (src) return cudaMemcpy(p, src, sizeof(T) * n, cudaMemcpyHostToDevice);
    return cudaMemset(p, 0, sizeof(T) * (n ? n : 1));
  }
};
mcpet_status probe_device() {
  int d = pick_device(-1);
  if (d < 0) return set_error(MCPET_ERR_CUDA, "no CUDA device available");
  CUDA_TRY(cudaSetDevice(d));
  return MCPET_OK;
}
}  // namespace

extern "C" {

mcpet_status mcpet_probe_rng(int n, int seed_input, const int64_t* stream_ids, int ndraw, int32_t* seeds_out,
                             float* draws, double* ddraws) {
  if (n <= 0 || !stream_ids || !seeds_out || ndraw < 0 || (ndraw > 0 && (!draws || !ddraws)))
    return set_error(MCPET_ERR_ARG, "invalid probe arguments");
  if (seed_input <= 0) return set_error(MCPET_ERR_ARG, "RANECU seed must be positive");
  mcpet_status s = probe_device();
  if (s != MCPET_OK) return s;
  TransportParams P;
  memset(&P, 0, sizeof(P));
  jump_tables(P.jump1, P.jump2);
  P.seed = seed_input;
  DBuf<int64_t> ids;
  DBuf<int2> sd;
  DBuf<float> f;
  DBuf<double> dd;
  CUDA_TRY(ids.alloc(n, stream_ids));
  CUDA_TRY(sd.alloc(n));
  CUDA_TRY(f.alloc((size_t)n * ndraw));
  CUDA_TRY(dd.alloc((size_t)n * ndraw));
  CUDA_TRY(launch_probe_rng(P, n, ids.p, ndraw, sd.p, f.p, dd.p, nullptr));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(seeds_out, sd.p, sizeof(int2) * n, cudaMemcpyDeviceToHost));
  if (ndraw > 0) {
    CUDA_TRY(cudaMemcpy(draws, f.p, sizeof(float) * n * ndraw, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(ddraws, dd.p, sizeof(double) * n * ndraw, cudaMemcpyDeviceToHost));
  }
  return MCPET_OK;
}

mcpet_status mcpet_probe_detector(const mcpet_scene* sc, int n, const float* e2, const float* e1, const float* pos2,
                                  const float* pos1, const float* dir2, const float* dir1, const int8_t* st2,
                                  const int8_t* st1, const int32_t* seeds, int32_t* out) {
  if (!sc || n <= 0 || !e2 || !e1 || !pos2 || !pos1 || !dir2 || !dir1 || !st2 || !st1 || !seeds || !out)
    return set_error(MCPET_ERR_ARG, "invalid probe arguments");
  mcpet_status s = probe_device();
  if (s != MCPET_OK) return s;
  TransportParams P;
  fill_params(sc, P);
  DBuf<float> de2, de1;
  DBuf<float3> dp2, dp1, dd2, dd1;
  DBuf<int8_t> ds2, ds1;
  DBuf<int2> dsd;
  DBuf<int> dout;
  CUDA_TRY(de2.alloc(n, e2));
  CUDA_TRY(de1.alloc(n, e1));
  CUDA_TRY(dp2.alloc(n, pos2));
  CUDA_TRY(dp1.alloc(n, pos1));
  CUDA_TRY(dd2.alloc(n, dir2));
  CUDA_TRY(dd1.alloc(n, dir1));
  CUDA_TRY(ds2.alloc(n, st2));
  CUDA_TRY(ds1.alloc(n, st1));
  CUDA_TRY(dsd.alloc(n, seeds));
  CUDA_TRY(dout.alloc((size_t)6 * n));
  CUDA_TRY(launch_probe_detector(P, n, de2.p, de1.p, dp2.p, dp1.p, dd2.p, dd1.p, ds2.p, ds1.p, dsd.p, dout.p,
                                 nullptr));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(out, dout.p, sizeof(int) * 6 * n, cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

mcpet_status mcpet_probe_compton(const mcpet_scene* sc, int n, const float* energy_in, const int32_t* mat,
                                 const int32_t* seeds_in, float* energy_out, double* costh_out, int32_t* seeds_out) {
  if (!sc || n <= 0 || !energy_in || !mat || !seeds_in || !energy_out || !costh_out || !seeds_out)
    return set_error(MCPET_ERR_ARG, "invalid probe arguments");
  for (int i = 0; i < n; ++i)
    if (mat[i] < 0 || mat[i] >= kMaxMaterials || !sc->material_loaded[mat[i]])
      return set_error(MCPET_ERR_ARG, "material %d not loaded", mat[i]);
  mcpet_status s = probe_device();
  if (s != MCPET_OK) return s;
  DBuf<ComptonTable> tab;
  DBuf<float> de;
  DBuf<int> dm;
  DBuf<int2> dsd;
  DBuf<double> dc;
  CUDA_TRY(tab.alloc(1, &sc->compton));
  CUDA_TRY(de.alloc(n, energy_in));
  CUDA_TRY(dm.alloc(n, mat));
  CUDA_TRY(dsd.alloc(n, seeds_in));
  CUDA_TRY(dc.alloc(n));
  CUDA_TRY(launch_probe_compton(tab.p, n, de.p, dm.p, dsd.p, dc.p, nullptr));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(energy_out, de.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(costh_out, dc.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(seeds_out, dsd.p, sizeof(int2) * n, cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

mcpet_status mcpet_probe_rayleigh(const mcpet_scene* sc, int n, const float* energy_in, const int32_t* mat,
                                  const float* pmax, const int32_t* seeds_in, double* costh_out, int32_t* seeds_out) {
  if (!sc || n <= 0 || !energy_in || !mat || !pmax || !seeds_in || !costh_out || !seeds_out)
    return set_error(MCPET_ERR_ARG, "invalid probe arguments");
  for (int i = 0; i < n; ++i)
    if (mat[i] < 0 || mat[i] >= kMaxMaterials || !sc->material_loaded[mat[i]])
      return set_error(MCPET_ERR_ARG, "material %d not loaded", mat[i]);
  mcpet_status s = probe_device();
  if (s != MCPET_OK) return s;
  const size_t nr = (size_t)kMaxMaterials * kNpRayleigh;
  std::vector<float> ray(4 * nr);
  std::copy(sc->xco.begin(), sc->xco.end(), ray.begin());
  std::copy(sc->pco.begin(), sc->pco.end(), ray.begin() + nr);
  std::copy(sc->aco.begin(), sc->aco.end(), ray.begin() + 2 * nr);
  std::copy(sc->bco.begin(), sc->bco.end(), ray.begin() + 3 * nr);
  std::vector<uint8_t> r8(2 * nr);
  std::copy(sc->itl.begin(), sc->itl.end(), r8.begin());
  std::copy(sc->itu.begin(), sc->itu.end(), r8.begin() + nr);
  DBuf<float> dray, de, dp;
  DBuf<uint8_t> dr8;
  DBuf<int> dm;
  DBuf<int2> dsd;
  DBuf<double> dc;
  CUDA_TRY(dray.alloc(4 * nr, ray.data()));
  CUDA_TRY(dr8.alloc(2 * nr, r8.data()));
  CUDA_TRY(de.alloc(n, energy_in));
  CUDA_TRY(dm.alloc(n, mat));
  CUDA_TRY(dp.alloc(n, pmax));
  CUDA_TRY(dsd.alloc(n, seeds_in));
  CUDA_TRY(dc.alloc(n));
  RayleighRows R{dray.p, dray.p + nr, dray.p + 2 * nr, dray.p + 3 * nr, dr8.p, dr8.p + nr};
  CUDA_TRY(launch_probe_rayleigh(R, n, de.p, dm.p, dp.p, dsd.p, dc.p, nullptr));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(costh_out, dc.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(seeds_out, dsd.p, sizeof(int2) * n, cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

mcpet_status mcpet_probe_source(int nx, int ny, int nz, const float inv_voxel_size[3], int background_mode,
                                const int32_t* seeds_in, float* out, int32_t* seeds_out) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !inv_voxel_size || !seeds_in || !out || !seeds_out ||
      background_mode < 0 || background_mode > 3)
    return set_error(MCPET_ERR_ARG, "invalid probe arguments");
  mcpet_status s = probe_device();
  if (s != MCPET_OK) return s;
  TransportParams P;
  memset(&P, 0, sizeof(P));
  P.nx = nx;
  P.ny = ny;
  P.nz = nz;
  P.inv_vx = inv_voxel_size[0];
  P.inv_vy = inv_voxel_size[1];
  P.inv_vz = inv_voxel_size[2];
  P.n_voxels = (long long)nx * ny * nz;
  DBuf<int2> dsd;
  DBuf<float3> dout;
  CUDA_TRY(dsd.alloc(P.n_voxels, seeds_in));
  CUDA_TRY(dout.alloc(4 * P.n_voxels));
  CUDA_TRY(launch_probe_source(P, background_mode, dsd.p, dout.p, nullptr));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(out, dout.p, sizeof(float3) * 4 * P.n_voxels, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(seeds_out, dsd.p, sizeof(int2) * P.n_voxels, cudaMemcpyDeviceToHost));
  return MCPET_OK;
}

}  // extern "C"
