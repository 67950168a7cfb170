/* Input formats and output writers of the transport path.
 *
 * Reads the reference's sectioned input file, penEasy/MCGPU-PET voxel files
 * (plain or gzip) and PENELOPE-derived material tables (plain or gzip), and
 * builds the interpolation tables with the same floating-point steps as the
 * reference loader so the tables are bit-identical.  Writes the reference's
 * output files.  Errors are returned as statuses (the reference exit()s).
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <sys/time.h>
#include <zlib.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "mcpet_scene.h"

namespace mcpet {

namespace {

constexpr int kLine = 250;   /* line buffer of the reference readers */

/* Line reader with fgets semantics (at most kLine-1 characters, stops after
 * the newline) over plain or gzip-compressed files. */
class LineReader {
 public:
  explicit LineReader(const char* path) { f_ = gzopen(path, "rb"); }
  ~LineReader() {
    if (f_) gzclose(f_);
  }
  LineReader(const LineReader&) = delete;
  LineReader& operator=(const LineReader&) = delete;
  bool ok() const { return f_ != nullptr; }
  bool get(char* buf) { return gzgets(f_, buf, kLine) != nullptr; }
  bool eof() const { return gzeof(f_) != 0; }

 private:
  gzFile f_ = nullptr;
};

/* Next non-empty line with leading blanks and the trailing '#' comment
 * removed (the reference fgets_trimmed, MCGPU-PET.cu:1320-1350).  Returns
 * false at end of file (out is then empty). */
bool next_value_line(LineReader& r, char* out) {
  char line[kLine];
  bool got;
  int n = 0;
  out[0] = '\0';
  do {
    n = 0;
    got = r.get(line);
    if (got) {
      int a = 0;
      while (line[a] == ' ') a++;
      while (line[a] != '\n' && line[a] != '#' && line[a] != '\0') out[n++] = line[a++];
      out[n] = '\0';
    }
  } while (got && out[0] == '\0');
  out[n] = '\0';
  return got;
}

/* First blank-delimited word of a value line (the reference trim_name,
 * MCGPU-PET.cu:1292-1311). */
void first_word(const char* in, char* out, size_t cap) {
  size_t a = 0, b = 0;
  while (in[a] == ' ') a++;
  while (in[a] != ' ' && in[a] != '#' && in[a] != '\0' && in[a] != '\t' && in[a] != '\r' && b + 1 < cap)
    out[b++] = in[a++];
  out[b] = '\0';
}

bool seek_section(LineReader& r, const char* key) {
  char line[kLine];
  for (;;) {
    if (!r.get(line)) return false;
    if (strstr(line, key) != nullptr) return true;
  }
}

/* Skip lines until one holds key a (returns 1) or key b (returns 2); 0 at
 * the end of the file. */
int seek_either(LineReader& r, const char* a, const char* b) {
  char line[kLine];
  for (;;) {
    if (!r.get(line)) return 0;
    if (strstr(line, a) != nullptr) return 1;
    if (strstr(line, b) != nullptr) return 2;
  }
}

bool yes_answer(const char* s) {
  return strncmp("YE", s, 2) == 0 || strncmp("Ye", s, 2) == 0 || strncmp("ye", s, 2) == 0;
}
bool no_answer(const char* s) {
  return strncmp("NO", s, 2) == 0 || strncmp("No", s, 2) == 0 || strncmp("no", s, 2) == 0;
}

}  // namespace

thread_local std::string g_error;

mcpet_status set_error(mcpet_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return s;
}

/* NSEG, NSINOS, NBINS from the sinogram geometry (MCGPU-PET.cu:1176-1189):
 * NSEG = 2*(MRD/SPAN)+1 segments; NSINOS = NSEG*NZS minus SPAN+1 planes for
 * every segment after the first and 2*floor((a-2)/2)*SPAN more for segment
 * a >= 4, i.e. 2*SPAN*floor(n/2)*ceil(n/2) in total with n = NSEG-2. */
void derive_sinogram_sizes(mcpet_config* c) {
  c->n_segments = 2 * (c->max_ring_difference / c->span) + 1;
  long long nseg = c->n_segments;
  long long ns = nseg * c->n_z_slices;
  if (nseg > 1) ns -= (nseg - 1) * (long long)(c->span + 1);
  if (nseg > 2) {
    long long n = nseg - 2;
    ns -= 2LL * c->span * ((n / 2) * ((n + 1) / 2));
  }
  c->n_sinograms = (int)ns;
  c->n_bins = (long long)c->n_radial * c->n_angles * ns;
}

/* The reference's read_input (MCGPU-PET.cu:866-1280): sections are located
 * in a fixed order by their header text, then a fixed sequence of value
 * lines is read. */
mcpet_status parse_input(const char* in_path, mcpet_config* cfg) {
  if (!in_path || !cfg) return set_error(MCPET_ERR_ARG, "null argument");
  memset(cfg, 0, sizeof(*cfg));
  LineReader r(in_path);
  if (!r.ok()) return set_error(MCPET_ERR_IO, "input file not found or not readable: '%s'", in_path);
  char v[kLine];

  if (!seek_section(r, "SECTION SIMULATION CONFIG v.2016-07-05"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION SIMULATION CONFIG v.2016-07-05'");
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->seed);
  if (cfg->seed == 0) {   /* time-based seed, MCGPU-PET.cu:920-928 */
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    cfg->seed = (int)((tv.tv_sec / 1000) + (tv.tv_usec * 1000));
  }
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->gpu_id);
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->threads_per_block);
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->density_factor);

  if (!seek_section(r, "SECTION SOURCE PET SCAN v.2017-03-14"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION SOURCE PET SCAN v.2017-03-14'");
  double seconds = 0.0;
  next_value_line(r, v);
  sscanf(v, "%lf", &seconds);
  cfg->acquisition_time_ps = (unsigned long long)(seconds * 1.0e12 + 0.5);
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->mean_life);
  {
    int mat = 0;
    float act = 0.0f;
    for (int i = 0; i < MCPET_MAX_MATERIALS; ++i) {
      next_value_line(r, v);
      sscanf(v, "%d %f", &mat, &act);   /* a line that does not parse keeps the previous pair */
      if (mat < 1) break;
      if (mat > MCPET_MAX_MATERIALS)
        return set_error(MCPET_ERR_FORMAT, "activity table material %d above %d", mat, MCPET_MAX_MATERIALS);
      cfg->material_activity[mat - 1] = act;
    }
  }

  if (!seek_section(r, "SECTION PHASE SPACE FILE v.2016-07-05"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION PHASE SPACE FILE v.2016-07-05'");
  next_value_line(r, v);
  first_word(v, cfg->psf_file, sizeof(cfg->psf_file));
  next_value_line(r, v);
  sscanf(v, "%f %f %f %f %f", &cfg->detector_center[0], &cfg->detector_center[1], &cfg->detector_center[2],
         &cfg->detector_height, &cfg->detector_radius);
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->psf_size);
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->tally_type);
  if (cfg->tally_type < 0 || cfg->tally_type > 2) cfg->tally_type = 0;
  next_value_line(r, v);
  sscanf(v, "%d", &cfg->tally_psf_sinogram);
  if (cfg->tally_psf_sinogram < 0 || cfg->tally_psf_sinogram > 2) cfg->tally_psf_sinogram = 0;

  {
    char line[kLine];
    bool found = false;
    while (r.get(line)) {
      if (strstr(line, "SECTION DOSE DEPOSITION v.2011-02-18") != nullptr)
        return set_error(MCPET_ERR_FORMAT,
                         "input file uses the old 'SECTION DOSE DEPOSITION v.2011-02-18'; update it to "
                         "v.2012-12-12");
      if (strstr(line, "SECTION DOSE DEPOSITION v.2012-12-12") != nullptr) {
        found = true;
        break;
      }
    }
    if (!found) return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION DOSE DEPOSITION v.2012-12-12'");
  }
  next_value_line(r, v);
  if (yes_answer(v)) cfg->tally_material_dose = 1;
  else if (no_answer(v)) cfg->tally_material_dose = 0;
  else return set_error(MCPET_ERR_FORMAT, "answer YES or NO to 'TALLY MATERIAL DOSE' (got '%s')", v);
  next_value_line(r, v);
  if (yes_answer(v)) {
    cfg->tally_voxel_dose = 1;
    next_value_line(r, v);
    first_word(v, cfg->dose_file, sizeof(cfg->dose_file));
    for (int k = 0; k < 3; ++k) {
      next_value_line(r, v);
      sscanf(v, "%hd %hd", &cfg->dose_roi[2 * k], &cfg->dose_roi[2 * k + 1]);
      cfg->dose_roi[2 * k] -= 1;
      cfg->dose_roi[2 * k + 1] -= 1;
    }
    const short* q = cfg->dose_roi;
    if (q[0] > q[1] || q[2] > q[3] || q[4] > q[5] || q[0] < 0 || q[2] < 0 || q[4] < 0)
      return set_error(MCPET_ERR_FORMAT, "invalid dose region of interest");
  } else if (no_answer(v)) {
    cfg->tally_voxel_dose = 0;
    for (int k = 0; k < 3; ++k) {
      cfg->dose_roi[2 * k] = (short)32500;
      cfg->dose_roi[2 * k + 1] = (short)-32500;
    }
  } else {
    return set_error(MCPET_ERR_FORMAT, "answer YES or NO to 'TALLY 3D VOXEL DOSE' (got '%s')", v);
  }

  if (!seek_section(r, "SECTION ENERGY PARAMETERS v.2019-04-25"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION ENERGY PARAMETERS v.2019-04-25'");
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->energy_resolution);
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->energy_window_low);
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->energy_window_high);

  if (!seek_section(r, "SECTION SINOGRAM PARAMETERS v.2019-04-25"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION SINOGRAM PARAMETERS v.2019-04-25'");
  next_value_line(r, v);
  sscanf(v, "%f", &cfg->fov_z);
  int* ints[] = {&cfg->n_rows, &cfg->n_crystals, &cfg->n_angles, &cfg->n_radial, &cfg->n_z_slices,
                 &cfg->image_res, &cfg->n_energy_bins, &cfg->max_ring_difference, &cfg->span};
  for (int* p : ints) {
    next_value_line(r, v);
    sscanf(v, "%d", p);
  }
  if (cfg->span <= 0) return set_error(MCPET_ERR_FORMAT, "SPAN must be positive (got %d)", cfg->span);
  derive_sinogram_sizes(cfg);

  /* optional prompt-gamma section before the voxel-file section */
  cfg->prompt_gamma_energy = 0.0f;
  cfg->prompt_gamma_yield = 0.0f;
  const int found = seek_either(r, "SECTION PROMPT GAMMA EMISSION v.2026-12-01",
                                "SECTION VOXELIZED GEOMETRY FILE v.2009-11-30");
  if (found == 1) {
    next_value_line(r, v);
    if (sscanf(v, "%f", &cfg->prompt_gamma_energy) != 1)
      return set_error(MCPET_ERR_FORMAT, "prompt gamma energy (eV) expected, got '%s'", v);
    next_value_line(r, v);
    if (sscanf(v, "%f", &cfg->prompt_gamma_yield) != 1)
      return set_error(MCPET_ERR_FORMAT, "prompt gamma yield per decay expected, got '%s'", v);
    if (!(cfg->prompt_gamma_energy >= 0.0f) || (cfg->prompt_gamma_energy > 0.0f &&
                                                !(cfg->prompt_gamma_yield > 0.0f && cfg->prompt_gamma_yield <= 1.0f)))
      return set_error(MCPET_ERR_FORMAT, "prompt gamma: energy %g eV must be >= 0 and the yield %g in (0, 1]",
                       cfg->prompt_gamma_energy, cfg->prompt_gamma_yield);
    if (!seek_section(r, "SECTION VOXELIZED GEOMETRY FILE v.2009-11-30"))
      return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION VOXELIZED GEOMETRY FILE v.2009-11-30'");
  } else if (found != 2) {
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION VOXELIZED GEOMETRY FILE v.2009-11-30'");
  }
  next_value_line(r, v);
  first_word(v, cfg->voxel_file, sizeof(cfg->voxel_file));

  if (!seek_section(r, "SECTION MATERIAL"))
    return set_error(MCPET_ERR_FORMAT, "input file lacks 'SECTION MATERIAL FILE LIST'");
  for (int i = 0; i < MCPET_MAX_MATERIALS; ++i) {
    if (!next_value_line(r, v)) cfg->material_files[i][0] = '\0';   /* list may end early */
    else first_word(v, cfg->material_files[i], sizeof(cfg->material_files[i]));
  }
  return MCPET_OK;
}

/* ---------------------------------------------------------------- voxels */

static void phantom_geometry(mcpet_scene* sc, int nx, int ny, int nz, const float vs[3]) {
  sc->nx = nx;
  sc->ny = ny;
  sc->nz = nz;
  for (int k = 0; k < 3; ++k) sc->voxel_size[k] = vs[k];
  sc->bbox[0] = nx * vs[0];
  sc->bbox[1] = ny * vs[1];
  sc->bbox[2] = nz * vs[2];
  for (int k = 0; k < 3; ++k) sc->inv_voxel_size[k] = 1.0f / vs[k];
  for (int m = 0; m < kMaxMaterials; ++m) sc->density_max[m] = -999.0f;
}

static mcpet_status check_voxel(mcpet_scene* sc, long long idx, int material, float density) {
  if (material > kMaxMaterials)
    return set_error(MCPET_ERR_FORMAT, "voxel material number too high: #mat=%d, MAX_MATERIALS=%d, voxel %lld",
                     material, kMaxMaterials, idx + 1);
  if (material < 1)
    return set_error(MCPET_ERR_FORMAT, "voxel material number can not be zero or negative: #mat=%d, voxel %lld",
                     material, idx + 1);
  if (density < 1.0e-9f)
    return set_error(MCPET_ERR_FORMAT, "voxel density can not be 0 or negative: #mat=%d, density=%f, voxel %lld",
                     material, density, idx + 1);
  if (density > sc->density_max[material - 1]) sc->density_max[material - 1] = density;
  return MCPET_OK;
}

/* The reference load_voxels (MCGPU-PET.cu:1381-1533): header with the grid
 * and voxel size, then one "material density activity" line per voxel, x
 * fastest, blank and '#' lines skipped (a line is skipped when its first or
 * second character is a newline or '#').  Unlike the reference, a missing or
 * malformed voxel line is an error (the reference repeats the previous line at
 * end of file and leaves the row unset on a short line). */
mcpet_status load_phantom_file(const char* path, float density_factor, mcpet_scene* sc) {
  LineReader r(path);
  if (!r.ok()) return set_error(MCPET_ERR_IO, "voxel file '%s' does not exist or is not readable", path);
  char line[kLine];
  if (!seek_section(r, "[SECTION VOXELS"))
    return set_error(MCPET_ERR_FORMAT, "voxel file lacks '[SECTION VOXELS HEADER'");
  int n[3] = {0, 0, 0};
  float vs[3] = {0, 0, 0};
  if (!r.get(line) || sscanf(line, "%d %d %d", &n[0], &n[1], &n[2]) != 3)
    return set_error(MCPET_ERR_FORMAT, "voxel file: cannot read the number of voxels");
  if (!r.get(line) || sscanf(line, "%f %f %f", &vs[0], &vs[1], &vs[2]) != 3)
    return set_error(MCPET_ERR_FORMAT, "voxel file: cannot read the voxel size");
  if (!seek_section(r, "[END OF VXH SECTION"))
    return set_error(MCPET_ERR_FORMAT, "voxel file lacks '[END OF VXH SECTION]'");
  if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0 || !(vs[0] > 0) || !(vs[1] > 0) || !(vs[2] > 0))
    return set_error(MCPET_ERR_FORMAT, "voxel file: invalid grid %d x %d x %d / size %g x %g x %g", n[0], n[1],
                     n[2], vs[0], vs[1], vs[2]);
  long long nv = (long long)n[0] * n[1] * n[2];
  if (nv >= (1LL << 31)) return set_error(MCPET_ERR_LIMIT, "phantom has %lld voxels (limit 2^31-1)", nv);
  phantom_geometry(sc, n[0], n[1], n[2], vs);
  sc->mat0.assign(nv, 0);
  sc->rho.assign(nv, 0.f);
  sc->activity.assign(nv, 0.f);
  for (long long i = 0; i < nv; ++i) {
    do {
      if (!r.get(line))
        return set_error(MCPET_ERR_FORMAT, "voxel file ended after %lld of %lld voxels", i, nv);
    } while (line[0] == '\n' || line[1] == '\n' || line[0] == '#' || line[1] == '#');
    int material = 0;
    float density = 0.f, act = 0.f;
    int items = sscanf(line, "%d %f %f", &material, &density, &act);
    if (items != 3)
      return set_error(MCPET_ERR_FORMAT, "voxel file: expecting 3 items per voxel (material, density, activity), "
                       "read %d at voxel %lld", items, i + 1);
    density *= density_factor;
    mcpet_status s = check_voxel(sc, i, material, density);
    if (s != MCPET_OK) return s;
    sc->mat0[i] = material - 1;
    sc->rho[i] = density;
    sc->activity[i] = act;
  }
  return MCPET_OK;
}

mcpet_status set_phantom_arrays(int nx, int ny, int nz, const float vs[3], const int32_t* material,
                                const float* density, const float* activity, float density_factor,
                                mcpet_scene* sc) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !vs || !(vs[0] > 0) || !(vs[1] > 0) || !(vs[2] > 0) || !material ||
      !density || !activity)
    return set_error(MCPET_ERR_ARG, "invalid phantom arrays");
  long long nv = (long long)nx * ny * nz;
  if (nv >= (1LL << 31)) return set_error(MCPET_ERR_LIMIT, "phantom has %lld voxels (limit 2^31-1)", nv);
  phantom_geometry(sc, nx, ny, nz, vs);
  sc->mat0.assign(nv, 0);
  sc->rho.assign(nv, 0.f);
  sc->activity.assign(activity, activity + nv);
  for (long long i = 0; i < nv; ++i) {
    float d = density[i] * density_factor;
    mcpet_status s = check_voxel(sc, i, material[i], d);
    if (s != MCPET_OK) return s;
    sc->mat0[i] = material[i] - 1;
    sc->rho[i] = d;
  }
  return MCPET_OK;
}

/* ------------------------------------------------------------- materials */

/* The reference load_material (MCGPU-PET.cu:1565-1831).  Per material: the
 * nominal density, N energy rows of (E, mfp Rayleigh, Compton, photoelectric,
 * total, Rayleigh pmax) with a constant energy step, 128 RITA rows and the
 * Compton shells.  Tables built with the reference's arithmetic:
 *   a = 1/(mfp*rho_nominal) per row (double, stored float),
 *   b = (a[i+1]-a[i])/dE (float difference, double quotient), last row
 *       repeats the previous slope,
 *   a -= (e0 + i dE) b  so that value = a + E b,
 *   majorant mfp = min over materials of mfp_total*rho_nominal/rho_max,
 *       with its slope and shift computed the same way.
 * Materials absent from the phantom are skipped, except the first slot,
 * which sets the table size. */
mcpet_status load_materials(mcpet_scene* sc) {
  const mcpet_config& cfg = sc->cfg;
  for (int m = 0; m < kMaxMaterials; ++m) {
    sc->density_nominal[m] = -1.0f;
    sc->material_loaded[m] = false;
    sc->compton.noscco[m] = 0;
  }
  memset(sc->compton.fco, 0, sizeof(sc->compton.fco));
  memset(sc->compton.uico, 0, sizeof(sc->compton.uico));
  memset(sc->compton.fj0, 0, sizeof(sc->compton.fj0));
  sc->xco.assign(kMaxMaterials * kNpRayleigh, 0.f);
  sc->pco.assign(kMaxMaterials * kNpRayleigh, 0.f);
  sc->aco.assign(kMaxMaterials * kNpRayleigh, 0.f);
  sc->bco.assign(kMaxMaterials * kNpRayleigh, 0.f);
  sc->itl.assign(kMaxMaterials * kNpRayleigh, 0);
  sc->itu.assign(kMaxMaterials * kNpRayleigh, 0);
  if (cfg.material_files[0][0] == '\0')
    return set_error(MCPET_ERR_FORMAT, "the first material file slot is empty (it defines the table size)");

  int num_values = 0;
  double delta_e = -99999.0;
  char line[kLine];
  for (int mat = 0; mat < kMaxMaterials; ++mat) {
    const char* fname = cfg.material_files[mat];
    if (fname[0] == '\0' || fname[0] == '\n') continue;
    LineReader r(fname);
    if (!r.ok()) return set_error(MCPET_ERR_IO, "material file %d '%s' does not exist", mat + 1, fname);
    if (!seek_section(r, "[NOMINAL DENSITY"))
      return set_error(MCPET_ERR_FORMAT, "material file '%s' lacks '[NOMINAL DENSITY'", fname);
    if (!r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    sscanf(line, "# %f", &sc->density_nominal[mat]);
    if (!(sc->density_max[mat] > 0)) {
      if (mat == 0) sc->density_max[mat] = 0.01f * sc->density_nominal[mat];
      else continue;   /* material not present in the phantom */
    }
    int n_in = 0;
    if (!r.get(line) || !r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    sscanf(line, "# %d", &n_in);
    if (mat == 0) {
      num_values = n_in;
      if (n_in > kMaxEnergyBins)
        return set_error(MCPET_ERR_LIMIT, "too many energy bins (%d > %d)", n_in, kMaxEnergyBins);
      if (n_in < 2) return set_error(MCPET_ERR_FORMAT, "material file '%s': %d energy rows", fname, n_in);
      sc->n_e = n_in;
      sc->woodcock.assign(2 * (size_t)n_in, 0.f);
      sc->mfp_a.assign(3 * (size_t)n_in * kMaxMaterials, 0.f);
      sc->mfp_b.assign(3 * (size_t)n_in * kMaxMaterials, 0.f);
      sc->pmax.assign((size_t)n_in * kMaxMaterials, 0.f);
      for (int i = 0; i < n_in; ++i) sc->woodcock[2 * i] = 99999999.99f;
    } else if (n_in != num_values) {
      return set_error(MCPET_ERR_FORMAT, "incorrect number of energy values in material '%s': input=%d, expected=%d",
                       fname, n_in, num_values);
    }
    if (!r.get(line) || !r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    float* A = sc->mfp_a.data();
    float* B = sc->mfp_b.data();
    float* W = sc->woodcock.data();
    double e_last = -1.0;
    for (int i = 0; i < num_values; ++i) {
      double e, ray, comp, photo, total, pmx;
      if (!r.get(line) || sscanf(line, "  %le  %le  %le  %le  %le  %le", &e, &ray, &comp, &photo, &total, &pmx) != 6)
        return set_error(MCPET_ERR_FORMAT, "material file '%s': bad mean free path row %d", fname, i + 1);
      float maj = total * (sc->density_nominal[mat]) / (sc->density_max[mat]);
      if (maj < W[2 * i]) W[2 * i] = maj;
      size_t bin = (size_t)i * kMaxMaterials + mat;
      A[3 * bin + 0] = 1.0 / (total * sc->density_nominal[mat]);
      A[3 * bin + 1] = 1.0 / (comp * sc->density_nominal[mat]);
      A[3 * bin + 2] = 1.0 / (ray * sc->density_nominal[mat]);
      sc->pmax[bin] = pmx;
      if (i == 0 && mat == 0) sc->e0 = e;
      if (i == 0) {
        if (fabs(e - sc->e0) > 1.0e-9)
          return set_error(MCPET_ERR_FORMAT, "incorrect first energy in material '%s': input=%f, expected=%f",
                           fname, e, (double)sc->e0);
      } else if (i == 1) {
        delta_e = e - e_last;
      } else if (((fabs((e - e_last) - delta_e)) / delta_e) > 0.001) {
        return set_error(MCPET_ERR_FORMAT, "the energy step between mean free path values is not constant "
                         "(row %d of '%s')", i + 1, fname);
      }
      e_last = e;
    }
    sc->ide = 1.0f / delta_e;
    for (int i = 0; i < num_values - 1; ++i) {
      size_t bin = (size_t)i * kMaxMaterials + mat;
      for (int c = 0; c < 3; ++c) B[3 * bin + c] = (A[3 * (bin + kMaxMaterials) + c] - A[3 * bin + c]) / delta_e;
    }
    {
      size_t last = (size_t)(num_values - 1) * kMaxMaterials + mat, prev = last - kMaxMaterials;
      for (int c = 0; c < 3; ++c) B[3 * last + c] = B[3 * prev + c];
    }
    for (int i = 0; i < num_values; ++i) {
      double e = sc->e0 + i * delta_e;
      size_t bin = (size_t)i * kMaxMaterials + mat;
      for (int c = 0; c < 3; ++c) A[3 * bin + c] = A[3 * bin + c] - e * B[3 * bin + c];
    }

    /* Rayleigh RITA rows */
    bool found = false;
    while (r.get(line)) {
      if (r.eof()) break;
      if (strstr(line, "[DATA VALUES") != nullptr) {
        found = true;
        break;
      }
    }
    if (!found) return set_error(MCPET_ERR_FORMAT, "Rayleigh data '[DATA VALUES' not found in '%s'", fname);
    int nray = 0;
    if (!r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    sscanf(line, "# %d", &nray);
    if (nray != kNpRayleigh)
      return set_error(MCPET_ERR_FORMAT, "%d Rayleigh sampling values in '%s' (expected %d)", nray, fname,
                       kNpRayleigh);
    if (!r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    for (int i = 0; i < kNpRayleigh; ++i) {
      int b = kNpRayleigh * mat + i, lo = 0, hi = 0;
      if (!r.get(line) || sscanf(line, "  %e  %e  %e  %e  %d  %d", &sc->xco[b], &sc->pco[b], &sc->aco[b],
                                 &sc->bco[b], &lo, &hi) != 6)
        return set_error(MCPET_ERR_FORMAT, "material file '%s': bad Rayleigh row %d", fname, i + 1);
      if (lo < 1 || hi < 1 || lo > kNpRayleigh || hi > kNpRayleigh)
        return set_error(MCPET_ERR_FORMAT, "material file '%s': Rayleigh interval index out of range", fname);
      sc->itl[b] = (uint8_t)lo;
      sc->itu[b] = (uint8_t)hi;
    }

    /* Compton shells */
    found = false;
    while (r.get(line)) {
      if (r.eof()) break;
      if (strstr(line, "[NUMBER OF SHELLS") != nullptr) {
        found = true;
        break;
      }
    }
    if (!found) return set_error(MCPET_ERR_FORMAT, "Compton data '[NUMBER OF SHELLS' not found in '%s'", fname);
    int nsh = 0;
    if (!r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    sscanf(line, "# %d", &nsh);
    if (nsh > kMaxShells || nsh < 1)
      return set_error(MCPET_ERR_FORMAT, "%d Compton shells in '%s' (1..%d allowed)", nsh, fname, kMaxShells);
    sc->compton.noscco[mat] = nsh;
    if (!r.get(line)) return set_error(MCPET_ERR_FORMAT, "material file '%s' truncated", fname);
    for (int i = 0; i < nsh; ++i) {
      int b = mat + i * kMaxMaterials, kz = 0, ks = 0;
      if (!r.get(line) || sscanf(line, " %e  %e  %e  %d  %d", &sc->compton.fco[b], &sc->compton.uico[b],
                                 &sc->compton.fj0[b], &kz, &ks) != 5)
        return set_error(MCPET_ERR_FORMAT, "material file '%s': bad Compton shell row %d", fname, i + 1);
    }
    sc->material_loaded[mat] = true;
  }
  sc->delta_e = delta_e;

  /* majorant slope and shift (the last row repeats the previous slope) */
  float* W = sc->woodcock.data();
  for (int i = 0; i < num_values - 1; ++i) W[2 * i + 1] = (W[2 * (i + 1)] - W[2 * i]) / delta_e;
  W[2 * (num_values - 1) + 1] = W[2 * (num_values - 2) + 1];
  for (int i = 0; i < num_values; ++i) W[2 * i] = W[2 * i] - (sc->e0 + i * delta_e) * W[2 * i + 1];
  return MCPET_OK;
}

/* Voxels of the dose ROI (0 when the voxel dose tally is off). */
long long dose_voxels(const mcpet_config& c) {
  const short* r = c.dose_roi;
  if (!c.tally_voxel_dose || r[1] < 0) return 0;
  return (long long)(r[1] - r[0] + 1) * (long long)(r[3] - r[2] + 1) * (long long)(r[5] - r[4] + 1);
}

/* Checks after loading (MCGPU-PET.cu:316-351) and palette compression. */
mcpet_status finalize_scene(mcpet_scene* sc) {
  mcpet_config& cfg = sc->cfg;
  if (cfg.tally_voxel_dose) {
    /* the ROI's upper corner is clipped to the phantom (load_voxels, MCGPU-PET.cu:1444-1452) */
    short* r = cfg.dose_roi;
    r[1] = (short)std::min<int>(sc->nx - 1, r[1]);
    r[3] = (short)std::min<int>(sc->ny - 1, r[3]);
    r[5] = (short)std::min<int>(sc->nz - 1, r[5]);
    if (r[0] > r[1] || r[2] > r[3] || r[4] > r[5])
      return set_error(MCPET_ERR_FORMAT, "the dose region of interest lies outside the phantom");
  }
  for (long long i = 0; i < (long long)sc->mat0.size(); ++i)
    if (!sc->material_loaded[sc->mat0[i]])
      return set_error(MCPET_ERR_FORMAT, "voxel %lld uses material %d which has no material file", i + 1,
                       sc->mat0[i] + 1);
  if (cfg.detector_radius < 0.0f) {
    cfg.detector_center[0] = sc->bbox[0] * 0.5f;
    cfg.detector_center[1] = sc->bbox[1] * 0.5f;
    cfg.detector_center[2] = sc->bbox[2] * 0.5f;
    cfg.detector_radius = -cfg.detector_radius;
    cfg.detector_auto_center = 1;
  }
  /* the tables must reach the annihilation energy (MCGPU-PET.cu:344-351) */
  if (510998.95f > (sc->e0 + (sc->n_e - 1) / sc->ide))
    return set_error(MCPET_ERR_FORMAT, "the material files do not have data up to %f keV", 510998.95f * 1e-3);

  /* palette of distinct (material, density) pairs; voxels keep an index */
  std::unordered_map<uint64_t, uint32_t> seen;
  sc->palette.clear();
  sc->voxel_key.resize(sc->mat0.size());
  for (size_t i = 0; i < sc->mat0.size(); ++i) {
    uint32_t bits;
    memcpy(&bits, &sc->rho[i], 4);
    uint64_t key = ((uint64_t)(uint32_t)sc->mat0[i] << 32) | bits;
    auto it = seen.find(key);
    if (it == seen.end()) {
      it = seen.emplace(key, (uint32_t)sc->palette.size()).first;
      sc->palette.push_back(PaletteEntry{sc->mat0[i], sc->rho[i]});
    }
    sc->voxel_key[i] = it->second;
  }
  return MCPET_OK;
}

/* --------------------------------------------------------------- writers */

static mcpet_status write_gz(const std::string& path, const void* data, size_t bytes) {
  gzFile f = gzopen(path.c_str(), "wb");
  if (!f) return set_error(MCPET_ERR_IO, "cannot write '%s'", path.c_str());
  const char* p = static_cast<const char*>(data);
  while (bytes > 0) {
    unsigned chunk = bytes > (1u << 30) ? (1u << 30) : (unsigned)bytes;
    if (gzwrite(f, p, chunk) != (int)chunk) {
      gzclose(f);
      return set_error(MCPET_ERR_IO, "short write to '%s'", path.c_str());
    }
    p += chunk;
    bytes -= chunk;
  }
  if (gzclose(f) != Z_OK) return set_error(MCPET_ERR_IO, "cannot close '%s'", path.c_str());
  return MCPET_OK;
}

static std::string join(const char* dir, const char* name) {
  if (!dir || !dir[0]) return name;
  std::string d(dir);
  if (d.back() != '/') d += '/';
  return d + name;
}

/* PSF record field access on the packed 44-byte layout. */
struct PsfView {
  const unsigned char* base;
  unsigned long long t(long long i) const { unsigned long long v; memcpy(&v, base + 44 * i, 8); return v; }
  float f(long long i, int off) const { float v; memcpy(&v, base + 44 * i + off, 4); return v; }
  int n(long long i, int off) const { int v; memcpy(&v, base + 44 * i + off, 4); return v; }
  short s(long long i, int off) const { short v; memcpy(&v, base + 44 * i + off, 2); return v; }
};

/* Materials dose report (report_materials_dose, MCGPU-PET.cu:2664-2725): per
 * defined material, dose = sum(Edep)/N/mass with mass = sum over the
 * phantom's voxels of density x voxel volume, and its 2-sigma uncertainty
 * from sum(Edep^2). */
std::string format_materials_dose(const mcpet_scene* sc, const unsigned long long* md, unsigned long long n_hist) {
  const double vol = 1.0 / ((double)sc->inv_voxel_size[0] * (double)sc->inv_voxel_size[1] *
                            (double)sc->inv_voxel_size[2]);
  double mass[kMaxMaterials] = {0};
  for (size_t v = 0; v < sc->mat0.size(); ++v) mass[sc->mat0[v]] += (double)sc->rho[v] * vol;
  const double inv_n = 1.0 / (double)(n_hist ? n_hist : 1);
  std::string out;
  char line[1024];
  snprintf(line, sizeof(line), "\n          *** MATERIALS TOTAL DOSE TALLY REPORT ***\n\n"
           "              Total number of simulated x rays: %llu\n\n"
           "\t [MAT]  [DOSE eV/g/hist]  [2*std_dev]  [Rel_error 2*std_dev, %%]  [E_dep eV/hist]  [DOSE mGy]  "
           "[Material mass g]  [Material file name]\n", n_hist);
  out += line;
  for (int m = 0; m < kMaxMaterials; ++m) {
    if (sc->density_nominal[m] < 0.0f) break;
    const char* name = sc->cfg.material_files[m];
    const char* slash = strrchr(name, '/');
    if (slash) name = slash + 1;
    const double edep = (double)md[2 * m] * inv_n;
    double sd = sqrt(((double)md[2 * m + 1] * inv_n - edep * edep) * inv_n);
    const double rel = edep > 0.0 ? sd / edep : 0.0;
    const double m_g = std::max(mass[m], 0.00001);
    snprintf(line, sizeof(line), "\t%d\t%.5lf\t\t%.5lf\t\t%.2lf\t\t%.5lf\t\t%.5lf\t\t%.5lf\t\t%s\n", m + 1, edep / m_g,
             2.0 * sd / m_g, 200.0 * rel, edep, (double)md[2 * m] / m_g * (1.0e3 / 6.2415e15), mass[m], name);
    out += line;
  }
  return out;
}

/* Voxel dose in the ROI (report_voxels_dose, MCGPU-PET.cu:2389-2640): the
 * text file holds the central Z plane of the ROI (dose and 2 sigma, eV/g per
 * history; one blank line between Y rows), the .raw files the whole ROI as
 * 32-bit floats (dose; % relative error at 2 sigma), x fastest.  Voxels of
 * density below 0.1 g/cm^3 (air) report 0. */
static mcpet_status write_voxel_dose(const mcpet_scene* sc, const mcpet_tallies* t, const std::string& path,
                                     double elapsed_s) {
  const mcpet_config& c = sc->cfg;
  const short* r = c.dose_roi;
  const int dx = r[1] - r[0] + 1, dy = r[3] - r[2] + 1, dz = r[5] - r[4] + 1;
  const int zplane = (r[5] + r[4]) / 2 - r[4];
  const unsigned long long n_hist = t->total_histories ? *t->total_histories : 0ull;
  const double inv_n = 1.0 / (double)(n_hist ? n_hist : 1);
  const double vol = 1.0 / ((double)sc->inv_voxel_size[0] * (double)sc->inv_voxel_size[1] *
                            (double)sc->inv_voxel_size[2]);
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return set_error(MCPET_ERR_IO, "cannot write '%s'", path.c_str());
  const std::string pm = path + ".raw", ps = path + "_PercentRelError2sigma.raw";
  FILE* fm = fopen(pm.c_str(), "wb");
  FILE* fs = fopen(ps.c_str(), "wb");
  if (!fm || !fs) {
    fclose(f);
    if (fm) fclose(fm);
    if (fs) fclose(fs);
    return set_error(MCPET_ERR_IO, "cannot write '%s'", pm.c_str());
  }
  fprintf(f, "#\n#  3D voxel dose (photon KERMA: energy deposited by photon interactions in each voxel, no electron\n"
             "#  transport) in the region of interest; 32-bit float binaries: %s (dose) and %s (%% relative error\n"
             "#  at 2 standard deviations).  This text: the ROI plane z_coord = %d (z_coord in ROI = %d).\n#\n",
          pm.c_str(), ps.c_str(), zplane + r[4], zplane);
  fprintf(f, "#  Voxel size:  %lf x %lf x %lf = %lf cm^3\n", 1.0 / (double)sc->inv_voxel_size[0],
          1.0 / (double)sc->inv_voxel_size[1], 1.0 / (double)sc->inv_voxel_size[2], vol);
  fprintf(f, "#  Number of voxels in the reported region of interest (ROI) X, Y and Z:\n#      %d  %d  %d\n", dx, dy,
          dz);
  fprintf(f, "#  Coordinates of the ROI inside the voxel volume = X[%d,%d], Y[%d,%d], Z[%d,%d]\n", r[0] + 1, r[1] + 1,
          r[2] + 1, r[3] + 1, r[4] + 1, r[5] + 1);
  fprintf(f, "#  Voxel dose units: eV/g per history\n#\n#    [DOSE]   [2*standard_deviation]\n"
             "# =====================================\n");
  unsigned long long total = 0;
  long long k = 0;
  for (int z = 0; z < dz; ++z) {
    for (int y = 0; y < dy; ++y) {
      for (int x = 0; x < dx; ++x, ++k) {
        const size_t g = (size_t)(x + r[0]) + (size_t)(y + r[2]) * sc->nx + (size_t)(z + r[4]) * sc->nx * sc->ny;
        const double rho = sc->rho[g];
        unsigned long long e1 = t->voxel_dose[2 * k], e2 = t->voxel_dose[2 * k + 1];
        if (rho < 0.1) e1 = e2 = 0;
        const double inv_mass = 1.0 / (rho * vol);
        double dose = (double)e1 * inv_n;
        total += e1;
        double sd = ((double)e2 * inv_n - dose * dose) * inv_n * inv_mass;
        if (sd > 0.0) sd = sqrt(sd);
        dose *= inv_mass;
        if (z == zplane) fprintf(f, "%.6lf %.6lf\n", dose, 2.0 * sd);
        const float df = (float)dose;
        const float ef = dose > 0.0 ? 200.0f * (float)(sd / dose) : 0.0f;
        fwrite(&df, sizeof(float), 1, fm);
        fwrite(&ef, sizeof(float), 1, fs);
      }
      if (z == zplane) fprintf(f, "\n");
    }
    if (z == zplane) fprintf(f, "\n");
  }
  fprintf(f, "#   ****** DOSE REPORT: TOTAL SIMULATION PERFORMANCE ******\n");
  fprintf(f, "#       Total number of simulated x rays: %llu\n", n_hist);
  fprintf(f, "#       Total simulation time [s]:  %.2f\n", elapsed_s);
  fprintf(f, "\n#       Total energy absorved inside the dose ROI: %.5lf keV/hist\n\n",
          0.001 * (double)total * inv_n);
  fclose(f);
  fclose(fm);
  fclose(fs);
  return MCPET_OK;
}

mcpet_status write_outputs(const mcpet_scene* sc, const mcpet_tallies* t, const char* out_dir, int bg,
                           double elapsed_s) {
  const mcpet_config& c = sc->cfg;
  const size_t nb = (size_t)c.n_bins, nv = (size_t)sc->mat0.size();
  if (c.tally_psf_sinogram == 0 || c.tally_psf_sinogram == 2) {
    const char* names_std[4] = {"sinogram_Trues.raw.gz", "sinogram_Scatter.raw.gz", "image_Trues.raw.gz",
                                "image_Scatter.raw.gz"};
    const char* names_bg[4] = {"sinogram_BG_Trues.raw.gz", "sinogram_BG_Scatter.raw.gz", "BG_image_True.raw.gz",
                               "BG_image_Scatter.raw.gz"};
    const char** names = bg ? names_bg : names_std;
    const void* bufs[4] = {t->trues, t->scatter, t->image_trues, t->image_scatter};
    size_t sizes[4] = {nb * 4, nb * 4, nv * 4, nv * 4};
    for (int k = 0; k < 4; ++k) {
      if (!bufs[k]) continue;
      mcpet_status s = write_gz(join(out_dir, names[k]), bufs[k], sizes[k]);
      if (s != MCPET_OK) return s;
    }
  }
  if (t->spectrum) {
    std::string p = join(out_dir, "Energy_Sinogram_Spectrum.dat");
    FILE* f = fopen(p.c_str(), "w");
    if (!f) return set_error(MCPET_ERR_IO, "cannot write '%s'", p.c_str());
    fprintf(f, "# HISTOGRAM OF ENERGIES (keV) OF DETECTED COINCIDENCE PHOTONS (before energy window selection)\n");
    fprintf(f, "#     Energy bin [keV]     Counts\n");
    for (int i = 0; i < c.n_energy_bins; ++i) fprintf(f, "%10d  %10d \n", i, t->spectrum[i]);
    fclose(f);
  }
  if ((c.tally_psf_sinogram == 0 || c.tally_psf_sinogram == 1) && t->psf && t->psf_count) {
    long long n = *t->psf_count;
    if (n > t->psf_capacity) n = t->psf_capacity;
    if (n < 0) n = 0;
    std::string p = join(out_dir, c.psf_file);
    FILE* f = fopen(p.c_str(), "w");
    if (!f) return set_error(MCPET_ERR_IO, "cannot write '%s'", p.c_str());
    std::string pb = p + ".raw";
    FILE* fb = fopen(pb.c_str(), "w");
    if (!fb) {
      fclose(f);
      return set_error(MCPET_ERR_IO, "cannot write '%s'", pb.c_str());
    }
    unsigned long long hist = t->total_histories ? *t->total_histories : 0ull;
    fprintf(f, "# \n#  Phase space file (PSF) of photon pairs arriving at the ideal cylindrical detector.\n# \n");
    fprintf(f, "#        Number of detections in the PSF = %lld\n", n);
    fprintf(f, "#        Allocated PSF elements = %d\n", c.psf_size);
    fprintf(f, "#        PET acquistion time    = %lf s\n", c.acquisition_time_ps * 1.0e-12);
    fprintf(f, "#        mean life isotope      = %f\n", c.mean_life);
    fprintf(f, "#        PSF detector center    = (%.5f,%.5f,%.5f) cm\n", c.detector_center[0], c.detector_center[1],
            c.detector_center[2]);
    fprintf(f, "#        PSF detector height and radius = %.5f, %.5f cm\n", c.detector_height, c.detector_radius);
    fprintf(f, "#        Input voxel file       = %s\n# \n", c.voxel_file);
    fprintf(f, "#        Reporting only the 5000 first elements below in ASCII. Complete PSF available in binary "
               "form in the file %s\n", pb.c_str());
    fprintf(f, "#        Binary record (44 bytes): emission_time (ps) uint64, travel_time (ps) float, emission voxel "
               "int32, energy (eV) z (cm) phi (rad) vx vy vz float, index1 (scatter flag) index2 int16\n# \n");
    fprintf(f, "#  [emission_time (ps)]    [travel_time (ps)]    [emission voxel]  [energy (eV)]  [z (cm)]  [phi (rad)]"
               "  [vx]  [vy]  [vz]  [index1]  [index2]\n");
    fprintf(f, "# ========================================================================================================"
               "================================\n");
    PsfView v{static_cast<const unsigned char*>(t->psf)};
    for (long long i = 0; i < (n < 5000 ? n : 5000); ++i)
      fprintf(f, "%lld %f %d %f %f %f %f %f %f %d %d\n", (long long)v.t(i), v.f(i, 8), v.n(i, 12), v.f(i, 16),
              v.f(i, 20), v.f(i, 24), v.f(i, 28), v.f(i, 32), v.f(i, 36), (int)v.s(i, 40), (int)v.s(i, 42));
    fprintf(f, "\n#        (...)\n");
    if (n > 0 && fwrite(t->psf, 44, (size_t)n, fb) != (size_t)n) {
      fclose(f);
      fclose(fb);
      return set_error(MCPET_ERR_IO, "short write to '%s'", pb.c_str());
    }
    fprintf(f, "# \n#   *** Simulation REPORT: ***\n");
    fprintf(f, "#       Simulated x rays:    %lld\n", (long long)hist);
    fprintf(f, "#       Simulation time [s]: %.2f\n", elapsed_s);
    if (elapsed_s > 0.000001) fprintf(f, "#       Speed [x-rays/s]:    %.2f\n\n", ((double)hist) / elapsed_s);
    fclose(f);
    fclose(fb);
  }
  if (c.tally_voxel_dose && t->voxel_dose && dose_voxels(c) > 0) {
    mcpet_status s = write_voxel_dose(sc, t, join(out_dir, c.dose_file), elapsed_s);
    if (s != MCPET_OK) return s;
  }
  if (c.tally_material_dose && t->material_dose) {
    std::string p = join(out_dir, "materials_dose.txt");
    FILE* f = fopen(p.c_str(), "w");
    if (!f) return set_error(MCPET_ERR_IO, "cannot write '%s'", p.c_str());
    const std::string txt = format_materials_dose(sc, t->material_dose, t->total_histories ? *t->total_histories : 0);
    fputs(txt.c_str(), f);
    fclose(f);
  }
  return MCPET_OK;
}

}  // namespace mcpet
