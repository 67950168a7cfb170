/* CPU oracle of the MCGPU-PET photon-transport path -- TEST INFRASTRUCTURE.
 *
 * Plain C restatement of the reference algorithm, one function per reference
 * routine (citations are to the reference sources).  Only tests/, the smoke
 * check and the benchmark's CPU-baseline leg use it, as the checker.
 *
 * Arithmetic follows the reference's host-compilable form: libm calls where
 * the CUDA build calls fast-math intrinsics, and the #ifndef USING_CUDA branch
 * of GCOa (division instead of rsqrtf).  Built with -ffp-contract=off so no
 * multiply-add is fused; the same operations in the same order as the
 * reference compiled for the host, hence bit-identical to it.
 */
#define _GNU_SOURCE
#include "mcpet_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846
#define EPS_SRC 0.00015f
#define E_ANNIHILATION 510998.95f
#define PS_PER_CM (1.0 / 29979245800e-12)
#define NM ORC_MAX_MATERIALS

typedef struct { int x, y; } rng_t;
typedef struct { float x, y, z; } vec3;

/* ---------------------------------------------------------------- RANECU */

/* One draw of L'Ecuyer's combined generator (ranecu / ranecu_double,
 * MCGPU-PET_kernel.cu:1045-1083): two MLCGs advanced with Schrage's
 * factorisation, combined and scaled. */
static int ranecu_int(rng_t* s) {
  int k = s->x / 53668;
  s->x = 40014 * (s->x - k * 53668) - k * 12211;
  if (s->x < 0) s->x += 2147483563;
  k = s->y / 52774;
  s->y = 40692 * (s->y - k * 52774) - k * 3791;
  if (s->y < 0) s->y += 2147483399;
  int z = s->x - s->y;
  if (z < 1) z += 2147483562;
  return z;
}
static float ranecu(rng_t* s) { return (float)ranecu_int(s) * 4.65661305739e-10f; }
static double ranecu_double(rng_t* s) { return (double)ranecu_int(s) * 4.6566130573917692e-10; }

/* a^e mod m and (a*b) mod m in exact 64-bit arithmetic. */
static uint64_t mulmod64(uint64_t a, uint64_t b, uint64_t m) { return (a * b) % m; }
static uint64_t powmod64(uint64_t a, uint64_t e, uint64_t m) {
  uint64_t r = 1;
  a %= m;
  while (e) {
    if (e & 1) r = mulmod64(r, a, m);
    a = mulmod64(a, a, m);
    e >>= 1;
  }
  return r;
}

/* Stream start: the seed advanced (stream+1)*555555*256 draws
 * (init_PRNG, MCGPU-PET_kernel.cu:925-978). */
static rng_t rng_stream(int seed, uint64_t stream) {
  const uint64_t leap = (stream + 1) * (uint64_t)(555555 * 256);
  rng_t r;
  r.x = (int)mulmod64((uint64_t)seed % 2147483563u, powmod64(40014, leap, 2147483563u), 2147483563u);
  r.y = (int)mulmod64((uint64_t)seed % 2147483399u, powmod64(40692, leap, 2147483399u), 2147483399u);
  return r;
}

/* ------------------------------------------------------------- helpers */

static int fl(float x) { return (int)floorf(x); }   /* __float2int_rd */

static unsigned long long round_u64(double x) {       /* __double2ull_rn */
  double r = nearbyint(x);
  if (!(r == r) || r <= 0.0) return 0ull;
  if (r >= 18446744073709551616.0) return ~0ull;
  return (unsigned long long)r;
}

/* Voxel containing a point, -100 outside the box shrunk by EPS
 * (locate_voxel, MCGPU-PET_kernel.cu:1098-1124). */
static int locate(const orc_params* p, vec3 r) {
  if ((r.y < EPS_SRC) || (r.y > (p->bby - EPS_SRC)) || (r.x < EPS_SRC) || (r.x > (p->bbx - EPS_SRC)) ||
      (r.z < EPS_SRC) || (r.z > (p->bbz - EPS_SRC)))
    return -100;
  int ix = fl(r.x * p->inv_vx), iy = fl(r.y * p->inv_vy), iz = fl(r.z * p->inv_vz);
  return ix + iy * p->nx + iz * p->nx * p->ny;
}

/* ------------------------------------------------------------- source */

/* Isotropic direction (MCGPU-PET_kernel.cu:673-680, 712-719). */
static void isotropic(rng_t* s, vec3* d) {
  d->z = 1.0f - 2.0f * ranecu(s);
  float phi = 6.28318530716f * ranecu(s);
  float st = sqrtf(1.0f - d->z * d->z);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  d->y = st * sp;
  d->x = st * cp;
}

/* First annihilation photon: direction, then a uniform point in the voxel
 * (MCGPU-PET_kernel.cu:670-704). */
static void source_first(rng_t* s, const orc_params* p, int vx, int vy, int vz, vec3* pos, vec3* dir) {
  isotropic(s, dir);
  float u[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = ranecu(s);
    u[k] = (EPS_SRC > u[k] - EPS_SRC) ? EPS_SRC : u[k] - EPS_SRC;
  }
  pos->x = ((float)vx + u[0]) / p->inv_vx;
  pos->y = ((float)vy + u[1]) / p->inv_vy;
  pos->z = ((float)vz + u[2]) / p->inv_vz;
}

/* Second photon: opposite direction with Gaussian acolinearity (sigma
 * 0.21276 deg doubled), or isotropic in background mode
 * (MCGPU-PET_kernel.cu:709-766). */
static void source_second(rng_t* s, int background, vec3 d1, vec3* d) {
  if (background) {
    isotropic(s, d);
    return;
  }
  float phi2 = (float)((double)atan2f(d1.y, d1.x) + PI_D);
  float theta2 = (float)(PI_D - (double)acosf(d1.z));
  float v1 = ranecu(s);
  float v2 = ranecu(s);
  float theta_nc = (float)((2.0 * 0.21276 * PI_D / 180.0) * (double)sqrtf(-2.0f * logf(v2 + 1e-8f)) *
                           (double)cosf((float)((2.0 * PI_D) * (double)v1)));
  float phi_nc = (float)((2.0 * PI_D) * (double)ranecu(s));
  float st, ct, sp, cp, st1, ct1, sp1, cp1;
  sincosf(theta_nc, &st, &ct);
  sincosf(phi_nc, &sp, &cp);
  sincosf(theta2, &st1, &ct1);
  sincosf(phi2, &sp1, &cp1);
  float gx = cp * st, gy = sp * st, gz = ct;
  d->x = gx * ct1 * cp1 - gy * sp1 + gz * st1 * cp1;
  d->y = gx * ct1 * sp1 + gy * cp1 + gz * st1 * sp1;
  d->z = -gx * st1 + gz * ct1;
}

/* ------------------------------------------------------------- rotation */

/* PENELOPE DIRECT in double precision (rotate_double,
 * MCGPU-PET_kernel.cu:1160-1200). */
static void rotate(vec3* d, double costh, double phi) {
  double sinphi, cosphi;
  double dxy = d->x * d->x + d->y * d->y;
  sincos(phi, &sinphi, &cosphi);
  double norm = dxy + d->z * d->z;
  if (fabs(norm - 1.0) > 1.0e-14) {
    norm = 1.0 / sqrt(norm);
    d->x = norm * d->x;
    d->y = norm * d->y;
    d->z = norm * d->z;
    dxy = d->x * d->x + d->y * d->y;
  }
  if (dxy > 1.0e-28) {
    double sdt = sqrt((1.0 - costh * costh) / dxy);
    float xin = d->x;
    float yin = d->y;
    float zin = d->z;
    d->x = xin * costh + sdt * (xin * zin * cosphi - yin * sinphi);
    d->y = yin * costh + sdt * (yin * zin * cosphi + xin * sinphi);
    d->z = zin * costh - dxy * sdt * cosphi;
  } else {
    double sdt = sqrt(1.0 - costh * costh);
    d->y = sdt * sinphi;
    if (d->z > 0.0) {
      d->x = sdt * cosphi;
      d->z = costh;
    } else {
      d->x = -sdt * cosphi;
      d->z = -costh;
    }
  }
}

/* ------------------------------------------------------------- Rayleigh */

/* PENELOPE 2006 GRAa: RITA sampling of x^2 from the squared form factor,
 * rejection on (1+cos^2)/2 (MCGPU-PET_kernel.cu:1231-1296). */
static double rayleigh(rng_t* s, float energy, int mat, float pmax, const orc_tables* t) {
  const int base = mat * ORC_NP_RAYLEIGH;
  double xmax = ((double)energy) * 8.065535669099010e-5;
  double xlast = (double)t->xco[base + ORC_NP_RAYLEIGH - 1];
  double x2max = ((xmax * xmax) < xlast) ? (xmax * xmax) : xlast;
  double c;
  if (xmax < 0.01) {
    do {
      c = 1.0 - ranecu_double(s) * 2.0;
    } while (ranecu_double(s) > ((c * c + 1.0) * 0.5));
    return c;
  }
  for (;;) {
    double ru = ranecu_double(s) * (double)pmax;
    int itn = (int)(ru * (ORC_NP_RAYLEIGH - 1));
    int lo = t->itlco[itn + base], hi = t->ituco[itn + base];
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (ru > t->pco[mid - 1 + base]) lo = mid;
      else hi = mid;
    }
    int i = lo - 1 + base;
    double rr = ru - t->pco[i], xx;
    if (rr > 1e-16) {
      double dp = (double)(t->pco[i + 1] - t->pco[i]);
      float a = t->aco[i], b = t->bco[i], x0 = t->xco[i];
      xx = (double)x0 + (double)(a + 1.0f + b) * dp * rr / (dp * dp + (a * dp + b * rr) * rr) *
                            (double)(t->xco[i + 1] - x0);
    } else {
      xx = t->xco[i];
    }
    if (xx < x2max) {
      c = 1.0 - 2.0 * xx / x2max;
      if (ranecu_double(s) < ((c * c + 1.0) * 0.5)) return c;
    }
  }
}

/* ------------------------------------------------------------- Compton */

/* One-electron Compton profile term of shell i for the momentum pz
 * (host form of MCGPU-PET_kernel.cu:1372-1379). */
static float pz_of(float fj0, float aux, float u) {
  return fj0 * (aux - u * 510998.918f) / (sqrtf(aux + aux + u * u) * 510998.918f);
}

/* PENELOPE 2006 GCOa: relativistic impulse approximation with analytical
 * profiles (MCGPU-PET_kernel.cu:1335-1563).  Updates the energy, returns
 * cos(theta). */
static double compton(rng_t* s, float* energy, int mat, const orc_tables* t) {
  const float E = *energy;
  const int nsh = t->noscco[mat];
  float rn[ORC_MAX_SHELLS];
  memset(rn, 0, sizeof(rn));
  float ek = E * 1.956951306108245e-6f;
  float ek2 = ek * 2.f + 1.f;
  float ek3 = ek * ek;
  float taumin = 1.f / ek2;
  float a1 = logf(ek2);

  float s0 = 0.0f;
  for (int i = 0; i < nsh; ++i) {
    float u = t->uico[mat + i * NM];
    if (u < E) {
      float aux = E * (E - u) * 2.f;
      float pz = pz_of(t->fj0[mat + i * NM], aux, u);
      float q;
      if (pz > 0.0f) q = (0.707106781186545f + pz * 1.4142135623731f) * (0.707106781186545f + pz * 1.4142135623731f);
      else q = (0.707106781186545f - pz * 1.4142135623731f) * (0.707106781186545f - pz * 1.4142135623731f);
      q = 0.5f * expf(0.5f - q);
      if (pz > 0.0f) q = 1.0f - q;
      s0 += t->fco[mat + i * NM] * q;
    }
  }

  float tau, sv;
  double cdt1;
  for (;;) {
    if (ranecu(s) * (a1 + 2. * ek * (ek + 1.f) * taumin * taumin) < a1) tau = powf(taumin, ranecu(s));
    else tau = sqrtf(1.f + ranecu(s) * (taumin * taumin - 1.f));
    cdt1 = (double)(1.f - tau) / (((double)tau) * ((double)E) * 1.956951306108245e-6);
    if (cdt1 > 2.0) cdt1 = 1.99999999;
    sv = 0.0f;
    for (int i = 0; i < nsh; ++i) {
      float u = t->uico[mat + i * NM];
      if (u < E) {
        float aux = E * (E - u) * ((float)cdt1);
        float pz = ((aux > 1.0e-12f) || (u > 1.0e-12f)) ? pz_of(t->fj0[mat + i * NM], aux, u) : 0.002f;
        float q = pz * 1.4142135623731f;
        if (pz > 0.0f) q = 0.5f - (q + 0.70710678118654502f) * (q + 0.70710678118654502f);
        else q = 0.5f - (0.70710678118654502f - q) * (0.70710678118654502f - q);
        q = 0.5f * expf(q);
        if (pz > 0.0f) q = 1.0f - q;
        sv += t->fco[mat + i * NM] * q;
        rn[i] = q;
      } else {
        rn[i] = 0.0f;   /* shell above the photon energy: the reference leaves it uninitialised */
      }
    }
    if (!((ranecu(s) * s0) > (sv * (1.0f + tau * ((ek3 - ek2 - 1.0f) + tau * (ek2 + tau * ek3)))) /
                                 (ek3 * tau * (tau * tau + 1.0f))))
      break;
  }
  double costh = 1.0 - cdt1;

  float pzomc, af;
  for (;;) {
    float q = sv * ranecu(s);
    float pac = 0.0f;
    int ish = nsh - 1;
    for (int i = 0; i < nsh - 1; ++i) {
      pac += t->fco[mat + i * NM] * rn[i];
      if (pac > q) {
        ish = i;
        break;
      }
    }
    q = ranecu(s) * rn[ish];
    if (q < 0.5f) pzomc = (0.70710678118654502f - sqrtf(0.5f - logf(q + q))) / (t->fj0[mat + ish * NM] * 1.4142135623731f);
    else pzomc = (sqrtf(0.5f - logf(2.0f - 2.0f * q)) - 0.70710678118654502f) / (t->fj0[mat + ish * NM] * 1.4142135623731f);
    if (pzomc < -1.0f) continue;
    q = (float)((double)tau * ((double)tau - costh * 2.f) + 1.f);
    if (q > 1.0e-20f) af = sqrtf(q) * (tau * (tau - ((float)costh)) / q + 1.f);
    else af = 0.00200f;
    q = (af > 0.0f) ? af * 0.2f + 1.f : 1.f - af * 0.2f;
    float pzc = (pzomc < 0.2f) ? pzomc : 0.2f;
    pzc = (pzc > -0.2f) ? pzc : -0.2f;
    if (ranecu(s) * q < (af * pzc + 1.f)) break;
  }
  {
    float tt = pzomc * pzomc;
    float b1 = 1.f - tt * tau * tau;
    float b2 = 1.f - tt * tau * ((float)costh);
    float q = sqrtf(fabsf(b2 * b2 - b1 * (1.0f - tt)));
    if (pzomc < 0.0f) q *= -1.0f;
    tt = (tau / b1) * (b2 + q);
    if (tt > 1.0f) tt = 1.0f;
    *energy *= tt;
  }
  return costh;
}

/* ------------------------------------------------------------- detector */

/* Ideal cylinder intersection (MCGPU-PET_kernel.cu:1645-1700); returns the
 * distance, writes the hit point relative to the detector centre. */
static float cylinder(const orc_params* p, vec3 r, vec3 d, vec3* h) {
  float x0 = r.x - p->cx, y0 = r.y - p->cy;
  float A = d.x * d.x + d.y * d.y;
  float B = 2.0f * (x0 * d.x + y0 * d.y);
  float C = x0 * x0 + y0 * y0 - p->radius * p->radius;
  float dist = (A == 0.0f) ? 99999999.9f : (-B + sqrtf(B * B - 4.0f * A * C)) / (2.0f * A);
  h->x = x0 + dist * d.x;
  h->y = y0 + dist * d.y;
  h->z = (r.z - p->cz) + dist * d.z;
  return dist;
}

long long orc_sinogram_bin(const orc_params* p, float phi2, float z2, float phi1, float z1) {
  /* MCGPU-PET_kernel.cu:1749-1791 with the reference's running sums */
  int ix1 = fl((float)(((double)phi2 / (2.0 * PI_D) + 0.5) * (double)p->ncrystals));
  int ix2 = fl((float)(((double)phi1 / (2.0 * PI_D) + 0.5) * (double)p->ncrystals));
  int iz1 = fl((float)(((double)(z2 / p->fovz) + 0.5) * (double)p->nrows));
  int iz2 = fl((float)(((double)(z1 / p->fovz) + 0.5) * (double)p->nrows));
  if (iz1 < 0 || iz2 < 0 || iz1 >= p->nrows || iz2 >= p->nrows) return -1;
  if (abs(iz2 - iz1) > p->mrd) return -1;
  float delta = (float)abs(iz2 - iz1);
  int incl = fl((delta - 1 + ((p->span + 1) / 2)) / (float)p->span);
  int iseg = 2 * incl;
  if (iz2 < iz1 && iseg > 0) iseg = iseg - 1;
  long long ofseg = (long long)iseg * p->nzs;
  for (int k = 0; k <= iseg; ++k) {
    float ofk = (float)((k - 2) * 0.5);
    if (k > 1) ofseg -= (p->span + 1);
    if (k > 3) ofseg -= (long long)fl(ofk) * 2 * p->span;
  }
  int ofz = 0;
  if (incl > 0) ofz = ((p->span + 1) / 2) + (incl - 1) * p->span;
  long long izm = ofseg + (iz1 + iz2) - ofz;
  if (ix2 < ix1) {
    int tmp = ix2;
    ix2 = ix1;
    ix1 = tmp;
  }
  int ith = ((ix1 + ix2 + p->nangles + 1) % p->ncrystals) / 2;
  int ir = abs(ix2 - ix1 - p->nangles);
  if ((ix1 < ith) || (ix2 >= (ith + p->nangles))) ir = -ir;
  ir = ir + p->nrad / 2;
  if (izm < 0 || izm >= p->nsinos || ir < 0 || ir >= p->nrad) return -1;
  return izm * (long long)p->nangles * p->nrad + (long long)ith * p->nrad + ir;
}

typedef struct {
  vec3 pos, dir;
  float energy, travel;
  int state;
} photon;

typedef struct {
  unsigned long long c[9];
} counts;

static void add_i32(int32_t* a, int v) { __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }
static void add_u64(unsigned long long* a, unsigned long long v) { __atomic_fetch_add(a, v, __ATOMIC_RELAXED); }

/* Dose of one real interaction, host branch of the reference
 * (MCGPU-PET_kernel.cu:396-410, 1593-1650, `#ifndef USING_CUDA`): `loss` is
 * E_after - E_before (Compton) or -E (photoelectric); tallied below -0.001 eV
 * with terms (u64)(Edep + 0.5f) and (u64)(Edep*Edep + 0.5f), SCALE_eV = 1. */
static void tally_dose(const orc_params* p, orc_outputs* o, float loss, int mat, vec3 pos) {
  if (!(loss < -0.001f)) return;
  const float edep = -1.0f * loss;
  const unsigned long long e1 = (unsigned long long)(edep * 1.0f + 0.5f);
  const unsigned long long e2 = (unsigned long long)(edep * edep + 0.5f);
  if (o->material_dose) {
    add_u64(&o->material_dose[2 * mat], e1);
    add_u64(&o->material_dose[2 * mat + 1], e2);
  }
  const int* r = p->dose_roi;
  if (!o->voxel_dose || r[1] < 0) return;
  const short x = (short)floorf(pos.x * p->inv_vx), y = (short)floorf(pos.y * p->inv_vy),
              z = (short)floorf(pos.z * p->inv_vz);
  if (x < r[0] || x > r[1] || y < r[2] || y > r[3] || z < r[4] || z > r[5]) return;
  const int dx = 1 + r[1] - r[0];
  const long long k = (long long)(x - r[0]) + (long long)(y - r[2]) * dx + (long long)(z - r[4]) * dx * (1 + r[3] - r[2]);
  add_u64(&o->voxel_dose[2 * k], e1);
  add_u64(&o->voxel_dose[2 * k + 1], e2);
}

static void put_record(unsigned char* rec, unsigned long long t_emit, float travel, int voxel, float energy,
                       float z, float phi, vec3 d, int state) {
  float tt = (float)((double)travel * PS_PER_CM);
  short i1 = (short)state, i2 = 0;
  memcpy(rec + 0, &t_emit, 8);
  memcpy(rec + 8, &tt, 4);
  memcpy(rec + 12, &voxel, 4);
  memcpy(rec + 16, &energy, 4);
  memcpy(rec + 20, &z, 4);
  memcpy(rec + 24, &phi, 4);
  memcpy(rec + 28, &d.x, 4);
  memcpy(rec + 32, &d.y, 4);
  memcpy(rec + 36, &d.z, 4);
  memcpy(rec + 40, &i1, 2);
  memcpy(rec + 42, &i2, 2);
}

/* Sinogram tally (tally_Sinogram, MCGPU-PET_kernel.cu:1624-1836) and phase
 * space tally (tally_PSF_coincidences, :531-644) of a pair whose photons both
 * escaped; b = second photon, a = first. */
static void detect(rng_t* s, const orc_params* p, orc_outputs* o, int voxel, unsigned long long t_left,
                   const photon* b, const photon* a, counts* cnt, int spurious) {
  const int sino = p->tally_psf_sinogram == 0 || p->tally_psf_sinogram == 2;
  const int psf = p->tally_psf_sinogram == 0 || p->tally_psf_sinogram == 1;
  if (sino) {
    vec3 hb, ha;
    cylinder(p, b->pos, b->dir, &hb);
    float phib = atan2f(hb.y, hb.x);
    if (fabsf(hb.z) < 0.5f * p->height) {
      cylinder(p, a->pos, a->dir, &ha);
      float phia = atan2f(ha.y, ha.x);
      if (fabsf(ha.z) < 0.5f * p->height) {
        long long bin = orc_sinogram_bin(p, phib, hb.z, phia, ha.z);
        if (bin >= 0) {
          float u1 = ranecu(s), u2 = ranecu(s);
          float g1 = sqrtf((float)(-2.0 * (double)logf(u1 + 1e-8f))) * cosf((float)(2.0 * PI_D * (double)u2));
          float u3 = ranecu(s), u4 = ranecu(s);
          float g2 = sqrtf((float)(-2.0 * (double)logf(u3 + 1.0e-8f))) * cosf((float)(2.0 * PI_D * (double)u4));
          float eb = b->energy + (p->e_resol / 2.35f) * b->energy * g1;
          float ea = a->energy + (p->e_resol / 2.35f) * a->energy * g2;
          int ib = fl(eb / 1000.0f), ia = fl(ea / 1000.0f);
          if (ib < p->ne && ib >= 0) {
            add_i32(&o->spectrum[ib], 1);
            cnt->c[3]++;
          }
          if (ia < p->ne && ia >= 0) {
            add_i32(&o->spectrum[ia], 1);
            cnt->c[3]++;
          }
          if (eb > p->e_low && eb < p->e_high && ea > p->e_low && ea < p->e_high) {
            if (!spurious && b->state == 0 && a->state == 0) {
              add_i32(&o->trues[bin], 1);
              add_i32(&o->image_trues[voxel], 1);
            } else {
              add_i32(&o->scatter[bin], 1);
              add_i32(&o->image_scatter[voxel], 1);
            }
            cnt->c[3] += 2;
          }
        }
      }
    }
  }
  if (psf) {
    vec3 hb, ha;
    float tb = b->travel + cylinder(p, b->pos, b->dir, &hb);
    float phib = atan2f(hb.y, hb.x);
    if (fabsf(hb.z) < 0.5f * p->height) {
      float ta = a->travel + cylinder(p, a->pos, a->dir, &ha);
      float phia = atan2f(ha.y, ha.x);
      float u1 = ranecu(s), u2 = ranecu(s);
      float g1 = sqrtf(-2.0f * logf(u1 + 1e-8f)) * cosf((float)(2.0 * PI_D * (double)u2));
      float u3 = ranecu(s), u4 = ranecu(s);
      float g2 = sqrtf(-2.0f * logf(u3 + 1.0e-8f)) * cosf((float)(2.0 * PI_D * (double)u4));
      float eb = b->energy + (p->e_resol * (1.0f / 2.35f)) * b->energy * g1;
      float ea = a->energy + (p->e_resol * (1.0f / 2.35f)) * a->energy * g2;
      if (fabsf(ha.z) < 0.5f * p->height && eb > p->e_low && eb < p->e_high && ea > p->e_low && ea < p->e_high) {
        int k = __atomic_fetch_add(&o->psf_count, 2, __ATOMIC_RELAXED);
        if (k < p->psf_capacity - 1 && o->psf) {
          int kb = (tb < ta) ? k : k + 1, ka = (tb < ta) ? k + 1 : k;
          unsigned long long te = p->acq_ps - t_left;
          put_record(o->psf + 44 * (size_t)kb, te, tb, voxel, eb, hb.z, phib, b->dir, b->state);
          put_record(o->psf + 44 * (size_t)ka, te, ta, voxel, ea, ha.z, phia, a->dir, a->state);
        }
      }
    }
  }
}

/* ------------------------------------------------------------- tracking */

/* Woodcock tracking and interactions of one photon (MCGPU-PET_kernel.cu:
 * 298-414); returns 1 when it leaves the voxel box, 0 when absorbed. */
static int track(rng_t* s, const orc_params* p, const orc_tables* t, const int32_t* mat0, const float* rho,
                 photon* ph, counts* cnt, orc_outputs* o) {
  float energy = ph->energy;
  int index = fl((energy - p->e0) * p->ide);
  if (index < 0 || index >= p->n_e - 1) return 0;   /* outside the tables (callers check the prompt energy) */
  float mfp_w = t->woodcock[2 * index] + energy * t->woodcock[2 * index + 1];
  cnt->c[2]++;
  int mat_old = -1, mat = 0;
  float a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
  for (;;) {
    int v = locate(p, ph->pos);
    if (v < 0) break;
    float prob = 0.f, u = 0.f, md = 0.f;
    do {
      float step = -(mfp_w)*logf(ranecu(s));
      ph->travel += step;
      ph->pos.x += step * ph->dir.x;
      ph->pos.y += step * ph->dir.y;
      ph->pos.z += step * ph->dir.z;
      v = locate(p, ph->pos);
      if (v < 0) break;
      mat = mat0[v];
      cnt->c[0]++;
      if (mat != mat_old) {
        for (int k = 0; k < 3; ++k) {
          a[k] = t->mfp_a[3 * ((size_t)index * NM + mat) + k];
          b[k] = t->mfp_b[3 * ((size_t)index * NM + mat) + k];
        }
        mat_old = mat;
        cnt->c[1]++;
      }
      md = mfp_w * rho[v];
      prob = 1.0f - md * (a[0] + energy * b[0]);
      u = ranecu(s);
    } while (u < prob);
    if (v < 0) break;
    prob += md * (a[1] + energy * b[1]);
    if (u < prob) {
      const float e_before = energy;
      double c = compton(s, &energy, mat, t);
      rotate(&ph->dir, c, 6.28318530717958647693 * ranecu_double(s));
      cnt->c[5]++;
      tally_dose(p, o, energy - e_before, mat, ph->pos);
      index = fl((energy - p->e0) * p->ide);
      if (index > -1) {
        mfp_w = t->woodcock[2 * index] + energy * t->woodcock[2 * index + 1];
        mat_old = -2;
        ph->state = ph->state == 0 ? 1 : 3;
        cnt->c[2]++;
      }
    } else {
      prob += md * (a[2] + energy * b[2]);
      if (u < prob) {
        double c = rayleigh(s, energy, mat, t->pmax[(size_t)(index + 1) * NM + mat], t);
        rotate(&ph->dir, c, 6.28318530717958647693 * ranecu_double(s));
        ph->state = ph->state == 0 ? 2 : 3;
        cnt->c[6]++;
      } else {
        index = -11;
        cnt->c[7]++;
        tally_dose(p, o, -energy, mat, ph->pos);
      }
    }
    if (index < 0) break;
  }
  ph->energy = energy;
  return index > -1;
}

/* One lane of the reference launch: Poisson decays of rate activity/tpb,
 * each giving a photon pair (MCGPU-PET_kernel.cu:153-463). */
static unsigned long long run_lane(const orc_params* p, const orc_tables* t, const int32_t* mat0,
                                   const float* rho, int voxel, float activity, uint64_t stream, orc_outputs* o,
                                   counts* cnt) {
  rng_t s = rng_stream(p->seed, stream);
  double inv_act = (p->tpb / (double)activity);
  const double inv_life = 1.0 / (double)p->mean_life;
  unsigned long long t_left = p->acq_ps, hist = 0;
  const int vx = voxel % p->nx, vy = (voxel / p->nx) % p->ny, vz = voxel / (p->nx * p->ny);
  cnt->c[8]++;
  for (;;) {
    double dt = -log(ranecu_double(&s)) * inv_act;
    unsigned long long dps = round_u64(dt * 1e12);
    if (!(dps < t_left)) break;
    t_left -= dps;
    hist += 2;
    inv_act = inv_act * exp(dt * inv_life);
    photon a, b;
    source_first(&s, p, vx, vy, vz, &a.pos, &a.dir);
    vec3 origin = a.pos, d0 = a.dir;
    a.energy = E_ANNIHILATION;
    a.travel = 0.f;
    a.state = 0;
    cnt->c[4] += 2;
    int esc_a = track(&s, p, t, mat0, rho, &a, cnt, o);
    source_second(&s, p->background, d0, &b.dir);
    b.pos = origin;
    b.energy = E_ANNIHILATION;
    b.travel = 0.f;
    b.state = 0;
    int esc_b = track(&s, p, t, mat0, rho, &b, cnt, o);
    if (esc_a && esc_b) {
      int pass = (p->tally_type == 0) || (p->tally_type == 1 && b.state == 0 && a.state == 0) ||
                 (p->tally_type == 2 && (b.state != 0 || a.state != 0));
      if (pass) detect(&s, p, o, voxel, t_left, &b, &a, cnt, 0);
    }
    /* Prompt gamma (no reference counterpart): emitted isotropically from
     * the decay point after the pair (a yield draw first when the yield is
     * below 1), tracked, then paired with each escaped annihilation photon,
     * photon 1 first; every such pair is a spurious coincidence, tallied with
     * the scatter and left out of a trues-only tally. */
    if (p->prompt_energy > 0.0f && (p->prompt_yield >= 1.0f || ranecu(&s) < p->prompt_yield)) {
      photon g;
      isotropic(&s, &g.dir);
      g.pos = origin;
      g.energy = p->prompt_energy;
      g.travel = 0.f;
      g.state = 0;
      hist += 1;
      cnt->c[4] += 1;
      int esc_g = track(&s, p, t, mat0, rho, &g, cnt, o);
      if (esc_g && p->tally_type != 1) {
        if (esc_a) detect(&s, p, o, voxel, t_left, &g, &a, cnt, 1);
        if (esc_b) detect(&s, p, o, voxel, t_left, &g, &b, cnt, 1);
      }
    }
  }
  return hist;
}

int orc_run(const orc_params* p, const orc_tables* t, const int32_t* mat0, const float* rho, const float* activity,
            const int32_t* voxel_list, long long n_list, int n_threads, orc_outputs* out) {
  const long long nv = (long long)p->nx * p->ny * p->nz;
  const long long n = voxel_list ? n_list : nv;
  unsigned long long hist = 0;
  unsigned long long tot[9] = {0};
  out->psf_count = 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel
  {
    counts cnt;
    memset(&cnt, 0, sizeof(cnt));
    unsigned long long h = 0;
#pragma omp for schedule(dynamic, 1)
    for (long long i = 0; i < n; ++i) {
      int v = voxel_list ? voxel_list[i] : (int)i;
      if (!(activity[v] > 1.0e-7f)) continue;
      for (int l = 0; l < p->tpb; ++l)
        h += run_lane(p, t, mat0, rho, v, activity[v], (uint64_t)v * p->tpb + l, out, &cnt);
    }
#pragma omp critical
    {
      hist += h;
      for (int k = 0; k < 9; ++k) tot[k] += cnt.c[k];
    }
  }
  out->histories = hist;
  memcpy(out->counters, tot, sizeof(tot));
  return 0;
}

/* ------------------------------------------------------------- probes */

void orc_rng(int seed, const int64_t* ids, int n, int ndraw, int32_t* seeds_out, float* draws, double* ddraws) {
  for (int i = 0; i < n; ++i) {
    rng_t s = rng_stream(seed, (uint64_t)ids[i]);
    seeds_out[2 * i] = s.x;
    seeds_out[2 * i + 1] = s.y;
    rng_t s2 = s;
    for (int d = 0; d < ndraw; ++d) draws[(size_t)i * ndraw + d] = ranecu(&s);
    for (int d = 0; d < ndraw; ++d) ddraws[(size_t)i * ndraw + d] = ranecu_double(&s2);
  }
}

void orc_detector(const orc_params* p, int n, const float* e2, const float* e1, const float* pos2, const float* pos1,
                  const float* dir2, const float* dir1, const int8_t* st2, const int8_t* st1, const int32_t* seeds,
                  int32_t* out) {
  for (int i = 0; i < n; ++i) {
    photon b = {{pos2[3 * i], pos2[3 * i + 1], pos2[3 * i + 2]}, {dir2[3 * i], dir2[3 * i + 1], dir2[3 * i + 2]},
                e2[i], 0.f, st2[i]};
    photon a = {{pos1[3 * i], pos1[3 * i + 1], pos1[3 * i + 2]}, {dir1[3 * i], dir1[3 * i + 1], dir1[3 * i + 2]},
                e1[i], 0.f, st1[i]};
    rng_t s = {seeds[2 * i], seeds[2 * i + 1]};
    int32_t* o = out + 6 * i;
    o[0] = -1;
    o[1] = 0;
    o[2] = -1;
    o[3] = -1;
    vec3 hb, ha;
    cylinder(p, b.pos, b.dir, &hb);
    float phib = atan2f(hb.y, hb.x);
    if (fabsf(hb.z) < 0.5f * p->height) {
      cylinder(p, a.pos, a.dir, &ha);
      float phia = atan2f(ha.y, ha.x);
      if (fabsf(ha.z) < 0.5f * p->height) {
        long long bin = orc_sinogram_bin(p, phib, hb.z, phia, ha.z);
        if (bin >= 0) {
          float u1 = ranecu(&s), u2 = ranecu(&s);
          float g1 = sqrtf((float)(-2.0 * (double)logf(u1 + 1e-8f))) * cosf((float)(2.0 * PI_D * (double)u2));
          float u3 = ranecu(&s), u4 = ranecu(&s);
          float g2 = sqrtf((float)(-2.0 * (double)logf(u3 + 1.0e-8f))) * cosf((float)(2.0 * PI_D * (double)u4));
          float eb = b.energy + (p->e_resol / 2.35f) * b.energy * g1;
          float ea = a.energy + (p->e_resol / 2.35f) * a.energy * g2;
          int ib = fl(eb / 1000.0f), ia = fl(ea / 1000.0f);
          if (ib < p->ne && ib >= 0) o[2] = ib;
          if (ia < p->ne && ia >= 0) o[3] = ia;
          if (eb > p->e_low && eb < p->e_high && ea > p->e_low && ea < p->e_high) {
            o[0] = (int32_t)bin;
            o[1] = (b.state == 0 && a.state == 0) ? 1 : 2;
          }
        }
      }
    }
    o[4] = s.x;
    o[5] = s.y;
  }
}

void orc_compton(const orc_tables* t, int n, const float* energy_in, const int32_t* mat, const int32_t* seeds_in,
                 float* energy_out, double* costh_out, int32_t* seeds_out) {
  for (int i = 0; i < n; ++i) {
    rng_t s = {seeds_in[2 * i], seeds_in[2 * i + 1]};
    float e = energy_in[i];
    costh_out[i] = compton(&s, &e, mat[i], t);
    energy_out[i] = e;
    seeds_out[2 * i] = s.x;
    seeds_out[2 * i + 1] = s.y;
  }
}

void orc_rayleigh(const orc_tables* t, int n, const float* energy_in, const int32_t* mat, const float* pmax,
                  const int32_t* seeds_in, double* costh_out, int32_t* seeds_out) {
  for (int i = 0; i < n; ++i) {
    rng_t s = {seeds_in[2 * i], seeds_in[2 * i + 1]};
    costh_out[i] = rayleigh(&s, energy_in[i], mat[i], pmax[i], t);
    seeds_out[2 * i] = s.x;
    seeds_out[2 * i + 1] = s.y;
  }
}

void orc_source(int nx, int ny, int nz, const float inv_voxel_size[3], int background, const int32_t* seeds_in,
                float* out, int32_t* seeds_out) {
  orc_params p;
  memset(&p, 0, sizeof(p));
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.inv_vx = inv_voxel_size[0];
  p.inv_vy = inv_voxel_size[1];
  p.inv_vz = inv_voxel_size[2];
  long long nv = (long long)nx * ny * nz;
  for (long long v = 0; v < nv; ++v) {
    rng_t s = {seeds_in[2 * v], seeds_in[2 * v + 1]};
    vec3 pos, d1, d2;
    source_first(&s, &p, (int)(v % nx), (int)((v / nx) % ny), (int)(v / ((long long)nx * ny)), &pos, &d1);
    source_second(&s, background, d1, &d2);
    float* o = out + 12 * v;
    o[0] = pos.x; o[1] = pos.y; o[2] = pos.z;
    o[3] = d1.x; o[4] = d1.y; o[5] = d1.z;
    o[6] = pos.x; o[7] = pos.y; o[8] = pos.z;
    o[9] = d2.x; o[10] = d2.y; o[11] = d2.z;
    seeds_out[2 * v] = s.x;
    seeds_out[2 * v + 1] = s.y;
  }
}

void orc_sinogram_sizes(int mrd, int span, int nzs, int* nseg, int* nsinos) {
  /* MCGPU-PET.cu:1176-1187 */
  int ns = 2 * (int)floor((double)(mrd / span)) + 1;
  int n = ns * nzs;
  for (int a = 1; a <= ns; ++a) {
    if (a > 1) n = n - (span + 1);
    if (a > 3) n = (int)(n - 2 * floor((double)((a - 2) / 2)) * span);
  }
  *nseg = ns;
  *nsinos = n;
}
