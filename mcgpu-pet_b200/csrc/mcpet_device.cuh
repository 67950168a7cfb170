/* Device building blocks of the photon-transport path (sm_100a).
 *
 * Each function restates one step of the reference kernel
 * (MCGPU-PET_kernel.cu).  The floating-point operations inside every step are
 * kept in the reference's order, types and intrinsic calls (the library is
 * built with -use_fast_math like the reference, Makefile:44), because a
 * history can only be replayed from its RANECU seed when every rounding is the
 * same; the surrounding structure (lane queue, state layout, table records,
 * palette voxels, RNG jump) is this library's own.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "mcpet_params.h"

namespace mcpet {
namespace dev {

/* Physical and geometric constants (values from MCGPU-PET.h:104-128). */
constexpr float kEps = 0.00015f;                 /* EPS_SOURCE */
constexpr double kPi = 3.14159265358979323846;   /* PI */
constexpr float kAnnihilation = 510998.95f;      /* ANNIHILATION_PHOTON_ENERGY */
constexpr double kInvLightSpeed = (1.0 / 29979245800e-12); /* ps per cm */

/* Loop guards (defaults of mcpet_run_opts.max_woodcock_steps and
 * max_rejections): far above anything a physical history reaches; when one
 * fires the photon is dropped and the run reports MCPET_ERR_DEVICE. */
constexpr int kMaxWoodcockSteps = 1 << 20;
constexpr int kMaxRejections = 1 << 16;

/* ------------------------------------------------------------------------
 * RANECU (L'Ecuyer 1988 combined MLCG; reference ranecu/ranecu_double,
 * MCGPU-PET_kernel.cu:1045-1083).  Each component is advanced with a 64-bit
 * product reduced modulo the pseudo-Mersenne moduli m1 = 2^31-85 and
 * m2 = 2^31-249, which yields exactly (a*s) mod m like the reference's Schrage
 * factorisation.  The output combination and scaling are the generator's
 * published ones. */
struct Rng {
  int x, y;
};

constexpr uint32_t kM1 = 2147483563u, kM2 = 2147483399u;

__device__ __forceinline__ uint32_t mlcg1(uint32_t s) {
  uint64_t p = (uint64_t)s * 40014u;                /* < 2^47 */
  uint32_t r = (uint32_t)(p & 0x7fffffffu) + (uint32_t)(p >> 31) * 85u;
  return r >= kM1 ? r - kM1 : r;
}
__device__ __forceinline__ uint32_t mlcg2(uint32_t s) {
  uint64_t p = (uint64_t)s * 40692u;
  uint32_t r = (uint32_t)(p & 0x7fffffffu) + (uint32_t)(p >> 31) * 249u;
  return r >= kM2 ? r - kM2 : r;
}
__device__ __forceinline__ int rng_combine(Rng& s) {
  s.x = (int)mlcg1((uint32_t)s.x);
  s.y = (int)mlcg2((uint32_t)s.y);
  int z = s.x - s.y;
  if (z < 1) z += 2147483562;
  return z;
}
__device__ __forceinline__ float ranecu(Rng& s) {
  return __int2float_rn(rng_combine(s)) * 4.65661305739e-10f;
}
__device__ __forceinline__ double ranecu_double(Rng& s) {
  return __int2double_rn(rng_combine(s)) * 4.6566130573917692e-10;
}

/* Full-range modular products for the stream jump (inputs < 2^31). */
__device__ __forceinline__ uint32_t mulmod_pm(uint32_t a, uint32_t b, uint32_t c, uint32_t m) {
  uint64_t p = (uint64_t)a * b;                     /* < 2^62 */
  uint64_t r = (p & 0x7fffffffull) + (p >> 31) * c; /* < 2^39 */
  uint32_t q = (uint32_t)(r & 0x7fffffffull) + (uint32_t)(r >> 31) * c;
  return q >= m ? q - m : q;
}

/* Start state of RANECU stream `stream` for a seed: the reference
 * jumps each thread (stream+1)*555555*256 draws ahead
 * (init_PRNG, MCGPU-PET_kernel.cu:925-978).  a^((s+1)C) = prod over the set
 * bits of (s+1) of (a^C)^(2^k), with the 32 powers precomputed on the host. */
__device__ __forceinline__ Rng rng_stream(const TransportParams& P, int seed, uint64_t stream) {
  uint64_t e = stream + 1;
  uint32_t y1 = 1, y2 = 1;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    if ((e >> k) & 1ull) {
      y1 = mulmod_pm(y1, (uint32_t)P.jump1[k], 85u, kM1);
      y2 = mulmod_pm(y2, (uint32_t)P.jump2[k], 249u, kM2);
    }
  }
  Rng r;
  r.x = (int)mulmod_pm((uint32_t)seed % kM1, y1, 85u, kM1);
  r.y = (int)mulmod_pm((uint32_t)seed % kM2, y2, 249u, kM2);
  return r;
}
__device__ __forceinline__ Rng rng_stream(const TransportParams& P, uint64_t stream) {
  return rng_stream(P, P.seed, stream);
}

/* ------------------------------------------------------------------------
 * Voxel lookup (locate_voxel, MCGPU-PET_kernel.cu:1098-1124). */
__device__ __forceinline__ int locate(const TransportParams& P, float x, float y, float z) {
  if ((y < kEps) || (y > (P.bby - kEps)) || (x < kEps) || (x > (P.bbx - kEps)) || (z < kEps) ||
      (z > (P.bbz - kEps)))
    return -100;
  int ix = __float2int_rd(x * P.inv_vx);
  int iy = __float2int_rd(y * P.inv_vy);
  int iz = __float2int_rd(z * P.inv_vz);
  return ix + iy * P.nx + iz * P.nx * P.ny;
}

/* ------------------------------------------------------------------------
 * Positron annihilation source (source, MCGPU-PET_kernel.cu:666-773). */
__device__ __forceinline__ void emit_isotropic(Rng& r, float3& d) {
  d.z = 1.0f - 2.0f * ranecu(r);
  float phi = 6.28318530716f * ranecu(r);
  float sin_t = sqrtf(1.0f - d.z * d.z);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  d.y = sin_t * sp;
  d.x = sin_t * cp;
}

/* First photon: isotropic direction, uniform point inside the voxel kept
 * EPS away from its faces. */
__device__ __forceinline__ void emit_first(Rng& r, const TransportParams& P, int vx, int vy, int vz,
                                           float3& pos, float3& dir) {
  emit_isotropic(r, dir);
  float r1 = ranecu(r);
  float r2 = ranecu(r);
  float r3 = ranecu(r);
  r1 = (kEps > (r1 - kEps)) ? kEps : (r1 - kEps);
  r2 = (kEps > (r2 - kEps)) ? kEps : (r2 - kEps);
  r3 = (kEps > (r3 - kEps)) ? kEps : (r3 - kEps);
  pos.x = ((float)vx + r1) / P.inv_vx;
  pos.y = ((float)vy + r2) / P.inv_vy;
  pos.z = ((float)vz + r3) / P.inv_vz;
}

/* Direction d turned by the polar angle with cosine c and sine s (s may be
 * negative: the azimuth turned by pi) around azimuth 2 pi u: the DIRECT
 * rotation of rotate_fast with the sine given, so that a small angle keeps
 * its precision. */
__device__ __forceinline__ void rotate_fast_cs(float3& d, float c, float s, float u) {
  float sinphi, cosphi;
  __sincosf(6.28318530717958647693f * u, &sinphi, &cosphi);
  const float dxy = d.x * d.x + d.y * d.y;
  if (dxy > 1.0e-14f) {
    const float sdt = s * rsqrtf(dxy);
    const float x_in = d.x;
    d.x = d.x * c + sdt * (x_in * d.z * cosphi - d.y * sinphi);
    d.y = d.y * c + sdt * (d.y * d.z * cosphi + x_in * sinphi);
    d.z = d.z * c - dxy * sdt * cosphi;
  } else {
    d.y = s * sinphi;
    if (d.z > 0.0f) {
      d.x = s * cosphi;
      d.z = c;
    } else {
      d.x = -s * cosphi;
      d.z = -c;
    }
  }
}

/* Second photon: anti-parallel to the first, tilted by the acolinearity
 * angle theta = 2*0.21276 deg * N(0,1) (Box-Muller, cosine branch) around a
 * uniform azimuth; or isotropic in background mode.  The reference builds it
 * from the spherical angles of -d1 and a rotation matrix (atan2, acos and
 * four sincos).  kFast (balanced lanes): the same three draws give theta
 * and the azimuth, and -d1 is turned by theta directly -- the same
 * distribution (the azimuth is uniform, so the frame does not matter) for
 * a fraction of the arithmetic. */
template <bool kFast = false>
__device__ __forceinline__ void emit_second(Rng& r, bool background, const float3& d1, float3& d) {
  if (background) {
    emit_isotropic(r, d);
    return;
  }
  float phi2, theta2, theta_nc, phi_nc;
  if (kFast) {
    const float v1 = ranecu(r);
    const float v2 = ranecu(r);
    theta_nc = (float)(2.0 * 0.21276 * kPi / 180.0) * sqrtf(-2.0f * __logf(v2 + 1e-8f)) *
               __cosf((float)(2.0 * kPi) * v1);
    float st, ct;
    __sincosf(theta_nc, &st, &ct);
    d = make_float3(-d1.x, -d1.y, -d1.z);
    rotate_fast_cs(d, ct, st, ranecu(r));
    return;
  } else {
    phi2 = (float)((double)atan2f(d1.y, d1.x) + kPi);
    theta2 = (float)(kPi - (double)acosf(d1.z));
    const float v1 = ranecu(r);
    const float v2 = ranecu(r);
    theta_nc = (float)((2.0 * 0.21276 * kPi / 180.0) * (double)sqrtf(-2.0f * logf(v2 + 1e-8f)) *
                       (double)cosf((float)((2.0 * kPi) * (double)v1)));
    phi_nc = (float)((2.0 * kPi) * (double)ranecu(r));
  }
  float st, ct, sp, cp, st1, ct1, sp1, cp1;
  sincosf(theta_nc, &st, &ct);
  sincosf(phi_nc, &sp, &cp);
  sincosf(theta2, &st1, &ct1);
  sincosf(phi2, &sp1, &cp1);
  float gx = cp * st;
  float gy = sp * st;
  float gz = ct;
  d.x = gx * ct1 * cp1 - gy * sp1 + gz * st1 * cp1;
  d.y = gx * ct1 * sp1 + gy * cp1 + gz * st1 * sp1;
  d.z = -gx * st1 + gz * ct1;
}

/* ------------------------------------------------------------------------
 * Direction change by polar cosine costh and azimuth phi in the particle
 * frame, in double precision (PENELOPE DIRECT; rotate_double,
 * MCGPU-PET_kernel.cu:1160-1200). */
__device__ __forceinline__ void rotate(float3& d, double costh, double phi) {
  double sinphi, cosphi;
  double dxy = d.x * d.x + d.y * d.y;
  sincos(phi, &sinphi, &cosphi);
  double norm = dxy + d.z * d.z;
  if (fabs(norm - 1.0) > 1.0e-14) {
    norm = 1.0 / sqrt(norm);
    d.x = norm * d.x;
    d.y = norm * d.y;
    d.z = norm * d.z;
    dxy = d.x * d.x + d.y * d.y;
  }
  if (dxy > 1.0e-28) {
    double sdt = sqrt((1.0 - costh * costh) / dxy);
    float x_in = d.x;
    d.x = d.x * costh + sdt * (x_in * d.z * cosphi - d.y * sinphi);
    d.y = d.y * costh + sdt * (d.y * d.z * cosphi + x_in * sinphi);
    d.z = d.z * costh - dxy * sdt * cosphi;
  } else {
    double sdt = sqrt(1.0 - costh * costh);
    d.y = sdt * sinphi;
    if (d.z > 0.0) {
      d.x = sdt * cosphi;
      d.z = costh;
    } else {
      d.x = -sdt * cosphi;
      d.z = -costh;
    }
  }
}

/* The same direction change in single precision, for balanced lanes (which
 * are held to statistical parity, not history replay): azimuth phi = 2 pi u
 * from the same random draw, the new direction from the same formulas.  The
 * double-precision sincos, square roots and divisions of the reference form
 * are the most expensive arithmetic of a scattering round on this part. */
__device__ __forceinline__ void rotate_fast(float3& d, float costh, float u) {
  float sinphi, cosphi;
  __sincosf(6.28318530717958647693f * u, &sinphi, &cosphi);
  float dxy = d.x * d.x + d.y * d.y;
  const float norm = dxy + d.z * d.z;
  if (fabsf(norm - 1.0f) > 1.0e-6f) {
    const float s = rsqrtf(norm);
    d.x *= s;
    d.y *= s;
    d.z *= s;
    dxy = d.x * d.x + d.y * d.y;
  }
  if (dxy > 1.0e-14f) {
    const float sdt = sqrtf((1.0f - costh * costh) / dxy);
    const float x_in = d.x;
    d.x = d.x * costh + sdt * (x_in * d.z * cosphi - d.y * sinphi);
    d.y = d.y * costh + sdt * (d.y * d.z * cosphi + x_in * sinphi);
    d.z = d.z * costh - dxy * sdt * cosphi;
  } else {
    const float sdt = sqrtf(1.0f - costh * costh);
    d.y = sdt * sinphi;
    if (d.z > 0.0f) {
      d.x = sdt * cosphi;
      d.z = costh;
    } else {
      d.x = -sdt * cosphi;
      d.z = -costh;
    }
  }
}

/* Time to a lane's next decay in ps, and the lane's decayed 1/rate
 * (MCGPU-PET_kernel.cu:267-291).  kFast: the exponential interval in single
 * precision from the same draw (balanced lanes); otherwise the reference's
 * double-precision form. */
template <bool kFast>
__device__ __forceinline__ unsigned long long decay_interval(Rng& r, double& inv_rate, double inv_mean_life) {
  if (kFast) {
    const float dt_ps = -__logf(ranecu(r)) * (float)(inv_rate * 1e12);
    inv_rate = inv_rate * (double)__expf(dt_ps * (float)(inv_mean_life * 1e-12));
    return __float2ull_rn(dt_ps);
  }
  const double dt = -log(ranecu_double(r)) * inv_rate;
  inv_rate = inv_rate * exp(dt * inv_mean_life);
  return __double2ull_rn(dt * 1e12);
}

/* ------------------------------------------------------------------------
 * Rayleigh scattering: RITA sampling of the squared molecular form factor
 * plus rejection (PENELOPE 2006 GRAa; MCGPU-PET_kernel.cu:1231-1296).
 * Returns false when the rejection guard fired. */
__device__ __forceinline__ bool sample_rayleigh(Rng& r, float energy, int mat, float pmax,
                                                const RayleighRows& R, double& costh,
                                                int max_rejections = kMaxRejections) {
  const int base = mat * kNpRayleigh;
  double xmax = ((double)energy) * 8.065535669099010e-5;
  double xlast = (double)__ldg(&R.xco[base + kNpRayleigh - 1]);
  double x2max = ((xmax * xmax) < xlast) ? (xmax * xmax) : xlast;
  if (xmax < 0.01) {
    for (int it = 0; it < max_rejections; ++it) {
      costh = 1.0 - ranecu_double(r) * 2.0;
      if (!(ranecu_double(r) > ((costh * costh + 1.0) * 0.5))) return true;
    }
    return false;
  }
  for (int it = 0; it < max_rejections; ++it) {
    double ru = ranecu_double(r) * (double)pmax;
    int itn = (int)(ru * (kNpRayleigh - 1));
    int lo = (int)__ldg(&R.itl[itn + base]);
    int hi = (int)__ldg(&R.itu[itn + base]);
    while ((hi - lo) > 1) {
      int mid = (lo + hi) >> 1;
      if (ru > (double)__ldg(&R.pco[mid - 1 + base])) lo = mid;
      else hi = mid;
    }
    int idx = lo - 1 + base;
    float p0 = __ldg(&R.pco[idx]);
    double rr = ru - p0;
    double xx;
    if (rr > 1e-16) {
      double dp = (double)(__ldg(&R.pco[idx + 1]) - p0);
      float a = __ldg(&R.aco[idx]), b = __ldg(&R.bco[idx]), x0 = __ldg(&R.xco[idx]);
      xx = (double)x0 + (double)(a + 1.0f + b) * dp * rr / (dp * dp + (a * dp + b * rr) * rr) *
                            (double)(__ldg(&R.xco[idx + 1]) - x0);
    } else {
      xx = __ldg(&R.xco[idx]);
    }
    if (xx < x2max) {
      costh = 1.0 - 2.0 * xx / x2max;
      if (ranecu_double(r) < ((costh * costh + 1.0) * 0.5)) return true;
    }
  }
  return false;
}

/* ------------------------------------------------------------------------
 * Compton scattering: relativistic impulse approximation with analytical
 * one-electron Compton profiles (PENELOPE 2006 GCOa;
 * MCGPU-PET_kernel.cu:1335-1563).  `C` is the block's shared copy of the
 * shell table, `rn` a per-thread scratch of max_shells floats.  Updates the
 * energy; returns false when a rejection guard fired. */
/* Incoherent scattering function at theta = pi, the normalisation of the
 * rejection step of GCOa (MCGPU-PET_kernel.cu:1366-1391).  It depends only on
 * the energy and material, so kernels evaluate it once per block for the
 * annihilation energy and pass the value in. */
__device__ __forceinline__ float compton_s0(float E, int mat, const ComptonTable& C) {
  const int nsh = C.noscco[mat];
  float s0 = 0.0f;
  for (int i = 0; i < nsh; ++i) {
    float u = C.uico[mat + i * kMaxMaterials];
    if (u < E) {
      float aux = E * (E - u) * 2.f;
      float pz = C.fj0[mat + i * kMaxMaterials] * (aux - u * 510998.918f) *
                 rsqrtf(aux + aux + u * u) * 1.956951306108245e-6f;
      float t;
      if (pz > 0.0f) t = (0.707106781186545f + pz * 1.4142135623731f) * (0.707106781186545f + pz * 1.4142135623731f);
      else t = (0.707106781186545f - pz * 1.4142135623731f) * (0.707106781186545f - pz * 1.4142135623731f);
      t = 0.5f * expf(0.5f - t);
      if (pz > 0.0f) t = 1.0f - t;
      s0 += C.fco[mat + i * kMaxMaterials] * t;
    }
  }
  return s0;
}

/* One trial of GCOa's first stage (MCGPU-PET_kernel.cu:1390-1451): tau = E'/E
 * from the Klein-Nishina-like envelope, then the rejection on the incoherent
 * scattering function, normalised by s0 (compton_s0 of E and the material).
 * Returns true on acceptance, with tau, cdt1 = 1 - cos(theta), the sum s and
 * the shell terms rn[] that the second stage reads.  A trial draws the same
 * random numbers whether the trials of one sampling run back to back or
 * with other work of the thread between them.  kFast (balanced lanes): the
 * envelope branch and cdt1 in single precision instead of the reference's
 * double-precision constant and division. */
template <bool kFast = false, typename Scratch>
__device__ __forceinline__ bool compton_trial(Rng& r, float E, int mat, const ComptonTable& C, Scratch rn,
                                              float s0, float& tau, float& s, double& cdt1) {
  const int nsh = C.noscco[mat];
  float ek = E * 1.956951306108245e-6f;
  float ek2 = ek * 2.f + 1.f;
  float ek3 = ek * ek;
  float taumin = 1.f / ek2;
  float a1 = logf(ek2);
  const bool first_branch = kFast ? (ranecu(r) * (a1 + 2.f * ek * (ek + 1.f) * taumin * taumin) < a1)
                                   : (ranecu(r) * (a1 + 2. * ek * (ek + 1.f) * taumin * taumin) < a1);
  if (first_branch) {
    tau = powf(taumin, ranecu(r));
  } else {
    tau = sqrtf(1.f + ranecu(r) * (taumin * taumin - 1.f));
  }
  if (kFast) {
    float c = (1.f - tau) / (tau * ek);
    if (c > 2.0f) c = 1.99999999f;
    cdt1 = c;
  } else {
    cdt1 = (double)(1.f - tau) / (((double)tau) * ((double)E) * 1.956951306108245e-6);
    if (cdt1 > 2.0) cdt1 = 1.99999999;
  }
  s = 0.0f;
  for (int i = 0; i < nsh; ++i) {
    float u = C.uico[mat + i * kMaxMaterials];
    if (u < E) {
      float aux = E * (E - u) * ((float)cdt1);
      float pz;
      if ((aux > 1.0e-12f) || (u > 1.0e-12f)) {
        pz = C.fj0[mat + i * kMaxMaterials] * (aux - u * 510998.918f) * rsqrtf(aux + aux + u * u) *
             1.956951306108245e-6f;
      } else {
        pz = 0.002f;
      }
      float t = pz * 1.4142135623731f;
      if (pz > 0.0f) t = 0.5f - (t + 0.70710678118654502f) * (t + 0.70710678118654502f);
      else t = 0.5f - (0.70710678118654502f - t) * (0.70710678118654502f - t);
      t = 0.5f * expf(t);
      if (pz > 0.0f) t = 1.0f - t;
      s += C.fco[mat + i * kMaxMaterials] * t;
      rn[i] = t;
    } else {
      rn[i] = 0.0f;   /* shell above the photon energy: the reference leaves it uninitialised */
    }
  }
  return !((ranecu(r) * s0) >
           (s * (1.0f + tau * ((ek3 - ek2 - 1.0f) + tau * (ek2 + tau * ek3)))) / (ek3 * tau * (tau * tau + 1.0f)));
}

/* GCOa's second stage after an accepted trial (MCGPU-PET_kernel.cu:1453-1562):
 * the target shell and projected momentum pz with the F(EP) rejection, then
 * the energy of the scattered photon.  costh = 1 - cdt1 of the trial.
 * Returns false when the rejection guard fired.  kFast (balanced lanes):
 * the angle term in single precision (the reference's mixes in double). */
template <bool kFast = false, typename Scratch>
__device__ __forceinline__ bool compton_doppler(Rng& r, float& energy, int mat, const ComptonTable& C, Scratch rn,
                                                float tau, float s, double costh,
                                                int max_rejections = kMaxRejections) {
  const int nsh = C.noscco[mat];
  float pzomc, af;
  int it = 0;
  for (;;) {
    if (++it > max_rejections) return false;
    float t = s * ranecu(r);
    float pac = 0.0f;
    int ish = nsh - 1;
    for (int i = 0; i < (nsh - 1); ++i) {
      pac += C.fco[mat + i * kMaxMaterials] * rn[i];
      if (pac > t) {
        ish = i;
        break;
      }
    }
    t = ranecu(r) * rn[ish];
    if (t < 0.5f) {
      pzomc = (0.70710678118654502f - sqrtf(0.5f - logf(t + t))) /
              (C.fj0[mat + ish * kMaxMaterials] * 1.4142135623731f);
    } else {
      pzomc = (sqrtf(0.5f - logf(2.0f - 2.0f * t)) - 0.70710678118654502f) /
              (C.fj0[mat + ish * kMaxMaterials] * 1.4142135623731f);
    }
    if (pzomc < -1.0f) continue;
    t = kFast ? tau * (tau - (float)costh * 2.f) + 1.f : tau * (tau - costh * 2.f) + 1.f;
    if (t > 1.0e-20f) {
      af = sqrtf(t) * (tau * (tau - ((float)costh)) / t + 1.f);
    } else {
      af = 0.00200f;
    }
    if (af > 0.0f) t = af * 0.2f + 1.f;
    else t = 1.f - af * 0.2f;
    float pzc = (pzomc < 0.2f) ? pzomc : 0.2f;
    pzc = (pzc > -0.2f) ? pzc : -0.2f;
    if (ranecu(r) * t < (af * pzc + 1.f)) break;
  }

  /* energy of the scattered photon */
  {
    float t = pzomc * pzomc;
    float b1 = 1.f - t * tau * tau;
    float b2 = 1.f - t * tau * ((float)costh);
    float q = sqrtf(fabsf(b2 * b2 - b1 * (1.0f - t)));
    if (pzomc < 0.0f) q *= -1.0f;
    t = (tau / b1) * (b2 + q);
    if (t > 1.0f) t = 1.0f;
    energy *= t;
  }
  return true;
}

/* The whole sampling: trials until one is accepted, then the second stage.
 * s0 < 0: the normaliser evaluated at the photon's energy (the reference's
 * arithmetic); else the bound given (MfpRecord::s0_bound). */
template <bool kFast = false, typename Scratch>
__device__ __forceinline__ bool sample_compton(Rng& r, float& energy, int mat, const ComptonTable& C,
                                               Scratch rn, double& costh, float s0_given = -1.0f,
                                               int max_rejections = kMaxRejections) {
  const float E = energy;
  const float s0 = s0_given < 0.0f ? compton_s0(E, mat, C) : s0_given;
  float tau, s;
  double cdt1;
  int it = 0;
  for (;;) {
    if (++it > max_rejections) return false;
    if (compton_trial<kFast>(r, E, mat, C, rn, s0, tau, s, cdt1)) break;
  }
  costh = 1.0 - cdt1;
  return compton_doppler<kFast>(r, energy, mat, C, rn, tau, s, costh, max_rejections);
}

/* ------------------------------------------------------------------------
 * Detector: intersection with the ideal cylinder of radius R around the axis
 * through (cx, cy) (MCGPU-PET_kernel.cu:1645-1700).  Outputs the hit point
 * relative to the detector centre and the travelled distance. */
__device__ __forceinline__ float to_cylinder(const TransportParams& P, const float3& centre, const float3& pos,
                                             const float3& dir, float& xn, float& yn, float& zn) {
  float x0 = pos.x - centre.x;
  float y0 = pos.y - centre.y;
  float A = dir.x * dir.x + dir.y * dir.y;
  float B = 2.0f * (x0 * dir.x + y0 * dir.y);
  float C = x0 * x0 + y0 * y0 - P.radius * P.radius;
  float dist;
  if (A == 0.0f) dist = 99999999.9f;
  else dist = (-B + sqrtf(B * B - 4.0f * A * C)) / (2.0f * A);
  xn = x0 + dist * dir.x;
  yn = y0 + dist * dir.y;
  zn = (pos.z - centre.z) + dist * dir.z;
  return dist;
}
__device__ __forceinline__ float to_cylinder(const TransportParams& P, const float3& pos, const float3& dir,
                                             float& xn, float& yn, float& zn) {
  return to_cylinder(P, make_float3(P.cx, P.cy, P.cz), pos, dir, xn, yn, zn);
}

/* Sinogram bin of a line of response (MCGPU-PET_kernel.cu:1749-1791) from the
 * azimuths and axial hit positions of the two photons (photon "a" is the one
 * tracked last).  Returns -1 when the pair falls outside the rings, the
 * maximum ring difference or the sinogram.  kFast (balanced lanes): the
 * crystal and ring indices in single precision (the reference divides in
 * double). */
template <bool kFast = false>
__device__ __forceinline__ long long sinogram_bin(const TransportParams& P, float phi_a, float z_a,
                                                  float phi_b, float z_b) {
  int xa, xb, za, zb;
  if (kFast) {
    const float inv_2pi = (float)(1.0 / (2.0 * kPi)), nc = (float)P.ncrystals, nr = (float)P.nrows;
    xa = __float2int_rd((phi_a * inv_2pi + 0.5f) * nc);
    xb = __float2int_rd((phi_b * inv_2pi + 0.5f) * nc);
    za = __float2int_rd((z_a / P.fovz + 0.5f) * nr);
    zb = __float2int_rd((z_b / P.fovz + 0.5f) * nr);
  } else {
    xa = __float2int_rd((float)(((double)phi_a / (2.0 * kPi) + 0.5) * (double)P.ncrystals));
    xb = __float2int_rd((float)(((double)phi_b / (2.0 * kPi) + 0.5) * (double)P.ncrystals));
    za = __float2int_rd((float)(((double)(z_a / P.fovz) + 0.5) * (double)P.nrows));
    zb = __float2int_rd((float)(((double)(z_b / P.fovz) + 0.5) * (double)P.nrows));
  }
  if (za < 0 || zb < 0 || za >= P.nrows || zb >= P.nrows) return -1;
  int dz = abs(zb - za);
  if (dz > P.mrd) return -1;
  /* segment of the ring difference (span grouping) */
  float fdz = (float)dz;
  int incl = __float2int_rd((fdz - 1 + ((P.span + 1) / 2)) / (float)P.span);
  int iseg = 2 * incl;
  if (zb < za && iseg > 0) iseg -= 1;
  /* first plane of segment iseg: iseg*NZS minus the planes the oblique
   * segments lack (closed form of the reference's running sum) */
  long long ofseg = (long long)iseg * P.nzs;
  if (iseg >= 2) {
    long long n = iseg - 2;
    ofseg -= (long long)(iseg - 1) * (P.span + 1);
    ofseg -= 2LL * P.span * ((n / 2) * ((n + 1) / 2));
  }
  int ofz = 0;
  if (incl > 0) ofz = ((P.span + 1) / 2) + (incl - 1) * P.span;
  long long izm = ofseg + (za + zb) - ofz;
  if (xb < xa) {
    int t = xa;
    xa = xb;
    xb = t;
  }
  int ith = ((xa + xb + P.nangles + 1) % P.ncrystals) / 2;
  int ir = abs(xb - xa - P.nangles);
  if ((xa < ith) || (xb >= (ith + P.nangles))) ir = -ir;
  ir = ir + P.nrad / 2;
  if (izm < 0 || izm >= P.nsinos || ir < 0 || ir >= P.nrad) return -1;
  return izm * (long long)P.nangles * P.nrad + (long long)ith * P.nrad + ir;
}

/* Gaussian energy blur of one photon as drawn by the sinogram tally
 * (MCGPU-PET_kernel.cu:1797-1802): sqrt(-2 ln(u1+1e-8)) cos(2 pi u2); kFast
 * (balanced lanes): in single precision. */
template <bool kFast = false>
__device__ __forceinline__ float blur_sinogram(Rng& r) {
  float u1 = ranecu(r);
  float u2 = ranecu(r);
  if (kFast) return sqrtf(-2.0f * __logf(u1 + 1e-8f)) * __cosf((float)(2.0 * kPi) * u2);
  return sqrtf((float)(-2.0 * (double)logf(u1 + 1e-8f))) * cosf((float)((double)(2.0f) * kPi * (double)u2));
}
/* ... and as drawn by the PSF tally (MCGPU-PET_kernel.cu:580-585). */
__device__ __forceinline__ float blur_psf(Rng& r) {
  float u1 = ranecu(r);
  float u2 = ranecu(r);
  return sqrtf(-2.0f * logf(u1 + 1e-8f)) * cosf((float)((double)(2.0f) * kPi * (double)u2));
}

}  // namespace dev
}  // namespace mcpet
