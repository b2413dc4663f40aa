// pic_mcc_kin.h -- one MCC_jw collision, device side.
//
// Restates, with Philox draws in place of RANDOM_NUMBER:
//   UpdateMCCParticleOne ........ mc/TypeMCC.f90:58-82 (Maxwellian gas target,
//                                 relative velocity g, energy 0.5*mu*g^2)
//   VelocityMaxwellianInit ...... base/ParticleOne.f90 (rejection sampling of |v|)
//   VelocityRandomInit .......... base/ParticleOne.f90 (isotropic direction)
//   SelectProbility ............. mc/TypeMCC.f90:155-198
//   PostCollisionVelocity ....... mc/TypeMCC.f90:101-133
//   CosKaiVahedi, IsotropicCosKai, CreatEnergyVehadi ... mc/MCCChi.f90
//   electron types 11/12/13 ..... mc/MCCElectron.F90:13-72
//   ion types 101/103 ........... mc/MCCIon.F90:6-20
// Draw order inside one collision is fixed: the k-th uniform of a collision
// is word pair (k mod 2) of Philox call k/2 with counter
// (id, step_lo, COLLIDE<<24 | species<<16 | call, step_hi).
#ifndef PIC_MCC_KIN_H
#define PIC_MCC_KIN_H

#include <math.h>
#include <stdint.h>

#include "../../include/picgpu.h"
#include "pic_common.h"

#define PIC_FORTRAN_EXP 2.71828 /* Constants.f90: exp=2.71828d0 */

struct McTable {
  int nr, ns;
  double emin, eint, emax;
  int type[PIC_MAX_REACTIONS];
  double thr[PIC_MAX_REACTIONS];
};

struct McGas {
  double mass, temperature;
};

struct McParticle {
  double vx, vy, vz;  // SI
};

struct McOut {
  int reaction;  // 1-based reaction index, 0 none
  int ionised;
  double e_new[3];    // created electron velocity (SI)
  double ion_new[3];  // created ion velocity (SI)
};

struct McRng {
  uint32_t id, slo, shi, sp, k0, k1, call;
  int have;
  double buf[2];
};

static inline McTable mc_table_from(const pic_mcc_table &t) {
  McTable m;
  m.nr = t.n_reaction;
  m.ns = t.n_sigma;
  m.emin = t.energy_min;
  m.eint = t.energy_interval;
  m.emax = t.energy_max;
  for (int r = 0; r < PIC_MAX_REACTIONS; ++r) {
    m.type[r] = t.reaction_type[r];
    m.thr[r] = t.threshold[r];
  }
  return m;
}

// Selection keys.  One Philox block per species and step draws two 32-bit
// round keys; a particle's key is two rounds of the lowbias32 integer hash
// (C. Wellons, "Prospecting for hash functions", 2018), each after an xor of
// a round key into the id.  For a given step the key is a bijection of the
// 32-bit id, so no two particles share a key, and it costs a dozen integer
// instructions where a Philox block per particle costs about eighty: the
// selection pass reads 8 bytes a particle and stays memory-bound.
PIC_HD uint32_t mcc_hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

typedef struct McSelect {
  uint32_t r0, r1;
} McSelect;

PIC_HD McSelect mcc_select_round_keys(uint32_t slo, uint32_t shi, uint32_t sp, uint32_t k0, uint32_t k1) {
  const pic_u32x4 o = pic_philox(0u, slo, (PIC_RNG_SELECT << 24) | (sp << 16), shi, k0, k1);
  McSelect r;
  r.r0 = o.v[0];
  r.r1 = o.v[1];
  return r;
}

PIC_HD uint32_t mcc_select_key(uint32_t id, McSelect k) { return mcc_hash32(mcc_hash32(id ^ k.r0) ^ k.r1); }

// Bounded selection: a key below `bound` enters bin floor(key 2^16 / bound)
// of a 65536-bin histogram and a compact list of (key << 32 | id, slot).
PIC_HD uint32_t mcc_bin(uint32_t key, uint64_t bound) { return (uint32_t)(((uint64_t)key << 16) / bound); }

// Where one species' bounded selection is built, by the key pass
// (k_mcc_scan) or by the push of the step (the particles it leaves live).
struct MccSink {
  int on;                   // 0: the push builds nothing
  McSelect rk;              // round keys of this step and species
  uint64_t bound;
  const uint32_t *id;       // particle ids (read by the push)
  uint32_t *hist;           // [65536]
  uint64_t *lkey;           // [cap]
  int32_t *lslot;           // [cap]
  int64_t cap;
  unsigned long long *cnt;  // list entries (may exceed cap: the selection then falls back)
};

#ifdef __CUDACC__
// One warp's particles (want: live and below the bound): one list
// reservation per warp; every lane takes part in the ballot.
__device__ __forceinline__ void mcc_sink_put(const MccSink &k, int lane, bool want, uint32_t key, uint32_t id,
                                             int64_t slot) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;  // the same for every lane of the warp
  const int leader = __ffs(m) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(k.cnt, (unsigned long long)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (want) {
    atomicAdd(k.hist + mcc_bin(key, k.bound), 1u);
    const int64_t i = (int64_t)base + __popc(m & ((1u << lane) - 1u));
    if (i < k.cap) {
      k.lkey[i] = ((uint64_t)key << 32) | (uint64_t)id;
      k.lslot[i] = (int32_t)slot;
    }
  }
}
#endif

static inline int64_t mcc_n_collisions(int64_t npar, double ratio, uint32_t slo, uint32_t shi,
                                       uint32_t sp, uint32_t k0, uint32_t k1) {
  double x = (double)npar * ratio;
  int64_t n = (int64_t)x;
  double residue = x - (double)n;
  pic_u32x4 o = pic_philox(0xFFFFFFFFu, slo, (PIC_RNG_RESIDUE << 24) | (sp << 16), shi, k0, k1);
  if (pic_u01(o.v[0], o.v[1]) < residue) ++n;
  return n;
}

PIC_HD void mc_rng_init(McRng *r, uint32_t id, uint32_t slo, uint32_t shi, uint32_t sp, uint32_t k0,
                        uint32_t k1) {
  r->id = id; r->slo = slo; r->shi = shi; r->sp = sp; r->k0 = k0; r->k1 = k1;
  r->call = 0; r->have = 0; r->buf[0] = r->buf[1] = 0.0;
}

PIC_HD double mc_u(McRng *r) {
  if (r->have == 0) {
    pic_u32x4 o = pic_philox(r->id, r->slo, (PIC_RNG_COLLIDE << 24) | (r->sp << 16) | r->call, r->shi,
                             r->k0, r->k1);
    r->call++;
    r->buf[0] = pic_u01(o.v[0], o.v[1]);
    r->buf[1] = pic_u01(o.v[2], o.v[3]);
    r->have = 2;
  }
  double u = r->buf[2 - r->have];
  r->have--;
  return u;
}

PIC_HD void mc_random_dir(McRng *r, double V, double v[3]) {
  double R = mc_u(r);
  double ct = 1.0 - 2.0 * R;
  double st = sqrt(1.0 - ct * ct);
  R = mc_u(r);
  double fai = 2.0 * PIC_PI * R;
  v[0] = V * ct;
  v[1] = V * st * cos(fai);
  v[2] = V * st * sin(fai);
}

PIC_HD void mc_maxwellian(McRng *r, double mass, double T, double v[3]) {
  double beta = 1.0 / (PIC_KB * T);
  double R = 0.5;
  for (int it = 0; it < 64; ++it) {
    R = mc_u(r);
    double fa = R * R;
    R = mc_u(r);
    if (R < 1e-300) R = 1e-300;
    double fb = -((PIC_FORTRAN_EXP * R) * log(R));
    if (!(fa > fb)) break;
  }
  double V = sqrt(((-3.0 * log(R)) / beta) / mass);
  mc_random_dir(r, V, v);
}

struct McState {
  double gx, gy, gz, gper, g, energy, mass_ratio;
};

// Vahedi (cos_type 0) or isotropic (cos_type 1) scattering of the relative velocity.
PIC_HD void mc_post_collision(McRng *r, McState *s, McParticle *P, int cos_type) {
  if (fabs(s->gper) < PIC_MINREAL) {
    double v[3];
    mc_random_dir(r, s->g, v);
    P->vx = v[0]; P->vy = v[1]; P->vz = v[2];
    return;
  }
  double ct;
  if (cos_type == 0) {
    if (s->energy < PIC_MINREAL) ct = 1.0;
    else {
      double R = mc_u(r);
      ct = ((s->energy + 2.0) - 2.0 * pow(s->energy + 1.0, R)) / s->energy;
    }
  } else {
    double R = mc_u(r);
    ct = 1.0 - 2.0 * R;
  }
  double fct = 1.0 - ct;
  double st = sqrt(1.0 - ct * ct);
  double R = mc_u(r);
  double aphi = 2.0 * PIC_PI * R;
  double cp = cos(aphi), sp = sin(aphi);
  double hx = s->gper * cp;
  double hy = -(s->gx * s->gy * cp + s->g * s->gz * sp) / s->gper;
  double hz = -(s->gx * s->gz * cp - s->g * s->gy * sp) / s->gper;
  P->vx = P->vx - s->mass_ratio * (s->gx * fct + hx * st);
  P->vy = P->vy - s->mass_ratio * (s->gy * fct + hy * st);
  P->vz = P->vz - s->mass_ratio * (s->gz * fct + hz * st);
}

PIC_HD void mc_scale(McState *s, McParticle *P, double f) {
  s->gx *= f; s->gy *= f; s->gz *= f; s->gper *= f; s->g *= f;
  P->vx *= f; P->vy *= f; P->vz *= f;
}

PIC_HD void mc_collide(McParticle *P, const McTable *t, const double *prob, const McGas *gas, double mass,
                       McRng *r, McOut *out) {
  out->reaction = 0;
  out->ionised = 0;
  // target gas particle (Updater)
  double vt[3];
  mc_maxwellian(r, gas->mass, gas->temperature, vt);
  McState s;
  double miu = mass * gas->mass / (mass + gas->mass);
  s.mass_ratio = gas->mass / (mass + gas->mass);
  s.gx = P->vx - vt[0];
  s.gy = P->vy - vt[1];
  s.gz = P->vz - vt[2];
  double gt = s.gy * s.gy + s.gz * s.gz;
  s.gper = sqrt(gt);
  double g2 = gt + s.gx * s.gx;
  s.g = sqrt(g2);
  s.energy = ((0.5 * miu) * g2) / PIC_JTOEV;
  // SelectProbility
  double E = s.energy;
  double tp[PIC_MAX_REACTIONS];
  double lg = log10(E);
  double pos = (lg - t->emin) / t->eint;
  double cpos = ceil(pos);
  int N = (cpos < -1.0e9) ? -1000000000 : (cpos > 1.0e9 ? 1000000000 : (int)cpos);
  for (int j = 0; j < t->nr; ++j) {
    if (N < 1) tp[j] = prob[j];
    else if (N < t->ns) {
      double S1 = (double)N - pos;
      double S2 = 1.0 - S1;
      tp[j] = prob[(size_t)(N - 1) * t->nr + j] * S1 + prob[(size_t)N * t->nr + j] * S2;
    } else {
      tp[j] = prob[(size_t)(t->ns - 1) * t->nr + j] * E / t->emax;
    }
    if (E < t->thr[j]) tp[j] = 0.0;
  }
  double R = mc_u(r);
  int idx = 0;
  for (int j = 0; j < t->nr; ++j)
    if (R < tp[j]) {
      idx = j + 1;
      break;
    }
  out->reaction = idx;
  if (idx == 0) return;
  int type = t->type[idx - 1];
  double thr = t->thr[idx - 1];
  if (type == 11) {
    mc_post_collision(r, &s, P, 0);
  } else if (type == 12) {
    double f = sqrt(1.0 - thr / s.energy);
    s.energy = s.energy - thr;
    mc_scale(&s, P, f);
    mc_post_collision(r, &s, P, 0);
  } else if (type == 13) {
    double v0[3] = {P->vx, P->vy, P->vz};
    double e0 = s.energy;
    double et = s.energy - thr;
    double Rr = mc_u(r);
    double eold = 10.0 * tan(Rr * atan(et) / 20.0);
    if (fabs(eold) < PIC_MINREAL) eold = PIC_MINREAL;
    double f = sqrt(eold / s.energy);
    mc_scale(&s, P, f);
    mc_post_collision(r, &s, P, 0);
    double enew = et - eold;
    double fn = sqrt(enew / e0);
    out->ionised = 1;
    for (int q = 0; q < 3; ++q) {
      out->e_new[q] = v0[q] * fn;
      out->ion_new[q] = vt[q];
    }
  } else if (type == 101) {
    mc_post_collision(r, &s, P, 1);
  } else if (type == 103) {
    P->vx = vt[0];
    P->vy = vt[1];
    P->vz = vt[2];
  }
}

#endif
