/*
 * oracle_tables.c -- the oracle's own restatement (FP64) of the MCC_jw
 * collision-table set-up: the normalised cross sections on the log-energy
 * grid and the cumulative collision probabilities with the null-collision
 * ratio.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/ load it.  It takes the raw
 * (energy [eV], sigma [cm^2]) points of each reaction as the Pegasus files
 * hold them and builds the tables without any code of the product's table
 * builder (pic_b200/mcc_tables.py), so that a test can compare the two.
 *
 * Reference paths are relative to PIC-IFE_GEC/MCC_jw/code of weqwoueu/pic-.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

/* Numrical.F90 `Locate` (Numerical Recipes' bisection) on xx[1..n], 1-based;
 * 0 or n when x is outside. */
static int nr_locate(const double *xx, int n, double x) {
  int jl = 0, ju = n + 1;
  const int asc = xx[n - 1] >= xx[0];
  while (ju - jl > 1) {
    int jm = (ju + jl) / 2;
    if (asc == (x >= xx[jm - 1])) jl = jm;
    else ju = jm;
  }
  if (x == xx[0]) return 1;
  if (x == xx[n - 1]) return n - 1;
  return jl;
}

/* SigmaNormalizedUpdate (mc/MCCSigma.f90:123-172) for one reaction, after
 * ConvertReactionOnePegasus2SigmaRaw (mc/ReactionOnePegasus.f90:444-450:
 * sigma / 1e4, cm^2 -> m^2).  n_raw points e_raw[], s_raw_cm2[];
 * out[nsigma] = sigma(E_i) in m^2 on E_i = 10^(emin + (i-1) eint).
 * Returns 0, or -1 for a bad table. */
int or_mcc_sigma(int n_raw, const double *e_raw, const double *s_raw_cm2, double threshold, double emin,
                 double eint, int nsigma, double *out) {
  if (n_raw < 2 || nsigma < 1) return -1;
  double *ix = malloc(sizeof(double) * (size_t)n_raw);
  double *sg = malloc(sizeof(double) * (size_t)n_raw);
  if (!ix || !sg) { free(ix); free(sg); return -1; }
  /* Maxloc of the raw energies: the table ends at its largest energy */
  int nraw = 1;
  for (int i = 1; i < n_raw; ++i)
    if (e_raw[i] > e_raw[nraw - 1]) nraw = i + 1;
  for (int i = 0; i < n_raw; ++i) sg[i] = s_raw_cm2[i] / 1.0e4;
  const double max_energy = e_raw[nraw - 1];
  const double alfa = sg[nraw - 1] * max_energy;
  /* raw energies -> fractional grid index; below 10^Emin the reference
   * stores Emin itself (not an index) */
  for (int i = 0; i < nraw; ++i)
    ix[i] = e_raw[i] < pow(10.0, emin) ? emin : (log10(e_raw[i]) - emin) / eint;
  for (int i = 1; i <= nsigma; ++i) {
    const double nenergy = (double)(i - 1);
    const double energy = pow(10.0, emin + (double)(i - 1) * eint);
    double s;
    if (energy <= threshold) s = 0.0;
    else if (energy >= max_energy) s = alfa / energy;
    else {
      int k = nr_locate(ix, nraw, nenergy);
      if (k < 1) k = 1;
      const double le = ix[k - 1], ue = ix[k];
      const double s1 = ((double)i - le) / (ue - le), s2 = 1.0 - s1;
      s = s2 * sg[k - 1] + s1 * sg[k];
    }
    out[i - 1] = s;
  }
  free(ix);
  free(sg);
  return 0;
}

/* ProbilityNonReactive (mc/MCCInit.F90:107-152) and the collision ratio of
 * MCCBundleElelctronInit / MCCBundleIonInit (MCCInit.F90:54, 88):
 * sigma [nr][ns] (row per reaction) -> prob [ns][nr] = cumulative over
 * reactions of sigma v n_gas, divided by its maximum; out3 = {SigmaMax,
 * CollisionRatio = 1 - exp(-SigmaMax dt), EnergyMax = 10^emax}. */
void or_mcc_probability(int nr, int ns, const double *sigma, double mass, double gas_mass, double n_gas,
                        double emin, double eint, double emax, double dt, double jtoev, double *prob,
                        double *out3) {
  const double miu = mass * gas_mass / (mass + gas_mass);
  for (int i = 1; i <= ns; ++i) {
    const double energy = pow(10.0, emin + (double)(i - 1) * eint);
    const double v = sqrt(2.0 * energy * jtoev / miu);
    for (int j = 0; j < nr; ++j) prob[(size_t)(i - 1) * nr + j] = sigma[(size_t)j * ns + (i - 1)] * v * n_gas;
  }
  for (int i = 0; i < ns; ++i)
    for (int j = 1; j < nr; ++j) prob[(size_t)i * nr + j] = prob[(size_t)i * nr + j] + prob[(size_t)i * nr + j - 1];
  double mx = 0.0;
  for (size_t q = 0; q < (size_t)ns * nr; ++q)
    if (prob[q] > mx) mx = prob[q];
  for (size_t q = 0; q < (size_t)ns * nr; ++q) prob[q] = prob[q] / mx;
  out3[0] = mx;
  out3[1] = 1.0 - exp(-mx * dt);
  out3[2] = pow(10.0, emax);
}
