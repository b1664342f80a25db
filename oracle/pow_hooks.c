/* pow_hooks.c -- pow() replacements for builds of the C oracle (TEST
 * INFRASTRUCTURE; linked only into liboracle_cr.so and liboracle_powcmp.so).
 *
 * or_cr_pow:     the correctly rounded pow() the engine's entropy fix uses
 *                (coolharm3d_b200/csrc/hg_crpow.h): the oracle built with it
 *                is the reference's algorithm evaluated with that pow(), and
 *                the engine must reproduce it bit for bit.
 * or_pow_cmp:    glibc's pow() (so the step follows the reference exactly),
 *                counting the calls and the calls where the correctly rounded
 *                pow() returns a different double; the first mismatching
 *                arguments are kept for inspection.
 * or_cr_pow_raw: hg_cr_pow itself, for direct tests against exact values.
 * or_pow_ulp_up: glibc's pow() moved up by one ulp, to measure how far the
 *                reference's own step carries a one-ulp change of pow(). */
#include <math.h>
#include <stdint.h>

#include "../coolharm3d_b200/csrc/hg_crpow.h"

double or_cr_pow(double x, double y) { return hg_cr_pow(x, y); }
double or_cr_pow_raw(double x, double y) { return hg_cr_pow(x, y); }
double or_pow_ulp_up(double x, double y) { return nextafter(pow(x, y), INFINITY); }

#define OR_POW_KEEP 64
static uint64_t n_calls = 0, n_diff = 0;
static double kept[OR_POW_KEEP][2];

double or_pow_cmp(double x, double y)
{
  const double a = pow(x, y);
  const double b = hg_cr_pow(x, y);
  n_calls++;
  if (a != b && !(a != a && b != b)) {
    if (n_diff < OR_POW_KEEP) {
      kept[n_diff][0] = x;
      kept[n_diff][1] = y;
    }
    n_diff++;
  }
  return a;
}

/* counts since the last reset; args receives up to OR_POW_KEEP (x, y) pairs */
void or_pow_counts(uint64_t *calls, uint64_t *diffs, double *args)
{
  *calls = n_calls;
  *diffs = n_diff;
  for (uint64_t i = 0; args && i < n_diff && i < OR_POW_KEEP; i++) {
    args[2 * i] = kept[i][0];
    args[2 * i + 1] = kept[i][1];
  }
}

void or_pow_reset(void) { n_calls = n_diff = 0; }
