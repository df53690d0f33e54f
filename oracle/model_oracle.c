/*
 * CPU oracle for the learned position model.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference has no learned model (it narrows searches with 128-cell rank
 * directories, GPULSMOpt.cuh:4605-4646); this file restates, in float64, the
 * model the GPU trains (piecewise-linear CDF over equal-width key segments) so
 * the GPU's forward/backward kernels can be checked:
 *   s     = min((key - kmin) >> shift, nseg - 1)
 *   xhat  = ((key - kmin) - (s << shift)) / 2^shift - 1/2
 *   r_i   = b_s + a_s * xhat_i - i
 *   L     = (1/N) sum r_i^2,  dL/da_s = (2/N) sum r_i xhat_i,  dL/db_s = (2/N) sum r_i
 */
#include <stdint.h>
#include <string.h>

void orc_model_gradients(const uint64_t *keys, uint64_t n, uint64_t kmin, uint32_t shift, uint32_t nseg,
                         const float *a, const float *b, double *ga, double *gb, double *loss) {
  memset(ga, 0, nseg * sizeof(double));
  memset(gb, 0, nseg * sizeof(double));
  double l = 0.0;
  const double scale = 1.0 / (double)(1ull << shift);
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t d = keys[i] - kmin;
    uint64_t s = d >> shift;
    if (s >= nseg) s = nseg - 1;
    const double xh = (double)(d - (s << shift)) * scale - 0.5;
    const double r = (double)b[s] + (double)a[s] * xh - (double)i;
    ga[s] += r * xh;
    gb[s] += r;
    l += r * r;
  }
  const double inv = n ? 1.0 / (double)n : 0.0;
  for (uint32_t s = 0; s < nseg; ++s) {
    ga[s] *= 2.0 * inv;
    gb[s] *= 2.0 * inv;
  }
  *loss = l * inv;
}
