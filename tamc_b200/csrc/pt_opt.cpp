// pt_opt.cpp -- the temperature-ladder update of tamc-pt-opt
// (pt_optimize_beta, src/bin/tamc-pt-opt.rs:37-190): from the round trips and
// diffusion histograms that PT runs at the current ladder recorded, place
// the next ladder so that the normalised inverse-temperature density eta,
// derived from the flow of replicas between the ends of the ladder, gives
// every interval the same mass; blend it with a momentum term.
//
// All arithmetic is f32 in the reference's order, with ndarray's sums
// (eight-way unrolled fold over contiguous data) and tamc-core's helpers
// (tamc-core/src/util.rs): finite_differences, StepwiseMeasure,
// monotonic_divisions by nested bisection.  Linear interpolation restates
// the interp crate (0.1.x, a dependency outside the reference tree): the
// segment that starts at the last knot below the point, among all but the
// last knot (the first segment when none is below), evaluated as
// slope * x + intercept, which extrapolates beyond the ends.
#include <cmath>
#include <cstdio>
#include <vector>

#include "internal.h"

namespace tamc {
namespace {

// ndarray 0.15 numeric_util::unrolled_fold with addition from 0.0
float nd_sum(const float* x, size_t n) {
  float acc = 0.0f;
  float p[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  size_t k = 0;
  for (; k + 8 <= n; k += 8)
    for (int j = 0; j < 8; ++j) p[j] = p[j] + x[k + j];
  acc = acc + (p[0] + p[4]);
  acc = acc + (p[1] + p[5]);
  acc = acc + (p[2] + p[6]);
  acc = acc + (p[3] + p[7]);
  for (; k < n; ++k) acc = acc + x[k];
  return acc;
}

// tamc-core/src/util.rs:5-21
std::vector<float> finite_differences(const std::vector<float>& x, const std::vector<float>& y) {
  const size_t n = x.size();
  std::vector<float> dx(n - 1), dy(n - 1), d(n, 0.0f);
  for (size_t i = 0; i + 1 < n; ++i) {
    dx[i] = x[i + 1] - x[i];
    dy[i] = y[i + 1] - y[i];
  }
  d[0] = dy[0] / dx[0];
  d[n - 1] = dy[n - 2] / dx[n - 2];
  for (size_t i = 1; i + 1 < n; ++i)
    d[i] = (dy[i - 1] * dx[i] / dx[i - 1] + dy[i] * dx[i - 1] / dx[i]) / (dx[i - 1] + dx[i]);
  return d;
}

// interp 0.1: linear interpolation / extrapolation of (x, y) at xp
float interp(const std::vector<float>& x, const std::vector<float>& y, float xp) {
  const size_t n = std::min(x.size(), y.size());
  if (n == 0) return 0.0f;
  if (n == 1) return y[0];
  size_t i = 0;
  for (size_t k = n - 1; k-- > 0;)
    if (x[k] < xp) { i = k; break; }
  const float slope = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
  const float intercept = y[i] - slope * x[i];
  return slope * xp + intercept;
}

struct EtaFn {
  const std::vector<float>* beta;
  const std::vector<float>* cdf;
  float bmin, bmax;
  float operator()(float x) const { return interp(*beta, *cdf, bmin + x * (bmax - bmin)); }
};

// monotonic_bisection (tamc-core/src/util.rs:56-84); false where the reference panics
bool bisection(const EtaFn& f, float y0, float xmin, float xmax, float& root) {
  const float tol = 1.0e-6f;
  if (!(xmin < xmax)) return false;  // assert!(xmin < xmax)
  float x0 = xmin, x1 = xmax;
  for (uint32_t it = 0; it < 1000000u; ++it) {
    const float xmid = (x0 + x1) / 2.0f;
    const float y = f(xmid);
    if (std::fabs(y - y0) < tol) {
      root = xmid;
      return true;
    }
    if (std::fabs(xmid - xmin) < tol) return false;  // LoBnd
    if (std::fabs(xmid - xmax) < tol) return false;  // UpBnd
    if (y < y0) x0 = xmid;
    else x1 = xmid;
  }
  return false;  // Failed
}

// bisect_array (tamc-core/src/util.rs:88-116): the middle root first, then
// each half within the bracket it leaves
bool bisect_array(const EtaFn& f, float* roots, const float* ytgt, size_t n, float xmin, float xmax) {
  if (n == 0) return true;
  if (n == 1) return bisection(f, ytgt[0], xmin, xmax, roots[0]);
  const size_t mid = n / 2;
  if (!bisect_array(f, roots + mid, ytgt + mid, 1, xmin, xmax)) return false;
  const float xmid = roots[mid];
  return bisect_array(f, roots, ytgt, mid, xmin, xmid) &&
         bisect_array(f, roots + mid + 1, ytgt + mid + 1, n - mid - 1, xmid, xmax);
}

}  // namespace
}  // namespace tamc

using namespace tamc;

extern "C" int tamc_pt_opt_step(uint32_t nt, float* betas, float* momentum, uint32_t num_instances,
                                const uint32_t* round_trips, const uint32_t* dhist, uint32_t num_sweeps,
                                uint32_t num_chains, float alpha, float m, float* tau, float* err) {
  TAMC_API_BEGIN
  if (nt < 3) fail(TAMC_E_INVAL, "the ladder needs at least 3 temperatures");
  if (!betas || !momentum || !round_trips || !dhist || !tau || !err || num_instances == 0)
    fail(TAMC_E_INVAL, "null argument");
  const std::vector<float> beta(betas, betas + nt);
  // StepwiseMeasure::new (tamc-core/src/util.rs:28-45)
  std::vector<float> weights(nt, 0.0f), difs(nt - 1);
  for (uint32_t i = 0; i + 1 < nt; ++i) difs[i] = beta[i + 1] - beta[i];
  weights[0] = difs[0] / 2.0f;
  for (uint32_t i = 1; i + 1 < nt; ++i) weights[i] = (difs[i - 1] + difs[i]) / 2.0f;
  weights[nt - 1] = difs[nt - 2] / 2.0f;
  // per instance: round-trip time and the finite-difference slope of the
  // fraction of visits that came from the top of the ladder
  std::vector<std::vector<float>> d_dif(num_instances);
  for (uint32_t s = 0; s < num_instances; ++s) {
    const uint32_t rts = round_trips[s];
    const float rt_per_rep = (float)rts / (float)(num_chains * nt);
    tau[s] = rts == 0 ? 0.0f : (float)num_sweeps / rt_per_rep;
    std::vector<float> probs(nt);
    for (uint32_t t = 0; t < nt; ++t) {
      const float a = (float)(dhist[((size_t)s * nt + t) * 2] + 1u);      // pseudocount of 1
      const float b = (float)(dhist[((size_t)s * nt + t) * 2 + 1] + 1u);
      probs[t] = b / (a + b);
    }
    d_dif[s] = finite_differences(beta, probs);
  }
  const float sum_tau = nd_sum(tau, num_instances);
  std::vector<float> wdd(nt, 0.0f);
  for (uint32_t s = 0; s < num_instances; ++s)
    for (uint32_t t = 0; t < nt; ++t) wdd[t] = wdd[t] + tau[s] * d_dif[s][t];
  for (uint32_t t = 0; t < nt; ++t) wdd[t] = wdd[t] / sum_tau;
  std::vector<float> eta(nt), eta_w(nt - 1);
  for (uint32_t t = 0; t < nt; ++t) eta[t] = std::sqrt(std::fmax(wdd[t] / weights[t], 0.0f));  // f32::max: NaN -> 0
  for (uint32_t t = 0; t + 1 < nt; ++t) eta_w[t] = ((eta[t] + eta[t + 1]) / 2.0f) * difs[t];
  const float z = nd_sum(eta_w.data(), nt - 1);
  if (z < 1.1920929e-7f) return 1;  // "Insufficient round trips for eta CDF" (f32::EPSILON): ladder unchanged
  std::vector<float> cdf(nt);
  float acc = 0.0f;
  for (uint32_t t = 0; t + 1 < nt; ++t) {
    cdf[t] = acc;
    acc += eta_w[t] / z;
  }
  cdf[nt - 1] = 1.0f;
  const EtaFn f{&beta, &cdf, beta[0], beta[nt - 1]};
  // monotonic_divisions (tamc-core/src/util.rs:121-137) into nt - 1 intervals
  std::vector<float> xd(nt, 0.0f), tgt(nt - 2);
  xd[nt - 1] = 1.0f;
  for (uint32_t i = 1; i + 1 < nt; ++i) tgt[i - 1] = (float)((double)i / (double)(nt - 1));
  if (!bisect_array(f, xd.data() + 1, tgt.data(), nt - 2, 0.0f, 1.0f))
    fail(TAMC_E_REFPANIC, "bisection for the eta CDF ended at a bound or failed (the reference panics)");
  std::vector<float> calc(nt);
  for (uint32_t t = 0; t < nt; ++t) calc[t] = xd[t] * (beta[nt - 1] - beta[0]) + beta[0];
  for (uint32_t t = 0; t < nt; ++t) momentum[t] = std::exp(m * std::log(momentum[t]) + (1.0f - m) * std::log(calc[t]));
  float e = 0.0f;
  std::vector<float> out(calc);
  for (uint32_t t = 1; t + 1 < nt; ++t) {
    const float b = std::exp(alpha * std::log(momentum[t]) + (1.0f - alpha) * std::log(beta[t]));
    e += std::fabs(std::log10(out[t]) - std::log10(beta[t]));
    out[t] = b;
  }
  *err = e / (float)nt;
  for (uint32_t t = 0; t < nt; ++t) betas[t] = out[t];
  TAMC_API_END
}
