// certify.hpp — rigorous verification of the engine's answers on the ORIGINAL model:
//   certified_dual_bound  a rounding-error-proof bound on the optimum from any row multipliers
//                         (reference src/core/safe_bound.{h,cpp}; Neumaier & Shcherbina, "Safe
//                         bounds in linear and mixed-integer linear programming", Math. Prog. 99,
//                         2004), with double-double sums and an explicit error bound
//   implied_bounds        feasibility-based bound tightening with outward rounding, used when a
//                         column bounded on one side only makes the plain bound −∞
//                         (reference src/core/implied_bounds.{h,cpp})
//   check_infeasibility_certificate / check_unboundedness_certificate
//                         the Farkas and recession-ray checks of Infeasible / Unbounded claims
//                         (reference src/core/certificates.{h,cpp})
// Host C++. The per-column work of the bound runs on all host threads; every sum is taken in
// the reference's order, so the bound's bits do not depend on the thread count.
#pragma once

#include <string>
#include <vector>

#include "solver.hpp"

namespace b200 {

struct SafeBound {
  bool finite = false;
  double bound = 0.0;  // MIN model: ≤ the optimum; MAX model: ≥ the optimum (offset included)
  int unbounded_row_terms = 0, unbounded_col_terms = 0;
};
// y: row multipliers in the model's own sense (Solution::y). use_implied_bounds = false skips the
// bound-tightening refinement (the result is still rigorous, possibly infinite).
SafeBound certified_dual_bound(const Model& model, const std::vector<double>& y, bool use_implied_bounds = true);

struct ImpliedBounds {
  std::vector<double> lower, upper;
  int tightened = 0;  // infinite model bounds made finite
};
ImpliedBounds implied_bounds(const Model& model, int max_passes = 20);

struct CertificateCheck {
  bool present = false, passed = false, rigorous = false;
  double measure = 0.0, violation = 0.0;
  std::string detail;
};
CertificateCheck check_infeasibility_certificate(const Model& model, const std::vector<double>& dual_ray);
CertificateCheck check_unboundedness_certificate(const Model& model, const std::vector<double>& x,
                                                 const std::vector<double>& primal_ray);

}  // namespace b200
