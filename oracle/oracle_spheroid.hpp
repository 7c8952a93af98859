// TEST INFRASTRUCTURE ONLY: one spheroid node of the adaptive ensemble's direct path
// (scatrs/src/ensemble/particle.rs:256-366), solved by the oracle's double-precision EBCM
// (oracle_tmatrix.cpp) and orientation average (oracle_random.cpp).
#pragma once

#include <vector>

#include "oracle_core.hpp"

namespace orc {

struct SpheroidNode {
  int n = 0, nth = 0;
  double q_ext = 0, q_sca = 0, q_abs = 0, q_back = 0, g = 0;
  double depol = 0;           // Q_back - Q_sca F22(180 deg) (particle.rs:276-285)
  std::vector<double> greek;  // unnormalized (alpha1_0 = Q_sca), [6][2N + 1]
};

// The spheroid of equal-volume size parameter x, aspect ratio eps and index s, converged to
// rtol as driver.rs:343-420 converges it. Returns 0 or the status (1 invalid, 2 not converged).
int spheroid_node(double x, double eps, cplx s, double rtol, SpheroidNode* out);

}  // namespace orc
