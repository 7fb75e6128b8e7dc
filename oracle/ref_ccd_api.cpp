// C entry points over the reference's own CPU CCD -- TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file together with the UNCHANGED reference
// sources silk/src/backend/cpu/collision/{ccd.cpp,interval_root_finder.cpp,
// interval.cpp} (read in place from the reference checkout) against the
// stand-in header oracle/ref_shim/Eigen/Core, into oracle/_ref/libref_ccd.so.
// Only the tests use it, to pin the oracle's CCD restatement and the GPU
// narrowphase to the reference's code bit for bit.
#include <cstdint>

#include "backend/cpu/collision/ccd.hpp"
#include "backend/cpu/collision/interval_root_finder.hpp"

namespace {

Eigen::Vector3f point(const float* x, int k) {
  return Eigen::Vector3f(x[3 * k], x[3 * k + 1], x[3 * k + 2]);
}

}  // namespace

extern "C" {

// One query: x24 = 4 points at t0 then the same 4 at t1 (vertex-face: the
// vertex first, then the face's three corners).  Calls
// silk::cpu::vertex_face_ccd / edge_edge_ccd (ccd.cpp:182-206).
// Returns 1 on a hit; t4 = (t lower, t upper, refined-separation t lower,
// refined-separation t upper); *use_small_ms = CCDResult::use_small_ms;
// *tolerance = CCDResult::tolerance.
int ref_ccd(int is_vf, const float* x24, const float* err3, float ms, float tol,
            long max_iter, int no_zero_toi, float max_time, float* t4,
            int* use_small_ms, float* tolerance) {
  Eigen::Array3f err(err3[0], err3[1], err3[2]);
  std::optional<silk::cpu::CCDResult> r;
  if (is_vf)
    r = silk::cpu::vertex_face_ccd(point(x24, 0), point(x24, 1), point(x24, 2),
                                   point(x24, 3), point(x24, 4), point(x24, 5),
                                   point(x24, 6), point(x24, 7), err, ms, tol,
                                   max_iter, no_zero_toi != 0, max_time);
  else
    r = silk::cpu::edge_edge_ccd(point(x24, 0), point(x24, 1), point(x24, 2),
                                 point(x24, 3), point(x24, 4), point(x24, 5),
                                 point(x24, 6), point(x24, 7), err, ms, tol,
                                 max_iter, no_zero_toi != 0, max_time);
  if (!r) return 0;
  t4[0] = r->t(0);
  t4[1] = r->t(1);
  t4[2] = r->small_ms_t(0);
  t4[3] = r->small_ms_t(1);
  *use_small_ms = r->use_small_ms ? 1 : 0;
  *tolerance = r->tolerance;
  return 1;
}

// silk::cpu::get_numerical_error (interval_root_finder.cpp:512-522).
void ref_numerical_error(const float* absmax3, int is_vf, float* out3) {
  Eigen::Array3f e = silk::cpu::get_numerical_error(
      Eigen::Vector3f(absmax3[0], absmax3[1], absmax3[2]), is_vf != 0);
  out3[0] = e(0);
  out3[1] = e(1);
  out3[2] = e(2);
}

}  // extern "C"
