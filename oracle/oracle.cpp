// CPU oracle for the Silk per-step cloth hot path.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU-baseline legs of bench.py as the checker.  Never part of the product.
//
// Every routine restates the reference algorithm it cites (paths relative to
// the reference project root).  The solver path is templated on the scalar
// type: float reproduces the reference's FP32 arithmetic for parity runs,
// double gives the FP64 error reference.  Continuous collision detection is
// always evaluated in float with the reference's exact operation order
// (this file is compiled with -ffp-contract=off).
#include "oracle_api.h"

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <optional>
#include <set>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

using u32 = uint32_t;
using u64 = uint64_t;

// ---------------------------------------------------------------------------
// Small fixed-size vector helpers (float, used by collision code).
// ---------------------------------------------------------------------------
struct V3 {
  float x[3];
  float& operator()(int i) { return x[i]; }
  float operator()(int i) const { return x[i]; }
};
static inline V3 v3(float a, float b, float c) { return V3{{a, b, c}}; }
static inline V3 vsub(const V3& a, const V3& b) {
  return v3(a(0) - b(0), a(1) - b(1), a(2) - b(2));
}
static inline V3 vadd(const V3& a, const V3& b) {
  return v3(a(0) + b(0), a(1) + b(1), a(2) + b(2));
}
static inline V3 vscale(float s, const V3& a) {
  return v3(s * a(0), s * a(1), s * a(2));
}
// axpby as in simple_linalg.cuh:330-345: a*x + b*y per element.
static inline V3 axpby(float a, const V3& x, float b, const V3& y) {
  return v3(a * x(0) + b * y(0), a * x(1) + b * y(1), a * x(2) + b * y(2));
}
static inline float dot3(const V3& a, const V3& b) {
  return a(0) * b(0) + a(1) * b(1) + a(2) * b(2);
}
static inline float fmin_std(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_std(float a, float b) { return (a < b) ? b : a; }
static inline V3 vmin(const V3& a, const V3& b) {
  return v3(fmin_std(a(0), b(0)), fmin_std(a(1), b(1)), fmin_std(a(2), b(2)));
}
static inline V3 vmax(const V3& a, const V3& b) {
  return v3(fmax_std(a(0), b(0)), fmax_std(a(1), b(1)), fmax_std(a(2), b(2)));
}

// ---------------------------------------------------------------------------
// Bbox (collision/bbox.cuh:10-37).
// ---------------------------------------------------------------------------
struct Bbox {
  V3 mn, mx;
};
static inline Bbox bbox_merge(const Bbox& a, const Bbox& b) {
  return {vmin(a.mn, b.mn), vmax(a.mx, b.mx)};
}
static inline Bbox bbox_pad(const Bbox& b, float p) {
  // axpb(1.0f, min, -padding): 1*x + b.
  return {v3(1.0f * b.mn(0) + -p, 1.0f * b.mn(1) + -p, 1.0f * b.mn(2) + -p),
          v3(1.0f * b.mx(0) + p, 1.0f * b.mx(1) + p, 1.0f * b.mx(2) + p)};
}
// Overlap test uses <= (bbox.cuh:25-29): touching boxes collide.
static inline bool bbox_colliding(const Bbox& a, const Bbox& b) {
  V3 mxmn = vmax(a.mn, b.mn);
  V3 mnmx = vmin(a.mx, b.mx);
  return mxmn(0) <= mnmx(0) && mxmn(1) <= mnmx(1) && mxmn(2) <= mnmx(2);
}

// ---------------------------------------------------------------------------
// Tight-Inclusion CCD, restated from the reference's in-tree CPU version
// (backend/cpu/collision/ccd.cpp:13-204, interval_root_finder.cpp:13-522,
// interval.cpp:5-11).  Float arithmetic, no contraction.
// ---------------------------------------------------------------------------
struct Interval {
  float lower, upper;
};
using IBox = std::array<Interval, 3>;

struct CCDResult {
  float t0, t1;
  float tolerance;
  bool use_small_ms;
  float small_t0, small_t1;
};

struct Coeffs {
  float c0[3], c1[3], c2[3], c3[3], c4[3], c5[3];
};

// interval.cpp:7-11: midpoint split.
static inline std::pair<Interval, Interval> bisect(const Interval& i) {
  float mid = (i.upper + i.lower) / 2;
  return {Interval{i.lower, mid}, Interval{mid, i.upper}};
}

// interval_root_finder.cpp:31-100.
template <bool VF>
static bool eval_unit_bbox_1d(const V3* P /*a0 b0 c0 d0 a1 b1 c1 d1*/,
                              float eps, float ms, int dim, bool& in_eps,
                              float& tol) {
  float minv, maxv;
  if (VF) {
    float A[6] = {P[0](dim), P[0](dim), P[0](dim),
                  P[4](dim), P[4](dim), P[4](dim)};
    float B[6] = {P[1](dim), P[2](dim), P[3](dim),
                  P[5](dim), P[6](dim), P[7](dim)};
    float D[6];
    for (int i = 0; i < 6; ++i) D[i] = A[i] - B[i];
    minv = D[0];
    maxv = D[0];
    for (int i = 1; i < 6; ++i) {
      if (D[i] < minv) minv = D[i];
      if (D[i] > maxv) maxv = D[i];
    }
  } else {
    float A[8] = {P[0](dim), P[0](dim), P[1](dim), P[1](dim),
                  P[4](dim), P[4](dim), P[5](dim), P[5](dim)};
    float B[8] = {P[2](dim), P[3](dim), P[2](dim), P[3](dim),
                  P[6](dim), P[7](dim), P[6](dim), P[7](dim)};
    float D[8];
    for (int i = 0; i < 8; ++i) D[i] = A[i] - B[i];
    minv = D[0];
    maxv = D[0];
    for (int i = 1; i < 8; ++i) {
      if (D[i] < minv) minv = D[i];
      if (D[i] > maxv) maxv = D[i];
    }
  }
  tol = maxv - minv;
  in_eps = false;
  const float eps_and_ms = eps + ms;
  if (minv > eps_and_ms || maxv < -eps_and_ms) return false;
  if (minv >= -eps_and_ms && maxv <= eps_and_ms) in_eps = true;
  return true;
}

// interval_root_finder.cpp:102-212.
static bool eval_vf_bbox_1d(const IBox& tuv, const Coeffs& co, float eps_ms,
                            int dim, bool& in_eps, float& tol) {
  float t_lo = tuv[0].lower, t_up = tuv[0].upper;
  float u_lo = tuv[1].lower, u_up = tuv[1].upper;
  float v_lo = tuv[2].lower, v_up = tuv[2].upper;
  float c0 = co.c0[dim], c1 = co.c1[dim], c2 = co.c2[dim], c3 = co.c3[dim],
        c4 = co.c4[dim], c5 = co.c5[dim];
  auto at_t = [&](float t, float& mn, float& mx) {
    float a = (c1 - c0) * t + c0;
    float b = (c3 - c2) * t + c2;
    float c = (c5 - c4) * t + c4;
    if (u_up + v_up <= 1.0f) {
      float bl = b * u_lo, bu = b * u_up, cl = c * v_lo, cu = c * v_up;
      mn = a + fmin_std(bl, bu) + fmin_std(cl, cu);
      mx = a + fmax_std(bl, bu) + fmax_std(cl, cu);
      return;
    }
    mn = std::numeric_limits<float>::infinity();
    mx = -std::numeric_limits<float>::infinity();
    auto inc = [&](float u, float v) {
      float val = a + b * u + c * v;
      mn = fmin_std(mn, val);
      mx = fmax_std(mx, val);
    };
    if (u_lo + v_lo <= 1.0f) inc(u_lo, v_lo);
    if (u_lo + v_up <= 1.0f) inc(u_lo, v_up);
    if (u_up + v_lo <= 1.0f) inc(u_up, v_lo);
    if (u_up + v_up <= 1.0f) inc(u_up, v_up);
    float v_at_u_lo = 1.0f - u_lo;
    if (v_at_u_lo >= v_lo && v_at_u_lo <= v_up) inc(u_lo, v_at_u_lo);
    float v_at_u_up = 1.0f - u_up;
    if (v_at_u_up >= v_lo && v_at_u_up <= v_up) inc(u_up, v_at_u_up);
    float u_at_v_lo = 1.0f - v_lo;
    if (u_at_v_lo >= u_lo && u_at_v_lo <= u_up) inc(u_at_v_lo, v_lo);
    float u_at_v_up = 1.0f - v_up;
    if (u_at_v_up >= u_lo && u_at_v_up <= u_up) inc(u_at_v_up, v_up);
  };
  float mn0, mx0, mn1, mx1;
  at_t(t_lo, mn0, mx0);
  at_t(t_up, mn1, mx1);
  float minv = fmin_std(mn0, mn1);
  float maxv = fmax_std(mx0, mx1);
  in_eps = false;
  if (minv > eps_ms || maxv < -eps_ms) return false;
  tol = maxv - minv;
  if (minv >= -eps_ms && maxv <= eps_ms) in_eps = true;
  return true;
}

// interval_root_finder.cpp:214-276.
static bool eval_ee_bbox_1d(const IBox& tuv, const Coeffs& co, float eps_ms,
                            int dim, bool& in_eps, float& tol) {
  float t_lo = tuv[0].lower, t_up = tuv[0].upper;
  float u_lo = tuv[1].lower, u_up = tuv[1].upper;
  float v_lo = tuv[2].lower, v_up = tuv[2].upper;
  float c0 = co.c0[dim], c1 = co.c1[dim], c2 = co.c2[dim], c3 = co.c3[dim],
        c4 = co.c4[dim], c5 = co.c5[dim];
  auto at_t = [&](float t, float& mn, float& mx) {
    float a = (c1 - c0) * t + c0;
    float b = (c3 - c2) * t + c2;
    float c = (c5 - c4) * t + c4;
    float bl = b * u_lo, bu = b * u_up, cl = c * v_lo, cu = c * v_up;
    mn = a + fmin_std(bl, bu) + fmin_std(cl, cu);
    mx = a + fmax_std(bl, bu) + fmax_std(cl, cu);
  };
  float mn0, mx0, mn1, mx1;
  at_t(t_lo, mn0, mx0);
  at_t(t_up, mn1, mx1);
  float minv = fmin_std(mn0, mn1);
  float maxv = fmax_std(mx0, mx1);
  in_eps = false;
  if (minv > eps_ms || maxv < -eps_ms) return false;
  tol = maxv - minv;
  if (minv >= -eps_ms && maxv <= eps_ms) in_eps = true;
  return true;
}

// interval_root_finder.cpp:280-320.
template <bool VF>
static bool origin_in_bbox_eval(const IBox& tuv, const V3* P, const float* eps,
                                float ms, bool unit, bool& in_eps, float* tol,
                                const Coeffs& co) {
  bool xyz[3];
  in_eps = false;
  for (int dim = 0; dim < 3; ++dim) {
    bool ok;
    if (unit) {
      ok = eval_unit_bbox_1d<VF>(P, eps[dim], ms, dim, xyz[dim], tol[dim]);
    } else if (VF) {
      ok = eval_vf_bbox_1d(tuv, co, eps[dim] + ms, dim, xyz[dim], tol[dim]);
    } else {
      ok = eval_ee_bbox_1d(tuv, co, eps[dim] + ms, dim, xyz[dim], tol[dim]);
    }
    if (!ok) return false;
  }
  in_eps = xyz[0] && xyz[1] && xyz[2];
  return true;
}

// interval_root_finder.cpp:323-330: largest relative width above tolerance;
// Eigen maxCoeff keeps the first maximum.
static int find_next_split(const float* w, const float* tol) {
  float tmp[3];
  for (int i = 0; i < 3; ++i)
    tmp[i] = (w[i] > tol[i]) ? w[i] / tol[i]
                             : -std::numeric_limits<float>::infinity();
  int best = 0;
  for (int i = 1; i < 3; ++i)
    if (tmp[i] > tmp[best]) best = i;
  return best;
}

// Largest number of pending boxes seen by any search (sizes GPU storage).
static thread_local size_t g_max_pending = 0;

// interval_root_finder.cpp:390-510 (bucket DFS keyed by t.lower).
template <bool VF>
static std::optional<CCDResult> root_finder_bucket_dfs(
    const V3* P, const IBox& iset, const float* tol, float co_tol,
    const float* err, float ms, long max_iter, bool is_unit) {
  std::map<float, std::vector<IBox>> stacks;
  IBox cur = iset;
  bool has_cur = true;
  long iter = 0;
  Coeffs co;
  for (int d = 0; d < 3; ++d) {
    if (VF) {
      co.c0[d] = P[0](d) - P[1](d);
      co.c1[d] = P[4](d) - P[5](d);
      co.c2[d] = P[1](d) - P[2](d);
      co.c3[d] = P[5](d) - P[6](d);
      co.c4[d] = P[1](d) - P[3](d);
      co.c5[d] = P[5](d) - P[7](d);
    } else {
      co.c0[d] = P[0](d) - P[2](d);
      co.c1[d] = P[4](d) - P[6](d);
      co.c2[d] = P[1](d) - P[0](d);
      co.c3[d] = P[5](d) - P[4](d);
      co.c4[d] = P[2](d) - P[3](d);
      co.c5[d] = P[6](d) - P[7](d);
    }
  }
  while (has_cur || !stacks.empty()) {
    auto bucket = stacks.end();
    if (!has_cur) {
      bucket = stacks.begin();
      cur = bucket->second.back();
      bucket->second.pop_back();
    }
    has_cur = false;
    ++iter;
    bool in_eps;
    float w_img[3];
    bool in_zero = origin_in_bbox_eval<VF>(cur, P, err, ms, is_unit, in_eps,
                                           w_img, co);
    is_unit = false;
    if (!in_zero) {
      if (bucket != stacks.end() && bucket->second.empty()) stacks.erase(bucket);
      continue;
    }
    bool small = (w_img[0] <= co_tol) && (w_img[1] <= co_tol) &&
                 (w_img[2] <= co_tol);
    if (small || in_eps) {
      return CCDResult{cur[0].lower, cur[0].upper, co_tol, false, 0.f, 0.f};
    }
    if (max_iter > 0 && iter > max_iter) {
      float mx = fmax_std(fmax_std(w_img[0], w_img[1]), w_img[2]);
      return CCDResult{cur[0].lower, cur[0].upper, fmax_std(co_tol, mx), false,
                       0.f, 0.f};
    }
    float widths[3] = {cur[0].upper - cur[0].lower, cur[1].upper - cur[1].lower,
                       cur[2].upper - cur[2].lower};
    int split = find_next_split(widths, tol);
    auto halves = bisect(cur[split]);
    // split_and_push (interval_root_finder.cpp:332-365).
    constexpr float SPLIT_LOWER_BOUND = 1e-12f;
    if (halves.first.upper < SPLIT_LOWER_BOUND) {
      float mx = fmax_std(fmax_std(w_img[0], w_img[1]), w_img[2]);
      return CCDResult{cur[0].lower, cur[0].upper, fmax_std(co_tol, mx), false,
                       0.f, 0.f};
    }
    IBox tmp = cur;
    auto push = [&](const IBox& b) {
      stacks[b[0].lower].push_back(b);
      size_t pending = 0;
      for (auto& kv : stacks) pending += kv.second.size();
      if (pending > g_max_pending) g_max_pending = pending;
    };
    if (split == 0 || !VF) {
      tmp[split] = halves.second;
      push(tmp);
      tmp[split] = halves.first;
      push(tmp);
    } else {
      const Interval& other = (split == 1) ? cur[2] : cur[1];
      if (halves.second.lower + other.lower <= 1.0f) {
        tmp[split] = halves.second;
        push(tmp);
      }
      if (halves.first.lower + other.lower <= 1.0f) {
        tmp[split] = halves.first;
        push(tmp);
      }
    }
    if (bucket != stacks.end() && bucket->second.empty()) stacks.erase(bucket);
  }
  return std::nullopt;
}

static float max_linf_4(const V3& p1, const V3& p2, const V3& p3, const V3& p4,
                        const V3& p1e, const V3& p2e, const V3& p3e,
                        const V3& p4e) {
  auto linf = [](const V3& a, const V3& b) {
    float m = std::fabs(a(0) - b(0));
    m = fmax_std(m, std::fabs(a(1) - b(1)));
    m = fmax_std(m, std::fabs(a(2) - b(2)));
    return m;
  };
  float r = linf(p1e, p1);
  r = fmax_std(r, linf(p2e, p2));
  r = fmax_std(r, linf(p3e, p3));
  r = fmax_std(r, linf(p4e, p4));
  return r;
}

static float clamp_div(float a, float b, float max_val) {
  if (b == 0) return max_val;
  return fmin_std(a / b, max_val);
}

// ccd.cpp:63-126: distance tolerance -> (t,u,v) tolerances.
template <bool VF>
static void ccd_tolerances(const V3* P, float dist_tol, float* out) {
  V3 p000, p001, p011, p010, p100, p101, p111, p110;
  if (VF) {
    p000 = vsub(P[0], P[1]);
    p001 = vsub(P[0], P[3]);
    p011 = vsub(P[0], vsub(vadd(P[2], P[3]), P[1]));
    p010 = vsub(P[0], P[2]);
    p100 = vsub(P[4], P[5]);
    p101 = vsub(P[4], P[7]);
    p111 = vsub(P[4], vsub(vadd(P[6], P[7]), P[5]));
    p110 = vsub(P[4], P[6]);
  } else {
    p000 = vsub(P[0], P[2]);
    p001 = vsub(P[0], P[3]);
    p010 = vsub(P[1], P[2]);
    p011 = vsub(P[1], P[3]);
    p100 = vsub(P[4], P[6]);
    p101 = vsub(P[4], P[7]);
    p110 = vsub(P[5], P[6]);
    p111 = vsub(P[5], P[7]);
  }
  float dl = 3 * max_linf_4(p000, p001, p011, p010, p100, p101, p111, p110);
  float e0 = 3 * max_linf_4(p000, p100, p101, p001, p010, p110, p111, p011);
  float e1 = 3 * max_linf_4(p000, p100, p110, p010, p001, p101, p111, p011);
  const float inf = std::numeric_limits<float>::infinity();
  out[0] = clamp_div(dist_tol, dl, inf);
  out[1] = clamp_div(dist_tol, e0, inf);
  out[2] = clamp_div(dist_tol, e1, inf);
}

// ccd.cpp:128-182.
template <bool VF>
static std::optional<CCDResult> ccd(const V3* P, const float* err, float ms,
                                    float tolerance, long max_iter,
                                    bool no_zero_toi, float max_time) {
  float tol[3];
  ccd_tolerances<VF>(P, tolerance, tol);
  IBox iset = {Interval{0.0f, max_time}, Interval{0.0f, 1.0f},
               Interval{0.0f, 1.0f}};
  auto res = root_finder_bucket_dfs<VF>(P, iset, tol, tolerance, err, ms,
                                        max_iter, max_time == 1.0f);
  if (!no_zero_toi) return res;
  if (!res || res->t0 > 0.0f) return res;
  ms *= 0.5f;
  auto refine = root_finder_bucket_dfs<VF>(P, iset, tol, tolerance, err, ms,
                                           max_iter, max_time == 1.0f);
  res->use_small_ms = true;
  if (!refine) {
    res->small_t0 = max_time;
    res->small_t1 = max_time;
  } else if (refine->t0 > 0.0f) {
    res->small_t0 = refine->t0;
    res->small_t1 = refine->t1;
  } else {
    res->small_t0 = 0.0f;
    res->small_t1 = 0.0f;
  }
  return res;
}

// interval_root_finder.cpp:512-522.
static void numerical_error(const float* absmax, bool vf, float* out) {
  constexpr float EE_FILTER = 3.814698e-06f;
  constexpr float VF_FILTER = 4.053116e-06f;
  float f = vf ? VF_FILTER : EE_FILTER;
  for (int i = 0; i < 3; ++i) out[i] = f * fmax_std(absmax[i], 1.0f);
}

// The production step consumes a CCD answer as a time of impact: the lower
// bound of the accepted interval, or of the refined-separation interval when
// the first answer started at t = 0 (narrowphase.cu:32-77 ignores toi == 0).
static bool ccd_toi(bool vf, const V3* P, const float* err, float ms,
                    float tolerance, long max_iter, float max_time,
                    float& toi) {
  auto r = vf ? ccd<true>(P, err, ms, tolerance, max_iter, true, max_time)
              : ccd<false>(P, err, ms, tolerance, max_iter, true, max_time);
  if (!r) return false;
  toi = r->use_small_ms ? r->small_t0 : r->t0;
  return true;
}

// ---------------------------------------------------------------------------
// Closest points (collision/dcd.cu:241-315).
// ---------------------------------------------------------------------------
static bool exact_pt_uv(const V3& x0, const V3& x1, const V3& x2, const V3& x3,
                        float eps, float& u, float& v) {
  V3 x21 = vsub(x2, x1), x31 = vsub(x3, x1), x01 = vsub(x0, x1);
  float a = dot3(x21, x21), b = dot3(x21, x31), c = dot3(x31, x31);
  float d = dot3(x21, x01), e = dot3(x31, x01);
  float det = a * c - b * b;
  float area_eps = eps * fmax_std(a, c);
  if (det < area_eps * area_eps) return false;
  float b1 = (c * d - b * e) / det;
  float b2 = (a * e - b * d) / det;
  if (b1 < 0.0f || b2 < 0.0f || b1 + b2 > 1.0f) return false;
  u = b1;
  v = b2;
  return true;
}

static bool exact_ee_uv(const V3& x0, const V3& x1, const V3& x2, const V3& x3,
                        float eps, float& uo, float& vo) {
  double d1x = (double)x1(0) - x0(0), d1y = (double)x1(1) - x0(1),
         d1z = (double)x1(2) - x0(2);
  double d2x = (double)x3(0) - x2(0), d2y = (double)x3(1) - x2(1),
         d2z = (double)x3(2) - x2(2);
  double rx = (double)x0(0) - x2(0), ry = (double)x0(1) - x2(1),
         rz = (double)x0(2) - x2(2);
  double a = d1x * d1x + d1y * d1y + d1z * d1z;
  double b = d1x * d2x + d1y * d2y + d1z * d2z;
  double c = d1x * rx + d1y * ry + d1z * rz;
  double e = d2x * d2x + d2y * d2y + d2z * d2z;
  double f = d2x * rx + d2y * ry + d2z * rz;
  double eps2 = (double)eps * eps;
  double ls2 = std::max(a, e);
  if (a <= eps2 * ls2 || e <= eps2 * ls2) return false;
  double den = a * e - b * b;
  double u = den > eps2 * a * e ? std::clamp((b * f - c * e) / den, 0.0, 1.0)
                                : 0.0;
  double v = (b * u + f) / e;
  if (v < 0.0) {
    v = 0.0;
    u = std::clamp(-c / a, 0.0, 1.0);
  } else if (v > 1.0) {
    v = 1.0;
    u = std::clamp((b - c) / a, 0.0, 1.0);
  }
  uo = (float)u;
  vo = (float)v;
  return true;
}

// contact_constraints.cu:391-411.
static V3 solve_coulomb(const V3& us, const V3& n, float mu) {
  float un = dot3(us, n);
  if (un >= 0.0f) return us;
  V3 ut = vsub(us, vscale(un, n));
  float utn = std::sqrt(dot3(ut, ut));
  float radius = -mu * un;
  if (utn <= radius) return v3(0, 0, 0);
  return vscale(1.0f - radius / utn, ut);
}

// ---------------------------------------------------------------------------
// 3x2 clamped projection (cloth_admm_helper.cu:19-51).  Any accurate SVD has
// the same projection; this one diagonalises F^T F in double by a Jacobi
// rotation.
// ---------------------------------------------------------------------------
static void clamp_projection(const double* f, double lo, double hi,
                             double* out) {
  // F columns: c0 = f[0..2], c1 = f[3..5].
  double g11 = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
  double g22 = f[3] * f[3] + f[4] * f[4] + f[5] * f[5];
  double g12 = f[0] * f[3] + f[1] * f[4] + f[2] * f[5];
  double theta = 0.5 * std::atan2(2.0 * g12, g11 - g22);
  double c = std::cos(theta), s = std::sin(theta);
  double v1[2] = {c, s}, v2[2] = {-s, c};
  double u1[3], u2[3];
  for (int i = 0; i < 3; ++i) {
    u1[i] = f[i] * v1[0] + f[3 + i] * v1[1];
    u2[i] = f[i] * v2[0] + f[3 + i] * v2[1];
  }
  double s1 = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  double s2 = std::sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
  if (s1 < s2) {  // order singular values descending
    std::swap(s1, s2);
    std::swap(u1, u2);
    double t0 = v1[0], t1 = v1[1];
    v1[0] = v2[0];
    v1[1] = v2[1];
    v2[0] = t0;
    v2[1] = t1;
  }
  if (s1 > 0) {
    for (int i = 0; i < 3; ++i) u1[i] /= s1;
  } else {
    u1[0] = 1;
    u1[1] = 0;
    u1[2] = 0;
  }
  if (s2 > 1e-12 * std::max(s1, 1e-30)) {
    for (int i = 0; i < 3; ++i) u2[i] /= s2;
  } else {
    // Degenerate: any unit vector orthogonal to u1.
    double a[3] = {std::fabs(u1[0]) < 0.9 ? 1.0 : 0.0,
                   std::fabs(u1[0]) < 0.9 ? 0.0 : 1.0, 0.0};
    double d = a[0] * u1[0] + a[1] * u1[1] + a[2] * u1[2];
    for (int i = 0; i < 3; ++i) a[i] -= d * u1[i];
    double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int i = 0; i < 3; ++i) u2[i] = a[i] / n;
  }
  double c1 = std::clamp(s1, lo, hi), c2 = std::clamp(s2, lo, hi);
  for (int i = 0; i < 3; ++i) {
    out[i] = c1 * u1[i] * v1[0] + c2 * u2[i] * v2[0];
    out[3 + i] = c1 * u1[i] * v1[1] + c2 * u2[i] * v2[1];
  }
}

// ---------------------------------------------------------------------------
// Sparse helpers.
// ---------------------------------------------------------------------------
struct Csr {
  int n = 0;
  std::vector<int> rows, cols;
  std::vector<double> vals;
};

static Csr csr_from_triplets(int n,
                             std::vector<std::tuple<int, int, double>>& t) {
  std::sort(t.begin(), t.end(), [](const auto& a, const auto& b) {
    if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) < std::get<0>(b);
    return std::get<1>(a) < std::get<1>(b);
  });
  Csr m;
  m.n = n;
  m.rows.assign(n + 1, 0);
  for (size_t i = 0; i < t.size();) {
    size_t j = i;
    double s = 0;
    while (j < t.size() && std::get<0>(t[j]) == std::get<0>(t[i]) &&
           std::get<1>(t[j]) == std::get<1>(t[i])) {
      s += std::get<2>(t[j]);
      ++j;
    }
    m.cols.push_back(std::get<1>(t[i]));
    m.vals.push_back(s);
    m.rows[std::get<0>(t[i]) + 1]++;
    i = j;
  }
  for (int i = 0; i < n; ++i) m.rows[i + 1] += m.rows[i];
  return m;
}

// ---------------------------------------------------------------------------
// Cloth static assembly (common/cloth_assembly_l2_cache.cpp:27-136 and
// backend/cuda/assembly/cloth_assembly_l1_cache.cu:16-97).  libigl's Voronoi
// mass and cotangent matrix are restated from their definitions (Meyer et al.
// 2003 mixed area; cotangent weights 0.5 cot).
// ---------------------------------------------------------------------------
struct Assembly {
  int nv = 0, nf = 0;
  std::vector<double> mass;   // Voronoi area per vertex (no density)
  std::vector<double> area;   // per face
  std::vector<double> jop;    // 54 per face, row-major 6x9
  Csr H;                      // 3V x 3V: k_e JWJ + k_b (CWC (x) I3)
  std::vector<double> mass3;  // density * mass, per DoF
  std::vector<double> contact_weight;  // per DoF
  std::vector<double> bending_rhs;     // k_b * C0, per DoF
};

static void triangle_jacobian(const double* v0, const double* v1,
                              const double* v2, double* jop /*6x9 rm*/) {
  double e0[3], e1[3];
  for (int i = 0; i < 3; ++i) {
    e0[i] = v1[i] - v0[i];
    e1[i] = v2[i] - v0[i];
  }
  double n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                 e0[0] * e1[1] - e0[1] * e1[0]};
  double l0 = std::sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
  double bx[3] = {e0[0] / l0, e0[1] / l0, e0[2] / l0};
  double by[3] = {n[1] * e0[2] - n[2] * e0[1], n[2] * e0[0] - n[0] * e0[2],
                  n[0] * e0[1] - n[1] * e0[0]};
  double lb = std::sqrt(by[0] * by[0] + by[1] * by[1] + by[2] * by[2]);
  for (int i = 0; i < 3; ++i) by[i] /= lb;
  double a = bx[0] * e0[0] + bx[1] * e0[1] + bx[2] * e0[2];
  double b = bx[0] * e1[0] + bx[1] * e1[1] + bx[2] * e1[2];
  double c = by[0] * e1[0] + by[1] * e1[1] + by[2] * e1[2];
  // dX = [[a, b], [0, c]]; B = (D dX^-1)^T with D = [[-1,-1],[1,0],[0,1]].
  double inv[2][2] = {{1.0 / a, -b / (a * c)}, {0.0, 1.0 / c}};
  double D[3][2] = {{-1, -1}, {1, 0}, {0, 1}};
  double B[2][3];
  for (int r = 0; r < 2; ++r)
    for (int k = 0; k < 3; ++k)
      B[r][k] = D[k][0] * inv[0][r] + D[k][1] * inv[1][r];
  // J = kron(B, I3): J(3r+a, 3k+b) = B(r,k) delta_ab.
  for (int i = 0; i < 54; ++i) jop[i] = 0.0;
  for (int r = 0; r < 2; ++r)
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) jop[(3 * r + d) * 9 + 3 * k + d] = B[r][k];
}

static Assembly assemble(const std::vector<double>& V, const std::vector<int>& F,
                         const oracle_cloth_config& cfg, double dt) {
  Assembly A;
  int nv = (int)V.size() / 3, nf = (int)F.size() / 3;
  A.nv = nv;
  A.nf = nf;
  A.mass.assign(nv, 0.0);
  A.area.assign(nf, 0.0);
  std::vector<std::tuple<int, int, double>> ct;  // cotangent Laplacian
  for (int f = 0; f < nf; ++f) {
    int id[3] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};
    const double* p[3] = {&V[3 * id[0]], &V[3 * id[1]], &V[3 * id[2]]};
    double e[3][3];  // e[i] = edge opposite vertex i: p[j] -> p[k]
    double l2[3];
    for (int i = 0; i < 3; ++i) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      for (int d = 0; d < 3; ++d) e[i][d] = p[k][d] - p[j][d];
      l2[i] = e[i][0] * e[i][0] + e[i][1] * e[i][1] + e[i][2] * e[i][2];
    }
    double ab[3], ac[3];
    for (int d = 0; d < 3; ++d) {
      ab[d] = p[1][d] - p[0][d];
      ac[d] = p[2][d] - p[0][d];
    }
    double cr[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
                    ab[0] * ac[1] - ab[1] * ac[0]};
    double dbl = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    double area = 0.5 * dbl;
    A.area[f] = area;
    // cot of angle at vertex i = (l_j^2 + l_k^2 - l_i^2) / (4 area)
    double cot[3], cosv[3];
    for (int i = 0; i < 3; ++i) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      cot[i] = (l2[j] + l2[k] - l2[i]) / (4.0 * area);
      cosv[i] = (l2[j] + l2[k] - l2[i]);
    }
    // Mixed Voronoi area.
    int obtuse = -1;
    for (int i = 0; i < 3; ++i)
      if (cosv[i] < 0) obtuse = i;
    for (int i = 0; i < 3; ++i) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      double m;
      if (obtuse < 0) {
        // 1/8 (|e_ij|^2 cot(k) + |e_ik|^2 cot(j)); |e_ij| is opposite k.
        m = 0.125 * (l2[k] * cot[k] + l2[j] * cot[j]);
      } else {
        m = (obtuse == i) ? 0.5 * area : 0.25 * area;
      }
      A.mass[id[i]] += m;
    }
    // Cotangent matrix: edge opposite i gets 0.5 cot(i).
    for (int i = 0; i < 3; ++i) {
      int j = id[(i + 1) % 3], k = id[(i + 2) % 3];
      double w = 0.5 * cot[i];
      ct.emplace_back(j, k, w);
      ct.emplace_back(k, j, w);
      ct.emplace_back(j, j, -w);
      ct.emplace_back(k, k, -w);
    }
  }
  Csr C = csr_from_triplets(nv, ct);
  // CWC = C^T W C, W = M^-1 (C is symmetric).
  std::vector<std::tuple<int, int, double>> cwc;
  {
    std::vector<double> acc(nv, 0.0);
    std::vector<int> mark(nv, -1), touched;
    for (int i = 0; i < nv; ++i) {
      touched.clear();
      for (int a = C.rows[i]; a < C.rows[i + 1]; ++a) {
        int k = C.cols[a];
        double cik = C.vals[a] / A.mass[k];
        for (int b = C.rows[k]; b < C.rows[k + 1]; ++b) {
          int j = C.cols[b];
          if (mark[j] != i) {
            mark[j] = i;
            acc[j] = 0.0;
            touched.push_back(j);
          }
          acc[j] += cik * C.vals[b];
        }
      }
      for (int j : touched) cwc.emplace_back(i, j, acc[j]);
    }
  }
  // Full 3V x 3V system the reference way.
  std::vector<std::tuple<int, int, double>> trip;
  A.jop.assign(54 * (size_t)nf, 0.0);
  for (int f = 0; f < nf; ++f) {
    int id[3] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};
    double* J = &A.jop[54 * (size_t)f];
    triangle_jacobian(&V[3 * id[0]], &V[3 * id[1]], &V[3 * id[2]], J);
    double w = A.area[f];
    for (int vi = 0; vi < 3; ++vi)
      for (int vj = 0; vj < 3; ++vj)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int r = 0; r < 6; ++r)
              s += J[r * 9 + 3 * vi + i] * J[r * 9 + 3 * vj + j];
            if (s != 0.0)
              trip.emplace_back(3 * id[vi] + i, 3 * id[vj] + j,
                                cfg.elastic_stiffness * w * s);
          }
  }
  for (auto& [i, j, v] : cwc)
    for (int d = 0; d < 3; ++d)
      trip.emplace_back(3 * i + d, 3 * j + d, cfg.bending_stiffness * v);
  A.H = csr_from_triplets(3 * nv, trip);
  // Vectors.
  A.mass3.assign(3 * nv, 0.0);
  A.contact_weight.assign(3 * nv, 0.0);
  A.bending_rhs.assign(3 * nv, 0.0);
  for (int i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) A.mass3[3 * i + d] = cfg.density * A.mass[i];
  // C0 = CWC * V; bending rhs = k_b C0.
  for (auto& [i, j, v] : cwc)
    for (int d = 0; d < 3; ++d)
      A.bending_rhs[3 * i + d] += cfg.bending_stiffness * v * V[3 * j + d];
  // Contact weight (cloth_assembly_l1_cache.cu:58-75): eta = smallest
  // eigenvalue of the 3x3 diagonal block of H + M/dt^2.
  for (int i = 0; i < nv; ++i) {
    double blk[3][3] = {};
    for (int d = 0; d < 3; ++d) {
      int r = 3 * i + d;
      for (int a = A.H.rows[r]; a < A.H.rows[r + 1]; ++a) {
        int c = A.H.cols[a];
        if (c / 3 == i) blk[d][c % 3] = A.H.vals[a];
      }
      blk[d][d] += A.mass3[3 * i] / (dt * dt);
    }
    // Symmetric 3x3 eigenvalues (Jacobi sweeps, double).
    double m[3][3];
    std::memcpy(m, blk, sizeof(m));
    for (int sweep = 0; sweep < 50; ++sweep) {
      double off = m[0][1] * m[0][1] + m[0][2] * m[0][2] + m[1][2] * m[1][2];
      if (off < 1e-30) break;
      for (int p = 0; p < 2; ++p)
        for (int q = p + 1; q < 3; ++q) {
          if (std::fabs(m[p][q]) < 1e-300) continue;
          double th = 0.5 * std::atan2(2 * m[p][q], m[q][q] - m[p][p]);
          double c = std::cos(th), s = std::sin(th);
          for (int k = 0; k < 3; ++k) {
            double mkp = m[k][p], mkq = m[k][q];
            m[k][p] = c * mkp - s * mkq;
            m[k][q] = s * mkp + c * mkq;
          }
          for (int k = 0; k < 3; ++k) {
            double mpk = m[p][k], mqk = m[q][k];
            m[p][k] = c * mpk - s * mqk;
            m[q][k] = s * mpk + c * mqk;
          }
        }
    }
    double eta = std::min(m[0][0], std::min(m[1][1], m[2][2]));
    double inertia = A.mass3[3 * i] / (dt * dt);
    double w = std::max(0.001 * eta, std::min(25.0 * inertia, eta));
    for (int d = 0; d < 3; ++d) A.contact_weight[3 * i + d] = w;
  }
  return A;
}

// ---------------------------------------------------------------------------
// Multilevel additive Schwarz preconditioner
// (backend/cuda/solver/mas_preconditioner.cu:50-989), banks of 32 vertices,
// 3 DoF per vertex, dense bank matrices inverted in double.
// ---------------------------------------------------------------------------
constexpr int BANK = 32;
constexpr int MAX_COARSE = 4;

template <class T>
struct Mas {
  int nv = 0;
  int levels = 0;  // coarse levels
  std::vector<int> real_to_padded;
  std::vector<int> padded_nodes;     // per level incl. level 0 (node slots)
  std::vector<std::vector<int>> map;  // map[lv][vertex] coarse id
  // Dense inverses per level: banks x 96 x 96.
  std::vector<std::vector<T>> inv;
  std::vector<int> nbank;

  void build_topology(const Csr& H, const std::vector<int>& part_offsets) {
    nv = H.n / 3;
    int nparts = (int)part_offsets.size() - 1;
    real_to_padded.assign(nv, -1);
    for (int p = 0; p < nparts; ++p)
      for (int v = part_offsets[p]; v < part_offsets[p + 1]; ++v)
        real_to_padded[v] = BANK * p + (v - part_offsets[p]);
    // Block adjacency graph of H.
    std::vector<std::vector<int>> adj(nv);
    for (int r = 0; r < H.n; r += 3) {
      int i = r / 3;
      for (int a = H.rows[r]; a < H.rows[r + 1]; ++a) {
        int j = H.cols[a] / 3;
        if (j != i) adj[i].push_back(j);
      }
    }
    for (auto& a : adj) {
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    // Level "node id" of each vertex at the previous level (padded ids first).
    std::vector<int> prev(nv);
    for (int v = 0; v < nv; ++v) prev[v] = real_to_padded[v];
    int prev_slots = nparts * BANK;
    int prev_count = -1;  // real nodes at previous level (unknown for lv0)
    map.clear();
    for (int lv = 0; lv < MAX_COARSE; ++lv) {
      // Connected components inside each bank of 32 consecutive prev ids.
      std::vector<int> uf(prev_slots);
      for (int i = 0; i < prev_slots; ++i) uf[i] = i;
      std::function<int(int)> find = [&](int x) {
        while (uf[x] != x) x = uf[x] = uf[uf[x]];
        return x;
      };
      std::vector<char> present(prev_slots, 0);
      for (int v = 0; v < nv; ++v) present[prev[v]] = 1;
      for (int v = 0; v < nv; ++v)
        for (int j : adj[v]) {
          int a = prev[v], b = prev[j];
          if (a / BANK != b / BANK) continue;
          int ra = find(a), rb = find(b);
          if (ra != rb) uf[std::max(ra, rb)] = std::min(ra, rb);
        }
      // CCO ids ordered by bank, then by lowest member lane.
      std::vector<int> cid(prev_slots, -1);
      int count = 0;
      for (int s = 0; s < prev_slots; ++s) {
        if (!present[s]) continue;
        int r = find(s);
        if (r == s) cid[s] = count++;
      }
      for (int s = 0; s < prev_slots; ++s)
        if (present[s]) cid[s] = cid[find(s)];
      std::vector<int> m(nv);
      for (int v = 0; v < nv; ++v) m[v] = cid[prev[v]];
      if (lv > 0 && count == prev_count) break;  // nothing merged
      map.push_back(m);
      prev = m;
      prev_slots = ((count + BANK - 1) / BANK) * BANK;
      prev_count = count;
    }
    levels = (int)map.size();
    nbank.assign(levels + 1, 0);
    nbank[0] = nparts;
    for (int lv = 0; lv < levels; ++lv) {
      int mx = 0;
      for (int v = 0; v < nv; ++v) mx = std::max(mx, map[lv][v] + 1);
      nbank[lv + 1] = (mx + BANK - 1) / BANK;
    }
  }

  // A = H + diag(d).
  void factorize(const Csr& H, const std::vector<double>& diag) {
    constexpr int N = 3 * BANK;
    inv.assign(levels + 1, {});
    for (int l = 0; l <= levels; ++l) {
      std::vector<double> M((size_t)nbank[l] * N * N, 0.0);
      auto node = [&](int v) {
        return l == 0 ? real_to_padded[v] : map[l - 1][v];
      };
      for (int r = 0; r < H.n; ++r) {
        int i = r / 3, di = r % 3;
        int ci = node(i);
        for (int a = H.rows[r]; a < H.rows[r + 1]; ++a) {
          int j = H.cols[a] / 3, dj = H.cols[a] % 3;
          int cj = node(j);
          if (ci / BANK != cj / BANK) continue;
          size_t base = (size_t)(ci / BANK) * N * N;
          M[base + (size_t)(3 * (ci % BANK) + di) * N + 3 * (cj % BANK) + dj] +=
              H.vals[a];
        }
        size_t base = (size_t)(ci / BANK) * N * N;
        M[base + (size_t)(3 * (ci % BANK) + di) * N + 3 * (ci % BANK) + di] +=
            diag[r];
      }
      inv[l].assign(M.size(), T(0));
      for (int b = 0; b < nbank[l]; ++b) {
        double* A = &M[(size_t)b * N * N];
        for (int i = 0; i < N; ++i)
          if (A[i * N + i] == 0.0) A[i * N + i] = 1.0;  // virtual padding
        // Gauss-Jordan with partial pivoting in double.
        std::vector<double> I(N * N, 0.0);
        for (int i = 0; i < N; ++i) I[i * N + i] = 1.0;
        for (int c = 0; c < N; ++c) {
          int piv = c;
          for (int r = c + 1; r < N; ++r)
            if (std::fabs(A[r * N + c]) > std::fabs(A[piv * N + c])) piv = r;
          if (piv != c)
            for (int k = 0; k < N; ++k) {
              std::swap(A[c * N + k], A[piv * N + k]);
              std::swap(I[c * N + k], I[piv * N + k]);
            }
          double p = A[c * N + c];
          for (int k = 0; k < N; ++k) {
            A[c * N + k] /= p;
            I[c * N + k] /= p;
          }
          for (int r = 0; r < N; ++r) {
            if (r == c) continue;
            double f = A[r * N + c];
            if (f == 0.0) continue;
            for (int k = 0; k < N; ++k) {
              A[r * N + k] -= f * A[c * N + k];
              I[r * N + k] -= f * I[c * N + k];
            }
          }
        }
        for (int k = 0; k < N * N; ++k) inv[l][(size_t)b * N * N + k] = (T)I[k];
      }
    }
  }

  void apply(const std::vector<T>& r, std::vector<T>& z) const {
    constexpr int N = 3 * BANK;
    z.assign(r.size(), T(0));
    for (int l = 0; l <= levels; ++l) {
      std::vector<double> rl((size_t)nbank[l] * N, 0.0);
      auto node = [&](int v) {
        return l == 0 ? real_to_padded[v] : map[l - 1][v];
      };
      for (int v = 0; v < nv; ++v)
        for (int d = 0; d < 3; ++d) rl[3 * node(v) + d] += (double)r[3 * v + d];
      std::vector<T> zl(rl.size(), T(0));
      for (int b = 0; b < nbank[l]; ++b) {
        const T* M = &inv[l][(size_t)b * N * N];
        for (int i = 0; i < N; ++i) {
          T s = 0;
          for (int k = 0; k < N; ++k) s += M[i * N + k] * (T)rl[b * N + k];
          zl[b * N + i] = s;
        }
      }
      for (int v = 0; v < nv; ++v)
        for (int d = 0; d < 3; ++d) z[3 * v + d] += zl[3 * node(v) + d];
    }
  }
};

// ---------------------------------------------------------------------------
// Colliders (collision/mesh_collider.cuh:11-75, object_collider.cu:21-466).
// ---------------------------------------------------------------------------
struct ObjectColl {
  u32 id;
  bool physical;
  int group;  // -1 disabled
  bool self_on;
  float padding;
  float friction;
  Bbox bbox;
  int state_offset;  // -1 for obstacles
  int nv;
  std::vector<int> F, E;       // solver-order indices
  std::vector<float> inv_mass;  // per vertex
  std::vector<float> x0, x1;    // per-vertex t0 / t1 positions (3 nv)
  std::vector<Bbox> tri_bb, edge_bb, pt_bb;
};

static void refit(ObjectColl& o) {
  int nf = (int)o.F.size() / 3, ne = (int)o.E.size() / 2;
  auto P0 = [&](int i) { return v3(o.x0[3 * i], o.x0[3 * i + 1], o.x0[3 * i + 2]); };
  auto P1 = [&](int i) { return v3(o.x1[3 * i], o.x1[3 * i + 1], o.x1[3 * i + 2]); };
  o.tri_bb.resize(nf);
  Bbox obj{v3(std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
              std::numeric_limits<float>::max()),
           v3(std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
              std::numeric_limits<float>::lowest())};
  for (int f = 0; f < nf; ++f) {
    int a = o.F[3 * f], b = o.F[3 * f + 1], c = o.F[3 * f + 2];
    V3 t0min = vmin(vmin(P0(a), P0(b)), P0(c));
    V3 t1min = vmin(vmin(P1(a), P1(b)), P1(c));
    V3 t0max = vmax(vmax(P0(a), P0(b)), P0(c));
    V3 t1max = vmax(vmax(P1(a), P1(b)), P1(c));
    o.tri_bb[f] = bbox_pad(Bbox{vmin(t0min, t1min), vmax(t0max, t1max)}, o.padding);
    obj = bbox_merge(obj, o.tri_bb[f]);
  }
  o.bbox = obj;
  o.edge_bb.resize(ne);
  for (int e = 0; e < ne; ++e) {
    int a = o.E[2 * e], b = o.E[2 * e + 1];
    Bbox bb{vmin(vmin(P0(a), P0(b)), vmin(P1(a), P1(b))),
            vmax(vmax(P0(a), P0(b)), vmax(P1(a), P1(b)))};
    o.edge_bb[e] = bbox_pad(bb, o.padding);
  }
  o.pt_bb.resize(o.nv);
  for (int i = 0; i < o.nv; ++i)
    o.pt_bb[i] = bbox_pad(Bbox{vmin(P0(i), P1(i)), vmax(P0(i), P1(i))}, o.padding);
}

struct Cand {
  int kind;  // 0 = PT (a = tri object/index, b = point), 1 = EE
  int oa, ia, ob, ib;  // object slot + primitive index
};

// find_collision.cu:17-138: object SAP + primitive filters; candidate set is
// every pair of padded boxes that overlap (<=) and passes the filters.
static std::vector<Cand> candidates(std::vector<ObjectColl*>& objs) {
  std::vector<Cand> out;
  int n = (int)objs.size();
  auto obj_filter = [](const ObjectColl& a, const ObjectColl& b) {
    return a.group != -1 && b.group != -1 && a.group == b.group &&
           (a.physical || b.physical);
  };
  // sap.cuh:37-99 (stable sort for determinism).
  std::vector<int> prox(n);
  for (int i = 0; i < n; ++i) prox[i] = i;
  std::vector<std::pair<int, int>> pairs;
  if (n > 0) {
    float mean[3] = {0, 0, 0}, var[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
      V3 c = axpby(0.5f, objs[i]->bbox.mn, 0.5f, objs[i]->bbox.mx);
      for (int d = 0; d < 3; ++d) {
        mean[d] += c(d);
        var[d] += c(d) * c(d);
      }
    }
    for (int d = 0; d < 3; ++d) {
      mean[d] = (1.0f / n) * mean[d];
      var[d] = (1.0f / n) * var[d] - mean[d] * mean[d];
    }
    int axis = (var[0] > var[1] && var[0] > var[2]) ? 0 : (var[1] > var[2] ? 1 : 2);
    std::stable_sort(prox.begin(), prox.end(), [&](int a, int b) {
      return objs[a]->bbox.mn(axis) < objs[b]->bbox.mn(axis);
    });
    for (int i = 0; i + 1 < n; ++i) {
      ObjectColl& ca = *objs[prox[i]];
      for (int j = i + 1; j < n; ++j) {
        ObjectColl& cb = *objs[prox[j]];
        if (ca.bbox.mx(axis) < cb.bbox.mn(axis)) break;
        if (!obj_filter(ca, cb)) continue;
        if (bbox_colliding(ca.bbox, cb.bbox)) pairs.emplace_back(prox[i], prox[j]);
      }
    }
  }
  auto pt = [&](int ot, int op, bool self) {
    ObjectColl& T = *objs[ot];
    ObjectColl& P = *objs[op];
    int nf = (int)T.F.size() / 3;
    for (int f = 0; f < nf; ++f)
      for (int p = 0; p < P.nv; ++p) {
        if (!bbox_colliding(P.pt_bb[p], T.tri_bb[f])) continue;
        int a = T.F[3 * f], b = T.F[3 * f + 1], c = T.F[3 * f + 2];
        float s = P.inv_mass[p] + T.inv_mass[a] + T.inv_mass[b] + T.inv_mass[c];
        if (s == 0.0f) continue;
        if (self && (a == p || b == p || c == p)) continue;
        out.push_back({0, ot, f, op, p});
      }
  };
  auto ee = [&](int oa, int ob, bool self) {
    ObjectColl& A = *objs[oa];
    ObjectColl& B = *objs[ob];
    int na = (int)A.E.size() / 2, nb = (int)B.E.size() / 2;
    for (int i = 0; i < na; ++i)
      for (int j = self ? i + 1 : 0; j < nb; ++j) {
        if (!bbox_colliding(A.edge_bb[i], B.edge_bb[j])) continue;
        int a0 = A.E[2 * i], a1 = A.E[2 * i + 1], b0 = B.E[2 * j], b1 = B.E[2 * j + 1];
        float s = A.inv_mass[a0] + A.inv_mass[a1] + B.inv_mass[b0] + B.inv_mass[b1];
        if (s == 0.0f) continue;
        if (self && (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1)) continue;
        out.push_back({1, oa, i, ob, j});
      }
  };
  for (auto& [a, b] : pairs) {
    pt(a, b, false);
    pt(b, a, false);
    ee(a, b, false);
  }
  for (int o = 0; o < n; ++o) {
    if (!objs[o]->physical || !objs[o]->self_on) continue;
    pt(o, o, true);
    ee(o, o, true);
  }
  return out;
}

// ---------------------------------------------------------------------------
// DCD collisions (collision/dcd.cu:23-238) and contact constraints
// (solver/contact_constraints.cu:24-599).
// ---------------------------------------------------------------------------
struct Collision {
  int type;  // 0 PT, 1 EE
  u32 obj_a, obj_b;
  int off_a, off_b;  // state offsets (-1 obstacle)
  int idx[4];
  float dact, friction;
  V3 normal;
  float coef[4], inv_mass[4];
  V3 x[4];
  V3 prescribed;
};

struct ContactKey {
  int type;
  u32 oa, ob;
  int idx[4];
  bool operator<(const ContactKey& o) const {
    return std::tie(type, oa, ob, idx[0], idx[1], idx[2], idx[3]) <
           std::tie(o.type, o.oa, o.ob, o.idx[0], o.idx[1], o.idx[2], o.idx[3]);
  }
  bool operator==(const ContactKey& o) const {
    return type == o.type && oa == o.oa && ob == o.ob && idx[0] == o.idx[0] &&
           idx[1] == o.idx[1] && idx[2] == o.idx[2] && idx[3] == o.idx[3];
  }
};

// contact_constraints.cu:24-47.
static ContactKey make_key(const Collision& c) {
  ContactKey k{c.type, c.obj_a, c.obj_b, {c.idx[0], c.idx[1], c.idx[2], c.idx[3]}};
  if (c.type == 0) {
    std::sort(k.idx + 1, k.idx + 4);
    return k;
  }
  if (k.idx[1] < k.idx[0]) std::swap(k.idx[0], k.idx[1]);
  if (k.idx[3] < k.idx[2]) std::swap(k.idx[2], k.idx[3]);
  auto ea = std::make_tuple(k.oa, k.idx[0], k.idx[1]);
  auto eb = std::make_tuple(k.ob, k.idx[2], k.idx[3]);
  if (eb < ea) {
    std::swap(k.oa, k.ob);
    std::swap(k.idx[0], k.idx[2]);
    std::swap(k.idx[1], k.idx[3]);
  }
  return k;
}

// Colouring priority of a contact: a 64-bit mix of its canonical key.  The
// product computes the same function, so both colourings are the greedy
// colouring in decreasing priority order.
static inline u64 mix64(u64 z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static u64 key_priority(const ContactKey& k) {
  u64 h = mix64((u64)k.type);
  h = mix64(h ^ k.oa);
  h = mix64(h ^ ((u64)k.ob << 1));
  for (int i = 0; i < 4; ++i) h = mix64(h ^ (u64)(u32)k.idx[i]);
  return h;
}

static inline V3 lerp_t(const V3& a, const V3& b, float t) {
  return axpby(1.0f - t, a, t, b);
}

constexpr float DCD_EPS = 1e-6f;

static std::optional<Collision> make_pt_collision(const ObjectColl& T, int f,
                                                  const ObjectColl& P, int p,
                                                  float time, float dact) {
  auto X0 = [](const ObjectColl& o, int i) {
    return v3(o.x0[3 * i], o.x0[3 * i + 1], o.x0[3 * i + 2]);
  };
  auto X1 = [](const ObjectColl& o, int i) {
    return v3(o.x1[3 * i], o.x1[3 * i + 1], o.x1[3 * i + 2]);
  };
  int a = T.F[3 * f], b = T.F[3 * f + 1], c = T.F[3 * f + 2];
  V3 x0 = lerp_t(X0(P, p), X1(P, p), time);
  V3 x1 = lerp_t(X0(T, a), X1(T, a), time);
  V3 x2 = lerp_t(X0(T, b), X1(T, b), time);
  V3 x3 = lerp_t(X0(T, c), X1(T, c), time);
  float u, v;
  if (!exact_pt_uv(x0, x1, x2, x3, DCD_EPS, u, v)) return std::nullopt;
  V3 tp = axpby(1.0f, axpby(1.0f - u - v, x1, u, x2), v, x3);
  V3 disp = vsub(tp, x0);
  float d2 = dot3(disp, disp);
  if (d2 == 0.0f) return std::nullopt;
  float dist = std::sqrt(d2);
  if (dist >= dact) return std::nullopt;
  V3 n = vscale(-1.0f / dist, disp);
  float param[4] = {1.0f, 1.0f - u - v, u, v};
  float coef[4] = {1.0f, -param[1], -param[2], -param[3]};
  float im[4] = {P.inv_mass[p], T.inv_mass[a], T.inv_mass[b], T.inv_mass[c]};
  float den = 0.0f;
  for (int i = 0; i < 4; ++i) den += param[i] * param[i] * im[i];
  if (den == 0.0f) return std::nullopt;
  Collision col;
  col.type = 0;
  col.obj_a = P.id;
  col.obj_b = T.id;
  col.off_a = P.state_offset;
  col.off_b = T.state_offset;
  col.idx[0] = p;
  col.idx[1] = a;
  col.idx[2] = b;
  col.idx[3] = c;
  col.dact = dact;
  col.friction = std::sqrt(P.friction * T.friction);
  col.normal = n;
  for (int i = 0; i < 4; ++i) {
    col.coef[i] = coef[i];
    col.inv_mass[i] = im[i];
  }
  col.x[0] = x0;
  col.x[1] = x1;
  col.x[2] = x2;
  col.x[3] = x3;
  col.prescribed = v3(0, 0, 0);
  if (P.state_offset < 0) col.prescribed = vscale(coef[0], vsub(X1(P, p), x0));
  if (T.state_offset < 0) {
    col.prescribed = vadd(
        col.prescribed,
        vadd(vscale(coef[1], vsub(X1(T, a), x1)),
             vadd(vscale(coef[2], vsub(X1(T, b), x2)), vscale(coef[3], vsub(X1(T, c), x3)))));
  }
  return col;
}

static std::optional<Collision> make_ee_collision(const ObjectColl& A, int i,
                                                  const ObjectColl& B, int j,
                                                  float time, float dact) {
  auto X0 = [](const ObjectColl& o, int k) {
    return v3(o.x0[3 * k], o.x0[3 * k + 1], o.x0[3 * k + 2]);
  };
  auto X1 = [](const ObjectColl& o, int k) {
    return v3(o.x1[3 * k], o.x1[3 * k + 1], o.x1[3 * k + 2]);
  };
  int a0 = A.E[2 * i], a1 = A.E[2 * i + 1], b0 = B.E[2 * j], b1 = B.E[2 * j + 1];
  V3 x0 = lerp_t(X0(A, a0), X1(A, a0), time);
  V3 x1 = lerp_t(X0(A, a1), X1(A, a1), time);
  V3 x2 = lerp_t(X0(B, b0), X1(B, b0), time);
  V3 x3 = lerp_t(X0(B, b1), X1(B, b1), time);
  float u, v;
  if (!exact_ee_uv(x0, x1, x2, x3, DCD_EPS, u, v)) return std::nullopt;
  V3 pa = axpby(1.0f - u, x0, u, x1);
  V3 pb = axpby(1.0f - v, x2, v, x3);
  V3 disp = vsub(pb, pa);
  float d2 = dot3(disp, disp);
  if (d2 == 0.0f) return std::nullopt;
  float dist = std::sqrt(d2);
  if (dist >= dact) return std::nullopt;
  V3 n = vscale(-1.0f / dist, disp);
  float param[4] = {1.0f - u, u, 1.0f - v, v};
  float coef[4] = {param[0], param[1], -param[2], -param[3]};
  float im[4] = {A.inv_mass[a0], A.inv_mass[a1], B.inv_mass[b0], B.inv_mass[b1]};
  float den = 0.0f;
  for (int k = 0; k < 4; ++k) den += param[k] * param[k] * im[k];
  if (den == 0.0f) return std::nullopt;
  Collision col;
  col.type = 1;
  col.obj_a = A.id;
  col.obj_b = B.id;
  col.off_a = A.state_offset;
  col.off_b = B.state_offset;
  col.idx[0] = a0;
  col.idx[1] = a1;
  col.idx[2] = b0;
  col.idx[3] = b1;
  col.dact = dact;
  col.friction = std::sqrt(A.friction * B.friction);
  col.normal = n;
  for (int k = 0; k < 4; ++k) {
    col.coef[k] = coef[k];
    col.inv_mass[k] = im[k];
  }
  col.x[0] = x0;
  col.x[1] = x1;
  col.x[2] = x2;
  col.x[3] = x3;
  col.prescribed = v3(0, 0, 0);
  if (A.state_offset < 0)
    col.prescribed = vadd(vscale(coef[0], vsub(X1(A, a0), x0)),
                          vscale(coef[1], vsub(X1(A, a1), x1)));
  if (B.state_offset < 0)
    col.prescribed = vadd(col.prescribed,
                          vadd(vscale(coef[2], vsub(X1(B, b0), x2)),
                               vscale(coef[3], vsub(X1(B, b1), x3))));
  return col;
}

struct Contact {
  int off[4];  // global DoF offset of each slot, -1 = kinematic
  float coef[4], gamma[4];
  V3 normal, affine;
  float friction;
  u64 prio;
  ContactKey key;
};

// build_contacts (contact_constraints.cu:73-137).
template <class T>
static Contact build_contact(const Collision& c, const std::vector<T>& weight) {
  Contact k;
  for (int s = 0; s < 4; ++s) k.coef[s] = c.coef[s];
  k.normal = c.normal;
  k.friction = c.friction;
  k.affine = vscale(-c.dact, c.normal);
  float norm = 0.0f;
  V3 ref = v3(0, 0, 0);
  for (int s = 0; s < 4; ++s) {
    float co = k.coef[s];
    ref = vadd(ref, vscale(co, c.x[s]));
    int off;
    if (c.type == 0) off = (s == 0) ? c.off_a : c.off_b;
    else off = (s < 2) ? c.off_a : c.off_b;
    off = off < 0 ? -1 : off + 3 * c.idx[s];
    k.off[s] = off;
    if (off < 0) {
      k.affine = vadd(k.affine, vscale(co, c.x[s]));
      continue;
    }
    if (c.inv_mass[s] > 0.0f) norm += co * co / (float)weight[off];
  }
  k.affine = vadd(k.affine, c.prescribed);
  float rn = dot3(ref, k.normal);
  V3 rt = vsub(ref, vscale(rn, k.normal));
  k.affine = vsub(k.affine, rt);
  for (int s = 0; s < 4; ++s) {
    if (k.off[s] >= 0 && c.inv_mass[s] > 0.0f)
      k.gamma[s] = k.coef[s] / (norm * (float)weight[k.off[s]]);
    else
      k.gamma[s] = 0.0f;
  }
  k.key = make_key(c);
  k.prio = key_priority(k.key);
  return k;
}

// Greedy colouring in decreasing priority order: each contact takes the
// smallest colour >= 1 not used by an already-coloured contact sharing a
// movable vertex (validity rule of contact_coloring.cu:121-213).
static int color_greedy(const std::vector<std::array<int, 4>>& verts,
                        const std::vector<u64>& prio, std::vector<int>& color) {
  int n = (int)verts.size();
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (prio[a] != prio[b]) return prio[a] > prio[b];
    return a < b;
  });
  std::unordered_map<int, std::vector<int>> inc;
  for (int i = 0; i < n; ++i)
    for (int s = 0; s < 4; ++s)
      if (verts[i][s] >= 0) inc[verts[i][s]].push_back(i);
  color.assign(n, 0);
  int maxc = 0;
  for (int c : order) {
    std::set<int> used;
    for (int s = 0; s < 4; ++s) {
      int v = verts[c][s];
      if (v < 0) continue;
      for (int o : inc[v])
        if (color[o] > 0) used.insert(color[o]);
    }
    int col = 1;
    while (used.count(col)) ++col;
    color[c] = col;
    maxc = std::max(maxc, col);
  }
  return maxc;
}

template <class T>
struct Contacts {
  int ndof = 0;
  std::vector<Contact> list;
  std::set<ContactKey> keys;
  std::vector<std::vector<int>> groups;  // contact ids per colour
  std::vector<T> base_weight, weight, aux, prev_aux, eta;
  std::vector<V3> corr;
  int active_dof = 0;

  void init(int n, const std::vector<T>& bw) {
    ndof = n;
    base_weight = bw;
    weight.assign(n, T(0));
    aux.assign(n, T(0));
    prev_aux.assign(n, T(0));
    eta.assign(n, T(0));
    list.clear();
    keys.clear();
    groups.clear();
    corr.clear();
    active_dof = 0;
  }

  int append(const std::vector<Collision>& cols) {
    std::vector<Contact> fresh;
    for (const Collision& c : cols) {
      ContactKey k = make_key(c);
      if (keys.insert(k).second) fresh.push_back(build_contact(c, base_weight));
    }
    if (fresh.empty()) return 0;
    std::sort(fresh.begin(), fresh.end(),
              [](const Contact& a, const Contact& b) { return a.key < b.key; });
    for (auto& f : fresh) {
      list.push_back(f);
      corr.push_back(v3(0, 0, 0));
    }
    rebuild();
    return (int)fresh.size();
  }

  void rebuild() {
    int nvert = ndof / 3;
    std::vector<int> count(nvert, 0);
    std::vector<std::array<int, 4>> verts(list.size());
    std::vector<u64> prio(list.size());
    for (size_t c = 0; c < list.size(); ++c) {
      prio[c] = list[c].prio;
      for (int s = 0; s < 4; ++s) {
        if (list[c].gamma[s] != 0.0f) {
          verts[c][s] = list[c].off[s] / 3;
          count[verts[c][s]]++;
        } else {
          verts[c][s] = -1;
        }
      }
    }
    int active = 0;
    for (int v = 0; v < nvert; ++v) active += count[v] > 0;
    active_dof = 3 * active;
    weight = base_weight;
    for (int i = 0; i < ndof; ++i)
      if (count[i / 3] == 0) weight[i] = T(0);
    std::vector<int> color;
    int nc = color_greedy(verts, prio, color);
    groups.assign(nc, {});
    for (size_t c = 0; c < list.size(); ++c) groups[color[c] - 1].push_back((int)c);
  }

  void eval(std::vector<T>& lhs, std::vector<T>& rhs) const {
    for (int i = 0; i < ndof; ++i) {
      T w = weight[i];
      if (w > T(0)) {
        lhs[i] += w;
        rhs[i] += w * aux[i] + eta[i];
      }
    }
  }

  // update_aux_var_and_lagrange_mul (contact_constraints.cu:575-593).
  void update(const std::vector<T>& x, double& pn2, std::vector<T>& dual,
              std::vector<T>& dcur, std::vector<T>& dprev) {
    prev_aux = aux;
    for (int i = 0; i < ndof; ++i) {
      T w = weight[i];
      aux[i] = w > T(0) ? x[i] - eta[i] / w : x[i];
    }
    auto getp = [&](int off) { return V3{{(float)aux[off], (float)aux[off + 1], (float)aux[off + 2]}}; };
    auto addp = [&](int off, const V3& d, float g) {
      for (int a = 0; a < 3; ++a) aux[off + a] = (T)((float)aux[off + a] + g * d(a));
    };
    for (auto& grp : groups)
      for (int c : grp) {
        const Contact& k = list[c];
        for (int s = 0; s < 4; ++s)
          if (k.gamma[s] != 0.0f) addp(k.off[s], corr[c], k.gamma[s]);
      }
    for (int sweep = 0; sweep < 10; ++sweep)
      for (auto& grp : groups)
        for (int c : grp) {
          const Contact& k = list[c];
          V3 u = k.affine;
          for (int s = 0; s < 4; ++s)
            if (k.off[s] >= 0) u = vadd(u, vscale(k.coef[s], getp(k.off[s])));
          V3 old = corr[c];
          V3 us = vsub(u, old);
          V3 un = solve_coulomb(us, k.normal, k.friction);
          V3 du = vsub(un, u);
          corr[c] = vadd(old, du);
          for (int s = 0; s < 4; ++s)
            if (k.gamma[s] != 0.0f) addp(k.off[s], du, k.gamma[s]);
        }
    for (int i = 0; i < ndof; ++i) {
      T w = weight[i];
      if (!(w > T(0))) continue;
      T xv = x[i], p = aux[i], pp = prev_aux[i];
      T pr = xv - p;
      eta[i] += w * (p - xv);
      pn2 += (double)pr * (double)pr;
      dual[i] += w * (p - pp);
      dcur[i] += eta[i];
      dprev[i] += eta[i];
    }
  }

  void project(std::vector<T>& x) const {
    for (int i = 0; i < ndof; ++i)
      if (weight[i] > T(0)) x[i] = aux[i];
  }
};

// ---------------------------------------------------------------------------
// World.
// ---------------------------------------------------------------------------
template <class T>
struct Cloth {
  u32 id;
  oracle_cloth_config cfg;
  oracle_collision_config col;
  int nv, nf;
  std::vector<int> perm, inv_perm, part_offsets;
  std::vector<float> rest_orig;  // original order
  std::vector<int> F_orig;
  std::vector<int> pins_orig;
  std::vector<float> pin_pos;  // 3 * npins target positions
  bool pin_static = true, pin_static_twice = true;
  std::vector<int> F, E;  // solver order
  float avg_edge = 0;
  Assembly asmb;
  double asm_dt = -1;
  Mas<T> mas;
  bool mas_topo = false;
  std::vector<T> x, v;       // solver order state
  std::vector<T> z, u;       // 6 per face
  std::vector<T> jop;        // 54 per face
  std::vector<T> area_sqrt;  // per face
  Csr H;
  int offset = 0;
  ObjectColl coll;
};

struct Obstacle {
  u32 id;
  oracle_collision_config col;
  int nv;
  std::vector<int> F, E;
  std::vector<float> cur, prev;
  bool is_static = true, is_static_twice = false;
  float avg_edge = 0;
  ObjectColl coll;
};

static void mesh_edges(const std::vector<int>& F, std::vector<int>& E) {
  std::vector<std::pair<int, int>> e;
  for (size_t f = 0; f < F.size() / 3; ++f)
    for (int i = 0; i < 3; ++i) {
      int a = F[3 * f + i], b = F[3 * f + (i + 1) % 3];
      e.emplace_back(std::min(a, b), std::max(a, b));
    }
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  E.clear();
  for (auto& [a, b] : e) {
    E.push_back(a);
    E.push_back(b);
  }
}

static float average_edge_length(const std::vector<float>& V,
                                 const std::vector<int>& E) {
  float s = 0.0f;
  int ne = (int)E.size() / 2;
  for (int i = 0; i < ne; ++i) {
    int a = E[2 * i], b = E[2 * i + 1];
    float dx = V[3 * a] - V[3 * b], dy = V[3 * a + 1] - V[3 * b + 1],
          dz = V[3 * a + 2] - V[3 * b + 2];
    s += std::sqrt(dx * dx + dy * dy + dz * dz);
  }
  return s / (float)ne;
}

template <class T>
struct World {
  oracle_global_config g{};
  std::vector<Cloth<T>> cloths;
  std::vector<Obstacle> obstacles;
  u32 next_id = 1;
  oracle_stats stats{};
  // Scratch shared with debug entry points.
  std::vector<ObjectColl*> objs;

  World() {
    g.acceleration[0] = 0;
    g.acceleration[1] = 0;
    g.acceleration[2] = -10.0f;
    g.max_outer_iteration = 100;
    g.max_inner_iteration = 100;
    g.dt = 1.0f / 60.0f;
    g.linear_solver_abs_tol = 1e-7f;
    g.linear_solver_rel_tol_min = 1e-6f;
    g.linear_solver_rel_tol_max = 1e-3f;
    g.initial_linear_rel_tol = 1e-2f;
    g.admm_abs_tol = 1e-5f;
    g.admm_rel_tol = 1e-3f;
    g.fixed_linear_rel_tol = 0.0f;
    g.cg_max_iter = 1000;
  }

  void setup_cloth(Cloth<T>& c) {
    double dt = g.dt;
    if (c.asm_dt == dt) return;
    std::vector<double> Vp(3 * (size_t)c.nv);
    for (int i = 0; i < c.nv; ++i)
      for (int d = 0; d < 3; ++d) Vp[3 * c.perm[i] + d] = c.rest_orig[3 * i + d];
    c.asmb = assemble(Vp, c.F, c.cfg, dt);
    c.H = c.asmb.H;
    c.jop.assign(c.asmb.jop.begin(), c.asmb.jop.end());
    c.area_sqrt.resize(c.nf);
    for (int f = 0; f < c.nf; ++f) c.area_sqrt[f] = (T)std::sqrt(c.asmb.area[f]);
    if (!c.mas_topo) {
      c.mas.build_topology(c.H, c.part_offsets);
      c.mas_topo = true;
    }
    c.asm_dt = dt;
  }

  void gather_obstacle_positions(Obstacle& o) {
    // obstacle_assembler.cu:50-63.
    if (o.is_static_twice) {
    } else if (o.is_static) {
      o.coll.x0 = o.cur;
      o.coll.x1 = o.cur;
      refit(o.coll);
    } else {
      o.coll.x0 = o.prev;
      o.coll.x1 = o.cur;
      refit(o.coll);
    }
  }

  void set_cloth_collider(Cloth<T>& c, const std::vector<T>& t1,
                          const std::vector<T>& t0) {
    for (int i = 0; i < 3 * c.nv; ++i) {
      c.coll.x0[i] = (float)t0[c.offset + i];
      c.coll.x1[i] = (float)t1[c.offset + i];
    }
    c.coll.state_offset = c.offset;
    refit(c.coll);
  }

  std::vector<Collision> find_active(float time, float dact) {
    std::vector<Collision> out;
    auto cand = candidates(objs);
    for (auto& k : cand) {
      std::optional<Collision> c;
      if (k.kind == 0)
        c = make_pt_collision(*objs[k.oa], k.ia, *objs[k.ob], k.ib, time, dact);
      else
        c = make_ee_collision(*objs[k.oa], k.ia, *objs[k.ob], k.ib, time, dact);
      if (c) out.push_back(*c);
    }
    return out;
  }

  // find_collision.cu:140-190 with every query searched over the full
  // remaining interval (the reference shrinks it with the running minimum).
  float find_min_toi(float time_start, float max_time, float ms, int* nq,
                     int* nh) {
    if (max_time == 0.0f) return 0.0f;
    float absmax[3] = {0, 0, 0};
    for (auto* o : objs)
      for (int d = 0; d < 3; ++d) {
        float mn = o->bbox.mn(d) + o->padding;
        float mx = o->bbox.mx(d) - o->padding;
        absmax[d] = fmax_std(absmax[d], std::fabs(mn));
        absmax[d] = fmax_std(absmax[d], std::fabs(mx));
      }
    float ee_err[3], vf_err[3];
    numerical_error(absmax, false, ee_err);
    numerical_error(absmax, true, vf_err);
    auto cand = candidates(objs);
    float local_max = max_time / max_time;
    float local_tol = 1e-6f / max_time;
    float best = local_max;
    int hits = 0;
    std::vector<float> tois(cand.size(), local_max);
    std::vector<char> hit(cand.size(), 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (long q = 0; q < (long)cand.size(); ++q) {
      const Cand& k = cand[q];
      V3 P[8];
      // ccd_fast_rejection.cu:16-77: trajectories, obstacle re-based.
      auto traj = [&](const ObjectColl& o, int vi, V3& p0, V3& p1) {
        V3 s0 = v3(o.x0[3 * vi], o.x0[3 * vi + 1], o.x0[3 * vi + 2]);
        V3 s1 = v3(o.x1[3 * vi], o.x1[3 * vi + 1], o.x1[3 * vi + 2]);
        V3 delta = vsub(s1, s0);
        if (o.state_offset == -1) {
          p0 = axpby(1.0f, s0, time_start, delta);
          p1 = axpby(1.0f, p0, max_time, delta);
        } else {
          p0 = s0;
          p1 = s1;
        }
      };
      bool vf = k.kind == 0;
      if (vf) {
        const ObjectColl& Tt = *objs[k.oa];
        const ObjectColl& Pp = *objs[k.ob];
        traj(Pp, k.ib, P[0], P[4]);
        traj(Tt, Tt.F[3 * k.ia], P[1], P[5]);
        traj(Tt, Tt.F[3 * k.ia + 1], P[2], P[6]);
        traj(Tt, Tt.F[3 * k.ia + 2], P[3], P[7]);
      } else {
        const ObjectColl& A = *objs[k.oa];
        const ObjectColl& B = *objs[k.ob];
        traj(A, A.E[2 * k.ia], P[0], P[4]);
        traj(A, A.E[2 * k.ia + 1], P[1], P[5]);
        traj(B, B.E[2 * k.ib], P[2], P[6]);
        traj(B, B.E[2 * k.ib + 1], P[3], P[7]);
      }
      float toi;
      if (ccd_toi(vf, P, vf ? vf_err : ee_err, ms, local_tol, 4096, local_max, toi)) {
        hit[q] = 1;
        tois[q] = toi;
      }
    }
    for (size_t q = 0; q < cand.size(); ++q) {
      if (!hit[q]) continue;
      ++hits;
      if (tois[q] == 0.0f) continue;
      best = fmin_std(best, tois[q]);
    }
    if (nq) *nq = (int)cand.size();
    if (nh) *nh = hits;
    return max_time * best;
  }

  void collect_objs() {
    objs.clear();
    for (auto& c : cloths) objs.push_back(&c.coll);
    for (auto& o : obstacles) objs.push_back(&o.coll);
  }

  // cg (mas_cg_solver.cu:193-311) on A = H + diag(lhs), x warm start.
  int cg(Cloth<T>& c, const std::vector<T>& lhs, const std::vector<T>& b,
         std::vector<T>& x, float rel_tol, float abs_tol) {
    int n = 3 * c.nv;
    auto spmv = [&](const std::vector<T>& in, std::vector<T>& out) {
      out.assign(n, T(0));
#pragma omp parallel for schedule(static)
      for (int r = 0; r < n; ++r) {
        T s = 0;
        for (int a = c.H.rows[r]; a < c.H.rows[r + 1]; ++a)
          s += (T)c.H.vals[a] * in[c.H.cols[a]];
        out[r] = s + lhs[r] * in[r];
      }
    };
    // Fixed chunks summed in chunk order: the same value for any thread count
    // (an OpenMP reduction adds the thread partials in the order they finish).
    auto dotp = [&](const std::vector<T>& a, const std::vector<T>& bb) {
      constexpr int kChunk = 4096;
      const int nch = (n + kChunk - 1) / kChunk;
      std::vector<double> part(nch, 0.0);
#pragma omp parallel for schedule(static)
      for (int ch = 0; ch < nch; ++ch) {
        double s = 0;
        const int e = std::min(n, (ch + 1) * kChunk);
        for (int i = ch * kChunk; i < e; ++i) s += (double)a[i] * (double)bb[i];
        part[ch] = s;
      }
      double s = 0;
      for (double v : part) s += v;
      return s;
    };
    std::vector<T> r, z, p, Ap;
    spmv(x, r);
    for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
    c.mas.apply(r, z);
    p = z;
    T rz = (T)dotp(r, z);
    T rr = (T)dotp(r, r);
    if (std::isnan((double)rz) || !std::isfinite((double)rz)) return 0;
    T rr0 = rr;
    int iter = 0;
    int max_iter = g.cg_max_iter > 0 ? g.cg_max_iter : 1000;
    while (true) {
      spmv(p, Ap);
      T pAp = (T)dotp(p, Ap);
      T alpha = (std::fabs((double)pAp) < 1e-20) ? T(0) : rz / pAp;
      for (int i = 0; i < n; ++i) {
        x[i] = alpha * p[i] + x[i];
        r[i] = -alpha * Ap[i] + r[i];
      }
      c.mas.apply(r, z);
      T rz_old = rz;
      rz = (T)dotp(r, z);
      rr = (T)dotp(r, r);
      ++iter;
      bool stop = iter >= max_iter || rr <= (T)abs_tol * (T)abs_tol ||
                  rr <= (T)rel_tol * (T)rel_tol * rr0;
      T beta = (std::fabs((double)rz_old) < 1e-20) ? T(0) : rz / rz_old;
      for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      if (stop) break;
    }
    return iter;
  }

  // ADMM solve (admm_solver.cu:173-342).
  bool admm(const std::vector<T>& prev, const std::vector<T>& prev_v,
            std::vector<T>& x, std::vector<char>& pin_ind,
            std::vector<T>& pin_tgt, Contacts<T>& con) {
    int n = (int)x.size();
    float dt = g.dt;
    std::vector<T> inertia(n);
    for (int i = 0; i < n; ++i)
      inertia[i] = -prev[i] / ((T)dt * (T)dt) - prev_v[i] / (T)dt -
                   (T)g.acceleration[i % 3];
    std::vector<T> lam(n, T(0));
    const T pin_rho = (T)1e4;
    const T maxmul = (T)1e8;
    int pin_dof = 0;
    for (int i = 0; i < n; ++i) pin_dof += pin_ind[i] ? 1 : 0;
    float init_p = 0, init_d = 0, ratio = 1.0f;
    std::vector<T> lhs(n), rhs(n), dual(n), dcur(n), dprev(n);
    for (int it = 0; it < g.max_inner_iteration; ++it) {
      if (it != 0) {
        std::fill(lhs.begin(), lhs.end(), T(0));
        std::fill(rhs.begin(), rhs.end(), T(0));
        for (int i = 0; i < n; ++i)
          if (pin_ind[i]) {
            lhs[i] += pin_rho;
            rhs[i] += pin_rho * pin_tgt[i] - lam[i];
          }
        con.eval(lhs, rhs);
        float rel = std::clamp(g.initial_linear_rel_tol * ratio,
                               g.linear_solver_rel_tol_min,
                               g.linear_solver_rel_tol_max);
        if (g.fixed_linear_rel_tol > 0) rel = g.fixed_linear_rel_tol;
        for (auto& c : cloths) {
          int o = c.offset, m = 3 * c.nv;
          std::vector<T> cl(m), cr(m), xl(m);
          for (int i = 0; i < m; ++i) {
            cl[i] = lhs[o + i] + (T)c.asmb.mass3[i] / ((T)dt * (T)dt);
            cr[i] = rhs[o + i] + (T)c.asmb.bending_rhs[i] -
                    (T)c.asmb.mass3[i] * inertia[o + i];
            xl[i] = x[o + i];
          }
          // assemble_elastic_rhs (cloth_admm_helper.cu:219-271).
          T rho = (T)c.cfg.elastic_stiffness;
          for (int f = 0; f < c.nf; ++f) {
            const T* J = &c.jop[54 * (size_t)f];
            T w = c.area_sqrt[f];
            for (int k = 0; k < 9; ++k) {
              T s = 0;
              for (int r = 0; r < 6; ++r)
                s += J[r * 9 + k] * (-w * c.u[6 * f + r] + w * w * rho * c.z[6 * f + r]);
              int vtx = c.F[3 * f + k / 3];
              cr[3 * vtx + k % 3] += s;
            }
          }
          if (it == 1) {
            std::vector<double> dg(cl.begin(), cl.end());
            c.mas.factorize(c.H, dg);
          }
          int its = cg(c, cl, cr, xl, rel, g.linear_solver_abs_tol);
          stats.cg_iterations += its;
          stats.cg_solves += 1;
          for (int i = 0; i < m; ++i) x[o + i] = xl[i];
        }
      }
      // Aux update.
      double pn2 = 0, px2 = 0, pa2 = 0;
      std::fill(dual.begin(), dual.end(), T(0));
      std::fill(dcur.begin(), dcur.end(), T(0));
      std::fill(dprev.begin(), dprev.end(), T(0));
      for (auto& c : cloths) {
        T rho = (T)c.cfg.elastic_stiffness, k = rho;
        for (int f = 0; f < c.nf; ++f) {
          const T* J = &c.jop[54 * (size_t)f];
          T w = c.area_sqrt[f];
          T xv[9];
          for (int i = 0; i < 3; ++i)
            for (int d = 0; d < 3; ++d) xv[3 * i + d] = x[c.offset + 3 * c.F[3 * f + i] + d];
          T Sx[6], u6[6], zo[6];
          for (int r = 0; r < 6; ++r) {
            T s = 0;
            for (int q = 0; q < 9; ++q) s += J[r * 9 + q] * xv[q];
            Sx[r] = s;
            u6[r] = c.u[6 * f + r];
            zo[r] = c.z[6 * f + r];
          }
          // solve_elastic_aux (cloth_admm_helper.cu:19-51).
          double y[6], proj[6];
          for (int r = 0; r < 6; ++r) y[r] = (double)(Sx[r] + (T(1) / (rho * w)) * u6[r]);
          clamp_projection(y, 0.9, 1.1, proj);
          T rr_ = k / (k + rho);
          T zn[6];
          for (int r = 0; r < 6; ++r) zn[r] = (T(1) - rr_) * (T)y[r] + rr_ * (T)proj[r];
          for (int r = 0; r < 6; ++r) {
            T pr = w * (Sx[r] - zn[r]);
            pn2 += (double)pr * pr;
            px2 += (double)(w * Sx[r]) * (w * Sx[r]);
            pa2 += (double)(w * zn[r]) * (w * zn[r]);
          }
          for (int q = 0; q < 9; ++q) {
            T sc = 0, sp = 0;
            for (int r = 0; r < 6; ++r) {
              sc += J[r * 9 + q] * zn[r];
              sp += J[r * 9 + q] * zo[r];
            }
            T cur = rho * w * w * sc, pv = rho * w * w * sp;
            int dof = c.offset + 3 * c.F[3 * f + q / 3] + q % 3;
            dual[dof] += cur - pv;
            dcur[dof] += cur;
            dprev[dof] += pv;
          }
          for (int r = 0; r < 6; ++r) {
            c.z[6 * f + r] = zn[r];
            T d = w * rho * Sx[r] + -w * rho * zn[r];
            c.u[6 * f + r] = std::clamp(u6[r] + d, -maxmul, maxmul);
          }
        }
      }
      for (int i = 0; i < n; ++i)
        if (pin_ind[i]) lam[i] = std::clamp(lam[i] + pin_rho * (x[i] - pin_tgt[i]), -maxmul, maxmul);
      for (int i = 0; i < n; ++i)
        if (pin_ind[i]) {
          T d = x[i] - pin_tgt[i];
          pn2 += (double)d * d;
          px2 += (double)x[i] * x[i];
          pa2 += (double)pin_tgt[i] * pin_tgt[i];
        }
      con.update(x, pn2, dual, dcur, dprev);
      stats.admm_iterations += 1;
      if (it == 0) continue;
      for (int i = 0; i < n; ++i)
        if (!std::isfinite((double)x[i])) return false;
      float pnorm = std::sqrt((float)pn2);
      if (it == 1) init_p = pnorm;
      int dof = 0;
      for (auto& c : cloths) dof += 6 * c.nf;
      dof += pin_dof + con.active_dof;
      auto crit = [&](int d, float a2, float b2) {
        return (float)std::sqrt((double)d) * g.admm_abs_tol +
               std::max(std::sqrt(a2), std::sqrt(b2)) * g.admm_rel_tol;
      };
      float peps = crit(dof, (float)px2, (float)pa2);
      double d2 = 0, c2 = 0, q2 = 0;
      for (int i = 0; i < n; ++i) {
        d2 += (double)dual[i] * dual[i];
        c2 += (double)dcur[i] * dcur[i];
        q2 += (double)dprev[i] * dprev[i];
      }
      float dnorm = std::sqrt((float)d2);
      if (it == 1) init_d = dnorm;
      float deps = crit(n, (float)c2, (float)q2);
      ratio = std::max(pnorm / std::max(init_p, g.admm_abs_tol),
                       dnorm / std::max(init_d, g.admm_abs_tol));
      if (pnorm <= peps && dnorm <= deps) break;
    }
    for (int i = 0; i < n; ++i)
      if (pin_ind[i]) x[i] = pin_tgt[i];
    con.project(x);
    return true;
  }

  // MainLoop::step (main_loop.cu:140-278).
  int step() {
    stats = oracle_stats{};
    int n = 0;
    for (auto& c : cloths) {
      setup_cloth(c);
      c.offset = n;
      n += 3 * c.nv;
    }
    if (n == 0) return 1;
    for (auto& o : obstacles) gather_obstacle_positions(o);
    float dt = g.dt;
    std::vector<T> prev(n), prev_v(n);
    for (auto& c : cloths) {
      T damp = T(1) - (T)c.cfg.damping;
      for (int i = 0; i < 3 * c.nv; ++i) {
        prev[c.offset + i] = c.x[i];
        prev_v[c.offset + i] = damp * c.v[i];
      }
      std::fill(c.z.begin(), c.z.end(), T(0));
      std::fill(c.u.begin(), c.u.end(), T(0));
    }
    collect_objs();
    float pad = objs[0]->padding;
    for (auto* o : objs) pad = fmin_std(pad, o->padding);
    float ms = 0.2f * pad;
    float dact = 1.0f * pad;
    std::vector<T> outer = prev, outer_v = prev_v, inner(n);
    // Pins (pin_constraints.cu:50-107).
    std::vector<char> pin_ind(n, 0);
    std::vector<T> pin_tgt(n, T(0));
    for (auto& c : cloths)
      for (size_t k = 0; k < c.pins_orig.size(); ++k) {
        int v = c.perm[c.pins_orig[k]];
        for (int d = 0; d < 3; ++d) {
          pin_ind[c.offset + 3 * v + d] = 1;
          pin_tgt[c.offset + 3 * v + d] = (T)c.pin_pos[3 * k + d];
        }
      }
    // Contacts.
    std::vector<T> bw(n, T(0));
    for (auto& c : cloths)
      for (int i = 0; i < 3 * c.nv; ++i) bw[c.offset + i] = (T)c.asmb.contact_weight[i];
    Contacts<T> con;
    con.init(n, bw);
    for (auto& c : cloths) set_cloth_collider(c, outer, outer);
    con.append(find_active(0.0f, dact));
    float remaining = 1.0f;
    for (int oit = 0; oit < g.max_outer_iteration; ++oit) {
      stats.outer_iterations += 1;
      // predict (main_loop.cu:78-98).
      for (int i = 0; i < n / 3; ++i)
        for (int d = 0; d < 3; ++d) {
          int k = 3 * i + d;
          T nx = T(1) * outer[k] + (T)dt * outer_v[k];
          inner[k] = T(1) * nx + (T)dt * (T)dt * (T)g.acceleration[d];
        }
      if (!admm(prev, prev_v, inner, pin_ind, pin_tgt, con)) return 2;
      for (auto& c : cloths) set_cloth_collider(c, inner, outer);
      float ts = 1.0f - remaining;
      int nq = 0, nh = 0;
      float toi = find_min_toi(ts, remaining, ms, &nq, &nh);
      stats.ccd_queries += nq;
      stats.ccd_hits += nh;
      stats.min_toi = toi;
      for (int i = 0; i < n; ++i) outer_v[i] = (inner[i] - outer[i]) / (T)dt;
      if (toi >= remaining) {
        outer = inner;
        break;
      }
      float rb = 0.8f * toi;
      float w = rb / remaining;
      for (int i = 0; i < n; ++i)
        outer[i] = (T)((double)((T)w * inner[i]) + (1.0 - (double)w) * (double)outer[i]);
      remaining -= rb;
      for (auto& c : cloths) set_cloth_collider(c, outer, outer);
      con.append(find_active(1.0f - remaining, dact));
    }
    for (int i = 0; i < n; ++i) outer_v[i] = (outer[i] - prev[i]) / (T)dt;
    for (auto& c : cloths) {
      for (int i = 0; i < 3 * c.nv; ++i) {
        c.x[i] = outer[c.offset + i];
        c.v[i] = outer_v[c.offset + i];
      }
    }
    for (auto& o : obstacles) {
      o.prev = o.cur;
      if (o.is_static) o.is_static_twice = true;
      else o.is_static = true;
    }
    stats.contacts = (int)con.list.size();
    stats.colors = (int)con.groups.size();
    return 0;
  }
};

struct AnyWorld {
  bool fp64;
  World<float>* f = nullptr;
  World<double>* d = nullptr;
};

template <class T>
static int add_cloth_impl(World<T>& W, const oracle_cloth_config* cc,
                          const oracle_collision_config* col, const float* verts,
                          int nv, const int* faces, int nf, const int* pins,
                          int np, const int* perm, const int* part_offsets,
                          int nparts, uint32_t* handle) {
  Cloth<T> c;
  c.id = W.next_id++;
  c.cfg = *cc;
  c.col = *col;
  c.nv = nv;
  c.nf = nf;
  c.rest_orig.assign(verts, verts + 3 * nv);
  c.F_orig.assign(faces, faces + 3 * nf);
  c.pins_orig.assign(pins, pins + np);
  c.perm.assign(perm, perm + nv);
  c.inv_perm.assign(nv, 0);
  for (int i = 0; i < nv; ++i) c.inv_perm[c.perm[i]] = i;
  c.part_offsets.assign(part_offsets, part_offsets + nparts + 1);
  std::vector<int> E_orig;
  mesh_edges(c.F_orig, E_orig);
  c.avg_edge = average_edge_length(c.rest_orig, E_orig);
  c.F.resize(3 * nf);
  for (int i = 0; i < 3 * nf; ++i) c.F[i] = c.perm[c.F_orig[i]];
  c.E.resize(E_orig.size());
  for (size_t i = 0; i < E_orig.size(); ++i) c.E[i] = c.perm[E_orig[i]];
  c.pin_pos.resize(3 * (size_t)np);
  for (int k = 0; k < np; ++k)
    for (int d = 0; d < 3; ++d) c.pin_pos[3 * k + d] = verts[3 * pins[k] + d];
  c.x.assign(3 * (size_t)nv, T(0));
  c.v.assign(3 * (size_t)nv, T(0));
  for (int i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) c.x[3 * c.perm[i] + d] = (T)verts[3 * i + d];
  c.z.assign(6 * (size_t)nf, T(0));
  c.u.assign(6 * (size_t)nf, T(0));
  // Collider (object_collider.cu:119-177).
  ObjectColl& o = c.coll;
  o.id = c.id;
  o.physical = true;
  o.group = col->is_collision_on ? col->group : -1;
  o.self_on = col->is_self_collision_on != 0;
  o.padding = 0.05f * c.avg_edge;
  o.friction = col->friction;
  o.state_offset = 0;
  o.nv = nv;
  o.F = c.F;
  o.E = c.E;
  o.x0.assign(3 * (size_t)nv, 0.f);
  for (int i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) o.x0[3 * c.perm[i] + d] = verts[3 * i + d];
  o.x1 = o.x0;
  W.cloths.push_back(std::move(c));
  Cloth<T>& cr = W.cloths.back();
  W.setup_cloth(cr);
  std::vector<char> pinned(nv, 0);
  for (int k = 0; k < np; ++k) pinned[cr.perm[pins[k]]] = 1;
  cr.coll.inv_mass.resize(nv);
  for (int i = 0; i < nv; ++i) {
    float m = cr.cfg.density * (float)cr.asmb.mass[i];
    cr.coll.inv_mass[i] = pinned[i] ? 0.0f : 1.0f / m;
  }
  refit(cr.coll);
  *handle = cr.id;
  return 0;
}

template <class T>
static int add_obstacle_impl(World<T>& W, const oracle_collision_config* col,
                             const float* verts, int nv, const int* faces,
                             int nf, uint32_t* handle) {
  Obstacle o;
  o.id = W.next_id++;
  o.col = *col;
  o.nv = nv;
  o.F.assign(faces, faces + 3 * nf);
  mesh_edges(o.F, o.E);
  o.cur.assign(verts, verts + 3 * nv);
  o.prev = o.cur;
  o.avg_edge = average_edge_length(o.cur, o.E);
  ObjectColl& c = o.coll;
  c.id = o.id;
  c.physical = false;
  c.group = col->is_collision_on ? col->group : -1;
  c.self_on = col->is_self_collision_on != 0;
  c.padding = 0.05f * o.avg_edge;
  c.friction = col->friction;
  c.state_offset = -1;
  c.nv = nv;
  c.F = o.F;
  c.E = o.E;
  c.inv_mass.assign(nv, 0.0f);
  c.x0 = o.cur;
  c.x1 = o.cur;
  refit(c);
  W.obstacles.push_back(std::move(o));
  *handle = W.obstacles.back().id;
  return 0;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void* oracle_world_new(int fp64) {
  AnyWorld* a = new AnyWorld;
  a->fp64 = fp64 != 0;
  if (a->fp64) a->d = new World<double>();
  else a->f = new World<float>();
  return a;
}

void oracle_world_free(void* w) {
  AnyWorld* a = (AnyWorld*)w;
  delete a->f;
  delete a->d;
  delete a;
}

int oracle_set_global_config(void* w, const oracle_global_config* c) {
  AnyWorld* a = (AnyWorld*)w;
  if (a->fp64) a->d->g = *c;
  else a->f->g = *c;
  return 0;
}

int oracle_add_cloth(void* w, const oracle_cloth_config* cc,
                     const oracle_collision_config* col, const float* verts,
                     int nv, const int* faces, int nf, const int* pins,
                     int npins, const int* perm, const int* part_offsets,
                     int nparts, uint32_t* handle) {
  AnyWorld* a = (AnyWorld*)w;
  if (a->fp64)
    return add_cloth_impl(*a->d, cc, col, verts, nv, faces, nf, pins, npins,
                          perm, part_offsets, nparts, handle);
  return add_cloth_impl(*a->f, cc, col, verts, nv, faces, nf, pins, npins,
                        perm, part_offsets, nparts, handle);
}

int oracle_add_obstacle(void* w, const oracle_collision_config* col,
                        const float* verts, int nv, const int* faces, int nf,
                        uint32_t* handle) {
  AnyWorld* a = (AnyWorld*)w;
  if (a->fp64) return add_obstacle_impl(*a->d, col, verts, nv, faces, nf, handle);
  return add_obstacle_impl(*a->f, col, verts, nv, faces, nf, handle);
}

int oracle_set_obstacle_position(void* w, uint32_t h, const float* pos, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& o : W.obstacles)
      if (o.id == h) {
        if (n != 3 * o.nv) return 7;
        o.is_static = false;
        o.is_static_twice = false;
        std::swap(o.cur, o.prev);
        o.cur.assign(pos, pos + n);
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_set_cloth_pin_position(void* w, uint32_t h, const float* pos, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if ((size_t)n != 3 * c.pins_orig.size()) return 6;
        c.pin_pos.assign(pos, pos + n);
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_solver_step(void* w) {
  AnyWorld* a = (AnyWorld*)w;
  return a->fp64 ? a->d->step() : a->f->step();
}

int oracle_set_cloth_state(void* w, uint32_t h, const float* x, const float* v,
                           int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        for (int i = 0; i < c.nv; ++i)
          for (int d = 0; d < 3; ++d) {
            c.x[3 * c.perm[i] + d] = x[3 * i + d];
            c.v[3 * c.perm[i] + d] = v[3 * i + d];
          }
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_get_cloth_position(void* w, uint32_t h, float* out, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        for (int i = 0; i < c.nv; ++i)
          for (int d = 0; d < 3; ++d) out[3 * i + d] = (float)c.x[3 * c.perm[i] + d];
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_get_cloth_velocity(void* w, uint32_t h, float* out, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        for (int i = 0; i < c.nv; ++i)
          for (int d = 0; d < 3; ++d) out[3 * i + d] = (float)c.v[3 * c.perm[i] + d];
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_get_cloth_position_f64(void* w, uint32_t h, double* out, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        for (int i = 0; i < c.nv; ++i)
          for (int d = 0; d < 3; ++d) out[3 * i + d] = (double)c.x[3 * c.perm[i] + d];
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_get_stats(void* w, oracle_stats* s) {
  AnyWorld* a = (AnyWorld*)w;
  *s = a->fp64 ? a->d->stats : a->f->stats;
  return 0;
}

int oracle_cloth_dense_scalar_matrix(void* w, uint32_t h, double* out, int nv) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (nv != c.nv) return 7;
        std::fill(out, out + (size_t)nv * nv, 0.0);
        for (int r = 0; r < c.H.n; r += 3)
          for (int k = c.H.rows[r]; k < c.H.rows[r + 1]; ++k)
            if (c.H.cols[k] % 3 == 0) out[(size_t)(r / 3) * nv + c.H.cols[k] / 3] = c.H.vals[k];
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_cloth_dense_full_matrix(void* w, uint32_t h, double* out, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        std::fill(out, out + (size_t)n * n, 0.0);
        for (int r = 0; r < c.H.n; ++r)
          for (int k = c.H.rows[r]; k < c.H.rows[r + 1]; ++k)
            out[(size_t)r * n + c.H.cols[k]] = c.H.vals[k];
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_cloth_vectors(void* w, uint32_t h, double* mass3, double* cw,
                         double* brhs, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    for (auto& c : W.cloths)
      if (c.id == h) {
        if (n != 3 * c.nv) return 7;
        for (int i = 0; i < n; ++i) {
          mass3[i] = c.asmb.mass3[i];
          cw[i] = c.asmb.contact_weight[i];
          brhs[i] = c.asmb.bending_rhs[i];
        }
        return 0;
      }
    return 4;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_debug_refit(void* w, const float* disp, int n) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    int off = 0;
    for (auto& c : W.cloths) {
      for (int i = 0; i < c.nv; ++i)
        for (int d = 0; d < 3; ++d) {
          int s = 3 * c.perm[i] + d;
          c.coll.x0[s] = (float)c.x[s];
          c.coll.x1[s] = (disp && off + 3 * i + d < n)
                             ? (float)c.x[s] + disp[off + 3 * i + d]
                             : (float)c.x[s];
        }
      refit(c.coll);
      off += 3 * c.nv;
    }
    for (auto& o : W.obstacles) W.gather_obstacle_positions(o);
    W.collect_objs();
    return 0;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_debug_candidates(void* w, int* out, int cap) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    auto cand = candidates(W.objs);
    int n = (int)cand.size();
    for (int i = 0; i < n && i < cap; ++i) {
      out[5 * i] = cand[i].kind;
      out[5 * i + 1] = (int)W.objs[cand[i].oa]->id;
      out[5 * i + 2] = cand[i].ia;
      out[5 * i + 3] = (int)W.objs[cand[i].ob]->id;
      out[5 * i + 4] = cand[i].ib;
    }
    return n;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

int oracle_debug_dcd(void* w, float t, float dact, int* keys, int cap) {
  AnyWorld* a = (AnyWorld*)w;
  auto impl = [&](auto& W) {
    auto cols = W.find_active(t, dact);
    std::vector<ContactKey> ks;
    for (auto& c : cols) ks.push_back(make_key(c));
    std::sort(ks.begin(), ks.end());
    int n = (int)ks.size();
    for (int i = 0; i < n && i < cap; ++i) {
      keys[7 * i] = ks[i].type;
      keys[7 * i + 1] = (int)ks[i].oa;
      keys[7 * i + 2] = (int)ks[i].ob;
      for (int k = 0; k < 4; ++k) keys[7 * i + 3 + k] = ks[i].idx[k];
    }
    return n;
  };
  return a->fp64 ? impl(*a->d) : impl(*a->f);
}

float oracle_debug_min_toi(void* w, float time_start, float max_time, float ms,
                           int* nq, int* nh) {
  AnyWorld* a = (AnyWorld*)w;
  return a->fp64 ? a->d->find_min_toi(time_start, max_time, ms, nq, nh)
                 : a->f->find_min_toi(time_start, max_time, ms, nq, nh);
}

long oracle_ccd_max_pending(int reset) {
  long r = (long)g_max_pending;
  if (reset) g_max_pending = 0;
  return r;
}

int oracle_ccd(int is_vf, const float* x, const float* err, float ms, float tol,
               long max_iter, int no_zero_toi, float max_time, float* t4,
               int* use_small) {
  V3 P[8];
  for (int i = 0; i < 8; ++i) P[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  auto r = is_vf ? ccd<true>(P, err, ms, tol, max_iter, no_zero_toi != 0, max_time)
                 : ccd<false>(P, err, ms, tol, max_iter, no_zero_toi != 0, max_time);
  if (!r) return 0;
  t4[0] = r->t0;
  t4[1] = r->t1;
  t4[2] = r->small_t0;
  t4[3] = r->small_t1;
  *use_small = r->use_small_ms ? 1 : 0;
  return 1;
}

int oracle_exact_ee_uv(const float* x, float eps, float* uv) {
  V3 P[4];
  for (int i = 0; i < 4; ++i) P[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  return exact_ee_uv(P[0], P[1], P[2], P[3], eps, uv[0], uv[1]) ? 1 : 0;
}

int oracle_exact_pt_uv(const float* x, float eps, float* uv) {
  V3 P[4];
  for (int i = 0; i < 4; ++i) P[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  return exact_pt_uv(P[0], P[1], P[2], P[3], eps, uv[0], uv[1]) ? 1 : 0;
}

void oracle_solve_coulomb(const float* u, const float* n, float mu, float* out) {
  V3 r = solve_coulomb(v3(u[0], u[1], u[2]), v3(n[0], n[1], n[2]), mu);
  out[0] = r(0);
  out[1] = r(1);
  out[2] = r(2);
}

void oracle_numerical_error(const float* absmax, int is_vf, float* out) {
  numerical_error(absmax, is_vf != 0, out);
}

int oracle_color_contacts(const int* verts4, const uint64_t* prio, int n,
                          int* colors) {
  std::vector<std::array<int, 4>> v(n);
  std::vector<u64> p(prio, prio + n);
  for (int i = 0; i < n; ++i)
    for (int s = 0; s < 4; ++s) v[i][s] = verts4[4 * i + s];
  std::vector<int> c;
  int nc = color_greedy(v, p, c);
  for (int i = 0; i < n; ++i) colors[i] = c[i];
  return nc;
}

void oracle_clamp_projection(const float* f6, float lo, float hi, float* out6) {
  double f[6], o[6];
  for (int i = 0; i < 6; ++i) f[i] = f6[i];
  clamp_projection(f, lo, hi, o);
  for (int i = 0; i < 6; ++i) out6[i] = (float)o[i];
}

}  // extern "C"
