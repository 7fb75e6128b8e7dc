// Collision pipeline on the GPU.
//
// Reference: backend/cuda/collision/object_collider.cu:21-378 (colliders and
// padded swept boxes), oibvh.cuh:43-688 (implicit-tree BVH over Morton-sorted
// colliders and stack traversal), find_collision.cu:17-211 (object SAP,
// primitive filters, candidate enumeration), dcd.cu:23-315 (active contacts),
// ccd_fast_rejection.cu:16-77 (CCD queries), narrowphase.cu:32-105 and the
// in-tree Tight-Inclusion restatement backend/cpu/collision/ccd.cpp:13-204 +
// interval_root_finder.cpp:13-522 (CCD), solver/contact_constraints.cu:24-599
// and contact_coloring.cu:26-373 (contacts and colouring).
//
// This file is compiled with --fmad=false: the CCD and DCD arithmetic keeps
// the reference's single-precision operation sequence so that hit / no-hit
// decisions and times of impact equal the CPU restatement bit for bit.
//
// Differences by design (documented, deterministic):
//  * every CCD query searches the full remaining interval (the reference lets
//    a shrinking running minimum cut later queries short, which makes its
//    answer depend on thread timing);
//  * contacts of one DCD call are appended in canonical key order and
//    coloured greedily in decreasing order of a 64-bit hash of the key
//    (Jones-Plassmann rounds), which is the same colouring the CPU oracle
//    computes sequentially;
//  * the tree is refitted between re-sorts; any leaf order yields the same
//    candidate set because the set is defined by box overlap alone.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "collision.cuh"
#include "grid_barrier.cuh"
#include "world.hpp"

namespace silkb {

namespace {

constexpr int kCollThreads = 128;
constexpr float kDcdEps = 1e-6f;       // dcd.cu:18
constexpr int kCcdMaxIter = 4096;      // main_loop.cuh:24
constexpr float kCcdTolerance = 1e-6f; // main_loop.cuh:23
constexpr int kGsSweeps = 10;          // contact_constraints.cuh:89
constexpr int kCcdStack = 96;

// std::min / std::max semantics.
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct Box {
  float3 mn, mx;
};

__device__ __forceinline__ Box box_pad(Box b, float p) {
  Box o;
  o.mn = make_float3(1.0f * b.mn.x + -p, 1.0f * b.mn.y + -p, 1.0f * b.mn.z + -p);
  o.mx = make_float3(1.0f * b.mx.x + p, 1.0f * b.mx.y + p, 1.0f * b.mx.z + p);
  return o;
}
__device__ __forceinline__ float3 vmin3(float3 a, float3 b) {
  return make_float3(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z));
}
__device__ __forceinline__ float3 vmax3(float3 a, float3 b) {
  return make_float3(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z));
}
__device__ __forceinline__ bool overlap(const Box& a, const Box& b) {
  float3 p = vmax3(a.mn, b.mn), q = vmin3(a.mx, b.mx);
  return p.x <= q.x && p.y <= q.y && p.z <= q.z;
}
__device__ __forceinline__ Box load_box(const float4* bb, int i) {
  float4 a = bb[2 * i], b = bb[2 * i + 1];
  return Box{make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z)};
}
__device__ __forceinline__ void store_box(float4* bb, int i, const Box& b) {
  bb[2 * i] = make_float4(b.mn.x, b.mn.y, b.mn.z, 0.f);
  bb[2 * i + 1] = make_float4(b.mx.x, b.mx.y, b.mx.z, 0.f);
}
__device__ __forceinline__ Box merge(const Box& a, const Box& b) {
  return Box{vmin3(a.mn, b.mn), vmax3(a.mx, b.mx)};
}
__device__ __forceinline__ Box empty_box() {
  const float inf = __int_as_float(0x7f800000);
  return Box{make_float3(inf, inf, inf), make_float3(-inf, -inf, -inf)};
}

struct ObjDev {
  const float4* x0;
  const float4* x1;
  const int4* F;
  const int2* E;
  const float* inv_mass;
  int nv, nf, ne;
  float padding, friction;
  int handle;
  int voff;  // global vertex offset of a cloth, -1 for an obstacle
  float4* tri_bb;
  float4* edge_bb;
  float4* pt_bb;
  // Trees (triangles, edges).
  int tri_D, edge_D;
  const float4* tri_nodes;
  const int* tri_order;
  const float4* edge_nodes;
  const int* edge_order;
  float4* obj_box;  // reduced box (2 float4)
};

__device__ __forceinline__ float3 P(const float4* x, int i) {
  float4 q = x[i];
  return make_float3(q.x, q.y, q.z);
}

// Padded swept boxes (object_collider.cu:280-378) and block partial boxes of
// the triangles for the object box.
__global__ void refit_kernel(const ObjDev* objs, int slot, float4* partial) {
  const ObjDev& o = objs[slot];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  Box tb = empty_box();
  if (i < o.nf) {
    int4 f = o.F[i];
    float3 a0 = P(o.x0, f.x), b0 = P(o.x0, f.y), c0 = P(o.x0, f.z);
    float3 a1 = P(o.x1, f.x), b1 = P(o.x1, f.y), c1 = P(o.x1, f.z);
    Box b;
    b.mn = vmin3(vmin3(vmin3(a0, b0), c0), vmin3(vmin3(a1, b1), c1));
    b.mx = vmax3(vmax3(vmax3(a0, b0), c0), vmax3(vmax3(a1, b1), c1));
    tb = box_pad(b, o.padding);
    store_box(o.tri_bb, i, tb);
  }
  if (i < o.ne) {
    int2 e = o.E[i];
    float3 a0 = P(o.x0, e.x), b0 = P(o.x0, e.y), a1 = P(o.x1, e.x), b1 = P(o.x1, e.y);
    Box b;
    b.mn = vmin3(vmin3(a0, b0), vmin3(a1, b1));
    b.mx = vmax3(vmax3(a0, b0), vmax3(a1, b1));
    store_box(o.edge_bb, i, box_pad(b, o.padding));
  }
  if (i < o.nv) {
    float3 a0 = P(o.x0, i), a1 = P(o.x1, i);
    Box b{vmin3(a0, a1), vmax3(a0, a1)};
    store_box(o.pt_bb, i, box_pad(b, o.padding));
  }
  // Block reduction of triangle boxes (min/max are exact in any order).
  __shared__ float sh[6][kCollThreads];
  sh[0][threadIdx.x] = tb.mn.x;
  sh[1][threadIdx.x] = tb.mn.y;
  sh[2][threadIdx.x] = tb.mn.z;
  sh[3][threadIdx.x] = tb.mx.x;
  sh[4][threadIdx.x] = tb.mx.y;
  sh[5][threadIdx.x] = tb.mx.z;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      for (int k = 0; k < 3; ++k)
        sh[k][threadIdx.x] = smin(sh[k][threadIdx.x], sh[k][threadIdx.x + s]);
      for (int k = 3; k < 6; ++k)
        sh[k][threadIdx.x] = smax(sh[k][threadIdx.x], sh[k][threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = make_float4(sh[0][0], sh[1][0], sh[2][0], 0.f);
    partial[2 * blockIdx.x + 1] = make_float4(sh[3][0], sh[4][0], sh[5][0], 0.f);
  }
}

__global__ void reduce_box_kernel(const ObjDev* objs, int slot, const float4* partial,
                                  int n) {
  __shared__ Box sb[kCollThreads];
  Box b = empty_box();
  for (int i = threadIdx.x; i < n; i += blockDim.x) b = merge(b, load_box(partial, i));
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sb[threadIdx.x] = merge(sb[threadIdx.x], sb[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) store_box(objs[slot].obj_box, 0, sb[0]);
}

__device__ __forceinline__ unsigned long long spread21(unsigned x) {
  unsigned long long y = x & 0x1fffffu;
  y = (y | y << 32) & 0x1f00000000ffffULL;
  y = (y | y << 16) & 0x1f0000ff0000ffULL;
  y = (y | y << 8) & 0x100f00f00f00f00fULL;
  y = (y | y << 4) & 0x10c30c30c30c30c3ULL;
  y = (y | y << 2) & 0x1249249249249249ULL;
  return y;
}

// 63-bit Morton code of box centres in the object box (oibvh.cuh:112-168).
__global__ void morton_kernel(const ObjDev* objs, int slot, int kind, int n,
                              unsigned long long* keys, int* vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ObjDev& o = objs[slot];
  Box root = load_box(o.obj_box, 0);
  Box b = load_box(kind == 0 ? o.tri_bb : o.edge_bb, i);
  float c[3] = {0.5f * b.mn.x + 0.5f * b.mx.x, 0.5f * b.mn.y + 0.5f * b.mx.y,
                0.5f * b.mn.z + 0.5f * b.mx.z};
  float lo[3] = {root.mn.x, root.mn.y, root.mn.z};
  float hi[3] = {root.mx.x, root.mx.y, root.mx.z};
  unsigned long long code = 0;
  for (int d = 0; d < 3; ++d) {
    float cell_len = (hi[d] - lo[d]) / 2097152.0f;
    float inv = cell_len < 1e-20f ? 1e20f : 1.0f / cell_len;
    float fc = (c[d] - lo[d]) * inv;
    fc = fminf(fmaxf(fc, 0.0f), 2097151.0f);
    code |= spread21((unsigned)floorf(fc)) << d;
  }
  keys[i] = code;
  vals[i] = i;
}

// Leaves of the implicit complete tree (2^D leaves, virtual leaves empty).
__global__ void tree_leaves_kernel(const float4* prim_bb, const int* order, int n,
                                   int P, float4* nodes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  Box b = i < n ? load_box(prim_bb, order[i]) : empty_box();
  store_box(nodes, (P - 1) + i, b);
}

// Up to 8 levels of bottom-up merging per launch, one subtree per block.
__global__ void tree_up_kernel(float4* nodes, int L, int k) {
  __shared__ Box sb[256];
  int count = 1 << L;
  int per = count < 256 ? count : 256;
  int base = blockIdx.x * per;
  int t = threadIdx.x;
  if (t < per) sb[t] = load_box(nodes, ((1 << L) - 1) + base + t);
  __syncthreads();
  for (int s = 1; s <= k; ++s) {
    int m = per >> s;
    Box b;
    if (t < m) b = merge(sb[2 * t], sb[2 * t + 1]);
    __syncthreads();
    if (t < m) {
      sb[t] = b;
      int lvl = L - s;
      store_box(nodes, ((1 << lvl) - 1) + (base >> s) + t, b);
    }
    __syncthreads();
  }
}

// Candidate record: x = primitive of A, y = primitive of B,
// z = (kind << 16) | slot A, w = slot B.  kind 0: A triangle / B point;
// kind 1: A edge / B edge.
struct Emitter {
  int4* out;
  int cap;
  int* counter;
  int4 buf[8];
  int n = 0;
  __device__ void flush() {
    if (n == 0) return;
    int at = atomicAdd(counter, n);
    for (int i = 0; i < n; ++i)
      if (at + i < cap) out[at + i] = buf[i];
    n = 0;
  }
  __device__ void push(int4 r) {
    buf[n++] = r;
    if (n == 8) flush();
  }
};

// One query primitive per thread against the tree of another primitive set
// (oibvh.cuh:418-516).  mode: 0 PT inter, 1 PT self, 2 EE inter, 3 EE self.
__global__ void traverse_kernel(const ObjDev* objs, int tslot, int qslot, int mode,
                                int4* out, int cap, int* counter) {
  const ObjDev& T = objs[tslot];
  const ObjDev& Q = objs[qslot];
  bool pt = mode < 2;
  bool self = (mode & 1) != 0;
  int nq = pt ? Q.nv : Q.ne;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  Emitter em{out, cap, counter};
  if (q < nq) {
    int qprim = (mode == 3) ? Q.edge_order[q] : q;
    Box qb = load_box(pt ? Q.pt_bb : Q.edge_bb, qprim);
    int D = pt ? T.tri_D : T.edge_D;
    int n = pt ? T.nf : T.ne;
    const float4* nodes = pt ? T.tri_nodes : T.edge_nodes;
    const int* order = pt ? T.tri_order : T.edge_order;
    const float4* prim_bb = pt ? T.tri_bb : T.edge_bb;
    int Pn = 1 << D;
    unsigned stack[64];
    int sp = 0;
    if (n > 0) stack[sp++] = 0u;
    while (sp > 0) {
      unsigned node = stack[--sp];
      int depth = 31 - __clz((int)(node + 1u));
      if (!overlap(qb, load_box(nodes, (int)node))) continue;
      if (depth == D) {
        int leaf = (int)node - (Pn - 1);
        if (leaf >= n) continue;
        if (mode == 3 && !(leaf < q)) continue;
        int tprim = order[leaf];
        if (!overlap(qb, load_box(prim_bb, tprim))) continue;
        if (pt) {
          int4 f = T.F[tprim];
          float s = Q.inv_mass[qprim] + T.inv_mass[f.x] + T.inv_mass[f.y] + T.inv_mass[f.z];
          if (s == 0.0f) continue;
          if (self && (f.x == qprim || f.y == qprim || f.z == qprim)) continue;
          em.push(make_int4(tprim, qprim, (0 << 16) | tslot, qslot));
        } else {
          int2 a = T.E[tprim], b = Q.E[qprim];
          float s = T.inv_mass[a.x] + T.inv_mass[a.y] + Q.inv_mass[b.x] + Q.inv_mass[b.y];
          if (s == 0.0f) continue;
          if (self && (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y)) continue;
          if (self) {
            int lo = tprim < qprim ? tprim : qprim, hi = tprim < qprim ? qprim : tprim;
            em.push(make_int4(lo, hi, (1 << 16) | tslot, qslot));
          } else {
            em.push(make_int4(tprim, qprim, (1 << 16) | tslot, qslot));
          }
        }
      } else {
        stack[sp++] = 2u * node + 2u;
        stack[sp++] = 2u * node + 1u;
      }
    }
  }
  em.flush();
}

// ---------------------------------------------------------------------------
// DCD (dcd.cu:23-238).
// ---------------------------------------------------------------------------
struct CollisionDev {
  int type;
  int slot_a, slot_b;
  int idx[4];
  float dact, friction;
  float3 normal;
  float coef[4];
  float inv_mass[4];
  float3 x[4];
  float3 prescribed;
};

__device__ __forceinline__ float3 lerp_t(float3 a, float3 b, float t) {
  return make_float3((1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y,
                     (1.0f - t) * a.z + t * b.z);
}
__device__ __forceinline__ float3 sub3(float3 a, float3 b) {
  return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ float3 add3(float3 a, float3 b) {
  return make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
}
__device__ __forceinline__ float3 sc3(float s, float3 a) {
  return make_float3(s * a.x, s * a.y, s * a.z);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}

// Exact Signorini-Coulomb projection of one contact's free displacement us
// onto the friction cone of unit normal n and coefficient mu: separating
// displacements (us.n >= 0) stay, sticking ones (tangential part inside the
// cone) become zero, sliding ones keep the tangential part shortened by the
// cone radius (solve_coulomb_contact, contact_constraints.cu:391-411).  The
// stick test compares squared lengths and the slide scales by
// 1 - radius * rsqrt(|u_t|^2): one reciprocal square root instead of a square
// root and a division.
// The arithmetic uses fused multiply-adds (explicitly: this file is built
// without contraction for the CCD), as does the rest of the contact
// Gauss-Seidel (gs_accum, gs_move).
__device__ __forceinline__ float3 coulomb_project(float3 us, float3 n, float mu) {
  const float un = fmaf(us.z, n.z, fmaf(us.y, n.y, us.x * n.x));
  if (un >= 0.0f) return us;
  const float3 ut = make_float3(fmaf(-un, n.x, us.x), fmaf(-un, n.y, us.y), fmaf(-un, n.z, us.z));
  const float ut2 = fmaf(ut.z, ut.z, fmaf(ut.y, ut.y, ut.x * ut.x));
  const float radius = -mu * un;
  return ut2 <= radius * radius ? make_float3(0.f, 0.f, 0.f)
                                : sc3(fmaf(-radius, rsqrtf(ut2), 1.0f), ut);
}

// Contact Gauss-Seidel updates shared by its three forms (identical bits):
// u += c x (relative position of a contact) and x += g d (a vertex moved by
// its share g of a correction d).
__device__ __forceinline__ float3 gs_accum(float3 u, float c, float4 x) {
  return make_float3(fmaf(c, x.x, u.x), fmaf(c, x.y, u.y), fmaf(c, x.z, u.z));
}
__device__ __forceinline__ float4 gs_move(float4 x, float g, float3 d) {
  return make_float4(fmaf(g, d.x, x.x), fmaf(g, d.y, x.y), fmaf(g, d.z, x.z), 0.f);
}
__device__ __forceinline__ float3 axpby3(float a, float3 x, float b, float3 y) {
  return make_float3(a * x.x + b * y.x, a * x.y + b * y.y, a * x.z + b * y.z);
}

__device__ bool exact_pt_uv(float3 x0, float3 x1, float3 x2, float3 x3, float eps,
                            float& u, float& v) {
  float3 x21 = sub3(x2, x1), x31 = sub3(x3, x1), x01 = sub3(x0, x1);
  float a = dot3(x21, x21), b = dot3(x21, x31), c = dot3(x31, x31);
  float d = dot3(x21, x01), e = dot3(x31, x01);
  float det = a * c - b * b;
  float area_eps = eps * smax(a, c);
  if (det < area_eps * area_eps) return false;
  float b1 = (c * d - b * e) / det;
  float b2 = (a * e - b * d) / det;
  if (b1 < 0.0f || b2 < 0.0f || b1 + b2 > 1.0f) return false;
  u = b1;
  v = b2;
  return true;
}

__device__ bool exact_ee_uv(float3 x0, float3 x1, float3 x2, float3 x3, float eps,
                            float& uo, float& vo) {
  double d1x = (double)x1.x - x0.x, d1y = (double)x1.y - x0.y, d1z = (double)x1.z - x0.z;
  double d2x = (double)x3.x - x2.x, d2y = (double)x3.y - x2.y, d2z = (double)x3.z - x2.z;
  double rx = (double)x0.x - x2.x, ry = (double)x0.y - x2.y, rz = (double)x0.z - x2.z;
  double a = d1x * d1x + d1y * d1y + d1z * d1z;
  double b = d1x * d2x + d1y * d2y + d1z * d2z;
  double c = d1x * rx + d1y * ry + d1z * rz;
  double e = d2x * d2x + d2y * d2y + d2z * d2z;
  double f = d2x * rx + d2y * ry + d2z * rz;
  double eps2 = (double)eps * eps;
  double ls2 = a < e ? e : a;
  if (a <= eps2 * ls2 || e <= eps2 * ls2) return false;
  double den = a * e - b * b;
  double u = den > eps2 * a * e ? fmin(fmax((b * f - c * e) / den, 0.0), 1.0) : 0.0;
  double v = (b * u + f) / e;
  if (v < 0.0) {
    v = 0.0;
    u = fmin(fmax(-c / a, 0.0), 1.0);
  } else if (v > 1.0) {
    v = 1.0;
    u = fmin(fmax((b - c) / a, 0.0), 1.0);
  }
  uo = (float)u;
  vo = (float)v;
  return true;
}

__global__ void dcd_kernel(const ObjDev* objs, const int4* cand, int n, float time,
                           float dact, CollisionDev* out, int cap, int* counter) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int4 c = cand[i];
  int kind = c.z >> 16, sa = c.z & 0xffff, sb = c.w;
  const ObjDev& A = objs[sa];
  const ObjDev& B = objs[sb];
  CollisionDev col;
  float3 x0, x1, x2, x3;
  float param[4], coef[4], im[4];
  int idx[4];
  float u, v;
  if (kind == 0) {
    // A = triangle object, B = point object; collision point first.
    int4 f = A.F[c.x];
    int p = c.y;
    x0 = lerp_t(P(B.x0, p), P(B.x1, p), time);
    x1 = lerp_t(P(A.x0, f.x), P(A.x1, f.x), time);
    x2 = lerp_t(P(A.x0, f.y), P(A.x1, f.y), time);
    x3 = lerp_t(P(A.x0, f.z), P(A.x1, f.z), time);
    if (!exact_pt_uv(x0, x1, x2, x3, kDcdEps, u, v)) return;
    float3 tp = axpby3(1.0f, axpby3(1.0f - u - v, x1, u, x2), v, x3);
    float3 disp = sub3(tp, x0);
    float d2 = dot3(disp, disp);
    if (d2 == 0.0f) return;
    float dist = sqrtf(d2);
    if (dist >= dact) return;
    col.normal = sc3(-1.0f / dist, disp);
    param[0] = 1.0f;
    param[1] = 1.0f - u - v;
    param[2] = u;
    param[3] = v;
    coef[0] = 1.0f;
    coef[1] = -param[1];
    coef[2] = -param[2];
    coef[3] = -param[3];
    im[0] = B.inv_mass[p];
    im[1] = A.inv_mass[f.x];
    im[2] = A.inv_mass[f.y];
    im[3] = A.inv_mass[f.z];
    idx[0] = p;
    idx[1] = f.x;
    idx[2] = f.y;
    idx[3] = f.z;
    col.slot_a = sb;
    col.slot_b = sa;
    col.friction = sqrtf(B.friction * A.friction);
  } else {
    int2 ea = A.E[c.x], eb = B.E[c.y];
    x0 = lerp_t(P(A.x0, ea.x), P(A.x1, ea.x), time);
    x1 = lerp_t(P(A.x0, ea.y), P(A.x1, ea.y), time);
    x2 = lerp_t(P(B.x0, eb.x), P(B.x1, eb.x), time);
    x3 = lerp_t(P(B.x0, eb.y), P(B.x1, eb.y), time);
    if (!exact_ee_uv(x0, x1, x2, x3, kDcdEps, u, v)) return;
    float3 pa = axpby3(1.0f - u, x0, u, x1);
    float3 pb = axpby3(1.0f - v, x2, v, x3);
    float3 disp = sub3(pb, pa);
    float d2 = dot3(disp, disp);
    if (d2 == 0.0f) return;
    float dist = sqrtf(d2);
    if (dist >= dact) return;
    col.normal = sc3(-1.0f / dist, disp);
    param[0] = 1.0f - u;
    param[1] = u;
    param[2] = 1.0f - v;
    param[3] = v;
    coef[0] = param[0];
    coef[1] = param[1];
    coef[2] = -param[2];
    coef[3] = -param[3];
    im[0] = A.inv_mass[ea.x];
    im[1] = A.inv_mass[ea.y];
    im[2] = B.inv_mass[eb.x];
    im[3] = B.inv_mass[eb.y];
    idx[0] = ea.x;
    idx[1] = ea.y;
    idx[2] = eb.x;
    idx[3] = eb.y;
    col.slot_a = sa;
    col.slot_b = sb;
    col.friction = sqrtf(A.friction * B.friction);
  }
  float den = 0.0f;
  for (int k = 0; k < 4; ++k) den += param[k] * param[k] * im[k];
  if (den == 0.0f) return;
  col.type = kind;
  col.dact = dact;
  col.x[0] = x0;
  col.x[1] = x1;
  col.x[2] = x2;
  col.x[3] = x3;
  for (int k = 0; k < 4; ++k) {
    col.idx[k] = idx[k];
    col.coef[k] = coef[k];
    col.inv_mass[k] = im[k];
  }
  // Prescribed obstacle displacement over the rest of the step (dcd.cu:84-96).
  float3 pres = make_float3(0.f, 0.f, 0.f);
  const ObjDev& OA = objs[col.slot_a];
  const ObjDev& OB = objs[col.slot_b];
  if (kind == 0) {
    if (OA.voff < 0) pres = sc3(coef[0], sub3(P(OA.x1, idx[0]), x0));
    if (OB.voff < 0)
      pres = add3(pres, add3(sc3(coef[1], sub3(P(OB.x1, idx[1]), x1)),
                             add3(sc3(coef[2], sub3(P(OB.x1, idx[2]), x2)),
                                  sc3(coef[3], sub3(P(OB.x1, idx[3]), x3)))));
  } else {
    if (OA.voff < 0)
      pres = add3(sc3(coef[0], sub3(P(OA.x1, idx[0]), x0)),
                  sc3(coef[1], sub3(P(OA.x1, idx[1]), x1)));
    if (OB.voff < 0)
      pres = add3(pres, add3(sc3(coef[2], sub3(P(OB.x1, idx[2]), x2)),
                             sc3(coef[3], sub3(P(OB.x1, idx[3]), x3))));
  }
  col.prescribed = pres;
  int at = atomicAdd(counter, 1);
  if (at < cap) out[at] = col;
}

// ---------------------------------------------------------------------------
// Tight-Inclusion CCD (ccd.cpp:13-204, interval_root_finder.cpp:13-522).
// ---------------------------------------------------------------------------
struct IBox {
  float t0, t1, u0, u1, v0, v1;
};

struct CcdCoeff {
  float c0[3], c1[3], c2[3], c3[3], c4[3], c5[3];
};

__device__ bool eval_unit_1d(bool vf, const float3* Pt, float eps, float ms, int dim,
                             bool& in_eps, float& tol) {
  auto comp = [&](const float3& p) { return dim == 0 ? p.x : (dim == 1 ? p.y : p.z); };
  float minv, maxv;
  if (vf) {
    float a0 = comp(Pt[0]), a1 = comp(Pt[4]);
    float D[6] = {a0 - comp(Pt[1]), a0 - comp(Pt[2]), a0 - comp(Pt[3]),
                  a1 - comp(Pt[5]), a1 - comp(Pt[6]), a1 - comp(Pt[7])};
    minv = D[0];
    maxv = D[0];
    for (int i = 1; i < 6; ++i) {
      if (D[i] < minv) minv = D[i];
      if (D[i] > maxv) maxv = D[i];
    }
  } else {
    float A[8] = {comp(Pt[0]), comp(Pt[0]), comp(Pt[1]), comp(Pt[1]),
                  comp(Pt[4]), comp(Pt[4]), comp(Pt[5]), comp(Pt[5])};
    float B[8] = {comp(Pt[2]), comp(Pt[3]), comp(Pt[2]), comp(Pt[3]),
                  comp(Pt[6]), comp(Pt[7]), comp(Pt[6]), comp(Pt[7])};
    minv = A[0] - B[0];
    maxv = minv;
    for (int i = 1; i < 8; ++i) {
      float d = A[i] - B[i];
      if (d < minv) minv = d;
      if (d > maxv) maxv = d;
    }
  }
  tol = maxv - minv;
  in_eps = false;
  float em = eps + ms;
  if (minv > em || maxv < -em) return false;
  if (minv >= -em && maxv <= em) in_eps = true;
  return true;
}

__device__ bool eval_box_1d(bool vf, const IBox& b, const CcdCoeff& co, float em,
                            int dim, bool& in_eps, float& tol) {
  float c0 = co.c0[dim], c1 = co.c1[dim], c2 = co.c2[dim], c3 = co.c3[dim],
        c4 = co.c4[dim], c5 = co.c5[dim];
  float mn[2], mx[2];
  float ts[2] = {b.t0, b.t1};
  for (int k = 0; k < 2; ++k) {
    float t = ts[k];
    float a = (c1 - c0) * t + c0;
    float bb = (c3 - c2) * t + c2;
    float c = (c5 - c4) * t + c4;
    if (!vf || b.u1 + b.v1 <= 1.0f) {
      float bl = bb * b.u0, bu = bb * b.u1, cl = c * b.v0, cu = c * b.v1;
      mn[k] = a + smin(bl, bu) + smin(cl, cu);
      mx[k] = a + smax(bl, bu) + smax(cl, cu);
    } else {
      const float inf = __int_as_float(0x7f800000);
      float lo = inf, hi = -inf;
      auto inc = [&](float u, float v) {
        float val = a + bb * u + c * v;
        lo = smin(lo, val);
        hi = smax(hi, val);
      };
      if (b.u0 + b.v0 <= 1.0f) inc(b.u0, b.v0);
      if (b.u0 + b.v1 <= 1.0f) inc(b.u0, b.v1);
      if (b.u1 + b.v0 <= 1.0f) inc(b.u1, b.v0);
      if (b.u1 + b.v1 <= 1.0f) inc(b.u1, b.v1);
      float v_at_u0 = 1.0f - b.u0;
      if (v_at_u0 >= b.v0 && v_at_u0 <= b.v1) inc(b.u0, v_at_u0);
      float v_at_u1 = 1.0f - b.u1;
      if (v_at_u1 >= b.v0 && v_at_u1 <= b.v1) inc(b.u1, v_at_u1);
      float u_at_v0 = 1.0f - b.v0;
      if (u_at_v0 >= b.u0 && u_at_v0 <= b.u1) inc(u_at_v0, b.v0);
      float u_at_v1 = 1.0f - b.v1;
      if (u_at_v1 >= b.u0 && u_at_v1 <= b.u1) inc(u_at_v1, b.v1);
      mn[k] = lo;
      mx[k] = hi;
    }
  }
  float minv = smin(mn[0], mn[1]);
  float maxv = smax(mx[0], mx[1]);
  in_eps = false;
  if (minv > em || maxv < -em) return false;
  tol = maxv - minv;
  if (minv >= -em && maxv <= em) in_eps = true;
  return true;
}

__device__ float max_linf4(const float3* p, const float3* q) {
  float r = 0.0f;
  for (int k = 0; k < 4; ++k) {
    float m = fabsf(q[k].x - p[k].x);
    m = smax(m, fabsf(q[k].y - p[k].y));
    m = smax(m, fabsf(q[k].z - p[k].z));
    r = k == 0 ? m : smax(r, m);
  }
  return r;
}

__device__ float clamp_div(float a, float b, float mx) {
  if (b == 0) return mx;
  return smin(a / b, mx);
}

// Pending boxes of one search: a small per-thread array for the first pass;
// queries that outgrow it are re-run with a global-memory array of
// max_iter + 2 entries, the most a search can hold (each evaluation pops one
// box and pushes at most two, and pushes stop after max_iter evaluations).
// Pending boxes of a search, in the reference's processing order: smallest
// t.lower first and, for equal t.lower, the most recently pushed (its
// std::map of per-t.lower stacks, interval_root_finder.cpp:430-500).  Two
// stores of that one total order: a sorted array (top = next; an insertion
// shifts the boxes with smaller t.lower, cheap while the search is shallow)
// and a binary heap keyed on (t.lower ascending, push sequence descending),
// O(log n) per operation for deep searches.
struct DfsStack {
  IBox local[kCcdStack];
  IBox* e;
  int* q = nullptr;  // heap: push sequence of each box
  int cap;
  int n;
  bool heap = false;
  int seq = 0;
  __device__ __forceinline__ bool before(const IBox& a, int qa, const IBox& b, int qb) const {
    return a.t0 < b.t0 || (a.t0 == b.t0 && qa > qb);
  }
  __device__ bool push(const IBox& b) {
    if (n >= cap) return false;
    if (heap) {
      const int sq = seq++;
      int i = n++;
      while (i > 0) {
        const int p = (i - 1) >> 1;
        if (!before(b, sq, e[p], q[p])) break;
        e[i] = e[p];
        q[i] = q[p];
        i = p;
      }
      e[i] = b;
      q[i] = sq;
      return true;
    }
    int pos = n;
    while (pos > 0 && e[pos - 1].t0 < b.t0) --pos;
    for (int k = n; k > pos; --k) e[k] = e[k - 1];
    e[pos] = b;
    ++n;
    return true;
  }
  // t.lower of the box pop() would return (n > 0).
  __device__ __forceinline__ float top_t0() const { return heap ? e[0].t0 : e[n - 1].t0; }
  __device__ IBox pop() {
    if (!heap) return e[--n];
    const IBox top = e[0];
    --n;
    if (n > 0) {
      const IBox last = e[n];
      const int lq = q[n];
      int i = 0;
      for (;;) {
        const int l = 2 * i + 1;
        if (l >= n) break;
        int c = l;
        if (l + 1 < n && before(e[l + 1], q[l + 1], e[l], q[l])) c = l + 1;
        if (!before(e[c], q[c], last, lq)) break;
        e[i] = e[c];
        q[i] = q[c];
        i = c;
      }
      e[i] = last;
      q[i] = lq;
    }
    return top;
  }
};

// Returns 0 = no root, 1 = root, 2 = storage overflow, 3 = pruned.
//
// Pruning (best != nullptr): boxes are processed in non-decreasing t.lower
// (every child keeps or raises its parent's t.lower and the smallest pending
// t.lower is always taken next), so once the current box starts at
// t.lower > 0 with t.lower >= the smallest time of impact already found by
// any query, no answer of this search can lower that minimum.  Stopping
// there leaves the minimum over all queries bit-identical to the full search.
__device__ int root_finder(bool vf, const float3* Pt, const float* tol,
                           float co_tol, const float* err, float ms, int max_iter,
                           float max_time, IBox& result, DfsStack& st,
                           const unsigned* best_bits = nullptr) {
  CcdCoeff co;
  for (int d = 0; d < 3; ++d) {
    auto comp = [&](const float3& p) { return d == 0 ? p.x : (d == 1 ? p.y : p.z); };
    if (vf) {
      co.c0[d] = comp(Pt[0]) - comp(Pt[1]);
      co.c1[d] = comp(Pt[4]) - comp(Pt[5]);
      co.c2[d] = comp(Pt[1]) - comp(Pt[2]);
      co.c3[d] = comp(Pt[5]) - comp(Pt[6]);
      co.c4[d] = comp(Pt[1]) - comp(Pt[3]);
      co.c5[d] = comp(Pt[5]) - comp(Pt[7]);
    } else {
      co.c0[d] = comp(Pt[0]) - comp(Pt[2]);
      co.c1[d] = comp(Pt[4]) - comp(Pt[6]);
      co.c2[d] = comp(Pt[1]) - comp(Pt[0]);
      co.c3[d] = comp(Pt[5]) - comp(Pt[4]);
      co.c4[d] = comp(Pt[2]) - comp(Pt[3]);
      co.c5[d] = comp(Pt[6]) - comp(Pt[7]);
    }
  }
  bool unit = max_time == 1.0f;
  IBox cur{0.0f, max_time, 0.0f, 1.0f, 0.0f, 1.0f};
  bool has_cur = true;
  st.n = 0;
  st.seq = 0;
  int iter = 0;
  auto push = [&](const IBox& b) -> bool { return st.push(b); };
  float best = __int_as_float(0x7f800000);
  while (has_cur || st.n > 0) {
    if (!has_cur) cur = st.pop();
    has_cur = false;
    if (best_bits) {
      if ((iter & 15) == 0) best = __uint_as_float(*(volatile const unsigned*)best_bits);
      if (cur.t0 > 0.0f && cur.t0 >= best) return 3;
    }
    ++iter;
    bool in_eps_all = true;
    float w_img[3];
    bool in_zero = true;
    for (int d = 0; d < 3; ++d) {
      bool ie;
      bool ok = unit ? eval_unit_1d(vf, Pt, err[d], ms, d, ie, w_img[d])
                     : eval_box_1d(vf, cur, co, err[d] + ms, d, ie, w_img[d]);
      if (!ok) {
        in_zero = false;
        break;
      }
      in_eps_all = in_eps_all && ie;
    }
    unit = false;
    if (!in_zero) continue;
    bool small = w_img[0] <= co_tol && w_img[1] <= co_tol && w_img[2] <= co_tol;
    if (small || in_eps_all) {
      result = cur;
      return 1;
    }
    if (max_iter > 0 && iter > max_iter) {
      result = cur;
      return 1;
    }
    float widths[3] = {cur.t1 - cur.t0, cur.u1 - cur.u0, cur.v1 - cur.v0};
    float tmp[3];
    for (int d = 0; d < 3; ++d)
      tmp[d] = widths[d] > tol[d] ? widths[d] / tol[d] : -__int_as_float(0x7f800000);
    int split = 0;
    if (tmp[1] > tmp[split]) split = 1;
    if (tmp[2] > tmp[split]) split = 2;
    float lo = split == 0 ? cur.t0 : (split == 1 ? cur.u0 : cur.v0);
    float hi = split == 0 ? cur.t1 : (split == 1 ? cur.u1 : cur.v1);
    float mid = (hi + lo) / 2;
    if (mid < 1e-12f) {  // first half's upper bound below the split limit
      result = cur;
      return 1;
    }
    IBox first = cur, second = cur;
    if (split == 0) {
      first.t1 = mid;
      second.t0 = mid;
    } else if (split == 1) {
      first.u1 = mid;
      second.u0 = mid;
    } else {
      first.v1 = mid;
      second.v0 = mid;
    }
    // The first half, pushed last, is the next box taken whenever no
    // pending box has a smaller t.lower (it is the most recent of any equal
    // ones): it then stays the current box instead of going through the
    // pending store and straight back, which leaves the order of the search
    // unchanged.
    auto push_first = [&]() -> bool {
      if (st.n == 0 || first.t0 <= st.top_t0()) {
        cur = first;
        has_cur = true;
        return true;
      }
      return push(first);
    };
    bool ok = true;
    if (split == 0 || !vf) {
      ok = push(second) && push_first();
    } else {
      float other_lo = split == 1 ? cur.v0 : cur.u0;
      float s_lo = split == 1 ? second.u0 : second.v0;
      float f_lo = split == 1 ? first.u0 : first.v0;
      if (s_lo + other_lo <= 1.0f) ok = push(second);
      if (ok && f_lo + other_lo <= 1.0f) ok = push_first();
    }
    if (!ok) {
      result = cur;
      return 2;
    }
  }
  return 0;
}

// Full query: tolerances, search, and the no-zero-toi refinement with half
// the minimum separation (ccd.cpp:128-182).  Returns the status of the first
// search; toi follows narrowphase.cu's use of the answer.
__device__ int ccd_query(bool vf, const float3* Pt, const float* err, float ms,
                         float tolerance, int max_iter, float max_time, float& toi,
                         float& t_upper, DfsStack& st,
                         const unsigned* best_bits = nullptr) {
  float3 p000, p001, p011, p010, p100, p101, p111, p110;
  if (vf) {
    p000 = sub3(Pt[0], Pt[1]);
    p001 = sub3(Pt[0], Pt[3]);
    p011 = sub3(Pt[0], sub3(add3(Pt[2], Pt[3]), Pt[1]));
    p010 = sub3(Pt[0], Pt[2]);
    p100 = sub3(Pt[4], Pt[5]);
    p101 = sub3(Pt[4], Pt[7]);
    p111 = sub3(Pt[4], sub3(add3(Pt[6], Pt[7]), Pt[5]));
    p110 = sub3(Pt[4], Pt[6]);
  } else {
    p000 = sub3(Pt[0], Pt[2]);
    p001 = sub3(Pt[0], Pt[3]);
    p010 = sub3(Pt[1], Pt[2]);
    p011 = sub3(Pt[1], Pt[3]);
    p100 = sub3(Pt[4], Pt[6]);
    p101 = sub3(Pt[4], Pt[7]);
    p110 = sub3(Pt[5], Pt[6]);
    p111 = sub3(Pt[5], Pt[7]);
  }
  float3 a1[4] = {p000, p001, p011, p010}, b1[4] = {p100, p101, p111, p110};
  float3 a2[4] = {p000, p100, p101, p001}, b2[4] = {p010, p110, p111, p011};
  float3 a3[4] = {p000, p100, p110, p010}, b3[4] = {p001, p101, p111, p011};
  float dl = 3 * max_linf4(a1, b1);
  float e0 = 3 * max_linf4(a2, b2);
  float e1 = 3 * max_linf4(a3, b3);
  const float inf = __int_as_float(0x7f800000);
  float tol[3] = {clamp_div(tolerance, dl, inf), clamp_div(tolerance, e0, inf),
                  clamp_div(tolerance, e1, inf)};
  IBox r;
  int s = root_finder(vf, Pt, tol, tolerance, err, ms, max_iter, max_time, r, st, best_bits);
  if (s == 0 || s == 3) return s;
  toi = r.t0;
  t_upper = r.t1;
  if (r.t0 > 0.0f) return s;
  IBox r2;
  int s2 = root_finder(vf, Pt, tol, tolerance, err, 0.5f * ms, max_iter, max_time, r2, st,
                       best_bits);
  if (s2 == 3) return 3;
  if (s2 == 0) {
    toi = max_time;
    t_upper = max_time;
  } else if (r2.t0 > 0.0f) {
    toi = r2.t0;
    t_upper = r2.t1;
  } else {
    toi = 0.0f;
    t_upper = 0.0f;
  }
  return s == 2 || s2 == 2 ? 2 : 1;
}

// Trajectory of one vertex for the CCD window (ccd_fast_rejection.cu:16-30).
__device__ void trajectory(const ObjDev& o, int v, float ts, float interval,
                           float3& p0, float3& p1) {
  float3 s0 = P(o.x0, v), s1 = P(o.x1, v);
  if (o.voff < 0) {
    float3 d = sub3(s1, s0);
    p0 = axpby3(1.0f, s0, ts, d);
    p1 = axpby3(1.0f, p0, interval, d);
  } else {
    p0 = s0;
    p1 = s1;
  }
}

// Storage of the pending boxes: with spill == nullptr the thread-local array
// (first pass), else a global slice of spill_cap boxes per query (second
// pass over the queries whose first pass overflowed).
struct CcdSpill {
  IBox* spill;
  int spill_cap;
  const int* list;    // second pass: query indices
  int* overflow;      // first pass: queries to re-run
  int* n_overflow;
  int smem_heap = 0;  // second pass: one query per block, a heap of spill_cap
                      // boxes in the block's shared memory (spill unused)
};

extern __shared__ __align__(16) unsigned char ccd_heap_smem[];

__device__ __forceinline__ void bind_stack(DfsStack& st, const CcdSpill& sp, int i) {
  if (sp.smem_heap) {
    st.e = reinterpret_cast<IBox*>(ccd_heap_smem);
    st.q = reinterpret_cast<int*>(ccd_heap_smem + (size_t)sp.spill_cap * sizeof(IBox));
    st.cap = sp.spill_cap;
    st.heap = true;
  } else if (sp.spill) {
    st.e = sp.spill + (size_t)i * sp.spill_cap;
    st.cap = sp.spill_cap;
  } else {
    st.e = st.local;
    st.cap = kCcdStack;
  }
}

__device__ __noinline__ void ccd_one(const ObjDev* objs, const int4* cand, int i, float ts,
                                     float interval, float ms, float3 vf_err, float3 ee_err,
                                     float local_tol, unsigned* min_bits, int* counts,
                                     const CcdSpill& sp, int prune) {
  int q = sp.list ? sp.list[i] : i;
  int4 c = cand[q];
  int kind = c.z >> 16, sa = c.z & 0xffff, sb = c.w;
  const ObjDev& A = objs[sa];
  const ObjDev& B = objs[sb];
  float3 Pt[8];
  bool vf = kind == 0;
  if (vf) {
    int4 f = A.F[c.x];
    trajectory(B, c.y, ts, interval, Pt[0], Pt[4]);
    trajectory(A, f.x, ts, interval, Pt[1], Pt[5]);
    trajectory(A, f.y, ts, interval, Pt[2], Pt[6]);
    trajectory(A, f.z, ts, interval, Pt[3], Pt[7]);
  } else {
    int2 ea = A.E[c.x], eb = B.E[c.y];
    trajectory(A, ea.x, ts, interval, Pt[0], Pt[4]);
    trajectory(A, ea.y, ts, interval, Pt[1], Pt[5]);
    trajectory(B, eb.x, ts, interval, Pt[2], Pt[6]);
    trajectory(B, eb.y, ts, interval, Pt[3], Pt[7]);
  }
  float err[3];
  float3 e = vf ? vf_err : ee_err;
  err[0] = e.x;
  err[1] = e.y;
  err[2] = e.z;
  DfsStack st;
  bind_stack(st, sp, i);
  float toi = 1.0f, tup = 1.0f;
  float local_max = interval / interval;
  int s = ccd_query(vf, Pt, err, ms, local_tol, kCcdMaxIter, local_max, toi, tup, st,
                    prune ? min_bits : nullptr);
  if (s == 2) {
    if (!sp.spill) sp.overflow[atomicAdd(sp.n_overflow, 1)] = q;
    else atomicAdd(&counts[1], 1);
    return;
  }
  if (s == 0 || s == 3) return;
  atomicAdd(&counts[0], 1);
  if (toi == 0.0f) return;
  atomicMin(min_bits, __float_as_uint(toi));  // toi >= 0: bit order = value order
}

// Queries are taken from a shared counter so that threads whose searches end
// early pick up new work instead of idling behind long searches.  With
// prune != 0 a search stops once it cannot lower the running minimum
// (root_finder); the hit count then covers completed searches only.
__global__ void __launch_bounds__(kCollThreads) ccd_kernel(
    const ObjDev* objs, const int4* cand, int n, float ts, float interval,
    float ms, float3 vf_err, float3 ee_err, float local_tol, unsigned* min_bits,
    int* counts, CcdSpill sp, int* next, int prune) {
  for (;;) {
    int i = atomicAdd(next, 1);
    if (i >= n) return;
    ccd_one(objs, cand, i, ts, interval, ms, vf_err, ee_err, local_tol, min_bits, counts,
            sp, prune);
  }
}

// Second pass of the searches that outgrew the per-thread storage: one
// query per block (block q takes list entry q), searched by thread 0 with
// its pending boxes in a heap in the block's shared memory.
__global__ void __launch_bounds__(32) ccd_heap_kernel(
    const ObjDev* objs, const int4* cand, int n, float ts, float interval, float ms,
    float3 vf_err, float3 ee_err, float local_tol, unsigned* min_bits, int* counts,
    CcdSpill sp, int prune) {
  if (threadIdx.x != 0 || (int)blockIdx.x >= n) return;
  ccd_one(objs, cand, blockIdx.x, ts, interval, ms, vf_err, ee_err, local_tol, min_bits, counts,
          sp, prune);
}

constexpr size_t kCcdHeapSmemMax = 200 * 1024;  // heap second pass: up to ~7,300 boxes

size_t ccd_heap_smem_bytes(int cap) {
  return (size_t)cap * (sizeof(IBox) + sizeof(int));
}

__global__ void ccd_batch_kernel(bool vf, const float* x, int n, float3 err,
                                 const float* ms, float tol, int max_iter,
                                 float max_time, int* hit, float* toi, float* tup,
                                 int* n_bad, CcdSpill sp) {
  int i = sp.smem_heap ? (threadIdx.x == 0 ? (int)blockIdx.x : n)
                       : blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int q = sp.list ? sp.list[i] : i;
  float3 Pt[8];
  for (int k = 0; k < 8; ++k)
    Pt[k] = make_float3(x[24 * q + 3 * k], x[24 * q + 3 * k + 1], x[24 * q + 3 * k + 2]);
  float e[3] = {err.x, err.y, err.z};
  DfsStack st;
  bind_stack(st, sp, i);
  float t = max_time, u = max_time;
  int s = ccd_query(vf, Pt, e, ms[q], tol, max_iter, max_time, t, u, st);
  if (s == 2) {
    if (!sp.spill) sp.overflow[atomicAdd(sp.n_overflow, 1)] = q;
    else atomicAdd(n_bad, 1);
    return;
  }
  hit[q] = s != 0 ? 1 : 0;
  toi[q] = s != 0 ? t : max_time;
  if (tup) tup[q] = s != 0 ? u : max_time;
}

// ---------------------------------------------------------------------------
// Contacts (contact_constraints.cu:73-374).
// ---------------------------------------------------------------------------
struct ContactDev {
  int v[4];  // global cloth vertex per slot, -1 kinematic
  float coef[4];
  float gamma[4];
  float3 normal;
  float friction;
  float3 affine;
  float pad;
};

__global__ void build_contacts_kernel(const ObjDev* objs, const CollisionDev* cols,
                                      const int* pick, int n, const float* base_w,
                                      ContactDev* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CollisionDev& c = cols[pick[i]];
  ContactDev k;
  k.normal = c.normal;
  k.friction = c.friction;
  k.affine = sc3(-c.dact, c.normal);
  float norm = 0.0f;
  float3 ref = make_float3(0.f, 0.f, 0.f);
  int dof[4];
  for (int s = 0; s < 4; ++s) {
    float co = c.coef[s];
    k.coef[s] = co;
    ref = add3(ref, sc3(co, c.x[s]));
    int slot = (c.type == 0) ? (s == 0 ? c.slot_a : c.slot_b) : (s < 2 ? c.slot_a : c.slot_b);
    const ObjDev& o = objs[slot];
    int v = o.voff < 0 ? -1 : o.voff + c.idx[s];
    k.v[s] = v;
    dof[s] = v;
    if (v < 0) {
      k.affine = add3(k.affine, sc3(co, c.x[s]));
      continue;
    }
    if (c.inv_mass[s] > 0.0f) norm += co * co / base_w[v];
  }
  k.affine = add3(k.affine, c.prescribed);
  float rn = dot3(ref, k.normal);
  float3 rt = sub3(ref, sc3(rn, k.normal));
  k.affine = sub3(k.affine, rt);
  for (int s = 0; s < 4; ++s)
    k.gamma[s] = (dof[s] >= 0 && c.inv_mass[s] > 0.0f) ? k.coef[s] / (norm * base_w[dof[s]])
                                                       : 0.0f;
  k.pad = 0.f;
  out[i] = k;
}

__global__ void incidence_count_kernel(const ContactDev* c, int n, int* count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int s = 0; s < 4; ++s)
    if (c[i].gamma[s] != 0.0f) atomicAdd(&count[c[i].v[s]], 1);
}

__global__ void incidence_fill_kernel(const ContactDev* c, int n, const int* off,
                                      int* cursor, int* list) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int s = 0; s < 4; ++s)
    if (c[i].gamma[s] != 0.0f) {
      int v = c[i].v[s];
      list[off[v] + atomicAdd(&cursor[v], 1)] = i;
    }
}

// activate_contact_weights + active vertex count (contact_constraints.cu:163-201).
__global__ void activate_weights_kernel(const int* count, int nv, const float* base,
                                        float* w, int* active_dof) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int act = 0;
  if (i < nv) {
    act = count[i] > 0;
    w[i] = act ? base[i] : 0.0f;
  }
  act = __syncthreads_count(act);
  if (threadIdx.x == 0 && act) atomicAdd(active_dof, 3 * act);
}

// One Jones-Plassmann round: a contact whose higher-priority neighbours are
// all coloured takes the smallest colour none of them uses.
// One Jones-Plassmann step of contact i: 0 when a higher-priority neighbour
// (sharing a movable vertex) is still uncoloured, else the smallest colour
// none of them holds (1025 past 1,024 colours).  A neighbour coloured in the
// same round may or may not be seen; either way contact i ends with the
// smallest colour its higher-priority neighbours leave free, so the result
// is the sequential greedy colouring in priority order.
__device__ int jp_pick(const ContactDev* c, const unsigned long long* prio, int i,
                       const int* off, const int* list, const int* color) {
  unsigned long long pi = prio[i];
  unsigned used[32];
  for (int k = 0; k < 32; ++k) used[k] = 0u;
  for (int s = 0; s < 4; ++s) {
    if (c[i].gamma[s] == 0.0f) continue;
    int v = c[i].v[s];
    for (int q = off[v]; q < off[v + 1]; ++q) {
      int j = list[q];
      if (j == i) continue;
      unsigned long long pj = prio[j];
      bool higher = pj > pi || (pj == pi && j < i);
      if (!higher) continue;
      int cj = ((const volatile int*)color)[j];
      if (cj == 0) return 0;
      if (cj <= 1024) used[(cj - 1) >> 5] |= 1u << ((cj - 1) & 31);
    }
  }
  int col = 0;
  for (int k = 0; k < 32 && col == 0; ++k)
    if (used[k] != 0xffffffffu) col = 32 * k + __ffs(~used[k]);
  return col == 0 ? 1025 : col;
}

// Every round in one cooperative launch: one thread per contact (grid-
// stride), the bounded grid barrier between rounds instead of launches and
// host checks.  Round r counts its uncoloured contacts in rem[r % 3]; the
// counter of round r + 1 is cleared during round r, after every block has
// read it for round r - 2.  info: [0] highest colour, [1] contacts past
// 1,024 colours, [3] set when a barrier wait gave up or the rounds ran out.
constexpr int kJpMaxRounds = 4096;
__global__ void jp_grid_kernel(const ContactDev* c, const unsigned long long* prio, int n,
                               const int* off, const int* list, int* color, int* info, int* rem,
                               unsigned* barrier, long long spin_limit) {
  GridBarrier bar{barrier, barrier + 1, barrier + 2, gridDim.x};
  if (spin_limit > 0) bar.limit = spin_limit;
  const int stride = gridDim.x * blockDim.x;
  for (int round = 0; round < kJpMaxRounds; ++round) {
    if (blockIdx.x == 0 && threadIdx.x == 0) rem[(round + 1) % 3] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      if (color[i] != 0) continue;
      const int col = jp_pick(c, prio, i, off, list, color);
      if (col == 0) {
        atomicAdd(rem + round % 3, 1);
        continue;
      }
      if (col > 1024) atomicAdd(info + 1, 1);
      atomicMax(info, col);
      color[i] = col;
    }
    if (!bar.sync()) {
      if (blockIdx.x == 0 && threadIdx.x == 0) info[3] = 1;  // a barrier wait gave up
      return;
    }
    if (((volatile int*)rem)[round % 3] == 0) return;  // the same in every block
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) info[3] = 1;  // rounds exhausted
}

__global__ void iota_kernel(int n, int* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

// Colour groups from the colours sorted ascending (stable, so contact index
// order inside a colour): group_off[k] = first position of colour k + 1,
// group_off[nc] = n; info[2] = the largest group.
__global__ void group_offsets_kernel(const int* sorted, int n, int* info, int* group_off) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = info[0];
  if (k > nc) return;
  auto lower = [&](int key) {
    int lo = 0, hi = n;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (sorted[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  const int a = lower(k + 1);
  group_off[k] = a;
  if (k < nc) atomicMax(info + 2, lower(k + 2) - a);
}

__global__ void gs_nslots_kernel(const int* slot, const int* flag, int nv, int* info) {
  info[4] = slot[nv - 1] + flag[nv - 1];
}



__global__ void contact_gs_kernel(const ContactDev* contacts, const int* groups,
                                  const int* group_off, int ncolors, float4* corr,
                                  float4* p, unsigned* barrier, const int* skip) {
  if (skip && *skip) return;  // the ADMM solve already ended (every block alike)
  GridBarrier bar{barrier, barrier + 1, barrier + 2, gridDim.x};
  int stride = gridDim.x * blockDim.x;
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  // Warm start with the saved corrections (apply_correction_group).
  for (int col = 0; col < ncolors; ++col) {
    for (int q = group_off[col] + tid; q < group_off[col + 1]; q += stride) {
      int ci = groups[q];
      const ContactDev& k = contacts[ci];
      float4 r = corr[ci];
      for (int s = 0; s < 4; ++s) {
        if (k.gamma[s] == 0.0f) continue;
        float4 x = p[k.v[s]];
        float g = k.gamma[s];
        p[k.v[s]] = gs_move(x, g, make_float3(r.x, r.y, r.z));
      }
    }
    if (!bar.sync()) return;
  }
  // Gauss-Seidel sweeps of the exact Signorini-Coulomb projection.
  for (int sweep = 0; sweep < kGsSweeps; ++sweep)
    for (int col = 0; col < ncolors; ++col) {
      for (int q = group_off[col] + tid; q < group_off[col + 1]; q += stride) {
        int ci = groups[q];
        const ContactDev& k = contacts[ci];
        float3 u = k.affine;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const float4 x = k.v[s] >= 0 ? p[k.v[s]] : make_float4(0.f, 0.f, 0.f, 0.f);
          u = gs_accum(u, k.coef[s], x);
        }
        float4 o = corr[ci];
        float3 old = make_float3(o.x, o.y, o.z);
        float3 us = sub3(u, old);
        float3 unew = coulomb_project(us, k.normal, k.friction);
        float3 du = sub3(unew, u);
        float3 nc = add3(old, du);
        corr[ci] = make_float4(nc.x, nc.y, nc.z, 0.f);
        for (int s = 0; s < 4; ++s) {
          if (k.gamma[s] == 0.0f) continue;
          float4 x = p[k.v[s]];
          float g = k.gamma[s];
          p[k.v[s]] = gs_move(x, g, make_float3(du.x, du.y, du.z));
        }
      }
      if (!bar.sync()) return;
    }
}

// Single-block form of contact_gs_kernel.  The contacts are stored in colour
// order with their cloth vertices renamed to compact slots (the vertices any
// contact touches), so a colour phase reads contact q = group_off[c] + thread
// directly and the positions of all touched vertices stay in shared memory for
// the whole solve; colour phases are separated by __syncthreads and the next
// phase's contact and correction are loaded while the current one is
// processed.  The corrections are gathered into colour order at the start and
// scattered back at the end.  Each contact goes through the same operations
// in the same order as in contact_gs_kernel (contacts of one colour touch
// disjoint vertices), so both forms give identical results.
constexpr int kGsBlockThreads = 1024;
constexpr size_t kGsBlockSmemMax = 226 * 1024;

struct GsContact {
  int slot[4];  // compact vertex slot, -1 kinematic
  float coef[4];
  float gamma[4];
  float3 normal;
  float friction;
  float3 affine;
  int ci;       // contact index (correction storage); bit 31: distinct slots
};
static_assert(sizeof(GsContact) == sizeof(ContactDev), "same record size");

// Every cloth vertex a contact reads (v >= 0), movable or not: the pinned
// ones (gamma = 0) still enter the contact's relative position u.
__global__ void gs_flag_kernel(const ContactDev* __restrict__ c, int total,
                               int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  for (int s = 0; s < 4; ++s)
    if (c[i].v[s] >= 0) flag[c[i].v[s]] = 1;
}

__global__ void gs_vlist_kernel(const int* __restrict__ flag, const int* __restrict__ slot, int nv,
                                int* __restrict__ vlist) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv && flag[v]) vlist[slot[v]] = v;
}

__global__ void gs_gather_kernel(const ContactDev* __restrict__ c, const int* __restrict__ groups,
                                 int total, const int* __restrict__ vslot,
                                 GsContact* __restrict__ out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= total) return;
  int ci = groups[q];
  const ContactDev& k = c[ci];
  GsContact g;
  for (int s = 0; s < 4; ++s) {
    g.slot[s] = k.v[s] >= 0 ? vslot[k.v[s]] : -1;
    g.coef[s] = k.coef[s];
    g.gamma[s] = k.gamma[s];
  }
  g.normal = k.normal;
  g.friction = k.friction;
  g.affine = k.affine;
  // Bit 31 of ci: the contact's cloth vertices are pairwise distinct, so the
  // positions gathered for its relative position are still current when it
  // is applied (the pipelined kernel then skips re-reading them).
  bool distinct = true;
  for (int a = 0; a < 4; ++a)
    for (int b = a + 1; b < 4; ++b)
      if (g.slot[a] >= 0 && g.slot[a] == g.slot[b]) distinct = false;
  g.ci = ci | (distinct ? (int)0x80000000u : 0);
  out[q] = g;
}

// Slot incidence of the colour-ordered contacts: entry e = 4 q + s (contact
// position q, vertex s) keyed by its slot when the vertex moves (gamma != 0),
// else by a key past every slot.  A stable sort by key leaves each slot's
// entries in (q, s) order, i.e. in colour order.
__global__ void gs_inc_keys_kernel(const GsContact* __restrict__ cc, int total, int* key,
                                   int* val) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 4 * total) return;
  const GsContact& k = cc[e >> 2];
  const int s = e & 3;
  key[e] = k.gamma[s] != 0.0f && k.slot[s] >= 0 ? k.slot[s] : 0x7fffffff;
  val[e] = e;
}
// The sorted entries as (contact position, share bits) pairs.
__global__ void gs_vent_kernel(const GsContact* __restrict__ cc, const int* __restrict__ code,
                               int n, int2* __restrict__ vent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int c = code[e], q = c >> 2;
  vent[e] = make_int2(q, __float_as_int(cc[q].gamma[c & 3]));
}
// voff[i] = first entry of slot i in the sorted keys, for i <= nslots (info[4]).
__global__ void gs_voff_kernel(const int* __restrict__ sorted, int n, const int* info, int nv,
                               int* voff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nv || i > info[4]) return;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (sorted[mid] < i) lo = mid + 1;
    else hi = mid;
  }
  voff[i] = lo;
}

__global__ void __launch_bounds__(kGsBlockThreads) contact_gs_block_kernel(
    const GsContact* __restrict__ cc, const int* __restrict__ group_off, int ncolors, int total,
    float4* __restrict__ corr, float4* __restrict__ ccorr, const int* __restrict__ vlist,
    int nslots, float4* __restrict__ p, const int* __restrict__ skip) {
  if (skip && *skip) return;  // the ADMM solve already ended
  extern __shared__ float4 sp[];
  const int t = threadIdx.x;
  for (int i = t; i < nslots; i += blockDim.x) sp[i] = p[vlist[i]];
  for (int q = t; q < total; q += blockDim.x) ccorr[q] = corr[cc[q].ci & 0x7fffffff];
  __syncthreads();
  // Warm start with the saved corrections.
  for (int col = 0; col < ncolors; ++col) {
    int q = group_off[col] + t;
    if (q < group_off[col + 1]) {
      const GsContact& k = cc[q];
      float4 r = ccorr[q];
      for (int s = 0; s < 4; ++s) {
        if (k.gamma[s] == 0.0f) continue;
        float4 x = sp[k.slot[s]];
        float g = k.gamma[s];
        sp[k.slot[s]] = gs_move(x, g, make_float3(r.x, r.y, r.z));
      }
    }
    __syncthreads();
  }
  // A thread always takes the same contact of a colour, so the correction it
  // prefetches was last written by itself.
  auto fetch = [&](int col, int& q, GsContact& k, float4& o) {
    q = group_off[col] + t;
    if (q < group_off[col + 1]) {
      k = cc[q];
      o = ccorr[q];
    } else {
      q = -1;
    }
  };
  const int phases = kGsSweeps * ncolors;
  int qn = -1;
  GsContact k;
  float4 on = make_float4(0.f, 0.f, 0.f, 0.f);
  if (phases > 0) fetch(0, qn, k, on);
  for (int ph = 0; ph < phases; ++ph) {
    const int cur = qn;
    const GsContact kc = k;
    const float4 o = on;
    if (ph + 1 < phases) fetch((ph + 1) % ncolors, qn, k, on);
    if (cur >= 0) {
      float3 u = kc.affine;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const float4 x = kc.slot[s] >= 0 ? sp[kc.slot[s]] : make_float4(0.f, 0.f, 0.f, 0.f);
        u = gs_accum(u, kc.coef[s], x);
      }
      float3 old = make_float3(o.x, o.y, o.z);
      float3 us = sub3(u, old);
      float3 unew = coulomb_project(us, kc.normal, kc.friction);
      float3 du = sub3(unew, u);
      float3 nc = add3(old, du);
      ccorr[cur] = make_float4(nc.x, nc.y, nc.z, 0.f);
      if (qn == cur) on = make_float4(nc.x, nc.y, nc.z, 0.f);  // one colour
      for (int s = 0; s < 4; ++s) {
        if (kc.gamma[s] == 0.0f) continue;
        float4 x = sp[kc.slot[s]];
        float g = kc.gamma[s];
        sp[kc.slot[s]] = gs_move(x, g, make_float3(du.x, du.y, du.z));
      }
    }
    __syncthreads();
  }
  for (int q = t; q < total; q += blockDim.x) corr[cc[q].ci & 0x7fffffff] = ccorr[q];
  for (int i = t; i < nslots; i += blockDim.x) p[vlist[i]] = sp[i];
}

// Pipelined single-block form: the contact records of the next ns colour
// phases (ns = 4 staging stages, or 2 or 1 when 4 do not fit shared memory)
// arrive in shared memory by bulk copies (one per colour: its
// records are contiguous in colour order) while the current phase is
// processed, each completing on its stage's mbarrier; the corrections and
// colour offsets stay in shared memory for the whole call, so a phase never
// waits on a global load.  Same per-contact operations as contact_gs_kernel.
constexpr int kGsStages = 4;  // most stages (2 or 1 when 4 do not fit shared memory)
static_assert(sizeof(GsContact) % 16 == 0, "bulk copies move whole 16-byte units");
constexpr int kGsWaitSpins = 1 << 20;  // mbarrier polls before a phase gives up

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of an mbarrier: false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  for (int spin = 0; spin < kGsWaitSpins; ++spin)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

struct GsPipeLayout {
  size_t sp, sc, go, stage, bytes;
};
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
__host__ __device__ inline GsPipeLayout gs_pipe_layout(int nslots, int total, int ncolors,
                                                       int threads, int stages) {
  GsPipeLayout L;
  L.sp = 0;
  // Two extra position slots: nslots reads as zero (kinematic vertices),
  // nslots + 1 takes the stores of zero-share vertices.
  L.sc = align16(L.sp + (size_t)(nslots + 2) * sizeof(float4));
  L.go = align16(L.sc + (size_t)total * sizeof(float4));
  L.stage = align16(L.go + (size_t)(ncolors + 1) * sizeof(int));
  L.bytes = L.stage + (size_t)stages * threads * sizeof(GsContact);
  return L;
}

__global__ void __launch_bounds__(kGsBlockThreads) contact_gs_pipe_kernel(
    const GsContact* __restrict__ cc, const int* __restrict__ group_off, int ncolors, int total,
    float4* __restrict__ corr, const int* __restrict__ vlist, int nslots, float4* __restrict__ p,
    int* __restrict__ fail, const int* __restrict__ skip, const int* __restrict__ voff,
    const int2* __restrict__ vent, int ns_log) {
  if (skip && *skip) return;  // the ADMM solve already ended
  extern __shared__ __align__(16) unsigned char gs_raw[];
  __shared__ __align__(8) uint64_t bars[kGsStages];
  const int ns = 1 << ns_log, nmask = ns - 1;  // staging stages: 1, 2 or 4
  const GsPipeLayout L = gs_pipe_layout(nslots, total, ncolors, blockDim.x, ns);
  float4* sp = reinterpret_cast<float4*>(gs_raw + L.sp);
  float4* sc = reinterpret_cast<float4*>(gs_raw + L.sc);
  int* sgo = reinterpret_cast<int*>(gs_raw + L.go);
  GsContact* stage = reinterpret_cast<GsContact*>(gs_raw + L.stage);
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < nslots; i += nt) sp[i] = p[vlist[i]];
  if (t < 2) sp[nslots + t] = make_float4(0.f, 0.f, 0.f, 0.f);
  const int zslot = nslots, tslot = nslots + 1;
  for (int q = t; q < total; q += nt) sc[q] = corr[cc[q].ci & 0x7fffffff];
  for (int c = t; c <= ncolors; c += nt) sgo[c] = group_off[c];
  __syncthreads();
  // Warm start with the saved corrections: each slot applies those of its
  // contacts in colour order (its entries of the slot incidence), the same
  // moves in the same order as colour phases would, without their barriers.
  // A slot's entries (at most 8 per load round) are loaded together.
  for (int i = t; i < nslots; i += nt) {
    float4 x = sp[i];
    const int e1 = voff[i + 1];
    for (int e0 = voff[i]; e0 < e1; e0 += 8) {
      int2 en[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) en[k] = e0 + k < e1 ? vent[e0 + k] : make_int2(0, 0);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (e0 + k >= e1) break;
        const float4 r = sc[en[k].x];
        x = gs_move(x, __int_as_float(en[k].y), make_float3(r.x, r.y, r.z));
      }
    }
    sp[i] = x;
  }
  __syncthreads();
  const int phases = kGsSweeps * ncolors;
  // The copies are issued by the block's last thread: its warp holds no
  // contact in most colours, so the issue stays off the contacts' path.
  const int producer = nt - 1;
  if (t == producer) {
    for (int s = 0; s < ns; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  // Copy the records of phase ph's colour into stage ph % ns.  A thread reads
  // its record of phase ph at the end of phase ph - 1, before that phase's
  // block barrier, so at phase ph the stage of phase ph is free again and
  // receives the records of phase ph + ns.
  auto issue = [&](int ph, int col) {
    if (t != producer || ph >= phases) return;
    uint64_t* bar = &bars[ph & nmask];
    const unsigned bytes = (unsigned)((sgo[col + 1] - sgo[col]) * (int)sizeof(GsContact));
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (bytes) {
      mbar_arrive_expect(bar, bytes);
      bulk_copy_g2s(stage + (size_t)(ph & nmask) * nt, cc + sgo[col], bytes, bar);
    } else {
      mbar_arrive(bar);
    }
  };
  int col_issue = 0;
#pragma unroll
  for (int s = 0; s < ns; ++s) {
    issue(s, col_issue);
    col_issue = col_issue + 1 == ncolors ? 0 : col_issue + 1;
  }
  // Registers carry the record and the correction of the phase about to run;
  // they are loaded before the previous phase's barrier, so their latency
  // overlaps the barrier.  A thread always takes the same contact of a
  // colour, so the correction it loads was last written by itself (with one
  // colour, in the phase just run, earlier in this thread's program order).
  GsContact kn;
  float4 on = make_float4(0.f, 0.f, 0.f, 0.f);
  int qn = -1;
  bool lost = false;  // a copy this thread waited for did not land in time
  auto fetch = [&](int ph, int col) {
    const bool landed = mbar_wait(&bars[ph & nmask], (unsigned)(ph >> ns_log) & 1u);
    qn = sgo[col] + t;
    if (landed && qn < sgo[col + 1]) {
      kn = stage[(size_t)(ph & nmask) * nt + t];
      on = sc[qn];
    } else {
      qn = -1;
    }
    lost = lost || !landed;
  };
  int col = 0;
  if (phases > 0) fetch(0, 0);
  __syncthreads();  // every thread has read stage 0 before phase 0 refills it
  int ph = 0;
  for (; ph < phases; ++ph) {
    issue(ph + ns, col_issue);
    col_issue = col_issue + 1 == ncolors ? 0 : col_issue + 1;
    const int cur = qn;
    const GsContact kc = kn;
    const float4 o = on;
    col = col + 1 == ncolors ? 0 : col + 1;
    if (cur >= 0) {
      // All four positions read at once, without branches (a kinematic
      // vertex reads the zero slot: u gains c * 0).
      float3 u = kc.affine;
      float4 xs[4];
#pragma unroll
      for (int s = 0; s < 4; ++s) xs[s] = sp[kc.slot[s] >= 0 ? kc.slot[s] : zslot];
#pragma unroll
      for (int s = 0; s < 4; ++s) u = gs_accum(u, kc.coef[s], xs[s]);
      float3 old = make_float3(o.x, o.y, o.z);
      float3 us = sub3(u, old);
      float3 unew = coulomb_project(us, kc.normal, kc.friction);
      float3 du = sub3(unew, u);
      float3 nc = add3(old, du);
      sc[cur] = make_float4(nc.x, nc.y, nc.z, 0.f);
      const bool distinct = kc.ci < 0;
      // Zero-share vertices (kinematic, pinned) store into the scratch slot.
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int sl = kc.gamma[s] != 0.0f && kc.slot[s] >= 0 ? kc.slot[s] : tslot;
        const float4 x = distinct ? xs[s] : sp[sl];
        sp[sl] = gs_move(x, kc.gamma[s], du);
      }
    }
    if (ph + 1 < phases) fetch(ph + 1, col);
    // The block barrier that orders the colours also agrees on a lost copy,
    // so every thread leaves the loop at the same phase.
    if (__syncthreads_or(lost)) break;
  }
  if (ph < phases) {
    // A copy did not land in time: wait (bounded) for the copies still in
    // flight, report the failure (the step then returns
    // IterativeSolveFail) and leave the positions untouched.
    if (t == producer) {
      // Phase ph's copy completed before phase ph - 1's barrier; ph + 1 ..
      // ph + ns may still be in flight.
      for (int q = ph + 1; q <= ph + ns && q < phases; ++q)
        mbar_wait(&bars[q & nmask], (unsigned)(q >> ns_log) & 1u);
      if (fail) atomicOr(fail, kFailContactWait);
    }
    return;
  }
  for (int q = t; q < total; q += nt) corr[cc[q].ci & 0x7fffffff] = sc[q];
  for (int i = t; i < nslots; i += nt) p[vlist[i]] = sp[i];
}

// Canonical contact key (contact_constraints.cu:24-47).
struct Key {
  int type;
  uint32_t oa, ob;
  int idx[4];
  bool operator<(const Key& o) const {
    return std::tie(type, oa, ob, idx[0], idx[1], idx[2], idx[3]) <
           std::tie(o.type, o.oa, o.ob, o.idx[0], o.idx[1], o.idx[2], o.idx[3]);
  }
};

Key make_key(int type, uint32_t oa, uint32_t ob, const int* idx) {
  Key k{type, oa, ob, {idx[0], idx[1], idx[2], idx[3]}};
  if (type == 0) {
    std::sort(k.idx + 1, k.idx + 4);
    return k;
  }
  if (k.idx[1] < k.idx[0]) std::swap(k.idx[0], k.idx[1]);
  if (k.idx[3] < k.idx[2]) std::swap(k.idx[2], k.idx[3]);
  if (std::make_tuple(k.ob, k.idx[2], k.idx[3]) < std::make_tuple(k.oa, k.idx[0], k.idx[1])) {
    std::swap(k.oa, k.ob);
    std::swap(k.idx[0], k.idx[2]);
    std::swap(k.idx[1], k.idx[3]);
  }
  return k;
}

// Colouring priority: 64-bit mix of the canonical key (splitmix64 finaliser).
uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
uint64_t key_priority(const Key& k) {
  uint64_t h = mix64((uint64_t)k.type);
  h = mix64(h ^ k.oa);
  h = mix64(h ^ ((uint64_t)k.ob << 1));
  for (int i = 0; i < 4; ++i) h = mix64(h ^ (uint64_t)(uint32_t)k.idx[i]);
  return h;
}

struct Tree {
  int n = 0, D = 0;
  DevBuf<int> order, vals_in;
  DevBuf<unsigned long long> keys_in, keys_out;
  DevBuf<float4> nodes;
  DevBuf<char> temp;
  size_t temp_bytes = 0;
  bool sorted = false;
};

struct ObjHost {
  bool cloth = false;
  int index = 0;
  uint32_t handle = 0;
  bool physical = false;
  int group = -1;
  bool self_on = false;
  float padding = 0.f;
  float friction = 0.f;
  int nv = 0, nf = 0, ne = 0;
  int voff = -1;
  DevBuf<int4> F;
  DevBuf<int2> E;
  DevBuf<float> inv_mass;
  DevBuf<float4> pos_cur, pos_prev;
  DevBuf<float4> tri_bb, edge_bb, pt_bb, partial, obj_box;
  Tree tri, edge;
  float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
};

}  // namespace

struct CollisionImpl {
  std::vector<std::unique_ptr<ObjHost>> objs;
  std::vector<ObjDev> table;
  DevBuf<ObjDev> table_d;
  DevBuf<int4> cand;
  int cand_cap = 0;
  int n_cand = 0;
  DevBuf<int> counter;  // [candidates, collisions, ...]
  DevBuf<CollisionDev> cols;
  int cols_cap = 0;
  DevBuf<unsigned> min_bits;
  DevBuf<int> ccd_counts;  // [hits, storage overflows, first-pass spills]
  DevBuf<int> ccd_overflow;
  // Contacts.
  cudaEvent_t ccd_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // narrowphase pass timing
  CollisionImpl() = default;
  CollisionImpl(const CollisionImpl&) = delete;
  CollisionImpl& operator=(const CollisionImpl&) = delete;
  ~CollisionImpl() {
    for (cudaEvent_t e : ccd_ev)
      if (e) cudaEventDestroy(e);
  }
  std::set<Key> keys;
  std::vector<Key> key_list;
  std::vector<uint64_t> prio_host;
  DevBuf<ContactDev> contacts;
  int n_contacts = 0, contacts_cap = 0;
  DevBuf<unsigned long long> prio;
  DevBuf<float4> corr;
  DevBuf<int> inc_count, inc_off, inc_cursor, inc_list, colors, groups, group_off;
  // Single-block Gauss-Seidel: compact slots of the touched vertices and the
  // contacts in colour order on those slots.
  DevBuf<int> gs_flag, gs_slot, gs_vlist;
  DevBuf<GsContact> gs_cc;
  DevBuf<float4> gs_ccorr;
  int gs_nslots = 0;
  bool gs_ready = false;
  DevBuf<int> active_dof;
  DevBuf<int> jp_flags;
  // Colouring results read by the host once per contact build: highest
  // colour, overflow, largest group, uncoloured left, Gauss-Seidel slots.
  DevBuf<int> col_info, col_sorted, grp_in;
  // Slot incidence of the colour-ordered contacts (entries 4 q + s, each
  // slot's in colour order; gs_voff[slot] = its first entry).
  DevBuf<int> gs_ikey, gs_ival, gs_ikey_s, gs_vinc, gs_voff;
  DevBuf<int2> gs_vent;  // sorted entries as (contact position, share bits)
  DevBuf<char> sort_temp;
  DevBuf<int> pick_d;  // DCD records picked as new contacts (grow-only)
  DevBuf<unsigned> gs_barrier;
  DevBuf<char> scan_temp;
  int n_colors = 0;
  int max_group = 0;
};

CollisionSystem::CollisionSystem(World& w) : w_(w), impl_(new CollisionImpl) {
  impl_->active_dof.alloc(1);
  CUDA_CHECK(cudaMemset(impl_->active_dof.p, 0, sizeof(int)));
  impl_->counter.alloc(4);
  impl_->min_bits.alloc(1);
  impl_->ccd_counts.alloc(4 + 64);
  impl_->jp_flags.alloc(3);
  impl_->col_info.alloc(5);
  impl_->gs_barrier.alloc(4);
  CUDA_CHECK(cudaMemset(impl_->gs_barrier.p, 0, 4 * sizeof(unsigned)));
}

CollisionSystem::~CollisionSystem() = default;

void CollisionSystem::rebuild() {
  CollisionImpl& I = *impl_;
  cudaStream_t st = w_.stream;
  I.objs.clear();
  auto common = [&](ObjHost& o) {
    o.tri_bb.alloc(2 * (size_t)std::max(o.nf, 1));
    o.edge_bb.alloc(2 * (size_t)std::max(o.ne, 1));
    o.pt_bb.alloc(2 * (size_t)std::max(o.nv, 1));
    o.partial.alloc(2 * (size_t)div_up(std::max({o.nf, o.ne, o.nv, 1}), kCollThreads));
    o.obj_box.alloc(2);
  };
  for (size_t c = 0; c < w_.cloths.size(); ++c) {
    Cloth& cl = *w_.cloths[c];
    const ClothSetup& S = *cl.setup;
    auto o = std::make_unique<ObjHost>();
    o->cloth = true;
    o->index = (int)c;
    o->handle = cl.handle;
    o->physical = true;
    o->group = cl.coll.is_collision_on ? cl.coll.group : -1;
    o->self_on = cl.coll.is_self_collision_on != 0;
    o->padding = 0.05f * S.avg_edge;
    o->friction = cl.coll.friction;
    o->nv = S.nv;
    o->nf = S.nf;
    o->ne = S.ne;
    o->voff = cl.voff;
    std::vector<int4> F(S.nf);
    for (int t = 0; t < S.nf; ++t) F[t] = make_int4(S.F[3 * t], S.F[3 * t + 1], S.F[3 * t + 2], 0);
    std::vector<int2> E(S.ne);
    for (int e = 0; e < S.ne; ++e) E[e] = make_int2(S.E[2 * e], S.E[2 * e + 1]);
    std::vector<char> pinned(S.nv, 0);
    for (int p : cl.pins) pinned[S.perm[p]] = 1;
    std::vector<float> im(S.nv);
    for (int i = 0; i < S.nv; ++i) {
      float m = cl.cfg.density * (float)S.voronoi[i];
      im[i] = pinned[i] ? 0.0f : 1.0f / m;
    }
    o->F.upload(F, st);
    o->E.upload(E, st);
    o->inv_mass.upload(im, st);
    common(*o);
    I.objs.push_back(std::move(o));
  }
  for (size_t k = 0; k < w_.obstacles.size(); ++k) {
    Obstacle& ob = *w_.obstacles[k];
    auto o = std::make_unique<ObjHost>();
    o->cloth = false;
    o->index = (int)k;
    o->handle = ob.handle;
    o->physical = false;
    o->group = ob.coll.is_collision_on ? ob.coll.group : -1;
    o->self_on = ob.coll.is_self_collision_on != 0;
    std::vector<int> E = mesh_edges(ob.faces.data(), ob.nf());
    o->padding = 0.05f * average_edge_length(ob.cur.data(), E);
    o->friction = ob.coll.friction;
    o->nv = ob.nv();
    o->nf = ob.nf();
    o->ne = (int)E.size() / 2;
    o->voff = -1;
    std::vector<int4> F(o->nf);
    for (int t = 0; t < o->nf; ++t)
      F[t] = make_int4(ob.faces[3 * t], ob.faces[3 * t + 1], ob.faces[3 * t + 2], 0);
    std::vector<int2> E2(o->ne);
    for (int e = 0; e < o->ne; ++e) E2[e] = make_int2(E[2 * e], E[2 * e + 1]);
    o->F.upload(F, st);
    o->E.upload(E2, st);
    o->inv_mass.upload(std::vector<float>(o->nv, 0.0f), st);
    o->pos_cur.alloc(o->nv);
    o->pos_prev.alloc(o->nv);
    ob.positions_dirty = true;
    common(*o);
    I.objs.push_back(std::move(o));
  }
  I.table.assign(I.objs.size(), ObjDev{});
  I.table_d.alloc(std::max<size_t>(I.objs.size(), 1));
  for (auto& o : I.objs) {
    o->tri.sorted = false;
    o->edge.sorted = false;
  }
  I.keys.clear();
  I.n_contacts = 0;
  CUDA_CHECK(cudaStreamSynchronize(st));
}

float CollisionSystem::scene_padding() const {
  float p = 0.f;
  bool first = true;
  for (auto& o : impl_->objs) {
    p = first ? o->padding : std::min(p, o->padding);
    first = false;
  }
  return p;
}

bool CollisionSystem::has_colliders() const {
  for (auto& o : impl_->objs)
    if (o->group != -1) return true;
  return false;
}

void CollisionSystem::refresh_obstacles() {
  for (auto& o : impl_->objs) {
    if (o->cloth) continue;
    Obstacle& ob = *w_.obstacles[o->index];
    if (!ob.positions_dirty) continue;
    std::vector<float4> cur(o->nv), prev(o->nv);
    for (int i = 0; i < o->nv; ++i) {
      cur[i] = make_float4(ob.cur[3 * i], ob.cur[3 * i + 1], ob.cur[3 * i + 2], 0.f);
      prev[i] = make_float4(ob.prev[3 * i], ob.prev[3 * i + 1], ob.prev[3 * i + 2], 0.f);
    }
    CUDA_CHECK(cudaMemcpyAsync(o->pos_cur.p, cur.data(), o->nv * sizeof(float4),
                               cudaMemcpyHostToDevice, w_.stream));
    CUDA_CHECK(cudaMemcpyAsync(o->pos_prev.p, prev.data(), o->nv * sizeof(float4),
                               cudaMemcpyHostToDevice, w_.stream));
    ob.positions_dirty = false;
  }
}

static void build_tree(cudaStream_t st, const ObjDev* table_d, int slot, int kind,
                       Tree& T, int n, const float4* prim_bb, bool resort) {
  T.n = n;
  if (n == 0) return;
  int D = 0;
  while ((1 << D) < n) ++D;
  if (T.D != D || !T.nodes.p) {
    T.D = D;
    T.nodes.alloc(2 * (size_t)((2 << D) - 1));
    T.order.alloc(n);
    T.vals_in.alloc(n);
    T.keys_in.alloc(n);
    T.keys_out.alloc(n);
    T.temp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, T.temp_bytes, T.keys_in.p, T.keys_out.p,
                                    T.vals_in.p, T.order.p, n, 0, 64, st);
    T.temp.alloc(T.temp_bytes);
    resort = true;
  }
  if (resort || !T.sorted) {
    morton_kernel<<<div_up(n, kCollThreads), kCollThreads, 0, st>>>(table_d, slot, kind, n,
                                                                     T.keys_in.p, T.vals_in.p);
    SILK_LAUNCHED();
    size_t tb = T.temp_bytes;
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(T.temp.p, tb, T.keys_in.p, T.keys_out.p,
                                               T.vals_in.p, T.order.p, n, 0, 64, st));
    SILK_LAUNCHED();
    T.sorted = true;
  }
  int P = 1 << D;
  tree_leaves_kernel<<<div_up(P, 256), 256, 0, st>>>(prim_bb, T.order.p, n, P, T.nodes.p);
  SILK_LAUNCHED();
  for (int L = D; L > 0;) {
    int k = std::min(8, L);
    int count = 1 << L;
    int grid = count < 256 ? 1 : count / 256;
    tree_up_kernel<<<grid, 256, 0, st>>>(T.nodes.p, L, k);
    SILK_LAUNCHED();
    L -= k;
  }
}

void CollisionSystem::refit(const float4* t1, const float4* t0) {
  CollisionImpl& I = *impl_;
  cudaStream_t st = w_.stream;
  for (size_t s = 0; s < I.objs.size(); ++s) {
    ObjHost& o = *I.objs[s];
    ObjDev& d = I.table[s];
    if (o.cloth) {
      d.x0 = t0 + o.voff;
      d.x1 = t1 + o.voff;
    } else {
      Obstacle& ob = *w_.obstacles[o.index];
      d.x1 = o.pos_cur.p;
      d.x0 = ob.is_static ? o.pos_cur.p : o.pos_prev.p;
    }
    d.F = o.F.p;
    d.E = o.E.p;
    d.inv_mass = o.inv_mass.p;
    d.nv = o.nv;
    d.nf = o.nf;
    d.ne = o.ne;
    d.padding = o.padding;
    d.friction = o.friction;
    d.handle = (int)o.handle;
    d.voff = o.cloth ? o.voff : -1;
    d.tri_bb = o.tri_bb.p;
    d.edge_bb = o.edge_bb.p;
    d.pt_bb = o.pt_bb.p;
    d.obj_box = o.obj_box.p;
  }
  // Tree depths are fixed by primitive counts; set them before upload.
  for (size_t s = 0; s < I.objs.size(); ++s) {
    ObjHost& o = *I.objs[s];
    ObjDev& d = I.table[s];
    int D = 0;
    while ((1 << D) < o.nf) ++D;
    d.tri_D = D;
    D = 0;
    while ((1 << D) < o.ne) ++D;
    d.edge_D = D;
    if (!o.tri.nodes.p || o.tri.D != d.tri_D) {
      o.tri.D = -1;  // force allocation in build_tree
    }
  }
  // Allocate tree storage first so that the table carries final pointers.
  for (size_t s = 0; s < I.objs.size(); ++s) {
    ObjHost& o = *I.objs[s];
    ObjDev& d = I.table[s];
    for (int kind = 0; kind < 2; ++kind) {
      Tree& T = kind == 0 ? o.tri : o.edge;
      int n = kind == 0 ? o.nf : o.ne;
      int D = kind == 0 ? d.tri_D : d.edge_D;
      if (n > 0 && (T.D != D || !T.nodes.p)) {
        T.D = D;
        T.n = n;
        T.nodes.alloc(2 * (size_t)((2 << D) - 1));
        T.order.alloc(n);
        T.vals_in.alloc(n);
        T.keys_in.alloc(n);
        T.keys_out.alloc(n);
        T.temp_bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, T.temp_bytes, T.keys_in.p, T.keys_out.p,
                                        T.vals_in.p, T.order.p, n, 0, 64, st);
        T.temp.alloc(T.temp_bytes);
        T.sorted = false;
      }
    }
    d.tri_nodes = o.tri.nodes.p;
    d.tri_order = o.tri.order.p;
    d.edge_nodes = o.edge.nodes.p;
    d.edge_order = o.edge.order.p;
  }
  CUDA_CHECK(cudaMemcpyAsync(I.table_d.p, I.table.data(), I.table.size() * sizeof(ObjDev),
                             cudaMemcpyHostToDevice, st));
  for (size_t s = 0; s < I.objs.size(); ++s) {
    ObjHost& o = *I.objs[s];
    int n = std::max({o.nf, o.ne, o.nv, 1});
    int grid = div_up(n, kCollThreads);
    refit_kernel<<<grid, kCollThreads, 0, st>>>(I.table_d.p, (int)s, o.partial.p);
    SILK_LAUNCHED();
    reduce_box_kernel<<<1, kCollThreads, 0, st>>>(I.table_d.p, (int)s, o.partial.p, grid);
    SILK_LAUNCHED();
    build_tree(st, I.table_d.p, (int)s, 0, o.tri, o.nf, o.tri_bb.p, false);
    build_tree(st, I.table_d.p, (int)s, 1, o.edge, o.ne, o.edge_bb.p, false);
  }
  // Object boxes to the host (object-level SAP and the CCD error filter).
  std::vector<float4> boxes(2 * I.objs.size());
  for (size_t s = 0; s < I.objs.size(); ++s)
    CUDA_CHECK(cudaMemcpyAsync(&boxes[2 * s], I.objs[s]->obj_box.p, 2 * sizeof(float4),
                               cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  for (size_t s = 0; s < I.objs.size(); ++s) {
    ObjHost& o = *I.objs[s];
    o.bmin[0] = boxes[2 * s].x;
    o.bmin[1] = boxes[2 * s].y;
    o.bmin[2] = boxes[2 * s].z;
    o.bmax[0] = boxes[2 * s + 1].x;
    o.bmax[1] = boxes[2 * s + 1].y;
    o.bmax[2] = boxes[2 * s + 1].z;
  }
}

namespace {

// Object pairs of the object-level SAP (sap.cuh:37-99, find_collision.cu:17-26).
std::vector<std::pair<int, int>> object_pairs(CollisionImpl& I) {
  int n = (int)I.objs.size();
  std::vector<std::pair<int, int>> pairs;
  if (n == 0) return pairs;
  float mean[3] = {0, 0, 0}, var[3] = {0, 0, 0};
  for (auto& o : I.objs)
    for (int d = 0; d < 3; ++d) {
      float c = 0.5f * o->bmin[d] + 0.5f * o->bmax[d];
      mean[d] += c;
      var[d] += c * c;
    }
  for (int d = 0; d < 3; ++d) {
    mean[d] = (1.0f / n) * mean[d];
    var[d] = (1.0f / n) * var[d] - mean[d] * mean[d];
  }
  int axis = (var[0] > var[1] && var[0] > var[2]) ? 0 : (var[1] > var[2] ? 1 : 2);
  std::vector<int> prox(n);
  for (int i = 0; i < n; ++i) prox[i] = i;
  std::stable_sort(prox.begin(), prox.end(), [&](int a, int b) {
    return I.objs[a]->bmin[axis] < I.objs[b]->bmin[axis];
  });
  auto filt = [](const ObjHost& a, const ObjHost& b) {
    return a.group != -1 && b.group != -1 && a.group == b.group && (a.physical || b.physical);
  };
  auto ovl = [](const ObjHost& a, const ObjHost& b) {
    for (int d = 0; d < 3; ++d) {
      float lo = a.bmin[d] < b.bmin[d] ? b.bmin[d] : a.bmin[d];
      float hi = b.bmax[d] < a.bmax[d] ? b.bmax[d] : a.bmax[d];
      if (!(lo <= hi)) return false;
    }
    return true;
  };
  for (int i = 0; i + 1 < n; ++i) {
    ObjHost& a = *I.objs[prox[i]];
    for (int j = i + 1; j < n; ++j) {
      ObjHost& b = *I.objs[prox[j]];
      if (a.bmax[axis] < b.bmin[axis]) break;
      if (!filt(a, b)) continue;
      if (ovl(a, b)) pairs.emplace_back(prox[i], prox[j]);
    }
  }
  return pairs;
}

int gather_candidates(CollisionImpl& I, cudaStream_t st) {
  auto pairs = object_pairs(I);
  struct Call {
    int t, q, mode, nq;
  };
  std::vector<Call> calls;
  for (auto& [a, b] : pairs) {
    calls.push_back({a, b, 0, I.objs[b]->nv});
    calls.push_back({b, a, 0, I.objs[a]->nv});
    calls.push_back({a, b, 2, I.objs[b]->ne});
  }
  for (size_t o = 0; o < I.objs.size(); ++o) {
    ObjHost& ob = *I.objs[o];
    if (!ob.physical || !ob.self_on || ob.group == -1) continue;
    calls.push_back({(int)o, (int)o, 1, ob.nv});
    calls.push_back({(int)o, (int)o, 3, ob.ne});
  }
  if (I.cand_cap == 0) {
    I.cand_cap = 1 << 16;
    I.cand.alloc(I.cand_cap);
  }
  for (int attempt = 0; attempt < 2; ++attempt) {
    CUDA_CHECK(cudaMemsetAsync(I.counter.p, 0, sizeof(int), st));
    for (auto& c : calls) {
      ObjHost& T = *I.objs[c.t];
      int ntree = c.mode < 2 ? T.nf : T.ne;
      if (c.nq == 0 || ntree == 0) continue;
      traverse_kernel<<<div_up(c.nq, kCollThreads), kCollThreads, 0, st>>>(
          I.table_d.p, c.t, c.q, c.mode, I.cand.p, I.cand_cap, I.counter.p);
      SILK_LAUNCHED();
    }
    int n = 0;
    CUDA_CHECK(cudaMemcpyAsync(&n, I.counter.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
    if (n <= I.cand_cap) {
      I.n_cand = n;
      return n;
    }
    I.cand_cap = n + n / 4 + 1024;
    I.cand.alloc(I.cand_cap);
  }
  throw CudaError("candidate buffer overflow");
}

}  // namespace

void CollisionSystem::begin_step() {
  CollisionImpl& I = *impl_;
  I.keys.clear();
  I.key_list.clear();
  I.prio_host.clear();
  I.n_contacts = 0;
  I.n_colors = 0;
  CUDA_CHECK(cudaMemsetAsync(I.active_dof.p, 0, sizeof(int), w_.stream));
  w_.contact_w.zero(w_.stream);
  w_.contact_eta.zero(w_.stream);
  w_.contact_p.zero(w_.stream);
}

int CollisionSystem::append_active(float time, float dact) {
  CollisionImpl& I = *impl_;
  using clk = std::chrono::steady_clock;
  auto lap = [](clk::time_point& t) {
    const clk::time_point now = clk::now();
    const double ms = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
    return ms;
  };
  clk::time_point t_lap = clk::now();
  last_dcd_gather_ms = last_dcd_build_ms = last_dcd_color_ms = last_dcd_layout_ms = 0.0;
  cudaStream_t st = w_.stream;
  int n = gather_candidates(I, st);
  last_dcd_gather_ms = lap(t_lap);
  if (n == 0) return 0;
  if (I.cols_cap < n) {
    I.cols_cap = n + n / 4;
    I.cols.alloc(I.cols_cap);
  }
  CUDA_CHECK(cudaMemsetAsync(I.counter.p + 1, 0, sizeof(int), st));
  dcd_kernel<<<div_up(n, kCollThreads), kCollThreads, 0, st>>>(
      I.table_d.p, I.cand.p, n, time, dact, I.cols.p, I.cols_cap, I.counter.p + 1);
  SILK_LAUNCHED();
  int m = 0;
  CUDA_CHECK(cudaMemcpyAsync(&m, I.counter.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  if (m == 0) return 0;
  // Host dedup against the contact set, canonical order (the reference also
  // deduplicates on the host, contact_constraints.cu:440-453).
  std::vector<CollisionDev> hc(m);
  CUDA_CHECK(cudaMemcpy(hc.data(), I.cols.p, m * sizeof(CollisionDev), cudaMemcpyDeviceToHost));
  std::vector<std::pair<Key, int>> fresh;
  for (int i = 0; i < m; ++i) {
    const CollisionDev& c = hc[i];
    Key k = make_key(c.type, I.objs[c.slot_a]->handle, I.objs[c.slot_b]->handle, c.idx);
    if (I.keys.insert(k).second) fresh.emplace_back(k, i);
  }
  if (fresh.empty()) return 0;
  std::sort(fresh.begin(), fresh.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });
  int add = (int)fresh.size();
  int old = I.n_contacts;
  int total = old + add;
  if (total > I.contacts_cap) {
    int cap = std::max(1024, total * 2);
    DevBuf<ContactDev> nc;
    nc.alloc(cap);
    DevBuf<float4> ncorr;
    ncorr.alloc(cap);
    DevBuf<unsigned long long> np;
    np.alloc(cap);
    if (old) {
      CUDA_CHECK(cudaMemcpyAsync(nc.p, I.contacts.p, old * sizeof(ContactDev),
                                 cudaMemcpyDeviceToDevice, st));
      CUDA_CHECK(cudaMemcpyAsync(ncorr.p, I.corr.p, old * sizeof(float4),
                                 cudaMemcpyDeviceToDevice, st));
      CUDA_CHECK(cudaMemcpyAsync(np.p, I.prio.p, old * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, st));
    }
    CUDA_CHECK(cudaStreamSynchronize(st));
    I.contacts = std::move(nc);
    I.corr = std::move(ncorr);
    I.prio = std::move(np);
    I.contacts_cap = cap;
  }
  std::vector<int> pick(add);
  std::vector<unsigned long long> pr(add);
  for (int i = 0; i < add; ++i) {
    pick[i] = fresh[i].second;
    pr[i] = key_priority(fresh[i].first);
    I.key_list.push_back(fresh[i].first);
    I.prio_host.push_back(pr[i]);
  }
  I.pick_d.upload(pick, st);
  CUDA_CHECK(cudaMemcpyAsync(I.prio.p + old, pr.data(), add * sizeof(unsigned long long),
                             cudaMemcpyHostToDevice, st));
  CUDA_CHECK(cudaMemsetAsync(I.corr.p + old, 0, add * sizeof(float4), st));
  build_contacts_kernel<<<div_up(add, kCollThreads), kCollThreads, 0, st>>>(
      I.table_d.p, I.cols.p, I.pick_d.p, add, w_.contact_w_base.p, I.contacts.p + old);
  SILK_LAUNCHED();
  I.n_contacts = total;
  // Vertex incidence (contact_constraints.cu:139-201).
  int nv = w_.nv_total;
  I.inc_count.alloc(nv + 1);
  I.inc_off.alloc(nv + 1);
  I.inc_cursor.alloc(nv + 1);
  I.inc_count.zero(st);
  I.inc_cursor.zero(st);
  incidence_count_kernel<<<div_up(total, kCollThreads), kCollThreads, 0, st>>>(
      I.contacts.p, total, I.inc_count.p);
  SILK_LAUNCHED();
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, I.inc_count.p, I.inc_off.p, nv + 1, st);
  if (I.scan_temp.n < tb) I.scan_temp.alloc(tb);
  CUDA_CHECK(cub::DeviceScan::ExclusiveSum(I.scan_temp.p, tb, I.inc_count.p, I.inc_off.p,
                                           nv + 1, st));
  SILK_LAUNCHED();
  int nlist = 0;
  CUDA_CHECK(cudaMemcpyAsync(&nlist, I.inc_off.p + nv, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  I.inc_list.alloc(std::max(nlist, 1));
  incidence_fill_kernel<<<div_up(total, kCollThreads), kCollThreads, 0, st>>>(
      I.contacts.p, total, I.inc_off.p, I.inc_cursor.p, I.inc_list.p);
  SILK_LAUNCHED();
  CUDA_CHECK(cudaMemsetAsync(I.active_dof.p, 0, sizeof(int), st));
  activate_weights_kernel<<<div_up(nv, 256), 256, 0, st>>>(I.inc_count.p, nv,
                                                           w_.contact_w_base.p,
                                                           w_.contact_w.p, I.active_dof.p);
  SILK_LAUNCHED();
  last_dcd_build_ms = lap(t_lap);
  // Colouring by Jones-Plassmann rounds, all in one cooperative launch (a
  // round after the last contact is coloured changes nothing, so stopping
  // at the first round that leaves none uncoloured gives the colours of the
  // sequential greedy colouring in priority order).
  I.colors.alloc(total);
  I.colors.zero(st);
  I.col_info.zero(st);
  {
    static const int max_coop = [] {
      int dev = 0, sms = 0, per = 0;
      CUDA_CHECK(cudaGetDevice(&dev));
      CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, jp_grid_kernel, 256, 0));
      return sms * std::max(per, 1);
    }();
    const int grid = std::min(max_coop, std::max(1, div_up(total, 256)));
    CUDA_CHECK(cudaMemsetAsync(I.jp_flags.p, 0, 3 * sizeof(int), st));
    CUDA_CHECK(cudaMemsetAsync(I.gs_barrier.p, 0, 2 * sizeof(unsigned), st));
    const ContactDev* cp = I.contacts.p;
    const unsigned long long* pp = I.prio.p;
    int n = total;
    const int* op = I.inc_off.p;
    const int* lp = I.inc_list.p;
    int* colp = I.colors.p;
    int* infop = I.col_info.p;
    int* remp = I.jp_flags.p;
    unsigned* barp = I.gs_barrier.p;
    long long limit = w_.opt.barrier_spin_limit;
    void* args[] = {&cp, &pp, &n, &op, &lp, &colp, &infop, &remp, &barp, &limit};
    CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)jp_grid_kernel, dim3(grid), dim3(256),
                                           args, 0, st));
    SILK_LAUNCHED();
  }
  // Groups on the device: a stable sort of the contacts by colour (contact
  // index order inside a colour) and the group offsets.
  I.col_sorted.alloc(total);
  I.grp_in.alloc(total);
  I.groups.alloc(total);
  I.group_off.alloc(1026);
  iota_kernel<<<div_up(total, 256), 256, 0, st>>>(total, I.grp_in.p);
  SILK_LAUNCHED();
  size_t sb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, sb, I.colors.p, I.col_sorted.p, I.grp_in.p,
                                  I.groups.p, total, 0, 11, st);
  if (I.sort_temp.n < sb) I.sort_temp.alloc(sb);
  CUDA_CHECK(cub::DeviceRadixSort::SortPairs(I.sort_temp.p, sb, I.colors.p, I.col_sorted.p,
                                             I.grp_in.p, I.groups.p, total, 0, 11, st));
  SILK_LAUNCHED();
  group_offsets_kernel<<<div_up(1026, 256), 256, 0, st>>>(I.col_sorted.p, total, I.col_info.p,
                                                          I.group_off.p);
  SILK_LAUNCHED();
  last_dcd_color_ms = lap(t_lap);
  // Colour-ordered contacts on compact vertex slots for the single-block
  // Gauss-Seidel form.
  {
    I.gs_flag.alloc(nv);
    I.gs_slot.alloc(nv);
    I.gs_flag.zero(st);
    gs_flag_kernel<<<div_up(total, kCollThreads), kCollThreads, 0, st>>>(I.contacts.p, total,
                                                                        I.gs_flag.p);
    SILK_LAUNCHED();
    size_t tb2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb2, I.gs_flag.p, I.gs_slot.p, nv, st);
    if (I.scan_temp.n < tb2) I.scan_temp.alloc(tb2);
    CUDA_CHECK(cub::DeviceScan::ExclusiveSum(I.scan_temp.p, tb2, I.gs_flag.p, I.gs_slot.p, nv,
                                             st));
    SILK_LAUNCHED();
    gs_nslots_kernel<<<1, 1, 0, st>>>(I.gs_slot.p, I.gs_flag.p, nv, I.col_info.p);
    SILK_LAUNCHED();
    I.gs_vlist.alloc(nv);  // the touched vertices are at most all of them
    gs_vlist_kernel<<<div_up(nv, 256), 256, 0, st>>>(I.gs_flag.p, I.gs_slot.p, nv, I.gs_vlist.p);
    SILK_LAUNCHED();
    I.gs_cc.alloc(total);
    I.gs_ccorr.alloc(total);
    gs_gather_kernel<<<div_up(total, kCollThreads), kCollThreads, 0, st>>>(
        I.contacts.p, I.groups.p, total, I.gs_slot.p, I.gs_cc.p);
    SILK_LAUNCHED();
    // Slot incidence in colour order for the pipelined form's warm start.
    const int ne = 4 * total;
    I.gs_ikey.alloc(ne);
    I.gs_ival.alloc(ne);
    I.gs_ikey_s.alloc(ne);
    I.gs_vinc.alloc(ne);
    I.gs_voff.alloc(nv + 1);
    gs_inc_keys_kernel<<<div_up(ne, 256), 256, 0, st>>>(I.gs_cc.p, total, I.gs_ikey.p,
                                                        I.gs_ival.p);
    SILK_LAUNCHED();
    size_t sb2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sb2, I.gs_ikey.p, I.gs_ikey_s.p, I.gs_ival.p,
                                    I.gs_vinc.p, ne, 0, 31, st);
    if (I.sort_temp.n < sb2) I.sort_temp.alloc(sb2);
    CUDA_CHECK(cub::DeviceRadixSort::SortPairs(I.sort_temp.p, sb2, I.gs_ikey.p, I.gs_ikey_s.p,
                                               I.gs_ival.p, I.gs_vinc.p, ne, 0, 31, st));
    SILK_LAUNCHED();
    gs_voff_kernel<<<div_up(nv + 1, 256), 256, 0, st>>>(I.gs_ikey_s.p, ne, I.col_info.p, nv,
                                                        I.gs_voff.p);
    SILK_LAUNCHED();
    I.gs_vent.alloc(ne);
    gs_vent_kernel<<<div_up(ne, 256), 256, 0, st>>>(I.gs_cc.p, I.gs_vinc.p, ne, I.gs_vent.p);
    SILK_LAUNCHED();
    I.gs_ready = true;
  }
  // The one host read of the contact build's colouring and layout.
  int info[5] = {0, 0, 0, 0, 0};
  CUDA_CHECK(cudaMemcpyAsync(info, I.col_info.p, sizeof(info), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  if (info[1] > 0 || info[3] > 0) throw CudaError("Too many colors");
  I.n_colors = info[0];
  I.max_group = info[2];
  I.gs_nslots = info[4];
  last_dcd_layout_ms = lap(t_lap);
  return add;
}

void CollisionSystem::contact_solve_launch() {
  CollisionImpl& I = *impl_;
  if (I.n_contacts == 0) return;
  cudaStream_t st = w_.stream;
  const size_t smem = (size_t)I.gs_nslots * sizeof(float4);
  if (I.gs_ready && w_.opt.contact_gs_form != 1 && I.max_group <= kGsBlockThreads &&
      smem <= kGsBlockSmemMax) {
    static const bool attr = [] {
      CUDA_CHECK(cudaFuncSetAttribute(contact_gs_block_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kGsBlockSmemMax));
      return true;
    }();
    (void)attr;
    // Only as many warps as the largest colour needs: every colour phase ends
    // in a block barrier, whose cost grows with the number of warps.
    const int threads = std::max(32, div_up(I.max_group, 32) * 32);
    // Four staging stages where they fit, else two, else one (the copy for a
    // colour is then issued 4, 2 or 1 phases ahead).
    int ns_log = 2;
    GsPipeLayout L = gs_pipe_layout(I.gs_nslots, I.n_contacts, I.n_colors, threads, 4);
    while (L.bytes > kGsBlockSmemMax && ns_log > 0) {
      --ns_log;
      L = gs_pipe_layout(I.gs_nslots, I.n_contacts, I.n_colors, threads, 1 << ns_log);
    }
    if (L.bytes <= kGsBlockSmemMax) {
      static const bool pattr = [] {
        CUDA_CHECK(cudaFuncSetAttribute(contact_gs_pipe_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kGsBlockSmemMax));
        return true;
      }();
      (void)pattr;
      contact_gs_pipe_kernel<<<1, threads, L.bytes, st>>>(
          I.gs_cc.p, I.group_off.p, I.n_colors, I.n_contacts, I.corr.p, I.gs_vlist.p,
          I.gs_nslots, w_.contact_p.p, w_.cg_fail.p, gs_skip_, I.gs_voff.p, I.gs_vent.p, ns_log);
      SILK_LAUNCHED();
      return;
    }
    contact_gs_block_kernel<<<1, threads, smem, st>>>(
        I.gs_cc.p, I.group_off.p, I.n_colors, I.n_contacts, I.corr.p, I.gs_ccorr.p,
        I.gs_vlist.p, I.gs_nslots, w_.contact_p.p, gs_skip_);
    SILK_LAUNCHED();
    return;
  }
  static const int max_coop = [] {
    int dev = 0, sms = 0, per = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, contact_gs_kernel, 256, 0));
    return sms * std::max(per, 1);
  }();
  int grid = std::min(max_coop, std::max(1, div_up(I.max_group, 256)));
  CUDA_CHECK(cudaMemsetAsync(I.gs_barrier.p, 0, 2 * sizeof(unsigned), st));
  const ContactDev* c = I.contacts.p;
  const int* g = I.groups.p;
  const int* go = I.group_off.p;
  int nc = I.n_colors;
  float4* corr = I.corr.p;
  float4* p = w_.contact_p.p;
  unsigned* bar = I.gs_barrier.p;
  const int* skip = gs_skip_;
  void* args[] = {&c, &g, &go, &nc, &corr, &p, &bar, &skip};
  CUDA_CHECK(cudaLaunchCooperativeKernel((const void*)contact_gs_kernel, dim3(grid), dim3(256),
                                         args, 0, st));
  SILK_LAUNCHED();
}

float CollisionSystem::min_toi(float ts, float max_time, float ms, int* nq, int* nh,
                               bool prune) {
  CollisionImpl& I = *impl_;
  cudaStream_t st = w_.stream;
  *nq = 0;
  *nh = 0;
  if (max_time == 0.0f) return 0.0f;
  const auto t_gather = std::chrono::steady_clock::now();
  int n = gather_candidates(I, st);
  last_gather_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_gather)
          .count();
  *nq = n;
  if (n == 0) return max_time;
  // Scene-wide magnitude for the numerical filter (find_collision.cu:157-172).
  float absmax[3] = {0, 0, 0};
  for (auto& o : I.objs)
    for (int d = 0; d < 3; ++d) {
      float mn = o->bmin[d] + o->padding, mx = o->bmax[d] - o->padding;
      absmax[d] = std::max(absmax[d], std::fabs(mn));
      absmax[d] = std::max(absmax[d], std::fabs(mx));
    }
  const float kEE = 3.814698e-06f, kVF = 4.053116e-06f;
  float3 ee = make_float3(kEE * std::max(absmax[0], 1.0f), kEE * std::max(absmax[1], 1.0f),
                          kEE * std::max(absmax[2], 1.0f));
  float3 vf = make_float3(kVF * std::max(absmax[0], 1.0f), kVF * std::max(absmax[1], 1.0f),
                          kVF * std::max(absmax[2], 1.0f));
  float local_tol = kCcdTolerance / max_time;
  unsigned one_bits;
  float one = max_time / max_time;
  std::memcpy(&one_bits, &one, 4);
  CUDA_CHECK(cudaMemcpyAsync(I.min_bits.p, &one_bits, 4, cudaMemcpyHostToDevice, st));
  // counts: [hits, storage overflows, first-pass spills, work counter]
  CUDA_CHECK(cudaMemsetAsync(I.ccd_counts.p, 0, 4 * sizeof(int), st));
  if ((int)I.ccd_overflow.n < n) I.ccd_overflow.alloc(n + n / 4);
  static const int sms = [] {
    int dev = 0, n = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
  }();
  auto grid_for = [&](int m) { return std::max(1, std::min(div_up(m, kCollThreads), 8 * sms)); };
  if (!I.ccd_ev[0]) {
    for (auto& e : I.ccd_ev) CUDA_CHECK(cudaEventCreate(&e));
  }
  CcdSpill first{nullptr, 0, nullptr, I.ccd_overflow.p, I.ccd_counts.p + 2};
  CUDA_CHECK(cudaEventRecord(I.ccd_ev[0], st));
  ccd_kernel<<<grid_for(n), kCollThreads, 0, st>>>(
      I.table_d.p, I.cand.p, n, ts, max_time, ms, vf, ee, local_tol, I.min_bits.p,
      I.ccd_counts.p, first, I.ccd_counts.p + 3, prune ? 1 : 0);
  SILK_LAUNCHED();
  CUDA_CHECK(cudaEventRecord(I.ccd_ev[1], st));
  int counts[3];
  CUDA_CHECK(cudaMemcpyAsync(counts, I.ccd_counts.p, sizeof(counts), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  last_second_pass_queries = counts[2];
  CUDA_CHECK(cudaEventRecord(I.ccd_ev[2], st));
  // Second pass for the searches that outgrew the per-thread array: one
  // query per block, its pending boxes in a heap in shared memory.
  if (counts[2] > 0) {
    const int cap = kCcdMaxIter + 2;
    const size_t smem = ccd_heap_smem_bytes(cap);
    static const bool attr = [smem] {
      CUDA_CHECK(cudaFuncSetAttribute(ccd_heap_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      return true;
    }();
    (void)attr;
    CcdSpill second{nullptr, cap, I.ccd_overflow.p, nullptr, nullptr, 1};
    ccd_heap_kernel<<<counts[2], 32, smem, st>>>(I.table_d.p, I.cand.p, counts[2], ts, max_time,
                                                 ms, vf, ee, local_tol, I.min_bits.p,
                                                 I.ccd_counts.p, second, prune ? 1 : 0);
    SILK_LAUNCHED();
  }
  CUDA_CHECK(cudaEventRecord(I.ccd_ev[3], st));
  unsigned bits = 0;
  CUDA_CHECK(cudaMemcpyAsync(&bits, I.min_bits.p, 4, cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaMemcpyAsync(counts, I.ccd_counts.p, sizeof(counts), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  {
    float a = 0.f, b = 0.f;
    CUDA_CHECK(cudaEventElapsedTime(&a, I.ccd_ev[0], I.ccd_ev[1]));
    CUDA_CHECK(cudaEventElapsedTime(&b, I.ccd_ev[2], I.ccd_ev[3]));
    last_first_pass_ms = a;
    last_second_pass_ms = b;
  }
  if (counts[1] > 0) throw CudaError("CCD search storage overflow");
  *nh = counts[0];
  float local;
  std::memcpy(&local, &bits, 4);
  return max_time * local;
}

int CollisionSystem::contact_count() const { return impl_->n_contacts; }
int CollisionSystem::color_count() const { return impl_->n_colors; }
const int* CollisionSystem::active_dof_device() const { return impl_->active_dof.p; }
int CollisionSystem::last_candidates() const { return impl_->n_cand; }

int CollisionSystem::debug_candidates(int* out, int64_t cap) {
  CollisionImpl& I = *impl_;
  int n = gather_candidates(I, w_.stream);
  std::vector<int4> h(n);
  if (n) CUDA_CHECK(cudaMemcpy(h.data(), I.cand.p, n * sizeof(int4), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n && i < cap; ++i) {
    int kind = h[i].z >> 16, sa = h[i].z & 0xffff, sb = h[i].w;
    out[5 * i] = kind;
    out[5 * i + 1] = (int)I.objs[sa]->handle;
    out[5 * i + 2] = h[i].x;
    out[5 * i + 3] = (int)I.objs[sb]->handle;
    out[5 * i + 4] = h[i].y;
  }
  return n;
}

int CollisionSystem::debug_contacts(int* keys, int64_t cap) {
  const CollisionImpl& I = *impl_;
  int i = 0;
  for (const Key& k : I.keys) {  // std::set: canonical key order
    if (i < cap) {
      keys[7 * i] = k.type;
      keys[7 * i + 1] = (int)k.oa;
      keys[7 * i + 2] = (int)k.ob;
      for (int q = 0; q < 4; ++q) keys[7 * i + 3 + q] = k.idx[q];
    }
    ++i;
  }
  return i;
}

int CollisionSystem::debug_dcd(float t, float dact, int* keys, int64_t cap) {
  CollisionImpl& I = *impl_;
  cudaStream_t st = w_.stream;
  int n = gather_candidates(I, st);
  if (n == 0) return 0;
  if (I.cols_cap < n) {
    I.cols_cap = n + n / 4;
    I.cols.alloc(I.cols_cap);
  }
  CUDA_CHECK(cudaMemsetAsync(I.counter.p + 1, 0, sizeof(int), st));
  dcd_kernel<<<div_up(n, kCollThreads), kCollThreads, 0, st>>>(
      I.table_d.p, I.cand.p, n, t, dact, I.cols.p, I.cols_cap, I.counter.p + 1);
  SILK_LAUNCHED();
  int m = 0;
  CUDA_CHECK(cudaMemcpyAsync(&m, I.counter.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_CHECK(cudaStreamSynchronize(st));
  std::vector<CollisionDev> hc(m);
  if (m) CUDA_CHECK(cudaMemcpy(hc.data(), I.cols.p, m * sizeof(CollisionDev), cudaMemcpyDeviceToHost));
  std::vector<Key> ks;
  for (auto& c : hc)
    ks.push_back(make_key(c.type, I.objs[c.slot_a]->handle, I.objs[c.slot_b]->handle, c.idx));
  std::sort(ks.begin(), ks.end());
  for (int i = 0; i < m && i < cap; ++i) {
    keys[7 * i] = ks[i].type;
    keys[7 * i + 1] = (int)ks[i].oa;
    keys[7 * i + 2] = (int)ks[i].ob;
    for (int k = 0; k < 4; ++k) keys[7 * i + 3 + k] = ks[i].idx[k];
  }
  return m;
}

void ccd_batch_host(bool vf, const float* x, int64_t n, const float* err3,
                    const float* ms, float tol, int max_iter, float max_time, int* hit,
                    float* toi, float* t_upper) {
  if (n == 0) return;
  DevBuf<float> xd, msd, toid, tupd;
  DevBuf<int> hitd;
  xd.alloc(24 * n);
  msd.alloc(n);
  toid.alloc(n);
  tupd.alloc(n);
  hitd.alloc(n);
  CUDA_CHECK(cudaMemcpy(xd.p, x, 24 * n * sizeof(float), cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(msd.p, ms, n * sizeof(float), cudaMemcpyHostToDevice));
  DevBuf<int> over, counts;
  over.alloc(n);
  counts.alloc(2);
  CUDA_CHECK(cudaMemset(counts.p, 0, 2 * sizeof(int)));
  float3 e3 = make_float3(err3[0], err3[1], err3[2]);
  CcdSpill first{nullptr, 0, nullptr, over.p, counts.p};
  ccd_batch_kernel<<<div_up((int)n, kCollThreads), kCollThreads>>>(
      vf, xd.p, (int)n, e3, msd.p, tol, max_iter, max_time, hitd.p, toid.p, tupd.p,
      counts.p + 1, first);
  SILK_LAUNCHED();
  CUDA_CHECK(cudaGetLastError());
  int h[2];
  CUDA_CHECK(cudaMemcpy(h, counts.p, sizeof(h), cudaMemcpyDeviceToHost));
  if (h[0] > 0) {
    // Second pass with max_iter + 2 pending boxes per search (unbounded
    // searches, max_iter <= 0, get 65536).
    int cap = max_iter > 0 ? max_iter + 2 : 65536;
    const size_t heap_smem = ccd_heap_smem_bytes(cap);
    if (heap_smem <= kCcdHeapSmemMax) {
      // One query per block, its pending boxes in a heap in shared memory.
      static const bool attr = [] {
        CUDA_CHECK(cudaFuncSetAttribute(ccd_batch_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kCcdHeapSmemMax));
        return true;
      }();
      (void)attr;
      CcdSpill second{nullptr, cap, over.p, nullptr, nullptr, 1};
      ccd_batch_kernel<<<h[0], 32, heap_smem>>>(vf, xd.p, h[0], e3, msd.p, tol, max_iter,
                                                max_time, hitd.p, toid.p, tupd.p, counts.p + 1,
                                                second);
      SILK_LAUNCHED();
    } else {
      int chunk =
          std::max(1, std::min(h[0], (int)((256ll << 20) / ((long long)cap * sizeof(IBox)))));
      DevBuf<IBox> spill;
      spill.alloc((size_t)chunk * cap);
      for (int start = 0; start < h[0]; start += chunk) {
        int m = std::min(chunk, h[0] - start);
        CcdSpill second{spill.p, cap, over.p + start, nullptr, nullptr};
        ccd_batch_kernel<<<div_up(m, kCollThreads), kCollThreads>>>(
            vf, xd.p, m, e3, msd.p, tol, max_iter, max_time, hitd.p, toid.p, tupd.p,
            counts.p + 1, second);
        SILK_LAUNCHED();
      }
    }
    CUDA_CHECK(cudaMemcpy(h, counts.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (h[1] > 0) throw CudaError("CCD search storage overflow");
  }
  CUDA_CHECK(cudaMemcpy(hit, hitd.p, n * sizeof(int), cudaMemcpyDeviceToHost));
  CUDA_CHECK(cudaMemcpy(toi, toid.p, n * sizeof(float), cudaMemcpyDeviceToHost));
  if (t_upper) CUDA_CHECK(cudaMemcpy(t_upper, tupd.p, n * sizeof(float), cudaMemcpyDeviceToHost));
}

namespace {
__global__ void color_explicit_round(const int4* v4, const unsigned long long* prio, int n,
                                     const int* off, const int* list, int* color,
                                     int* remaining, int* overflow) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || color[i] != 0) return;
  unsigned long long pi = prio[i];
  unsigned used[32];
  for (int k = 0; k < 32; ++k) used[k] = 0u;
  int vs[4] = {v4[i].x, v4[i].y, v4[i].z, v4[i].w};
  for (int s = 0; s < 4; ++s) {
    int v = vs[s];
    if (v < 0) continue;
    for (int q = off[v]; q < off[v + 1]; ++q) {
      int j = list[q];
      if (j == i) continue;
      unsigned long long pj = prio[j];
      if (!(pj > pi || (pj == pi && j < i))) continue;
      int cj = ((volatile int*)color)[j];
      if (cj == 0) {
        atomicAdd(remaining, 1);
        return;
      }
      if (cj <= 1024) used[(cj - 1) >> 5] |= 1u << ((cj - 1) & 31);
    }
  }
  int col = 0;
  for (int k = 0; k < 32 && col == 0; ++k)
    if (used[k] != 0xffffffffu) col = 32 * k + __ffs(~used[k]);
  if (col == 0) {
    atomicAdd(overflow, 1);
    col = 1025;
  }
  color[i] = col;
}
}  // namespace

namespace {
__global__ void coulomb_debug_kernel(int n, const float* u, const float* nrm, const float* mu,
                                     float* out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  float3 r = coulomb_project(make_float3(u[3 * q], u[3 * q + 1], u[3 * q + 2]),
                             make_float3(nrm[3 * q], nrm[3 * q + 1], nrm[3 * q + 2]), mu[q]);
  out[3 * q] = r.x;
  out[3 * q + 1] = r.y;
  out[3 * q + 2] = r.z;
}
}  // namespace

void coulomb_debug_host(const float* u, const float* nrm, const float* mu, int64_t n,
                        float* out) {
  if (n == 0) return;
  DevBuf<float> ud, nd, md, od;
  ud.alloc(3 * n);
  nd.alloc(3 * n);
  md.alloc(n);
  od.alloc(3 * n);
  CUDA_CHECK(cudaMemcpy(ud.p, u, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(nd.p, nrm, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  CUDA_CHECK(cudaMemcpy(md.p, mu, n * sizeof(float), cudaMemcpyHostToDevice));
  coulomb_debug_kernel<<<div_up((int)n, 256), 256>>>((int)n, ud.p, nd.p, md.p, od.p);
  SILK_LAUNCHED();
  CUDA_CHECK(cudaGetLastError());
  CUDA_CHECK(cudaMemcpy(out, od.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost));
}

int color_contacts_host(const int* verts4, const uint64_t* prio, int64_t n, int* colors) {
  if (n == 0) return 0;
  int maxv = -1;
  for (int64_t i = 0; i < 4 * n; ++i) maxv = std::max(maxv, verts4[i]);
  int nv = maxv + 1;
  std::vector<int> cnt(nv + 1, 0);
  for (int64_t i = 0; i < 4 * n; ++i)
    if (verts4[i] >= 0) cnt[verts4[i] + 1]++;
  for (int v = 0; v < nv; ++v) cnt[v + 1] += cnt[v];
  std::vector<int> list(std::max(cnt[nv], 1)), cur(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < 4; ++s) {
      int v = verts4[4 * i + s];
      if (v >= 0) list[cur[v]++] = (int)i;
    }
  std::vector<int4> v4(n);
  for (int64_t i = 0; i < n; ++i)
    v4[i] = make_int4(verts4[4 * i], verts4[4 * i + 1], verts4[4 * i + 2], verts4[4 * i + 3]);
  DevBuf<int4> v4d;
  DevBuf<unsigned long long> pd;
  DevBuf<int> offd, listd, cold, flags;
  v4d.upload(v4, 0);
  std::vector<unsigned long long> pv(prio, prio + n);
  pd.upload(pv, 0);
  offd.upload(cnt, 0);
  listd.upload(list, 0);
  cold.alloc(n);
  cold.zero(0);
  flags.alloc(2);
  for (int round = 0; round < 100000; ++round) {
    CUDA_CHECK(cudaMemset(flags.p, 0, 2 * sizeof(int)));
    color_explicit_round<<<div_up((int)n, kCollThreads), kCollThreads>>>(
        v4d.p, pd.p, (int)n, offd.p, listd.p, cold.p, flags.p, flags.p + 1);
    SILK_LAUNCHED();
    int f[2];
    CUDA_CHECK(cudaMemcpy(f, flags.p, sizeof(f), cudaMemcpyDeviceToHost));
    if (f[1] > 0) return -1;
    if (f[0] == 0) break;
  }
  CUDA_CHECK(cudaMemcpy(colors, cold.p, n * sizeof(int), cudaMemcpyDeviceToHost));
  int nc = 0;
  for (int64_t i = 0; i < n; ++i) nc = std::max(nc, colors[i]);
  return nc;
}

// ---------------------------------------------------------------------------
// CCD batch over caller-owned device buffers that allocates nothing.
//
// Its only working memory is one statically sized device array, created
// with this module on every device that loads the library:
//   [0, 256)                 counters, which must be zero when the first pass
//                            starts (each call zeroes them on its stream):
//                            [0] queries whose search overflowed the
//                            96-box per-thread storage, [1] second-pass
//                            searches that exhausted their storage, [2] next
//                            overflowed query for the second pass to take
//   [256, 256 + 4 MiB)       indices of the overflowed queries (written by
//                            the first pass before they are read; no
//                            initial value needed)
//   [.., + 6,294,528 B)      pending-box storage of the second pass:
//                            kNoAllocSpillSlots regions of max_iter + 2 boxes
//                            (the most a search of max_iter steps can hold)
// The first pass is ccd_batch_kernel itself; the second pass runs the
// overflowed queries on kNoAllocSpillSlots threads that each reuse one
// storage region, so the scratch size does not grow with the batch.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocListOffset = 256;
constexpr size_t kNoAllocSpillOffset =
    kNoAllocListOffset + sizeof(int) * (size_t)kNoAllocMaxQueries;
constexpr size_t kNoAllocScratchBytes =
    kNoAllocSpillOffset + sizeof(IBox) * (size_t)kNoAllocSpillSlots * (kNoAllocMaxIter + 2);
static_assert(kNoAllocSpillOffset % 256 == 0, "spill region alignment");

static __device__ __align__(256) unsigned char g_ccd_noalloc_scratch[kNoAllocScratchBytes];

__global__ void __launch_bounds__(kNoAllocSpillSlots) ccd_batch_spill_kernel(
    bool vf, const float* x, float3 err, const float* ms, float tol, int max_iter,
    float max_time, int* hit, float* toi, float* tup, int* counters, const int* list,
    IBox* spill) {
  const int n_over = counters[0];
  DfsStack st;
  st.cap = max_iter + 2;
  st.e = spill + (size_t)threadIdx.x * st.cap;
  const float e[3] = {err.x, err.y, err.z};
  for (;;) {
    int j = atomicAdd(&counters[2], 1);
    if (j >= n_over) return;
    int q = list[j];
    float3 Pt[8];
    for (int k = 0; k < 8; ++k)
      Pt[k] = make_float3(x[24 * q + 3 * k], x[24 * q + 3 * k + 1], x[24 * q + 3 * k + 2]);
    float t = max_time, u = max_time;
    int s = ccd_query(vf, Pt, e, ms[q], tol, max_iter, max_time, t, u, st);
    if (s == 2) {
      // Storage ran out: report the conservative answer (a hit at time 0).
      atomicAdd(&counters[1], 1);
      hit[q] = 1;
      toi[q] = 0.0f;
      if (tup) tup[q] = max_time;
      continue;
    }
    hit[q] = s != 0 ? 1 : 0;
    toi[q] = s != 0 ? t : max_time;
    if (tup) tup[q] = s != 0 ? u : max_time;
  }
}

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex[kNoAllocMaxDevices];
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

bool device_buffer(const void* p, int dev) {
  if (!p || (reinterpret_cast<uintptr_t>(p) & 3u)) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}
}  // namespace

NoAllocStatus ccd_batch_noalloc(bool vf, const float* x, int64_t n, const float* err3,
                                const float* ms, float tol, int max_iter, float max_time,
                                int* hit, float* toi, float* t_upper, cudaStream_t stream,
                                int* n_spilled) {
  if (n < 0 || !err3) return NoAllocStatus::kBadArgument;
  if (n > kNoAllocMaxQueries || max_iter < 1 || max_iter > kNoAllocMaxIter)
    return NoAllocStatus::kBeyondLimits;
  // A stream under capture is refused before anything is queued on it: the
  // call reads results back and synchronises, which would invalidate the
  // caller's capture.
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess ||
      capture != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return NoAllocStatus::kBadArgument;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    cudaGetLastError();
    return NoAllocStatus::kCudaError;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex[dev]);
  if (!g_noalloc_addr[dev]) {
    // One-time setup on this device (the device is current): resolving the
    // symbol loads this module's kernels and its scratch array.
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_ccd_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return NoAllocStatus::kCudaError;
    }
    g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
  }
  if (n_spilled) *n_spilled = 0;
  if (n == 0) return NoAllocStatus::kOk;
  if (!device_buffer(x, dev) || !device_buffer(ms, dev) || !device_buffer(hit, dev) ||
      !device_buffer(toi, dev) || (t_upper && !device_buffer(t_upper, dev)))
    return NoAllocStatus::kBadArgument;

  unsigned char* base = g_noalloc_addr[dev];
  int* counters = reinterpret_cast<int*>(base);
  int* list = reinterpret_cast<int*>(base + kNoAllocListOffset);
  IBox* spill = reinterpret_cast<IBox*>(base + kNoAllocSpillOffset);
  const float3 e3 = make_float3(err3[0], err3[1], err3[2]);
  // Any failure after work was queued waits for that work before returning,
  // so the lock is released only once the scratch array is idle.
  auto fail_after_queue = [&]() {
    cudaGetLastError();
    cudaStreamSynchronize(stream);
    cudaGetLastError();
    return NoAllocStatus::kCudaError;
  };
  cudaGetLastError();  // an earlier, unrelated error is not this call's
  if (cudaMemsetAsync(counters, 0, 4 * sizeof(int), stream) != cudaSuccess)
    return fail_after_queue();
  CcdSpill first{nullptr, 0, nullptr, list, counters};
  ccd_batch_kernel<<<div_up((int)n, kCollThreads), kCollThreads, 0, stream>>>(
      vf, x, (int)n, e3, ms, tol, max_iter, max_time, hit, toi, t_upper, counters + 1, first);
  SILK_LAUNCHED();
  if (cudaGetLastError() != cudaSuccess) return fail_after_queue();
  ccd_batch_spill_kernel<<<1, kNoAllocSpillSlots, 0, stream>>>(
      vf, x, e3, ms, tol, max_iter, max_time, hit, toi, t_upper, counters, list, spill);
  SILK_LAUNCHED();
  if (cudaGetLastError() != cudaSuccess) return fail_after_queue();
  int h[4] = {0, 0, 0, 0};
  if (cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    return fail_after_queue();
  if (cudaStreamSynchronize(stream) != cudaSuccess) {
    cudaGetLastError();
    return NoAllocStatus::kCudaError;
  }
  if (n_spilled) *n_spilled = h[0];
  return h[1] > 0 ? NoAllocStatus::kStorageExhausted : NoAllocStatus::kOk;
}

}  // namespace silkb
