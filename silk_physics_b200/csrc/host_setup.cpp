// Host-side static setup of a cloth (runs once per cloth / dt change).
//
// Reference counterparts: common/mesh.cpp (checks), backend/cuda/
// mesh_partition.cu + graph_partition.cpp (partition), common/
// cloth_assembly_l2_cache.cpp and backend/cuda/assembly/
// cloth_assembly_l1_cache.cu (assembly), backend/cuda/solver/
// mas_preconditioner.cu:50-478 (MAS topology and coarse spaces).
#include "host_setup.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <cstdint>
#include <map>
#include <numeric>
#include <unordered_map>

namespace silkb {

namespace {

constexpr int kBank = 32;
constexpr int kMaxCoarse = 4;

std::string check_schema(const float* v, long nvf, const int* f, long nfi,
                         int min_v, int min_f) {
  if (v == nullptr || (nfi > 0 && f == nullptr) || (min_f > 0 && f == nullptr))
    return "null pointer in verts or faces";
  if (nvf % 3 != 0 || nfi % 3 != 0) return "verts/faces size not a multiple of 3";
  if (nvf / 3 < min_v) return "too few vertices";
  if (nfi / 3 < min_f) return "too few faces";
  return {};
}

std::string check_finite_and_index(const float* v, long nvf, const int* f,
                                   long nfi) {
  for (long i = 0; i < nvf; ++i)
    if (!std::isfinite(v[i])) return "vertex positions contain NaN/Inf";
  long nv = nvf / 3;
  for (long i = 0; i < nfi / 3; ++i) {
    int a = f[3 * i], b = f[3 * i + 1], c = f[3 * i + 2];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv)
      return "face index out of range";
    if (a == b || b == c || c == a) return "triangle with repeated vertex";
  }
  return {};
}

}  // namespace

std::string check_mesh_indices(const float* v, long nvf, const int* f, long nfi) {
  std::string r = check_schema(v, nvf, f, nfi, 0, 0);
  if (!r.empty()) return r;
  return check_finite_and_index(v, nvf, f, nfi);
}

std::string check_cloth_mesh(const float* v, long nvf, const int* f, long nfi) {
  std::string r = check_schema(v, nvf, f, nfi, 3, 1);
  if (!r.empty()) return r;
  r = check_finite_and_index(v, nvf, f, nfi);
  if (!r.empty()) return r;
  int nv = (int)(nvf / 3), nf = (int)(nfi / 3);
  // Internal angles within [0.5, 179.5] degrees (mesh.cpp:124-146).
  const float kPi = 3.14159265358979323846f;
  const float min_rad = 0.5f * kPi / 180.0f;
  const float max_rad = kPi - min_rad;
  for (int t = 0; t < nf; ++t) {
    double p[3][3];
    for (int k = 0; k < 3; ++k)
      for (int d = 0; d < 3; ++d) p[k][d] = v[3 * f[3 * t + k] + d];
    for (int k = 0; k < 3; ++k) {
      const double* o = p[k];
      const double* a = p[(k + 1) % 3];
      const double* b = p[(k + 2) % 3];
      double ea[3], eb[3];
      for (int d = 0; d < 3; ++d) {
        ea[d] = a[d] - o[d];
        eb[d] = b[d] - o[d];
      }
      double la = std::sqrt(ea[0] * ea[0] + ea[1] * ea[1] + ea[2] * ea[2]);
      double lb = std::sqrt(eb[0] * eb[0] + eb[1] * eb[1] + eb[2] * eb[2]);
      if (la == 0.0 || lb == 0.0) return "degenerate triangle";
      double c = (ea[0] * eb[0] + ea[1] * eb[1] + ea[2] * eb[2]) / (la * lb);
      c = std::max(-1.0, std::min(1.0, c));
      float ang = (float)std::acos(c);
      if (!(ang >= min_rad && ang <= max_rad)) return "poor triangle angle quality";
    }
  }
  // Edge manifold (mesh.cpp:148-160): every undirected edge in <= 2 faces.
  std::map<std::pair<int, int>, int> ecount;
  for (int t = 0; t < nf; ++t)
    for (int k = 0; k < 3; ++k) {
      int a = f[3 * t + k], b = f[3 * t + (k + 1) % 3];
      if (++ecount[{std::min(a, b), std::max(a, b)}] > 2)
        return "non-manifold edge";
    }
  // Vertex manifold (mesh.cpp:162-175): faces around a vertex form one fan
  // connected through edges incident to that vertex.
  std::vector<std::vector<int>> vf(nv);
  for (int t = 0; t < nf; ++t)
    for (int k = 0; k < 3; ++k) vf[f[3 * t + k]].push_back(t);
  for (int vtx = 0; vtx < nv; ++vtx) {
    auto& fs = vf[vtx];
    if (fs.size() <= 1) continue;
    std::vector<int> parent(fs.size());
    std::iota(parent.begin(), parent.end(), 0);
    std::function<int(int)> find = [&](int x) {
      while (parent[x] != x) x = parent[x] = parent[parent[x]];
      return x;
    };
    std::map<int, int> other_owner;  // other endpoint of an incident edge
    for (size_t i = 0; i < fs.size(); ++i) {
      int t = fs[i];
      for (int k = 0; k < 3; ++k) {
        int o = f[3 * t + k];
        if (o == vtx) continue;
        auto it = other_owner.find(o);
        if (it == other_owner.end()) {
          other_owner[o] = (int)i;
        } else {
          int ra = find((int)i), rb = find(it->second);
          if (ra != rb) parent[ra] = rb;
        }
      }
    }
    int root = find(0);
    for (size_t i = 1; i < fs.size(); ++i)
      if (find((int)i) != root) return "non-manifold vertex";
  }
  // Single connected component of faces through shared edges
  // (mesh.cpp:177-189).
  {
    std::vector<int> parent(nf);
    std::iota(parent.begin(), parent.end(), 0);
    std::function<int(int)> find = [&](int x) {
      while (parent[x] != x) x = parent[x] = parent[parent[x]];
      return x;
    };
    std::map<std::pair<int, int>, int> first;
    for (int t = 0; t < nf; ++t)
      for (int k = 0; k < 3; ++k) {
        int a = f[3 * t + k], b = f[3 * t + (k + 1) % 3];
        auto key = std::make_pair(std::min(a, b), std::max(a, b));
        auto it = first.find(key);
        if (it == first.end()) {
          first[key] = t;
        } else {
          int ra = find(t), rb = find(it->second);
          if (ra != rb) parent[ra] = rb;
        }
      }
    int root = find(0);
    for (int t = 1; t < nf; ++t)
      if (find(t) != root) return "mesh has more than one connected component";
  }
  return {};
}

std::string check_obstacle_mesh(const float* v, long nvf, const int* f,
                                long nfi) {
  std::string r = check_schema(v, nvf, f, nfi, 1, 0);
  if (!r.empty()) return r;
  return check_finite_and_index(v, nvf, f, nfi);
}

std::vector<int> mesh_edges(const int* faces, int nf) {
  std::vector<std::pair<int, int>> e;
  e.reserve(3 * (size_t)nf);
  for (int t = 0; t < nf; ++t)
    for (int k = 0; k < 3; ++k) {
      int a = faces[3 * t + k], b = faces[3 * t + (k + 1) % 3];
      e.emplace_back(std::min(a, b), std::max(a, b));
    }
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  std::vector<int> out;
  out.reserve(2 * e.size());
  for (auto& [a, b] : e) {
    out.push_back(a);
    out.push_back(b);
  }
  return out;
}

float average_edge_length(const float* v, const std::vector<int>& E) {
  // mesh.cpp:262-268: float accumulation in edge order.
  float s = 0.0f;
  int ne = (int)E.size() / 2;
  if (ne == 0) return 0.0f;
  for (int i = 0; i < ne; ++i) {
    int a = E[2 * i], b = E[2 * i + 1];
    float dx = v[3 * a] - v[3 * b], dy = v[3 * a + 1] - v[3 * b + 1],
          dz = v[3 * a + 2] - v[3 * b + 2];
    s += std::sqrt(dx * dx + dy * dy + dz * dz);
  }
  return s / (float)ne;
}

// Greedy breadth-first growth of connected parts of <= 32 vertices, seeded in
// Morton order of the rest positions so that consecutive parts are spatially
// close (which keeps the coarse MAS levels compact).  Small leftover parts are
// merged into an adjacent part when the union still fits in a bank.
void partition_mesh(const float* verts, int nv, const int* faces, int nf,
                    std::vector<int>& perm, std::vector<int>& part_offsets) {
  std::vector<std::vector<int>> adj(nv);
  for (int t = 0; t < nf; ++t)
    for (int k = 0; k < 3; ++k) {
      int a = faces[3 * t + k], b = faces[3 * t + (k + 1) % 3];
      adj[a].push_back(b);
      adj[b].push_back(a);
    }
  float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
  for (int i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], verts[3 * i + d]);
      hi[d] = std::max(hi[d], verts[3 * i + d]);
    }
  auto spread = [](uint32_t x) {
    uint64_t y = x & 0x1fffff;
    y = (y | y << 32) & 0x1f00000000ffffULL;
    y = (y | y << 16) & 0x1f0000ff0000ffULL;
    y = (y | y << 8) & 0x100f00f00f00f00fULL;
    y = (y | y << 4) & 0x10c30c30c30c30c3ULL;
    y = (y | y << 2) & 0x1249249249249249ULL;
    return y;
  };
  // One scale for all axes (a cube around the mesh): a nearly flat axis must
  // not have its noise stretched over the full code range.
  double ext = 0.0;
  for (int d = 0; d < 3; ++d) ext = std::max(ext, (double)hi[d] - lo[d]);
  std::vector<uint64_t> code(nv);
  for (int i = 0; i < nv; ++i) {
    uint64_t c = 0;
    for (int d = 0; d < 3; ++d) {
      double u = ext > 0 ? ((double)verts[3 * i + d] - lo[d]) / ext : 0.0;
      uint32_t q = (uint32_t)std::min(2097151.0, std::max(0.0, u * 2097151.0));
      c |= spread(q) << d;
    }
    code[i] = c;
  }
  std::vector<int> order(nv);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return code[a] < code[b]; });
  std::vector<int> rank(nv);
  for (int i = 0; i < nv; ++i) rank[order[i]] = i;
  for (auto& a : adj) {
    std::sort(a.begin(), a.end(), [&](int x, int y) { return rank[x] < rank[y]; });
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  std::vector<int> part(nv, -1);
  std::vector<std::vector<int>> parts;
  for (int seed : order) {
    if (part[seed] != -1) continue;
    int p = (int)parts.size();
    parts.emplace_back();
    auto& members = parts.back();
    members.push_back(seed);
    part[seed] = p;
    for (size_t head = 0; head < members.size() && members.size() < kBank; ++head) {
      int u = members[head];
      for (int w : adj[u]) {
        if (members.size() >= kBank) break;
        if (part[w] != -1) continue;
        part[w] = p;
        members.push_back(w);
      }
    }
  }
  // Merge small parts into the smallest adjacent part that can absorb them.
  for (size_t p = 0; p < parts.size(); ++p) {
    if (parts[p].empty() || parts[p].size() >= 12) continue;
    int best = -1;
    size_t best_size = kBank + 1;
    for (int u : parts[p])
      for (int w : adj[u]) {
        int q = part[w];
        if (q == (int)p || parts[q].empty()) continue;
        if (parts[q].size() + parts[p].size() <= (size_t)kBank &&
            parts[q].size() < best_size) {
          best = q;
          best_size = parts[q].size();
        }
      }
    if (best < 0) continue;
    for (int u : parts[p]) {
      part[u] = best;
      parts[best].push_back(u);
    }
    parts[p].clear();
  }
  perm.assign(nv, -1);
  part_offsets.assign(1, 0);
  int next = 0;
  for (auto& m : parts) {
    if (m.empty()) continue;
    for (int u : m) perm[u] = next++;
    part_offsets.push_back(next);
  }
}

namespace {

struct Trip {
  int r, c;
  double v;
};

void csr_from(int n, std::vector<Trip>& t, std::vector<int>& rows,
              std::vector<int>& cols, std::vector<double>& vals) {
  std::sort(t.begin(), t.end(), [](const Trip& a, const Trip& b) {
    return a.r != b.r ? a.r < b.r : a.c < b.c;
  });
  rows.assign(n + 1, 0);
  cols.clear();
  vals.clear();
  for (size_t i = 0; i < t.size();) {
    size_t j = i;
    double s = 0;
    while (j < t.size() && t[j].r == t[i].r && t[j].c == t[i].c) s += t[j++].v;
    cols.push_back(t[i].c);
    vals.push_back(s);
    rows[t[i].r + 1]++;
    i = j;
  }
  for (int i = 0; i < n; ++i) rows[i + 1] += rows[i];
}

// Connected components inside banks of 32 consecutive slots.  slot_of_node
// gives the slot of each member; edges are pairs of members.  Returns per slot
// the local CCO index (-1 for empty slots) and per bank the CCO count.
void bank_components(int nslots, const std::vector<char>& present,
                     const std::vector<std::pair<int, int>>& slot_edges,
                     std::vector<int>& slot_cco, std::vector<int>& bank_ncco) {
  std::vector<int> uf(nslots);
  std::iota(uf.begin(), uf.end(), 0);
  auto find = [&](int x) {
    while (uf[x] != x) x = uf[x] = uf[uf[x]];
    return x;
  };
  for (auto& [a, b] : slot_edges) {
    if (a / kBank != b / kBank) continue;
    int ra = find(a), rb = find(b);
    if (ra != rb) uf[std::max(ra, rb)] = std::min(ra, rb);
  }
  int nbank = nslots / kBank;
  slot_cco.assign(nslots, -1);
  bank_ncco.assign(nbank, 0);
  std::vector<int> lead_local(nslots, -1);
  for (int s = 0; s < nslots; ++s) {
    if (!present[s]) continue;
    int r = find(s);
    if (r == s) lead_local[s] = bank_ncco[s / kBank]++;
  }
  for (int s = 0; s < nslots; ++s)
    if (present[s]) slot_cco[s] = lead_local[find(s)];
}

}  // namespace

void build_cloth_setup(const float* verts, int nv, const int* faces, int nf,
                       const ClothParams& prm, ClothSetup& S) {
  S.nv = nv;
  S.nf = nf;
  std::vector<int> E_orig = mesh_edges(faces, nf);
  S.ne = (int)E_orig.size() / 2;
  S.avg_edge = average_edge_length(verts, E_orig);
  partition_mesh(verts, nv, faces, nf, S.perm, S.part_offsets);
  S.inv_perm.assign(nv, 0);
  for (int i = 0; i < nv; ++i) S.inv_perm[S.perm[i]] = i;
  S.F.resize(3 * (size_t)nf);
  for (size_t i = 0; i < S.F.size(); ++i) S.F[i] = S.perm[faces[i]];
  S.E.resize(E_orig.size());
  for (size_t i = 0; i < E_orig.size(); ++i) S.E[i] = S.perm[E_orig[i]];

  // Rest positions in solver order (double).
  std::vector<double> V(3 * (size_t)nv);
  for (int i = 0; i < nv; ++i)
    for (int d = 0; d < 3; ++d) V[3 * S.perm[i] + d] = verts[3 * i + d];

  // Voronoi mass, areas, cotangent Laplacian.
  S.voronoi.assign(nv, 0.0);
  S.area.assign(nf, 0.0);
  S.B.assign(6 * (size_t)nf, 0.0f);
  S.area_sqrt.assign(nf, 0.0f);
  std::vector<Trip> cot;
  std::vector<Trip> lt;  // k_e * area * B^T B
  cot.reserve(12 * (size_t)nf);
  lt.reserve(9 * (size_t)nf);
  for (int t = 0; t < nf; ++t) {
    int id[3] = {S.F[3 * t], S.F[3 * t + 1], S.F[3 * t + 2]};
    const double* p[3] = {&V[3 * id[0]], &V[3 * id[1]], &V[3 * id[2]]};
    double l2[3];
    for (int i = 0; i < 3; ++i) {
      const double* a = p[(i + 1) % 3];
      const double* b = p[(i + 2) % 3];
      l2[i] = (b[0] - a[0]) * (b[0] - a[0]) + (b[1] - a[1]) * (b[1] - a[1]) +
              (b[2] - a[2]) * (b[2] - a[2]);
    }
    double e0[3], e1[3];
    for (int d = 0; d < 3; ++d) {
      e0[d] = p[1][d] - p[0][d];
      e1[d] = p[2][d] - p[0][d];
    }
    double n[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                   e0[0] * e1[1] - e0[1] * e1[0]};
    double dbl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    double area = 0.5 * dbl;
    S.area[t] = area;
    S.area_sqrt[t] = (float)std::sqrt(area);
    double cotv[3];
    int obtuse = -1;
    for (int i = 0; i < 3; ++i) {
      double num = l2[(i + 1) % 3] + l2[(i + 2) % 3] - l2[i];
      cotv[i] = num / (4.0 * area);
      if (num < 0) obtuse = i;
    }
    for (int i = 0; i < 3; ++i) {
      int j = (i + 1) % 3, k = (i + 2) % 3;
      double m = obtuse < 0 ? 0.125 * (l2[k] * cotv[k] + l2[j] * cotv[j])
                            : (obtuse == i ? 0.5 * area : 0.25 * area);
      S.voronoi[id[i]] += m;
    }
    for (int i = 0; i < 3; ++i) {
      int a = id[(i + 1) % 3], b = id[(i + 2) % 3];
      double w = 0.5 * cotv[i];
      cot.push_back({a, b, w});
      cot.push_back({b, a, w});
      cot.push_back({a, a, -w});
      cot.push_back({b, b, -w});
    }
    // Chart operator B = (D dX^-1)^T (cloth_assembly_l2_cache.cpp:27-69).
    double l0 = std::sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
    double bx[3] = {e0[0] / l0, e0[1] / l0, e0[2] / l0};
    double by[3] = {n[1] * e0[2] - n[2] * e0[1], n[2] * e0[0] - n[0] * e0[2],
                    n[0] * e0[1] - n[1] * e0[0]};
    double lb = std::sqrt(by[0] * by[0] + by[1] * by[1] + by[2] * by[2]);
    for (int d = 0; d < 3; ++d) by[d] /= lb;
    double a = bx[0] * e0[0] + bx[1] * e0[1] + bx[2] * e0[2];
    double b = bx[0] * e1[0] + bx[1] * e1[1] + bx[2] * e1[2];
    double c = by[0] * e1[0] + by[1] * e1[1] + by[2] * e1[2];
    double Bm[2][3] = {{-1.0 / a, 1.0 / a, 0.0},
                       {b / (a * c) - 1.0 / c, -b / (a * c), 1.0 / c}};
    for (int r = 0; r < 2; ++r)
      for (int k = 0; k < 3; ++k) S.B[6 * t + 3 * r + k] = (float)Bm[r][k];
    for (int vi = 0; vi < 3; ++vi)
      for (int vj = 0; vj < 3; ++vj) {
        double s = Bm[0][vi] * Bm[0][vj] + Bm[1][vi] * Bm[1][vj];
        lt.push_back({id[vi], id[vj], prm.elastic_stiffness * area * s});
      }
  }
  std::vector<int> Cr, Cc;
  std::vector<double> Cv;
  csr_from(nv, cot, Cr, Cc, Cv);
  // CWC = C M^-1 C (C symmetric), scaled by k_b.
  std::vector<double> acc(nv, 0.0);
  std::vector<int> mark(nv, -1), touched;
  for (int i = 0; i < nv; ++i) {
    touched.clear();
    for (int x = Cr[i]; x < Cr[i + 1]; ++x) {
      int k = Cc[x];
      double inv_m = S.voronoi[k] > 0 ? 1.0 / S.voronoi[k] : 0.0;
      double cik = Cv[x] * inv_m;
      for (int y = Cr[k]; y < Cr[k + 1]; ++y) {
        int j = Cc[y];
        if (mark[j] != i) {
          mark[j] = i;
          acc[j] = 0.0;
          touched.push_back(j);
        }
        acc[j] += cik * Cv[y];
      }
    }
    for (int j : touched) lt.push_back({i, j, prm.bending_stiffness * acc[j]});
  }
  csr_from(nv, lt, S.Lrows, S.Lcols, S.Lvals);
  // Bending RHS = k_b CWC V: recompute from the bending part only.
  S.bending_rhs.assign(3 * (size_t)nv, 0.0);
  for (int i = 0; i < nv; ++i) {
    touched.clear();
    for (int x = Cr[i]; x < Cr[i + 1]; ++x) {
      int k = Cc[x];
      double inv_m = S.voronoi[k] > 0 ? 1.0 / S.voronoi[k] : 0.0;
      double cik = Cv[x] * inv_m;
      for (int y = Cr[k]; y < Cr[k + 1]; ++y) {
        int j = Cc[y];
        for (int d = 0; d < 3; ++d)
          S.bending_rhs[3 * i + d] += prm.bending_stiffness * cik * Cv[y] * V[3 * j + d];
      }
    }
  }
  S.mass.resize(nv);
  for (int i = 0; i < nv; ++i) S.mass[i] = prm.density * S.voronoi[i];
  // Vertex -> incident faces.
  S.vf_offsets.assign(nv + 1, 0);
  for (int t = 0; t < nf; ++t)
    for (int k = 0; k < 3; ++k) S.vf_offsets[S.F[3 * t + k] + 1]++;
  for (int i = 0; i < nv; ++i) S.vf_offsets[i + 1] += S.vf_offsets[i];
  S.vf_list.assign(S.vf_offsets[nv], 0);
  {
    std::vector<int> cur(S.vf_offsets.begin(), S.vf_offsets.end() - 1);
    for (int t = 0; t < nf; ++t)
      for (int k = 0; k < 3; ++k) S.vf_list[cur[S.F[3 * t + k]]++] = (t << 2) | k;
  }

  // ---------------- MAS hierarchy (mas_preconditioner.cu:99-478) ----------
  int nparts = (int)S.part_offsets.size() - 1;
  // Matrix graph edges between vertices (off-diagonal nnz of L).
  std::vector<std::pair<int, int>> vedges;
  for (int i = 0; i < nv; ++i)
    for (int x = S.Lrows[i]; x < S.Lrows[i + 1]; ++x)
      if (S.Lcols[x] != i) vedges.emplace_back(i, S.Lcols[x]);
  // Level 0: slots are padded vertex slots.
  std::vector<int> slot_of(nv);
  for (int p = 0; p < nparts; ++p)
    for (int v = S.part_offsets[p]; v < S.part_offsets[p + 1]; ++v)
      slot_of[v] = kBank * p + (v - S.part_offsets[p]);
  std::vector<int> node_of(nv);  // current level node (slot index space)
  for (int v = 0; v < nv; ++v) node_of[v] = slot_of[v];
  int nslots = nparts * kBank;
  int prev_count = -1;
  S.cmap.assign(4 * (size_t)nv, -1);
  std::vector<MasLevelPlan> plans;
  std::vector<std::vector<int>> maps;  // map per coarse space
  for (int lv = 0; lv <= kMaxCoarse; ++lv) {
    MasLevelPlan plan;
    plan.nbank = nslots / kBank;
    std::vector<char> present(nslots, 0);
    int count_present = 0;
    for (int v = 0; v < nv; ++v) present[node_of[v]] = 1;
    for (int s = 0; s < nslots; ++s) count_present += present[s];
    plan.nnode = lv == 0 ? nv : count_present;
    std::vector<std::pair<int, int>> sedges;
    sedges.reserve(vedges.size());
    for (auto& [a, b] : vedges) sedges.emplace_back(node_of[a], node_of[b]);
    bank_components(nslots, present, sedges, plan.slot_cco, plan.bank_ncco);
    plan.bank_cco_base.assign(plan.nbank, 0);
    int total = 0;
    for (int b = 0; b < plan.nbank; ++b) {
      plan.bank_cco_base[b] = total;
      total += plan.bank_ncco[b];
    }
    plans.push_back(plan);
    if ((int)maps.size() >= kMaxCoarse) break;
    if (lv > 0 && total == prev_count) {
      // No merge at this level: the next coarse space is not created.
      plans.back().slot_cco.assign(nslots, -1);
      break;
    }
    // Next coarse space: CCO ids.
    std::vector<int> m(nv);
    for (int v = 0; v < nv; ++v) {
      int s = node_of[v];
      m[v] = plan.bank_cco_base[s / kBank] + plan.slot_cco[s];
    }
    maps.push_back(m);
    node_of = m;
    prev_count = total;
    nslots = ((total + kBank - 1) / kBank) * kBank;
  }
  // A level exists for the fine banks and one per coarse space.
  S.levels = (int)maps.size();
  plans.resize(S.levels + 1);
  S.fine = plans[0];
  S.coarse.assign(plans.begin() + 1, plans.end());
  // The last matrix level has no next coarse space.
  if (!S.coarse.empty())
    S.coarse.back().slot_cco.assign(S.coarse.back().nbank * kBank, -1);
  else
    S.fine.slot_cco.assign(S.fine.nbank * kBank, -1);
  for (int k = 0; k < S.levels; ++k)
    for (int v = 0; v < nv; ++v) S.cmap[4 * v + k] = maps[k][v];

  // Galerkin operators G_k over coarse space k nodes and their gather plans.
  S.galerkin.assign(S.levels, {});
  for (int k = 0; k < S.levels; ++k) {
    auto& G = S.galerkin[k];
    const std::vector<int>& mk = maps[k];
    int n = 0;
    for (int v = 0; v < nv; ++v) n = std::max(n, mk[v] + 1);
    G.n = n;
    // Source entries: (row node, col node, source index).
    std::vector<std::tuple<int, int, int>> srcs;
    if (k == 0) {
      for (int i = 0; i < nv; ++i)
        for (int x = S.Lrows[i]; x < S.Lrows[i + 1]; ++x)
          srcs.emplace_back(mk[i], mk[S.Lcols[x]], x);
    } else {
      const auto& P = S.galerkin[k - 1];
      // Node map from coarse space k-1 to k.
      std::vector<int> up(P.n, -1);
      for (int v = 0; v < nv; ++v) up[maps[k - 1][v]] = mk[v];
      for (int a = 0; a < P.n; ++a)
        for (int x = P.rows[a]; x < P.rows[a + 1]; ++x)
          srcs.emplace_back(up[a], up[P.cols[x]], x);
    }
    std::sort(srcs.begin(), srcs.end());
    G.rows.assign(n + 1, 0);
    G.src_off.assign(1, 0);
    for (size_t i = 0; i < srcs.size();) {
      size_t j = i;
      while (j < srcs.size() && std::get<0>(srcs[j]) == std::get<0>(srcs[i]) &&
             std::get<1>(srcs[j]) == std::get<1>(srcs[i])) {
        G.src.push_back(std::get<2>(srcs[j]));
        ++j;
      }
      G.cols.push_back(std::get<1>(srcs[i]));
      G.rows[std::get<0>(srcs[i]) + 1]++;
      G.src_off.push_back((int)G.src.size());
      i = j;
    }
    for (int a = 0; a < n; ++a) G.rows[a + 1] += G.rows[a];
    // Dynamic diagonal only enters G_0 (higher levels aggregate it).
    G.diag_off.assign(G.cols.size() + 1, 0);
    if (k == 0) {
      std::vector<std::vector<int>> members(n);
      for (int v = 0; v < nv; ++v) members[mk[v]].push_back(v);
      for (int a = 0; a < n; ++a)
        for (int x = G.rows[a]; x < G.rows[a + 1]; ++x)
          if (G.cols[x] == a) {
            G.diag_off[x + 1] = (int)members[a].size();
          }
      for (size_t e = 0; e < G.cols.size(); ++e) G.diag_off[e + 1] += G.diag_off[e];
      G.diag.assign(G.diag_off.back(), 0);
      for (int a = 0; a < n; ++a)
        for (int x = G.rows[a]; x < G.rows[a + 1]; ++x)
          if (G.cols[x] == a) {
            int o = G.diag_off[x];
            for (int v : members[a]) G.diag[o++] = v;
          }
    }
  }
  // Bank fill plans: packed upper 528 entries per bank.
  const int NP = kBank * (kBank + 1) / 2;
  auto find_entry = [](const std::vector<int>& rows, const std::vector<int>& cols,
                       int a, int b) {
    auto beg = cols.begin() + rows[a], end = cols.begin() + rows[a + 1];
    auto it = std::lower_bound(beg, end, b);
    return (it != end && *it == b) ? (int)(it - cols.begin()) : -1;
  };
  S.fine.fill_src.assign((size_t)S.fine.nbank * NP, -1);
  for (int p = 0; p < nparts; ++p) {
    int base = S.part_offsets[p], size = S.part_offsets[p + 1] - base;
    for (int i = 0; i < size; ++i)
      for (int j = i; j < size; ++j)
        S.fine.fill_src[(size_t)p * NP + (i * kBank - i * (i + 1) / 2 + j)] =
            find_entry(S.Lrows, S.Lcols, base + i, base + j);
  }
  for (int l = 1; l <= S.levels; ++l) {
    auto& plan = S.coarse[l - 1];
    const auto& G = S.galerkin[l - 1];
    plan.fill_src.assign((size_t)plan.nbank * NP, -1);
    for (int b = 0; b < plan.nbank; ++b)
      for (int i = 0; i < kBank; ++i) {
        int a = kBank * b + i;
        if (a >= G.n) continue;
        for (int j = i; j < kBank; ++j) {
          int c = kBank * b + j;
          if (c >= G.n) continue;
          plan.fill_src[(size_t)b * NP + (i * kBank - i * (i + 1) / 2 + j)] =
              find_entry(G.rows, G.cols, a, c);
        }
      }
  }
}

void contact_weights(const ClothSetup& S, double dt, std::vector<double>& w) {
  w.assign(S.nv, 0.0);
  for (int i = 0; i < S.nv; ++i) {
    double lii = 0.0;
    for (int x = S.Lrows[i]; x < S.Lrows[i + 1]; ++x)
      if (S.Lcols[x] == i) lii = S.Lvals[x];
    double inertia = S.mass[i] / (dt * dt);
    double eta = lii + inertia;  // smallest eigenvalue of (L_ii + m/dt^2) I3
    w[i] = std::max(0.001 * eta, std::min(25.0 * inertia, eta));
  }
}

// Rows per bank (one per lane of a warp) of the resident CG's ELL slices.
constexpr int kSchedRows = 32;

// Order of the entries of one bank's rows in its ELL slice (round j of lane
// l at out[j * kSchedRows + l]).  In round j the 32 lanes of the warp gather p from
// shared memory (float4 per slot), and a 128-bit shared load is served per
// quarter-warp: two lanes of a quarter whose slots differ but share slot % 8
// (the 16-byte bank group) cost an extra pass.  Each quarter's entries are
// placed round by round, the lanes with the least slack first, each taking
// an entry whose bank group is still free in the round (or whose slot is
// already read, a broadcast), else an entry outside the block (a global
// load, no shared-memory access), else, when it has no slack left, any
// entry.  Padding entries (value 0) read a slot another lane of the quarter
// reads.  Entries outside the block have column >= 0; the kernel reads slot
// -1 - column otherwise.  A row's terms are summed in round order.
void schedule_bank_rows(const std::vector<std::vector<std::pair<int, int>>>& rows, int width,
                        int slot0, std::pair<int, int>* out) {
  for (int q = 0; q < kSchedRows / 8; ++q) {
    std::vector<std::vector<std::pair<int, int>>> rem(8);
    for (int l = 0; l < 8; ++l) rem[l] = rows[8 * q + l];
    for (int j = 0; j < width; ++j) {
      const int left = width - j;
      int order[8];
      for (int l = 0; l < 8; ++l) order[l] = l;
      std::stable_sort(order, order + 8, [&](int a, int b) {
        return left - (int)rem[a].size() < left - (int)rem[b].size();
      });
      int group_slot[8];  // slot read in this round per bank group, -1: free
      for (int g = 0; g < 8; ++g) group_slot[g] = -1;
      bool pad[8] = {false, false, false, false, false, false, false, false};
      for (int oi = 0; oi < 8; ++oi) {
        const int l = order[oi];
        auto& r = rem[l];
        if (r.empty()) {
          pad[l] = true;
          continue;
        }
        int pick = -1;
        for (int e = 0; e < (int)r.size() && pick < 0; ++e)
          if (r[e].first < 0) {
            int slot = -1 - r[e].first;
            int g = slot & 7;
            if (group_slot[g] < 0 || group_slot[g] == slot) pick = e;
          }
        if (pick < 0)
          for (int e = 0; e < (int)r.size() && pick < 0; ++e)
            if (r[e].first >= 0) pick = e;
        if (pick < 0 && (int)r.size() >= left) pick = 0;
        if (pick < 0) {
          pad[l] = true;
          continue;
        }
        std::pair<int, int> e = r[pick];
        r.erase(r.begin() + pick);
        if (e.first < 0) {
          int slot = -1 - e.first;
          if (group_slot[slot & 7] < 0) group_slot[slot & 7] = slot;
        }
        out[j * kSchedRows + 8 * q + l] = e;
      }
      for (int l = 0; l < 8; ++l) {
        if (!pad[l]) continue;
        int slot = slot0 + 8 * q + l;
        for (int g = 0; g < 8; ++g)
          if (group_slot[g] >= 0) {
            slot = group_slot[g];
            break;
          }
        if (group_slot[slot & 7] < 0) group_slot[slot & 7] = slot;
        out[j * kSchedRows + 8 * q + l] = std::make_pair(-1 - slot, 0);
      }
    }
  }
}

}  // namespace silkb
