// Host-side static setup of a cloth: mesh checks, vertex partition, assembly
// of the decoupled system matrix and the static plans of the MAS hierarchy.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace silkb {

struct ClothParams {
  float elastic_stiffness = 100.0f;
  float bending_stiffness = 1e-4f;
  float density = 0.1f;
  float damping = 0.01f;
};

// Checks of common/mesh.cpp:231-276 (cloth) and :278-303 (obstacle).
// Returns an empty string when valid, otherwise the reason.
// Sizes, finite positions and face indices in range (the part of the mesh
// checks every consumer of a face list needs); "" if valid.
std::string check_mesh_indices(const float* verts, long nverts_floats, const int* faces,
                               long nfaces_ints);
std::string check_cloth_mesh(const float* verts, long nverts_floats,
                             const int* faces, long nfaces_ints);
std::string check_obstacle_mesh(const float* verts, long nverts_floats,
                                const int* faces, long nfaces_ints);

// Unique undirected edges (i < j) sorted lexicographically.
std::vector<int> mesh_edges(const int* faces, int nf);
float average_edge_length(const float* verts, const std::vector<int>& edges);

// Vertex partition into connected parts of at most 32 vertices.
// perm: original -> solver id; part_offsets: CSR offsets in solver order.
void partition_mesh(const float* verts, int nv, const int* faces, int nf,
                    std::vector<int>& perm, std::vector<int>& part_offsets);

// One level of the multilevel additive Schwarz hierarchy.
struct MasLevelPlan {
  int nbank = 0;                 // banks of 32 slots at this level
  int nnode = 0;                 // real nodes (slots in use)
  std::vector<int> slot_cco;     // per slot: local CCO index or -1
  std::vector<int> bank_cco_base;  // per bank: first global CCO id
  std::vector<int> bank_ncco;      // per bank: CCO count
  // Bank matrix fill: per bank, 528 packed-upper entries; source index into
  // the level's Galerkin operator values (-1 = zero) -- coarse levels only.
  std::vector<int> fill_src;
};

// Static system of one cloth in solver order.
struct ClothSetup {
  int nv = 0, nf = 0, ne = 0;
  std::vector<int> perm, inv_perm, part_offsets;
  std::vector<int> F;  // 3 per face (solver ids, original face order)
  std::vector<int> E;  // 2 per edge (solver ids)
  float avg_edge = 0.0f;
  std::vector<double> voronoi;  // per vertex, no density
  std::vector<double> area;     // per face
  std::vector<float> B;         // 6 per face: rows of the 2x3 chart operator
  std::vector<float> area_sqrt;
  // Scalar matrix L (V x V) with H = L (x) I3; CSR including the diagonal.
  std::vector<int> Lrows, Lcols;
  std::vector<double> Lvals;
  std::vector<double> bending_rhs;  // 3 per vertex
  std::vector<double> mass;         // density * voronoi per vertex
  // Vertex -> incident face list (face << 2 | corner).
  std::vector<int> vf_offsets, vf_list;
  // MAS hierarchy.
  int levels = 0;                      // coarse levels
  std::vector<int> cmap;               // 4 per vertex: lv0..lv3 node (-1)
  MasLevelPlan fine;                   // level 0 (banks = parts)
  std::vector<MasLevelPlan> coarse;    // level l = 1..levels
  // Galerkin operators G_k over coarse-space-k nodes (k = 0..levels-1):
  // values gathered from L (k = 0) or G_{k-1}; CSR over nodes.
  struct Galerkin {
    int n = 0;
    std::vector<int> rows, cols;
    // Gather plan: entry e sums src[src_off[e]..src_off[e+1]) of the source
    // operator values, plus the dynamic diagonal of vertices in diag list.
    std::vector<int> src_off, src;
    std::vector<int> diag_off, diag;  // per entry (diagonal entries only)
  };
  std::vector<Galerkin> galerkin;
};

void build_cloth_setup(const float* verts, int nv, const int* faces, int nf,
                       const ClothParams& p, ClothSetup& out);

// Per-vertex contact weight (cloth_assembly_l1_cache.cu:58-75) for a dt.
void contact_weights(const ClothSetup& s, double dt, std::vector<double>& w);

// Entry order of one bank's 32 rows in the resident CG's ELL slice: out has
// width x 32 (column, value bits) pairs, round j of row l at out[j * 32 + l];
// a column < 0 is shared-memory slot -1 - column.  Rows no longer than width.
void schedule_bank_rows(const std::vector<std::vector<std::pair<int, int>>>& rows, int width,
                        int slot0, std::pair<int, int>* out);

}  // namespace silkb
