// Host orchestration of the per-step pipeline (reference:
// backend/cuda/cuda_backend.cu:31-352, main_loop.cu:24-278,
// admm_solver.cu:173-342, cloth_admm_helper.cu:306-347,
// assembly/cloth_assembler.cu:64-172, pin_constraints.cu:50-107).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>

#include <nvtx3/nvToolsExt.h>

#include "collision.cuh"
#include "world.hpp"
#include "learned.cuh"

namespace silkb {

namespace {
// Named host range for profiler timelines (nsys, ncu's NVTX filters); a
// cheap no-op when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

namespace {

std::vector<float4> to_float4(const std::vector<float>& v3, const std::vector<int>& perm) {
  int n = (int)perm.size();
  std::vector<float4> out(n);
  for (int i = 0; i < n; ++i)
    out[perm[i]] = make_float4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 0.f);
  return out;
}

}  // namespace

World::World() {
  silk_global_config_default(&g);
  silk_solver_options_default(&opt);
}

World::~World() {
  coll_.reset();
  for (auto* pool : {&events, &events_other, &events_gs})
    for (auto& e : *pool) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  for (cudaStream_t cs : cloth_streams_) cudaStreamDestroy(cs);
  for (cudaEvent_t e : cloth_done_) cudaEventDestroy(e);
  if (fork_ev_) cudaEventDestroy(fork_ev_);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

void World::ensure_stream() {
  if (!stream) {
    CUDA_CHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
}

void World::sync() { CUDA_CHECK(cudaStreamSynchronize(stream)); }

void World::ensure_cloth_streams(size_t n) {
  if (!fork_ev_) CUDA_CHECK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
  while (cloth_streams_.size() < n) {
    cudaStream_t s;
    cudaEvent_t e;
    CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cloth_streams_.push_back(s);
    cloth_done_.push_back(e);
  }
}

silk_status World::init(int backend) {
  if (backend != SILK_BACKEND_GPU) {
    last_error = "only the GPU backend is provided";
    return SILK_ERR_INVALID_CONFIG;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    last_error = "CUDA runtime/device not available";
    return SILK_ERR_NO_CUDA_SUPPORT;
  }
  CUDA_CHECK(cudaGetDevice(&device));
  ensure_stream();
  if (!coll_) coll_ = std::make_unique<CollisionSystem>(*this);
  initialized = true;
  return SILK_OK;
}

silk_status World::set_global_config(const silk_global_config& c) {
  if (c.dt != g.dt) invalidate_layout();
  g = c;
  return SILK_OK;
}

void World::clear() {
  if (stream) cudaStreamSynchronize(stream);
  coll_.reset();
  cloths.clear();
  obstacles.clear();
  initialized = false;
  layout_valid_ = false;
  nv_total = nf_total = 0;
}

silk_status World::set_solver_options(const silk_solver_options& o) {
  // The CG launch form is chosen when the solver layout is built.
  if (o.cg_form != opt.cg_form || o.resident_halo_limit != opt.resident_halo_limit)
    invalidate_layout();
  opt = o;
  if (opt.cg_max_iter <= 0) opt.cg_max_iter = 1000;
  return SILK_OK;
}

silk_status World::set_stream(void* s) {
  if (stream) cudaStreamSynchronize(stream);
  if (own_stream && stream) cudaStreamDestroy(stream);
  own_stream = false;
  stream = (cudaStream_t)s;
  if (!stream) ensure_stream();
  return SILK_OK;
}

Cloth* World::find_cloth(uint32_t h) {
  for (auto& c : cloths)
    if (c->handle == h) return c.get();
  return nullptr;
}

Obstacle* World::find_obstacle(uint32_t h) {
  for (auto& o : obstacles)
    if (o->handle == h) return o.get();
  return nullptr;
}

void World::invalidate_layout() {
  if (!layout_valid_) return;
  // Keep the simulated states on the host while the layout is rebuilt.
  sync();
  for (auto& c : cloths) {
    if (!c->on_device) continue;
    int nv = c->nv();
    std::vector<float4> xs(nv), vs(nv);
    CUDA_CHECK(cudaMemcpy(xs.data(), sx.p + c->voff, nv * sizeof(float4),
                          cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(vs.data(), sv.p + c->voff, nv * sizeof(float4),
                          cudaMemcpyDeviceToHost));
    c->x_host.resize(3 * nv);
    c->v_host.resize(3 * nv);
    for (int i = 0; i < nv; ++i) {
      int s = c->setup->perm[i];
      c->x_host[3 * i] = xs[s].x;
      c->x_host[3 * i + 1] = xs[s].y;
      c->x_host[3 * i + 2] = xs[s].z;
      c->v_host[3 * i] = vs[s].x;
      c->v_host[3 * i + 1] = vs[s].y;
      c->v_host[3 * i + 2] = vs[s].z;
    }
    c->on_device = false;
  }
  layout_valid_ = false;
}

silk_status World::solver_reset() {
  if (stream) sync();
  for (auto& c : cloths) {
    c->x_host = c->rest;
    c->v_host.assign(c->rest.size(), 0.0f);
    c->on_device = false;
    c->pin_pos.clear();
    for (int p : c->pins)
      for (int d = 0; d < 3; ++d) c->pin_pos.push_back(c->rest[3 * p + d]);
  }
  for (auto& o : obstacles) {
    o->is_static = true;
    o->is_static_twice = true;
  }
  layout_valid_ = false;
  return SILK_OK;
}

silk_status World::add_cloth(const silk_cloth_config& cc,
                             const silk_collision_config& col, const float* v,
                             int64_t nvf, const int* f, int64_t nfi,
                             const int* pins, int64_t npins, uint32_t* handle) {
  if (handle) *handle = 0;
  std::string why = check_cloth_mesh(v, nvf, f, nfi);
  if (!why.empty()) {
    last_error = why;
    return SILK_ERR_INVALID_MESH;
  }
  int nv = (int)(nvf / 3);
  if (npins > nv || (npins > 0 && pins == nullptr)) {
    last_error = "too many pins";
    return SILK_ERR_INVALID_PIN;
  }
  for (int64_t i = 0; i < npins; ++i)
    if (pins[i] < 0 || pins[i] >= nv) {
      last_error = "pin index out of range";
      return SILK_ERR_INVALID_PIN;
    }
  invalidate_layout();
  auto c = std::make_unique<Cloth>();
  c->handle = next_handle_++;
  c->cfg = cc;
  c->coll = col;
  c->rest.assign(v, v + nvf);
  c->faces.assign(f, f + nfi);
  c->pins.assign(pins, pins + npins);
  for (int p : c->pins)
    for (int d = 0; d < 3; ++d) c->pin_pos.push_back(c->rest[3 * p + d]);
  c->x_host = c->rest;
  c->v_host.assign(c->rest.size(), 0.0f);
  *handle = c->handle;
  cloths.push_back(std::move(c));
  return SILK_OK;
}

silk_status World::remove_cloth(uint32_t h) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  invalidate_layout();
  cloths.erase(std::remove_if(cloths.begin(), cloths.end(),
                              [h](auto& p) { return p->handle == h; }),
               cloths.end());
  return SILK_OK;
}

silk_status World::get_cloth_position(uint32_t h, float* out, int64_t n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  int nv = c->nv();
  if (n != 3 * (int64_t)nv) return SILK_ERR_INVALID_POSITION;
  if (!c->on_device) {
    std::memcpy(out, c->x_host.data(), sizeof(float) * 3 * nv);
    return SILK_OK;
  }
  std::vector<float4> xs(nv);
  CUDA_CHECK(cudaMemcpyAsync(xs.data(), sx.p + c->voff, nv * sizeof(float4),
                             cudaMemcpyDeviceToHost, stream));
  sync();
  const auto& perm = c->setup->perm;
  for (int i = 0; i < nv; ++i) {
    float4 q = xs[perm[i]];
    out[3 * i] = q.x;
    out[3 * i + 1] = q.y;
    out[3 * i + 2] = q.z;
  }
  return SILK_OK;
}

// Restart a cloth from a stored state.  The state between steps is exactly
// the positions and velocities: contacts are rebuilt by DCD and the ADMM
// variables reset at the start of every step (main_loop.cu:140-176).  The
// warm-start feature history becomes the positions one and two steps back
// along the given velocity.
silk_status World::set_cloth_state(uint32_t h, const float* xin, int64_t nx,
                                   const float* vin, int64_t nvel) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  const int nv = c->nv();
  if (!xin || nx != 3 * (int64_t)nv || (vin && nvel != 3 * (int64_t)nv))
    return SILK_ERR_INVALID_POSITION;
  for (int64_t i = 0; i < nx; ++i)
    if (!std::isfinite(xin[i]) || (vin && !std::isfinite(vin[i]))) {
      last_error = "non-finite state";
      return SILK_ERR_INVALID_POSITION;
    }
  ensure_layout();
  std::vector<float4> xs(nv), vs(nv), h1(nv), h2(nv);
  const auto& perm = c->setup->perm;
  const float dt = g.dt;
  for (int i = 0; i < nv; ++i) {
    float px = xin[3 * i], py = xin[3 * i + 1], pz = xin[3 * i + 2];
    float vx = vin ? vin[3 * i] : 0.f, vy = vin ? vin[3 * i + 1] : 0.f,
          vz = vin ? vin[3 * i + 2] : 0.f;
    int s = perm[i];
    xs[s] = make_float4(px, py, pz, 0.f);
    vs[s] = make_float4(vx, vy, vz, 0.f);
    h1[s] = make_float4(px - dt * vx, py - dt * vy, pz - dt * vz, 0.f);
    h2[s] = make_float4(px - 2.f * dt * vx, py - 2.f * dt * vy, pz - 2.f * dt * vz, 0.f);
  }
  const size_t bytes = nv * sizeof(float4);
  CUDA_CHECK(cudaMemcpyAsync(sx.p + c->voff, xs.data(), bytes, cudaMemcpyHostToDevice, stream));
  CUDA_CHECK(cudaMemcpyAsync(sv.p + c->voff, vs.data(), bytes, cudaMemcpyHostToDevice, stream));
  CUDA_CHECK(cudaMemcpyAsync(hist1.p + c->voff, h1.data(), bytes, cudaMemcpyHostToDevice, stream));
  CUDA_CHECK(cudaMemcpyAsync(hist2.p + c->voff, h2.data(), bytes, cudaMemcpyHostToDevice, stream));
  sync();
  return SILK_OK;
}

silk_status World::set_cloth_config(uint32_t h, const silk_cloth_config& cfg) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  invalidate_layout();
  c->cfg = cfg;
  c->setup_valid = false;
  return SILK_OK;
}

silk_status World::set_cloth_collision_config(uint32_t h,
                                              const silk_collision_config& col) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  invalidate_layout();
  c->coll = col;
  return SILK_OK;
}

silk_status World::set_cloth_pin_index(uint32_t h, const int* pins, int64_t n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  for (int64_t i = 0; i < n; ++i)
    if (pins[i] < 0 || pins[i] >= c->nv()) return SILK_ERR_INVALID_PIN;
  invalidate_layout();
  c->pins.assign(pins, pins + n);
  // PinPosition is rebuilt from the initial vertices (cloth_assembler.cu:79).
  c->pin_pos.clear();
  for (int p : c->pins)
    for (int d = 0; d < 3; ++d) c->pin_pos.push_back(c->rest[3 * p + d]);
  return SILK_OK;
}

silk_status World::set_cloth_pin_position(uint32_t h, const float* pos,
                                          int64_t n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  if (n != 3 * (int64_t)c->pins.size()) return SILK_ERR_INVALID_PIN;
  c->pin_pos.assign(pos, pos + n);
  pins_dirty_ = true;
  return SILK_OK;
}

silk_status World::add_obstacle(const silk_collision_config& col,
                                const float* v, int64_t nvf, const int* f,
                                int64_t nfi, uint32_t* handle) {
  if (handle) *handle = 0;
  std::string why = check_obstacle_mesh(v, nvf, f, nfi);
  if (!why.empty()) {
    last_error = why;
    return SILK_ERR_INVALID_MESH;
  }
  invalidate_layout();
  auto o = std::make_unique<Obstacle>();
  o->handle = next_handle_++;
  o->coll = col;
  o->cur.assign(v, v + nvf);
  o->prev = o->cur;
  if (nfi > 0) o->faces.assign(f, f + nfi);
  *handle = o->handle;
  obstacles.push_back(std::move(o));
  return SILK_OK;
}

silk_status World::remove_obstacle(uint32_t h) {
  if (!find_obstacle(h)) return SILK_ERR_INVALID_HANDLE;
  invalidate_layout();
  obstacles.erase(std::remove_if(obstacles.begin(), obstacles.end(),
                                 [h](auto& p) { return p->handle == h; }),
                  obstacles.end());
  return SILK_OK;
}

silk_status World::set_obstacle_collision_config(uint32_t h,
                                                 const silk_collision_config& c) {
  Obstacle* o = find_obstacle(h);
  if (!o) return SILK_ERR_INVALID_HANDLE;
  invalidate_layout();
  o->coll = c;
  return SILK_OK;
}

silk_status World::set_obstacle_position(uint32_t h, const float* pos,
                                         int64_t n) {
  Obstacle* o = find_obstacle(h);
  if (!o) return SILK_ERR_INVALID_HANDLE;
  if (n != (int64_t)o->cur.size()) return SILK_ERR_INVALID_POSITION;
  // cuda_backend.cu:323-344: the previous target becomes the start of the
  // obstacle motion over the next step.
  o->is_static = false;
  o->is_static_twice = false;
  std::swap(o->cur, o->prev);
  o->cur.assign(pos, pos + n);
  o->positions_dirty = true;
  return SILK_OK;
}

SolverView World::view() {
  SolverView s;
  s.nv = nv_total;
  s.nf = nf_total;
  s.dt = g.dt;
  s.acc = make_float4(g.acceleration_x, g.acceleration_y, g.acceleration_z, 0.f);
  s.x = x.p;
  s.prev = sx.p;
  s.prev_v = prev_v.p;
  s.mass = mass.p;
  s.bending_rhs = bending_rhs.p;
  s.faces = faces_d.p;
  s.B0 = B0.p;
  s.B1 = B1.p;
  s.zu = zu.p;
  s.zold = zold.p;
  s.vf_off = vf_off.p;
  s.vf_list = vf_list.p;
  s.pin_flag = pin_flag.p;
  s.pin_target = pin_target.p;
  s.pin_lambda = pin_lambda.p;
  s.contact_w = contact_w.p;
  s.contact_p = contact_p.p;
  s.contact_p_prev = contact_p_prev.p;
  s.contact_eta = contact_eta.p;
  s.lhs = lhs.p;
  s.rhs = rhs.p;
  s.inertia = inertia.p;
  return s;
}

// Per-cloth static device data: sliced-ELL off-diagonal L, MAS plans.
// Resident CG layout (cg_resident_kernel): block k owns fine banks
// 32k .. 32k+31 with thread 32 w + lane on slot `lane` of fine bank 32k + w.
// Possible when every fine bank is one coarse node (parts are connected), so
// that first-level coarse bank k is exactly this group, and the coarse levels
// above fit the shared memory of a block.  The off-diagonal part of L is
// re-sliced per fine bank; a column inside the block is stored as -1 - slot,
// and the entries from other blocks come first in each row.
namespace {

// Per-fine-bank ELL slices of the off-diagonal rows of L for CTAs of `bpb`
// fine banks: a column inside the CTA is its shared-memory slot
// (bank within the CTA * 32 + lane), a column outside it the next free halo
// slot bpb * 32 + i (at most halo_cap halo vertices per CTA; further columns
// stay global vertex indices and halo_full becomes false), entries ordered
// by schedule_bank_rows.
struct BlockLayout {
  std::vector<int> ptr, width, halo_off, halo_col;
  std::vector<int2> ent;
  bool halo_full = true;
};

BlockLayout block_layout(const ClothSetup& S, int bpb, int halo_cap) {
  BlockLayout L;
  const int nbank0 = S.fine.nbank;
  const int nblocks = div_up(nbank0, bpb);
  const int nthreads = bpb * BANK;
  const int nv = S.nv;
  std::vector<int> part_of(nv), lane_of(nv);
  for (int b = 0; b < nbank0; ++b)
    for (int v = S.part_offsets[b]; v < S.part_offsets[b + 1]; ++v) {
      part_of[v] = b;
      lane_of[v] = v - S.part_offsets[b];
    }
  L.ptr.assign(nbank0 + 1, 0);
  L.width.assign(nbank0, 0);
  for (int b = 0; b < nbank0; ++b) {
    int w = 0;
    for (int v = S.part_offsets[b]; v < S.part_offsets[b + 1]; ++v)
      w = std::max(w, S.Lrows[v + 1] - S.Lrows[v] - 1);
    L.width[b] = w;
    L.ptr[b + 1] = L.ptr[b] + BANK * w;
  }
  L.halo_off.assign(nblocks + 1, 0);
  std::vector<int> halo_slot(nv, -1), halo_mark(nv, -1);
  for (int k = 0; k < nblocks; ++k) {
    L.halo_off[k] = (int)L.halo_col.size();
    for (int bb = k * bpb; bb < std::min(nbank0, (k + 1) * bpb); ++bb)
      for (int v = S.part_offsets[bb]; v < S.part_offsets[bb + 1]; ++v)
        for (int q = S.Lrows[v]; q < S.Lrows[v + 1]; ++q) {
          int col = S.Lcols[q];
          if (part_of[col] / bpb == k || halo_mark[col] == k) continue;
          if ((int)L.halo_col.size() - L.halo_off[k] >= halo_cap) {
            L.halo_full = false;
            continue;
          }
          halo_mark[col] = k;
          L.halo_col.push_back(col);
        }
  }
  L.halo_off[nblocks] = (int)L.halo_col.size();
  L.ent.assign(std::max(L.ptr[nbank0], 1), make_int2(0, 0));
  std::vector<std::vector<std::pair<int, int>>> row(BANK);
  std::vector<std::pair<int, int>> sched;
  int halo_block = -1;
  for (int b = 0; b < nbank0; ++b) {
    const int k = b / bpb;
    if (k != halo_block) {
      if (halo_block >= 0)
        for (int i = L.halo_off[halo_block]; i < L.halo_off[halo_block + 1]; ++i)
          halo_slot[L.halo_col[i]] = -1;
      for (int i = L.halo_off[k]; i < L.halo_off[k + 1]; ++i)
        halo_slot[L.halo_col[i]] = nthreads + i - L.halo_off[k];
      halo_block = k;
    }
    for (int lane = 0; lane < BANK; ++lane) {
      row[lane].clear();
      const int v = S.part_offsets[b] + lane;
      if (v >= S.part_offsets[b + 1]) continue;
      for (int q = S.Lrows[v]; q < S.Lrows[v + 1]; ++q) {
        int col = S.Lcols[q];
        if (col == v) continue;
        float val = (float)S.Lvals[q];
        int bits;
        std::memcpy(&bits, &val, 4);
        int cb = part_of[col];
        if (cb / bpb == k)
          row[lane].emplace_back(-1 - ((cb - k * bpb) * BANK + lane_of[col]), bits);
        else if (halo_slot[col] >= 0)
          row[lane].emplace_back(-1 - halo_slot[col], bits);
        else
          row[lane].emplace_back(col, bits);
      }
    }
    sched.resize((size_t)BANK * L.width[b]);
    schedule_bank_rows(row, L.width[b], (b - k * bpb) * BANK, sched.data());
    for (size_t i = 0; i < sched.size(); ++i)
      L.ent[L.ptr[b] + i] = make_int2(sched[i].first, sched[i].second);
  }
  if (L.halo_col.empty()) L.halo_col.push_back(0);
  return L;
}

// Row store of the cluster and resident CG forms in tensor memory: the
// bpb / 4 warps of a CTA that share a 32-lane quarter of it each hold their
// bank's rows in 2 tm_rw columns (two per entry, the widest bank's entries
// rounded up to 8); the allocation is the next power of two, at most the
// 512 columns of an SM.  Off (cg_form 3 and 4): rows read from global memory.
void set_row_store(ClothDev& d, const BlockLayout& L, int bpb, bool on) {
  int wmax = 0;
  for (int wd : L.width) wmax = std::max(wmax, wd);
  const int rwpad = std::max(8, div_up(wmax, 8) * 8);
  int cols = 32;
  while (cols < (bpb / 4) * 2 * rwpad) cols *= 2;
  d.tm_rw = rwpad;
  d.tm_cols = on && cols <= 512 ? cols : 0;
}

}  // namespace

// Launch form of the cloth's CG solve, chosen when its layout is built:
//  1. the cluster form with redundant coarse levels (CTAs of 8 or 16 fine
//     banks, one cluster of at most 16 CTAs, every coarse bank held by every
//     CTA, every off-CTA column in the CTA's halo);
//  2. the resident form (one CTA per first-level coarse bank, a cluster of up
//     to 16 or a cooperative grid);
//  3. otherwise the streaming form.
// Forms 1 and 2 need every fine bank to be one first-level coarse node.
// solver option cg_form: 0 all forms, 2 forms 2 and 3, 1 form 3 only; 3 and
// 4 as 0 and 2 with forms 1 and 2 reading their matrix rows from global
// memory in every SpMV instead of holding them in tensor memory.
void World::build_resident_layout(Cloth& c) {
  const ClothSetup& S = *c.setup;
  ClothDev& d = c.dev;
  d.res_blocks = 0;
  d.res_grid = 0;
  d.dsm_ctas = 0;
  d.dsm_f = 0;
  d.tm_cols = 0;
  d.tm_rw = 0;
  const int nbank0 = S.fine.nbank;
  const int nblocks = div_up(nbank0, BANK);
  int upper = 0, all_coarse = 0;
  if (S.levels > 0) {
    for (int b = 0; b < nbank0; ++b)
      if (S.fine.bank_ncco[b] != 1 || S.fine.bank_cco_base[b] != b) return;
    if (S.coarse[0].nbank != nblocks) return;
    for (int l = 1; l <= S.levels; ++l) {
      all_coarse += S.coarse[l - 1].nbank;
      if (l >= 2) upper += S.coarse[l - 1].nbank;
    }
  }
  if (opt.cg_form == 1) return;
  cudaStream_t st = stream;
  auto upload = [&](const BlockLayout& L) {
    d.rb_ptr.upload(L.ptr, st);
    d.rb_w.upload(L.width, st);
    d.rent.upload(L.ent, st);
    d.res_halo_off.upload(L.halo_off, st);
    d.res_halo_full = L.halo_full;
    d.res_halo_col.upload(L.halo_col, st);
  };
  if ((opt.cg_form == 0 || opt.cg_form == 3) && S.levels > 0 &&
      all_coarse <= kDsmCoarseBankLimit) {
    for (int f : {8, 16}) {
      const int n = cg_dsm_ctas(nbank0, f);
      if (n == 0) continue;
      BlockLayout L = block_layout(S, f, BANK * f);
      if (!L.halo_full) continue;
      // Pushes of fine-level z: each halo vertex of CTA k is stored by its
      // owner into slot i of k's halo (entry: own slot | k << 10 | i << 15).
      std::vector<std::vector<int>> pushes(n);
      for (int k = 0; k < n; ++k)
        for (int i = L.halo_off[k]; i < L.halo_off[k + 1]; ++i) {
          const int col = L.halo_col[i];
          int b = (int)(std::upper_bound(S.part_offsets.begin(), S.part_offsets.end(), col) -
                        S.part_offsets.begin()) - 1;
          const int owner = b / f;
          const int slot = (b - owner * f) * BANK + (col - S.part_offsets[b]);
          pushes[owner].push_back(slot | (k << 10) | ((i - L.halo_off[k]) << 15));
        }
      bool fits = true;
      std::vector<int> poff(1, 0), plist;
      for (auto& v : pushes) {
        if ((int)v.size() > kDsmPushPerThread * BANK * f) fits = false;
        plist.insert(plist.end(), v.begin(), v.end());
        poff.push_back((int)plist.size());
      }
      if (!fits) continue;
      if (plist.empty()) plist.push_back(0);
      upload(L);
      d.dsm_push_off.upload(poff, st);
      d.dsm_push.upload(plist, st);
      d.dsm_ctas = n;
      d.dsm_f = f;
      set_row_store(d, L, f, opt.cg_form == 0);
      return;
    }
  }
  if (S.levels > 0 && upper > kResCoarseBanks) return;
  int grid = cg_resident_grid(nblocks);
  if (grid == 0) return;
  const int halo_cap = opt.resident_halo_limit > 0 ? std::min(opt.resident_halo_limit, kResHalo)
                                                   : kResHalo;
  const BlockLayout L = block_layout(S, BANK, halo_cap);
  upload(L);
  set_row_store(d, L, BANK, opt.cg_form == 0 || opt.cg_form == 2);
  d.res_blocks = nblocks;
  d.res_grid = grid;
}

void World::build_cloth_device(Cloth& c) {
  const ClothSetup& S = *c.setup;
  ClothDev& d = c.dev;
  cudaStream_t st = stream;
  int nv = S.nv;
  // Sliced ELL of the off-diagonal part, 32 rows per slice.
  int nsl = div_up(nv, 32);
  std::vector<int> sl_ptr(nsl + 1, 0), sl_w(nsl, 0);
  std::vector<float> ldiag(nv, 0.f);
  for (int s = 0; s < nsl; ++s) {
    int w = 0;
    for (int r = 32 * s; r < std::min(nv, 32 * s + 32); ++r) {
      int cnt = 0;
      for (int k = S.Lrows[r]; k < S.Lrows[r + 1]; ++k)
        if (S.Lcols[k] != r) ++cnt;
      w = std::max(w, cnt);
    }
    sl_w[s] = w;
    sl_ptr[s + 1] = sl_ptr[s] + 32 * w;
  }
  std::vector<int2> ent(sl_ptr[nsl]);
  for (int s = 0; s < nsl; ++s)
    for (int lane = 0; lane < 32; ++lane) {
      int r = 32 * s + lane;
      int k = 0;
      if (r < nv) {
        for (int q = S.Lrows[r]; q < S.Lrows[r + 1]; ++q) {
          if (S.Lcols[q] == r) {
            ldiag[r] = (float)S.Lvals[q];
            continue;
          }
          float val = (float)S.Lvals[q];
          int bits;
          std::memcpy(&bits, &val, 4);
          ent[sl_ptr[s] + k * 32 + lane] = make_int2(S.Lcols[q], bits);
          ++k;
        }
      }
      for (; k < sl_w[s]; ++k)
        ent[sl_ptr[s] + k * 32 + lane] = make_int2(r < nv ? r : 0, 0);
    }
  d.sl_ptr.upload(sl_ptr, st);
  d.sl_w.upload(sl_w, st);
  d.ent.upload(ent, st);
  build_resident_layout(c);
  d.Ldiag.upload(ldiag, st);
  d.Lvals.upload(S.Lvals, st);
  d.part_off.upload(S.part_offsets, st);
  std::vector<int4> cm(nv);
  for (int v = 0; v < nv; ++v)
    cm[v] = make_int4(S.cmap[4 * v], S.cmap[4 * v + 1], S.cmap[4 * v + 2],
                      S.cmap[4 * v + 3]);
  d.cmap.upload(cm, st);
  auto upload_level = [&](const MasLevelPlan& P, ClothDev::Level& L, int nnode,
                          int nrout) {
    L.fill_src.upload(P.fill_src, st);
    std::vector<signed char> sc(P.slot_cco.size());
    for (size_t i = 0; i < sc.size(); ++i) sc[i] = (signed char)P.slot_cco[i];
    L.slot_cco.upload(sc, st);
    L.cco_base.upload(P.bank_cco_base, st);
    L.ncco.upload(P.bank_ncco, st);
    L.M.alloc((size_t)P.nbank * kPacked);
    L.Mb.alloc((size_t)P.nbank * kPacked);
    if (nnode > 0) {
      L.zout.alloc(nnode);
      L.zout.zero(st);
    }
    if (nrout > 0) {
      L.rout.alloc(nrout);
      L.rout.zero(st);
    }
  };
  int n0 = S.levels > 0 ? S.galerkin[0].n : 0;
  upload_level(S.fine, d.fine, 0, S.levels > 0 ? n0 : 0);
  d.coarse.clear();
  d.coarse.resize(S.levels);
  for (int l = 1; l <= S.levels; ++l) {
    int nnode = S.galerkin[l - 1].n;
    int nnext = l < S.levels ? S.galerkin[l].n : 0;
    upload_level(S.coarse[l - 1], d.coarse[l - 1], nnode, nnext);
    if (l >= 2) {
      // Members of each node of this level: the slots of the level below
      // whose connected component it is, in slot order.
      const MasLevelPlan& below = S.coarse[l - 2];
      std::vector<std::vector<int>> mem(nnode);
      for (int g = 0; g < below.nbank; ++g)
        for (int j = 0; j < BANK; ++j) {
          const int c = below.slot_cco[(size_t)g * BANK + j];
          if (c < 0) continue;
          const int node = below.bank_cco_base[g] + c;
          if (node >= 0 && node < nnode) mem[node].push_back(g * BANK + j);
        }
      std::vector<int> off(1, 0), list;
      for (auto& m : mem) {
        list.insert(list.end(), m.begin(), m.end());
        off.push_back((int)list.size());
      }
      if (list.empty()) list.push_back(0);
      d.coarse[l - 1].member_off.upload(off, st);
      d.coarse[l - 1].member.upload(list, st);
    }
  }
  d.gal.clear();
  d.gal.resize(S.levels);
  for (int k = 0; k < S.levels; ++k) {
    const auto& G = S.galerkin[k];
    d.gal[k].src_off.upload(G.src_off, st);
    d.gal[k].src.upload(G.src, st);
    if (k == 0) {
      d.gal[k].diag_off.upload(G.diag_off, st);
      d.gal[k].diag.upload(G.diag, st);
    }
    d.gal[k].vals.alloc(G.cols.size());
  }
  d.r.alloc(nv);
  d.z0.alloc(nv);
  d.p.alloc(nv);
  d.Ap.alloc(nv);
  d.p.zero(st);
  int nbank0 = S.fine.nbank;
  // Negative: one thread-block cluster of that many CTAs.
  d.cg_grid = cg_grid_size(nsl, nbank0);
  d.partials.alloc(4 * (size_t)std::max(std::abs(d.cg_grid), d.res_blocks));
  d.coarse_partial.alloc(1);
  d.barrier.alloc(4);
  d.barrier.zero(st);
  d.result.alloc(2);
  d.result_rr.alloc(1);
  d.stats.alloc(kCgStats);
  d.stats.zero(st);
  // Compulsory DRAM bytes of one CG iteration: off-diagonal entries (8 B),
  // per row Ldiag + dynamic diagonal + p read + Ap write (40 B) in the SpMV
  // phase, r/p/Ap/x read + x/r/z0 write (112 B) in the fine MAS phase, z0/p/
  // cmap read + p write (64 B) in the prolongation, plus every bank inverse.
  {
    long nnz_off = (long)S.Lcols.size() - nv;
    long banks = S.fine.nbank;
    for (auto& c : S.coarse) banks += c.nbank;
    double base = 8.0 * nnz_off + 216.0 * nv;
    d.bytes_per_iter_fp32 = base + (double)banks * kPacked * 4.0;
    d.bytes_per_iter_bf16 = base + (double)banks * kPacked * 2.0;
  }
  // CG argument template (vectors are bound per solve).
  CgArgs& a = d.cg;
  a = CgArgs{};
  a.nv = nv;
  a.nslices = nsl;
  a.sl_ptr = d.sl_ptr.p;
  a.sl_w = d.sl_w.p;
  a.ent = d.ent.p;
  a.Ldiag = d.Ldiag.p;
  a.r = d.r.p;
  a.z0 = d.z0.p;
  a.p = d.p.p;
  a.Ap = d.Ap.p;
  a.cmap = d.cmap.p;
  a.nbank0 = nbank0;
  a.part_off = d.part_off.p;
  auto lv_dev = [&](const MasLevelPlan& P, ClothDev::Level& L, int nnode,
                    float4* rin) {
    MasLevelDev m;
    m.nbank = P.nbank;
    m.nnode = nnode;
    m.fill_src = L.fill_src.p;
    m.slot_cco = L.slot_cco.p;
    m.cco_base = L.cco_base.p;
    m.ncco = L.ncco.p;
    m.M = L.M.p;
    m.Mb = L.Mb.p;
    m.rin = rin;
    m.zout = L.zout.p;
    m.rout = L.rout.p;
    m.member_off = L.member_off.p;
    m.member = L.member.p;
    return m;
  };
  a.fine = lv_dev(S.fine, d.fine, nv, nullptr);
  a.levels = S.levels;
  for (int l = 1; l <= S.levels; ++l) {
    float4* rin = l == 1 ? d.fine.rout.p : d.coarse[l - 2].rout.p;
    a.coarse[l - 1] = lv_dev(S.coarse[l - 1], d.coarse[l - 1],
                             S.galerkin[l - 1].n, rin);
  }
  if (d.dsm_ctas > 0) {
    a.dsm_f = d.dsm_f;
    a.push_off = d.dsm_push_off.p;
    a.push = d.dsm_push.p;
    a.rb_ptr = d.rb_ptr.p;
    a.rb_w = d.rb_w.p;
    a.rent = d.rent.p;
    a.halo_off = d.res_halo_off.p;
    a.halo_col = d.res_halo_col.p;
    a.halo_full = 1;
  }
  a.tm_cols = d.tm_cols;
  a.tm_rw = d.tm_rw;
  if (d.res_grid != 0) {
    a.res_blocks = d.res_blocks;
    a.rb_ptr = d.rb_ptr.p;
    a.rb_w = d.rb_w.p;
    a.rent = d.rent.p;
    a.halo_off = d.res_halo_off.p;
    a.halo_col = d.res_halo_col.p;
    a.halo_full = d.res_halo_full ? 1 : 0;
  }
  a.partials = d.partials.p;
  a.coarse_partial = d.coarse_partial.p;
  a.barrier = d.barrier.p;
  a.result = d.result.p;
  a.result_rr = d.result_rr.p;
}

void World::ensure_layout() {
  ensure_stream();
  if (layout_valid_ && layout_dt_ == g.dt) return;
  if (layout_valid_) invalidate_layout();
  cudaStream_t st = stream;
  nv_total = nf_total = 0;
  for (auto& c : cloths) {
    if (!c->setup_valid) {
      c->setup = std::make_unique<ClothSetup>();
      ClothParams prm;
      prm.elastic_stiffness = c->cfg.elastic_stiffness;
      prm.bending_stiffness = c->cfg.bending_stiffness;
      prm.density = c->cfg.density;
      prm.damping = c->cfg.damping;
      build_cloth_setup(c->rest.data(), c->nv(), c->faces.data(), c->nf(), prm,
                        *c->setup);
      build_cloth_device(*c);
      c->setup_valid = true;
    }
    c->voff = nv_total;
    c->foff = nf_total;
    nv_total += c->nv();
    nf_total += c->nf();
  }
  int nv = nv_total, nf = nf_total;
  for (DevBuf<float4>* b : {&sx, &sv, &prev_v, &outer, &outer_v, &x, &bending_rhs,
                            &rhs, &inertia, &pin_target, &pin_lambda, &contact_p,
                            &contact_p_prev, &contact_eta})
    b->alloc(nv);
  for (DevBuf<float>* b : {&mass, &damp, &lhs, &contact_w, &contact_w_base}) b->alloc(nv);
  pin_flag.alloc(nv);
  faces_d.alloc(nf);
  B0.alloc(nf);
  B1.alloc(nf);
  zu.alloc(3 * (size_t)nf);
  zold.alloc(2 * (size_t)nf);
  std::vector<float4> hx, hv, hbr;
  std::vector<float> hm, hd, hcw;
  std::vector<int4> hf;
  std::vector<float4> hb0, hb1;
  std::vector<int> hvo(1, 0), hvl;
  for (auto& c : cloths) {
    const ClothSetup& S = *c->setup;
    auto xs = to_float4(c->x_host, S.perm);
    auto vs = to_float4(c->v_host, S.perm);
    hx.insert(hx.end(), xs.begin(), xs.end());
    hv.insert(hv.end(), vs.begin(), vs.end());
    std::vector<double> cw;
    contact_weights(S, g.dt, cw);
    for (int i = 0; i < S.nv; ++i) {
      hbr.push_back(make_float4((float)S.bending_rhs[3 * i], (float)S.bending_rhs[3 * i + 1],
                                (float)S.bending_rhs[3 * i + 2], 0.f));
      hm.push_back((float)S.mass[i]);
      hd.push_back(1.0f - c->cfg.damping);
      hcw.push_back((float)cw[i]);
    }
    for (int t = 0; t < S.nf; ++t) {
      hf.push_back(make_int4(c->voff + S.F[3 * t], c->voff + S.F[3 * t + 1],
                             c->voff + S.F[3 * t + 2], 0));
      hb0.push_back(make_float4(S.B[6 * t], S.B[6 * t + 1], S.B[6 * t + 2], S.area_sqrt[t]));
      hb1.push_back(make_float4(S.B[6 * t + 3], S.B[6 * t + 4], S.B[6 * t + 5],
                                c->cfg.elastic_stiffness));
    }
    for (int i = 0; i < S.nv; ++i) {
      for (int k = S.vf_offsets[i]; k < S.vf_offsets[i + 1]; ++k) {
        int code = S.vf_list[k];
        hvl.push_back(((c->foff + (code >> 2)) << 2) | (code & 3));
      }
      hvo.push_back((int)hvl.size());
    }
  }
  auto up4 = [&](DevBuf<float4>& b, const std::vector<float4>& h) {
    if (!h.empty())
      CUDA_CHECK(cudaMemcpyAsync(b.p, h.data(), h.size() * sizeof(float4),
                                 cudaMemcpyHostToDevice, st));
  };
  up4(sx, hx);
  up4(sv, hv);
  up4(bending_rhs, hbr);
  mass.upload(hm, st);
  damp.upload(hd, st);
  contact_w_base.upload(hcw, st);
  faces_d.upload(hf, st);
  B0.upload(hb0, st);
  B1.upload(hb1, st);
  vf_off.upload(hvo, st);
  vf_list.upload(hvl, st);
  zu.zero(st);
  zold.zero(st);
  pin_lambda.zero(st);
  contact_w.zero(st);
  contact_p.zero(st);
  contact_p_prev.zero(st);
  contact_eta.zero(st);
  face_partials.alloc((size_t)face_step_blocks(nf) * kAdmmSlots);
  vertex_partials.alloc((size_t)vertex_step_blocks(nv) * kAdmmSlots);
  ctl.alloc(1);
  cg_fail.alloc(1);
  cg_fail.zero(st);
  // Learned warm start: 1-ring CSR over all cloths, step history (starting at
  // the current positions, i.e. zero displacements), feature buffers.
  {
    std::vector<int> roff(1, 0), rl;
    for (auto& c : cloths) {
      const ClothSetup& S = *c->setup;
      std::vector<std::vector<int>> nb(S.nv);
      for (size_t e = 0; e + 1 < S.E.size(); e += 2) {
        nb[S.E[e]].push_back(c->voff + S.E[e + 1]);
        nb[S.E[e + 1]].push_back(c->voff + S.E[e]);
      }
      for (int i = 0; i < S.nv; ++i) {
        rl.insert(rl.end(), nb[i].begin(), nb[i].end());
        roff.push_back((int)rl.size());
      }
    }
    if (rl.empty()) rl.push_back(0);
    ring_off.upload(roff, st);
    ring.upload(rl, st);
  }
  for (DevBuf<float4>* b : {&hist1, &hist2, &step_start, &ypred, &xpred}) b->alloc(nv);
  up4(hist1, hx);
  up4(hist2, hx);
  warm_feat.alloc((size_t)kMlpK * nv);
  warm_tgt.alloc((size_t)4 * nv);
  mlp_out.alloc((size_t)kMlpOut * nv);
  samples_valid = false;
  pinned_dof = 0;
  for (auto& c : cloths) c->on_device = true;
  pins_dirty_ = true;
  if (coll_) coll_->rebuild();
  layout_valid_ = true;
  layout_dt_ = g.dt;
}

void World::upload_pins() {
  if (!pins_dirty_) return;
  std::vector<unsigned char> flag(nv_total, 0);
  std::vector<float4> tgt(nv_total, make_float4(0, 0, 0, 0));
  pinned_dof = 0;
  for (auto& c : cloths) {
    const auto& perm = c->setup->perm;
    for (size_t k = 0; k < c->pins.size(); ++k) {
      int v = c->voff + perm[c->pins[k]];
      if (!flag[v]) pinned_dof += 3;
      flag[v] = 1;
      tgt[v] = make_float4(c->pin_pos[3 * k], c->pin_pos[3 * k + 1],
                           c->pin_pos[3 * k + 2], 0.f);
    }
  }
  if (nv_total) {
    CUDA_CHECK(cudaMemcpyAsync(pin_flag.p, flag.data(), nv_total,
                               cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaMemcpyAsync(pin_target.p, tgt.data(), nv_total * sizeof(float4),
                               cudaMemcpyHostToDevice, stream));
    sync();  // host vectors go out of scope
  }
  pins_dirty_ = false;
}

// MASPreconditioner::factorize on A = L + diag(lhs) (mas_preconditioner.cu:903).
void World::factorize(Cloth& c, cudaStream_t st) {
  ClothDev& d = c.dev;
  const ClothSetup& S = *c.setup;
  const float* dyn = lhs.p + c.voff;
  for (int k = 0; k < S.levels; ++k) {
    GalerkinDev gd;
    gd.n_entries = (int)S.galerkin[k].cols.size();
    gd.src_off = d.gal[k].src_off.p;
    gd.src = d.gal[k].src.p;
    gd.diag_off = k == 0 ? d.gal[k].diag_off.p : nullptr;
    gd.diag = k == 0 ? d.gal[k].diag.p : nullptr;
    gd.vals = d.gal[k].vals.p;
    launch_galerkin_fill(gd, k == 0 ? d.Lvals.p : d.gal[k - 1].vals.p, dyn, st);
  }
  launch_bank_invert(d.cg.fine, true, d.part_off.p, d.Lvals.p, dyn, cg_fail.p, st);
  for (int l = 1; l <= S.levels; ++l)
    launch_bank_invert(d.cg.coarse[l - 1], false, nullptr, d.gal[l - 1].vals.p,
                       nullptr, cg_fail.p, st);
}

float World::warm_sigma() const {
  float ax = g.acceleration_x, ay = g.acceleration_y, az = g.acceleration_z;
  float s = g.dt * g.dt * std::sqrt(ax * ax + ay * ay + az * az);
  return std::max(s, 1e-12f);
}

void World::cg_solve(Cloth& c, float rel_tol, bool first, cudaStream_t st) {
  CgArgs a = c.dev.cg;
  a.first_solve = first ? 1 : 0;
  if (first && has_model && opt.learned_warm_start) {
    a.x_alt = xpred.p + c.voff;
    a.alt_stat = 3;
  } else if (!first && iter_ready) {
    a.x_alt = iter_pred.p + c.voff;
    a.alt_stat = 5;
  } else if (!first && admm_ext_ready) {
    a.x_alt = admm_ext.p + c.voff;
    a.alt_stat = 4;
  }
  a.dyn = lhs.p + c.voff;
  a.b = rhs.p + c.voff;
  a.x = x.p + c.voff;
  a.bf16 = opt.mas_bf16 ? 1 : 0;
  a.rel_tol = rel_tol;
  a.abs_tol = g.linear_solver_abs_tol;
  a.max_iter = opt.cg_max_iter > 0 ? opt.cg_max_iter : 1000;
  a.stats = c.dev.stats.p;
  if (opt.profile >= 2) {
    if (c.dev.cg_trace.n < (size_t)kCgTraceLen) c.dev.cg_trace.alloc(kCgTraceLen);
    a.trace = c.dev.cg_trace.p;
  }
  a.fail = cg_fail.p;
  a.barrier_spin_limit = opt.barrier_spin_limit;
  a.withhold_block = opt.debug_withhold_block - 1;
  const bool dsm = c.dev.dsm_ctas > 0;
  const bool resident = !dsm && c.dev.res_grid != 0;
  // Counted by admm_solve for the iterations that ran.
  if (dsm || resident) solve_resident_ += 1;
  if (dsm) solve_cluster_ += 1;
  a.skip = cg_skip_;
  a.rel_tol_dev = cg_skip_ ? &ctl.p->next_rel_tol : nullptr;
  auto launch = [&]() {
    if (dsm)
      launch_cg_dsm(a, c.dev.dsm_ctas, st);
    else if (resident)
      launch_cg_resident(a, c.dev.res_grid, st);
    else
      launch_cg(a, c.dev.cg_grid, st);
  };
  if (opt.profile) {
    auto* ev = next_event_pair(events, events_used);
    CUDA_CHECK(cudaEventRecord(ev->first, st));
    launch();
    CUDA_CHECK(cudaEventRecord(ev->second, st));
  } else {
    launch();
  }
}

std::pair<cudaEvent_t, cudaEvent_t>* World::next_event_pair(
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& pool, size_t& used) {
  if (used == pool.size()) {
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    pool.emplace_back(e0, e1);
  }
  return &pool[used++];
}

silk_status World::debug_cg_trace(uint32_t h, int64_t* out, int64_t cap, int32_t* n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  *n = 0;
  if (!c->dev.cg_trace.p) return SILK_OK;
  if (cap < kCgTraceLen) return SILK_ERR_INVALID_CONFIG;
  sync();
  CUDA_CHECK(cudaMemcpy(out, c->dev.cg_trace.p, kCgTraceLen * sizeof(long long),
                        cudaMemcpyDeviceToHost));
  *n = kCgTraceLen;
  return SILK_OK;
}

// n = kMlpParams: the first-solve model; n = 2 kMlpParams: the first-solve
// model followed by the iterate model.
silk_status World::set_warm_start_model(const float* params, int64_t n) {
  if (!params) {
    has_model = false;
    has_iter_model = false;
    return SILK_OK;
  }
  if (n != kMlpParams && n != 2 * (int64_t)kMlpParams) return SILK_ERR_INVALID_CONFIG;
  for (int64_t m = 0; m < n; m += kMlpParams)
    for (int i = kOffStd; i < kOffStd + kMlpK; ++i)
      if (!(params[m + i] > 0.0f)) return SILK_ERR_INVALID_CONFIG;
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(params[i])) return SILK_ERR_INVALID_CONFIG;
  ensure_stream();
  mlp_params.alloc(kMlpParams);
  mlp_image_buf.alloc(kMlpWeightImage);
  CUDA_CHECK(cudaMemcpyAsync(mlp_params.p, params, kMlpParams * sizeof(float),
                             cudaMemcpyHostToDevice, stream));
  mlp_image(mlp_params.p, mlp_image_buf.p, stream);
  has_iter_model = n == 2 * (int64_t)kMlpParams;
  if (has_iter_model) {
    mlp2_params.alloc(kMlpParams);
    mlp2_image_buf.alloc(kMlpWeightImage);
    CUDA_CHECK(cudaMemcpyAsync(mlp2_params.p, params + kMlpParams, kMlpParams * sizeof(float),
                               cudaMemcpyHostToDevice, stream));
    mlp_image(mlp2_params.p, mlp2_image_buf.p, stream);
  }
  sync();
  has_model = true;
  return SILK_OK;
}

silk_status World::get_iterate_samples(float* feat, float* target, int64_t cap, int* n) {
  *n = 0;
  if (!iter_samp_n.p) return SILK_OK;
  sync();
  int total = 0;
  CUDA_CHECK(cudaMemcpy(&total, iter_samp_n.p, sizeof(int), cudaMemcpyDeviceToHost));
  const int64_t m = std::min<int64_t>(std::min(total, kIterSampleCap), cap);
  if (m > 0) {
    CUDA_CHECK(cudaMemcpy(feat, iter_samp_feat.p, (size_t)m * kMlpK * sizeof(float),
                          cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(target, iter_samp_tgt.p, (size_t)m * 4 * sizeof(float),
                          cudaMemcpyDeviceToHost));
  }
  *n = (int)m;
  return SILK_OK;
}

silk_status World::get_warm_start_samples(uint32_t h, float* feat, float* target, int64_t nv,
                                          int* valid) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  if (nv != c->nv()) return SILK_ERR_INVALID_POSITION;
  *valid = 0;
  if (!samples_valid || !c->on_device) return SILK_OK;
  sync();
  CUDA_CHECK(cudaMemcpy(feat, warm_feat.p + (size_t)kMlpK * c->voff,
                        (size_t)kMlpK * nv * sizeof(float), cudaMemcpyDeviceToHost));
  CUDA_CHECK(cudaMemcpy(target, warm_tgt.p + (size_t)4 * c->voff, (size_t)4 * nv * sizeof(float),
                        cudaMemcpyDeviceToHost));
  *valid = 1;
  return SILK_OK;
}

silk_status World::get_profile(silk_profile* p, bool reset) {
  *p = prof;
  if (reset) prof = silk_profile{};
  return SILK_OK;
}

silk_status World::get_cloth_velocity(uint32_t h, float* out, int64_t n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  int nv = c->nv();
  if (n != 3 * (int64_t)nv) return SILK_ERR_INVALID_POSITION;
  if (!c->on_device) {
    std::memcpy(out, c->v_host.data(), sizeof(float) * 3 * nv);
    return SILK_OK;
  }
  std::vector<float4> vs(nv);
  CUDA_CHECK(cudaMemcpyAsync(vs.data(), sv.p + c->voff, nv * sizeof(float4),
                             cudaMemcpyDeviceToHost, stream));
  sync();
  const auto& perm = c->setup->perm;
  for (int i = 0; i < nv; ++i) {
    float4 q = vs[perm[i]];
    out[3 * i] = q.x;
    out[3 * i + 1] = q.y;
    out[3 * i + 2] = q.z;
  }
  return SILK_OK;
}

bool World::admm_solve() {
  NvtxRange admm_range("ADMM solve");
  SolverView s = view();
  cudaStream_t st = stream;
  launch_compute_inertia(s, st);
  pin_lambda.zero(st);
  float rel = std::min(std::max(g.initial_linear_rel_tol, g.linear_solver_rel_tol_min),
                       g.linear_solver_rel_tol_max);
  if (opt.fixed_linear_rel_tol > 0) rel = opt.fixed_linear_rel_tol;
  // Iterations are decided on the device: the convergence test (run by the
  // vertex step's last block) sets AdmmControl::done when the solve
  // converges or diverges, and every kernel
  // of a later iteration returns at entry; the host enqueues
  // admm_check_interval iterations between reads of the control block, so
  // the GPU does not idle on a host round trip after every iteration.  The
  // CG takes each solve's tolerance from the control block.
  {
    AdmmControl init{};
    init.next_rel_tol = rel;
    CUDA_CHECK(cudaMemcpyAsync(ctl.p, &init, sizeof(AdmmControl), cudaMemcpyHostToDevice, st));
  }
  const int check_every = opt.admm_check_interval > 0 ? opt.admm_check_interval : 4;
  ctl_host_ = AdmmControl{};
  const int* done = &ctl.p->done;
  s.skip = done;
  cg_skip_ = done;
  struct SkipReset {
    const int*& p;
    ~SkipReset() { p = nullptr; }
  } skip_reset{cg_skip_};
  solve_resident_ = solve_cluster_ = 0;
  const int prior_iterations = stats.admm_iterations;
  int enqueued = 0;
  int fb = face_step_blocks(nf_total), vb = vertex_step_blocks(nv_total);
  AdmmFinalizeArgs fa;
  fa.face_partials = face_partials.p;
  fa.face_blocks = fb;
  fa.vertex_partials = vertex_partials.p;
  fa.vertex_blocks = vb;
  fa.dof_primal_static = 6 * nf_total + pinned_dof;
  fa.contact_active_dof = coll_ ? coll_->active_dof_device() : nullptr;
  fa.state_dof = 3 * nv_total;
  fa.abs_tol = g.admm_abs_tol;
  fa.rel_tol = g.admm_rel_tol;
  fa.init_lin_rel = g.initial_linear_rel_tol;
  fa.lin_rel_min = g.linear_solver_rel_tol_min;
  fa.lin_rel_max = g.linear_solver_rel_tol_max;
  fa.fixed_rel = opt.fixed_linear_rel_tol;
  fa.ctl = ctl.p;
  fa.cg_fail = cg_fail.p;
  bool contacts = coll_ && coll_->contact_count() > 0;
  admm_ext_ready = false;
  iter_ready = false;
  // Learned iterate start and its sample capture (solver options
  // learned_warm_start with an iterate model loaded, capture_samples bit 2).
  const bool iter_model = has_iter_model && opt.learned_warm_start;
  const bool iter_capture = (opt.capture_samples & 2) != 0;
  if (iter_model || iter_capture) {
    for (DevBuf<float4>* b : {&iter_hist0, &iter_hist1, &iter_hist2, &iter_pred})
      if (b->n < (size_t)nv_total) b->alloc(nv_total);
    if (iter_feat.n < (size_t)kMlpK * nv_total) iter_feat.alloc((size_t)kMlpK * nv_total);
    if (iter_out.n < (size_t)kMlpOut * nv_total) iter_out.alloc((size_t)kMlpOut * nv_total);
    if (!iter_sigma.p) iter_sigma.alloc(1);
  }
  DevBuf<float4>* iter_ring[3] = {&iter_hist0, &iter_hist1, &iter_hist2};
  for (int it = 0; it < g.max_inner_iteration; ++it) {
    if (it != 0 && (iter_model || iter_capture)) {
      // x holds x_(it-1); slots (it-1) % 3 and (it-2) % 3 hold x_(it-2) and
      // x_(it-3) from the previous iterations.
      if (it >= 3) {
        MlpDev m{iter_model ? mlp2_params.p : nullptr, mlp2_image_buf.p, cg_fail.p};
        iterate_predict(m, nv_total, x.p, iter_ring[(it - 1) % 3]->p, iter_ring[(it - 2) % 3]->p,
                        pin_flag.p, ring_off.p, ring.p, iter_sigma.p, iter_feat.p, iter_out.p,
                        iter_pred.p, st);
      }
      CUDA_CHECK(cudaMemcpyAsync(iter_ring[it % 3]->p, x.p, nv_total * sizeof(float4),
                                 cudaMemcpyDeviceToDevice, st));
      iter_ready = iter_model && it >= 3;
    }
    if (it != 0) {
      // Extrapolated start: from the third solve on, 2 x_k - x_(k-1) of the
      // last two iterates of this ADMM solve (the first solve starts from the
      // outer state, whose step to x_1 is not an ADMM iterate difference).
      if (opt.admm_extrapolated_start && it >= 2) {
        if (admm_prev.n < (size_t)nv_total) {
          admm_prev.alloc(nv_total);
          admm_ext.alloc(nv_total);
        }
        launch_extrapolate(nv_total, it >= 3, x.p, admm_prev.p, admm_ext.p, st);
        admm_ext_ready = it >= 3;
      }
      // Cloths are independent systems.  Those whose CG runs as one
      // thread-block cluster (scheduled as a unit) go on their own streams,
      // forked from and joined back into the world's stream; cooperative
      // grids stay on the world's stream, one after another.
      std::vector<int> forked;
      for (int k = 0; k < (int)cloths.size(); ++k) {
        const ClothDev& d = cloths[k]->dev;
        const bool resident = d.res_grid != 0;
        const bool cluster = d.dsm_ctas > 0 || (resident ? d.res_grid < 0 : d.cg_grid < 0);
        if (cloths.size() > 1 && cluster) forked.push_back(k);
      }
      if (!forked.empty()) {
        ensure_cloth_streams(cloths.size());
        CUDA_CHECK(cudaEventRecord(fork_ev_, st));
      }
      size_t f = 0;
      for (int k = 0; k < (int)cloths.size(); ++k) {
        Cloth& c = *cloths[k];
        cudaStream_t cs = st;
        if (f < forked.size() && forked[f] == k) {
          cs = cloth_streams_[k];
          CUDA_CHECK(cudaStreamWaitEvent(cs, fork_ev_, 0));
        }
        if (it == 1) factorize(c, cs);
        cg_solve(c, rel, it == 1, cs);
        if (cs != st) {
          CUDA_CHECK(cudaEventRecord(cloth_done_[k], cs));
          ++f;
        }
      }
      for (int k : forked) CUDA_CHECK(cudaStreamWaitEvent(st, cloth_done_[k], 0));
      if (it == 1 && (opt.capture_samples & 1) && warm_first_) {
        warm_target(nv_total, x.p, ypred.p, 1.0f / warm_sigma(), warm_tgt.p, st);
        samples_valid = true;
      }
      if (iter_capture && it >= 3)
        iterate_samples(kIterSamplesPerSolve, nv_total, (unsigned)(it * 7919 + prior_iterations + it),
                        iter_feat.p, x.p, iter_ring[it % 3]->p, iter_sigma.p, iter_samp_feat.p,
                        iter_samp_tgt.p, iter_samp_n.p, kIterSampleCap, done, st);
    }
    std::pair<cudaEvent_t, cudaEvent_t>* oe = opt.profile ? next_event_pair(events_other, events_other_used) : nullptr;
    if (oe) CUDA_CHECK(cudaEventRecord(oe->first, st));
    launch_face_step(s, face_partials.p, fb, contacts, st);
    if (contacts) {
      std::pair<cudaEvent_t, cudaEvent_t>* ge =
          opt.profile ? next_event_pair(events_gs, events_gs_used) : nullptr;
      if (ge) CUDA_CHECK(cudaEventRecord(ge->first, st));
      coll_->contact_solve(done);
      if (ge) CUDA_CHECK(cudaEventRecord(ge->second, st));
    }
    fa.iteration = it;
    launch_vertex_step(s, fa, st);
    if (oe) CUDA_CHECK(cudaEventRecord(oe->second, st));
    enqueued = it + 1;
    if (it == 0) continue;
    if (it % check_every != 0 && it + 1 < g.max_inner_iteration) continue;
    CUDA_CHECK(cudaMemcpyAsync(&ctl_host_, ctl.p, sizeof(AdmmControl), cudaMemcpyDeviceToHost, st));
    sync();
    if (ctl_host_.done) break;
  }
  // Iterations that ran: 0 .. the last one finalized (the first has no
  // finalize); each one from the second on ran one CG solve per cloth.
  const int ran = enqueued <= 1 ? enqueued : ctl_host_.iteration + 1;
  stats.admm_iterations += ran;
  if (enqueued > 1) {
    const int per_it_res = solve_resident_ / (enqueued - 1), per_it_cl = solve_cluster_ / (enqueued - 1);
    stats.cg_resident_solves += per_it_res * (ran - 1);
    stats.cg_cluster_solves += per_it_cl * (ran - 1);
  }
  if (ctl_host_.diverged) return false;
  launch_enforce(s, st);
  return true;
}

silk_status World::solver_step() {
  NvtxRange step_range("silk::solver_step");
  if (!initialized) return SILK_ERR_NOT_INITIALIZED;
  try {
    long long launches0 = g_launch_count;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t) {
      return std::chrono::duration<double, std::milli>(clk::now() - t).count();
    };
    auto t_step = clk::now();
    stats = silk_step_stats{};
    if (cloths.empty()) {
      last_error = "nothing to solve";
      return SILK_ERR_UNKNOWN;
    }
    ensure_layout();
    upload_pins();
    cudaStream_t st = stream;
    int nv = nv_total;
    for (auto& c : cloths) c->dev.stats.zero(st);
    events_used = 0;
    events_other_used = 0;
    events_gs_used = 0;
    CUDA_CHECK(cudaMemcpyAsync(step_start.p, sx.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    if (opt.capture_samples & 1) samples_valid = false;
    if (opt.capture_samples & 2) {
      if (!iter_samp_n.p) {
        iter_samp_n.alloc(1);
        iter_samp_feat.alloc((size_t)kIterSampleCap * kMlpK);
        iter_samp_tgt.alloc((size_t)kIterSampleCap * 4);
      }
      iter_samp_n.zero(st);
    }
    // init (main_loop.cu:24-76): damped velocity, fresh ADMM aux variables.
    launch_damp(nv, damp.p, sv.p, prev_v.p, st);
    zu.zero(st);
    CUDA_CHECK(cudaMemcpyAsync(outer.p, sx.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_CHECK(cudaMemcpyAsync(outer_v.p, prev_v.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    bool collide = coll_ && coll_->has_colliders();
    float ms = 0.f, dact = 0.f;
    auto add_dcd_profile = [&]() {
      prof.dcd_candidates_host_ms += coll_->last_dcd_gather_ms;
      prof.dcd_build_host_ms += coll_->last_dcd_build_ms;
      prof.dcd_coloring_host_ms += coll_->last_dcd_color_ms;
      prof.dcd_layout_host_ms += coll_->last_dcd_layout_ms;
      prof.dcd_calls += 1;
    };
    if (coll_) {
      coll_->refresh_obstacles();
      coll_->begin_step();
    }
    if (collide) {
      float pad = coll_->scene_padding();
      ms = 0.2f * pad;
      dact = 1.0f * pad;
      NvtxRange dcd_range("refit + DCD + contact rebuild");
      auto t0 = clk::now();
      coll_->refit(outer.p, outer.p);
      prof.dcd_refit_host_ms += ms_since(t0);
      coll_->append_active(0.0f, dact);
      add_dcd_profile();
      prof.dcd_host_ms += ms_since(t0);
    }
    float remaining = 1.0f;
    for (int oit = 0; oit < g.max_outer_iteration; ++oit) {
      NvtxRange outer_range("outer iteration");
      stats.outer_iterations += 1;
      launch_predict(nv, g.dt, make_float4(g.acceleration_x, g.acceleration_y, g.acceleration_z, 0.f),
                     outer.p, outer_v.p, x.p, st);
      warm_first_ = oit == 0;
      if (warm_active()) {
        const float sigma = warm_sigma();
        CUDA_CHECK(cudaMemcpyAsync(ypred.p, x.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        warm_features(nv, outer.p, hist1.p, hist2.p, ypred.p, pin_flag.p, ring_off.p, ring.p,
                      1.0f / sigma, warm_feat.p, st);
        if (has_model && opt.learned_warm_start) {
          MlpDev m{mlp_params.p, mlp_image_buf.p, cg_fail.p};
          warm_predict(m, nv, warm_feat.p, ypred.p, sigma, mlp_out.p, xpred.p, st);
        }
      }
      auto t_admm = clk::now();
      if (!admm_solve()) {
        int f = 0;
        CUDA_CHECK(cudaMemcpy(&f, cg_fail.p, sizeof(int), cudaMemcpyDeviceToHost));
        last_error = (f & kFailMasPivot) ? "MAS bank inverse failed: zero or non-finite pivot"
                     : (f & kFailBarrier) ? "CG barrier wait gave up"
                     : (f & kFailContactWait) ? "contact Gauss-Seidel copy wait gave up"
                     : (f & kFailMlpWait) ? "learned warm start tensor-core wait gave up"
                                          : "solver diverged";
        if (f) cg_fail.zero(st);
        return SILK_ERR_ITERATIVE_SOLVE_FAIL;
      }
      prof.admm_host_ms += ms_since(t_admm);
      float toi = remaining;
      if (collide) {
        NvtxRange ccd_range("refit + CCD");
        auto t0 = clk::now();
        coll_->refit(x.p, outer.p);
        prof.ccd_refit_host_ms += ms_since(t0);
        int nq = 0, nh = 0;
        toi = coll_->min_toi(1.0f - remaining, remaining, ms, &nq, &nh);
        prof.ccd_candidates_host_ms += coll_->last_gather_ms;
        prof.ccd_first_pass_ms += coll_->last_first_pass_ms;
        prof.ccd_second_pass_ms += coll_->last_second_pass_ms;
        prof.ccd_second_pass_queries += coll_->last_second_pass_queries;
        prof.ccd_calls += 1;
        stats.ccd_queries += nq;
        stats.ccd_hits += nh;
        prof.ccd_host_ms += ms_since(t0);
      }
      stats.min_toi = toi;
      launch_velocity(nv, g.dt, x.p, outer.p, outer_v.p, st);
      if (toi >= remaining) {
        CUDA_CHECK(cudaMemcpyAsync(outer.p, x.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        break;
      }
      float rollback = 0.8f * toi;
      float frac = rollback / remaining;
      launch_mix(nv, frac, x.p, outer.p, st);
      remaining -= rollback;
      NvtxRange dcd_range("refit + DCD + contact rebuild");
      auto t0 = clk::now();
      coll_->refit(outer.p, outer.p);
      prof.dcd_refit_host_ms += ms_since(t0);
      coll_->append_active(1.0f - remaining, dact);
      add_dcd_profile();
      prof.dcd_host_ms += ms_since(t0);
    }
    // Final velocity from the whole accepted displacement (main_loop.cu:248).
    launch_velocity(nv, g.dt, outer.p, sx.p, sv.p, st);
    CUDA_CHECK(cudaMemcpyAsync(sx.p, outer.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    // Step history of the warm-start features.
    CUDA_CHECK(cudaMemcpyAsync(hist2.p, hist1.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    CUDA_CHECK(cudaMemcpyAsync(hist1.p, step_start.p, nv * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    std::vector<int> cgs(kCgStats * cloths.size());
    for (size_t k = 0; k < cloths.size(); ++k)
      CUDA_CHECK(cudaMemcpyAsync(&cgs[kCgStats * k], cloths[k]->dev.stats.p,
                                 kCgStats * sizeof(int), cudaMemcpyDeviceToHost, st));
    sync();
    for (size_t k = 0; k < cloths.size(); ++k) {
      const int* q = &cgs[kCgStats * k];
      stats.cg_iterations += q[0];
      stats.cg_solves += q[1];
      stats.cg_first_solve_iterations += q[2];
      stats.learned_starts += q[3];
      stats.extrapolated_starts += q[4];
      stats.learned_iterate_starts += q[5];
      if (opt.profile) {
        double bpi = opt.mas_bf16 ? cloths[k]->dev.bytes_per_iter_bf16
                                  : cloths[k]->dev.bytes_per_iter_fp32;
        prof.cg_algorithmic_bytes += bpi * (q[0] + q[1]);
        prof.cg_iterations += q[0];
      }
    }
    if (opt.profile) {
      for (size_t e = 0; e < events_used; ++e) {
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, events[e].first, events[e].second));
        prof.cg_time_ms += ms;
      }
      // Solves that ran (launches of iterations enqueued after the ADMM
      // solve ended return at entry; their events add a few us).
      for (size_t k = 0; k < cloths.size(); ++k) prof.cg_launches += cgs[kCgStats * k + 1];
      for (size_t e = 0; e < events_gs_used; ++e) {
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, events_gs[e].first, events_gs[e].second));
        prof.contact_gs_ms += ms;
      }
      for (size_t e = 0; e < events_other_used; ++e) {
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, events_other[e].first, events_other[e].second));
        prof.admm_other_ms += ms;
      }
    }
    if (coll_) {
      stats.contacts = coll_->contact_count();
      stats.colors = coll_->color_count();
      stats.broadphase_candidates = coll_->last_candidates();
    }
    for (auto& o : obstacles) {
      o->prev = o->cur;
      if (o->is_static) o->is_static_twice = true;
      else o->is_static = true;
    }
    stats.kernel_launches = g_launch_count - launches0;
    prof.step_host_ms += ms_since(t_step);
    return SILK_OK;
  } catch (const std::exception& e) {
    last_error = e.what();
    return SILK_ERR_UNKNOWN;
  }
}

silk_status World::debug_partition(uint32_t h, int* perm, int64_t perm_len,
                                   int* offs, int64_t cap, int* nparts) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  ensure_layout();
  const ClothSetup& S = *c->setup;
  if (perm_len != S.nv) return SILK_ERR_INVALID_POSITION;
  for (int i = 0; i < S.nv; ++i) perm[i] = S.perm[i];
  int np = (int)S.part_offsets.size() - 1;
  *nparts = np;
  for (int i = 0; i <= np && i < cap; ++i) offs[i] = S.part_offsets[i];
  return SILK_OK;
}

silk_status World::debug_matrix(uint32_t h, double* dense, int64_t n) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  ensure_layout();
  const ClothSetup& S = *c->setup;
  if (n != (int64_t)S.nv * S.nv) return SILK_ERR_INVALID_POSITION;
  std::fill(dense, dense + n, 0.0);
  for (int i = 0; i < S.nv; ++i)
    for (int k = S.Lrows[i]; k < S.Lrows[i + 1]; ++k)
      dense[(size_t)i * S.nv + S.Lcols[k]] = S.Lvals[k];
  return SILK_OK;
}

silk_status World::debug_mas_fine(uint32_t h, float* inv, int64_t ninv, float* diag,
                                  int64_t ndiag) {
  Cloth* c = find_cloth(h);
  if (!c) return SILK_ERR_INVALID_HANDLE;
  ensure_layout();
  const ClothSetup& S = *c->setup;
  const int64_t need = (int64_t)S.fine.nbank * BANK * (BANK + 1) / 2;
  if (ninv != need || ndiag != S.nv || c->dev.fine.M.n < (size_t)need)
    return SILK_ERR_INVALID_POSITION;
  sync();
  CUDA_CHECK(cudaMemcpy(inv, c->dev.fine.M.p, need * sizeof(float), cudaMemcpyDeviceToHost));
  CUDA_CHECK(cudaMemcpy(diag, lhs.p + c->voff, S.nv * sizeof(float), cudaMemcpyDeviceToHost));
  return SILK_OK;
}

silk_status World::debug_refit(const float* disp, int64_t n) {
  if (!initialized) return SILK_ERR_NOT_INITIALIZED;
  ensure_layout();
  std::vector<float4> h(nv_total);
  int64_t off = 0;
  for (auto& c : cloths) {
    for (int i = 0; i < c->nv(); ++i) {
      float4 q = make_float4(0, 0, 0, 0);
      if (disp && off + 3 * i + 2 < n)
        q = make_float4(disp[off + 3 * i], disp[off + 3 * i + 1], disp[off + 3 * i + 2], 0.f);
      h[c->voff + c->setup->perm[i]] = q;
    }
    off += 3 * c->nv();
  }
  // x = sx + disp.
  std::vector<float4> xs(nv_total);
  CUDA_CHECK(cudaMemcpy(xs.data(), sx.p, nv_total * sizeof(float4), cudaMemcpyDeviceToHost));
  for (int i = 0; i < nv_total; ++i) {
    xs[i].x += h[i].x;
    xs[i].y += h[i].y;
    xs[i].z += h[i].z;
  }
  CUDA_CHECK(cudaMemcpy(x.p, xs.data(), nv_total * sizeof(float4), cudaMemcpyHostToDevice));
  coll_->refresh_obstacles();
  coll_->refit(x.p, sx.p);
  sync();
  return SILK_OK;
}

silk_status World::debug_candidates(int* out, int64_t cap, int* n) {
  *n = coll_->debug_candidates(out, cap);
  return SILK_OK;
}

silk_status World::debug_dcd(float t, float dact, int* keys, int64_t cap, int* n) {
  *n = coll_->debug_dcd(t, dact, keys, cap);
  return SILK_OK;
}

silk_status World::debug_contacts(int* keys, int64_t cap, int* n) {
  *n = coll_ ? coll_->debug_contacts(keys, cap) : 0;
  return SILK_OK;
}

silk_status World::debug_min_toi(float ts, float mt, float ms, bool prune,
                                 float* toi, int* nq, int* nh) {
  *toi = coll_->min_toi(ts, mt, ms, nq, nh, prune);
  return SILK_OK;
}

}  // namespace silkb
