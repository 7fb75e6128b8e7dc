// Collision pipeline (placeholder until the broadphase/CCD kernels land).
#include "collision.cuh"
#include "world.hpp"

namespace silkb {

struct CollisionImpl {
  DevBuf<int> zero;
};

CollisionSystem::CollisionSystem(World& w) : w_(w), impl_(new CollisionImpl) {
  impl_->zero.alloc(1);
  CUDA_CHECK(cudaMemset(impl_->zero.p, 0, sizeof(int)));
}
CollisionSystem::~CollisionSystem() = default;
void CollisionSystem::rebuild() {}
float CollisionSystem::scene_padding() const { return 0.0f; }
bool CollisionSystem::has_colliders() const { return false; }
void CollisionSystem::refresh_obstacles() {}
void CollisionSystem::refit(const float4*, const float4*) {}
void CollisionSystem::begin_step() {}
int CollisionSystem::append_active(float, float) { return 0; }
float CollisionSystem::min_toi(float, float max_time, float, int* nq, int* nh) {
  *nq = 0;
  *nh = 0;
  return max_time;
}
void CollisionSystem::contact_solve() {}
int CollisionSystem::contact_count() const { return 0; }
int CollisionSystem::color_count() const { return 0; }
const int* CollisionSystem::active_dof_device() const { return impl_->zero.p; }
int CollisionSystem::last_candidates() const { return 0; }
int CollisionSystem::debug_candidates(int*, int64_t) { return 0; }
int CollisionSystem::debug_dcd(float, float, int*, int64_t) { return 0; }

void ccd_batch_host(bool, const float*, int64_t, const float*, const float*,
                    float, int, float, int*, float*, float*) {
  throw std::runtime_error("not built");
}
int color_contacts_host(const int*, const uint64_t*, int64_t, int*) { return -1; }

}  // namespace silkb
