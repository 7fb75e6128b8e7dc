// Drives the B200 library through the reference-compatible C++ header
// (include/silk/silk.hpp): the calls a reference user makes, unchanged.
// Exit code 0 on success; prints the failing check otherwise.
#include <silk/silk.hpp>

#include <cmath>
#include <cstdio>
#include <vector>

#define CHECK(cond)                                              \
  do {                                                           \
    if (!(cond)) {                                               \
      std::fprintf(stderr, "check failed: %s (line %d)\n", #cond, \
                   __LINE__);                                    \
      return 1;                                                  \
    }                                                            \
  } while (0)

int main() {
  silk::World world;
  silk::Result r = world.init(silk::Backend::GPU);
  if (!r) {
    std::fprintf(stderr, "%s\n", r.to_string().c_str());
    return 2;
  }
  silk::GlobalConfig cfg;
  cfg.acceleration_z = -9.81f;
  CHECK(world.set_global_config(cfg));

  // 8 x 8 sheet, pinned at one corner.
  const int s = 8;
  std::vector<float> verts;
  std::vector<int> faces;
  for (int j = 0; j < s; ++j)
    for (int i = 0; i < s; ++i) {
      verts.push_back(i / float(s - 1));
      verts.push_back(j / float(s - 1));
      verts.push_back(1.0f);
    }
  for (int j = 0; j + 1 < s; ++j)
    for (int i = 0; i + 1 < s; ++i) {
      int a = j * s + i, b = a + 1, c = a + s, d = c + 1;
      int tri[6] = {a, b, d, a, d, c};
      faces.insert(faces.end(), tri, tri + 6);
    }
  std::vector<int> pins = {0};
  uint32_t handle = 0;
  CHECK(world.add_cloth(silk::ClothConfig{}, silk::CollisionConfig{},
                        silk::MeshConfig{verts, faces}, pins, handle));
  CHECK(handle != 0);

  for (int k = 0; k < 3; ++k) CHECK(world.solver_step());
  std::vector<float> x(verts.size());
  CHECK(world.get_cloth_position(handle, x));
  CHECK(std::fabs(x[2] - 1.0f) < 1e-5f);       // pinned vertex holds
  CHECK(x[3 * (s * s - 1) + 2] < 1.0f - 1e-3f);  // far corner falls

  // Error behaviour of the reference API.
  std::vector<float> wrong(3);
  r = world.get_cloth_position(handle, wrong);
  CHECK(!r && r.code == silk::ErrorCode::InvalidPosition);
  r = world.remove_cloth(handle + 77);
  CHECK(!r && r.code == silk::ErrorCode::InvalidHandle);
  std::vector<int> bad_faces = {0, 0, 1};
  uint32_t h2 = 123;
  r = world.add_cloth(silk::ClothConfig{}, silk::CollisionConfig{},
                      silk::MeshConfig{verts, bad_faces}, {}, h2);
  CHECK(!r && r.code == silk::ErrorCode::InvalidMesh && h2 == 0);
  CHECK(world.solver_reset());
  CHECK(world.get_cloth_position(handle, x));
  CHECK(x == verts);
  std::printf("drop-in silk::World ok\n");
  return 0;
}
