// Host-side scene object behind the enc_scene handle: a triangle soup in
// primitive-list order plus what the scene-file front-end records about it.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "encore_b200.h"

struct enc_scene_s {
  std::vector<float> verts;           // 9 floats per triangle
  uint32_t ntris = 0;
  // Filled by the loaders; empty for enc_scene_create (then triangle i is
  // primitive i with the default material).
  std::vector<int32_t> prim_of_tri;
  std::vector<int32_t> material_of_tri;
  std::vector<std::array<float, 13>> materials;
  std::vector<enc_scene_light> lights;
  enc_scene_desc desc{};
};
