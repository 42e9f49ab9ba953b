// gg_scene_host.h -- host-side scene preparation (gg_scene_build.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/gargantua_gpu.h"
#include "gg_params.h"

namespace gg {

// Checks `prims`, resolves their materials and builds the hierarchy:
// out_prims in leaf order, out_nodes with the root at index 0, and the
// tree's depth.  Returns GG_OK, GG_ERR_INVALID_ARG (empty, non-finite or
// degenerate primitives, unknown kinds) or GG_ERR_UNSUPPORTED (a fuzzed
// metal, whose shading the reference draws at random).
int build_scene(const gg_prim_t* prims, uint32_t n, std::vector<ScenePrim>* out_prims,
                std::vector<SceneNode>* out_nodes, uint32_t* depth);

}  // namespace gg
