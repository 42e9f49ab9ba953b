// gg_host.h -- host-side helpers shared by the C ABI translation units.
#pragma once

#include "../../include/gargantua_gpu.h"
#include "gg_params.h"

namespace gg {

// Checks every field a render would use (the rules of gg_validate).
int validate_render(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
                    const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
                    uint32_t height);

// Builds the kernel parameter block of a validated render.
void make_params(const gg_metric_t* metric, const gg_camera_t* camera, const gg_disk_t* disk,
                 const gg_integrator_t* integ, const gg_render_opts_t* opts, uint32_t width,
                 uint32_t height, DevParams* out);

}  // namespace gg
