// Internal interface of the raymarcher (lbm_render.cu) for the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "lbm_b200.h"

namespace lbm {

// Per-frame constants of the reference's fragment shader (its uniforms).
struct RenderSetup {
  float inv[16];  // inverse view-projection, column-major
  float cam[3], gridInv[3], boxMax[3], light[3];
  float sph[4];  // centre and radius in the shader's world units (cells / max(nx, ny, nz))
};

void render_frame_setup(int nx, int ny, int nz, const lbm_sphere *sphere, const lbm_camera *cam, int width,
                        int height, RenderSetup *out);
cudaError_t render_launch(const uint8_t *d_vol, int nx, int ny, int nz, const RenderSetup &r, int width,
                          int height, uint8_t *d_out, cudaStream_t st);

}  // namespace lbm
