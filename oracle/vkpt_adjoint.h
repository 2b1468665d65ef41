/*
 * vkpt_adjoint.h -- FP64 CPU adjoint of the render path (test infrastructure).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library includes, links
 * or calls this; only tests/ use it, as the checker of vkptc_forward /
 * vkptc_backward.
 *
 * The reference has no derivative path, so this oracle restates the
 * reference's trace loop (src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289,
 * sample_direct_light :1022-1118, sample_phong_lobe :996-1020, camera_rays
 * src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119, shade_pixel :228-284)
 * in double precision with forward-mode dual numbers over a chosen subset of
 * the material parameters, and differentiates the estimator the GPU adjoint
 * differentiates:
 *   - Phong-lobe directions are reparameterized (same uniforms; they move
 *     with roughness and with the incoming direction);
 *   - the Russian-roulette probability is held constant;
 *   - discrete decisions come from the (double) primal, so visibility
 *     boundaries contribute nothing.
 * Intersection is brute force over all triangles (Moller-Trumbore in double
 * with the reference's thresholds), which suits the small scenes the
 * gradient tests use.  Parity with the reference is "unpinned" (there is no
 * reference derivative); the primal image is checked against the reference
 * render statistically by the tests.
 */
#ifndef VKPT_ADJOINT_H
#define VKPT_ADJOINT_H

#include <stdint.h>

#include "vkpt_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

#define VKO_ADJ_PARAMS_PER_MATERIAL 7u
#define VKO_ADJ_MAX_TANGENTS 160u

typedef struct vko_adjoint_request {
  const float* params;         /* 7 per material: albedo rgb, roughness, emission rgb */
  uint32_t param_count;
  uint32_t spp;
  uint32_t first_sample;
  uint32_t frame;
  const float* target;         /* W*H*3, or NULL (loss 0) */
  const uint32_t* grad_index;  /* parameter indices to differentiate */
  uint32_t grad_count;         /* <= VKO_ADJ_MAX_TANGENTS */
  uint32_t threads;
  const float* rr_params;      /* NULL = params; else the parameters whose throughput sets the
                                  Russian-roulette probabilities and decisions (for finite differences) */
} vko_adjoint_request;

/* loss: mean over pixels and channels of (image - target)^2.
 * grad (grad_count doubles): dloss/dparams[grad_index[i]].
 * image (optional, W*H*3 doubles): the primal image.
 * Returns 0 on success, non-zero on failure (message via vko_adjoint_last_error). */
int vko_adjoint(const vko_scene* scene, const vko_settings* settings, const vko_adjoint_request* request,
                double* loss, double* grad, double* image);

/* Central finite differences of the same estimator with common random
 * numbers and the roulette of `params`: for each grad_index parameter, the
 * loss is linearised at `params` (per-pixel weights from its image) and every
 * path is re-traced at params +- h.  A path whose discrete decisions differ
 * from the unperturbed one (a "flip": another triangle, visibility, lobe
 * fallback or termination) is left out and counted in flips_out, so the
 * result converges to the derivative the adjoint computes. */
int vko_adjoint_fd(const vko_scene* scene, const vko_settings* settings, const vko_adjoint_request* request, double h,
                   double* fd_out, uint64_t* flips_out);

const char* vko_adjoint_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* VKPT_ADJOINT_H */
