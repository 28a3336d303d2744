/*
 * cuda_engine.h - drop-in replacement for the reference engine's API.
 *
 * Same C++ declarations (and so the same mangled symbols) as
 * cuda_engine.h:5-32 of lakshya076/Galaxy-Collision-Simulator, so the
 * reference's main.cpp links against libgcs unchanged.  Each function is a
 * thin wrapper over one process-wide gcs_ctx (include/gcs.h):
 *
 *   cuda_init                    cuda_engine.cu:219-285  -> gcs_create on device 0
 *   cuda_cleanup                 cuda_engine.cu:303-340  -> gcs_destroy
 *   cuda_allocate_pinned_stars   cuda_engine.cu:287-289  -> cudaMallocHost
 *   cuda_free_pinned_stars       cuda_engine.cu:291-293  -> cudaFreeHost
 *   cuda_allocate_pinned_playback cuda_engine.cu:295-297 -> cudaMallocHost
 *   cuda_free_pinned_playback    cuda_engine.cu:299-301  -> cudaFreeHost
 *   cuda_upload_initial_stars    cuda_engine.cu:342-352  -> gcs_upload_stars
 *   cuda_register_vbo            cuda_engine.cu:354-356  -> headless: records the id
 *   cuda_unregister_vbo          cuda_engine.cu:358-363  -> headless: forgets it
 *   cuda_get_center_of_mass      cuda_engine.cu:365-376  -> root node COM
 *   cuda_physics_step            cuda_engine.cu:379-451  -> gcs_step (+ pack, D2H)
 *
 * Behaviour kept from the reference: only cuda_init reports failure; the
 * step is synchronous and returns its dt argument; host_stars is output
 * only (overwritten with the stepped particles in this step's Morton order).
 * With use_interop=true and a registered VBO id the reference writes the
 * Stars into the GL buffer; there is no graphics stack here, so the stepped
 * Stars go to a device buffer (gcs_dropin_device_stars) instead and
 * host_stars is left untouched, as in the reference's interop branch.
 *
 * The reference's walk has no theta or leaf-size argument (theta = 1,
 * one particle per leaf); gcs_dropin_set_params changes those for callers
 * that want them, everything else keeps the reference's behaviour.
 */
#pragma once
#include "gcs_types.h"
#include "gcs.h"

bool cuda_init(int num_stars);
void cuda_cleanup();

void cuda_allocate_pinned_stars(Star** stars, int num_stars);
void cuda_free_pinned_stars(Star* stars);
void cuda_allocate_pinned_playback(PlaybackStar** buf, int size);
void cuda_free_pinned_playback(PlaybackStar* buf);

void cuda_upload_initial_stars(const Star* host_stars, int num_stars);

void cuda_register_vbo(unsigned int vbo_id);
void cuda_unregister_vbo();
void cuda_get_center_of_mass(float* cx, float* cy, float* cz);

float cuda_physics_step(
    Star* host_stars,
    int num_stars,
    float G,
    float epsilon_sq,
    float dt,
    float global_min,
    float global_max,
    bool use_interop
);

extern "C" {
/* Theta, leaf size, bounds mode, COM precision and walk tuning used by
 * cuda_physics_step; G, epsilon_sq, dt and the bounds still come from its
 * arguments.  Defaults: gcs_params_reference. */
int gcs_dropin_set_params(const gcs_params* p);
/* The process-wide context behind the drop-in functions (NULL before
 * cuda_init). */
gcs_ctx* gcs_dropin_context(void);
/* Device Star[] written by cuda_physics_step when use_interop is true and a
 * VBO id is registered: the headless stand-in for the mapped GL buffer. */
const Star* gcs_dropin_device_stars(void);
}
