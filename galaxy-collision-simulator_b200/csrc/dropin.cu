// dropin.cu - the reference's C++ engine API (cuda_engine.h:5-32) over one
// process-wide gcs_ctx.  See include/cuda_engine.h for the mapping.
#include <cstdio>
#include <mutex>

#include "../../include/cuda_engine.h"
#include "gcs_internal.h"

namespace {

gcs_ctx* g_ctx = nullptr;
gcs_params g_params;
bool g_params_set = false;
unsigned int g_vbo = 0;
bool g_vbo_registered = false;
Star* g_interop_stars = nullptr;   // headless stand-in for the mapped VBO
std::mutex g_mu;

const gcs_params& dropin_params() {
    if (!g_params_set) {
        gcs_params_reference(&g_params);
        g_params_set = true;
    }
    return g_params;
}

}  // namespace

bool cuda_init(int num_stars) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (num_stars < 1) return false;
    if (g_ctx) {
        gcs_destroy(g_ctx);
        g_ctx = nullptr;
    }
    gcs_ctx* c = nullptr;
    const int rc = gcs_create(&c, num_stars, 1, 0);
    if (rc != GCS_OK) {
        fprintf(stderr, "CUDA Error: engine initialisation failed (%s)\n", gcs_status_string(rc));
        return false;
    }
    if (cudaMalloc(&g_interop_stars, sizeof(Star) * (size_t)num_stars) != cudaSuccess) {
        gcs_destroy(c);
        g_interop_stars = nullptr;
        return false;
    }
    g_ctx = c;
    return true;
}

void cuda_cleanup() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_ctx) gcs_destroy(g_ctx);
    g_ctx = nullptr;
    if (g_interop_stars) cudaFree(g_interop_stars);
    g_interop_stars = nullptr;
}

void cuda_allocate_pinned_stars(Star** stars, int num_stars) {
    if (!stars) return;
    if (cudaMallocHost(reinterpret_cast<void**>(stars), sizeof(Star) * (size_t)num_stars) != cudaSuccess)
        *stars = nullptr;
}

void cuda_free_pinned_stars(Star* stars) {
    if (stars) cudaFreeHost(stars);
}

void cuda_allocate_pinned_playback(PlaybackStar** buf, int size) {
    if (!buf) return;
    if (cudaMallocHost(reinterpret_cast<void**>(buf), sizeof(PlaybackStar) * (size_t)size) != cudaSuccess)
        *buf = nullptr;
}

void cuda_free_pinned_playback(PlaybackStar* buf) {
    if (buf) cudaFreeHost(buf);
}

void cuda_upload_initial_stars(const Star* host_stars, int num_stars) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx || !host_stars) return;
    int64_t cnt = num_stars;
    if (gcs_num_particles(g_ctx) != num_stars) gcs_set_segments(g_ctx, 1, &cnt);
    gcs_upload_stars(g_ctx, host_stars, 0, num_stars);
}

void cuda_register_vbo(unsigned int vbo_id) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_vbo = vbo_id;
    g_vbo_registered = true;
}

void cuda_unregister_vbo() {
    std::lock_guard<std::mutex> lk(g_mu);
    g_vbo = 0;
    g_vbo_registered = false;
}

void cuda_get_center_of_mass(float* cx, float* cy, float* cz) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!cx || !cy || !cz) return;
    *cx = *cy = *cz = 0.0f;
    if (!g_ctx || gcs_num_internal_nodes(g_ctx) < 1) return;
    BvhNodeTraverse root;
    if (gcs_read_buffer(g_ctx, GCS_BUF_NODES, &root, 0, 1) == GCS_OK) {
        *cx = root.com_x;
        *cy = root.com_y;
        *cz = root.com_z;
    }
}

float cuda_physics_step(Star* host_stars, int num_stars, float G, float epsilon_sq, float dt,
                        float global_min, float global_max, bool use_interop) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx) return dt;
    gcs_params p = dropin_params();
    p.G = G;
    p.epsilon_sq = epsilon_sq;
    p.dt = dt;
    p.global_min = global_min;
    p.global_max = global_max;
    if (gcs_num_particles(g_ctx) != num_stars) return dt;
    if (use_interop && g_vbo_registered) {
        // No graphics stack here: the Stars go to the device buffer a mapped
        // VBO would have received (cuda_engine.cu:427-440), host untouched.
        if (gcs_step(g_ctx, &p) != GCS_OK) return dt;
        gcs::pack_to_device(g_ctx, g_interop_stars);
    } else if (host_stars) {
        // the step with the Star copy (cuda_engine.cu:442-448) overlapped
        // with the walk
        gcs_step_host(g_ctx, &p, host_stars);
    } else {
        gcs_step(g_ctx, &p);
    }
    return dt;
}

extern "C" {

int gcs_dropin_set_params(const gcs_params* p) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!p) return GCS_ERR_ARG;
    if (p->leaf_size < 1 || p->leaf_size > 32) return GCS_ERR_ARG;
    g_params = *p;
    g_params_set = true;
    return GCS_OK;
}

gcs_ctx* gcs_dropin_context(void) { return g_ctx; }

const Star* gcs_dropin_device_stars(void) { return g_interop_stars; }

}  // extern "C"
