// ref_cpu_shim.cpp - headless driver for the reference's CPU Barnes-Hut
// engine, compiled together with the reference's own engine.cpp,
// gravity_aggregator.cpp (theta made a variable, see build_ref.py) and
// generator.cpp into oracle/_ref/libref_cpu.so.
//
// TEST/BASELINE INFRASTRUCTURE ONLY: bench.py times it as the reference's
// CPU implementation, tests use it for golden vectors.  ref_cpu_step repeats
// the CPU step sequence of the reference's driver (main.cpp:152-252):
// bounds, Morton sort (__gnu_parallel::sort), arena reset + insert_star,
// node_physics, OpenMP query_gravity (dynamic,256), OpenMP integrate.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <limits>
#include <parallel/algorithm>
#include <random>
#include <utility>
#include <vector>

#include "arena_allocator.h"
#include "engine.h"
#include "generator.h"
#include "gravity_aggregator.h"
#include "morton.h"

float ref_cpu_theta = 0.8f;  // read by the theta-variable gravity_aggregator copy

namespace {

struct State {
    ArenaAllocator* arena = nullptr;
    size_t max_nodes = 0;
    uint32_t* leaf_idx = nullptr;
    float *node_m = nullptr, *node_x = nullptr, *node_y = nullptr, *node_z = nullptr;
    std::vector<float> acc;
};
State g;

void release() {
    delete g.arena;
    delete[] g.leaf_idx;
    delete[] g.node_m;
    delete[] g.node_x;
    delete[] g.node_y;
    delete[] g.node_z;
    g = State();
}

}  // namespace

extern "C" {

// Arena of `arena_bytes` (the reference uses 64 MiB, main.cpp:102-108).
int ref_cpu_init(int64_t n, int64_t arena_bytes) {
    release();
    if (arena_bytes <= 0) arena_bytes = 1024ll * 1024 * 64;
    g.arena = new ArenaAllocator((size_t)arena_bytes);
    g.max_nodes = (size_t)arena_bytes / sizeof(OctreeNode);
    g.leaf_idx = new uint32_t[g.max_nodes * 32];
    g.node_m = new float[g.max_nodes];
    g.node_x = new float[g.max_nodes];
    g.node_y = new float[g.max_nodes];
    g.node_z = new float[g.max_nodes];
    g.acc.assign((size_t)n * 3, 0.0f);
    return 0;
}

void ref_cpu_cleanup(void) { release(); }

void ref_cpu_set_theta(float theta) { ref_cpu_theta = theta; }

int ref_cpu_threads(void) { return omp_get_max_threads(); }

// One CPU step over stars[0..n); accel_out (3n floats, may be NULL) gets the
// accelerations of the sorted particles.  times (may be NULL): seconds for
// {sort, build, walk, integrate}.
int ref_cpu_step(Star* stars, int n, float G, float epsilon_sq, float dt, float* accel_out,
                 double* times) {
    using clk = std::chrono::steady_clock;
    if (!g.arena || (int64_t)g.acc.size() < 3ll * n) return -1;
    const auto t0 = clk::now();
    float min_x = std::numeric_limits<float>::max(), min_y = min_x, min_z = min_x;
    float max_x = std::numeric_limits<float>::lowest(), max_y = max_x, max_z = max_x;
    for (int i = 0; i < n; i++) {
        min_x = std::min(min_x, stars[i].x);
        min_y = std::min(min_y, stars[i].y);
        min_z = std::min(min_z, stars[i].z);
        max_x = std::max(max_x, stars[i].x);
        max_y = std::max(max_y, stars[i].y);
        max_z = std::max(max_z, stars[i].z);
    }
    const float gmin = std::min({min_x, min_y, min_z});
    const float gmax = std::max({max_x, max_y, max_z});
    std::vector<std::pair<uint64_t, Star>> buf((size_t)n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        buf[i].first = get_morton_code(stars[i].x, stars[i].y, stars[i].z, gmin, gmax);
        buf[i].second = stars[i];
    }
    __gnu_parallel::sort(buf.begin(), buf.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) stars[i] = buf[i].second;
    const auto t1 = clk::now();

    g.arena->reset();
    OctreeNode* root = g.arena->alloc<OctreeNode>();
    const float span = std::max({max_x - min_x, max_y - min_y, max_z - min_z});
    root->center_x = (min_x + max_x) * 0.5f;
    root->center_y = (min_y + max_y) * 0.5f;
    root->center_z = (min_z + max_z) * 0.5f;
    root->half_width = span * 0.5f;
    root->is_leaf = true;
    root->start_star_index = 0;
    root->star_count = 0;
    uint32_t next_free = 32;
    for (uint32_t i = 0; i < (uint32_t)n; i++) insert_star(root, i, stars, *g.arena, g.leaf_idx, next_free);
    node_physics(root, root, stars, g.node_m, g.node_x, g.node_y, g.node_z, g.leaf_idx);
    const auto t2 = clk::now();

    float* acc = g.acc.data();
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i)
        query_gravity(root, stars[i], (uint32_t)i, stars, g.node_m, g.node_x, g.node_y, g.node_z,
                      g.leaf_idx, G, epsilon_sq, acc[3 * i], acc[3 * i + 1], acc[3 * i + 2]);
    const auto t3 = clk::now();

#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        stars[i].vx += acc[3 * i] * dt;
        stars[i].vy += acc[3 * i + 1] * dt;
        stars[i].vz += acc[3 * i + 2] * dt;
        stars[i].x += stars[i].vx * dt;
        stars[i].y += stars[i].vy * dt;
        stars[i].z += stars[i].vz * dt;
    }
    const auto t4 = clk::now();
    if (accel_out) std::copy(acc, acc + 3 * (size_t)n, accel_out);
    if (times) {
        times[0] = std::chrono::duration<double>(t1 - t0).count();
        times[1] = std::chrono::duration<double>(t2 - t1).count();
        times[2] = std::chrono::duration<double>(t3 - t2).count();
        times[3] = std::chrono::duration<double>(t4 - t3).count();
    }
    return 0;
}

// The reference's own initial conditions (generator.cpp:169-210) with a
// seeded mt19937 in place of random_device (main.cpp:66).
void ref_initial_setup(uint32_t seed, int num_dm, int num_disc, int num_bulge, Star* out) {
    std::mt19937 rng(seed);
    initial_setup(out, num_dm, num_disc, num_bulge, rng);
}

}  // extern "C"
