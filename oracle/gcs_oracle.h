/*
 * gcs_oracle.h - CPU restatement of the reference's per-step Barnes-Hut path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke()
 * and bench.py's cpu_baseline leg compare against; the engine never calls
 * it.  Each function cites the reference file:line it restates
 * (lakshya076/Galaxy-Collision-Simulator).  Arithmetic whose rounding
 * decides a result is written with the same explicit fmaf() forms the CUDA
 * kernels use, and the GPU's saturating float->uint conversion is emulated,
 * so keys, permutations, topology and opening decisions match bit for bit;
 * 1/sqrt is IEEE here and rsqrtf on the GPU, so forces agree to FP32
 * rounding, not bitwise.
 *
 * Pinning: the restatement is checked against the reference's own code
 * compiled from its sources (oracle/_ref, built by oracle/build_ref.py) and
 * against golden vectors that code produced (tests/golden/).
 */
#ifndef GCS_ORACLE_H
#define GCS_ORACLE_H
#include <stdint.h>
#include "../include/gcs_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Saturating round-toward-zero float -> u32, NaN -> 0 (the GPU's cvt.rzi). */
uint32_t gcs_oracle_f2u_rz(float f);
/* morton.h:11-19 */
uint64_t gcs_oracle_spread21(uint32_t v);
/* morton.h:22-28 with GPU conversion semantics. */
uint64_t gcs_oracle_morton(float x, float y, float z, float lo, float hi);
/* Keys of n particles (xyzm: 4 floats per particle). */
void gcs_oracle_encode(const float* xyzm, int64_t n, float lo, float hi, uint64_t* keys);
/* main.cpp:152-166: scalar min over x,y,z and max over x,y,z. */
void gcs_oracle_bounds(const float* xyzm, int64_t n, float* lo, float* hi);
/* cub::DeviceRadixSort::SortPairs over (key, position) (cuda_engine.cu:397):
 * stable, so equal keys keep position order. */
void gcs_oracle_sort(const uint64_t* keys, int64_t n, uint64_t* keys_out, uint32_t* idx_out);
/* karras_bvh.cuh:73-131 for one segment of n >= 2 sorted keys, with node
 * numbering base `node_base`, particle (leaf) numbering base `leaf_base` and
 * particle offset `off` (range_end is off + j).  parent has n-1 entries
 * (root: -1), leaf_parent has n. */
void gcs_oracle_build(const uint64_t* keys, int n, int node_base, int leaf_base, int off,
                      int32_t* child_left, int32_t* child_right, int32_t* range_end,
                      int32_t* parent, int32_t* leaf_parent);
/* karras_bvh.cuh:175-225 over one segment: fills com/mass/width of `nodes`
 * (n-1 entries, children already set, numbering as in gcs_oracle_build with
 * node_base 0 and leaf_base n-1) and box (6 floats per node).  com_fp64
 * selects, for nodes of at least GCS_ORACLE_COM_FP64_MIN particles (the top
 * of the tree), FP64 mass-weighted sums instead of the FP32 pairwise formula;
 * a child below that size (or a particle) enters those sums as the exact
 * double product of its FP32 mass and centre of mass (or position). */
#define GCS_ORACLE_COM_FP64_MIN 1024
void gcs_oracle_aggregate(int n, const float* xyzm, BvhNodeTraverse* nodes, float* box,
                          int com_fp64);
/* cuda_engine.cu:91-161 with theta and leaf size L, for every particle of
 * one segment (sorted order, nodes numbered from 0, leaves from n-1).
 * acc: 4 floats per particle (ax, ay, az, potential).  counts (may be NULL):
 * 2 per particle (monopole terms, particle terms). */
void gcs_oracle_walk(int n, const float* xyzm, const BvhNodeTraverse* nodes, float G, float eps2,
                     float theta, int leaf_size, float* acc, int64_t* counts);
/* gcs_oracle_walk for the listed targets only (sorted indices): acc gets 4
 * floats and counts (may be NULL) 2 per listed target. */
void gcs_oracle_walk_targets(int n, const float* xyzm, const BvhNodeTraverse* nodes, float G, float eps2,
                             float theta, int leaf_size, const int64_t* targets, int64_t n_targets, float* acc,
                             int64_t* counts);
/* cuda_engine.cu:164-216 (vel4: vx, vy, vz, bits of type|r|g|b). */
void gcs_oracle_integrate(int64_t n, float* xyzm, float* vel4, const float* acc4, float dt,
                          int recolor);
/* FP64 direct sum excluding only i == j. out: 3 doubles per target. */
void gcs_oracle_direct_fp64(int64_t n, const float* xyzm, const int64_t* targets, int64_t n_targets,
                            double G, double eps2, double* out);
/* One full reference step of one segment (bounds caller-given when
 * use_bounds, else reduced): encode, sort, gather, build, aggregate, walk,
 * integrate.  xyzm/vel4 are permuted into sorted order and stepped in place;
 * acc (4/particle) receives the accelerations; nodes (n-1) the tree. */
void gcs_oracle_step(int n, float* xyzm, float* vel4, int use_bounds, float lo, float hi, float G,
                     float eps2, float theta, int leaf_size, float dt, int recolor, int com_fp64,
                     float* acc, BvhNodeTraverse* nodes);

/* Headless point-splat renderer (renderer.cpp:97-148, 203, 248): every
 * Star as a GL point through view and proj (row-major 4x4, column vectors),
 * fragments added to acc (width*height*3, 2^-24 units per channel, zeroed
 * by the caller); rgba (may be NULL) gets the resolved RGBA8 frame, row 0 at
 * the bottom. */
void gcs_oracle_render(const Star* stars, int64_t n, const float view[16], const float proj[16], int width,
                       int height, uint64_t* acc, uint8_t* rgba);

#ifdef __cplusplus
}
#endif
#endif
