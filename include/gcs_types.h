/*
 * gcs_types.h - host/device record layouts shared by the engine, its C ABI and
 * its callers.
 *
 * Star and PlaybackStar are byte-identical to the reference's records
 * (types.h:5-18 of lakshya076/Galaxy-Collision-Simulator), so a caller that
 * fills a Star[] for the reference engine can hand the same buffer to this
 * one, and frames written by the bake writer are the same bytes as the
 * reference's simulation.bin frames.
 *
 * BvhNodeTraverse and BvhNodeBuild have the layout of the reference's split
 * tree nodes (karras_bvh.cuh:7-21).  The traverse node's last word, which is
 * padding in the reference, holds the far end of the node's particle range
 * (Karras 2012: internal node i covers the sorted range [min(i,j), max(i,j)];
 * the word stores j), so the walk can tell a node's particle count without a
 * second array.
 *
 * Plain C so that ctypes / cgo / JNI bindings can mirror it.
 */
#ifndef GCS_TYPES_H
#define GCS_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
#define GCS_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define GCS_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

/* One particle as the reference's host code, its VBO and its uploads see it:
 * x0 y4 z8 vx12 vy16 vz20 mass24 type28 r29 g30 b31 (32 bytes, 4-aligned).
 * type: 0 = galaxy A star, 1 = dark matter, 2 = galaxy B star. */
typedef struct Star {
    float x, y, z;
    float vx, vy, vz;
    float mass;
    uint8_t type;
    uint8_t r, g, b;
} Star;

/* One particle of a simulation.bin frame: position and colour, and the type
 * in the last byte (the reference's bake loop writes `type` into `padding`,
 * main.cpp:266). 16 bytes. */
typedef struct PlaybackStar {
    float x, y, z;
    uint8_t r, g, b;
    uint8_t padding;
} PlaybackStar;

/* Traversal record of one tree node (32 bytes, read as two 16-byte loads).
 * Internal nodes are 0 .. n_internal-1 (root of segment s at
 * seg_off[s] - s); a child index >= n_internal names the particle
 * (child - n_internal) in sorted order, which for one segment is the
 * reference's leaf numbering N-1+i. */
typedef struct BvhNodeTraverse {
    float com_x, com_y, com_z;
    float mass;
    float width;        /* max extent of the node's bounding box */
    int32_t child_left;
    int32_t child_right;
    int32_t range_end;  /* reference: padding; here the far end j of the range */
} BvhNodeTraverse;

/* Build/aggregation record of one internal node (32 bytes). */
typedef struct BvhNodeBuild {
    float min_x, min_y, min_z;
    float max_x, max_y, max_z;
    int32_t flag;       /* arrival counter of the bottom-up pass */
    int32_t parent;     /* -1 at a segment root */
} BvhNodeBuild;

GCS_STATIC_ASSERT(sizeof(Star) == 32, "Star must be 32 bytes");
GCS_STATIC_ASSERT(sizeof(PlaybackStar) == 16, "PlaybackStar must be 16 bytes");
GCS_STATIC_ASSERT(sizeof(BvhNodeTraverse) == 32, "BvhNodeTraverse must be 32 bytes");
GCS_STATIC_ASSERT(sizeof(BvhNodeBuild) == 32, "BvhNodeBuild must be 32 bytes");

#endif /* GCS_TYPES_H */
