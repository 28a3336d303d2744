/*
 * gcs_oracle.c - CPU restatement of the reference's per-step Barnes-Hut path.
 *
 * TEST INFRASTRUCTURE ONLY (see gcs_oracle.h).  Compile without FMA
 * contraction or fast-math (-ffp-contract=off): every fused multiply-add
 * below is an explicit fmaf() mirroring the CUDA kernels.
 */
#include "gcs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

uint32_t gcs_oracle_f2u_rz(float f) {
    if (isnan(f) || f <= 0.0f) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)f;
}

/* morton.h:11-19: bit k of the 21-bit input moves to bit 3k. */
uint64_t gcs_oracle_spread21(uint32_t v) {
    uint64_t x = v & 0x1FFFFFu;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

/* morton.h:22-28: scale = 2097151/(max-min) in FP32; (c-min)*scale truncated. */
uint64_t gcs_oracle_morton(float x, float y, float z, float lo, float hi) {
    const float scale = 2097151.0f / (hi - lo);
    const uint32_t ix = gcs_oracle_f2u_rz((x - lo) * scale);
    const uint32_t iy = gcs_oracle_f2u_rz((y - lo) * scale);
    const uint32_t iz = gcs_oracle_f2u_rz((z - lo) * scale);
    return (gcs_oracle_spread21(ix) << 2) | (gcs_oracle_spread21(iy) << 1) | gcs_oracle_spread21(iz);
}

/* karras_bvh.cuh:34-41 */
void gcs_oracle_encode(const float* xyzm, int64_t n, float lo, float hi, uint64_t* keys) {
    for (int64_t i = 0; i < n; ++i)
        keys[i] = gcs_oracle_morton(xyzm[4 * i], xyzm[4 * i + 1], xyzm[4 * i + 2], lo, hi);
}

/* main.cpp:152-166 */
void gcs_oracle_bounds(const float* xyzm, int64_t n, float* lo, float* hi) {
    float mn = INFINITY, mx = -INFINITY;
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float v = xyzm[4 * i + a];
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
    *lo = mn;
    *hi = mx;
}

/* Stable LSD counting sort, 8-bit digits over all 64 bits: the ordering
 * cub::DeviceRadixSort::SortPairs produces (cuda_engine.cu:397). */
void gcs_oracle_sort(const uint64_t* keys, int64_t n, uint64_t* keys_out, uint32_t* idx_out) {
    uint64_t* ka = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    uint32_t* va = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    uint64_t* kb = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    uint32_t* vb = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) {
        ka[i] = keys[i];
        va[i] = (uint32_t)i;
    }
    for (int pass = 0; pass < 8; ++pass) {
        int64_t count[257];
        memset(count, 0, sizeof count);
        const int sh = 8 * pass;
        for (int64_t i = 0; i < n; ++i) count[((ka[i] >> sh) & 255u) + 1]++;
        for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
        for (int64_t i = 0; i < n; ++i) {
            const int64_t p = count[(ka[i] >> sh) & 255u]++;
            kb[p] = ka[i];
            vb[p] = va[i];
        }
        uint64_t* tk = ka;
        ka = kb;
        kb = tk;
        uint32_t* tv = va;
        va = vb;
        vb = tv;
    }
    memcpy(keys_out, ka, sizeof(uint64_t) * (size_t)n);
    memcpy(idx_out, va, sizeof(uint32_t) * (size_t)n);
    free(ka);
    free(va);
    free(kb);
    free(vb);
}

/* karras_bvh.cuh:23-31 */
static int lcp(int i, int j, int n, const uint64_t* k) {
    if (j < 0 || j >= n) return -1;
    if (k[i] == k[j]) return 64 + __builtin_clz((unsigned)(i ^ j));
    return __builtin_clzll(k[i] ^ k[j]);
}

/* karras_bvh.cuh:73-131 */
void gcs_oracle_build(const uint64_t* k, int n, int node_base, int leaf_base, int off,
                      int32_t* child_left, int32_t* child_right, int32_t* range_end,
                      int32_t* parent, int32_t* leaf_parent) {
    if (n < 2) {
        if (n == 1) leaf_parent[0] = -1;
        return;
    }
    parent[0] = -1;
    for (int i = 0; i < n - 1; ++i) {
        const int d = (lcp(i, i + 1, n, k) - lcp(i, i - 1, n, k)) > 0 ? 1 : -1;
        const int dmin = lcp(i, i - d, n, k);
        int lmax = 2;
        while (lcp(i, i + lmax * d, n, k) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (lcp(i, i + (l + t) * d, n, k) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = lcp(i, j, n, k);
        int s = 0, step = l;
        do {
            step = (step + 1) >> 1;
            if (lcp(i, i + (s + step) * d, n, k) > dnode) s += step;
        } while (step > 1);
        const int split = i + s * d + (d > 0 ? 0 : -1);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const int node = node_base + i;
        const int cl = (lo == split) ? leaf_base + split : node_base + split;
        const int cr = (hi == split + 1) ? leaf_base + split + 1 : node_base + split + 1;
        child_left[i] = cl;
        child_right[i] = cr;
        range_end[i] = off + j;
        if (lo == split) leaf_parent[split] = node;
        else parent[split] = node;
        if (hi == split + 1) leaf_parent[split + 1] = node;
        else parent[split + 1] = node;
    }
}

typedef struct {
    float lo[3], hi[3], com[3], m;
    double mx[3], md;
} Agg;

/* karras_bvh.cuh:175-225, evaluated in post-order (the result does not
 * depend on which sibling arrives second). */
void gcs_oracle_aggregate(int n, const float* xyzm, BvhNodeTraverse* nodes, float* box,
                          int com_fp64) {
    if (n < 2) return;
    const int ni = n - 1;
    Agg* agg = (Agg*)malloc(sizeof(Agg) * (size_t)ni);
    /* iterative post-order */
    int* stack = (int*)malloc(sizeof(int) * (size_t)(2 * ni + 2));
    unsigned char* seen = (unsigned char*)calloc((size_t)ni, 1);
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        const int v = stack[top - 1];
        if (!seen[v]) {
            seen[v] = 1;
            const int c[2] = {nodes[v].child_left, nodes[v].child_right};
            for (int s = 0; s < 2; ++s)
                if (c[s] < ni) stack[top++] = c[s];
            continue;
        }
        --top;
        Agg ch[2];
        const int c[2] = {nodes[v].child_left, nodes[v].child_right};
        for (int s = 0; s < 2; ++s) {
            if (c[s] >= ni) {
                const float* p = xyzm + 4 * (size_t)(c[s] - ni);
                for (int a = 0; a < 3; ++a) {
                    ch[s].lo[a] = ch[s].hi[a] = ch[s].com[a] = p[a];
                    ch[s].mx[a] = (double)p[3] * (double)p[a];
                }
                ch[s].m = p[3];
                ch[s].md = p[3];
            } else {
                ch[s] = agg[c[s]];
            }
        }
        Agg r;
        for (int a = 0; a < 3; ++a) {
            r.lo[a] = fminf(ch[0].lo[a], ch[1].lo[a]);
            r.hi[a] = fmaxf(ch[0].hi[a], ch[1].hi[a]);
        }
        const float w = fmaxf(r.hi[0] - r.lo[0], fmaxf(r.hi[1] - r.lo[1], r.hi[2] - r.lo[2]));
        /* particles in the node: its range [min(v, j), max(v, j)] */
        const int re = nodes[v].range_end;
        const int count = (re > v ? re - v : v - re) + 1;
        const int big = com_fp64 && count >= GCS_ORACLE_COM_FP64_MIN;
        r.m = ch[0].m + ch[1].m;
        r.md = ch[0].md + ch[1].md;
        for (int a = 0; a < 3; ++a) r.mx[a] = ch[0].mx[a] + ch[1].mx[a];
        for (int a = 0; a < 3; ++a) {
            if (r.m > 0.0f) {
                if (big) r.com[a] = (float)(r.mx[a] / r.md);
                else r.com[a] = fmaf(ch[0].com[a], ch[0].m, ch[1].com[a] * ch[1].m) / r.m;
            } else {
                r.com[a] = (r.lo[a] + r.hi[a]) * 0.5f;
                r.mx[a] = 0.0;
            }
        }
        if (!(r.m > 0.0f)) r.md = 0.0;
        if (!big && r.m > 0.0f) {
            /* a node below the FP64 size hands its parent the exact double
             * product of its FP32 mass and centre of mass */
            for (int a = 0; a < 3; ++a) r.mx[a] = (double)r.m * (double)r.com[a];
            r.md = (double)r.m;
        }
        agg[v] = r;
        nodes[v].com_x = r.com[0];
        nodes[v].com_y = r.com[1];
        nodes[v].com_z = r.com[2];
        nodes[v].mass = r.m;
        nodes[v].width = w;
        if (box)
            for (int a = 0; a < 3; ++a) {
                box[6 * (size_t)v + a] = r.lo[a];
                box[6 * (size_t)v + 3 + a] = r.hi[a];
            }
    }
    free(seen);
    free(stack);
    free(agg);
}

/* The kernels' softened distance: fma(dz,dz, fma(dy,dy, dx*dx)) + eps^2. */
static float softened_d2(float dx, float dy, float dz, float eps2) {
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx)) + eps2;
}

static void add_term(float gm, float dx, float dy, float dz, float d2, float* a) {
    const float inv = 1.0f / sqrtf(d2);
    const float inv3 = (inv * inv) * inv;
    const float f = gm * inv3;
    a[0] = fmaf(dx, f, a[0]);
    a[1] = fmaf(dy, f, a[1]);
    a[2] = fmaf(dz, f, a[2]);
    a[3] = fmaf(-gm, inv, a[3]);
}

/* cuda_engine.cu:91-161, with theta (criterion width^2 < theta^2 d2,
 * cuda_engine.cu:143) and leaf size L (an opened node of <= L particles is
 * summed directly).  Leaves use the 1.01 eps^2 exclusion
 * (cuda_engine.cu:134).  Depth-first, left pushed before right. */
/* One target's walk (cuda_engine.cu:91-161 with theta and leaf size L):
 * acc4 gets ax, ay, az, potential; nm / np the monopole and particle terms. */
static void walk_one(int t, int n, const float* xyzm, const BvhNodeTraverse* nodes, float G, float eps2,
                     float theta2, float leaf_thr, int leaf_size, float* acc4, int64_t* nm_out, int64_t* np_out) {
    const int ni = n - 1;
    int stack[256];
    const float px = xyzm[4 * (size_t)t], py = xyzm[4 * (size_t)t + 1], pz = xyzm[4 * (size_t)t + 2];
    float a[4] = {0.f, 0.f, 0.f, 0.f};
    int64_t nm = 0, np = 0;
    if (n >= 2) {
        int top = 0;
        stack[top++] = 0;
        while (top > 0) {
            const int c = stack[--top];
            if (c >= ni) {
                const float* q = xyzm + 4 * (size_t)(c - ni);
                const float dx = q[0] - px, dy = q[1] - py, dz = q[2] - pz;
                const float d2 = softened_d2(dx, dy, dz, eps2);
                if (d2 > leaf_thr) {
                    add_term(G * q[3], dx, dy, dz, d2, a);
                    ++np;
                }
                continue;
            }
            const BvhNodeTraverse* nd = nodes + c;
            const float dx = nd->com_x - px, dy = nd->com_y - py, dz = nd->com_z - pz;
            const float d2 = softened_d2(dx, dy, dz, eps2);
            if (nd->width * nd->width < d2 * theta2) {
                add_term(G * nd->mass, dx, dy, dz, d2, a);
                ++nm;
                continue;
            }
            const int own = c, re = nd->range_end;
            const int lo = own < re ? own : re, hi = own < re ? re : own;
            if (hi - lo + 1 <= leaf_size) {
                for (int s = lo; s <= hi; ++s) {
                    const float* q = xyzm + 4 * (size_t)s;
                    const float ex = q[0] - px, ey = q[1] - py, ez = q[2] - pz;
                    const float e2 = softened_d2(ex, ey, ez, eps2);
                    if (e2 > leaf_thr) {
                        add_term(G * q[3], ex, ey, ez, e2, a);
                        ++np;
                    }
                }
                continue;
            }
            if (top + 2 > 256) break; /* deeper than any valid tree of < 2^31 particles */
            stack[top++] = nd->child_left;
            stack[top++] = nd->child_right;
        }
    }
    for (int k = 0; k < 4; ++k) acc4[k] = a[k];
    *nm_out = nm;
    *np_out = np;
}

void gcs_oracle_walk(int n, const float* xyzm, const BvhNodeTraverse* nodes, float G, float eps2,
                     float theta, int leaf_size, float* acc, int64_t* counts) {
    const float theta2 = theta * theta;
    const float leaf_thr = eps2 * 1.01f;
    for (int t = 0; t < n; ++t) {
        int64_t nm, np;
        walk_one(t, n, xyzm, nodes, G, eps2, theta2, leaf_thr, leaf_size, acc + 4 * (size_t)t, &nm, &np);
        if (counts) {
            counts[2 * (size_t)t] = nm;
            counts[2 * (size_t)t + 1] = np;
        }
    }
}

void gcs_oracle_walk_targets(int n, const float* xyzm, const BvhNodeTraverse* nodes, float G, float eps2,
                             float theta, int leaf_size, const int64_t* targets, int64_t n_targets, float* acc,
                             int64_t* counts) {
    const float theta2 = theta * theta;
    const float leaf_thr = eps2 * 1.01f;
    for (int64_t k = 0; k < n_targets; ++k) {
        int64_t nm, np;
        walk_one((int)targets[k], n, xyzm, nodes, G, eps2, theta2, leaf_thr, leaf_size, acc + 4 * (size_t)k, &nm,
                 &np);
        if (counts) {
            counts[2 * (size_t)k] = nm;
            counts[2 * (size_t)k + 1] = np;
        }
    }
}

/* cuda_engine.cu:184-215 */
static uint32_t recolour(uint32_t tcol, float vx, float vy, float vz) {
    const uint32_t type = tcol & 0xFFu;
    if (type != 0u && type != 2u) return tcol;
    const float speed = sqrtf(fmaf(vz, vz, fmaf(vy, vy, vx * vx)));
    const float t = fminf(speed / 150.0f, 1.0f);
    uint32_t r, g, b;
    if (type == 0u) {
        if (t < 0.5f) {
            const float nt = t * 2.0f;
            r = 255u;
            g = (uint8_t)gcs_oracle_f2u_rz(fmaf(150.0f, nt, 50.0f));
            b = 0u;
        } else {
            const float nt = (t - 0.5f) * 2.0f;
            r = 255u;
            g = (uint8_t)gcs_oracle_f2u_rz(fmaf(55.0f, nt, 200.0f));
            b = (uint8_t)gcs_oracle_f2u_rz(150.0f * nt);
        }
    } else {
        if (t < 0.5f) {
            const float nt = t * 2.0f;
            r = 0u;
            g = (uint8_t)gcs_oracle_f2u_rz(fmaf(100.0f, nt, 100.0f));
            b = 255u;
        } else {
            const float nt = (t - 0.5f) * 2.0f;
            r = (uint8_t)gcs_oracle_f2u_rz(200.0f * nt);
            g = (uint8_t)gcs_oracle_f2u_rz(fmaf(55.0f, nt, 200.0f));
            b = 255u;
        }
    }
    return type | (r << 8) | (g << 16) | (b << 24);
}

/* cuda_engine.cu:164-216: v += a dt; x += v dt; recolour. */
void gcs_oracle_integrate(int64_t n, float* xyzm, float* vel4, const float* acc4, float dt,
                          int recolor) {
    for (int64_t i = 0; i < n; ++i) {
        float* p = xyzm + 4 * i;
        float* v = vel4 + 4 * i;
        const float* a = acc4 + 4 * i;
        for (int k = 0; k < 3; ++k) v[k] = fmaf(a[k], dt, v[k]);
        for (int k = 0; k < 3; ++k) p[k] = fmaf(v[k], dt, p[k]);
        if (recolor) {
            uint32_t tc;
            memcpy(&tc, &v[3], 4);
            tc = recolour(tc, v[0], v[1], v[2]);
            memcpy(&v[3], &tc, 4);
        }
    }
}

void gcs_oracle_direct_fp64(int64_t n, const float* xyzm, const int64_t* targets, int64_t n_targets,
                            double G, double eps2, double* out) {
    for (int64_t t = 0; t < n_targets; ++t) {
        const int64_t i = targets[t];
        const double px = xyzm[4 * i], py = xyzm[4 * i + 1], pz = xyzm[4 * i + 2];
        double ax = 0, ay = 0, az = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = xyzm[4 * j] - px, dy = xyzm[4 * j + 1] - py, dz = xyzm[4 * j + 2] - pz;
            const double r2 = dx * dx + dy * dy + dz * dz + eps2;
            const double inv = 1.0 / sqrt(r2);
            const double f = G * (double)xyzm[4 * j + 3] * inv * inv * inv;
            ax += f * dx;
            ay += f * dy;
            az += f * dz;
        }
        out[3 * t] = ax;
        out[3 * t + 1] = ay;
        out[3 * t + 2] = az;
    }
}

/* cuda_engine.cu:379-451 for one segment. */
void gcs_oracle_step(int n, float* xyzm, float* vel4, int use_bounds, float lo, float hi, float G,
                     float eps2, float theta, int leaf_size, float dt, int recolor, int com_fp64,
                     float* acc, BvhNodeTraverse* nodes) {
    if (n < 1) return;
    if (!use_bounds) gcs_oracle_bounds(xyzm, n, &lo, &hi);
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint64_t* sk = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint32_t* idx = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    float* tmp = (float*)malloc(sizeof(float) * 8 * (size_t)n);
    gcs_oracle_encode(xyzm, n, lo, hi, keys);
    gcs_oracle_sort(keys, n, sk, idx);
    for (int i = 0; i < n; ++i) {
        memcpy(tmp + 4 * (size_t)i, xyzm + 4 * (size_t)idx[i], 16);
        memcpy(tmp + 4 * (size_t)n + 4 * (size_t)i, vel4 + 4 * (size_t)idx[i], 16);
    }
    memcpy(xyzm, tmp, 16 * (size_t)n);
    memcpy(vel4, tmp + 4 * (size_t)n, 16 * (size_t)n);
    if (n >= 2) {
        int32_t* cl = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        int32_t* cr = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        int32_t* re = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        int32_t* par = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        int32_t* lp = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        gcs_oracle_build(sk, n, 0, n - 1, 0, cl, cr, re, par, lp);
        for (int i = 0; i < n - 1; ++i) {
            nodes[i].child_left = cl[i];
            nodes[i].child_right = cr[i];
            nodes[i].range_end = re[i];
        }
        gcs_oracle_aggregate(n, xyzm, nodes, NULL, com_fp64);
        free(cl);
        free(cr);
        free(re);
        free(par);
        free(lp);
    }
    gcs_oracle_walk(n, xyzm, nodes, G, eps2, theta, leaf_size, acc, NULL);
    gcs_oracle_integrate(n, xyzm, vel4, acc, dt, recolor);
    free(keys);
    free(sk);
    free(idx);
    free(tmp);
}

/* ---- headless point-splat renderer --------------------------------------
 * The reference's GL point pipeline restated on the CPU, in the operation
 * order of the CUDA splat kernel: vertex shader renderer.cpp:106-122 (view,
 * projection, size by view-space distance), fragment shader
 * renderer.cpp:130-147 (r^2 from gl_PointCoord, exp(-3 r^2), colour and
 * alpha by type), additive blend renderer.cpp:203 over the clear colour
 * renderer.cpp:248.  Fragments are added to acc in 2^-24 units per
 * channel. */
static float row_dot3(const float* m, int r, float x, float y, float z) {
    return fmaf(m[4 * r + 0], x, fmaf(m[4 * r + 1], y, fmaf(m[4 * r + 2], z, m[4 * r + 3])));
}
static float row_dot4(const float* m, int r, float x, float y, float z, float w) {
    return fmaf(m[4 * r + 0], x, fmaf(m[4 * r + 1], y, fmaf(m[4 * r + 2], z, m[4 * r + 3] * w)));
}

void gcs_oracle_render(const Star* stars, int64_t n, const float view[16], const float proj[16], int width,
                       int height, uint64_t* acc, uint8_t* rgba) {
    const float W = (float)width, H = (float)height;
    for (int64_t i = 0; i < n; ++i) {
        const Star* s = stars + i;
        const float vx = row_dot3(view, 0, s->x, s->y, s->z);
        const float vy = row_dot3(view, 1, s->x, s->y, s->z);
        const float vz = row_dot3(view, 2, s->x, s->y, s->z);
        const float vw = row_dot3(view, 3, s->x, s->y, s->z);
        const float dist = sqrtf(fmaf(vz, vz, fmaf(vy, vy, vx * vx)));
        const int dm = s->type == 1;
        const float size = dm ? fminf(fmaxf(2500.0f / dist, 1.0f), 6.0f) : fminf(fmaxf(1000.0f / dist, 1.0f), 3.0f);
        const float cx = row_dot4(proj, 0, vx, vy, vz, vw);
        const float cy = row_dot4(proj, 1, vx, vy, vz, vw);
        const float cz = row_dot4(proj, 2, vx, vy, vz, vw);
        const float cw = row_dot4(proj, 3, vx, vy, vz, vw);
        if (!(cw > 0.0f && fabsf(cx) <= cw && fabsf(cy) <= cw && fabsf(cz) <= cw)) continue;
        const float xw = fmaf(cx / cw, 0.5f * W, 0.5f * W);
        const float yw = fmaf(cy / cw, 0.5f * H, 0.5f * H);
        const float half = size * 0.5f;
        int i0 = (int)ceilf((xw - half) - 0.5f), i1 = (int)ceilf((xw + half) - 0.5f) - 1;
        int j0 = (int)ceilf((yw - half) - 0.5f), j1 = (int)ceilf((yw + half) - 0.5f) - 1;
        if (i0 < 0) i0 = 0;
        if (j0 < 0) j0 = 0;
        if (i1 > width - 1) i1 = width - 1;
        if (j1 > height - 1) j1 = height - 1;
        float cr, cg, cb, amul;
        if (dm) {
            cr = 0.4f;
            cg = 0.0f;
            cb = 0.8f;
            amul = 0.03f;
        } else {
            cr = (float)s->r / 255.0f;
            cg = (float)s->g / 255.0f;
            cb = (float)s->b / 255.0f;
            amul = 0.15f;
        }
        for (int pj = j0; pj <= j1; ++pj) {
            const float py = (2.0f * (((float)pj + 0.5f) - yw)) / size;
            for (int pi = i0; pi <= i1; ++pi) {
                const float px = (2.0f * (((float)pi + 0.5f) - xw)) / size;
                const float r2 = fmaf(py, py, px * px);
                if (r2 > 1.0f) continue;
                const float a = expf(-r2 * 3.0f) * amul;
                uint64_t* p = acc + 3 * ((size_t)pj * width + pi);
                p[0] += (uint64_t)llrintf((cr * a) * 16777216.0f);
                p[1] += (uint64_t)llrintf((cg * a) * 16777216.0f);
                p[2] += (uint64_t)llrintf((cb * a) * 16777216.0f);
            }
        }
    }
    if (!rgba) return;
    const double clear[3] = {(double)0.01f, (double)0.01f, (double)0.02f};
    for (int64_t p = 0; p < (int64_t)width * height; ++p) {
        for (int k = 0; k < 3; ++k) {
            double v = clear[k] + (double)acc[3 * p + k] * (1.0 / 16777216.0);
            if (v > 1.0) v = 1.0;
            rgba[4 * p + k] = (uint8_t)nearbyint(v * 255.0);
        }
        rgba[4 * p + 3] = 255;
    }
}
