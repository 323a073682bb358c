/*
 * oracle_host.h -- TEST INFRASTRUCTURE (oracle).  Restatement of the
 * reference's Java host logic on the render path, with Java's strict float
 * semantics: IEEE single operations evaluated left to right with no fused
 * multiply-add (build with -ffp-contract=off), (int) casts truncating,
 * Math.sqrt/sin/cos/tan/atan evaluated in double and cast to float, and
 * Math.min/max(float) with Java's NaN and signed-zero rules.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this.
 */
#ifndef RC_ORACLE_HOST_H
#define RC_ORACLE_HOST_H

#include <math.h>
#include <stdint.h>
#include <string.h>
#include <vector>

#include "retrocam.h"

namespace oracle {

/* java.lang.Math.min(float,float) / max(float,float). */
static inline bool neg_zero(float f) { uint32_t u; memcpy(&u, &f, 4); return u == 0x80000000u; }
static inline float jmin(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f && neg_zero(b)) return b;
    return (a <= b) ? a : b;
}
static inline float jmax(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f && neg_zero(a)) return b;
    return (a >= b) ? a : b;
}
static inline float jsqrtf(float x) { return (float)sqrt((double)x); }
static const float JFLOAT_MAX = 3.4028234663852886e38f;

/* scene/GpuTriangle.java:38-50. */
static inline void with_flat_normal(rc_triangle& t) {
    float ax = t.v1[0] - t.v0[0], ay = t.v1[1] - t.v0[1], az = t.v1[2] - t.v0[2];
    float bx = t.v2[0] - t.v0[0], by = t.v2[1] - t.v0[1], bz = t.v2[2] - t.v0[2];
    float nx = ay * bz - az * by;
    float ny = az * bx - ax * bz;
    float nz = ax * by - ay * bx;
    float len = jsqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 1e-8f) { nx /= len; ny /= len; nz /= len; }
    t.n0[0] = t.n1[0] = t.n2[0] = nx;
    t.n0[1] = t.n1[1] = t.n2[1] = ny;
    t.n0[2] = t.n1[2] = t.n2[2] = nz;
}

/* scene/GpuTriangle.java:53-66. */
static inline float tri_min(const rc_triangle& t, int a) { return jmin(t.v0[a], jmin(t.v1[a], t.v2[a])); }
static inline float tri_max(const rc_triangle& t, int a) { return jmax(t.v0[a], jmax(t.v1[a], t.v2[a])); }
static inline float tri_centroid(const rc_triangle& t, int a) { return (t.v0[a] + t.v1[a] + t.v2[a]) / 3.0f; }

/* scene/Box.java:25-76. */
void tess_box(float cx, float cy, float cz, float hx, float hy, float hz, int mat,
              std::vector<rc_triangle>& out);
/* scene/Sphere.java:34-101. */
void tess_sphere(float cx, float cy, float cz, float radius, int mat, int stacks, int slices,
                 std::vector<rc_triangle>& out);
/* scene/TransformedPrimitive.java:32-95 applied in place to tris[first..]. */
void rotate_about(std::vector<rc_triangle>& tris, size_t first, float cx, float cy, float cz,
                  float degx, float degy, float degz);
/* scene/BVHBuilder.java:35-202. */
void build_bvh(std::vector<rc_triangle>& tris, std::vector<rc_bvh_node>& nodes);
/* scene/SceneUploader.java:144-216. */
void build_lights(const std::vector<rc_triangle>& tris, const rc_material* mats,
                  std::vector<rc_light>& lights, float& total_power);

}  // namespace oracle

#endif
