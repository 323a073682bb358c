/*
 * oracle_host.cpp -- TEST INFRASTRUCTURE (oracle).  Java host logic of the
 * render path restated in C++ (see oracle_host.h for the float rules).
 */
#include "oracle_host.h"

#include <algorithm>

namespace oracle {

static rc_triangle blank_tri() {
    rc_triangle t;
    memset(&t, 0, sizeof(t));
    return t;
}

/* Box.java:93-120 addQuad: (a,b,c) and (a,c,d) with fixed UVs. */
static void add_quad(std::vector<rc_triangle>& out, int mat,
                     float ax, float ay, float az, float bx, float by, float bz,
                     float cx, float cy, float cz, float dx, float dy, float dz) {
    rc_triangle t1 = blank_tri();
    t1.v0[0] = ax; t1.v0[1] = ay; t1.v0[2] = az;
    t1.v1[0] = bx; t1.v1[1] = by; t1.v1[2] = bz;
    t1.v2[0] = cx; t1.v2[1] = cy; t1.v2[2] = cz;
    t1.uv0[0] = 0; t1.uv0[1] = 0; t1.uv1[0] = 0; t1.uv1[1] = 1; t1.uv2[0] = 1; t1.uv2[1] = 1;
    t1.mat_index = mat;
    with_flat_normal(t1);
    rc_triangle t2 = blank_tri();
    t2.v0[0] = ax; t2.v0[1] = ay; t2.v0[2] = az;
    t2.v1[0] = cx; t2.v1[1] = cy; t2.v1[2] = cz;
    t2.v2[0] = dx; t2.v2[1] = dy; t2.v2[2] = dz;
    t2.uv0[0] = 0; t2.uv0[1] = 0; t2.uv1[0] = 1; t2.uv1[1] = 1; t2.uv2[0] = 1; t2.uv2[1] = 0;
    t2.mat_index = mat;
    with_flat_normal(t2);
    out.push_back(t1);
    out.push_back(t2);
}

/* Box.java:69-90: faces +X, -X, +Y, -Y, +Z, -Z. */
void tess_box(float cx, float cy, float cz, float hx, float hy, float hz, int mat,
              std::vector<rc_triangle>& out) {
    const float x0 = cx - hx, x1 = cx + hx;
    const float y0 = cy - hy, y1 = cy + hy;
    const float z0 = cz - hz, z1 = cz + hz;
    add_quad(out, mat, x1, y0, z1, x1, y1, z1, x1, y1, z0, x1, y0, z0);
    add_quad(out, mat, x0, y0, z0, x0, y1, z0, x0, y1, z1, x0, y0, z1);
    add_quad(out, mat, x0, y1, z1, x0, y1, z0, x1, y1, z0, x1, y1, z1);
    add_quad(out, mat, x0, y0, z0, x0, y0, z1, x1, y0, z1, x1, y0, z0);
    add_quad(out, mat, x0, y0, z1, x0, y1, z1, x1, y1, z1, x1, y0, z1);
    add_quad(out, mat, x1, y0, z0, x1, y1, z0, x0, y1, z0, x0, y0, z0);
}

/* Sphere.java:85-93 spherePt. */
static void sphere_pt(float cx, float cy, float cz, float radius, float phi, float theta, float p[3]) {
    const float sinP = (float)sin((double)phi);
    p[0] = cx + radius * sinP * (float)cos((double)theta);
    p[1] = cy + radius * (float)cos((double)phi);
    p[2] = cz + radius * sinP * (float)sin((double)theta);
}

/* Sphere.java:114-123 setNormal. */
static void sphere_normal(float cx, float cy, float cz, const float p[3], float n[3]) {
    float nx = p[0] - cx, ny = p[1] - cy, nz = p[2] - cz;
    float len = jsqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 1e-8f) { nx /= len; ny /= len; nz /= len; }
    n[0] = nx; n[1] = ny; n[2] = nz;
}

static rc_triangle sphere_tri(float cx, float cy, float cz, int mat, const float* p0, const float* p1,
                              const float* p2, const float* uv0, const float* uv1, const float* uv2) {
    rc_triangle t = blank_tri();
    for (int k = 0; k < 3; ++k) { t.v0[k] = p0[k]; t.v1[k] = p1[k]; t.v2[k] = p2[k]; }
    sphere_normal(cx, cy, cz, p0, t.n0);
    sphere_normal(cx, cy, cz, p1, t.n1);
    sphere_normal(cx, cy, cz, p2, t.n2);
    t.uv0[0] = uv0[0]; t.uv0[1] = uv0[1];
    t.uv1[0] = uv1[0]; t.uv1[1] = uv1[1];
    t.uv2[0] = uv2[0]; t.uv2[1] = uv2[1];
    t.mat_index = mat;
    return t;
}

/* Sphere.java:54-83. */
void tess_sphere(float cx, float cy, float cz, float radius, int mat, int stacks, int slices,
                 std::vector<rc_triangle>& out) {
    const double PI = 3.141592653589793;
    for (int i = 0; i < stacks; ++i) {
        const float phi0 = (float)(PI * i / stacks);
        const float phi1 = (float)(PI * (i + 1) / stacks);
        for (int j = 0; j < slices; ++j) {
            const float theta0 = (float)(2 * PI * j / slices);
            const float theta1 = (float)(2 * PI * (j + 1) / slices);
            float A[3], B[3], C[3], D[3];
            sphere_pt(cx, cy, cz, radius, phi0, theta0, A);
            sphere_pt(cx, cy, cz, radius, phi0, theta1, B);
            sphere_pt(cx, cy, cz, radius, phi1, theta1, C);
            sphere_pt(cx, cy, cz, radius, phi1, theta0, D);
            const float uvA[2] = {(float)j / slices, (float)i / stacks};
            const float uvB[2] = {(float)(j + 1) / slices, (float)i / stacks};
            const float uvC[2] = {(float)(j + 1) / slices, (float)(i + 1) / stacks};
            const float uvD[2] = {(float)j / slices, (float)(i + 1) / stacks};
            if (i != 0) out.push_back(sphere_tri(cx, cy, cz, mat, A, B, C, uvA, uvB, uvC));
            if (i != stacks - 1) out.push_back(sphere_tri(cx, cy, cz, mat, A, C, D, uvA, uvC, uvD));
        }
    }
}

/* TransformedPrimitive.java:80-95: Rz*Ry*Rx, column-major.  Java 9+
 * Math.toRadians multiplies by the double nearest pi/180. */
static void build_rotation(float degx, float degy, float degz, float rot[9]) {
    const double D2R = 0.017453292519943295;
    const double rx = (double)degx * D2R, ry = (double)degy * D2R, rz = (double)degz * D2R;
    const float cx = (float)cos(rx), sx = (float)sin(rx);
    const float cy = (float)cos(ry), sy = (float)sin(ry);
    const float cz = (float)cos(rz), sz = (float)sin(rz);
    rot[0] = cy * cz;              rot[1] = cy * sz;              rot[2] = -sy;
    rot[3] = sx * sy * cz - cx * sz; rot[4] = sx * sy * sz + cx * cz; rot[5] = sx * cy;
    rot[6] = cx * sy * cz + sx * sz; rot[7] = cx * sy * sz - sx * cz; rot[8] = cx * cy;
}

static void rot_vec(const float r[9], float x, float y, float z, float o[3]) {
    o[0] = r[0] * x + r[3] * y + r[6] * z;
    o[1] = r[1] * x + r[4] * y + r[7] * z;
    o[2] = r[2] * x + r[5] * y + r[8] * z;
}

/* TransformedPrimitive.java:32-65. */
void rotate_about(std::vector<rc_triangle>& tris, size_t first, float cx, float cy, float cz,
                  float degx, float degy, float degz) {
    float R[9];
    build_rotation(degx, degy, degz, R);
    for (size_t i = first; i < tris.size(); ++i) {
        rc_triangle& t = tris[i];
        float v[3];
        float* verts[3] = {t.v0, t.v1, t.v2};
        for (int k = 0; k < 3; ++k) {
            rot_vec(R, verts[k][0] - cx, verts[k][1] - cy, verts[k][2] - cz, v);
            verts[k][0] = v[0] + cx; verts[k][1] = v[1] + cy; verts[k][2] = v[2] + cz;
        }
        float* norms[3] = {t.n0, t.n1, t.n2};
        for (int k = 0; k < 3; ++k) {
            rot_vec(R, norms[k][0], norms[k][1], norms[k][2], v);
            norms[k][0] = v[0]; norms[k][1] = v[1]; norms[k][2] = v[2];
        }
    }
}

/* ---------------------------------------------------------------------
 * BVHBuilder.java
 * ------------------------------------------------------------------- */
namespace {

struct Box3 {
    float mn[3], mx[3];
};

struct JNode {
    float mn[3], mx[3];
    int left = -1, right = -1, prim_start = 0, prim_count = 0;
};

/* BVHNode.java:56-61. */
float surface_area(const float mn[3], const float mx[3]) {
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

/* BVHBuilder.java:182-202 Bucket. */
struct Bucket {
    int count = 0;
    float mn[3] = {JFLOAT_MAX, JFLOAT_MAX, JFLOAT_MAX};
    float mx[3] = {-JFLOAT_MAX, -JFLOAT_MAX, -JFLOAT_MAX};
    void expand(const rc_triangle& t) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = jmin(mn[a], tri_min(t, a));
            mx[a] = jmax(mx[a], tri_max(t, a));
        }
    }
    void merge(const Bucket& o) {
        count += o.count;
        if (o.count == 0) return;
        for (int a = 0; a < 3; ++a) {
            mn[a] = jmin(mn[a], o.mn[a]);
            mx[a] = jmax(mx[a], o.mx[a]);
        }
    }
    float sa() const {
        if (count == 0) return 0.0f;
        return surface_area(mn, mx);
    }
};

struct Builder {
    std::vector<rc_triangle>& tris;
    std::vector<JNode> nodes;
    explicit Builder(std::vector<rc_triangle>& t) : tris(t) {}

    /* BVHNode.java:58-64 fromTriangles. */
    JNode from_triangles(int start, int count) {
        JNode n;
        for (int a = 0; a < 3; ++a) { n.mn[a] = JFLOAT_MAX; n.mx[a] = -JFLOAT_MAX; }
        for (int i = start; i < start + count; ++i)
            for (int a = 0; a < 3; ++a) {
                n.mn[a] = jmin(n.mn[a], tri_min(tris[i], a));
                n.mx[a] = jmax(n.mx[a], tri_max(tris[i], a));
            }
        return n;
    }

    /* BVHBuilder.java:100-145. Returns false when no split exists. */
    bool find_best_split(const JNode& parent, int start, int count, int& best_axis,
                         float& best_pos, float& best_cost) {
        const float parent_sa = surface_area(parent.mn, parent.mx);
        if (parent_sa < 1e-8f) return false;
        bool have = false;
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = parent.mn[axis], hi = parent.mx[axis];
            if (hi - lo < 1e-6f) continue;
            Bucket b[8];
            for (int i = start; i < start + count; ++i) {
                const float c = tri_centroid(tris[i], axis);
                int k = (int)(8.0f * (c - lo) / (hi - lo));
                if (k > 7) k = 7;
                if (k < 0) k = 0; /* Java's (int)NaN is 0 */
                b[k].count++;
                b[k].expand(tris[i]);
            }
            for (int s = 0; s < 7; ++s) {
                Bucket left, right;
                for (int i = 0; i <= s; ++i) left.merge(b[i]);
                for (int i = s + 1; i < 8; ++i) right.merge(b[i]);
                if (left.count == 0 || right.count == 0) continue;
                const float cost = 1.0f + (left.sa() * (float)left.count * 1.5f) / parent_sa
                                 + (right.sa() * (float)right.count * 1.5f) / parent_sa;
                const float split_pos = lo + (hi - lo) * (float)(s + 1) / 8.0f;
                if (!have || cost < best_cost) {
                    have = true;
                    best_axis = axis; best_pos = split_pos; best_cost = cost;
                }
            }
        }
        return have;
    }

    /* BVHBuilder.java:150-164. */
    int partition(int start, int count, int axis, float split_pos) {
        int lo = start, hi = start + count - 1;
        while (lo <= hi) {
            if (tri_centroid(tris[lo], axis) < split_pos) {
                lo++;
            } else {
                std::swap(tris[lo], tris[hi]);
                hi--;
            }
        }
        return lo;
    }

    /* BVHBuilder.java:61-96. */
    int subdivide(int start, int count) {
        const int idx = (int)nodes.size();
        nodes.push_back(from_triangles(start, count));
        if (count <= 4) {
            nodes[idx].prim_start = start; nodes[idx].prim_count = count;
            return idx;
        }
        int axis = 0; float pos = 0.0f, cost = 0.0f;
        const bool have = find_best_split(nodes[idx], start, count, axis, pos, cost);
        const float leaf_cost = 1.5f * (float)count;
        if (!have || cost >= leaf_cost) {
            nodes[idx].prim_start = start; nodes[idx].prim_count = count;
            return idx;
        }
        const int mid = partition(start, count, axis, pos);
        if (mid == start || mid == start + count) {
            nodes[idx].prim_start = start; nodes[idx].prim_count = count;
            return idx;
        }
        const int l = subdivide(start, mid - start);
        const int r = subdivide(mid, start + count - mid);
        nodes[idx].left = l;
        nodes[idx].right = r;
        return idx;
    }
};

}  // namespace

void build_bvh(std::vector<rc_triangle>& tris, std::vector<rc_bvh_node>& out) {
    Builder b(tris);
    b.subdivide(0, (int)tris.size());
    out.resize(b.nodes.size());
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        const JNode& n = b.nodes[i];
        rc_bvh_node& o = out[i];
        memset(&o, 0, sizeof(o));
        for (int a = 0; a < 3; ++a) { o.aabb_min[a] = n.mn[a]; o.aabb_max[a] = n.mx[a]; }
        o.left_child = n.left; o.right_child = n.right;
        o.prim_start = n.prim_start; o.prim_count = n.prim_count;
    }
}

/* SceneUploader.java:144-216. */
void build_lights(const std::vector<rc_triangle>& tris, const rc_material* mats,
                  std::vector<rc_light>& lights, float& total_power) {
    lights.clear();
    float sum = 0.0f;
    for (const rc_triangle& t : tris) {
        const rc_material& m = mats[t.mat_index];
        if (m.emission_strength <= 0.0f) continue;
        const float e1x = t.v1[0] - t.v0[0], e1y = t.v1[1] - t.v0[1], e1z = t.v1[2] - t.v0[2];
        const float e2x = t.v2[0] - t.v0[0], e2y = t.v2[1] - t.v0[1], e2z = t.v2[2] - t.v0[2];
        const float cx = e1y * e2z - e1z * e2y;
        const float cy = e1z * e2x - e1x * e2z;
        const float cz = e1x * e2y - e1y * e2x;
        const float area = 0.5f * jsqrtf(cx * cx + cy * cy + cz * cz);
        if (area < 1e-8f) continue;
        const float er = m.emission[0] * m.emission_strength;
        const float eg = m.emission[1] * m.emission_strength;
        const float eb = m.emission[2] * m.emission_strength;
        const float lum = 0.299f * er + 0.587f * eg + 0.114f * eb;
        const float power = lum * area * (float)3.141592653589793;
        sum += power;
        rc_light L;
        memset(&L, 0, sizeof(L));
        for (int a = 0; a < 3; ++a) { L.v0[a] = t.v0[a]; L.v1[a] = t.v1[a]; L.v2[a] = t.v2[a]; }
        L.area = area;
        L.emission[0] = er; L.emission[1] = eg; L.emission[2] = eb;
        L.power = power;
        L.normal[0] = t.n0[0]; L.normal[1] = t.n0[1]; L.normal[2] = t.n0[2];
        lights.push_back(L);
    }
    total_power = sum;
    if (lights.empty()) return;
    float cumulative = 0.0f;
    for (rc_light& L : lights) {
        cumulative += L.power;
        L.cdf_weight = (sum > 0.0f) ? cumulative / sum : 1.0f;
    }
    lights.back().cdf_weight = 1.0f;
}

}  // namespace oracle
