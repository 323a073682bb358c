// host_scene.cpp -- host half of the C ABI: the scene logic the reference
// runs in Java before its SSBO upload, with Java's float semantics so the
// outputs are bit-identical to what the Java host would upload.
//
// Float rules: IEEE single, left-to-right evaluation, no contraction (this
// file is compiled with -ffp-contract=off); Math.sqrt/sin/cos/tan/atan are
// evaluated in double and rounded to float; Math.min/max(float) keep Java's
// NaN and signed-zero behaviour.
//
// The BVH builder (scene/BVHBuilder.java:35-202) works on an index
// permutation with per-triangle bounds and centroids computed once, instead
// of re-deriving them from the triangle records at every level.  Bounds
// reductions use min/max, which are order-independent under Java's rules, so
// the node boxes, SAH costs and the in-place partition (which alone fixes the
// triangle order) are those of the reference.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "retrocam.h"

namespace rc_host {

static inline bool is_neg_zero(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u == 0x80000000u;
}
// java.lang.Math.min/max(float, float)
static inline float jmin(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f && is_neg_zero(b)) return b;
    return (a <= b) ? a : b;
}
static inline float jmax(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f && is_neg_zero(a)) return b;
    return (a >= b) ? a : b;
}
static inline float dsqrtf(float x) { return (float)sqrt((double)x); }
static const float kFloatMax = 3.4028234663852886e38f;

// GpuTriangle.withFlatNormal (scene/GpuTriangle.java:38-50)
static void flat_normal(rc_triangle& t) {
    const float ax = t.v1[0] - t.v0[0], ay = t.v1[1] - t.v0[1], az = t.v1[2] - t.v0[2];
    const float bx = t.v2[0] - t.v0[0], by = t.v2[1] - t.v0[1], bz = t.v2[2] - t.v0[2];
    float nx = ay * bz - az * by;
    float ny = az * bx - ax * bz;
    float nz = ax * by - ay * bx;
    const float len = dsqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 1e-8f) {
        nx /= len;
        ny /= len;
        nz /= len;
    }
    for (float* n : {t.n0, t.n1, t.n2}) {
        n[0] = nx;
        n[1] = ny;
        n[2] = nz;
    }
}

static rc_triangle make_tri(const float* a, const float* b, const float* c) {
    rc_triangle t;
    memset(&t, 0, sizeof(t));
    for (int k = 0; k < 3; ++k) {
        t.v0[k] = a[k];
        t.v1[k] = b[k];
        t.v2[k] = c[k];
    }
    return t;
}

// scene/Box.java:69-120: six faces, two triangles each, flat normals.
static void box(float cx, float cy, float cz, float hx, float hy, float hz, int mat, rc_triangle* out) {
    const float x0 = cx - hx, x1 = cx + hx;
    const float y0 = cy - hy, y1 = cy + hy;
    const float z0 = cz - hz, z1 = cz + hz;
    const float q[6][4][3] = {
        {{x1, y0, z1}, {x1, y1, z1}, {x1, y1, z0}, {x1, y0, z0}},
        {{x0, y0, z0}, {x0, y1, z0}, {x0, y1, z1}, {x0, y0, z1}},
        {{x0, y1, z1}, {x0, y1, z0}, {x1, y1, z0}, {x1, y1, z1}},
        {{x0, y0, z0}, {x0, y0, z1}, {x1, y0, z1}, {x1, y0, z0}},
        {{x0, y0, z1}, {x0, y1, z1}, {x1, y1, z1}, {x1, y0, z1}},
        {{x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0}, {x0, y0, z0}},
    };
    for (int f = 0; f < 6; ++f) {
        rc_triangle t1 = make_tri(q[f][0], q[f][1], q[f][2]);
        t1.uv1[1] = 1.0f;
        t1.uv2[0] = 1.0f;
        t1.uv2[1] = 1.0f;
        t1.mat_index = mat;
        flat_normal(t1);
        rc_triangle t2 = make_tri(q[f][0], q[f][2], q[f][3]);
        t2.uv1[0] = 1.0f;
        t2.uv1[1] = 1.0f;
        t2.uv2[0] = 1.0f;
        t2.mat_index = mat;
        flat_normal(t2);
        out[2 * f] = t1;
        out[2 * f + 1] = t2;
    }
}

// scene/Sphere.java:54-123
static int sphere(float cx, float cy, float cz, float radius, int mat, int stacks, int slices,
                  rc_triangle* out, int cap) {
    const double PI = 3.141592653589793;
    auto pt = [&](float phi, float theta, float* p) {
        const float s = (float)sin((double)phi);
        p[0] = cx + radius * s * (float)cos((double)theta);
        p[1] = cy + radius * (float)cos((double)phi);
        p[2] = cz + radius * s * (float)sin((double)theta);
    };
    auto nrm = [&](const float* p, float* n) {
        float nx = p[0] - cx, ny = p[1] - cy, nz = p[2] - cz;
        const float len = dsqrtf(nx * nx + ny * ny + nz * nz);
        if (len > 1e-8f) {
            nx /= len;
            ny /= len;
            nz /= len;
        }
        n[0] = nx;
        n[1] = ny;
        n[2] = nz;
    };
    auto tri = [&](const float* p0, const float* p1, const float* p2, const float* u0, const float* u1,
                   const float* u2) {
        rc_triangle t = make_tri(p0, p1, p2);
        nrm(p0, t.n0);
        nrm(p1, t.n1);
        nrm(p2, t.n2);
        t.uv0[0] = u0[0]; t.uv0[1] = u0[1];
        t.uv1[0] = u1[0]; t.uv1[1] = u1[1];
        t.uv2[0] = u2[0]; t.uv2[1] = u2[1];
        t.mat_index = mat;
        return t;
    };
    int n = 0;
    for (int i = 0; i < stacks; ++i) {
        const float phi0 = (float)(PI * i / stacks);
        const float phi1 = (float)(PI * (i + 1) / stacks);
        for (int j = 0; j < slices; ++j) {
            const float th0 = (float)(2 * PI * j / slices);
            const float th1 = (float)(2 * PI * (j + 1) / slices);
            float A[3], B[3], Cc[3], D[3];
            pt(phi0, th0, A);
            pt(phi0, th1, B);
            pt(phi1, th1, Cc);
            pt(phi1, th0, D);
            const float uA[2] = {(float)j / slices, (float)i / stacks};
            const float uB[2] = {(float)(j + 1) / slices, (float)i / stacks};
            const float uC[2] = {(float)(j + 1) / slices, (float)(i + 1) / stacks};
            const float uD[2] = {(float)j / slices, (float)(i + 1) / stacks};
            if (i != 0) {
                if (n >= cap) return -1;
                out[n++] = tri(A, B, Cc, uA, uB, uC);
            }
            if (i != stacks - 1) {
                if (n >= cap) return -1;
                out[n++] = tri(A, Cc, D, uA, uC, uD);
            }
        }
    }
    return n;
}

// scene/TransformedPrimitive.java:32-95 (R = Rz Ry Rx, column-major; Java 9+
// Math.toRadians multiplies by the double nearest pi/180).
static void rotate(rc_triangle* t, int n, float cx, float cy, float cz, float dx, float dy, float dz) {
    const double k = 0.017453292519943295;
    const double ax = (double)dx * k, ay = (double)dy * k, az = (double)dz * k;
    const float c_x = (float)cos(ax), s_x = (float)sin(ax);
    const float c_y = (float)cos(ay), s_y = (float)sin(ay);
    const float c_z = (float)cos(az), s_z = (float)sin(az);
    const float R[9] = {c_y * c_z, c_y * s_z, -s_y,
                        s_x * s_y * c_z - c_x * s_z, s_x * s_y * s_z + c_x * c_z, s_x * c_y,
                        c_x * s_y * c_z + s_x * s_z, c_x * s_y * s_z - s_x * c_z, c_x * c_y};
    auto mv = [&](float x, float y, float z, float* o) {
        o[0] = R[0] * x + R[3] * y + R[6] * z;
        o[1] = R[1] * x + R[4] * y + R[7] * z;
        o[2] = R[2] * x + R[5] * y + R[8] * z;
    };
    for (int i = 0; i < n; ++i) {
        float o[3];
        for (float* v : {t[i].v0, t[i].v1, t[i].v2}) {
            mv(v[0] - cx, v[1] - cy, v[2] - cz, o);
            v[0] = o[0] + cx;
            v[1] = o[1] + cy;
            v[2] = o[2] + cz;
        }
        for (float* v : {t[i].n0, t[i].n1, t[i].n2}) {
            mv(v[0], v[1], v[2], o);
            v[0] = o[0];
            v[1] = o[1];
            v[2] = o[2];
        }
    }
}

// ---------------------------------------------------------------------------
// SAH BVH
// ---------------------------------------------------------------------------
struct Bounds {
    float mn[3], mx[3];
    void reset() {
        for (int a = 0; a < 3; ++a) {
            mn[a] = kFloatMax;
            mx[a] = -kFloatMax;
        }
    }
    void grow(const Bounds& o) {
        for (int a = 0; a < 3; ++a) {
            mn[a] = jmin(mn[a], o.mn[a]);
            mx[a] = jmax(mx[a], o.mx[a]);
        }
    }
    float area() const {  // BVHNode.surfaceArea / Bucket.sa
        const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

class SahBuilder {
public:
    SahBuilder(const rc_triangle* tris, int n) : n_(n), box_(n), cen_(3 * (size_t)n), perm_(n) {
        for (int i = 0; i < n; ++i) {
            const rc_triangle& t = tris[i];
            for (int a = 0; a < 3; ++a) {
                box_[i].mn[a] = jmin(t.v0[a], jmin(t.v1[a], t.v2[a]));
                box_[i].mx[a] = jmax(t.v0[a], jmax(t.v1[a], t.v2[a]));
                cen_[3 * (size_t)i + a] = (t.v0[a] + t.v1[a] + t.v2[a]) / 3.0f;
            }
            perm_[i] = i;
        }
        nodes_.reserve(2 * (size_t)n + 1);
    }

    void build() { subdivide(0, n_); }

    const std::vector<int>& perm() const { return perm_; }
    const std::vector<rc_bvh_node>& nodes() const { return nodes_; }

private:
    float centroid(int slot, int axis) const { return cen_[3 * (size_t)perm_[slot] + axis]; }

    int subdivide(int start, int count) {
        const int idx = (int)nodes_.size();
        Bounds nb;
        nb.reset();
        for (int i = start; i < start + count; ++i) nb.grow(box_[perm_[i]]);
        rc_bvh_node node;
        memset(&node, 0, sizeof(node));
        for (int a = 0; a < 3; ++a) {
            node.aabb_min[a] = nb.mn[a];
            node.aabb_max[a] = nb.mx[a];
        }
        node.left_child = -1;
        node.right_child = -1;
        nodes_.push_back(node);
        if (count <= 4) return make_leaf(idx, start, count);
        int axis = 0;
        float pos = 0.0f, cost = 0.0f;
        if (!best_split(nb, start, count, axis, pos, cost) || cost >= 1.5f * (float)count)
            return make_leaf(idx, start, count);
        // BVHBuilder.partition: in-place, unstable; this order is the output order.
        int lo = start, hi = start + count - 1;
        while (lo <= hi) {
            if (centroid(lo, axis) < pos) {
                ++lo;
            } else {
                std::swap(perm_[lo], perm_[hi]);
                --hi;
            }
        }
        const int mid = lo;
        if (mid == start || mid == start + count) return make_leaf(idx, start, count);
        const int l = subdivide(start, mid - start);
        const int r = subdivide(mid, start + count - mid);
        nodes_[idx].left_child = l;
        nodes_[idx].right_child = r;
        return idx;
    }

    int make_leaf(int idx, int start, int count) {
        nodes_[idx].prim_start = start;
        nodes_[idx].prim_count = count;
        return idx;
    }

    // BVHBuilder.findBestSplit: 8 buckets per axis, 7 candidate planes,
    // first strict minimum in axis order x, y, z.
    bool best_split(const Bounds& parent, int start, int count, int& best_axis, float& best_pos,
                    float& best_cost) {
        const float psa = parent.area();
        if (psa < 1e-8f) return false;
        bool have = false;
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = parent.mn[axis], hi = parent.mx[axis];
            if (hi - lo < 1e-6f) continue;
            int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            Bounds bb[8];
            for (int k = 0; k < 8; ++k) bb[k].reset();
            const float ext = hi - lo;
            for (int i = start; i < start + count; ++i) {
                int k = (int)(8.0f * (centroid(i, axis) - lo) / ext);
                if (k > 7) k = 7;
                if (k < 0) k = 0;
                cnt[k]++;
                bb[k].grow(box_[perm_[i]]);
            }
            // prefix (left) and suffix (right) merges of non-empty buckets
            Bounds lb[8], rb[8];
            int lc[8], rcnt[8];
            Bounds acc;
            acc.reset();
            int c = 0;
            for (int k = 0; k < 8; ++k) {
                c += cnt[k];
                if (cnt[k]) acc.grow(bb[k]);
                lb[k] = acc;
                lc[k] = c;
            }
            acc.reset();
            c = 0;
            for (int k = 7; k >= 0; --k) {
                c += cnt[k];
                if (cnt[k]) acc.grow(bb[k]);
                rb[k] = acc;
                rcnt[k] = c;
            }
            for (int s = 0; s < 7; ++s) {
                const int nl = lc[s], nr = rcnt[s + 1];
                if (nl == 0 || nr == 0) continue;
                const float cst = 1.0f + (lb[s].area() * (float)nl * 1.5f) / psa
                                + (rb[s + 1].area() * (float)nr * 1.5f) / psa;
                const float sp = lo + (hi - lo) * (float)(s + 1) / 8.0f;
                if (!have || cst < best_cost) {
                    have = true;
                    best_axis = axis;
                    best_pos = sp;
                    best_cost = cst;
                }
            }
        }
        return have;
    }

    int n_;
    std::vector<Bounds> box_;
    std::vector<float> cen_;
    std::vector<int> perm_;
    std::vector<rc_bvh_node> nodes_;
};

}  // namespace rc_host

using namespace rc_host;

extern "C" {

int rc_abi_version(void) { return RC_ABI_VERSION; }

int rc_tessellate_box(float cx, float cy, float cz, float hx, float hy, float hz, int mat_index, float rx,
                      float ry, float rz, rc_triangle* out12) {
    if (!out12) return RC_ERR_INVALID_ARG;
    box(cx, cy, cz, hx, hy, hz, mat_index, out12);
    if (rx != 0.0f || ry != 0.0f || rz != 0.0f) rotate(out12, 12, cx, cy, cz, rx, ry, rz);
    return RC_OK;
}

int rc_tessellate_sphere(float cx, float cy, float cz, float radius, int mat_index, int stacks, int slices,
                         float rx, float ry, float rz, rc_triangle* out, int capacity, int* count) {
    if (!out || !count || stacks < 1 || slices < 1) return RC_ERR_INVALID_ARG;
    const int n = sphere(cx, cy, cz, radius, mat_index, stacks, slices, out, capacity);
    if (n < 0) return RC_ERR_CAPACITY;
    if (rx != 0.0f || ry != 0.0f || rz != 0.0f) rotate(out, n, cx, cy, cz, rx, ry, rz);
    *count = n;
    return RC_OK;
}

int rc_triangles_from_positions(const float* p, int count, int mat_index, rc_triangle* out) {
    if ((!p || !out) && count > 0) return RC_ERR_INVALID_ARG;
    for (int i = 0; i < count; ++i) {
        out[i] = make_tri(p + 9 * (size_t)i, p + 9 * (size_t)i + 3, p + 9 * (size_t)i + 6);
        out[i].mat_index = mat_index;
        flat_normal(out[i]);
    }
    return RC_OK;
}

int rc_build_bvh(const rc_triangle* in, int count, rc_triangle* out_tris, rc_bvh_node* out_nodes,
                 int node_capacity, int* node_count) {
    if (!in || !out_tris || !out_nodes || !node_count || count < 1) return RC_ERR_INVALID_ARG;
    SahBuilder b(in, count);
    b.build();
    if ((int)b.nodes().size() > node_capacity) return RC_ERR_CAPACITY;
    const std::vector<int>& perm = b.perm();
    for (int i = 0; i < count; ++i) out_tris[i] = in[perm[i]];
    memcpy(out_nodes, b.nodes().data(), b.nodes().size() * sizeof(rc_bvh_node));
    *node_count = (int)b.nodes().size();
    return RC_OK;
}

int rc_build_lights(const rc_triangle* tris, int count, const rc_material* mats, int material_count,
                    rc_light* out, int capacity, int* light_count, float* total_power) {
    if (!tris || !mats || !out || !light_count || !total_power || capacity < 1) return RC_ERR_INVALID_ARG;
    int n = 0;
    float sum = 0.0f;
    for (int i = 0; i < count; ++i) {
        const rc_triangle& t = tris[i];
        if (t.mat_index < 0 || t.mat_index >= material_count) return RC_ERR_INVALID_ARG;
        const rc_material& m = mats[t.mat_index];
        if (m.emission_strength <= 0.0f) continue;
        const float e1x = t.v1[0] - t.v0[0], e1y = t.v1[1] - t.v0[1], e1z = t.v1[2] - t.v0[2];
        const float e2x = t.v2[0] - t.v0[0], e2y = t.v2[1] - t.v0[1], e2z = t.v2[2] - t.v0[2];
        const float cx = e1y * e2z - e1z * e2y;
        const float cy = e1z * e2x - e1x * e2z;
        const float cz = e1x * e2y - e1y * e2x;
        const float area = 0.5f * dsqrtf(cx * cx + cy * cy + cz * cz);
        if (area < 1e-8f) continue;
        if (n >= capacity) return RC_ERR_CAPACITY;
        rc_light& L = out[n++];
        memset(&L, 0, sizeof(L));
        L.emission[0] = m.emission[0] * m.emission_strength;
        L.emission[1] = m.emission[1] * m.emission_strength;
        L.emission[2] = m.emission[2] * m.emission_strength;
        const float lum = 0.299f * L.emission[0] + 0.587f * L.emission[1] + 0.114f * L.emission[2];
        L.power = lum * area * (float)3.141592653589793;
        sum += L.power;
        for (int a = 0; a < 3; ++a) {
            L.v0[a] = t.v0[a];
            L.v1[a] = t.v1[a];
            L.v2[a] = t.v2[a];
            L.normal[a] = t.n0[a];
        }
        L.area = area;
    }
    *total_power = sum;
    *light_count = n;
    if (n == 0) {
        memset(out, 0, sizeof(rc_light));  // SceneUploader's zeroed stub
        return RC_OK;
    }
    float cum = 0.0f;
    for (int i = 0; i < n; ++i) {
        cum += out[i].power;
        out[i].cdf_weight = (sum > 0.0f) ? cum / sum : 1.0f;
    }
    out[n - 1].cdf_weight = 1.0f;
    return RC_OK;
}

int rc_thin_lens(float focal_length_mm, float f_stop, float* lens_radius, float* fov_tan_half) {
    if (!lens_radius || !fov_tan_half) return RC_ERR_INVALID_ARG;
    const float fm = focal_length_mm / 1000.0f;
    *lens_radius = fm / (2.0f * f_stop);
    *fov_tan_half = (float)tan(atan((double)(0.012f / fm)));
    return RC_OK;
}

int rc_orbit_basis(float theta, float phi, float radius, float tx, float ty, float tz, float* o) {
    if (!o) return RC_ERR_INVALID_ARG;
    const float sp = (float)sin((double)phi);
    const float ex = tx + radius * sp * (float)cos((double)theta);
    const float ey = ty + radius * (float)cos((double)phi);
    const float ez = tz + radius * sp * (float)sin((double)theta);
    float fx = tx - ex, fy = ty - ey, fz = tz - ez;
    const float fl = dsqrtf(fx * fx + fy * fy + fz * fz);
    fx /= fl;
    fy /= fl;
    fz /= fl;
    float rx = fy * 0.0f - fz * 1.0f, ry = fz * 0.0f - fx * 0.0f, rz = fx * 1.0f - fy * 0.0f;
    const float rl = dsqrtf(rx * rx + ry * ry + rz * rz);
    rx /= rl;
    ry /= rl;
    rz /= rl;
    const float v[12] = {ex, ey, ez, fx, fy, fz, rx, ry, rz,
                         ry * fz - rz * fy, rz * fx - rx * fz, rx * fy - ry * fx};
    memcpy(o, v, sizeof(v));
    return RC_OK;
}

float rc_sppm_next_radius(float radius, int iteration, float alpha) {
    const float num = (float)iteration + alpha;  // int + float is float in Java
    return radius * (float)sqrt((double)num / ((double)iteration + 1.0));
}

float rc_keyframe_evaluate(const float* tm, const float* val, const int32_t* interp, int n, float time,
                           float def) {
    if (n <= 0 || !tm || !val || !interp) return def;
    if (n == 1) return val[0];
    if (time <= tm[0]) return val[0];
    if (time >= tm[n - 1]) return val[n - 1];
    int hi = 1;
    while (hi < n && tm[hi] < time) ++hi;
    const int lo = hi - 1;
    const float t = (time - tm[lo]) / (tm[hi] - tm[lo]);
    switch (interp[lo]) {
        case 0:
            return val[lo];
        case 1:
            return val[lo] + (val[hi] - val[lo]) * t;
        default: {
            const float dt = tm[hi] - tm[lo];
            const float m0 = lo > 0 ? (val[hi] - val[lo - 1]) / (tm[hi] - tm[lo - 1]) : (val[hi] - val[lo]) / dt;
            const float m1 = hi < n - 1 ? (val[hi + 1] - val[lo]) / (tm[hi + 1] - tm[lo])
                                        : (val[hi] - val[lo]) / dt;
            const float t2 = t * t, t3 = t2 * t;
            const float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f;
            const float h10 = t3 - 2.0f * t2 + t;
            const float h01 = -2.0f * t3 + 3.0f * t2;
            const float h11 = t3 - t2;
            return h00 * val[lo] + h10 * dt * m0 + h01 * val[hi] + h11 * dt * m1;
        }
    }
}

}  // extern "C"
