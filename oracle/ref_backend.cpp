// ORACLE — test infrastructure only. Never linked into, called by or shipped with the product path.
//
// The reference's own CPU integrator, `integratePaths<Backend>` (xpu2/interactive/async_integrator.h:1986-3042),
// compiled UNMODIFIED from the reference's headers (oracle/Makefile) and driven by OracleBackend, which this
// file writes following the reference's CpuBackend (xpu2/interactive/async_cpu.h:586-1163): a hit is
// reconstructed by the reference's resume::geometryHit (resume_core.h:17-45), shaded by the reference's
// hitState + shadeMaterial (shade_material.h:121, :787), lit by the reference's lights::sample/eval/intersect
// (light_core.h:988-1025). The only part not from the reference is traversal: the reference delegates it to
// Embree (async_cpu.h:669-720, :944-967), which is absent here, so this file supplies a binary BVH whose
// triangle test (Woop et al. 2013, watertight, fp32, no contraction) and tie break (nearest t, then lowest
// triangle) are the same arithmetic the device traversal uses: both devices then choose the same primitive.
// The film and the chunk loop follow renderChunk (async_cpu.h:1584-1667) and the audit async_render.h:992-1048.
#define XPU2_PATHS_ONLY 1
#include "async_integrator.h"
#include "async_adaptive.h"
#include "async_grid.h"

#include "../include/x2.h"
#ifdef X2REF_REPLAY
#include "replay.h"
#endif

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace xi = xpu2::interactive;
using xi::sample::U32;
using xi::sample::U64;
using xi::surface::V3;

namespace {

// ---- traversal (the Embree stand-in) ----
struct Node {
    float lo[3], hi[3];
    U32 first, count;  // leaf: triangles [first, first+count) of order; inner: left child = first, right = first+1
};

struct Bvh {
    std::vector<Node> nodes;
    std::vector<U32> order;
};

struct TriTest {  // Woop, Benthin, Wald 2013: the ray's shear, once a ray
    int kx, ky, kz;
    float Sx, Sy, Sz;
};
inline TriTest shear(V3 d) {
    const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    TriTest s;
    s.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    s.kx = s.kz == 2 ? 0 : s.kz + 1;
    s.ky = s.kx == 2 ? 0 : s.kx + 1;
    const float dz = (&d.x)[s.kz];
    if (dz < 0.0f) std::swap(s.kx, s.ky);
    s.Sx = (&d.x)[s.kx] / dz;
    s.Sy = (&d.x)[s.ky] / dz;
    s.Sz = 1.0f / dz;
    return s;
}
// The hit distance t of the ray against triangle (a, b, c), or false. Same operations as the device test.
inline bool triHit(const TriTest& s, V3 o, V3 a, V3 b, V3 c, float tmin, float tmax, float& tOut) {
    const float A[3] = {a.x - o.x, a.y - o.y, a.z - o.z}, B[3] = {b.x - o.x, b.y - o.y, b.z - o.z},
                C[3] = {c.x - o.x, c.y - o.y, c.z - o.z};
    const float Ax = A[s.kx] - s.Sx * A[s.kz], Ay = A[s.ky] - s.Sy * A[s.kz];
    const float Bx = B[s.kx] - s.Sx * B[s.kz], By = B[s.ky] - s.Sy * B[s.kz];
    const float Cx = C[s.kx] - s.Sx * C[s.kz], Cy = C[s.ky] - s.Sy * C[s.kz];
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = s.Sz * A[s.kz], Bz = s.Sz * B[s.kz], Cz = s.Sz * C[s.kz];
    const float T = U * Az + V * Bz + W * Cz;
    const float t = T / det;
    if (!(t >= tmin && t <= tmax)) return false;
    tOut = t;
    return true;
}

struct Scene {
    std::vector<V3> vertices;
    std::vector<U32> tris;       // 3 a triangle
    std::vector<U32> triGeom;    // mesh of each triangle
    std::vector<U32> meshFirst;  // mesh_count + 1
    std::vector<xi::lights::Light> lights;
    std::vector<xi::shade::MaterialRecord> records;  // one a mesh
    std::vector<float> pool;
    xi::mixed::Config config{};
    Bvh bvh;
    V3 vertex(U32 i) const { return vertices[i]; }
    // Volumes: their shaders, their bounds as closed meshes (twelve triangles a box, outward), their dense grids.
    std::vector<xi::volume::Shader> volumes;
    std::vector<V3> volumeTris;  // 3 vertices a triangle, 12 triangles a volume
    std::vector<std::vector<float>> gridValues;
    std::vector<nanovdb::FloatGrid> floatGrids;
    std::vector<nanovdb::Vec3fGrid> vecGrids;
    std::vector<xi::volume::Grid> grids;
    // Texture coordinates (2 a vertex; empty: none) and the textures as the reference's images: one level of fp32 RGB
    // texels (format 0) in 32x32 tile pages, each page's texels row-major at the tile's own width.
    std::vector<float> uvs;
    std::vector<xi::tex::Image> images;
    std::vector<std::vector<const V3*>> pagePointers;
    std::vector<std::vector<std::vector<V3>>> pages;
};

// The reference's texture source for its map programs (shadeMaterial's Tex): the scene's images, looked up by
// texture_core.h's lookup.
struct OracleTextures {
    const Scene* s;
    unsigned lookup(unsigned texture, xi::tex::Binding b, const xi::tex::Footprint& f, V3& out) const {
        if (texture >= s->images.size()) return xi::tex::Invalid;
        b.image = &s->images[texture];
#ifdef X2REF_REPLAY
        const unsigned status = xi::tex::lookup(b, f, out);
        replay::event(3, b.mode, f.u, f.v, out.x, out.y);
        replay::event(4, status, out.z, 0.0f, 0.0f, 0.0f);
        return status;
#else
        return xi::tex::lookup(b, f, out);
#endif
    }
};

// A box's 12 triangles by corner (corner i: hi on x for bit 0, y for bit 1, z for bit 2), each counter-clockwise seen
// from outside, so cross(b - a, c - a) points out. The engine's device code uses the same table.
const int kBoxTriangles[12][3] = {{0, 4, 6}, {0, 6, 2}, {1, 3, 7}, {1, 7, 5}, {0, 1, 5}, {0, 5, 4},
                                  {2, 6, 7}, {2, 7, 3}, {0, 2, 3}, {0, 3, 1}, {4, 5, 7}, {4, 7, 6}};

void buildBvh(Scene& s) {
    const U32 n = U32(s.tris.size() / 3);
    std::vector<float> cen(size_t(n) * 3);
    std::vector<float> blo(size_t(n) * 3), bhi(size_t(n) * 3);
    for (U32 t = 0; t < n; ++t) {
        const V3 a = s.vertex(s.tris[3 * t]), b = s.vertex(s.tris[3 * t + 1]), c = s.vertex(s.tris[3 * t + 2]);
        const float lo[3] = {std::min({a.x, b.x, c.x}), std::min({a.y, b.y, c.y}), std::min({a.z, b.z, c.z})};
        const float hi[3] = {std::max({a.x, b.x, c.x}), std::max({a.y, b.y, c.y}), std::max({a.z, b.z, c.z})};
        for (int k = 0; k < 3; ++k) {
            blo[3 * t + k] = lo[k];
            bhi[3 * t + k] = hi[k];
            cen[3 * t + k] = 0.5f * (lo[k] + hi[k]);
        }
    }
    s.bvh.order.resize(n);
    for (U32 i = 0; i < n; ++i) s.bvh.order[i] = i;
    s.bvh.nodes.clear();
    s.bvh.nodes.reserve(size_t(n) * 2 / 2 + 16);
    struct Item { U32 node, first, count; };
    std::vector<Item> work;
    s.bvh.nodes.push_back(Node{});
    work.push_back({0, 0, n});
    while (!work.empty()) {
        const Item it = work.back();
        work.pop_back();
        Node nd{};
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 3; ++k) { nd.lo[k] = INFINITY; nd.hi[k] = -INFINITY; }
        for (U32 i = it.first; i < it.first + it.count; ++i) {
            const U32 t = s.bvh.order[i];
            for (int k = 0; k < 3; ++k) {
                nd.lo[k] = std::min(nd.lo[k], blo[3 * t + k]);
                nd.hi[k] = std::max(nd.hi[k], bhi[3 * t + k]);
                clo[k] = std::min(clo[k], cen[3 * t + k]);
                chi[k] = std::max(chi[k], cen[3 * t + k]);
            }
        }
        if (it.count <= 4) {
            nd.first = it.first;
            nd.count = it.count;
            s.bvh.nodes[it.node] = nd;
            continue;
        }
        int axis = 0;
        for (int k = 1; k < 3; ++k)
            if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
        const U32 mid = it.first + it.count / 2;
        std::nth_element(s.bvh.order.begin() + it.first, s.bvh.order.begin() + mid, s.bvh.order.begin() + it.first + it.count,
                         [&](U32 x, U32 y) { return cen[3 * x + axis] < cen[3 * y + axis] || (cen[3 * x + axis] == cen[3 * y + axis] && x < y); });
        const U32 left = U32(s.bvh.nodes.size());
        s.bvh.nodes.push_back(Node{});
        s.bvh.nodes.push_back(Node{});
        nd.first = left;
        nd.count = 0;
        s.bvh.nodes[it.node] = nd;
        work.push_back({left, it.first, mid - it.first});
        work.push_back({left + 1, mid, it.first + it.count - mid});
    }
}

inline bool boxHit(const Node& nd, V3 o, V3 inv, float tmin, float tmax) {
    float t0 = tmin, t1 = tmax;
    const float oo[3] = {o.x, o.y, o.z}, ii[3] = {inv.x, inv.y, inv.z};
    for (int k = 0; k < 3; ++k) {
        float a = (nd.lo[k] - oo[k]) * ii[k], b = (nd.hi[k] - oo[k]) * ii[k];
        if (a > b) std::swap(a, b);
        a -= std::fabs(a) * 4e-7f;  // widened by 2 gamma(3) each way: the slab test stays conservative
        b += std::fabs(b) * 4e-7f;
        t0 = a > t0 ? a : t0;  // NaN (0 * inf) keeps the bound
        t1 = b < t1 ? b : t1;
    }
    return t0 <= t1;
}

// The triangle test's t is a convex combination of the vertices' sheared depths, rounded: its absolute error is a
// few ulps of the distance to the vertices. Boxes are tested against [tmin - eps, tmax + eps], eps = 2^-18 times
// the origin's distance to the far corner of the scene's bounds, so no box holding an accepted hit is culled.
inline float rayTolerance(const Scene& s, V3 o) {
    const Node& root = s.bvh.nodes[0];
    const float x = std::max(std::fabs(root.lo[0] - o.x), std::fabs(root.hi[0] - o.x));
    const float y = std::max(std::fabs(root.lo[1] - o.y), std::fabs(root.hi[1] - o.y));
    const float z = std::max(std::fabs(root.lo[2] - o.z), std::fabs(root.hi[2] - o.z));
    return (x + y + z) * 0x1p-18f;
}

// Closest hit on [tmin, tmax]: the nearest t, then the lowest triangle index. Returns ~0u on a miss.
U32 closest(const Scene& s, V3 o, V3 d, float tmin, float tmax, float& tBest) {
    const TriTest sh = shear(d);
    const V3 inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    const float eps = rayTolerance(s, o);
    U32 best = ~0u;
    tBest = tmax;
    U32 stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node& nd = s.bvh.nodes[stack[--sp]];
        if (!boxHit(nd, o, inv, tmin - eps, tBest + eps)) continue;
        if (nd.count) {
            for (U32 i = nd.first; i < nd.first + nd.count; ++i) {
                const U32 t = s.bvh.order[i];
                float th;
                if (!triHit(sh, o, s.vertex(s.tris[3 * t]), s.vertex(s.tris[3 * t + 1]), s.vertex(s.tris[3 * t + 2]), tmin, tBest, th)) continue;
                if (th < tBest || (th == tBest && t < best)) {
                    tBest = th;
                    best = t;
                }
            }
        } else {
            stack[sp++] = nd.first;
            stack[sp++] = nd.first + 1;
        }
    }
    return best;
}
bool occluded(const Scene& s, V3 o, V3 d, float tmin, float tmax) {
    const TriTest sh = shear(d);
    const V3 inv{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    const float eps = rayTolerance(s, o);
    U32 stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node& nd = s.bvh.nodes[stack[--sp]];
        if (!boxHit(nd, o, inv, tmin - eps, tmax + eps)) continue;
        if (nd.count) {
            for (U32 i = nd.first; i < nd.first + nd.count; ++i) {
                const U32 t = s.bvh.order[i];
                float th;
                if (triHit(sh, o, s.vertex(s.tris[3 * t]), s.vertex(s.tris[3 * t + 1]), s.vertex(s.tris[3 * t + 2]), tmin, tmax, th)) return true;
            }
        } else {
            stack[sp++] = nd.first;
            stack[sp++] = nd.first + 1;
        }
    }
    return false;
}

// ---- the Backend concept (async_integrator.h:52-57), after CpuBackend ----
struct Counts {
    uint64_t trace = 0, nee = 0, bsdf = 0, held = 0;
};

struct OracleBackend {
    const Scene& s;
    Counts* counts;
    struct Scratch {
        xi::shade::Bsdf bsdf;
        xi::async::paths::Pending pending[xi::async::paths::MaxPending];
    };
    static Scratch& scratch() {
        static thread_local std::unique_ptr<Scratch> p;
        if (!p) p = std::make_unique<Scratch>();
        return *p;
    }
    // Members the reference integrator reads directly (subsurface exits' light set, the sample's time, the
    // shadow ray's receiver): unused by the admitted scenes, kept at CpuBackend's initial values.
    U32 exitLightSet = ~0u, shadowLight = ~0u, shadowReceiver = ~0u;
    float time = 0.0f;
    void setTime(float t) { time = t; }
    xi::resume::Hit trace(const xi::surface::Ray& ray) const {
        ++counts->trace;
        xi::resume::Hit out;
        float t;
        const U32 tri = closest(s, ray.origin, ray.direction, ray.nearT, ray.farT, t);
#ifdef X2REF_REPLAY
        replay::event(1, tri, tri == ~0u ? 0.0f : t, ray.direction.x, ray.direction.y, ray.direction.z);
#endif
        if (tri == ~0u) return out;
        out.geom = s.triGeom[tri];
        out.prim = tri - s.meshFirst[out.geom];
        out.t = t;
        if (!xi::resume::geometryHit(out, ray, s.vertex(s.tris[3 * tri]), s.vertex(s.tris[3 * tri + 1]), s.vertex(s.tris[3 * tri + 2])))
            out.normal = {};
        return out;
    }
    bool visible(V3 o, V3 d) const { return visible(o, d, INFINITY); }
    bool visible(V3 o, V3 d, float distance) const { return visible(o, d, 0.0f, distance); }
    bool visible(V3 o, V3 d, float near, float distance) const {
        const bool v = !occluded(s, o, d, near, distance);
#ifdef X2REF_REPLAY
        replay::event(2, v ? 1u : 0u, distance, d.x, d.y, d.z);
#endif
        return v;
    }
    void countRay(U32 kind) const {
        if (kind == xi::async::paths::RayCountNee) ++counts->nee;
        else if (kind == xi::async::paths::RayCountBsdf) ++counts->bsdf;
        else ++counts->held;
    }
    bool deferred() const { return false; }
    bool textureMissed() const { return false; }
    xi::shade::Bsdf& bsdf() const { return scratch().bsdf; }
    xi::async::paths::Pending* pending() const { return scratch().pending; }
    const xi::lights::Light& light(U32 i) const { return s.lights[i]; }
    U32 lightSet(U32) const { return 0; }
    bool inSet(U32, U32 i) const { return i < s.lights.size(); }
    bool inLobeSet(U32 set, U32) const { return set == ~0u; }
    const xi::lights::TreeNode* treeNodes() const { return nullptr; }
    int treeRoot(U32) const { return -1; }
    void shadowFor(U32, U32) {}
    bool castsShadow(U32, bool) const { return true; }
    const xi::volume::Shader* volumes() const { return s.volumes.empty() ? nullptr : s.volumes.data(); }
    xi::volume::Grids volumeGrids() const {
        xi::volume::Grids g;
        g.grids = s.grids.empty() ? nullptr : s.grids.data();
        g.count = U32(s.grids.size());
        g.maps = nullptr;
        g.time = time;
        return g;
    }
    // The ray's crossings of the volumes' bounds from tnear on, as the reference's CPU backend collects them
    // (async_cpu.h:1089-1149): the nearest crossing from t, entering where the ray runs against the outward normal,
    // then on from just past it; a repeat of the same crossing at the same t dropped. Every ray type sees volumes.
    U32 volumeCrossings(V3 o, V3 d, float tnear, xi::volume::Crossing* x, U32 max, U32) const {
        if (s.volumes.empty()) return 0;
        const TriTest sh = shear(d);
        const U32 tris = U32(s.volumeTris.size() / 3);
        U32 n = 0;
        float t = tnear;
        for (U32 k = 0; k < 4 * max && n < max; ++k) {
            float best = INFINITY;
            U32 hitTri = ~0u;
            for (U32 i = 0; i < tris; ++i) {
                float th;
                if (triHit(sh, o, s.volumeTris[3 * i], s.volumeTris[3 * i + 1], s.volumeTris[3 * i + 2], t, INFINITY, th) && th < best) {
                    best = th;
                    hitTri = i;
                }
            }
            if (hitTri == ~0u) break;
            const V3 a = s.volumeTris[3 * hitTri], b = s.volumeTris[3 * hitTri + 1], c = s.volumeTris[3 * hitTri + 2];
            const V3 e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{c.x - a.x, c.y - a.y, c.z - a.z};
            const V3 ng{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
            const U32 v = hitTri / 12;
            const U32 flags = d.x * ng.x + d.y * ng.y + d.z * ng.z < 0.0f ? xi::volume::Entry : xi::volume::Exit;
            if (!(n > 0 && x[n - 1].t == best && x[n - 1].volume == v && x[n - 1].flags == flags)) x[n++] = xi::volume::Crossing{best, v, flags};
            t = best + std::fmax(1e-6f, best * 1e-6f);
        }
        return n;
    }
    xi::volume::Regions emissiveRegions() const { return xi::volume::Regions{nullptr, 0, nullptr}; }
    const xi::aov::Tables& aovs() const {
        static const xi::aov::Tables none{};
        return none;
    }
    int geomLabel(U32) const { return -1; }
    const float* walkSequences() const { return nullptr; }
    const xi::lights::Filter* filters() const { return nullptr; }
    const xi::lights::FilterList* filterList(U32, U32) const { return nullptr; }
    float filterVdb(U32, U32, V3) const { return 1.0f; }
    V3 filterMap(U32, U32, float, float) const { return V3{1, 1, 1}; }
    U32 materialId(U32 geom) const { return geom < s.records.size() ? s.records[geom].offset : ~0u; }
    xi::resume::Hit traceMaterial(xi::surface::Ray ray, U32 material) const {
        for (int k = 0; k < 64; ++k) {
            const xi::resume::Hit h = trace(ray);
            if (h.geom == ~0u || materialId(h.geom) == material) return h;
            ray.nearT = h.t + fmaxf(1e-6f, h.t * 1e-6f);
            if (!(ray.nearT < ray.farT)) break;
        }
        return xi::resume::Hit{};
    }
    bool stateOf(const xi::resume::Hit& h, const xi::surface::Ray& ray, xi::shade::State& st) const {
        const U32 tri = s.meshFirst[h.geom] + h.prim;
        const U32 ia = s.tris[3 * tri], ib = s.tris[3 * tri + 1], ic = s.tris[3 * tri + 2];
        xi::shade::MeshAttributes attributes;  // no normals: the geometric normal; the vertices' uvs when the scene has them
        if (!s.uvs.empty()) {
            attributes.uvs = s.uvs.data();
            attributes.uvRate = xi::shade::RateVertex;
        }
        if (!xi::shade::hitState(attributes, h.prim, ia, ib, ic, s.vertex(ia), s.vertex(ib), s.vertex(ic), h.u, h.v, h.point,
                                 ray.direction, st))
            return false;
        st.geom = h.geom;
        return true;
    }
    bool surfaceState(const xi::resume::Hit& h, const xi::surface::Ray& ray, xi::shade::State& st) const { return stateOf(h, ray, st); }
    unsigned presenceAt(const xi::resume::Hit&, const xi::surface::Ray&, float& presence) const {
        presence = 1.0f;
        return xi::tex::Ready;
    }
    unsigned shade(const xi::resume::Hit& h, const xi::surface::Ray& ray, xi::shade::State& st, xi::shade::Bsdf& bsdf, float& presence) const {
        if (!stateOf(h, ray, st)) return xi::tex::Invalid;
        if (h.geom >= s.records.size()) return xi::tex::Invalid;
        const OracleTextures textures{&s};
        return xi::shade::shadeMaterial(s.records[h.geom], s.pool.data(), st, textures, bsdf, presence, nullptr, nullptr);
    }
};

xi::lights::Light toLight(const x2_light& x, U32 index) {
    xi::lights::Light l;
    std::memset(&l, 0, sizeof(l));
    l.type = x.type == X2_LIGHT_ENV ? xi::lights::Env : x.type == X2_LIGHT_DISTANT ? xi::lights::Distant : xi::lights::Rect;
    l.cosThetaMax = x.cos_theta_max;
    l.versineThetaMax = x.versine_theta_max;
    l.sidedness = x.sidedness;
    l.index = index;
    l.radiance = V3{x.radiance[0], x.radiance[1], x.radiance[2]};
    l.position = V3{x.position[0], x.position[1], x.position[2]};
    l.direction = V3{x.direction[0], x.direction[1], x.direction[2]};
    for (int i = 0; i < 3; ++i) {
        l.local2Render[i] = V3{x.local2render[i][0], x.local2render[i][1], x.local2render[i][2]};
        l.render2Local[i] = V3{x.render2local[i][0], x.render2local[i][1], x.render2local[i][2]};
        l.render2LocalRot[i] = V3{x.render2local_rot[i][0], x.render2local_rot[i][1], x.render2local_rot[i][2]};
    }
    l.scale = x.scale;
    l.invArea = x.inv_area;
    l.planeOffset = x.plane_offset;
    l.halfWidth = x.half_width;
    l.halfHeight = x.half_height;
    l.image = nullptr;
    l.visibleInCamera = x.visible_in_camera;
    l.hemispherical = x.hemispherical;
    l.fallback = V3{1, 1, 1};
    l.spread = 1.0f;
    l.mesh = nullptr;
    l.lpeLabel = -1;
    l.ref = nullptr;
    l.visibilityMask = x.visibility_mask;
    return l;
}

xi::mixed::Config toConfig(const x2_config& x, const x2_camera& cam) {
    xi::mixed::Config c{};
    std::memset(c.camera.rasterToCamera.m, 0, sizeof(c.camera.rasterToCamera.m));
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            c.camera.rasterToCamera.m[i][j] = cam.raster_to_camera[i][j];
            c.camera.cameraToRender.m[i][j] = cam.camera_to_render[i][j];
        }
    c.camera.nearClip = cam.near_clip;
    c.camera.farClip = cam.far_clip;
    c.camera.type = xi::surface::CameraPerspective;
    c.sky = V3{0, 0, 0};
    c.width = x.width;
    c.height = x.height;
    c.seed = x.seed;
    c.meshes = 0;
    c.filter = xi::surface::Filter(x.filter);
    c.filterWidth = x.filter_width;
    c.spp = x.spp;
    c.sampling = x.sampling;
    c.paths = 1;
    c.lightCount = x.light_count;
    c.bsdfSamples = x.bsdf_samples;
    c.lightSamples = x.light_samples;
    c.maxDepth = x.max_depth;
    c.maxDiffuseDepth = x.max_diffuse_depth;
    c.clampDepth = x.clamp_depth;
    c.rrThreshold = x.rr_threshold;
    c.clampValue = x.clamp_value;
    c.maxGlossyDepth = x.max_glossy_depth;
    c.maxMirrorDepth = x.max_mirror_depth;
    c.maxHairDepth = x.max_hair_depth;
    c.maxPresenceDepth = x.max_presence_depth;
    c.shadowTerminatorFix = x.shadow_terminator_fix;
    c.roughnessClamping = x.roughness_clamping;
    c.transparencyThreshold = x.transparency_threshold;
    c.visibleLights = x.visible_lights;
    c.presenceThreshold = x.presence_threshold;
    c.presenceQuality = x.presence_quality;
    c.shadowReuse = x.shadow_reuse;
    c.volumeCount = x.volume_count;
    c.maxVolumeDepth = x.max_volume_depth;
    c.volumeIlluminationSamples = x.volume_illumination_samples;
    c.volumeOverlapMode = x.volume_overlap_mode;
    c.volumeTransmittanceThreshold = x.volume_transmittance_threshold;
    c.volumeAttenuationFactor = x.volume_attenuation_factor;
    c.volumeContributionFactor = x.volume_contribution_factor;
    c.volumePhaseAttenuationFactor = x.volume_phase_attenuation_factor;
    c.invVolumeQuality = x.inv_volume_quality;
    c.invVolumeShadowQuality = x.inv_volume_shadow_quality;
    return c;
}

#include "adjoint64.h"

struct Handle {
    Scene scene;
    Counts counts;
    adj64::Scene64 x;  // the engine's own records, for the FP64 adjoint
};

}  // namespace

extern "C" {

// The scene and config as the engine takes them (x2.h), built into the reference's records.
void* x2ref_open(const x2_scene_desc* d, const x2_config* cfg) {
    if (!d || !cfg) return nullptr;
    auto* h = new Handle();
    Scene& s = h->scene;
    s.vertices.resize(d->vertex_count);
    for (U32 i = 0; i < d->vertex_count; ++i) s.vertices[i] = V3{d->vertices[3 * i], d->vertices[3 * i + 1], d->vertices[3 * i + 2]};
    s.tris.assign(d->triangles, d->triangles + size_t(d->triangle_count) * 3);
    s.meshFirst.assign(d->mesh_first, d->mesh_first + d->mesh_count + 1);
    s.triGeom.resize(d->triangle_count);
    for (U32 m = 0; m < d->mesh_count; ++m)
        for (U32 t = d->mesh_first[m]; t < d->mesh_first[m + 1]; ++t) s.triGeom[t] = m;
    // Textures: each a one-level image of 32x32 pages (texture_core.h Mip), and the vertices' uvs.
    if (d->uvs) s.uvs.assign(d->uvs, d->uvs + 2 * size_t(d->vertex_count));
    s.images.resize(d->texture_count);
    s.pagePointers.resize(d->texture_count);
    s.pages.resize(d->texture_count);
    for (U32 t = 0; t < d->texture_count; ++t) {
        const x2_texture& xt = d->textures[t];
        const U32 T = xi::tex::Tile, nx = (xt.width + T - 1) / T, ny = (xt.height + T - 1) / T;
        s.pages[t].resize(size_t(nx) * ny);
        s.pagePointers[t].resize(size_t(nx) * ny);
        for (U32 ty = 0; ty < ny; ++ty)
            for (U32 tx = 0; tx < nx; ++tx) {
                const U32 stride = std::min(T, xt.width - tx * T), rows = std::min(T, xt.height - ty * T);
                std::vector<V3>& page = s.pages[t][size_t(ty) * nx + tx];
                page.resize(size_t(stride) * rows);
                for (U32 y = 0; y < rows; ++y)
                    for (U32 x = 0; x < stride; ++x) {
                        const float* v = xt.rgb + 3 * (size_t(ty * T + y) * xt.width + tx * T + x);
                        page[size_t(y) * stride + x] = V3{v[0], v[1], v[2]};
                    }
                s.pagePointers[t][size_t(ty) * nx + tx] = page.data();
            }
        xi::tex::Image& img = s.images[t];
        img.count = 1;
        img.levels[0].width = xt.width;
        img.levels[0].height = xt.height;
        img.levels[0].pages = s.pagePointers[t].data();
        img.levels[0].tileBase = 0;
        img.levels[0].format = 0;
    }
    // A textured material's map program, once a material: a UsdPrimvarReader of st (mode 2) into register 0, a
    // UsdUVTexture of the texture at that st (its st bound BindVec2 to register 0) into register 1; the material's
    // diffuseColor bound BindColor to register 1 (shade_mapnodes.h, shade_maps.h). Returns (program, bindings).
    auto words = [&](const std::vector<U32>& w) {
        const U32 at = U32(s.pool.size());
        for (U32 v : w) {
            float f;
            std::memcpy(&f, &v, sizeof(f));
            s.pool.push_back(f);
        }
        return at;
    };
    auto floats = [&](const float* f, size_t n) { s.pool.insert(s.pool.end(), f, f + n); };
    std::vector<std::pair<U32, U32>> programs(d->material_count, {xi::shade::NoMapProgram, 0});
    for (U32 i = 0; i < d->material_count; ++i) {
        const x2_material& x = d->materials[i];
        if (!x.diffuse_texture) continue;
        namespace sh = xi::shade;
        const U32 headerFloats = sizeof(sh::MapNodeHeader) / sizeof(float);
        // The primvar reader.
        const U32 node0 = U32(s.pool.size());
        sh::MapNodeHeader h0{};
        h0.kind = sh::MapUsdPrimvar;
        h0.reg = 0;
        h0.paramCount = sizeof(sh::MapUsdPrimvarParams) / sizeof(float);
        h0.bindingCount = 0;
        h0.texture = sh::MapNoTexture;
        floats(reinterpret_cast<const float*>(&h0), headerFloats);
        sh::MapUsdPrimvarParams q0{};
        q0.mode = 2.0f;
        q0.components = 2.0f;
        floats(reinterpret_cast<const float*>(&q0), h0.paramCount);
        // The texture.
        const U32 node1 = U32(s.pool.size());
        sh::MapNodeHeader h1{};
        h1.kind = sh::MapUsdUVTexture;
        h1.reg = 1;
        h1.paramCount = sizeof(sh::MapUsdUVTextureParams) / sizeof(float);
        h1.bindingCount = 1;
        h1.texture = x.diffuse_texture - 1;
        h1.wrap = d->textures[x.diffuse_texture - 1].wrap;
        h1.gamma = 0;
        floats(reinterpret_cast<const float*>(&h1), headerFloats);
        sh::MapUsdUVTextureParams q1{};
        q1.output_mode = 0.0f;
        q1.fallback = sh::Color{1.0f, 1.0f, 1.0f};
        q1.scale = sh::Color{1.0f, 1.0f, 1.0f};
        q1.bias = sh::Color{0.0f, 0.0f, 0.0f};
        floats(reinterpret_cast<const float*>(&q1), h1.paramCount);
        words({U32(offsetof(sh::MapUsdUVTextureParams, st) / sizeof(float)), U32(sh::BindVec2), 0u});
        // The program: its nodes in order, then no required attributes.
        const U32 program = words({2u, node0, node1, 0u});
        const U32 bindings = words({U32(offsetof(sh::UsdPreviewSurfaceParams, diffuseColor) / sizeof(float)), U32(sh::BindColor), 1u});
        programs[i] = {program, bindings};
    }
    // One UsdPreviewSurface record a mesh (its material's parameters in the pool).
    for (U32 m = 0; m < d->mesh_count; ++m) {
        const x2_material& x = d->materials[d->mesh_material[m]];
        xi::shade::UsdPreviewSurfaceParams p{};
        p.diffuseColor = V3{x.diffuse[0], x.diffuse[1], x.diffuse[2]};
        p.emissiveColor = V3{x.emission[0], x.emission[1], x.emission[2]};
        p.specularColor = V3{x.specular[0], x.specular[1], x.specular[2]};
        p.useSpecularWorkflow = 1.0f;
        p.metallic = 0.0f;
        p.roughness = x.roughness;
        p.clearcoat = 0.0f;
        p.clearcoatRoughness = 0.01f;
        p.opacity = 1.0f;
        p.opacityThreshold = 0.0f;
        p.ior = 1.5f;
        p.normal = V3{0, 0, 1};
        xi::shade::MaterialRecord r;
        r.kind = xi::shade::MatUsdPreviewSurface;
        r.flags = x.kind == X2_MAT_GGX ? U32(xi::shade::MatModoUsdSpecular) : 0u;
        r.offset = U32(s.pool.size());
        r.count = xi::shade::UsdPreviewSurfaceFloats;
        const float* f = reinterpret_cast<const float*>(&p);
        s.pool.insert(s.pool.end(), f, f + xi::shade::UsdPreviewSurfaceFloats);
        if (x.diffuse_texture) {
            r.maps = programs[d->mesh_material[m]].first;
            r.bindings = programs[d->mesh_material[m]].second;
            r.bindingCount = 1;
        }
        s.records.push_back(r);
    }
    for (U32 i = 0; i < d->light_count; ++i) s.lights.push_back(toLight(d->lights[i], i));
    s.config = toConfig(*cfg, d->camera);
    h->x.materials.assign(d->materials, d->materials + d->material_count);
    h->x.meshMaterial.assign(d->mesh_material, d->mesh_material + d->mesh_count);
    h->x.lights.assign(d->lights, d->lights + d->light_count);
    h->x.camera = d->camera;
    h->x.config = *cfg;
    if (d->uvs) h->x.uvs.assign(d->uvs, d->uvs + 2 * size_t(d->vertex_count));
    for (U32 t = 0; t < d->texture_count; ++t) {
        const x2_texture& xt = d->textures[t];
        adj64::Texture64 tx{xt.width, xt.height, xt.wrap, h->x.texels, {}};
        tx.rgb.assign(xt.rgb, xt.rgb + 3 * size_t(xt.width) * xt.height);
        h->x.texels += U64(xt.width) * xt.height;
        h->x.textures.push_back(std::move(tx));
    }
    // Grids (dense, as the NanoVDB stand-in holds them) and the VdbVolume shaders over them.
    s.gridValues.resize(d->grid_count);
    s.floatGrids.resize(d->grid_count);
    s.vecGrids.resize(d->grid_count);
    s.grids.resize(d->grid_count);
    for (U32 g = 0; g < d->grid_count; ++g) {
        const x2_grid& xg = d->grids[g];
        const size_t voxels = size_t(xg.dims[0]) * xg.dims[1] * xg.dims[2];
        s.gridValues[g].assign(xg.values, xg.values + voxels * xg.channels);
        xi::volume::Grid& vg = s.grids[g];
        for (int i = 0; i < 16; ++i) vg.worldToIndex[i] = xg.world_to_index[i];
        vg.vec3 = xg.channels == 3 ? 1u : 0u;
        if (xg.channels == 3) {
            nanovdb::Vec3fGrid& ng = s.vecGrids[g];
            ng.values = reinterpret_cast<const nanovdb::Vec3f*>(s.gridValues[g].data());
            ng.background = nanovdb::Vec3f{{0, 0, 0}};
            for (int a = 0; a < 3; ++a) ng.lo[a] = xg.lo[a], ng.dims[a] = xg.dims[a];
            vg.data = &ng;
        } else {
            nanovdb::FloatGrid& ng = s.floatGrids[g];
            ng.values = s.gridValues[g].data();
            ng.background = 0.0f;
            for (int a = 0; a < 3; ++a) ng.lo[a] = xg.lo[a], ng.dims[a] = xg.dims[a];
            vg.data = &ng;
        }
    }
    for (U32 v = 0; v < d->volume_count; ++v) {
        const x2_volume& xv = d->volumes[v];
        xi::volume::Shader sh;
        std::memset(&sh, 0, sizeof(sh));
        sh.kind = xi::volume::KindVdb;
        sh.g = xv.g;
        sh.flags = 0;
        sh.lightSet = xv.light_set;
        sh.densityGrid = xv.density_grid;
        sh.emissionGrid = xv.emission_grid;
        sh.interpolation = xv.interpolation;
        sh.featureSize = xv.feature_size;
        for (int i = 0; i < 12; ++i) sh.worldToGrid[i] = xv.world_to_grid[i];
        sh.gain = V3{xv.gain[0], xv.gain[1], xv.gain[2]};
        sh.colorMult = V3{xv.color_mult[0], xv.color_mult[1], xv.color_mult[2]};
        sh.incandescence = V3{xv.incandescence[0], xv.incandescence[1], xv.incandescence[2]};
        sh.visibility = ~0u;
        sh.lpeLabel = -1;
        sh.bakedGrid = xi::volume::NoGrid;
        sh.velocityGrid = xi::volume::NoGrid;
        sh.surfaceOpacityThreshold = xv.surface_opacity_threshold;
        s.volumes.push_back(sh);
        V3 corner[8];
        for (int i = 0; i < 8; ++i)
            corner[i] = V3{(i & 1) ? xv.bound_hi[0] : xv.bound_lo[0], (i & 2) ? xv.bound_hi[1] : xv.bound_lo[1], (i & 4) ? xv.bound_hi[2] : xv.bound_lo[2]};
        for (const auto& t : kBoxTriangles)
            for (int k = 0; k < 3; ++k) s.volumeTris.push_back(corner[t[k]]);
    }
    buildBvh(s);
    return h;
}

void x2ref_close(void* p) { delete static_cast<Handle*>(p); }

// integrate() for n (pixel, index) pairs on `threads` host threads.
int x2ref_integrate(void* p, const uint32_t* pairs, uint64_t n, double* rgba, uint32_t* status, int threads) {
    auto* h = static_cast<Handle*>(p);
    if (!h || (!pairs && n)) return X2_EINVAL;
    std::atomic<uint64_t> next{0};
    std::vector<Counts> per(std::max(threads, 1));
    auto work = [&](int w) {
        OracleBackend backend{h->scene, &per[w]};
        for (;;) {
            const uint64_t i = next.fetch_add(1);
            if (i >= n) break;
            xi::async::Radiance r;
            const auto st = xi::async::integratePaths(h->scene.config, pairs[2 * i], pairs[2 * i + 1], backend, r);
            rgba[4 * i] = r.rgb[0];
            rgba[4 * i + 1] = r.rgb[1];
            rgba[4 * i + 2] = r.rgb[2];
            rgba[4 * i + 3] = r.alpha;
            status[i] = U32(st);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    for (const auto& c : per) {
        h->counts.trace += c.trace;
        h->counts.nee += c.nee;
        h->counts.bsdf += c.bsdf;
        h->counts.held += c.held;
    }
    return X2_OK;
}

#ifdef X2REF_REPLAY
// One sample through the reference integrator on this thread, replaying the given transcendental values (the
// device's records, x2_diag.h; null or n = 0: libm's own), with the calls it made and the backend's events logged.
// Returns the number of table misses in *misses; the logs are truncated to their capacities (the full counts in
// *ncalls and *nevents).
int x2ref_replay(void* p, uint32_t pixel, uint32_t index, const x2_diag_call* table, uint32_t n, double* rgba, uint32_t* status,
                 x2_diag_call* calls, uint32_t callCap, uint32_t* ncalls, void* events, uint32_t eventCap, uint32_t* nevents,
                 uint64_t* misses) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return X2_EINVAL;
    replay::State st;
    st.useTable = table && n;
    for (uint32_t i = 0; i < n; ++i) st.table[replay::key(table[i].fn, table[i].a, table[i].b)] = {table[i].r0, table[i].r1};
    Counts c;
    OracleBackend backend{h->scene, &c};
    xi::async::Radiance r;
    replay::t_state = &st;
    const auto code = xi::async::integratePaths(h->scene.config, pixel, index, backend, r);
    replay::t_state = nullptr;
    rgba[0] = r.rgb[0];
    rgba[1] = r.rgb[1];
    rgba[2] = r.rgb[2];
    rgba[3] = r.alpha;
    *status = U32(code);
    *ncalls = uint32_t(st.calls.size());
    *nevents = uint32_t(st.events.size());
    std::memcpy(calls, st.calls.data(), sizeof(x2_diag_call) * std::min<size_t>(callCap, st.calls.size()));
    std::memcpy(events, st.events.data(), sizeof(replay::Event) * std::min<size_t>(eventCap, st.events.size()));
    *misses = st.misses;
    return X2_OK;
}
#endif

// renderChunk (async_cpu.h:1584-1667): workers claim 8x8 tiles and render their samples [first, first+count)
// into an FP64 film: sums (4 a pixel), odd-index sums and counts. Ray counts in rays[4] (trace, nee, bsdf, held).
int x2ref_render(void* p, uint32_t first, uint32_t count, int threads, double* sums, double* odd, uint32_t* counts, uint64_t* rays) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return X2_EINVAL;
    const auto& c = h->scene.config;
    const U32 tilesX = (c.width + 7) / 8, tilesY = (c.height + 7) / 8, tiles = tilesX * tilesY;
    std::atomic<U32> next{0};
    std::vector<Counts> per(std::max(threads, 1));
    std::atomic<uint64_t> errors{0};
    auto work = [&](int w) {
        OracleBackend backend{h->scene, &per[w]};
        for (;;) {
            const U32 tile = next.fetch_add(1);
            if (tile >= tiles) break;
            for (U32 s = 0; s < count; ++s)
                for (U32 pos = 0; pos < 64; ++pos) {
                    const U32 pixel = xi::async::tilePixel(tile, pos, c.width, c.height);
                    if (pixel == ~0u) continue;
                    const U32 index = first + s;
                    xi::async::Radiance r;
                    const auto st = xi::async::integratePaths(c, pixel, index, backend, r);
                    if (st == xi::async::SampleStatus::Done) {
                        // Each tile is one worker's: no two threads share a pixel.
                        for (int k = 0; k < 3; ++k) sums[4 * size_t(pixel) + k] += r.rgb[k];
                        sums[4 * size_t(pixel) + 3] += r.alpha;
                        if (odd && (index & 1)) {
                            for (int k = 0; k < 3; ++k) odd[4 * size_t(pixel) + k] += r.rgb[k];
                            odd[4 * size_t(pixel) + 3] += r.alpha;
                        }
                        ++counts[pixel];
                    } else if (st == xi::async::SampleStatus::Skip) {
                        ++counts[pixel];
                    } else {
                        ++errors;
                    }
                }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    Counts total;
    for (const auto& k : per) {
        total.trace += k.trace;
        total.nee += k.nee;
        total.bsdf += k.bsdf;
        total.held += k.held;
    }
    if (rays) {
        rays[0] = total.trace;
        rays[1] = total.nee;
        rays[2] = total.bsdf;
        rays[3] = total.held;
    }
    return errors ? X2_EDEVICE : X2_OK;
}

// renderChunk over a list of tiles only (a bounded sample of a frame for the CPU baseline): each tile's 64 pixels
// times samples [first, first+count); returns the samples rendered in *samples and ray counts in rays[4].
int x2ref_render_tiles(void* p, const uint32_t* tiles, uint32_t ntiles, uint32_t first, uint32_t count, int threads, uint64_t* samples,
                       uint64_t* rays) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !tiles) return X2_EINVAL;
    const auto& c = h->scene.config;
    std::atomic<U32> next{0};
    std::atomic<uint64_t> done{0}, errors{0};
    std::vector<Counts> per(std::max(threads, 1));
    auto work = [&](int w) {
        OracleBackend backend{h->scene, &per[w]};
        for (;;) {
            const U32 k = next.fetch_add(1);
            if (k >= ntiles) break;
            for (U32 s = 0; s < count; ++s)
                for (U32 pos = 0; pos < 64; ++pos) {
                    const U32 pixel = xi::async::tilePixel(tiles[k], pos, c.width, c.height);
                    if (pixel == ~0u) continue;
                    xi::async::Radiance r;
                    const auto st = xi::async::integratePaths(c, pixel, first + s, backend, r);
                    if (st == xi::async::SampleStatus::Done) ++done;
                    else ++errors;
                }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    Counts total;
    for (const auto& k : per) {
        total.trace += k.trace;
        total.nee += k.nee;
        total.bsdf += k.bsdf;
        total.held += k.held;
    }
    if (samples) *samples = done;
    if (rays) {
        rays[0] = total.trace;
        rays[1] = total.nee;
        rays[2] = total.bsdf;
        rays[3] = total.held;
    }
    return errors ? X2_EDEVICE : X2_OK;
}

// renderChunk over a list of tiles with their film: tile k's position pos (pixel tilePixel(tiles[k], pos)) sums its
// samples [first, first+count) in FP64 into sums[4 (64 k + pos) ...] (rgb, alpha) and counts them in counts[64 k +
// pos]; positions past the frame's edge stay zero. Each tile is one worker's, so no two threads share a sum.
int x2ref_render_tiles_film(void* p, const uint32_t* tiles, uint32_t ntiles, uint32_t first, uint32_t count, int threads, double* sums,
                            uint32_t* counts) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !tiles || !sums || !counts) return X2_EINVAL;
    const auto& c = h->scene.config;
    std::atomic<U32> next{0};
    std::atomic<uint64_t> errors{0};
    std::vector<Counts> per(std::max(threads, 1));
    auto work = [&](int w) {
        OracleBackend backend{h->scene, &per[w]};
        for (;;) {
            const U32 k = next.fetch_add(1);
            if (k >= ntiles) break;
            for (U32 s = 0; s < count; ++s)
                for (U32 pos = 0; pos < 64; ++pos) {
                    const U32 pixel = xi::async::tilePixel(tiles[k], pos, c.width, c.height);
                    if (pixel == ~0u) continue;
                    xi::async::Radiance r;
                    const auto st = xi::async::integratePaths(c, pixel, first + s, backend, r);
                    double* sum = sums + 4 * (64 * size_t(k) + pos);
                    if (st == xi::async::SampleStatus::Done) {
                        for (int j = 0; j < 3; ++j) sum[j] += r.rgb[j];
                        sum[3] += r.alpha;
                        ++counts[64 * size_t(k) + pos];
                    } else if (st == xi::async::SampleStatus::Skip) {
                        ++counts[64 * size_t(k) + pos];
                    } else {
                        ++errors;
                    }
                }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    return errors ? X2_EDEVICE : X2_OK;
}

// The FP64 adjoint (adjoint64.h) of samples [first, first + count) of every pixel: given dL/dimage (3 floats a pixel,
// the image being the mean of those samples), the gradients with respect to each material's albedo (3 a material),
// roughness (1 a material) and each light's radiance (3 a light), summed in double; `image` (3 doubles a pixel, or
// null) gets each pixel's radiance summed over the samples in double; `mass` (or null) each gradient's sum of credit
// magnitudes, in the gradients' order (albedo, roughness, radiance). Requires no volumes and bsdf_samples = 1.
// Parameters as set with x2ref_set_params (or the scene's own).
int x2ref_adjoint64(void* p, uint32_t first, uint32_t count, const float* dldi, int threads, double* albedo, double* roughness,
                    double* radiance, double* image, double* mass, double* texture) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !dldi || !albedo || !roughness || !radiance || count == 0) return X2_EINVAL;
    const auto& c = h->x.config;
    if (c.volume_count || c.bsdf_samples != 1 || c.max_depth >= 128) return X2_EINVAL;
    const U32 pixels = c.width * c.height, M = U32(h->x.materials.size()), L = U32(h->x.lights.size());
    threads = std::max(threads, 1);
    std::vector<adj64::Grads> per(threads);
    std::atomic<U32> next{0};
    auto work = [&](int w) {
        adj64::Grads& g = per[w];
        g.albedo.assign(3 * M, 0.0);
        g.roughness.assign(M, 0.0);
        g.radiance.assign(3 * L, 0.0);
        g.albedoMass.assign(3 * M, 0.0);
        g.roughnessMass.assign(M, 0.0);
        g.radianceMass.assign(3 * L, 0.0);
        if (texture) g.texture.assign(3 * h->x.texels, 0.0);
        for (;;) {
            const U32 px = next.fetch_add(1);
            if (px >= pixels) break;
            const adj64::D3 delta{double(dldi[3 * size_t(px)]) / count, double(dldi[3 * size_t(px) + 1]) / count, double(dldi[3 * size_t(px) + 2]) / count};
            adj64::Tracer t{h->scene, h->x, g, delta};
            adj64::D3 sum{0, 0, 0};
            for (U32 k = 0; k < count; ++k) sum = sum + t.sample(px, first + k);
            if (image) {
                image[3 * size_t(px)] = sum.x;
                image[3 * size_t(px) + 1] = sum.y;
                image[3 * size_t(px) + 2] = sum.z;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < threads; ++w) pool.emplace_back(work, w);
    work(0);
    for (auto& t : pool) t.join();
    for (U32 i = 0; i < 3 * M; ++i) albedo[i] = 0;
    for (U32 i = 0; i < M; ++i) roughness[i] = 0;
    for (U32 i = 0; i < 3 * L; ++i) radiance[i] = 0;
    if (mass)
        for (U32 i = 0; i < 4 * M + 3 * L; ++i) mass[i] = 0;
    if (texture) {
        for (U64 i = 0; i < 3 * h->x.texels; ++i) texture[i] = 0;
        for (const auto& g : per)
            for (U64 i = 0; i < 3 * h->x.texels; ++i) texture[i] += g.texture[i];
    }
    for (const auto& g : per) {
        for (U32 i = 0; i < 3 * M; ++i) albedo[i] += g.albedo[i];
        for (U32 i = 0; i < M; ++i) roughness[i] += g.roughness[i];
        for (U32 i = 0; i < 3 * L; ++i) radiance[i] += g.radiance[i];
        if (!mass) continue;
        for (U32 i = 0; i < 3 * M; ++i) mass[i] += g.albedoMass[i];
        for (U32 i = 0; i < M; ++i) mass[3 * M + i] += g.roughnessMass[i];
        for (U32 i = 0; i < 3 * L; ++i) mass[4 * M + i] += g.radianceMass[i];
    }
    return X2_OK;
}

// A texture's texels for the FP64 adjoint (as x2_scene_set_texture sets the engine's); the reference integrator's
// images are left as they are.
int x2ref_set_texture(void* p, uint32_t texture, const float* rgb) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !rgb || texture >= h->x.textures.size()) return X2_EINVAL;
    auto& t = h->x.textures[texture];
    t.rgb.assign(rgb, rgb + 3 * size_t(t.width) * t.height);
    return X2_OK;
}

// The FP64 adjoint's parameters, as x2_scene_set_params sets the engine's (null leaves a set as it is). The reference
// integrator's records are left as they are: after this, only x2ref_adjoint64 sees the new values.
int x2ref_set_params(void* p, const float* albedo, const float* roughness, const float* radiance) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return X2_EINVAL;
    for (size_t m = 0; m < h->x.materials.size(); ++m) {
        if (albedo)
            for (int k = 0; k < 3; ++k) h->x.materials[m].diffuse[k] = albedo[3 * m + k];
        if (roughness) h->x.materials[m].roughness = roughness[m];
    }
    if (radiance)
        for (size_t j = 0; j < h->x.lights.size(); ++j)
            for (int k = 0; k < 3; ++k) h->x.lights[j].radiance[k] = radiance[3 * j + k];
    return X2_OK;
}

// Traversal parity: closest hit (triangle, t) or ~0u, and occlusion, for n rays (origin, direction, near, far).
int x2ref_trace(void* p, const float* rays, uint64_t n, uint32_t* tri, float* t, uint32_t* occl) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return X2_EINVAL;
    for (uint64_t i = 0; i < n; ++i) {
        const float* r = rays + 8 * i;
        const V3 o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
        float th;
        tri[i] = closest(h->scene, o, d, r[6], r[7], th);
        t[i] = tri[i] == ~0u ? 0.0f : th;
        occl[i] = occluded(h->scene, o, d, r[6], r[7]) ? 1u : 0u;
    }
    return X2_OK;
}

// The same queries by testing every triangle (no BVH): the arbiter when two traversals disagree.
int x2ref_trace_brute(void* p, const float* rays, uint64_t n, uint32_t* tri, float* t, uint32_t* occl) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return X2_EINVAL;
    const Scene& s = h->scene;
    const U32 nt = U32(s.tris.size() / 3);
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        for (uint64_t i; (i = next.fetch_add(1)) < n;) {
            const float* r = rays + 8 * i;
            const V3 o{r[0], r[1], r[2]}, d{r[3], r[4], r[5]};
            const TriTest sh = shear(d);
            U32 best = ~0u;
            float tBest = r[7];
            bool any = false;
            for (U32 k = 0; k < nt; ++k) {
                float th;
                const V3 a = s.vertex(s.tris[3 * k]), b = s.vertex(s.tris[3 * k + 1]), c = s.vertex(s.tris[3 * k + 2]);
                if (triHit(sh, o, a, b, c, r[6], r[7], th)) any = true;
                if (triHit(sh, o, a, b, c, r[6], tBest, th) && (th < tBest || (th == tBest && k < best))) {
                    tBest = th;
                    best = k;
                }
            }
            tri[i] = best;
            t[i] = best == ~0u ? 0.0f : tBest;
            occl[i] = any ? 1u : 0u;
        }
    };
    std::vector<std::thread> pool;
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned w = 1; w < threads; ++w) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    return X2_OK;
}

// ---- adaptive sampling (async_integrator.h:3088-3125, async_adaptive.h, async_adaptive_core.h), the reference's own ----
// Each pixel's error (pixelError) from a film: sums and odd sums (4 doubles a pixel) and counts.
int x2ref_pixel_errors(const double* sums, const double* odd, const uint32_t* counts, uint64_t pixels, float* errors) {
    for (uint64_t i = 0; i < pixels; ++i) errors[i] = xi::async::pixelError(sums + 4 * i, odd + 4 * i, counts[i]);
    return X2_OK;
}
// The region trees over a width x height image rebuilt from per-pixel errors (Regions, target error), and each 8x8
// tile's mask of pixels still to sample (sampleArea, bit y * 8 + x, masked to the image); *done = 1 when every region
// has converged. masks: one a tile, tiles in row-major order.
int x2ref_adaptive_masks(uint32_t width, uint32_t height, float target, const float* errors, uint64_t* masks, uint32_t* done) {
    namespace ad = xi::async::adaptive;
    ad::Regions regions(int(width), int(height), target);
    for (size_t r = 0; r < regions.count(); ++r) regions.update(r, errors);
    const uint32_t tilesX = (width + 7) / 8, tilesY = (height + 7) / 8;
    for (uint32_t ty = 0; ty < tilesY; ++ty)
        for (uint32_t tx = 0; tx < tilesX; ++tx) {
            uint64_t inImage = 0;
            for (uint32_t p = 0; p < 64; ++p)
                if (tx * 8 + p % 8 < width && ty * 8 + p / 8 < height) inImage |= uint64_t(1) << p;
            masks[size_t(ty) * tilesX + tx] = inImage & regions.sampleArea(int(tx * 8), int(ty * 8));
        }
    *done = regions.done() ? 1u : 0u;
    return X2_OK;
}
// MoonRay's pass schedule for maxSamples (schedule): passes[2 k], passes[2 k + 1] = start, end; returns the count.
uint32_t x2ref_adaptive_schedule(uint32_t maxSamples, uint32_t* passes, uint32_t capacity) {
    const auto s = xi::async::adaptive::schedule(maxSamples);
    for (size_t k = 0; k < s.size() && k < capacity; ++k) {
        passes[2 * k] = s[k].start;
        passes[2 * k + 1] = s[k].end;
    }
    return uint32_t(s.size());
}

// sample::samplingWord (sample_stream.h:127-144), the reference's own.
int x2ref_sample_words(const x2_identity* ids, const uint32_t* dims, uint64_t n, uint32_t policy, uint32_t* out) {
    for (uint64_t i = 0; i < n; ++i) {
        const xi::sample::Identity id{ids[i].pixel, ids[i].index, ids[i].stream, ids[i].branch};
        out[i] = xi::sample::samplingWord(id, dims[i], policy);
    }
    return X2_OK;
}

// ---- the reference's cellular generations (async_adaptive.h Cellular) ----
void* x2ref_cellular_open(int width, int height, float target, const uint64_t* inImage, uint32_t tiles) {
    auto* c = new xi::async::adaptive::Cellular(width, height, target);
    c->deadForever(std::vector<std::uint64_t>(inImage, inImage + tiles));
    return c;
}
void x2ref_cellular_free(void* c) { delete static_cast<xi::async::adaptive::Cellular*>(c); }
uint64_t x2ref_cellular_update(void* c, const float* errors) { return static_cast<xi::async::adaptive::Cellular*>(c)->update(errors); }
uint64_t x2ref_cellular_update_budget(void* c, const float* errors, const uint32_t* planned, uint64_t pixels, double remaining,
                                      uint32_t most, float floor) {
    const std::vector<uint32_t> samples(planned, planned + pixels);
    const xi::async::adaptive::Budget b{&samples, remaining, most, floor};
    return static_cast<xi::async::adaptive::Cellular*>(c)->update(errors, &b);
}
void x2ref_cellular_ratio(void* c, float* out, uint32_t tiles) {
    for (uint32_t t = 0; t < tiles; ++t) out[t] = static_cast<xi::async::adaptive::Cellular*>(c)->ratio(t);
}
void x2ref_cellular_alive(void* c, uint8_t* out, uint32_t tiles) {
    for (uint32_t t = 0; t < tiles; ++t) out[t] = static_cast<xi::async::adaptive::Cellular*>(c)->alive(t) ? 1 : 0;
}

// ---- the reference's work grid (async_grid.h Grid), driven call by call ----
void* x2ref_grid_open(uint32_t width, uint32_t height, uint32_t spp, uint32_t cellSize, uint32_t samplesPerChunk, int mode,
                      int progressive, uint32_t sampleFirst, uint32_t sampleCount, const uint32_t* owners, uint32_t ownerCount,
                      int empty, const int32_t* viewport) {
    namespace A = xi::async;
    A::GridOptions o;
    o.cellSize = cellSize;
    o.samplesPerChunk = samplesPerChunk;
    o.mode = mode;
    o.progressive = progressive != 0;
    o.sampleFirst = sampleFirst;
    o.sampleCount = sampleCount;
    std::vector<A::Device> own;
    for (uint32_t i = 0; owners && i < ownerCount; ++i) own.push_back(owners[i] ? A::Device::Gpu : A::Device::Cpu);
    int view[4];
    if (viewport)
        for (int k = 0; k < 4; ++k) view[k] = viewport[k];
    try {
        return new A::Grid(width, height, spp, o, owners ? &own : nullptr, empty != 0, viewport ? view : nullptr);
    } catch (...) {
        return nullptr;
    }
}
void x2ref_grid_free(void* g) { delete static_cast<xi::async::Grid*>(g); }
uint32_t x2ref_grid_cells(void* g) { return static_cast<xi::async::Grid*>(g)->cellCount(); }
uint64_t x2ref_grid_total(void* g) { return static_cast<xi::async::Grid*>(g)->totalChunks(); }
uint32_t x2ref_grid_ranges(void* g, uint32_t* out, uint32_t capacity) {
    const auto& r = static_cast<xi::async::Grid*>(g)->ranges();
    for (size_t k = 0; k < r.size() && k < capacity; ++k) {
        out[2 * k] = r[k].first;
        out[2 * k + 1] = r[k].count;
    }
    return uint32_t(r.size());
}
uint32_t x2ref_grid_claim(void* g, uint32_t cell, uint32_t n, x2_chunk* out, uint32_t device) {
    static_assert(sizeof(xi::async::Chunk) == sizeof(x2_chunk), "chunk layouts");
    return static_cast<xi::async::Grid*>(g)->claim(cell, n, reinterpret_cast<xi::async::Chunk*>(out), xi::async::Device(device));
}
uint32_t x2ref_grid_claimable(void* g, uint32_t cell, uint32_t device) {
    return static_cast<xi::async::Grid*>(g)->claimable(cell, xi::async::Device(device));
}
uint32_t x2ref_grid_remaining(void* g, uint32_t cell) { return static_cast<xi::async::Grid*>(g)->remaining(cell); }
uint32_t x2ref_grid_empty(void* g) { return static_cast<xi::async::Grid*>(g)->empty() ? 1u : 0u; }
uint32_t x2ref_grid_frontier(void* g, uint32_t device) { return static_cast<xi::async::Grid*>(g)->frontier(xi::async::Device(device)); }
uint32_t x2ref_grid_choose(void* g, uint32_t device, uint32_t current, uint32_t salt) {
    return static_cast<xi::async::Grid*>(g)->choose(xi::async::Device(device), current, salt);
}
uint32_t x2ref_grid_seed(void* g, uint32_t device, uint32_t worker, uint32_t workers) {
    return static_cast<xi::async::Grid*>(g)->seed(xi::async::Device(device), worker, workers);
}
void x2ref_grid_set_scores(void* g, const float* scores, uint32_t n) {
    static_cast<xi::async::Grid*>(g)->setScores(std::vector<float>(scores, scores + n));
}
void x2ref_grid_append(void* g, uint32_t cell, const x2_chunk* chunks, uint32_t n) {
    static_cast<xi::async::Grid*>(g)->append(cell, reinterpret_cast<const xi::async::Chunk*>(chunks), n);
}
void x2ref_grid_close(void* g) { static_cast<xi::async::Grid*>(g)->close(); }

// paths::childBranch (async_integrator.h:281-287), the reference's own.
uint64_t x2ref_child_branch(uint64_t parent, uint32_t a, uint32_t b) { return xi::async::paths::childBranch(parent, a, b); }

}  // extern "C"
