// Seeded synthetic scenes: the inputs of the tests and the bench (host code, not the hot path).
//
// Config 0, the closed box: five quads spanning [-1,1]^3 (floor, ceiling and back wall grey 0.73, left wall
// (0.63,0.065,0.05), right wall (0.14,0.45,0.09)), a 0.6 box and a 0.6x1.2x0.6 box rotated -18/+18 degrees about
// y (albedo 0.73), a 0.5x0.5 one-sided rect light (radiance 15) just below the ceiling facing down, a 40 degree
// pinhole at z = 3.5, 256x256, 16 spp, depth 8.
// Config 1: a 64x64 grid of 16x16-quad heightfield tiles (6-octave fBm, amplitude 0.3) plus 2000 level-4
// icospheres (centres uniform in a 20x20x4 box, radii log-uniform 0.05-0.5): 2,097,152 + 10,240,000 triangles.
// Materials 50/50 Lambert (albedo U[0.05,0.9]^3) or GGX (roughness U[0.05,0.8], F0 0.04 or metal U[0.5,1]^3),
// 16 rect lights of radiance U[1,20] and a constant environment of 0.2; 1920x1080, 64 spp, depth 12.
// Config 11: config 1 at about 1.2M triangles (32x32 tiles, level-2 icospheres). Config 100+k: config 1 scaled
// down by k for tests. Random numbers: xoshiro256** seeded by splitmix64.
#include "../../include/x2.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <new>
#include <vector>

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (int i = 0; i < 4; ++i) {  // splitmix64
            seed += 0x9e3779b97f4a7c15ull;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return double(next() >> 11) * 0x1p-53; }
    float uniform(float lo, float hi) { return float(lo + (hi - lo) * uniform()); }
};

struct V { float x, y, z; };
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V normalized(V a) { return a * (1.0f / std::sqrt(dot(a, a))); }

// The generator's scene: the descriptor first, so the library hands out the descriptor's address.
struct Holder {
    x2_scene_desc desc;
    std::vector<float> vertices;
    std::vector<uint32_t> triangles, meshFirst, meshMaterial;
    std::vector<x2_material> materials;
    std::vector<x2_light> lights;
    std::vector<x2_volume> volumes;
    std::vector<x2_grid> grids;
    std::vector<std::vector<float>> gridValues;
    std::vector<float> uvs;  // 2 a vertex when a mesh has texture coordinates (then every vertex has them)
    std::vector<x2_texture> textures;
    std::vector<std::vector<float>> textureValues;

    uint32_t vertex(V p) {
        vertices.push_back(p.x);
        vertices.push_back(p.y);
        vertices.push_back(p.z);
        return uint32_t(vertices.size() / 3 - 1);
    }
    void tri(uint32_t a, uint32_t b, uint32_t c) {
        triangles.push_back(a);
        triangles.push_back(b);
        triangles.push_back(c);
    }
    uint32_t triangleCount() const { return uint32_t(triangles.size() / 3); }
    void beginMesh(uint32_t material) {
        meshFirst.push_back(triangleCount());
        meshMaterial.push_back(material);
    }
    uint32_t material(const x2_material& m) {
        materials.push_back(m);
        return uint32_t(materials.size() - 1);
    }
    void quad(V a, V b, V c, V d) {  // a b c d counter-clockwise
        const uint32_t i = vertex(a), j = vertex(b), k = vertex(c), l = vertex(d);
        tri(i, j, k);
        tri(i, k, l);
    }
    void finish() {  // again after more lights or volumes: the descriptor refreshed, the meshes closed once
        if (meshFirst.size() == meshMaterial.size()) meshFirst.push_back(triangleCount());
        std::memset(&desc, 0, sizeof(desc));
        desc.vertex_count = uint32_t(vertices.size() / 3);
        desc.triangle_count = triangleCount();
        desc.mesh_count = uint32_t(meshMaterial.size());
        desc.material_count = uint32_t(materials.size());
        desc.light_count = uint32_t(lights.size());
        desc.vertices = vertices.data();
        desc.triangles = triangles.data();
        desc.mesh_first = meshFirst.data();
        desc.mesh_material = meshMaterial.data();
        desc.materials = materials.data();
        desc.lights = lights.data();
        for (size_t g = 0; g < grids.size(); ++g) grids[g].values = gridValues[g].data();
        desc.volume_count = uint32_t(volumes.size());
        desc.grid_count = uint32_t(grids.size());
        desc.volumes = volumes.data();
        desc.grids = grids.data();
        for (size_t t = 0; t < textures.size(); ++t) textures[t].rgb = textureValues[t].data();
        desc.texture_count = uint32_t(textures.size());
        desc.textures = textures.data();
        desc.uvs = uvs.empty() ? nullptr : uvs.data();
    }
};

x2_material lambert(float r, float g, float b) {
    x2_material m{};
    m.kind = X2_MAT_LAMBERT;
    m.diffuse[0] = r;
    m.diffuse[1] = g;
    m.diffuse[2] = b;
    m.roughness = 1.0f;
    return m;
}
x2_material ggx(float f0r, float f0g, float f0b, float roughness) {
    x2_material m{};
    m.kind = X2_MAT_GGX;
    m.specular[0] = f0r;
    m.specular[1] = f0g;
    m.specular[2] = f0b;
    m.roughness = roughness;
    return m;
}

// A one-sided rect light centred at c with edge vectors eu, ev (full lengths) shining along n = its local +Z
// (lights::Light's layout: rows of the local frame, scale 1, half sizes in local units).
x2_light rectLight(V c, V eu, V ev, V n, float r, float g, float b) {
    x2_light l{};
    l.type = X2_LIGHT_RECT;
    l.sidedness = X2_SIDE_REGULAR;
    l.visible_in_camera = 1;
    l.radiance[0] = r;
    l.radiance[1] = g;
    l.radiance[2] = b;
    const V x = normalized(eu), y = normalized(ev), z = normalized(n);
    const float hw = 0.5f * std::sqrt(dot(eu, eu)), hh = 0.5f * std::sqrt(dot(ev, ev));
    const V rows[3] = {x, y, z};
    for (int i = 0; i < 3; ++i) {
        l.local2render[i][0] = rows[i].x;
        l.local2render[i][1] = rows[i].y;
        l.local2render[i][2] = rows[i].z;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) l.render2local[i][j] = l.render2local_rot[i][j] = l.local2render[j][i];
    l.position[0] = c.x;
    l.position[1] = c.y;
    l.position[2] = c.z;
    l.direction[0] = z.x;
    l.direction[1] = z.y;
    l.direction[2] = z.z;
    l.scale = 1.0f;
    l.half_width = hw;
    l.half_height = hh;
    l.inv_area = 1.0f / (4.0f * hw * hh);
    l.plane_offset = -dot(z, c);
    l.visibility_mask = 0xfcu;
    return l;
}
x2_light envLight(float v) {
    x2_light l{};
    l.type = X2_LIGHT_ENV;
    l.visible_in_camera = 1;
    l.radiance[0] = l.radiance[1] = l.radiance[2] = v;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) l.local2render[i][j] = l.render2local[i][j] = l.render2local_rot[i][j] = i == j ? 1.0f : 0.0f;
    l.direction[2] = 1.0f;
    l.scale = 1.0f;
    l.inv_area = 0.0795774715459476678845f;  // 1 / (4 pi): the whole sphere
    l.visibility_mask = 0xfcu;
    return l;
}

// A pinhole camera at eye looking at target (vertical field of view fovDeg), raster width x height, as
// perspectiveRay (camera_core.h:217) reads it: raster (x, y, -1) to a camera-space point on z = -1.
x2_camera pinhole(V eye, V target, float fovDeg, uint32_t width, uint32_t height) {
    x2_camera c{};
    const float s = 2.0f * std::tan(0.5f * fovDeg * 3.14159265358979f / 180.0f) / float(height);
    c.raster_to_camera[0][0] = s;
    c.raster_to_camera[1][1] = -s;
    c.raster_to_camera[2][2] = 1.0f;
    c.raster_to_camera[3][0] = -0.5f * float(width) * s;
    c.raster_to_camera[3][1] = 0.5f * float(height) * s;
    c.raster_to_camera[3][3] = 1.0f;
    const V forward = normalized(target - eye);
    V right = cross(forward, V{0, 1, 0});
    if (dot(right, right) < 1e-12f) right = V{1, 0, 0};
    right = normalized(right);
    const V up = cross(right, forward), back = forward * -1.0f;
    const V rows[3] = {right, up, back};
    for (int i = 0; i < 3; ++i) {
        c.camera_to_render[i][0] = rows[i].x;
        c.camera_to_render[i][1] = rows[i].y;
        c.camera_to_render[i][2] = rows[i].z;
    }
    c.camera_to_render[3][0] = eye.x;
    c.camera_to_render[3][1] = eye.y;
    c.camera_to_render[3][2] = eye.z;
    c.camera_to_render[3][3] = 1.0f;
    c.near_clip = 1e-3f;
    c.far_clip = 1e5f;
    return c;
}

void boxMesh(Holder& h, V center, V size, float angleDeg) {
    const float a = angleDeg * 3.14159265358979f / 180.0f, cs = std::cos(a), sn = std::sin(a);
    auto at = [&](float x, float y, float z) {
        const V p{x * size.x * 0.5f, y * size.y * 0.5f, z * size.z * 0.5f};
        return V{cs * p.x + sn * p.z, p.y, -sn * p.x + cs * p.z} + center;
    };
    const V c[8] = {at(-1, -1, -1), at(1, -1, -1), at(1, 1, -1), at(-1, 1, -1),
                    at(-1, -1, 1),  at(1, -1, 1),  at(1, 1, 1),  at(-1, 1, 1)};
    const int f[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {3, 7, 6, 2}, {0, 4, 7, 3}, {1, 2, 6, 5}};
    for (auto& q : f) h.quad(c[q[0]], c[q[1]], c[q[2]], c[q[3]]);
}

void fillConfig(x2_config* c, uint32_t width, uint32_t height, uint32_t spp, uint32_t depth, uint32_t lights,
                uint32_t visible) {
    x2_config_defaults(c);
    c->width = width;
    c->height = height;
    c->seed = 1;
    c->spp = spp;
    c->light_count = lights;
    c->visible_lights = visible;
    c->max_depth = c->max_diffuse_depth = c->max_glossy_depth = c->max_mirror_depth = depth;
    // MoonRay's russian_roulette_threshold default (run_paths_benchmark.py uses it): RR past the first
    // non-mirror vertex (async_integrator.h:2450).
    c->rr_threshold = 0.0375f;
}

Holder* makeBox(x2_config* cfg) {
    auto* h = new Holder();
    const uint32_t grey = h->material(lambert(0.73f, 0.73f, 0.73f));
    const uint32_t red = h->material(lambert(0.63f, 0.065f, 0.05f));
    const uint32_t green = h->material(lambert(0.14f, 0.45f, 0.09f));
    h->beginMesh(grey);  // floor
    h->quad({-1, -1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, -1, -1});
    h->beginMesh(grey);  // ceiling
    h->quad({-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1});
    h->beginMesh(grey);  // back wall
    h->quad({-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1});
    h->beginMesh(red);  // left wall
    h->quad({-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1});
    h->beginMesh(green);  // right wall
    h->quad({1, -1, -1}, {1, -1, 1}, {1, 1, 1}, {1, 1, -1});
    h->beginMesh(grey);
    boxMesh(*h, {0.33f, -0.7f, 0.3f}, {0.6f, 0.6f, 0.6f}, -18.0f);
    h->beginMesh(grey);
    boxMesh(*h, {-0.35f, -0.4f, -0.3f}, {0.6f, 1.2f, 0.6f}, 18.0f);
    h->lights.push_back(rectLight({0, 0.99f, 0}, {0.5f, 0, 0}, {0, 0, 0.5f}, {0, -1, 0}, 15, 15, 15));
    h->desc.camera = pinhole({0, 0, 3.5f}, {0, 0, 0}, 40.0f, 256, 256);
    const x2_camera cam = h->desc.camera;
    fillConfig(cfg, 256, 256, 16, 8, 1, 1);
    h->finish();
    h->desc.camera = cam;
    return h;
}

// Hash value noise with a smooth interpolant, summed over octaves (fBm).
float hashLattice(int x, int z, uint32_t seed) {
    uint32_t h = uint32_t(x) * 0x8da6b343u ^ uint32_t(z) * 0xd8163841u ^ seed * 0xcb1ab31fu;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    return float(h & 0xffffff) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}
float valueNoise(float x, float z, uint32_t seed) {
    const int ix = int(std::floor(x)), iz = int(std::floor(z));
    const float fx = x - float(ix), fz = z - float(iz);
    const float sx = fx * fx * (3 - 2 * fx), sz = fz * fz * (3 - 2 * fz);
    const float a = hashLattice(ix, iz, seed), b = hashLattice(ix + 1, iz, seed);
    const float c = hashLattice(ix, iz + 1, seed), d = hashLattice(ix + 1, iz + 1, seed);
    return (a + (b - a) * sx) + ((c + (d - c) * sx) - (a + (b - a) * sx)) * sz;
}
float fbm(float x, float z, int octaves, uint32_t seed) {
    float sum = 0, amp = 0.5f, freq = 1;
    for (int o = 0; o < octaves; ++o) {
        sum += amp * valueNoise(x * freq, z * freq, seed + uint32_t(o));
        amp *= 0.5f;
        freq *= 2.0f;
    }
    return sum;
}

// A unit icosphere subdivided `level` times (20 * 4^level faces).
void icosphere(int level, std::vector<V>& verts, std::vector<uint32_t>& faces) {
    const float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    verts = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
             {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& v : verts) v = normalized(v);
    faces = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
             3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int l = 0; l < level; ++l) {
        std::map<uint64_t, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) {
            const uint64_t key = a < b ? (uint64_t(a) << 32 | b) : (uint64_t(b) << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            verts.push_back(normalized((verts[a] + verts[b]) * 0.5f));
            const uint32_t i = uint32_t(verts.size() - 1);
            mid[key] = i;
            return i;
        };
        std::vector<uint32_t> next;
        next.reserve(faces.size() * 4);
        for (size_t f = 0; f < faces.size(); f += 3) {
            const uint32_t a = faces[f], b = faces[f + 1], c = faces[f + 2];
            const uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            const uint32_t add[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
            next.insert(next.end(), add, add + 12);
        }
        faces.swap(next);
    }
}

x2_material randomMaterial(Rng& r) {
    if (r.uniform() < 0.5) return lambert(r.uniform(0.05f, 0.9f), r.uniform(0.05f, 0.9f), r.uniform(0.05f, 0.9f));
    const float roughness = r.uniform(0.05f, 0.8f);
    if (r.uniform() < 0.5) return ggx(0.04f, 0.04f, 0.04f, roughness);
    return ggx(r.uniform(0.5f, 1.0f), r.uniform(0.5f, 1.0f), r.uniform(0.5f, 1.0f), roughness);
}

Holder* makeField(uint64_t seed, int tilesPerSide, int spheres, int icoLevel, uint32_t width, uint32_t height, uint32_t spp,
                  uint32_t depth, x2_config* cfg, float radiusScale = 1.0f) {
    auto* h = new Holder();
    Rng r(seed);
    const int quadsPerTile = 16, n = tilesPerSide * quadsPerTile;
    const float extent = 20.0f, cell = extent / float(n);
    // The heightfield's shared vertex grid, (n+1)^2 vertices over [-10,10]^2 in x and z.
    const uint32_t first = h->desc.vertex_count;
    (void)first;
    const uint32_t base = uint32_t(h->vertices.size() / 3);
    h->vertices.reserve(size_t(n + 1) * (n + 1) * 3);
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
            const float x = -10.0f + float(i) * cell, z = -10.0f + float(j) * cell;
            h->vertex({x, 0.3f * fbm(x * 0.25f, z * 0.25f, 6, uint32_t(seed)), z});
        }
    auto at = [&](int i, int j) { return base + uint32_t(j) * uint32_t(n + 1) + uint32_t(i); };
    for (int tj = 0; tj < tilesPerSide; ++tj)
        for (int ti = 0; ti < tilesPerSide; ++ti) {
            h->beginMesh(h->material(randomMaterial(r)));
            for (int qj = 0; qj < quadsPerTile; ++qj)
                for (int qi = 0; qi < quadsPerTile; ++qi) {
                    const int i = ti * quadsPerTile + qi, j = tj * quadsPerTile + qj;
                    h->tri(at(i, j), at(i, j + 1), at(i + 1, j + 1));
                    h->tri(at(i, j), at(i + 1, j + 1), at(i + 1, j));
                }
        }
    std::vector<V> unitVerts;
    std::vector<uint32_t> unitFaces;
    icosphere(icoLevel, unitVerts, unitFaces);
    for (int s = 0; s < spheres; ++s) {
        const V c{r.uniform(-10.0f, 10.0f), r.uniform(0.0f, 4.0f), r.uniform(-10.0f, 10.0f)};
        const float radius = radiusScale * float(0.05 * std::exp(r.uniform() * std::log(10.0)));
        h->beginMesh(h->material(randomMaterial(r)));
        const uint32_t b = uint32_t(h->vertices.size() / 3);
        for (const V& v : unitVerts) h->vertex(c + v * radius);
        for (size_t f = 0; f < unitFaces.size(); f += 3) h->tri(b + unitFaces[f], b + unitFaces[f + 1], b + unitFaces[f + 2]);
    }
    for (int l = 0; l < 16; ++l) {
        const V c{r.uniform(-9.0f, 9.0f), r.uniform(5.0f, 8.0f), r.uniform(-9.0f, 9.0f)};
        const float w = r.uniform(1.0f, 2.0f), d = r.uniform(1.0f, 2.0f);
        const float rad = r.uniform(1.0f, 20.0f);
        h->lights.push_back(rectLight(c, {w, 0, 0}, {0, 0, d}, {0, -1, 0}, rad, rad, rad));
    }
    h->lights.push_back(envLight(0.2f));
    fillConfig(cfg, width, height, spp, depth, uint32_t(h->lights.size()), uint32_t(h->lights.size()));
    h->finish();
    h->desc.camera = pinhole({0, 7, 17}, {0, 0, -1}, 45.0f, width, height);
    return h;
}

// fp16 rounding (round to nearest, ties to even) of a finite float in half's range: the density grid is stored at
// half precision, as the scene gives it, and read back as the floats it rounds to.
float roundHalf(float f) {
    if (f == 0.0f) return f;
    int e;
    std::frexp(f, &e);                      // f = m 2^e, 0.5 <= |m| < 1
    const int bits = e - 1 >= -14 ? 10 : 10 - (-14 - (e - 1));  // mantissa bits kept (subnormals keep fewer)
    const float q = std::ldexp(1.0f, (e - 1) - bits);
    return float(std::nearbyint(double(f) / double(q)) * double(q));
}

// Value noise in 3D with a smooth interpolant, summed over octaves.
float hash3(int x, int y, int z, uint32_t seed) {
    uint32_t h = uint32_t(x) * 0x8da6b343u ^ uint32_t(y) * 0x68e31da4u ^ uint32_t(z) * 0xd8163841u ^ seed * 0xcb1ab31fu;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    return float(h & 0xffffff) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}
float noise3(float x, float y, float z, uint32_t seed) {
    const int ix = int(std::floor(x)), iy = int(std::floor(y)), iz = int(std::floor(z));
    const float fx = x - float(ix), fy = y - float(iy), fz = z - float(iz);
    const float sx = fx * fx * (3 - 2 * fx), sy = fy * fy * (3 - 2 * fy), sz = fz * fz * (3 - 2 * fz);
    float v[2][2];
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 2; ++k) {
            const float a = hash3(ix, iy + j, iz + k, seed), b = hash3(ix + 1, iy + j, iz + k, seed);
            v[j][k] = a + (b - a) * sx;
        }
    const float y0 = v[0][0] + (v[1][0] - v[0][0]) * sy, y1 = v[0][1] + (v[1][1] - v[0][1]) * sy;
    return y0 + (y1 - y0) * sz;
}
float fbm3(float x, float y, float z, int octaves, uint32_t seed) {
    float sum = 0, amp = 0.5f, freq = 1;
    for (int o = 0; o < octaves; ++o) {
        sum += amp * noise3(x * freq, y * freq, z * freq, seed + uint32_t(o));
        amp *= 0.5f;
        freq *= 2.0f;
    }
    return sum;
}

// A blackbody's colour at kelvin, normalised to unit maximum (Tanner Helland's fit to the CIE blackbody locus).
V blackbody(float kelvin) {
    const double t = kelvin / 100.0;
    double r, g, b;
    if (t <= 66.0) {
        r = 255.0;
        g = 99.4708025861 * std::log(t) - 161.1195681661;
    } else {
        r = 329.698727446 * std::pow(t - 60.0, -0.1332047592);
        g = 288.1221695283 * std::pow(t - 60.0, -0.0755148492);
    }
    if (t >= 66.0) b = 255.0;
    else if (t <= 19.0) b = 0.0;
    else b = 138.5177312231 * std::log(t - 10.0) - 305.0447927307;
    auto c = [](double v) { return float(std::min(255.0, std::max(0.0, v)) / 255.0); };
    return {c(r), c(g), c(b)};
}

// A Distant light of radiance v from direction `toward` (the way its light travels), angular diameter 0.53 degrees.
x2_light distantLight(V toward, float v) {
    x2_light l{};
    l.type = X2_LIGHT_DISTANT;
    l.radiance[0] = l.radiance[1] = l.radiance[2] = v;
    const V d = normalized(toward);
    const V a = std::fabs(d.x) < 0.9f ? V{1, 0, 0} : V{0, 1, 0};
    const V u = normalized(cross(a, d)), w = cross(d, u);
    const V rowsOf[3] = {u, w, d};
    for (int i = 0; i < 3; ++i) {
        const float r[3] = {rowsOf[i].x, rowsOf[i].y, rowsOf[i].z};
        for (int j = 0; j < 3; ++j) l.local2render[i][j] = l.render2local_rot[j][i] = l.render2local[j][i] = r[j];
    }
    l.direction[0] = d.x;
    l.direction[1] = d.y;
    l.direction[2] = d.z;
    l.scale = 1.0f;
    const double half = 0.5 * 0.53 * 3.14159265358979323846 / 180.0;
    l.cos_theta_max = float(std::cos(half));
    l.versine_theta_max = float(1.0 - std::cos(half));
    l.inv_area = float(1.0 / (2.0 * 3.14159265358979323846 * (1.0 - std::cos(half))));
    l.visibility_mask = 0xfcu;
    return l;
}

// The participating medium (config 3): an n^3 grid over the cube [-0.9, 0.9]^3 inside the config-0 box, density from
// seeded 5-octave 3D fBm, its lowest 40% empty, scaled to [0, 8] per unit length and stored at half precision; a
// temperature channel on the hottest 10% of voxels (1000-3000 K, half precision) glowing with its blackbody colour; a
// VdbVolume (trilinear density, HG g = 0.6, albedo 0.9); the box's rect light and a sun (Distant, radiance 5).
Holder* makeVolumeBox(uint64_t seed, int n, uint32_t width, uint32_t height, uint32_t spp, uint32_t depth, x2_config* cfg) {
    x2_config boxCfg;
    Holder* h = makeBox(&boxCfg);
    const float lo = -0.9f, extent = 1.8f, voxel = extent / float(n);
    const size_t cells = size_t(n) * n * n;
    std::vector<float> raw(cells), heat(cells);
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const float x = (float(i) + 0.5f) / float(n) * 4.0f, y = (float(j) + 0.5f) / float(n) * 4.0f, z = (float(k) + 0.5f) / float(n) * 4.0f;
                const size_t c = (size_t(k) * n + j) * n + i;
                raw[c] = fbm3(x, y, z, 5, uint32_t(seed));
                heat[c] = fbm3(x + 17.0f, y + 5.0f, z + 11.0f, 3, uint32_t(seed) + 101u);
            }
    std::vector<float> sorted = raw;
    std::nth_element(sorted.begin(), sorted.begin() + long(cells * 2 / 5), sorted.end());
    const float threshold = sorted[cells * 2 / 5];
    float top = threshold;
    for (float v : raw) top = std::max(top, v);
    std::vector<float> hs = heat;
    std::nth_element(hs.begin(), hs.begin() + long(cells * 9 / 10), hs.end());
    const float hot = hs[cells * 9 / 10];
    float hottest = hot;
    for (float v : heat) hottest = std::max(hottest, v);
    std::vector<float> density(cells), emission(3 * cells, 0.0f);
    for (size_t c = 0; c < cells; ++c) {
        density[c] = raw[c] > threshold ? roundHalf(8.0f * (raw[c] - threshold) / (top - threshold)) : 0.0f;
        if (heat[c] > hot && density[c] > 0.0f) {
            const float kelvin = roundHalf(1000.0f + 2000.0f * (heat[c] - hot) / std::max(hottest - hot, 1e-6f));
            const V rgb = blackbody(kelvin);
            const float power = 4.0f * (kelvin / 3000.0f) * (kelvin / 3000.0f) * (kelvin / 3000.0f) * (kelvin / 3000.0f);
            emission[3 * c] = rgb.x * power;
            emission[3 * c + 1] = rgb.y * power;
            emission[3 * c + 2] = rgb.z * power;
        }
    }
    auto grid = [&](uint32_t channels, std::vector<float>&& values) {
        x2_grid g{};
        g.channels = channels;
        g.lo[0] = g.lo[1] = g.lo[2] = 0;
        g.dims[0] = g.dims[1] = g.dims[2] = n;
        for (int i = 0; i < 16; ++i) g.world_to_index[i] = 0.0;
        for (int a = 0; a < 3; ++a) {
            g.world_to_index[a * 4 + a] = 1.0 / double(voxel);
            g.world_to_index[12 + a] = -double(lo) / double(voxel) - 0.5;
        }
        g.world_to_index[15] = 1.0;
        h->grids.push_back(g);
        h->gridValues.push_back(std::move(values));
        return uint32_t(h->grids.size() - 1);
    };
    x2_volume v{};
    for (int a = 0; a < 3; ++a) {
        v.bound_lo[a] = lo;
        v.bound_hi[a] = lo + extent;
    }
    v.density_grid = grid(1, std::move(density));
    v.emission_grid = grid(3, std::move(emission));
    v.interpolation = 1;
    v.feature_size = voxel;
    for (int i = 0; i < 12; ++i) v.world_to_grid[i] = 0.0f;
    v.world_to_grid[0] = v.world_to_grid[5] = v.world_to_grid[10] = 1.0f;
    for (int a = 0; a < 3; ++a) {
        v.gain[a] = 1.0f;
        v.color_mult[a] = 0.9f;
        v.incandescence[a] = 1.0f;
    }
    v.g = 0.6f;
    v.light_set = ~0u;
    v.surface_opacity_threshold = 0.5f;
    h->volumes.push_back(v);
    h->lights.push_back(distantLight({0.25f, -0.45f, -1.0f}, 5.0f));
    const x2_camera cam = pinhole({0, 0, 3.5f}, {0, 0, 0}, 40.0f, width, height);
    fillConfig(cfg, width, height, spp, depth, uint32_t(h->lights.size()), uint32_t(h->lights.size()));
    cfg->volume_count = 1;
    h->finish();
    h->desc.camera = cam;
    return h;
}

// The differentiable scene (config 4): config 1's construction reduced to about 250k triangles (18x18 heightfield
// tiles of 16x16 quads, 64 level-3 icospheres), the heightfield's meshes sharing one Lambert material whose diffuse
// colour is a texture (an fp32 RGB texture of `texels` x `texels` from seeded 4-octave colour fBm in [0.05, 0.9],
// periodic, over the heightfield's uvs: vertex (i, j) of its (n+1)^2 grid at (i/n, j/n)), the icospheres each one
// of a pool of `spheres` materials (sphere k takes material k). 512x512. (Config 44, the tests' shrunk copy, makes its
// icospheres three times larger so that their materials cover enough pixels for finite differences.)
Holder* makeAdjointField(uint64_t seed, int tiles, int spheres, int icoLevel, uint32_t texels, uint32_t width, uint32_t height, uint32_t spp,
                         uint32_t depth, x2_config* cfg, float radiusScale = 1.0f) {
    Holder* h = makeField(seed, tiles, spheres, icoLevel, width, height, spp, depth, cfg, radiusScale);
    const uint32_t tileMeshes = uint32_t(tiles * tiles);
    // The icospheres' own materials (each made after its heightfield tiles' by makeField) become the pool.
    std::vector<x2_material> pool(h->materials.begin() + tileMeshes, h->materials.end());
    x2_material textured = lambert(1.0f, 1.0f, 1.0f);
    textured.diffuse_texture = 1;
    pool.push_back(textured);
    h->materials = pool;
    for (size_t m = 0; m < h->meshMaterial.size(); ++m)
        h->meshMaterial[m] = m < tileMeshes ? uint32_t(pool.size() - 1) : uint32_t(m - tileMeshes);
    const int n = tiles * 16;
    h->uvs.assign(h->vertices.size() / 3 * 2, 0.0f);
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
            const size_t v = size_t(j) * (n + 1) + i;
            h->uvs[2 * v] = float(i) / float(n);
            h->uvs[2 * v + 1] = float(j) / float(n);
        }
    x2_texture t{};
    t.width = t.height = texels;
    t.wrap = 1;
    std::vector<float> rgb(size_t(texels) * texels * 3);
    for (uint32_t y = 0; y < texels; ++y)
        for (uint32_t x = 0; x < texels; ++x)
            for (int c = 0; c < 3; ++c) {
                const float u = 8.0f * float(x) / float(texels), v = 8.0f * float(y) / float(texels);
                const float f = fbm(u, v, 4, uint32_t(seed) + 31u * uint32_t(c + 1));
                rgb[(size_t(y) * texels + x) * 3 + c] = std::min(0.9f, std::max(0.05f, 0.475f + 0.6f * f));
            }
    h->textures.push_back(t);
    h->textureValues.push_back(std::move(rgb));
    const x2_camera cam = h->desc.camera;
    h->finish();
    h->desc.camera = cam;
    return h;
}

// Batched requests (one frame a request, each its own scene and frame seed): request r draws a triangle count
// log-uniform in [0.1M, 2M] (half heightfield tiles of 16x16 quads, half level-4 icospheres), a square resolution among
// 128, 256, 512 and 1024, log-uniform 4..256 spp and a uniform 4..32 depth; its frame seed is 1 + r. `shrink` > 1
// divides the triangle count by shrink^2 and the resolution and spp by shrink (the parity tests' small copies).
Holder* makeRequest(uint32_t r, uint64_t seed, uint32_t shrink, x2_config* cfg) {
    Rng g(seed ^ (0x51ed270b27a4f1c3ull * (uint64_t(r) + 1)));
    const double tris = std::exp(std::log(1e5) + g.uniform() * (std::log(2e6) - std::log(1e5))) / (double(shrink) * shrink);
    const uint32_t res = 128u << uint32_t(g.next() % 4);
    const double sppReal = std::exp(std::log(4.0) + g.uniform() * (std::log(256.0) - std::log(4.0)));
    const uint32_t depth = 4u + uint32_t(g.next() % 29u);
    const int tiles = std::max(1, int(std::lround(std::sqrt(tris / 2.0 / 512.0))));
    const int spheres = std::max(1, int(std::lround(tris / 2.0 / 5120.0)));
    const uint32_t side = std::max(8u, res / shrink);
    const uint32_t spp = std::max(1u, uint32_t(std::lround(sppReal / double(shrink))));
    Holder* h = makeField(seed + r, tiles, spheres, 4, side, side, spp, depth, cfg);
    cfg->seed = 1u + r;
    return h;
}

}  // namespace

extern "C" void x2_config_defaults(x2_config* c) {
    std::memset(c, 0, sizeof(*c));
    // mixed::Config defaults (gpu_jobs.h:11-44), with the path tracer switched on as mixed::config does for a
    // path-traced plan (cpu_jobs.h:13-27): sampling policy 3 | 4 | 8, every lobe ray type reused as a shadow ray.
    c->width = c->height = 1;
    c->spp = 1;
    c->sampling = 15;
    c->filter = X2_FILTER_BOX;
    c->filter_width = 1.0f;
    c->bsdf_samples = 1;
    c->light_samples = 1;
    c->clamp_depth = 1;
    c->transparency_threshold = 1.0f;
    c->presence_threshold = 0.999f;
    c->presence_quality = 0.75f;
    c->shadow_reuse = 0xfcu;
    c->max_volume_depth = 1;
    c->volume_illumination_samples = 4;
    c->volume_overlap_mode = 0;
    c->volume_transmittance_threshold = 0.005f;
    c->volume_attenuation_factor = 0.65f;
    c->volume_contribution_factor = 0.65f;
    c->volume_phase_attenuation_factor = 0.5f;
    c->inv_volume_quality = 2.0f;
    c->inv_volume_shadow_quality = 1.0f;
}

extern "C" int x2_scene_generate(uint32_t config_id, uint64_t seed, x2_scene_desc** out, x2_config* config) {
    if (!out || !config) return X2_EINVAL;
    Holder* h = nullptr;
    try {
        if (config_id == 0) {
            h = makeBox(config);
        } else if (config_id == 1) {
            h = makeField(seed, 64, 2000, 4, 1920, 1080, 64, 12, config);
        } else if (config_id == 11) {
            h = makeField(seed, 32, 2000, 2, 1920, 1080, 64, 12, config);
        } else if (config_id == 4) {
            h = makeAdjointField(seed, 18, 64, 3, 1024, 512, 512, 32, 12, config);
        } else if (config_id == 44) {
            h = makeAdjointField(seed, 4, 32, 2, 64, 64, 64, 4, 6, config, 3.0f);
        } else if (config_id == 3) {
            h = makeVolumeBox(seed, 256, 512, 512, 256, 64, config);
        } else if (config_id == 33) {
            h = makeVolumeBox(seed, 32, 64, 64, 4, 8, config);
        } else if (config_id >= 200 && config_id < 248) {
            h = makeRequest(config_id - 200, seed, 1, config);
        } else if (config_id >= 300 && config_id < 348) {
            h = makeRequest(config_id - 300, seed, 8, config);
        } else if (config_id > 100 && config_id <= 164) {
            const int k = int(config_id - 100);
            const int tiles = 64 / k > 0 ? 64 / k : 1, spheres = 2000 / (k * k) > 0 ? 2000 / (k * k) : 1;
            const uint32_t w = 1920u / uint32_t(k) > 8 ? 1920u / uint32_t(k) : 8u, hh = 1080u / uint32_t(k) > 8 ? 1080u / uint32_t(k) : 8u;
            h = makeField(seed, tiles, spheres, 4, w, hh, 64, 12, config);
        } else {
            return X2_EINVAL;
        }
    } catch (const std::bad_alloc&) {
        delete h;
        return X2_ENOMEM;
    }
    *out = &h->desc;
    return X2_OK;
}

extern "C" void x2_scene_desc_free(x2_scene_desc* desc) {
    if (!desc) return;
    delete reinterpret_cast<Holder*>(desc);  // the descriptor is the holder's first member
}
