// A dense-grid stand-in for the small part of NanoVDB's API the reference's volume sampler reads
// (volume_grid.h): Coord, Vec3f, FloatGrid / Vec3fGrid with getAccessor().getValue(Coord).
// Test infrastructure for the oracle build only; NanoVDB itself is not part of this repository.
#pragma once
namespace nanovdb {
struct Coord {
    int x, y, z;
    Coord(int i, int j, int k) : x(i), y(j), z(k) {}
};
struct Vec3f {
    float v[3];
    float operator[](int i) const { return v[i]; }
};
// A dense grid: dims voxels from index `lo`, x fastest; the background outside.
template <class T>
struct DenseGrid {
    const T* values;
    int lo[3], dims[3];
    T background;
    struct Accessor {
        const DenseGrid* g;
        T getValue(const Coord& c) const {
            const int i = c.x - g->lo[0], j = c.y - g->lo[1], k = c.z - g->lo[2];
            if (i < 0 || j < 0 || k < 0 || i >= g->dims[0] || j >= g->dims[1] || k >= g->dims[2]) return g->background;
            return g->values[(long(k) * g->dims[1] + j) * long(g->dims[0]) + i];
        }
    };
    Accessor getAccessor() const { return Accessor{this}; }
};
using FloatGrid = DenseGrid<float>;
using Vec3fGrid = DenseGrid<Vec3f>;
}  // namespace nanovdb
