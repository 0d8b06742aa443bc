// Marching tetrahedra on the device (src/surface.cpp:66-200 of chem-kumo):
// the crossed edges (one per surface vertex) and the polygons of the
// isosurface f = iso of samples on a grid, numbered exactly as the
// reference's sequential sweep over the cells (k fastest) numbers them.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

namespace kumo_dev {

struct IsoGrid {
    double origin[3];
    double steps[9];  // steps[3a + r]: component r of the step vector of axis a
    int n[3];         // points per axis
};

/// A crossed tetrahedron edge: the linear indices of its inside (f >= iso)
/// and outside end points, their samples, and the grid indices of its lower
/// end (the corner with the smaller cell mask).
struct IsoEdge {
    long long inside, outside;
    double f_inside, f_outside;
    int cell[3];
    int pad;
};

/// A triangle or quadrilateral of vertex (edge) ids, oriented with its normal
/// from the inside corners to the outside ones.
struct IsoPolygon {
    long long vertex[4];
    int count;
    int pad;
};

/// Whether any sample on the grid's boundary faces is >= iso (the
/// reference's isosurface_reaches_boundary), from device samples.
bool iso_reaches_boundary(const IsoGrid& g, const double* samples, double iso, cudaStream_t stream);

/// Polygonization of device samples (n[a] >= 2): edges in vertex order and
/// polygons in the reference's order, copied to the host.
void iso_polygonize(const IsoGrid& g, const double* samples, double iso, std::vector<IsoEdge>& edges,
                    std::vector<IsoPolygon>& polygons, cudaStream_t stream);

}  // namespace kumo_dev
