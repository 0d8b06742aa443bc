// Marching tetrahedra on the device with the vertex and polygon numbering of
// chem-kumo's sequential sweep (src/surface.cpp:150-200).
//
// The reference walks the cells in order (k fastest) and, in each cell, the
// six tetrahedra around the main diagonal and the corners of each polygon;
// a vertex is numbered when its edge is met for the first time.  An edge that
// the isosurface crosses is met by every cell that contains it (each of its
// tetrahedra is crossed, and the polygon of a crossed tetrahedron has a
// corner on each of its crossed edges), so it is first met in the containing
// cell of smallest index, its owner, and there at the position of its first
// occurrence in that cell's sequence.  One kernel counts, per cell, its
// polygons and the edges it owns; exclusive scans give each cell its first
// vertex and polygon number; a second kernel writes the edges a cell owns
// and its polygons, finding the number of an edge owned by an earlier cell by
// replaying that cell's sequence.
#include <cub/cub.cuh>

#include <stdexcept>
#include <string>

#include "func_attr.cuh"
#include "isosurface.cuh"

namespace kumo_dev {
namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Corner masks of the six tetrahedra (corners 0, e_a, e_a + e_b, (1,1,1)).
__constant__ unsigned char kTet[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                         {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
// For an edge direction d = high ^ low, the lower corner masks of the
// tetrahedron edges with that direction (the cells containing an edge sit at
// its lower end minus these offsets); count in kLowCount.
__constant__ unsigned char kLows[8][4] = {{0, 0, 0, 0}, {0, 2, 4, 6}, {0, 1, 4, 5}, {0, 4, 0, 0},
                                          {0, 1, 2, 3}, {0, 2, 0, 0}, {0, 1, 0, 0}, {0, 0, 0, 0}};
__constant__ unsigned char kLowCount[8] = {0, 4, 4, 2, 4, 2, 2, 1};

struct Cell {
    int i, j, k;
};

__device__ __forceinline__ long long point_index(const IsoGrid& g, int i, int j, int k) {
    return (static_cast<long long>(i) * g.n[1] + j) * g.n[2] + k;
}

__device__ __forceinline__ long long cell_index(const IsoGrid& g, int i, int j, int k) {
    return (static_cast<long long>(i) * (g.n[1] - 1) + j) * (g.n[2] - 1) + k;
}

__device__ __forceinline__ Cell cell_of(const IsoGrid& g, long long c) {
    const long long nz = g.n[2] - 1, ny = g.n[1] - 1;
    return {static_cast<int>(c / (ny * nz)), static_cast<int>((c / nz) % ny), static_cast<int>(c % nz)};
}

__device__ __forceinline__ void position(const IsoGrid& g, int i, int j, int k, double p[3]) {
    for (int r = 0; r < 3; ++r)
        p[r] = g.origin[r] + ((g.steps[r] * i + g.steps[3 + r] * j) + g.steps[6 + r] * k);
}

// The polygon corners of one cell in the reference's order: for corner q,
// the masks of its inside end a[q] and outside end b[q]; polygons of
// count[p] corners.
struct Sequence {
    int npoly = 0, ncorner = 0;
    unsigned char count[6];
    unsigned char a[24], b[24];
    long long corner[8];
};

__device__ bool cell_sequence(const IsoGrid& g, const double* f, double iso, Cell c, Sequence& s) {
    bool inside[8];
    int nin_total = 0;
    for (int m = 0; m < 8; ++m) {
        s.corner[m] = point_index(g, c.i + (m & 1), c.j + ((m >> 1) & 1), c.k + (m >> 2));
        inside[m] = f[s.corner[m]] >= iso;
        nin_total += inside[m];
    }
    if (nin_total == 0 || nin_total == 8) return false;
    double pos[8][3];
    for (int m = 0; m < 8; ++m) position(g, c.i + (m & 1), c.j + ((m >> 1) & 1), c.k + (m >> 2), pos[m]);
    s.npoly = s.ncorner = 0;
    for (int t = 0; t < 6; ++t) {
        unsigned char in[4], out[4];
        int nin = 0, nout = 0;
        for (int v = 0; v < 4; ++v) {
            const unsigned char m = kTet[t][v];
            if (inside[m])
                in[nin++] = m;
            else
                out[nout++] = m;
        }
        if (nin == 0 || nout == 0) continue;
        unsigned char ea[4], eb[4];
        int cnt;
        if (nin == 1) {
            ea[0] = ea[1] = ea[2] = in[0];
            eb[0] = out[0], eb[1] = out[1], eb[2] = out[2];
            cnt = 3;
        } else if (nout == 1) {
            ea[0] = in[0], ea[1] = in[1], ea[2] = in[2];
            eb[0] = eb[1] = eb[2] = out[0];
            cnt = 3;
        } else {
            ea[0] = in[0], eb[0] = out[0];
            ea[1] = in[0], eb[1] = out[1];
            ea[2] = in[1], eb[2] = out[1];
            ea[3] = in[1], eb[3] = out[0];
            cnt = 4;
        }
        // Orientation from the edge midpoints (they depend on the cell only):
        // the normal must point from the inside corners to the outside ones.
        double mid[4][3];
        for (int q = 0; q < cnt; ++q)
            for (int r = 0; r < 3; ++r) mid[q][r] = 0.5 * (pos[ea[q]][r] + pos[eb[q]][r]);
        double u[3], v[3];
        for (int r = 0; r < 3; ++r) {
            u[r] = cnt == 3 ? mid[1][r] - mid[0][r] : mid[2][r] - mid[0][r];
            v[r] = cnt == 3 ? mid[2][r] - mid[0][r] : mid[3][r] - mid[1][r];
        }
        const double nrm[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        double outward[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < nout; ++q)
            for (int r = 0; r < 3; ++r) outward[r] += pos[out[q]][r] / nout;
        for (int q = 0; q < nin; ++q)
            for (int r = 0; r < 3; ++r) outward[r] -= pos[in[q]][r] / nin;
        const bool reverse = nrm[0] * outward[0] + nrm[1] * outward[1] + nrm[2] * outward[2] < 0;
        for (int q = 0; q < cnt; ++q) {
            const int src = reverse ? cnt - 1 - q : q;
            s.a[s.ncorner + q] = ea[src];
            s.b[s.ncorner + q] = eb[src];
        }
        s.count[s.npoly++] = static_cast<unsigned char>(cnt);
        s.ncorner += cnt;
    }
    return true;
}

// Edge key: lower end point index * 8 + direction.
__device__ __forceinline__ long long edge_key(const Sequence& s, int q) {
    const unsigned char lo = s.a[q] < s.b[q] ? s.a[q] : s.b[q];
    const unsigned char hi = s.a[q] < s.b[q] ? s.b[q] : s.a[q];
    return s.corner[lo] * 8 + (hi ^ lo);
}

// Index of the cell that meets the edge (lower end of cell c's corner `lo`,
// direction d) first: the containing cell of smallest index.
__device__ long long edge_owner(const IsoGrid& g, Cell c, unsigned char lo, unsigned char d) {
    const int p[3] = {c.i + (lo & 1), c.j + ((lo >> 1) & 1), c.k + (lo >> 2)};
    long long best = -1;
    for (int t = 0; t < kLowCount[d]; ++t) {
        const unsigned char l = kLows[d][t];
        const int ci = p[0] - (l & 1), cj = p[1] - ((l >> 1) & 1), ck = p[2] - (l >> 2);
        if (ci < 0 || cj < 0 || ck < 0 || ci > g.n[0] - 2 || cj > g.n[1] - 2 || ck > g.n[2] - 2) continue;
        const long long idx = cell_index(g, ci, cj, ck);
        if (best < 0 || idx < best) best = idx;
    }
    return best;
}

__device__ __forceinline__ bool first_in_cell(const Sequence& s, int q, long long key) {
    for (int r = 0; r < q; ++r)
        if (edge_key(s, r) == key) return false;
    return true;
}

// Whether corner q of cell c's sequence is the first meeting of its edge in
// the whole sweep.
__device__ __forceinline__ bool owns(const IsoGrid& g, Cell c, long long ci, const Sequence& s, int q) {
    const long long key = edge_key(s, q);
    if (!first_in_cell(s, q, key)) return false;
    const unsigned char lo = s.a[q] < s.b[q] ? s.a[q] : s.b[q];
    const unsigned char hi = s.a[q] < s.b[q] ? s.b[q] : s.a[q];
    return edge_owner(g, c, lo, hi ^ lo) == ci;
}

__global__ void count_kernel(IsoGrid g, const double* f, double iso, long long ncells, int* vcount, int* pcount) {
    const long long ci = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ci >= ncells) return;
    const Cell c = cell_of(g, ci);
    Sequence s;
    int nv = 0, np = 0;
    if (cell_sequence(g, f, iso, c, s)) {
        np = s.npoly;
        for (int q = 0; q < s.ncorner; ++q) nv += owns(g, c, ci, s, q);
    }
    vcount[ci] = nv;
    pcount[ci] = np;
}

__global__ void emit_kernel(IsoGrid g, const double* f, double iso, long long ncells, const int* vbase,
                            const int* pbase, IsoEdge* edges, IsoPolygon* polys) {
    const long long ci = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ci >= ncells) return;
    const Cell c = cell_of(g, ci);
    Sequence s;
    if (!cell_sequence(g, f, iso, c, s)) return;
    long long ids[24];
    int next = vbase[ci];
    for (int q = 0; q < s.ncorner; ++q) {
        const long long key = edge_key(s, q);
        long long id = -1;
        for (int r = 0; r < q && id < 0; ++r)
            if (edge_key(s, r) == key) id = ids[r];
        if (id < 0) {
            const unsigned char lo = s.a[q] < s.b[q] ? s.a[q] : s.b[q];
            const unsigned char hi = s.a[q] < s.b[q] ? s.b[q] : s.a[q];
            const long long owner = edge_owner(g, c, lo, hi ^ lo);
            if (owner == ci) {
                id = next++;
                IsoEdge e;
                e.inside = s.corner[s.a[q]];
                e.outside = s.corner[s.b[q]];
                e.f_inside = f[e.inside];
                e.f_outside = f[e.outside];
                e.cell[0] = c.i + (lo & 1);
                e.cell[1] = c.j + ((lo >> 1) & 1);
                e.cell[2] = c.k + (lo >> 2);
                e.pad = 0;
                edges[id] = e;
            } else {
                // Replay the owner's sequence to find the edge's number there.
                const Cell oc = cell_of(g, owner);
                Sequence os;
                cell_sequence(g, f, iso, oc, os);
                int n = vbase[owner];
                for (int r = 0; r < os.ncorner; ++r) {
                    if (!owns(g, oc, owner, os, r)) continue;
                    if (edge_key(os, r) == key) {
                        id = n;
                        break;
                    }
                    ++n;
                }
            }
        }
        ids[q] = id;
    }
    int q = 0;
    for (int p = 0; p < s.npoly; ++p) {
        IsoPolygon poly;
        poly.count = s.count[p];
        poly.pad = 0;
        for (int v = 0; v < 4; ++v) poly.vertex[v] = v < poly.count ? ids[q + v] : -1;
        q += poly.count;
        polys[pbase[ci] + p] = poly;
    }
}

__global__ void boundary_kernel(IsoGrid g, const double* f, double iso, long long npoints, int* hit) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= npoints) return;
    const long long i = q / (static_cast<long long>(g.n[1]) * g.n[2]);
    const long long j = (q / g.n[2]) % g.n[1];
    const long long k = q % g.n[2];
    const bool face = i == 0 || i == g.n[0] - 1 || j == 0 || j == g.n[1] - 1 || k == 0 || k == g.n[2] - 1;
    if (face && f[q] >= iso) atomicOr(hit, 1);
}

}  // namespace

bool iso_reaches_boundary(const IsoGrid& g, const double* samples, double iso, cudaStream_t stream) {
    const long long n = static_cast<long long>(g.n[0]) * g.n[1] * g.n[2];
    int* hit = nullptr;
    check(cudaMallocAsync(reinterpret_cast<void**>(&hit), sizeof(int), stream), "cudaMallocAsync (isosurface)");
    check(cudaMemsetAsync(hit, 0, sizeof(int), stream), "cudaMemsetAsync (isosurface)");
    KUMO_REGISTER_KERNEL(boundary_kernel);
    boundary_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(g, samples, iso, n, hit);
    int h = 0;
    check(cudaMemcpyAsync(&h, hit, sizeof(int), cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync (isosurface)");
    check(cudaFreeAsync(hit, stream), "cudaFreeAsync (isosurface)");
    check(cudaStreamSynchronize(stream), "isosurface boundary check");
    return h != 0;
}

void iso_polygonize(const IsoGrid& g, const double* samples, double iso, std::vector<IsoEdge>& edges,
                    std::vector<IsoPolygon>& polygons, cudaStream_t stream) {
    edges.clear();
    polygons.clear();
    const long long ncells = static_cast<long long>(g.n[0] - 1) * (g.n[1] - 1) * (g.n[2] - 1);
    if (ncells <= 0) return;
    if (ncells > 0x7fffffffll) throw std::invalid_argument("isosurface grid has too many cells");
    const int n = static_cast<int>(ncells);
    int *counts = nullptr, *bases = nullptr;
    check(cudaMallocAsync(reinterpret_cast<void**>(&counts), sizeof(int) * 2 * static_cast<size_t>(n), stream),
          "cudaMallocAsync (isosurface counts)");
    check(cudaMallocAsync(reinterpret_cast<void**>(&bases), sizeof(int) * 2 * static_cast<size_t>(n), stream),
          "cudaMallocAsync (isosurface bases)");
    int* vcount = counts;
    int* pcount = counts + n;
    int* vbase = bases;
    int* pbase = bases + n;
    const unsigned blocks = static_cast<unsigned>((ncells + 127) / 128);
    KUMO_REGISTER_KERNEL(count_kernel);
    KUMO_REGISTER_KERNEL(emit_kernel);
    count_kernel<<<blocks, 128, 0, stream>>>(g, samples, iso, ncells, vcount, pcount);
    check(cudaGetLastError(), "isosurface count kernel");
    size_t tmp_bytes = 0;
    check(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, vcount, vbase, n, stream), "cub scan (size)");
    void* tmp = nullptr;
    check(cudaMallocAsync(&tmp, tmp_bytes, stream), "cudaMallocAsync (scan)");
    check(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, vcount, vbase, n, stream), "cub scan (vertices)");
    check(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, pcount, pbase, n, stream), "cub scan (polygons)");
    int tail[4];
    check(cudaMemcpyAsync(&tail[0], vbase + n - 1, sizeof(int), cudaMemcpyDeviceToHost, stream), "isosurface totals");
    check(cudaMemcpyAsync(&tail[1], vcount + n - 1, sizeof(int), cudaMemcpyDeviceToHost, stream), "isosurface totals");
    check(cudaMemcpyAsync(&tail[2], pbase + n - 1, sizeof(int), cudaMemcpyDeviceToHost, stream), "isosurface totals");
    check(cudaMemcpyAsync(&tail[3], pcount + n - 1, sizeof(int), cudaMemcpyDeviceToHost, stream), "isosurface totals");
    check(cudaStreamSynchronize(stream), "isosurface scan");
    const long long nv = static_cast<long long>(tail[0]) + tail[1];
    const long long np = static_cast<long long>(tail[2]) + tail[3];
    IsoEdge* d_edges = nullptr;
    IsoPolygon* d_polys = nullptr;
    if (nv > 0)
        check(cudaMallocAsync(reinterpret_cast<void**>(&d_edges), sizeof(IsoEdge) * static_cast<size_t>(nv), stream),
              "cudaMallocAsync (isosurface edges)");
    if (np > 0)
        check(cudaMallocAsync(reinterpret_cast<void**>(&d_polys), sizeof(IsoPolygon) * static_cast<size_t>(np), stream),
              "cudaMallocAsync (isosurface polygons)");
    if (nv > 0 || np > 0) {
        emit_kernel<<<blocks, 128, 0, stream>>>(g, samples, iso, ncells, vbase, pbase, d_edges, d_polys);
        check(cudaGetLastError(), "isosurface emit kernel");
    }
    edges.resize(static_cast<size_t>(nv));
    polygons.resize(static_cast<size_t>(np));
    if (nv > 0)
        check(cudaMemcpyAsync(edges.data(), d_edges, sizeof(IsoEdge) * static_cast<size_t>(nv), cudaMemcpyDeviceToHost,
                              stream),
              "isosurface edges");
    if (np > 0)
        check(cudaMemcpyAsync(polygons.data(), d_polys, sizeof(IsoPolygon) * static_cast<size_t>(np),
                              cudaMemcpyDeviceToHost, stream),
              "isosurface polygons");
    cudaFreeAsync(tmp, stream);
    cudaFreeAsync(counts, stream);
    cudaFreeAsync(bases, stream);
    if (d_edges) cudaFreeAsync(d_edges, stream);
    if (d_polys) cudaFreeAsync(d_polys, stream);
    check(cudaStreamSynchronize(stream), "isosurface polygonization");
}

}  // namespace kumo_dev
