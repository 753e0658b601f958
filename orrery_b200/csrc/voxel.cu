// Mesh voxelization on the device: the solid flags of a grid from the
// generalized winding number of a triangle mesh, and the narrow-band signed
// distance to it (geom::voxelize and geom::signed_distance_band,
// src/geom/voxel_grid.cpp:84-140, evaluated with the bounding-volume tree of
// src/geom/winding_number.cpp:164-309).  The adapter builds the mask and wall
// distances of every lattice this way (lbm_aero_solver3d.cpp:249-258); on the
// host it is the largest part of setting up a lattice.
//
// Layout: the tree is built on the host (it is small: about n / 4 nodes for n
// triangles) and copied with the triangles' corners in tree order, 9 doubles
// per triangle, so a leaf's triangles are one contiguous run.  One thread per
// grid cell.  For the winding number the 32 cells of a warp (a 4 x 4 x 2
// brick) walk the tree together on one stack in shared memory; for the
// distance each thread walks on its own with a stack of at most 64 entries in
// local memory (its nearest-first order is its own).
//
// Results: the tree has the reference's node ranges, triangle order and node
// quantities (same median split with the same tie-break, same sums in the same
// order; the host uses the same standard-library routines), and the device
// repeats the reference's traversal order.  This translation unit is built
// without FMA contraction, and the distance to a triangle (products, sums,
// correctly rounded division and sqrt) is the reference's bit for bit, so the
// band distances are.  The winding sum differs from the reference's only
// through atan2, whose CUDA and C library results may differ in the last
// bits: a few 1e-16 per triangle term.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numbers>
#include <numeric>
#include <string>
#include <vector>

#include "common.h"
#include "host_copy.h"
#include "orrery_lbm.h"

namespace orr::geo {

// Largest grid accepted, as the reference's geom::max_grid_cells (2^27).
constexpr uint64_t kMaxGridCells = uint64_t{1} << 27;
// Far-field ratio and leaf size of the reference's MeshTree defaults.
constexpr double kBeta = 2.0;
constexpr uint32_t kLeafSize = 8;
// Traversal stack entries per thread; a walk holds at most depth + 1.
constexpr int kStack = 64;

struct V3 {
    double x, y, z;
};
__host__ __device__ inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Length of (x, y, z) as the C++ standard library's three-argument hypot of
// this toolchain evaluates it (the reference's norm): the largest magnitude
// m times sqrt of the sum of the squared ratios, added left to right.
__host__ __device__ inline double length3(V3 v) {
    const double x = fabs(v.x), y = fabs(v.y), z = fabs(v.z);
    const double m = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (m == 0.0) {
        return 0.0;
    }
    const double qx = x / m, qy = y / m, qz = z / m;
    return m * sqrt(qx * qx + qy * qy + qz * qz);
}

// Tree node (128 bytes): bounds, area-weighted centre, area vector over
// scale^2, radius about the centre, triangle range (tree order) or children.
struct Node {
    double lo[3], hi[3];
    double centre[3];
    double area[3];
    double radius;
    uint32_t first, count, left, right;
    uint32_t leaf, unused;
};
static_assert(sizeof(Node) == 128, "node layout");

struct Tree {
    std::vector<Node> nodes;
    std::vector<double> corners;  // 9 per triangle, tree order
    double scale = 1.0;
    uint32_t depth = 0;
};

// ------------------------------------------------------------------ host --

// The tree of a mesh (src/geom/winding_number.cpp:164-240 gives the rules:
// node bounds and area sums over the range, median split of the centroids
// along their longest axis with ties broken by triangle index).  Nodes are
// made breadth first; every range is permuted only by its own split, which
// leaves the same order in each range as a depth-first build.
Tree build_tree(const double* vertices, uint64_t nv, const uint32_t* triangles, uint32_t nt) {
    Tree tree;
    auto vertex = [&](uint32_t i) { return V3{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]}; };
    auto corner = [&](uint32_t t, int k) { return vertex(triangles[3 * t + k]); };
    auto centroid = [&](uint32_t t) { return (corner(t, 0) + corner(t, 1) + corner(t, 2)) / 3.0; };
    // Power of two near the largest extent of the vertices' bounds.
    if (nv > 0) {
        V3 lo = vertex(0), hi = vertex(0);
        for (uint64_t i = 0; i < nv; ++i) {
            const V3 v = vertex(static_cast<uint32_t>(i));
            lo = {std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z)};
            hi = {std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z)};
        }
        const double extent = std::max({hi.x - lo.x, hi.y - lo.y, hi.z - lo.z});
        if (extent > 0.0 && std::isfinite(extent)) {
            tree.scale = std::ldexp(1.0, std::ilogb(extent));
        }
    }
    if (nt == 0) {
        return tree;
    }
    std::vector<uint32_t> order(nt);
    std::iota(order.begin(), order.end(), 0u);
    std::vector<uint32_t> level_of;
    tree.nodes.reserve(2 * (nt / kLeafSize + 1));
    auto make = [&](uint32_t first, uint32_t count, uint32_t level) {
        Node n{};
        n.first = first;
        n.count = count;
        const V3 v0 = corner(order[first], 0);
        V3 lo = v0, hi = v0;
        V3 clo = centroid(order[first]), chi = clo;
        V3 area_vec{0.0, 0.0, 0.0}, weighted{0.0, 0.0, 0.0};
        double area = 0.0;
        for (uint32_t i = first; i < first + count; ++i) {
            const uint32_t t = order[i];
            for (int k = 0; k < 3; ++k) {
                const V3 v = corner(t, k);
                lo = {std::min(lo.x, v.x), std::min(lo.y, v.y), std::min(lo.z, v.z)};
                hi = {std::max(hi.x, v.x), std::max(hi.y, v.y), std::max(hi.z, v.z)};
            }
            const V3 c = centroid(t);
            clo = {std::min(clo.x, c.x), std::min(clo.y, c.y), std::min(clo.z, c.z)};
            chi = {std::max(chi.x, c.x), std::max(chi.y, c.y), std::max(chi.z, c.z)};
            const V3 a = corner(t, 0);
            const V3 n2 = cross((corner(t, 1) - a) / tree.scale, (corner(t, 2) - a) / tree.scale);
            const double half_area = 0.5 * std::hypot(n2.x, n2.y, n2.z);
            area_vec = area_vec + n2 * 0.5;
            weighted = weighted + c * half_area;
            area += half_area;
        }
        const V3 centre = area > 0.0 ? weighted / area : (lo + hi) * 0.5;
        const double b[3][3] = {{lo.x, lo.y, lo.z}, {hi.x, hi.y, hi.z}, {centre.x, centre.y, centre.z}};
        std::memcpy(n.lo, b[0], sizeof n.lo);
        std::memcpy(n.hi, b[1], sizeof n.hi);
        std::memcpy(n.centre, b[2], sizeof n.centre);
        n.area[0] = area_vec.x;
        n.area[1] = area_vec.y;
        n.area[2] = area_vec.z;
        n.leaf = count <= kLeafSize ? 1u : 0u;
        tree.nodes.push_back(n);
        level_of.push_back(level);
        tree.depth = std::max(tree.depth, level);
        // The split axis comes from the centroid bounds, kept for the queue.
        const V3 e = chi - clo;
        return e.x >= e.y && e.x >= e.z ? 0 : (e.y >= e.z ? 1 : 2);
    };
    std::vector<int> axis_of;
    axis_of.push_back(make(0, nt, 0));
    for (std::size_t k = 0; k < tree.nodes.size(); ++k) {
        if (tree.nodes[k].leaf) {
            continue;
        }
        const uint32_t first = tree.nodes[k].first, count = tree.nodes[k].count, half = count / 2;
        const int axis = axis_of[k];
        auto key = [&](uint32_t t) {
            const V3 c = centroid(t);
            return axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
        };
        std::nth_element(order.begin() + first, order.begin() + first + half, order.begin() + first + count,
                         [&](uint32_t a, uint32_t b) {
                             const double ka = key(a), kb = key(b);
                             return ka != kb ? ka < kb : a < b;
                         });
        const uint32_t level = level_of[k] + 1;
        tree.nodes[k].left = static_cast<uint32_t>(tree.nodes.size());
        axis_of.push_back(make(first, half, level));
        tree.nodes[k].right = static_cast<uint32_t>(tree.nodes.size());
        axis_of.push_back(make(first + half, count - half, level));
    }
    // Radii, children before parents (they come later in breadth-first order).
    for (std::size_t k = tree.nodes.size(); k-- > 0;) {
        Node& n = tree.nodes[k];
        const V3 c{n.centre[0], n.centre[1], n.centre[2]};
        double r = 0.0;
        if (n.leaf) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) {
                for (int j = 0; j < 3; ++j) {
                    const V3 d = corner(order[i], j) - c;
                    r = std::max(r, std::hypot(d.x, d.y, d.z));
                }
            }
        } else {
            for (const uint32_t child : {n.left, n.right}) {
                const Node& m = tree.nodes[child];
                const V3 d = V3{m.centre[0], m.centre[1], m.centre[2]} - c;
                r = std::max(r, std::hypot(d.x, d.y, d.z) + m.radius);
            }
        }
        n.radius = r;
    }
    tree.corners.resize(static_cast<std::size_t>(nt) * 9);
    for (uint32_t i = 0; i < nt; ++i) {
        for (int k = 0; k < 3; ++k) {
            const V3 v = corner(order[i], k);
            tree.corners[9 * static_cast<std::size_t>(i) + 3 * k] = v.x;
            tree.corners[9 * static_cast<std::size_t>(i) + 3 * k + 1] = v.y;
            tree.corners[9 * static_cast<std::size_t>(i) + 3 * k + 2] = v.z;
        }
    }
    return tree;
}

// ---------------------------------------------------------------- device --

struct Grid {
    double ox, oy, oz, h;
    uint32_t nx, ny, nz;
};

__device__ inline V3 cell_centre(const Grid& g, uint32_t c) {
    const uint32_t i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    return {g.ox + (static_cast<double>(i) + 0.5) * g.h, g.oy + (static_cast<double>(j) + 0.5) * g.h,
            g.oz + (static_cast<double>(k) + 0.5) * g.h};
}

__device__ inline V3 load3(const double* p) { return {__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }

// Signed solid angle of triangle (a, b, c) seen from p on unit vectors (Van
// Oosterom and Strackee; solid_angle, winding_number.cpp:101-122).
__device__ inline double solid_angle(V3 p, V3 a, V3 b, V3 c) {
    const V3 ra = a - p, rb = b - p, rc = c - p;
    const double la = length3(ra), lb = length3(rb), lc = length3(rc);
    if (!(la > 0.0) || !(lb > 0.0) || !(lc > 0.0)) {
        return 0.0;
    }
    const V3 ua = ra / la, ub = rb / lb, uc = rc / lc;
    const double num = dot(ua, cross(ub, uc));
    const double den = 1.0 + dot(ua, ub) + dot(ub, uc) + dot(uc, ua);
    return 2.0 * atan2(num, den);
}

// Closest point of segment a-b to p (a when it has no length).
__device__ inline V3 segment_point(V3 p, V3 a, V3 b) {
    const V3 ab = b - a;
    const double l2 = dot(ab, ab);
    if (!(l2 > 0.0)) {
        return a;
    }
    double t = dot(p - a, ab) / l2;
    t = t < 0.0 ? 0.0 : (1.0 < t ? 1.0 : t);
    return a + ab * t;
}

// A triangle without area: the closest of its edges' closest points.
__device__ inline V3 edges_point(V3 p, V3 a, V3 b, V3 c) {
    V3 best = segment_point(p, a, b);
    V3 d = best - p;
    double best2 = dot(d, d);
    const V3 q1 = segment_point(p, b, c), q2 = segment_point(p, c, a);
    d = q1 - p;
    const double d1 = dot(d, d);
    if (d1 < best2) {
        best = q1;
        best2 = d1;
    }
    d = q2 - p;
    if (dot(d, d) < best2) {
        best = q2;
    }
    return best;
}

// Closest point of triangle (a, b, c) to p by its Voronoi regions (Ericson,
// Real-Time Collision Detection 5.1.5; closest_point_on_triangle,
// winding_number.cpp:131-176, with the same degenerate fallbacks).
__device__ inline V3 triangle_point(V3 p, V3 a, V3 b, V3 c) {
    const V3 ab = b - a, ac = c - a;
    const V3 n = cross(ab, ac);
    if (!(dot(n, n) > 0.0)) {
        return edges_point(p, a, b, c);
    }
    const V3 ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) {
        return a;
    }
    const V3 bp = p - b;
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) {
        return b;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        return a + ab * (d1 / (d1 - d3));
    }
    const V3 cp = p - c;
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) {
        return c;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        return a + ac * (d2 / (d2 - d6));
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    }
    const double sum = va + vb + vc;
    if (!(sum > 0.0)) {
        return edges_point(p, a, b, c);
    }
    return a + ab * (vb / sum) + ac * (vc / sum);
}

// Largest of (below, 0, above), the first one on ties.
__device__ inline double gap(double below, double above) {
    double m = below;
    m = m < 0.0 ? 0.0 : m;
    return m < above ? above : m;
}

__device__ inline double box_distance2(const Node& n, V3 p) {
    const double dx = gap(n.lo[0] - p.x, p.x - n.hi[0]);
    const double dy = gap(n.lo[1] - p.y, p.y - n.hi[1]);
    const double dz = gap(n.lo[2] - p.z, p.z - n.hi[2]);
    return dx * dx + dy * dy + dz * dz;
}

// Cells of a warp: a brick of 4 x 4 x 2 neighbouring cells (lane l at
// (l % 4, l / 4 % 4, l / 16) of its brick), whose tree walks differ little.
constexpr uint32_t kBrickX = 4, kBrickY = 4, kBrickZ = 2;
constexpr int kWarpsPerBlock = 4;

struct Bricks {
    uint32_t bx, by, bz;
};

__host__ __device__ inline Bricks bricks_of(const Grid& g) {
    return {(g.nx + kBrickX - 1) / kBrickX, (g.ny + kBrickY - 1) / kBrickY, (g.nz + kBrickZ - 1) / kBrickZ};
}

// Generalized winding number of every cell centre (hierarchical evaluation
// of Barill et al. 2018; MeshTree::winding_number, winding_number.cpp:242-279):
// a node far enough away (distance above beta times its radius) counts as its
// dipole, a near leaf as the exact solid angles of its triangles.
//
// The 32 lanes of a warp walk the tree together: one stack per warp in
// shared memory holds (node, lanes that reach it).  Each lane of the popped
// entry either adds the node's dipole or opens it; the lanes that open a
// leaf add its solid angles together, those that open an inner node push its
// children (left, then right) with their mask.  The walk is the union of the
// lanes' own depth-first walks in the same order, so every lane adds the same
// terms in the same order as a walk of its own (the reference's order), with
// one instruction stream per warp instead of 32 diverging ones.
__global__ void __launch_bounds__(128) winding_kernel(Grid g, const Node* __restrict__ nodes,
                                                      const double* __restrict__ corners, uint32_t node_count,
                                                      double scale, double threshold, uint8_t* __restrict__ solid,
                                                      double* __restrict__ winding, uint32_t* __restrict__ overflow) {
    __shared__ uint2 stacks[kWarpsPerBlock][kStack];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint2* stack = stacks[warp];
    const Bricks nb = bricks_of(g);
    const uint64_t brick = static_cast<uint64_t>(blockIdx.x) * kWarpsPerBlock + warp;
    const uint32_t bi = static_cast<uint32_t>(brick % nb.bx), bj = static_cast<uint32_t>((brick / nb.bx) % nb.by);
    const uint64_t bk = brick / (static_cast<uint64_t>(nb.bx) * nb.by);
    const uint32_t i = bi * kBrickX + lane % kBrickX, j = bj * kBrickY + (lane / kBrickX) % kBrickY;
    const uint64_t k = bk * kBrickZ + lane / (kBrickX * kBrickY);
    const bool valid = i < g.nx && j < g.ny && k < g.nz;
    const uint32_t lanes = __ballot_sync(0xffffffffu, valid);
    if (lanes == 0u) {
        return;
    }
    const uint32_t c = valid ? i + g.nx * (j + g.ny * static_cast<uint32_t>(k)) : 0u;
    const V3 p = cell_centre(g, c);
    double sum = 0.0;
    int top = 0;
    if (node_count > 0) {
        if (lane == 0) {
            stack[0] = make_uint2(0u, lanes);
        }
        top = 1;
    }
    __syncwarp();
    while (top > 0) {
        --top;
        const uint2 e = stack[top];
        __syncwarp();
        const Node& n = nodes[e.x];
        bool open = false;
        if ((e.y >> lane) & 1u) {
            const V3 d = V3{__ldg(&n.centre[0]), __ldg(&n.centre[1]), __ldg(&n.centre[2])} - p;
            const double dist = length3(d);
            if (dist > kBeta * __ldg(&n.radius)) {
                const double flux = dot(V3{__ldg(&n.area[0]), __ldg(&n.area[1]), __ldg(&n.area[2])}, d / dist);
                if (flux != 0.0) {
                    const double ratio = scale / dist;
                    sum += flux * ratio * ratio;
                }
            } else {
                open = true;
            }
        }
        const uint32_t opened = __ballot_sync(0xffffffffu, open);
        if (opened == 0u) {
            continue;
        }
        if (__ldg(&n.leaf)) {
            if (open) {
                const uint32_t first = __ldg(&n.first), count = __ldg(&n.count);
                for (uint32_t t = first; t < first + count; ++t) {
                    const double* tri = corners + 9 * static_cast<size_t>(t);
                    sum += solid_angle(p, load3(tri), load3(tri + 3), load3(tri + 6));
                }
            }
            continue;
        }
        if (top + 2 > kStack) {
            if (lane == 0) {
                atomicOr(overflow, 1u);
            }
            break;
        }
        if (lane == 0) {
            stack[top] = make_uint2(__ldg(&n.left), opened);
            stack[top + 1] = make_uint2(__ldg(&n.right), opened);
        }
        top += 2;
        __syncwarp();
    }
    if (valid) {
        const double w = sum / (4.0 * std::numbers::pi);
        if (winding != nullptr) {
            winding[c] = w;
        }
        solid[c] = static_cast<uint8_t>(w >= threshold);
    }
}

// Distance from every cell centre to the surface, up to `band`, signed by the
// cell's solid flag (MeshTree::distance, winding_number.cpp:281-307, and
// signed_distance_band, voxel_grid.cpp:110-138): subtrees whose box is no
// closer than the best distance so far are skipped, the nearer child first.
__global__ void __launch_bounds__(128) distance_kernel(Grid g, const Node* __restrict__ nodes,
                                                       const double* __restrict__ corners, uint32_t node_count,
                                                       double band, const uint8_t* __restrict__ solid,
                                                       double* __restrict__ distance, uint8_t* __restrict__ in_band,
                                                       uint32_t* __restrict__ overflow) {
    const uint32_t cells = g.nx * g.ny * g.nz;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) {
        return;
    }
    const V3 p = cell_centre(g, c);
    double best2 = band * band;
    uint32_t stack[kStack];
    int top = 0;
    if (node_count > 0) {
        stack[top++] = 0;
    }
    while (top > 0) {
        const Node& n = nodes[stack[--top]];
        if (box_distance2(n, p) >= best2) {
            continue;
        }
        if (n.leaf) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i) {
                const double* t = corners + 9 * static_cast<size_t>(i);
                const V3 q = triangle_point(p, load3(t), load3(t + 3), load3(t + 6)) - p;
                const double d2 = dot(q, q);
                best2 = d2 < best2 ? d2 : best2;
            }
            continue;
        }
        if (top + 2 > kStack) {
            atomicOr(overflow, 1u);
            break;
        }
        const double dl = box_distance2(nodes[n.left], p), dr = box_distance2(nodes[n.right], p);
        const bool left_first = dl <= dr;
        stack[top++] = left_first ? n.right : n.left;
        stack[top++] = left_first ? n.left : n.right;
    }
    const double d = node_count > 0 ? sqrt(best2) : band;
    in_band[c] = static_cast<uint8_t>(d < band);
    distance[c] = (solid[c] != 0 ? -1.0 : 1.0) * d;
}

// --------------------------------------------------------------- host API --

// A grid is usable when its cell count is in range, its origin finite and
// its spacing positive and finite, and so is its last cell centre
// (check_spec, voxel_grid.cpp:22-47; the texts are the reference's).
void check_grid(const orr_grid_spec& s, const char* who) {
    const bool count_ok = s.nx > 0 && s.ny > 0 && s.nz > 0 && s.nx <= kMaxGridCells / s.ny &&
                          s.nx * s.ny <= kMaxGridCells / s.nz;
    if (!count_ok) {
        throw Refusal{ORR_ERR_INVALID, std::string(who) + ": grid empty or too large"};
    }
    const bool origin_ok = std::isfinite(s.origin[0]) && std::isfinite(s.origin[1]) && std::isfinite(s.origin[2]);
    if (!origin_ok || !std::isfinite(s.spacing) || !(s.spacing > 0.0)) {
        throw Refusal{ORR_ERR_INVALID,
                      std::string(who) + ": grid origin must be finite and spacing positive and finite"};
    }
    const double last[3] = {s.origin[0] + (static_cast<double>(s.nx - 1) + 0.5) * s.spacing,
                            s.origin[1] + (static_cast<double>(s.ny - 1) + 0.5) * s.spacing,
                            s.origin[2] + (static_cast<double>(s.nz - 1) + 0.5) * s.spacing};
    if (!std::isfinite(last[0]) || !std::isfinite(last[1]) || !std::isfinite(last[2])) {
        throw Refusal{ORR_ERR_INVALID, std::string(who) + ": grid extends beyond finite coordinates"};
    }
}

void check_mesh(const orr_mesh* m, const char* who) {
    if (m == nullptr || (m->vertex_count > 0 && m->vertices == nullptr) ||
        (m->triangle_count > 0 && m->triangles == nullptr)) {
        throw Refusal{ORR_ERR_INVALID, std::string(who) + ": null mesh arrays"};
    }
    if (m->triangle_count > std::numeric_limits<uint32_t>::max()) {
        throw Refusal{ORR_ERR_INVALID, "MeshTree: too many triangles"};
    }
    for (uint64_t i = 0; i < 3 * m->triangle_count; ++i) {
        if (m->triangles[i] >= m->vertex_count) {
            throw Refusal{ORR_ERR_INVALID, std::string(who) + ": triangle corner index out of range"};
        }
    }
}

// Device copies of a tree, freed on scope exit.
struct DeviceTree {
    Node* nodes = nullptr;
    double* corners = nullptr;
    uint32_t* overflow = nullptr;
    uint32_t node_count = 0;
    ~DeviceTree() {
        cudaFree(nodes);
        cudaFree(corners);
        cudaFree(overflow);
    }
};

template <class T> T* alloc(std::size_t count, const char* what) {
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<std::size_t>(count, 1) * sizeof(T)), what);
    return static_cast<T*>(p);
}

void upload(const Tree& t, DeviceTree& d, cudaStream_t s) {
    d.node_count = static_cast<uint32_t>(t.nodes.size());
    d.nodes = alloc<Node>(t.nodes.size(), "tree nodes");
    d.corners = alloc<double>(t.corners.size(), "tree triangles");
    d.overflow = alloc<uint32_t>(1, "tree status");
    if (!t.nodes.empty()) {
        check(cudaMemcpyAsync(d.nodes, t.nodes.data(), t.nodes.size() * sizeof(Node), cudaMemcpyHostToDevice, s),
              "tree upload");
        check(cudaMemcpyAsync(d.corners, t.corners.data(), t.corners.size() * sizeof(double),
                              cudaMemcpyHostToDevice, s),
              "tree upload");
    }
    check(cudaMemsetAsync(d.overflow, 0, sizeof(uint32_t), s), "tree status");
}

Grid grid_of(const orr_grid_spec& s) {
    return Grid{s.origin[0], s.origin[1], s.origin[2], s.spacing, static_cast<uint32_t>(s.nx),
                static_cast<uint32_t>(s.ny), static_cast<uint32_t>(s.nz)};
}

// A stream and two events for one call, released on scope exit.
struct Call {
    cudaStream_t stream = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int device;
    explicit Call(int device) : device(device) {
        require_device(device);
        check(cudaSetDevice(device), "cudaSetDevice");
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check(cudaEventCreate(&t0), "event");
        check(cudaEventCreate(&t1), "event");
    }
    ~Call() {
        if (stream) cudaStreamSynchronize(stream);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        cudaStreamDestroy(stream);
    }
};

} // namespace orr::geo

using namespace orr;
using namespace orr::geo;

orr_status orr_grid_around(const double box_min[3], const double box_max[3], double spacing, uint64_t padding,
                           orr_grid_spec* out) {
    return guarded(nullptr, [&]() -> orr_status {
        if (box_min == nullptr || box_max == nullptr || out == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "grid_around: null argument"};
        }
        if (!std::isfinite(spacing) || !(spacing > 0.0)) {
            throw Refusal{ORR_ERR_INVALID, "grid_around: spacing must be positive and finite"};
        }
        bool finite = true;
        for (int k = 0; k < 3; ++k) {
            finite = finite && std::isfinite(box_min[k]) && std::isfinite(box_max[k]);
        }
        if (!finite || !(box_min[0] <= box_max[0]) || !(box_min[1] <= box_max[1]) || !(box_min[2] <= box_max[2])) {
            throw Refusal{ORR_ERR_INVALID, "grid_around: bounds must be finite and ordered (min <= max)"};
        }
        uint64_t n[3];
        for (int k = 0; k < 3; ++k) {
            const double cells = std::ceil((box_max[k] - box_min[k]) / spacing) + 2.0 * static_cast<double>(padding);
            if (!std::isfinite(cells) || !(cells >= 0.0) || cells > static_cast<double>(kMaxGridCells)) {
                throw Refusal{ORR_ERR_INVALID, "grid_around: grid too large"};
            }
            n[k] = std::max<uint64_t>(1, static_cast<uint64_t>(cells));
        }
        orr_grid_spec g{};
        g.spacing = spacing;
        g.nx = n[0];
        g.ny = n[1];
        g.nz = n[2];
        if (!(g.nx <= kMaxGridCells / g.ny && g.nx * g.ny <= kMaxGridCells / g.nz)) {
            throw Refusal{ORR_ERR_INVALID, "grid_around: grid too large"};
        }
        // Centred on the box.
        for (int k = 0; k < 3; ++k) {
            const double centre = (box_min[k] + box_max[k]) * 0.5;
            const double size = static_cast<double>(n[k]) * spacing;
            g.origin[k] = centre - size * 0.5;
        }
        check_grid(g, "grid_around");
        *out = g;
        return ORR_OK;
    });
}

orr_status orr_voxelize(const orr_mesh* mesh, const orr_grid_spec* spec, double threshold, int32_t device,
                        uint8_t* solid, double* winding, double* device_ms) {
    return guarded(nullptr, [&]() -> orr_status {
        if (spec == nullptr || solid == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "voxelize: null argument"};
        }
        check_grid(*spec, "voxelize");
        if (!std::isfinite(threshold)) {
            throw Refusal{ORR_ERR_INVALID, "voxelize: threshold must be finite"};
        }
        check_mesh(mesh, "voxelize");
        const Tree tree = build_tree(mesh->vertices, mesh->vertex_count, mesh->triangles,
                                     static_cast<uint32_t>(mesh->triangle_count));
        if (tree.depth + 1 >= static_cast<uint32_t>(kStack)) {
            throw Refusal{ORR_ERR_INVALID, "voxelize: mesh tree too deep"};
        }
        const uint64_t cells = spec->nx * spec->ny * spec->nz;
        Call call(device);
        DeviceTree d;
        upload(tree, d, call.stream);
        uint8_t* dsolid = alloc<uint8_t>(cells, "voxel flags");
        double* dwinding = winding != nullptr ? alloc<double>(cells, "winding numbers") : nullptr;
        struct Free {
            void* a;
            void* b;
            ~Free() {
                cudaFree(a);
                cudaFree(b);
            }
        } release{dsolid, dwinding};
        const Bricks nb = bricks_of(grid_of(*spec));
        const uint64_t bricks = static_cast<uint64_t>(nb.bx) * nb.by * nb.bz;
        const unsigned blocks = static_cast<unsigned>((bricks + kWarpsPerBlock - 1) / kWarpsPerBlock);
        check(cudaEventRecord(call.t0, call.stream), "event");
        winding_kernel<<<blocks, 32 * kWarpsPerBlock, 0, call.stream>>>(grid_of(*spec), d.nodes, d.corners, d.node_count,
                                                        tree.scale, threshold, dsolid, dwinding, d.overflow);
        check(cudaGetLastError(), "winding kernel");
        check(cudaEventRecord(call.t1, call.stream), "event");
        uint32_t overflow = 0;
        check(cudaMemcpyAsync(&overflow, d.overflow, sizeof overflow, cudaMemcpyDeviceToHost, call.stream),
              "status read-back");
        const HostSpan out[2] = {{solid, dsolid, cells},
                                 {winding, dwinding, winding != nullptr ? cells * sizeof(double) : 0}};
        copy_to_host(out, 2, call.stream, call.device);
        if (overflow != 0) {
            throw Refusal{ORR_ERR_STATE, "voxelize: tree walk exceeded its stack"};
        }
        if (device_ms != nullptr) {
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, call.t0, call.t1), "event");
            *device_ms = ms;
        }
        return ORR_OK;
    });
}

orr_status orr_signed_distance_band(const orr_mesh* mesh, const orr_grid_spec* spec, const uint8_t* solid,
                                    uint64_t solid_count, double band_cells, int32_t device, double* distance,
                                    uint8_t* in_band, double* band_out, double* device_ms) {
    return guarded(nullptr, [&]() -> orr_status {
        if (!std::isfinite(band_cells) || !(band_cells > 0.0)) {
            throw Refusal{ORR_ERR_INVALID, "signed_distance_band: band must be positive"};
        }
        if (spec == nullptr || solid == nullptr || distance == nullptr || in_band == nullptr) {
            throw Refusal{ORR_ERR_INVALID, "signed_distance_band: null argument"};
        }
        check_grid(*spec, "signed_distance_band");
        const uint64_t cells = spec->nx * spec->ny * spec->nz;
        if (solid_count != cells) {
            throw Refusal{ORR_ERR_INVALID, "signed_distance_band: voxel grid does not match its spec"};
        }
        const double band = band_cells * spec->spacing;
        if (!std::isfinite(band)) {
            throw Refusal{ORR_ERR_INVALID, "signed_distance_band: band is not finite"};
        }
        check_mesh(mesh, "signed_distance_band");
        const Tree tree = build_tree(mesh->vertices, mesh->vertex_count, mesh->triangles,
                                     static_cast<uint32_t>(mesh->triangle_count));
        if (tree.depth + 1 >= static_cast<uint32_t>(kStack)) {
            throw Refusal{ORR_ERR_INVALID, "signed_distance_band: mesh tree too deep"};
        }
        Call call(device);
        DeviceTree d;
        upload(tree, d, call.stream);
        uint8_t* dsolid = alloc<uint8_t>(cells, "voxel flags");
        uint8_t* dband = alloc<uint8_t>(cells, "band flags");
        double* ddist = alloc<double>(cells, "distances");
        struct Free {
            void* a;
            void* b;
            void* c;
            ~Free() {
                cudaFree(a);
                cudaFree(b);
                cudaFree(c);
            }
        } release{dsolid, dband, ddist};
        check(cudaMemcpyAsync(dsolid, solid, cells, cudaMemcpyHostToDevice, call.stream), "voxel upload");
        const unsigned blocks = static_cast<unsigned>((cells + 127) / 128);
        check(cudaEventRecord(call.t0, call.stream), "event");
        distance_kernel<<<blocks, 128, 0, call.stream>>>(grid_of(*spec), d.nodes, d.corners, d.node_count, band,
                                                         dsolid, ddist, dband, d.overflow);
        check(cudaGetLastError(), "distance kernel");
        check(cudaEventRecord(call.t1, call.stream), "event");
        uint32_t overflow = 0;
        check(cudaMemcpyAsync(&overflow, d.overflow, sizeof overflow, cudaMemcpyDeviceToHost, call.stream),
              "status read-back");
        const HostSpan out[2] = {{distance, ddist, cells * sizeof(double)}, {in_band, dband, cells}};
        copy_to_host(out, 2, call.stream, call.device);
        if (overflow != 0) {
            throw Refusal{ORR_ERR_STATE, "signed_distance_band: tree walk exceeded its stack"};
        }
        if (band_out != nullptr) {
            *band_out = band;
        }
        if (device_ms != nullptr) {
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, call.t0, call.t1), "event");
            *device_ms = ms;
        }
        return ORR_OK;
    });
}
