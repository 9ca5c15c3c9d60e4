// Boundary-condition inputs of a mesh problem: shell elements, outward
// normals at points, region masks and region force fields.
//
// The reference builds them on the host with CGAL and Eigen:
//  - shell elements: HierarchyGrid::setSolidShellElement (grid/Grid.cpp:
//    253-322) walks every face's grown index box and asks the AABB tree for
//    the squared distance of each element centre to the mesh;
//  - normals: Grid::outwardNormal (grid/Grid.cpp:2838-2854), the closest
//    point of the mesh and its triangle's supporting-plane vector;
//  - regions and fields: the range and field classes of
//    boundary/BoundaryCondition.h, evaluated at node positions in
//    computeProjectionMatrix (grid/Grid.cpp:2694-2760).
// Here each is one FP64 kernel: a block per face for the shell (an element
// in a face's index box within w of that face is within w of the mesh, and an
// element within w of the mesh lies in the index box of its nearest face, so
// the union over faces is the reference's set), a thread per point for the
// normals (the nearest face with the lowest index on a tie, found by a ring
// search over a uniform face grid, or by scanning all faces of small meshes),
// a thread per node or point for the regions and fields.  The file is compiled without
// multiply-add contraction so every product and sum rounds as in the host
// restatement the tests compare with.
#include "rso_internal.cuh"
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>

namespace rso {
namespace {

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 axpy(D3 a, double s, D3 d) { return {a.x + s * d.x, a.y + s * d.y, a.z + s * d.z}; }
__device__ __forceinline__ double qdiv(double n, double d) { return d != 0.0 ? n / d : 0.0; }
// Eigen normalized(): v / sqrt(|v|^2) when |v|^2 > 0, else v
__device__ __forceinline__ D3 unit(D3 v) {
  const double n = dot(v, v);
  if (!(n > 0.0)) return v;
  const double s = sqrt(n);
  return {v.x / s, v.y / s, v.z / s};
}

// Closest point of triangle (a, b, c) to p by Voronoi regions (Ericson,
// Real-Time Collision Detection, 5.1.5); degenerate edges give parameter 0.
__device__ D3 closest_on_triangle(D3 p, D3 a, D3 b, D3 c) {
  const D3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return a;
  const D3 bp = sub(p, b);
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return b;
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return axpy(a, qdiv(d1, d1 - d3), ab);
  const D3 cp = sub(p, c);
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return axpy(a, qdiv(d2, d2 - d6), ac);
  const double va = d3 * d6 - d5 * d4;
  const double e43 = d4 - d3, e56 = d5 - d6;
  if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) return axpy(b, qdiv(e43, e43 + e56), sub(c, b));
  const double den = va + vb + vc;
  const double v = qdiv(vb, den), w = qdiv(vc, den);
  return axpy(axpy(a, v, ab), w, ac);
}

__device__ __forceinline__ D3 vertex(const float* __restrict__ vtx, int i) {
  return {(double)vtx[3 * i], (double)vtx[3 * i + 1], (double)vtx[3 * i + 2]};
}

// one block per face: the face's grown index box, element centres within w of it
__global__ void k_shell(const float* __restrict__ vtx, const int* __restrict__ faces, int nf, double b0x, double b0y,
                        double b0z, double eh, double wshell, int R, const uint8_t* __restrict__ solid,
                        uint8_t* __restrict__ shell) {
  const int f = blockIdx.x;
  if (f >= nf) return;
  const D3 a = vertex(vtx, faces[3 * f]), b = vertex(vtx, faces[3 * f + 1]), c = vertex(vtx, faces[3 * f + 2]);
  const double b0[3] = {b0x, b0y, b0z};
  const double lo[3] = {fmin(fmin(a.x, b.x), c.x), fmin(fmin(a.y, b.y), c.y), fmin(fmin(a.z, b.z), c.z)};
  const double hi[3] = {fmax(fmax(a.x, b.x), c.x), fmax(fmax(a.y, b.y), c.y), fmax(fmax(a.z, b.z), c.z)};
  int lid[3], rid[3];
  for (int j = 0; j < 3; j++) {
    const double ql = (lo[j] - wshell * 1.3 - b0[j] - 0.5 * eh) / eh;
    const double qr = (hi[j] + wshell * 1.3 - b0[j] - 0.5 * eh) / eh + 1;
    // int conversion truncates; out-of-range quotients saturate before the clamp
    lid[j] = (int)fmax(fmin(ql, 2147483647.0), -2147483648.0);
    rid[j] = (int)fmax(fmin(qr, 2147483647.0), -2147483648.0);
    lid[j] = min(max(lid[j], 0), R - 1);
    rid[j] = min(max(rid[j], 0), R - 1);
  }
  const int nbx = rid[0] - lid[0], nby = rid[1] - lid[1], nbz = rid[2] - lid[2];
  if (nbx <= 0 || nby <= 0 || nbz <= 0) return;
  const double sh2 = wshell * wshell;
  const long long nbox = (long long)nbx * nby * nbz;
  for (long long k = threadIdx.x; k < nbox; k += blockDim.x) {
    const int x = lid[0] + (int)(k % nbx), y = lid[1] + (int)((k / nbx) % nby), z = lid[2] + (int)(k / ((long long)nbx * nby));
    const long long e = (long long)x + (long long)R * (y + (long long)R * z);
    if (!solid[e]) continue;
    const D3 p = {(x + 0.5) * eh + b0x, (y + 0.5) * eh + b0y, (z + 0.5) * eh + b0z};
    const D3 d = sub(p, closest_on_triangle(p, a, b, c));
    if (dot(d, d) < sh2) shell[e] = 1;
  }
}

constexpr int kNormalTile = 128;

// outwardNormal's rule for the closest point q of face bf to p: the supporting
// plane's vector (a - c) x (b - c) of CGAL's plane through three points when
// |q - p| < 1e-6, else (q - p) / |q - p| oriented along it
__device__ void emit_normal(const float* __restrict__ vtx, const int* __restrict__ faces, int bf, D3 bq, D3 p,
                            double* __restrict__ out) {
  const D3 ba = vertex(vtx, faces[3 * bf]), bb = vertex(vtx, faces[3 * bf + 1]), bc = vertex(vtx, faces[3 * bf + 2]);
  const D3 tn = cross(sub(ba, bc), sub(bb, bc));
  const D3 pq = sub(bq, p);
  double len = sqrt(dot(pq, pq));
  D3 n;
  if (len < 1e-6) {
    n = unit(tn);
  } else {
    if (dot(pq, tn) < 0.0) len = -len;
    n = {pq.x / len, pq.y / len, pq.z / len};
  }
  out[0] = n.x;
  out[1] = n.y;
  out[2] = n.z;
}

// one thread per point; faces staged through shared memory a tile at a time
__global__ void __launch_bounds__(kNormalTile) k_normals(const float* __restrict__ vtx, const int* __restrict__ faces,
                                                         int nf, const double* __restrict__ pts, int np,
                                                         double* __restrict__ nrm) {
  __shared__ double tri[kNormalTile][9];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  D3 p = {0.0, 0.0, 0.0};
  if (i < np) p = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  double best = INFINITY;
  D3 bq = p;
  int bf = 0;  // face 0 when no distance compares (degenerate faces only)
  for (int t0 = 0; t0 < nf; t0 += kNormalTile) {
    __syncthreads();
    const int f = t0 + threadIdx.x;
    if (f < nf) {
      const D3 a = vertex(vtx, faces[3 * f]), b = vertex(vtx, faces[3 * f + 1]), c = vertex(vtx, faces[3 * f + 2]);
      tri[threadIdx.x][0] = a.x, tri[threadIdx.x][1] = a.y, tri[threadIdx.x][2] = a.z;
      tri[threadIdx.x][3] = b.x, tri[threadIdx.x][4] = b.y, tri[threadIdx.x][5] = b.z;
      tri[threadIdx.x][6] = c.x, tri[threadIdx.x][7] = c.y, tri[threadIdx.x][8] = c.z;
    }
    __syncthreads();
    const int nt = min(kNormalTile, nf - t0);
    if (i < np)
      for (int t = 0; t < nt; t++) {
        const double* q = tri[t];
        const D3 a = {q[0], q[1], q[2]}, b = {q[3], q[4], q[5]}, c = {q[6], q[7], q[8]};
        const D3 cq = closest_on_triangle(p, a, b, c);
        const D3 d = sub(cq, p);
        const double d2 = dot(d, d);
        if (d2 < best) {
          best = d2;
          bq = cq;
          bf = t0 + t;
        }
      }
  }
  if (i >= np) return;
  emit_normal(vtx, faces, bf, bq, p, nrm + 3 * i);
}

// A uniform grid over the mesh's bounding box: cell (x, y, z) lists the faces
// whose bounding box overlaps it (start[cell] .. start[cell + 1] in items).
struct FaceGrid {
  double lo[3], cs[3];
  int g[3];
  double slack;  // absolute slack on distances to cell boundaries (cell-index rounding)
  const int* start;
  const int* items;
};

__device__ __forceinline__ int cell_of(double x, double lo, double cs, int g) {
  const double q = floor((x - lo) / cs);
  return !(q >= 0.0) ? 0 : (q >= (double)g ? g - 1 : (int)q);
}

__device__ __forceinline__ void face_cells(const FaceGrid& G, D3 a, D3 b, D3 c, int* c0, int* c1) {
  const double lo[3] = {fmin(fmin(a.x, b.x), c.x), fmin(fmin(a.y, b.y), c.y), fmin(fmin(a.z, b.z), c.z)};
  const double hi[3] = {fmax(fmax(a.x, b.x), c.x), fmax(fmax(a.y, b.y), c.y), fmax(fmax(a.z, b.z), c.z)};
  for (int j = 0; j < 3; j++) {
    c0[j] = cell_of(lo[j], G.lo[j], G.cs[j], G.g[j]);
    c1[j] = cell_of(hi[j], G.lo[j], G.cs[j], G.g[j]);
  }
}

// FILL false: count the faces of every cell; true: write them (cursor per cell)
template <bool FILL>
__global__ void k_bin_faces(const float* __restrict__ vtx, const int* __restrict__ faces, int nf, FaceGrid G,
                            int* __restrict__ counts, int* __restrict__ items) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  int c0[3], c1[3];
  face_cells(G, vertex(vtx, faces[3 * f]), vertex(vtx, faces[3 * f + 1]), vertex(vtx, faces[3 * f + 2]), c0, c1);
  for (int z = c0[2]; z <= c1[2]; z++)
    for (int y = c0[1]; y <= c1[1]; y++)
      for (int x = c0[0]; x <= c1[0]; x++) {
        const long long cell = x + (long long)G.g[0] * (y + (long long)G.g[1] * z);
        const int slot = atomicAdd(&counts[cell], 1);
        if (FILL) items[G.start[cell] + slot] = f;
      }
}

// one thread per point: cells in rings of growing Chebyshev radius around the
// point's cell, until no face outside the visited block can come as close as
// the best so far (the faces that could still tie or win lie within the
// bound); the best is the lexicographic minimum of (squared distance, face
// index), the brute-force scan's answer
__global__ void k_normals_grid(const float* __restrict__ vtx, const int* __restrict__ faces, FaceGrid G,
                               const double* __restrict__ pts, int np, double* __restrict__ nrm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const D3 p = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  const double pc[3] = {p.x, p.y, p.z};
  int c[3];
  for (int j = 0; j < 3; j++) c[j] = cell_of(pc[j], G.lo[j], G.cs[j], G.g[j]);
  double best = INFINITY;
  D3 bq = p;
  int bf = 0x7fffffff;
  const int rmax = max(G.g[0], max(G.g[1], G.g[2]));
  auto visit = [&](int x, int y, int z) {
    const long long cell = x + (long long)G.g[0] * (y + (long long)G.g[1] * z);
    for (int k = G.start[cell]; k < G.start[cell + 1]; k++) {
      const int f = G.items[k];
      const D3 a = vertex(vtx, faces[3 * f]), b = vertex(vtx, faces[3 * f + 1]), cc = vertex(vtx, faces[3 * f + 2]);
      const D3 q = closest_on_triangle(p, a, b, cc);
      const D3 d = sub(q, p);
      const double d2 = dot(d, d);
      if (d2 < best || (d2 == best && f < bf)) {
        best = d2;
        bq = q;
        bf = f;
      }
    }
  };
  for (int r = 0; r <= rmax; r++) {
    const int z0 = max(c[2] - r, 0), z1 = min(c[2] + r, G.g[2] - 1);
    const int y0 = max(c[1] - r, 0), y1 = min(c[1] + r, G.g[1] - 1);
    const int x0 = max(c[0] - r, 0), x1 = min(c[0] + r, G.g[0] - 1);
    for (int z = z0; z <= z1; z++) {
      const bool zs = z == c[2] - r || z == c[2] + r;
      for (int y = y0; y <= y1; y++) {
        const bool ys = zs || y == c[1] - r || y == c[1] + r;
        if (ys) {
          for (int x = x0; x <= x1; x++) visit(x, y, z);
        } else {
          if (c[0] - r >= 0) visit(c[0] - r, y, z);
          if (r > 0 && c[0] + r < G.g[0]) visit(c[0] + r, y, z);
        }
      }
    }
    // lower bound on the distance from p to cells outside the block: the
    // nearest of the slabs of the grid beyond each block face
    const int b0[3] = {x0, y0, z0}, b1[3] = {x1, y1, z1};
    double bound = INFINITY;
    for (int a = 0; a < 3; a++)
      for (int side = 0; side < 2; side++) {
        if (side == 0 ? b0[a] == 0 : b1[a] == G.g[a] - 1) continue;
        double d2 = 0;
        for (int j = 0; j < 3; j++) {
          double lo = G.lo[j], hi = G.lo[j] + G.g[j] * G.cs[j];
          if (j == a) {
            if (side == 0) hi = G.lo[j] + b0[j] * G.cs[j];
            else lo = G.lo[j] + (b1[j] + 1) * G.cs[j];
          }
          const double e = pc[j] < lo ? lo - pc[j] : (pc[j] > hi ? pc[j] - hi : 0.0);
          d2 += e * e;
        }
        bound = fmin(bound, sqrt(d2));
      }
    if (bound == INFINITY) break;  // the block covers the grid
    const double bd = bound - G.slack;
    if (bd > 0.0 && best < bd * bd * (1.0 - 1e-12)) break;
  }
  emit_normal(vtx, faces, bf == 0x7fffffff ? 0 : bf, bq, p, nrm + 3 * i);
}

__device__ bool region_contains(const rso_region& r, D3 p) {
  const double* q = r.p;
  bool in = false;
  switch (r.kind) {
    case RSO_REGION_SPHERE: {
      const double dx = p.x - q[0], dy = p.y - q[1], dz = p.z - q[2];
      const double s = dx * dx + dy * dy + dz * dz, r2 = q[3] * q[3];
      in = s < r2 || (r.closed && (s - r2) < 1e-8);
      break;
    }
    case RSO_REGION_BOX: {
      const bool inner = q[0] < p.x && p.x < q[3] && q[1] < p.y && p.y < q[4] && q[2] < p.z && p.z < q[5];
      const bool closed_in = q[0] <= p.x && p.x <= q[3] && q[1] <= p.y && p.y <= q[4] && q[2] <= p.z && p.z <= q[5];
      in = inner || (r.closed && closed_in);
      break;
    }
    case RSO_REGION_HALFSPACE: {
      const double s = q[0] * p.x + q[1] * p.y + q[2] * p.z + q[3];
      in = s > 0.0 || (r.closed && s == 0.0);
      break;
    }
    case RSO_REGION_CYLINDER: {
      D3 z = {q[4], q[5], q[6]};
      const double height = sqrt(dot(z, z));
      z = {z.x / height, z.y / height, z.z / height};
      const D3 v = sub(p, D3{q[0], q[1], q[2]});
      const double proj = dot(v, z);
      if (proj > height || proj < 0.0) return false;
      const D3 cr = cross(v, z);
      return !(sqrt(dot(cr, cr)) >= q[3]);
    }
    default:
      return false;
  }
  return in != (r.complement != 0);
}

__global__ void k_region_mask(const rso_region* __restrict__ regions, int nr, double ox, double oy, double oz,
                              double h, int nx, int ny, long long nn, uint8_t* __restrict__ mask) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
  const D3 p = {ox + x * h, oy + y * h, oz + z * h};
  bool in = false;
  for (int k = 0; k < nr; k++) in |= region_contains(regions[k], p);
  mask[i] = in ? 1 : 0;
}

__device__ double field_norm(const rso_field& f, D3 p) {
  const double* q = f.norm_p;
  switch (f.norm_kind) {
    case RSO_FIELD_CONSTANT:
      return q[0];
    case RSO_FIELD_RADIAL: {
      const D3 d = sub(D3{q[0], q[1], q[2]}, p);
      const double radi = sqrt(dot(d, d));
      return q[3] * exp(-pow(radi, q[4] * 2));
    }
    case RSO_FIELD_TWIST: {
      const D3 s = {q[0], q[1], q[2]};
      const D3 ax = unit(sub(D3{q[3], q[4], q[5]}, s));
      const D3 cr = cross(sub(p, s), ax);
      return sqrt(dot(cr, cr)) * q[6];
    }
    default:
      return 0.0;
  }
}

__device__ D3 field_dir(const rso_field& f, D3 p) {
  const double* q = f.dir_p;
  switch (f.dir_kind) {
    case RSO_FIELD_CONSTANT:
      return unit(D3{q[0], q[1], q[2]});
    case RSO_FIELD_RADIAL:
      return unit(sub(D3{q[0], q[1], q[2]}, p));
    case RSO_FIELD_TWIST: {
      const D3 s = {q[0], q[1], q[2]};
      return unit(cross(sub(p, s), sub(D3{q[3], q[4], q[5]}, s)));
    }
    default:
      return {0.0, 0.0, 0.0};
  }
}

__global__ void k_region_field(const rso_field* __restrict__ fields, int nfld, const double* __restrict__ pts,
                               int np, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const D3 p = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
  D3 s = {0.0, 0.0, 0.0};
  for (int k = 0; k < nfld; k++) {
    if (!region_contains(fields[k].region, p)) continue;
    const double m = field_norm(fields[k], p);
    const D3 d = field_dir(fields[k], p);
    s = {s.x + m * d.x, s.y + m * d.y, s.z + m * d.z};
  }
  out[3 * i] = s.x;
  out[3 * i + 1] = s.y;
  out[3 * i + 2] = s.z;
}

// device copies of a host array; frees everything it allocated on destruction
// Device blocks of these entry points, cached per device in power-of-two
// size classes between calls: repeated calls reuse them instead of
// allocating and freeing (a free lets the driver unmap the memory and the
// next allocation map it again, which made the call times vary by tens of
// milliseconds).  At most kCacheCap bytes per device stay cached.
constexpr int kCacheDevices = 64;
constexpr size_t kCacheCap = size_t(1) << 30;
struct BlockCache {
  std::mutex m;
  std::vector<std::pair<size_t, void*>> blocks[kCacheDevices];
  size_t held[kCacheDevices] = {};
};
BlockCache g_blocks;

cudaError_t block_get(int dev, size_t bytes, void** p, size_t* cls) {
  size_t c = 256;
  while (c < bytes) c <<= 1;
  *cls = c;
  if (dev >= 0 && dev < kCacheDevices) {
    std::lock_guard<std::mutex> lk(g_blocks.m);
    auto& v = g_blocks.blocks[dev];
    for (size_t i = 0; i < v.size(); i++)
      if (v[i].first == c) {
        *p = v[i].second;
        g_blocks.held[dev] -= c;
        v.erase(v.begin() + i);
        return cudaSuccess;
      }
  }
  return cudaMalloc(p, c);
}

void block_put(int dev, size_t cls, void* p) {
  if (dev >= 0 && dev < kCacheDevices) {
    std::lock_guard<std::mutex> lk(g_blocks.m);
    if (g_blocks.held[dev] + cls <= kCacheCap) {
      g_blocks.blocks[dev].push_back({cls, p});
      g_blocks.held[dev] += cls;
      return;
    }
  }
  cudaFree(p);
}

// device copies of host arrays and work buffers for one call; the blocks go
// back to the cache when the call returns (every kernel of the call has
// finished by then: each entry point ends with a synchronous copy)
struct Scratch {
  struct Block {
    void* p;
    size_t cls;
  };
  std::vector<Block> blocks;
  int dev = -1;
  cudaError_t err = cudaSuccess;
  Scratch() { err = cudaGetDevice(&dev); }
  template <typename T>
  T* upload(const T* host, size_t n) {
    if (err != cudaSuccess) return nullptr;
    void* p = nullptr;
    size_t cls = 0;
    err = block_get(dev, sizeof(T) * (n ? n : 1), &p, &cls);
    if (err != cudaSuccess) return nullptr;
    blocks.push_back({p, cls});
    if (host && n) err = cudaMemcpy(p, host, sizeof(T) * n, cudaMemcpyHostToDevice);
    return static_cast<T*>(p);
  }
  template <typename T>
  T* alloc(size_t n) { return upload<T>(nullptr, n); }
  ~Scratch() {
    // a failed call may have left work in flight on the device
    if (err != cudaSuccess) cudaDeviceSynchronize();
    for (const Block& b : blocks) block_put(dev, b.cls, b.p);
  }
};

static_assert(sizeof(rso_region) == 80 && sizeof(rso_field) == 192, "rso_region / rso_field layout is part of the ABI");

bool faces_valid(const int* faces, int nf, int nv) {
  for (long long k = 0; k < 3LL * nf; k++)
    if (faces[k] < 0 || faces[k] >= nv) return false;
  return true;
}

bool regions_valid(const rso_region* r, int n) {
  for (int k = 0; k < n; k++)
    if (r[k].kind < RSO_REGION_SPHERE || r[k].kind > RSO_REGION_CYLINDER) return false;
  return true;
}

}  // namespace
}  // namespace rso

using namespace rso;

extern "C" rso_status rso_shell_elements(const float* vertices_host, int n_vertices, const int* faces_host,
                                         int n_faces, const float* box_host, int resolution, double shell_width,
                                         const uint8_t* solid_host, uint8_t* shell_host) {
  if (!vertices_host || !faces_host || !box_host || !solid_host || !shell_host || n_vertices < 3 || n_faces < 1 ||
      resolution < 1 || resolution > 2048 || !(shell_width >= 0) || !faces_valid(faces_host, n_faces, n_vertices))
    return RSO_ERR_INVALID_ARG;
  const int R = resolution;
  const long long nvox = (long long)R * R * R;
  // element edge as the reference forms it: an FP32 difference over an FP32 quotient
  const double eh = (double)((box_host[3] - box_host[0]) / (float)R);
  const double wshell = shell_width * eh;
  Scratch s;
  const float* dv = s.upload(vertices_host, 3 * (size_t)n_vertices);
  const int* df = s.upload(faces_host, 3 * (size_t)n_faces);
  const uint8_t* dsolid = s.upload(solid_host, (size_t)nvox);
  uint8_t* dshell = s.alloc<uint8_t>((size_t)nvox);
  if (s.err == cudaSuccess) s.err = cudaMemset(dshell, 0, (size_t)nvox);
  if (s.err == cudaSuccess && wshell > 0) {
    k_shell<<<n_faces, 256>>>(dv, df, n_faces, box_host[0], box_host[1], box_host[2], eh, wshell, R, dsolid, dshell);
    note_launch();
    s.err = cudaGetLastError();
  }
  if (s.err == cudaSuccess) s.err = cudaMemcpy(shell_host, dshell, (size_t)nvox, cudaMemcpyDeviceToHost);
  return s.err == cudaSuccess ? RSO_OK : RSO_ERR_CUDA;
}

extern "C" rso_status rso_mesh_normals(const float* vertices_host, int n_vertices, const int* faces_host, int n_faces,
                                       const double* points_host, int n_points, double* normals_host) {
  if (!vertices_host || !faces_host || n_vertices < 3 || n_faces < 1 || n_points < 0 ||
      (n_points > 0 && (!points_host || !normals_host)) || !faces_valid(faces_host, n_faces, n_vertices))
    return RSO_ERR_INVALID_ARG;
  if (n_points == 0) return RSO_OK;
  Scratch s;
  const float* dv = s.upload(vertices_host, 3 * (size_t)n_vertices);
  const int* df = s.upload(faces_host, 3 * (size_t)n_faces);
  const double* dp = s.upload(points_host, 3 * (size_t)n_points);
  double* dn = s.alloc<double>(3 * (size_t)n_points);
  // meshes of a few hundred faces or more: bin the faces on a uniform grid
  // of about two faces per cell and search rings of cells around each point
  bool grid = false;
  FaceGrid G{};
  if (s.err == cudaSuccess && n_faces >= 256) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (long long k = 0; k < 3LL * n_faces; k++) {
      const int v = faces_host[k];
      for (int a = 0; a < 3; a++) {
        lo[a] = std::fmin(lo[a], (double)vertices_host[3 * v + a]);
        hi[a] = std::fmax(hi[a], (double)vertices_host[3 * v + a]);
      }
    }
    double ext[3], emax = 0, mag = 0;
    for (int a = 0; a < 3; a++) {
      ext[a] = hi[a] - lo[a];
      emax = std::fmax(emax, ext[a]);
      mag = std::fmax(mag, std::fmax(std::fabs(lo[a]), std::fabs(hi[a])));
    }
    if (emax > 0 && std::isfinite(emax) && std::isfinite(mag)) {
      const double target = std::min(std::max(n_faces / 2.0, 1.0), (double)(1 << 21));
      double vol = 1;
      for (int a = 0; a < 3; a++) vol *= std::fmax(ext[a], 1e-3 * emax);
      const double cs = std::cbrt(vol / target);
      long long ncell = 1;
      double csmin = INFINITY;
      for (int a = 0; a < 3; a++) {
        G.g[a] = (int)std::min(std::max(std::ceil(ext[a] / cs), 1.0), 1024.0);
        G.cs[a] = ext[a] > 0 ? ext[a] / G.g[a] : cs;
        G.lo[a] = lo[a];
        ncell *= G.g[a];
        csmin = std::fmin(csmin, G.cs[a]);
      }
      G.slack = 1e-9 * csmin + 1e-14 * mag;
      int* counts = s.alloc<int>((size_t)ncell);
      if (s.err == cudaSuccess) s.err = cudaMemset(counts, 0, sizeof(int) * ncell);
      if (s.err == cudaSuccess) {
        k_bin_faces<false><<<cdiv(n_faces, 256), 256>>>(dv, df, n_faces, G, counts, nullptr);
        note_launch();
        s.err = cudaGetLastError();
      }
      std::vector<int> hc((size_t)ncell);
      if (s.err == cudaSuccess) s.err = cudaMemcpy(hc.data(), counts, sizeof(int) * ncell, cudaMemcpyDeviceToHost);
      std::vector<int> hs((size_t)ncell + 1, 0);
      long long total = 0;
      for (long long cidx = 0; cidx < ncell; cidx++) {
        hs[cidx] = (int)std::min(total, (long long)INT32_MAX);
        total += hc[cidx];
      }
      hs[ncell] = (int)std::min(total, (long long)INT32_MAX);
      if (s.err == cudaSuccess && total <= (1LL << 25)) {
        int* start = s.upload(hs.data(), hs.size());
        int* items = s.alloc<int>((size_t)std::max(total, 1LL));
        if (s.err == cudaSuccess) s.err = cudaMemset(counts, 0, sizeof(int) * ncell);
        if (s.err == cudaSuccess) {
          G.start = start;
          G.items = items;
          k_bin_faces<true><<<cdiv(n_faces, 256), 256>>>(dv, df, n_faces, G, counts, items);
          note_launch();
          s.err = cudaGetLastError();
          grid = s.err == cudaSuccess;
        }
      }
    }
  }
  if (s.err == cudaSuccess && grid) {
    k_normals_grid<<<cdiv(n_points, 128), 128>>>(dv, df, G, dp, n_points, dn);
    note_launch();
    s.err = cudaGetLastError();
  } else if (s.err == cudaSuccess) {
    k_normals<<<cdiv(n_points, kNormalTile), kNormalTile>>>(dv, df, n_faces, dp, n_points, dn);
    note_launch();
    s.err = cudaGetLastError();
  }
  if (s.err == cudaSuccess)
    s.err = cudaMemcpy(normals_host, dn, sizeof(double) * 3 * (size_t)n_points, cudaMemcpyDeviceToHost);
  return s.err == cudaSuccess ? RSO_OK : RSO_ERR_CUDA;
}

extern "C" rso_status rso_region_mask(const rso_region* regions_host, int n_regions, const double* origin_host,
                                      double h, int nx, int ny, int nz, uint8_t* mask_host) {
  if (n_regions < 0 || (n_regions > 0 && !regions_host) || !origin_host || !mask_host || nx < 1 || ny < 1 || nz < 1 ||
      !regions_valid(regions_host, n_regions))
    return RSO_ERR_INVALID_ARG;
  const long long nn = (long long)nx * ny * nz;
  Scratch s;
  const rso_region* dr = s.upload(regions_host, (size_t)n_regions);
  uint8_t* dm = s.alloc<uint8_t>((size_t)nn);
  if (s.err == cudaSuccess) {
    k_region_mask<<<cdiv(nn, 256), 256>>>(dr, n_regions, origin_host[0], origin_host[1], origin_host[2], h, nx, ny,
                                          nn, dm);
    note_launch();
    s.err = cudaGetLastError();
  }
  if (s.err == cudaSuccess) s.err = cudaMemcpy(mask_host, dm, (size_t)nn, cudaMemcpyDeviceToHost);
  return s.err == cudaSuccess ? RSO_OK : RSO_ERR_CUDA;
}

extern "C" rso_status rso_region_field(const rso_field* fields_host, int n_fields, const double* points_host,
                                       int n_points, double* vectors_host) {
  if (n_fields < 0 || (n_fields > 0 && !fields_host) || n_points < 0 ||
      (n_points > 0 && (!points_host || !vectors_host)))
    return RSO_ERR_INVALID_ARG;
  for (int k = 0; k < n_fields; k++)
    if (!regions_valid(&fields_host[k].region, 1) || fields_host[k].norm_kind < 0 || fields_host[k].norm_kind > 2 ||
        fields_host[k].dir_kind < 0 || fields_host[k].dir_kind > 2)
      return RSO_ERR_INVALID_ARG;
  if (n_points == 0) return RSO_OK;
  Scratch s;
  const rso_field* df = s.upload(fields_host, (size_t)n_fields);
  const double* dp = s.upload(points_host, 3 * (size_t)n_points);
  double* dout = s.alloc<double>(3 * (size_t)n_points);
  if (s.err == cudaSuccess) {
    k_region_field<<<cdiv(n_points, 128), 128>>>(df, n_fields, dp, n_points, dout);
    note_launch();
    s.err = cudaGetLastError();
  }
  if (s.err == cudaSuccess)
    s.err = cudaMemcpy(vectors_host, dout, sizeof(double) * 3 * (size_t)n_points, cudaMemcpyDeviceToHost);
  return s.err == cudaSuccess ? RSO_OK : RSO_ERR_CUDA;
}
