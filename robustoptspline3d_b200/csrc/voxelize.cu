// Solid voxelisation of a closed triangle mesh (the mesh -> voxel-mask input
// of the reference's drivers).
//
// The reference vendors cuda_voxelizer (voxelizer/, Jeroen Baert's
// cuda_voxelizer with its solid-voxelisation extension) and calls it from
// voxelize_mesh (voxelizer/voxelize_main.cpp:344-399):
//  - the grid is a cube of R^3 voxels, R the smallest power of two above the
//    preferred resolution, around the mesh's bounding box enlarged to
//    max_len * R / preferred on every axis and centred
//    (padd2SatifyResolution, voxelize_main.cpp:313-342), so the mesh spans
//    `preferred` voxels along its longest axis;
//  - a voxel is solid when its centre has an odd number of mesh crossings on
//    its +x side: every triangle (skipped when its normal is perpendicular to
//    x) is projected on the yz plane, the voxel-centre columns (y, z) inside
//    it, with the top-left rule deciding points on an edge, get the x of the
//    crossing, and the voxels x = 0 .. int(x / unit - 0.5) of that column flip
//    (cpu_voxelize_mesh_solid, voxelizer/cpu_voxelizer.cpp:206-330).
// Here a thread per triangle writes each crossing as one XOR into a crossing
// table at (int(x / unit - 0.5), y, z), and a scan along x turns the table into
// the parity of crossings at or above each x: the same voxels, one atomic per
// crossing instead of one per flipped voxel.
#include "rso_internal.cuh"
#include <cmath>
#include <vector>

namespace rso {
namespace {

constexpr float kVoxEps = 0.000001f;  // float_error of the reference

__device__ __forceinline__ bool top_left(float2 v0, float2 v1) {
  return (v1.y < v0.y) || (v1.y == v0.y && v0.x > v1.x);
}

__device__ __forceinline__ int point_in_triangle(float2 v0, float2 v1, float2 v2, float2 p) {
  const float2 pa = make_float2(p.x - v0.x, p.y - v0.y), pb = make_float2(p.x - v1.x, p.y - v1.y),
               pc = make_float2(p.x - v2.x, p.y - v2.y);
  const float t1 = pa.x * pb.y - pa.y * pb.x;
  if (fabsf(t1) < kVoxEps && pa.x * pb.x <= 0 && pa.y * pb.y <= 0) return 1;
  const float t2 = pb.x * pc.y - pb.y * pc.x;
  if (fabsf(t2) < kVoxEps && pb.x * pc.x <= 0 && pb.y * pc.y <= 0) return 2;
  const float t3 = pc.x * pa.y - pc.y * pa.x;
  if (fabsf(t3) < kVoxEps && pc.x * pa.x <= 0 && pc.y * pa.y <= 0) return 3;
  return (t1 * t2 > 0 && t1 * t3 > 0) ? 0 : -1;
}

// one thread per triangle; crossings XOR-ed into cross[(z * R + y) * R + x] (bytes)
__global__ void k_vox_cross(const float* __restrict__ tri, long long ntri, float3 bmin, float unit, int R,
                            unsigned int* __restrict__ cross_words) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= ntri) return;
  const float* q = tri + 9 * t;
  const float3 v0 = make_float3(q[0] - bmin.x, q[1] - bmin.y, q[2] - bmin.z);
  const float3 v1 = make_float3(q[3] - bmin.x, q[4] - bmin.y, q[5] - bmin.z);
  const float3 v2 = make_float3(q[6] - bmin.x, q[7] - bmin.y, q[8] - bmin.z);
  const float3 e0 = make_float3(v1.x - v0.x, v1.y - v0.y, v1.z - v0.z);
  const float3 e1 = make_float3(v2.x - v1.x, v2.y - v1.y, v2.z - v1.z);
  float3 n = make_float3(e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x);
  // glm::normalize: v * (1 / sqrt(v . v)); this file is compiled without
  // multiply-add contraction, so every step rounds as on the host
  const float nd = n.x * n.x + n.y * n.y + n.z * n.z;
  if (!(nd > 0.f)) return;
  const float inv = 1.0f / sqrtf(nd);
  n = make_float3(n.x * inv, n.y * inv, n.z * inv);
  if (fabsf(n.x) < kVoxEps) return;
  float2 a = make_float2(v0.y, v0.z), b = make_float2(v1.y, v1.z), c = make_float2(v2.y, v2.z);
  {
    const float2 d0 = make_float2(b.x - a.x, b.y - a.y), d1 = make_float2(c.x - a.x, c.y - a.y);
    if (!(d0.x * d1.y - d1.x * d0.y > 0)) {  // make the projection counterclockwise
      const float2 w = b;
      b = c;
      c = w;
    }
  }
  const float ymaxw = fmaxf(a.x, fmaxf(b.x, c.x)), zmaxw = fmaxf(a.y, fmaxf(b.y, c.y));
  const float yminw = fminf(a.x, fminf(b.x, c.x)), zminw = fminf(a.y, fminf(b.y, c.y));
  // the reference subtracts a double 0.5 from the FP32 quotients and forms the
  // sample points in double before storing them as FP32
  const int y1 = max((int)floor((double)(ymaxw / unit) - 0.5), -1), z1 = max((int)floor((double)(zmaxw / unit) - 0.5), -1);
  const int y0 = max((int)ceil((double)(yminw / unit) - 0.5), 0), z0 = max((int)ceil((double)(zminw / unit) - 0.5), 0);
  for (int y = y0; y <= min(y1, R - 1); y++)
    for (int z = z0; z <= min(z1, R - 1); z++) {
      const float2 p = make_float2((float)((y + 0.5) * (double)unit), (float)((z + 0.5) * (double)unit));
      const int k = point_in_triangle(a, b, c, p);
      if ((k == 1 && top_left(a, b)) || (k == 2 && top_left(b, c)) || (k == 3 && top_left(c, a)) || k == 0) {
        const float xi = -(n.y * (p.x - v0.y) + n.z * (p.y - v0.z)) / n.x + v0.x;
        const int xm = (int)((double)(xi / unit) - 0.5);
        if (xm < 0) continue;  // no voxel centre lies before the crossing
        const int x = min(xm, R - 1);
        const long long idx = ((long long)z * R + y) * R + x;
        atomicXor(cross_words + idx / 4, 1u << (8 * (idx % 4)));
      }
    }
}

// solid[x] = parity of the crossings at x' >= x along each (y, z) column
__global__ void k_vox_scan(const unsigned char* __restrict__ cross, int R, unsigned char* __restrict__ solid) {
  const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (col >= (long long)R * R) return;
  const unsigned char* c = cross + col * R;
  unsigned char* s = solid + col * R;
  unsigned char p = 0;
  for (int x = R - 1; x >= 0; x--) {
    p ^= c[x] & 1;
    s[x] = p;
  }
}

}  // namespace
}  // namespace rso

using namespace rso;

extern "C" rso_status rso_voxelize(const float* vertices_host, int n_vertices, const int* faces_host, int n_faces,
                                   int preferred_resolution, uint8_t* solid_host, int* resolution_out,
                                   float* box_out) {
  if (!vertices_host || !faces_host || n_vertices < 3 || n_faces < 1 || preferred_resolution < 1 ||
      !resolution_out)
    return RSO_ERR_INVALID_ARG;
  // padded cubic grid (padd2SatifyResolution)
  int R = 1;
  for (int i = 0; i < 32 && !(preferred_resolution < R); i++) R <<= 1;
  if (R > 2048) return RSO_ERR_INVALID_ARG;
  *resolution_out = R;
  if (!solid_host && !box_out) return RSO_OK;  // size query
  float lo[3], hi[3];
  for (int a = 0; a < 3; a++) { lo[a] = INFINITY; hi[a] = -INFINITY; }
  for (int i = 0; i < n_vertices; i++)
    for (int a = 0; a < 3; a++) {
      lo[a] = std::fmin(lo[a], vertices_host[3 * i + a]);
      hi[a] = std::fmax(hi[a], vertices_host[3 * i + a]);
    }
  const float len[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const float maxlen = std::fmax(std::fmax(len[0], len[1]), len[2]);
  if (!(maxlen > 0)) return RSO_ERR_INVALID_ARG;
  float bmin[3], bmax[3];
  for (int a = 0; a < 3; a++) {
    const float pad = maxlen * R / preferred_resolution;
    bmin[a] = lo[a] - (pad - len[a]) / 2;
    bmax[a] = hi[a] + (pad - len[a]) / 2;
  }
  if (box_out)
    for (int a = 0; a < 3; a++) { box_out[a] = bmin[a]; box_out[3 + a] = bmax[a]; }
  if (!solid_host) return RSO_OK;
  const float unit = (bmax[0] - bmin[0]) / R;  // voxinfo unit of a cubic grid
  std::vector<float> tri((size_t)9 * n_faces);
  for (int f = 0; f < n_faces; f++)
    for (int k = 0; k < 3; k++) {
      const int v = faces_host[3 * f + k];
      if (v < 0 || v >= n_vertices) return RSO_ERR_INVALID_ARG;
      for (int a = 0; a < 3; a++) tri[(size_t)9 * f + 3 * k + a] = vertices_host[3 * v + a];
    }
  const long long nvox = (long long)R * R * R;
  float* dtri = nullptr;
  unsigned char *cross = nullptr, *solid = nullptr;
  cudaError_t e = cudaMalloc(&dtri, sizeof(float) * tri.size());
  if (e == cudaSuccess) e = cudaMalloc(&cross, (size_t)nvox);
  if (e == cudaSuccess) e = cudaMalloc(&solid, (size_t)nvox);
  if (e == cudaSuccess) e = cudaMemcpy(dtri, tri.data(), sizeof(float) * tri.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(cross, 0, (size_t)nvox);
  if (e == cudaSuccess) {
    k_vox_cross<<<(unsigned)cdiv(n_faces, 128), 128>>>(dtri, n_faces, make_float3(bmin[0], bmin[1], bmin[2]), unit,
                                                      R, reinterpret_cast<unsigned int*>(cross));
    note_launch();
    k_vox_scan<<<(unsigned)cdiv((long long)R * R, 256), 256>>>(cross, R, solid);
    note_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(solid_host, solid, (size_t)nvox, cudaMemcpyDeviceToHost);
  cudaFree(dtri);
  cudaFree(cross);
  cudaFree(solid);
  return e == cudaSuccess ? RSO_OK : RSO_ERR_CUDA;
}
