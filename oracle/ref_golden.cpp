// Host harness around definitions extracted from the reference by
// ref_extract.py (test infrastructure, built into oracle/_ref/ only; see
// tests/golden/make_golden.py, which runs it and writes the golden fixtures).
//
// The extracted code is the reference's own, unmodified: the Heaviside and
// Dirac functions and the self-support penalty functions (grid/Grid.cu:76-190),
// the spline basis recursion and its derivatives (grid/Grid.cu:427-857), the
// knot series (grid/Grid.cpp:3307-3431), the density-map kernel with its
// element-centre functor (grid/Grid.cu:3405-3502), the sensitivity-filter
// kernel with its weight functor (grid/Grid.cu:4210-4309), the projection
// kernels (optimization/optimization.cu:167-189, :324-348) and the bit-array
// rank structure gBitSAT (culib/lib.cuh:1473-1550), and for the surface-point
// self-support the background marching-cubes values (grid/Grid.cu:4109-4160),
// generateEquidistantIntegers (grid/Grid.cpp:3831-3847) and the per-point
// normal, orientation probe, flag, constraint and coefficient-gradient
// functors (grid/Grid.cu:5711-5760, :5810-5860, :5949-5975, :6216-6262,
// :6379-6490) with oh/doh/norm/dot (:139-155, :858-876).  Below, the CUDA keywords
// are empty, the __constant__ symbols are host globals, and a kernel "launch"
// runs every thread index in turn.  Host libm's tanhf/expf/sqrtf stand in for
// CUDA's and the host compiler does not contract multiply-adds, so results
// may differ from the reference's GPU run by a few FP32 ulps.
//
// Usage (every array a raw little-endian file):
//   ref_golden funcs N x.f32 beta a mid c out.f32
//   ref_golden proj N beta rhomin rho.f32 shellflag.i32 sens.f32 out_rho.f32 out_sens.f32
//   ref_golden spline ereso order px py pz nword bits.u32 sat.i32 coeff.f32 eflag.i32 rhomin
//                     out_knots.f32 out_axis.f32 out_rho.f32
//   ref_golden filter ereso nword bits.u32 sat.i32 n_active sens.f32 radius out.f32
//   ref_golden surface ereso order px py pz coeff.f32 mc npts pts.f32 beta opt_ratio default_ratio
//                      out_mc.f32 out_equi.i32 out_pts.f32 out_dc.f32 out_scalar.f32
#include <math.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#define __device__
#define __host__
#define __global__
#define __constant__
#define __forceinline__ inline

static inline int __popc(unsigned int v) { return __builtin_popcount(v); }
struct HostIdx {
  unsigned int x = 0, y = 0, z = 0;
};
static HostIdx threadIdx, blockIdx, blockDim;

// gBitSAT's allocating constructor and destroy() name these; the harness
// builds gBitSAT from host pointers only and never calls either
enum HostMemcpyKind { cudaMemcpyHostToDevice };
template <typename T>
static int cudaMalloc(T**, size_t) { return 1; }
static int cudaMemcpy(void*, const void*, size_t, HostMemcpyKind) { return 1; }
static int cudaFree(void*) { return 0; }

// the reference's spline order is a compile-time constant (grid/Grid.h:37)
constexpr static int m_iM = 3;

// node and element flag bits (grid/Grid.h:399-439): only the shell-element bit is read
namespace grid {
struct Grid {
  enum Bitmask { mask_shellelement = 1 << 12 };
};
}  // namespace grid

template <typename T>
struct BitCount {
  static constexpr int value = sizeof(T) * 8;
};

// __constant__ symbols read by the extracted code
static float gnBoundMin[3], gnstep[3];
static int gorder[1], gnbasis[3];
static float* gpu_KnotSer[3];
static float* gpu_cijk;
static float* gpu_SurfacePoints[3];
static float* gpu_surface_normal[3];
static int* gV2E[8];
static int* gEflag[1];

#include "lib_bits.inc"
#include "grid_funcs.inc"
#include "grid_kernels.inc"
#include "opt_kernels.inc"
#include <iostream>
#include "surf_funcs.inc"

// the reference's upload helper, a no-op on the host
struct gpu_manager_t {
  static void upload_buf(void*, const void*, size_t) {}
};

// the members set_spline_knot_series reads and writes (grid/Grid.h:243-312, :448)
struct KnotGrid {
  int n_order;
  size_t n_partitionx, n_partitiony, n_partitionz;
  int spknotspan[3];
  float m_sStep[3];
  float m_3sBoundMin[3], m_3sBoundMax[3];
  std::vector<float> KnotSer[3];
  float m_sStepX, m_sStepY, m_sStepZ;
  struct {
    float* KnotSer[3];
  } _gbuf;
  float _box[2][3];
  void set_spline_knot_series(void)
#include "knots_body.inc"
};

// ---------------------------------------------------------------- host plumbing
template <typename T>
static std::vector<T> load(const char* path, size_t n) {
  std::vector<T> v(n);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(T), n, f) != n) {
    std::fprintf(stderr, "cannot read %zu values from %s\n", n, path);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}
template <typename T>
static void save(const char* path, const std::vector<T>& v) {
  FILE* f = std::fopen(path, "wb");
  if (!f || std::fwrite(v.data(), sizeof(T), v.size(), f) != v.size()) {
    std::fprintf(stderr, "cannot write %s\n", path);
    std::exit(2);
  }
  std::fclose(f);
}
// runs kernel(args...) for every thread of a 1-D grid of `blocks` x `threads`
template <typename K>
static void launch(long long n_threads, int threads, K kernel) {
  blockDim.x = threads;
  const long long blocks = (n_threads + threads - 1) / threads;
  for (long long b = 0; b < blocks; b++)
    for (int t = 0; t < threads; t++) {
      blockIdx.x = (unsigned)b;
      threadIdx.x = (unsigned)t;
      kernel();
    }
}

static int cmd_funcs(char** a) {
  const size_t n = std::atol(a[0]);
  std::vector<float> x = load<float>(a[1], n);
  const float beta = std::atof(a[2]), pa = std::atof(a[3]), mid = std::atof(a[4]), c = std::atof(a[5]);
  std::vector<float> out(10 * n);
  for (size_t i = 0; i < n; i++) {
    out[0 * n + i] = Heaviside(x[i], beta);
    out[1 * n + i] = Dirac(x[i], beta);
    out[2 * n + i] = h(x[i], pa);
    out[3 * n + i] = dh(x[i], pa);
    out[4 * n + i] = inner_(x[i], pa);
    out[5 * n + i] = dinner_(x[i], pa);
    out[6 * n + i] = overhang(x[i], mid, c);
    out[7 * n + i] = doverhang(x[i], mid, c);
    out[8 * n + i] = normal_distri(x[i], pa);
    out[9 * n + i] = dnormal_distri(x[i], pa);
  }
  save(a[6], out);
  return 0;
}

static int cmd_proj(char** a) {
  const int n = std::atoi(a[0]);
  const float beta = std::atof(a[1]), rhomin = std::atof(a[2]);
  std::vector<float> rho = load<float>(a[3], n), sens = load<float>(a[5], n);
  std::vector<int> flag = load<int>(a[4], n);
  // one "vertex" per element, its corner-7 element being the element itself
  std::vector<int> v2e7(n);
  for (int i = 0; i < n; i++) v2e7[i] = i;
  gV2E[7] = v2e7.data();
  gEflag[0] = flag.data();
  std::vector<float> out_rho(n, 0.f), out_sens(n, 0.f);
  launch(n, 256, [&] { computeProjection_kernel(n, rho.data(), rhomin, out_rho.data(), beta); });
  launch(n, 256, [&] { computeProjectionSensitivity_kernel(n, rho.data(), sens.data(), out_sens.data(), beta); });
  save(a[6], out_rho);
  save(a[7], out_sens);
  return 0;
}

// HierarchyGrid::set_spline_partition (grid/Grid.cu:3187-3256) sets these;
// the knot series of a box [0, ereso]^3 with unit elements
static KnotGrid& setup_knots(int ereso, int order, const int* part) {
  static KnotGrid g;
  g.n_order = order;
  g.n_partitionx = part[0];
  g.n_partitiony = part[1];
  g.n_partitionz = part[2];
  for (int i = 0; i < 3; i++) {
    g.spknotspan[i] = 2 * order + part[i];
    g._box[0][i] = 0.f;
    g._box[1][i] = (float)ereso;
  }
  g.set_spline_knot_series();
  gorder[0] = order;
  for (int i = 0; i < 3; i++) {
    gnbasis[i] = order + part[i];
    gnBoundMin[i] = g.m_3sBoundMin[i];
    gnstep[i] = g.m_sStep[i];
    gpu_KnotSer[i] = g.KnotSer[i].data();
  }
  return g;
}

static int cmd_spline(char** a) {
  const int ereso = std::atoi(a[0]), order = std::atoi(a[1]);
  const int part[3] = {std::atoi(a[2]), std::atoi(a[3]), std::atoi(a[4])};
  const int nword = std::atoi(a[5]);
  std::vector<unsigned int> bits = load<unsigned int>(a[6], nword);
  std::vector<int> sat = load<int>(a[7], nword + 1);
  const int nb[3] = {order + part[0], order + part[1], order + part[2]};
  std::vector<float> coeff = load<float>(a[8], (size_t)nb[0] * nb[1] * nb[2]);
  const int n_active = sat[nword];
  std::vector<int> eflag = load<int>(a[9], n_active);
  const float min_Density = std::atof(a[10]);
  if (order != m_iM) {
    std::fprintf(stderr, "the reference's basis functions are compiled for order %d\n", m_iM);
    return 2;
  }
  KnotGrid& g = setup_knots(ereso, order, part);
  std::vector<float> knots;
  for (int i = 0; i < 3; i++) {
    knots.push_back(g.m_3sBoundMin[i]);
    knots.push_back(g.m_3sBoundMax[i]);
    knots.push_back(g.m_sStep[i]);
    knots.insert(knots.end(), g.KnotSer[i].begin(), g.KnotSer[i].end());
  }
  save(a[11], knots);
  // per axis and element coordinate: SplineBasisX (m_iM + 1 values), the
  // derivative routine's values (n = 1) and first derivatives (n = 2)
  std::vector<float> axis;
  for (int ax = 0; ax < 3; ax++)
    for (int x = 0; x < ereso; x++) {
      const float pos = 0.f + x * 1.f + 0.5 * 1.f;
      float b[m_iM + 1], v[m_iM], d[m_iM];
      if (ax == 0) { SplineBasisX(pos, b); SplineBasisDeriX(pos, 1, v); SplineBasisDeriX(pos, 2, d); }
      if (ax == 1) { SplineBasisY(pos, b); SplineBasisDeriY(pos, 1, v); SplineBasisDeriY(pos, 2, d); }
      if (ax == 2) { SplineBasisZ(pos, b); SplineBasisDeriZ(pos, 1, v); SplineBasisDeriZ(pos, 2, d); }
      axis.insert(axis.end(), b, b + m_iM + 1);
      axis.insert(axis.end(), v, v + m_iM);
      axis.insert(axis.end(), d, d + m_iM);
    }
  save(a[12], axis);
  // Grid::coeff2density (grid/Grid.cu:3439-3502) on a box with origin 0 and unit elements
  float* cijk_value = coeff.data();
  const float eh = 1.f;
  const float boxOrigin[3] = {0.f, 0.f, 0.f};
#include "calc_node.inc"
  gBitSAT<unsigned int> esat(bits.data(), sat.data());
  std::vector<float> rho(n_active, 0.f);
  launch(nword, 512, [&] {
    coeff2density_kernel(nword, min_Density, esat, ereso, rho.data(), calc_node, (const int*)nullptr, eflag.data());
  });
  save(a[13], rho);
  return 0;
}

static int cmd_filter(char** a) {
  const int ereso = std::atoi(a[0]), nword = std::atoi(a[1]);
  std::vector<unsigned int> bits = load<unsigned int>(a[2], nword);
  std::vector<int> sat = load<int>(a[3], nword + 1);
  const int n_active = std::atoi(a[4]);
  std::vector<float> sens = load<float>(a[5], n_active);
  const double radii = std::atof(a[6]);
#include "filter_weight.inc"
  gBitSAT<unsigned int> esat(bits.data(), sat.data());
  std::vector<float> out(n_active, 0.f);
  launch(nword, 512, [&] {
    filterSensitivity_kernel(nword, esat, ereso, sens.data(), out.data(), radii, fr, (const int*)nullptr);
  });
  save(a[7], out);
  return 0;
}

// surface-point self-support on a box [0, ereso]^3 (the model box) with the
// given points; every mode 0..5 (GlobalSSMode, grid/Grid.h:177-184)
static int cmd_surface(char** a) {
  const int ereso = std::atoi(a[0]), order = std::atoi(a[1]);
  const int part[3] = {std::atoi(a[2]), std::atoi(a[3]), std::atoi(a[4])};
  if (order != m_iM) {
    std::fprintf(stderr, "the reference's basis functions are compiled for order %d\n", m_iM);
    return 2;
  }
  const int nb[3] = {order + part[0], order + part[1], order + part[2]};
  const long ncoef = (long)nb[0] * nb[1] * nb[2];
  std::vector<float> coeff = load<float>(a[5], ncoef);
  const int mc_ereso = std::atoi(a[6]);
  const int npts = std::atoi(a[7]);
  std::vector<float> pts = load<float>(a[8], 3 * (size_t)npts);
  const float beta = std::atof(a[9]);
  const float opt_angle = std::atof(a[10]) * M_PI, default_print_angle = std::atof(a[11]) * M_PI;
  setup_knots(ereso, order, part);
  gpu_cijk = coeff.data();

  // Grid::compute_background_mcPoints_value (grid/Grid.cu:4066-4175), model box [0, ereso]^3
  {
    float* cijk_value = coeff.data();
    const int ereso_mc = mc_ereso + 2;
    const float ehx = ((float)ereso - 0.f) / mc_ereso, ehy = ehx, ehz = ehx;
    const float boxOrigin[3] = {0.f, 0.f, 0.f};
    const float boxEnd[3] = {(float)ereso, (float)ereso, (float)ereso};
    const float boxOrispan[3] = {0.f - ehx, 0.f - ehy, 0.f - ehz};
    const int n3 = ereso_mc * ereso_mc * ereso_mc;
    std::vector<float> out(4 * (size_t)n3);
    float* nodex = out.data();
    float* nodey = nodex + n3;
    float* nodez = nodey + n3;
    float* node_value = nodez + n3;
    {
      const int ereso = ereso_mc;
#include "surf_mc.inc"
      for (int id = 0; id < n3; id++) calc_node(id);
    }
    save(a[12], out);
  }
  // generateEquidistantIntegers (grid/Grid.cpp:3831-3847) on fixed pairs
  {
    const int pairs[6][2] = {{100, 10}, {1000, 300}, {1574, 1500}, {12345, 600}, {50, 49}, {7, 3}};
    std::vector<int> out;
    for (auto& pr : pairs) {
      std::vector<int> v = generateEquidistantIntegers(pr[0], pr[1]);
      out.insert(out.end(), v.begin(), v.end());
    }
    save(a[13], out);
  }
  // per point: normal (5709-5760), orientation (5800-5943), flag (5945-5992)
  for (int i = 0; i < 3; i++) gpu_SurfacePoints[i] = pts.data() + (size_t)i * npts;
  std::vector<float> nrm(3 * (size_t)npts, 0.f), dir(npts, 0.f), flag(npts, 0.f);
  for (int i = 0; i < 3; i++) gpu_surface_normal[i] = nrm.data() + (size_t)i * npts;
  {
#include "surf_normal.inc"
    for (int id = 0; id < npts; id++) calc_normal(id);
  }
  double dirsum = 0;
  {
    float* direction_tmp = dir.data();
#include "surf_dir.inc"
    for (int id = 0; id < npts; id++) calc_node(id);
    for (int id = 0; id < npts; id++) dirsum += dir[id];
  }
  if (dirsum < 0)
    for (auto& v : nrm) v = -v;
  {
#include "surf_flag.inc"
    for (int id = 0; id < npts; id++) flag[id] = calc_node(id);
  }
  // per mode: constraint (6198-6283), mean (6285-6328), gradient (6330-6505) / count (Grid.cpp:4263-4280)
  std::vector<float> per(6 * (size_t)npts), dcs(6 * (size_t)ncoef), scalars;
  scalars.push_back((float)dirsum);
  int down = 0;
  for (int id = 0; id < npts; id++) down += nrm[2 * (size_t)npts + id] < 0;
  for (int modeid = 0; modeid < 6; modeid++) {
    const float print_angle = opt_angle;
    const float func_para = modeid <= 1 ? 8.0f : (modeid <= 3 ? 10.0f : 0.09f);  // grid/Grid.h:371-375
    {
#include "surf_ss.inc"
      for (int id = 0; id < npts; id++) per[(size_t)modeid * npts + id] = calc_node(id);
    }
    const float count = modeid % 2 == 0 ? (float)down : (float)npts;
    double sum = 0;
    for (int id = 0; id < npts; id++) sum += per[(size_t)modeid * npts + id];
    float value = 0.f;
    if (count != 0) value = modeid <= 1 ? std::pow((float)sum / count, 1 / func_para) - 1 : (float)sum / count;
    scalars.push_back(count);
    scalars.push_back(value);
    std::vector<float> dc_acc(ncoef, 0.f);
    {
      float* dc_tmp = dc_acc.data();
      float* normal_dirction = dir.data();
      const float direction = dirsum > 0 ? 1.0f : -1.0f;
#include "surf_dss.inc"
      for (int id = 0; id < npts; id++) calc_node_value(id);
    }
    for (long i = 0; i < ncoef; i++) dcs[(size_t)modeid * ncoef + i] = count == 0 ? 0.f : dc_acc[i] * (1 / count);
  }
  std::vector<float> pts_out;
  pts_out.insert(pts_out.end(), nrm.begin(), nrm.end());
  pts_out.insert(pts_out.end(), dir.begin(), dir.end());
  pts_out.insert(pts_out.end(), flag.begin(), flag.end());
  pts_out.insert(pts_out.end(), per.begin(), per.end());
  save(a[14], pts_out);
  save(a[15], dcs);
  save(a[16], scalars);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string c = argv[1];
  if (c == "funcs" && argc == 9) return cmd_funcs(argv + 2);
  if (c == "proj" && argc == 10) return cmd_proj(argv + 2);
  if (c == "spline" && argc == 16) return cmd_spline(argv + 2);
  if (c == "filter" && argc == 10) return cmd_filter(argv + 2);
  if (c == "surface" && argc == 19) return cmd_surface(argv + 2);
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
