// Hierarchy and topology on the device: element/vertex masks of every level,
// fine-level node classes (surface / support / load), the reference's compact
// numbering (lexicographic ranks, GS-colour order padded to 32) and the
// load-node list.  All integer work, bit-exact with the reference rules.
#include "rso_internal.cuh"
#include <algorithm>
#include <cstring>

namespace rso {

// ---------------------------------------------------------------- kernels
__global__ void k_pad_emask(Level L, const uint8_t* dense, uint8_t* pad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.ne) return;
  int x = i % L.ex, y = (i / L.ex) % L.ey, z = i / ((long long)L.ex * L.ey);
  pad[L.eidx(x, y, z)] = dense[i] ? 1 : 0;
}

// fine-level node classes: active = touches an active element; surface =
// mark_surface_nodes_kernel (grid/Grid.cu:2824-2858); support = surface and
// in the fixed area; load = surface, in the load area, not support
// (grid/Grid.cpp:2715-2745).
__global__ void k_classify_fine(Level L, const uint8_t* fixed_area, const uint8_t* load_area) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  bool s[2][2][2];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    bool a = L.emask[L.eidx(x - 1 + k % 2, y - 1 + k / 2 % 2, z - 1 + k / 4)] != 0;
    s[k % 2][k / 2 % 2][k / 4] = a;
    any |= a;
  }
  uint8_t c = 0;
  if (any) {
    bool ax0 = false, ax1 = false, ax2 = false;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++) {
        ax0 |= s[0][a][b] && s[1][a][b];
        ax1 |= s[a][0][b] && s[a][1][b];
        ax2 |= s[a][b][0] && s[a][b][1];
      }
    bool surf = !ax0 || !ax1 || !ax2;
    c = NC_ACTIVE;
    if (surf) {
      c |= NC_SURFACE;
      if (fixed_area[i]) c |= NC_SUPPORT;
      else if (load_area[i]) c |= NC_LOAD;
    }
  }
  L.vclass[L.nidx(x, y, z)] = c;
}

__global__ void k_coarsen_emask(Level F, Level C, int factor) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= C.ne) return;
  int X = i % C.ex, Y = (i / C.ex) % C.ey, Z = i / ((long long)C.ex * C.ey);
  uint8_t a = 0;
  for (int dz = 0; dz < factor; dz++)
    for (int dy = 0; dy < factor; dy++)
      for (int dx = 0; dx < factor; dx++) {
        int x = X * factor + dx, y = Y * factor + dy, z = Z * factor + dz;
        if (x < F.ex && y < F.ey && z < F.ez) a |= F.emask[F.eidx(x, y, z)];
      }
  C.emask[C.eidx(X, Y, Z)] = a ? 1 : 0;
}

__global__ void k_vertex_active(Level L) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  uint8_t a = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) a |= L.emask[L.eidx(x - 1 + k % 2, y - 1 + k / 2 % 2, z - 1 + k / 4)];
  L.vclass[L.nidx(x, y, z)] = a ? NC_ACTIVE : 0;
}

__global__ void k_count_u8(const uint8_t* p, long long n, uint8_t mask, unsigned long long* out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned v = (i < n && (p[i] & mask)) ? 1u : 0u;
  unsigned b = __ballot_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(out, (unsigned long long)__popc(b));
}

__global__ void k_unpad_u8(const uint8_t* pad, long long n, int nx, int ny, int px, int py, uint8_t mask,
                           uint8_t* dense) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int x = i % nx, y = (i / nx) % ny, z = i / ((long long)nx * ny);
  long long j = (long long)(x + 1) + (long long)px * ((y + 1) + (long long)py * (z + 1));
  dense[i] = (pad[j] & mask) ? (mask == 0xff ? pad[j] : 1) : 0;
}

// Stable multi-key ranking.  Item i carries key[i] in [-1, K); rank[i] is
// the number of earlier items with the same key; totals[k] counts key k.
// Three passes: per-block counts, per-key scan of block counts, final ranks.
constexpr int RANK_BLOCK = 1024;

__global__ void k_rank_block_counts(const int8_t* key, long long n, int K, int* bcount) {
  __shared__ int cnt[16];
  if (threadIdx.x < 16) cnt[threadIdx.x] = 0;
  __syncthreads();
  long long i = blockIdx.x * (long long)RANK_BLOCK + threadIdx.x;
  int k = (i < n) ? key[i] : -1;
  for (int kk = 0; kk < K; kk++) {
    unsigned b = __ballot_sync(0xffffffffu, k == kk);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(&cnt[kk], __popc(b));
  }
  __syncthreads();
  if (threadIdx.x < K) bcount[(long long)threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void k_rank_scan(int* bcount, int nblocks, int K, long long* totals) {
  int k = threadIdx.x;
  if (k >= K) return;
  long long acc = 0;
  int* c = bcount + (long long)k * nblocks;
  for (int b = 0; b < nblocks; b++) {
    int v = c[b];
    c[b] = (int)acc;
    acc += v;
  }
  totals[k] = acc;
}

__global__ void k_rank_final(const int8_t* key, long long n, int K, const int* boff, int* rank) {
  __shared__ int wcnt[16][RANK_BLOCK / 32];
  long long i = blockIdx.x * (long long)RANK_BLOCK + threadIdx.x;
  int k = (i < n) ? key[i] : -1;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int my = 0;
  for (int kk = 0; kk < K; kk++) {
    unsigned b = __ballot_sync(0xffffffffu, k == kk);
    if (lane == 0) wcnt[kk][warp] = __popc(b);
    if (k == kk) my = __popc(b & ((1u << lane) - 1u));
  }
  __syncthreads();
  if (i >= n || k < 0) return;
  int before = 0;
  for (int w = 0; w < warp; w++) before += wcnt[k][w];
  rank[i] = boff[(long long)k * gridDim.x + blockIdx.x] + before + my;
}

// keys for the reference numbering: GS colour (x%2)+2(y%2)+4(z%2) of active items
__global__ void k_keys_colour(Level L, int elements, int8_t* key, int8_t* key_any) {
  long long n = elements ? L.ne : L.nn;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int ax = elements ? L.ex : L.nx, ay = elements ? L.ey : L.ny;
  int x = i % ax, y = (i / ax) % ay, z = i / ((long long)ax * ay);
  bool act = elements ? L.emask[L.eidx(x, y, z)] != 0 : (L.vclass[L.nidx(x, y, z)] & NC_ACTIVE) != 0;
  key[i] = act ? (int8_t)(x % 2 + 2 * (y % 2) + 4 * (z % 2)) : (int8_t)-1;
  key_any[i] = act ? 0 : -1;
}

// gs ids, lexicographic ids and flag words (grid/Grid.h:399-439)
__global__ void k_ref_numbering(Level L, int elements, int level0, const int8_t* key, const int* crank,
                                const int* lrank, const long long* coff, int* lexi2gs, int* flag_gs) {
  long long n = elements ? L.ne : L.nn;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = key[i];
  if (c < 0) return;
  int ax = elements ? L.ex : L.nx, ay = elements ? L.ey : L.ny;
  int x = i % ax, y = (i / ax) % ay, z = i / ((long long)ax * ay);
  long long gs = coff[c] + crank[i];
  if (lexi2gs) lexi2gs[lrank[i]] = (int)gs;
  if (flag_gs) {
    int w;
    if (elements) {
      w = c << 9;  // element position bits are never set by the reference (Grid.cpp:1063-1065)
    } else {
      w = (x % 8) | ((y % 8) << 3) | ((z % 8) << 6) | (c << 9);
      if (level0) {
        uint8_t cl = L.vclass[L.nidx(x, y, z)];
        if (cl & NC_SURFACE) w |= 1 << 13;
        if (cl & NC_LOAD) w |= 1 << 14;
        if (cl & NC_SUPPORT) w |= 1 << 19;
      }
    }
    flag_gs[gs] = w;
  }
}

__global__ void k_fill_i32(int* p, long long n, int v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// load-node list in reference order (GS id ascending = colour, then lexicographic)
__global__ void k_keys_load(Level L, int8_t* key) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  bool ld = (L.vclass[L.nidx(x, y, z)] & NC_LOAD) != 0;
  key[i] = ld ? (int8_t)(x % 2 + 2 * (y % 2) + 4 * (z % 2)) : (int8_t)-1;
}

__global__ void k_scatter_load(Level L, const int8_t* key, const int* rank, const long long* totals, int* out_dense,
                               int* out_pad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= L.nn) return;
  int c = key[i];
  if (c < 0) return;
  long long base = 0;
  for (int k = 0; k < c; k++) base += totals[k];
  long long pos = base + rank[i];
  int x = i % L.nx, y = (i / L.nx) % L.ny, z = i / ((long long)L.nx * L.ny);
  out_dense[pos] = (int)i;
  out_pad[pos] = (int)L.nidx(x, y, z);
}

// BitSAT rank over 32-bit words (gBitSAT::operator(), culib/lib.cuh:1474-1550)
__global__ void k_bits_to_keys(const uint32_t* words, long long nbits, int8_t* key) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nbits) return;
  key[i] = ((words[i >> 5] >> (i & 31)) & 1u) ? 0 : -1;
}
__global__ void k_rank_or_minus1(const int8_t* key, const int* rank, long long n, int* out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = key[i] >= 0 ? rank[i] : -1;
}

// ---------------------------------------------------------------- host helpers
static rso_status stable_rank(rso_handle* h, const int8_t* key, long long n, int K, int* rank, long long* totals_dev) {
  int nb = cdiv(n, RANK_BLOCK);
  int* bcount = nullptr;
  RSO_CHECK_CUDA(h, cudaMallocAsync(&bcount, sizeof(int) * (size_t)nb * K, h->stream));
  k_rank_block_counts<<<nb, RANK_BLOCK, 0, h->stream>>>(key, n, K, bcount); rso::note_launch();
  k_rank_scan<<<1, 32, 0, h->stream>>>(bcount, nb, K, totals_dev); rso::note_launch();
  k_rank_final<<<nb, RANK_BLOCK, 0, h->stream>>>(key, n, K, bcount, rank); rso::note_launch();
  RSO_TRY(launch_check(h, "stable_rank"));
  RSO_CHECK_CUDA(h, cudaFreeAsync(bcount, h->stream));
  return RSO_OK;
}

static rso_status count_mask(rso_handle* h, const uint8_t* p, long long n, uint8_t mask, long long* out) {
  unsigned long long* d = nullptr;
  RSO_CHECK_CUDA(h, cudaMallocAsync(&d, sizeof(unsigned long long), h->stream));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(d, 0, sizeof(unsigned long long), h->stream));
  k_count_u8<<<cdiv(n, 256), 256, 0, h->stream>>>(p, n, mask, d); rso::note_launch();
  RSO_TRY(launch_check(h, "count_mask"));
  unsigned long long v = 0;
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  RSO_CHECK_CUDA(h, cudaFreeAsync(d, h->stream));
  *out = (long long)v;
  return RSO_OK;
}

Level make_level(int ex, int ey, int ez, int factor) {
  Level l;
  l.ex = ex; l.ey = ey; l.ez = ez;
  l.nx = ex + 1; l.ny = ey + 1; l.nz = ez + 1;
  l.px = ((l.nx + 2 + 3) / 4) * 4; l.py = l.ny + 2; l.pz = l.nz + 2;
  l.qx = ((ex + 2 + 3) / 4) * 4; l.qy = ey + 2; l.qz = ez + 2;
  l.NP = (long long)l.px * l.py * l.pz;
  l.NQ = (long long)l.qx * l.qy * l.qz;
  l.nn = (long long)l.nx * l.ny * l.nz;
  l.ne = (long long)ex * ey * ez;
  l.factor = factor;
  return l;
}

static rso_status alloc_level_masks(rso_handle* h, Level& l) {
  RSO_CHECK_CUDA(h, cudaMalloc(&l.emask, l.NQ));
  RSO_CHECK_CUDA(h, cudaMalloc(&l.vclass, l.NP));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(l.emask, 0, l.NQ, h->stream));
  RSO_CHECK_CUDA(h, cudaMemsetAsync(l.vclass, 0, l.NP, h->stream));
  return RSO_OK;
}

static rso_status coarsen_level(rso_handle* h, const Level& f, int factor, Level& c) {
  c = make_level((f.ex + factor - 1) / factor, (f.ey + factor - 1) / factor, (f.ez + factor - 1) / factor, factor);
  RSO_TRY(alloc_level_masks(h, c));
  k_coarsen_emask<<<cdiv(c.ne, 256), 256, 0, h->stream>>>(f, c, factor); rso::note_launch();
  k_vertex_active<<<cdiv(c.nn, 256), 256, 0, h->stream>>>(c); rso::note_launch();
  RSO_TRY(launch_check(h, "coarsen"));
  RSO_TRY(count_mask(h, c.emask, c.NQ, 0xff, &c.n_active_e));
  RSO_TRY(count_mask(h, c.vclass, c.NP, NC_ACTIVE, &c.n_active_v));
  return RSO_OK;
}

static void free_level_masks(Level& l) {
  cudaFree(l.emask);
  cudaFree(l.vclass);
  l.emask = nullptr;
  l.vclass = nullptr;
}

static rso_status host_masks(rso_handle* h, int li) {
  const Level& l = h->L[li];
  std::vector<uint8_t>& hem = h->h_emask[li];
  std::vector<uint8_t>& hvm = h->h_vmask[li];
  uint8_t* d = nullptr;
  long long n = std::max(l.ne, l.nn);
  RSO_CHECK_CUDA(h, cudaMallocAsync(&d, n, h->stream));
  hem.resize(l.ne);
  hvm.resize(l.nn);
  k_unpad_u8<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l.emask, l.ne, l.ex, l.ey, l.qx, l.qy, 0xff, d); rso::note_launch();
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(hem.data(), d, l.ne, cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  k_unpad_u8<<<cdiv(l.nn, 256), 256, 0, h->stream>>>(l.vclass, l.nn, l.nx, l.ny, l.px, l.py, NC_ACTIVE, d); rso::note_launch();
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(hvm.data(), d, l.nn, cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  RSO_CHECK_CUDA(h, cudaFreeAsync(d, h->stream));
  return RSO_OK;
}

rso_status build_topology(rso_handle* h, const uint8_t* emask, const uint8_t* fixed_area, const uint8_t* load_area,
                          const double* load_normals) {
  Level& l0 = h->L[0];
  RSO_TRY(alloc_level_masks(h, l0));
  uint8_t *d_em = nullptr, *d_fa = nullptr, *d_la = nullptr;
  RSO_CHECK_CUDA(h, cudaMalloc(&d_em, l0.ne));
  RSO_CHECK_CUDA(h, cudaMalloc(&d_fa, l0.nn));
  RSO_CHECK_CUDA(h, cudaMalloc(&d_la, l0.nn));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(d_em, emask, l0.ne, cudaMemcpyHostToDevice, h->stream));
  if (fixed_area) RSO_CHECK_CUDA(h, cudaMemcpyAsync(d_fa, fixed_area, l0.nn, cudaMemcpyHostToDevice, h->stream));
  else RSO_CHECK_CUDA(h, cudaMemsetAsync(d_fa, 0, l0.nn, h->stream));
  if (load_area) RSO_CHECK_CUDA(h, cudaMemcpyAsync(d_la, load_area, l0.nn, cudaMemcpyHostToDevice, h->stream));
  else RSO_CHECK_CUDA(h, cudaMemsetAsync(d_la, 0, l0.nn, h->stream));
  k_pad_emask<<<cdiv(l0.ne, 256), 256, 0, h->stream>>>(l0, d_em, l0.emask); rso::note_launch();
  k_classify_fine<<<cdiv(l0.nn, 256), 256, 0, h->stream>>>(l0, d_fa, d_la); rso::note_launch();
  RSO_TRY(launch_check(h, "classify"));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaFree(d_em); cudaFree(d_fa); cudaFree(d_la);
  RSO_TRY(count_mask(h, l0.emask, l0.NQ, 0xff, &l0.n_active_e));
  RSO_TRY(count_mask(h, l0.vclass, l0.NP, NC_ACTIVE, &l0.n_active_v));
  if (l0.n_active_e == 0) { h->err = "no active element"; return RSO_ERR_INVALID_ARG; }

  // hierarchy (grid/Grid.cpp:1011-1034 policy, or an explicit level count)
  int ff = h->cfg.first_factor == 2 ? 2 : 4;
  if (h->cfg.n_levels > 0) {
    for (int i = 1; i < h->cfg.n_levels; i++) {
      Level c;
      RSO_TRY(coarsen_level(h, h->L.back(), i == 1 ? ff : 2, c));
      h->L.push_back(c);
    }
  } else {
    std::vector<Level> halves;
    halves.push_back(l0);
    while (halves.back().n_active_e > 400) {
      Level c;
      RSO_TRY(coarsen_level(h, halves.back(), 2, c));
      halves.push_back(c);
    }
    for (size_t i = 1; i < halves.size(); i++) {
      if (ff == 4 && i == 1) continue;
      if (ff == 4 && i == 2) {
        Level c;
        RSO_TRY(coarsen_level(h, h->L[0], 4, c));
        h->L.push_back(c);
      } else {
        halves[i].factor = 2;
        h->L.push_back(halves[i]);
        halves[i].emask = nullptr;  // ownership moved
        halves[i].vclass = nullptr;
      }
    }
    for (size_t i = 1; i < halves.size(); i++) free_level_masks(halves[i]);
    // keep at least one coarse level: the coarsest level is solved directly
    // from its stencil (the reference would be left with only a dummy layer)
    if (h->L.size() == 1) {
      Level c;
      RSO_TRY(coarsen_level(h, h->L[0], 2, c));
      h->L.push_back(c);
    }
  }
  h->h_emask.assign(h->L.size(), {});
  h->h_vmask.assign(h->L.size(), {});
  for (int li = 0; li < (int)h->L.size(); li++) RSO_TRY(host_masks(h, li));
  // h->L may have been reallocated by push_back: take the finest level afresh
  Level& lf = h->L[0];

  // load nodes in reference order
  int8_t* key = nullptr;
  int *rank = nullptr, *ld_dense = nullptr;
  long long* totals = nullptr;
  RSO_CHECK_CUDA(h, cudaMalloc(&key, lf.nn));
  RSO_CHECK_CUDA(h, cudaMalloc(&rank, sizeof(int) * lf.nn));
  RSO_CHECK_CUDA(h, cudaMalloc(&totals, sizeof(long long) * 16));
  k_keys_load<<<cdiv(lf.nn, 256), 256, 0, h->stream>>>(lf, key); rso::note_launch();
  RSO_TRY(stable_rank(h, key, lf.nn, 8, rank, totals));
  long long tot[8];
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  long long nl = 0;
  for (int k = 0; k < 8; k++) nl += tot[k];
  h->n_load = (int)nl;
  RSO_CHECK_CUDA(h, cudaMalloc(&ld_dense, sizeof(int) * std::max(nl, 1LL)));
  RSO_CHECK_CUDA(h, cudaMalloc(&h->load_nodes, sizeof(int) * std::max(nl, 1LL)));
  k_scatter_load<<<cdiv(lf.nn, 256), 256, 0, h->stream>>>(lf, key, rank, totals, ld_dense, h->load_nodes); rso::note_launch();
  RSO_TRY(launch_check(h, "load nodes"));
  h->h_load_nodes.resize(nl);
  if (nl) RSO_CHECK_CUDA(h, cudaMemcpyAsync(h->h_load_nodes.data(), ld_dense, sizeof(int) * nl, cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaFree(key); cudaFree(rank); cudaFree(totals); cudaFree(ld_dense);
  // load normals (one unit vector per load node)
  std::vector<double> nrm(3 * std::max(nl, 1LL), 0.0);
  if (load_normals)
    for (long long k = 0; k < nl; k++)
      for (int c = 0; c < 3; c++) nrm[3 * k + c] = load_normals[3 * (long long)h->h_load_nodes[k] + c];
  RSO_CHECK_CUDA(h, cudaMalloc(&h->load_normals, sizeof(double) * nrm.size()));
  RSO_CHECK_CUDA(h, cudaMemcpy(h->load_normals, nrm.data(), sizeof(double) * nrm.size(), cudaMemcpyHostToDevice));
  return RSO_OK;
}

}  // namespace rso

using namespace rso;

// reference compact numbering of one level
extern "C" rso_status rso_ref_numbering(rso_handle* h, int level, int* counts, int* gs_num, int* vlexi2gs,
                                        int* elexi2gs, int* vflag, int* eflag) {
  if (!h || level < 0 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  Level& l = h->L[level];
  long long tot_c[2][8];
  long long coff[2][8];
  long long ngs[2] = {0, 0};
  long long nact[2] = {0, 0};
  for (int el = 0; el < 2; el++) {
    long long n = el ? l.ne : l.nn;
    int8_t *key = nullptr, *key_any = nullptr;
    int *crank = nullptr, *lrank = nullptr, *lexi = nullptr, *flag = nullptr;
    long long *tot = nullptr, *tot_any = nullptr, *d_coff = nullptr;
    RSO_CHECK_CUDA(h, cudaMalloc(&key, n));
    RSO_CHECK_CUDA(h, cudaMalloc(&key_any, n));
    RSO_CHECK_CUDA(h, cudaMalloc(&crank, sizeof(int) * n));
    RSO_CHECK_CUDA(h, cudaMalloc(&lrank, sizeof(int) * n));
    RSO_CHECK_CUDA(h, cudaMalloc(&tot, sizeof(long long) * 16));
    RSO_CHECK_CUDA(h, cudaMalloc(&tot_any, sizeof(long long) * 16));
    RSO_CHECK_CUDA(h, cudaMalloc(&d_coff, sizeof(long long) * 8));
    k_keys_colour<<<cdiv(n, 256), 256, 0, h->stream>>>(l, el, key, key_any); rso::note_launch();
    RSO_TRY(stable_rank(h, key, n, 8, crank, tot));
    RSO_TRY(stable_rank(h, key_any, n, 1, lrank, tot_any));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(tot_c[el], tot, sizeof(long long) * 8, cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaMemcpyAsync(&nact[el], tot_any, sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    for (int c = 0; c < 8; c++) {
      coff[el][c] = ngs[el];
      ngs[el] += (tot_c[el][c] + 31) / 32 * 32;
    }
    int* want_lexi = el ? elexi2gs : vlexi2gs;
    int* want_flag = el ? eflag : vflag;
    if (want_lexi || want_flag) {
      RSO_CHECK_CUDA(h, cudaMalloc(&lexi, sizeof(int) * std::max(nact[el], 1LL)));
      RSO_CHECK_CUDA(h, cudaMalloc(&flag, sizeof(int) * std::max(ngs[el], 1LL)));
      k_fill_i32<<<cdiv(ngs[el], 256), 256, 0, h->stream>>>(flag, ngs[el], -1); rso::note_launch();
      RSO_CHECK_CUDA(h, cudaMemcpyAsync(d_coff, coff[el], sizeof(long long) * 8, cudaMemcpyHostToDevice, h->stream));
      k_ref_numbering<<<cdiv(n, 256), 256, 0, h->stream>>>(l, el, level == 0, key, crank, lrank, d_coff, lexi, flag); rso::note_launch();
      RSO_TRY(launch_check(h, "ref numbering"));
      if (want_lexi && nact[el])
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(want_lexi, lexi, sizeof(int) * nact[el], cudaMemcpyDeviceToHost, h->stream));
      if (want_flag && ngs[el])
        RSO_CHECK_CUDA(h, cudaMemcpyAsync(want_flag, flag, sizeof(int) * ngs[el], cudaMemcpyDeviceToHost, h->stream));
      RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    cudaFree(key); cudaFree(key_any); cudaFree(crank); cudaFree(lrank); cudaFree(tot); cudaFree(tot_any);
    cudaFree(d_coff); cudaFree(lexi); cudaFree(flag);
  }
  if (counts) { counts[0] = (int)nact[0]; counts[1] = (int)nact[1]; counts[2] = (int)ngs[0]; counts[3] = (int)ngs[1]; }
  if (gs_num) for (int c = 0; c < 8; c++) gs_num[c] = (int)((tot_c[0][c] + 31) / 32 * 32);
  if (level == 0) h->n_gs_elements = ngs[1];
  return RSO_OK;
}

extern "C" rso_status rso_bitsat_rank(rso_handle* h, const uint32_t* words, int64_t nbits, int32_t* rank_out) {
  if (!h || !words || !rank_out || nbits <= 0) return RSO_ERR_INVALID_ARG;
  int8_t* key = nullptr;
  int* rank = nullptr;
  long long* tot = nullptr;
  RSO_CHECK_CUDA(h, cudaMalloc(&key, nbits));
  RSO_CHECK_CUDA(h, cudaMalloc(&rank, sizeof(int) * nbits));
  RSO_CHECK_CUDA(h, cudaMalloc(&tot, sizeof(long long) * 16));
  k_bits_to_keys<<<cdiv(nbits, 256), 256, 0, h->stream>>>(words, nbits, key); rso::note_launch();
  RSO_TRY(stable_rank(h, key, nbits, 1, rank, tot));
  k_rank_or_minus1<<<cdiv(nbits, 256), 256, 0, h->stream>>>(key, rank, nbits, rank_out); rso::note_launch();
  RSO_TRY(launch_check(h, "bitsat rank"));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaFree(key); cudaFree(rank); cudaFree(tot);
  return RSO_OK;
}

extern "C" rso_status rso_level_masks(rso_handle* h, int level, uint8_t* em, uint8_t* vm) {
  if (!h || level < 0 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  Level& l = h->L[level];
  if (em) std::memcpy(em, h->h_emask[level].data(), l.ne);
  if (vm) std::memcpy(vm, h->h_vmask[level].data(), l.nn);
  return RSO_OK;
}

extern "C" rso_status rso_level_bitwords(rso_handle* h, int level, uint32_t* eb, uint32_t* vb) {
  if (!h || level < 0 || level >= (int)h->L.size()) return RSO_ERR_INVALID_ARG;
  Level& l = h->L[level];
  if (eb) {
    std::memset(eb, 0, sizeof(uint32_t) * ((l.ne + 31) / 32));
    const uint8_t* m = h->h_emask[level].data();
    for (long long i = 0; i < l.ne; i++) if (m[i]) eb[i >> 5] |= 1u << (i & 31);
  }
  if (vb) {
    std::memset(vb, 0, sizeof(uint32_t) * ((l.nn + 31) / 32));
    const uint8_t* m = h->h_vmask[level].data();
    for (long long i = 0; i < l.nn; i++) if (m[i]) vb[i >> 5] |= 1u << (i & 31);
  }
  return RSO_OK;
}

extern "C" rso_status rso_node_class(rso_handle* h, uint8_t* out) {
  if (!h || !out) return RSO_ERR_INVALID_ARG;
  Level& l = h->L[0];
  uint8_t* d = nullptr;
  RSO_CHECK_CUDA(h, cudaMalloc(&d, l.nn));
  k_unpad_u8<<<cdiv(l.nn, 256), 256, 0, h->stream>>>(l.vclass, l.nn, l.nx, l.ny, l.px, l.py, 0xff, d); rso::note_launch();
  RSO_TRY(launch_check(h, "node class"));
  RSO_CHECK_CUDA(h, cudaMemcpyAsync(out, d, l.nn, cudaMemcpyDeviceToHost, h->stream));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaFree(d);
  return RSO_OK;
}

extern "C" rso_status rso_load_nodes(rso_handle* h, int* nodes, int* n) {
  if (!h || !n) return RSO_ERR_INVALID_ARG;
  *n = h->n_load;
  if (nodes) std::memcpy(nodes, h->h_load_nodes.data(), sizeof(int) * h->n_load);
  return RSO_OK;
}
