// Sensitivity filter that allocates no device memory.
//
// rso_filter builds its table of filter taps (offset + weight) on the host
// and copies it into a device allocation owned by the handle, made on the
// first call and again whenever the radius grows.  Some
// callers cannot allow a device allocation inside their loop: an application
// that has handed all free device memory to its own pool up front (so any
// allocation outside that pool fails), one that must keep a fixed, known
// device footprint, or one that cannot accept the pool growth or the
// synchronisation an allocation may cause.  rso_filter_noalloc gives them
// the same filter with the tap table held in a fixed device array of this
// library, so no call makes an allocation, the first one included.
//
// The table holds the full cube of offsets |dx|,|dy|,|dz| <= reach, with a
// flag for the offsets inside the filter ball; reach = int(radius + 0.5) is
// limited to RSO_FILTER_NOALLOC_MAX_REACH (radius < 6.5), which bounds the
// array at 13^3 = 2197 taps of 24 bytes (52,728 bytes per device).
#include "rso_internal.cuh"

#include <mutex>

using namespace rso;

namespace {

constexpr int kMaxReach = RSO_FILTER_NOALLOC_MAX_REACH;
constexpr int kMaxSide = 2 * kMaxReach + 1;
constexpr int kMaxTaps = kMaxSide * kMaxSide * kMaxSide;
constexpr int kMaxDevices = 64;

struct Tap {
  double w;
  int dx, dy, dz, in_ball;
};
static_assert(sizeof(Tap) == 24, "tap layout");

// One table per device, shared by every call on that device.  A call writes
// every entry it reads (the side^3 cube of its own reach) before the filter
// kernel reads it, so nothing has to start at zero and the entries beyond
// the current reach, left from earlier calls, are never read.  Two calls
// that overlap on one device (two host threads, or two streams without an
// ordering between them) race on this table and must be serialised.
static __device__ __align__(256) Tap g_filter_taps[kMaxTaps];

std::mutex g_taps_mu;
Tap* g_taps_addr[kMaxDevices] = {};

// Device address of g_filter_taps on `device`, looked up once per device
// with that device current (the first call on a device may load the module
// there, which is why that first call belongs before any stream capture).
rso_status taps_address(rso_handle* h, Tap** out) {
  if (h->device < 0 || h->device >= kMaxDevices) {
    h->err = "rso_filter_noalloc: device ordinal out of range";
    return RSO_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_taps_mu);
  if (!g_taps_addr[h->device]) {
    int cur = -1;
    RSO_CHECK_CUDA(h, cudaGetDevice(&cur));
    if (cur != h->device) RSO_CHECK_CUDA(h, cudaSetDevice(h->device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_filter_taps);
    if (cur != h->device) RSO_CHECK_CUDA(h, cudaSetDevice(cur));
    if (e != cudaSuccess || !p) {
      h->err = std::string("rso_filter_noalloc: cudaGetSymbolAddress of the tap table: ") + cudaGetErrorString(e);
      return RSO_ERR_CUDA;
    }
    g_taps_addr[h->device] = static_cast<Tap*>(p);
  }
  *out = g_taps_addr[h->device];
  return RSO_OK;
}

// Tap (dx,dy,dz) at cube index ((dx+R)*side + dy+R)*side + dz+R, the same
// dx-major order, weight 1 - 6r^2 + 8r^3 - 3r^4 (r = |d|/radius) and
// rounding steps as the host-built table of rso_filter (operations written
// out so no contraction changes a weight).
__global__ void k_build_taps(Tap* __restrict__ taps, int reach, double radius) {
  const int side = 2 * reach + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= side * side * side) return;
  const int dx = i / (side * side) - reach, dy = (i / side) % side - reach, dz = i % side - reach;
  const double R2 = __dmul_rn(radius, radius);
  const double r2 = (double)(dx * dx + dy * dy + dz * dz);
  Tap t;
  t.dx = dx;
  t.dy = dy;
  t.dz = dz;
  t.in_ball = r2 <= R2;
  const double r = __dsqrt_rn(__ddiv_rn(r2, R2)), rr = __dmul_rn(r, r);
  double w = __dsub_rn(1.0, __dmul_rn(6.0, rr));
  w = __dadd_rn(w, __dmul_rn(__dmul_rn(8.0, rr), r));
  w = __dsub_rn(w, __dmul_rn(__dmul_rn(3.0, rr), rr));
  t.w = t.in_ball ? w : 0.0;
  taps[i] = t;
}

// out_e = sum_k w_k in_{e+d_k} / sum_k w_k over active neighbours inside the
// box; the taps are visited in table order, as in rso_filter.
__global__ void k_filter_taps(const Level L, const Tap* __restrict__ taps, int ntaps, const float* __restrict__ in,
                              float* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.ne) return;
  const int x = t % L.ex, y = (t / L.ex) % L.ey, z = t / ((long long)L.ex * L.ey);
  const long long e = L.eidx(x, y, z);
  if (!L.emask[e]) { out[e] = 0.f; return; }
  double gs = 0, ws = 0;
  for (int k = 0; k < ntaps; k++) {
    const Tap tp = taps[k];
    if (!tp.in_ball) continue;
    const int xx = x + tp.dx, yy = y + tp.dy, zz = z + tp.dz;
    if (xx < 0 || yy < 0 || zz < 0 || xx >= L.ex || yy >= L.ey || zz >= L.ez) continue;
    const long long n = L.eidx(xx, yy, zz);
    if (!L.emask[n]) continue;
    ws += tp.w;
    gs += tp.w * (double)in[n];
  }
  out[e] = (float)(gs / ws);
}

}  // namespace

extern "C" rso_status rso_filter_noalloc(rso_handle* h, double radius, const float* in, float* out) {
  if (!h || !in || !out || !(radius > 0)) return RSO_ERR_INVALID_ARG;
  if (!(radius < kMaxReach + 0.5)) {
    h->err = "rso_filter_noalloc: radius " + std::to_string(radius) + " reaches more than " +
             std::to_string(kMaxReach) + " elements; the fixed tap table allows radius < " +
             std::to_string(kMaxReach + 0.5) + " (use rso_filter for larger radii)";
    return RSO_ERR_INVALID_ARG;
  }
  const int reach = (int)(radius + 0.5);
  const int side = 2 * reach + 1, ntaps = side * side * side;
  Tap* taps = nullptr;
  RSO_TRY(taps_address(h, &taps));
  const Level& l = h->L[0];
  k_build_taps<<<cdiv(ntaps, 256), 256, 0, h->stream>>>(taps, reach, radius); rso::note_launch();
  RSO_TRY(launch_check(h, "filter_noalloc taps"));
  RSO_TRY(pad_elems_f(h, in, h->e_a));
  k_filter_taps<<<cdiv(l.ne, 256), 256, 0, h->stream>>>(l, taps, ntaps, h->e_a, h->e_b); rso::note_launch();
  RSO_TRY(launch_check(h, "filter_noalloc"));
  RSO_TRY(unpad_elems_f(h, h->e_b, out));
  RSO_CHECK_CUDA(h, cudaStreamSynchronize(h->stream));
  return RSO_OK;
}
