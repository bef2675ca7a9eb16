// Host side of libfoilb200.so: the C ABI declared in include/foilb200.h.
//
// A solver owns one device arena with the MAC state, its rollback copy, the cell-field
// planes, the pressure/Krylov vectors and the preconditioner tables. Each substep is one
// cooperative launch of fb::step_kernel; the host only plans substeps, handles retries
// and rollback (stable_fluids.py:332-603) and reads a small report once per call.

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/foilb200.h"
#include "fb_step.cuh"

using namespace fb;

namespace fb {
void *step_kernel_f64(int vpt, int r0);
void *step_kernel_f32r(int vpt, int r0);
void *step_kernel_f32m(int vpt, int r0);
void *step_kernel_batch_f32m();
}  // namespace fb

namespace {

thread_local std::string g_err;

int set_err(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

}  // namespace

namespace fb {
void set_last_error(const char *message) { g_err = message; }
}  // namespace fb

namespace {

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      return set_err(e_ == cudaErrorMemoryAllocation ? FB_ERR_OUT_OF_MEMORY : FB_ERR_CUDA,        \
                     "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    }                                                                                            \
  } while (0)

constexpr int kThreads = 512;
constexpr int kSplitCtas = 256;  // CTAs with spectrum scratch for split row transforms
constexpr unsigned long long kBarrierLimitNs = 2000000000ull;  // 2 s per barrier wait

double deg2rad(double a) { return a * (M_PI / 180.0); }

struct Layout {
  size_t N, NU, NV;
  int vsz, psz, csz;  // bytes of a field word, a Krylov word, a cell-plane word
  int pf, logp;
  size_t bytes;
  // offsets
  size_t u, v, u2, v2, uck, vck, cells, scal, scal2, scalck, solid, solidck;
  size_t b, x, r64, r, z, pa, pb, q, e, t;
  size_t chirp, filt, twp, tw2, mu, logmu, kappa, inv1m;
  size_t plane;  // bytes per cell plane
  size_t part, gs, rep, staging, count;
  size_t staging_bytes;
  // tensor-core row transforms (fb_umma.cuh): DST table, data operands, partial sums
  int tc, tc_nkb, tc_nrb, tc_nwb;
  size_t tab, a1, tc_bytes;
  // double-precision rows over 4096 points: the Bluestein convolution in two halves of
  // split_h points (pf is then the half convolution's length), spectrum scratch for
  // kSplitCtas CTAs
  int split_h;
  size_t spec;
};

size_t align_up(size_t a, size_t al) { return (a + al - 1) / al * al; }

// Whether the preconditioner's row transforms run on the tensor cores: the mixed scheme's DST
// preconditioner (no periodic axis), forced by FB_ROW_TRANSFORM_TENSOR, or under AUTO when the
// grid gives at least 64 work units (128 rows x 128 wavenumbers, one parity each): measured
// faster per step at 2048 x 1024 (128 units) and 4096 x 2048 (512 units); on smaller grids
// the units do not fill the SMs and the FFT spread over all of them wins.
bool tc_selected(const fb_scenario_desc *d) {
  if (d->pressure_scheme != FB_PRESSURE_MIXED || d->periodic_x || d->periodic_y) return false;
  if (d->row_transform == FB_ROW_TRANSFORM_FFT) return false;
  if (d->row_transform == FB_ROW_TRANSFORM_TENSOR) return true;
  const long long kh = (d->nx + 1) / 2;
  return 2 * ((d->ny + 127) / 128) * ((kh + 127) / 128) >= 64;
}

bool desc_valid(const fb_scenario_desc *d, std::string &why) {
  if (!d) { why = "null scenario"; return false; }
  if (d->nx < 4 || d->ny < 4) { why = "each resolution axis must contain at least four cells"; return false; }
  if ((long long)d->nx * d->ny > (1ll << 31) - 1) { why = "grid too large"; return false; }
  if (d->ny > 32768) { why = "at most 32768 cells along y"; return false; }
  if (!(std::isfinite(d->x0) && std::isfinite(d->x1) && d->x1 > d->x0 && std::isfinite(d->y0) &&
        std::isfinite(d->y1) && d->y1 > d->y0)) { why = "invalid bounds"; return false; }
  for (int i = 0; i < 4; ++i)
    if (d->naca[i] < '0' || d->naca[i] > '9') { why = "NACA code must contain exactly four digits"; return false; }
  if (!(d->chord > 0.0) || !std::isfinite(d->chord)) { why = "foil chord must be positive"; return false; }
  if (d->precision != FB_FLOAT32 && d->precision != FB_FLOAT64) { why = "precision"; return false; }
  if (d->pressure_scheme != FB_PRESSURE_REFERENCE && d->pressure_scheme != FB_PRESSURE_MIXED) { why = "scheme"; return false; }
  if (d->advection < FB_ADVECT_SEMI_LAGRANGIAN || d->advection > FB_ADVECT_SKEW_RK2) { why = "advection"; return false; }
  if (d->precision == FB_FLOAT64 && d->pressure_scheme == FB_PRESSURE_MIXED) {
    why = "the mixed pressure scheme is provided for float32 fields";
    return false;
  }
  if (!(d->pressure_tolerance > 0.0)) { why = "pressure_tolerance must be positive"; return false; }
  if (d->row_transform < FB_ROW_TRANSFORM_AUTO || d->row_transform > FB_ROW_TRANSFORM_TENSOR) {
    why = "row_transform";
    return false;
  }
  if (d->row_transform == FB_ROW_TRANSFORM_TENSOR &&
      (d->pressure_scheme != FB_PRESSURE_MIXED || d->periodic_x || d->periodic_y)) {
    why = "the tensor-core row transform serves the mixed scheme's DST preconditioner (no periodic axis)";
    return false;
  }
  if (d->pressure_max_iterations < 0) { why = "pressure_max_iterations must be >= 0"; return false; }
  return true;
}

Layout make_layout(const fb_scenario_desc *d) {
  Layout L{};
  L.N = (size_t)d->nx * d->ny;
  L.NU = (size_t)d->ny * (d->nx + 1);
  L.NV = (size_t)(d->ny + 1) * d->nx;
  L.vsz = d->precision == FB_FLOAT64 ? 8 : 4;
  L.psz = (d->pressure_scheme == FB_PRESSURE_MIXED) ? 4 : 8;
  int logp = 1;
  while ((1 << logp) < 2 * d->nx - 1) ++logp;
  // A double-precision convolution over 8192 points exceeds a CTA's shared memory: split it
  // (two halves of h = ceil(nx / 2) points; 2 h <= Pf / 2, so half the length suffices)
  if (L.psz == 8 && logp > 13) {
    L.split_h = (d->nx + 1) / 2;
    --logp;
  }
  L.logp = logp;
  L.pf = 1 << logp;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes, 256);
    return at;
  };
  L.u = take(L.NU * L.vsz);
  L.v = take(L.NV * L.vsz);
  L.u2 = take(L.NU * L.vsz);
  L.v2 = take(L.NV * L.vsz);
  L.uck = take(L.NU * L.vsz);
  L.vck = take(L.NV * L.vsz);
  // eight planes, each large enough for a face array (the face-centred and skew transports
  // use six of them as face temporaries)
  // cell planes hold the stencil type: FP64 for the mixed scheme on float32 fields
  L.csz = (d->precision == FB_FLOAT32 && d->pressure_scheme == FB_PRESSURE_MIXED) ? 8 : L.vsz;
  L.plane = align_up((L.N + (size_t)std::max(d->nx, d->ny) + 1) * L.csz, 256);
  L.cells = take(8 * L.plane);
  if (d->passive_scalar) {
    L.scal = take(L.N * L.vsz);
    L.scal2 = take(L.N * L.vsz);
    L.scalck = take(L.N * L.vsz);
  }
  L.solid = take(L.N);
  L.solidck = take(L.N);
  L.b = take(L.N * 8);
  L.x = take(L.N * 8);
  if (d->pressure_scheme == FB_PRESSURE_MIXED) L.r64 = take(L.N * 8);
  L.r = take(L.N * L.psz);
  L.z = take(L.N * L.psz);
  L.pa = take(L.N * L.psz);
  L.pb = take(L.N * L.psz);
  L.q = take(L.N * L.psz);
  if (d->pressure_scheme == FB_PRESSURE_MIXED) L.e = take(L.N * L.psz);
  L.t = take(L.N * L.psz);
  if (tc_selected(d)) {
    const int kh = (d->nx + 1) / 2;
    L.tc = 1;
    L.tc_nkb = (kh + 31) / 32;
    L.tc_nrb = (d->ny + 127) / 128;
    L.tc_nwb = (kh + 127) / 128;
    const size_t tile = (size_t)128 * 32 * 4;
    const size_t o0 = o;
    L.tab = take((size_t)L.tc_nwb * 2 * L.tc_nkb * tile);
    L.a1 = take((size_t)L.tc_nrb * 2 * L.tc_nkb * tile);  // both transforms' data operand
    L.tc_bytes = o - o0;
  }
  L.chirp = take((size_t)(d->nx + 1) * 2 * L.psz);
  L.filt = take((size_t)(L.split_h ? 3 : 1) * L.pf * 2 * L.psz);
  if (L.split_h) L.spec = take((size_t)kSplitCtas * 2 * L.pf * 2 * L.psz);
  L.twp = take((size_t)2 * L.pf * 2 * L.psz);  // per-pass twiddle tables (at most 2 Pf entries)
  L.tw2 = take((size_t)(128 + std::max(1, L.pf / 128)) * 2 * L.psz);  // two-level twiddles (long rows)
  L.mu = take((size_t)d->nx * 8);
  L.logmu = take((size_t)d->nx * 8);
  L.kappa = take((size_t)d->nx * 8);
  L.inv1m = take((size_t)d->nx * 8);
  L.part = take((size_t)SL_COUNT * 2048 * 8);
  L.gs = take(sizeof(GridSync));
  L.count = take(sizeof(unsigned long long));
  L.rep = take(sizeof(DevReport));
  // staging: interleaved cell velocity for import/export, and the diagnostics row partials
  // (8 doubles per row plus 8 results)
  L.staging_bytes = std::max({(size_t)L.N * 2 * L.vsz, (size_t)L.N * 8, ((size_t)d->ny * 8 + 8) * 8});
  L.staging = take(L.staging_bytes);
  L.bytes = o;
  return L;
}

// Surface forces on the solid body, per row (one CTA per row i): the fluid's kinematic
// pressure and viscous shear on every face between a fluid cell and a solid cell (periodic
// neighbours wrap). Pressure: the fluid cell's pressure times the face length, pushing into
// the solid. Shear: nu (t_fluid - t_wall) / (h / 2) times the face length along the face's
// tangent, with the fluid cell's centred velocity and the rigid wall velocity at the face.
// rows[4 i + k] = (Fx_pressure, Fy_pressure, Fx_viscous, Fy_viscous) of row i.
template <class V>
__global__ void forces_rows_kernel(const V *u, const V *v, const double *p, const unsigned char *solid, int nx, int ny,
                                   double dx, double dy, double x0, double y0, int perx, int pery, double omega,
                                   double px, double py, double nu, double *rows) {
  const int i = blockIdx.x;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < nx; j += blockDim.x) {
    const size_t idx = (size_t)i * nx + j;
    if (solid[idx]) continue;
    const double uf = 0.5 * ((double)u[(size_t)i * (nx + 1) + j] + (double)u[(size_t)i * (nx + 1) + j + 1]);
    const double vf = 0.5 * ((double)v[idx] + (double)v[(size_t)(i + 1) * nx + j]);
    const double pc = p[idx];
    const int jr = j + 1 < nx ? j + 1 : (perx ? 0 : -1), jl = j > 0 ? j - 1 : (perx ? nx - 1 : -1);
    const int iu = i + 1 < ny ? i + 1 : (pery ? 0 : -1), id = i > 0 ? i - 1 : (pery ? ny - 1 : -1);
    if (jr >= 0 && solid[(size_t)i * nx + jr]) {
      a[0] += pc * dy;
      const double vw = omega * ((x0 + (double)(j + 1) * dx) - px);
      a[3] += nu * (vf - vw) / (0.5 * dx) * dy;
    }
    if (jl >= 0 && solid[(size_t)i * nx + jl]) {
      a[0] -= pc * dy;
      const double vw = omega * ((x0 + (double)j * dx) - px);
      a[3] += nu * (vf - vw) / (0.5 * dx) * dy;
    }
    if (iu >= 0 && solid[(size_t)iu * nx + j]) {
      a[1] += pc * dx;
      const double uw = -omega * ((y0 + (double)(i + 1) * dy) - py);
      a[2] += nu * (uf - uw) / (0.5 * dy) * dx;
    }
    if (id >= 0 && solid[(size_t)id * nx + j]) {
      a[1] -= pc * dx;
      const double uw = -omega * ((y0 + (double)i * dy) - py);
      a[2] += nu * (uf - uw) / (0.5 * dy) * dx;
    }
  }
  __shared__ double red[32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  if (lane == 0)
    for (int k = 0; k < 4; ++k) red[warp][k] = a[k];
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w][threadIdx.x];
    rows[(size_t)4 * i + threadIdx.x] = t;
  }
}

// Fixed-order fold of the row partials: lane-strided sums, then a butterfly.
__global__ void forces_fold_kernel(const double *rows, int ny, double *out) {
  const int lane = threadIdx.x;
  for (int k = 0; k < 4; ++k) {
    double t = 0.0;
    for (int i = lane; i < ny; i += 32) t += rows[(size_t)4 * i + k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) out[k] = t;
  }
}

// Direct DFT of the Bluestein kernel conj(w_m), |m| < N, in natural frequency order, scaled
// by sqrt(2/L)/Pf (the DST normalisation and the inverse-FFT 1/Pf). Setup only.
__global__ void bluestein_filter_kernel(const double2 *chirp, int n, int pf, int logp, double scale, double2 *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= pf) return;
  double re = 0.0, im = 0.0;
  for (int m = -(n - 1); m <= n - 1; ++m) {
    const int j = m < 0 ? m + pf : m;
    const double2 w = chirp[m < 0 ? -m : m];
    // b_j = conj(w) ; e^{-2 pi i j k / pf}
    const long long jk = ((long long)j * k) % pf;
    double sn, cs;
    sincospi(2.0 * (double)jk / (double)pf, &sn, &cs);
    const double br = w.x, bi = -w.y;
    re += br * cs + bi * sn;
    im += bi * cs - br * sn;
  }
  (void)logp;
  out[k] = make_double2(re * scale, im * scale);
}

// Filter slices of the split convolution (dst_rows_split2): slice d in {-1, 0, 1} is the
// direct DFT of b_{d h + x} = conj(w_|d h + x|) (zero where |d h + x| >= N) at x mod pf for
// |x| < h, with bluestein_filter_kernel's scale; out[(d + 1) pf + k]. Setup only.
__global__ void bluestein_split_filter_kernel(const double2 *chirp, int n, int h, int pf, double scale, double2 *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = (int)blockIdx.y - 1;
  if (k >= pf) return;
  double re = 0.0, im = 0.0;
  for (int x = -(h - 1); x <= h - 1; ++x) {
    const int j = d * h + x, aj = j < 0 ? -j : j;
    if (aj >= n) continue;
    const double2 w = chirp[aj];
    const long long jk = ((long long)(x < 0 ? x + pf : x) * k) % pf;
    double sn, cs;
    sincospi(2.0 * (double)jk / (double)pf, &sn, &cs);
    const double br = w.x, bi = -w.y;
    re += br * cs + bi * sn;
    im += bi * cs - br * sn;
  }
  out[(size_t)(d + 1) * pf + k] = make_double2(re * scale, im * scale);
}

template <class T>
__global__ void convert_c2_kernel(const double2 *in, int n, T *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    out[2 * k] = (T)in[k].x;
    out[2 * k + 1] = (T)in[k].y;
  }
}

template <class V, class C>
__global__ void deinterleave_kernel(const V *in, size_t n, C *cx, C *cy) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    cx[i] = (C)in[2 * i];
    cy[i] = (C)in[2 * i + 1];
  }
}

template <class C, class V>
__global__ void interleave_kernel(const C *cx, const C *cy, size_t n, V *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    out[2 * i] = (V)cx[i];
    out[2 * i + 1] = (V)cy[i];
  }
}

// Cell velocity from faces (faces_to_cell, grid.py:25-29), interleaved (ny, nx, 2);
// solid cells zeroed when requested (export_state, stable_fluids.py:613-618).
// With `nonfinite` given, also counts the non-finite values written (one atomic per warp
// that saw any), so a caller can trust the exported array without scanning it again.
template <class V>
__global__ void export_cells_kernel(const V *u, const V *v, const unsigned char *solid, int nx, int ny, int zero_solids,
                                    V *out, unsigned long long *nonfinite = nullptr) {
  const size_t n = (size_t)nx * ny;
  unsigned bad = 0;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nx), j = (int)(idx - (size_t)i * nx);
    V a = (V)0.5 * (u[(size_t)i * (nx + 1) + j] + u[(size_t)i * (nx + 1) + j + 1]);
    V b = (V)0.5 * (v[(size_t)i * nx + j] + v[(size_t)(i + 1) * nx + j]);
    if (zero_solids && solid[idx]) a = b = V(0);
    out[2 * idx] = a;
    out[2 * idx + 1] = b;
    bad += (isfinite((double)a) ? 0u : 1u) + (isfinite((double)b) ? 0u : 1u);
  }
  if (nonfinite) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(nonfinite, (unsigned long long)bad);
  }
}

template <class V>
__global__ void sample_kernel(const V *u, const V *v, Axis ax, Axis ay, int nx, int ny, const double *pts, long long n,
                              double *out) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double gxv = (pts[2 * k] - ax.lo) / ax.h - 0.5, gyv = (pts[2 * k + 1] - ay.lo) / ay.h - 0.5;
  int ix0, ix1, iy0, iy1;
  double tx, ty;
  sample_coord(gxv, nx, ax.periodic, ix0, ix1, tx);
  sample_coord(gyv, ny, ay.periodic, iy0, iy1, ty);
  auto cval = [&](int comp, int i, int j) -> double {
    if (comp == 0) return (double)((V)0.5 * (u[(size_t)i * (nx + 1) + j] + u[(size_t)i * (nx + 1) + j + 1]));
    return (double)((V)0.5 * (v[(size_t)i * nx + j] + v[(size_t)(i + 1) * nx + j]));
  };
  for (int c = 0; c < 2; ++c) {
    const double a = cval(c, iy0, ix0), b = cval(c, iy0, ix1), cc = cval(c, iy1, ix0), d = cval(c, iy1, ix1);
    out[2 * k + c] = (double)(V)((1.0 - tx) * (1.0 - ty) * a + tx * (1.0 - ty) * b + (1.0 - tx) * ty * cc + tx * ty * d);
  }
}

__global__ void mask_kernel(Foil f, Axis ax, Axis ay, double c, double s, unsigned char *out) {
  const size_t n = (size_t)ax.n * ay.n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / ax.n), j = (int)(idx - (size_t)i * ax.n);
    out[idx] = naca_contains(f, c, s, lin_at(j, ax.n, ax.start, ax.step, ax.stop), lin_at(i, ay.n, ay.start, ay.step, ay.stop))
                   ? 1
                   : 0;
  }
}

__global__ void sdf_kernel(Foil f, double c, double s, const double *pts, long long n, double *out) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k < n) out[k] = naca_sdf(f, c, s, pts[2 * k], pts[2 * k + 1]);
}

// Diagnostics (stable_fluids.py:708-731, metrics.py:24-105): one CTA per row writes row
// partials; a single CTA folds them in row order.
template <class V>
__global__ void diag_rows_kernel(const V *u, const V *v, const unsigned char *solid, int nx, int ny, double dx, double dy,
                                 Axis ax, Axis ay, double omega, double px, double py, double wake_x, double recirc_x,
                                 double fsu, double *rows) {
  const int i = blockIdx.x;
  if (i >= ny) return;
  __shared__ double sh[8][32];
  double ke = 0, ens = 0, dv2 = 0, dlin = 0, leak = 0, wake = 0, rec = 0;
  auto cu = [&](int ii, int jj) -> double {
    return (double)((V)0.5 * (u[(size_t)ii * (nx + 1) + jj] + u[(size_t)ii * (nx + 1) + jj + 1]));
  };
  auto cv = [&](int ii, int jj) -> double { return (double)((V)0.5 * (v[(size_t)ii * nx + jj] + v[(size_t)(ii + 1) * nx + jj])); };
  auto ddy = [&](int comp, int jj) -> double {
    auto f = [&](int ii) { return comp == 0 ? cu(ii, jj) : cv(ii, jj); };
    if (i == 0) return (f(1) - f(0)) / dy;
    if (i == ny - 1) return (f(ny - 1) - f(ny - 2)) / dy;
    return (f(i + 1) - f(i - 1)) / (2.0 * dy);
  };
  auto ddx = [&](int comp, int jj) -> double {
    auto f = [&](int j2) { return comp == 0 ? cu(i, j2) : cv(i, j2); };
    if (jj == 0) return (f(1) - f(0)) / dx;
    if (jj == nx - 1) return (f(nx - 1) - f(nx - 2)) / dx;
    return (f(jj + 1) - f(jj - 1)) / (2.0 * dx);
  };
  const double wu = -omega * (lin_at(i, ny, ay.start, ay.step, ay.stop) - py);
  for (int j = threadIdx.x; j < nx; j += blockDim.x) {
    const double a = cu(i, j), b = cv(i, j);
    ke += a * a + b * b;
    const double w = ddx(1, j) - ddy(0, j);
    ens += w * w;
    const double dvv = ddx(0, j) + ddy(1, j);
    dv2 += dvv * dvv;
    const size_t idx = (size_t)i * nx + j;
    const double xc = lin_at(j, nx, ax.start, ax.step, ax.stop);
    if (!solid[idx]) {
      const V d = (u[(size_t)i * (nx + 1) + j + 1] - u[(size_t)i * (nx + 1) + j]) / (V)dx +
                  (v[(size_t)(i + 1) * nx + j] - v[(size_t)i * nx + j]) / (V)dy;
      dlin = fmax(dlin, fabs((double)d));
      if (xc > wake_x && fsu - a > 0.1 * fabs(fsu)) wake = 1.0;
      if (xc > recirc_x && a < 0.0) rec += 1.0;
    }
    if (j > 0 && solid[idx - 1] != solid[idx]) leak = fmax(leak, fabs((double)u[(size_t)i * (nx + 1) + j] - wu));
    if (i > 0 && solid[idx - nx] != solid[idx]) {
      const double wv = omega * (xc - px);
      leak = fmax(leak, fabs((double)v[(size_t)i * nx + j] - wv));
    }
  }
  double vals[7] = {ke, ens, dv2, dlin, leak, wake, rec};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 7; ++k) {
    double x = vals[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = (k == 3 || k == 4 || k == 5) ? fmax(x, y) : x + y;
    }
    if (lane == 0) sh[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < 7; ++k) {
      double x = sh[k][0];
      for (int w = 1; w < nw; ++w) x = (k == 3 || k == 4 || k == 5) ? fmax(x, sh[k][w]) : x + sh[k][w];
      rows[(size_t)i * 8 + k] = x;
    }
  }
}

__global__ void diag_fold_kernel(const double *rows, int nx, int ny, double dx, double dy, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < ny; ++i) {
    for (int k = 0; k < 7; ++k) {
      const double x = rows[(size_t)i * 8 + k];
      if (k == 3 || k == 4) s[k] = fmax(s[k], x);
      else s[k] += x;
    }
  }
  const double n = (double)nx * ny;
  out[0] = 0.5 * s[0] / n;
  out[1] = 0.5 * s[1] / n;
  out[2] = sqrt(s[2] / n);
  out[3] = s[3];
  out[4] = s[4];
  out[5] = s[5] * dy;
  out[6] = s[6] * dx * dy;
}

Axis make_axis(double lo, double hi, int n, int periodic) {
  Axis a{};
  a.lo = lo;
  a.hi = hi;
  a.h = (hi - lo) / n;
  a.ih = 1.0 / a.h;
  a.start = lo + 0.5 * a.h;
  a.stop = hi - 0.5 * a.h;
  a.step = (a.stop - a.start) / (double)(n - 1);
  a.n = n;
  a.periodic = periodic;
  return a;
}

Foil make_foil(const char naca[4], double chord, double px, double py) {
  Foil f{};
  f.m = (naca[0] - '0') / 100.0;
  f.p = (naca[1] - '0') / 10.0;
  f.t = ((naca[2] - '0') * 10 + (naca[3] - '0')) / 100.0;
  f.chord = chord;
  f.px = px;
  f.py = py;
  f.quarter = 0.25 * chord;
  f.thick_scale = 5.0 * f.t * chord;
  f.cambered = (f.m > 0.0 && f.p > 0.0) ? 1 : 0;
  if (f.cambered) {
    f.front_k = f.m / (f.p * f.p);
    f.back_k = f.m / ((1.0 - f.p) * (1.0 - f.p));
  }
  f.two_p = 2.0 * f.p;
  f.one_m_2p = 1.0 - 2.0 * f.p;
  return f;
}

double naca_max_radius(const Foil &f) {
  return std::hypot(0.75 * f.chord, (f.m + 0.51 * f.t) * f.chord);
}

}  // namespace

// =====================================================================================
struct fb_ctx {
  int device;
  uint64_t budget;
  uint64_t in_use;
  int sm_count;
  cudaStream_t stream;
};

struct fb_solver {
  fb_ctx *ctx;
  fb_scenario_desc d;
  Layout L;
  char *arena;
  DevReport *rep_host;
  unsigned long long *count_host;  // page-locked word for small device counters
  cudaEvent_t ev0, ev1;
  Axis ax, ay;
  Foil foil;
  int nblocks;
  size_t smem;
  FftPlan fft;
  int col_w;
  int tw_smem_off;
  int filt_smem_off, chirp_smem_off;  // -1: table read from global memory
  int tw2_smem_off;                   // two-level twiddles of the long-row path, -1 when unused
  void *kernel;
  unsigned long long *trace;
  int trace_cap;
  unsigned withhold = 0;                           // test hook of the grid barrier (0: off)
  int col_w_max = 16;                              // widest column tile that fits (configure_launch)
  int nblocks_max = 1;                             // co-resident CTAs of the cooperative launch
  double tuned_inner_rtol = 0.0;                   // autotuned mixed-scheme inner floor (0: default)
  unsigned long long limit_ns = kBarrierLimitNs;   // bound of every barrier wait
  int tc_on = 0;                                   // row transforms on the tensor cores (needs L.tc)
  int tc_stages = 4;                               // depth of the tensor-core operand ring
  // host-side state
  int initialized;
  double time, angle, omega, nu, cell_speed;
  double cg_per_substep;  // CG iterations per substep of the last accepted advance (batch weights)
  double skew_rate;       // staggered advection rate of the current faces (skew-RK2 planning)
  double batch_cost = 0.0;  // measured CTA-seconds per unit of expected work in batched launches (0: none yet)
  int launches;
  template <class T>
  T *at(size_t off) const {
    return reinterpret_cast<T *>(arena + off);
  }
};

namespace {

void fill_report_from_dev(const DevReport &r, fb_report *out) {
  if (!out) return;
  out->status = r.status == ST_OK ? FB_OK : (r.status == ST_TIMEOUT ? FB_ERR_DEVICE_TIMEOUT : FB_ERR_NUMERICAL);
  out->reason = r.reason;
  out->stage = r.stage;
  out->pressure_iterations = r.cg_iters;
  out->pressure_outer_iterations = r.cg_outer;
  out->pressure_converged = r.cg_converged;
  out->pressure_relative_residual = r.cg_rel;
  out->viscosity_iterations = r.visc_iters;
  out->viscosity_converged = r.visc_converged;
  out->viscosity_final_residual = r.visc_resid;
  out->max_speed = r.final_speed;
  out->divergence_linf = r.div_linf;
  out->solid_leakage = r.leakage;
  out->total_pressure_iterations = r.total_cg_iters;
  for (int i = 0; i < 6; ++i) out->evidence[i] = r.ev[i];
}

int grid_of(size_t n);

// Velocity in the host layout (ny, nx, 2) of the field type, in the staging area, to the first
// two cell planes (cell type), and the result planes 6, 7 back to the staging area.
void cells_from_staging(fb_solver *s, cudaStream_t st) {
  const Layout &L = s->L;
  const int g = grid_of(L.N);
  char *c0 = s->arena + L.cells, *c1 = c0 + L.plane;
  if (L.vsz == 8)
    deinterleave_kernel<double, double><<<g, 256, 0, st>>>(s->at<double>(L.staging), L.N, (double *)c0, (double *)c1);
  else if (L.csz == 8)
    deinterleave_kernel<float, double><<<g, 256, 0, st>>>(s->at<float>(L.staging), L.N, (double *)c0, (double *)c1);
  else
    deinterleave_kernel<float, float><<<g, 256, 0, st>>>(s->at<float>(L.staging), L.N, (float *)c0, (float *)c1);
}

void staging_from_result_cells(fb_solver *s, cudaStream_t st) {
  const Layout &L = s->L;
  const int g = grid_of(L.N);
  const char *c6 = s->arena + L.cells + 6 * L.plane, *c7 = c6 + L.plane;
  if (L.vsz == 8)
    interleave_kernel<double, double><<<g, 256, 0, st>>>((const double *)c6, (const double *)c7, L.N, s->at<double>(L.staging));
  else if (L.csz == 8)
    interleave_kernel<double, float><<<g, 256, 0, st>>>((const double *)c6, (const double *)c7, L.N, s->at<float>(L.staging));
  else
    interleave_kernel<float, float><<<g, 256, 0, st>>>((const float *)c6, (const float *)c7, L.N, s->at<float>(L.staging));
}

// Kernel parameters of one substep (or operator call) of solver s. `allow_tc` = false keeps the
// FFT row transforms (the batched launch, whose per-member shapes use the staged FFT path).
template <class V, class P>
StepParams<V, P> make_params(const fb_solver *s, unsigned phases, double dt, double angle_deg, double omega_deg,
                             double nu, double vtol, int vmaxit, bool allow_tc = true) {
  const fb_scenario_desc &d = s->d;
  const Layout &L = s->L;
  StepParams<V, P> p{};
  p.nx = d.nx;
  p.ny = d.ny;
  p.ax = s->ax;
  p.ay = s->ay;
  p.channel = d.channel_walls;
  p.fs_x = d.freestream_x;
  p.fs_y = d.freestream_y;
  p.foil = s->foil;
  p.phases = phases;
  p.initial_condition = d.initial_condition;
  p.maccormack = d.advection == FB_ADVECT_MACCORMACK;
  p.skew = d.advection == FB_ADVECT_SKEW_RK2;
  p.face_adv = d.face_advection != 0;
  p.dt = dt;
  const double a = deg2rad(angle_deg);
  p.cos_a = std::cos(a);
  p.sin_a = std::sin(a);
  p.omega = deg2rad(omega_deg);
  p.nu = nu;
  p.vtol = vtol;
  p.vmaxit = vmaxit;
  p.ptol = d.pressure_tolerance;
  p.pmaxit = d.pressure_max_iterations;
  p.pfixed = d.pressure_fixed_iterations;
  p.scheme = d.pressure_scheme == FB_PRESSURE_MIXED ? SCHEME_MIXED : SCHEME_REFERENCE;
  p.inner_floor = d.mixed_inner_rtol > 0.0 ? d.mixed_inner_rtol : (s->tuned_inner_rtol > 0.0 ? s->tuned_inner_rtol : 3.0e-6);
  // skew-RK2 caps the configured CFL at 0.4 (stable_fluids.py:264-266)
  p.proj_cfl_limit = std::max(1.0, 2.0 * (d.advection == FB_ADVECT_SKEW_RK2 ? std::min(d.cfl, 0.4) : d.cfl));
  p.singular = d.periodic_x && d.periodic_y;
  p.dst_precond = !(d.periodic_x || d.periodic_y);
  p.u = s->at<V>(L.u);
  p.v = s->at<V>(L.v);
  p.u2 = s->at<V>(L.u2);
  p.v2 = s->at<V>(L.v2);
  p.solid = s->at<unsigned char>(L.solid);
  const size_t plane = L.plane;
  using C = typename StencilArith<V, P>::type;
  C *cells[8];
  for (int i = 0; i < 8; ++i) cells[i] = reinterpret_cast<C *>(s->arena + L.cells + i * plane);
  p.cx = cells[0];
  p.cy = cells[1];
  p.fx = cells[2];
  p.fy = cells[3];
  p.gx = cells[4];
  p.gy = cells[5];
  p.hx = cells[6];
  p.hy = cells[7];
  if (d.passive_scalar) {
    p.scal = s->at<V>(L.scal);
    p.scal2 = s->at<V>(L.scal2);
  }
  p.b = s->at<double>(L.b);
  p.x = s->at<double>(L.x);
  p.r64 = d.pressure_scheme == FB_PRESSURE_MIXED ? s->at<double>(L.r64) : nullptr;
  p.r = s->at<P>(L.r);
  p.z = s->at<P>(L.z);
  p.pa = s->at<P>(L.pa);
  p.pb = s->at<P>(L.pb);
  p.q = s->at<P>(L.q);
  p.e = d.pressure_scheme == FB_PRESSURE_MIXED ? s->at<P>(L.e) : reinterpret_cast<P *>(p.x);
  p.t = s->at<P>(L.t);
  p.dst.chirp = s->at<Cx<P>>(L.chirp);
  p.dst.filt = s->at<Cx<P>>(L.filt);
  p.dst.twp = s->at<Cx<P>>(L.twp);
  p.dst.tw_lo = s->at<Cx<P>>(L.tw2);
  p.dst.tw_hi = s->at<Cx<P>>(L.tw2) + 128;
  p.dst.tw2_soff = s->tw2_smem_off;
  p.dst.split_h = L.split_h;
  p.dst.spec = L.split_h ? s->at<Cx<P>>(L.spec) : nullptr;
  p.dst.n = d.nx;
  p.dst.logp = L.logp;
  p.col.mu = s->at<double>(L.mu);
  p.col.logmu = s->at<double>(L.logmu);
  p.col.kappa = s->at<double>(L.kappa);
  p.col.inv1m = s->at<double>(L.inv1m);
  p.dy2 = s->ay.h * s->ay.h;
  p.fft = s->fft;
  p.tw_smem_off = s->tw_smem_off;
  p.filt_smem_off = s->filt_smem_off;
  p.chirp_smem_off = s->chirp_smem_off;
  if (L.tc && s->tc_on && allow_tc) {
    // the row transforms run on the tensor cores: no FFT tables in shared memory, whose
    // start holds the transform's operand ring
    p.um.tab = s->at<float>(L.tab);
    p.um.a1 = s->at<float>(L.a1);
    p.um.a2 = p.um.a1;  // the column solve writes the second operand over the first (dead by then)
    p.um.out1 = s->at<float>(L.t);  // y, accumulated into the FFT path's t buffer
    p.um.out2 = s->at<float>(L.z);  // z
    p.um.n = d.nx;
    p.um.kh = (d.nx + 1) / 2;
    p.um.nkb = L.tc_nkb;
    p.um.nrb = L.tc_nrb;
    p.um.nwb = L.tc_nwb;
    p.um.soff = 0;
    p.um.stages = s->tc_stages;
    {
      // the column solve's copy of y follows its tile and scan scratch when shared memory allows
      const size_t tile = align_up((size_t)(d.ny * s->col_w + kThreads / s->col_w) * 4, 16);
      p.um.ycopy_soff = 2 * tile + 64 * 8 <= s->smem ? (int)(tile + 64 * 8) : -1;
    }
    p.um.on = 1;
    p.tw_smem_off = p.filt_smem_off = p.chirp_smem_off = -1;
    p.dst.tw2_soff = -1;
    p.fft.io_soff = -1;
  }
  p.col_w = s->col_w;
  p.part = s->at<double>(L.part);
  p.gs = s->at<GridSync>(L.gs);
  p.rep = s->at<DevReport>(L.rep);
  p.limit_ns = s->limit_ns;
  p.withhold = s->withhold;
  p.trace = s->trace;
  p.trace_cap = s->trace_cap;
  return p;
}

template <class V, class P>
int launch_step(fb_solver *s, unsigned phases, double dt, double angle_deg, double omega_deg, double nu, double vtol,
                int vmaxit) {
  StepParams<V, P> p = make_params<V, P>(s, phases, dt, angle_deg, omega_deg, nu, vtol, vmaxit);
  void *args[] = {&p};
  // the grid barrier counts arrivals from zero in every launch (the abort flag stays sticky)
  CK(cudaMemsetAsync(&s->at<GridSync>(s->L.gs)->count, 0, sizeof(unsigned int), s->ctx->stream));
  CK(cudaLaunchCooperativeKernel(s->kernel, dim3(s->nblocks), dim3(kThreads), args, s->smem, s->ctx->stream));
  s->launches += 1;
  return FB_OK;
}

int launch(fb_solver *s, unsigned phases, double dt, double angle_deg, double omega_deg, double nu, double vtol,
           int vmaxit) {
  if (s->d.precision == FB_FLOAT64) return launch_step<double, double>(s, phases, dt, angle_deg, omega_deg, nu, vtol, vmaxit);
  if (s->d.pressure_scheme == FB_PRESSURE_MIXED)
    return launch_step<float, float>(s, phases, dt, angle_deg, omega_deg, nu, vtol, vmaxit);
  return launch_step<float, double>(s, phases, dt, angle_deg, omega_deg, nu, vtol, vmaxit);
}

int reset_report(fb_solver *s) {
  CK(cudaMemsetAsync(s->at<DevReport>(s->L.rep), 0, sizeof(DevReport), s->ctx->stream));
  CK(cudaMemsetAsync(s->at<GridSync>(s->L.gs), 0, sizeof(GridSync), s->ctx->stream));
  return FB_OK;
}

int read_report(fb_solver *s) {
  CK(cudaMemcpyAsync(s->rep_host, s->at<DevReport>(s->L.rep), sizeof(DevReport), cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  CK(cudaGetLastError());
  return FB_OK;
}

int checkpoint(fb_solver *s, bool restore) {
  const Layout &L = s->L;
  cudaStream_t st = s->ctx->stream;
  auto cp = [&](size_t dst, size_t src, size_t bytes) {
    return cudaMemcpyAsync(s->arena + dst, s->arena + src, bytes, cudaMemcpyDeviceToDevice, st);
  };
  if (!restore) {
    CK(cp(L.uck, L.u, L.NU * L.vsz));
    CK(cp(L.vck, L.v, L.NV * L.vsz));
    CK(cp(L.solidck, L.solid, L.N));
    if (s->d.passive_scalar) CK(cp(L.scalck, L.scal, L.N * L.vsz));
  } else {
    CK(cp(L.u, L.uck, L.NU * L.vsz));
    CK(cp(L.v, L.vck, L.NV * L.vsz));
    CK(cp(L.solid, L.solidck, L.N));
    if (s->d.passive_scalar) CK(cp(L.scal, L.scalck, L.N * L.vsz));
  }
  return FB_OK;
}

// Kernel selection per precision and row-transform shape (fb_kern_*.cu).
void *select_step_kernel(const fb_scenario_desc &d, const FftPlan &pl) {
  if (d.precision == FB_FLOAT64) return step_kernel_f64(pl.vpt, pl.radix[0]);
  if (d.pressure_scheme == FB_PRESSURE_MIXED) return step_kernel_f32m(pl.vpt, pl.radix[0]);
  return step_kernel_f32r(pl.vpt, pl.radix[0]);
}

int setup_tables(fb_solver *s) {
  const fb_scenario_desc &d = s->d;
  const Layout &L = s->L;
  const int n = d.nx, pf = L.pf;
  const double Lh = (double)(n + 1);
  // chirp w_m = exp(i pi m^2 / (2L)), reduced exactly modulo 4L
  std::vector<double> chirp(2 * (n + 1));
  const long long four_l = 4ll * (n + 1);
  for (int m = 0; m <= n; ++m) {
    const long long r = ((long long)m * m) % four_l;
    const double ang = M_PI * (double)r / (2.0 * Lh);
    chirp[2 * m] = std::cos(ang);
    chirp[2 * m + 1] = std::sin(ang);
  }
  // per-pass Stockham twiddles of the row FFT (layout fixed by the plan, independent of
  // the shared-memory budget)
  const size_t csz = 2 * (size_t)L.psz;
  const FftPlan plan = make_fft_plan(pf, L.logp, kThreads, 110 * 1024, csz);
  // two-level twiddles: lo[k] = W^k (k < 128), hi[k] = W^{128 k} (k < Pf / 128), W = exp(-2 pi i / Pf)
  {
    const int nhi = std::max(1, pf / 128);
    std::vector<double> t2(2 * (size_t)(128 + nhi));
    for (int k = 0; k < 128 + nhi; ++k) {
      const long long e = k < 128 ? k : (long long)128 * (k - 128);
      const double a = -2.0 * M_PI * (double)(e % pf) / (double)pf;
      t2[2 * k] = std::cos(a);
      t2[2 * k + 1] = std::sin(a);
    }
    double2 *dt2 = nullptr;
    CK(cudaMalloc(&dt2, sizeof(double2) * (128 + nhi)));
    CK(cudaMemcpy(dt2, t2.data(), sizeof(double2) * (128 + nhi), cudaMemcpyHostToDevice));
    if (L.psz == 8)
      CK(cudaMemcpyAsync(s->arena + L.tw2, dt2, sizeof(double2) * (128 + nhi), cudaMemcpyDeviceToDevice, s->ctx->stream));
    else
      convert_c2_kernel<float><<<(128 + nhi + 255) / 256, 256, 0, s->ctx->stream>>>(dt2, 128 + nhi, s->at<float>(L.tw2));
    CK(cudaStreamSynchronize(s->ctx->stream));
    cudaFree(dt2);
  }
  const int ntw = plan.tw_entries;
  std::vector<double> tw(2 * (size_t)ntw, 0.0);
  fft_pass_twiddles(plan, csz == 8 ? MainRadix<float>::value : MainRadix<double>::value, tw.data());
  double2 *dchirp = nullptr, *dfilt = nullptr, *dtw = nullptr;
  CK(cudaMalloc(&dchirp, sizeof(double2) * (n + 1)));
  const int nfilt = (L.split_h ? 3 : 1) * pf;
  CK(cudaMalloc(&dfilt, sizeof(double2) * nfilt));
  CK(cudaMalloc(&dtw, sizeof(double2) * ntw));
  CK(cudaMemcpy(dchirp, chirp.data(), sizeof(double2) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dtw, tw.data(), sizeof(double2) * ntw, cudaMemcpyHostToDevice));
  const double scale = std::sqrt(2.0 / Lh) / (double)pf;
  if (L.split_h)
    bluestein_split_filter_kernel<<<dim3((pf + 127) / 128, 3), 128, 0, s->ctx->stream>>>(dchirp, n, L.split_h, pf,
                                                                                       scale, dfilt);
  else
    bluestein_filter_kernel<<<(pf + 127) / 128, 128, 0, s->ctx->stream>>>(dchirp, n, pf, L.logp, scale, dfilt);
  CK(cudaGetLastError());
  if (L.psz == 8) {
    CK(cudaMemcpyAsync(s->arena + L.chirp, dchirp, sizeof(double2) * (n + 1), cudaMemcpyDeviceToDevice, s->ctx->stream));
    CK(cudaMemcpyAsync(s->arena + L.filt, dfilt, sizeof(double2) * nfilt, cudaMemcpyDeviceToDevice, s->ctx->stream));
    CK(cudaMemcpyAsync(s->arena + L.twp, dtw, sizeof(double2) * ntw, cudaMemcpyDeviceToDevice, s->ctx->stream));
  } else {
    convert_c2_kernel<float><<<(n + 1 + 255) / 256, 256, 0, s->ctx->stream>>>(dchirp, n + 1, s->at<float>(L.chirp));
    convert_c2_kernel<float><<<(pf + 255) / 256, 256, 0, s->ctx->stream>>>(dfilt, pf, s->at<float>(L.filt));
    convert_c2_kernel<float><<<(ntw + 255) / 256, 256, 0, s->ctx->stream>>>(dtw, ntw, s->at<float>(L.twp));
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s->ctx->stream));
  cudaFree(dchirp);
  cudaFree(dfilt);
  cudaFree(dtw);
  // column constants of the tridiagonal solve (see fb_dst.cuh)
  std::vector<double> mu(n), lmu(n), kap(n), i1m(n);
  const double dx = s->ax.h, dy = s->ay.h;
  const int ny = d.ny;
  for (int k = 0; k < n; ++k) {
    const double lam = 2.0 * (1.0 - std::cos(M_PI * (double)(k + 1) / (double)(n + 1))) * (1.0 / (dx * dx));
    const double e = lam * dy * dy;
    const double sq = std::sqrt(e * (e + 4.0));
    const double m = 2.0 / (2.0 + e + sq);
    const double one_m = (e + sq) / (2.0 + e + sq);
    const double lg = std::log1p(-one_m);
    const double one_m2 = one_m * (1.0 + m);
    const double h0 = -std::expm1(2.0 * ny * lg) / one_m2;
    mu[k] = m;
    lmu[k] = lg;
    kap[k] = m * m / (1.0 + m * m * h0);
    i1m[k] = 1.0 / one_m2;
  }
  CK(cudaMemcpy(s->arena + L.mu, mu.data(), 8 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->arena + L.logmu, lmu.data(), 8 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->arena + L.kappa, kap.data(), 8 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->arena + L.inv1m, i1m.data(), 8 * n, cudaMemcpyHostToDevice));
  if (L.tc) {
    // DST table of the tensor-core transform: S[nn][k] = sqrt(2/L) sin(pi nn k / L) (argument
    // reduced exactly modulo 2L), rounded to TF32 (nearest, ties away); zero past Kh and N.
    // The operands' padding is zeroed once here and never written afterwards.
    const int kh = (n + 1) / 2, nkb = L.tc_nkb;
    std::vector<float> tab((size_t)L.tc_nwb * 2 * nkb * 128 * 32, 0.0f);
    const double c = std::sqrt(2.0 / Lh);
    const long long two_l = 2ll * (n + 1);
    auto tf32 = [](double v) {
      float f = (float)v;
      uint32_t b;
      std::memcpy(&b, &f, 4);
      b = (b + 0x1000u) & 0xFFFFE000u;
      std::memcpy(&f, &b, 4);
      return f;
    };
    for (int k = 1; k <= kh; ++k)
      for (int p = 0; p < 2; ++p)
        for (int i = 0; i < nkb * 32; ++i) {
          const long long nn = 2ll * i + 1 + p;
          if (nn > n) break;
          const long long r = (nn * k) % two_l;
          tab[umma_index(nkb, k - 1, p, i)] = tf32(c * std::sin(M_PI * (double)r / Lh));
        }
    CK(cudaMemset(s->arena + L.tab, 0, L.tc_bytes));
    CK(cudaMemcpy(s->arena + L.tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice));
  }
  return FB_OK;
}

// ---- autotuner cache ---------------------------------------------------------------------------
// Launch shapes (column tile width, CTA count) and the mixed scheme's inner sweep floor that
// fb_autotune measured fastest, per grid, precision, scheme, transport, periodicity and device;
// solvers created later with the same key start from them.
struct TuneKey {
  int nx, ny, precision, scheme, transport, periodic, device;
  bool operator<(const TuneKey &o) const {
    return std::tie(nx, ny, precision, scheme, transport, periodic, device) <
           std::tie(o.nx, o.ny, o.precision, o.scheme, o.transport, o.periodic, o.device);
  }
};
struct TuneChoice {
  int col_w, nblocks;
  double inner_rtol;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune;

TuneKey tune_key(const fb_solver *s) {
  const fb_scenario_desc &d = s->d;
  return TuneKey{d.nx, d.ny, d.precision, d.pressure_scheme, d.advection * 2 + (d.face_advection ? 1 : 0),
                 d.periodic_x * 2 + d.periodic_y, s->ctx->device};
}

void apply_cached_tuning(fb_solver *s) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(tune_key(s));
  if (it == g_tune.end()) return;
  if (it->second.col_w <= s->col_w_max) s->col_w = it->second.col_w;
  if (it->second.nblocks <= s->nblocks_max) s->nblocks = it->second.nblocks;
  s->tuned_inner_rtol = it->second.inner_rtol;
}

int configure_launch(fb_solver *s) {
  const fb_scenario_desc &d = s->d;
  const Layout &L = s->L;
  const size_t csz = 2 * (size_t)L.psz;
  const size_t row_bytes = (size_t)fft_pad(L.pf) * csz;
  size_t budget = 110 * 1024;
  if (row_bytes > budget) budget = row_bytes;
  s->fft = make_fft_plan(L.pf, L.logp, kThreads, budget, csz);
  if (s->fft.tr > kThreads) return set_err(FB_ERR_INVALID_ARGUMENT, "row transform of %d points is too long", L.pf);
  size_t rows_smem = (size_t)s->fft.rows * row_bytes;
  // column tiles of the tridiagonal solve: W in {16, 8, 4, 2} columns (see fb_dst.cuh)
  int W = 16;
  auto col_bytes = [&](int w) {
    const int S = kThreads / w;
    return align_up((size_t)(d.ny * w + S) * L.psz, 16) + (size_t)64 * 8;
  };
  while (W > 2 && col_bytes(W) > std::max(budget, rows_smem)) W >>= 1;
  const size_t cbytes = col_bytes(W);
  // Fast layout: row buffers, then per-row-slot staging buffers for the bulk copies (two
  // halves of an input row plus its mask), overlapping the column tile; then shared copies
  // of the transform tables. It needs the three-pass transform shape, rows of whole 16-byte
  // units (nx % 16 == 0), at most 16 row slots (32 mbarriers) and room for everything;
  // otherwise the transform reads its inputs and tables from global memory.
  const size_t kSmemMax = 227 * 1024 - 4 * 1024;  // leave room for the static reductions
  const size_t tab_bytes = align_up((size_t)s->fft.tw_entries * csz, 16) + align_up((size_t)L.pf * csz, 16) +
                           align_up((size_t)(d.nx + 1) * csz, 16);
  const size_t io_slot = align_up(2 * ((size_t)d.nx * L.psz + (size_t)d.nx), 16);
  const size_t work_fast = std::max(align_up(rows_smem, 16) + (size_t)s->fft.rows * io_slot, cbytes);
  s->tw_smem_off = s->filt_smem_off = s->chirp_smem_off = -1;
  s->tw2_smem_off = -1;
  s->fft.io_soff = -1;
  s->fft.io_slot = 0;
  size_t smem;
  const bool fixed_shape = s->fft.npass == 3 && s->fft.rows * s->fft.tr == kThreads;  // dst_rows_body3
  if (fixed_shape && d.nx % 16 == 0 && s->fft.rows <= 16 && align_up(work_fast, 16) + tab_bytes <= kSmemMax) {
    s->fft.io_soff = (int)align_up(rows_smem, 16);
    s->fft.io_slot = (int)io_slot;
    smem = align_up(work_fast, 16);
    s->tw_smem_off = (int)smem;
    smem += align_up((size_t)s->fft.tw_entries * csz, 16);
    s->filt_smem_off = (int)smem;
    smem += align_up((size_t)L.pf * csz, 16);
    s->chirp_smem_off = (int)smem;
    smem += align_up((size_t)(d.nx + 1) * csz, 16);
  } else if (s->fft.npass == 4 && s->fft.rows * s->fft.tr == kThreads && d.nx % 16 == 0 && s->fft.rows <= 16 &&
             L.pf >= 128 && align_up(work_fast, 16) + align_up((size_t)(128 + L.pf / 128) * csz, 16) <= kSmemMax) {
    // long rows (dst_rows_body4): staged inputs, two-level twiddles in shared memory, filter
    // and chirp read through the cache
    s->fft.io_soff = (int)align_up(rows_smem, 16);
    s->fft.io_slot = (int)io_slot;
    smem = align_up(work_fast, 16);
    s->tw2_smem_off = (int)smem;
    smem += align_up((size_t)(128 + L.pf / 128) * csz, 16);
  } else {
    smem = align_up(std::max(rows_smem, cbytes), 16);
  }
  // the tensor-core row transform's operand ring (fb_umma.cuh) starts at offset 0
  if (s->L.tc) smem = std::max(smem, (size_t)umma_smem_bytes(s->tc_stages));
  if (smem > kSmemMax) return set_err(FB_ERR_INVALID_ARGUMENT, "grid needs %zu bytes of shared memory per CTA", smem);
  s->col_w = W;
  s->smem = smem;
  s->kernel = select_step_kernel(d, s->fft);
  if (!s->kernel)
    return set_err(FB_ERR_INVALID_ARGUMENT, "no step kernel for a %d-point row transform in this precision", L.pf);
  CK(cudaFuncSetAttribute(s->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s->kernel, kThreads, smem));
  if (occ < 1) return set_err(FB_ERR_CUDA, "step kernel cannot be resident (smem %zu)", smem);
  // two cells per thread at least, and at least one CTA per transformed row, so that the row
  // transforms of small grids spread over the SMs (one row slot per CTA runs fastest)
  const long long want = std::max<long long>(std::max<long long>(1, (long long)((L.N + 2 * kThreads - 1) / (2 * kThreads))),
                                             (long long)d.ny);
  s->nblocks = (int)std::min<long long>((long long)occ * s->ctx->sm_count, want);
  s->nblocks = std::min(s->nblocks, 2048);
  if (L.split_h) {
    // split rows: one row per CTA, spectrum scratch for kSplitCtas CTAs
    if (s->fft.rows != 1 || s->fft.tr != kThreads)
      return set_err(FB_ERR_INVALID_ARGUMENT, "no split row transform for a %d-point convolution", L.pf);
    s->nblocks = std::min(s->nblocks, kSplitCtas);
  }
  s->col_w_max = W;
  s->nblocks_max = s->nblocks;
  apply_cached_tuning(s);
  return FB_OK;
}

bool report_ok(const DevReport &r) { return r.status == ST_OK; }

int numerical_status(fb_solver *s, fb_report *out) {
  fill_report_from_dev(*s->rep_host, out);
  if (s->rep_host->status == ST_TIMEOUT) return set_err(FB_ERR_DEVICE_TIMEOUT, "device barrier wait timed out");
  return set_err(FB_ERR_NUMERICAL, "numerical failure reason=%d stage=%d", s->rep_host->reason, s->rep_host->stage);
}

int full_projection(fb_solver *s, unsigned phases, double dt, double angle, double omega, fb_report *out) {
  int rc = reset_report(s);
  if (rc) return rc;
  rc = launch(s, phases | PH_GUARD | PH_PROJECT | PH_FINALIZE, dt, angle, omega, s->nu, 0.0, 0);
  if (rc) return rc;
  rc = read_report(s);
  if (rc) return rc;
  if (!report_ok(*s->rep_host)) return numerical_status(s, out);
  fill_report_from_dev(*s->rep_host, out);
  s->cell_speed = s->rep_host->final_speed;
  s->skew_rate = s->rep_host->skew_rate;
  return FB_OK;
}

}  // namespace

namespace fb {
// The device report's status mapping, shared with the allocation-free entry point.
void fill_report(const DevReport &r, fb_report *out) { fill_report_from_dev(r, out); }
}  // namespace fb

// =====================================================================================
extern "C" {

int32_t fb_abi_version(void) { return FB_ABI_VERSION; }

int32_t fb_abi_struct_sizes(uint64_t *desc_bytes, uint64_t *report_bytes) {
  if (desc_bytes) *desc_bytes = sizeof(fb_scenario_desc);
  if (report_bytes) *report_bytes = sizeof(fb_report);
  return FB_OK;
}

const char *fb_last_error(void) { return g_err.c_str(); }

int32_t fb_device_count(int32_t *count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    if (count) *count = 0;
    return set_err(FB_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  if (count) *count = n;
  return FB_OK;
}

int32_t fb_ctx_create(int32_t device, uint64_t hbm_budget, fb_ctx **out) {
  if (!out) return set_err(FB_ERR_INVALID_ARGUMENT, "null out");
  *out = nullptr;
  int n = 0;
  CK(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return set_err(FB_ERR_INVALID_ARGUMENT, "device %d out of range (%d)", device, n);
  CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (!prop.cooperativeLaunch) return set_err(FB_ERR_CUDA, "device lacks cooperative launch");
  fb_ctx *c = new (std::nothrow) fb_ctx();
  if (!c) return set_err(FB_ERR_OUT_OF_MEMORY, "host allocation");
  c->device = device;
  c->budget = hbm_budget;
  c->in_use = 0;
  c->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return set_err(FB_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  }
  *out = c;
  return FB_OK;
}

int32_t fb_ctx_destroy(fb_ctx *ctx) {
  if (!ctx) return FB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return FB_OK;
}

int32_t fb_ctx_bytes_in_use(fb_ctx *ctx, uint64_t *bytes) {
  if (!ctx || !bytes) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = ctx->in_use;
  return FB_OK;
}

namespace {
// Page-locked host pool: blocks by size (portable, so any device can copy into them), reused
// after fb_host_free, the most recently freed first; the held total (in use + cached) stays
// under FB_HOST_POOL_BYTES.
struct HostPool {
  std::mutex mu;
  std::multimap<uint64_t, void *> free_blocks;
  std::map<void *, uint64_t> live;
  uint64_t held = 0;
};
HostPool &host_pool() {
  static HostPool *pool = new HostPool();  // never destroyed: blocks may be freed at exit
  return *pool;
}
}  // namespace

int32_t fb_host_alloc(uint64_t bytes, void **out) {
  if (!out || bytes == 0) return set_err(FB_ERR_INVALID_ARGUMENT, "fb_host_alloc: null output or zero size");
  HostPool &hp = host_pool();
  std::lock_guard<std::mutex> lock(hp.mu);
  auto range = hp.free_blocks.equal_range(bytes);
  if (range.first != range.second) {
    auto it = std::prev(range.second);  // the most recently freed block of this size
    *out = it->second;
    hp.free_blocks.erase(it);
    hp.live[*out] = bytes;
    return FB_OK;
  }
  // make room by releasing cached blocks of other sizes
  while (hp.held + bytes > FB_HOST_POOL_BYTES && !hp.free_blocks.empty()) {
    auto f = hp.free_blocks.begin();
    cudaFreeHost(f->second);
    hp.held -= f->first;
    hp.free_blocks.erase(f);
  }
  if (hp.held + bytes > FB_HOST_POOL_BYTES) return set_err(FB_ERR_BUDGET, "host pool full");
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return set_err(FB_ERR_OUT_OF_MEMORY, "cudaHostAlloc %llu bytes", (unsigned long long)bytes);
  }
  hp.held += bytes;
  hp.live[p] = bytes;
  *out = p;
  return FB_OK;
}

int32_t fb_host_free(void *p) {
  if (!p) return FB_OK;
  HostPool &hp = host_pool();
  std::lock_guard<std::mutex> lock(hp.mu);
  auto it = hp.live.find(p);
  if (it == hp.live.end()) return set_err(FB_ERR_INVALID_ARGUMENT, "fb_host_free: not a pool block");
  hp.free_blocks.emplace(it->second, p);
  hp.live.erase(it);
  return FB_OK;
}

int32_t fb_solver_bytes(const fb_scenario_desc *desc, uint64_t *bytes) {
  std::string why;
  if (!desc_valid(desc, why)) return set_err(FB_ERR_INVALID_ARGUMENT, "%s", why.c_str());
  if (bytes) *bytes = make_layout(desc).bytes;
  return FB_OK;
}

int32_t fb_solver_create(fb_ctx *ctx, const fb_scenario_desc *desc, fb_solver **out) {
  if (!ctx || !out) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  std::string why;
  if (!desc_valid(desc, why)) return set_err(FB_ERR_INVALID_ARGUMENT, "%s", why.c_str());
  CK(cudaSetDevice(ctx->device));
  Layout L = make_layout(desc);
  if (ctx->budget && ctx->in_use + L.bytes > ctx->budget)
    return set_err(FB_ERR_BUDGET, "solver needs %zu bytes; %llu of %llu in use", L.bytes,
                   (unsigned long long)ctx->in_use, (unsigned long long)ctx->budget);
  fb_solver *s = new (std::nothrow) fb_solver();
  if (!s) return set_err(FB_ERR_OUT_OF_MEMORY, "host allocation");
  s->ctx = ctx;
  s->d = *desc;
  s->L = L;
  s->ax = make_axis(desc->x0, desc->x1, desc->nx, desc->periodic_x);
  s->ay = make_axis(desc->y0, desc->y1, desc->ny, desc->periodic_y);
  s->foil = make_foil(desc->naca, desc->chord, desc->pivot_x, desc->pivot_y);
  cudaError_t e = cudaMalloc(&s->arena, L.bytes);
  if (e != cudaSuccess) {
    delete s;
    return set_err(FB_ERR_OUT_OF_MEMORY, "cudaMalloc %zu bytes: %s", L.bytes, cudaGetErrorString(e));
  }
  // one page-locked block: the device report, then the counter word
  const size_t rep_bytes = (sizeof(DevReport) + 15) / 16 * 16;
  e = cudaMallocHost(&s->rep_host, rep_bytes + 16);
  if (e != cudaSuccess) {
    cudaFree(s->arena);
    delete s;
    return set_err(FB_ERR_OUT_OF_MEMORY, "pinned report: %s", cudaGetErrorString(e));
  }
  s->count_host = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(s->rep_host) + rep_bytes);
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  ctx->in_use += L.bytes;
  int rc = cudaMemsetAsync(s->arena, 0, L.bytes, ctx->stream) == cudaSuccess ? FB_OK : FB_ERR_CUDA;
  if (!rc) rc = setup_tables(s);
  s->tc_on = s->L.tc;
  if (!rc) rc = configure_launch(s);
  if (rc) {
    fb_solver_destroy(s);
    return rc;
  }
  *out = s;
  return FB_OK;
}

int32_t fb_solver_destroy(fb_solver *s) {
  if (!s) return FB_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  if (s->arena) cudaFree(s->arena);
  if (s->trace) cudaFree(s->trace);
  if (s->rep_host) cudaFreeHost(s->rep_host);
  cudaEventDestroy(s->ev0);
  cudaEventDestroy(s->ev1);
  s->ctx->in_use -= s->L.bytes;
  delete s;
  return FB_OK;
}

int32_t fb_set_viscosity(fb_solver *s, double viscosity) {
  if (!s) return set_err(FB_ERR_INVALID_ARGUMENT, "null solver");
  if (!std::isfinite(viscosity) || viscosity < 0.0) return set_err(FB_ERR_INVALID_ARGUMENT, "viscosity");
  s->nu = viscosity;
  return FB_OK;
}

int32_t fb_initialize(fb_solver *s, double angle0_degrees, double reynolds, double project_dt, fb_report *out) {
  if (!s) return set_err(FB_ERR_INVALID_ARGUMENT, "null solver");
  if (!(reynolds > 0.0) || !std::isfinite(angle0_degrees) || !(project_dt > 0.0))
    return set_err(FB_ERR_INVALID_ARGUMENT, "invalid initialize arguments");
  CK(cudaSetDevice(s->ctx->device));
  if (out) std::memset(out, 0, sizeof(*out));
  s->initialized = 0;
  s->time = 0.0;
  s->angle = angle0_degrees;
  s->omega = 0.0;
  s->nu = s->d.reference_speed * s->d.chord / reynolds;
  s->launches = 0;
  CK(cudaEventRecord(s->ev0, s->ctx->stream));
  int rc = full_projection(s, PH_IC | PH_MASK | PH_FROM_CELLS, project_dt, angle0_degrees, 0.0, out);
  CK(cudaEventRecord(s->ev1, s->ctx->stream));
  if (rc) return rc;
  s->initialized = 1;
  if (out) {
    out->status = FB_OK;
    float ms = 0;
    cudaEventSynchronize(s->ev1);
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    out->device_ms = ms;
    out->kernel_launches = s->launches;
  }
  return FB_OK;
}
}  // extern "C"

namespace {

int require(fb_solver *s) {
  if (!s) return set_err(FB_ERR_INVALID_ARGUMENT, "null solver");
  if (!s->initialized) return set_err(FB_ERR_NOT_INITIALIZED, "solver has not been initialized");
  CK(cudaSetDevice(s->ctx->device));
  return FB_OK;
}

void finish_timing(fb_solver *s, fb_report *out) {
  if (!out) return;
  float ms = 0;
  cudaEventSynchronize(s->ev1);
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  out->device_ms = ms;
  out->kernel_launches = s->launches;
}

int grid_of(size_t n) { return (int)std::min<size_t>(4096, std::max<size_t>(1, (n + 255) / 256)); }

}  // namespace

extern "C" {

int32_t fb_restart(fb_solver *s, double time, double angle_degrees, double reynolds, double project_dt, fb_report *out) {
  int rc = require(s);
  if (rc) return rc;
  if (!(reynolds > 0.0) || !std::isfinite(time) || time < 0.0 || !std::isfinite(angle_degrees) || !(project_dt > 0.0))
    return set_err(FB_ERR_INVALID_ARGUMENT, "restart state must be finite, time nonnegative and Reynolds positive");
  if (out) std::memset(out, 0, sizeof(*out));
  s->launches = 0;
  const double nu = s->d.reference_speed * s->d.chord / reynolds;
  const double prev_nu = s->nu;
  s->nu = nu;
  CK(cudaEventRecord(s->ev0, s->ctx->stream));
  rc = full_projection(s, PH_IC | PH_MASK | PH_WALL_FILL | PH_FROM_CELLS, project_dt, angle_degrees, 0.0, out);
  CK(cudaEventRecord(s->ev1, s->ctx->stream));
  if (rc) {
    s->nu = prev_nu;
    return rc;
  }
  s->time = time;
  s->angle = angle_degrees;
  s->omega = 0.0;
  finish_timing(s, out);
  return FB_OK;
}

int32_t fb_update_options(fb_solver *s, const fb_scenario_desc *desc) {
  if (!s || !desc) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  if (!(desc->pressure_tolerance > 0.0) || desc->pressure_max_iterations < 0 || !(desc->cfl > 0.0))
    return set_err(FB_ERR_INVALID_ARGUMENT, "invalid run-time options");
  s->d.cfl = desc->cfl;
  s->d.pressure_tolerance = desc->pressure_tolerance;
  s->d.pressure_max_iterations = desc->pressure_max_iterations;
  s->d.pressure_fixed_iterations = desc->pressure_fixed_iterations;
  s->d.mixed_inner_rtol = desc->mixed_inner_rtol;
  s->d.divergence_limit = desc->divergence_limit;
  s->d.leakage_limit = desc->leakage_limit;
  s->d.advection = desc->advection;
  s->d.face_advection = desc->face_advection;
  return FB_OK;
}

int32_t fb_trace_enable(fb_solver *s, int32_t capacity) {
  if (!s || capacity < 0) return set_err(FB_ERR_INVALID_ARGUMENT, "invalid trace request");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaStreamSynchronize(s->ctx->stream));
  if (s->trace) {
    cudaFree(s->trace);
    s->trace = nullptr;
    s->trace_cap = 0;
  }
  if (capacity == 0) return FB_OK;
  CK(cudaMalloc(&s->trace, sizeof(unsigned long long) * (size_t)(capacity + 1)));
  CK(cudaMemset(s->trace, 0, sizeof(unsigned long long) * (size_t)(capacity + 1)));
  s->trace_cap = capacity + 1;
  return FB_OK;
}

int32_t fb_debug_barrier_timeout(fb_solver *s, int32_t withhold_barrier, uint64_t limit_ns) {
  if (!s || withhold_barrier < 0) return set_err(FB_ERR_INVALID_ARGUMENT, "invalid barrier test request");
  s->withhold = (unsigned)withhold_barrier;
  s->limit_ns = limit_ns == 0 ? kBarrierLimitNs : (unsigned long long)limit_ns;
  return FB_OK;
}

int32_t fb_trace_read(fb_solver *s, uint64_t *host, int64_t capacity, int64_t *count) {
  if (!s || capacity < 0 || (capacity > 0 && !host)) return set_err(FB_ERR_INVALID_ARGUMENT, "invalid trace read");
  if (!s->trace) {
    if (count) *count = 0;
    return FB_OK;
  }
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaStreamSynchronize(s->ctx->stream));
  unsigned long long n = 0;
  CK(cudaMemcpy(&n, s->trace, sizeof(n), cudaMemcpyDeviceToHost));
  const int64_t take = std::min<int64_t>((int64_t)n, capacity);
  if (take > 0) CK(cudaMemcpy(host, s->trace + 1, sizeof(unsigned long long) * take, cudaMemcpyDeviceToHost));
  if (count) *count = (int64_t)n;
  CK(cudaMemset(s->trace, 0, sizeof(unsigned long long)));
  return FB_OK;
}

int32_t fb_get_pose(fb_solver *s, double *time, double *angle_degrees, double *angular_velocity_degrees) {
  int rc = require(s);
  if (rc) return rc;
  if (time) *time = s->time;
  if (angle_degrees) *angle_degrees = s->angle;
  if (angular_velocity_degrees) *angular_velocity_degrees = s->omega;
  return FB_OK;
}

// StableFluidsSolver.advance (stable_fluids.py:332-603) for the cell-centred transport.
// ---- advance: substep plan, substeps, acceptance (stable_fluids.py:332-603) ------------------
// One advance of one solver, split so that a batch can interleave many of them: plan, then
// launch `substeps` substeps, then evaluate the device report (accept, retry with more
// substeps, or fail with the state restored).
struct AdvanceState {
  double target_dt, control_angle, omega_deg;
  double start_time, start_angle;
  double wall_speed, sweep, spacing;
  int substeps, retries;
  double dt;
  unsigned base;
  bool skew;
};

namespace {

int plan_advance(fb_solver *s, double control_angle_degrees, double control_angular_velocity_degrees, double target_dt,
                 AdvanceState &a, fb_report *o) {
  const fb_scenario_desc &d = s->d;
  a.target_dt = target_dt;
  a.control_angle = control_angle_degrees;
  a.omega_deg = control_angular_velocity_degrees;
  a.spacing = std::min(s->ax.h, s->ay.h);
  const double max_speed = std::max(std::max(s->cell_speed, std::fabs(d.freestream_x)), 1.0e-6);
  const bool skew = d.advection == FB_ADVECT_SKEW_RK2;
  const double cfl = skew ? std::min(d.cfl, 0.4) : d.cfl;
  const double radius = naca_max_radius(s->foil);
  a.wall_speed = std::fabs(deg2rad(control_angular_velocity_degrees)) * radius;
  a.sweep = std::fabs(deg2rad(control_angle_degrees - s->angle)) * radius / a.spacing;
  const double rate = skew ? s->skew_rate : max_speed / a.spacing;
  const double measure = target_dt * rate;
  const double required =
      std::max(std::max(1.05 * measure / cfl, target_dt * a.wall_speed / (cfl * a.spacing)), a.sweep / cfl);
  a.substeps = std::max(1, (int)std::ceil(required));
  o->wall_speed = a.wall_speed;
  if (!(required <= 512.0) || a.substeps > 512) {
    o->status = FB_ERR_NUMERICAL;
    o->reason = FB_REASON_STABILITY_LIMIT;
    o->stage = skew ? FB_STAGE_ADVECTION : FB_STAGE_BOUNDARY;
    o->required_substeps = std::isfinite(required) ? std::ceil(required) : required;
    o->max_speed = max_speed;
    o->boundary_sweep = a.sweep;
    return set_err(FB_ERR_NUMERICAL, "Stable Fluids motion requires too many internal substeps");
  }
  a.dt = target_dt / a.substeps;
  a.start_time = s->time;
  a.start_angle = s->angle;
  a.retries = 0;
  if (skew)
    a.base = PH_FACE | PH_MASK_LATE | PH_GUARD | PH_PROJECT;
  else if (d.face_advection)
    a.base = PH_F2C | PH_MASK | PH_FACE | PH_GUARD | PH_PROJECT;
  else
    a.base = PH_F2C | PH_ADVECT | PH_MASK | PH_DIFFUSE | PH_FROM_CELLS | PH_GUARD | PH_PROJECT;
  if (d.passive_scalar && !skew && !d.face_advection) a.base |= PH_SCALAR;
  a.skew = skew;
  return FB_OK;
}

// Substep k of the plan: phases and pose.
unsigned substep_phases(const AdvanceState &a, int k) { return a.base | (k == a.substeps - 1 ? PH_FINALIZE : 0u); }
double substep_angle(const AdvanceState &a, int k) {
  const double frac = (double)(k + 1) / a.substeps;
  return a.start_angle + frac * (a.control_angle - a.start_angle);
}

enum AdvanceOutcome { ADV_ACCEPTED = 0, ADV_RETRY = 1, ADV_FAILED = 2 };

// Judge the device report (already in s->rep_host) after the plan's substeps ran.
AdvanceOutcome evaluate_advance(fb_solver *s, AdvanceState &a, fb_report *o, int &rc) {
  const fb_scenario_desc &d = s->d;
  const DevReport &r = *s->rep_host;
  rc = FB_OK;
  if (!report_ok(r)) {
    checkpoint(s, true);
    cudaStreamSynchronize(s->ctx->stream);
    rc = numerical_status(s, o);
    o->substeps = a.substeps;
    o->stability_retries = a.retries;
    return ADV_FAILED;
  }
  const double final_speed = r.final_speed;
  const double rate = a.skew ? r.skew_rate : final_speed / a.spacing;
  const double accepted = a.dt * rate;
  const double cfl = a.skew ? std::min(d.cfl, 0.4) : d.cfl;
  if (!(accepted <= cfl * (1.0 + 1.0e-6))) {
    const int next = std::max(a.substeps + 1, (int)std::ceil(1.05 * a.substeps * accepted / cfl));
    rc = checkpoint(s, true);
    if (rc) return ADV_FAILED;
    if (next > 512) {
      cudaStreamSynchronize(s->ctx->stream);
      o->status = FB_ERR_NUMERICAL;
      o->reason = FB_REASON_STABILITY_LIMIT;
      o->stage = FB_STAGE_ADVECTION;
      o->required_substeps = next;
      o->accepted_measure = accepted;
      o->stability_retries = a.retries;
      rc = set_err(FB_ERR_NUMERICAL, "Stable Fluids retry requires too many internal substeps");
      return ADV_FAILED;
    }
    ++a.retries;
    a.substeps = next;
    a.dt = a.target_dt / a.substeps;
    return ADV_RETRY;
  }
  fill_report_from_dev(r, o);
  o->substeps = a.substeps;
  o->stability_retries = a.retries;
  o->max_speed = final_speed;
  o->wall_speed = a.wall_speed;
  o->accepted_measure = accepted;
  o->advective_rate = rate;
  o->boundary_sweep = a.sweep / a.substeps;
  if (r.div_linf > d.divergence_limit || r.leakage > d.leakage_limit) {
    checkpoint(s, true);
    cudaStreamSynchronize(s->ctx->stream);
    o->status = FB_ERR_NUMERICAL;
    o->reason = FB_REASON_POSTCONDITION_FAILURE;
    o->stage = FB_STAGE_POSTCONDITION;
    o->evidence[0] = r.div_linf;
    o->evidence[1] = d.divergence_limit;
    o->evidence[2] = r.leakage;
    o->evidence[3] = d.leakage_limit;
    rc = set_err(FB_ERR_NUMERICAL, "Stable Fluids exceeded a configured MAC postcondition limit");
    return ADV_FAILED;
  }
  s->time = a.start_time + a.target_dt;
  s->angle = a.control_angle;
  s->omega = a.omega_deg;
  s->cell_speed = final_speed;
  s->skew_rate = r.skew_rate;
  s->cg_per_substep = std::max(1.0, (double)r.total_cg_iters / a.substeps);
  o->status = FB_OK;
  return ADV_ACCEPTED;
}

int validate_advance_args(double control_time, double control_angle_degrees, double control_angular_velocity_degrees,
                          double target_dt) {
  if (!std::isfinite(target_dt) || target_dt <= 0.0)
    return set_err(FB_ERR_INVALID_ARGUMENT, "target_dt must be finite and positive");
  if (!std::isfinite(control_time) || !std::isfinite(control_angle_degrees) ||
      !std::isfinite(control_angular_velocity_degrees))
    return set_err(FB_ERR_INVALID_ARGUMENT, "control state must be finite");
  return FB_OK;
}

}  // namespace

int32_t fb_advance(fb_solver *s, double control_time, double control_angle_degrees,
                   double control_angular_velocity_degrees, double target_dt, fb_report *out) {
  int rc = require(s);
  if (rc) return rc;
  rc = validate_advance_args(control_time, control_angle_degrees, control_angular_velocity_degrees, target_dt);
  if (rc) return rc;
  fb_report local{};
  fb_report *o = out ? out : &local;
  std::memset(o, 0, sizeof(*o));
  s->launches = 0;
  AdvanceState a{};
  rc = plan_advance(s, control_angle_degrees, control_angular_velocity_degrees, target_dt, a, o);
  if (rc) return rc;
  CK(cudaEventRecord(s->ev0, s->ctx->stream));
  rc = checkpoint(s, false);
  if (rc) return rc;
  for (;;) {
    rc = reset_report(s);
    if (rc) return rc;
    for (int k = 0; k < a.substeps; ++k) {
      rc = launch(s, substep_phases(a, k), a.dt, substep_angle(a, k), control_angular_velocity_degrees, s->nu,
                  s->d.pressure_tolerance, s->d.pressure_max_iterations);
      if (rc) {
        checkpoint(s, true);
        return rc;
      }
    }
    rc = read_report(s);
    if (rc) {
      checkpoint(s, true);
      return rc;
    }
    const AdvanceOutcome out_ = evaluate_advance(s, a, o, rc);
    if (out_ == ADV_RETRY) continue;
    if (out_ == ADV_FAILED) return rc;
    break;
  }
  CK(cudaEventRecord(s->ev1, s->ctx->stream));
  (void)control_time;
  finish_timing(s, o);
  return FB_OK;
}

int32_t fb_set_launch_shape(fb_solver *s, int32_t ctas, int32_t column_tile) {
  int rc = require(s);
  if (rc) return rc;
  if (ctas < 0 || ctas > s->nblocks_max)
    return set_err(FB_ERR_INVALID_ARGUMENT, "ctas must be in [1, %d] (0 keeps the current count)", s->nblocks_max);
  if (column_tile != 0 && (column_tile > s->col_w_max || (column_tile & (column_tile - 1)) || column_tile < 2))
    return set_err(FB_ERR_INVALID_ARGUMENT, "column tile must be a power of two in [2, %d] (0 keeps it)", s->col_w_max);
  if (ctas > 0) s->nblocks = ctas;
  if (column_tile > 0) s->col_w = column_tile;
  return FB_OK;
}

int32_t fb_get_launch_shape(fb_solver *s, int32_t *ctas, int32_t *column_tile, double *inner_rtol) {
  int rc = require(s);
  if (rc) return rc;
  if (ctas) *ctas = s->nblocks;
  if (column_tile) *column_tile = s->col_w;
  if (inner_rtol)
    *inner_rtol = s->d.mixed_inner_rtol > 0.0 ? s->d.mixed_inner_rtol
                                              : (s->tuned_inner_rtol > 0.0 ? s->tuned_inner_rtol : 3.0e-6);
  return FB_OK;
}

int32_t fb_autotune(fb_solver *s, double target_dt, int32_t reps, double *out, int32_t n) {
  int rc = require(s);
  if (rc) return rc;
  if (!(target_dt > 0.0) || !std::isfinite(target_dt) || reps < 1 || reps > 15 || (n > 0 && !out))
    return set_err(FB_ERR_INVALID_ARGUMENT, "invalid autotune request");
  if (s->trace) return set_err(FB_ERR_INVALID_ARGUMENT, "disable tracing before tuning");
  CK(cudaSetDevice(s->ctx->device));
  // one substep of an advance from the current state, as fb_advance would plan it
  fb_report scratch{};
  AdvanceState a{};
  rc = plan_advance(s, s->angle, 0.0, target_dt, a, &scratch);
  if (rc) return rc;
  const unsigned phases = a.base | (a.substeps == 1 ? PH_FINALIZE : 0u);
  rc = checkpoint(s, false);
  if (rc) return rc;
  const fb_scenario_desc &d = s->d;
  const bool mixed = d.pressure_scheme == FB_PRESSURE_MIXED;
  int trials = 0;
  auto trial = [&](const TuneChoice &c, double &ms) -> int {
    s->col_w = c.col_w;
    s->nblocks = c.nblocks;
    s->tuned_inner_rtol = c.inner_rtol;
    std::vector<float> t;
    for (int k = 0; k < reps; ++k) {
      int r = reset_report(s);
      if (r) return r;
      CK(cudaEventRecord(s->ev0, s->ctx->stream));
      r = launch(s, phases, a.dt, substep_angle(a, 0), 0.0, s->nu, d.pressure_tolerance, d.pressure_max_iterations);
      if (r) return r;
      CK(cudaEventRecord(s->ev1, s->ctx->stream));
      r = read_report(s);
      if (r) return r;
      if (!report_ok(*s->rep_host)) {
        checkpoint(s, true);
        cudaStreamSynchronize(s->ctx->stream);
        return set_err(FB_ERR_NUMERICAL, "autotune trial failed (reason=%d stage=%d)", s->rep_host->reason,
                       s->rep_host->stage);
      }
      float e = 0.f;
      CK(cudaEventElapsedTime(&e, s->ev0, s->ev1));
      t.push_back(e);
      r = checkpoint(s, true);
      if (r) return r;
      ++trials;
    }
    std::sort(t.begin(), t.end());
    ms = t[t.size() / 2];
    return FB_OK;
  };
  const TuneChoice start{s->col_w, s->nblocks, s->tuned_inner_rtol};
  TuneChoice heur{s->col_w_max, s->nblocks_max, 0.0};
  double heur_ms = 0.0;
  rc = trial(heur, heur_ms);
  TuneChoice best = heur;
  double best_ms = heur_ms;
  auto consider = [&](TuneChoice c) -> int {
    double ms = 0.0;
    const int r = trial(c, ms);
    if (r) return r;
    if (ms < best_ms * 0.995) {
      best = c;
      best_ms = ms;
    }
    return FB_OK;
  };
  // coordinate search: CTA count, then column tile width, then (mixed) the inner sweep floor
  if (!rc) {
    const int full = s->nblocks_max, sms = s->ctx->sm_count;
    std::vector<int> counts;
    for (int c : {full, sms * 7 / 8, sms * 3 / 4, sms * 5 / 8, sms / 2})
      if (c >= 1 && c <= full && std::find(counts.begin(), counts.end(), c) == counts.end()) counts.push_back(c);
    // a CTA count that gives the row transforms whole rounds (no partial last round)
    if (s->fft.rows >= 1) {
      const int per = s->fft.rows;
      for (int rounds = 1; rounds <= 64; ++rounds) {
        const int c = (d.ny + per * rounds - 1) / (per * rounds);
        if (c <= full && c >= sms / 2) {
          if (std::find(counts.begin(), counts.end(), c) == counts.end()) counts.push_back(c);
          break;
        }
      }
    }
    for (int c : counts)
      if (!rc && c != heur.nblocks) rc = consider(TuneChoice{best.col_w, c, best.inner_rtol});
    for (int w = s->col_w_max >> 1; !rc && w >= 2; w >>= 1) rc = consider(TuneChoice{w, best.nblocks, best.inner_rtol});
    if (mixed && d.pressure_fixed_iterations <= 0 && d.mixed_inner_rtol <= 0.0)
      for (double f : {1.0e-6, 1.0e-5, 3.0e-5})
        if (!rc) rc = consider(TuneChoice{best.col_w, best.nblocks, f});
  }
  if (rc) {  // leave the solver as it was
    s->col_w = start.col_w;
    s->nblocks = start.nblocks;
    s->tuned_inner_rtol = start.inner_rtol;
    return rc;
  }
  s->col_w = best.col_w;
  s->nblocks = best.nblocks;
  s->tuned_inner_rtol = best.inner_rtol;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[tune_key(s)] = best;
  }
  const double vals[8] = {(double)best.col_w, (double)best.nblocks, best.inner_rtol > 0.0 ? best.inner_rtol : 3.0e-6,
                          heur_ms, best_ms, (double)trials, (double)heur.col_w, (double)heur.nblocks};
  for (int i = 0; i < n && i < 8; ++i) out[i] = vals[i];
  return FB_OK;
}

// ---- batched advance ----------------------------------------------------------------------
// One launch per attempt: the running members form the groups of the launch, each with a
// contiguous CTA range sized by its expected work, and run all their planned substeps.
struct fb_batch {
  fb_ctx *ctx;
  std::vector<fb_solver *> members;
  std::vector<int> last_ctas;       // CTAs of each member in the latest launch (0: not running)
  StepParams<float, float> *table_host = nullptr, *table_dev = nullptr;
  size_t table_cap = 0;             // entries
  int *index_host = nullptr;        // first[m + 1] then sub_first[m + 1]
  int *index_dev = nullptr;
  unsigned long long *timing_host = nullptr, *timing_dev = nullptr;  // per group: first start, last end
  void *kernel = nullptr;
  size_t smem = 0;
  int capacity = 0;                 // CTAs the device holds at once
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

bool batch_member_ok(const fb_solver *s, std::string &why) {
  if (!s->initialized) { why = "every member must be initialized"; return false; }
  if (s->d.precision != FB_FLOAT32 || s->d.pressure_scheme != FB_PRESSURE_MIXED) {
    why = "batched members use float32 fields with the mixed pressure scheme";
    return false;
  }
  if (!(!s->d.periodic_x && !s->d.periodic_y) || s->tw_smem_off < 0 || s->fft.io_soff < 0 || s->fft.npass != 3 ||
      s->fft.vpt != 16) {
    why = "batched members need the staged three-pass row transform (non-periodic, nx a multiple of 16, 129..2048 columns)";
    return false;
  }
  if (s->trace) { why = "tracing is not available for batched members"; return false; }
  return true;
}

// CTAs per group in proportion to its weight (largest remainder), at least one each and at
// most what a single-solve launch of that member would use.
std::vector<int> split_ctas(const std::vector<double> &w, const std::vector<int> &cap, int total) {
  const size_t n = w.size();
  std::vector<int> c(n, 1);
  double sum = 0.0;
  for (double x : w) sum += x;
  int left = total - (int)n;
  std::vector<std::pair<double, size_t>> rem;
  for (size_t i = 0; i < n; ++i) {
    const double share = sum > 0.0 ? w[i] / sum * (double)(total - (int)n) : 0.0;
    int extra = std::max(0, std::min({(int)share, cap[i] - 1, left}));
    c[i] += extra;
    left -= extra;
    rem.push_back({share - (double)(int)share, i});
  }
  std::sort(rem.begin(), rem.end(), [](const std::pair<double, size_t> &x, const std::pair<double, size_t> &y) {
    return x.first > y.first;
  });
  for (bool grew = true; left > 0 && grew;) {
    grew = false;
    for (size_t k = 0; left > 0 && k < rem.size(); ++k) {
      const size_t i = rem[k].second;
      if (c[i] < cap[i]) {
        ++c[i];
        --left;
        grew = true;
      }
    }
  }
  return c;
}

int batch_reserve(fb_batch *b, size_t entries) {
  if (entries <= b->table_cap) return FB_OK;
  const size_t cap = std::max(entries, 2 * b->table_cap);
  if (b->table_host) cudaFreeHost(b->table_host);
  if (b->table_dev) cudaFree(b->table_dev);
  b->table_host = nullptr;
  b->table_dev = nullptr;
  b->table_cap = 0;
  if (cudaMallocHost(&b->table_host, sizeof(StepParams<float, float>) * cap) != cudaSuccess ||
      cudaMalloc(&b->table_dev, sizeof(StepParams<float, float>) * cap) != cudaSuccess)
    return set_err(FB_ERR_OUT_OF_MEMORY, "batch table of %zu entries", cap);
  b->table_cap = cap;
  return FB_OK;
}

}  // namespace

int32_t fb_batch_create(fb_ctx *ctx, fb_solver *const *solvers, int32_t count, fb_batch **out) {
  if (!ctx || !solvers || !out || count < 1) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument or empty batch");
  *out = nullptr;
  std::string why;
  size_t smem = 0;
  for (int i = 0; i < count; ++i) {
    if (!solvers[i] || solvers[i]->ctx != ctx) return set_err(FB_ERR_INVALID_ARGUMENT, "member %d is not a solver of this context", i);
    for (int j = 0; j < i; ++j)
      if (solvers[j] == solvers[i]) return set_err(FB_ERR_INVALID_ARGUMENT, "member %d appears twice", i);
    if (!batch_member_ok(solvers[i], why)) return set_err(FB_ERR_INVALID_ARGUMENT, "member %d: %s", i, why.c_str());
    smem = std::max(smem, solvers[i]->smem);
  }
  CK(cudaSetDevice(ctx->device));
  void *kernel = step_kernel_batch_f32m();
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreads, smem));
  const int total = occ * ctx->sm_count;
  if (occ < 1 || count > total)
    return set_err(FB_ERR_INVALID_ARGUMENT, "a batch holds at most %d members on this device", std::max(total, 0));
  fb_batch *b = new (std::nothrow) fb_batch();
  if (!b) return set_err(FB_ERR_OUT_OF_MEMORY, "host allocation");
  b->ctx = ctx;
  b->members.assign(solvers, solvers + count);
  b->last_ctas.assign(count, 0);
  b->kernel = kernel;
  b->smem = smem;
  b->capacity = total;
  int rc = batch_reserve(b, (size_t)count * 4);
  if (!rc && (cudaMallocHost(&b->index_host, sizeof(int) * 2 * (count + 1)) != cudaSuccess ||
              cudaMalloc(&b->index_dev, sizeof(int) * 2 * (count + 1)) != cudaSuccess ||
              cudaMallocHost(&b->timing_host, sizeof(unsigned long long) * 2 * count) != cudaSuccess ||
              cudaMalloc(&b->timing_dev, sizeof(unsigned long long) * 2 * count) != cudaSuccess))
    rc = set_err(FB_ERR_OUT_OF_MEMORY, "batch index arrays");
  if (rc) {
    fb_batch_destroy(b);
    return rc;
  }
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  *out = b;
  return FB_OK;
}

int32_t fb_batch_destroy(fb_batch *b) {
  if (!b) return FB_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  if (b->table_host) cudaFreeHost(b->table_host);
  if (b->table_dev) cudaFree(b->table_dev);
  if (b->index_host) cudaFreeHost(b->index_host);
  if (b->index_dev) cudaFree(b->index_dev);
  if (b->timing_host) cudaFreeHost(b->timing_host);
  if (b->timing_dev) cudaFree(b->timing_dev);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
  return FB_OK;
}

int32_t fb_batch_ctas(const fb_batch *b, int32_t *ctas, int32_t count) {
  if (!b || !ctas || count != (int32_t)b->members.size()) return set_err(FB_ERR_INVALID_ARGUMENT, "ctas needs one slot per member");
  for (int32_t i = 0; i < count; ++i) ctas[i] = b->last_ctas[i];
  return FB_OK;
}

int32_t fb_batch_advance(fb_batch *b, const double *control_time, const double *control_angle_degrees,
                         const double *control_angular_velocity_degrees, const double *target_dt, fb_report *reports,
                         int32_t *status) {
  if (!b || !control_time || !control_angle_degrees || !control_angular_velocity_degrees || !target_dt || !reports ||
      !status)
    return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  const int n = (int)b->members.size();
  CK(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  std::vector<AdvanceState> a(n);
  std::vector<int> state(n, 0);  // 0 running, 1 accepted, 2 failed
  for (int i = 0; i < n; ++i) {
    fb_solver *s = b->members[i];
    std::memset(&reports[i], 0, sizeof(fb_report));
    s->launches = 0;
    int rc = validate_advance_args(control_time[i], control_angle_degrees[i], control_angular_velocity_degrees[i],
                                   target_dt[i]);
    if (!rc) rc = plan_advance(s, control_angle_degrees[i], control_angular_velocity_degrees[i], target_dt[i], a[i],
                               &reports[i]);
    if (!rc) rc = checkpoint(s, false);
    if (!rc) rc = reset_report(s);
    status[i] = rc;
    if (rc) {
      if (reports[i].status == 0) reports[i].status = rc;
      state[i] = 2;
    }
  }
  CK(cudaEventRecord(b->ev0, st));
  int launches = 0;
  for (;;) {
    std::vector<int> run;
    for (int i = 0; i < n; ++i)
      if (state[i] == 0) run.push_back(i);
    if (run.empty()) break;
    const int m = (int)run.size();
    size_t entries = 0;
    for (int i : run) entries += (size_t)a[i].substeps;
    int rc = batch_reserve(b, entries);
    if (rc) return rc;
    // expected work: cells x substeps x (outer phases ~ 6 CG iterations + CG iterations),
    // scaled by each member's measured cost per unit of it in earlier batched launches (the
    // CTA-seconds its group took), so that the CTA split evens out the groups' finish times
    std::vector<double> w(m), wexp(m);
    std::vector<int> cap(m);
    double cost_sum = 0.0;
    int cost_n = 0;
    for (int g = 0; g < m; ++g) {
      const fb_solver *s = b->members[run[g]];
      wexp[g] = (double)s->L.N * a[run[g]].substeps * (6.0 + (s->cg_per_substep > 0.0 ? s->cg_per_substep : 15.0));
      cap[g] = s->nblocks_max;
      if (s->batch_cost > 0.0) {
        cost_sum += s->batch_cost;
        ++cost_n;
      }
    }
    const double cost_mean = cost_n ? cost_sum / cost_n : 1.0;
    for (int g = 0; g < m; ++g) {
      const double k = b->members[run[g]]->batch_cost;
      w[g] = wexp[g] * (k > 0.0 ? k : cost_mean);
    }
    const std::vector<int> c = split_ctas(w, cap, b->capacity);
    int *first = b->index_host, *sub_first = b->index_host + (m + 1);
    first[0] = 0;
    sub_first[0] = 0;
    size_t e = 0;
    std::fill(b->last_ctas.begin(), b->last_ctas.end(), 0);
    for (int g = 0; g < m; ++g) {
      const int i = run[g];
      fb_solver *s = b->members[i];
      first[g + 1] = first[g] + c[g];
      b->last_ctas[i] = c[g];
      for (int k = 0; k < a[i].substeps; ++k, ++e)
        b->table_host[e] = make_params<float, float>(s, substep_phases(a[i], k), a[i].dt, substep_angle(a[i], k),
                                                     a[i].omega_deg, s->nu, s->d.pressure_tolerance,
                                                     s->d.pressure_max_iterations, false);
      sub_first[g + 1] = (int)e;
      s->launches += 1;
    }
    CK(cudaMemcpyAsync(b->table_dev, b->table_host, sizeof(StepParams<float, float>) * e, cudaMemcpyHostToDevice, st));
    // first[] and sub_first[] at the same offsets on the device
    CK(cudaMemcpyAsync(b->index_dev, b->index_host, sizeof(int) * 2 * (m + 1), cudaMemcpyHostToDevice, st));
    int *first_dev = b->index_dev, *sub_first_dev = b->index_dev + (m + 1);
    for (int g = 0; g < m; ++g) {
      b->timing_host[2 * g] = ~0ull;
      b->timing_host[2 * g + 1] = 0ull;
    }
    CK(cudaMemcpyAsync(b->timing_dev, b->timing_host, sizeof(unsigned long long) * 2 * m, cudaMemcpyHostToDevice, st));
    void *args[] = {&b->table_dev, &first_dev, &sub_first_dev, (void *)&m, &b->timing_dev};
    CK(cudaLaunchCooperativeKernel(b->kernel, dim3(first[m]), dim3(kThreads), args, b->smem, st));
    ++launches;
    for (int i : run)
      CK(cudaMemcpyAsync(b->members[i]->rep_host, b->members[i]->at<DevReport>(b->members[i]->L.rep), sizeof(DevReport),
                         cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(b->timing_host, b->timing_dev, sizeof(unsigned long long) * 2 * m, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));  // also frees the pinned tables for the next attempt
    CK(cudaGetLastError());
    // measured cost per unit of expected work of each group (CTA-seconds), averaged with the
    // earlier launches' so one noisy launch does not swing the split
    for (int g = 0; g < m; ++g) {
      const unsigned long long t0 = b->timing_host[2 * g], t1 = b->timing_host[2 * g + 1];
      if (t0 == ~0ull || t1 <= t0 || wexp[g] <= 0.0) continue;
      fb_solver *s = b->members[run[g]];
      const double measured = (double)(t1 - t0) * 1e-9 * c[g] / wexp[g];
      s->batch_cost = s->batch_cost > 0.0 ? 0.5 * (s->batch_cost + measured) : measured;
    }
    for (int i : run) {
      int rc2 = FB_OK;
      const AdvanceOutcome oc = evaluate_advance(b->members[i], a[i], &reports[i], rc2);
      if (oc == ADV_ACCEPTED) {
        state[i] = 1;
      } else if (oc == ADV_FAILED) {
        state[i] = 2;
        status[i] = rc2;
      } else {
        rc2 = reset_report(b->members[i]);
        if (rc2) {
          state[i] = 2;
          status[i] = rc2;
        }
      }
    }
  }
  CK(cudaEventRecord(b->ev1, st));
  CK(cudaEventSynchronize(b->ev1));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  int failed = 0;
  for (int i = 0; i < n; ++i) {
    reports[i].device_ms = ms;  // the batch's device time, shared by its members
    reports[i].kernel_launches = launches;
    if (state[i] != 1) ++failed;
  }
  if (failed) return set_err(FB_ERR_NUMERICAL, "%d of %d batch members did not advance (see status)", failed, n);
  return FB_OK;
}

int32_t fb_export_velocity(fb_solver *s, void *host, size_t bytes, int32_t zero_solids) {
  int rc = require(s);
  if (rc) return rc;
  const Layout &L = s->L;
  if (!host || bytes != L.N * 2 * L.vsz) return set_err(FB_ERR_INVALID_ARGUMENT, "export buffer must be %zu bytes", L.N * 2 * (size_t)L.vsz);
  const int g = grid_of(L.N);
  if (s->d.precision == FB_FLOAT64)
    export_cells_kernel<double><<<g, 256, 0, s->ctx->stream>>>(s->at<double>(L.u), s->at<double>(L.v), s->at<unsigned char>(L.solid),
                                                               s->d.nx, s->d.ny, zero_solids, s->at<double>(L.staging));
  else
    export_cells_kernel<float><<<g, 256, 0, s->ctx->stream>>>(s->at<float>(L.u), s->at<float>(L.v), s->at<unsigned char>(L.solid),
                                                              s->d.nx, s->d.ny, zero_solids, s->at<float>(L.staging));
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, s->arena + L.staging, bytes, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_export_state(fb_solver *s, void *host, size_t bytes, int64_t *nonfinite) {
  int rc = require(s);
  if (rc) return rc;
  const Layout &L = s->L;
  if (!host || !nonfinite || bytes != L.N * 2 * L.vsz)
    return set_err(FB_ERR_INVALID_ARGUMENT, "export buffer must be %zu bytes", L.N * 2 * (size_t)L.vsz);
  const int g = grid_of(L.N);
  unsigned long long *cnt = s->at<unsigned long long>(L.count);
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s->ctx->stream));
  if (s->d.precision == FB_FLOAT64)
    export_cells_kernel<double><<<g, 256, 0, s->ctx->stream>>>(s->at<double>(L.u), s->at<double>(L.v), s->at<unsigned char>(L.solid),
                                                               s->d.nx, s->d.ny, 1, s->at<double>(L.staging), cnt);
  else
    export_cells_kernel<float><<<g, 256, 0, s->ctx->stream>>>(s->at<float>(L.u), s->at<float>(L.v), s->at<unsigned char>(L.solid),
                                                              s->d.nx, s->d.ny, 1, s->at<float>(L.staging), cnt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, s->arena + L.staging, bytes, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaMemcpyAsync(s->count_host, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  *nonfinite = (int64_t)*s->count_host;
  return FB_OK;
}

int32_t fb_export_faces(fb_solver *s, void *host_u, size_t bytes_u, void *host_v, size_t bytes_v) {
  int rc = require(s);
  if (rc) return rc;
  const Layout &L = s->L;
  if (!host_u || !host_v || bytes_u != L.NU * L.vsz || bytes_v != L.NV * L.vsz)
    return set_err(FB_ERR_INVALID_ARGUMENT, "face buffers must be %zu and %zu bytes", L.NU * (size_t)L.vsz, L.NV * (size_t)L.vsz);
  CK(cudaMemcpyAsync(host_u, s->arena + L.u, bytes_u, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaMemcpyAsync(host_v, s->arena + L.v, bytes_v, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_export_pressure(fb_solver *s, double *host, size_t bytes) {
  int rc = require(s);
  if (rc) return rc;
  if (!host || bytes != s->L.N * 8) return set_err(FB_ERR_INVALID_ARGUMENT, "pressure buffer must be %zu bytes", s->L.N * 8);
  CK(cudaMemcpyAsync(host, s->arena + s->L.x, bytes, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_export_mask(fb_solver *s, uint8_t *host, size_t bytes) {
  int rc = require(s);
  if (rc) return rc;
  if (!host || bytes != s->L.N) return set_err(FB_ERR_INVALID_ARGUMENT, "mask buffer must be %zu bytes", s->L.N);
  CK(cudaMemcpyAsync(host, s->arena + s->L.solid, bytes, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_export_scalar(fb_solver *s, void *host, size_t bytes) {
  int rc = require(s);
  if (rc) return rc;
  if (!s->d.passive_scalar) return set_err(FB_ERR_INVALID_ARGUMENT, "solver carries no passive scalar");
  if (!host || bytes != s->L.N * s->L.vsz) return set_err(FB_ERR_INVALID_ARGUMENT, "scalar buffer size");
  CK(cudaMemcpyAsync(host, s->arena + s->L.scal, bytes, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_import_scalar(fb_solver *s, const void *host, size_t bytes) {
  int rc = require(s);
  if (rc) return rc;
  if (!s->d.passive_scalar) return set_err(FB_ERR_INVALID_ARGUMENT, "solver carries no passive scalar");
  if (!host || bytes != s->L.N * s->L.vsz) return set_err(FB_ERR_INVALID_ARGUMENT, "scalar buffer size");
  CK(cudaMemcpyAsync(s->arena + s->L.scal, host, bytes, cudaMemcpyHostToDevice, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

// StableFluidsSolver.import_state (stable_fluids.py:636-706) after validation: solid cells
// take the wall velocity, faces are rebuilt and re-projected; rollback on failure.
int32_t fb_import_velocity(fb_solver *s, const void *host, size_t bytes, double time, double angle_degrees,
                           double angular_velocity_degrees, double project_dt, fb_report *out) {
  int rc = require(s);
  if (rc) return rc;
  const Layout &L = s->L;
  if (!host || bytes != L.N * 2 * L.vsz) return set_err(FB_ERR_INVALID_ARGUMENT, "import buffer must be %zu bytes", L.N * 2 * (size_t)L.vsz);
  if (!std::isfinite(time) || !std::isfinite(angle_degrees) || !std::isfinite(angular_velocity_degrees) || !(project_dt > 0.0))
    return set_err(FB_ERR_INVALID_ARGUMENT, "import pose must be finite");
  if (out) std::memset(out, 0, sizeof(*out));
  s->launches = 0;
  CK(cudaEventRecord(s->ev0, s->ctx->stream));
  rc = checkpoint(s, false);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->arena + L.staging, host, bytes, cudaMemcpyHostToDevice, s->ctx->stream));
  cells_from_staging(s, s->ctx->stream);
  CK(cudaGetLastError());
  rc = full_projection(s, PH_MASK | PH_WALL_FILL | PH_FROM_CELLS, project_dt, angle_degrees, angular_velocity_degrees, out);
  CK(cudaEventRecord(s->ev1, s->ctx->stream));
  if (rc) {
    checkpoint(s, true);
    cudaStreamSynchronize(s->ctx->stream);
    if (out) out->stage = out->stage;
    return rc;
  }
  s->time = time;
  s->angle = angle_degrees;
  s->omega = angular_velocity_degrees;
  finish_timing(s, out);
  return FB_OK;
}

int32_t fb_sample_velocity(fb_solver *s, const double *points, int64_t n, double *out) {
  int rc = require(s);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!points || !out))) return set_err(FB_ERR_INVALID_ARGUMENT, "points");
  if (n == 0) return FB_OK;
  double *dp = nullptr;
  CK(cudaMallocAsync(&dp, sizeof(double) * 4 * n, s->ctx->stream));
  CK(cudaMemcpyAsync(dp, points, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, s->ctx->stream));
  const int g = (int)((n + 255) / 256);
  if (s->d.precision == FB_FLOAT64)
    sample_kernel<double><<<g, 256, 0, s->ctx->stream>>>(s->at<double>(s->L.u), s->at<double>(s->L.v), s->ax, s->ay, s->d.nx,
                                                         s->d.ny, dp, n, dp + 2 * n);
  else
    sample_kernel<float><<<g, 256, 0, s->ctx->stream>>>(s->at<float>(s->L.u), s->at<float>(s->L.v), s->ax, s->ay, s->d.nx,
                                                        s->d.ny, dp, n, dp + 2 * n);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dp + 2 * n, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaFreeAsync(dp, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_diagnostics(fb_solver *s, double *values, int32_t count) {
  int rc = require(s);
  if (rc) return rc;
  if (!values || count < 7) return set_err(FB_ERR_INVALID_ARGUMENT, "diagnostics needs 7 values");
  const fb_scenario_desc &d = s->d;
  double *rows = s->at<double>(s->L.staging);  // ny * 8 doubles fit: staging >= N * 8 bytes
  double *res = rows + (size_t)d.ny * 8;
  const double om = deg2rad(s->omega);
  if (d.precision == FB_FLOAT64)
    diag_rows_kernel<double><<<d.ny, 256, 0, s->ctx->stream>>>(s->at<double>(s->L.u), s->at<double>(s->L.v),
                                                               s->at<unsigned char>(s->L.solid), d.nx, d.ny, s->ax.h, s->ay.h,
                                                               s->ax, s->ay, om, d.pivot_x, d.pivot_y, d.pivot_x + d.chord,
                                                               d.pivot_x, d.freestream_x, rows);
  else
    diag_rows_kernel<float><<<d.ny, 256, 0, s->ctx->stream>>>(s->at<float>(s->L.u), s->at<float>(s->L.v),
                                                              s->at<unsigned char>(s->L.solid), d.nx, d.ny, s->ax.h, s->ay.h,
                                                              s->ax, s->ay, om, d.pivot_x, d.pivot_y, d.pivot_x + d.chord,
                                                              d.pivot_x, d.freestream_x, rows);
  diag_fold_kernel<<<1, 32, 0, s->ctx->stream>>>(rows, d.nx, d.ny, s->ax.h, s->ay.h, res);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(values, res, sizeof(double) * 7, cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  return FB_OK;
}

int32_t fb_forces(fb_solver *s, double *values, int32_t count) {
  int rc = require(s);
  if (rc) return rc;
  if (!values || count < 8) return set_err(FB_ERR_INVALID_ARGUMENT, "forces needs 8 values");
  const fb_scenario_desc &d = s->d;
  double *rows = s->at<double>(s->L.staging);  // 4 ny + 4 doubles fit in the staging area
  double *res = rows + (size_t)4 * d.ny;
  const double om = deg2rad(s->omega);
  if (d.precision == FB_FLOAT64)
    forces_rows_kernel<double><<<d.ny, 256, 0, s->ctx->stream>>>(
        s->at<double>(s->L.u), s->at<double>(s->L.v), s->at<double>(s->L.x), s->at<unsigned char>(s->L.solid), d.nx, d.ny,
        s->ax.h, s->ay.h, d.x0, d.y0, d.periodic_x, d.periodic_y, om, d.pivot_x, d.pivot_y, s->nu, rows);
  else
    forces_rows_kernel<float><<<d.ny, 256, 0, s->ctx->stream>>>(
        s->at<float>(s->L.u), s->at<float>(s->L.v), s->at<double>(s->L.x), s->at<unsigned char>(s->L.solid), d.nx, d.ny,
        s->ax.h, s->ay.h, d.x0, d.y0, d.periodic_x, d.periodic_y, om, d.pivot_x, d.pivot_y, s->nu, rows);
  forces_fold_kernel<<<1, 32, 0, s->ctx->stream>>>(rows, d.ny, res);
  CK(cudaGetLastError());
  double f[4];
  CK(cudaMemcpyAsync(f, res, sizeof(f), cudaMemcpyDeviceToHost, s->ctx->stream));
  CK(cudaStreamSynchronize(s->ctx->stream));
  const double fx = f[0] + f[2], fy = f[1] + f[3];
  double ux = d.freestream_x, uy = d.freestream_y, speed = std::hypot(ux, uy);
  if (!(speed > 0.0)) {
    ux = 1.0;
    uy = 0.0;
    speed = d.reference_speed > 0.0 ? d.reference_speed : 1.0;
  } else {
    ux /= speed;
    uy /= speed;
  }
  const double q = 0.5 * speed * speed * d.chord;
  values[0] = f[0];
  values[1] = f[1];
  values[2] = f[2];
  values[3] = f[3];
  values[4] = fx;
  values[5] = fy;
  values[6] = (fx * ux + fy * uy) / q;   // drag coefficient (along the freestream)
  values[7] = (-fx * uy + fy * ux) / q;  // lift coefficient (freestream turned +90 deg)
  return FB_OK;
}

int32_t fb_compute_mask(fb_ctx *ctx, const fb_scenario_desc *desc, double angle_degrees, uint8_t *host_mask, size_t bytes) {
  if (!ctx || !desc || !host_mask) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  std::string why;
  if (!desc_valid(desc, why)) return set_err(FB_ERR_INVALID_ARGUMENT, "%s", why.c_str());
  const size_t n = (size_t)desc->nx * desc->ny;
  if (bytes != n) return set_err(FB_ERR_INVALID_ARGUMENT, "mask buffer must be %zu bytes", n);
  CK(cudaSetDevice(ctx->device));
  unsigned char *dm = nullptr;
  CK(cudaMallocAsync(&dm, n, ctx->stream));
  const Axis ax = make_axis(desc->x0, desc->x1, desc->nx, desc->periodic_x);
  const Axis ay = make_axis(desc->y0, desc->y1, desc->ny, desc->periodic_y);
  const Foil f = make_foil(desc->naca, desc->chord, desc->pivot_x, desc->pivot_y);
  const double a = deg2rad(angle_degrees);
  mask_kernel<<<grid_of(n), 256, 0, ctx->stream>>>(f, ax, ay, std::cos(a), std::sin(a), dm);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host_mask, dm, n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaFreeAsync(dm, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FB_OK;
}

int32_t fb_naca_signed_distance(fb_ctx *ctx, const char naca[4], double chord, double pivot_x, double pivot_y,
                                const double *points, int64_t n, double angle_degrees, double *out) {
  if (!ctx || !naca || (n > 0 && (!points || !out)) || n < 0) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  for (int i = 0; i < 4; ++i)
    if (naca[i] < '0' || naca[i] > '9') return set_err(FB_ERR_INVALID_ARGUMENT, "NACA code must contain exactly four digits");
  if (n == 0) return FB_OK;
  CK(cudaSetDevice(ctx->device));
  double *dp = nullptr;
  CK(cudaMallocAsync(&dp, sizeof(double) * 3 * n, ctx->stream));
  CK(cudaMemcpyAsync(dp, points, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, ctx->stream));
  const Foil f = make_foil(naca, chord, pivot_x, pivot_y);
  const double a = deg2rad(angle_degrees);
  sdf_kernel<<<(int)((n + 255) / 256), 256, 0, ctx->stream>>>(f, std::cos(a), std::sin(a), dp, n, dp + 2 * n);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dp + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaFreeAsync(dp, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return FB_OK;
}

// ---- operator-level entry points -------------------------------------------------------

int32_t fb_op_advect_velocity(fb_ctx *ctx, const fb_scenario_desc *desc, const void *vel_in, void *vel_out, double dt,
                              int32_t maccormack) {
  if (!vel_in || !vel_out || !std::isfinite(dt)) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  fb_scenario_desc d = *desc;
  d.advection = maccormack ? FB_ADVECT_MACCORMACK : FB_ADVECT_SEMI_LAGRANGIAN;
  fb_solver *s = nullptr;
  int rc = fb_solver_create(ctx, &d, &s);
  if (rc) return rc;
  const Layout &L = s->L;
  const size_t bytes = L.N * 2 * L.vsz;
  do {
    if (cudaMemcpyAsync(s->arena + L.staging, vel_in, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    cells_from_staging(s, ctx->stream);
    if ((rc = reset_report(s))) break;
    if ((rc = launch(s, PH_ADVECT | PH_CELLS_ONLY, dt, 0.0, 0.0, 0.0, 0.0, 0))) break;
    staging_from_result_cells(s, ctx->stream);
    if (cudaMemcpyAsync(vel_out, s->arena + L.staging, bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if ((rc = read_report(s))) break;
    if (s->rep_host->status != ST_OK) rc = set_err(FB_ERR_DEVICE_TIMEOUT, "advection kernel did not complete");
  } while (0);
  if (rc == FB_ERR_CUDA) set_err(rc, "CUDA error in fb_op_advect_velocity: %s", cudaGetErrorString(cudaGetLastError()));
  fb_solver_destroy(s);
  return rc;
}

int32_t fb_op_implicit_diffuse(fb_ctx *ctx, const fb_scenario_desc *desc, const void *vel_in, void *vel_out, double viscosity,
                               double dt, double tolerance, int32_t max_iterations, fb_report *out) {
  if (!vel_in || !vel_out) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  fb_solver *s = nullptr;
  int rc = fb_solver_create(ctx, desc, &s);
  if (rc) return rc;
  if (out) std::memset(out, 0, sizeof(*out));
  const Layout &L = s->L;
  const size_t bytes = L.N * 2 * L.vsz;
  do {
    if (cudaMemcpyAsync(s->arena + L.staging, vel_in, bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    cells_from_staging(s, ctx->stream);
    if ((rc = reset_report(s))) break;
    if ((rc = launch(s, PH_DIFFUSE | PH_CELLS_ONLY, dt, 0.0, 0.0, viscosity, tolerance, max_iterations))) break;
    staging_from_result_cells(s, ctx->stream);
    if (cudaMemcpyAsync(vel_out, s->arena + L.staging, bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if ((rc = read_report(s))) break;
    fill_report_from_dev(*s->rep_host, out);
    if (s->rep_host->status != ST_OK) rc = set_err(FB_ERR_DEVICE_TIMEOUT, "viscosity kernel did not complete");
  } while (0);
  if (rc == FB_ERR_CUDA) set_err(rc, "CUDA error in fb_op_implicit_diffuse");
  fb_solver_destroy(s);
  return rc;
}

int32_t fb_op_solve_masked_poisson(fb_ctx *ctx, const fb_scenario_desc *desc, const double *rhs, const uint8_t *fluid,
                                   double *pressure, fb_report *out) {
  if (!rhs || !fluid || !pressure) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  fb_solver *s = nullptr;
  int rc = fb_solver_create(ctx, desc, &s);
  if (rc) return rc;
  if (out) std::memset(out, 0, sizeof(*out));
  const Layout &L = s->L;
  std::vector<uint8_t> solid(L.N);
  for (size_t i = 0; i < L.N; ++i) solid[i] = fluid[i] ? 0 : 1;
  do {
    if (cudaMemcpyAsync(s->arena + L.b, rhs, L.N * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if (cudaMemcpyAsync(s->arena + L.solid, solid.data(), L.N, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if ((rc = reset_report(s))) break;
    if ((rc = launch(s, PH_PROJECT | PH_RHS_GIVEN | PH_NO_GRADIENT, 1.0, 0.0, 0.0, 0.0, 0.0, 0))) break;
    if (cudaMemcpyAsync(pressure, s->arena + L.x, L.N * 8, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if ((rc = read_report(s))) break;
    fill_report_from_dev(*s->rep_host, out);
    if (out) out->pressure_converged = s->rep_host->cg_info == 0 ? 1 : 0;
    if (s->rep_host->status != ST_OK) rc = numerical_status(s, out);
  } while (0);
  if (rc == FB_ERR_CUDA) set_err(rc, "CUDA error in fb_op_solve_masked_poisson");
  fb_solver_destroy(s);
  return rc;
}

int32_t fb_op_project_faces(fb_ctx *ctx, const fb_scenario_desc *desc, void *u, void *v, const uint8_t *solid,
                            double omega_degrees, double dt, fb_report *out) {
  if (!u || !v || !solid) return set_err(FB_ERR_INVALID_ARGUMENT, "null argument");
  fb_solver *s = nullptr;
  int rc = fb_solver_create(ctx, desc, &s);
  if (rc) return rc;
  if (out) std::memset(out, 0, sizeof(*out));
  const Layout &L = s->L;
  do {
    if (cudaMemcpyAsync(s->arena + L.u, u, L.NU * L.vsz, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if (cudaMemcpyAsync(s->arena + L.v, v, L.NV * L.vsz, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if (cudaMemcpyAsync(s->arena + L.solid, solid, L.N, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if ((rc = reset_report(s))) break;
    if ((rc = launch(s, PH_PROJECT, dt, 0.0, omega_degrees, 0.0, 0.0, 0))) break;
    if ((rc = read_report(s))) break;
    fill_report_from_dev(*s->rep_host, out);
    if (s->rep_host->status != ST_OK) {
      rc = numerical_status(s, out);
      break;
    }
    if (cudaMemcpyAsync(u, s->arena + L.u, L.NU * L.vsz, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if (cudaMemcpyAsync(v, s->arena + L.v, L.NV * L.vsz, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { rc = FB_ERR_CUDA; break; }
  } while (0);
  if (rc == FB_ERR_CUDA) set_err(rc, "CUDA error in fb_op_project_faces");
  fb_solver_destroy(s);
  return rc;
}

}  // extern "C"
