// Persistent, cooperatively launched kernel for one Stable Fluids substep (or a part of
// one, selected by phase bits). All CTAs are co-resident; phases are separated by the
// bounded grid barrier of fb_device.cuh and all data-dependent loops (Jacobi viscosity,
// pressure CG, FP64 defect correction) run on the device, so a substep is one launch.
//
// Reference: PY/solvers/stable_fluids.py:424-494 (substep body) with PY/core/grid.py and
// PY/core/_scipy_adapter.py; PY = implementations/python/src/foilbench_py.
#pragma once

#include "fb_device.cuh"
#include "fb_dst.cuh"
#include "fb_fft.cuh"
#include "fb_umma.cuh"

namespace fb {

enum PhaseBits : unsigned {
  PH_IC = 1u << 0,          // write the initial condition into the cell planes cx, cy
  PH_F2C = 1u << 1,         // cell velocity cx, cy from faces u, v
  PH_MASK = 1u << 2,        // recompute the solid mask at (cos_a, sin_a)
  PH_ADVECT = 1u << 3,      // semi-Lagrangian / MacCormack advection of cx, cy
  PH_DIFFUSE = 1u << 4,     // Jacobi backward-Euler viscosity
  PH_FROM_CELLS = 1u << 5,  // faces u, v from the current cell field
  PH_WALL_FILL = 1u << 6,   // solid cells of the cell field take the wall velocity first
  PH_GUARD = 1u << 7,       // projection guard (finite input, projection CFL)
  PH_PROJECT = 1u << 8,     // BCs, RHS, pressure solve, gradient subtraction
  PH_RHS_GIVEN = 1u << 9,   // pressure solve on a caller RHS in b (no divergence)
  PH_NO_GRADIENT = 1u << 10,// stop after the pressure solve
  PH_FINALIZE = 1u << 11,   // final speed, divergence / leakage postconditions
  PH_SCALAR = 1u << 12,     // passive scalar advected with the first trace
  PH_CELLS_ONLY = 1u << 13, // stop after advection / viscosity (operator entry points)
  PH_FACE = 1u << 14,       // face-centred or skew-RK2 transport and face viscosity into u, v
  PH_MASK_LATE = 1u << 15,  // solid mask at the substep pose after the transport (skew-RK2)
};

enum Scheme : int { SCHEME_REFERENCE = 0, SCHEME_MIXED = 1 };

// Arithmetic type of the velocity stencils (traces, averages, Jacobi, divergence, limiter)
// and storage type of the cell planes (the within-substep cell velocity: faces -> cells,
// advection, Jacobi iterates). With FP64 Krylov vectors (the reference's scheme) it is the
// field type V, so float32 fields reproduce numpy's float32 expressions operation by
// operation, as the reference's float32 path computes them. With FP32 Krylov vectors (the
// mixed scheme) the face velocities stay FP32 in memory, but every stencil is evaluated in
// FP64 and the cell planes are kept in FP64: the float32 expressions of the reference path,
// and FP32 rounding of the cell planes, put their rounding into the divergence, and so into
// the pressure, at several times the size that rounding the faces alone does.
template <class V, class P>
struct StencilArith {
  using type = V;
};
// The mixed scheme is the instantiation with FP32 Krylov vectors.
template <class P>
__host__ __device__ constexpr bool is_mixed() {
  return sizeof(P) == 4;
}
template <>
struct StencilArith<float, float> {
  using type = double;
};

// Reduction slots of the partials array.
enum Slots : int {
  SL_A = 0,   // generic 8-wide block of slots per phase
  SL_B = 8,
  SL_C = 16,
  SL_COUNT = 24
};

template <class V, class P>
struct StepParams {
  int nx, ny;
  Axis ax, ay;
  int channel;
  double fs_x, fs_y;
  Foil foil;
  unsigned phases;
  int initial_condition;
  int maccormack;
  double dt;
  double cos_a, sin_a;  // solid pose
  double omega;         // wall angular velocity (rad/s)
  double nu, vtol;
  int vmaxit;
  double ptol;
  int pmaxit, pfixed, scheme;
  double inner_floor;
  double proj_cfl_limit;
  int singular, dst_precond;
  int skew, face_adv;     // transport: skew-symmetric RK2 / face-centred (PH_FACE)
  // fields
  V *u, *v, *u2, *v2;
  unsigned char *solid;
  typename StencilArith<V, P>::type *cx, *cy, *fx, *fy, *gx, *gy, *hx, *hy;  // cell planes
  V *scal, *scal2;
  double *b, *x, *r64;
  P *r, *z, *pa, *pb, *q, *e, *t;
  DstTables<P> dst;
  ColTables col;
  double dy2;
  FftPlan fft;         // register Stockham plan of the row transforms
  int col_w;           // columns per tridiagonal tile
  int tw_smem_off;     // byte offsets of the shared-memory copies of the FFT twiddles, the
  int filt_smem_off;   // Bluestein filter and the chirp; -1 when read from global memory
  int chirp_smem_off;
  UmmaDst um;          // tensor-core row transforms of the mixed scheme (um.on = 0: FFT)
  double *part;
  GridSync *gs;
  DevReport *rep;
  unsigned long long limit_ns;
  unsigned withhold;          // test hook of grid_sync (0: off)
  unsigned long long *trace;  // optional phase trace: [0] = count, then (tag << 56 | ns)
  int trace_cap;
};

// Phase tags of the optional device trace (CTA 0 stamps %globaltimer after each barrier).
enum TraceTag : unsigned {
  TR_START = 0, TR_P0 = 1, TR_ADVECT = 2, TR_MACCORMACK = 3, TR_JACOBI = 4, TR_GUARD = 5, TR_BC = 6, TR_RHS = 7,
  TR_CG_UPDATE_DST = 8, TR_CG_COLUMN = 9, TR_CG_DST2 = 10, TR_CG_MATVEC = 11, TR_DEFECT = 12, TR_RESIDUAL = 13,
  TR_GRADIENT = 14, TR_FINAL = 15, TR_SCALE = 16, TR_MIXED_INIT = 17, TR_MEAN = 18, TR_FACE = 19,
  TR_CG_UPDATE = 20, TR_CG_TC1 = 21, TR_CG_TC2 = 22, TR_END = 63
};

template <class V, class P>
__device__ __forceinline__ void trace_mark(const StepParams<V, P> &s, unsigned tag) {
  if (s.trace != nullptr && vcta() == 0 && threadIdx.x == 0) {
    const unsigned long long n = s.trace[0];
    if (n + 1 < (unsigned long long)s.trace_cap) {
      s.trace[1 + n] = ((unsigned long long)tag << 56) | (global_ns() & ((1ull << 56) - 1));
      s.trace[0] = n + 1;
    }
  }
}

// ------------------------------------------------------------------------------------------
// small helpers

// Grid-stride walk over a (rows x cols) array carrying (i, j) incrementally: one division
// per walk instead of one per element.
struct Walk {
  int idx, i, j, stride, di, dj, cols, total;
  __device__ __forceinline__ Walk(int start, int stride_, int cols_, int total_)
      : idx(start), stride(stride_), cols(cols_), total(total_) {
    i = start / cols_;
    j = start - i * cols_;
    di = stride_ / cols_;
    dj = stride_ - di * cols_;
  }
  __device__ __forceinline__ bool ok() const { return idx < total; }
  __device__ __forceinline__ void next() {
    idx += stride;
    i += di;
    j += dj;
    if (j >= cols) {
      j -= cols;
      ++i;
    }
  }
};

// Grid-stride walk in batches of U positions, in Walk's order: ld(idx, i, j) runs for every
// position of a batch before op(idx, i, j, operands) runs for any, so a thread keeps U
// independent groups of loads in flight where a plain walk keeps one (the elementwise phases
// are otherwise bound by one memory latency per element). Each thread still visits its
// positions in the same order, so its reduction partials are bitwise those of a plain walk.
template <int U, class T, class Ld, class Op>
__device__ __forceinline__ void walk_batched(Walk w, Ld ld, Op op) {
  while (w.ok()) {
    T o[U];
    int ix[U], ii[U], jj[U];
    int n = 0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (w.ok()) {
        ix[u] = w.idx;
        ii[u] = w.i;
        jj[u] = w.j;
        o[u] = ld(w.idx, w.i, w.j);
        w.next();
        n = u + 1;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (u < n) op(ix[u], ii[u], jj[u], o[u]);
  }
}


template <class V, class P>
__device__ __forceinline__ double cell_x(const StepParams<V, P> &s, int j) {
  return lin_at(j, s.nx, s.ax.start, s.ax.step, s.ax.stop);
}
template <class V, class P>
__device__ __forceinline__ double cell_y(const StepParams<V, P> &s, int i) {
  return lin_at(i, s.ny, s.ay.start, s.ay.step, s.ay.stop);
}

template <class V>
__device__ __forceinline__ bool finite_v(V a) {
  return isfinite((double)a);
}

// Sample a cell-centred plane at a world point (sample_scalar, interpolation.py:55).
template <class V, class P, class T>
__device__ __forceinline__ double sample_cell(const StepParams<V, P> &s, const T *__restrict__ f, double px,
                                              double py) {
  // grid coordinates: the reference divides by the spacing (as numpy does); the mixed scheme,
  // which evaluates its own FP64 stencils, multiplies by the reciprocal (one rounding apart)
  const double gxv = (is_mixed<P>() ? (px - s.ax.lo) * s.ax.ih : (px - s.ax.lo) / s.ax.h) - 0.5;
  const double gyv = (is_mixed<P>() ? (py - s.ay.lo) * s.ay.ih : (py - s.ay.lo) / s.ay.h) - 0.5;
  int ix0, ix1, iy0, iy1;
  double tx, ty;
  sample_coord(gxv, s.nx, s.ax.periodic, ix0, ix1, tx);
  sample_coord(gyv, s.ny, s.ay.periodic, iy0, iy1, ty);
  return bilinear(f, s.nx, iy0, iy1, ix0, ix1, tx, ty);
}

// Midpoint RK2 departure point through the frozen field (fx_, fy_) (grid.py:527-537). The
// velocity samples are rounded to the stencil type A and the dt products formed in A, as numpy
// does with a Python-float coefficient: with A = float the reference's float32 arithmetic.
template <class V, class P, class T>
__device__ __forceinline__ void rk2_trace(const StepParams<V, P> &s, const T *fx_, const T *fy_, double px,
                                          double py, double dt, double &dxp, double &dyp) {
  using A = typename StencilArith<V, P>::type;
  const A k1x = (A)sample_cell(s, fx_, px, py), k1y = (A)sample_cell(s, fy_, px, py);
  const A hdt = (A)(0.5 * dt);
  const double mx = px - (double)(hdt * k1x), my = py - (double)(hdt * k1y);
  const A k2x = (A)sample_cell(s, fx_, mx, my), k2y = (A)sample_cell(s, fy_, mx, my);
  const A vdt = (A)dt;
  dxp = px - (double)(vdt * k2x);
  dyp = py - (double)(vdt * k2y);
}

__device__ __forceinline__ int wrap_or_clamp(int i, int n, int periodic) {
  if (periodic) return i < 0 ? i + n : (i >= n ? i - n : i);
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// Final value of u face (i, j) after apply_domain_boundaries (grid.py:47-78) given the
// pre-boundary face values `uu` (ny x nx+1).
template <class V, class P>
__device__ __forceinline__ V bc_u(const StepParams<V, P> &s, const V *__restrict__ uu, int i, int j,
                                  int channel = -1) {
  const int ld = s.nx + 1;
  const int ch = channel < 0 ? s.channel : channel;
  if (!s.ay.periodic && (i == 0 || i == s.ny - 1)) return ch ? V(0) : (V)s.fs_x;
  if (s.ax.periodic) {
    using A = typename StencilArith<V, P>::type;
    if (j == 0 || j == s.nx) return (V)((A)0.5 * ((A)uu[(size_t)i * ld] + (A)uu[(size_t)i * ld + s.nx]));
    return uu[(size_t)i * ld + j];
  }
  if (j == 0) return (V)s.fs_x;
  if (j == s.nx) return uu[(size_t)i * ld + s.nx - 1];
  return uu[(size_t)i * ld + j];
}

template <class V, class P>
__device__ __forceinline__ V bcx_v(const StepParams<V, P> &s, const V *__restrict__ vv, int i, int j) {
  if (!s.ax.periodic) {
    if (j == 0) return (V)s.fs_y;
    if (j == s.nx - 1) return vv[(size_t)i * s.nx + s.nx - 2];
  }
  return vv[(size_t)i * s.nx + j];
}

template <class V, class P>
__device__ __forceinline__ V bc_v(const StepParams<V, P> &s, const V *__restrict__ vv, int i, int j,
                                  int channel = -1) {
  const int ch = channel < 0 ? s.channel : channel;
  if (i == 0 || i == s.ny) {
    using A = typename StencilArith<V, P>::type;
    if (s.ay.periodic) return (V)((A)0.5 * ((A)bcx_v(s, vv, 0, j) + (A)bcx_v(s, vv, s.ny, j)));
    return ch ? V(0) : (V)s.fs_y;
  }
  return bcx_v(s, vv, i, j);
}

__device__ __forceinline__ bool solid_u_face(const unsigned char *sol, int nx, int i, int j) {
  const unsigned char *row = sol + (size_t)i * nx;
  if (j == 0) return row[0];
  if (j == nx) return row[nx - 1];
  return row[j - 1] | row[j];
}
__device__ __forceinline__ bool solid_v_face(const unsigned char *sol, int nx, int ny, int i, int j) {
  if (i == 0) return sol[j];
  if (i == ny) return sol[(size_t)(ny - 1) * nx + j];
  return sol[(size_t)(i - 1) * nx + j] | sol[(size_t)i * nx + j];
}

// Rigid-rotation wall velocity interpolated to faces (cell_to_faces of wall_velocity_grid):
// the x component depends only on the row and the y component only on the column, so the
// face averages equal the cell values.
template <class V, class P>
__device__ __forceinline__ double wall_u(const StepParams<V, P> &s, int i) {
  return -s.omega * (cell_y(s, i) - s.foil.py);
}
template <class V, class P>
__device__ __forceinline__ double wall_v(const StepParams<V, P> &s, int j) {
  return s.omega * (cell_x(s, j) - s.foil.px);
}

// Masked negative Laplacian (_scipy_adapter.py:31-70) applied at cell (i, j) to a field
// given by a functor f(i, j) -> double.
template <class V, class P, class F>
__device__ __forceinline__ double apply_a(const StepParams<V, P> &s, const unsigned char *__restrict__ sol, int i,
                                          int j, double pc, F f) {
  if (sol[(size_t)i * s.nx + j]) return pc;
  const double ix2 = 1.0 / (s.ax.h * s.ax.h), iy2 = 1.0 / (s.ay.h * s.ay.h);
  double acc = 0.0;
  // x neighbours
  if (j > 0) {
    if (!sol[(size_t)i * s.nx + j - 1]) acc += (pc - f(i, j - 1)) * ix2;
  } else if (s.ax.periodic) {
    if (!sol[(size_t)i * s.nx + s.nx - 1]) acc += (pc - f(i, s.nx - 1)) * ix2;
  } else {
    acc += pc * ix2;
  }
  if (j < s.nx - 1) {
    if (!sol[(size_t)i * s.nx + j + 1]) acc += (pc - f(i, j + 1)) * ix2;
  } else if (s.ax.periodic) {
    if (!sol[(size_t)i * s.nx]) acc += (pc - f(i, 0)) * ix2;
  } else {
    acc += pc * ix2;
  }
  if (i > 0) {
    if (!sol[(size_t)(i - 1) * s.nx + j]) acc += (pc - f(i - 1, j)) * iy2;
  } else if (s.ay.periodic) {
    if (!sol[(size_t)(s.ny - 1) * s.nx + j]) acc += (pc - f(s.ny - 1, j)) * iy2;
  } else {
    acc += pc * iy2;
  }
  if (i < s.ny - 1) {
    if (!sol[(size_t)(i + 1) * s.nx + j]) acc += (pc - f(i + 1, j)) * iy2;
  } else if (s.ay.periodic) {
    if (!sol[j]) acc += (pc - f(0, j)) * iy2;
  } else {
    acc += pc * iy2;
  }
  return acc;
}

// Operands of apply_a for the four cells (i, j0..j0+3) of a field of any precision: the row,
// its y neighbours (16-byte accesses) and the outer x neighbours, with their solid flags.
template <class T>
struct A4Ops {
  T c4[4], d4[4], u4[4], fl, fr;
  uchar4 sc, sd, su;
  unsigned char sl, sr;
};

template <class V, class P, class T>
__device__ __forceinline__ A4Ops<T> a4_load(const StepParams<V, P> &s, const unsigned char *__restrict__ sol,
                                            const T *__restrict__ f, int i, int j0) {
  const int nx = s.nx, ny = s.ny;
  const size_t base = (size_t)i * nx + j0;
  A4Ops<T> o;
#pragma unroll
  for (int k = 0; k < 4; ++k) o.d4[k] = o.u4[k] = T(0);
  ld4(f + base, o.c4);
  o.sc = *reinterpret_cast<const uchar4 *>(sol + base);
  o.sd = o.su = o.sc;
  const bool hd = i > 0 || s.ay.periodic, hu = i < ny - 1 || s.ay.periodic;
  const int id = i > 0 ? i - 1 : ny - 1, iu = i < ny - 1 ? i + 1 : 0;
  if (hd) {
    ld4(f + (size_t)id * nx + j0, o.d4);
    o.sd = *reinterpret_cast<const uchar4 *>(sol + (size_t)id * nx + j0);
  }
  if (hu) {
    ld4(f + (size_t)iu * nx + j0, o.u4);
    o.su = *reinterpret_cast<const uchar4 *>(sol + (size_t)iu * nx + j0);
  }
  const bool hl = j0 > 0 || s.ax.periodic, hr = j0 + 4 < nx || s.ax.periodic;
  const int jl = j0 > 0 ? j0 - 1 : nx - 1, jr = j0 + 4 < nx ? j0 + 4 : 0;
  o.fl = o.fr = T(0);
  o.sl = o.sr = 1;
  if (hl) {
    o.fl = f[(size_t)i * nx + jl];
    o.sl = sol[(size_t)i * nx + jl];
  }
  if (hr) {
    o.fr = f[(size_t)i * nx + jr];
    o.sr = sol[(size_t)i * nx + jr];
  }
  return o;
}

// apply_a for the four cells (i, j0..j0+3) from their loaded operands (nx % 4 == 0). Same
// terms in the same order as apply_a, so results are identical. pc returns f there.
template <class V, class P, class T>
__device__ __forceinline__ void a4_apply(const StepParams<V, P> &s, const A4Ops<T> &o, int i, int j0,
                                         double (&out)[4], double (&pc)[4]) {
  const int nx = s.nx, ny = s.ny;
  const double ix2 = 1.0 / (s.ax.h * s.ax.h), iy2 = 1.0 / (s.ay.h * s.ay.h);
  const bool hd = i > 0 || s.ay.periodic, hu = i < ny - 1 || s.ay.periodic;
  const bool hl = j0 > 0 || s.ax.periodic, hr = j0 + 4 < nx || s.ax.periodic;
  const T(&c4)[4] = o.c4;
  const T(&d4)[4] = o.d4;
  const T(&u4)[4] = o.u4;
  const T fl = o.fl, fr = o.fr;
  const unsigned char sl = o.sl, sr = o.sr;
  const unsigned char scv[4] = {o.sc.x, o.sc.y, o.sc.z, o.sc.w}, sdv[4] = {o.sd.x, o.sd.y, o.sd.z, o.sd.w},
                      suv[4] = {o.su.x, o.su.y, o.su.z, o.su.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double c = (double)c4[k];
    pc[k] = c;
    if (scv[k]) {
      out[k] = c;
      continue;
    }
    const bool lx = k > 0 || hl, rx = k < 3 || hr;
    const double lv = k > 0 ? (double)c4[k - 1] : (double)fl, rv = k < 3 ? (double)c4[k + 1] : (double)fr;
    const unsigned char ls = k > 0 ? scv[k - 1] : sl, rs = k < 3 ? scv[k + 1] : sr;
    double acc = 0.0;
    if (lx) {
      if (!ls) acc += (c - lv) * ix2;
    } else {
      acc += c * ix2;
    }
    if (rx) {
      if (!rs) acc += (c - rv) * ix2;
    } else {
      acc += c * ix2;
    }
    if (hd) {
      if (!sdv[k]) acc += (c - (double)d4[k]) * iy2;
    } else {
      acc += c * iy2;
    }
    if (hu) {
      if (!suv[k]) acc += (c - (double)u4[k]) * iy2;
    } else {
      acc += c * iy2;
    }
    out[k] = acc;
  }
}

// apply_a for the four cells (i, j0..j0+3) of a field f of any precision (nx % 4 == 0), all
// loads issued before any arithmetic.
template <class V, class P, class T>
__device__ __forceinline__ void apply_a4(const StepParams<V, P> &s, const unsigned char *__restrict__ sol,
                                         const T *__restrict__ f, int i, int j0, double (&out)[4], double (&pc)[4]) {
  a4_apply(s, a4_load(s, sol, f, i, j0), i, j0, out, pc);
}

// Diagonal of the masked operator (Jacobi preconditioner for periodic domains).
template <class V, class P>
__device__ __forceinline__ double diag_a(const StepParams<V, P> &s, const unsigned char *__restrict__ sol, int i,
                                         int j) {
  if (sol[(size_t)i * s.nx + j]) return 1.0;
  const double ix2 = 1.0 / (s.ax.h * s.ax.h), iy2 = 1.0 / (s.ay.h * s.ay.h);
  double d = 0.0;
  if (j > 0) d += sol[(size_t)i * s.nx + j - 1] ? 0.0 : ix2;
  else d += s.ax.periodic ? (sol[(size_t)i * s.nx + s.nx - 1] ? 0.0 : ix2) : ix2;
  if (j < s.nx - 1) d += sol[(size_t)i * s.nx + j + 1] ? 0.0 : ix2;
  else d += s.ax.periodic ? (sol[(size_t)i * s.nx] ? 0.0 : ix2) : ix2;
  if (i > 0) d += sol[(size_t)(i - 1) * s.nx + j] ? 0.0 : iy2;
  else d += s.ay.periodic ? (sol[(size_t)(s.ny - 1) * s.nx + j] ? 0.0 : iy2) : iy2;
  if (i < s.ny - 1) d += sol[(size_t)(i + 1) * s.nx + j] ? 0.0 : iy2;
  else d += s.ay.periodic ? (sol[j] ? 0.0 : iy2) : iy2;
  return d;
}

// ---- face-centred and skew-symmetric transport (PY/core/grid.py:306-503) -------------------

// Index and weight along one axis of a face array for sample_staggered_scalar
// (interpolation.py:9-52): periodic axes wrap with the domain period, others clamp to the
// array's extent (one more than the period along the staggered axis).
__device__ __forceinline__ void face_coord(double g, int extent, int period, int periodic, int &i0, int &i1,
                                           double &t) {
  if (!(g == g)) {
    i0 = 0;
    i1 = 0;
    t = g;
    return;
  }
  if (periodic) {
    double m = fmod(g, (double)period);
    if (m < 0.0) m += (double)period;
    g = m;
  } else {
    g = fmin(fmax(g, 0.0), (double)(extent - 1));
  }
  int i = (int)floor(g);
  i = max(0, min(i, extent - 1));
  t = g - (double)i;
  i0 = i;
  i1 = periodic ? (i + 1) % period : min(i + 1, extent - 1);
}

// Bilinear sample of a (rows x cols) face array at a world point with a cell-unit offset.
template <class V, class P, class T>
__device__ __forceinline__ double sample_face(const StepParams<V, P> &s, const T *__restrict__ f, int rows, int cols,
                                              double px, double py, double offx, double offy) {
  const double gx = (is_mixed<P>() ? (px - s.ax.lo) * s.ax.ih : (px - s.ax.lo) / s.ax.h) - offx;
  const double gy = (is_mixed<P>() ? (py - s.ay.lo) * s.ay.ih : (py - s.ay.lo) / s.ay.h) - offy;
  int ix0, ix1, iy0, iy1;
  double tx, ty;
  face_coord(gx, cols, s.nx, s.ax.periodic, ix0, ix1, tx);
  face_coord(gy, rows, s.ny, s.ay.periodic, iy0, iy1, ty);
  return bilinear(f, cols, iy0, iy1, ix0, ix1, tx, ty);
}

// x of u-face column j and y of v-face row i (numpy linspace over the domain bounds).
template <class V, class P>
__device__ __forceinline__ double face_x(const StepParams<V, P> &s, int j) {
  return lin_at(j, s.nx + 1, s.ax.lo, (s.ax.hi - s.ax.lo) / (double)s.nx, s.ax.hi);
}
template <class V, class P>
__device__ __forceinline__ double face_y(const StepParams<V, P> &s, int i) {
  return lin_at(i, s.ny + 1, s.ay.lo, (s.ay.hi - s.ay.lo) / (double)s.ny, s.ay.hi);
}

// centered_derivative (grid.py:379-406) of the field f(i, j) at (i, j) along x or y: periodic
// centred differences (a duplicated periodic endpoint takes the first entry's value), else
// numpy.gradient with second-order one-sided ends. ext: the array's extent along the axis.
template <class V, class F>
__device__ __forceinline__ V cderiv(F f, int i, int j, bool along_x, int ext, int periodic, int dup, double h) {
  const int k = along_x ? j : i;
  auto at = [&](int kk) -> V { return along_x ? f(i, kk) : f(kk, j); };
  if (periodic) {
    const int n = ext - dup;
    const int kk = (dup && k == n) ? 0 : k;
    const int kp = kk + 1 == n ? 0 : kk + 1, km = kk == 0 ? n - 1 : kk - 1;
    return (at(kp) - at(km)) / (V)(2.0 * h);
  }
  if (k == 0) return (V)(-1.5 / h) * at(0) + (V)(2.0 / h) * at(1) + (V)(-0.5 / h) * at(2);
  if (k == ext - 1) return (V)(0.5 / h) * at(ext - 3) + (V)(-2.0 / h) * at(ext - 2) + (V)(1.5 / h) * at(ext - 1);
  return (at(k + 1) - at(k - 1)) / (V)(2.0 * h);
}

// _cross_velocity_on_faces (grid.py:409-432): v at u face (i, j) and u at v face (i, j).
template <class V, class P>
__device__ __forceinline__ typename StencilArith<V, P>::type v_on_u(const StepParams<V, P> &s,
                                                                    const V *__restrict__ v, int i, int j) {
  using A = typename StencilArith<V, P>::type;
  const int nx = s.nx;
  auto cv = [&](int jj) -> A { return (A)0.5 * ((A)v[(size_t)i * nx + jj] + (A)v[(size_t)(i + 1) * nx + jj]); };
  if (j >= 1 && j <= nx - 1) return (A)0.5 * (cv(j - 1) + cv(j));
  if (s.ax.periodic) return (A)0.5 * (cv(nx - 1) + cv(0));
  return j == 0 ? cv(0) : cv(nx - 1);
}
template <class V, class P>
__device__ __forceinline__ typename StencilArith<V, P>::type u_on_v(const StepParams<V, P> &s,
                                                                    const V *__restrict__ u, int i, int j) {
  using A = typename StencilArith<V, P>::type;
  const int ny = s.ny, ld = s.nx + 1;
  auto cu = [&](int ii) -> A { return (A)0.5 * ((A)u[(size_t)ii * ld + j] + (A)u[(size_t)ii * ld + j + 1]); };
  if (i >= 1 && i <= ny - 1) return (A)0.5 * (cu(i - 1) + cu(i));
  if (s.ay.periodic) return (A)0.5 * (cu(ny - 1) + cu(0));
  return i == 0 ? cu(0) : cu(ny - 1);
}

// _skew_symmetric_convection (grid.py:448-481) at u face (i, j) and v face (i, j).
template <class V, class P>
__device__ __forceinline__ typename StencilArith<V, P>::type conv_u(const StepParams<V, P> &s,
                                                                    const V *__restrict__ u, const V *__restrict__ v,
                                                                    int i, int j) {
  using A = typename StencilArith<V, P>::type;
  const int nx = s.nx, ny = s.ny, px = s.ax.periodic, py = s.ay.periodic;
  auto U = [&](int a, int b) -> A { return (A)u[(size_t)a * (nx + 1) + b]; };
  auto UU = [&](int a, int b) -> A { const A x = U(a, b); return x * x; };
  auto VUU = [&](int a, int b) -> A { return v_on_u(s, v, a, b) * U(a, b); };
  const A du_dx = cderiv<A>(U, i, j, true, nx + 1, px, px, s.ax.h);
  const A du_dy = cderiv<A>(U, i, j, false, ny, py, 0, s.ay.h);
  const A adv = U(i, j) * du_dx + v_on_u(s, v, i, j) * du_dy;
  const A con = cderiv<A>(UU, i, j, true, nx + 1, px, px, s.ax.h) + cderiv<A>(VUU, i, j, false, ny, py, 0, s.ay.h);
  return (A)0.5 * (adv + con);
}
template <class V, class P>
__device__ __forceinline__ typename StencilArith<V, P>::type conv_v(const StepParams<V, P> &s,
                                                                    const V *__restrict__ u, const V *__restrict__ v,
                                                                    int i, int j) {
  using A = typename StencilArith<V, P>::type;
  const int nx = s.nx, ny = s.ny, px = s.ax.periodic, py = s.ay.periodic;
  auto W = [&](int a, int b) -> A { return (A)v[(size_t)a * nx + b]; };
  auto UVV = [&](int a, int b) -> A { return u_on_v(s, u, a, b) * W(a, b); };
  auto VV = [&](int a, int b) -> A { const A x = W(a, b); return x * x; };
  const A dv_dx = cderiv<A>(W, i, j, true, nx, px, 0, s.ax.h);
  const A dv_dy = cderiv<A>(W, i, j, false, ny + 1, py, py, s.ay.h);
  const A adv = u_on_v(s, u, i, j) * dv_dx + W(i, j) * dv_dy;
  const A con = cderiv<A>(UVV, i, j, true, nx, px, 0, s.ax.h) + cderiv<A>(VV, i, j, false, ny + 1, py, py, s.ay.h);
  return (A)0.5 * (adv + con);
}

#define FB_SYNC(tag)                                               \
  do {                                                             \
    if (!grid_sync(s.gs, nblocks, s.limit_ns, s.rep, s.withhold)) return; \
    trace_mark(s, tag);                                            \
  } while (0)

#define FB_SYNC_B(tag)                                             \
  do {                                                             \
    if (!grid_sync(s.gs, nblocks, s.limit_ns, s.rep, s.withhold)) return false; \
    trace_mark(s, tag);                                            \
  } while (0)

template <class V, class P>
__device__ __forceinline__ void fail(const StepParams<V, P> &s, int reason, int stage) {
  if (vcta() == 0 && threadIdx.x == 0) {
    s.rep->status = ST_NUMERICAL;
    s.rep->reason = reason;
    s.rep->stage = stage;
  }
}

struct Acc3 {
  double a, b, c;
};

// Row transforms of the rows too long for one shared-memory convolution (double precision,
// over 4096 points): two half convolutions per row (dst_rows_split2), one row per CTA, with
// dst_phase's inputs and outputs (stage 0: t = S(m . r); stage 1: z = S t on fluid cells and
// r on solid ones, returning this CTA's r . z). Out of line so the other transform bodies keep
// their registers.
template <class P, int VPT, int R0>
__device__ __noinline__ double dst_split_phase(DstTables<P> tb, FftPlan pl, int nx, int ny, int nblocks, int stage,
                                               const P *__restrict__ rr, P *__restrict__ tt, P *__restrict__ zz,
                                               const unsigned char *__restrict__ sol) {
  double a2 = 0.0;
  auto in = [&](int row, int n) -> P {
    const size_t idx = (size_t)row * nx + n;
    if (stage) return tt[idx];
    return sol[idx] ? P(0) : rr[idx];
  };
  auto out = [&](int row, int n, P val) {
    const size_t idx = (size_t)row * nx + n;
    if (!stage) {
      tt[idx] = val;
    } else {
      const P rv = rr[idx];
      const P zv = sol[idx] ? rv : val;
      zz[idx] = zv;
      a2 += (double)rv * (double)zv;
    }
  };
  Cx<P> *buf = reinterpret_cast<Cx<P> *>(fb_smem);
  Cx<P> *spec = tb.spec + (size_t)vcta() * 2 * pl.P;
  for (int row = vcta(); row < ny; row += nblocks)
    dst_rows_split2<P, VPT, R0>(tb, pl, buf, spec, row, true, threadIdx.x, in, out);
  return a2;
}

// Both row-transform stages of a CG iteration, out of line with explicit arguments so the
// transform's register allocation is independent of the CG loop's live state.
//   stage 0: CG update of e and r (when upd; or r = src64, e = 0 on the first pass of a
//            mixed inner solve), then t = row DST of m . r; returns (|r|^2, #nonfinite e, 0).
//   stage 1: z = row DST of t, solid cells passing r through; returns (0, 0, r . z).
// Each CTA updates exactly the rows it transforms next, so no grid barrier separates them.
// SHAPE selects the transform: 0, the run-time plan reading inputs and tables from global
// memory; 3, the fixed three-pass shape with the Bluestein tables in the CTA's shared copies;
// 4, the fixed four-pass shape (long rows) with the tables read through the cache. With 3 and
// 4 each row slot stages its inputs in shared memory with bulk asynchronous copies issued one
// row ahead: buffer A holds the transform input (r and the mask for stage 0, t for stage 1),
// buffer B the r row and mask that the stage-1 output needs.
template <class P, int VPT, int R0, int SHAPE>
__device__ __noinline__ Acc3 dst_phase(DstTables<P> tb, FftPlan pl, int nx, int ny, int nblocks, int stage,
                                       int upd, P pal, const double *__restrict__ src64, P *__restrict__ ee,
                                       const P *__restrict__ pin, P *__restrict__ rr, const P *__restrict__ qq,
                                       P *__restrict__ tt, P *__restrict__ zz, const unsigned char *__restrict__ sol,
                                       GridSync *gs, DevReport *rep, unsigned long long limit_ns) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  // row buffers at the start of the dynamic shared memory; with SHAPE 3 the tables are the
  // kernel's shared copies
  constexpr bool ST = SHAPE >= 3;
  Cx<P> *buf = reinterpret_cast<Cx<P> *>(fb_smem);
  if constexpr (SHAPE == 4) {
    tb.tw_lo = reinterpret_cast<const Cx<P> *>(fb_smem + tb.tw2_soff);
    tb.tw_hi = tb.tw_lo + 128;
  }
  if constexpr (SHAPE == 3) {
    tb.twp = reinterpret_cast<const Cx<P> *>(fb_smem + tb.tw_soff);
    tb.filt = reinterpret_cast<const Cx<P> *>(fb_smem + tb.filt_soff);
    tb.chirp = reinterpret_cast<const Cx<P> *>(fb_smem + tb.chirp_soff);
  }
  const int R = pl.rows;
  const int slot = threadIdx.x / pl.tr, tl = threadIdx.x - slot * pl.tr;
  const int rstride = nblocks * R;

  // Rows of round k (k * rstride + ...): slot-major with the fixed three-pass shape, so a CTA's
  // slots take rows nblocks apart and a last, partial round spreads one row over as many CTAs
  // as possible (a lone slot runs faster than two sharing an SM); R consecutive rows per CTA
  // with the other shapes (the long-row shape has one slot per CTA anyway).
  auto row_of = [&](int rbase, int sl) -> int {
    return SHAPE == 3 ? rbase + sl * nblocks + vcta() : rbase + vcta() * R + sl;
  };

  // ---- CG update of every row this CTA transforms. With the three-pass shape a round's R
  // rows form one index space of (slot, element group), so that all threads have work even
  // when rows are short; otherwise the R rows of a round are contiguous.
  if (stage == 0 && (upd || src64)) {
    const int T = blockDim.x;
    if constexpr (SHAPE == 3) {
      const bool vec = upd && (nx & 3) == 0;
      const int gpr = vec ? nx >> 2 : nx;  // element groups per row
      for (int rb = 0; rb < ny; rb += rstride) {
        for (int v = threadIdx.x; v < R * gpr; v += T) {
          const int sl = v / gpr, g = v - sl * gpr;
          const int rw = row_of(rb, sl);
          if (rw >= ny) continue;
          if (vec) {
            const int k = rw * nx + 4 * g;
            P e4[4], p4[4], r4[4], q4[4];
            ld4(ee + k, e4);
            ld4(pin + k, p4);
            ld4(rr + k, r4);
            ld4(qq + k, q4);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              e4[c] = e4[c] + pal * p4[c];
              r4[c] = r4[c] - pal * q4[c];
              a0 += (double)r4[c] * (double)r4[c];
              a1 += isfinite((double)e4[c]) ? 0.0 : 1.0;
            }
            st4(ee + k, e4);
            st4(rr + k, r4);
          } else if (upd) {
            const int k = rw * nx + g;
            const P ev = ee[k] + pal * pin[k];
            ee[k] = ev;
            const P rv = rr[k] - pal * qq[k];
            rr[k] = rv;
            a0 += (double)rv * (double)rv;
            a1 += isfinite((double)ev) ? 0.0 : 1.0;
          } else {
            const int k = rw * nx + g;
            rr[k] = (P)src64[k];
            ee[k] = P(0);
          }
        }
      }
    } else {
      for (int row0 = vcta() * R; row0 < ny; row0 += rstride) {
        const int lo = row0 * nx, hi = min(row0 + R, ny) * nx;
        if (upd && (nx & 3) == 0) {
          for (int k = lo + 4 * threadIdx.x; k < hi; k += 4 * T) {
            P e4[4], p4[4], r4[4], q4[4];
            ld4(ee + k, e4);
            ld4(pin + k, p4);
            ld4(rr + k, r4);
            ld4(qq + k, q4);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              e4[c] = e4[c] + pal * p4[c];
              r4[c] = r4[c] - pal * q4[c];
              a0 += (double)r4[c] * (double)r4[c];
              a1 += isfinite((double)e4[c]) ? 0.0 : 1.0;
            }
            st4(ee + k, e4);
            st4(rr + k, r4);
          }
        } else if (upd) {
          for (int k = lo + threadIdx.x; k < hi; k += T) {
            const P ev = ee[k] + pal * pin[k];
            ee[k] = ev;
            const P rv = rr[k] - pal * qq[k];
            rr[k] = rv;
            a0 += (double)rv * (double)rv;
            a1 += isfinite((double)ev) ? 0.0 : 1.0;
          }
        } else {
          for (int k = lo + threadIdx.x; k < hi; k += T) {
            rr[k] = (P)src64[k];
            ee[k] = P(0);
          }
        }
      }
    }
    if constexpr (ST) fence_proxy_async();  // the bulk copies below read r
    __syncthreads();
  }

  if constexpr (ST) {
    // ---- staged pipeline: one row slot = pl.tr threads, its lead thread issues the copies
    const unsigned vbytes = (unsigned)nx * (unsigned)sizeof(P);
    char *stA = fb_smem + pl.io_soff + (size_t)slot * pl.io_slot;
    char *stB = stA + vbytes + nx;
    unsigned long long *barA = &fb_mbar[2 * slot], *barB = &fb_mbar[2 * slot + 1];
    const bool in_slot = slot < R;
    const bool lead = in_slot && tl == 0;
    unsigned doneA = in_slot ? fb_mbar_uses[2 * slot] : 0u, doneB = in_slot ? fb_mbar_uses[2 * slot + 1] : 0u;
    auto issueA = [&](int row) {
      if (lead) {
        fence_proxy_async();
        const size_t off = (size_t)row * nx;
        mbar_expect_tx(barA, stage ? vbytes : vbytes + (unsigned)nx);
        bulk_copy_g2s(stA, (stage ? tt : rr) + off, vbytes, barA);
        if (!stage) bulk_copy_g2s(stA + vbytes, sol + off, (unsigned)nx, barA);
      }
    };
    auto issueB = [&](int row) {
      if (lead) {
        fence_proxy_async();
        const size_t off = (size_t)row * nx;
        mbar_expect_tx(barB, vbytes + (unsigned)nx);
        bulk_copy_g2s(stB, rr + off, vbytes, barB);
        bulk_copy_g2s(stB + vbytes, sol + off, (unsigned)nx, barB);
      }
    };
    constexpr int M = MainRadix<P>::value, PS = SHAPE == 3 ? R0 * M * M : R0 * M * M * M, TR = PS / VPT;
    Cx<P> *rowbuf = buf + (size_t)(in_slot ? slot : 0) * fft_pad(PS);
    const P *va = reinterpret_cast<const P *>(stA);
    const unsigned char *ma = reinterpret_cast<const unsigned char *>(stA + vbytes);
    const P *vb = reinterpret_cast<const P *>(stB);
    const unsigned char *mb = reinterpret_cast<const unsigned char *>(stB + vbytes);
    {
      const int first = row_of(0, slot);
      if (in_slot && first < ny) {
        issueA(first);
        if (stage) issueB(first);
      }
    }
    for (int rb = (SHAPE == 3 ? 0 : vcta() * R); rb < ny; rb += rstride) {
      const int row = SHAPE == 3 ? row_of(rb, slot) : rb + slot;
      const bool live = in_slot && row < ny;
      if (SHAPE == 3 && !live) break;  // the slot's later rows are past the end too
      const int nxt = row + rstride;
      if (live) {
        mbar_wait(barA, doneA & 1u, limit_ns, gs, rep);
        ++doneA;
      }
      auto in = [&](int, int n) -> P {
        if (stage) return va[n];
        return ma[n] ? P(0) : va[n];
      };
      auto after_in = [&]() {
        slot_sync(slot, TR);  // every thread of the slot has its inputs in registers
        if (live && nxt < ny) issueA(nxt);
      };
      auto before_out = [&]() {
        if (stage && live) {
          mbar_wait(barB, doneB & 1u, limit_ns, gs, rep);
          ++doneB;
        }
      };
      auto out = [&](int rw, int n, P val) {
        const size_t idx = (size_t)rw * nx + n;
        if (!stage) {
          tt[idx] = val;
        } else {
          const P rv = vb[n];
          const P zv = mb[n] ? rv : val;
          zz[idx] = zv;
          a2 += (double)rv * (double)zv;
        }
      };
      if constexpr (SHAPE == 3)
        dst_rows_body3<P, VPT, R0>(tb, rowbuf, in_slot, live, row, tl, slot, in, out, after_in, before_out);
      else
        dst_rows_body4<P, VPT, R0>(tb, rowbuf, in_slot, live, row, tl, slot, in, out, after_in, before_out);
      if (stage) {
        slot_sync(slot, TR);  // buffer B consumed
        if (live && nxt < ny) issueB(nxt);
      }
    }
    if (lead) {
      fb_mbar_uses[2 * slot] = doneA;
      fb_mbar_uses[2 * slot + 1] = doneB;
    }
  } else {
    // ---- direct global reads; rows of the CTA run independently (per-slot barriers)
    auto in = [&](int row, int n) -> P {
      const size_t idx = (size_t)row * nx + n;
      if (stage) return tt[idx];
      return sol[idx] ? P(0) : rr[idx];
    };
    auto out = [&](int row, int n, P val) {
      const size_t idx = (size_t)row * nx + n;
      if (!stage) {
        tt[idx] = val;
      } else {
        const P rv = rr[idx];
        const P zv = sol[idx] ? rv : val;
        zz[idx] = zv;
        a2 += (double)rv * (double)zv;
      }
    };
    if constexpr (sizeof(P) == 8) {
      if (tb.split_h > 0) {
        a2 = dst_split_phase<P, VPT, R0>(tb, pl, nx, ny, nblocks, stage, rr, tt, zz, sol);
        return Acc3{a0, a1, a2};
      }
    }
    for (int row0 = vcta() * R; row0 < ny; row0 += rstride) dst_rows_regs<P, VPT, R0>(tb, pl, buf, row0, ny, in, out);
  }
  (void)tl;
  return Acc3{a0, a1, a2};
}

// CG update ahead of the tensor-core row transform (mixed scheme): e += alpha p and
// r -= alpha q (or r = src64 and e = 0 on an inner solve's first pass), with ||r||^2 and the
// count of non-finite e, and the first transform's data operand: TF32(m . r), x split by
// parity (umma_index). Returns (||r||^2, #nonfinite e, 0).
static __device__ __noinline__ Acc3 cg_update_phase(const UmmaDst um, int nx, int ny, int nblocks, int upd, float pal,
                                             const double *__restrict__ src64, float *__restrict__ ee,
                                             const float *__restrict__ pin, float *__restrict__ rr,
                                             const float *__restrict__ qq, const unsigned char *__restrict__ sol) {
  double a0 = 0.0, a1 = 0.0;
  const int T = blockDim.x;
  const int gtid = vcta() * T + threadIdx.x, gstride = nblocks * T;
  const size_t N = (size_t)nx * ny;
  float *__restrict__ op = um.a1;
  const int nkb = um.nkb;
  // the masked TF32 residual of columns j0 .. j0 + 3 into the operand: columns j0, j0 + 2
  // (odd x) and j0 + 1, j0 + 3 (even x), two adjacent values each
  auto put = [&](int i, int j0, const float (&r4)[4], unsigned f) {
    float m4[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) m4[c] = ((f >> (8 * c)) & 0xffu) ? 0.0f : to_tf32(r4[c]);
    *reinterpret_cast<float2 *>(op + umma_index(nkb, i, 0, j0 >> 1)) = make_float2(m4[0], m4[2]);
    *reinterpret_cast<float2 *>(op + umma_index(nkb, i, 1, j0 >> 1)) = make_float2(m4[1], m4[3]);
  };
  if ((nx & 3) == 0 && upd) {
    // two groups of four per pass, all loads issued before either is used
    for (Walk w_(gtid, gstride, nx >> 2, (int)(N >> 2)); w_.ok();) {
      const int i0 = w_.i, j00 = w_.j << 2;
      w_.next();
      const bool two = w_.ok();
      const int i1 = w_.i, j01 = w_.j << 2;
      if (two) w_.next();
      const size_t k0 = (size_t)i0 * nx + j00, k1 = two ? (size_t)i1 * nx + j01 : k0;
      float e0[4], p0[4], r0[4], q0[4], e1[4], p1[4], r1[4], q1[4];
      ld4(ee + k0, e0);
      ld4(pin + k0, p0);
      ld4(rr + k0, r0);
      ld4(qq + k0, q0);
      ld4(ee + k1, e1);
      ld4(pin + k1, p1);
      ld4(rr + k1, r1);
      ld4(qq + k1, q1);
      const unsigned f0 = *reinterpret_cast<const unsigned *>(sol + k0);
      const unsigned f1 = *reinterpret_cast<const unsigned *>(sol + k1);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        e0[c] = e0[c] + pal * p0[c];
        r0[c] = r0[c] - pal * q0[c];
        a0 += (double)r0[c] * (double)r0[c];
        a1 += isfinite(e0[c]) ? 0.0 : 1.0;
      }
      st4(ee + k0, e0);
      st4(rr + k0, r0);
      put(i0, j00, r0, f0);
      if (two) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          e1[c] = e1[c] + pal * p1[c];
          r1[c] = r1[c] - pal * q1[c];
          a0 += (double)r1[c] * (double)r1[c];
          a1 += isfinite(e1[c]) ? 0.0 : 1.0;
        }
        st4(ee + k1, e1);
        st4(rr + k1, r1);
        put(i1, j01, r1, f1);
      }
    }
  } else if ((nx & 3) == 0) {
    for (Walk w_(gtid, gstride, nx >> 2, (int)(N >> 2)); w_.ok(); w_.next()) {
      const int i = w_.i, j0 = w_.j << 2;
      const size_t k = (size_t)i * nx + j0;
      double s4[4];
      ld4(src64 + k, s4);
      float r4[4];
      const float z4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int c = 0; c < 4; ++c) r4[c] = (float)s4[c];
      st4(rr + k, r4);
      st4(ee + k, z4);
      put(i, j0, r4, *reinterpret_cast<const unsigned *>(sol + k));
    }
  } else {
    for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
      const int idx = w_.idx, i = w_.i, j = w_.j;
      float rv;
      if (upd) {
        const float ev = ee[idx] + pal * pin[idx];
        ee[idx] = ev;
        rv = rr[idx] - pal * qq[idx];
        rr[idx] = rv;
        a0 += (double)rv * (double)rv;
        a1 += isfinite(ev) ? 0.0 : 1.0;
      } else {
        rv = (float)src64[idx];
        rr[idx] = rv;
        ee[idx] = 0.0f;
      }
      op[umma_index(nkb, i, j & 1, j >> 1)] = sol[idx] ? 0.0f : to_tf32(rv);
    }
  }
  return Acc3{a0, a1, 0.0};
}

// The tridiagonal column solves of the preconditioner over this CTA's column tiles (out of
// line so their registers are their own).
// With TC (tensor-core row transforms) the input is the first transform's parity arrays
// (t + io.pe), the output the second transform's operand, and the return value this thread's
// share of y . w (see ColIO).
template <class P, bool TC = false>
__device__ __noinline__ double column_phase(P *t, int nx, int ny, int W, double dy2, ColTables col, int nblocks,
                                            const ColIO io = ColIO{}) {
  P *tile = reinterpret_cast<P *>(fb_smem);
  double *scan = reinterpret_cast<double *>(fb_smem + (((size_t)(ny * W + 512 / W) * sizeof(P) + 15) & ~(size_t)15));
  const int ntiles = (nx + W - 1) / W;
  P *yc = (TC && io.ycopy_soff >= 0) ? reinterpret_cast<P *>(fb_smem + io.ycopy_soff) : nullptr;
  double acc = 0.0;
  // the tile width is a template argument, so tile indexing divides by constants
  switch (W) {
    case 16:
      for (int tti = vcta(); tti < ntiles; tti += nblocks)
        acc += column_solve_tile<P, 16, TC>(t, nx, ny, tti * 16, dy2, col, tile, scan, io, yc);
      break;
    case 8:
      for (int tti = vcta(); tti < ntiles; tti += nblocks)
        acc += column_solve_tile<P, 8, TC>(t, nx, ny, tti * 8, dy2, col, tile, scan, io, yc);
      break;
    case 4:
      for (int tti = vcta(); tti < ntiles; tti += nblocks)
        acc += column_solve_tile<P, 4, TC>(t, nx, ny, tti * 4, dy2, col, tile, scan, io, yc);
      break;
    default:
      for (int tti = vcta(); tti < ntiles; tti += nblocks)
        acc += column_solve_tile<P, 2, TC>(t, nx, ny, tti * 2, dy2, col, tile, scan, io, yc);
      break;
  }
  return acc;
}

// CG direction update and operator: p = z + beta p (p = z on the first pass), q = A p with the
// masked Laplacian of apply_a (same terms, same order), returning p . q over this CTA's cells.
// Out of line with explicit arguments so its registers are its own.
// ZMASK (tensor-core row transforms): z is not masked by its writer, so solid cells (where r,
// and so z, vanish) read 0.
template <class P, bool ZMASK = false>
__device__ __noinline__ double pap_phase(int nx, int ny, double hx, double hy, int perx, int pery, int nblocks,
                                         bool first, P pbeta, const unsigned char *__restrict__ so,
                                         const P *__restrict__ zz, const P *__restrict__ pp, P *__restrict__ po,
                                         P *__restrict__ qo) {
  const int T = blockDim.x;
  const int gtid = vcta() * T + threadIdx.x, gstride = nblocks * T;
  const size_t N = (size_t)nx * ny;
  const double ix2 = 1.0 / (hx * hx), iy2 = 1.0 / (hy * hy);
  const P pix2 = (P)ix2, piy2 = (P)iy2;
  double pq = 0.0;
  auto p1 = [&](int i, int j) -> P {
    const size_t k = (size_t)i * nx + j;
    P zv = zz[k];
    if constexpr (ZMASK) zv = so[k] ? P(0) : zv;
    return first ? zv : (P)fma(pbeta, pp[k], zv);
  };
  if ((nx & 3) == 0) {
    // Row streams: each warp owns a strip of 128 columns (four cells per lane) over a
    // contiguous run of rows, the runs of all warps covering (strip, row) pairs evenly. A
    // lane forms p for the rows below, at and above the current one once, keeps them in
    // registers as it walks up the strip, and has the next two rows' loads in flight, so z,
    // p and the mask are read once per run; left and right neighbours come from the adjacent
    // lanes, the strip's edge lanes load their outer neighbour.
    const int lane = threadIdx.x & 31;
    const int nwarp = nblocks * (T >> 5), gw = vcta() * (T >> 5) + (threadIdx.x >> 5);
    const int nseg = (nx + 127) >> 7;
    const long long S = (long long)nseg * ny;
    long long s0 = S * gw / nwarp;
    const long long s1 = S * (gw + 1) / nwarp;
    struct Raw {
      P z[4], p[4], zl, pl, zr, pr;
      unsigned f;
      unsigned char fl, fr;
    };
    struct Row {
      P c[4];
      unsigned f;
    };
    while (s0 < s1) {
      const int seg = (int)(s0 / ny), ib = (int)(s0 - (long long)seg * ny);
      const int ie = (int)min((long long)ny, ib + (s1 - s0));
      s0 += ie - ib;
      const int j0 = seg * 128 + lane * 4;
      const bool act = j0 < nx;
      const bool hl = j0 > 0 || perx, hr = j0 + 4 < nx || perx;
      // outer neighbours loaded by the strip's edge lanes (-1: from the adjacent lane or none)
      const int el = (lane == 0 && act && hl) ? (j0 > 0 ? j0 - 1 : nx - 1) : -1;
      const int er = ((lane == 31 || j0 + 4 >= nx) && act && hr) ? (j0 + 4 < nx ? j0 + 4 : 0) : -1;
      auto rowof = [&](int r) -> int { return r < 0 ? (pery ? ny - 1 : -1) : (r >= ny ? (pery ? 0 : -1) : r); };
      auto load = [&](Raw &w, int r) {
        const int i = rowof(r);
        if (!act || i < 0) {
#pragma unroll
          for (int k = 0; k < 4; ++k) w.z[k] = w.p[k] = P(0);
          w.zl = w.pl = w.zr = w.pr = P(0);
          w.f = 0u;
          w.fl = w.fr = 1;
          return;
        }
        const size_t rb = (size_t)i * nx;
        ld4(zz + rb + j0, w.z);
        if (!first) ld4(pp + rb + j0, w.p);
        w.f = *reinterpret_cast<const unsigned *>(so + rb + j0);
        if constexpr (ZMASK) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if ((w.f >> (8 * k)) & 0xffu) w.z[k] = P(0);
        }
        w.fl = w.fr = 1;
        if (el >= 0) {
          w.zl = zz[rb + el];
          if constexpr (ZMASK) w.zl = so[rb + el] ? P(0) : w.zl;
          if (!first) w.pl = pp[rb + el];
          w.fl = so[rb + el];
        }
        if (er >= 0) {
          w.zr = zz[rb + er];
          if constexpr (ZMASK) w.zr = so[rb + er] ? P(0) : w.zr;
          if (!first) w.pr = pp[rb + er];
          w.fr = so[rb + er];
        }
      };
      auto pnew = [&](P z, P q) -> P { return first ? z : (P)fma(pbeta, q, z); };
      struct Edge {
        P l, r;
        unsigned char fl, fr;
      };
      auto form = [&](const Raw &w, Row &o) {
#pragma unroll
        for (int k = 0; k < 4; ++k) o.c[k] = pnew(w.z[k], w.p[k]);
        o.f = w.f;
      };
      auto edges = [&](const Raw &w) -> Edge {
        return Edge{el >= 0 ? pnew(w.zl, w.pl) : P(0), er >= 0 ? pnew(w.zr, w.pr) : P(0), w.fl, w.fr};
      };
      const bool own_l = lane == 0, own_r = lane == 31 || j0 + 4 >= nx;
      auto cell_rows = [&](int i, const Row &D, const Row &C, const Row &U, const Edge &e) {
        // left / right neighbours of the lane's cells: adjacent lanes; the edge lanes their loads
        P nl = __shfl_up_sync(0xffffffffu, C.c[3], 1), nr = __shfl_down_sync(0xffffffffu, C.c[0], 1);
        const unsigned gl = __shfl_up_sync(0xffffffffu, C.f, 1), gr = __shfl_down_sync(0xffffffffu, C.f, 1);
        unsigned sl = gl >> 24, sr = gr & 0xffu;
        if (own_l) {
          nl = e.l;
          sl = e.fl;
        }
        if (own_r) {
          nr = e.r;
          sr = e.fr;
        }
        if (!act) return;
        const bool hd = i > 0 || pery, hu = i < ny - 1 || pery;
        P qv4[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          // the operator's terms in the Krylov type: FP64 for the reference scheme (the same
          // terms in the same order as apply_a), FP32 for the mixed scheme's inner solve, whose
          // residual the FP64 defect correction recomputes
          const P c = C.c[k];
          P acc;
          if ((C.f >> (8 * k)) & 0xffu) {
            acc = c;
          } else {
            const bool lx = k > 0 || hl, rx = k < 3 || hr;
            const P lv = k > 0 ? C.c[k - 1] : nl, rv = k < 3 ? C.c[k + 1] : nr;
            const unsigned ls = k > 0 ? (C.f >> (8 * (k - 1))) & 0xffu : sl;
            const unsigned rs = k < 3 ? (C.f >> (8 * (k + 1))) & 0xffu : sr;
            acc = lx ? (ls ? P(0) : (c - lv) * pix2) : c * pix2;
            acc += rx ? (rs ? P(0) : (c - rv) * pix2) : c * pix2;
            acc += hd ? (((D.f >> (8 * k)) & 0xffu) ? P(0) : (c - D.c[k]) * piy2) : c * piy2;
            acc += hu ? (((U.f >> (8 * k)) & 0xffu) ? P(0) : (c - U.c[k]) * piy2) : c * piy2;
          }
          qv4[k] = acc;
          pq += (double)c * (double)acc;
        }
        const size_t base = (size_t)i * nx + j0;
        st4(po + base, C.c);
        st4(qo + base, qv4);
      };
      // rows ib-1 .. ie are read; while row i is computed, rows i+2 and i+3 are in flight
      Raw ra, rb;
      Row D, C, U;
      load(ra, ib - 1);
      load(rb, ib);
      form(ra, D);
      load(ra, ib + 1);
      form(rb, C);
      Edge eC = edges(rb);
      if (ib + 2 <= ie) load(rb, ib + 2);
      for (int i = ib; i < ie; i += 2) {
        // ra holds row i+1, rb row i+2
        form(ra, U);
        Edge eU = edges(ra);
        if (i + 3 <= ie) load(ra, i + 3);
        cell_rows(i, D, C, U, eC);
        D = C;
        C = U;
        eC = eU;
        if (i + 1 >= ie) break;
        form(rb, U);
        eU = edges(rb);
        if (i + 4 <= ie) load(rb, i + 4);
        cell_rows(i + 1, D, C, U, eC);
        D = C;
        C = U;
        eC = eU;
      }
    }
  } else {
    for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
      const int idx = w_.idx, i = w_.i, j = w_.j;
      const P pv = p1(i, j);
      po[idx] = pv;
      const double c = (double)pv;
      double acc;
      if (so[idx]) {
        acc = c;
      } else {
        acc = 0.0;
        if (j > 0) {
          if (!so[idx - 1]) acc += (c - (double)p1(i, j - 1)) * ix2;
        } else if (perx) {
          if (!so[(size_t)i * nx + nx - 1]) acc += (c - (double)p1(i, nx - 1)) * ix2;
        } else {
          acc += c * ix2;
        }
        if (j < nx - 1) {
          if (!so[idx + 1]) acc += (c - (double)p1(i, j + 1)) * ix2;
        } else if (perx) {
          if (!so[(size_t)i * nx]) acc += (c - (double)p1(i, 0)) * ix2;
        } else {
          acc += c * ix2;
        }
        if (i > 0) {
          if (!so[idx - nx]) acc += (c - (double)p1(i - 1, j)) * iy2;
        } else if (pery) {
          if (!so[(size_t)(ny - 1) * nx + j]) acc += (c - (double)p1(ny - 1, j)) * iy2;
        } else {
          acc += c * iy2;
        }
        if (i < ny - 1) {
          if (!so[idx + nx]) acc += (c - (double)p1(i + 1, j)) * iy2;
        } else if (pery) {
          if (!so[j]) acc += (c - (double)p1(0, j)) * iy2;
        } else {
          acc += c * iy2;
        }
      }
      const P qp = (P)acc;
      qo[idx] = qp;
      pq += c * (double)qp;
    }
  }
  return pq;
}

// ------------------------------------------------------------------------------------------
// Uniform control state of the pressure CG, in shared memory: the out-of-line phases get the
// registers their callers leave free, so the CG loop keeps nothing but the kernel parameters
// in registers across a phase call. Written by thread 0 and read after a CTA barrier.
struct CgCtl {
  double rn0, rho, rho_prev, alpha, atol;
  const double *src64;
  int budget, fixed, iters, info, pass, flip, bad;
  int total_it, outer;  // of the whole pressure solve (pressure_solve)
  double final_rn2;     // mixed scheme: ||b - A x64||^2 after the last correction (-1: not kept)
};
static __shared__ CgCtl fb_cg;

// Pressure CG (scipy.sparse.linalg.cg as called at _scipy_adapter.py:134-145) on A e = r0,
// e = 0 initially, operating on P-precision vectors. `src64` (optional) is the FP64 right
// hand side copied into r at the first pass (mixed scheme). Returns false when the kernel
// must stop (barrier abort). On exit fb_cg holds iters, info (0 converged, otherwise the
// budget was hit) and bad (a non-finite iterate or breakdown).
//
// Per iteration (DST preconditioner): [update x, r; ||r||; row DST of m.r] | column solve |
// [row DST -> z; r.z] | [p = z + beta p; q = A p; p.q]. Both row transforms go through one
// call site (stage flag) so the kernel carries a single transform body. With the row
// transforms on the tensor cores (s.um.on, FP32 vectors): [update x, r; ||r||; TF32 m.r] |
// [row DST -> parity arrays t, z] | [column solve of y = t + z; r.z as y.w; z = 0] |
// [row DST accumulated into z] | [p = z + beta p; q = A p; p.q].
template <class V, class P, int VPT, int R0>
__device__ __noinline__ bool pcg_solve(const StepParams<V, P> &s, const DstTables<P> &dstl, unsigned nblocks,
                                       double r0norm2, const double *src64, double atol, int budget, int fixed) {
  if (threadIdx.x == 0) {
    fb_cg.rn0 = r0norm2;
    fb_cg.rho = 0.0;
    fb_cg.rho_prev = 1.0;
    fb_cg.alpha = 0.0;
    fb_cg.atol = atol;
    fb_cg.src64 = src64;
    fb_cg.budget = budget;
    fb_cg.fixed = fixed;
    fb_cg.iters = 0;
    fb_cg.info = budget;
    fb_cg.pass = 0;
    fb_cg.flip = 0;
    fb_cg.bad = 0;
  }
  __syncthreads();
  if (budget <= 0) {  // scipy's loop body never runs; it reports info = maxiter = 0
    if (threadIdx.x == 0) fb_cg.info = 0;
    __syncthreads();
    return true;
  }
  // sets the exit state (thread 0) and returns true after a CTA barrier
  auto finish = [&](int info, bool bad) -> bool {
    if (threadIdx.x == 0) {
      fb_cg.info = info;
      fb_cg.bad = bad ? 1 : 0;
    }
    __syncthreads();
    return true;
  };
  int stage = 0;
  // tensor-core row transforms (mixed scheme, FP32 Krylov vectors)
  const bool tc = sizeof(P) == 4 && s.dst_precond && s.um.on;
  for (;;) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int pass = fb_cg.pass;
    const bool upd = pass > 0;
    P *const pin = fb_cg.flip ? s.pb : s.pa;
    if (s.dst_precond) {
      const P pal = (P)fb_cg.alpha;
      const double *const sr64 = fb_cg.src64;
      Acc3 r3{0.0, 0.0, 0.0};
      if (tc) {
        if constexpr (sizeof(P) == 4) {
          if (stage == 0)
            r3 = cg_update_phase(s.um, s.nx, s.ny, (int)nblocks, upd ? 1 : 0, pal, sr64, s.e, pin, s.r, s.q, s.solid);
          else
            umma_dst_phase(s.um, 1, s.ny, (int)nblocks, s.gs, s.rep, s.limit_ns);
        }
      } else if constexpr (R0 == 0) {
        // batched launch: per-scenario transform shape, always the staged three-pass path
#define FB_DST_CASE(RX)                                                                                            \
  case RX:                                                                                                         \
    r3 = dst_phase<P, VPT, RX, 3>(dstl, s.fft, s.nx, s.ny, (int)nblocks, stage, upd ? 1 : 0, pal, sr64, s.e, pin,   \
                                    s.r, s.q, s.t, s.z, s.solid, s.gs, s.rep, s.limit_ns);                          \
    break;
        switch (s.fft.radix[0]) {
          FB_DST_CASE(2)
          FB_DST_CASE(4)
          FB_DST_CASE(8)
          FB_DST_CASE(16)
          default: break;
        }
#undef FB_DST_CASE
      } else {
        if (dstl.tw_soff >= 0)
          r3 = dst_phase<P, VPT, R0, 3>(dstl, s.fft, s.nx, s.ny, (int)nblocks, stage, upd ? 1 : 0, pal, sr64, s.e,
                                        pin, s.r, s.q, s.t, s.z, s.solid, s.gs, s.rep, s.limit_ns);
        else if (s.fft.io_soff >= 0)
          r3 = dst_phase<P, VPT, R0, 4>(dstl, s.fft, s.nx, s.ny, (int)nblocks, stage, upd ? 1 : 0, pal, sr64, s.e,
                                        pin, s.r, s.q, s.t, s.z, s.solid, s.gs, s.rep, s.limit_ns);
        else
          r3 = dst_phase<P, VPT, R0, 0>(dstl, s.fft, s.nx, s.ny, (int)nblocks, stage, upd ? 1 : 0, pal, sr64, s.e,
                                        pin, s.r, s.q, s.t, s.z, s.solid, s.gs, s.rep, s.limit_ns);
      }
      acc[0] += r3.a;
      acc[1] += r3.b;
      acc[2] += r3.c;
    } else {
      // Jacobi preconditioner (periodic domains): update, z = r / diag and r.z in one pass
      const int nx = s.nx;
      const size_t N = (size_t)nx * s.ny;
      const int gtid = vcta() * blockDim.x + threadIdx.x, gstride = nblocks * blockDim.x;
      const P pal = (P)fb_cg.alpha;
      const double *const sr64 = fb_cg.src64;
      P *__restrict__ rr = s.r;
      P *__restrict__ ee = s.e;
      for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
        const int idx = w_.idx, i = w_.i, j = w_.j;
        P rv;
        if (!upd) {
          if (sr64) {
            rv = (P)sr64[idx];
            rr[idx] = rv;
            ee[idx] = P(0);
          } else {
            rv = rr[idx];
          }
        } else {
          const P ev = ee[idx] + pal * pin[idx];
          ee[idx] = ev;
          rv = rr[idx] - pal * s.q[idx];
          rr[idx] = rv;
          acc[0] += (double)rv * (double)rv;
          acc[1] += isfinite((double)ev) ? 0.0 : 1.0;
        }
        const double d = fmax(diag_a(s, s.solid, i, j), 2.220446049250313e-16);
        const P zv = (P)((double)rv * (1.0 / d));
        s.z[idx] = zv;
        acc[2] += (double)rv * (double)zv;
      }
    }
    const int ops[3] = {OP_SUM, OP_SUM, OP_SUM};
    // (tensor-core transforms: r . z was published by the column phase at SL_B)
    if (!(tc && stage == 1)) cta_publish<3>(acc, ops, fb_red, s.part, stage == 0 ? SL_A : SL_B, nblocks);
    FB_SYNC_B(stage == 0 ? (tc ? TR_CG_UPDATE : TR_CG_UPDATE_DST) : (tc ? TR_CG_TC2 : TR_CG_DST2));
    double tot[3];
    grid_total<3>(s.part, stage == 0 ? SL_A : SL_B, ops, nblocks, fb_red, tot);
    if (stage == 0) {
      int iters = fb_cg.iters;
      const int budget_ = fb_cg.budget, fixed_ = fb_cg.fixed;
      const double rnorm2 = upd ? tot[0] : fb_cg.rn0;
      if (upd) {
        ++iters;
        __syncthreads();  // every thread has read fb_cg.iters
        if (threadIdx.x == 0) fb_cg.iters = iters;
        if (tot[1] != 0.0) return finish(budget_, true);
      }
      if (upd && iters >= budget_) return finish(budget_, false);
      if (fixed_ > 0) {
        if (iters >= fixed_) return finish(0, false);
      } else if (sqrt(rnorm2) < fb_cg.atol) {
        return finish(0, false);
      }
      if (s.dst_precond) {
        // constant-coefficient tridiagonal solve along y for each x wavenumber
        if (tc) {
          if constexpr (sizeof(P) == 4) {
            // y goes to z's buffer (dead until the second transform writes z), and the column
            // solve's output to the first transform's operand (dead after it): a smaller L2
            // working set
            // the first transform writes y's parity arrays t and z (y = t + z); the column solve
            // sums them and zeroes z, into which the second transform accumulates
            umma_dst_phase(s.um, 0, s.ny, (int)nblocks, s.gs, s.rep, s.limit_ns);
            FB_SYNC_B(TR_CG_TC1);
            double rz[3] = {0.0, 0.0,
                            column_phase<P, true>(s.t, s.nx, s.ny, s.col_w, s.dy2, s.col, (int)nblocks,
                                                  ColIO{s.z, s.um.a2, s.um.nkb, s.um.ycopy_soff})};
            const int o3[3] = {OP_SUM, OP_SUM, OP_SUM};
            cta_publish<3>(rz, o3, fb_red, s.part, SL_B, nblocks);
          }
        } else {
          column_phase<P>(s.t, s.nx, s.ny, s.col_w, s.dy2, s.col, (int)nblocks);
        }
        FB_SYNC_B(TR_CG_COLUMN);
        stage = 1;
        continue;
      }
    }
    // ---- E4: p = z + beta p ; q = A p ; pq = p . q
    {
      const double rho = tot[2];
      const int pass_ = fb_cg.pass, flip = fb_cg.flip;
      const double beta = pass_ > 0 ? rho / fb_cg.rho_prev : 0.0;
      __syncthreads();  // every thread has read fb_cg before thread 0 updates it
      if (threadIdx.x == 0) fb_cg.rho = rho;
      double pq;
      if (tc)
        pq = pap_phase<P, true>(s.nx, s.ny, s.ax.h, s.ay.h, s.ax.periodic, s.ay.periodic, (int)nblocks, pass_ == 0,
                                (P)beta, s.solid, s.z, flip ? s.pb : s.pa, flip ? s.pa : s.pb, s.q);
      else
        pq = pap_phase<P>(s.nx, s.ny, s.ax.h, s.ay.h, s.ax.periodic, s.ay.periodic, (int)nblocks, pass_ == 0,
                          (P)beta, s.solid, s.z, flip ? s.pb : s.pa, flip ? s.pa : s.pb, s.q);
      double a2[2] = {pq, isfinite(beta) ? 0.0 : 1.0};
      const int o2[2] = {OP_SUM, OP_MAX};
      cta_publish<2>(a2, o2, fb_red, s.part, SL_C, nblocks);
      FB_SYNC_B(TR_CG_MATVEC);
      double t2[2];
      grid_total<2>(s.part, SL_C, o2, nblocks, fb_red, t2);
      const double rho2 = fb_cg.rho;
      const double alpha = rho2 / t2[0];
      if (!isfinite(alpha) || !isfinite(rho2) || t2[0] == 0.0) return finish(fb_cg.budget, true);
      __syncthreads();  // every thread has read fb_cg.rho
      if (threadIdx.x == 0) {
        fb_cg.alpha = alpha;
        fb_cg.rho_prev = rho2;
        fb_cg.flip ^= 1;
        fb_cg.pass += 1;
      }
      __syncthreads();
    }
    stage = 0;
  }
}

// ---- P7: pressure solve (project_faces, grid.py:148-163): the masked Poisson CG in the
// configured scheme. Out of line, taking only the parameters and ||b||^2, so that none of the
// step's own state is live across it; results in fb_cg (total_it, outer, info). The FFT
// twiddles are read at data-dependent positions by every pass, so each CTA keeps its own copy
// in shared memory. Returns false when the kernel must stop (barrier abort or failure).
template <class V, class P, int VPT, int R0>
__device__ __noinline__ bool pressure_solve(const StepParams<V, P> &s, double bnorm2) {
  char *const smem = fb_smem;
  double *const shm = fb_red;
  const unsigned nblocks = vncta();
  const int T = blockDim.x;
  const int nx = s.nx, ny = s.ny;
  const size_t N = (size_t)nx * ny;
  const int gtid = vcta() * T + threadIdx.x, gstride = nblocks * T;
  DevReport *rep = s.rep;
  const bool lead = vcta() == 0 && threadIdx.x == 0;
  (void)ny;
  DstTables<P> dstl = s.dst;
  if (s.dst_precond) {
    dstl.tw_soff = s.tw_smem_off;
    dstl.filt_soff = s.filt_smem_off;
    dstl.chirp_soff = s.chirp_smem_off;
    if (s.dst.tw2_soff >= 0) {  // two-level twiddles of the long-row path
      Cx<P> *t2 = reinterpret_cast<Cx<P> *>(smem + s.dst.tw2_soff);
      const int n2 = 128 + (s.fft.P >> 7);
      for (int k = threadIdx.x; k < n2; k += T) t2[k] = k < 128 ? s.dst.tw_lo[k] : s.dst.tw_hi[k - 128];
    }
    // mbarriers of the row slots' staging copies (fb_device.cuh), once per launch
    if (s.fft.io_soff >= 0 && fb_mbar_ready == 0 && threadIdx.x < 2 * s.fft.rows) {
      mbar_init(&fb_mbar[threadIdx.x], 1);
      fb_mbar_uses[threadIdx.x] = 0;
      mbar_fence_init();
    }
    if (s.tw_smem_off >= 0) {
      Cx<P> *tws = reinterpret_cast<Cx<P> *>(smem + s.tw_smem_off);
      for (int k = threadIdx.x; k < s.fft.tw_entries; k += T) tws[k] = s.dst.twp[k];
      Cx<P> *fs = reinterpret_cast<Cx<P> *>(smem + s.filt_smem_off);
      for (int k = threadIdx.x; k < s.fft.P; k += T) fs[k] = s.dst.filt[k];
      Cx<P> *cs = reinterpret_cast<Cx<P> *>(smem + s.chirp_smem_off);
      for (int k = threadIdx.x; k <= nx; k += T) cs[k] = s.dst.chirp[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) fb_mbar_ready = 1;
  }
  const double bnorm = sqrt(bnorm2);
  int total_it = 0, info = 0, outer = 0;
  bool bad = false;
  double final_rn2 = bnorm > 0.0 ? -1.0 : 0.0;
  if (bnorm > 0.0) {
    if (s.scheme == SCHEME_REFERENCE) {
      if (!pcg_solve<V, P, VPT, R0>(s, dstl, nblocks, bnorm2, nullptr, 0.9 * s.ptol * bnorm, s.pmaxit, s.pfixed))
        return false;
      total_it = fb_cg.iters;
      info = fb_cg.info;
      bad = fb_cg.bad != 0;
      outer = 1;
    } else {
      // FP64 defect correction around an FP32 CG: r64 = b - A x64 kept in FP64. x64 starts
      // at zero and r64 at b without being written: the first inner solve reads b, and the
      // first correction writes x64 = e and r64 = b - A e.
      double rn2 = bnorm2;
      const double goal = 0.9 * s.ptol * bnorm;
      info = s.pmaxit;
      for (;;) {
        const double rn = sqrt(rn2);
        if (s.pfixed > 0 ? outer >= 1 : rn < goal) {
          info = 0;
          break;
        }
        if (total_it >= s.pmaxit) {
          info = s.pmaxit;
          break;
        }
        const double inner_atol = fmax(0.5 * goal, s.inner_floor * rn);
        const bool first = outer == 0;
        if (!pcg_solve<V, P, VPT, R0>(s, dstl, nblocks, rn2, first ? s.b : s.r64, inner_atol, s.pmaxit - total_it,
                                      s.pfixed))
          return false;
        total_it += fb_cg.iters;
        bad = fb_cg.bad != 0;
        ++outer;
        if (bad) break;
        // x64 += e ; r64 -= A e   (FP64); the first pass starts from x64 = 0, r64 = b
        double g2[2] = {0.0, 0.0};
        const int o2[2] = {OP_SUM, OP_SUM};
        if ((nx & 3) == 0) {
          const P *__restrict__ ep = s.e;
          double *__restrict__ xp = s.x;
          double *__restrict__ rp = s.r64;
          const double *__restrict__ rsrc = first ? s.b : s.r64;
          for (Walk w_(gtid, gstride, nx >> 2, (int)(N >> 2)); w_.ok(); w_.next()) {
            const int i = w_.i, j0 = w_.j << 2;
            const size_t base = (size_t)i * nx + j0;
            double x4[4] = {0.0, 0.0, 0.0, 0.0}, r4[4], ae[4], ev[4];
            if (!first) ld4(xp + base, x4);
            ld4(rsrc + base, r4);
            apply_a4(s, s.solid, ep, i, j0, ae, ev);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              x4[k] = x4[k] + ev[k];
              r4[k] = r4[k] - ae[k];
              g2[0] += r4[k] * r4[k];
              g2[1] += isfinite(x4[k]) ? 0.0 : 1.0;
            }
            st4(xp + base, x4);
            st4(rp + base, r4);
          }
        } else {
          for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
            const int idx = w_.idx, i = w_.i, j = w_.j;
            const double ev = (double)s.e[idx];
            const double xv = (first ? 0.0 : s.x[idx]) + ev;
            s.x[idx] = xv;
            const double ae =
                apply_a(s, s.solid, i, j, ev, [&](int a, int c) { return (double)s.e[(size_t)a * nx + c]; });
            const double rv = (first ? s.b[idx] : s.r64[idx]) - ae;
            s.r64[idx] = rv;
            g2[0] += rv * rv;
            g2[1] += isfinite(xv) ? 0.0 : 1.0;
          }
        }
        cta_publish<2>(g2, o2, shm, s.part, SL_C, nblocks);
        FB_SYNC_B(TR_DEFECT);
        double tot[2];
        grid_total<2>(s.part, SL_C, o2, nblocks, shm, tot);
        rn2 = tot[0];
        final_rn2 = rn2;
        if (tot[1] != 0.0) {
          bad = true;
          break;
        }
      }
      if (outer == 0) {  // no correction ran: the pressure is zero
        for (int k = gtid; k < (int)N; k += gstride) s.x[k] = 0.0;
        FB_SYNC_B(TR_DEFECT);
      }
    }
  } else if (s.scheme != SCHEME_REFERENCE) {  // zero right-hand side: zero pressure
    for (int k = gtid; k < (int)N; k += gstride) s.x[k] = 0.0;
    FB_SYNC_B(TR_DEFECT);
  }
  if (bad) {
    if (lead) {
      rep->cg_iters = total_it;
      rep->cg_outer = outer;
    }
    fail(s, RS_PROJECTION, SG_POSTCONDITION);
    return false;
  }
  __syncthreads();  // every thread has read fb_cg
  if (threadIdx.x == 0) {
    fb_cg.total_it = total_it;
    fb_cg.outer = outer;
    fb_cg.info = info;
    fb_cg.final_rn2 = s.scheme == SCHEME_REFERENCE ? -1.0 : final_rn2;
  }
  __syncthreads();
  return true;
}

// ------------------------------------------------------------------------------------------
template <class V, class P, int VPT, int R0>
__device__ __forceinline__ void step_body(const StepParams<V, P> &s) {
  using A = typename StencilArith<V, P>::type;
  char *const smem = fb_smem;
  double *const shm = fb_red;
  const unsigned nblocks = vncta();
  const int T = blockDim.x;
  const int nx = s.nx, ny = s.ny;
  const size_t N = (size_t)nx * ny;
  const size_t NU = (size_t)ny * (nx + 1), NV = (size_t)(ny + 1) * nx;
  const int gtid = vcta() * T + threadIdx.x, gstride = nblocks * T;
  const unsigned ph = s.phases;
  DevReport *rep = s.rep;
  if (*(volatile int *)&rep->status != ST_OK) return;
  const bool lead = vcta() == 0 && threadIdx.x == 0;
  trace_mark(s, TR_START);

  // ---- P0: initial condition / faces->cells / mask (no advection)
  if (ph & (PH_IC | PH_F2C | PH_MASK)) {
    const bool mask_here = (ph & PH_MASK) && !(ph & PH_ADVECT);
    if ((ph & PH_F2C) && !(ph & PH_IC) && !mask_here) {
      // faces -> cells alone (every substep): four face values per cell, loaded a batch ahead
      struct Ops {
        V ul, ur, vd, vu;
      };
      const V *uu = s.u, *vv = s.v;
      walk_batched<4, Ops>(
          Walk(gtid, gstride, nx, (int)N),
          [&](int, int i, int j) {
            Ops o;
            o.ul = uu[(size_t)i * (nx + 1) + j];
            o.ur = uu[(size_t)i * (nx + 1) + j + 1];
            o.vd = vv[(size_t)i * nx + j];
            o.vu = vv[(size_t)(i + 1) * nx + j];
            return o;
          },
          [&](int idx, int, int, const Ops &o) {
            s.cx[idx] = (A)0.5 * ((A)o.ul + (A)o.ur);
            s.cy[idx] = (A)0.5 * ((A)o.vd + (A)o.vu);
          });
    } else
    for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
      const int idx = w_.idx, i = w_.i, j = w_.j;
      if (ph & PH_IC) {
        // _initial_velocity, stable_fluids.py:102-116
        const double xc = cell_x(s, j), yc = cell_y(s, i);
        double vx = s.fs_x, vy = s.fs_y;
        if (s.initial_condition == 1) {
          vx = sin(xc) * cos(yc);
          vy = -cos(xc) * sin(yc);
        } else if (s.initial_condition == 2) {
          const double rr = 0.5 * (s.ay.hi - s.ay.lo), cc = 0.5 * (s.ay.lo + s.ay.hi);
          const double e = (yc - cc) / rr;
          vx = 1.5 * (1.0 - e * e);
          vy = 0.0;
        }
        s.cx[idx] = (A)vx;
        s.cy[idx] = (A)vy;
      } else if (ph & PH_F2C) {
        const V *uu = s.u, *vv = s.v;
        s.cx[idx] = (A)0.5 * ((A)uu[(size_t)i * (nx + 1) + j] + (A)uu[(size_t)i * (nx + 1) + j + 1]);
        s.cy[idx] = (A)0.5 * ((A)vv[(size_t)i * nx + j] + (A)vv[(size_t)(i + 1) * nx + j]);
      }
      if (mask_here) s.solid[idx] = naca_contains(s.foil, s.cos_a, s.sin_a, cell_x(s, j), cell_y(s, i)) ? 1 : 0;
    }
    FB_SYNC(TR_P0);
  }

  // Cell field that feeds the faces (updated by advection / viscosity below).
  const A *srcx = s.cx, *srcy = s.cy;
  double scale[2] = {1.0, 1.0};
  bool have_scale = false;

  // ---- P1/P2: advection (grid.py:506-524), mask at the substep pose, passive scalar
  if (ph & PH_ADVECT) {
    double mx[2] = {0.0, 0.0};
    const int om[2] = {OP_MAX, OP_MAX};
    for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
      const int idx = w_.idx, i = w_.i, j = w_.j;
      const double px = cell_x(s, j), py = cell_y(s, i);
      double dxp, dyp;
      rk2_trace(s, s.cx, s.cy, px, py, s.dt, dxp, dyp);
      const A fxv = (A)sample_cell(s, s.cx, dxp, dyp), fyv = (A)sample_cell(s, s.cy, dxp, dyp);
      s.fx[idx] = fxv;
      s.fy[idx] = fyv;
      mx[0] = fmax(mx[0], fabs((double)fxv));
      mx[1] = fmax(mx[1], fabs((double)fyv));
      if (ph & PH_SCALAR) s.scal2[idx] = (V)sample_cell(s, s.scal, dxp, dyp);
      if (ph & PH_MASK) s.solid[idx] = naca_contains(s.foil, s.cos_a, s.sin_a, px, py) ? 1 : 0;
    }
    if (!s.maccormack) cta_publish<2>(mx, om, shm, s.part, SL_A, nblocks);
    FB_SYNC(TR_ADVECT);
    srcx = s.fx;
    srcy = s.fy;
    if (s.maccormack) {
      // forward trace of the first estimate, corrector, 3x3 limiter (grid.py:517-524,540-569)
      double mg[2] = {0.0, 0.0};
      for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
        const int idx = w_.idx, i = w_.i, j = w_.j;
        const double px = cell_x(s, j), py = cell_y(s, i);
        double dxp, dyp;
        rk2_trace(s, s.fx, s.fy, px, py, -s.dt, dxp, dyp);
        const A bx = (A)sample_cell(s, s.fx, dxp, dyp), by = (A)sample_cell(s, s.fy, dxp, dyp);
        const A f0x = (A)s.fx[idx], f0y = (A)s.fy[idx];
        A cxv = f0x + (A)0.5 * ((A)s.cx[idx] - bx);
        A cyv = f0y + (A)0.5 * ((A)s.cy[idx] - by);
        A lox = (A)s.cx[idx], hix = lox, loy = (A)s.cy[idx], hiy = loy;
        for (int oy = -1; oy <= 1; ++oy) {
          const int ii = wrap_or_clamp(i + oy, ny, s.ay.periodic);
          for (int ox = -1; ox <= 1; ++ox) {
            const int jj = wrap_or_clamp(j + ox, nx, s.ax.periodic);
            const size_t k = (size_t)ii * nx + jj;
            lox = fmin(lox, (A)s.cx[k]);
            hix = fmax(hix, (A)s.cx[k]);
            loy = fmin(loy, (A)s.cy[k]);
            hiy = fmax(hiy, (A)s.cy[k]);
          }
        }
        lox = fmin(lox, f0x);
        hix = fmax(hix, f0x);
        loy = fmin(loy, f0y);
        hiy = fmax(hiy, f0y);
        cxv = fmin(fmax(cxv, lox), hix);
        cyv = fmin(fmax(cyv, loy), hiy);
        s.gx[idx] = cxv;
        s.gy[idx] = cyv;
        mg[0] = fmax(mg[0], fabs((double)cxv));
        mg[1] = fmax(mg[1], fabs((double)cyv));
      }
      cta_publish<2>(mg, om, shm, s.part, SL_A, nblocks);
      FB_SYNC(TR_MACCORMACK);
      srcx = s.gx;
      srcy = s.gy;
    }
    double tot[2];
    grid_total<2>(s.part, SL_A, om, nblocks, shm, tot);
    scale[0] = fmax(tot[0], 1.0);
    scale[1] = fmax(tot[1], 1.0);
    have_scale = true;
  }

  // ---- P3: Jacobi viscosity (grid.py:183-275), per component with its own stop test
  if (ph & PH_DIFFUSE) {
    if (!have_scale) {
      double mx[2] = {0.0, 0.0};
      const int om[2] = {OP_MAX, OP_MAX};
      for (int idx = gtid; idx < (int)N; idx += gstride) {
        mx[0] = fmax(mx[0], fabs((double)srcx[idx]));
        mx[1] = fmax(mx[1], fabs((double)srcy[idx]));
      }
      cta_publish<2>(mx, om, shm, s.part, SL_A, nblocks);
      FB_SYNC(TR_SCALE);
      double tot[2];
      grid_total<2>(s.part, SL_A, om, nblocks, shm, tot);
      scale[0] = fmax(tot[0], 1.0);
      scale[1] = fmax(tot[1], 1.0);
    }
    int iters[2] = {0, 0};
    double resid[2] = {0.0, 0.0};
    bool done[2] = {true, true};
    const A *orig[2] = {srcx, srcy};
    const A *cur[2] = {srcx, srcy};
    // buffers not aliasing the original field
    A *bufs[2][2];
    if (srcx == s.gx) {
      bufs[0][0] = s.fx; bufs[0][1] = s.hx; bufs[1][0] = s.fy; bufs[1][1] = s.hy;
    } else if (srcx == s.fx) {
      bufs[0][0] = s.gx; bufs[0][1] = s.hx; bufs[1][0] = s.gy; bufs[1][1] = s.hy;
    } else {
      bufs[0][0] = s.fx; bufs[0][1] = s.gx; bufs[1][0] = s.fy; bufs[1][1] = s.gy;
    }
    if (s.nu > 0.0) {
      done[0] = done[1] = false;
      resid[0] = resid[1] = 1.0 / 0.0;
      const double axc = s.nu * s.dt / (s.ax.h * s.ax.h), ayc = s.nu * s.dt / (s.ay.h * s.ay.h);
      const A vax = (A)axc, vay = (A)ayc, vden = (A)(1.0 + 2.0 * axc + 2.0 * ayc);
      for (int it = 1; it <= s.vmaxit && !(done[0] && done[1]); ++it) {
        double dm[4] = {0.0, 0.0, 0.0, 0.0};
        const int o4[4] = {OP_MAX, OP_MAX, OP_SUM, OP_SUM};
        for (int c = 0; c < 2; ++c) {
          if (done[c]) continue;
          const A *cc = cur[c];
          const A *oo = orig[c];
          A *out = bufs[c][(it - 1) & 1];
          double dmax = 0.0, nf = 0.0;
          const bool al16 = ((reinterpret_cast<uintptr_t>(cc) | reinterpret_cast<uintptr_t>(oo) |
                              reinterpret_cast<uintptr_t>(out)) & 15u) == 0;  // caller planes may be unaligned
          if ((nx & 3) == 0 && al16) {
            // four cells per thread, all loads first (same arithmetic as the scalar loop)
            for (Walk w_(gtid, gstride, nx >> 2, (int)(N >> 2)); w_.ok(); w_.next()) {
              const int i = w_.i, j0 = w_.j << 2;
              const size_t base = (size_t)i * nx + j0;
              const int id = wrap_or_clamp(i - 1, ny, s.ay.periodic), iu = wrap_or_clamp(i + 1, ny, s.ay.periodic);
              const int jl = wrap_or_clamp(j0 - 1, nx, s.ax.periodic), jr = wrap_or_clamp(j0 + 4, nx, s.ax.periodic);
              A c4[4], d4[4], u4[4], o4[4], n4[4];
              ld4(cc + base, c4);
              ld4(cc + (size_t)id * nx + j0, d4);
              ld4(cc + (size_t)iu * nx + j0, u4);
              ld4(oo + base, o4);
              const A vl = cc[(size_t)i * nx + jl], vr = cc[(size_t)i * nx + jr];
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const A l = k > 0 ? c4[k - 1] : vl, r = k < 3 ? c4[k + 1] : vr;
                const A nv = (o4[k] + vax * (l + r) + vay * (d4[k] + u4[k])) / vden;
                n4[k] = nv;
                const double df = fabs((double)nv - (double)c4[k]);
                if (df == df) dmax = fmax(dmax, df);
                else nf += 1.0;
              }
              st4(out + base, n4);
            }
          } else {
            for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
              const int idx = w_.idx, i = w_.i, j = w_.j;
              const int jl = wrap_or_clamp(j - 1, nx, s.ax.periodic), jr = wrap_or_clamp(j + 1, nx, s.ax.periodic);
              const int id = wrap_or_clamp(i - 1, ny, s.ay.periodic), iu = wrap_or_clamp(i + 1, ny, s.ay.periodic);
              const A l = cc[(size_t)i * nx + jl], r = cc[(size_t)i * nx + jr];
              const A d = cc[(size_t)id * nx + j], up = cc[(size_t)iu * nx + j];
              const A nv = (oo[idx] + vax * (l + r) + vay * (d + up)) / vden;
              out[idx] = nv;
              const double df = fabs((double)nv - (double)cc[idx]);
              if (df == df) dmax = fmax(dmax, df);
              else nf += 1.0;
            }
          }
          dm[c] = dmax;
          dm[2 + c] = nf;
        }
        cta_publish<4>(dm, o4, shm, s.part, SL_B, nblocks);
        FB_SYNC(TR_JACOBI);
        double tot[4];
        grid_total<4>(s.part, SL_B, o4, nblocks, shm, tot);
        for (int c = 0; c < 2; ++c) {
          if (done[c]) continue;
          iters[c] = it;
          resid[c] = tot[2 + c] != 0.0 ? (0.0 / 0.0) : tot[c] / scale[c];
          cur[c] = bufs[c][(it - 1) & 1];
          if (resid[c] <= s.vtol) done[c] = true;
        }
      }
    }
    const bool conv = (resid[0] <= s.vtol || s.nu <= 0.0) && (resid[1] <= s.vtol || s.nu <= 0.0);
    if (lead) {
      rep->visc_iters = iters[0] > iters[1] ? iters[0] : iters[1];
      const double r0 = s.nu > 0.0 ? resid[0] : 0.0, r1 = s.nu > 0.0 ? resid[1] : 0.0;
      rep->visc_resid = (r0 != r0 || r1 != r1) ? (0.0 / 0.0) : fmax(r0, r1);
      rep->visc_converged = conv ? 1 : 0;
    }
    srcx = cur[0];
    srcy = cur[1];
    if (!conv && !(ph & PH_CELLS_ONLY)) {
      fail(s, RS_CONVERGENCE, SG_VISCOSITY);
      return;
    }
  }
  // ---- P3b: face-centred or skew-RK2 transport, then face viscosity, straight into u, v
  //      (stable_fluids.py:432-466; grid.py:276-503). The six cell planes fx..hy, sized for a
  //      face array, hold the face temporaries.
  if (ph & PH_FACE) {
    const int NUi = (int)NU, NVi = (int)NV, ld = nx + 1;
    // face temporaries in the field type (the planes hold at least that many 8-byte words)
    V *Au = reinterpret_cast<V *>(s.fx), *Av = reinterpret_cast<V *>(s.fy), *Bu = reinterpret_cast<V *>(s.gx),
      *Bv = reinterpret_cast<V *>(s.gy), *Cu = reinterpret_cast<V *>(s.hx), *Cv = reinterpret_cast<V *>(s.hy);
    const V *Tu, *Tv;
    V *J1u, *J1v, *J2u, *J2v;
    if (s.skew) {
      const A h1 = (A)(0.5 * s.dt), h2 = (A)s.dt;
      // midpoint u - dt/2 c(u, v), then domain boundaries (no channel walls) and solid faces at
      // the substep's wall velocity over the pre-substep mask
      for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next())
        Au[w_.idx] = (V)((A)s.u[w_.idx] - h1 * conv_u(s, s.u, s.v, w_.i, w_.j));
      for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next())
        Av[w_.idx] = (V)((A)s.v[w_.idx] - h1 * conv_v(s, s.u, s.v, w_.i, w_.j));
      FB_SYNC(TR_FACE);
      for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next())
        Bu[w_.idx] = solid_u_face(s.solid, nx, w_.i, w_.j) ? (V)wall_u(s, w_.i) : bc_u(s, Au, w_.i, w_.j, 0);
      for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next())
        Bv[w_.idx] = solid_v_face(s.solid, nx, ny, w_.i, w_.j) ? (V)wall_v(s, w_.j) : bc_v(s, Av, w_.i, w_.j, 0);
      FB_SYNC(TR_FACE);
      // full step u - dt c(midpoint), then the same boundary treatment
      for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next())
        Au[w_.idx] = (V)((A)s.u[w_.idx] - h2 * conv_u(s, Bu, Bv, w_.i, w_.j));
      for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next())
        Av[w_.idx] = (V)((A)s.v[w_.idx] - h2 * conv_v(s, Bu, Bv, w_.i, w_.j));
      FB_SYNC(TR_FACE);
      for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next())
        Cu[w_.idx] = solid_u_face(s.solid, nx, w_.i, w_.j) ? (V)wall_u(s, w_.i) : bc_u(s, Au, w_.i, w_.j, 0);
      for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next())
        Cv[w_.idx] = solid_v_face(s.solid, nx, ny, w_.i, w_.j) ? (V)wall_v(s, w_.j) : bc_v(s, Av, w_.i, w_.j, 0);
      FB_SYNC(TR_FACE);
      Tu = Cu;
      Tv = Cv;
      J1u = Au;
      J1v = Av;
      J2u = Bu;
      J2v = Bv;
    } else {
      // first estimate: each face value at the RK2 departure of its centre through the cell
      // velocity (cx, cy)
      for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next()) {
        double dxp, dyp;
        rk2_trace(s, s.cx, s.cy, face_x(s, w_.j), cell_y(s, w_.i), s.dt, dxp, dyp);
        Au[w_.idx] = (V)sample_face(s, s.u, ny, ld, dxp, dyp, 0.0, 0.5);
      }
      for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next()) {
        double dxp, dyp;
        rk2_trace(s, s.cx, s.cy, cell_x(s, w_.j), face_y(s, w_.i), s.dt, dxp, dyp);
        Av[w_.idx] = (V)sample_face(s, s.v, ny + 1, nx, dxp, dyp, 0.5, 0.0);
      }
      FB_SYNC(TR_FACE);
      if (s.maccormack) {
        // cell velocity of the first estimate (cell-shaped, in C)
        for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
          const int i = w_.i, j = w_.j;
          Cu[w_.idx] = (V)((A)0.5 * ((A)Au[(size_t)i * ld + j] + (A)Au[(size_t)i * ld + j + 1]));
          Cv[w_.idx] = (V)((A)0.5 * ((A)Av[(size_t)i * nx + j] + (A)Av[(size_t)(i + 1) * nx + j]));
        }
        FB_SYNC(TR_FACE);
        // forward trace, corrector and the 3x3 edge-padded limiter of the original faces
        auto limit = [&](const V *f, int rows, int cols, int i, int j, A x) -> V {
          A lo = (A)f[(size_t)i * cols + j], hi = lo;
          for (int oy = -1; oy <= 1; ++oy) {
            const int ii = min(max(i + oy, 0), rows - 1);
            for (int ox = -1; ox <= 1; ++ox) {
              const int jj = min(max(j + ox, 0), cols - 1);
              const A q = (A)f[(size_t)ii * cols + jj];
              lo = fmin(lo, q);
              hi = fmax(hi, q);
            }
          }
          return (V)fmin(fmax(x, lo), hi);
        };
        for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next()) {
          double dxp, dyp;
          rk2_trace(s, (const V *)Cu, (const V *)Cv, face_x(s, w_.j), cell_y(s, w_.i), -s.dt, dxp, dyp);
          const A back = (A)sample_face(s, (const V *)Au, ny, ld, dxp, dyp, 0.0, 0.5);
          const A corr = (A)Au[w_.idx] + (A)0.5 * ((A)s.u[w_.idx] - back);
          Bu[w_.idx] = limit(s.u, ny, ld, w_.i, w_.j, corr);
        }
        for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next()) {
          double dxp, dyp;
          rk2_trace(s, (const V *)Cu, (const V *)Cv, cell_x(s, w_.j), face_y(s, w_.i), -s.dt, dxp, dyp);
          const A back = (A)sample_face(s, (const V *)Av, ny + 1, nx, dxp, dyp, 0.5, 0.0);
          const A corr = (A)Av[w_.idx] + (A)0.5 * ((A)s.v[w_.idx] - back);
          Bv[w_.idx] = limit(s.v, ny + 1, nx, w_.i, w_.j, corr);
        }
        FB_SYNC(TR_FACE);
        Tu = Bu;
        Tv = Bv;
        J1u = Au;
        J1v = Av;
        J2u = Cu;
        J2v = Cv;
      } else {
        Tu = Au;
        Tv = Av;
        J1u = Bu;
        J1v = Bv;
        J2u = Cu;
        J2v = Cv;
      }
    }
    // implicit_diffuse_faces: Jacobi on each face array's logical part (a periodic axis drops
    // the duplicated endpoint and restores it at the end), per component stop test
    const int rows_l[2] = {ny, ny + 1 - (s.ay.periodic ? 1 : 0)};
    const int cols_l[2] = {nx + 1 - (s.ax.periodic ? 1 : 0), nx};
    const int lds[2] = {ld, nx};
    const V *orig[2] = {Tu, Tv};
    const V *cur[2] = {Tu, Tv};
    V *pp[2][2] = {{J1u, J2u}, {J1v, J2v}};
    int iters[2] = {0, 0};
    double resid[2] = {0.0, 0.0};
    bool done[2] = {true, true};
    if (s.nu > 0.0) {
      double mx[2] = {0.0, 0.0};
      const int om[2] = {OP_MAX, OP_MAX};
      for (int c = 0; c < 2; ++c)
        for (Walk w_(gtid, gstride, cols_l[c], rows_l[c] * cols_l[c]); w_.ok(); w_.next())
          mx[c] = fmax(mx[c], fabs((double)orig[c][(size_t)w_.i * lds[c] + w_.j]));
      cta_publish<2>(mx, om, shm, s.part, SL_A, nblocks);
      FB_SYNC(TR_SCALE);
      double sc2[2];
      grid_total<2>(s.part, SL_A, om, nblocks, shm, sc2);
      const double scale[2] = {fmax(sc2[0], 1.0), fmax(sc2[1], 1.0)};
      done[0] = done[1] = false;
      resid[0] = resid[1] = 1.0 / 0.0;
      const double axc = s.nu * s.dt / (s.ax.h * s.ax.h), ayc = s.nu * s.dt / (s.ay.h * s.ay.h);
      const A vax = (A)axc, vay = (A)ayc, vden = (A)(1.0 + 2.0 * axc + 2.0 * ayc);
      for (int it = 1; it <= s.vmaxit && !(done[0] && done[1]); ++it) {
        double dm[4] = {0.0, 0.0, 0.0, 0.0};
        const int o4[4] = {OP_MAX, OP_MAX, OP_SUM, OP_SUM};
        for (int c = 0; c < 2; ++c) {
          if (done[c]) continue;
          const int R = rows_l[c], C = cols_l[c], L = lds[c];
          const V *cc = cur[c];
          const V *oo = orig[c];
          V *out = pp[c][(it - 1) & 1];
          double dmax = 0.0, nf = 0.0;
          for (Walk w_(gtid, gstride, C, R * C); w_.ok(); w_.next()) {
            const int i = w_.i, j = w_.j;
            const int jl = wrap_or_clamp(j - 1, C, s.ax.periodic), jr = wrap_or_clamp(j + 1, C, s.ax.periodic);
            const int id = wrap_or_clamp(i - 1, R, s.ay.periodic), iu = wrap_or_clamp(i + 1, R, s.ay.periodic);
            const size_t k = (size_t)i * L + j;
            const A l = cc[(size_t)i * L + jl], r = cc[(size_t)i * L + jr];
            const A d = cc[(size_t)id * L + j], up = cc[(size_t)iu * L + j];
            const V nv = (V)(((A)oo[k] + vax * (l + r) + vay * (d + up)) / vden);
            out[k] = nv;
            const double df = fabs((double)nv - (double)cc[k]);
            if (df == df) dmax = fmax(dmax, df);
            else nf += 1.0;
          }
          dm[c] = dmax;
          dm[2 + c] = nf;
        }
        cta_publish<4>(dm, o4, shm, s.part, SL_B, nblocks);
        FB_SYNC(TR_JACOBI);
        double tot[4];
        grid_total<4>(s.part, SL_B, o4, nblocks, shm, tot);
        for (int c = 0; c < 2; ++c) {
          if (done[c]) continue;
          iters[c] = it;
          resid[c] = tot[2 + c] != 0.0 ? (0.0 / 0.0) : tot[c] / scale[c];
          cur[c] = pp[c][(it - 1) & 1];
          if (resid[c] <= s.vtol) done[c] = true;
        }
      }
    }
    const bool conv = (resid[0] <= s.vtol || s.nu <= 0.0) && (resid[1] <= s.vtol || s.nu <= 0.0);
    if (lead) {
      rep->visc_iters = iters[0] > iters[1] ? iters[0] : iters[1];
      const double r0 = s.nu > 0.0 ? resid[0] : 0.0, r1 = s.nu > 0.0 ? resid[1] : 0.0;
      rep->visc_resid = (r0 != r0 || r1 != r1) ? (0.0 / 0.0) : fmax(r0, r1);
      rep->visc_converged = conv ? 1 : 0;
    }
    if (!conv) {
      fail(s, RS_CONVERGENCE, SG_VISCOSITY);
      return;
    }
    // result into u, v (duplicated periodic endpoints restored); the skew transport's solid
    // mask moves to the substep pose only now
    for (Walk w_(gtid, gstride, ld, NUi); w_.ok(); w_.next()) {
      const int j = (s.ax.periodic && w_.j == nx) ? 0 : w_.j;
      s.u[w_.idx] = cur[0][(size_t)w_.i * ld + j];
    }
    for (Walk w_(gtid, gstride, nx, NVi); w_.ok(); w_.next()) {
      const int i = (s.ay.periodic && w_.i == ny) ? 0 : w_.i;
      s.v[w_.idx] = cur[1][(size_t)i * nx + w_.j];
    }
    if (ph & PH_MASK_LATE)
      for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next())
        s.solid[w_.idx] = naca_contains(s.foil, s.cos_a, s.sin_a, cell_x(s, w_.j), cell_y(s, w_.i)) ? 1 : 0;
    FB_SYNC(TR_FACE);
  }

  if (ph & PH_CELLS_ONLY) {
    // operator entry points: leave the result in the cell planes hx, hy
    if (srcx != s.hx) {
      for (int idx = gtid; idx < (int)N; idx += gstride) {
        s.hx[idx] = srcx[idx];
        s.hy[idx] = srcy[idx];
      }
    }
    return;
  }

  // ---- P4: faces from cells (cell_to_faces, grid.py:32-44) and the projection guard
  //      (stable_fluids.py:268-298)
  if (ph & (PH_FROM_CELLS | PH_GUARD)) {
    const bool fill = (ph & PH_WALL_FILL) != 0;
    double g[4] = {0.0, 0.0, 0.0, 0.0};  // nonfinite count, max|u|, max|v|, max wall speed on solids
    const int og[4] = {OP_SUM, OP_MAX, OP_MAX, OP_MAX};
    // the two cells of a face (the same cell at a domain edge) and their solid flags are
    // loaded up front; with the wall fill, a solid cell contributes the rigid-rotation wall
    // velocity instead of its value (cell_to_faces of the wall-filled field)
    const bool from_cells = (ph & PH_FROM_CELLS) != 0;
    struct Ops {
      A a, b;  // the face's two cells (from_cells) or the face value itself (a)
      unsigned char sa, sb;
    };
    walk_batched<4, Ops>(
        Walk(gtid, gstride, nx + 1, (int)NU),
        [&](int idx, int i, int j) {
          Ops o;
          if (from_cells) {
            const size_t rb = (size_t)i * nx;
            const int jl = j > 0 ? j - 1 : 0, jr = j < nx ? j : nx - 1;
            o.a = srcx[rb + jl];
            o.b = srcx[rb + jr];
            o.sa = s.solid[rb + jl];
            o.sb = s.solid[rb + jr];
          } else {
            o.a = (A)s.u[idx];
            o.b = A(0);
            o.sa = o.sb = 0;
          }
          return o;
        },
        [&](int idx, int i, int j, const Ops &o) {
          V uv;
          if (from_cells) {
            const A w = fill ? (A)wall_u(s, i) : A(0);
            const A cl = (fill && o.sa) ? w : o.a, cr = (fill && o.sb) ? w : o.b;
            uv = (V)((j == 0 || j == nx) ? (j == 0 ? cr : cl) : (A)0.5 * (cl + cr));
            s.u[idx] = uv;
          } else {
            uv = (V)o.a;
          }
          if (!finite_v(uv)) g[0] += 1.0;
          else g[1] = fmax(g[1], fabs((double)uv));
        });
    walk_batched<4, Ops>(
        Walk(gtid, gstride, nx, (int)NV),
        [&](int idx, int i, int j) {
          Ops o;
          if (from_cells) {
            const int id = i > 0 ? i - 1 : 0, iu = i < ny ? i : ny - 1;
            o.a = srcy[(size_t)id * nx + j];
            o.b = srcy[(size_t)iu * nx + j];
            o.sa = s.solid[(size_t)id * nx + j];
            o.sb = s.solid[(size_t)iu * nx + j];
          } else {
            o.a = (A)s.v[idx];
            o.b = A(0);
            o.sa = o.sb = 0;
          }
          return o;
        },
        [&](int idx, int i, int j, const Ops &o) {
          V vv;
          if (from_cells) {
            const A w = fill ? (A)wall_v(s, j) : A(0);
            const A cd = (fill && o.sa) ? w : o.a, cu = (fill && o.sb) ? w : o.b;
            vv = (V)((i == 0 || i == ny) ? (i == 0 ? cu : cd) : (A)0.5 * (cd + cu));
            s.v[idx] = vv;
          } else {
            vv = (V)o.a;
          }
          if (!finite_v(vv)) g[0] += 1.0;
          else g[2] = fmax(g[2], fabs((double)vv));
        });
    walk_batched<8, unsigned char>(
        Walk(gtid, gstride, nx, (int)N), [&](int idx, int, int) { return s.solid[idx]; },
        [&](int, int i, int j, unsigned char sol) {
          if (!sol) return;
          const double wx = wall_u(s, i), wy = wall_v(s, j);
          g[3] = fmax(g[3], sqrt(wx * wx + wy * wy));
        });
    cta_publish<4>(g, og, shm, s.part, SL_C, nblocks);
    FB_SYNC(TR_GUARD);
    double tot[4];
    grid_total<4>(s.part, SL_C, og, nblocks, shm, tot);
    if (ph & PH_GUARD) {
      const double face_speed = fmax(tot[1], tot[2]);
      const double cfl = fmax(face_speed, tot[3]) * s.dt / fmin(s.ax.h, s.ay.h);
      if (lead) {
        rep->face_speed = face_speed;
        rep->wall_speed = tot[3];
        rep->proj_cfl = cfl;
      }
      if (tot[0] != 0.0) {
        fail(s, RS_NONFINITE, SG_PROJECTION);
        return;
      }
      if (cfl > s.proj_cfl_limit) {
        if (lead) {
          rep->ev[0] = cfl;
          rep->ev[1] = s.proj_cfl_limit;
        }
        fail(s, RS_EXCESSIVE_VELOCITY, SG_PROJECTION);
        return;
      }
    }
  }

  if (!(ph & PH_PROJECT)) return;

  // ---- P5: boundary conditions and solid faces on a copy (grid.py:146-147)
  if (!(ph & PH_RHS_GIVEN)) {
    // As in the gradient phase: each face's operands are loaded up front at valid indices and
    // the cases of solid_u_face / bc_u (solid_v_face / bc_v) select among them afterwards.
    const bool px = s.ax.periodic;
    const int ld = nx + 1;
    struct Ops {
      unsigned char sa, sb;
      V a, b;
    };
    walk_batched<4, Ops>(
        Walk(gtid, gstride, nx + 1, (int)NU),
        [&](int, int i, int j) {
          Ops o;
          const unsigned char *srow = s.solid + (size_t)i * nx;
          o.sa = srow[j > 0 ? j - 1 : 0];
          o.sb = srow[j < nx ? j : nx - 1];
          const bool pedge = px && (j == 0 || j == nx);
          const int ca = pedge ? 0 : (j == nx ? nx - 1 : j);
          o.a = s.u[(size_t)i * ld + ca];
          o.b = s.u[(size_t)i * ld + nx];
          return o;
        },
        [&](int idx, int i, int j, const Ops &o) {
          const bool pedge = px && (j == 0 || j == nx);
          V val;
          if (o.sa | o.sb) val = (V)wall_u(s, i);
          else if (!s.ay.periodic && (i == 0 || i == ny - 1)) val = s.channel ? V(0) : (V)s.fs_x;
          else if (pedge) val = (V)((A)0.5 * ((A)o.a + (A)o.b));
          else if (!px && j == 0) val = (V)s.fs_x;
          else val = o.a;
          s.u2[idx] = val;
        });
    if (!s.ay.periodic) {
      walk_batched<4, Ops>(
          Walk(gtid, gstride, nx, (int)NV),
          [&](int, int i, int j) {
            Ops o;
            const int ia = i > 0 ? i - 1 : 0, ib = i < ny ? i : ny - 1;
            o.sa = s.solid[(size_t)ia * nx + j];
            o.sb = s.solid[(size_t)ib * nx + j];
            int c = (!px && j == nx - 1) ? nx - 2 : j;
            c = c < 0 ? 0 : c;
            o.a = s.v[(size_t)i * nx + c];
            o.b = V(0);
            return o;
          },
          [&](int idx, int i, int j, const Ops &o) {
            V val;
            if (o.sa | o.sb) val = (V)wall_v(s, j);
            else if (i == 0 || i == ny) val = s.channel ? V(0) : (V)s.fs_y;
            else if (!px && j == 0) val = (V)s.fs_y;
            else val = o.a;
            s.v2[idx] = val;
          });
    } else {
      for (Walk w_(gtid, gstride, nx, (int)NV); w_.ok(); w_.next()) {
        const int idx = w_.idx, i = w_.i, j = w_.j;
        s.v2[idx] = solid_v_face(s.solid, nx, ny, i, j) ? (V)wall_v(s, j) : bc_v(s, s.v, i, j);
      }
    }
    FB_SYNC(TR_BC);
  }

  // ---- P6: divergence -> RHS (grid.py:148-150), compatible RHS and its guards
  //      (_scipy_adapter.py:108-120)
  double bnorm2;
  {
    double g[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // nonfinite, max|b|, |b|^2, sum fluid b, fluid count
    const int og[5] = {OP_SUM, OP_MAX, OP_SUM, OP_SUM, OP_SUM};
    const A vdx = (A)s.ax.h, vdy = (A)s.ay.h, vdt = (A)fmax(s.dt, 1.0e-12);
    struct Ops {
      V ul, ur, vd, vu;
      double bg;
      unsigned char sol;
    };
    const bool given = (ph & PH_RHS_GIVEN) != 0;
    walk_batched<4, Ops>(
        Walk(gtid, gstride, nx, (int)N),
        [&](int idx, int i, int j) {
          Ops o;
          o.sol = s.solid[idx];
          if (given) {
            o.bg = s.b[idx];
            o.ul = o.ur = o.vd = o.vu = V(0);
          } else {
            o.bg = 0.0;
            o.ul = s.u2[(size_t)i * (nx + 1) + j];
            o.ur = s.u2[(size_t)i * (nx + 1) + j + 1];
            o.vd = s.v2[(size_t)i * nx + j];
            o.vu = s.v2[(size_t)(i + 1) * nx + j];
          }
          return o;
        },
        [&](int idx, int, int, const Ops &o) {
          double bv;
          if (given) {
            bv = o.sol ? 0.0 : o.bg;
          } else {
            const A du = (A)o.ur - (A)o.ul;
            const A dv = (A)o.vu - (A)o.vd;
            const A div = du / vdx + dv / vdy;
            bv = o.sol ? 0.0 : (double)(-div / vdt);
          }
          s.b[idx] = bv;
          if (s.scheme == SCHEME_REFERENCE) {
            s.x[idx] = 0.0;
            s.r[idx] = (P)bv;
          }
          if (!isfinite(bv)) g[0] += 1.0;
          else g[1] = fmax(g[1], fabs(bv));
          g[2] += bv * bv;
          if (!o.sol) {
            g[3] += bv;
            g[4] += 1.0;
          }
        });
    cta_publish<5>(g, og, shm, s.part, SL_A, nblocks);
    FB_SYNC(TR_RHS);
    double tot[5];
    grid_total<5>(s.part, SL_A, og, nblocks, shm, tot);
    bnorm2 = tot[2];
    if (s.singular && tot[4] > 0.0) {
      const double mean = tot[3] / tot[4];
      double g2[3] = {0.0, 0.0, 0.0};
      const int o3[3] = {OP_SUM, OP_MAX, OP_SUM};
      for (int idx = gtid; idx < (int)N; idx += gstride) {
        double bv = s.b[idx];
        if (!s.solid[idx]) bv -= mean;
        s.b[idx] = bv;
        if (s.scheme == SCHEME_REFERENCE) s.r[idx] = (P)bv;
        if (!isfinite(bv)) g2[0] += 1.0;
        else g2[1] = fmax(g2[1], fabs(bv));
        g2[2] += bv * bv;
      }
      cta_publish<3>(g2, o3, shm, s.part, SL_B, nblocks);
      FB_SYNC(TR_RHS);
      double t3[3];
      grid_total<3>(s.part, SL_B, o3, nblocks, shm, t3);
      tot[0] = t3[0];
      tot[1] = t3[1];
      bnorm2 = t3[2];
    }
    if (tot[0] != 0.0) {
      fail(s, RS_NONFINITE, SG_POSTCONDITION);
      return;
    }
    if (tot[1] > 0.25 * sqrt(1.7976931348623157e308 / (double)(N > 0 ? N : 1))) {
      fail(s, RS_PROJECTION, SG_POSTCONDITION);
      return;
    }
  }

  // ---- P7: pressure CG (pressure_solve)
  if (!pressure_solve<V, P, VPT, R0>(s, bnorm2)) return;
  const double bnorm = sqrt(bnorm2);
  const int total_it = fb_cg.total_it, outer = fb_cg.outer, info = fb_cg.info;

  // ---- P8: (singular) mean removal, true residual ||b - A x|| / ||b||
  if (s.singular && bnorm > 0.0) {
    double g2[2] = {0.0, 0.0};
    const int o2[2] = {OP_SUM, OP_SUM};
    for (int idx = gtid; idx < (int)N; idx += gstride)
      if (!s.solid[idx]) {
        g2[0] += s.x[idx];
        g2[1] += 1.0;
      }
    cta_publish<2>(g2, o2, shm, s.part, SL_A, nblocks);
    FB_SYNC(TR_MEAN);
    double tot[2];
    grid_total<2>(s.part, SL_A, o2, nblocks, shm, tot);
    if (tot[1] > 0.0) {
      const double mean = tot[0] / tot[1];
      for (int idx = gtid; idx < (int)N; idx += gstride)
        if (!s.solid[idx]) s.x[idx] -= mean;
      FB_SYNC(TR_MEAN);
    }
  }
  double rel;
  {
    double g2[2] = {0.0, 0.0};
    const int o2[2] = {OP_SUM, OP_SUM};
    // The mixed scheme's defect correction already holds r64 = b - A x64 in FP64 and checked
    // x64 for non-finite values; without a later mean removal its norm is the true residual.
    const double kept = fb_cg.final_rn2;
    const bool have = kept >= 0.0 && !s.singular;
    if (have) {
      // nothing to sweep
    } else if ((nx & 3) == 0) {
      for (Walk w_(gtid, gstride, nx >> 2, (int)(N >> 2)); w_.ok(); w_.next()) {
        const int i = w_.i, j0 = w_.j << 2;
        double b4[4], ax4[4], x4[4];
        ld4(s.b + (size_t)i * nx + j0, b4);
        apply_a4(s, s.solid, (const double *)s.x, i, j0, ax4, x4);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double rv = b4[k] - ax4[k];
          g2[0] += rv * rv;
          g2[1] += isfinite(x4[k]) ? 0.0 : 1.0;
        }
      }
    } else {
      for (Walk w_(gtid, gstride, nx, (int)N); w_.ok(); w_.next()) {
        const int idx = w_.idx, i = w_.i, j = w_.j;
        const double xv = s.x[idx];
        const double ax_ = apply_a(s, s.solid, i, j, xv, [&](int a, int c) { return s.x[(size_t)a * nx + c]; });
        const double rv = s.b[idx] - ax_;
        g2[0] += rv * rv;
        g2[1] += isfinite(xv) ? 0.0 : 1.0;
      }
    }
    double tot[2] = {kept, 0.0};
    if (!have) {
      cta_publish<2>(g2, o2, shm, s.part, SL_B, nblocks);
      FB_SYNC(TR_RESIDUAL);
      grid_total<2>(s.part, SL_B, o2, nblocks, shm, tot);
    }
    rel = sqrt(tot[0]) / fmax(bnorm, 2.220446049250313e-16);
    // with a fixed sweep count the solve is accepted after its sweeps whatever the residual
    const bool conv = info == 0 && (s.pfixed > 0 || rel <= s.ptol * (1.0 + 1.0e-6));
    if (lead) {
      rep->cg_iters = total_it;
      rep->cg_outer = outer;
      rep->cg_info = info;
      rep->cg_rel = rel;
      rep->cg_converged = conv ? 1 : 0;
      rep->total_cg_iters += total_it;
    }
    if (tot[1] != 0.0) {
      fail(s, RS_NONFINITE, SG_POSTCONDITION);
      return;
    }
    if (ph & PH_NO_GRADIENT) return;
    if (!conv) {
      if (lead) {
        rep->ev[0] = total_it;
        rep->ev[1] = s.ptol;
        rep->ev[2] = rel;
      }
      fail(s, RS_PROJECTION, SG_PROJECTION);
      return;
    }
  }

  // ---- P9: gradient subtraction, boundaries, solid faces (grid.py:164-173)
  {
    double nf = 0.0;
    const double dtdx = s.dt, idx_ = 1.0 / s.ax.h, idy_ = 1.0 / s.ay.h;
    (void)idx_;
    (void)idy_;
    auto gv = [&](int i, int j) -> V {
      const V base = s.v2[(size_t)i * nx + j];
      if (i >= 1 && i <= ny - 1)
        return (V)((double)base - dtdx * (s.x[(size_t)i * nx + j] - s.x[(size_t)(i - 1) * nx + j]) / s.ay.h);
      if (s.ay.periodic)
        return (V)((double)s.v2[j] - dtdx * (s.x[j] - s.x[(size_t)(ny - 1) * nx + j]) / s.ay.h);
      return base;
    };
    // Every operand a face can need is loaded up front at valid indices and the boundary cases
    // select among the results afterwards, so a face costs one round of loads instead of a
    // chain of dependent ones. A face's value is u2 - dt (x_r - x_l) / dx at the column the
    // boundary rule picks (the periodic wrap takes x_0 - x_{nx-1}), as in grid.py:164-173.
    const bool px = s.ax.periodic;
    // operands of a face: its two cells' solid flags, the pre-gradient value and the two
    // pressures at the column (row) its boundary rule picks
    struct Ops {
      unsigned char sa, sb;
      V base;
      double xa, xb;
    };
    walk_batched<4, Ops>(
        Walk(gtid, gstride, nx + 1, (int)NU),
        [&](int, int i, int j) {
          Ops o;
          const unsigned char *srow = s.solid + (size_t)i * nx;
          o.sa = srow[j > 0 ? j - 1 : 0];  // solid_u_face
          o.sb = srow[j < nx ? j : nx - 1];
          // column whose gradient-updated value (gu) the face takes
          const int g = (px && (j == 0 || j == nx)) ? 0 : (j == nx ? nx - 1 : j);
          o.base = s.u2[(size_t)i * (nx + 1) + g];
          const int xa = g >= 1 ? g : 0, xb = g >= 1 ? g - 1 : nx - 1;
          o.xa = s.x[(size_t)i * nx + xa];
          o.xb = s.x[(size_t)i * nx + xb];
          return o;
        },
        [&](int idx, int i, int j, const Ops &o) {
          const int g = (px && (j == 0 || j == nx)) ? 0 : (j == nx ? nx - 1 : j);
          const bool grad = (g >= 1 && g <= nx - 1) || px;
          const V gval = grad ? (V)((double)o.base - dtdx * (o.xa - o.xb) / s.ax.h) : o.base;
          V val;
          if (o.sa | o.sb) {
            val = (V)wall_u(s, i);
          } else if (!s.ay.periodic && (i == 0 || i == ny - 1)) {
            val = s.channel ? V(0) : (V)s.fs_x;
          } else if (px && (j == 0 || j == nx)) {
            val = (V)0.5 * (gval + gval);
          } else if (!px && j == 0) {
            val = (V)s.fs_x;
          } else {
            val = gval;  // interior: gu(i, j); non-periodic outlet: gu(i, nx - 1)
          }
          s.u[idx] = val;
          if (!finite_v(val)) nf += 1.0;
        });
    if (!s.ay.periodic) {
      const int hi = ny - 1 > 0 ? ny - 1 : 0;
      walk_batched<4, Ops>(
          Walk(gtid, gstride, nx, (int)NV),
          [&](int, int i, int j) {
            Ops o;
            const int ia = i > 0 ? i - 1 : 0, ib = i < ny ? i : ny - 1;
            o.sa = s.solid[(size_t)ia * nx + j];  // solid_v_face
            o.sb = s.solid[(size_t)ib * nx + j];
            // gv(i, c) for an interior row, c the column after the x-direction boundary rule (gvx)
            int c = (!px && j == nx - 1) ? nx - 2 : j;
            c = c < 0 ? 0 : c;
            const int ic = i < 1 ? (hi < 1 ? hi : 1) : (i > hi ? hi : i), id = ic > 0 ? ic - 1 : 0;
            o.base = s.v2[(size_t)ic * nx + c];
            o.xa = s.x[(size_t)ic * nx + c];
            o.xb = s.x[(size_t)id * nx + c];
            return o;
          },
          [&](int idx, int i, int j, const Ops &o) {
            const V gval = (V)((double)o.base - dtdx * (o.xa - o.xb) / s.ay.h);
            V val;
            if (o.sa | o.sb) {
              val = (V)wall_v(s, j);
            } else if (i == 0 || i == ny) {
              val = s.channel ? V(0) : (V)s.fs_y;
            } else if (!px && j == 0) {
              val = (V)s.fs_y;
            } else {
              val = gval;
            }
            s.v[idx] = val;
            if (!finite_v(val)) nf += 1.0;
          });
    } else {
      auto gvx = [&](int i, int j) -> V {  // v after the x-direction boundary rule
        if (!s.ax.periodic) {
          if (j == 0) return (V)s.fs_y;
          if (j == nx - 1) return gv(i, nx - 2);
        }
        return gv(i, j);
      };
      for (Walk w_(gtid, gstride, nx, (int)NV); w_.ok(); w_.next()) {
        const int idx = w_.idx, i = w_.i, j = w_.j;
        V val;
        if (solid_v_face(s.solid, nx, ny, i, j)) {
          val = (V)wall_v(s, j);
        } else if (i == 0 || i == ny) {
          if (s.ay.periodic) val = (V)((A)0.5 * ((A)gvx(0, j) + (A)gvx(ny, j)));
          else val = s.channel ? V(0) : (V)s.fs_y;
        } else {
          val = gvx(i, j);
        }
        s.v[idx] = val;
        if (!finite_v(val)) nf += 1.0;
      }
    }
    double a1[1] = {nf};
    const int o1[1] = {OP_SUM};
    cta_publish<1>(a1, o1, shm, s.part, SL_C, nblocks);
    FB_SYNC(TR_GRADIENT);
    double tot[1];
    grid_total<1>(s.part, SL_C, o1, nblocks, shm, tot);
    if (tot[0] != 0.0) {
      fail(s, RS_NONFINITE, SG_PROJECTION);
      return;
    }
  }
  if (ph & PH_SCALAR) {
    for (int idx = gtid; idx < (int)N; idx += gstride) s.scal[idx] = s.scal2[idx];
  }

  // ---- P10: final state checks (stable_fluids.py:495-509, 541-554)
  if (ph & PH_FINALIZE) {
    double g[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // nonfinite, max speed, fluid div Linf, leakage, skew rate
    const int og[5] = {OP_SUM, OP_MAX, OP_MAX, OP_MAX, OP_MAX};
    const A vdx = (A)s.ax.h, vdy = (A)s.ay.h;
    struct CellOps {
      V ul, ur, vb, vt;
      unsigned char sol;
    };
    walk_batched<4, CellOps>(
        Walk(gtid, gstride, nx, (int)N),
        [&](int idx, int i, int j) {
          CellOps o;
          o.ul = s.u[(size_t)i * (nx + 1) + j];
          o.ur = s.u[(size_t)i * (nx + 1) + j + 1];
          o.vb = s.v[(size_t)i * nx + j];
          o.vt = s.v[(size_t)(i + 1) * nx + j];
          o.sol = s.solid[idx];
          return o;
        },
        [&](int, int, int, const CellOps &o) {
          const A ul = o.ul, ur = o.ur, vb = o.vb, vt = o.vt;
          const V cxv = (V)((A)0.5 * (ul + ur)), cyv = (V)((A)0.5 * (vb + vt));
          if (!finite_v(cxv) || !finite_v(cyv)) g[0] += 1.0;
          else g[1] = fmax(g[1], sqrt((double)cxv * (double)cxv + (double)cyv * (double)cyv));
          if (!o.sol) {
            const A dv = (ur - ul) / vdx + (vt - vb) / vdy;
            g[2] = fmax(g[2], fabs((double)dv));
          }
        });
    // skew_face_advection_rate (grid.py:435-445): the skew transport plans its substeps with
    // it, and the transport mode can change between advances. The cross velocity of a face
    // (v_on_u / u_on_v: the average of one or two cell averages) has its four operands loaded
    // with the face's own value and solid flags.
    struct FaceOps {
      V f, c0, c1, c2, c3;  // the face value; the two pairs averaged into the cross velocity
      unsigned char sa, sb;
    };
    const bool pxx = s.ax.periodic, pyy = s.ay.periodic;
    walk_batched<4, FaceOps>(
        Walk(gtid, gstride, nx + 1, (int)NU),
        [&](int idx, int i, int j) {
          FaceOps o;
          o.f = s.u[idx];
          const bool inner = j >= 1 && j <= nx - 1;
          const int ca = inner ? j - 1 : (pxx ? nx - 1 : (j == 0 ? 0 : nx - 1));
          const int cb = inner ? j : (pxx ? 0 : ca);
          o.c0 = s.v[(size_t)i * nx + ca];
          o.c1 = s.v[(size_t)(i + 1) * nx + ca];
          o.c2 = s.v[(size_t)i * nx + cb];
          o.c3 = s.v[(size_t)(i + 1) * nx + cb];
          const int jl = j > 0 ? j - 1 : 0, jr = j < nx ? j : nx - 1;
          o.sa = s.solid[(size_t)i * nx + jl];
          o.sb = s.solid[(size_t)i * nx + jr];
          return o;
        },
        [&](int, int i, int j, const FaceOps &o) {
          // v_on_u(s, v, i, j) from the loaded operands, same operations
          const A cva = (A)0.5 * ((A)o.c0 + (A)o.c1), cvb = (A)0.5 * ((A)o.c2 + (A)o.c3);
          const bool both = (j >= 1 && j <= nx - 1) || pxx;
          const A cross = both ? (A)0.5 * (cva + cvb) : cva;
          g[4] = fmax(g[4], (double)(fabs(o.f) / (V)s.ax.h + fabs(cross) / (V)s.ay.h));
          if (j == 0 || j == nx) return;
          if (o.sa != o.sb) g[3] = fmax(g[3], fabs((double)o.f - wall_u(s, i)));
        });
    walk_batched<4, FaceOps>(
        Walk(gtid, gstride, nx, (int)NV),
        [&](int idx, int i, int j) {
          FaceOps o;
          o.f = s.v[idx];
          const int ld = nx + 1;
          const bool inner = i >= 1 && i <= ny - 1;
          const int ra = inner ? i - 1 : (pyy ? ny - 1 : (i == 0 ? 0 : ny - 1));
          const int rb = inner ? i : (pyy ? 0 : ra);
          o.c0 = s.u[(size_t)ra * ld + j];
          o.c1 = s.u[(size_t)ra * ld + j + 1];
          o.c2 = s.u[(size_t)rb * ld + j];
          o.c3 = s.u[(size_t)rb * ld + j + 1];
          const int id = i > 0 ? i - 1 : 0, iu = i < ny ? i : ny - 1;
          o.sa = s.solid[(size_t)id * nx + j];
          o.sb = s.solid[(size_t)iu * nx + j];
          return o;
        },
        [&](int, int i, int j, const FaceOps &o) {
          // u_on_v(s, u, i, j) from the loaded operands, same operations
          const A cua = (A)0.5 * ((A)o.c0 + (A)o.c1), cub = (A)0.5 * ((A)o.c2 + (A)o.c3);
          const bool both = (i >= 1 && i <= ny - 1) || pyy;
          const A cross = both ? (A)0.5 * (cua + cub) : cua;
          g[4] = fmax(g[4], (double)(fabs(cross) / (V)s.ax.h + fabs(o.f) / (V)s.ay.h));
          if (i == 0 || i == ny) return;
          if (o.sa != o.sb) g[3] = fmax(g[3], fabs((double)o.f - wall_v(s, j)));
        });
    cta_publish<5>(g, og, shm, s.part, SL_A, nblocks);
    FB_SYNC(TR_FINAL);
    double tot[5];
    grid_total<5>(s.part, SL_A, og, nblocks, shm, tot);
    if (lead) {
      rep->final_speed = tot[1];
      rep->div_linf = tot[2];
      rep->leakage = tot[3];
      rep->skew_rate = tot[4];
    }
    if (tot[0] != 0.0) {
      fail(s, RS_NONFINITE, SG_POSTCONDITION);
      return;
    }
  }
  if (lead) rep->substeps_done += 1;
  trace_mark(s, TR_END);
}

#undef FB_SYNC
#undef FB_SYNC_B

// Single solve: the hardware grid is the solve's grid.
template <class V, class P, int VPT, int R0>
__global__ void __launch_bounds__(512) step_kernel(const __grid_constant__ StepParams<V, P> s) {
  if (threadIdx.x == 0) {
    fb_vgrid[0] = blockIdx.x;
    fb_vgrid[1] = gridDim.x;
    fb_mbar_ready = 0;
    fb_bar_target = 0;
  }
  __syncthreads();
  step_body<V, P, VPT, R0>(s);
}

// Batched solves: scenario g owns CTAs [first[g], first[g + 1]) and runs, in order, the
// substeps described by table[sub_first[g] .. sub_first[g + 1]) with a barrier of its own
// group between them; an empty range means nothing to do in this launch. Groups share no
// data and synchronise only within themselves, so one launch advances every scenario by all
// of its planned substeps. With R0 = 0 the row-transform shape is chosen per scenario at run
// time (every scenario uses the fixed three-pass transform). timing[2g] / timing[2g + 1]
// receive the earliest start and latest end (%globaltimer) of group g's CTAs, from which the
// host balances the next launch's CTA split.
template <class V, class P, int VPT, int R0>
__global__ void __launch_bounds__(512) step_kernel_batch(const StepParams<V, P> *__restrict__ table,
                                                         const int *__restrict__ first,
                                                         const int *__restrict__ sub_first, int ngroups,
                                                         unsigned long long *__restrict__ timing) {
  const unsigned long long t0 = global_ns();
  int lo = 0, hi = ngroups;  // largest g with first[g] <= blockIdx.x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= (int)blockIdx.x) lo = mid;
    else hi = mid;
  }
  const int g = lo;
  if (threadIdx.x == 0) {
    fb_vgrid[0] = (int)blockIdx.x - first[g];
    fb_vgrid[1] = first[g + 1] - first[g];
    fb_mbar_ready = 0;
    fb_bar_target = 0;
  }
  __syncthreads();
  const int e0 = sub_first[g], e1 = sub_first[g + 1];
  for (int e = e0; e < e1; ++e) {
    if (e > e0 && !grid_sync(table[e].gs, (unsigned)vncta(), table[e].limit_ns, table[e].rep)) return;
    step_body<V, P, VPT, R0>(table[e]);
  }
  __syncthreads();
  if (timing != nullptr && threadIdx.x == 0) {
    atomicMin(&timing[2 * g], t0);
    atomicMax(&timing[2 * g + 1], global_ns());
  }
}

}  // namespace fb
