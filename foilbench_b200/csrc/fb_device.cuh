// Device building blocks shared by the Stable Fluids kernels: the bounded grid
// barrier of the persistent step kernel, deterministic CTA/grid reductions, NACA
// geometry and bilinear sampling on the MAC grid.
#pragma once

#include <cstdint>
#include <cuda/atomic>
#include <cuda_runtime.h>

namespace fb {

// Dynamic shared memory of the step kernel and the CTA reduction scratch. Functions that
// are not inlined into the kernel address them through these symbols (plus byte offsets),
// never through pointer arguments, so their accesses compile to shared-memory instructions
// instead of generic ones.
extern __shared__ __align__(16) char fb_smem[];
static __shared__ double fb_red[32 * 8 + 16];

// Virtual grid: this CTA's index within the solve it serves and that solve's CTA count. A
// single-solve launch uses the hardware grid; a batched launch gives every scenario its own
// contiguous group of CTAs (with its own barrier word, partials and report).
static __shared__ int fb_vgrid[2];
__device__ __forceinline__ int vcta() { return fb_vgrid[0]; }
__device__ __forceinline__ int vncta() { return fb_vgrid[1]; }

// ------------------------------------------------------------------------------------------
// Status words written by the device (mirrors fb_status / fb_reason / fb_stage in foilb200.h)
enum DevStatus : int { ST_OK = 0, ST_NUMERICAL = 5, ST_TIMEOUT = 6 };
enum DevReason : int {
  RS_NONE = 0, RS_EXCESSIVE_VELOCITY = 1, RS_STABILITY_LIMIT = 2, RS_NONFINITE = 3,
  RS_CONVERGENCE = 4, RS_PROJECTION = 5, RS_POSTCONDITION = 6
};
enum DevStage : int {
  SG_NONE = 0, SG_ADVECTION = 1, SG_VISCOSITY = 2, SG_PROJECTION = 3, SG_BOUNDARY = 4, SG_POSTCONDITION = 5,
  SG_IMPORT = 6
};

// Report written by CTA 0 of the step kernel and read back by the host once per call.
struct DevReport {
  int status, reason, stage;
  int cg_iters, cg_outer, cg_info, cg_converged;
  int visc_iters, visc_converged;
  int total_cg_iters;
  int substeps_done;
  int pad0;
  double cg_rel, visc_resid;
  double face_speed, wall_speed, proj_cfl;
  double final_speed, div_linf, leakage;
  double skew_rate;  // max staggered advection rate of the final faces (skew-RK2 CFL)
  double ev[6];
};

// Barrier state of the persistent kernel. `gen` only grows; `abort` is sticky until the
// host clears it.
struct GridSync {
  unsigned int count;  // barrier arrivals of the current launch (cleared before each launch)
  unsigned int gen;    // unused
  unsigned int abort;
  unsigned int pad;
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier for a cooperatively launched kernel (all CTAs co-resident). Arrivals
// add to a counter that only grows during a launch (the host clears it before every launch);
// a CTA's k-th barrier waits until the counter reaches k x nblocks, so no CTA has to reset it
// and arrival needs no returned value. The spin is bounded: after `limit_ns` a waiting CTA
// raises the sticky abort flag and every CTA leaves; the caller returns and the host sees
// ST_TIMEOUT. Returns false on abort. Every CTA of a launch sets fb_bar_target = 0 first.
// `withhold` is a test hook (0 in normal runs): CTA 0 of the solve does not arrive at its
// withhold-th barrier, so that barrier's waits run out and the launch ends with ST_TIMEOUT.
static __shared__ unsigned int fb_bar_target;  // arrivals this CTA's next barrier waits for
__device__ __forceinline__ bool grid_sync(GridSync *gs, unsigned int nblocks, unsigned long long limit_ns,
                                          DevReport *rep, unsigned int withhold = 0u) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(gs->count), ab(gs->abort);
    int ok = 1;
    const unsigned int target = fb_bar_target + nblocks;
    fb_bar_target = target;
    __threadfence();
    if (!(withhold != 0u && vcta() == 0 && target == withhold * nblocks)) cnt.fetch_add(1u, cuda::memory_order_release);
    const unsigned long long t0 = global_ns();
    unsigned int spins = 0;
    while ((int)(cnt.load(cuda::memory_order_acquire) - target) < 0) {
      if ((++spins & 63u) == 0u) {
        if (ab.load(cuda::memory_order_relaxed)) { ok = 0; break; }
        if (global_ns() - t0 > limit_ns) {
          ab.store(1u, cuda::memory_order_relaxed);
          atomicExch(&rep->status, (int)ST_TIMEOUT);
          ok = 0;
          break;
        }
      }
      __nanosleep(32);
    }
    if (ab.load(cuda::memory_order_relaxed)) ok = 0;
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ------------------------------------------------------------------------------------------
// Deterministic reductions. Each CTA reduces K values (sum or max) and publishes them to
// part[(slot + k) * nblocks + vcta()]; after a barrier every CTA folds all partials in
// the same fixed order, so all CTAs obtain bitwise identical totals and take identical
// control-flow decisions.
enum { OP_SUM = 0, OP_MAX = 1 };

__device__ __forceinline__ double op_apply(int op, double a, double b) { return op == OP_MAX ? fmax(a, b) : a + b; }
__device__ __forceinline__ double op_identity(int op) { return op == OP_MAX ? -1.0 / 0.0 : 0.0; }

template <int K>
__device__ __forceinline__ void cta_publish(double (&v)[K], const int (&op)[K], double *shm, double *part,
                                            int slot, int nblocks) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] = op_apply(op[k], v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) shm[warp * K + k] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double a = lane < nw ? shm[lane * K + k] : op_identity(op[k]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a = op_apply(op[k], a, __shfl_xor_sync(0xffffffffu, a, o));
      if (lane == 0) part[(size_t)(slot + k) * nblocks + vcta()] = a;
    }
  }
  __syncthreads();
}

template <int K>
__device__ __forceinline__ void grid_total(const double *part, int slot, const int (&op)[K], int nblocks,
                                           double *shm, double (&out)[K]) {
  // Warp k folds slot k: lane-strided partial sums in block order, then a fixed butterfly.
  // The partials are read through L2 (__ldcg; other CTAs wrote them) in batches of eight
  // independent loads so the fold waits on few round trips.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (warp == k) {
      double a = op_identity(op[k]);
      const double *src = part + (size_t)(slot + k) * nblocks;
      for (int b0 = lane; b0 < nblocks; b0 += 8 * 32) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = b0 + u * 32 < nblocks ? __ldcg(src + b0 + u * 32) : op_identity(op[k]);
#pragma unroll
        for (int u = 0; u < 8; ++u) a = op_apply(op[k], a, v[u]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a = op_apply(op[k], a, __shfl_xor_sync(0xffffffffu, a, o));
      if (lane == 0) shm[k] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = shm[k];
  __syncthreads();
}

// ------------------------------------------------------------------------------------------
// Bulk asynchronous global->shared copies (cp.async.bulk, completion counted in bytes on a
// shared-memory mbarrier). Only plain per-CTA copies of this GPU's memory; no multicast.
// Source, destination and size must be multiples of 16 bytes.
static __shared__ __align__(8) unsigned long long fb_mbar[32];
static __shared__ unsigned int fb_mbar_uses[32];  // completed phases per mbarrier
static __shared__ int fb_mbar_ready;               // set once the mbarriers are initialised in this launch

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Invalidate an mbarrier whose phases have all been waited for, so that its memory may be
// initialised again (re-initialising a valid mbarrier is undefined).
__device__ __forceinline__ void mbar_inval(unsigned long long *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Order this thread's earlier generic-proxy accesses (global writes seen through the grid
// barrier, reads of the destination buffer) before its following bulk copies.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity, giving up after limit_ns. A copy that never
// lands (which would mean a broken address) is reported, waited for once more with the
// same bound, and left to the caller, whose next grid barrier then aborts the kernel.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned long long limit_ns,
                                          GridSync *gs, DevReport *rep) {
  if (mbar_try_wait(bar, parity)) return true;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const unsigned long long t0 = global_ns();
    for (unsigned spins = 1;; ++spins) {
      if (mbar_try_wait(bar, parity)) return attempt == 0;
      if ((spins & 31u) == 0u && global_ns() - t0 > limit_ns) break;
    }
    if (attempt == 0) {
      cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ab(gs->abort);
      ab.store(1u, cuda::memory_order_relaxed);
      atomicExch(&rep->status, (int)ST_TIMEOUT);
    }
  }
  return false;
}

// ------------------------------------------------------------------------------------------
// Four consecutive values with 16-byte accesses (the address must be 16-byte aligned).
__device__ __forceinline__ void ld4(const float *p, float (&o)[4]) {
  const float4 a = *reinterpret_cast<const float4 *>(p);
  o[0] = a.x;
  o[1] = a.y;
  o[2] = a.z;
  o[3] = a.w;
}
__device__ __forceinline__ void ld4(const double *p, double (&o)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
  o[0] = a.x;
  o[1] = a.y;
  o[2] = b.x;
  o[3] = b.y;
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double (&v)[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

// ------------------------------------------------------------------------------------------
// Coordinates. numpy.linspace(start, stop, n)[j] = j * step + start with the last point
// set to stop exactly; evaluated without FMA contraction so cell centres (and with them the
// solid mask) are bit-identical to the reference's.
__device__ __forceinline__ double lin_at(int j, int n, double start, double step, double stop) {
  return (n > 1 && j == n - 1) ? stop : __dadd_rn(__dmul_rn((double)j, step), start);
}

struct Axis {
  double start, step, stop;  // cell-centre linspace
  double lo, h;              // domain lower bound and spacing
  double hi;                 // domain upper bound
  double ih;                 // 1 / h
  int n;
  int periodic;
};

// ------------------------------------------------------------------------------------------
// NACA four-digit section (geometry.py:13-159). Products that decide the solid mask are
// rounded exactly like the reference's numpy expressions: no FMA contraction, and the
// integer powers x**3, x**4 (libm pow in numpy) are computed as correctly rounded
// products through an exact double-double square.
struct Foil {
  double m, p, t;         // max camber, camber position, thickness (fractions)
  double chord, px, py;   // chord, pivot
  double quarter;         // 0.25 * chord
  double thick_scale;     // 5.0 * t * chord
  double front_k, back_k; // m / p**2, m / (1 - p)**2
  double two_p, one_m_2p; // 2p, 1 - 2p
  int cambered;
};

__device__ __forceinline__ double cr_cube(double x) {
  const double hi = __dmul_rn(x, x);
  const double lo = fma(x, x, -hi);
  const double h3 = __dmul_rn(hi, x);
  const double e = fma(hi, x, -h3) + lo * x;  // exact low part of hi*x plus lo*x
  return h3 + e;
}

__device__ __forceinline__ double cr_pow4(double x) {
  const double hi = __dmul_rn(x, x);
  const double lo = fma(x, x, -hi);
  const double h4 = __dmul_rn(hi, hi);
  const double e = fma(hi, hi, -h4) + 2.0 * hi * lo;
  return h4 + e;
}

__device__ __forceinline__ void naca_surfaces(const Foil &f, double x_local, double &upper, double &lower) {
  double xc = __ddiv_rn(x_local, f.chord);
  xc = fmin(fmax(xc, 0.0), 1.0);
  const double x2 = __dmul_rn(xc, xc);
  double poly = __dmul_rn(0.2969, sqrt(fmax(xc, 0.0)));
  poly = __dsub_rn(poly, __dmul_rn(0.1260, xc));
  poly = __dsub_rn(poly, __dmul_rn(0.3516, x2));
  poly = __dadd_rn(poly, __dmul_rn(0.2843, cr_cube(xc)));
  poly = __dsub_rn(poly, __dmul_rn(0.1036, cr_pow4(xc)));
  const double half = __dmul_rn(f.thick_scale, poly);
  double camber = 0.0;
  if (f.cambered) {
    if (xc < f.p) {
      camber = __dmul_rn(f.front_k, __dsub_rn(__dmul_rn(f.two_p, xc), x2));
    } else {
      camber = __dmul_rn(f.back_k, __dsub_rn(__dadd_rn(f.one_m_2p, __dmul_rn(f.two_p, xc)), x2));
    }
    camber = __dmul_rn(camber, f.chord);
  }
  upper = __dadd_rn(camber, half);
  lower = __dsub_rn(camber, half);
}

__device__ __forceinline__ void naca_local(const Foil &f, double c, double s, double x, double y, double &lx,
                                           double &ly) {
  const double tx = __dsub_rn(x, f.px), ty = __dsub_rn(y, f.py);
  lx = __dadd_rn(__dadd_rn(__dmul_rn(c, tx), __dmul_rn(s, ty)), f.quarter);
  ly = __dadd_rn(__dmul_rn(-s, tx), __dmul_rn(c, ty));
}

// signed_distance <= 0  <=>  inside the chord range and between the surfaces.
__device__ __forceinline__ bool naca_contains(const Foil &f, double c, double s, double x, double y) {
  double lx, ly;
  naca_local(f, c, s, x, y, lx, ly);
  if (!(lx >= 0.0 && lx <= f.chord)) return false;
  double up, lo;
  naca_surfaces(f, lx, up, lo);
  return ly <= up && ly >= lo;
}

__device__ __forceinline__ double naca_sdf(const Foil &f, double c, double s, double x, double y) {
  double lx, ly, up, lo;
  naca_local(f, c, s, x, y, lx, ly);
  naca_surfaces(f, lx, up, lo);
  const bool within = (lx >= 0.0) && (lx <= f.chord);
  const double outside_v = fmax(ly - up, lo - ly);
  const double inside_v = -fmin(up - ly, ly - lo);
  const double vertical = (ly <= up && ly >= lo) ? inside_v : outside_v;
  const double beyond = fmax(fmax(-lx, lx - f.chord), 0.0);
  return within ? vertical : hypot(beyond, fmax(vertical, 0.0));
}

// ------------------------------------------------------------------------------------------
// Bilinear sampling of a cell-centred field (interpolation.py:9-64): grid coordinate with a
// half-cell offset, clamp (or numpy-style modulo on periodic axes), floor, weights. Indices
// are always forced in range, so non-finite positions cannot address outside the field.
__device__ __forceinline__ void sample_coord(double g, int n, int periodic, int &i0, int &i1, double &t) {
  if (!(g == g)) {  // NaN position: sample element 0 with a NaN weight so the result stays NaN
    i0 = 0;
    i1 = 0;
    t = g;
    return;
  }
  if (periodic) {
    double m = fmod(g, (double)n);
    if (m != 0.0 && m < 0.0) m += (double)n;
    g = m;
  }
  g = fmin(fmax(g, 0.0), (double)(n - 1) + (periodic ? 0.999999999999 : 0.0));
  int i = (int)floor(g);
  if (i < 0) i = 0;
  if (i > n - 1) i = n - 1;
  t = g - (double)i;
  i0 = i;
  i1 = periodic ? (i + 1 == n ? 0 : i + 1) : (i + 1 < n ? i + 1 : n - 1);
}

template <class V>
__device__ __forceinline__ double bilinear(const V *__restrict__ f, int ld, int iy0, int iy1, int ix0, int ix1,
                                           double tx, double ty) {
  const double a = (double)f[(size_t)iy0 * ld + ix0], b = (double)f[(size_t)iy0 * ld + ix1];
  const double c = (double)f[(size_t)iy1 * ld + ix0], d = (double)f[(size_t)iy1 * ld + ix1];
  return (1.0 - tx) * (1.0 - ty) * a + tx * (1.0 - ty) * b + (1.0 - tx) * ty * c + tx * ty * d;
}

}  // namespace fb
