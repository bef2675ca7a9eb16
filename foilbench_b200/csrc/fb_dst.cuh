// Fast application of the reference's DST-I pressure preconditioner.
//
// The reference preconditioner (_scipy_adapter.py:76-96) is
//     z = S (Lambda^-1 o (S (m . r))),   S = S_y (x) S_x the 2D orthonormal DST-I,
//     Lambda_{ky,kx} = lam_x(kx) + lam_y(ky),  lam(k) = 2 (1 - cos(pi k / (n + 1))) / h^2,
// with solid rows passed through. Because S_y diagonalises the 1D Dirichlet Laplacian
// T_y = tridiag(-1, 2, -1) / dy^2 (S_y Lam_y S_y = T_y), the middle factor is, for every
// x-wavenumber kx, exactly the tridiagonal solve (lam_x(kx) I + T_y)^-1 along y. The
// device therefore applies the same operator as
//     row DST-I along x  ->  constant-coefficient tridiagonal solve per column  ->  row DST-I,
// which needs two transforms per application instead of four.
//
// Row DST-I (length N, L = N + 1) by Bluestein's chirp-z identity:
//     sum_n x_n e^{i pi n k / L} = w_k sum_n (x_n w_n) conj(w_{k-n}),  w_m = e^{i pi m^2 / (2L)},
// i.e. a circular convolution of length Pf >= 2N - 1 (power of two): forward FFT, pointwise
// product with the precomputed transform of conj(w) (natural order), inverse FFT (the
// register Stockham FFT of fb_fft.cuh). The DST-I value is sqrt(2/L) Im(w_k conv_k); the
// factor and the 1/Pf inverse-FFT scale are folded into the filter table.
//
// Column solve of A w = g, A = tridiag(-1, d, -1) (n x n, zero Dirichlet ends), d = 2 +
// lam_x dy^2 > 2. With mu = 2 / (d + sqrt(d^2 - 4)) in (0, 1):
//     mu A = (I - mu S-)(I - mu S+) + mu^2 e0 e0^T      (S-/S+ shift down/up),
// so w = y - kappa y_0 h with y = (I - mu S+)^-1 (I - mu S-)^-1 (mu g) (a causal and an
// anti-causal first-order recurrence), h_j = (mu^j - mu^{2n-j}) / (1 - mu^2) and
// kappa = mu^2 / (1 + mu^2 h_0) (Sherman-Morrison). Each recurrence is evaluated by a CTA
// over a W-column tile staged in shared memory: every thread owns one segment of one
// column, runs the recurrence locally, and segment carries are combined by warp scans.
#pragma once

#include <cuda_runtime.h>

#include "fb_umma.cuh"

namespace fb {

// Complex value, aligned to its size so a value moves in one 8- (float) or 16-byte (double)
// access.
template <class T>
struct __align__(2 * sizeof(T)) Cx {
  T x, y;
};

template <class T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return Cx<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class T>
__device__ __forceinline__ Cx<T> cmulc(Cx<T> a, Cx<T> b) {  // a * conj(b)
  return Cx<T>{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}

// Tables for the row transform of length N (device memory, precision T).
template <class T>
struct DstTables {
  const Cx<T> *chirp;  // w_m, m = 0..N
  const Cx<T> *filt;   // FFT(conj(w)) * sqrt(2/L) / Pf, natural order, Pf entries (split: 3 Pf)
  const Cx<T> *twp;    // per-pass Stockham twiddle tables (FftPlan layout)
  int n;               // N
  int logp;            // log2(Pf)
  // byte offsets of shared-memory copies of twp, filt and chirp in the dynamic shared
  // memory (all three present, or tw_soff < 0 when the transform reads global memory)
  int tw_soff, filt_soff, chirp_soff;
  // two-level twiddles of the long-row path: W_Pf^e = tw_hi[e >> 7] * tw_lo[e & 127]
  // (tw_lo: 128 entries, tw_hi: Pf / 128), global copies and the shared copy's byte offset
  const Cx<T> *tw_lo, *tw_hi;
  int tw2_soff;
  // Rows whose length-Pf convolution does not fit one CTA's shared memory (double precision,
  // N over 4096): the convolution runs in two halves of split_h points (dst_rows_split2)
  // with Pf = the half convolution's length, three filter slices at filt (3 Pf entries) and
  // 2 Pf spectrum values of scratch per CTA at spec. split_h = 0: one convolution.
  Cx<T> *spec;
  int split_h;
};

template <class T>
__device__ __forceinline__ Cx<T> dst_stage(const DstTables<T> &tb, int n, T x) {
  const Cx<T> w = tb.chirp[n + 1];
  return Cx<T>{x * w.x, x * w.y};
}

// Per-column constants of the tridiagonal solve (double precision tables).
struct ColTables {
  const double *mu;       // mu(kx)
  const double *logmu;    // log(mu)
  const double *kappa;    // mu^2 / (1 + mu^2 h_0)
  const double *inv1m;    // 1 / (1 - mu^2)
};

// Input and output of the column solve when the row transforms run on the tensor cores: the
// input is y = t + pe (the first transform's parity arrays), the output the second
// transform's data operand (TF32, split by the parity of the wavenumber, umma_index) instead
// of t itself. The solve then zeroes its columns of pe (the second transform's output, which
// that transform accumulates into) and accumulates y . w over its columns (with z = S w, the
// preconditioned residual's r . z).
struct ColIO {
  float *pe;
  float *a2;
  int nkb;
  int ycopy_soff;  // byte offset in the dynamic shared memory of a copy of the tile's y (-1: read y again)
};

// Solve A w = dy2 * t for the W columns [c0, c0 + W) of the (ny, nx) array t (row-major,
// x fastest), in place. 512 threads; W in {2, 4, 8, 16}. Each column is split into
// S = 512 / W segments of m = ceil(ny / S) rows, one per thread, so a column is served by
// G = S / 32 consecutive warps and segment carries are combined with warp-shuffle scans
// (plus a short shared-memory step when G > 1). Three sweeps over the segment:
//   1. causal recurrence s_j = mu (g_j + s_{j-1}) from a zero carry;
//   2. anti-causal recurrence y_j = s_j + mu y_{j+1} from a zero carry;
//   3. add the carries' closed-form responses and the Sherman-Morrison term.
// With C the true s entering the segment and D the true y leaving it at the bottom,
//   y_j = y_j(local) + C rho_j + D mu^{j1-j},   rho_j = (mu^{j-j0+1} - mu^{2 j1-j-j0+1}) / (1 - mu^2).
// sm: ny * W + S values of T (tile); xs: 3 * 16 + 16 doubles of scan scratch; yc (TC): ny * W
// values, 16-byte aligned, the tile's input y unpadded.
template <class T, int W, bool TC = false>
__device__ __forceinline__ double column_solve_tile(T *__restrict__ t, int nx, int ny, int c0, double dy2,
                                                    const ColTables &ct, T *sm, double *xs, const ColIO io = ColIO{},
                                                    T *yc = nullptr) {
  double ydotw = 0.0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int S = 512 / W;            // segments per column
  constexpr int G = S >> 5;             // warps per column
  const int m = (ny + S - 1) / S;       // rows per segment
  // row / m by a multiply-high (exact for row, m < 2^16)
  const unsigned magic = m > 1 ? (unsigned)(0xFFFFFFFFu / (unsigned)m) + 1u : 0u;
  auto seg_of = [&](int row) -> int { return m > 1 ? (int)__umulhi((unsigned)row, magic) : row; };
  // Tile layout: (row, c) at row * W + c + row / m. A warp's lanes are consecutive segments
  // of one column, m * W + 1 elements apart (an odd stride), so they never share a bank.
  constexpr int V4 = 16 / (int)sizeof(T);
  const bool vec = (W % V4) == 0 && (nx % V4) == 0;
  if (vec) {
    constexpr int vpr = W / V4 > 0 ? W / V4 : 1;  // vectors per tile row
    const int total = ny * vpr;
    for (int v0 = tid; v0 < total; v0 += 4 * 512) {
      T buf[4][V4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int v = v0 + u * 512;
        const int row = v / vpr, cv = (v - row * vpr) * V4;
        if (v < total && c0 + cv < nx) {
          const T *src = t + (size_t)row * nx + c0 + cv;
          if constexpr (V4 == 4) {
            float4 q = *reinterpret_cast<const float4 *>(src);
            if constexpr (TC) {
              const float4 e = *reinterpret_cast<const float4 *>(io.pe + (src - t));
              q.x += e.x;
              q.y += e.y;
              q.z += e.z;
              q.w += e.w;
            }
            buf[u][0] = q.x;
            buf[u][1] = q.y;
            buf[u][2] = q.z;
            buf[u][3] = q.w;
          } else {
            const double2 q = *reinterpret_cast<const double2 *>(src);
            buf[u][0] = q.x;
            buf[u][1] = q.y;
          }
        } else {
#pragma unroll
          for (int e = 0; e < V4; ++e) buf[u][e] = T(0);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int v = v0 + u * 512;
        if (v < total) {
          const int row = v / vpr, cv = (v - row * vpr) * V4;
          T *dst = sm + row * W + cv + seg_of(row);
#pragma unroll
          for (int e = 0; e < V4; ++e) dst[e] = buf[u][e];
          if constexpr (TC) {
            // y's copy is unpadded (row * W + cv), so one aligned 16-byte store
            if (yc != nullptr)
              *reinterpret_cast<float4 *>(yc + row * W + cv) = make_float4(buf[u][0], buf[u][1], buf[u][2], buf[u][3]);
          }
        }
      }
    }
  } else {
    for (int i = tid; i < ny * W; i += 512) {
      const int row = i / W, c = i - row * W, col = c0 + c;
      T val = T(0);
      if (col < nx) {
        val = t[(size_t)row * nx + col];
        if constexpr (TC) val += io.pe[(size_t)row * nx + col];
      }
      sm[row * W + c + seg_of(row)] = val;
    }
  }
  __syncthreads();
  const int c = warp / G, g = warp - c * G;
  const int col = c0 + c;
  const bool live = col < nx;
  const int k = g * 32 + lane;  // segment
  const int j0 = k * m;
  const int j1 = min(j0 + m, ny);
  const int len = j1 > j0 ? j1 - j0 : 0;
  double mu = 0.5, lmu = -0.6931471805599453, kap = 0.0, i1m = 1.0;
  if (live) {
    mu = ct.mu[col];
    lmu = ct.logmu[col];
    kap = ct.kappa[col];
    i1m = ct.inv1m[col];
  }
  const T tmu = (T)mu, tdy2 = (T)dy2;
  T *colp = sm + c + k;  // element (row j) of this column/segment at colp[j * W]
  const double a = exp((double)m * lmu);  // mu^m, the carry factor across a full segment
  // apow[q] = a^(2^q); a^e for e < 2^8 is the product of the apow of e's bits (segment and
  // lane powers below are products of these instead of further exp calls)
  double apow[8];
  apow[0] = a;
#pragma unroll
  for (int q = 1; q < 8; ++q) apow[q] = apow[q - 1] * apow[q - 1];
  auto a_to = [&](int e) -> double {
    double r = 1.0;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if ((e >> q) & 1) r *= apow[q];
    return r;
  };
  const bool full = len == m;                       // every segment but possibly the last
  const double a_len = full ? a : exp((double)len * lmu);  // mu^len
  double *wtot = xs;            // [16 columns][G] warp totals (reused by both scans)
  double *y0s = xs + 3 * 16;    // [16] true y_0 per column

  // ---- sweep 1: causal, zero carry in
  T sv = T(0);
  for (int j = j0; j < j1; ++j) {
    sv = tmu * (tdy2 * colp[j * W] + sv);
    colp[j * W] = sv;
  }
  // inclusive scan X_k = e_k + a X_{k-1} over the column's segments; carry C_k = X_{k-1}
  double X = (double)sv;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const double up = __shfl_up_sync(0xffffffffu, X, 1 << q);
    if (lane >= (1 << q)) X += apow[q] * up;
  }
  double Cin = __shfl_up_sync(0xffffffffu, X, 1);
  if (lane == 0) Cin = 0.0;
  if (G > 1) {
    if (lane == 31) wtot[c * G + g] = X;
    __syncthreads();
    double carry = 0.0;  // true s at the end of warp g - 1's segments
    const double a32 = apow[4] * apow[4];
    for (int h = 0; h < g; ++h) carry = wtot[c * G + h] + a32 * carry;
    Cin += carry * a_to(lane);
    __syncthreads();
  }

  // ---- sweep 2: anti-causal on the local causal values, zero carry in
  T yv = T(0);
  for (int j = j1 - 1; j >= j0; --j) {
    yv = colp[j * W] + tmu * yv;
    colp[j * W] = yv;
  }
  // true segment-top value with the causal carry: f = y_loc(j0) + C rho_{j0}
  const double rho0 = len > 0 ? mu * (1.0 - a_len * a_len) * i1m : 0.0;
  const double f = (double)yv + Cin * rho0;
  // reverse inclusive scan Y_k = f_k + a Y_{k+1}; D_k = Y_{k+1}
  double Y = f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const double dn = __shfl_down_sync(0xffffffffu, Y, 1 << q);
    if (lane + (1 << q) < 32) Y += apow[q] * dn;
  }
  double Din = __shfl_down_sync(0xffffffffu, Y, 1);
  if (lane == 31) Din = 0.0;
  if (G > 1) {
    if (lane == 0) wtot[c * G + g] = Y;
    __syncthreads();
    double carry = 0.0;  // true y at the top of warp g + 1's segments
    const double a32 = apow[4] * apow[4];
    for (int h = G - 1; h > g; --h) carry = wtot[c * G + h] + a32 * carry;
    Din += carry * a_to(31 - lane);
  }
  if (k == 0) y0s[c] = (double)yv + Din * a_len;  // C_0 = 0
  __syncthreads();
  const double y0 = y0s[c];

  // ---- sweep 3: carries' responses and the Sherman-Morrison correction
  if (len > 0) {
    const double inv_mu = 1.0 / mu;
    const double cc = Cin * i1m, sm_coef = kap * y0 * i1m;
    double pa = mu;                                           // mu^{j-j0+1}
    double pb = a_len * a_len * mu;                           // mu^{2 j1-j-j0+1}
    double pc = a_len;                                        // mu^{j1-j}
    double ha = a_to(k);                                      // mu^j (j0 = k m)
    double hb = exp((double)(2 * ny - j0) * lmu);             // mu^{2n-j}
    for (int j = j0; j < j1; ++j) {
      const double corr = cc * (pa - pb) + Din * pc - sm_coef * (ha - hb);
      colp[j * W] = (T)((double)colp[j * W] + corr);
      pa *= mu;
      pb *= inv_mu;
      pc *= inv_mu;
      ha *= mu;
      hb *= inv_mu;
    }
  }
  __syncthreads();
  if (vec) {
    constexpr int vpr = W / V4 > 0 ? W / V4 : 1;
    const int total = ny * vpr;
    for (int v = tid; v < total; v += 512) {
      const int row = v / vpr, cv = (v - row * vpr) * V4;
      if (c0 + cv < nx) {
        const T *srcp = sm + row * W + cv + seg_of(row);
        T *dst = t + (size_t)row * nx + c0 + cv;
        if constexpr (TC) {
          // y . w (y read again), pe zeroed, then the operand: columns c, c + 2 (odd
          // wavenumbers) and c + 1, c + 3 (even), two adjacent values each
          float *pez = io.pe + (dst - t);
          if (yc != nullptr) {
            const float4 ys = *reinterpret_cast<const float4 *>(yc + row * W + cv);
            ydotw += (double)(ys.x * srcp[0] + ys.y * srcp[1] + ys.z * srcp[2] + ys.w * srcp[3]);
          } else {
            const float4 ya = *reinterpret_cast<const float4 *>(dst), yb = *reinterpret_cast<const float4 *>(pez);
            ydotw += (double)((ya.x + yb.x) * srcp[0] + (ya.y + yb.y) * srcp[1] + (ya.z + yb.z) * srcp[2] +
                              (ya.w + yb.w) * srcp[3]);
          }
          *reinterpret_cast<float4 *>(pez) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          const int c = c0 + cv;
          *reinterpret_cast<float2 *>(io.a2 + umma_index(io.nkb, row, 0, c >> 1)) =
              make_float2(to_tf32(srcp[0]), to_tf32(srcp[2]));
          *reinterpret_cast<float2 *>(io.a2 + umma_index(io.nkb, row, 1, c >> 1)) =
              make_float2(to_tf32(srcp[1]), to_tf32(srcp[3]));
        } else if constexpr (V4 == 4) {
          *reinterpret_cast<float4 *>(dst) = make_float4(srcp[0], srcp[1], srcp[2], srcp[3]);
        } else {
          *reinterpret_cast<double2 *>(dst) = make_double2(srcp[0], srcp[1]);
        }
      }
    }
  } else {
    for (int i = tid; i < ny * W; i += 512) {
      const int row = i / W, cc2 = i - row * W, cl = c0 + cc2;
      if (cl < nx) {
        if constexpr (TC) {
          const size_t ix = (size_t)row * nx + cl;
          const T w = sm[row * W + cc2 + seg_of(row)];
          ydotw += (double)((t[ix] + io.pe[ix]) * w);
          io.pe[ix] = 0.0f;
          io.a2[umma_index(io.nkb, row, cl & 1, cl >> 1)] = to_tf32(w);
        } else
          t[(size_t)row * nx + cl] = sm[row * W + cc2 + seg_of(row)];
      }
    }
  }
  __syncthreads();
  return ydotw;
}

}  // namespace fb
