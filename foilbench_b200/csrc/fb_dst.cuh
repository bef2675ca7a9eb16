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
// column, runs the recurrence locally, and segment carries are combined by a short scan.
#pragma once

#include <cuda_runtime.h>

namespace fb {

template <class T>
struct Cx {
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
  const Cx<T> *filt;   // FFT(conj(w)) * sqrt(2/L) / Pf, natural order, Pf entries
  const Cx<T> *tw;     // e^{-2 pi i k / Pf}, k < Pf/2
  int n;               // N
  int logp;            // log2(Pf)
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

// Solve A w = dy2 * t for the W columns [c0, c0 + W) of the (ny, nx) array t (row-major,
// x fastest), in place. sm: ny * (W + 1) + S values of T, then 2 * S * W + W doubles of carries.
template <class T>
__device__ void column_solve_tile(T *__restrict__ t, int nx, int ny, int c0, int W, double dy2,
                                  const ColTables &ct, T *sm, double *carry) {
  // Tile layout: row j of column c at j * (W + 1) + c + j / m. The extra element per
  // segment of m rows shifts neighbouring segments by one bank, so the two segments that
  // share a warp (m rows apart) never hit the same bank.
  const int ld = W + 1;
  const int S = blockDim.x / W;
  const int m = (ny + S - 1) / S;
  const int tid = threadIdx.x;
  for (int i = tid; i < ny * W; i += blockDim.x) {
    const int row = i / W, c = i - row * W, col = c0 + c;
    sm[row * ld + c + row / m] = col < nx ? t[(size_t)row * nx + col] : T(0);
  }
  __syncthreads();
  const int k = tid / W, c = tid - (tid / W) * W, col = c0 + c;
  const bool active = (k < S) && (col < nx);
  const int j0 = k * m;
  const int j1 = min(j0 + m, ny);
  const int len = j1 > j0 ? j1 - j0 : 0;
  double mu = 0.5, lmu = -0.6931471805599453, kap = 0.0, i1m = 1.0;
  if (active) {
    mu = ct.mu[col];
    lmu = ct.logmu[col];
    kap = ct.kappa[col];
    i1m = ct.inv1m[col];
  }
  const T tmu = (T)mu;
  double *endc = carry;              // [S][W] local causal end values, then carries-in
  double *startc = carry + S * W;    // [S][W] local anti-causal start values, then carries-in
  double *y0c = carry + 2 * S * W;   // [W] true y_0 per column
  // causal: s_j = mu (g_j + s_{j-1})
  if (active) {
    T s = T(0);
    for (int j = j0; j < j1; ++j) {
      s = tmu * ((T)dy2 * sm[j * ld + c + k] + s);
      sm[j * ld + c + k] = s;
    }
    endc[k * W + c] = (double)s;
  }
  __syncthreads();
  if (k == 0 && col < nx) {
    // Full segments have length m; only the last non-empty one may be shorter, and its
    // carry-out feeds no later rows, so mu^m serves every step of the scan.
    const double mum = exp((double)m * lmu);
    double run = 0.0;
    for (int q = 0; q < S; ++q) {
      const double e = endc[q * W + c];
      endc[q * W + c] = run;  // carry-in for segment q
      run = e + mum * run;
    }
  }
  __syncthreads();
  if (active) {
    const double cin = endc[k * W + c];
    if (cin != 0.0) {
      T pw = tmu;
      const T tc = (T)cin;
      for (int j = j0; j < j1; ++j) {
        sm[j * ld + c + k] += pw * tc;
        pw *= tmu;
      }
    }
    // anti-causal: y_j = s_j + mu y_{j+1}
    T y = T(0);
    for (int j = j1 - 1; j >= j0; --j) {
      y = sm[j * ld + c + k] + tmu * y;
      sm[j * ld + c + k] = y;
    }
    startc[k * W + c] = (double)y;
  }
  __syncthreads();
  if (k == 0 && col < nx) {
    // scanning from the bottom, the carry entering the last non-empty segment is zero, so
    // its (possibly shorter) length never multiplies a nonzero carry
    const double mum = exp((double)m * lmu);
    double run = 0.0;
    for (int q = S - 1; q >= 0; --q) {
      const double e = startc[q * W + c];
      startc[q * W + c] = run;  // true y at the start of segment q + 1
      run = e + mum * run;
    }
    y0c[c] = run;  // true y_0
  }
  __syncthreads();
  if (active && len > 0) {
    const double cin = startc[k * W + c];
    if (cin != 0.0) {
      T pw = tmu;
      const T tc = (T)cin;
      for (int j = j1 - 1; j >= j0; --j) {
        sm[j * ld + c + k] += pw * tc;
        pw *= tmu;
      }
    }
    // Sherman-Morrison correction w_j = y_j - kappa y_0 h_j
    const double coef = kap * y0c[c] * i1m;
    double a = exp((double)j0 * lmu);
    double b = exp((double)(2 * ny - j0) * lmu);
    const double inv_mu = 1.0 / mu;
    for (int j = j0; j < j1; ++j) {
      sm[j * ld + c + k] -= (T)(coef * (a - b));
      a *= mu;
      b *= inv_mu;
    }
  }
  __syncthreads();
  for (int i = tid; i < ny * W; i += blockDim.x) {
    const int row = i / W, cc = i - row * W, cl = c0 + cc;
    if (cl < nx) t[(size_t)row * nx + cl] = sm[row * ld + cc + row / m];
  }
  __syncthreads();
}

}  // namespace fb
