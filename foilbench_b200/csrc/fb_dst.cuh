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
// i.e. a circular convolution of length Pf >= 2N - 1 (power of two) evaluated with a
// radix-2 decimation-in-frequency FFT, a pointwise product with the precomputed transform
// of conj(w) (kept in the same bit-reversed order, so no permutation pass is needed) and a
// decimation-in-time inverse FFT. The DST-I value is sqrt(2/L) Im(w_k conv_k); the factor
// and the 1/Pf inverse-FFT scale are folded into the filter table.
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

// In-place radix-2 DIF forward FFT (e^{-2 pi i jk / Pf}) of R rows of length Pf held in
// shared memory; natural order in, bit-reversed order out. tw[k] = e^{-2 pi i k / Pf},
// k < Pf/2.
template <class T>
__device__ __forceinline__ void fft_dif_rows(Cx<T> *buf, int rows, int logp, const Cx<T> *__restrict__ tw) {
  const int half = 1 << (logp - 1);
  const int total = rows << (logp - 1);
  for (int s = 0; s < logp; ++s) {
    const int lh = logp - 1 - s;
    const int h = 1 << lh;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int row = b >> (logp - 1);
      const int k = b & (half - 1);
      const int j = k & (h - 1);
      const int i0 = ((k >> lh) << (lh + 1)) + j;
      Cx<T> *base = buf + ((size_t)row << logp);
      const Cx<T> a = base[i0], c = base[i0 + h];
      base[i0] = Cx<T>{a.x + c.x, a.y + c.y};
      base[i0 + h] = cmul(Cx<T>{a.x - c.x, a.y - c.y}, tw[j << s]);
    }
    __syncthreads();
  }
}

// In-place radix-2 DIT inverse FFT (e^{+2 pi i jk / Pf}, unnormalised); bit-reversed order
// in, natural order out.
template <class T>
__device__ __forceinline__ void fft_dit_inv_rows(Cx<T> *buf, int rows, int logp, const Cx<T> *__restrict__ tw) {
  const int half = 1 << (logp - 1);
  const int total = rows << (logp - 1);
  for (int s = logp - 1; s >= 0; --s) {
    const int lh = logp - 1 - s;
    const int h = 1 << lh;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int row = b >> (logp - 1);
      const int k = b & (half - 1);
      const int j = k & (h - 1);
      const int i0 = ((k >> lh) << (lh + 1)) + j;
      Cx<T> *base = buf + ((size_t)row << logp);
      const Cx<T> a = base[i0];
      const Cx<T> c = cmulc(base[i0 + h], tw[j << s]);
      base[i0] = Cx<T>{a.x + c.x, a.y + c.y};
      base[i0 + h] = Cx<T>{a.x - c.x, a.y - c.y};
    }
    __syncthreads();
  }
}

// Tables for the row transform of length N (device memory, precision T).
template <class T>
struct DstTables {
  const Cx<T> *chirp;  // w_m, m = 0..N
  const Cx<T> *filt;   // DIF(conj(w)) * sqrt(2/L) / Pf, bit-reversed order, Pf entries
  const Cx<T> *tw;     // e^{-2 pi i k / Pf}, k < Pf/2
  int n;               // N
  int logp;            // log2(Pf)
};

// Orthonormal DST-I of `rows` rows staged by the caller: buf holds, for each row, the
// complex sequence a_n = x_{n+1} w_{n+1} (n < N) followed by zeros up to Pf. On return
// buf[row * Pf + k] holds the convolution whose imaginary part after multiplying by
// w_{k+1} is the transform; use dst_value() to read it.
template <class T>
__device__ __forceinline__ void dst_rows_core(Cx<T> *buf, int rows, const DstTables<T> &tb) {
  fft_dif_rows(buf, rows, tb.logp, tb.tw);
  const int pf = 1 << tb.logp;
  const int total = rows << tb.logp;
  for (int i = threadIdx.x; i < total; i += blockDim.x) buf[i] = cmul(buf[i], tb.filt[i & (pf - 1)]);
  __syncthreads();
  fft_dit_inv_rows(buf, rows, tb.logp, tb.tw);
}

template <class T>
__device__ __forceinline__ T dst_value(const Cx<T> *buf_row, const DstTables<T> &tb, int k) {
  const Cx<T> w = tb.chirp[k + 1];
  const Cx<T> c = buf_row[k];
  return w.x * c.y + w.y * c.x;  // Im(w * c)
}

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
// x fastest), in place. sm: (ny x (W + 1)) tile of T plus 3 * S * W doubles of carries.
template <class T>
__device__ void column_solve_tile(T *__restrict__ t, int nx, int ny, int c0, int W, double dy2,
                                  const ColTables &ct, T *sm, double *carry) {
  const int ld = W + 1;
  const int S = blockDim.x / W;
  const int tid = threadIdx.x;
  for (int i = tid; i < ny * W; i += blockDim.x) {
    const int row = i / W, c = i - row * W, col = c0 + c;
    sm[row * ld + c] = col < nx ? t[(size_t)row * nx + col] : T(0);
  }
  __syncthreads();
  const int k = tid / W, c = tid - (tid / W) * W, col = c0 + c;
  const bool active = (k < S) && (col < nx);
  const int m = (ny + S - 1) / S;
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
      s = tmu * ((T)dy2 * sm[j * ld + c] + s);
      sm[j * ld + c] = s;
    }
    endc[k * W + c] = (double)s;
  }
  __syncthreads();
  if (k == 0 && col < nx) {
    double run = 0.0;
    for (int q = 0; q < S; ++q) {
      const int a0 = q * m, a1 = min(a0 + m, ny);
      const int l = a1 > a0 ? a1 - a0 : 0;
      const double e = endc[q * W + c];
      endc[q * W + c] = run;  // carry-in for segment q
      run = e + exp((double)l * lmu) * run;
    }
  }
  __syncthreads();
  if (active) {
    const double cin = endc[k * W + c];
    if (cin != 0.0) {
      T pw = tmu;
      const T tc = (T)cin;
      for (int j = j0; j < j1; ++j) {
        sm[j * ld + c] += pw * tc;
        pw *= tmu;
      }
    }
    // anti-causal: y_j = s_j + mu y_{j+1}
    T y = T(0);
    for (int j = j1 - 1; j >= j0; --j) {
      y = sm[j * ld + c] + tmu * y;
      sm[j * ld + c] = y;
    }
    startc[k * W + c] = (double)y;
  }
  __syncthreads();
  if (k == 0 && col < nx) {
    double run = 0.0;
    for (int q = S - 1; q >= 0; --q) {
      const int a0 = q * m, a1 = min(a0 + m, ny);
      const int l = a1 > a0 ? a1 - a0 : 0;
      const double e = startc[q * W + c];
      startc[q * W + c] = run;  // true y at the start of segment q + 1
      run = e + exp((double)l * lmu) * run;
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
        sm[j * ld + c] += pw * tc;
        pw *= tmu;
      }
    }
    // Sherman-Morrison correction w_j = y_j - kappa y_0 h_j
    const double coef = kap * y0c[c] * i1m;
    double a = exp((double)j0 * lmu);
    double b = exp((double)(2 * ny - j0) * lmu);
    const double inv_mu = 1.0 / mu;
    for (int j = j0; j < j1; ++j) {
      sm[j * ld + c] -= (T)(coef * (a - b));
      a *= mu;
      b *= inv_mu;
    }
  }
  __syncthreads();
  for (int i = tid; i < ny * W; i += blockDim.x) {
    const int row = i / W, cc = i - row * W, cl = c0 + cc;
    if (cl < nx) t[(size_t)row * nx + cl] = sm[row * ld + cc];
  }
  __syncthreads();
}

}  // namespace fb
