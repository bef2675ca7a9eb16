// Register-resident Stockham FFT for the Bluestein row DST-I (see fb_dst.cuh).
//
// A row of the convolution (length P = 2^logp) is owned by Tr = P / VPT threads, each holding
// VPT complex values in registers. A pass of radix R (R in {2, 4, 8, 16}) computes, for every
// j in [0, P/R), the R-point DFT of the inputs j + r P/R (r < R) after the Stockham twiddle
// W_{Ns R}^{(j mod Ns) r}, and writes output r to position (j / Ns) Ns R + (j mod Ns) + r Ns;
// passes run with Ns = 1, R1, R1 R2, ... and leave natural order. Between passes the row
// goes through shared memory once (padded one slot in 16 to avoid bank conflicts).
//
// The forward transform's last pass and the inverse transform's first pass touch the same
// (j, r) positions, so the pointwise product with the filter happens in registers and the
// inverse starts without a shared-memory round trip. The inverse runs the radix sequence
// in reverse order with conjugate twiddles; its last pass writes natural-order outputs
// straight to the caller.
#pragma once

#include "fb_dst.cuh"

namespace fb {

struct FftPlan {
  int P;          // transform length (power of two)
  int logp;
  int tr;         // threads per row = P / VPT
  int vpt;        // values per thread (16 or 32)
  int npass;      // number of radix passes
  int radix[6];   // forward radix sequence (product = P)
  int rows;       // rows transformed concurrently by one CTA
};

__host__ __device__ inline int fft_pad(int i) { return i + (i >> 4); }

// Exact 16th roots of unity, W16^k = exp(-2 pi i k / 16) (forward sign).
template <class T>
__device__ __forceinline__ Cx<T> w16(int k) {
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, h = (T)0.70710678118654752440;
  k &= 15;
  T c, s;
  switch (k & 3) {
    case 0: c = 1; s = 0; break;
    case 1: c = c1; s = s1; break;
    case 2: c = h; s = h; break;
    default: c = s1; s = c1; break;
  }
  // rotate by quadrant: exp(-i pi/2 * q)
  const int q = k >> 2;
  T re = c, im = -s;
  if (q == 1) { const T t = re; re = im; im = -t; }
  else if (q == 2) { re = -re; im = -im; }
  else if (q == 3) { const T t = re; re = -im; im = t; }
  return Cx<T>{re, im};
}

// In-register DFT of R points (R | 16), natural order in and out. inv selects e^{+i}.
template <class T, int R>
__device__ __forceinline__ void dft_reg(Cx<T> *v, bool inv) {
#pragma unroll
  for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; ++j) {
        const Cx<T> a = v[b + j], c = v[b + j + h];
        v[b + j] = Cx<T>{a.x + c.x, a.y + c.y};
        Cx<T> d{a.x - c.x, a.y - c.y};
        if (j != 0) {
          Cx<T> w = w16<T>(j * (16 / (2 * h)));
          if (inv) w.y = -w.y;
          d = cmul(d, w);
        }
        v[b + j + h] = d;
      }
    }
  }
  // undo the bit reversal of the radix-2 DIF network
#pragma unroll
  for (int i = 0; i < R; ++i) {
    int r = 0;
#pragma unroll
    for (int bit = 1, k = i; bit < R; bit <<= 1, k >>= 1) r = (r << 1) | (k & 1);
    if (r > i) {
      const Cx<T> t = v[i];
      v[i] = v[r];
      v[r] = t;
    }
  }
}

// Twiddle W_P^e from the table tw (P/2 entries of W_P^k, k < P/2), e in [0, P).
template <class T>
__device__ __forceinline__ Cx<T> tw_at(const Cx<T> *__restrict__ tw, int e, int half) {
  if (e < half) return tw[e];
  const Cx<T> w = tw[e - half];
  return Cx<T>{-w.x, -w.y};
}

// Radix-R butterflies of one pass for the q-th group of registers (VPT / R groups).
template <class T, int R, int VPT>
__device__ __forceinline__ void pass_compute(Cx<T> (&v)[VPT], int t, int tr, int P, int Ns, bool inv,
                                             const Cx<T> *__restrict__ tw) {
  const int half = P >> 1;
  const int step = P / (Ns * R);  // twiddle exponent stride
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
    if (Ns > 1) {
      const int e = (j & (Ns - 1)) * step;
#if FB_TWIDDLE_TABLE_ALL
#pragma unroll
      for (int r = 1; r < R; ++r) {
        Cx<T> w = tw_at(tw, (e * r) & (P - 1), half);
        if (inv) w.y = -w.y;
        v[q * R + r] = cmul(v[q * R + r], w);
      }
#else
      // W^{e r} as a product of the table powers W^{e 2^b} over the set bits of r: log2 R
      // table reads per DFT instead of R - 1, at most two extra roundings per twiddle.
      Cx<T> wp[4];
#pragma unroll
      for (int b = 0; (1 << b) < R; ++b) {
        wp[b] = tw_at(tw, (e << b) & (P - 1), half);
        if (inv) wp[b].y = -wp[b].y;
      }
#pragma unroll
      for (int r = 1; r < R; ++r) {
        Cx<T> w{T(1), T(0)};
        bool first = true;
#pragma unroll
        for (int b = 0; (1 << b) < R; ++b) {
          if (r & (1 << b)) {
            w = first ? wp[b] : cmul(w, wp[b]);
            first = false;
          }
        }
        v[q * R + r] = cmul(v[q * R + r], w);
      }
#endif
    }
    dft_reg<T, R>(&v[q * R], inv);
  }
}

template <class T, int R, int VPT>
__device__ __forceinline__ void pass_store(const Cx<T> (&v)[VPT], Cx<T> *row, int t, int tr, int Ns) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
    const int base = (j / Ns) * Ns * R + (j & (Ns - 1));
#pragma unroll
    for (int r = 0; r < R; ++r) row[fft_pad(base + r * Ns)] = v[q * R + r];
  }
}

template <class T, int R, int VPT>
__device__ __forceinline__ void pass_load(Cx<T> (&v)[VPT], const Cx<T> *row, int t, int tr, int P) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = row[fft_pad(j + r * (P / R))];
  }
}

template <class T, int VPT>
__device__ __forceinline__ void pass_compute_any(int R, Cx<T> (&v)[VPT], int t, int tr, int P, int Ns, bool inv,
                                                 const Cx<T> *tw) {
  switch (R) {
    case 16: pass_compute<T, 16, VPT>(v, t, tr, P, Ns, inv, tw); break;
    case 8: pass_compute<T, 8, VPT>(v, t, tr, P, Ns, inv, tw); break;
    case 4: pass_compute<T, 4, VPT>(v, t, tr, P, Ns, inv, tw); break;
    default: pass_compute<T, 2, VPT>(v, t, tr, P, Ns, inv, tw); break;
  }
}
template <class T, int VPT>
__device__ __forceinline__ void pass_store_any(int R, const Cx<T> (&v)[VPT], Cx<T> *row, int t, int tr, int Ns) {
  switch (R) {
    case 16: pass_store<T, 16, VPT>(v, row, t, tr, Ns); break;
    case 8: pass_store<T, 8, VPT>(v, row, t, tr, Ns); break;
    case 4: pass_store<T, 4, VPT>(v, row, t, tr, Ns); break;
    default: pass_store<T, 2, VPT>(v, row, t, tr, Ns); break;
  }
}
template <class T, int VPT>
__device__ __forceinline__ void pass_load_any(int R, Cx<T> (&v)[VPT], const Cx<T> *row, int t, int tr, int P) {
  switch (R) {
    case 16: pass_load<T, 16, VPT>(v, row, t, tr, P); break;
    case 8: pass_load<T, 8, VPT>(v, row, t, tr, P); break;
    case 4: pass_load<T, 4, VPT>(v, row, t, tr, P); break;
    default: pass_load<T, 2, VPT>(v, row, t, tr, P); break;
  }
}

template <class T, int R, int VPT, class In>
__device__ __forceinline__ void stage_input(Cx<T> (&v)[VPT], const DstTables<T> &tb, int t, int tr, int P, bool live,
                                            int row, In in) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * (P / R);
      Cx<T> a{T(0), T(0)};
      if (live && n < tb.n) a = dst_stage(tb, n, in(row, n));
      v[q * R + r] = a;
    }
  }
}

template <class T, int R, int VPT>
__device__ __forceinline__ void apply_filter(Cx<T> (&v)[VPT], const Cx<T> *__restrict__ filt, int t, int tr, int P) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = cmul(v[q * R + r], filt[j + r * (P / R)]);
  }
}

template <class T, int R, int VPT, class Out>
__device__ __forceinline__ void emit_output(const Cx<T> (&v)[VPT], const DstTables<T> &tb, int t, int tr, int P,
                                            bool live, int row, Out out) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * (P / R);
      if (live && n < tb.n) {
        const Cx<T> w = tb.chirp[n + 1];
        const Cx<T> c = v[q * R + r];
        out(row, n, w.x * c.y + w.y * c.x);
      }
    }
  }
}

// Main radix of the register passes: 16 in single precision; 8 in double precision, where
// 16 complex doubles plus twiddles exceed the register budget of a 512-thread CTA.
template <class T>
struct MainRadix {
  static constexpr int value = sizeof(T) == 4 ? 16 : 8;
};

// Body of the row transform for a first-pass radix R0; all further passes use kMainRadix.
template <class T, int VPT, int R0, class In, class Out>
__device__ __forceinline__ void dst_rows_body(const DstTables<T> &tb, const FftPlan &pl, Cx<T> *rowbuf, bool active,
                                              bool live, int row, int t, In in, Out out) {
  constexpr int kMainRadix = MainRadix<T>::value;
  const int P = pl.P, tr = pl.tr, nm = pl.npass - 1;
  Cx<T> v[VPT];
  stage_input<T, R0, VPT>(v, tb, t, tr, P, live, row, in);
  pass_compute<T, R0, VPT>(v, t, tr, P, 1, false, tb.tw);
  int Ns = R0;
  if (nm > 0) {
    if (active) pass_store<T, R0, VPT>(v, rowbuf, t, tr, 1);
    __syncthreads();
    if (active) pass_load<T, kMainRadix, VPT>(v, rowbuf, t, tr, P);
    __syncthreads();
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, kMainRadix, VPT>(v, t, tr, P, Ns, false, tb.tw);
      if (ps + 1 < nm) {
        if (active) pass_store<T, kMainRadix, VPT>(v, rowbuf, t, tr, Ns);
        __syncthreads();
        if (active) pass_load<T, kMainRadix, VPT>(v, rowbuf, t, tr, P);
        __syncthreads();
      }
      Ns *= kMainRadix;
    }
    // filter in natural frequency order, then the inverse runs radix-16 passes first
    apply_filter<T, kMainRadix, VPT>(v, tb.filt, t, tr, P);
    Ns = 1;
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, kMainRadix, VPT>(v, t, tr, P, Ns, true, tb.tw);
      if (active) pass_store<T, kMainRadix, VPT>(v, rowbuf, t, tr, Ns);
      __syncthreads();
      if (ps + 1 < nm) {
        if (active) pass_load<T, kMainRadix, VPT>(v, rowbuf, t, tr, P);
      } else {
        if (active) pass_load<T, R0, VPT>(v, rowbuf, t, tr, P);
      }
      __syncthreads();
      Ns *= kMainRadix;
    }
    pass_compute<T, R0, VPT>(v, t, tr, P, Ns, true, tb.tw);
  } else {
    apply_filter<T, R0, VPT>(v, tb.filt, t, tr, P);
    pass_compute<T, R0, VPT>(v, t, tr, P, 1, true, tb.tw);
  }
  // the last inverse pass (radix R0, Ns = P / R0) left output n = j + r P/R0
  emit_output<T, R0, VPT>(v, tb, t, tr, P, live, row, out);
}

// Orthonormal DST-I of rows [row0, row0 + plan.rows) of an (ny, N) array. `in(row, n)`
// returns input n < N of a row; `out(row, n, value)` receives output n < N. Rows beyond ny
// are computed on zeros and not stored. VPT and the first-pass radix R0 must match the
// plan (they are template parameters so one kernel holds exactly one transform body).
// Every thread of the CTA must call this.
template <class T, int VPT, int R0, class In, class Out>
__device__ __forceinline__ void dst_rows_regs(const DstTables<T> &tb, const FftPlan &pl, Cx<T> *smem, int row0, int ny,
                                              In in, Out out) {
  const int slot = threadIdx.x / pl.tr;
  const int t = threadIdx.x - slot * pl.tr;
  const bool active = slot < pl.rows;
  const int row = row0 + slot;
  const bool live = active && row < ny;
  Cx<T> *rowbuf = smem + (size_t)(active ? slot : 0) * fft_pad(pl.P);
  dst_rows_body<T, VPT, R0>(tb, pl, rowbuf, active, live, row, t, in, out);
}

// Host-side plan: main-radix passes, the first pass taking the remaining factor (or the
// main radix); VPT = main radix values per thread, more when a row would need over
// `threads`.
inline FftPlan make_fft_plan(int P, int logp, int threads, size_t smem_budget, size_t csz) {
  const int kMainRadix = csz == 8 ? MainRadix<float>::value : MainRadix<double>::value;
  FftPlan pl{};
  pl.P = P;
  pl.logp = logp;
  pl.vpt = kMainRadix;
  while (P / pl.vpt > threads) pl.vpt *= 2;
  pl.tr = P / pl.vpt;
  if (pl.tr < 1) pl.tr = 1;
  const int lm = kMainRadix == 16 ? 4 : 3;
  const int rem = logp % lm;
  int n = 0;
  pl.radix[n++] = rem ? (1 << rem) : kMainRadix;
  for (int k = 0; k < (logp - (rem ? rem : lm)) / lm; ++k) pl.radix[n++] = kMainRadix;
  pl.npass = n;
  int rows = threads / pl.tr;
  const size_t row_bytes = (size_t)fft_pad(P) * csz;
  while (rows > 1 && (size_t)rows * row_bytes > smem_budget) --rows;
  pl.rows = rows < 1 ? 1 : rows;
  return pl;
}

}  // namespace fb
