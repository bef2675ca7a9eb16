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

#include <cmath>

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
  // Per-pass twiddle tables (entries of Cx, see fft_pass_twiddles): the forward passes 1..
  // (Ns = R0, R0 M, ...) are stored back to back from twf1; the inverse passes 1.. before
  // the last (Ns = M, M^2, ...) from twi1; the last inverse pass (radix R0) at twi_last.
  int twf1, twi1, twi_last;
  int tw_entries;
  // Shared staging of row inputs (step kernel with shared tables): byte offset of the area
  // and bytes per row slot (two halves: input row + mask, output-side r + mask).
  int io_soff, io_slot;
};

__host__ __device__ inline int fft_pad(int i) { return i + (i >> 4); }

// Barrier of the tr threads that transform one row (slot): a named barrier (ids 1..8, id 0
// being __syncthreads) when a row spans whole warps, the warp barrier when rows share a warp.
// Rows of one CTA therefore run their passes independently of each other.
__device__ __forceinline__ void slot_sync(int slot, int tr) {
  if (tr <= 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(slot + 1), "r"(tr) : "memory");
  }
}

// d * W16^k (forward, W16 = exp(-2 pi i / 16)) or d * conj(W16^k) (inverse). k is a
// compile-time constant after unrolling, so the quarter turns reduce to moves and signs.
template <class T>
__device__ __forceinline__ Cx<T> mul_w16(Cx<T> d, int k, bool inv) {
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, h = (T)0.70710678118654752440;
  k &= 15;
  if (k == 0) return d;
  if (k == 8) return Cx<T>{-d.x, -d.y};
  if (k == 4) return inv ? Cx<T>{-d.y, d.x} : Cx<T>{d.y, -d.x};
  if (k == 12) return inv ? Cx<T>{d.y, -d.x} : Cx<T>{-d.y, d.x};
  T c, sn;
  switch (k & 3) {
    case 1: c = c1; sn = s1; break;
    case 2: c = h; sn = h; break;
    default: c = s1; sn = c1; break;
  }
  T re = c, im = -sn;  // W16^(k mod 4) in the first quadrant, then rotate by -pi/2 (k >> 2) times
  const int q = k >> 2;
  if (q == 1) { const T t = re; re = im; im = -t; }
  else if (q == 2) { re = -re; im = -im; }
  else if (q == 3) { const T t = re; re = -im; im = t; }
  if (inv) im = -im;
  return cmul(d, Cx<T>{re, im});
}

// In-register DFT of R points (R | 16), natural order in and out. INV selects e^{+i}.
template <class T, int R, bool INV>
__device__ __forceinline__ void dft_reg(Cx<T> *v) {
#pragma unroll
  for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; ++j) {
        const Cx<T> a = v[b + j], c = v[b + j + h];
        v[b + j] = Cx<T>{a.x + c.x, a.y + c.y};
        v[b + j + h] = mul_w16<T>(Cx<T>{a.x - c.x, a.y - c.y}, j * (16 / (2 * h)), INV);
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

// Radix-R butterflies of one pass (VPT / R groups per thread). For Ns > 1 the inputs r >= 1
// of group j first take the Stockham twiddle W_{Ns R}^{(j mod Ns) r}, read from this pass's
// table tw[(r - 1) Ns + (j mod Ns)] (conjugated for the inverse).
template <class T, int R, int VPT, bool INV>
__device__ __forceinline__ void pass_compute(Cx<T> (&v)[VPT], int t, int tr, int Ns, const Cx<T> *__restrict__ tw) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    if (Ns > 1) {
      const Cx<T> *w = tw + ((t + q * tr) & (Ns - 1));
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const Cx<T> ww = w[(r - 1) * Ns];
        v[q * R + r] = INV ? cmulc(v[q * R + r], ww) : cmul(v[q * R + r], ww);
      }
    }
    dft_reg<T, R, INV>(&v[q * R]);
  }
}

// pass_compute with twiddles from the two-level table: W_{Ns R}^{jm r} = W_P^{e},
// e = jm r P / (Ns R) mod P, formed as tw_hi[e >> 7] * tw_lo[e & 127] (one product, so a
// long transform needs only P / 128 + 128 table entries).
template <class T, int R, int VPT, bool INV>
__device__ __forceinline__ void pass_compute_tw2(Cx<T> (&v)[VPT], int t, int tr, int Ns, int P,
                                                 const Cx<T> *__restrict__ lo, const Cx<T> *__restrict__ hi) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    if (Ns > 1) {
      const int e1 = ((t + q * tr) & (Ns - 1)) * (P / (Ns * R));
      int e = 0;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        e = (e + e1) & (P - 1);
        const Cx<T> w = cmul(hi[e >> 7], lo[e & 127]);
        v[q * R + r] = INV ? cmulc(v[q * R + r], w) : cmul(v[q * R + r], w);
      }
    }
    dft_reg<T, R, INV>(&v[q * R]);
  }
}

// Output r of group j goes to position (j / Ns) Ns R + (j mod Ns) + r Ns. With the padding
// of one slot per 16, the R addresses of a group are a constant stride apart whenever Ns is
// 1 (the group stays inside one 16-slot line) or a multiple of 16.
template <class T, int R, int VPT>
__device__ __forceinline__ void pass_store(const Cx<T> (&v)[VPT], Cx<T> *row, int t, int tr, int Ns) {
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
    const int jm = j & (Ns - 1);
    const int base = (j - jm) * R + jm;
    Cx<T> *p = row + fft_pad(base);
    if (Ns == 1) {
#pragma unroll
      for (int r = 0; r < R; ++r) p[r] = v[q * R + r];
    } else if ((Ns & 15) == 0) {
      const int st = Ns + (Ns >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) p[r * st] = v[q * R + r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) row[fft_pad(base + r * Ns)] = v[q * R + r];
    }
  }
}

// Inputs of group j are positions j + r P / R.
template <class T, int R, int VPT>
__device__ __forceinline__ void pass_load(Cx<T> (&v)[VPT], const Cx<T> *row, int t, int tr, int P) {
  const int S = P / R;
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
    if ((S & 15) == 0) {
      const Cx<T> *p = row + fft_pad(j);
      const int st = S + (S >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = p[r * st];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = row[fft_pad(j + r * S)];
    }
  }
}

template <class T, int R, int VPT, class In>
__device__ __forceinline__ void stage_input(Cx<T> (&v)[VPT], const DstTables<T> &tb, int t, int tr, int P, bool live,
                                            int row, In in) {
  const int S = P / R;
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * S;
      Cx<T> a{T(0), T(0)};
      if (live && n < tb.n) a = dst_stage(tb, n, in(row, n));
      v[q * R + r] = a;
    }
  }
}

template <class T, int R, int VPT>
__device__ __forceinline__ void apply_filter(Cx<T> (&v)[VPT], const Cx<T> *__restrict__ filt, int t, int tr, int P) {
  const int S = P / R;
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const Cx<T> *f = filt + t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = cmul(v[q * R + r], f[r * S]);
  }
}

template <class T, int R, int VPT, class Out>
__device__ __forceinline__ void emit_output(const Cx<T> (&v)[VPT], const DstTables<T> &tb, int t, int tr, int P,
                                            bool live, int row, Out out) {
  const int S = P / R;
#pragma unroll
  for (int q = 0; q < VPT / R; ++q) {
    const int j = t + q * tr;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * S;
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

// Body of the row transform for a first-pass radix R0; all further passes use the main
// radix M. Forward radices R0, M, M, ...; the inverse runs them in reverse order.
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

// `after_in()` runs once the row's inputs are in registers (the staging buffer may be
// refilled), `before_out()` right before the outputs are emitted.
template <class T, int VPT, int R0, class In, class Out, class AfterIn, class BeforeOut>
__device__ __forceinline__ void dst_rows_body(const DstTables<T> &tb, const FftPlan &pl, Cx<T> *rowbuf, bool active,
                                              bool live, int row, int t, int slot, In in, Out out, AfterIn after_in,
                                              BeforeOut before_out) {
  constexpr int M = MainRadix<T>::value;
  const int P = pl.P, tr = pl.tr, nm = pl.npass - 1;
  Cx<T> v[VPT];
  stage_input<T, R0, VPT>(v, tb, t, tr, P, live, row, in);
  after_in();
  pass_compute<T, R0, VPT, false>(v, t, tr, 1, tb.twp);
  if (nm > 0) {
    if (active) pass_store<T, R0, VPT>(v, rowbuf, t, tr, 1);
    slot_sync(slot, tr);
    if (active) pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
    slot_sync(slot, tr);
    int Ns = R0;
    const Cx<T> *tw = tb.twp + pl.twf1;
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, M, VPT, false>(v, t, tr, Ns, tw);
      if (ps + 1 < nm) {
        if (active) pass_store<T, M, VPT>(v, rowbuf, t, tr, Ns);
        slot_sync(slot, tr);
        if (active) pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
        slot_sync(slot, tr);
      }
      tw += (M - 1) * Ns;
      Ns *= M;
    }
    // filter in natural frequency order, then the inverse runs the main-radix passes first
    apply_filter<T, M, VPT>(v, tb.filt, t, tr, P);
    Ns = 1;
    tw = tb.twp + pl.twi1;
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, M, VPT, true>(v, t, tr, Ns, tw);
      if (active) pass_store<T, M, VPT>(v, rowbuf, t, tr, Ns);
      slot_sync(slot, tr);
      if (ps + 1 < nm) {
        if (active) pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
      } else {
        if (active) pass_load<T, R0, VPT>(v, rowbuf, t, tr, P);
      }
      slot_sync(slot, tr);
      if (Ns > 1) tw += (M - 1) * Ns;
      Ns *= M;
    }
    pass_compute<T, R0, VPT, true>(v, t, tr, Ns, tb.twp + pl.twi_last);
  } else {
    apply_filter<T, R0, VPT>(v, tb.filt, t, tr, P);
    pass_compute<T, R0, VPT, true>(v, t, tr, 1, tb.twp);
  }
  // the last inverse pass (radix R0, Ns = P / R0) left output n = j + r P/R0
  before_out();
  emit_output<T, R0, VPT>(v, tb, t, tr, P, live, row, out);
}

// Fixed-shape body for three radix passes (P = R0 M^2, the 512..4096-point transforms of
// the production grids): every stride, pass size and table offset is a compile-time
// constant, so the transform keeps only its values and a few addresses in registers. The
// table layout is the one make_fft_plan builds for npass = 3.
template <class T, int VPT, int R0, class In, class Out, class AfterIn, class BeforeOut>
__device__ __forceinline__ void dst_rows_body3(const DstTables<T> &tb, Cx<T> *rowbuf, bool active, bool live, int row,
                                               int t, int slot, In in, Out out, AfterIn after_in,
                                               BeforeOut before_out) {
  constexpr int M = MainRadix<T>::value;
  constexpr int P = R0 * M * M;
  constexpr int TR = P / VPT;
  constexpr int TWF1 = 0, TWF2 = (M - 1) * R0, FEND = TWF2 + (M - 1) * R0 * M;
  constexpr int TWI1 = R0 == M ? TWF1 : FEND;
  constexpr int TWIL = R0 == M ? TWF2 : FEND + (M - 1) * M;
  Cx<T> v[VPT];
  stage_input<T, R0, VPT>(v, tb, t, TR, P, live, row, in);
  after_in();
  // forward: radices R0, M, M
  pass_compute<T, R0, VPT, false>(v, t, TR, 1, tb.twp);
  if (active) pass_store<T, R0, VPT>(v, rowbuf, t, TR, 1);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute<T, M, VPT, false>(v, t, TR, R0, tb.twp + TWF1);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, R0);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute<T, M, VPT, false>(v, t, TR, R0 * M, tb.twp + TWF2);
  apply_filter<T, M, VPT>(v, tb.filt, t, TR, P);
  // inverse: radices M, M, R0
  pass_compute<T, M, VPT, true>(v, t, TR, 1, tb.twp);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, 1);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute<T, M, VPT, true>(v, t, TR, M, tb.twp + TWI1);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, M);
  slot_sync(slot, TR);
  if (active) pass_load<T, R0, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute<T, R0, VPT, true>(v, t, TR, M * M, tb.twp + TWIL);
  before_out();
  emit_output<T, R0, VPT>(v, tb, t, TR, P, live, row, out);
}

// Fixed-shape body for four radix passes (P = R0 M^3, the 2^13..2^16-point transforms of
// grids over 2048 columns), twiddles from the two-level table (DstTables::tw_lo / tw_hi).
template <class T, int VPT, int R0, class In, class Out, class AfterIn, class BeforeOut>
__device__ __forceinline__ void dst_rows_body4(const DstTables<T> &tb, Cx<T> *rowbuf, bool active, bool live, int row,
                                               int t, int slot, In in, Out out, AfterIn after_in,
                                               BeforeOut before_out) {
  constexpr int M = MainRadix<T>::value;
  constexpr int P = R0 * M * M * M;
  constexpr int TR = P / VPT;
  const Cx<T> *lo = tb.tw_lo, *hi = tb.tw_hi;
  Cx<T> v[VPT];
  stage_input<T, R0, VPT>(v, tb, t, TR, P, live, row, in);
  after_in();
  // forward: radices R0, M, M, M
  pass_compute_tw2<T, R0, VPT, false>(v, t, TR, 1, P, lo, hi);
  if (active) pass_store<T, R0, VPT>(v, rowbuf, t, TR, 1);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, M, VPT, false>(v, t, TR, R0, P, lo, hi);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, R0);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, M, VPT, false>(v, t, TR, R0 * M, P, lo, hi);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, R0 * M);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, M, VPT, false>(v, t, TR, R0 * M * M, P, lo, hi);
  apply_filter<T, M, VPT>(v, tb.filt, t, TR, P);
  // inverse: radices M, M, M, R0
  pass_compute_tw2<T, M, VPT, true>(v, t, TR, 1, P, lo, hi);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, 1);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, M, VPT, true>(v, t, TR, M, P, lo, hi);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, M);
  slot_sync(slot, TR);
  if (active) pass_load<T, M, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, M, VPT, true>(v, t, TR, M * M, P, lo, hi);
  if (active) pass_store<T, M, VPT>(v, rowbuf, t, TR, M * M);
  slot_sync(slot, TR);
  if (active) pass_load<T, R0, VPT>(v, rowbuf, t, TR, P);
  slot_sync(slot, TR);
  pass_compute_tw2<T, R0, VPT, true>(v, t, TR, M * M * M, P, lo, hi);
  before_out();
  emit_output<T, R0, VPT>(v, tb, t, TR, P, live, row, out);
}

// One row's DST-I with the Bluestein convolution split in two halves, for rows whose
// length-2^ceil(log2(2N - 1)) convolution would not fit one CTA (double precision, N over
// 4096). With h = tb.split_h = ceil(N / 2), input half i holds a_m for m in [i h, i h + h)
// and output half o the outputs n in [o h, o h + h); their differences n - m = d h + x with
// d = o - i and |x| < h, so each (o, i) pair is a circular convolution of length P >= 2 h
// without wrap-around, against the filter slice d (tb.filt + (d + 1) P, the spectrum of
// b_{d h + x}). The forward spectra G_0, G_1 of the two input halves go to this CTA's scratch
// `spec` (2 P values, each thread reading back only the positions it wrote), and output half
// o is the inverse transform of G_0 H_(o - 0) + G_1 H_(o - 1). Same passes, tables and
// emission as dst_rows_body; the plan has one row per CTA (tr = blockDim.x).
template <class T, int VPT, int R0, class In, class Out>
__device__ __forceinline__ void dst_rows_split2(const DstTables<T> &tb, const FftPlan &pl, Cx<T> *rowbuf,
                                                Cx<T> *__restrict__ spec, int row, bool live, int t, In in, Out out) {
  constexpr int M = MainRadix<T>::value;
  const int P = pl.P, tr = pl.tr, nm = pl.npass - 1, h = tb.split_h;
  const int S0 = P / R0, SM = P / M;
#pragma unroll 1
  for (int i = 0; i < 2; ++i) {
    Cx<T> v[VPT];
#pragma unroll
    for (int q = 0; q < VPT / R0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int m = t + q * tr + r * S0, n = i * h + m;
        Cx<T> a{T(0), T(0)};
        if (live && m < h && n < tb.n) a = dst_stage(tb, n, in(row, n));
        v[q * R0 + r] = a;
      }
    pass_compute<T, R0, VPT, false>(v, t, tr, 1, tb.twp);
    pass_store<T, R0, VPT>(v, rowbuf, t, tr, 1);
    slot_sync(0, tr);
    pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
    slot_sync(0, tr);
    int Ns = R0;
    const Cx<T> *tw = tb.twp + pl.twf1;
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, M, VPT, false>(v, t, tr, Ns, tw);
      if (ps + 1 < nm) {
        pass_store<T, M, VPT>(v, rowbuf, t, tr, Ns);
        slot_sync(0, tr);
        pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
        slot_sync(0, tr);
      }
      tw += (M - 1) * Ns;
      Ns *= M;
    }
    // spectrum value (q, r) is frequency t + q tr + r P / M; scratch index (q M + r) tr + t
    Cx<T> *g = spec + (size_t)i * P;
#pragma unroll
    for (int k = 0; k < VPT; ++k) g[k * tr + t] = v[k];
  }
#pragma unroll 1
  for (int o = 0; o < 2; ++o) {
    Cx<T> v[VPT];
    const Cx<T> *h0 = tb.filt + (size_t)(o + 1) * P;  // d = o - 0
    const Cx<T> *h1 = tb.filt + (size_t)o * P;        // d = o - 1
#pragma unroll
    for (int q = 0; q < VPT / M; ++q)
#pragma unroll
      for (int r = 0; r < M; ++r) {
        const int k = q * M + r, f = t + q * tr + r * SM;
        const Cx<T> a = cmul(spec[k * tr + t], h0[f]), b = cmul(spec[(size_t)P + k * tr + t], h1[f]);
        v[k] = Cx<T>{a.x + b.x, a.y + b.y};
      }
    int Ns = 1;
    const Cx<T> *tw = tb.twp + pl.twi1;
#pragma unroll 1
    for (int ps = 0; ps < nm; ++ps) {
      pass_compute<T, M, VPT, true>(v, t, tr, Ns, tw);
      pass_store<T, M, VPT>(v, rowbuf, t, tr, Ns);
      slot_sync(0, tr);
      if (ps + 1 < nm)
        pass_load<T, M, VPT>(v, rowbuf, t, tr, P);
      else
        pass_load<T, R0, VPT>(v, rowbuf, t, tr, P);
      slot_sync(0, tr);
      if (Ns > 1) tw += (M - 1) * Ns;
      Ns *= M;
    }
    pass_compute<T, R0, VPT, true>(v, t, tr, Ns, tb.twp + pl.twi_last);
#pragma unroll
    for (int q = 0; q < VPT / R0; ++q)
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int m = t + q * tr + r * S0, n = o * h + m;
        if (live && m < h && n < tb.n) {
          const Cx<T> w = tb.chirp[n + 1], c = v[q * R0 + r];
          out(row, n, w.x * c.y + w.y * c.x);
        }
      }
  }
}

// Orthonormal DST-I of rows [row0, row0 + plan.rows) of an (ny, N) array. `in(row, n)`
// returns input n < N of a row; `out(row, n, value)` receives output n < N. Rows beyond ny
// are computed on zeros and not stored. VPT and the first-pass radix R0 must match the
// plan (they are template parameters so one kernel holds exactly one transform body).
// Every thread of the CTA must call this; the threads of one row synchronise only among
// themselves (slot_sync), so the caller separates uses of the row buffer by other rows.
template <class T, int VPT, int R0, class In, class Out, class AfterIn = NoHook, class BeforeOut = NoHook>
__device__ __forceinline__ void dst_rows_regs(const DstTables<T> &tb, const FftPlan &pl, Cx<T> *smem, int row0, int ny,
                                              In in, Out out, AfterIn after_in = AfterIn(),
                                              BeforeOut before_out = BeforeOut()) {
  const int slot = threadIdx.x / pl.tr;
  const int t = threadIdx.x - slot * pl.tr;
  const bool active = slot < pl.rows;
  const int row = row0 + slot;
  const bool live = active && row < ny;
  Cx<T> *rowbuf = smem + (size_t)(active ? slot : 0) * fft_pad(pl.P);
  dst_rows_body<T, VPT, R0>(tb, pl, rowbuf, active, live, row, t, slot, in, out, after_in, before_out);
}

// Host-side plan: main-radix passes, the first pass taking the remaining factor (or the
// main radix); VPT = main radix values per thread, more when a row would need over
// `threads`. Also lays out the per-pass twiddle tables (fft_pass_twiddles).
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
  // twiddle tables: forward passes 1.. (Ns = R0 M^(k-1)); inverse passes 1..npass-2
  // (Ns = M^k); last inverse pass (radix R0, Ns = P / R0). When R0 == M the inverse
  // tables coincide with the forward ones.
  const int R0 = pl.radix[0], M = kMainRadix;
  int off = 0;
  pl.twf1 = 0;
  for (int k = 1, Ns = R0; k < n; ++k, Ns *= M) off += (M - 1) * Ns;
  if (R0 == M) {
    pl.twi1 = 0;
    pl.twi_last = n > 1 ? off - (M - 1) * (P / M) : 0;
  } else {
    pl.twi1 = off;
    for (int k = 1, Ns = M; k < n - 1; ++k, Ns *= M) off += (M - 1) * Ns;
    pl.twi_last = off;
    if (n > 1) off += (R0 - 1) * (P / R0);
  }
  pl.tw_entries = off > 0 ? off : 1;
  return pl;
}

// Values of the per-pass twiddle tables laid out by make_fft_plan, as interleaved
// (re, im) doubles with the forward sign: entry (r - 1) Ns + jm = exp(-2 pi i jm r / (Ns R)).
inline void fft_pass_twiddles(const FftPlan &pl, int main_radix, double *out) {
  const int n = pl.npass, R0 = pl.radix[0], M = main_radix, P = pl.P;
  auto fill = [&](int off, int Ns, int R) {
    for (int r = 1; r < R; ++r)
      for (int jm = 0; jm < Ns; ++jm) {
        const long long e = ((long long)jm * r) % ((long long)Ns * R);
        const double a = -2.0 * 3.14159265358979323846 * (double)e / ((double)Ns * R);
        out[2 * (off + (r - 1) * Ns + jm)] = std::cos(a);
        out[2 * (off + (r - 1) * Ns + jm) + 1] = std::sin(a);
      }
  };
  int off = pl.twf1;
  for (int k = 1, Ns = R0; k < n; ++k, Ns *= M) {
    fill(off, Ns, M);
    off += (M - 1) * Ns;
  }
  if (R0 != M && n > 1) {
    off = pl.twi1;
    for (int k = 1, Ns = M; k < n - 1; ++k, Ns *= M) {
      fill(off, Ns, M);
      off += (M - 1) * Ns;
    }
    fill(pl.twi_last, P / R0, R0);
  }
}

}  // namespace fb
