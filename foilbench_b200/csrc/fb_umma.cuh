// Row DST-I of the pressure preconditioner on the 5th-generation tensor cores (tcgen05, TF32
// operands, FP32 accumulators in tensor memory), for the mixed scheme's FP32 inner CG.
//
// The row transform of fb_dst.cuh (_scipy_adapter.py:76-96 applies the orthonormal DST-I
// along x) is a product with the symmetric matrix S[n][k] = sqrt(2/L) sin(pi n k / L),
// L = N + 1. Because S[n][L - k] = (-1)^(n+1) S[n][k], splitting the sum by the parity of n
// halves the work:
//     O_k = sum_{n odd} x_n S[n][k],  E_k = sum_{n even} x_n S[n][k]     (k = 1 .. Kh)
//     y_k = O_k + E_k,  y_{L-k} = O_k - E_k                              (Kh = ceil(N / 2))
// so a transform of an (ny x N) array is two GEMMs (ny x Kh) . (Kh x Kh), one per parity.
// A work unit is one parity of a 128-wavenumber x 128-row output tile: the DST table is the
// MMA's M operand (wavenumbers on the TMEM lanes), the data the N operand (rows on the TMEM
// columns), one 128-column FP32 accumulator, K swept in blocks of 32 sum indices (one
// 128-byte swizzle atom row of FP32). A unit never switches accumulators (switching between
// two accumulators every block halves the tensor core's rate). Each block's two operand tiles
// are brought into shared memory by bulk asynchronous copies from operands that are already
// laid out in global memory exactly as the tensor core reads them (K-major, 128-byte
// swizzle: 16-byte chunk c of row r at chunk c ^ (r & 7) of the row, 8-row atoms of 1024
// bytes), so no tensor map is needed. The unit writes its partial sums (O or E) straight
// from the TMEM registers: lane = wavenumber, so a warp's store covers 32 consecutive
// wavenumbers of one row. Each unit puts its sums at k and, with the parity's sign (+ for
// odd n, - for even n), at the mirror L - k, so that y_k = O_k + E_k and y_{L-k} = O_k - E_k
// are elementwise sums of the two parities' contributions:
//   first transform: stores into two parity arrays (odd -> out1, even -> out2), which the
//     column solve adds while reading;
//   second transform: red.global.add of both parities into out2, zeroed by the column solve;
//     every element receives exactly two additions onto zero, so the result does not depend
//     on their order.
// No unit waits for another.
//
// Operands (every tile 128 rows x 32 values, [blocks of 128 rows][parity][nkb] tiles):
//   table  rows = output wavenumbers k = 128 wb + row + 1, values S[n][k] with sum index
//          n = 2i + 1 (parity block 0) or 2i + 2 (block 1); zero past Kh or N.
//   data   rows = grid rows, values x_n split the same way (the first transform: masked r
//          split by the parity of x; the second: the column solve's output split by the
//          parity of the wavenumber). Writers round to TF32 (cvt.rna) and never touch the
//          padding (rows >= ny, indices past the block), which stays zero.
// Outputs: (ny x N) row-major.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fb_device.cuh"

namespace fb {

// Geometry of the tensor-core transform of one solve (device pointers).
struct UmmaDst {
  const float *tab;  // DST table tiles
  float *a1;         // data tiles of the first transform
  float *a2;         // data tiles of the second transform (may alias a1: written after the first ran)
  float *out1;       // odd-parity array of the first transform's output
  float *out2;       // even-parity array of the first transform's output; the second's output
  int n;             // N, the row length
  int kh;            // ceil(N / 2): output wavenumbers per parity and length of the odd block
  int nkb;           // blocks of 32 sum indices per parity block
  int nrb;           // blocks of 128 grid rows
  int nwb;           // blocks of 128 output wavenumbers
  int soff;          // byte offset of the stage region in the dynamic shared memory
  int stages;        // pipeline depth (1 .. kUmmaMaxStages)
  int ycopy_soff;    // shared-memory byte offset of the column solve's copy of y (-1: none)
  int on;            // 1: the preconditioner's row transforms use this path
};

constexpr int kUmmaMaxStages = 6;
constexpr int kUmmaTile = 128 * 32 * 4;      // bytes of one operand tile
constexpr int kUmmaStage = 2 * kUmmaTile;    // table tile + data tile

// Address (in floats) of operand element (row m, parity block p, index i).
__host__ __device__ __forceinline__ size_t umma_index(int nkb, int m, int p, int i) {
  const int mb = m >> 7, r = m & 127, kb = i >> 5, c = i & 31;
  return ((size_t)(mb * 2 + p) * nkb + kb) * (size_t)(128 * 32) + (size_t)r * 32 +
         (size_t)((((c >> 2) ^ (r & 7)) << 2) | (c & 3));
}
// Shared-memory bytes of the stage ring plus the 1024-byte alignment slack.
__host__ __device__ constexpr int umma_smem_bytes(int stages) { return 1024 + stages * kUmmaStage; }

// ------------------------------------------------------------------------------------------
// tcgen05 primitives (PTX ISA 8.6+, sm_100a)
static __shared__ __align__(8) unsigned long long fb_ubar[2 * kUmmaMaxStages + 1];
static __shared__ unsigned fb_tmem_addr;

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// whole warp; writes the allocated TMEM address to fb_tmem_addr
__device__ __forceinline__ void tmem_alloc(unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&fb_tmem_addr)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (TMEM) (+)= A (smem) . B (smem), TF32 operands, FP32 accumulation; one thread issues
__device__ __forceinline__ void umma_tf32(unsigned dtmem, uint64_t adesc, uint64_t bdesc, unsigned idesc, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
// arrive (once) on the mbarrier when every tcgen05.mma this thread issued so far has completed
__device__ __forceinline__ void umma_commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32 (w % 4) ..)
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// FP32 -> TF32 (round to nearest, ties away), kept in an FP32 container
__device__ __forceinline__ float to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Shared-memory matrix descriptor of a K-major operand tile with 128-byte swizzling (rows of
// 128 bytes, 8-row atoms 1024 bytes apart): low word = start address >> 4 (14 bits) | leading
// byte offset 1 << 16 (unused with swizzling); high word = stride byte offset 1024 >> 4 |
// descriptor version 1 (bit 46) | swizzle mode 2 = 128 bytes (bits 61-63). The high word is a
// constant, so the MMA thread steps start addresses with 32-bit adds on the low word.
__device__ __forceinline__ uint32_t umma_desc_lo(unsigned saddr) { return ((saddr >> 4) & 0x3FFFu) | (1u << 16); }
__device__ __forceinline__ uint64_t umma_desc_from_lo(uint32_t lo) {
  constexpr uint32_t hi = (1024u >> 4) | (1u << 14) | (2u << 29);
  return ((uint64_t)hi << 32) | lo;
}

// Instruction descriptor: TF32 x TF32 -> FP32, both operands K-major, M = 128, N = 128.
__device__ __forceinline__ constexpr unsigned umma_idesc_tf32_128() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(128 >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
}

// One row transform of an (ny x N) array: this CTA's work units (unit = vcta() + j nblocks
// over nrb x nwb x 2 units, parity fastest). 512 threads: thread 0 issues the bulk copies of
// the operand tiles through a `stages`-deep ring, thread 32 issues the MMAs (four K = 8 steps
// per block of 32 sum indices), and all 16 warps drain the accumulator: warp w reads TMEM
// lanes 32 (w % 4) .. (its 32 wavenumbers) and the 16-row column chunks w / 4 and w / 4 + 4.
// Stage 0 transforms the first operand into the parity arrays u.out1 / u.out2, stage 1 the
// second into u.out2 (accumulated).
// Every wait is bounded (limit_ns): on a timeout the abort flag and ST_TIMEOUT are set, the
// unit loop ends, TMEM is released and the caller's next grid barrier stops the kernel.
static __device__ __noinline__ void umma_dst_phase(const UmmaDst u, int stage, int ny, int nblocks, GridSync *gs,
                                                   DevReport *rep, unsigned long long limit_ns) {
  constexpr unsigned NCOLS = 128;
  const int nunits = u.nrb * u.nwb * 2;
  if (vcta() >= nunits) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned sraw = smem_u32(fb_smem + u.soff);
  const unsigned sal = (sraw + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
  char *sbase = fb_smem + u.soff + (sal - sraw);
  unsigned long long *full = fb_ubar, *empty = fb_ubar + kUmmaMaxStages, *done = fb_ubar + 2 * kUmmaMaxStages;
  const int ST = u.stages, N = u.n, kh = u.kh, nkb = u.nkb;
  const float *D = stage ? u.a2 : u.a1;
  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_fence_init();
  }
  if (warp == 0) {
    __syncwarp();
    tmem_alloc(NCOLS);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tbase = fb_tmem_addr;
  const int myunits = (nunits - vcta() + nblocks - 1) / nblocks;
  const int F = myunits * nkb;  // operand blocks this CTA streams through the ring
  bool ok = true;
  int ui = 0;
  // ring position of the producer (thread 0) and of the MMA thread (thread 32), kept
  // incrementally: slot s and `use` = how many times the slot was filled before
  int ps = 0, puse = 0, ms = 0, muse = 0, mf = 0;
  for (int unit = vcta(); unit < nunits; unit += nblocks, ++ui) {
    const int par = unit & 1, wr = unit >> 1, rb = wr / u.nwb, wb = wr - rb * u.nwb;
    if (tid == 0) {
      fence_proxy_async();  // generic accesses to the ring (earlier phases) before the copies
      const float *tsrc = u.tab + (size_t)(wb * 2 + par) * nkb * (128 * 32);
      const float *dsrc = D + (size_t)(rb * 2 + par) * nkb * (128 * 32);
      for (int kb = 0; kb < nkb; ++kb) {
        if (puse > 0 && !mbar_wait(&empty[ps], (unsigned)(puse - 1) & 1u, limit_ns, gs, rep)) {
          ok = false;
          break;
        }
        char *st = sbase + ps * kUmmaStage;
        mbar_expect_tx(&full[ps], (unsigned)kUmmaStage);
        bulk_copy_g2s(st, tsrc + (size_t)kb * (128 * 32), kUmmaTile, &full[ps]);
        bulk_copy_g2s(st + kUmmaTile, dsrc + (size_t)kb * (128 * 32), kUmmaTile, &full[ps]);
        if (++ps == ST) {
          ps = 0;
          ++puse;
        }
      }
    } else if (tid == 32) {
      constexpr unsigned idesc = umma_idesc_tf32_128();
      const uint32_t lo0 = umma_desc_lo(sal);                 // slot 0's table tile
      constexpr uint32_t kSlot = kUmmaStage >> 4, kData = kUmmaTile >> 4;
      uint32_t lo = lo0 + (uint32_t)ms * kSlot;
      for (int kb = 0; kb < nkb; ++kb) {
        if (!mbar_wait(&full[ms], (unsigned)muse & 1u, limit_ns, gs, rep)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          umma_tf32(tbase, umma_desc_from_lo(lo + 2u * kk), umma_desc_from_lo(lo + kData + 2u * kk), idesc,
                    (kb | kk) != 0);
        if (mf + ST < F) umma_commit(&empty[ms]);  // only the ring slots the producer reuses
        ++mf;
        if (++ms == ST) {
          ms = 0;
          ++muse;
          lo = lo0;
        } else {
          lo += kSlot;
        }
      }
      umma_commit(done);  // also after a failed wait, so that the epilogue's wait ends
    }
    __syncwarp();
    const bool dok = mbar_wait(done, (unsigned)ui & 1u, limit_ns, gs, rep);
    if (__syncthreads_or(!(ok && dok))) {
      ok = false;
      break;
    }
    tc_fence_after();
    // ---- TMEM -> global: this thread's wavenumber k and its mirror, 16 rows per chunk
    {
      const int q = warp & 3;
      const int k = wb * 128 + q * 32 + lane + 1;
      const int km = N + 1 - k;  // mirror wavenumber L - k
      float *__restrict__ dst = (stage || par) ? u.out2 : u.out1;
      const float sgn = par ? -1.0f : 1.0f;
      for (int cc = warp >> 2; cc < 8; cc += 4) {
        float v[16];
        tmem_ld16(tbase + ((unsigned)(q * 32) << 16) + (unsigned)(cc * 16), v);
        tmem_wait_ld();
        if (k > kh) continue;
        const int m0 = rb * 128 + cc * 16;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          if (m0 + j >= ny) continue;
          float *row = dst + (size_t)(m0 + j) * N;
          if (stage) {
            atomicAdd(row + (k - 1), v[j]);  // no return value used: a reduction, not a fetch
            if (km != k) atomicAdd(row + (km - 1), sgn * v[j]);
          } else {
            row[k - 1] = v[j];
            if (km != k) row[km - 1] = sgn * v[j];
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();  // TMEM free for the next unit; this unit's stores done
  }
  (void)ok;
  __syncthreads();
  if (tid == 0) {
    // every phase of the ring's mbarriers was waited for (the MMA thread commits to a ring
    // slot only when the producer will wait for that commit), so they can be invalidated
    // and initialised afresh by the next call in this launch
    for (int s = 0; s < ST; ++s) {
      mbar_inval(&full[s]);
      mbar_inval(&empty[s]);
    }
    mbar_inval(done);
  }
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, NCOLS);
  }
  return;
}

}  // namespace fb
