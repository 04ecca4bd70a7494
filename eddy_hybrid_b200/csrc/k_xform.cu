// k_xform.cu -- the x eigen-transforms of the mixed-precision Poisson solve on
// the 5th-generation tensor cores.
//
// Out[p][n] = sum_k In[p][k] B[n][k] for all P = L*N spectral lines p (the
// (J,k) lines of the solve, x index contiguous), K = N = M = NX-2.  Storage is
// FP32; products use the 3xTF32 split (a = a_hi + a_lo with a_hi the TF32
// truncation): A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32 in TMEM by
// tcgen05.mma kind::tf32, which keeps the transform at FP32 accuracy (the
// refinement sweeps then see the same convergence as with an FP32 GEMM).
//
// Mirror-symmetric x operators (a grid symmetric about its centre, the same
// boundary type at both ends: the eigenvectors are even or odd about the
// centre) take the split form with half the work: with H = M/2 and the modes
// ordered even then odd,
//   forward:  c_even = F_e (f[x] + f[M-1-x]),  c_odd = F_o (f[x] - f[M-1-x]),
//   backward: e = B_e c_even, o = B_o c_odd, f[x] = e + o, f[M-1-x] = e - o,
// all four matrices H x H.
//
// One CTA per 128-line tile, all M outputs in TMEM columns 0..M-1 (M <= 512).
// K is streamed in chunks of 8 through a multi-stage shared-memory pipeline:
// each A chunk arrives by one 2-D TMA box (32 bytes x 128 lines) with the
// 32-byte swizzle, which is the canonical SWIZZLE_32B K-major layout (rows of
// 32 bytes, the two 16-byte halves of row r exchanged when bit 2 of r is
// set); the B chunks of a stage (prepared on the host, in chunk order, as the
// no-swizzle K-major layout [k/4][n][4] of each block's hi and lo parts)
// arrive by one 1-D bulk copy.  Loading, splitting A into hi/lo (and, for
// the symmetric forward transform, forming the mirror sums and differences)
// and the MMAs run in separate warps so the three overlap across stages; the
// epilogue reads TMEM (lane = line) and stores rows.
#include <cmath>
#include <cstring>
#include <vector>

#include "eddy_internal.h"
#include "tma_ring.cuh"
#include "umma.cuh"

namespace {

constexpr int XT = 192;   // threads per CTA: loader warp, MMA warp, 4 splitter/epilogue warps
constexpr int KC = 8;     // K per pipeline stage (one MMA k-step)
constexpr int MAXST = 8;  // pipeline stages at most

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tma::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tma::smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(tma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(tma::smem_u32(bar))
      : "memory");
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major
__device__ __forceinline__ uint32_t idesc_tf32(int M, int N) {
  uint32_t d = 0;
  d |= 1u << 4;                   // D format f32
  d |= 2u << 7;                   // A format tf32
  d |= 2u << 10;                  // B format tf32
  d |= (uint32_t)(N >> 3) << 17;  // N / 8
  d |= (uint32_t)(M >> 4) << 24;  // M / 16
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tma::smem_u32(bar)) : "memory");
}

// 32 lanes x 32 bit, 32 consecutive columns, load and wait in one asm block
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ float4 tf32_hi(float4 v) {
  float4 h;
  h.x = __uint_as_float(__float_as_uint(v.x) & 0xFFFFE000u);
  h.y = __uint_as_float(__float_as_uint(v.y) & 0xFFFFE000u);
  h.z = __uint_as_float(__float_as_uint(v.z) & 0xFFFFE000u);
  h.w = __uint_as_float(__float_as_uint(v.w) & 0xFFFFE000u);
  return h;
}

__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// SWIZZLE_32B K-major descriptor: rows of 32 bytes, 8-row groups 256 bytes
// apart (SBO), LBO 16 bytes (unused inside the swizzle atom), version 1
__device__ __forceinline__ uint64_t make_desc_sw32(const void *smem_base) {
  const uint64_t addr = tma::smem_u32(smem_base);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= (uint64_t)(16 >> 4) << 16;
  d |= (uint64_t)(256 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)6 << 61;  // layout type SWIZZLE_32B
  return d;
}

// Per-stage layout.  mode 0 (plain): A, A_lo, B_hi, B_lo with B of M rows.
// modes 1/2 (symmetric): A1, A1_lo, A2, A2_lo, B1_hi, B1_lo, B2_hi, B2_lo with
// B1, B2 of H rows each.  The B part of a stage is contiguous, in the order of
// one chunk of the host-prepared matrix array.
struct StageGeom {
  int nb;             // rows of one B block (M or H)
  int na;             // A blocks per stage (1 or 2)
  uint32_t a_bytes;   // 128 x KC floats
  uint32_t b_bytes;   // nb x KC floats (one of hi / lo)
  uint32_t stage;     // bytes per stage
};

// output passes of the epilogue: rows of more than 432 floats are staged
// in two halves (128 rows of W + 4 floats must fit the shared memory)
__host__ __device__ inline int xform_passes(int M) { return M > 432 ? 2 : 1; }

__host__ __device__ inline StageGeom stage_geom(int mode, int M) {
  StageGeom g;
  g.na = mode ? 2 : 1;
  g.nb = mode ? M / 2 : M;
  g.a_bytes = 128u * KC * 4u;
  g.b_bytes = (uint32_t)g.nb * KC * 4u;
  g.stage = g.na * (2u * g.a_bytes + 2u * g.b_bytes);
  return g;
}

// Warp roles: warp 0 loads (one lane issues the TMA and bulk copies of a
// stage once the MMAs that read it have completed), warp 1 issues the MMAs
// (one lane), warps 2-5 split each A chunk into hi/lo and, at the end, drain
// TMEM (warp w reads lanes 32 (w % 4) .. +31).  Stage barriers: full (copies
// landed), split (128 splitter arrivals), empty (MMAs done, tcgen05.commit),
// and done after the last chunk.  Every wait is bounded; a timeout raises the
// error flag, the roles stop issuing work and wait (bounded) for what they
// already issued before TMEM is released.
__global__ void __launch_bounds__(XT, 1)
    k_xform_tf32(const __grid_constant__ CUtensorMap amap, const float *__restrict__ bmat, float *__restrict__ out, long long P, int M, int mode, int nst,
                 int *err) {
  extern __shared__ __align__(1024) unsigned char xsm[];
  __shared__ __align__(8) uint64_t full[MAXST], split[MAXST], empty[MAXST], done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  // 1024-byte aligned stage area, as an offset into the shared array (the
  // shared address space stays visible to the compiler)
  unsigned char *base = xsm + ((1024u - (unsigned)(reinterpret_cast<uintptr_t>(xsm) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const StageGeom G = stage_geom(mode, M);
  const int H = M / 2;
  const int nch = (mode ? H : M) / KC;
  const long long p0 = (long long)blockIdx.x * 128;
  uint32_t ncols = 64;
  while ((int)ncols < M) ncols <<= 1;
  if (warp == 1) {
    umma::tmem_alloc(&tmem_base, ncols);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < nst; s++) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&split[s], 128);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(&done, 1);
    tma::fence_mbar_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tm = tmem_base;
  // block h (0 or 1) of a stage: A_hi, A_lo (A blocks first), B_hi, B_lo
  auto st_a = [&](int s, int h) { return base + (size_t)s * G.stage + h * 2 * G.a_bytes; };
  auto st_alo = [&](int s, int h) { return st_a(s, h) + G.a_bytes; };
  auto st_bhi = [&](int s, int h) {
    return base + (size_t)s * G.stage + G.na * 2 * G.a_bytes + h * 2 * G.b_bytes;
  };
  auto st_blo = [&](int s, int h) { return st_bhi(s, h) + G.b_bytes; };
  auto fail = [&]() {
    abort_flag = 1;
    atomicExch(err, 1);
  };
  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {
      // the per-chunk bookkeeping is kept to increments (stage, phase, B
      // offset): this thread's issue rate paces the pipeline
      int issued = 0, s = 0;
      uint32_t ph = 0;
      const uint32_t bbytes = G.na * 2 * G.b_bytes;  // B of one chunk, all blocks, hi and lo
      const uint32_t txb = G.na * G.a_bytes + bbytes;
      const float *bsrc = bmat;
      for (int c = 0; c < nch && !abort_flag; c++) {
        if (c >= nst && !umma::mbar_wait(&empty[s], ph ^ 1u)) { fail(); break; }
        tma::mbar_expect_tx(&full[s], txb);
        // K offset of the A block: plain / first half at 8c; mirror block
        // (forward) at M - 8(c+1); odd-mode block (backward) at H + 8c
        load_2d(st_a(s, 0), &amap, c * KC, (int)p0, &full[s]);
        if (G.na == 2) load_2d(st_a(s, 1), &amap, mode == 1 ? M - (c + 1) * KC : H + c * KC, (int)p0, &full[s]);
        bulk_load(st_bhi(s, 0), bsrc, bbytes, &full[s]);
        bsrc += bbytes / 4;
        issued = c + 1;
        if (++s == nst) { s = 0; ph ^= 1u; }
      }
      // copies still in flight land before the CTA may exit
      for (int c = issued - nst < 0 ? 0 : issued - nst; c < issued; c++)
        if (!umma::mbar_wait(&full[c % nst], (c / nst) & 1, 1u << 20)) atomicExch(err, 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // Descriptors of stage 0, computed once: stage s adds s * stage bytes
      // / 16 to the 14-bit start-address field (every stage lies inside the
      // shared window, so the field cannot carry).  Keeping the per-chunk
      // work to the MMAs lets them issue back to back.  Columns of block h:
      // [h*H, h*H + nb) in the symmetric form; the plain form splits its M
      // columns into MMAs of at most 256 (j = 0, 1).
      const uint32_t lbo_b = (uint32_t)G.nb * 16;
      const uint64_t dstep = (uint64_t)(G.stage >> 4);
      uint64_t dah[2], dal[2], dbh[2][2], dbl[2][2];
      uint32_t idj[2], dcol[2][2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        dah[h] = make_desc_sw32(st_a(0, h));
        dal[h] = make_desc_sw32(st_alo(0, h));
#pragma unroll
        for (int j = 0; j < 2; j++) {
          dbh[h][j] = umma::make_desc(st_bhi(0, h) + j * 256 * 16, lbo_b, 128);
          dbl[h][j] = umma::make_desc(st_blo(0, h) + j * 256 * 16, lbo_b, 128);
          dcol[h][j] = tm + (uint32_t)(h * H + j * 256);
        }
      }
      const int nj = G.nb > 256 ? 2 : 1;
      idj[0] = idesc_tf32(128, G.nb < 256 ? G.nb : 256);
      idj[1] = idesc_tf32(128, G.nb > 256 ? G.nb - 256 : 16);
      int s = 0;
      uint32_t ph = 0;
      for (int c = 0; c < nch; c++) {
        if (abort_flag || !umma::mbar_wait(&split[s], ph)) { fail(); break; }
        umma::fence_after_sync();
        const uint64_t off = (uint64_t)s * dstep;
        const uint32_t acc = c == 0 ? 0u : 1u;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          if (h < G.na) {
#pragma unroll
            for (int j = 0; j < 2; j++) {
              if (j < nj) {
                mma_tf32(dcol[h][j], dah[h] + off, dbh[h][j] + off, idj[j], acc);
                mma_tf32(dcol[h][j], dah[h] + off, dbl[h][j] + off, idj[j], 1u);
                mma_tf32(dcol[h][j], dal[h] + off, dbh[h][j] + off, idj[j], 1u);
              }
            }
          }
        }
        umma::commit(&empty[s]);
        if (++s == nst) { s = 0; ph ^= 1u; }
      }
      // the commit after the last issued MMA completes once all of them have
      umma::commit(&done);
    }
  } else {
    const int t = tid - 64;
    const int qsw = (t >> 2) & 1;
    int s = 0;
    uint32_t ph = 0;
    for (int c = 0; c < nch; c++, s = (s + 1 == nst ? 0 : s + 1), ph ^= (s == 0 ? 1u : 0u)) {
      if (abort_flag) { ok = false; break; }
      if (!umma::mbar_wait(&full[s], ph)) { fail(); ok = false; break; }
      // 128 rows of 32 bytes = 256 float4 per A block; thread t handles row t
      // (float4 2t, 2t + 1; which holds which k half depends on the swizzle,
      // the element-wise split does not care).  Each access takes slot
      // 2t + (e ^ q), q = bit 2 of t: the eight threads of one 128-bit phase
      // then cover all 32 banks (slot 2t + e alone would pair t with t + 4).
      float4 *a1 = reinterpret_cast<float4 *>(st_a(s, 0)) + 2 * t;
      float4 *l1 = reinterpret_cast<float4 *>(st_alo(s, 0)) + 2 * t;
      if (mode == 1) {
        // mirror sums and differences: local k of the mirror block is 7 - k.
        // Half c of row t sits in 16-byte slot c ^ sw(t) of both blocks, so
        // slot p of A1 pairs with slot 1 - p of A2 (reversed) whatever sw(t)
        float4 *a2 = reinterpret_cast<float4 *>(st_a(s, 1)) + 2 * t;
        float4 *l2 = reinterpret_cast<float4 *>(st_alo(s, 1)) + 2 * t;
        // all four reads before any write: slot p of A2 is read for slot 1 - p
        float4 xs[2], ys[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          xs[e] = a1[e ^ qsw];
          ys[e] = a2[1 - (e ^ qsw)];
        }
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int p = e ^ qsw;
          const float4 x = xs[e], y = ys[e];
          const float4 r = make_float4(y.w, y.z, y.y, y.x);
          const float4 sm = make_float4(x.x + r.x, x.y + r.y, x.z + r.z, x.w + r.w), df = sub4(x, r);
          float4 h;
          h = tf32_hi(sm); a1[p] = h; l1[p] = sub4(sm, h);
          h = tf32_hi(df); a2[p] = h; l2[p] = sub4(df, h);
        }
      } else {
        for (int hb = 0; hb < G.na; hb++) {
          float4 *a = reinterpret_cast<float4 *>(st_a(s, hb)) + 2 * t;
          float4 *l = reinterpret_cast<float4 *>(st_alo(s, hb)) + 2 * t;
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const int p = e ^ qsw;
            const float4 v = a[p], h = tf32_hi(v);
            a[p] = h;
            l[p] = sub4(v, h);
          }
        }
      }
      umma::fence_smem_to_async();
      mbar_arrive(&split[s]);
    }
    // epilogue: all MMAs complete, so every stage buffer is free.  Thread t
    // (row t of the tile) assembles its output row in shared memory (rows
    // padded to W + 4 floats against bank conflicts) and writes it back with
    // one bulk copy (the row is contiguous in global memory).  Rows wider
    // than 432 floats go out in two halves of W = M/2 columns, the second
    // staged once the first copy has read the buffer.
    if (ok && !umma::mbar_wait(&done, 0)) { fail(); ok = false; }
    umma::fence_after_sync();
    if (ok && !abort_flag) {
      const int q4 = warp & 3;
      const int rt = q4 * 32 + lane;
      const long long row = p0 + rt;
      const uint32_t tl = tm + ((uint32_t)(q4 * 32) << 16);
      const int npass = xform_passes(M), W = M / npass;
      float *srow = reinterpret_cast<float *>(base) + (size_t)rt * (W + 4);
      for (int pass = 0; pass < npass; pass++) {
        if (pass) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        if (mode == 2) {
          // f[x] = e + o, f[M-1-x] = e - o; with two passes the first writes
          // columns 0..H-1 (the sums), the second H..M-1 (the differences)
          for (int c0 = 0; c0 < H; c0 += 32) {
            uint32_t e[32], o[32];
            tmem_ld32(tl + (uint32_t)c0, e);
            tmem_ld32(tl + (uint32_t)(H + c0), o);
            const int nv = (H - c0 < 32 ? H - c0 : 32) / 4;
#pragma unroll
            for (int q = 0; q < 8; q++) {
              if (q < nv) {
                float pv[4], mv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                  const float ev = __uint_as_float(e[4 * q + u]), ov = __uint_as_float(o[4 * q + u]);
                  pv[u] = ev + ov;
                  mv[u] = ev - ov;
                }
                const int x = c0 + 4 * q;
                if (pass == 0)
                  *reinterpret_cast<float4 *>(srow + x) = make_float4(pv[0], pv[1], pv[2], pv[3]);
                if (npass == 1 || pass == 1)
                  *reinterpret_cast<float4 *>(srow + (M - 4 - x - pass * W)) =
                      make_float4(mv[3], mv[2], mv[1], mv[0]);
              }
            }
          }
        } else {
          const int cb = pass * W, ce = cb + W;
          for (int c0 = cb; c0 < ce; c0 += 64) {
            uint32_t r[64];
            umma::tmem_ld64(tl + (uint32_t)c0, r);
            float4 *dst = reinterpret_cast<float4 *>(srow + (c0 - cb));
            const int nv = (ce - c0 < 64 ? ce - c0 : 64) / 4;
#pragma unroll
            for (int q = 0; q < 16; q++)
              if (q < nv)
                dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                     __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
          }
        }
        umma::fence_smem_to_async();
        if (row < P) {
          asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(out + row * M + pass * W),
                       "r"(tma::smem_u32(srow)), "r"((uint32_t)W * 4u)
                       : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
      }
      if (row < P) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
  }
  // on the error path the MMAs already issued may still run: wait (bounded)
  // for their commit before TMEM is released
  if (warp == 1 && lane == 0 && abort_flag) umma::mbar_wait(&done, 0, 1u << 20);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tm, ncols);
  }
}

// hi/lo split of an FP64 value: hi the TF32 truncation of its FP32 rounding
void split_tf32(double x, float &h, float &l) {
  float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u &= 0xFFFFE000u;
  std::memcpy(&h, &u, 4);
  l = (float)(x - (double)h);
}

// The na blocks B_h[n][k] = T(h, n, k) (nb x nb each, T given as a callable)
// as one array in the order the kernel streams them: for each chunk of KC k
// values, for each block, its hi part then its lo part, each in the
// no-swizzle K-major layout [KC/4][nb][4] of one stage
template <class F>
std::vector<float> chunked(int na, int nb, F T) {
  std::vector<float> v((size_t)na * 2 * nb * nb);
  size_t o = 0;
  for (int c = 0; c < nb / KC; c++)
    for (int h = 0; h < na; h++)
      for (int part = 0; part < 2; part++)
        for (int kq = 0; kq < KC / 4; kq++)
          for (int n = 0; n < nb; n++)
            for (int e = 0; e < 4; e++) {
              float hi, lo;
              split_tf32(T(h, n, c * KC + kq * 4 + e), hi, lo);
              v[o++] = part ? lo : hi;
            }
  return v;
}

int upload(eddy_ctx *ctx, const std::vector<float> &h, float **d) {
  EDDY_CUDA(cudaMalloc(d, sizeof(float) * h.size()));
  EDDY_CUDA(cudaMemcpy(*d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
  return EDDY_OK;
}

int xform_stages(int mode, int M) {
  const size_t st = stage_geom(mode, M).stage;
  int n = (int)((227 * 1024 - 2048) / st);
  return n > MAXST ? MAXST : n;
}

// dynamic shared memory: the stages, which the epilogue reuses for its
// 128 output rows of W + 4 floats (W = M / passes)
size_t xform_smem(int mode, int M) {
  const size_t st = (size_t)xform_stages(mode, M) * stage_geom(mode, M).stage;
  const size_t ep = (size_t)128 * (M / xform_passes(M) + 4) * 4;
  return (st > ep ? st : ep) + 1024;
}

}  // namespace

// M <= 512: all M accumulator columns fit the 512 TMEM columns of an SM (one
// CTA per SM), the epilogue stages rows in at most two passes
bool xform_supported(int M) { return M >= 16 && M <= 512 && M % 16 == 0; }

// Transform matrices from the FP64 plan.  Af (col-major, Af(n, x)) maps
// x values to mode coefficients, Ab (col-major, Ab(x, n)) back.  The split
// form is used when every mode is even or odd about the centre to within
// 1e-9 of its largest entry, H of each.
int xform_prepare(eddy_ctx *ctx, XformPlan *xp) {
  const PoissonPlan &pp = ctx->pp;
  const int M = pp.M, H = M / 2;
  std::vector<double> Af((size_t)M * M), Ab((size_t)M * M), lam(M);
  EDDY_CUDA(cudaMemcpy(Af.data(), pp.Af, sizeof(double) * Af.size(), cudaMemcpyDeviceToHost));
  EDDY_CUDA(cudaMemcpy(Ab.data(), pp.Ab, sizeof(double) * Ab.size(), cudaMemcpyDeviceToHost));
  EDDY_CUDA(cudaMemcpy(lam.data(), pp.lam, sizeof(double) * M, cudaMemcpyDeviceToHost));
  auto af = [&](int n, int x) { return Af[(size_t)n + (size_t)M * x]; };
  auto ab = [&](int x, int n) { return Ab[(size_t)x + (size_t)M * n]; };
  std::vector<int> even, odd;
  bool sym = (M % 32 == 0) && H <= 256;
  for (int n = 0; n < M && sym; n++) {
    double dot = 0., mf = 0., mb = 0.;
    for (int x = 0; x < M; x++) {
      dot += af(n, x) * af(n, M - 1 - x);
      mf = std::fmax(mf, std::fabs(af(n, x)));
      mb = std::fmax(mb, std::fabs(ab(x, n)));
    }
    const double sg = dot >= 0. ? 1. : -1.;
    for (int x = 0; x < M && sym; x++) {
      if (std::fabs(af(n, x) - sg * af(n, M - 1 - x)) > 1e-9 * mf) sym = false;
      if (std::fabs(ab(x, n) - sg * ab(M - 1 - x, n)) > 1e-9 * mb) sym = false;
    }
    (sg > 0. ? even : odd).push_back(n);
  }
  if (sym && ((int)even.size() != H || (int)odd.size() != H)) sym = false;
  std::vector<float> fm, bm;
  std::vector<double> lp(M);
  int m0 = pp.m0;
  if (sym) {
    std::vector<int> perm(even);
    perm.insert(perm.end(), odd.begin(), odd.end());
    for (int m = 0; m < M; m++) {
      lp[m] = lam[perm[m]];
      if (perm[m] == pp.m0) m0 = m;
    }
    // forward: B1[m][x] = Af(even[m], x), B2[m][x] = Af(odd[m], x), x < H
    fm = chunked(2, H, [&](int h, int m, int x) { return af((h ? odd : even)[m], x); });
    // backward: B1[x][m] = Ab(x, even[m]), B2[x][m] = Ab(x, odd[m]), x < H
    bm = chunked(2, H, [&](int h, int x, int m) { return ab(x, (h ? odd : even)[m]); });
  } else {
    lp = lam;
    fm = chunked(1, M, [&](int, int n, int x) { return af(n, x); });
    bm = chunked(1, M, [&](int, int x, int n) { return ab(x, n); });
  }
  xp->sym = sym ? 1 : 0;
  xp->m0 = m0;
  int rc;
  if ((rc = upload(ctx, fm, &xp->fmat)) || (rc = upload(ctx, bm, &xp->bmat))) return rc;
  EDDY_CUDA(cudaMalloc(&xp->lam, sizeof(double) * M));
  EDDY_CUDA(cudaMemcpy(xp->lam, lp.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
  size_t smax = 0;
  for (int mode = sym ? 1 : 0; mode < (sym ? 3 : 1); mode++) {
    const size_t smem = xform_smem(mode, M);
    smax = smem > smax ? smem : smax;
  }
  EDDY_CUDA(cudaFuncSetAttribute(k_xform_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
  return EDDY_OK;
}

void xform_release(XformPlan *xp) {
  float *p[] = {xp->fmat, xp->bmat};
  for (float *q : p)
    if (q) cudaFree(q);
  if (xp->lam) cudaFree(xp->lam);
  *xp = XformPlan{};
}

// out (P x M) = transform of in (P x M) on the tensor cores; dir 0 forward
// (x values -> mode coefficients), 1 backward
int launch_xform(eddy_ctx *ctx, const XformPlan *xp, int dir, const float *in, float *out) {
  const int M = ctx->pp.M;
  const long long P = (long long)ctx->pp.L * ctx->pp.N;
  const CUtensorMap *mp = nullptr;
  for (TmaEntry &e : ctx->tmaps)
    if (e.ptr == in && e.bx == 8 && e.by == -128) mp = &e.map;
  if (!mp) {
    TmaEntry e;
    e.ptr = in;
    e.bx = 8;
    e.by = -128;  // key: 2-D (M, P) view with an 8 x 128 box, 32-byte swizzle
    int r = make_tensor_map_2d(&e.map, in, M, P, 8, 128, 1);
    if (r != 0) {
      ctx->err = "cuTensorMapEncodeTiled (transform) failed (" + std::to_string(r) + ")";
      return EDDY_ECUDA;
    }
    ctx->tmaps.push_back(e);
    mp = &ctx->tmaps.back().map;
  }
  const int mode = xp->sym ? 1 + dir : 0;
  const int nst = xform_stages(mode, M);
  const size_t smem = xform_smem(mode, M);
  const unsigned grid = (unsigned)((P + 127) / 128);
  k_xform_tf32<<<grid, XT, smem, ctx->stream>>>(*mp, dir ? xp->bmat : xp->fmat, out, P, M,
                                                mode, nst, ctx->err_flag);
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}
