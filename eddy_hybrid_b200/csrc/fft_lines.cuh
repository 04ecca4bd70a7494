// fft_lines.cuh -- in-place complex FFT of TI interleaved lines in shared
// memory (re[j*TI + ii], im[j*TI + ii], input in bit-reversed order),
// decimation in time.  Stages are fused in pairs into radix-2^2 butterflies
// (one pass over shared memory and one barrier per two stages); each
// butterfly performs exactly the operations of the two radix-2 stages it
// replaces, with the same table twiddles, so results equal the radix-2
// sequence of FFTPACK order used by the oracle bit for bit.
// tw*: shared-memory table exp(s 2 pi i r / L), r < L/2.
#pragma once

template <class T, int TI>
__device__ __forceinline__ void fft_lines_r22(T *re, T *im, int logL, const T *twr, const T *twi) {
  const int L = 1 << logL;
  int s = 0;
  if (logL & 1) {  // one radix-2 stage of half-length 1 (twiddle index 0)
    const T wr = twr[0], wi = twi[0];
    for (int bf = threadIdx.x; bf < TI * (L >> 1); bf += blockDim.x) {
      const int ii = bf % TI, a = (bf / TI) * 2, b = a + 1;
      const T xr = re[b * TI + ii], xi = im[b * TI + ii];
      const T tr = wr * xr - wi * xi;
      const T ti = wr * xi + wi * xr;
      const T ar = re[a * TI + ii], ai = im[a * TI + ii];
      re[b * TI + ii] = ar - tr;
      im[b * TI + ii] = ai - ti;
      re[a * TI + ii] = ar + tr;
      im[a * TI + ii] = ai + ti;
    }
    __syncthreads();
    s = 1;
  }
  for (; s < logL; s += 2) {
    const int h = 1 << s;
    const int st1 = L >> (s + 1), st2 = L >> (s + 2);
    for (int bf = threadIdx.x; bf < TI * (L >> 2); bf += blockDim.x) {
      const int ii = bf % TI, pq = bf / TI;
      const int q = pq & (h - 1), grp = pq >> s;
      const int i0 = grp * 4 * h + q;
      const T w1r = twr[q * st1], w1i = twi[q * st1];
      const T w2r = twr[q * st2], w2i = twi[q * st2];
      const T w3r = twr[(q + h) * st2], w3i = twi[(q + h) * st2];
      T x0r = re[i0 * TI + ii], x0i = im[i0 * TI + ii];
      T x1r = re[(i0 + h) * TI + ii], x1i = im[(i0 + h) * TI + ii];
      T x2r = re[(i0 + 2 * h) * TI + ii], x2i = im[(i0 + 2 * h) * TI + ii];
      T x3r = re[(i0 + 3 * h) * TI + ii], x3i = im[(i0 + 3 * h) * TI + ii];
      // first stage (half-length h): pairs (x0,x1), (x2,x3)
      T tr = w1r * x1r - w1i * x1i, ti = w1r * x1i + w1i * x1r;
      const T y1r = x0r - tr, y1i = x0i - ti, y0r = x0r + tr, y0i = x0i + ti;
      tr = w1r * x3r - w1i * x3i;
      ti = w1r * x3i + w1i * x3r;
      const T y3r = x2r - tr, y3i = x2i - ti, y2r = x2r + tr, y2i = x2i + ti;
      // second stage (half-length 2h): pairs (y0,y2) and (y1,y3)
      tr = w2r * y2r - w2i * y2i;
      ti = w2r * y2i + w2i * y2r;
      re[(i0 + 2 * h) * TI + ii] = y0r - tr;
      im[(i0 + 2 * h) * TI + ii] = y0i - ti;
      re[i0 * TI + ii] = y0r + tr;
      im[i0 * TI + ii] = y0i + ti;
      tr = w3r * y3r - w3i * y3i;
      ti = w3r * y3i + w3i * y3r;
      re[(i0 + 3 * h) * TI + ii] = y1r - tr;
      im[(i0 + 3 * h) * TI + ii] = y1i - ti;
      re[(i0 + h) * TI + ii] = y1r + tr;
      im[(i0 + h) * TI + ii] = y1i + ti;
    }
    __syncthreads();
  }
}

// copy a twiddle table of L/2 entries from global to shared memory
template <class T>
__device__ __forceinline__ void load_twiddles(T *sr, T *si, const T *__restrict__ gr, const T *__restrict__ gi,
                                              int half) {
  for (int r = threadIdx.x; r < half; r += blockDim.x) {
    sr[r] = gr[r];
    si[r] = gi[r];
  }
}
