// fft_lines.cuh -- in-place complex FFT of TI interleaved lines in shared
// memory (re[j*TI + ii], im[j*TI + ii], input in bit-reversed order),
// decimation in time.  Stages are fused in pairs into radix-2^2 butterflies
// (one pass over shared memory and one barrier per two stages); each
// butterfly performs exactly the operations of the two radix-2 stages it
// replaces, with the same table twiddles, so results equal the radix-2
// sequence of FFTPACK order used by the oracle bit for bit.
// tw*: shared-memory table exp(s 2 pi i r / L), r < L/2 (read with stride ts:
// a sub-transform of length L/ts uses every ts-th entry).
//
// Lines of length L = r 2^m, r = 1 or 3 (the periodic extents FFTPACK's
// radix-2/3 factors cover, e.g. 384 = 3 x 128): with r = 3 the input is
// decimated by 3 (element j to block j mod 3, at the bit-reversed position of
// j / 3), each block is transformed by the radix-2^2 passes, and one pass of
// radix-3 butterflies combines them.  A length is passed as the code
// m | r << 8.
#pragma once

__host__ __device__ inline int fft_len(int code) { return (code >> 8) << (code & 255); }

// the code of a line length L = r 2^m (r = 1 or 3, m >= 1), or -1
inline int fft_code(int L) {
  int r = 1;
  if (L % 3 == 0) {
    r = 3;
    L /= 3;
  }
  int m = 0;
  while ((1 << m) < L) m++;
  if (m < 1 || (1 << m) != L) return -1;
  return m | (r << 8);
}

__device__ __forceinline__ int fft_bitrev(int x, int logn) {
  return (int)(__brev((unsigned)x) >> (32 - logn));
}

// the shared-memory slot of input element j of a line
__device__ __forceinline__ int fft_slot(int j, int code) {
  const int m = code & 255;
  if ((code >> 8) == 1) return fft_bitrev(j, m);
  return (j % 3) * (1 << m) + fft_bitrev(j / 3, m);
}

template <class T, int TI>
__device__ __forceinline__ void fft_lines_r22(T *re, T *im, int logL, const T *twr, const T *twi, int ts = 1) {
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
      const T w1r = twr[q * st1 * ts], w1i = twi[q * st1 * ts];
      const T w2r = twr[q * st2 * ts], w2i = twi[q * st2 * ts];
      const T w3r = twr[(q + h) * st2 * ts], w3i = twi[(q + h) * st2 * ts];
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

// a line of length fft_len(code), input in fft_slot order, output in
// natural order (in place)
template <class T, int TI>
__device__ __forceinline__ void fft_lines_any(T *re, T *im, int code, const T *twr, const T *twi) {
  const int m = code & 255;
  if ((code >> 8) == 1) {
    fft_lines_r22<T, TI>(re, im, m, twr, twi, 1);
    return;
  }
  const int L3 = 1 << m, half = 3 * L3 / 2;
  for (int b = 0; b < 3; b++) fft_lines_r22<T, TI>(re + b * L3 * TI, im + b * L3 * TI, m, twr, twi, 3);
  // W^e from the table of e < L/2 (W^(L/2) = -1 beyond)
  auto tw = [&](int e, T &wr, T &wi) {
    if (e < half) {
      wr = twr[e];
      wi = twi[e];
    } else {
      wr = -twr[e - half];
      wi = -twi[e - half];
    }
  };
  T ur, ui, vr, vi;  // the cube roots W^(L/3), W^(2L/3)
  tw(L3, ur, ui);
  tw(2 * L3, vr, vi);
  for (int bf = threadIdx.x; bf < TI * L3; bf += blockDim.x) {
    const int ii = bf % TI, k = bf / TI;
    T w1r, w1i, w2r, w2i;
    tw(k, w1r, w1i);
    tw(2 * k, w2r, w2i);
    const int pa = k * TI + ii, pb = (L3 + k) * TI + ii, pc = (2 * L3 + k) * TI + ii;
    const T ar = re[pa], ai = im[pa], br = re[pb], bi = im[pb], cr = re[pc], ci = im[pc];
    const T t1r = w1r * br - w1i * bi, t1i = w1r * bi + w1i * br;
    const T t2r = w2r * cr - w2i * ci, t2i = w2r * ci + w2i * cr;
    re[pa] = ar + t1r + t2r;
    im[pa] = ai + t1i + t2i;
    re[pb] = ar + (ur * t1r - ui * t1i) + (vr * t2r - vi * t2i);
    im[pb] = ai + (ur * t1i + ui * t1r) + (vr * t2i + vi * t2r);
    re[pc] = ar + (vr * t1r - vi * t1i) + (ur * t2r - ui * t2i);
    im[pc] = ai + (vr * t1i + vi * t1r) + (ur * t2i + ui * t2r);
  }
  __syncthreads();
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
