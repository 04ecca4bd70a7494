// k_sgs_impl.cuh -- the kernels and launch helper of the dynamic eddy
// viscosity (TURVIS, src/vt.f:16-442), included inside an anonymous namespace
// by k_sgs.cu (the FP64 instantiation, compiled with -fmad=false: the
// reference's operation order) and by k_sgs32.cu (the mixed form's FP32
// instantiation, compiled with FMA contraction).
#pragma once


constexpr int TI = 32;      // lanes: x columns ia-1 .. ia+30
constexpr int TO = 30;      // output columns per tile
constexpr int KT = 8;       // output z rows per tile
constexpr int NW = KT + 2;  // warps: z rows ka-1 .. ka+KT
constexpr int CR = KT + 4;  // centred-velocity ring rows ka-2 .. ka+KT+1
constexpr int CC = TI + 2;  // centred-velocity ring columns ia-2 .. ia+31
constexpr int RR = KT + 5;  // raw-velocity ring rows ka-3 .. ka+KT+1
constexpr int RC = TI + 4;  // raw-velocity ring columns ia-3 .. ia+32
constexpr int NQ = 22;      // filtered quantities

template <typename T>
struct MarchSmem {
  T cen[4][3][CR][CC];  // [plane slot j%4][uc,vc,wc][row][column]
  T raw[4][3][RR][RC];  // [plane slot j%4][u,v,w][row][column]
  T yb[NQ][NW][TI];     // completed y-filtered quantities of one plane
  T sgb[7][NW][TI];     // |S| and S_ij of plane jy1: the periodic copy in ghost row NY
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// centred velocities (vt.f:64-74) at (i,j,k), ghost formulas included
template <typename T>
__device__ __forceinline__ T cen_u(const Dims &d, int px, const T *__restrict__ u, int i, int j, int k) {
  long long q = pidx(d, px, i, j, k);
  if (i >= d.ix1 && i <= d.ix2) return T(0.5) * (u[q - 1] + u[q]);
  if (i == 1) return T(2.) * u[q] - T(0.5) * (u[pidx(d, px, d.ix1 - 1, j, k)] + u[pidx(d, px, d.ix1, j, k)]);
  return T(2.) * u[pidx(d, px, d.ix2, j, k)] - T(0.5) * (u[pidx(d, px, d.ix2 - 1, j, k)] + u[pidx(d, px, d.ix2, j, k)]);
}
template <typename T>
__device__ __forceinline__ T cen_v(const Dims &d, int px, const T *__restrict__ v, int i, int j, int k) {
  if (j >= d.jy1 && j <= d.jy2) return T(0.5) * (v[pidx(d, px, i, j - 1, k)] + v[pidx(d, px, i, j, k)]);
  if (j == 1)
    return T(2.) * v[pidx(d, px, i, 1, k)] - T(0.5) * (v[pidx(d, px, i, d.jy1 - 1, k)] + v[pidx(d, px, i, d.jy1, k)]);
  return T(2.) * v[pidx(d, px, i, d.jy2, k)] - T(0.5) * (v[pidx(d, px, i, d.jy2 - 1, k)] + v[pidx(d, px, i, d.jy2, k)]);
}
template <typename T>
__device__ __forceinline__ T cen_w(const Dims &d, int px, const T *__restrict__ w, int i, int j, int k) {
  if (k >= d.kz1 && k <= d.kz2) return T(0.5) * (w[pidx(d, px, i, j, k - 1)] + w[pidx(d, px, i, j, k)]);
  if (k == 1)
    return T(2.) * w[pidx(d, px, i, j, 1)] - T(0.5) * (w[pidx(d, px, i, j, d.kz1 - 1)] + w[pidx(d, px, i, j, d.kz1)]);
  return T(2.) * w[pidx(d, px, i, j, d.kz2)] - T(0.5) * (w[pidx(d, px, i, j, d.kz2 - 1)] + w[pidx(d, px, i, j, d.kz2)]);
}

// STRAIN (vt.f:955-1018) from the seven centred values around a point of each
// component: c0 centre, then x-, x+, y-, y+, z-, z+.  s: xx,yy,zz,xy,xz,yz.
template <typename T>
__device__ __forceinline__ void strain7(const T (&uc)[7], const T (&vc)[7], const T (&wc)[7], T aui, T auim, T bvj,
                                        T bvjm, T cwk, T cwkm, T (&s)[6], T &g) {
  T dudxp = aui * (uc[2] - uc[0]);
  T dudxm = auim * (uc[0] - uc[1]);
  T dudyp = bvj * (uc[4] - uc[0]);
  T dudym = bvjm * (uc[0] - uc[3]);
  T dudzp = cwk * (uc[6] - uc[0]);
  T dudzm = cwkm * (uc[0] - uc[5]);
  T dvdxp = aui * (vc[2] - vc[0]);
  T dvdxm = auim * (vc[0] - vc[1]);
  T dvdyp = bvj * (vc[4] - vc[0]);
  T dvdym = bvjm * (vc[0] - vc[3]);
  T dvdzp = cwk * (vc[6] - vc[0]);
  T dvdzm = cwkm * (vc[0] - vc[5]);
  T dwdxp = aui * (wc[2] - wc[0]);
  T dwdxm = auim * (wc[0] - wc[1]);
  T dwdyp = bvj * (wc[4] - wc[0]);
  T dwdym = bvjm * (wc[0] - wc[3]);
  T dwdzp = cwk * (wc[6] - wc[0]);
  T dwdzm = cwkm * (wc[0] - wc[5]);
  s[0] = T(0.5) * (dudxp + dudxm);
  s[1] = T(0.5) * (dvdyp + dvdym);
  s[2] = T(0.5) * (dwdzp + dwdzm);
  s[3] = T(0.25) * (dudyp + dudym + dvdxp + dvdxm);
  s[4] = T(0.25) * (dudzp + dudzm + dwdxp + dwdxm);
  s[5] = T(0.25) * (dwdyp + dwdym + dvdzp + dvdzm);
  g = sqrt(T(2.) * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + T(4.) * (s[3] * s[3] + s[5] * s[5] + s[4] * s[4]));
}

// the base values a point contributes to the 22 filtered quantities
template <typename T>
struct Base {
  T uc, vc, wc, g, s[6];
};

template <typename T>
__device__ __forceinline__ T shfl(T v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// centred velocities of plane j over the ring tile (zero outside the array)
template <typename T>
__device__ __forceinline__ void center_plane(const Dims &d, int px, const T *__restrict__ u, const T *__restrict__ v,
                                             const T *__restrict__ w, int j, int ia, int ka, MarchSmem<T> &sm) {
  const int slot = j % 4;
  for (int p = threadIdx.x; p < CR * CC; p += blockDim.x) {
    int c = p % CC, r = p / CC;
    int i = ia - 2 + c, k = ka - 2 + r;
    T a = T(0), b = T(0), e = T(0);
    if (i >= 1 && i <= d.nx && k >= 1 && k <= d.nz) {
      a = cen_u(d, px, u, i, j, k);
      b = cen_v(d, px, v, i, j, k);
      e = cen_w(d, px, w, i, j, k);
    }
    sm.cen[slot][0][r][c] = a;
    sm.cen[slot][1][r][c] = b;
    sm.cen[slot][2][r][c] = e;
  }
}

// raw u, v, w of plane j (2 <= j <= NY-1) over the raw tile into ring slot
// j%4, 8-byte cp.async copies (FP32 rows start at even elements: ia is even)
template <typename T>
__device__ __forceinline__ void issue_raw(const Dims &d, int px, const T *__restrict__ u, const T *__restrict__ v,
                                          const T *__restrict__ w, int j, int ia, int ka, MarchSmem<T> &sm) {
  constexpr int EPU = 8 / sizeof(T);  // elements per copy
  constexpr int UPR = RC / EPU;       // copies per row
  const int slot = j % 4, i0 = ia - 3, k0 = ka - 3;
  const int ilim = sizeof(T) == 8 ? d.nx : px;  // last element a copy may touch
  const bool inside = i0 >= 1 && i0 + RC - 1 <= ilim && k0 >= 1 && k0 + RR - 1 <= d.nz;  // CTA-uniform
  for (int e = threadIdx.x; e < 3 * RR * UPR; e += blockDim.x) {
    int uu = e % UPR, rest = e / UPR, rr = rest % RR, q = rest / RR;
    int i = i0 + uu * EPU, k = k0 + rr;
    if (!inside && (i < 1 || i + EPU - 1 > ilim || k < 1 || k > d.nz)) continue;
    const T *src = q == 0 ? u : (q == 1 ? v : w);
    cp_async8(&sm.raw[slot][q][rr][uu * EPU], src + pidx(d, px, i, j, k));
  }
}

// centred velocities (vt.f:64-74) of an interior plane j from the raw ring
// (slots of j-1 and j); the same formulas and operation order as cen_u/v/w
template <typename T>
__device__ __forceinline__ void center_raw(const Dims &d, int j, int ia, int ka, MarchSmem<T> &sm) {
  const int slot = j % 4, rs = j % 4, rm = (j + 3) % 4, i0 = ia - 3, k0 = ka - 3;
  auto U = [&](int i, int k) { return sm.raw[rs][0][k - k0][i - i0]; };
  auto W = [&](int i, int k) { return sm.raw[rs][2][k - k0][i - i0]; };
  // the ghost formulas apply only in tiles that reach a ghost layer (CTA-uniform)
  const bool xg = ia - 2 <= 1 || ia + TI - 1 >= d.nx, zg = ka - 2 <= 1 || ka + KT + 1 >= d.nz;
  for (int p = threadIdx.x; p < CR * CC; p += blockDim.x) {
    int c = p % CC, r = p / CC;
    int i = ia - 2 + c, k = ka - 2 + r;
    // raw-tile coordinates of (i, k), (i-1, k), (i, k-1)
    int rc = c + 1, rr = r + 1;
    T a = T(0.5) * (sm.raw[rs][0][rr][rc - 1] + sm.raw[rs][0][rr][rc]);
    T b = T(0.5) * (sm.raw[rm][1][rr][rc] + sm.raw[rs][1][rr][rc]);
    T e = T(0.5) * (sm.raw[rs][2][rr - 1][rc] + sm.raw[rs][2][rr][rc]);
    if (xg) {
      if (i == 1) a = T(2.) * U(1, k) - T(0.5) * (U(d.ix1 - 1, k) + U(d.ix1, k));
      else if (i == d.nx) a = T(2.) * U(d.ix2, k) - T(0.5) * (U(d.ix2 - 1, k) + U(d.ix2, k));
    }
    if (zg) {
      if (k == 1) e = T(2.) * W(i, 1) - T(0.5) * (W(i, d.kz1 - 1) + W(i, d.kz1));
      else if (k == d.nz) e = T(2.) * W(i, d.kz2) - T(0.5) * (W(i, d.kz2 - 1) + W(i, d.kz2));
    }
    // positions outside the array are never read by an interior strain
    sm.cen[slot][0][r][c] = a;
    sm.cen[slot][1][r][c] = b;
    sm.cen[slot][2][r][c] = e;
  }
}

// strain of plane j at this thread's (i,k) from the ring (slots of j-1, j, j+1)
template <typename T>
__device__ __forceinline__ void strain_at(const Dims &d, const DevMetrics &m, const MarchSmem<T> &sm, int j, int i,
                                          int k, int lane, int wr, T (&s)[6], T &g) {
  const int c = lane + 1, r = wr + 1;
  const int s0 = j % 4, sm1 = (j + 3) % 4, sp1 = (j + 1) % 4;
  T uc[7], vc[7], wc[7];
  auto gather = [&](int q, T(&a)[7]) {
    a[0] = sm.cen[s0][q][r][c];
    a[1] = sm.cen[s0][q][r][c - 1];
    a[2] = sm.cen[s0][q][r][c + 1];
    a[3] = sm.cen[sm1][q][r][c];
    a[4] = sm.cen[sp1][q][r][c];
    a[5] = sm.cen[s0][q][r - 1][c];
    a[6] = sm.cen[s0][q][r + 1][c];
  };
  gather(0, uc);
  gather(1, vc);
  gather(2, wc);
  strain7<T>(uc, vc, wc, (T)m.au[i], (T)m.au[i - 1], (T)m.bv[j], (T)m.bv[j - 1], (T)m.cw[k], (T)m.cw[k - 1], s, g);
}

template <typename T>
__global__ void __launch_bounds__(NW * 32, sizeof(T) == 4 ? 2 : 1)
    k_dynamic_march(Dims d, DevMetrics m, int px, const T *__restrict__ u, const T *__restrict__ v,
                    const T *__restrict__ w, const double *__restrict__ dxdydz, T *__restrict__ gs, int gpitch,
                    T *__restrict__ imm2, T *__restrict__ ilm2) {
  extern __shared__ __align__(16) unsigned char smraw[];
  MarchSmem<T> &sm = *reinterpret_cast<MarchSmem<T> *>(smraw);
  const int lane = threadIdx.x & 31, wr = threadIdx.x >> 5;
  int ia = d.ix1 + blockIdx.x * TO;
  if (ia > d.ix2 - TO + 1) ia = d.ix2 - TO + 1;
  if (ia < d.ix1) ia = d.ix1;
  int ka = d.kz1 + blockIdx.y * KT;
  if (ka > d.kz2 - KT + 1) ka = d.kz2 - KT + 1;
  if (ka < d.kz1) ka = d.kz1;
  const int i = ia - 1 + lane, k = ka - 1 + wr;
  const bool inner = i >= d.ix1 && i <= d.ix2 && k >= d.kz1 && k <= d.kz2;  // strain is defined here
  const bool out = inner && lane >= 1 && lane <= TO && wr >= 1 && wr <= KT;  // this thread owns an output column
  // x pass (vt.f:1156-1169): interior X = w0 q(i-1) + w1 q(i) + w2 q(i+1);
  // at ix1 X = w0 q(ix1) + w1 q(ix1+1) + w2 q(ix1+2), at ix2 mirrored
  const bool xedge = (i == d.ix1) || (i == d.ix2);
  int srcA, srcB;
  if (i == d.ix1) { srcA = lane + 1; srcB = lane + 2; }
  else if (i == d.ix2) { srcA = lane - 1; srcB = lane - 2; }
  else { srcA = lane - 1; srcB = lane + 1; }
  srcA = min(max(srcA, 0), 31);
  srcB = min(max(srcB, 0), 31);
  T wx0 = T(0), wx1 = T(0), wx2 = T(0);
  if (i >= 1 && i <= d.nx) { wx0 = (T)m.whx[i * 3]; wx1 = (T)m.whx[i * 3 + 1]; wx2 = (T)m.whx[i * 3 + 2]; }
  // z pass (vt.f:1216-1264), one-sided at kz1 and kz2 (ITYPE(5), ITYPE(6) > 0)
  T wz0 = T(0), wz1 = T(0), wz2 = T(0);
  int zr0 = wr - 1, zr1 = wr, zr2 = wr + 1;
  if (out) {
    wz0 = (T)m.whz[k * 3]; wz1 = (T)m.whz[k * 3 + 1]; wz2 = (T)m.whz[k * 3 + 2];
    if (k == d.kz1) { zr0 = wr; zr1 = wr + 1; zr2 = wr + 2; }
    else if (k == d.kz2) { zr0 = wr; zr1 = wr - 1; zr2 = wr - 2; }
  }

  T Ya[NQ] = {}, Yb[NQ] = {};  // partial y sums: Ya of plane j-1 (two terms), Yb of plane j (one term)
  T acc_m = T(0), acc_l = T(0);

  // x pass of the 22 quantities of this column's plane from its base and its
  // x neighbours', folded into the y partial sums; the completed Y of the
  // plane before goes to shared memory (row wr) for the z pass.  Tiles whose
  // output columns are all interior (the CTA-uniform common case) take the
  // interior stencil without selects.
  const bool xfast = ia > d.ix1 && ia + TO - 1 < d.ix2;
  auto fold = [&](int c, T x) {
    sm.yb[c][wr][lane] = Ya[c] + T(0.25) * x;
    Ya[c] = Yb[c] + T(0.50) * x;
    Yb[c] = T(0.25) * x;
  };
  // F, S, B: the values at the first, second and third x-stencil points of
  // this lane's column; inside (i-1, i, i+1), at ix1 (ix1, ix1+1, ix1+2), at
  // ix2 (ix2, ix2-1, ix2-2)
  auto nbr3 = [&](auto &V, auto &F, auto &S, auto &B) {
    constexpr int N = sizeof(V) / sizeof(T);
    if (xfast) {
#pragma unroll
      for (int n = 0; n < N; n++) {
        F[n] = shfl(V[n], max(lane - 1, 0));
        S[n] = V[n];
        B[n] = shfl(V[n], min(lane + 1, 31));
      }
    } else {
#pragma unroll
      for (int n = 0; n < N; n++) {
        T a = shfl(V[n], srcA);
        F[n] = xedge ? V[n] : a;
        S[n] = xedge ? a : V[n];
        B[n] = shfl(V[n], srcB);
      }
    }
  };
  auto x_and_y = [&](const Base<T> &b) {
    // quantities 0-12 from |S| and S_ij (G*S and S in the order xx,yy,zz,xy,yz,xz; G)
    {
      T V[7] = {b.g, b.s[0], b.s[1], b.s[2], b.s[3], b.s[5], b.s[4]};
      T F[7], S[7], B[7];
      nbr3(V, F, S, B);
#pragma unroll
      for (int c = 0; c < 6; c++)
        fold(c, (wx0 * (F[0] * F[1 + c]) + wx1 * (S[0] * S[1 + c])) + wx2 * (B[0] * B[1 + c]));
#pragma unroll
      for (int c = 0; c < 6; c++) fold(6 + c, (wx0 * F[1 + c] + wx1 * S[1 + c]) + wx2 * B[1 + c]);
      fold(12, (wx0 * F[0] + wx1 * S[0]) + wx2 * B[0]);
    }
    // quantities 13-21 from the centred velocities
    {
      T V[3] = {b.uc, b.vc, b.wc};
      T F[3], S[3], B[3];
      nbr3(V, F, S, B);
#pragma unroll
      for (int c = 0; c < 3; c++) fold(13 + c, (wx0 * F[c] + wx1 * S[c]) + wx2 * B[c]);
      const int pa[6] = {0, 1, 2, 0, 1, 0}, pb[6] = {0, 1, 2, 1, 2, 2};  // uu vv ww uv vw uw
#pragma unroll
      for (int c = 0; c < 6; c++)
        fold(16 + c, (wx0 * (F[pa[c]] * F[pb[c]]) + wx1 * (S[pa[c]] * S[pb[c]])) + wx2 * (B[pa[c]] * B[pb[c]]));
    }
  };
  // z pass of the completed plane j from shared memory, M_ij and L_ij
  // (vt.f:216-290), clipped sums in j order
  auto z_and_ml = [&](int j) {
    // filtered quantity c at this cell, read when first needed (fewer live registers)
    auto zq = [&](int c) {
      return (wz0 * sm.yb[c][zr0][lane] + wz1 * sm.yb[c][zr1][lane]) + wz2 * sm.yb[c][zr2][lane];
    };
    const T C = T(1.0), R = T(6.);
    T dx = (T)dxdydz[fidx(d, i, j, k)];
    T gb = zq(12);
    T mxx = C * dx * (R * gb * zq(6) - zq(0));
    T myy = C * dx * (R * gb * zq(7) - zq(1));
    T mzz = C * dx * (R * gb * zq(8) - zq(2));
    T mxy = C * dx * (R * gb * zq(9) - zq(3));
    T myz = C * dx * (R * gb * zq(10) - zq(4));
    T mxz = C * dx * (R * gb * zq(11) - zq(5));
    T mmv = mxx * mxx + myy * myy + mzz * mzz + T(2.) * (mxy * mxy + myz * myz + mxz * mxz);
    T uh = zq(13), vh = zq(14), wh = zq(15);
    T lxx = (zq(16) - uh * uh) * mxx;
    T lyy = (zq(17) - vh * vh) * myy;
    T lzz = (zq(18) - wh * wh) * mzz;
    T lxy = (zq(19) - uh * vh) * mxy;
    T lyz = (zq(20) - vh * wh) * myz;
    T lxz = (zq(21) - uh * wh) * mxz;
    T lmv = lxx + lyy + lzz + T(2.) * (lxy + lyz + lxz);
    acc_m += mmv;
    if (lmv < T(0)) lmv = T(0);
    acc_l += lmv;
  };

  // prologue: |S|, S_ij of plane jy2 (the periodic copy in ghost row 1)
  const int jy1 = d.jy1, jy2 = d.jy2, ny = d.ny;
  center_plane(d, px, u, v, w, jy2 - 1, ia, ka, sm);
  center_plane(d, px, u, v, w, jy2, ia, ka, sm);
  center_plane(d, px, u, v, w, ny, ia, ka, sm);
  __syncthreads();
  Base<T> b{};
  if (inner) strain_at(d, m, sm, jy2, i, k, lane, wr, b.s, b.g);
  __syncthreads();
  // raw planes 3, 4, 5 in flight (one copy group each), planes 1..3 centred
  // directly
  for (int p = jy1 + 1; p <= jy1 + 3; p++) {
    if (p <= ny - 1) issue_raw(d, px, u, v, w, p, ia, ka, sm);
    cp_async_commit();
  }
  center_plane(d, px, u, v, w, 1, ia, ka, sm);
  center_plane(d, px, u, v, w, jy1, ia, ka, sm);
  if (jy1 + 1 <= ny) center_plane(d, px, u, v, w, jy1 + 1, ia, ka, sm);
  __syncthreads();
  // ghost row 1: centred velocities of row 1, strain of row jy2
  b.uc = sm.cen[1 % 4][0][wr + 1][lane + 1];
  b.vc = sm.cen[1 % 4][1][wr + 1][lane + 1];
  b.wc = sm.cen[1 % 4][2][wr + 1][lane + 1];
#pragma unroll
  for (int c = 0; c < NQ; c++) { Ya[c] = T(0); Yb[c] = T(0); }
  x_and_y(b);  // only Yb (first term of Y(jy1)) is used
  for (int j = jy1; j <= jy2; j++) {
    // raw plane j+2 has landed (j+3 may still be in flight); after the
    // barrier every thread's copies are visible and every read of the slots
    // reused below (centred plane j-2, raw plane j) is done
    cp_async_wait<1>();
    __syncthreads();
    const int pc = j + 2;
    if (pc <= ny - 1) center_raw(d, pc, ia, ka, sm);
    else if (pc == ny) center_plane(d, px, u, v, w, ny, ia, ka, sm);
    if (j + 4 <= ny - 1) issue_raw(d, px, u, v, w, j + 4, ia, ka, sm);
    cp_async_commit();
    Base<T> bj{};
    if (inner) strain_at(d, m, sm, j, i, k, lane, wr, bj.s, bj.g);
    bj.uc = sm.cen[j % 4][0][wr + 1][lane + 1];
    bj.vc = sm.cen[j % 4][1][wr + 1][lane + 1];
    bj.wc = sm.cen[j % 4][2][wr + 1][lane + 1];
    if (j == jy1) {
      sm.sgb[0][wr][lane] = bj.g;
#pragma unroll
      for (int c = 0; c < 6; c++) sm.sgb[1 + c][wr][lane] = bj.s[c];
    }
    if (out) gs[pidx(d, gpitch, i, j, k)] = bj.g;
    x_and_y(bj);  // completes Y(j-1) (unused for j = jy1)
    __syncthreads();
    if (j > jy1 && out) z_and_ml(j - 1);
  }
  cp_async_wait<0>();
  // ghost row NY: centred velocities of row NY, strain of row jy1
  {
    Base<T> bn{};
    bn.uc = sm.cen[ny % 4][0][wr + 1][lane + 1];
    bn.vc = sm.cen[ny % 4][1][wr + 1][lane + 1];
    bn.wc = sm.cen[ny % 4][2][wr + 1][lane + 1];
    bn.g = sm.sgb[0][wr][lane];
#pragma unroll
    for (int c = 0; c < 6; c++) bn.s[c] = sm.sgb[1 + c][wr][lane];
    __syncthreads();  // every z pass of the last loop iteration has read yb
    x_and_y(bn);
    __syncthreads();
    if (out) z_and_ml(jy2);
  }
  if (out) {
    imm2[(i - 1) + d.nx * (k - 1)] = acc_m / T(d.ny - 2);
    ilm2[(i - 1) + d.nx * (k - 1)] = acc_l / T(d.ny - 2);
  }
}

// BOUNDTURB on a j-independent (NX,NZ) array: x sides then z sides
template <typename T>
__global__ void k_boundturb2(Dims d, T *a, int iflg) {
  // single block: the x-side fills, then the z-side fills, in order
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    int mode = 0;
    if (iflg == 0) {
      if (t > 700) mode = 2;
      else if (t != 0 && t != 500 && t != 300) mode = 1;
    } else {
      if (t != 0 && t != 500 && t != 300) mode = 2;
    }
    if (!mode || ib == 3 || ib == 4) continue;
    T sg = mode == 1 ? T(-1.) : T(1.);
    if (ib <= 2) {
      int dst = ib == 1 ? 1 : d.nx, src = ib == 1 ? 2 : d.ix2;
      for (int k = 1 + threadIdx.x; k <= d.nz; k += blockDim.x)
        a[(dst - 1) + d.nx * (k - 1)] = sg * a[(src - 1) + d.nx * (k - 1)];
    } else {
      int dst = ib == 5 ? 1 : d.nz, src = ib == 5 ? 2 : d.kz2;
      for (int i = 1 + threadIdx.x; i <= d.nx; i += blockDim.x)
        a[(i - 1) + d.nx * (dst - 1)] = sg * a[(i - 1) + d.nx * (src - 1)];
    }
    __syncthreads();
  }
}

// TV = (ILM/IMM) Delta^2 |S| where IMM > sqrt(eps), >= 0 (vt.f:416-427) at
// interior cells (BOUNDTURB fills the ghosts afterwards)
template <typename T>
__global__ void __launch_bounds__(256)
    k_tv(Dims d, const T *__restrict__ ilm2, const T *__restrict__ imm2, const double *__restrict__ dxdydz,
         const T *__restrict__ gs, int gpitch, double *__restrict__ tv, T seps) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncell) return;
  int i = 1 + (int)(q % d.nx);
  int k = 1 + (int)(q / ((long long)d.nx * d.ny));
  int j = 1 + (int)((q / d.nx) % d.ny);
  if (i < d.ix1 || i > d.ix2 || j < d.jy1 || j > d.jy2 || k < d.kz1 || k > d.kz2) return;
  T il = ilm2[(i - 1) + d.nx * (k - 1)], im = imm2[(i - 1) + d.nx * (k - 1)];
  if (il < T(0)) il = T(0);
  T v = T(0);
  if (im > seps) v = (il / im) * (T)dxdydz[q] * gs[pidx(d, gpitch, i, j, k)];
  if (v < T(0)) v = T(0);
  tv[q] = (double)v;
}

// Smagorinsky (isgs = 1): TV = css^2 Delta^2 |S| (vt.f:160-168), the strain
// from the centred velocities of the seven points around each cell
__global__ void __launch_bounds__(256)
    k_smag(Dims d, DevMetrics m, const double *__restrict__ u, const double *__restrict__ v,
           const double *__restrict__ w, const double *__restrict__ dxdydz, double *__restrict__ tv, double css) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.ncell) return;
  int i = 1 + (int)(q % d.nx);
  int k = 1 + (int)(q / ((long long)d.nx * d.ny));
  int j = 1 + (int)((q / d.nx) % d.ny);
  double g = 0.;
  if (i >= d.ix1 && i <= d.ix2 && j >= d.jy1 && j <= d.jy2 && k >= d.kz1 && k <= d.kz2) {
    const int di[7] = {0, -1, 1, 0, 0, 0, 0}, dj[7] = {0, 0, 0, -1, 1, 0, 0}, dk[7] = {0, 0, 0, 0, 0, -1, 1};
    double uc[7], vc[7], wc[7];
#pragma unroll
    for (int p = 0; p < 7; p++) {
      uc[p] = cen_u(d, d.nx, u, i + di[p], j + dj[p], k + dk[p]);
      vc[p] = cen_v(d, d.nx, v, i + di[p], j + dj[p], k + dk[p]);
      wc[p] = cen_w(d, d.nx, w, i + di[p], j + dj[p], k + dk[p]);
    }
    double s[6];
    strain7<double>(uc, vc, wc, m.au[i], m.au[i - 1], m.bv[j], m.bv[j - 1], m.cw[k], m.cw[k - 1], s, g);
  }
  tv[q] = css * css * 1.0 * dxdydz[q] * g;
}

template <typename T>
int turvis_dynamic(eddy_ctx *ctx, int px, const T *u, const T *v, const T *w, T *gs, T *imm2, T *ilm2) {
  const Dims &d = ctx->d;
  cudaStream_t st = ctx->stream;
  const size_t smem = sizeof(MarchSmem<T>);
  EDDY_CUDA(cudaFuncSetAttribute(k_dynamic_march<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int mi = d.ix2 - d.ix1 + 1, mk = d.kz2 - d.kz1 + 1;
  dim3 g((mi + TO - 1) / TO, (mk + KT - 1) / KT);
  k_dynamic_march<T><<<g, NW * 32, smem, st>>>(d, ctx->m, px, u, v, w, ctx->dxdydz, gs, px, imm2, ilm2);
  EDDY_LAUNCHED(ctx);
  k_boundturb2<T><<<1, 256, 0, st>>>(d, ilm2, 0);
  EDDY_LAUNCHED(ctx);
  k_boundturb2<T><<<1, 256, 0, st>>>(d, imm2, 1);
  EDDY_LAUNCHED(ctx);
  long long nb = (d.ncell + 255) / 256;
  k_tv<T><<<(unsigned)nb, 256, 0, st>>>(d, ilm2, imm2, ctx->dxdydz, gs, px, ctx->f[EDDY_TV], (T)std::sqrt(ctx->sc.eps));
  EDDY_LAUNCHED(ctx);
  return EDDY_OK;
}

// BOUNDTURB(TV,0) (vt.f:700-757)
int boundturb_tv(eddy_ctx *ctx) {
  const Dims &d = ctx->d;
  double *tv = ctx->f[EDDY_TV];
  int rc;
#define F(...) \
  if ((rc = launch_fill_plane(ctx, __VA_ARGS__)) != EDDY_OK) return rc
  for (int ib = 1; ib <= 6; ib++) {
    int t = d.itype[ib];
    int mode = 0;
    if (t > 700) mode = 2;
    else if (t != 0 && t != 500 && t != 300) mode = 1;
    if (!mode) continue;
    double sg = mode == 1 ? -1. : 1.;
    switch (ib) {
      case 1: F(tv, 0, 1, 2, sg, 0); break;
      case 2: F(tv, 0, d.nx, d.ix2, sg, 0); break;
      case 3: F(tv, 1, 1, 2, sg, 0); break;
      case 4: F(tv, 1, d.ny, d.jy2, sg, 0); break;
      case 5: F(tv, 2, 1, 2, sg, 0); break;
      case 6: F(tv, 2, d.nz, d.kz2, sg, 0); break;
    }
  }
  for (int ib = 1; ib <= 4; ib++) {
    if (d.itype[ib] != 500) continue;
    switch (ib) {
      case 1: F(tv, 0, 1, d.ix2, 1., 0); break;
      case 2: F(tv, 0, d.nx, 2, 1., 0); break;
      case 3: F(tv, 1, 1, d.jy2, 1., 0); break;
      case 4: F(tv, 1, d.ny, 2, 1., 0); break;
    }
  }
#undef F
  return EDDY_OK;
}
