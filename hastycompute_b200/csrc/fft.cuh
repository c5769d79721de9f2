// Register-resident small DFTs and the "team" FFT used by every pass.
//
// A team of S lanes (inside one warp) transforms one line of length L = E*S; each lane
// holds E complex values in registers.  The transform is the classic two-factor
// (four-step) split L = E x S:
//   forward : lane t holds x[t + S*e] (e < E)          -- layout D_in
//             E-point DFT in registers, twiddle w_L^(t*k1), one shared-memory exchange,
//             S-point DFTs in registers
//             -> lane t holds X[(t + S*c) + E*k2] in v[c*S + k2]  -- layout D_out
//   inverse : the exact transpose (D_out -> D_in), unnormalised.
// Zero-padded inputs (upper half zero, the 2x Toeplitz embedding) and cropped outputs
// (only the lower half needed) are pruned at compile time.
#pragma once

#include "common.cuh"

namespace hb {

// ---- constants: cos/sin of k*pi/8 (exact mathematical values rounded to float) ----
constexpr float kC8 = 0.70710678118654752f;  // cos(pi/4)
constexpr float kC16 = 0.92387953251128676f; // cos(pi/8)
constexpr float kS16 = 0.38268343236508977f; // sin(pi/8)

// multiply by exp(DIR * 2*pi*i * P / 16)
template <int P, int DIR>
HB_DEV float2 tw16(float2 a) {
  constexpr int p = ((P % 16) + 16) % 16;
  if constexpr (p == 0) return a;
  else if constexpr (p == 4) return rot90<DIR>(a);
  else if constexpr (p == 8) return make_float2(-a.x, -a.y);
  else if constexpr (p == 12) return rot90<-DIR>(a);
  else {
    constexpr float c = (p == 1 || p == 15) ? kC16 : (p == 2 || p == 14) ? kC8 : (p == 3 || p == 13) ? kS16
                      : (p == 5 || p == 11) ? -kS16 : (p == 6 || p == 10) ? -kC8 : -kC16;
    constexpr float s0 = (p == 1 || p == 7) ? kS16 : (p == 2 || p == 6) ? kC8 : (p == 3 || p == 5) ? kC16
                       : (p == 9 || p == 15) ? -kS16 : (p == 10 || p == 14) ? -kC8 : -kC16;
    constexpr float s = DIR < 0 ? -s0 : s0;
    return crot(a, c, s);
  }
}

// ---- compile-time cos/sin of 2*pi*p/R for any R (Taylor series, evaluated by the compiler) ----
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double ct_sin_series(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 30; ++k) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
// reduce to [-pi, pi] first so the series converges fast
constexpr double ct_reduce(double x) {
  while (x > 0.5 * kTwoPi) x -= kTwoPi;
  while (x < -0.5 * kTwoPi) x += kTwoPi;
  return x;
}
constexpr double ct_sin(double x) { return ct_sin_series(ct_reduce(x)); }
constexpr double ct_cos(double x) { return ct_sin_series(ct_reduce(x + 0.25 * kTwoPi)); }

// multiply by exp(DIR * 2*pi*i * P / R)
template <int R, int P, int DIR>
HB_DEV float2 twR(float2 a) {
  constexpr int p = ((P % R) + R) % R;
  if constexpr (p == 0) return a;
  else if constexpr (4 * p == R) return rot90<DIR>(a);
  else if constexpr (2 * p == R) return make_float2(-a.x, -a.y);
  else if constexpr (4 * p == 3 * R) return rot90<-DIR>(a);
  else {
    constexpr float c = (float)ct_cos(kTwoPi * p / R);
    constexpr float s0 = (float)ct_sin(kTwoPi * p / R);
    constexpr float s = DIR < 0 ? -s0 : s0;
    return crot(a, c, s);
  }
}

template <int DIR>
HB_DEV void dft2(float2& a, float2& b) {
  float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int DIR>
HB_DEV void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  float2 t0 = cadd(v0, v2), t1 = csub(v0, v2);
  float2 t2 = cadd(v1, v3), t3 = rot90<DIR>(csub(v1, v3));
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3);
  v3 = csub(t1, t3);
}

// ---- generic natural-order DFT of size R in registers ----
template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<1, DIR> {
  static HB_DEV void run(float2*) {}
};
template <int DIR>
struct Dft<2, DIR> {
  static HB_DEV void run(float2* v) { dft2<DIR>(v[0], v[1]); }
};
template <int DIR>
struct Dft<4, DIR> {
  static HB_DEV void run(float2* v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }
};
template <int DIR>
struct Dft<8, DIR> {
  static HB_DEV void run(float2* v) {
    // radix-2 DIT over two 4-point DFTs
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    o1 = tw16<2, DIR>(o1);
    o2 = tw16<4, DIR>(o2);
    o3 = tw16<6, DIR>(o3);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
  }
};
template <int DIR>
struct Dft<16, DIR> {
  // n = n1 + 4*n2, k = 4*k1 + k2: 4-point DFTs over n2, twiddle w16^(n1*k2), 4-point over n1
  static HB_DEV void run(float2* v) {
    float2 y[4][4];
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) {
      y[n1][0] = v[n1]; y[n1][1] = v[n1 + 4]; y[n1][2] = v[n1 + 8]; y[n1][3] = v[n1 + 12];
      dft4<DIR>(y[n1][0], y[n1][1], y[n1][2], y[n1][3]);
    }
    y[1][1] = tw16<1, DIR>(y[1][1]); y[1][2] = tw16<2, DIR>(y[1][2]); y[1][3] = tw16<3, DIR>(y[1][3]);
    y[2][1] = tw16<2, DIR>(y[2][1]); y[2][2] = tw16<4, DIR>(y[2][2]); y[2][3] = tw16<6, DIR>(y[2][3]);
    y[3][1] = tw16<3, DIR>(y[3][1]); y[3][2] = tw16<6, DIR>(y[3][2]); y[3][3] = tw16<9, DIR>(y[3][3]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float2 a = y[0][k2], b = y[1][k2], c = y[2][k2], d = y[3][k2];
      dft4<DIR>(a, b, c, d);
      v[k2] = a; v[4 + k2] = b; v[8 + k2] = c; v[12 + k2] = d;
    }
  }
};

template <int DIR>
struct Dft<3, DIR> {
  // X1,2 = a - (b+c)/2 +- i*DIR*(sqrt(3)/2)*(b - c)
  static HB_DEV void run(float2* v) {
    constexpr float h = 0.86602540378443865f;  // sqrt(3)/2
    const float2 a = v[0], t1 = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const float2 m = make_float2(fmaf(-0.5f, t1.x, a.x), fmaf(-0.5f, t1.y, a.y));
    const float2 r = rot90<DIR>(cscale(d, h));
    v[0] = cadd(a, t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
};
template <int DIR>
struct Dft<5, DIR> {
  static HB_DEV void run(float2* v) {
    constexpr float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;   // cos(2pi/5), cos(4pi/5)
    constexpr float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;    // sin(2pi/5), sin(4pi/5)
    const float2 x0 = v[0];
    const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const float2 a1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
    const float2 a2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
    // b1 = s1 t3 + s2 t4, b2 = s2 t3 - s1 t4, multiplied by DIR * i
    const float2 b1 = rot90<DIR>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    const float2 b2 = rot90<DIR>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(x0, cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

// Mixed radix R = R1 * R2:  n = n1 + R1*n2,  k = k2 + R2*k1
//   R2-point DFTs over n2, twiddle w_R^(n1*k2), R1-point DFTs over n1.
template <int R1, int R2, int DIR>
struct DftMixed {
  static constexpr int R = R1 * R2;
  template <int N1 = 0, int K2 = 0>
  static HB_DEV void twiddle(float2 (&y)[R1][R2]) {
    if constexpr (N1 < R1) {
      if constexpr (K2 < R2) {
        y[N1][K2] = twR<R, N1 * K2, DIR>(y[N1][K2]);
        twiddle<N1, K2 + 1>(y);
      } else {
        twiddle<N1 + 1, 0>(y);
      }
    }
  }
  static HB_DEV void run(float2* v) {
    float2 y[R1][R2];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) y[n1][n2] = v[n1 + R1 * n2];
      Dft<R2, DIR>::run(y[n1]);
    }
    twiddle(y);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      float2 u[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) u[n1] = y[n1][k2];
      Dft<R1, DIR>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) v[k2 + R2 * k1] = u[k1];
    }
  }
};
template <int DIR> struct Dft<6, DIR> : DftMixed<3, 2, DIR> {};
template <int DIR> struct Dft<10, DIR> : DftMixed<5, 2, DIR> {};
template <int DIR> struct Dft<12, DIR> : DftMixed<3, 4, DIR> {};
template <int DIR> struct Dft<20, DIR> : DftMixed<5, 4, DIR> {};
template <int DIR> struct Dft<24, DIR> : DftMixed<3, 8, DIR> {};
template <int DIR> struct Dft<40, DIR> : DftMixed<5, 8, DIR> {};
template <int DIR> struct Dft<32, DIR> : DftMixed<4, 8, DIR> {};

// DFT of size R whose inputs v[R/2..R-1] are zero (they are not read).
// X[2k] = DFT_{R/2}(v)[k];  X[2k+1] = DFT_{R/2}(v[n] * w_R^n)[k]
template <int R, int DIR>
struct DftHalfIn {
  template <int N>
  static HB_DEV void twiddle_half(const float2* v, float2* b) {
    if constexpr (N < R / 2) {
      b[N] = twR<R, N, DIR>(v[N]);
      twiddle_half<N + 1>(v, b);
    }
  }
  static HB_DEV void run(float2* v) {
    constexpr int H = R / 2;
    float2 a[H], b[H];
#pragma unroll
    for (int n = 0; n < H; ++n) a[n] = v[n];
    b[0] = v[0];
    if constexpr (R == 2) {
    } else if constexpr (R == 4) {
      b[1] = rot90<DIR>(v[1]);
    } else if constexpr (R == 8) {
      b[1] = tw16<2, DIR>(v[1]); b[2] = tw16<4, DIR>(v[2]); b[3] = tw16<6, DIR>(v[3]);
    } else if constexpr (R == 16) {
      b[1] = tw16<1, DIR>(v[1]); b[2] = tw16<2, DIR>(v[2]); b[3] = tw16<3, DIR>(v[3]);
      b[4] = tw16<4, DIR>(v[4]); b[5] = tw16<5, DIR>(v[5]); b[6] = tw16<6, DIR>(v[6]);
      b[7] = tw16<7, DIR>(v[7]);
    } else {
      twiddle_half<1>(v, b);
    }
    Dft<H, DIR>::run(a);
    Dft<H, DIR>::run(b);
#pragma unroll
    for (int k = 0; k < H; ++k) { v[2 * k] = a[k]; v[2 * k + 1] = b[k]; }
  }
};

// ---- team configuration for a line of length L ----
template <int L>
struct TeamCfg;
template <> struct TeamCfg<8> { static constexpr int E = 4, S = 2; };
template <> struct TeamCfg<16> { static constexpr int E = 4, S = 4; };
template <> struct TeamCfg<32> { static constexpr int E = 8, S = 4; };
template <> struct TeamCfg<64> { static constexpr int E = 8, S = 8; };
template <> struct TeamCfg<128> { static constexpr int E = 16, S = 8; };
template <> struct TeamCfg<256> { static constexpr int E = 16, S = 16; };
template <> struct TeamCfg<96> { static constexpr int E = 24, S = 4; };
template <> struct TeamCfg<160> { static constexpr int E = 40, S = 4; };
template <> struct TeamCfg<192> { static constexpr int E = 24, S = 8; };
template <> struct TeamCfg<320> { static constexpr int E = 40, S = 8; };
template <> struct TeamCfg<512> { static constexpr int E = 32, S = 16; };

// Shared-memory float2 slots one team needs for its exchange buffer.  The stride is
// chosen so that teams sharing a half-warp land on disjoint banks.
template <int L>
constexpr int team_buf_stride() {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
  constexpr int base = E * (S + 1);
  constexpr int want = S % 16;
  return base + ((want - base % 16) + 32) % 16;
}

// Forward (DIR=-1) or inverse (DIR=+1) transform D_in -> D_out.
//   v    : E registers, v[e] = x[t + S*e]; on return v[c*S + k2] = X[(t+S*c) + E*k2]
//   tw   : table of L entries, tw[k1*S + t] = exp(-2*pi*i*t*k1/L)  (forward sign)
//   buf  : this team's exchange buffer (team_buf_stride<L>() float2)
template <int L, int DIR, bool HALF_IN>
__device__ __forceinline__ void team_fft_din_to_dout(float2* v, int t, float2* buf, const float2* tw) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
  static_assert(E % S == 0, "a lane runs E/S S-point DFTs after the exchange: S must divide E");
  if constexpr (HALF_IN) DftHalfIn<E, DIR>::run(v);
  else Dft<E, DIR>::run(v);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    float2 w = tw[k1 * S + t];
    if (DIR > 0) w.y = -w.y;
    buf[k1 * (S + 1) + t] = cmul(v[k1], w);
  }
  __syncwarp();
#pragma unroll
  for (int c = 0; c < E / S; ++c) {
    float2 u[S];
#pragma unroll
    for (int j = 0; j < S; ++j) u[j] = buf[(t + S * c) * (S + 1) + j];
    Dft<S, DIR>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) v[c * S + k2] = u[k2];
  }
  __syncwarp();
}

// Transpose of the above: D_out -> D_in.  With HALF_OUT only v[0..E/2) (x[n], n < L/2)
// are meaningful on return.
template <int L, int DIR, bool HALF_OUT>
__device__ __forceinline__ void team_fft_dout_to_din(float2* v, int t, float2* buf, const float2* tw) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
#pragma unroll
  for (int c = 0; c < E / S; ++c) {
    float2 u[S];
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) u[k2] = v[c * S + k2];
    Dft<S, DIR>::run(u);
#pragma unroll
    for (int j = 0; j < S; ++j) buf[(t + S * c) * (S + 1) + j] = u[j];
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    float2 w = tw[k1 * S + t];
    if (DIR > 0) w.y = -w.y;
    v[k1] = cmul(buf[k1 * (S + 1) + t], w);
  }
  __syncwarp();
  Dft<E, DIR>::run(v);
  (void)HALF_OUT;  // unused outputs are removed by dead-code elimination
}

// Variants with this lane's twiddles held in registers: twr[k1] = tw[k1*S + t]
// (forward sign).  Lane t's twiddles never change, so kernels that run many lines of
// the same length load them once.
template <int L>
__device__ __forceinline__ void load_lane_twiddles(float2* twr, const float2* tw, int t) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) twr[k1] = tw[k1 * S + t];
}

template <int L, int DIR, bool HALF_IN>
__device__ __forceinline__ void team_fft_din_to_dout_r(float2* v, int t, float2* buf, const float2* twr) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
  if constexpr (HALF_IN) DftHalfIn<E, DIR>::run(v);
  else Dft<E, DIR>::run(v);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    float2 w = twr[k1];
    if (DIR > 0) w.y = -w.y;
    buf[k1 * (S + 1) + t] = k1 == 0 ? v[0] : cmul(v[k1], w);
  }
  __syncwarp();
#pragma unroll
  for (int c = 0; c < E / S; ++c) {
    float2 u[S];
#pragma unroll
    for (int j = 0; j < S; ++j) u[j] = buf[(t + S * c) * (S + 1) + j];
    Dft<S, DIR>::run(u);
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) v[c * S + k2] = u[k2];
  }
  __syncwarp();
}

template <int L, int DIR, bool HALF_OUT>
__device__ __forceinline__ void team_fft_dout_to_din_r(float2* v, int t, float2* buf, const float2* twr) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
#pragma unroll
  for (int c = 0; c < E / S; ++c) {
    float2 u[S];
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) u[k2] = v[c * S + k2];
    Dft<S, DIR>::run(u);
#pragma unroll
    for (int j = 0; j < S; ++j) buf[(t + S * c) * (S + 1) + j] = u[j];
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    float2 w = twr[k1];
    if (DIR > 0) w.y = -w.y;
    const float2 b = buf[k1 * (S + 1) + t];
    v[k1] = k1 == 0 ? b : cmul(b, w);
  }
  __syncwarp();
  Dft<E, DIR>::run(v);
  (void)HALF_OUT;
}

// Team shape (E, S) of a line of length L at run time (the TeamCfg table).
__host__ __device__ inline void team_shape(int L, int* E, int* S) {
  switch (L) {
    case 8: *E = 4; *S = 2; return;
    case 16: *E = 4; *S = 4; return;
    case 32: *E = 8; *S = 4; return;
    case 64: *E = 8; *S = 8; return;
    case 128: *E = 16; *S = 8; return;
    case 256: *E = 16; *S = 16; return;
    case 96: *E = 24; *S = 4; return;
    case 160: *E = 40; *S = 4; return;
    case 192: *E = 24; *S = 8; return;
    case 320: *E = 40; *S = 8; return;
    case 512: *E = 32; *S = 16; return;
    default: *E = L; *S = 1; return;
  }
}

// The frequency a z-column position p holds in the packed diagonal.  Lane t's registers
// r = 4j + c (c < 4) sit at p = (j*S + t)*4 + c: the S lanes of a team read their j-th
// group of four values as one contiguous run of S 16-byte vectors.  The value is the output
// index dout_index<L>(t, r) = (t + S*(r/S)) + E*(r%S) of lane t, register r.
__host__ __device__ inline int column_kz(int L, int p) {
  int E, S;
  team_shape(L, &E, &S);
  const int c = p % 4, q = p / 4;
  const int t = q % S, r = 4 * (q / S) + c;
  return (t + S * (r / S)) + E * (r % S);
}

// team_fft_dout_to_din with an unpadded exchange buffer of exactly L = E*S entries: entry
// (row, col) of the E x S exchange lies at row*S + (col ^ (row % S)).  Both transpose
// directions then touch S distinct banks per team, so a team can exchange inside any L
// contiguous entries, e.g. the part of a tile it has just read into registers.
template <int L, int DIR>
__device__ __forceinline__ void team_fft_dout_to_din_xor(float2* v, int t, float2* buf, const float2* tw) {
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
#pragma unroll
  for (int c = 0; c < E / S; ++c) {
    float2 u[S];
#pragma unroll
    for (int k2 = 0; k2 < S; ++k2) u[k2] = v[c * S + k2];
    Dft<S, DIR>::run(u);
#pragma unroll
    for (int j = 0; j < S; ++j) buf[(t + S * c) * S + (j ^ t)] = u[j];
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) {
    float2 w = tw[k1 * S + t];
    if (DIR > 0) w.y = -w.y;
    v[k1] = cmul(buf[k1 * S + (t ^ (k1 % S))], w);
  }
  __syncwarp();
  Dft<E, DIR>::run(v);
}

// Index helpers for the two layouts.
template <int L>
HB_DEV int din_index(int t, int e) { return t + TeamCfg<L>::S * e; }
template <int L>
HB_DEV int dout_index(int t, int r) {  // r = c*S + k2
  constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
  return (t + S * (r / S)) + E * (r % S);
}

}  // namespace hb
