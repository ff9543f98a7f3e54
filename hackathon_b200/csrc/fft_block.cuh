// Block-cooperative FP32 FFTs for sm_100a.
//
// An n-point complex transform is spread over n/8 threads, each holding 8
// points in registers. Stages are radix-8 Stockham butterflies computed in
// registers (with a final radix-4 or radix-2 stage when log2(n) is not a
// multiple of 3); between stages the points are exchanged through shared
// memory, ping-ponging between two padded buffers so each stage needs one
// __syncthreads. The output is in natural order, like the reference's
// radix-2 Stockham (motility-ddm/src/fft.js:59-93): same transform, unscaled
// in both directions, fewer passes.
//
// Layout contract: on entry to a stage thread t holds v[q] = x[t + q*n/8],
// q = 0..7, so a caller can feed the first stage straight from registers and
// read the natural-order result from shared memory at pad(k).
//
// Twiddles come from a host table computed in FP64 and rounded once to FP32
// (as the reference's gpuTwiddles, ddm_ref.js:566-574); no sin/cos is
// evaluated on the device. The table holds, for every stage with stride
// Ns > 1 and radix R, a block w[(m-1)*Ns + k] = exp(-2*pi*i*m*k/(Ns*R)),
// m = 1..R-1, k = 0..Ns-1: the lanes of a warp read consecutive k, so a
// load is one wavefront (shared memory) or one cache line (global).
#pragma once

#include <cuda_runtime.h>

namespace ddm {

// Shared-memory index: an XOR swizzle inside each aligned block of 16
// float2, i ^ ((i >> 3) & 15). 64-bit accesses are served per half-warp (16
// lanes over 16 bank pairs); with this swizzle every Stockham stage store
// (strides 1, 8, 64, 512 and the radix-4/2 tails) and every stage load is
// conflict-free, and no padding memory is needed (checked by simulating
// every access pattern of the 512- and 2048-point transforms).
__device__ __forceinline__ int pad(int i) { return i ^ ((i >> 3) & 15); }
__host__ __device__ constexpr int padded(int n) { return n; }

#define DDM_HD __host__ __device__ __forceinline__
DDM_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DDM_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DDM_HD float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
DDM_HD float2 rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// Number of stages of an n-point transform (radix 8 while possible, then 4/2).
__host__ __device__ constexpr int fft_stages(int n) {
  int s = 0;
  for (int ns = 1; ns < n; ns *= ((n / ns) >= 8 ? 8 : (n / ns))) s++;
  return s;
}

// Offset of the twiddle block of the stage with stride Ns, and table size.
__host__ __device__ constexpr int tw_offset(int n, int Ns) {
  int off = 0;
  for (int ns = 1; ns < Ns;) {
    const int r = (n / ns) >= 8 ? 8 : (n / ns);
    if (ns > 1) off += (r - 1) * ns;
    ns *= r;
  }
  return off;
}
__host__ __device__ constexpr int tw_size(int n) { return tw_offset(n, n); }

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  static DDM_HD void run(float2* a) {
    const float2 t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  }
};

template <bool INV>
struct Dft<4, INV> {
  static DDM_HD void run(float2* a) {
    const float2 s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
    const float2 s13 = cadd(a[1], a[3]), d13 = rot<INV>(csub(a[1], a[3]));
    a[0] = cadd(s02, s13);
    a[2] = csub(s02, s13);
    a[1] = cadd(d02, d13);
    a[3] = csub(d02, d13);
  }
};

template <bool INV>
struct Dft<8, INV> {
  static DDM_HD void run(float2* a) {
    float2 e[4] = {a[0], a[2], a[4], a[6]};
    float2 o[4] = {a[1], a[3], a[5], a[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    const float c = 0.70710678118654752f;
    // o[k] *= W8^k, W8 = exp(-+ 2 pi i / 8)
    float2 w1, w3;
    if (!INV) {
      w1 = make_float2(c * (o[1].x + o[1].y), c * (o[1].y - o[1].x));
      w3 = make_float2(c * (o[3].y - o[3].x), -c * (o[3].x + o[3].y));
    } else {
      w1 = make_float2(c * (o[1].x - o[1].y), c * (o[1].x + o[1].y));
      w3 = make_float2(-c * (o[3].x + o[3].y), c * (o[3].x - o[3].y));
    }
    const float2 w2 = rot<INV>(o[2]);
    a[0] = cadd(e[0], o[0]);
    a[4] = csub(e[0], o[0]);
    a[1] = cadd(e[1], w1);
    a[5] = csub(e[1], w1);
    a[2] = cadd(e[2], w2);
    a[6] = csub(e[2], w2);
    a[3] = cadd(e[3], w3);
    a[7] = csub(e[3], w3);
  }
};

// 3-point DFT: X1,2 = a0 - (a1 + a2)/2 -+ i (sqrt(3)/2)(a1 - a2) (forward).
template <bool INV>
struct Dft<3, INV> {
  static DDM_HD void run(float2* a) {
    const float h = 0.86602540378443865f;  // sin(2 pi / 3)
    const float2 s = cadd(a[1], a[2]), d = csub(a[1], a[2]);
    const float2 m = make_float2(fmaf(-0.5f, s.x, a[0].x), fmaf(-0.5f, s.y, a[0].y));
    const float2 r = rot<INV>(make_float2(h * d.x, h * d.y));  // -+ i h d
    a[0] = cadd(a[0], s);
    a[1] = cadd(m, r);
    a[2] = csub(m, r);
  }
};

// 6-point DFT as 2 x 3: DFT-3 of the even and the odd inputs, then
// X[k] = E[k] + W6^k O[k], X[k + 3] = E[k] - W6^k O[k], k < 3.
template <bool INV>
struct Dft<6, INV> {
  static DDM_HD void run(float2* a) {
    float2 e[3] = {a[0], a[2], a[4]};
    float2 o[3] = {a[1], a[3], a[5]};
    Dft<3, INV>::run(e);
    Dft<3, INV>::run(o);
    const float h = 0.86602540378443865f, sg = INV ? 1.f : -1.f;
    const float2 w1 = cmul(o[1], make_float2(0.5f, sg * h));   // W6^1
    const float2 w2 = cmul(o[2], make_float2(-0.5f, sg * h));  // W6^2
    a[0] = cadd(e[0], o[0]);
    a[3] = csub(e[0], o[0]);
    a[1] = cadd(e[1], w1);
    a[4] = csub(e[1], w1);
    a[2] = cadd(e[2], w2);
    a[5] = csub(e[2], w2);
  }
};

// 16-point DFT as 4 x 4: inner DFT-4 over n1 of x[4 n1 + n2], twiddle
// W16^(n2 k1), outer DFT-4 over n2; output X[k1 + 4 k2].
template <bool INV>
struct Dft<16, INV> {
  static DDM_HD void run(float2* a) {
    // W16^p = (cos(2 pi p / 16), -+ sin(2 pi p / 16)), p = n2 * k1
    const float c1 = 0.92387953251128676f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
      float2 b[4] = {a[n2], a[n2 + 4], a[n2 + 8], a[n2 + 12]};
      Dft<4, INV>::run(b);
#pragma unroll
      for (int k1 = 0; k1 < 4; k1++) y[n2][k1] = b[k1];
    }
    const float sg = INV ? 1.f : -1.f;
    // (n2, k1) -> p: (1,1)=1 (1,2)=2 (1,3)=3 (2,1)=2 (2,2)=4 (2,3)=6 (3,1)=3 (3,2)=6 (3,3)=9
    const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h), w3 = make_float2(s1, sg * c1);
    const float2 w6 = make_float2(-h, sg * h), w9 = make_float2(-c1, -sg * s1);
    y[1][1] = cmul(y[1][1], w1);
    y[1][2] = cmul(y[1][2], w2);
    y[1][3] = cmul(y[1][3], w3);
    y[2][1] = cmul(y[2][1], w2);
    y[2][2] = rot<INV>(y[2][2]);
    y[2][3] = cmul(y[2][3], w6);
    y[3][1] = cmul(y[3][1], w3);
    y[3][2] = cmul(y[3][2], w6);
    y[3][3] = cmul(y[3][3], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      float2 c[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      Dft<4, INV>::run(c);
#pragma unroll
      for (int k2 = 0; k2 < 4; k2++) a[k1 + 4 * k2] = c[k2];
    }
  }
};

// One radix-R Stockham stage at stride Ns. Thread t owns butterflies
// j = t + i*n/8 (i < 8/R); butterfly j reads x[j + m*n/R] = v[i + (8/R)*m],
// twiddles input m by exp(-+2*pi*i*m*(j%Ns)/(Ns*R)) and writes output m to
// (j - j%Ns)*R + j%Ns + m*Ns.
// TW_SMEM: the twiddle table is in shared memory (plain loads) rather than
// global memory (read-only cache loads).
template <int n, int R, int Ns, bool INV, bool TW_SMEM, bool TW_REC = false>
__device__ __forceinline__ void stage(float2 (&v)[8], int t, float2* __restrict__ out,
                                      const float2* __restrict__ tw) {
  constexpr int NT = n / 8;
  constexpr int B = 8 / R;
#pragma unroll
  for (int i = 0; i < B; i++) {
    const int j = t + i * NT;
    const int k = j & (Ns - 1);
    float2 a[R];
#pragma unroll
    for (int m = 0; m < R; m++) a[m] = v[i + B * m];
    if (Ns > 1) {
      const float2* tws = tw + tw_offset(n, Ns) + k;
      if constexpr (TW_REC) {
        // W^1 from the FP64-derived table, the higher powers as products
        // (one table load instead of R - 1; each product adds a rounding)
        float2 w1 = TW_SMEM ? tws[0] : __ldg(&tws[0]);
        if (INV) w1.y = -w1.y;
        float2 wm[R];
        wm[1] = w1;
#pragma unroll
        for (int m = 2; m < R; m++) wm[m] = cmul(wm[m / 2], wm[m - m / 2]);
#pragma unroll
        for (int m = 1; m < R; m++) a[m] = cmul(a[m], wm[m]);
      } else {
        // every W^m from the FP64-derived table
#pragma unroll
        for (int m = 1; m < R; m++) {
          float2 w = TW_SMEM ? tws[(m - 1) * Ns] : __ldg(&tws[(m - 1) * Ns]);
          if (INV) w.y = -w.y;
          a[m] = cmul(a[m], w);
        }
      }
    }
    Dft<R, INV>::run(a);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int m = 0; m < R; m++) out[pad(base + m * Ns)] = a[m];
  }
}

template <int n>
__device__ __forceinline__ void load8(float2 (&v)[8], int t, const float2* __restrict__ buf) {
  constexpr int NT = n / 8;
#pragma unroll
  for (int q = 0; q < 8; q++) v[q] = buf[pad(t + q * NT)];
}

// Barrier between stages, scoped to the threads that share the transform:
// SYNC_CTA the whole CTA; SYNC_GROUP a named barrier of the n/8 threads of
// this group (id 1 + group); SYNC_WARP the warp (groups of <= 32 threads).
enum { SYNC_CTA = 0, SYNC_GROUP = 1, SYNC_WARP = 2 };

template <int n, int SYNC>
__device__ __forceinline__ void stage_sync(int bar_id) {
  if constexpr (SYNC == SYNC_WARP) {
    __syncwarp();
  } else if constexpr (SYNC == SYNC_GROUP) {
    asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "n"(n / 8) : "memory");
  } else {
    __syncthreads();
  }
}

// Sync scope for groups of n/8 threads, `groups` of them per CTA.
__host__ __device__ constexpr int sync_kind(int n, int groups) {
  return groups == 1 ? SYNC_CTA : (n / 8 <= 32 ? SYNC_WARP : SYNC_GROUP);
}

template <int n, int Ns, bool INV, bool TW_SMEM, int SYNC, bool TW_REC = false>
struct Stages {
  // Runs the stages from stride Ns on; the stage writes `a`, the next one
  // writes `b`. Ends with a barrier after the last store.
  static __device__ __forceinline__ void run(float2 (&v)[8], int t, float2* a, float2* b,
                                             const float2* __restrict__ tw, int bar_id) {
    constexpr int R = (n / Ns) >= 8 ? 8 : (n / Ns);
    stage<n, R, Ns, INV, TW_SMEM, TW_REC>(v, t, a, tw);
    stage_sync<n, SYNC>(bar_id);
    if constexpr (Ns * R < n) {
      load8<n>(v, t, a);
      Stages<n, Ns * R, INV, TW_SMEM, SYNC, TW_REC>::run(v, t, b, a, tw, bar_id);
    }
  }
};

// Full n-point FFT of the 8 register points per thread (layout contract
// above). Returns the buffer holding the natural-order result (read it at
// pad(k)); the result lands in buf0 when the stage count is odd, else buf1.
template <int n, bool INV, bool TW_SMEM = false, int SYNC = SYNC_CTA, bool TW_REC = false>
__device__ __forceinline__ float2* fft(float2 (&v)[8], int t, float2* buf0, float2* buf1,
                                       const float2* __restrict__ tw, int bar_id = 0) {
  Stages<n, 1, INV, TW_SMEM, SYNC, TW_REC>::run(v, t, buf0, buf1, tw, bar_id);
  return (fft_stages(n) & 1) ? buf0 : buf1;
}

}  // namespace ddm

// ---------------------------------------------------------------------------
// 16 points per thread, radix-16 stages, one exchange buffer per group.
//
// An n-point transform over n/16 threads; stages are radix 16 while n/Ns >= 16
// (then the remaining radix 8/4/2): 2048 = 16 x 16 x 8 takes three passes
// through shared memory instead of the four of the radix-8 plan. Layout
// contract as above with 16 points: on entry to a stage thread t holds
// v[q] = x[t + q*n/16]. Each stage computes its butterflies in registers,
// waits until the group has finished reading the buffer, stores, and waits
// for the stores: one buffer per group, two group barriers per stage. The
// swizzle for this access pattern is i ^ ((i >> 4) & 15) (conflict-free for
// every stage store and load, by simulation). Twiddles: a host FP64 table
// laid out per stage like the radix-8 one, for this plan.

namespace ddm {

__device__ __forceinline__ int pad16(int i) { return i ^ ((i >> 4) & 15); }

__host__ __device__ constexpr int radix16(int n, int ns) { return (n / ns) >= 16 ? 16 : (n / ns); }
__host__ __device__ constexpr int tw_offset16(int n, int Ns) {
  int off = 0;
  for (int ns = 1; ns < Ns;) {
    const int r = radix16(n, ns);
    if (ns > 1) off += (r - 1) * ns;
    ns *= r;
  }
  return off;
}
__host__ __device__ constexpr int tw_size16(int n) { return tw_offset16(n, n); }

// barrier of the NTG threads of group `id` (named barrier 1 + group)
template <int NTG>
__device__ __forceinline__ void group_sync(int id) {
  if constexpr (NTG <= 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(NTG) : "memory");
}

template <int n, int R, int Ns, bool INV>
__device__ __forceinline__ void stage16_compute(float2 (&v)[16], int t, const float2* __restrict__ tw) {
  constexpr int NT = n / 16, B = 16 / R;
#pragma unroll
  for (int i = 0; i < B; i++) {
    const int j = t + i * NT;
    const int k = j & (Ns - 1);
    float2 a[R];
#pragma unroll
    for (int m = 0; m < R; m++) a[m] = v[i + B * m];
    if (Ns > 1) {
      const float2* tws = tw + tw_offset16(n, Ns) + k;
#pragma unroll
      for (int m = 1; m < R; m++) {
        float2 w = tws[(m - 1) * Ns];
        if (INV) w.y = -w.y;
        a[m] = cmul(a[m], w);
      }
    }
    Dft<R, INV>::run(a);
    // butterfly i owns slots i + B*m: in place
#pragma unroll
    for (int m = 0; m < R; m++) v[i + B * m] = a[m];
  }
}

template <int n, int R, int Ns>
__device__ __forceinline__ void stage16_store(const float2 (&v)[16], int t, float2* __restrict__ buf) {
  constexpr int NT = n / 16, B = 16 / R;
#pragma unroll
  for (int i = 0; i < B; i++) {
    const int j = t + i * NT;
    const int k = j & (Ns - 1);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int m = 0; m < R; m++) buf[pad16(base + m * Ns)] = v[i + B * m];
  }
}

template <int n>
__device__ __forceinline__ void load16(float2 (&v)[16], int t, const float2* __restrict__ buf) {
  constexpr int NT = n / 16;
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = buf[pad16(t + q * NT)];
}

template <int n, bool INV, int Ns = 1>
struct Stages16 {
  static __device__ __forceinline__ void run(float2 (&v)[16], int t, float2* buf, const float2* __restrict__ tw,
                                             int bar_id) {
    constexpr int R = radix16(n, Ns);
    stage16_compute<n, R, Ns, INV>(v, t, tw);
    group_sync<n / 16>(bar_id);  // the group is done reading buf
    stage16_store<n, R, Ns>(v, t, buf);
    group_sync<n / 16>(bar_id);  // the stores are visible
    if constexpr (Ns * R < n) {
      load16<n>(v, t, buf);
      Stages16<n, INV, Ns * R>::run(v, t, buf, tw, bar_id);
    }
  }
};

// Full n-point FFT of the 16 register points per thread; the natural-order
// result is left in buf (read it at pad16(k)). The first store waits for the
// group, so buf may hold this FFT's own input until then.
template <int n, bool INV>
__device__ __forceinline__ void fft16(float2 (&v)[16], int t, float2* buf, const float2* __restrict__ tw,
                                      int bar_id) {
  Stages16<n, INV>::run(v, t, buf, tw, bar_id);
}

}  // namespace ddm

// ---------------------------------------------------------------------------
// P points per thread, mixed radix (sizes with a factor 3: 384, 768).
//
// An n-point transform over n/P threads, P = 24 (= 8 x 3) points per thread;
// stage radices are 8 while n/Ns is a multiple of 8, then 6, 4, 3 or 2
// (384 = 8 x 8 x 6, 768 = 8 x 8 x 6 x 2); every radix divides P, so a stage
// is P/R butterflies per thread. Same layout contract, ping-pong buffers,
// swizzle (n is a multiple of 16) and twiddle-table layout as the radix-8
// transforms, with this plan.

namespace ddm {

__host__ __device__ constexpr int radix_p(int n, int ns) {
  return (n / ns) % 8 == 0 ? 8 : (n / ns) % 6 == 0 ? 6 : (n / ns) % 4 == 0 ? 4 : (n / ns) % 3 == 0 ? 3 : 2;
}
__host__ __device__ constexpr int fft_stages_p(int n) {
  int s = 0;
  for (int ns = 1; ns < n; ns *= radix_p(n, ns)) s++;
  return s;
}
__host__ __device__ constexpr int tw_offset_p(int n, int Ns) {
  int off = 0;
  for (int ns = 1; ns < Ns;) {
    const int r = radix_p(n, ns);
    if (ns > 1) off += (r - 1) * ns;
    ns *= r;
  }
  return off;
}
__host__ __device__ constexpr int tw_size_p(int n) { return tw_offset_p(n, n); }

template <int n, int P, int R, int Ns, bool INV>
__device__ __forceinline__ void stage_p(float2 (&v)[P], int t, float2* __restrict__ out,
                                        const float2* __restrict__ tw) {
  constexpr int NT = n / P;
  constexpr int B = P / R;
  static_assert(P % R == 0, "the radix divides the points per thread");
#pragma unroll
  for (int i = 0; i < B; i++) {
    const int j = t + i * NT;
    const int k = j % Ns;
    float2 a[R];
#pragma unroll
    for (int m = 0; m < R; m++) a[m] = v[i + B * m];
    if (Ns > 1) {
      const float2* tws = tw + tw_offset_p(n, Ns) + k;
#pragma unroll
      for (int m = 1; m < R; m++) {
        float2 w = tws[(m - 1) * Ns];
        if (INV) w.y = -w.y;
        a[m] = cmul(a[m], w);
      }
    }
    Dft<R, INV>::run(a);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int m = 0; m < R; m++) out[pad(base + m * Ns)] = a[m];
  }
}

template <int n, int P>
__device__ __forceinline__ void load_p(float2 (&v)[P], int t, const float2* __restrict__ buf) {
  constexpr int NT = n / P;
#pragma unroll
  for (int q = 0; q < P; q++) v[q] = buf[pad(t + q * NT)];
}

template <int n, int P, int Ns, bool INV, int SYNC>
struct StagesP {
  static __device__ __forceinline__ void run(float2 (&v)[P], int t, float2* a, float2* b,
                                             const float2* __restrict__ tw, int bar_id) {
    constexpr int R = radix_p(n, Ns);
    stage_p<n, P, R, Ns, INV>(v, t, a, tw);
    stage_sync<n * 8 / P, SYNC>(bar_id);  // the group's n/P threads
    if constexpr (Ns * R < n) {
      load_p<n, P>(v, t, a);
      StagesP<n, P, Ns * R, INV, SYNC>::run(v, t, b, a, tw, bar_id);
    }
  }
};

// Full n-point transform of the P register points per thread; returns the
// buffer holding the natural-order result (read it at pad(k)).
template <int n, int P, bool INV, int SYNC>
__device__ __forceinline__ float2* fft_p(float2 (&v)[P], int t, float2* buf0, float2* buf1,
                                         const float2* __restrict__ tw, int bar_id = 0) {
  StagesP<n, P, 1, INV, SYNC>::run(v, t, buf0, buf1, tw, bar_id);
  return (fft_stages_p(n) & 1) ? buf0 : buf1;
}

}  // namespace ddm
