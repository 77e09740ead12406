// Shared-memory batched FFT building blocks for the PM mesh transforms.
//
// A CTA holds a tile of B complex lines of length L and runs a self-sorting
// (Stockham) decimation-in-time FFT on it, one radix stage at a time: every
// thread loads the butterfly legs it owns into registers, twiddles them,
// does its radix-R DFTs in registers and writes the outputs.  The first
// stage may load straight from global memory and the last may store straight
// to global memory, so a pass over a mesh reads and writes HBM once; the
// exchanges between stages go through a padded shared tile.  Radices 16, 8,
// 4, 2 and 3, largest first up to a maximum radix RM.  Twiddles come from a
// table W_L[k] = exp(-2 pi i k / L) computed on the host in double precision
// and rounded once to float (one table per line length).
//
// Stage s with radix R after sub-transforms of size NS (Stockham autosort):
//   inputs   a[j + r L/R],                          r = 0..R-1
//   twiddle  a_r *= W_L^{(j mod NS) r L/(NS R)}     (conjugated for inverse)
//   DFT_R
//   outputs  a[(j / NS) NS R + (j mod NS) + r NS]
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cgfft {

// ------------------------------------------------------------ complex ops
struct cplx { float x, y; };

// The fused multiply-adds are explicit, so that every kernel built on these
// butterflies rounds a product the same way (the compiler's own contraction
// may fuse either product, differently from one kernel to the next).
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x))};
}
// Complex sums as paired fp32 instructions (sm_100's two-lane add and fma,
// through the CUDA float2 intrinsics): one instruction for both components,
// each rounded exactly as the scalar operation.  fma(b, +-1, a) is a +- b
// rounded once, so the sign pairs below give mixed-sign sums in one
// instruction as well.
__device__ __forceinline__ float2 f2(cplx a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cplx c2(float2 a) { return {a.x, a.y}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return c2(__fadd2_rn(f2(a), f2(b))); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) {
  return c2(__ffma2_rn(f2(b), make_float2(-1.0f, -1.0f), f2(a)));
}
// a + (s.x b.x, s.y b.y), one rounding per component
__device__ __forceinline__ cplx cfma(cplx b, float2 s, cplx a) {
  return c2(__ffma2_rn(f2(b), s, f2(a)));
}
// multiply by -i (forward) or +i (inverse):  DIR = -1 forward, +1 inverse
template <int DIR> __device__ __forceinline__ cplx mul_i(cplx a) {
  return DIR < 0 ? cplx{a.y, -a.x} : cplx{-a.y, a.x};
}
// a +- i_DIR t, given t with its components swapped, ts = (t.y, t.x):
// i_DIR t = DIR < 0 ? (t.y, -t.x) : (-t.y, t.x) = ts * isgn<DIR>()
template <int DIR> __device__ __forceinline__ float2 isgn() {
  return DIR < 0 ? make_float2(1.0f, -1.0f) : make_float2(-1.0f, 1.0f);
}
// Twiddle sources: the global table (read through the read-only path), or a
// shared-memory pack of the stage blocks one transform reads (TwPack, below).
// tw_at<B>(tw, i): entry B + i of the table, B the start of a stage block.
template <int B> __device__ __forceinline__ float2 tw_at(const float2* __restrict__ tw, int i) {
  return __ldg(tw + B + i);
}
// two entries (B + i even: 16-byte aligned in the table and in a pack)
template <int B> __device__ __forceinline__ float4 tw_at2(const float2* __restrict__ tw, int i) {
  return __ldg(reinterpret_cast<const float4*>(tw + B + i));
}
template <class TW> struct IsTwPack { static constexpr bool v = false; };
__device__ __forceinline__ float2 tw_ld(const float2* __restrict__ tw, int i) {
  return __ldg(tw + i);
}
template <int DIR> __device__ __forceinline__ cplx twiddle(const float2* __restrict__ tw, int t) {
  float2 w = tw_ld(tw, t);
  return DIR < 0 ? cplx{w.x, w.y} : cplx{w.x, -w.y};
}

// ------------------------------------------------------- radix-R kernels
// In-register DFT of R points with exp(DIR * 2 pi i k m / R).
template <int DIR> __device__ __forceinline__ void dft2(cplx* v) {
  cplx a = v[0], b = v[1];
  v[0] = cadd(a, b); v[1] = csub(a, b);
}

template <int DIR> __device__ __forceinline__ void dft3(cplx* v) {
  // c = cos(2 pi/3) = -1/2, s = sin(2 pi/3) = sqrt(3)/2
  const float s = 0.866025403784438646763723170753f;
  cplx a = v[0], b = v[1], c = v[2];
  cplx t = cadd(b, c);
  // d = b - c with its components swapped, for r = DIR i s d = ds * (s isgn)
  const cplx ds = {b.y - c.y, b.x - c.x};
  const cplx m = cfma(t, make_float2(-0.5f, -0.5f), a);
  const float2 sr = DIR < 0 ? make_float2(s, -s) : make_float2(-s, s);
  v[0] = cadd(a, t);
  v[1] = cfma(ds, sr, m);
  v[2] = cfma(ds, make_float2(-sr.x, -sr.y), m);
}

// OUT2 = 0: plain; 1: output 2 multiplied by i_DIR; 2: output 2 with its
// components swapped (for a following cfma).  Either costs one scalar
// subtraction more than the plain output.
template <int DIR, int OUT2 = 0> __device__ __forceinline__ void dft4(cplx* v) {
  cplx s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
  cplx s1 = cadd(v[1], v[3]);
  // v1 - v3 with its components swapped (two scalar subtractions)
  const cplx ts = {v[1].y - v[3].y, v[1].x - v[3].x};
  const float2 sg = isgn<DIR>();
  v[0] = cadd(s0, s1);
  if constexpr (OUT2 == 0) v[2] = csub(s0, s1);
  else if constexpr (OUT2 == 2) v[2] = cplx{s0.y - s1.y, s0.x - s1.x};
  else v[2] = DIR < 0 ? cplx{s0.y - s1.y, s1.x - s0.x} : cplx{s1.y - s0.y, s0.x - s1.x};
  v[1] = cfma(ts, sg, d0);
  v[3] = cfma(ts, make_float2(-sg.x, -sg.y), d0);
}

// 8-point: two 4-point DFTs on even/odd samples, then the W8 butterflies.
template <int DIR> __device__ __forceinline__ void dft8(cplx* v) {
  const float h = 0.707106781186547524400844362105f;
  cplx e[4] = {v[0], v[2], v[4], v[6]};
  cplx o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR, 2>(o);    // o[2] comes back swapped
  // o[k] *= W8^{DIR k}: k=1: (h, DIR h), k=2: DIR i, k=3: (-h, DIR h)
  cplx o1 = o[1], o3 = o[3];
  o[1] = DIR < 0 ? cplx{h * (o1.x + o1.y), h * (o1.y - o1.x)}
                 : cplx{h * (o1.x - o1.y), h * (o1.y + o1.x)};
  o[3] = DIR < 0 ? cplx{h * (o3.y - o3.x), -h * (o3.x + o3.y)}
                 : cplx{-h * (o3.x + o3.y), h * (o3.x - o3.y)};
  const float2 sg = isgn<DIR>();
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (k == 2) {
      // e2 +- i_DIR o2, o2 swapped
      v[2] = cfma(o[2], sg, e[2]);
      v[6] = cfma(o[2], make_float2(-sg.x, -sg.y), e[2]);
    } else {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
}

// 16-point: 4x4 decomposition, n = 4 n1 + n2, k = k1 + 4 k2.
template <int DIR> __device__ __forceinline__ void dft16(cplx* v) {
  // W16^m = (cos(2 pi m/16), DIR sin(2 pi m/16)) for the chosen direction
  const float c1 = 0.923879532511286756128183189397f;  // cos(pi/8)
  const float s1 = 0.382683432365089771728459984030f;  // sin(pi/8)
  const float h = 0.707106781186547524400844362105f;
  cplx a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    cplx t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
    // a[2][2]'s twiddle W16^{DIR 4} = i_DIR is applied as it is formed
    if (n2 == 2) dft4<DIR, 1>(t);
    else dft4<DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) a[n2][k1] = t[k1];
  }
  // twiddle a[n2][k1] *= W16^{DIR n2 k1}
  const float ds = DIR < 0 ? -1.0f : 1.0f;
  const cplx w1 = {c1, ds * s1}, w2 = {h, ds * h}, w3 = {s1, ds * c1};
  const cplx w6 = {-h, ds * h}, w9 = {-c1, -ds * s1};
  a[1][1] = cmul(a[1][1], w1); a[1][2] = cmul(a[1][2], w2); a[1][3] = cmul(a[1][3], w3);
  a[2][1] = cmul(a[2][1], w2); a[2][3] = cmul(a[2][3], w6);
  a[3][1] = cmul(a[3][1], w3); a[3][2] = cmul(a[3][2], w6); a[3][3] = cmul(a[3][3], w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    cplx t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft4<DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
  }
}

template <int R, int DIR> __device__ __forceinline__ void dft(cplx* v) {
  if constexpr (R == 2) dft2<DIR>(v);
  else if constexpr (R == 3) dft3<DIR>(v);
  else if constexpr (R == 4) dft4<DIR>(v);
  else if constexpr (R == 8) dft8<DIR>(v);
  else if constexpr (R == 16) dft16<DIR>(v);
}

// ------------------------------------------------- factorisation of L
// Radices in application order: RM as often as it divides, then one smaller
// power of two, then 3s.  RM is 16 or 8.
__host__ __device__ constexpr int radix_at(int L, int s, int RM = 16) {
  int m = L;
  int idx = 0;
  while (m % RM == 0) {
    if (idx == s) return RM;
    m /= RM; idx++;
  }
  for (int r = RM / 2; r >= 2; r /= 2) {
    if (m % r == 0) {
      if (idx == s) return r;
      m /= r; idx++;
      break;
    }
  }
  while (m % 3 == 0) {
    if (idx == s) return 3;
    m /= 3; idx++;
  }
  return 0;
}
__host__ __device__ constexpr int num_stages(int L, int RM = 16) {
  int s = 0;
  while (radix_at(L, s, RM) != 0) s++;
  return s;
}
__host__ __device__ constexpr int ns_before(int L, int s, int RM = 16) {
  int ns = 1;
  for (int i = 0; i < s; i++) ns *= radix_at(L, i, RM);
  return ns;
}
__host__ __device__ constexpr bool supported_length(int L, int RM = 16) {
  int prod = 1;
  for (int s = 0; s < num_stages(L, RM); s++) prod *= radix_at(L, s, RM);
  return prod == L && L >= 2;
}

// ------------------------------------------------ per-stage twiddle rows
// The twiddle table of length L is followed by one block per distinct stage
// (NS, R), NS > 1, of the radix-16 and the radix-8 schedules of L: NS rows
// of stage_rp(R) entries, row jm holding W_L^{jm r STEP} for r = 1 .. R-1
// (STEP = L / (NS R); the same values as entries jm r STEP of the table)
// and a zero pad to an even count.  A butterfly's R-1 twiddles are then one
// contiguous, 16-byte-aligned run read by float4 loads at constant offsets.
__host__ __device__ constexpr int stage_rp(int R) { return (R - 1 + 1) / 2 * 2; }

// Offset of stage (NS, R)'s block in a table for length L, or -1; with
// NS = 0 the table's total length.
__host__ __device__ constexpr int stage_tw_offset(int L, int NS, int R) {
  int off = L;
  for (int pass = 0; pass < 2; pass++) {
    const int rm = pass == 0 ? 16 : 8;
    if (!supported_length(L, rm)) continue;
    for (int st = 1; st < num_stages(L, rm); st++) {
      const int ns = ns_before(L, st, rm), r = radix_at(L, st, rm);
      bool seen = false;      // the same (ns, r) earlier in the walk
      for (int p2 = 0; p2 <= pass && !seen; p2++) {
        const int rm2 = p2 == 0 ? 16 : 8;
        if (!supported_length(L, rm2)) continue;
        const int last = p2 < pass ? num_stages(L, rm2) : st;
        for (int s2 = 1; s2 < last; s2++)
          if (ns_before(L, s2, rm2) == ns && radix_at(L, s2, rm2) == r) seen = true;
      }
      if (seen) continue;
      if (NS > 0 && ns == NS && r == R) return off;
      off += ns * stage_rp(r);
    }
  }
  return NS > 0 ? -1 : off;
}
// The same stages' twiddles once more, transposed, after the row blocks:
// R-1 runs of NS entries, run r-1 holding W_L^{jm r STEP} for jm = 0 ..
// NS-1.  Along a line consecutive threads take consecutive jm, so a warp's
// loads of one r fall on one contiguous run.  Offset of stage (NS, R)'s
// block, or -1; with NS = 0 the table's total length.
__host__ __device__ constexpr int stage_twt_offset(int L, int NS, int R) {
  int off = stage_tw_offset(L, 0, 0);
  for (int pass = 0; pass < 2; pass++) {
    const int rm = pass == 0 ? 16 : 8;
    if (!supported_length(L, rm)) continue;
    for (int st = 1; st < num_stages(L, rm); st++) {
      const int ns = ns_before(L, st, rm), r = radix_at(L, st, rm);
      bool seen = false;
      for (int p2 = 0; p2 <= pass && !seen; p2++) {
        const int rm2 = p2 == 0 ? 16 : 8;
        if (!supported_length(L, rm2)) continue;
        const int last = p2 < pass ? num_stages(L, rm2) : st;
        for (int s2 = 1; s2 < last; s2++)
          if (ns_before(L, s2, rm2) == ns && radix_at(L, s2, rm2) == r) seen = true;
      }
      if (seen) continue;
      if (NS > 0 && ns == NS && r == R) return off;
      off += ns * (r - 1);
    }
  }
  return NS > 0 ? -1 : off;
}
__host__ __device__ constexpr int twiddle_table_len(int L) { return stage_twt_offset(L, 0, 0); }

// The table blocks an L-point transform (maximum radix RM, stage mappings LM
// and LML as in fft_io) reads, one per stage after the first: the stage's
// rows where it is column-mapped, its transposed runs where it is
// line-major.  TwPack packs them back to back in shared memory, each rounded
// up to an even count of entries so that the rows stay 16-byte aligned.
__host__ __device__ constexpr int tw_block(int L, int RM, bool LM, bool LML, int st, bool len) {
  const int ns = num_stages(L, RM);
  const int n = ns_before(L, st, RM), r = radix_at(L, st, RM);
  const bool line = st == ns - 1 ? LML : LM;
  if (!len) return line ? stage_twt_offset(L, n, r) : stage_tw_offset(L, n, r);
  return ((line ? n * (r - 1) : n * stage_rp(r)) + 1) / 2 * 2;
}
// Position in the pack of the block that starts at table entry B (-1: none);
// with B < 0 the pack's length.
__host__ __device__ constexpr int tw_pack_pos(int L, int RM, bool LM, bool LML, int B) {
  int pos = 0;
  for (int st = 1; st < num_stages(L, RM); st++) {
    if (B >= 0 && tw_block(L, RM, LM, LML, st, false) == B) return pos;
    pos += tw_block(L, RM, LM, LML, st, true);
  }
  return B >= 0 ? -1 : pos;
}
__host__ __device__ constexpr bool tw_blocks_even(int L, int RM, bool LM, bool LML) {
  for (int st = 1; st < num_stages(L, RM); st++)
    if (tw_block(L, RM, LM, LML, st, false) % 2) return false;
  return true;
}
template <int L, int RM, bool LM, bool LML> struct TwPack {
  static_assert(tw_blocks_even(L, RM, LM, LML), "stage blocks start on even table entries");
  const float2* p;      // the pack in shared memory, 16-byte aligned
  static constexpr int entries = tw_pack_pos(L, RM, LM, LML, -1);
  static constexpr int bytes = entries * 8;
  static constexpr int kL = L, kRM = RM;
  static constexpr bool kLM = LM, kLML = LML;
  // the blocks of the table tw into dst, by T threads (stage ST on)
  template <int T, int ST = 1>
  __device__ static __forceinline__ void copy(float2* dst, const float2* __restrict__ tw) {
    if constexpr (ST < num_stages(L, RM)) {
      constexpr int b = tw_block(L, RM, LM, LML, ST, false);
      constexpr int n = tw_block(L, RM, LM, LML, ST, true);
      constexpr int pos = tw_pack_pos(L, RM, LM, LML, b);
      const float4* src = reinterpret_cast<const float4*>(tw + b);
      float4* d = reinterpret_cast<float4*>(dst + pos);
      for (int i = (int)threadIdx.x; i < n / 2; i += T) d[i] = __ldg(src + i);
      copy<T, ST + 1>(dst, tw);
    }
  }
};
template <int L, int RM, bool LM, bool LML> struct IsTwPack<TwPack<L, RM, LM, LML>> {
  static constexpr bool v = true;
};
template <int B, int L, int RM, bool LM, bool LML>
__device__ __forceinline__ float2 tw_at(const TwPack<L, RM, LM, LML>& tw, int i) {
  constexpr int pos = tw_pack_pos(L, RM, LM, LML, B);
  static_assert(pos >= 0, "the pack does not hold this stage block");
  return tw.p[pos + i];
}
template <int B, int L, int RM, bool LM, bool LML>
__device__ __forceinline__ float4 tw_at2(const TwPack<L, RM, LM, LML>& tw, int i) {
  constexpr int pos = tw_pack_pos(L, RM, LM, LML, B);
  static_assert(pos >= 0, "the pack does not hold this stage block");
  return *reinterpret_cast<const float4*>(tw.p + pos + i);
}

// ------------------------------------------------------------ tile access
// The first stage reads its legs j + r L/R and the last writes its outputs
// (j/NS) NS R + (j mod NS) + r NS; with consecutive threads on consecutive
// butterflies of a line both are coalesced in global memory.  Shared tiles
// are padded (one element per 16 along a line, one per 32 in
// column-interleaved tiles) to spread the stride-R writes over the banks.

// Line-major shared tile: element n of line b at b*SB + n + n/16.
template <int SB>
struct SmemLine {
  cplx* s;
  __device__ __forceinline__ cplx ld(int b, int n) const { return s[b * SB + n + (n >> 4)]; }
  __device__ __forceinline__ void st(int b, int n, cplx v) const { s[b * SB + n + (n >> 4)] = v; }
  // element n of line b sits at line(b) + n + n/16: a stage whose legs are
  // a multiple of 16 apart reaches them at constant offsets from one base
  __device__ __forceinline__ cplx* line(int b) const { return s + b * SB; }
  static constexpr bool kShared = true;
  static constexpr bool kPad16 = true;
};
// Line pitch >= the padded length, rounded to 1 (mod 16) elements: when
// consecutive threads walk across lines (same n, consecutive b), the 8-byte
// accesses then fall 2 words apart mod 32 banks -- conflict-free.
template <int L> __host__ __device__ constexpr int line_pitch() {
  return ((L + L / 16 + 1 + 14) / 16) * 16 + 1;
}

// Column-interleaved shared tile: element n of column b at i = n*B + b,
// stored at i + i/32.
template <int B>
struct SmemCol {
  cplx* s;
  __device__ __forceinline__ int at(int b, int n) const {
    const int i = n * B + b;
    return i + (i >> 5);
  }
  __device__ __forceinline__ cplx ld(int b, int n) const { return s[at(b, n)]; }
  __device__ __forceinline__ void st(int b, int n, cplx v) const { s[at(b, n)] = v; }
  static constexpr bool kShared = true;
};
template <int L, int B> __host__ __device__ constexpr int col_tile_elems() {
  return L * B + (L * B) / 32 + 1;
}

// Dense tile of 16 lines stored n-major ([n][b], 128-byte rows of 16
// complex) as a TMA load with the 128-byte swizzle writes it: the 16-byte
// chunk c of row n sits at chunk c ^ (n mod 8) (the tile starts on a
// 1024-byte boundary).  Consecutive threads on consecutive lines at one n
// touch one 128-byte row: conflict-free; consecutive n of one line fall on
// 8 distinct chunks per 8 rows: two-way conflicts per half-warp.
struct SmemSw16 {
  cplx* s;
  __device__ __forceinline__ int at(int b, int n) const {
    return (n << 4) + ((((b >> 1) ^ n) & 7) << 1) + (b & 1);
  }
  __device__ __forceinline__ cplx ld(int b, int n) const { return s[at(b, n)]; }
  __device__ __forceinline__ void st(int b, int n, cplx v) const { s[at(b, n)] = v; }
  static constexpr bool kShared = true;
};

// The same for 8 columns in 64-byte rows ([n][b]) as a TMA load with the
// 64-byte swizzle writes them: chunk c of row n sits at chunk
// c ^ ((n / 2) mod 4) (the tile starts on a 1024-byte boundary).
struct SmemSw8 {
  cplx* s;
  __device__ __forceinline__ int at(int b, int n) const {
    return (n << 3) + ((((b >> 1) ^ (n >> 1)) & 3) << 1) + (b & 1);
  }
  __device__ __forceinline__ cplx ld(int b, int n) const { return s[at(b, n)]; }
  __device__ __forceinline__ void st(int b, int n, cplx v) const { s[at(b, n)] = v; }
  static constexpr bool kShared = true;
};

// Global lines with compile-time strides: element n of line b at
// p[b * LS + n * ES] (a stage's legs then sit at constant offsets).
template <size_t LS, size_t ES>
struct GmemC {
  float2* p;
  __device__ __forceinline__ cplx ld(int b, int n) const {
    const float2 v = __ldg(p + (size_t)b * LS + (size_t)n * ES);
    return cplx{v.x, v.y};
  }
  __device__ __forceinline__ void st(int b, int n, cplx v) const {
    p[(size_t)b * LS + (size_t)n * ES] = make_float2(v.x, v.y);
  }
  static constexpr bool kShared = false;
  static constexpr bool kPad16 = false;
};

// Global lines: element n of line b at p[b * ls + n * es].
struct Gmem {
  float2* p;
  size_t ls;
  size_t es;
  static constexpr bool kPad16 = false;
  __device__ __forceinline__ cplx ld(int b, int n) const {
    const float2 v = __ldg(p + b * ls + (size_t)n * es);
    return cplx{v.x, v.y};
  }
  __device__ __forceinline__ void st(int b, int n, cplx v) const {
    p[b * ls + (size_t)n * es] = make_float2(v.x, v.y);
  }
  static constexpr bool kShared = false;
};

// Accessors that declare kPad16 = true (SmemLine) take the constant-offset
// paths of stage_io; every other accessor goes through ld / st.
template <class A, class = void> struct HasPad16 { static constexpr bool v = false; };
template <class A> struct HasPad16<A, decltype((void)A::kPad16)> {
  static constexpr bool v = A::kPad16;
};
template <class A> __host__ __device__ constexpr bool has_pad16() { return HasPad16<A>::v; }

// Accessors that declare kDistinct = true are never the same buffer as the
// shared tile `mid` of the transform they start or end (the Green pass's
// loader of the forward-transformed tile, which feeds a second tile), so
// the first stage (first -> mid) and the last (mid -> last) need no barrier
// between their loads and their stores.
template <class A, class = void> struct IsDistinct { static constexpr bool v = false; };
template <class A> struct IsDistinct<A, decltype((void)A::kDistinct)> {
  static constexpr bool v = A::kDistinct;
};
template <class A> __host__ __device__ constexpr bool distinct() { return IsDistinct<A>::v; }

// T = 32: the tile belongs to one warp (thread = lane, barriers are warp
// barriers), so warps of a CTA run their tiles independently.  Otherwise the
// tile belongs to the CTA's T threads.
template <int T> __device__ __forceinline__ void tile_sync() {
  if constexpr (T == 32) __syncwarp();
  else __syncthreads();
}
template <int T> __device__ __forceinline__ int tile_tid() {
  return T == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
}

template <int L, int R, int NS, int B, int T, bool LINE_MAJOR, int DIR, class In, class Out,
          class TW>
__device__ __forceinline__ void stage_io(const In& in, const Out& out, const TW& tw,
                                         bool inplace) {
  constexpr int NBF = L / R;
  constexpr int TOTAL = NBF * B;
  constexpr int PER = (TOTAL + T - 1) / T;
  cplx v[PER][R];
  const int tid = tile_tid<T>();
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int idx = tid + q * T;
    if (TOTAL % T == 0 || idx < TOTAL) {
      const int b = LINE_MAJOR ? idx / NBF : idx % B;
      const int j = LINE_MAJOR ? idx % NBF : idx / B;
      if constexpr (has_pad16<In>() && NBF % 16 == 0) {
        // legs j + r NBF, r NBF a multiple of 16: padded offsets r NBF 17/16
        const cplx* p = in.line(b) + j + (j >> 4);
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = p[r * (NBF + NBF / 16)];
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) v[q][r] = in.ld(b, j + r * NBF);
      }
    }
  }
  if (inplace) tile_sync<T>();
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int idx = tid + q * T;
    if (TOTAL % T == 0 || idx < TOTAL) {
      const int b = LINE_MAJOR ? idx / NBF : idx % B;
      const int j = LINE_MAJOR ? idx % NBF : idx / B;
      const int jm = NS == 1 ? 0 : j % NS;
      if constexpr (NS > 1) {
        // per-stage rows where consecutive threads share a row (the same
        // butterfly of consecutive lines): one broadcast 16-byte load per
        // pair of twiddles.  Along a line consecutive threads would read
        // consecutive rows, R-1 entries apart (768-point Green pass: 2.61
        // ms with rows against 1.85 ms with strided table reads); there they
        // read the transposed runs instead.
        constexpr int OFF = LINE_MAJOR ? -1 : stage_tw_offset(L, NS, R);
        constexpr int OFFT = LINE_MAJOR ? stage_twt_offset(L, NS, R) : -1;
        if constexpr (OFFT >= 0) {
          // along a line: the transposed runs, one contiguous run per r
#pragma unroll
          for (int r = 1; r < R; r++) {
            const float2 w = tw_at<OFFT>(tw, (r - 1) * NS + jm);
            v[q][r] = cmul(v[q][r], DIR < 0 ? cplx{w.x, w.y} : cplx{w.x, -w.y});
          }
        } else if constexpr (OFF >= 0) {
          // the stage's row jm: R-1 twiddles, two per 16-byte load
#pragma unroll
          for (int i = 0; i < stage_rp(R) / 2; i++) {
            const float4 w = tw_at2<OFF>(tw, jm * stage_rp(R) + 2 * i);
            const int r1 = 2 * i + 1, r2 = 2 * i + 2;
            v[q][r1] = cmul(v[q][r1], DIR < 0 ? cplx{w.x, w.y} : cplx{w.x, -w.y});
            if (r2 < R) v[q][r2] = cmul(v[q][r2], DIR < 0 ? cplx{w.z, w.w} : cplx{w.z, -w.w});
          }
        } else {
          static_assert(!IsTwPack<TW>::v, "a twiddle pack holds stage rows and runs only");
          constexpr int STEP = L / (NS * R);
#pragma unroll
          for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], twiddle<DIR>(tw, jm * r * STEP));
        }
      }
      dft<R, DIR>(v[q]);
      const int base = (j / NS) * NS * R + jm;
      if constexpr (has_pad16<Out>() && NS % 16 == 0) {
        // outputs base + r NS, r NS a multiple of 16
        cplx* p = out.line(b) + base + (base >> 4);
#pragma unroll
        for (int r = 0; r < R; r++) p[r * (NS + NS / 16)] = v[q][r];
      } else if constexpr (has_pad16<Out>() && NS == 1 && R == 16) {
        // outputs 16 j + r, r < 16: padded 17 j + r
        cplx* p = out.line(b) + 17 * j;
#pragma unroll
        for (int r = 0; r < R; r++) p[r] = v[q][r];
      } else if constexpr (has_pad16<Out>() && NS == 1 && R == 8) {
        // outputs 8 j + r, r < 8: padded 8 j + j/2 + r
        cplx* p = out.line(b) + 8 * j + (j >> 1);
#pragma unroll
        for (int r = 0; r < R; r++) p[r] = v[q][r];
      } else {
#pragma unroll
        for (int r = 0; r < R; r++) out.st(b, base + r * NS, v[q][r]);
      }
    }
  }
}

// ------------------------------------------------------------ one pass
// Stages S..end of an L-point FFT (maximum radix RM): stage 0 reads `first`,
// the last stage writes `last`, the stages in between work in place on the
// shared tile `mid`.  Every stage that writes `mid` is followed by a barrier.
// LML: the thread mapping of the last stage (the others use LM).
template <int L, int S, int B, int T, bool LM, int DIR, int RM, bool LML, class First, class Mid,
          class Last, class TW>
__device__ __forceinline__ void fft_io_from(const First& first, const Mid& mid, const Last& last,
                                            const TW& tw) {
  constexpr int NSTAGE = num_stages(L, RM);
  constexpr int R = radix_at(L, S, RM);
  constexpr int NS = ns_before(L, S, RM);
  if constexpr (S == NSTAGE - 1) {
    if constexpr (S == 0)
      stage_io<L, R, NS, B, T, LML, DIR>(first, last, tw, First::kShared && Last::kShared);
    else
      stage_io<L, R, NS, B, T, LML, DIR>(mid, last, tw, Last::kShared && !distinct<Last>());
    if constexpr (Last::kShared) tile_sync<T>();
  } else {
    if constexpr (S == 0)
      stage_io<L, R, NS, B, T, LM, DIR>(first, mid, tw, First::kShared && !distinct<First>());
    else
      stage_io<L, R, NS, B, T, LM, DIR>(mid, mid, tw, true);
    tile_sync<T>();
    fft_io_from<L, S + 1, B, T, LM, DIR, RM, LML>(first, mid, last, tw);
  }
}

// One L-point FFT of each of the B lines of a tile.  LM: consecutive threads
// take consecutive butterflies of one line (true) or the same butterfly of
// consecutive lines (false); LML: the same choice for the last stage alone.
// DIR = -1 forward, +1 inverse (unnormalised).
template <int L, int B, int T, bool LM, int DIR, int RM = 16, bool LML = LM, class First,
          class Mid, class Last, class TW>
__device__ __forceinline__ void fft_io(const First& first, const Mid& mid, const Last& last,
                                       const TW& tw) {
  static_assert(supported_length(L, RM), "FFT length must be 2^a 3^b");
  fft_io_from<L, 0, B, T, LM, DIR, RM, LML>(first, mid, last, tw);
}

}  // namespace cgfft
