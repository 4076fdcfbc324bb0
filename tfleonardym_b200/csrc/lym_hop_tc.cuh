// Tensor-core form of the solver's FP16 hop for 4D SU(3) with 16 right-hand
// sides per CTA (builder-defined; the reference applies the operator one vector
// at a time through TensorFlow einsums, dirac.py:458-523).
//
// With 16 right-hand sides per site the hop at one output site is a small dense
// contraction.  For direction mu the spin projection of the forward and the
// backward neighbour gives two upper half-spinor components h_a (a = 0, 1; three
// colours each), and with W = U_mu(x) (forward) or U_mu(x-mu)^dag (backward)
//     out[a]       += W h_a                    (upper spins)
//     out[j(mu,a)] += lambda(mu,a,+-) W h_a    (lower spins, lambda a unit phase)
// In real form, with the three colours' (re, im) pairs along K and one zero complex
// of padding per hop, direction mu is K = 16 (forward 8, backward 8), and for the
// 16 rhs of one site and one upper spin a
//     C_a (16 x 8)     += A_a (16 x 16) B       with B   = the two links in real form,
//     C_j(mu,a) (16x8) += A_a (16 x 16) B'_a    with B'_a = B with each half times lambda,
// one mma.sync.m16n8k16 each (FP16 operands, FP32 accumulation; 6 of 8 columns
// used).  The phase lives in the B operand, which each lane builds from its two
// link entries, so only the upper spins are projected and staged.
//
// Each CTA covers S = 8 consecutive checkerboard sites x 16 right-hand sides
// (blockIdx.y = group of 16 rhs), one thread per (site, rhs) for the global loads
// and the epilogue:
//   1. the FP16 links of the tile go to shared memory once (shared by the 16 rhs);
//   2. each thread reads its 8 neighbours' norms; every neighbour's half spinor
//      is scaled by norm / (largest of the 8), so one FP32 factor per (site, rhs)
//      restores the scale after the contraction (the FP16 operand never exceeds 2);
//   3. per mu: each thread projects its two neighbour spinors in packed FP16 and
//      stores the two upper rows into a double-buffered shared tile (the spinors of
//      mu + 1 are requested meanwhile); each warp then runs, for each of its two
//      sites, 2 ldmatrix and 4 mma;
//   4. the FP32 results go through shared memory back to one thread per
//      (site, rhs), which runs the same epilogue as the register-tiled kernels.
// The only roundings beyond the FP16 storage are h's (as in the mixed-precision
// hop) and the norm-ratio scaling of h (2^-11 relative each).
#pragma once

#include "lym_eo.cuh"

namespace lym {

namespace tc {

constexpr int kRG = 16;             // right-hand sides per CTA
constexpr int kS = 8;               // sites per CTA
constexpr int kThreads = kS * kRG;  // one thread per (site, rhs)
constexpr int kSPW = 2;             // sites per warp in the mma stage
static_assert(kThreads / 32 * kSPW == kS, "every site has one mma warp");

// shared-memory plan of one CTA (bytes)
struct Plan {
  static constexpr int kSiteStride = 2 * kRG * 32 + 16;  // 2 spin rows x 16 rhs x 32 B, +16 B against bank conflicts
  static constexpr int kTile = kS * kSiteStride;         // one staged direction
  static constexpr int kLinks = kS * 8 * 10 * 4;         // [site][dir][10 half2]
  static constexpr int kRed = kThreads * 8;              // reduction scratch (doubles)
  static constexpr int kBytes = 2 * kTile + kLinks + kRed;
  static_assert(kS * kRG * 96 <= 2 * kTile, "the FP32 results reuse both tiles");
};

LYM_D unsigned h2u(__half2 h) { return *reinterpret_cast<unsigned*>(&h); }
LYM_D __half2 u2h(unsigned u) { return *reinterpret_cast<__half2*>(&u); }
LYM_D unsigned swap_halves(unsigned u) { return __byte_perm(u, 0, 0x1032); }

LYM_D void mma16816(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

LYM_D void ldmatrix_x4(unsigned addr, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

// The B-operand entry of column g (odd: the imaginary part of output colour g/2)
// for the link times the unit phase k (0: +1, 1: +i, 2: -1, 3: -i), from the
// lane's real-part column value bre and imaginary-part column value bim.
LYM_D unsigned phased_b(int k, unsigned bre, unsigned bim, bool odd) {
  switch (k & 3) {
    case 0: return odd ? bim : bre;
    case 2: return (odd ? bim : bre) ^ 0x80008000u;
    case 1: return odd ? bre : (bim ^ 0x80008000u);  // Re(iX) = -Im X, Im(iX) = Re X
    default: return odd ? (bre ^ 0x80008000u) : bim;  // Re(-iX) = Im X, Im(-iX) = -Re X
  }
}

// The hop of the CTA's tile: on return, acc holds sum over the 8 hops for the
// thread's (site, rhs) = (i, r) (zero for inactive rhs or sites past Vh), in
// FP32 with the neighbour norms applied.  `smem` is the dynamic shared memory
// (Plan::kBytes).  Every thread of the block must call it.
template <bool G5IN>
LYM_D void hop_tc(const EoGeom& g, const HopGauge& hg, const EoField& in, int par, int site0, int rhs_base,
                  int i, int r, bool act, char* smem, cx<float> (&acc)[4][3]) {
  constexpr int ND = 4, NC = 3;
  const int tid = threadIdx.x;
  const int vh = (int)g.Vh;
  char* tiles = smem;
  unsigned* lk = reinterpret_cast<unsigned*>(smem + 2 * Plan::kTile);  // [site][dir][10]
  const int* nb = g.nbr + par * 2 * ND * vh;
  const int cb = site0 + i;
  const bool site_ok = cb < vh;
  const bool live = act && site_ok;
  const int rg = rhs_base + r;
  const uint4* inb = reinterpret_cast<const uint4*>(in.data) + (size_t)rg * in.nunits * in.Vh;

  // prologue: neighbour codes, norms, links, the spinors of direction 0
  int code[8];
#pragma unroll
  for (int d = 0; d < 8; ++d) code[d] = site_ok ? (__ldg(nb + d * vh + cb) & 0x7fffffff) : 0;
  float ratio[8];
#pragma unroll
  for (int d = 0; d < 8; ++d) ratio[d] = live ? __ldg(in.norm + (size_t)rg * in.Vh + code[d]) : 0.f;
  uint4 raw[2][3];
#pragma unroll
  for (int dir = 0; dir < 2; ++dir)
#pragma unroll
    for (int u = 0; u < 3; ++u)
      raw[dir][u] = live ? __ldg(inb + (size_t)u * vh + code[dir]) : make_uint4(0u, 0u, 0u, 0u);
  {
    // FP16 links of the tile: forward links on the tile's sites (parity par),
    // backward links on the neighbours (parity 1 - par); 5 uint2 units each
    const uint2* lbase = reinterpret_cast<const uint2*>(hg.data);
    for (int k = tid; k < kS * 8 * 5; k += kThreads) {
      const int s = k % kS, rest = k / kS;
      const int u = rest % 5, d = rest / 5;  // d = 2 mu + dir
      const int mu = d >> 1, dir = d & 1;
      const int lcb0 = site0 + s;
      uint2 v = make_uint2(0u, 0u);
      if (lcb0 < vh) {
        const int lcb = dir == 0 ? lcb0 : (__ldg(nb + d * vh + lcb0) & 0x7fffffff);
        const int lpar = dir == 0 ? par : 1 - par;
        v = __ldg(lbase + (size_t)((mu * 2 + lpar) * hg.nunits + u) * vh + lcb);
      }
      unsigned* dst = lk + (s * 8 + d) * 10 + 2 * u;
      dst[0] = v.x;
      dst[1] = v.y;
    }
  }
  float nmax = 0.f;
#pragma unroll
  for (int d = 0; d < 8; ++d) nmax = fmaxf(nmax, ratio[d]);
  {
    const float inv = nmax > 0.f ? 1.0f / nmax : 0.f;
#pragma unroll
    for (int d = 0; d < 8; ++d) ratio[d] *= inv;
  }

  // mma roles: warp w owns sites 2w, 2w + 1; accumulators per site and spin
  const int lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const bool odd = (gq & 1) != 0;
  const bool bcol = gq < 6 && tq < 3;  // columns 6, 7 and rows of the padding complex are zero
  float c[kSPW][4][4];
#pragma unroll
  for (int a = 0; a < kSPW; ++a)
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int k = 0; k < 4; ++k) c[a][s][k] = 0.f;
  // ldmatrix row address of this lane within a 16-row tile (one spin, 16 rhs)
  const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8, lhalf = lane >> 4;
  const unsigned tiles_s = (unsigned)__cvta_generic_to_shared(tiles);

#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
    char* tile = tiles + (mu & 1) * Plan::kTile;
    // project, scale and store the upper rows of the two hops of direction mu
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int d = 2 * mu + dir;
      const unsigned psi[12] = {raw[dir][0].x, raw[dir][0].y, raw[dir][0].z, raw[dir][0].w,
                                raw[dir][1].x, raw[dir][1].y, raw[dir][1].z, raw[dir][1].w,
                                raw[dir][2].x, raw[dir][2].y, raw[dir][2].z, raw[dir][2].w};
      const __half2 sc = __float2half2_rn(ratio[d]);
      const bool s2pos = fwd != G5IN;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
        const int kph = s2pos ? phase_neg(ph) : ph;
        unsigned h[3];
#pragma unroll
        for (int cc = 0; cc < NC; ++cc)
          h[cc] = h2u(__hmul2(proj_h2(u2h(psi[a * NC + cc]), u2h(psi[jb * NC + cc]), kph), sc));
        // row m = a * 16 + r; the 16-byte half of the row is swizzled by bit 2 of m
        const int m = a * kRG + r;
        *reinterpret_cast<uint4*>(tile + i * Plan::kSiteStride + m * 32 + ((dir ^ ((m >> 2) & 1)) * 16)) =
            make_uint4(h[0], h[1], h[2], 0u);
      }
    }
    // request direction mu + 1 while this one is contracted
    if (mu + 1 < ND) {
#pragma unroll
      for (int dir = 0; dir < 2; ++dir)
#pragma unroll
        for (int u = 0; u < 3; ++u)
          raw[dir][u] = live ? __ldg(inb + (size_t)u * vh + code[2 * (mu + 1) + dir]) : make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < kSPW; ++a) {
      const int site = warp * kSPW + a;
      // B for this lane's column: real and imaginary column values of the forward
      // (rows 0-7) and backward (rows 8-15) link entries
      unsigned bre_f = 0u, bim_f = 0u, bre_b = 0u, bim_b = 0u;
      if (bcol) {
        const int cp = gq >> 1;
        const unsigned uf = lk[(site * 8 + 2 * mu) * 10 + cp * 3 + tq];      // U_mu(x)[c'][t]
        const unsigned ub = lk[(site * 8 + 2 * mu + 1) * 10 + tq * 3 + cp];  // U_mu(x-mu)[t][c']
        bre_f = uf ^ 0x80000000u;               // (re, -im)
        bim_f = swap_halves(uf);                // (im, re)
        bre_b = ub;                             // adjoint: (re, im) of U[t][c']
        bim_b = swap_halves(ub) ^ 0x00008000u;  // (-im, re)
      }
      const unsigned b0 = odd ? bim_f : bre_f, b1 = odd ? bim_b : bre_b;
#pragma unroll
      for (int sa = 0; sa < 2; ++sa) {
        const int row = sa * kRG + lrow;
        const unsigned addr = tiles_s + (mu & 1) * Plan::kTile + site * Plan::kSiteStride + row * 32 +
                              ((lhalf ^ ((row >> 2) & 1)) * 16);
        unsigned a0, a1, a2, a3;
        ldmatrix_x4(addr, a0, a1, a2, a3);
        // upper spin sa
        mma16816(c[a][sa], a0, a1, a2, a3, b0, b1);
        // lower spin j(mu, sa) with the forward / backward reconstruction phases
        const int jb = Gamma<ND>::col(mu, sa), ph = Gamma<ND>::phase(mu, sa);
        const int lph_f = phase_neg(phase_conj(ph)), lph_b = phase_conj(ph);
        mma16816(c[a][jb], a0, a1, a2, a3, phased_b(lph_f, bre_f, bim_f, odd), phased_b(lph_b, bre_b, bim_b, odd));
      }
    }
  }
  // results to shared memory (both tiles), then per thread
  __syncthreads();
  float* cout = reinterpret_cast<float*>(tiles);  // [site][rhs][spin][colour] complex
  if (tq < 3) {
#pragma unroll
    for (int a = 0; a < kSPW; ++a) {
      const int site = warp * kSPW + a;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
#pragma unroll
        for (int hrow = 0; hrow < 2; ++hrow) {
          const int rr = gq + 8 * hrow;
          float2* p = reinterpret_cast<float2*>(cout + ((site * kRG + rr) * 12 + s * 3 + tq) * 2);
          *p = make_float2(c[a][s][2 * hrow], c[a][s][2 * hrow + 1]);
        }
      }
    }
  }
  __syncthreads();
  const float4* mine = reinterpret_cast<const float4*>(cout + (i * kRG + r) * 24);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float4 v = mine[k];
    const int e = 2 * k;  // complex element index e, e + 1 of [spin][colour]
    acc[e / 3][e % 3] = {nmax * v.x, nmax * v.y};
    acc[(e + 1) / 3][(e + 1) % 3] = {nmax * v.z, nmax * v.w};
  }
}

// Deterministic sum over the CTA of one double per thread, per rhs (threads
// with the same r = tid / S): red[tid] = v, then thread r < 16 adds its S
// values in site order.  Result in threads r < 16.  Every thread calls it.
LYM_D double block_rhs_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < kRG) {
    for (int k = 0; k < kS; ++k) s += red[threadIdx.x * kS + k];
  }
  __syncthreads();
  return s;
}

// Grid-level per-rhs sum with the last-block pattern: each block of the rhs group
// (blockIdx.y) stores 16 partials; the last block to arrive adds them in block
// order.  Returns true in the last block, with the totals in `tot` (threads r < 16).
LYM_D bool grid_rhs_sum(double v, double* red, double* partials, unsigned* counter, int nblk, double& tot) {
  __shared__ bool last;
  const double bsum = block_rhs_sum(v, red);
  double* part = partials + (size_t)blockIdx.y * nblk * kRG;
  if (threadIdx.x < kRG) part[(size_t)blockIdx.x * kRG + threadIdx.x] = bsum;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter + blockIdx.y, 1u) == (unsigned)nblk - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // thread (i, r) adds blocks i, i + S, ... of rhs r; then the S per-thread sums in order
  const int i = threadIdx.x % kS, r = threadIdx.x / kS;
  double s = 0.0;
  for (int b = i; b < nblk; b += kS) s += ((volatile double*)part)[(size_t)b * kRG + r];
  tot = block_rhs_sum(s, red);
  if (threadIdx.x == 0) counter[blockIdx.y] = 0u;  // ready for the next use of this slot
  return true;
}

}  // namespace tc

}  // namespace lym
