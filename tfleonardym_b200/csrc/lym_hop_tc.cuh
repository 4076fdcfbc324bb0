// Tensor-core form of the solver's FP16 hop for 4D SU(3) with several right-hand
// sides (builder-defined; the reference applies the operator one vector at a
// time through TensorFlow einsums, dirac.py:458-523).
//
// With RG right-hand sides per site the hop at one output site is a small dense
// contraction.  Writing the spin projection of direction (mu, +-) as
// h = P psi(x +- mu) (two spins) and the reconstruction of the lower spins as a
// unit phase times an upper one, every one of the 4 spins s of every rhs r gets
//     out[s, r] = sum_{mu, +-} W_{mu,+-} H_{mu,+-}[s, r],     W = U or U^dag,
// where H holds the projected (upper) or phased (lower) half spinor.  In real
// form, with the three colours' (re, im) pairs along K, this is
//     C (4 RG x 6) = sum over 4 pairs of K-blocks  A (4 RG x 16) B (16 x 8)
// with A = the projected spinors of the forward and the backward neighbour of
// direction mu (three colours plus one zero complex each, in FP16) and B = the
// forward link and the backward link's adjoint in real form (6 of 8 columns used).
// One mma.sync.m16n8k16 (FP16 operands, FP32 accumulation) covers 16 rows of
// (spin, rhs) for one mu; a site takes RG/4 x 4 of them.
//
// Each CTA covers S = 256/RG consecutive checkerboard sites x RG right-hand
// sides (blockIdx.y = group of RG rhs), one thread per (site, rhs) for the
// global loads and the epilogue:
//   1. the neighbour table entries and the FP16 links of the tile go to shared
//      memory once (shared by the RG right-hand sides);
//   2. each thread reads its 8 neighbours' norms; every neighbour's half spinor
//      is scaled by norm / (largest of the 8), so one FP32 factor per (site, rhs)
//      restores the scale after the contraction (the FP16 operand never exceeds 2);
//   3. per mu: each thread loads the two neighbour spinors (coalesced 16-byte
//      loads), projects them in packed FP16 and stores the four spin rows into a
//      double-buffered shared tile; the warps then run ldmatrix + mma on it;
//   4. the FP32 results go through shared memory back to one thread per
//      (site, rhs), which runs the same epilogue as the register-tiled kernels.
// The only roundings beyond the FP16 storage are h's (as in the mixed-precision
// hop) and the norm-ratio scaling of h (2^-11 relative each).
#pragma once

#include "lym_eo.cuh"

namespace lym {

namespace tc {

// shared-memory plan of one CTA (bytes)
template <int RG>
struct Plan {
  static constexpr int S = 256 / RG;                 // sites per CTA
  static constexpr int kSiteStride = 128 * RG + 16;  // 4 RG rows of 32 B, +16 B against bank conflicts
  static constexpr int kTile = S * kSiteStride;      // one spin-row tile
  static constexpr int kLinks = S * 8 * 10 * 4;      // [site][dir][10 half2]
  static constexpr int kCodes = S * 8 * 4;           // [dir][site] neighbour codes
  static constexpr int kRed = 256 * 8;               // reduction scratch (doubles)
  static constexpr int kBytes = 2 * kTile + kLinks + kCodes + kRed;
  static_assert(S * RG * 96 <= kTile, "the FP32 results reuse the first tile");
};

LYM_D unsigned h2u(__half2 h) { return *reinterpret_cast<unsigned*>(&h); }
LYM_D __half2 u2h(unsigned u) { return *reinterpret_cast<__half2*>(&u); }
LYM_D unsigned swap_halves(unsigned u) { return __byte_perm(u, 0, 0x1032); }

// unit phase k (0: +1, 1: +i, 2: -1, 3: -i) times a (re, im) half2, by bit operations
LYM_D unsigned phase_h2(int k, unsigned v) {
  switch (k & 3) {
    case 0: return v;
    case 1: return swap_halves(v) ^ 0x00008000u;  // (-im, re)
    case 2: return v ^ 0x80008000u;               // (-re, -im)
    default: return swap_halves(v) ^ 0x80000000u; // (im, -re)
  }
}

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

// The hop of the CTA's tile: on return, acc holds sum over the 8 hops for the
// thread's (site, rhs) = (i, r) (zero for inactive rhs or sites past Vh), in
// FP32 with the neighbour norms applied.  `smem` is the dynamic shared memory
// (Plan<RG>::kBytes).  Every thread of the block must call it.
template <bool G5IN, int RG>
LYM_D void hop_tc(const EoGeom& g, const HopGauge& hg, const EoField& in, int par, int site0, int rhs_base,
                  int i, int r, bool act, char* smem, cx<float> (&acc)[4][3]) {
  using P = Plan<RG>;
  constexpr int S = P::S;
  constexpr int ND = 4, NC = 3;
  const int tid = threadIdx.x;
  const int vh = (int)g.Vh;
  char* tiles = smem;
  unsigned* lk = reinterpret_cast<unsigned*>(smem + 2 * P::kTile);  // [site][dir][10]
  int* codes = reinterpret_cast<int*>(smem + 2 * P::kTile + P::kLinks);  // [dir][site]

  // 1. neighbour codes of the tile (8 x S, coalesced along sites)
  for (int k = tid; k < 8 * S; k += 256) {
    const int d = k / S, s = k - d * S;
    const int cb = site0 + s;
    codes[k] = cb < vh ? __ldg(g.nbr + (par * 2 * ND + d) * vh + cb) : 0;
  }
  __syncthreads();

  // 2. FP16 links of the tile: forward links on the tile's sites (parity par),
  // backward links on the neighbours (parity 1 - par); 5 uint2 units each
  {
    const uint2* lbase = reinterpret_cast<const uint2*>(hg.data);
    for (int k = tid; k < S * 8 * 5; k += 256) {
      const int s = k % S, rest = k / S;
      const int u = rest % 5, d = rest / 5;  // d = 2 mu + dir
      const int mu = d >> 1, dir = d & 1;
      const int cb = site0 + s;
      uint2 v = make_uint2(0u, 0u);
      if (cb < vh) {
        const int lcb = dir == 0 ? cb : (codes[d * S + s] & 0x7fffffff);
        const int lpar = dir == 0 ? par : 1 - par;
        v = __ldg(lbase + (size_t)((mu * 2 + lpar) * hg.nunits + u) * vh + lcb);
      }
      unsigned* dst = lk + (s * 8 + d) * 10 + 2 * u;
      dst[0] = v.x;
      dst[1] = v.y;
    }
  }

  // 3. neighbour norms -> per-hop scale relative to the largest
  float ratio[8];
  float nmax = 0.f;
  const bool live = act && (site0 + i) < vh;
  const int rg = rhs_base + r;
#pragma unroll
  for (int d = 0; d < 8; ++d) {
    ratio[d] = live ? __ldg(in.norm + (size_t)rg * in.Vh + (codes[d * S + i] & 0x7fffffff)) : 0.f;
    nmax = fmaxf(nmax, ratio[d]);
  }
  {
    const float inv = nmax > 0.f ? 1.0f / nmax : 0.f;
#pragma unroll
    for (int d = 0; d < 8; ++d) ratio[d] *= inv;
  }

  // mma roles: warp w owns sites w*(S/8) .. +S/8-1, all RG/4 m-tiles of each
  constexpr int SPW = S / 8, MT = RG / 4;
  const int lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  float c[SPW][MT][4];
#pragma unroll
  for (int a = 0; a < SPW; ++a)
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
      for (int k = 0; k < 4; ++k) c[a][m][k] = 0.f;
  // ldmatrix row address of this lane within a 16-row m-tile
  const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8, lhalf = lane >> 4;
  const unsigned tiles_s = (unsigned)__cvta_generic_to_shared(tiles);
  const uint4* inb = reinterpret_cast<const uint4*>(in.data) + (size_t)rg * in.nunits * in.Vh;

#pragma unroll
  for (int mu = 0; mu < ND; ++mu) {
    char* tile = tiles + (mu & 1) * P::kTile;
    // 3a. load, project, scale and store the two hops of direction mu
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int d = 2 * mu + dir;
      uint4 raw[3] = {make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u)};
      if (live) {
        const int ncb = codes[d * S + i] & 0x7fffffff;
#pragma unroll
        for (int u = 0; u < 3; ++u) raw[u] = __ldg(inb + (size_t)u * vh + ncb);
      }
      const unsigned psi[12] = {raw[0].x, raw[0].y, raw[0].z, raw[0].w, raw[1].x, raw[1].y,
                                raw[1].z, raw[1].w, raw[2].x, raw[2].y, raw[2].z, raw[2].w};
      const __half2 sc = __float2half2_rn(ratio[d]);
      const bool s2pos = fwd != G5IN;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const int jb = Gamma<ND>::col(mu, a), ph = Gamma<ND>::phase(mu, a);
        const int kph = s2pos ? phase_neg(ph) : ph;
        const int lph = fwd ? phase_neg(phase_conj(ph)) : phase_conj(ph);
        unsigned h[3], l[3];
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          const __half2 pr = proj_h2(u2h(psi[a * NC + cc]), u2h(psi[jb * NC + cc]), kph);
          h[cc] = h2u(__hmul2(pr, sc));
          l[cc] = phase_h2(lph, h[cc]);
        }
        // rows m = s * RG + r; the 16-byte half of the row is swizzled by bit 2 of m
        const int mu_ = a * RG + r, ml = jb * RG + r;
        const int hu = dir ^ ((mu_ >> 2) & 1), hl = dir ^ ((ml >> 2) & 1);
        *reinterpret_cast<uint4*>(tile + i * P::kSiteStride + mu_ * 32 + hu * 16) = make_uint4(h[0], h[1], h[2], 0u);
        *reinterpret_cast<uint4*>(tile + i * P::kSiteStride + ml * 32 + hl * 16) = make_uint4(l[0], l[1], l[2], 0u);
      }
    }
    __syncthreads();
    // 3b. tensor cores: for each of the warp's sites, B from the links, A by ldmatrix
#pragma unroll
    for (int a = 0; a < SPW; ++a) {
      const int site = warp * SPW + a;
      unsigned b0 = 0u, b1 = 0u;
      if (gq < 6 && tq < 3) {
        const int cp = gq >> 1;
        const unsigned uf = lk[(site * 8 + 2 * mu) * 10 + cp * 3 + tq];      // U_mu(x)[c'][t]
        const unsigned ub = lk[(site * 8 + 2 * mu + 1) * 10 + tq * 3 + cp];  // U_mu(x-mu)[t][c']
        if ((gq & 1) == 0) {
          b0 = uf ^ 0x80000000u;  // (re, -im)
          b1 = ub;                // adjoint: (re, im) of U[t][c']
        } else {
          b0 = swap_halves(uf);                // (im, re)
          b1 = swap_halves(ub) ^ 0x00008000u;  // (-im, re)
        }
      }
#pragma unroll
      for (int m = 0; m < MT; ++m) {
        const int row = m * 16 + lrow;
        const unsigned addr = tiles_s + (mu & 1) * P::kTile + site * P::kSiteStride + row * 32 +
                              ((lhalf ^ ((row >> 2) & 1)) * 16);
        unsigned a0, a1, a2, a3;
        ldmatrix_x4(addr, a0, a1, a2, a3);
        mma16816(c[a][m], a0, a1, a2, a3, b0, b1);
      }
    }
  }
  // 4. results to shared memory (first tile, last read at mu = 2), then per thread
  float* cout = reinterpret_cast<float*>(tiles);  // [site][rhs][spin][colour] complex
  if (tq < 3) {
#pragma unroll
    for (int a = 0; a < SPW; ++a) {
      const int site = warp * SPW + a;
#pragma unroll
      for (int m = 0; m < MT; ++m) {
#pragma unroll
        for (int hrow = 0; hrow < 2; ++hrow) {
          const int row = m * 16 + gq + 8 * hrow;
          const int s = row / RG, rr = row - s * RG;
          float2* p = reinterpret_cast<float2*>(cout + ((site * RG + rr) * 12 + s * 3 + tq) * 2);
          *p = make_float2(c[a][m][2 * hrow], c[a][m][2 * hrow + 1]);
        }
      }
    }
  }
  __syncthreads();
  const float4* mine = reinterpret_cast<const float4*>(cout + (i * RG + r) * 24);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float4 v = mine[k];
    const int e = 2 * k;  // complex element index e, e + 1 of [spin][colour]
    acc[e / 3][e % 3] = {nmax * v.x, nmax * v.y};
    acc[(e + 1) / 3][(e + 1) % 3] = {nmax * v.z, nmax * v.w};
  }
}

// Deterministic sum over the CTA of one double per thread, per rhs (threads
// with the same r = tid / S): red[tid] = v, then thread r < RG adds its S
// values in site order.  Result in out_r (threads r < RG).  Every thread calls it.
template <int RG>
LYM_D double block_rhs_sum(double v, double* red) {
  constexpr int S = 256 / RG;
  red[threadIdx.x] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < RG) {
    for (int k = 0; k < S; ++k) s += red[threadIdx.x * S + k];
  }
  __syncthreads();
  return s;
}

// Grid-level per-rhs sum with the last-block pattern: each block of the rhs group
// (blockIdx.y) stores RG partials; the last block to arrive adds them in block
// order.  Returns true in the last block, with the totals in `tot` (threads r < RG).
template <int RG>
LYM_D bool grid_rhs_sum(double v, double* red, double* partials, unsigned* counter, int nblk, double& tot) {
  constexpr int S = 256 / RG;
  __shared__ bool last;
  const double bsum = block_rhs_sum<RG>(v, red);
  double* part = partials + (size_t)blockIdx.y * nblk * RG;
  if (threadIdx.x < RG) part[(size_t)blockIdx.x * RG + threadIdx.x] = bsum;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter + blockIdx.y, 1u) == (unsigned)nblk - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // thread (i, r) adds blocks i, i + S, ... of rhs r; then the S per-thread sums in order
  const int i = threadIdx.x % S, r = threadIdx.x / S;
  double s = 0.0;
  for (int b = i; b < nblk; b += S) s += ((volatile double*)part)[(size_t)b * RG + r];
  tot = block_rhs_sum<RG>(s, red);
  if (threadIdx.x == 0) counter[blockIdx.y] = 0u;  // ready for the next use of this slot
  return true;
}

}  // namespace tc

}  // namespace lym
