// ilc_walk4.cuh -- the nn8 walk for the 4 integrand points of one RKF step,
// done as one pass over the grid.
//
// The 4 points of a step lie within one step length (typically < 1 kpc) of
// each other, so almost always in the same grid cell and subcell: they then
// share the reference's spiral cell order, and one walk serves all four. Each
// point keeps its own 8 slots, its own search radius and its own early break
// (volumetric_nn8_reconstruction.cl:157-171): a point stops taking part at the
// cell where its own break condition holds, exactly as its single-point walk
// would. Every point therefore sees the same cells and candidates in the same
// order as alone, and its slots evolve identically -- the result is the
// reference's, bit for bit. What is shared is the spiral/cell bookkeeping and
// the candidate loads (one 16-byte load serves four distance tests). Points in
// a different cell or subcell are walked in a further pass.
#pragma once

#include "ilc_device.cuh"

namespace ilc {

// Threads per block of every kernel that walks with Step4: the slot arrays of
// thread i live in shared memory at index i of each of the 64 rows.
constexpr int kSlotThreads = 128;
constexpr int kSlotRows = 4 * 8;  // (point, slot) pairs

// Shared-memory storage of one block's slot arrays: distance rows, then value
// (or index) rows; row (j, t) holds entry t of point j for all threads.
struct SlotMem {
  float d[kSlotRows][kSlotThreads];
  float v[kSlotRows][kSlotThreads];
};

struct Step4 {
  float qx[4], qy[4], qz[4];
  float* sd;      // this thread's distance column: sd[(j * 8 + t) * kSlotThreads]
  float* sv;      // this thread's value column
  float R[4];
  float rr[4];    // (R + cell_radius)^2: the early-break threshold
  float crad;     // cell radius
  unsigned mi;    // per point j, bits 4j..4j+3: its first maximal slot; while
                  // R == FLT_MAX: its next empty slot
};

__device__ __forceinline__ float& s4_d(const Step4& s, int j, int t) {
  return s.sd[(j * 8 + t) * kSlotThreads];
}
__device__ __forceinline__ float& s4_v(const Step4& s, int j, int t) {
  return s.sv[(j * 8 + t) * kSlotThreads];
}

__device__ __forceinline__ void s4_bind(Step4& s, SlotMem& m) {
  s.sd = &m.d[0][threadIdx.x];
  s.sv = &m.v[0][threadIdx.x];
}

template <int J> __device__ __forceinline__ void s4_set_mi(Step4& s, unsigned k) {
  s.mi = (s.mi & ~(15u << (4 * J))) | (k << (4 * J));
}

// The larger of two (distance, slot) pairs, the left one on ties.
__device__ __forceinline__ void max_left(float& d, int& i, float d2, int i2) {
  const bool right = d2 > d;
  d = right ? d2 : d;
  i = right ? i2 : i;
}

// Search radius and first maximal slot (volumetric_nn8_reconstruction.cl:
// 135-143), as a pairwise tournament: three levels instead of a chain of
// eight; keeping the left pair on ties gives the first slot holding the
// maximum, as the sequential scan does (distances are non-negative, so the
// scan's start at 0 changes nothing).
template <int J> __device__ __forceinline__ void s4_rescan(Step4& s) {
  float d[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) d[t] = s4_d(s, J, t);
  int i0 = 0, i2 = 2, i4 = 4, i6 = 6;
  float a0 = d[0], a2 = d[2], a4 = d[4], a6 = d[6];
  max_left(a0, i0, d[1], 1);
  max_left(a2, i2, d[3], 3);
  max_left(a4, i4, d[5], 5);
  max_left(a6, i6, d[7], 7);
  max_left(a0, i0, a2, i2);
  max_left(a4, i4, a6, i6);
  max_left(a0, i0, a4, i4);
  const float r = a0;
  const int m = i0;
  s.R[J] = r;
  s4_set_mi<J>(s, (unsigned)m);
  const float b = r + s.crad;
  s.rr[J] = b * b;
}

template <int J> __device__ __forceinline__ void s4_init(Step4& s, float empty_value) {
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    s4_d(s, J, t) = FLT_MAX;
    s4_v(s, J, t) = empty_value;
  }
  s.R[J] = FLT_MAX;
  const float b = FLT_MAX + s.crad;
  s.rr[J] = b * b;
  s4_set_mi<J>(s, 0u);
}

// Insertion into point J's slots. While fewer than 8 slots are filled the
// search radius is FLT_MAX (a full set of 8 finite distances makes it
// smaller) and the first-max slot is the next empty one, so the k-th
// accepted candidate goes to slot k without a rescan; the 8th insertion
// rescans. Afterwards: replace the first-max slot and rescan.
template <int J> __device__ __forceinline__ void s4_insert(Step4& s, float dist, float val) {
  const int k = (int)((s.mi >> (4 * J)) & 15u);
  s4_d(s, J, k) = dist;
  s4_v(s, J, k) = val;
  if (s.R[J] == FLT_MAX) {
    s4_set_mi<J>(s, (unsigned)(k + 1));
    if (k == 7) s4_rescan<J>(s);
  } else {
    s4_rescan<J>(s);
  }
}

// Squared-distance threshold of point J: R*R rounded up (a squared distance
// above it cannot give dist < R); +inf while R is FLT_MAX.
template <int J> __device__ __forceinline__ float s4_r2up(const Step4& s) {
  return __fmul_ru(s.R[J], s.R[J]);
}

// Candidate test of point J against its threshold thr: s4_r2up while J takes
// part in the walk, -1 once it has left it (no squared distance passes). thr
// follows R through insertions.
template <int J>
__device__ __forceinline__ void s4_test(Step4& s, float& thr, float d2, float val) {
  if (d2 <= thr) {
    const float dist = sqrtf(d2);
    if (dist < s.R[J]) {
      s4_insert<J>(s, dist, val);
      thr = s4_r2up<J>(s);
    }
  }
}

template <int J> __device__ __forceinline__ float s4_finalize(const Step4& s) {
  float w[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) w[t] = weight3d(s4_d(s, J, t));
  float ws = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) ws = ws + w[t];
  float dot = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) dot = __fmaf_rn(w[t], s4_v(s, J, t), dot);
  float res = 0.0f;
  if (ws != 0.0f && dot != 0.0f) res = dot / ws;
  return res;
}

// Distance tests of one candidate against the active points.
template <bool kSharedXY>
__device__ __forceinline__ void cand_d2(const Step4& s, const float4& P, float d2[4]) {
  if (kSharedXY) {
    const float fx = P.x - s.qx[0], fy = P.y - s.qy[0];
    const float fxy = fx * fx + fy * fy;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float fz = P.z - s.qz[j];
      d2[j] = fxy + fz * fz;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float fx = P.x - s.qx[j], fy = P.y - s.qy[j], fz = P.z - s.qz[j];
      d2[j] = (fx * fx + fy * fy) + fz * fz;
    }
  }
}

template <bool kIdx>
__device__ __forceinline__ void cand_insert(Step4& s, float thr[4], const float d2[4],
                                            const float4& P, int p) {
  const float pay = kIdx ? __int_as_float(p) : P.w;
  s4_test<0>(s, thr[0], d2[0], pay);
  s4_test<1>(s, thr[1], d2[1], pay);
  s4_test<2>(s, thr[2], d2[2], pay);
  s4_test<3>(s, thr[3], d2[3], pay);
}

template <bool kSharedXY, bool kIdx>
__device__ __forceinline__ void test_candidate(Step4& s, float thr[4], const float4& P, int p) {
  float d2[4];
  cand_d2<kSharedXY>(s, P, d2);
  cand_insert<kIdx>(s, thr, d2, P, p);
}

// With a shared x/y part, every point's squared distance is fl(fxy + fz^2)
// >= fxy (rounding is monotone and fz^2 >= 0), so a candidate whose fxy
// exceeds the largest threshold thrmax cannot be inserted for any point.
// thrmax may be stale (larger than the current thresholds): the test only
// skips work that could not insert.
template <bool kSharedXY, bool kIdx>
__device__ __forceinline__ void test_candidate_xy(Step4& s, float thr[4], float thrmax,
                                                  const float4& P, int p) {
  if (kSharedXY) {
    const float fx = P.x - s.qx[0], fy = P.y - s.qy[0];
    const float fxy = fx * fx + fy * fy;
    if (fxy > thrmax) return;
    float d2[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float fz = P.z - s.qz[j];
      d2[j] = fxy + fz * fz;
    }
    cand_insert<kIdx>(s, thr, d2, P, p);
  } else {
    test_candidate<false, kIdx>(s, thr, P, p);
  }
}

// Cells with more candidates than this are scanned through their sub-box codes.
constexpr int kPruneMin = 16;

// Quarters [lo, hi] of one cell axis that the interval [a, b] touches, as a
// 4-bit mask (0: none). t = (x - cell min) * 4 / cell size.
__device__ __forceinline__ unsigned quarter_mask(float a, float b, float cmin, float inv_w) {
  const float tl = (a - cmin) * inv_w, th = (b - cmin) * inv_w;
  if (!(th >= 0.0f) || !(tl < 4.0f)) return 0u;
  const int lo = tl > 0.0f ? (int)tl : 0;
  const int hi = th < 4.0f ? (int)th : 3;
  return (0xFu >> (3 - hi)) & (0xFu << lo);
}

// Bit (sx + 4 sy + 16 sz) set for every sub-box of the cell that meets the
// box [qlo - ext, qhi + ext]: the union of the cubes of half-width
// ext = max R + margin around the active points. A candidate in any other
// sub-box is farther than its point's R from every active point (the margin
// exceeds every rounding error of the codes and of the distance), so it
// would not be inserted.
__device__ __forceinline__ unsigned long long prune_mask(const GridView& g, int ix, int iy,
                                                         int iz, const float qlo[3],
                                                         const float qhi[3], float ext) {
  const float mx = g.min0 + (float)ix * g.cs0;
  const float my = g.min1 + (float)iy * g.cs1;
  const float mz = g.min2 + (float)iz * g.cs2;
  const unsigned xm = quarter_mask(qlo[0] - ext, qhi[0] + ext, mx, g.inv_w0);
  const unsigned ym = quarter_mask(qlo[1] - ext, qhi[1] + ext, my, g.inv_w1);
  const unsigned zm = quarter_mask(qlo[2] - ext, qhi[2] + ext, mz, g.inv_w2);
  const unsigned ys = (ym & 1u) | ((ym & 2u) << 3) | ((ym & 4u) << 6) | ((ym & 8u) << 9);
  const unsigned long long zs = (unsigned long long)(zm & 1u) |
                                ((unsigned long long)(zm & 2u) << 15) |
                                ((unsigned long long)(zm & 4u) << 30) |
                                ((unsigned long long)(zm & 8u) << 45);
  return (unsigned long long)(xm * ys) * zs;
}

// One walk over the spiral of (cx, cy, cz, sub) for the points in `mask`.
// kSharedXY: all 4 points have bit-identical x and y (a view along the z
// axis), so the x/y part of every squared distance, (dx*dx + dy*dy), is one
// value for the 4 points and is evaluated once -- the same operations in the
// same order, hence the same bits, as evaluating it per point.
// kIdx: the slots carry the candidate's sorted index (as float bits) in
// place of its value, for callers that look up several value channels.
template <bool kSharedXY, bool kIdx>
__device__ __forceinline__ void walk4(const GridView& g, const char4* __restrict__ spiral,
                                      Step4& s, unsigned mask, int cx, int cy, int cz, int sub,
                                      WalkStats& st) {
  const char4* order = spiral + sub * 125;
  unsigned act = mask;
  float thr[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) thr[j] = ((mask >> j) & 1u) ? __fmul_ru(s.R[j], s.R[j]) : -1.0f;
  // bounding box of the group's points (for the sub-box pruning)
  float qlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, qhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if ((mask >> j) & 1u) {
      qlo[0] = fminf(qlo[0], s.qx[j]); qhi[0] = fmaxf(qhi[0], s.qx[j]);
      qlo[1] = fminf(qlo[1], s.qy[j]); qhi[1] = fmaxf(qhi[1], s.qy[j]);
      qlo[2] = fminf(qlo[2], s.qz[j]); qhi[2] = fmaxf(qhi[2], s.qz[j]);
    }
  for (int it = 0; it < 125; ++it) {
    const char4 o = order[it];
    const int ix = cx + o.x, iy = cy + o.y, iz = cz + o.z;
    const float ccx = (g.min0 + (float)ix * g.cs0) + g.half0;
    const float ccy = (g.min1 + (float)iy * g.cs1) + g.half1;
    const float ccz = (g.min2 + (float)iz * g.cs2) + g.half2;
    {
      // early break per point: |c - q|^2 > (R + cell_radius)^2
      unsigned brk = 0;
      if (kSharedXY) {
        const float ex = ccx - s.qx[0], ey = ccy - s.qy[0];
        const float exy = ex * ex + ey * ey;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float ez = ccz - s.qz[j];
          if (exy + ez * ez > s.rr[j]) brk |= 1u << j;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float ex = ccx - s.qx[j], ey = ccy - s.qy[j], ez = ccz - s.qz[j];
          if ((ex * ex + ey * ey) + ez * ez > s.rr[j]) brk |= 1u << j;
        }
      }
      act &= ~brk;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if ((brk >> j) & 1u) thr[j] = -1.0f;
    }
    if (!act) break;
    if ((unsigned)ix >= (unsigned)g.n0 || (unsigned)iy >= (unsigned)g.n1 ||
        (unsigned)iz >= (unsigned)g.n2)
      continue;
    // largest insertion threshold of the points still walking, fixed for
    // this cell (thresholds only shrink, so it stays an upper bound)
    const float thrmax = fmaxf(fmaxf(thr[0], thr[1]), fmaxf(thr[2], thr[3]));
    // ix + iy nx + iz nx ny, in 32 bits (the grid build rejects 2^32 cells or more)
    const uint32_t key = (uint32_t)ix + (uint32_t)g.n0 * ((uint32_t)iy + (uint32_t)g.n1 * (uint32_t)iz);
    const int2 be = __ldg(&g.cells[key]);
    const unsigned na = __popc(act);
    st.cells += na;
    st.cands += na * (uint32_t)max(be.y - be.x, 0);
    if (be.x >= be.y) continue;
    {
      // Every particle of the cell lies in its box (to within the rounding of
      // the cell keys, which g.margin covers). If the box is farther from the
      // points' bounding box than the largest threshold allows, no candidate
      // of the cell can be inserted for any point: the cell is counted as
      // visited, and its scan is skipped.
      const float gx = fmaxf(fmaxf(qlo[0] - (ccx + g.half0), (ccx - g.half0) - qhi[0]) - g.margin,
                             0.0f);
      const float gy = fmaxf(fmaxf(qlo[1] - (ccy + g.half1), (ccy - g.half1) - qhi[1]) - g.margin,
                             0.0f);
      const float gz = fmaxf(fmaxf(qlo[2] - (ccz + g.half2), (ccz - g.half2) - qhi[2]) - g.margin,
                             0.0f);
      if ((gx * gx + gy * gy) + gz * gz > thrmax) continue;
    }
    if (be.y - be.x > kPruneMin) {
      // Dense cell: candidates in ascending index order, 16 codes per chunk.
      // The sub-box mask follows the search radius as it shrinks while the
      // cell is scanned (a mask from a larger radius stays conservative), and
      // once no sub-box is within reach no later candidate of the cell can be
      // inserted.
      float rused = -1.0f;
      unsigned long long m = ~0ull;
      for (int pw = be.x & ~15; pw < be.y; pw += 16) {
        float rmax = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if ((act >> j) & 1u) rmax = fmaxf(rmax, s.R[j]);
        if (rmax != rused) {
          m = prune_mask(g, ix, iy, iz, qlo, qhi, rmax + g.margin);
          rused = rmax;
          if (m == 0ull) break;
        }
        const uint4 w4 = __ldg(reinterpret_cast<const uint4*>(g.codes) + (pw >> 4));
        const uint32_t words[4] = {w4.x, w4.y, w4.z, w4.w};
        unsigned hits = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
          for (int q = 0; q < 4; ++q)
            hits |= (unsigned)((m >> ((words[k] >> (8 * q)) & 63u)) & 1ull) << (4 * k + q);
        if (pw < be.x) hits &= 0xFFFFu << (be.x - pw);
        if (be.y - pw < 16) hits &= 0xFFFFu >> (16 - (be.y - pw));
        while (hits) {
          const int p = pw + __ffs(hits) - 1;
          hits &= hits - 1;
          test_candidate_xy<kSharedXY, kIdx>(s, thr, thrmax, __ldg(&g.parts[p]), p);
        }
      }
      continue;
    }
    float4 P = __ldg(&g.parts[be.x]);
    for (int p = be.x; p < be.y; ++p) {
      const float4 N = (p + 1 < be.y) ? __ldg(&g.parts[p + 1]) : P;  // prefetch
      test_candidate_xy<kSharedXY, kIdx>(s, thr, thrmax, P, p);
      P = N;
    }
  }
}

// Cell index and subcell half (0/1) of a point along one axis
// (volumetric_nn8_reconstruction.cl:129-155, one component).
__device__ __forceinline__ void locate_axis(float q, float mn, float cs, float half, int& c,
                                            int& sh) {
  c = clamp_cell(to_int_sat(floorf((q - mn) / cs)));
  const float m = mn + (float)c * cs;
  const int si = to_int_sat(floorf((q - m) / half));
  sh = min(max(si, 0), 1);
}

// nn8 walk of the 4 points of one step; the slots are left in s.
// kAxis: the caller guarantees lx == ly == 0 (a view along z). Then every
// point's x is px + zq * 0 = px + 0, the same value for the 4 points whatever
// their zq (zq * 0 is +0 for the positive distances along the ray, and NaN
// for all 4 if the step is NaN), so the points share x and y without the
// run-time test and only the shared-x/y walk is compiled.
template <bool kIdx, bool kAxis = false>
__device__ __forceinline__ void nn8_walk_step4(const GridView& g,
                                               const char4* __restrict__ spiral, float px,
                                               float py, float pz, float lx, float ly, float lz,
                                               const float zq[4], Step4& s, WalkStats& st) {
  int cx[4], cy[4], cz[4], sb[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    s.qx[j] = px + zq[kAxis ? 0 : j] * lx;
    s.qy[j] = py + zq[kAxis ? 0 : j] * ly;
    s.qz[j] = pz + zq[j] * lz;
  }
  const bool shared_xy = kAxis || (s.qx[0] == s.qx[1] && s.qx[0] == s.qx[2] &&
                                   s.qx[0] == s.qx[3] && s.qy[0] == s.qy[1] &&
                                   s.qy[0] == s.qy[2] && s.qy[0] == s.qy[3]);
  // points with bit-identical x and y (a view along z) share their x/y cell
  // and subcell: located once
  int cx0, sx0, cy0, sy0;
  locate_axis(s.qx[0], g.min0, g.cs0, g.half0, cx0, sx0);
  locate_axis(s.qy[0], g.min1, g.cs1, g.half1, cy0, sy0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int sx = sx0, sy = sy0, sz;
    cx[j] = cx0;
    cy[j] = cy0;
    if (j > 0 && !shared_xy) {
      locate_axis(s.qx[j], g.min0, g.cs0, g.half0, cx[j], sx);
      locate_axis(s.qy[j], g.min1, g.cs1, g.half1, cy[j], sy);
    }
    locate_axis(s.qz[j], g.min2, g.cs2, g.half2, cz[j], sz);
    sb[j] = sx + 2 * sy + 4 * sz;
  }
  s.crad = g.cell_radius;
  const float empty = kIdx ? __int_as_float(-1) : 0.0f;  // empty slots carry index -1
  s4_init<0>(s, empty);
  s4_init<1>(s, empty);
  s4_init<2>(s, empty);
  s4_init<3>(s, empty);
  unsigned todo = 0xFu;
  while (todo) {
    const int j0 = __ffs(todo) - 1;
    int c0x = cx[0], c0y = cy[0], c0z = cz[0], s0 = sb[0];
#pragma unroll
    for (int j = 1; j < 4; ++j)
      if (j == j0) { c0x = cx[j]; c0y = cy[j]; c0z = cz[j]; s0 = sb[j]; }
    unsigned mask = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (((todo >> j) & 1u) && cx[j] == c0x && cy[j] == c0y && cz[j] == c0z && sb[j] == s0)
        mask |= 1u << j;
    if (shared_xy)
      walk4<true, kIdx>(g, spiral, s, mask, c0x, c0y, c0z, s0, st);
    else
      walk4<false, kIdx>(g, spiral, s, mask, c0x, c0y, c0z, s0, st);
    todo &= ~mask;
  }
}

// nn8 values of the 4 points of one step (e[j] for point j).
__device__ __forceinline__ void nn8_step4(const GridView& g, const char4* __restrict__ spiral,
                                          SlotMem& sm, float px, float py, float pz, float lx,
                                          float ly, float lz, const float zq[4], float e[4],
                                          WalkStats& st) {
  Step4 s;
  s4_bind(s, sm);
  nn8_walk_step4<false>(g, spiral, px, py, pz, lx, ly, lz, zq, s, st);
  e[0] = s4_finalize<0>(s);
  e[1] = s4_finalize<1>(s);
  e[2] = s4_finalize<2>(s);
  e[3] = s4_finalize<3>(s);
}

}  // namespace ilc
