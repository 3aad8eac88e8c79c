// Field kernels of the FELIS slice loop, FP64 plain path (--fmad=false).
//
//  * Ordered source deposit (solveField.cpp:233-312).  The reference adds
//    each particle's bilinear current into ScUx/ScUy one particle after the
//    other, so every cell is a sequential sum in particle order.  Here one
//    CTA owns one slice: it sorts the slice's (cell, particle) keys in shared
//    memory (bitonic, 32-bit composite keys), then one thread per target cell
//    merges the four source buckets (cells t, t-1, t-nx, t-nx-1) by particle
//    index and accumulates in exactly that order.  No float atomics; the
//    result equals the sequential CPU sum bit for bit.
//  * Ez space charge (solveField.cpp:315-399) the same way over radial bins,
//    followed by the per-slice Thomas solve in r.
//  * ADI (solveField.cpp:80-185).  One CTA owns one (slice, harmonic,
//    polarisation) plane.  The x sweep runs one thread per row with the
//    forward elimination stored in a shared-memory plane, the back
//    substitution overwrites it with Uc; the y sweep runs one thread per
//    column on that plane and writes U back to HBM coalesced.  The
//    data-independent recurrence coefficients (CC) are host tables.
#include "field.cuh"
#include "bulk.cuh"

namespace felis {

namespace {

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)((blockDim.x + 31) >> 5); ++k) t += red[k];
  return t;
}

// First index in s[0, n) with s[idx] >= v (s sorted ascending).
__device__ __forceinline__ int lower_bound_u32(const uint32_t* s, int n, uint32_t v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Maps a slice-local deposit index q (species-major) to the global particle index.
__device__ __forceinline__ int64_t q_to_n(const DepositLaunch& a, int s, uint32_t q) {
  const int S = a.G.S;
  for (int sp = 0; sp < a.G.nspecies; ++sp) {
    const int64_t b = a.soff[(size_t)sp * (S + 1) + s], e = a.soff[(size_t)sp * (S + 1) + s + 1];
    if ((int64_t)q < e - b) return b + q;
    q -= (uint32_t)(e - b);
  }
  return -1;
}

// Stable LSD radix sort (4-bit digits) of n <= C packed items held in a[]
// (the key in the high bits above `qb` index bits), NT threads in a blocked
// arrangement.  cnt[16*NT] u16 scratch; result left in a[] (b[] is the
// ping-pong buffer).  Equal keys keep their input order.
template <int NT>
__device__ void block_radix_sort(uint32_t* a, uint32_t* b, int n, int qb, int nbits, uint16_t* cnt, uint32_t* wsum) {
  const int t = threadIdx.x;
  const int K = (n + NT - 1) / NT;
  const int i0 = t * K, i1 = min(n, i0 + K);
  uint32_t* src = a;
  uint32_t* dst = b;
  for (int shift = 0; shift < nbits; shift += 4) {
    for (int d = 0; d < 16; ++d) cnt[d * NT + t] = 0;
    for (int i = i0; i < i1; ++i) cnt[((src[i] >> (qb + shift)) & 15u) * NT + t] += 1;
    __syncthreads();
    // exclusive scan of cnt (digit-major): thread t owns entries [16t, 16t+16)
    uint32_t run = 0;
    uint16_t loc[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) { loc[k] = cnt[16 * t + k]; run += loc[k]; }
    uint32_t incl = run;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if ((t & 31) >= o) incl += v;
    }
    if ((t & 31) == 31) wsum[t >> 5] = incl;
    __syncthreads();
    if (t == 0) {
      uint32_t acc = 0;
      for (int w = 0; w < NT / 32; ++w) { const uint32_t v = wsum[w]; wsum[w] = acc; acc += v; }
    }
    __syncthreads();
    uint32_t pre = wsum[t >> 5] + incl - run;
#pragma unroll
    for (int k = 0; k < 16; ++k) { const uint32_t v = loc[k]; cnt[16 * t + k] = (uint16_t)pre; pre += v; }
    __syncthreads();
    for (int i = i0; i < i1; ++i) {
      const uint32_t v = src[i];
      const int d = (int)((v >> (qb + shift)) & 15u);
      const uint16_t pos = cnt[d * NT + t];
      cnt[d * NT + t] = pos + 1;
      dst[pos] = v;
    }
    __syncthreads();
    uint32_t* tmp = src; src = dst; dst = tmp;
  }
  if (src != a) {
    for (int i = t; i < n; i += NT) a[i] = src[i];
    __syncthreads();
  }
}

// Shared-memory layout of one deposit CTA (one chunk of C particles at a
// time): sort buffers A, B (u32[C] each), digit counters u16[16*512],
// 2-D records {wx1, wy1, coef[H], fx/fy[even H]} in sorted order, or the
// radial chain terms double2[2C][L*F]; radial bin starts and chain starts;
// radial accumulators and the Thomas diagonal.
struct DepLayout {
  int C, qb;
  size_t A, B, cnt, wsum, wx, wy, coef, fx, fy, rterm, bstart, cstart, bins, bmod, total;
};

__host__ __device__ inline int ilog2_ceil(int v) {
  int b = 0;
  while ((1 << b) < v) ++b;
  return b;
}

__host__ __device__ inline DepLayout dep_layout(int C, int H, int neven, int LF, int nr) {
  DepLayout L;
  L.C = C;
  L.qb = ilog2_ceil(C);
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t r = o; o += (bytes + 15) & ~(size_t)15; return r; };
  L.A = take((size_t)C * 4);
  L.B = take((size_t)C * 4);
  L.cnt = take((size_t)16 * 512 * 2);
  L.wsum = take(16 * 4);
  const size_t rec = o;
  L.wx = take((size_t)C * 8);
  L.wy = take((size_t)C * 8);
  L.coef = take((size_t)C * 16 * H);
  L.fx = take((size_t)C * 16 * neven);
  L.fy = take((size_t)C * 16 * neven);
  const size_t rec_end = o;
  o = rec;
  L.rterm = take((size_t)2 * C * 16 * LF);
  if (o < rec_end) o = rec_end;
  L.bstart = take((size_t)(nr + 2) * 4);
  L.cstart = take((size_t)(nr + 2) * 4);
  L.bins = take((size_t)LF * nr * 16);
  L.bmod = take((size_t)LF * nr * 8);
  L.total = o;
  return L;
}

__global__ void __launch_bounds__(512) k_deposit(DepositLaunch a) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ int red_i[4][16];
  __shared__ int sbox[4];
  const DevGeom& G = a.G;
  const int s = blockIdx.x;
  const int S = G.S, nx = G.nx, ny = G.ny, N = G.N, H = G.H;
  const int nr = G.nr, LFn = G.L * G.F;
  const DepLayout Ly = dep_layout(a.cap, H, a.neven, LFn, nr);
  const int CH = Ly.C, qb = Ly.qb;
  const uint32_t qmask = (1u << qb) - 1u;
  uint32_t* A = reinterpret_cast<uint32_t*>(dsm + Ly.A);
  uint32_t* Bf = reinterpret_cast<uint32_t*>(dsm + Ly.B);
  uint16_t* cnt = reinterpret_cast<uint16_t*>(dsm + Ly.cnt);
  uint32_t* wsum = reinterpret_cast<uint32_t*>(dsm + Ly.wsum);
  double* rwx = reinterpret_cast<double*>(dsm + Ly.wx);
  double* rwy = reinterpret_cast<double*>(dsm + Ly.wy);
  double2* rcoef = reinterpret_cast<double2*>(dsm + Ly.coef);
  double2* rfx = reinterpret_cast<double2*>(dsm + Ly.fx);
  double2* rfy = reinterpret_cast<double2*>(dsm + Ly.fy);
  double2* rterm = reinterpret_cast<double2*>(dsm + Ly.rterm);
  int* bstart = reinterpret_cast<int*>(dsm + Ly.bstart);
  int* cstart = reinterpret_cast<int*>(dsm + Ly.cstart);
  double2* dbin = reinterpret_cast<double2*>(dsm + Ly.bins);
  double* bmod = reinterpret_cast<double*>(dsm + Ly.bmod);
  const size_t tot = (size_t)a.total;
  // key bits: 2-D cells (plus one invalid value) and radial bins
  const int kbits2 = ilog2_ceil(N + 1), kbitsr = ilog2_ceil(nr + 1);
  const uint32_t inval2 = (1u << kbits2) - 1u, invalr = (1u << kbitsr) - 1u;
  // ---- slice particle count (all species) ----
  int64_t Pt = 0, Plast0 = 0, Plast = 0;
  for (int sp = 0; sp < G.nspecies; ++sp) {
    const int64_t b = a.soff[(size_t)sp * (S + 1) + s], e = a.soff[(size_t)sp * (S + 1) + s + 1];
    if (sp == G.nspecies - 1) { Plast0 = Pt; Plast = e - b; }
    Pt += e - b;
  }
  // ---- box of reachable interior cells over the whole slice ----
  {
    int cmin_i = 1 << 30, cmax_i = -1, cmin_j = 1 << 30, cmax_j = -1;
    for (int64_t q = threadIdx.x; q < Pt; q += blockDim.x) {
      const int k = a.dep.key[q_to_n(a, s, (uint32_t)q)];
      if (k >= 0) {
        const int ki = k % nx, kj = k / nx;
        cmin_i = min(cmin_i, ki); cmax_i = max(cmax_i, ki);
        cmin_j = min(cmin_j, kj); cmax_j = max(cmax_j, kj);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      cmin_i = min(cmin_i, __shfl_down_sync(0xffffffffu, cmin_i, o));
      cmax_i = max(cmax_i, __shfl_down_sync(0xffffffffu, cmax_i, o));
      cmin_j = min(cmin_j, __shfl_down_sync(0xffffffffu, cmin_j, o));
      cmax_j = max(cmax_j, __shfl_down_sync(0xffffffffu, cmax_j, o));
    }
    if ((threadIdx.x & 31) == 0) {
      const int w = threadIdx.x >> 5;
      red_i[0][w] = cmin_i; red_i[1][w] = cmax_i; red_i[2][w] = cmin_j; red_i[3][w] = cmax_j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int i0 = 1 << 30, i1 = -1, j0 = 1 << 30, j1 = -1;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        i0 = min(i0, red_i[0][w]); i1 = max(i1, red_i[1][w]);
        j0 = min(j0, red_i[2][w]); j1 = max(j1, red_i[3][w]);
      }
      const int ti0 = max(1, i0), ti1 = min(nx - 2, i1 + 1), tj0 = max(1, j0), tj1 = min(ny - 2, j1 + 1);
      const bool any = i1 >= 0 && ti0 <= ti1 && tj0 <= tj1;
      sbox[0] = any ? ti0 : 1; sbox[1] = any ? ti1 : 0; sbox[2] = any ? tj0 : 1; sbox[3] = any ? tj1 : 0;
      a.box[s] = make_int4(sbox[0], sbox[1], sbox[2], sbox[3]);
    }
    __syncthreads();
  }
  const int bi0 = sbox[0], bi1 = sbox[1], bj0 = sbox[2], bj1 = sbox[3];
  const int bw = bi1 - bi0 + 1, bh = bj1 - bj0 + 1;
  if (bw > 0 && bh > 0)
    for (int c = threadIdx.x; c < bw * bh; c += blockDim.x) {
      const int t = (bj0 + c / bw) * nx + bi0 + c % bw;
      for (int h = 0; h < H; ++h) {
        a.Sc[(((size_t)h * 2 + 0) * S + s) * N + t] = make_double2(0.0, 0.0);
        a.Sc[(((size_t)h * 2 + 1) * S + s) * N + t] = make_double2(0.0, 0.0);
      }
    }
  __syncthreads();
  // ---- phase A: 2-D source, chunk by chunk in particle order ----
  for (int64_t c0 = 0; c0 < Pt && bw > 0 && bh > 0; c0 += CH) {
    const int nc = (int)((Pt - c0) < CH ? (Pt - c0) : CH);
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
      const int k = a.dep.key[q_to_n(a, s, (uint32_t)(c0 + q))];
      A[q] = ((k >= 0 ? (uint32_t)k : inval2) << qb) | (uint32_t)q;
    }
    __syncthreads();
    block_radix_sort<512>(A, Bf, nc, qb, kbits2, cnt, wsum);
    const int V = lower_bound_u32(A, nc, inval2 << qb);
    // records of the chunk, in sorted order
    for (int pos = threadIdx.x; pos < V; pos += blockDim.x) {
      const int64_t n = q_to_n(a, s, (uint32_t)(c0 + (A[pos] & qmask)));
      rwx[pos] = a.dep.wx1[n];
      rwy[pos] = a.dep.wy1[n];
      int e = 0;
      for (int h = 0; h < H; ++h) {
        rcoef[(size_t)h * CH + pos] = a.dep.coef[(size_t)h * tot + n];
        if (G.harmony[h] % 2 == 0) {
          rfx[(size_t)e * CH + pos] = a.dep.fx[(size_t)h * tot + n];
          rfy[(size_t)e * CH + pos] = a.dep.fy[(size_t)h * tot + n];
          ++e;
        }
      }
    }
    __syncthreads();
    if (V > 0) {
      const int kfirst = (int)(A[0] >> qb), klast = (int)(A[V - 1] >> qb);
      const int rj0 = max(bj0, kfirst / nx), rj1 = min(bj1, klast / nx + 1);
      const int rh = rj1 - rj0 + 1;
      for (int c = threadIdx.x; c < bw * max(rh, 0); c += blockDim.x) {
        const int ti = bi0 + c % bw, tj = rj0 + c / bw;
        const int t = tj * nx + ti;
        int lo[4], hi[4];
        bool any = false;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
          const int k = t - (cb >> 1) * nx - (cb & 1);
          lo[cb] = lower_bound_u32(A, V, (uint32_t)k << qb);
          hi[cb] = lower_bound_u32(A, V, (uint32_t)(k + 1) << qb);
          any |= lo[cb] < hi[cb];
        }
        if (!any) continue;
        cd accx[FELIS_MAX_HARMONY], accy[FELIS_MAX_HARMONY];
        for (int h = 0; h < H; ++h) {
          const double2 vx = a.Sc[(((size_t)h * 2 + 0) * S + s) * N + t];
          const double2 vy = a.Sc[(((size_t)h * 2 + 1) * S + s) * N + t];
          accx[h] = C(vx.x, vx.y);
          accy[h] = C(vy.x, vy.y);
        }
        uint32_t head[4];
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) head[cb] = lo[cb] < hi[cb] ? (A[lo[cb]] & qmask) : 0xFFFFFFFFu;
        while (true) {
          int best = 0;
          uint32_t bq = head[0];
#pragma unroll
          for (int cb = 1; cb < 4; ++cb)
            if (head[cb] < bq) { bq = head[cb]; best = cb; }
          if (bq == 0xFFFFFFFFu) break;
          const int pos = lo[best]++;
          head[best] = lo[best] < hi[best] ? (A[lo[best]] & qmask) : 0xFFFFFFFFu;
          const int ii = best & 1, jj = best >> 1;
          const double wx1 = rwx[pos], wy1 = rwy[pos];
          const double wxv = ii ? wx1 : 1.0 - wx1;
          const double wyv = jj ? wy1 : 1.0 - wy1;
          const cd ex = cscale(cscale(a.etaX, wxv), wyv);
          const cd ey = cscale(cscale(a.etaY, wxv), wyv);
          int e = 0;
          for (int h = 0; h < H; ++h) {
            const double2 m = rcoef[(size_t)h * CH + pos];
            const cd mc = C(m.x, m.y);
            cd fx, fy;
            if (G.harmony[h] % 2 == 1) {
              fx = C(a.fconst[h][0].x, a.fconst[h][0].y);
              fy = C(a.fconst[h][1].x, a.fconst[h][1].y);
            } else {
              const double2 v1 = rfx[(size_t)e * CH + pos], v2 = rfy[(size_t)e * CH + pos];
              fx = C(v1.x, v1.y);
              fy = C(v2.x, v2.y);
              ++e;
            }
            accx[h] = csub(accx[h], cmul(cmul(ex, fx), mc));
            accy[h] = csub(accy[h], cmul(cmul(ey, fy), mc));
          }
        }
        for (int h = 0; h < H; ++h) {
          a.Sc[(((size_t)h * 2 + 0) * S + s) * N + t] = make_double2(accx[h].re, accx[h].im);
          a.Sc[(((size_t)h * 2 + 1) * S + s) * N + t] = make_double2(accy[h].re, accy[h].im);
        }
      }
    }
    __syncthreads();
  }
  // ---- phase B: Ez of the last species (solveField.cpp:315-399) ----
  for (int idx = threadIdx.x; idx < LFn * nr; idx += blockDim.x) dbin[idx] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int64_t c0 = 0; c0 < Plast; c0 += CH) {
    const int nc = (int)((Plast - c0) < CH ? (Plast - c0) : CH);
    for (int q = threadIdx.x; q < nc; q += blockDim.x) {
      const int rk = a.dep.rkey[q_to_n(a, s, (uint32_t)(Plast0 + c0 + q))];
      A[q] = ((rk >= 0 ? (uint32_t)rk : invalr) << qb) | (uint32_t)q;
    }
    __syncthreads();
    block_radix_sort<512>(A, Bf, nc, qb, kbitsr, cnt, wsum);
    const int V = lower_bound_u32(A, nc, invalr << qb);
    // bucket starts per bin (bstart[nr] = V) and chain starts: bin b's chain
    // merges bucket b (weight wr0) and bucket b-1 (weight wr1) by particle
    for (int b = threadIdx.x; b <= nr; b += blockDim.x) bstart[b] = lower_bound_u32(A, V, (uint32_t)b << qb);
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int b = 0; b <= nr - 2; ++b) {
        cstart[b] = acc;
        int len = bstart[b + 1] - bstart[b];
        if (b >= 2) len += bstart[b] - bstart[b - 1];
        acc += len;
      }
      cstart[nr - 1] = acc;
    }
    __syncthreads();
    // every (particle, bin) term at its place in the bin's chain
    for (int pos = threadIdx.x; pos < V; pos += blockDim.x) {
      const uint32_t it = A[pos];
      const int rk = (int)(it >> qb);
      const uint32_t q = it & qmask;
      const int64_t n = q_to_n(a, s, (uint32_t)(Plast0 + c0 + q));
      const double wr1 = a.dep.wr1[n];
      const int rank = pos - bstart[rk];
      for (int jj = 0; jj < 2; ++jj) {
        const int b = rk + jj;
        if (b > nr - 2 || (rk == 0 && jj == 1)) continue;
        // the other bucket of chain b: b-1 (for jj = 0, b >= 2) or b (for jj = 1)
        int other = 0;
        if (jj == 0 && b >= 2) other = lower_bound_u32(A + bstart[b - 1], bstart[b] - bstart[b - 1], ((uint32_t)(b - 1) << qb) | q);
        if (jj == 1) other = lower_bound_u32(A + bstart[b], bstart[b + 1] - bstart[b], ((uint32_t)b << qb) | q);
        const int slot = cstart[b] + rank + other;
        for (int lf = 0; lf < LFn; ++lf) {
          const double2 v = a.dep.ez[(size_t)lf * tot + n];
          double2 tt;
          if (b == 0) tt = v;  // idxR == 0 branch: no radial weight
          else {
            const double w = jj ? wr1 : 1.0 - wr1;
            tt = make_double2(v.x * w, v.y * w);
          }
          rterm[(size_t)slot * LFn + lf] = tt;
        }
      }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < LFn * (nr - 1); idx += blockDim.x) {
      const int lf = idx / (nr - 1), b = idx % (nr - 1);
      if (b == 0 && (lf % G.F) > 0) continue;  // bin 0 of f > 0 stays zero
      const int k0 = cstart[b], k1 = cstart[b + 1];
      if (k0 == k1) continue;
      double2 acc = dbin[(size_t)lf * nr + b];
      for (int k = k0; k < k1; ++k) {
        const double2 tt = rterm[(size_t)k * LFn + lf];
        acc.x = acc.x + tt.x;
        acc.y = acc.y + tt.y;
      }
      dbin[(size_t)lf * nr + b] = acc;
    }
    __syncthreads();
  }
  // Thomas solve in r, one thread per (l, f)
  if ((int)threadIdx.x < LFn) {
    const int lf = threadIdx.x, l = lf / G.F, f = lf % G.F;
    const double Acoef = a.A;
    double2* d = dbin + lf * nr;
    auto acoef = [&](int j) -> double { return (j == 0) ? (f == 0 ? 1.0 : 0.0) : (j == nr - 1 ? 0.0 : j + 0.5); };
    auto ccoef = [&](int j) -> double { return (j == 0 || j == nr - 1) ? 0.0 : j - 0.5; };
    double* bm = bmod + (size_t)lf * nr;
    double bprev;
    if (f == 0) bprev = -(1.0 + (l + 1.0) * (l + 1.0) * Acoef / 8.0);
    else { bprev = 1.0; d[0] = make_double2(0.0, 0.0); }
    bm[0] = bprev;
    for (int j = 1; j < nr; ++j) {
      double bj = (j == nr - 1) ? 1.0 : -2.0 * j - (l + 1.0) * (l + 1.0) * Acoef * j - f * f * G.logtab[j];
      const double ww = ccoef(j) / bprev;
      bj -= ww * acoef(j - 1);
      cd dj = (j == nr - 1) ? C(0, 0) : C(d[j].x, d[j].y);
      const cd dp = C(d[j - 1].x, d[j - 1].y);
      dj = csub(dj, cscale(dp, ww));
      d[j] = make_double2(dj.re, dj.im);
      bm[j] = bj;
      bprev = bj;
    }
    const size_t ezs = (size_t)(S + 2) * nr * G.F;
    const int sliceI = s + 1;
    for (int j = nr - 2; j >= 0; --j) {
      const cd dj = C(d[j].x, d[j].y);
      const cd r = cdivr(csub(dj, cscale(C(0.0, 0.0), acoef(j))), bm[j]);
      a.Ez[(size_t)l * ezs + (size_t)sliceI * G.F * nr + (size_t)f * nr + j] = make_double2(r.re, r.im);
    }
  }
}

// ---- ADI -------------------------------------------------------------------
__global__ void __launch_bounds__(256, 1) k_adi(AdiLaunch a) {
  extern __shared__ double2 Apl[];  // ny rows of nxp complex, then the recurrence tables
  __shared__ double red[8];
  const DevGeom& G = a.G;
  const int S = G.S, nx = G.nx, ny = G.ny, N = G.N, nxp = a.nxp;
  const int s = blockIdx.x % S;
  const int hp = blockIdx.x / S;  // h*2 + pol
  const int h = hp >> 1, pol = hp & 1;
  const AdiTab Tg = a.tab[h];
  // recurrence coefficients of this harmonic, read at every step: shared memory
  cd* tx = reinterpret_cast<cd*>(Apl + (size_t)ny * nxp);   // ax_p, ax_a, ax_q, ax_cc [nx each]
  cd* ty = tx + 4 * nx;                                     // ay_p, ay_a, ay_q, ay_cc [ny each]
  double* dx_ = reinterpret_cast<double*>(ty + 4 * ny);     // ax_pinv, ax_qinv, ax_ccinv [nx each]
  double* dy_ = dx_ + 3 * nx;                               // ay_*inv [ny each]
  for (int k = threadIdx.x; k < nx; k += blockDim.x) {
    tx[k] = Tg.ax_p[k]; tx[nx + k] = Tg.ax_a[k]; tx[2 * nx + k] = Tg.ax_q[k]; tx[3 * nx + k] = Tg.ax_cc[k];
    dx_[k] = Tg.ax_pinv[k]; dx_[nx + k] = Tg.ax_qinv[k]; dx_[2 * nx + k] = Tg.ax_ccinv[k];
  }
  for (int k = threadIdx.x; k < ny; k += blockDim.x) {
    ty[k] = Tg.ay_p[k]; ty[ny + k] = Tg.ay_a[k]; ty[2 * ny + k] = Tg.ay_q[k]; ty[3 * ny + k] = Tg.ay_cc[k];
    dy_[k] = Tg.ay_pinv[k]; dy_[ny + k] = Tg.ay_qinv[k]; dy_[2 * ny + k] = Tg.ay_ccinv[k];
  }
  AdiTab T = Tg;
  T.ax_p = tx; T.ax_a = tx + nx; T.ax_q = tx + 2 * nx; T.ax_cc = tx + 3 * nx;
  T.ax_pinv = dx_; T.ax_qinv = dx_ + nx; T.ax_ccinv = dx_ + 2 * nx;
  T.ay_p = ty; T.ay_a = ty + ny; T.ay_q = ty + 2 * ny; T.ay_cc = ty + 3 * ny;
  T.ay_pinv = dy_; T.ay_qinv = dy_ + ny; T.ay_ccinv = dy_ + 2 * ny;
  double2* U = a.U + field_plane(S, h, pol, s, a.ring_base) * N;
  const double2* Sc = a.Sc + ((size_t)hp * S + s) * N;
  const int4 bx = a.box[s];
  const bool src = a.use_source != 0;
  const int tid = threadIdx.x;
  // ---- stage the plane: one bulk copy per row (rows of complex FP64 start on
  // 16-byte boundaries in global and in shared memory) ----
  __shared__ __align__(8) unsigned long long pbar;
  if (tid == 0) bar_init_tx(smem_u32(&pbar), (unsigned)((size_t)N * sizeof(double2)));
  __syncthreads();
  for (int r = tid; r < ny; r += blockDim.x)
    bulk_g2s(Apl + (size_t)r * nxp, U + (size_t)r * nx, (unsigned)(nx * sizeof(double2)), smem_u32(&pbar));
  if (!bar_wait0(smem_u32(&pbar), kBulkWaitTries)) {
    set_flag(a.err, ERR_TIMEOUT);
    bar_wait0(smem_u32(&pbar), kBulkWaitTries);  // once more for the copies in flight
  }
  __syncthreads();
  // ---- x sweep: thread per row j; one barrier per column so that every row
  // has read column i of U before any row overwrites it with DD ----
  const int j = tid;
  const bool row = j >= 1 && j <= ny - 2;
  {
    cd rm = C(0, 0), r0 = C(0, 0), rp = C(0, 0);
    if (row) { rm = T.rx_m[j]; r0 = T.rx_0[j]; rp = T.rx_p[j]; }
    const bool rowin = row && src && j >= bx.z && j <= bx.w;
    cd DD = C(0, 0);
    for (int i = 1; i <= nx - 2; ++i) {
      double2 up = make_double2(0, 0), u0 = up, um = up, sv = up;
      if (row) {
        up = Apl[(j + 1) * nxp + i]; u0 = Apl[j * nxp + i]; um = Apl[(j - 1) * nxp + i];
        if (rowin && i >= bx.x && i <= bx.y) sv = Sc[j * nx + i];
      }
      __syncthreads();
      if (row) {
        cd t = cmul(rm, C(up.x, up.y));
        t = cadd(t, cmul(r0, C(u0.x, u0.y)));
        t = csub(t, cmul(rp, C(um.x, um.y)));
        if (rowin && i >= bx.x && i <= bx.y) t = cadd(t, C(sv.x, sv.y));
        if (i == 1) {
          DD = cdiv_inv(t, T.ax_p[1], T.ax_pinv[1]);
        } else if (i < nx - 2) {
          DD = csub(cdiv_inv(t, T.ax_p[i], T.ax_pinv[i]), cdiv_inv(cmul(T.ax_a[i], DD), T.ax_q[i], T.ax_qinv[i]));
        } else {
          DD = csub(t, cdiv_inv(DD, T.ax_cc[nx - 3], T.ax_ccinv[nx - 3]));
        }
        Apl[j * nxp + i] = make_double2(DD.re, DD.im);
      }
    }
    if (row) {
      cd Uc = cdiv_inv(DD, T.ax_cc[nx - 2], T.ax_ccinv[nx - 2]);
      Apl[j * nxp + nx - 2] = make_double2(Uc.re, Uc.im);
      for (int i = nx - 3; i > 0; --i) {
        const double2 d = Apl[j * nxp + i];
        Uc = cdiv_inv(csub(C(d.x, d.y), Uc), T.ax_cc[i], T.ax_ccinv[i]);
        Apl[j * nxp + i] = make_double2(Uc.re, Uc.im);
      }
      Apl[j * nxp + 0] = make_double2(0.0, 0.0);
      Apl[j * nxp + nx - 1] = make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  // ---- y sweep: thread per column i, one barrier per row ----
  const int i = tid;
  const bool col = i >= 1 && i <= nx - 2;
  cd rm = C(0, 0), r0 = C(0, 0), rp = C(0, 0);
  if (col) { rm = T.ry_m[i]; r0 = T.ry_0[i]; rp = T.ry_p[i]; }
  const bool colin = col && src && i >= bx.x && i <= bx.y;
  cd DD = C(0, 0);
  for (int jr = 1; jr <= ny - 2; ++jr) {
    double2 up = make_double2(0, 0), u0 = up, um = up, sv = up;
    if (col) {
      up = Apl[jr * nxp + i + 1]; u0 = Apl[jr * nxp + i]; um = Apl[jr * nxp + i - 1];
      if (colin && jr >= bx.z && jr <= bx.w) sv = Sc[jr * nx + i];
    }
    __syncthreads();
    if (col) {
      cd t = cmul(rm, C(up.x, up.y));
      t = cadd(t, cmul(r0, C(u0.x, u0.y)));
      t = csub(t, cmul(rp, C(um.x, um.y)));
      if (colin && jr >= bx.z && jr <= bx.w) t = cadd(t, C(sv.x, sv.y));
      if (jr == 1) {
        DD = cdiv_inv(t, T.ay_p[1], T.ay_pinv[1]);
      } else if (jr < ny - 2) {
        DD = csub(cdiv_inv(t, T.ay_p[jr], T.ay_pinv[jr]), cdiv_inv(cmul(T.ay_a[jr], DD), T.ay_q[jr], T.ay_qinv[jr]));
      } else {
        DD = csub(t, cdiv_inv(DD, T.ay_cc[ny - 3], T.ay_ccinv[ny - 3]));
      }
      Apl[jr * nxp + i] = make_double2(DD.re, DD.im);
    }
  }
  if (col) {
    cd Un = cdiv_inv(DD, T.ay_cc[ny - 2], T.ay_ccinv[ny - 2]);
    Apl[(ny - 2) * nxp + i] = make_double2(Un.re, Un.im);
    for (int jr = ny - 3; jr > 0; --jr) {
      const double2 d = Apl[jr * nxp + i];
      Un = cdiv_inv(csub(C(d.x, d.y), Un), T.ay_cc[jr], T.ay_ccinv[jr]);
      Apl[jr * nxp + i] = make_double2(Un.re, Un.im);
    }
  }
  __syncthreads();
  // ---- write the interior back (coalesced) and sum |U|^2 over the plane;
  // edge columns keep their old values (the ADI never writes them) ----
  double e = 0.0;
  for (int k = tid; k < N; k += blockDim.x) {
    const int jj = k / nx, ii = k % nx;
    double2 v;
    if (jj >= 1 && jj <= ny - 2 && ii >= 1 && ii <= nx - 2) {
      v = Apl[jj * nxp + ii];
      U[k] = v;
    } else if (jj == 0 || jj == ny - 1) {
      v = Apl[jj * nxp + ii];
    } else {
      v = U[k];
    }
    e += v.x * v.x + v.y * v.y;
  }
  if (a.energy) {
    const double t = block_sum(e, red);
    if (tid == 0) a.energy[(size_t)hp * S + s] = t;
  }
}

// ADI of planes too large for shared memory: the same arithmetic in the same
// order as k_adi, with the plane in global memory.  The x sweep writes its
// result to a per-CTA scratch plane X (so the rows never wait for one another)
// and the y sweep reads X and writes U in place; one CTA per plane, planes
// taken in a grid-stride loop.
__global__ void __launch_bounds__(256) k_adi_big(AdiLaunch a) {
  extern __shared__ double2 Atb[];  // recurrence tables of the harmonic
  __shared__ double red[8];
  const DevGeom& G = a.G;
  const int S = G.S, nx = G.nx, ny = G.ny, N = G.N;
  const int tid = threadIdx.x;
  double2* X = a.scratch + (size_t)blockIdx.x * N;
  cd* tx = reinterpret_cast<cd*>(Atb);
  cd* ty = tx + 4 * nx;
  double* dx_ = reinterpret_cast<double*>(ty + 4 * ny);
  double* dy_ = dx_ + 3 * nx;
  int staged_h = -1;
  for (int plane = blockIdx.x; plane < S * G.H * 2; plane += gridDim.x) {
    const int s = plane % S, hp = plane / S, h = hp >> 1, pol = hp & 1;
    const AdiTab Tg = a.tab[h];
    if (h != staged_h) {
      __syncthreads();
      for (int k = tid; k < nx; k += blockDim.x) {
        tx[k] = Tg.ax_p[k]; tx[nx + k] = Tg.ax_a[k]; tx[2 * nx + k] = Tg.ax_q[k]; tx[3 * nx + k] = Tg.ax_cc[k];
        dx_[k] = Tg.ax_pinv[k]; dx_[nx + k] = Tg.ax_qinv[k]; dx_[2 * nx + k] = Tg.ax_ccinv[k];
      }
      for (int k = tid; k < ny; k += blockDim.x) {
        ty[k] = Tg.ay_p[k]; ty[ny + k] = Tg.ay_a[k]; ty[2 * ny + k] = Tg.ay_q[k]; ty[3 * ny + k] = Tg.ay_cc[k];
        dy_[k] = Tg.ay_pinv[k]; dy_[ny + k] = Tg.ay_qinv[k]; dy_[2 * ny + k] = Tg.ay_ccinv[k];
      }
      staged_h = h;
      __syncthreads();
    }
    AdiTab T = Tg;
    T.ax_p = tx; T.ax_a = tx + nx; T.ax_q = tx + 2 * nx; T.ax_cc = tx + 3 * nx;
    T.ax_pinv = dx_; T.ax_qinv = dx_ + nx; T.ax_ccinv = dx_ + 2 * nx;
    T.ay_p = ty; T.ay_a = ty + ny; T.ay_q = ty + 2 * ny; T.ay_cc = ty + 3 * ny;
    T.ay_pinv = dy_; T.ay_qinv = dy_ + ny; T.ay_ccinv = dy_ + 2 * ny;
    double2* U = a.U + field_plane(S, h, pol, s, a.ring_base) * N;
    const double2* Sc = a.Sc + ((size_t)hp * S + s) * N;
    const int4 bx = a.box[s];
    const bool src = a.use_source != 0;
    // ---- x sweep: thread per row j, result in X ----
    const int j = tid;
    if (j >= 1 && j <= ny - 2) {
      const cd rm = T.rx_m[j], r0 = T.rx_0[j], rp = T.rx_p[j];
      const bool rowin = src && j >= bx.z && j <= bx.w;
      cd DD = C(0, 0);
      for (int i = 1; i <= nx - 2; ++i) {
        const double2 up = U[(j + 1) * nx + i], u0 = U[j * nx + i], um = U[(j - 1) * nx + i];
        cd t = cmul(rm, C(up.x, up.y));
        t = cadd(t, cmul(r0, C(u0.x, u0.y)));
        t = csub(t, cmul(rp, C(um.x, um.y)));
        if (rowin && i >= bx.x && i <= bx.y) {
          const double2 sv = Sc[j * nx + i];
          t = cadd(t, C(sv.x, sv.y));
        }
        if (i == 1) {
          DD = cdiv_inv(t, T.ax_p[1], T.ax_pinv[1]);
        } else if (i < nx - 2) {
          DD = csub(cdiv_inv(t, T.ax_p[i], T.ax_pinv[i]), cdiv_inv(cmul(T.ax_a[i], DD), T.ax_q[i], T.ax_qinv[i]));
        } else {
          DD = csub(t, cdiv_inv(DD, T.ax_cc[nx - 3], T.ax_ccinv[nx - 3]));
        }
        X[j * nx + i] = make_double2(DD.re, DD.im);
      }
      cd Uc = cdiv_inv(DD, T.ax_cc[nx - 2], T.ax_ccinv[nx - 2]);
      X[j * nx + nx - 2] = make_double2(Uc.re, Uc.im);
      for (int i = nx - 3; i > 0; --i) {
        const double2 d = X[j * nx + i];
        Uc = cdiv_inv(csub(C(d.x, d.y), Uc), T.ax_cc[i], T.ax_ccinv[i]);
        X[j * nx + i] = make_double2(Uc.re, Uc.im);
      }
      X[j * nx + 0] = make_double2(0.0, 0.0);
      X[j * nx + nx - 1] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    // ---- y sweep: thread per column i, reads X, writes U in place ----
    const int i = tid;
    if (i >= 1 && i <= nx - 2) {
      const cd rm = T.ry_m[i], r0 = T.ry_0[i], rp = T.ry_p[i];
      const bool colin = src && i >= bx.x && i <= bx.y;
      cd DD = C(0, 0);
      for (int jr = 1; jr <= ny - 2; ++jr) {
        const double2 up = X[jr * nx + i + 1], u0 = X[jr * nx + i], um = X[jr * nx + i - 1];
        cd t = cmul(rm, C(up.x, up.y));
        t = cadd(t, cmul(r0, C(u0.x, u0.y)));
        t = csub(t, cmul(rp, C(um.x, um.y)));
        if (colin && jr >= bx.z && jr <= bx.w) {
          const double2 sv = Sc[jr * nx + i];
          t = cadd(t, C(sv.x, sv.y));
        }
        if (jr == 1) {
          DD = cdiv_inv(t, T.ay_p[1], T.ay_pinv[1]);
        } else if (jr < ny - 2) {
          DD = csub(cdiv_inv(t, T.ay_p[jr], T.ay_pinv[jr]), cdiv_inv(cmul(T.ay_a[jr], DD), T.ay_q[jr], T.ay_qinv[jr]));
        } else {
          DD = csub(t, cdiv_inv(DD, T.ay_cc[ny - 3], T.ay_ccinv[ny - 3]));
        }
        U[jr * nx + i] = make_double2(DD.re, DD.im);
      }
      cd Un = cdiv_inv(DD, T.ay_cc[ny - 2], T.ay_ccinv[ny - 2]);
      U[(ny - 2) * nx + i] = make_double2(Un.re, Un.im);
      for (int jr = ny - 3; jr > 0; --jr) {
        const double2 d = U[jr * nx + i];
        Un = cdiv_inv(csub(C(d.x, d.y), Un), T.ay_cc[jr], T.ay_ccinv[jr]);
        U[jr * nx + i] = make_double2(Un.re, Un.im);
      }
    }
    __syncthreads();
    // ---- |U|^2 over the plane (edge rows and columns keep their values) ----
    double e = 0.0;
    for (int k = tid; k < N; k += blockDim.x) {
      const double2 v = U[k];
      e += v.x * v.x + v.y * v.y;
    }
    if (a.energy) {
      const double t = block_sum(e, red);
      if (tid == 0) a.energy[(size_t)hp * S + s] = t;
    }
    __syncthreads();
  }
}

// Plane sums of |U|^2 (updateTotalEnergy.cpp:25-33), one block per plane.
__global__ void __launch_bounds__(256) k_energy(DevGeom G, const double2* U, int ring_base, double* out) {
  __shared__ double red[8];
  const int S = G.S;
  const int s = blockIdx.x % S, hp = blockIdx.x / S;
  const double2* P = U + field_plane(S, hp >> 1, hp & 1, s, ring_base) * G.N;
  double e = 0.0;
  for (int k = threadIdx.x; k < G.N; k += blockDim.x) {
    const double2 v = P[k];
    e += v.x * v.x + v.y * v.y;
  }
  const double t = block_sum(e, red);
  if (threadIdx.x == 0) out[(size_t)hp * S + s] = t;
}

// out[hp] = sum over planes s of planes[hp][s], s < S - skip_last (fixed order).
__global__ void __launch_bounds__(256) k_sum_planes(const double* planes, int S, int skip_last, double* out) {
  __shared__ double red[8];
  const int hp = blockIdx.x;
  double e = 0.0;
  for (int s = threadIdx.x; s < S - skip_last; s += blockDim.x) e += planes[(size_t)hp * S + s];
  const double t = block_sum(e, red);
  if (threadIdx.x == 0) out[hp] = t;
}

}  // namespace

size_t deposit_smem_bytes(int chunk, int H, int neven, int L, int F, int nr) {
  return dep_layout(chunk, H, neven, L * F, nr).total;
}

void launch_deposit(const DepositLaunch& a, cudaStream_t st) {
  const size_t smem = deposit_smem_bytes(a.cap, a.G.H, a.neven, a.G.L, a.G.F, a.G.nr);
  k_deposit<<<a.G.S, 512, smem, st>>>(a);
}

void deposit_set_smem(size_t bytes) {
  cudaFuncSetAttribute(k_deposit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

void adi_set_smem(size_t bytes) {
  cudaFuncSetAttribute(k_adi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

size_t adi_smem_bytes(int nx, int ny, int nxp) {
  return (size_t)ny * nxp * sizeof(double2) + (size_t)4 * (nx + ny) * sizeof(double2) + (size_t)3 * (nx + ny) * sizeof(double);
}

void launch_adi(const AdiLaunch& a, cudaStream_t st) {
  const int mx = a.G.nx > a.G.ny ? a.G.nx : a.G.ny;
  const int threads = ((mx + 31) / 32) * 32;
  k_adi<<<a.G.S * a.G.H * 2, threads, adi_smem_bytes(a.G.nx, a.G.ny, a.nxp), st>>>(a);
}

size_t adi_big_smem_bytes(int nx, int ny) {
  return (size_t)4 * (nx + ny) * sizeof(double2) + (size_t)3 * (nx + ny) * sizeof(double);
}

void launch_adi_big(const AdiLaunch& a, int grid, cudaStream_t st) {
  const int mx = a.G.nx > a.G.ny ? a.G.nx : a.G.ny;
  const int threads = ((mx + 31) / 32) * 32;
  k_adi_big<<<grid, threads, adi_big_smem_bytes(a.G.nx, a.G.ny), st>>>(a);
}

void launch_energy(const DevGeom& G, const double2* U, int ring_base, double* out_planes, cudaStream_t st) {
  k_energy<<<G.S * G.H * 2, 256, 0, st>>>(G, U, ring_base, out_planes);
}

void launch_sum_planes(const double* planes, int H, int S, int skip_last, double* out, cudaStream_t st) {
  k_sum_planes<<<H * 2, 256, 0, st>>>(planes, S, skip_last, out);
}

}  // namespace felis
