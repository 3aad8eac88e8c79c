// Mixed-precision ensemble kernels: two launches per iteration.
//
//   k_batch_adi   one CTA per field plane (instance, slice, harmonic,
//                 polarisation): the ADI of solveField.cpp:80-185 in FP32 with
//                 the interior plane, the recurrence tables and the slice's
//                 source box in shared memory, four threads per line
//                 (partitioned recurrences); emits the plane's |U|^2 sum.
//   k_batch_push  one CTA per (instance, slice): both transverse half-pushes,
//                 push_theta_gamma or the drift and the theta wrap
//                 (particlePush.cpp, rearrangeParticles.cpp) in a loop
//                 specialised on the mode, then, reading the pushed particles
//                 back, the source deposit and the radial Ez solve of the next
//                 iteration's solveField (solveField.cpp:233-399) together with
//                 the beam partial sums (twiss.cpp, saveFile.cpp).
//
// Every (instance, slice) of an iteration is independent of the others: the
// slippage shift only renames planes (ring buffer), and the CTA of the last
// slice clears the plane that becomes the new first slice.
//
// The deposit accumulates 32-bit fixed-point integers (shared-memory
// atomics), so the sums do not depend on the order of the atomics: a run is
// reproducible bit for bit and independent of the launch shape and of the
// other instances.
#include <type_traits>

#include "batch.cuh"
#include "bulk.cuh"

namespace felis {

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ __forceinline__ float2 cm(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cs(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cad(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csb(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// e^{i x} for an FP32 phase of moderate size (|x| < 2^14): Cody-Waite
// reduction by 2 pi with a two-part constant (6.28125 is exact in 9 bits, so
// k * 6.28125 is exact), then the hardware sin/cos on [-pi, pi].
__device__ __forceinline__ float2 expif(float x) {
  const float k = rintf(x * 0.159154943091895336f);
  float r = fmaf(-k, 6.28125f, x);
  r = fmaf(-k, 1.93530717958647692e-3f, r);
  float s, c;
  __sincosf(r, &s, &c);
  return make_float2(c, s);
}

// theta (FP64, up to 2 pi numSlice) reduced to [-pi, pi] in FP32.
__device__ __forceinline__ float theta_red(double th) { return (float)(th - kTwoPi * rint(th * (1.0 / kTwoPi))); }

__device__ __forceinline__ double block_sum_d(double v, double* red) {
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

// xi2 and e^{i (B - Phi/2)} of particlePush.cpp:272-279 / solveField.cpp:259-266.
__device__ __forceinline__ void pol_phase(float K0, float ue, float K0a, float Phi_half, float px, float py,
                                          float* xi2, float2* eP) {
  *xi2 = 1.41421356f * K0 / (1.f + K0 * K0 * 0.5f * (1.f + ue * ue)) *
         sqrtf((1.f + K0a) * (px * px + ue * ue * py * py) + (1.f - K0a) * (px * px * ue * ue + py * py));
  const float B = atanf(2.f * K0a * ue * (px - py) /
                        ((1.f + K0a) * (px + ue * ue * py) + (1.f - K0a) * (px * ue * ue + py)));
  *eP = expif(B - Phi_half);
}

// Asynchronous 8-byte global -> shared copies (all in flight at once), then
// one wait for every copy of the thread.
__device__ __forceinline__ void cp_async8(void* dst_smem, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }


// ---- fixed-point accumulation ------------------------------------------------
constexpr int kAccBits = 31;

// v / q rounded to the nearest integer (ties to even), for |v / q| < 2^22,
// on the FMA pipe: q is a power of two, so v * (1/q) is exact, and adding
// 1.5 * 2^23 rounds it once to an integer held in the low mantissa bits.  The
// same value as __float2int_rn(v * inv_q) in that range, without the
// conversion unit.
__device__ __forceinline__ acc_t fix(float v, float inv_q) {
  return (acc_t)(__float_as_int(__fmaf_rn(v, inv_q, 12582912.f)) - 0x4B400000);
}
// quantum 2^e with bound / 2^e < 2^(kAccBits - 1): the rounded terms add at
// most half a quantum each on top of the exact sum, so no sum overflows; and
// term / 2^e < 2^22 for fix's range, `term` bounding a single term (it decides
// only for slices of a few hundred particles or fewer)
__device__ __forceinline__ float quantum(float bound, float term) {
  if (!(bound > 0.f)) return 1.f;
  int e = ilogbf(bound) + 2 - kAccBits;
  if (term > 0.f) e = max(e, ilogbf(term) - 21);
  e = max(e, -120);  // 1/q stays a finite float
  return ldexpf(1.f, e);
}

// ============================================================================
// ADI (solveField.cpp:80-185), one CTA per plane.
//
// Each sweep is a forward and a backward first-order linear recurrence along
// every interior row (x) or column (y), with data-independent coefficients.
// Each line is split into four chunks.  Thread (q, l) runs chunk q of line l:
// q = tid / NL and l = tid % NL with NL = max(mx, my), the threads rounded up
// to whole warps, so the lanes of a warp work on the same chunk of 32
// neighbouring lines (all but the one warp at each chunk boundary, which
// holds the last lines of chunk q and the first of chunk q + 1) and, the
// chunks being equal, run the same trip counts.  No lane is idle for lack of
// a line, as a line count rounded up to 32 per chunk would leave them (28 of
// 128 lanes on a 102-point grid).  A thread runs the recurrence over its
// chunk from a zero start and publishes the chunk's end value; after a
// barrier, chunk q composes the carry of the chunks before it (forward) or
// after it (backward) with the chunk products at their ends, at most three
// steps.  It then corrects its own points by the carry times the chunk
// product of the coefficients (host tables G, Q).  This is exact in real
// arithmetic; in FP32 the rounding differs from the serial order by a few
// ulps.  The products fall off geometrically (by |alpha| / H per point,
// about 0.01 on the usual grids), so the correction runs only over the points
// where a component is still 2^-40 or more.  Outside the absorbing layers
// every coefficient table holds one value, which those points take from
// registers (BInst::adi_k).
//
// The right-hand side of each sweep reads the neighbouring lines, which other
// threads overwrite.  The x sweep's is formed in place in the staged plane
// (thread per column and row chunk; the rows either side of the chunk are
// read before a barrier).  The y sweep's is formed while the x sweep's result
// is finished (thread per row and column chunk).  The source term is added
// afterwards, on the source box only.  Seven barriers per plane; the final
// values go straight to global memory (edge cells keep their values: the
// ADI never writes them).
// ============================================================================

// An interior index range [lo, hi) split at the range [k0, k1) where the
// coefficient tables hold one value: [lo, a) and [b, hi) read the tables,
// [a, b) uses that value from registers.
__device__ __forceinline__ void split3(int lo, int hi, int k0, int k1, int& a, int& b) {
  a = min(max(k0, lo), hi);
  b = min(max(k1, a), hi);
}

// The loops below run along one line of a plane in shared memory, stride
// `st` (1 along a row, the pitch along a column), in place.  Each loads the
// next point before it stores the current one: the compiler cannot move a
// shared-memory load above a store to the same array.  The forward loop's
// load one point past its range stays inside the shared-memory allocation
// (rows have pitch >= nx - 2, the tables follow the plane); its value is not
// used.

// Right-hand side v_k = ka_k u_{k+1} + kb_k u_k - kc_k u_{k-1}, k in [a, b)
// of a chunk that ends at `end`.  (um, u0, up) hold u_{k-1}, u_k, u_{k+1} and
// are advanced; u_{end} is `ue` (the point past the chunk, read before it
// changed).
template <bool K>
__device__ __forceinline__ void rhs_run(float2* __restrict__ v, int st, int a, int b, int end,
                                        const float2* ra, const float2* rb, const float2* rc, float2 ca, float2 cb,
                                        float2 cc, float2& um, float2& u0, float2& up, float2 ue) {
  const int bm = min(b, end - 2);  // below bm, u_{k+2} lies inside the chunk
  int k = a;
  for (; k < bm; ++k) {
    const float2 un = v[(k + 2) * st];
    const float2 ka = K ? ca : ra[k], kb = K ? cb : rb[k], kc = K ? cc : rc[k];
    v[k * st] = csb(cad(cm(ka, up), cm(kb, u0)), cm(kc, um));
    um = u0;
    u0 = up;
    up = un;
  }
  for (; k < b; ++k) {
    const float2 un = ue;  // used only where k + 2 == end
    const float2 ka = K ? ca : ra[k], kb = K ? cb : rb[k], kc = K ? cc : rc[k];
    v[k * st] = csb(cad(cm(ka, up), cm(kb, u0)), cm(kc, um));
    um = u0;
    u0 = up;
    up = un;
  }
}

// Forward recurrence L_k = v_k ka_k - km_k L_{k-1}, k in [a, b).
template <bool K>
__device__ __forceinline__ float2 fwd_run(float2* __restrict__ v, int st, int a, int b, const float2* ta,
                                          const float2* tm, float2 ca, float2 cmv, float2 L) {
  if (a < b) {
    float2 x = v[a * st];
    for (int k = a; k < b; ++k) {
      const float2 xn = v[(k + 1) * st];
      const float2 ka = K ? ca : ta[k], km = K ? cmv : tm[k];
      L = csb(cm(x, ka), cm(km, L));
      v[k * st] = L;
      x = xn;
    }
  }
  return L;
}

// Backward recurrence B_k = (v_k - B_{k+1}) kr_k, k from b - 1 down to a.
template <bool K>
__device__ __forceinline__ float2 bwd_run(float2* __restrict__ v, int st, int a, int b, const float2* tr, float2 cr,
                                          float2 B) {
  if (a < b) {
    float2 x = v[(b - 1) * st];
    for (int k = b - 1; k > a; --k) {
      const float2 xn = v[(k - 1) * st];
      const float2 kr = K ? cr : tr[k];
      B = cm(csb(x, B), kr);
      v[k * st] = B;
      x = xn;
    }
    const float2 kr = K ? cr : tr[a];
    B = cm(csb(x, B), kr);
    v[a * st] = B;
  }
  return B;
}

// Carry correction v_k += g_k d, k in [a, b).
__device__ __forceinline__ void axpy_run(float2* __restrict__ v, int st, int a, int b, const float2* g, float2 d) {
  for (int k = a; k < b; ++k) v[k * st] = cad(v[k * st], cm(g[k], d));
}

// Source term v_k += f src[(k + 1 - k0) * ss], k in [a, b), along a line of
// stride st, for a source box too large to stage (in global memory): read
// eight points at a time before the stores, since a generic pointer's loads
// cannot be moved past the shared-memory stores.
__device__ __forceinline__ void add_source(float2* __restrict__ v, int st, int a, int b, const float2* src, int k0,
                                           int ss, float2 f) {
  for (int k = a; k < b; k += 8) {
    float2 t[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) t[u] = k + u < b ? src[(k + u + 1 - k0) * ss] : make_float2(0.f, 0.f);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k + u < b) v[(k + u) * st] = cad(v[(k + u) * st], cm(f, t[u]));
  }
}

__global__ void __launch_bounds__(1024) k_batch_adi(BatchLaunch a) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ double redd[32];
  const int4 wi = a.work[blockIdx.x];
  const BInst& I = a.inst[wi.x];
  const BStep& T = a.step[wi.x];
  const int s = wi.y, hp = wi.z, h = hp >> 1, pol = hp & 1;
  const int S = I.S, nx = I.nx, ny = I.ny, P = I.pitch, Mx = nx > ny ? nx : ny;
  const int mx = nx - 2, my = ny - 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int NL = Mx - 2;  // lines per chunk: max(mx, my)
  // thread (chunk q, line l), q = tid / NL; the threads that round the block up
  // to whole warps get no line (l = NL fails every line test below)
  int q = tid / NL, l = tid - q * NL;
  if (q > 3) { q = 3; l = NL; }
  float2* U = I.U + ((size_t)hp * S + (s + T.ring_base) % S) * I.N;
  const float2* ad = I.adi_c + (size_t)h * 16 * Mx;
  float2* pl = reinterpret_cast<float2*>(sm);  // interior cells, [my][P]
  float2* tb = pl + (size_t)my * P;            // 16 tables of Mx
  float2* cf = tb + 16 * Mx;                   // forward end values of chunks 0-2, [3][NL]
  float2* cb = cf + 3 * NL;                    // backward start values of chunks 1-3
  float2* ce = cb + 3 * NL;                    // backward end values of chunks 0-2 (x sweep)
  float2* ssrc = ce + 3 * NL;
  // the 16 coefficient tables are one contiguous run: one bulk copy when both
  // ends are 16-byte aligned (an even number of staged plane cells)
  const bool tb_bulk = ((my * P) & 1) == 0 && (reinterpret_cast<uintptr_t>(ad) & 15) == 0;
  __shared__ __align__(8) unsigned long long tbar;
  if (tb_bulk) {
    if (tid == 0) {
      bar_init_tx(smem_u32(&tbar), (unsigned)(16 * Mx * sizeof(float2)));
      bulk_g2s(tb, ad, (unsigned)(16 * Mx * sizeof(float2)), smem_u32(&tbar));
    }
  } else {
    for (int k = tid; k < 16 * Mx; k += nt) cp_async8(tb + k, ad + k);
  }
  {
    const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
    for (int r = warp; r < my; r += nwarp)
      for (int c = lane; c < mx; c += 32) cp_async8(pl + r * P + c, U + (size_t)(r + 1) * nx + c + 1);
  }
  // source of this plane: odd harmonic -eta f m (one plane m for both
  // polarisations), even harmonic its own plane
  int bi0 = 1, bi1 = 0, bj0 = 1, bj1 = 0, bw = 0;
  const float2* Sc = nullptr;
  const float2 sfac = T.sfac[h][pol];
  if (T.current) {
    const int4 b = I.sbox[s];
    bi0 = b.x; bi1 = b.y; bj0 = b.z; bj1 = b.w;
    bw = bi1 - bi0 + 1;
    const int cells = (bw > 0 && bj1 >= bj0) ? bw * (bj1 - bj0 + 1) : 0;
    // the deposit packs the slice's source planes back to back, `cells` each
    const int p = I.src_plane[h] + ((I.harmony[h] & 1) ? 0 : pol);
    const float2* g = I.src + (size_t)s * I.nsrc * I.N + (size_t)p * cells;
    const size_t used = ((size_t)my * P + 16 * (size_t)Mx + 9 * (size_t)NL) * sizeof(float2);
    if (cells > 0 && used + (size_t)cells * sizeof(float2) <= (size_t)a.smem_bytes) {
      for (int k = tid; k < cells; k += nt) cp_async8(ssrc + k, g + k);
      Sc = ssrc;
    } else if (cells > 0) {
      Sc = g;
    } else {
      bi0 = 1; bi1 = 0;
    }
  }
  const bool src = Sc != nullptr;
  cp_async_wait_all();
  if (tb_bulk && !bar_wait0(smem_u32(&tbar), kBulkWaitTries)) {
    atomicOr(I.err + ERR_TIMEOUT, 1);
    bar_wait0(smem_u32(&tbar), kBulkWaitTries);  // once more for the copy in flight
  }
  __syncthreads();
  const float2 zero = make_float2(0.f, 0.f);
  const int* K8 = I.adi_k[h];
  const int kx0 = K8[0], kx1 = K8[1], ky0 = K8[2], ky1 = K8[3], gx = K8[4], qx = K8[5], gy = K8[6], qy = K8[7];
  const int kcx = kx0 < kx1 ? kx0 : 0, kcy = ky0 < ky1 ? ky0 : 0;  // where the constants are read
  const int c0 = I.cx[q], c1 = I.cx[q + 1];  // this thread's chunk of a row (x sweep)
  const int r0 = I.cy[q], r1 = I.cy[q + 1];  // and of a column (x right-hand side, y sweep)
  double e = 0.0;
  // ---- x sweep right-hand side: thread (column l, row chunk q), in place in
  // the staged plane; the rows either side of the chunk are read first
  {
    const bool valid = l < mx;
    const int c = valid ? l : 0, i = c + 1;
    float2 um = zero, ul = zero;
    if (valid) {
      um = r0 == 0 ? U[i] : pl[(r0 - 1) * P + c];
      ul = r1 == my ? U[(size_t)(ny - 1) * nx + i] : pl[r1 * P + c];
    }
    // |U|^2 of the edge cells, which keep their values
    const int ne = 2 * nx + 2 * my;
    for (int k = tid; k < ne; k += nt) {
      float2 v;
      if (k < nx) v = U[k];
      else if (k < 2 * nx) v = U[(size_t)(ny - 1) * nx + (k - nx)];
      else v = U[(size_t)(((k - 2 * nx) >> 1) + 1) * nx + (((k - 2 * nx) & 1) ? nx - 1 : 0)];
      e += (double)(v.x * v.x + v.y * v.y);
    }
    __syncthreads();
    if (valid) {
      const float2* ra = tb + 10 * Mx;
      const float2* rb = tb + 11 * Mx;
      const float2* rc = tb + 12 * Mx;
      float2* v = pl + c;
      float2 u0 = v[r0 * P];
      float2 up = r0 + 1 < r1 ? v[(r0 + 1) * P] : ul;
      int ka_, kb_;
      split3(r0, r1, ky0, ky1, ka_, kb_);
      const float2 ca = ra[kcy], cb_ = rb[kcy], cc = rc[kcy];
      rhs_run<false>(v, P, r0, ka_, r1, ra, rb, rc, ca, cb_, cc, um, u0, up, ul);
      rhs_run<true>(v, P, ka_, kb_, r1, ra, rb, rc, ca, cb_, cc, um, u0, up, ul);
      rhs_run<false>(v, P, kb_, r1, r1, ra, rb, rc, ca, cb_, cc, um, u0, up, ul);
      // the source term, on the rows of the slice's source box only
      if (src && i >= bi0 && i <= bi1) {
        const int ra0 = max(r0, bj0 - 1), ra1 = min(r1, bj1);
        const float2* sc = Sc + (i - bi0);
        if (Sc == ssrc)
          for (int r = ra0; r < ra1; ++r) v[r * P] = cad(v[r * P], cm(sfac, sc[(r + 1 - bj0) * bw]));
        else
          add_source(v, P, ra0, ra1, sc, bj0, bw, sfac);
      }
    }
  }
  __syncthreads();
  // ---- x sweep: thread (row l, column chunk q)
  {
    const float2* pa = tb;
    const float2* pm = tb + Mx;
    const float2* pr = tb + 2 * Mx;
    const float2* pG = tb + 3 * Mx;
    const float2* pQ = tb + 4 * Mx;
    const bool valid = l < my;
    float2* row = pl + (valid ? l : 0) * P;
    int ka_, kb_;
    split3(c0, c1, kx0, kx1, ka_, kb_);
    if (valid) {
      const float2 ca = pa[kcx], cmv = pm[kcx];
      float2 L = fwd_run<false>(row, 1, c0, ka_, pa, pm, ca, cmv, zero);
      L = fwd_run<true>(row, 1, ka_, kb_, pa, pm, ca, cmv, L);
      L = fwd_run<false>(row, 1, kb_, c1, pa, pm, ca, cmv, L);
      if (q < 3) cf[q * NL + l] = L;
    }
    __syncthreads();
    if (valid) {
      // carry into the chunk: the forward result left of it, composed over the chunks before
      float2 din = zero;
      for (int p = 0; p < q; ++p) din = cad(cf[p * NL + l], cm(pG[I.cx[p + 1] - 1], din));
      axpy_run(row, 1, c0, min(c1, c0 + gx), pG, din);
      const float2 cr = pr[kcx];
      float2 B = bwd_run<false>(row, 1, kb_, c1, pr, cr, zero);
      B = bwd_run<true>(row, 1, ka_, kb_, pr, cr, B);
      B = bwd_run<false>(row, 1, c0, ka_, pr, cr, B);
      if (q > 0) cb[(q - 1) * NL + l] = B;
      if (q < 3) ce[q * NL + l] = row[c1 - 1];
    }
    __syncthreads();
    if (valid) {
      // carry into the chunk from the right: the x sweep's result at c1
      float2 uin = zero;
      for (int p = 3; p > q; --p) uin = cad(cb[(p - 1) * NL + l], cm(pQ[I.cx[p]], uin));
      axpy_run(row, 1, max(c0, c1 - qx), c1, pQ, uin);
      // the x sweep's result left of the chunk (zero left of the first column):
      // the previous chunk's last point corrected by its carry, the result at c0
      const float2 uprev = q > 0 ? cad(ce[(q - 1) * NL + l], cm(pQ[c0 - 1], row[c0])) : zero;
      // ---- the y sweep's right-hand side from the x sweep's result
      const float2* ra = tb + 13 * Mx;
      const float2* rb = tb + 14 * Mx;
      const float2* rc = tb + 15 * Mx;
      const int j = l + 1;
      float2 um = uprev;
      float2 u0 = row[c0];
      float2 up = c0 + 1 < c1 ? row[c0 + 1] : uin;
      const float2 ca = ra[kcx], cb_ = rb[kcx], cc = rc[kcx];
      rhs_run<false>(row, 1, c0, ka_, c1, ra, rb, rc, ca, cb_, cc, um, u0, up, uin);
      rhs_run<true>(row, 1, ka_, kb_, c1, ra, rb, rc, ca, cb_, cc, um, u0, up, uin);
      rhs_run<false>(row, 1, kb_, c1, c1, ra, rb, rc, ca, cb_, cc, um, u0, up, uin);
      if (src && j >= bj0 && j <= bj1) {
        const int ca0 = max(c0, bi0 - 1), ca1 = min(c1, bi1);
        const float2* sr = Sc + (j - bj0) * bw;
        if (Sc == ssrc)
          for (int c = ca0; c < ca1; ++c) row[c] = cad(row[c], cm(sfac, sr[c + 1 - bi0]));
        else
          add_source(row, 1, ca0, ca1, sr, bi0, 1, sfac);
      }
    }
  }
  __syncthreads();
  // ---- y sweep: thread (column l, row chunk q); results to global memory
  {
    const float2* pa = tb + 5 * Mx;
    const float2* pm = tb + 6 * Mx;
    const float2* pr = tb + 7 * Mx;
    const float2* pG = tb + 8 * Mx;
    const float2* pQ = tb + 9 * Mx;
    const bool valid = l < mx;
    const int c = valid ? l : 0;
    float2* v = pl + c;
    int ka_, kb_;
    split3(r0, r1, ky0, ky1, ka_, kb_);
    if (valid) {
      const float2 ca = pa[kcy], cmv = pm[kcy];
      float2 L = fwd_run<false>(v, P, r0, ka_, pa, pm, ca, cmv, zero);
      L = fwd_run<true>(v, P, ka_, kb_, pa, pm, ca, cmv, L);
      L = fwd_run<false>(v, P, kb_, r1, pa, pm, ca, cmv, L);
      if (q < 3) cf[q * NL + l] = L;
    }
    __syncthreads();
    if (valid) {
      float2 din = zero;
      for (int p = 0; p < q; ++p) din = cad(cf[p * NL + l], cm(pG[I.cy[p + 1] - 1], din));
      axpy_run(v, P, r0, min(r1, r0 + gy), pG, din);
      const float2 cr = pr[kcy];
      float2 B = bwd_run<false>(v, P, kb_, r1, pr, cr, zero);
      B = bwd_run<true>(v, P, ka_, kb_, pr, cr, B);
      B = bwd_run<false>(v, P, r0, ka_, pr, cr, B);
      if (q > 0) cb[(q - 1) * NL + l] = B;
    }
    __syncthreads();
    if (valid) {
      float2 uin = zero;
      for (int p = 3; p > q; --p) uin = cad(cb[(p - 1) * NL + l], cm(pQ[I.cy[p]], uin));
      // y sweep result u_r = v_r + Q_r uin; Q matters on the last qy rows only
      float2* Ug = U + nx + c + 1;
      const int rq = max(r0, r1 - qy);
      float2 x = v[r0 * P];
      for (int r = r0; r < rq; ++r) {
        const float2 xn = v[(r + 1) * P];
        Ug[(size_t)r * nx] = x;
        e += (double)(x.x * x.x + x.y * x.y);
        x = xn;
      }
      for (int r = rq; r < r1; ++r) {
        const float2 xn = v[(r + 1) * P];
        const float2 o = cad(x, cm(pQ[r], uin));
        Ug[(size_t)r * nx] = o;
        e += (double)(o.x * o.x + o.y * o.y);
        x = xn;
      }
    }
  }
  const double et = block_sum_d(e, redd);
  if (tid == 0) I.part_e[(size_t)s * 2 * I.H + hp] = et;
}

// ============================================================================
// Push and the next deposit, one CTA per (instance, slice).
// ============================================================================
// Bessel table lookup held in registers.
struct BesselTab {
  const float* __restrict__ t;
  int bn, bcols;
  float idb;  // 1 / dBessel
};
__device__ __forceinline__ float bjt(const BesselTab& B, int row, int col) {
  row = row < 0 ? 0 : (row >= B.bn ? B.bn - 1 : row);
  return __ldg(B.t + row * B.bcols + col);
}

// fx, fy of harmonic H for the push (sign conventions of
// particlePush.cpp:336-360) or the deposit (solveField.cpp:277-300).
__device__ __forceinline__ void ffac_t(const BesselTab& B, int H, float xi, float xi2, float K0a, float2 eP,
                                       bool deposit, float2* fx, float2* fy) {
  const float x = (float)H * xi * B.idb;
  const int idx = (int)x;
  const float w1 = x - (float)idx, w0 = 1.f - w1;
  const float2 eM = make_float2(eP.x, -eP.y);
  if (H & 1) {
    const float sign = (((H - 1) / 2) % 2 == 0) ? 1.f : -1.f;
    const float J1 = bjt(B, idx, (H - 1) / 2) * w0 + bjt(B, idx + 1, (H - 1) / 2) * w1;
    const float J2 = bjt(B, idx, (H + 1) / 2) * w0 + bjt(B, idx + 1, (H + 1) / 2) * w1;
    if (deposit) { *fx = make_float2(sign * (J1 - K0a * J2), 0.f); *fy = make_float2(sign * (J1 + K0a * J2), 0.f); }
    else { *fx = make_float2(sign * (K0a * J1 - J2), 0.f); *fy = make_float2(sign * (K0a * J1 + J2), 0.f); }
  } else {
    const float sign = ((H / 2) % 2 == 0) ? 1.f : -1.f;
    const float J1 = bjt(B, idx, (H - 2) / 2) * w0 + bjt(B, idx + 1, (H - 2) / 2) * w1;
    const float J2 = bjt(B, idx, H / 2) * w0 + bjt(B, idx + 1, H / 2) * w1;
    const float J3 = bjt(B, idx, (H + 2) / 2) * w0 + bjt(B, idx + 1, (H + 2) / 2) * w1;
    const float sx = sign * xi2 * H * 0.5f;
    if (deposit) {
      *fx = cs(cad(cs(eM, J1 - K0a * J2), cs(eP, J2 - K0a * J3)), sx);
      *fy = cs(cad(cs(eM, J1 + K0a * J2), cs(eP, J2 + K0a * J3)), sx);
    } else {
      *fx = cs(cad(cs(eP, K0a * J1 - J2), cs(eM, K0a * J2 - J3)), sx);
      *fy = cs(cad(cs(eP, K0a * J1 + J2), cs(eM, K0a * J2 + J3)), sx);
    }
  }
}

// The push's fx, fy of an odd harmonic H (real) at xi0 and their slopes
// d/dxi, from the table cell that holds H xi0: the table interpolant is linear
// in xi inside a cell, and a particle's xi = xi0 / (1 + d)^2 moves off xi0 by
// about 2 |d| xi0 (|d| = |gamma / gamR - 1| <~ 1e-3), a small fraction of a
// cell, so fx = fx0 + dfx (xi - xi0) is the interpolant itself up to the
// cell edges.
__device__ __forceinline__ void odd_factors(const BesselTab& B, int H, float xi0, float K0a, float* fx0, float* fy0,
                                            float* dfx, float* dfy) {
  const float x = (float)H * xi0 * B.idb;
  const int idx = (int)x;
  const float w1 = x - (float)idx, w0 = 1.f - w1;
  const float sign = (((H - 1) / 2) % 2 == 0) ? 1.f : -1.f;
  const float a1 = bjt(B, idx, (H - 1) / 2), b1 = bjt(B, idx + 1, (H - 1) / 2);
  const float a2 = bjt(B, idx, (H + 1) / 2), b2 = bjt(B, idx + 1, (H + 1) / 2);
  const float J1 = a1 * w0 + b1 * w1, J2 = a2 * w0 + b2 * w1;
  const float sl = (float)H * B.idb;  // d(x) / d(xi)
  const float dJ1 = (b1 - a1) * sl, dJ2 = (b2 - a2) * sl;
  *fx0 = sign * (K0a * J1 - J2);
  *fy0 = sign * (K0a * J1 + J2);
  *dfx = sign * (K0a * dJ1 - dJ2);
  *dfy = sign * (K0a * dJ1 + dJ2);
}

// Shrinks [i0, i1] x [j0, j1] to its central window of at most `cap` cells
// (about the same aspect); empty (i1 < i0) when no 2 x 2 window fits.  The
// same for every thread of a CTA.
__device__ __forceinline__ void shrink_window(int& i0, int& i1, int& j0, int& j1, int cap) {
  const int w = i1 - i0 + 1, h = j1 - j0 + 1;
  if (w <= 0 || h <= 0 || w * h <= cap) return;
  if (cap < 4) { i1 = i0 - 1; return; }
  const float sc = sqrtf((float)cap / ((float)w * (float)h));
  int w2 = max(2, min(w, (int)((float)w * sc))), h2 = max(2, min(h, (int)((float)h * sc)));
  while (w2 * h2 > cap) {
    if (w2 >= h2 && w2 > 2) --w2;
    else if (h2 > 2) --h2;
    else break;
  }
  if (w2 * h2 > cap) { i1 = i0 - 1; return; }
  i0 += (w - w2) / 2; i1 = i0 + w2 - 1;
  j0 += (h - h2) / 2; j1 = j0 + h2 - 1;
}

// Fixed-point adds without a return value: shared-memory accumulators by
// their 32-bit shared address, global ones by pointer.
__device__ __forceinline__ void red_s(unsigned saddr, acc_t v) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.s32 p, %1, 0;\n\t"
      "@p red.shared.add.s32 [%0], %1;\n\t}\n" ::"r"(saddr),
      "r"(v)
      : "memory");
}
// SH: every accumulator in shared memory, at idx.  Otherwise the box's
// accumulators are in global memory (idx) and those of its central window in
// shared memory (widx, -1 outside the window).
template <bool SH>
__device__ __forceinline__ void acc_to(acc_t* gbase, unsigned sbase, int idx, int widx, acc_t v) {
  if (SH) red_s(sbase + 4u * (unsigned)idx, v);
  else if (widx >= 0) red_s(sbase + 4u * (unsigned)widx, v);
  else if (v != 0) atomicAdd(gbase + idx, v);
}

// Constants of the deposit launch in registers.
struct DepConst {
  float K0, ue, K0a, Phi_half, coef_U, xi, coef_Ez;
  float2 etaX, etaY;
};

// Pass 2: the source deposit (solveField.cpp:252-357) of the pushed
// particles into the fixed-point accumulators (2D: shared, or global with the
// window [wi0, wi1] x [wj0, wj1] of wcells cells in shared memory; radial:
// shared).
// With SUMS, the pass also accumulates the twiss and bunching partial sums of
// the (pushed) particles (twiss.cpp, saveFile.cpp): acc7 = x^2, y^2, x'^2,
// y'^2, x x', y y', count; bre / bim = sum of e^{i H theta} per harmonic.
template <int HM>
__device__ __forceinline__ void beam_sums(float (&acc7)[7], float (&bre)[HM], float (&bim)[HM], const float2 (&eb)[HM],
                                          int H, float x, float y, float px, float py, float g) {
  const float ig = 1.f / g, xp = px * ig, yp = py * ig;
  acc7[0] += x * x; acc7[1] += y * y; acc7[2] += xp * xp;
  acc7[3] += yp * yp; acc7[4] += x * xp; acc7[5] += y * yp; acc7[6] += 1.f;
#pragma unroll
  for (int h = 0; h < HM; ++h) {
    if (h >= H) break;
    bre[h] += eb[h].x;
    bim[h] += eb[h].y;
  }
}
// e^{i H theta} of every harmonic from the reduced phase
template <int HM>
__device__ __forceinline__ void harmonic_phases(float2 (&eb)[HM], const int (&hh)[HM], int H, float thn) {
#pragma unroll
  for (int h = 0; h < HM; ++h) eb[h] = h < H ? expif((float)hh[h] * thn) : make_float2(1.f, 0.f);
}

template <int HM, bool SH, bool SUMS>
__device__ __forceinline__ void deposit_pass(const float* __restrict__ xs, const float* __restrict__ ys,
                                             const float* __restrict__ pxs, const float* __restrict__ pys,
                                             const float* __restrict__ dgs, const double* __restrict__ ths,
                                             int64_t p0, int P, const int (&hh)[HM], const int (&sp)[HM], int H,
                                             bool has_even, const DepConst& D, const BesselTab& B, float weight,
                                             float gRf, float minX, float minY, float idx_, float idy_, int nx,
                                             int ny, int bi0, int bi1, int bj0, int bj1, int bw, int cells,
                                             int wi0, int wi1, int wj0, int wj1, int wcells, float iq2, float iqr,
                                             acc_t* gacc, unsigned sacc, unsigned sR, float dr, float idr2, int nr,
                                             int L, int F, float (&acc7)[7], float (&bre)[HM], float (&bim)[HM]) {
  const int ww = wi1 - wi0 + 1;
  float2 ePhi[HM];  // e^{-i H Phi/2} of the deposit's lattice
#pragma unroll
  for (int h = 0; h < HM; ++h) ePhi[h] = expif(-(float)hh[h] * D.Phi_half);
  // The particles are visited in the reverse of the push's order, so that the
  // first reads find the push's latest stores still in L2.  The next
  // particle's state is loaded one iteration ahead: the accumulator adds below
  // are compiler memory barriers, so no load moves above them.
  const int nt = blockDim.x, t0 = threadIdx.x;
  float nxv = 0.f, nyv = 0.f, ndg = 0.f, npx = 0.f, npy = 0.f;
  double nth = 0.0;
  const int qlast = t0 < P ? t0 + (P - 1 - t0) / nt * nt : -1;  // this thread's last particle
  if (qlast >= 0) {
    const int64_t n = p0 + qlast;
    nxv = xs[n]; nyv = ys[n]; ndg = dgs[n]; nth = ths[n];
    if (SUMS || has_even) { npx = pxs[n]; npy = pys[n]; }
  }
  for (int q = qlast; q >= 0; q -= nt) {
    const float x = nxv, y = nyv, g = gRf + ndg, px = npx, py = npy;
    const double th = nth;
    if (q >= nt) {
      const int64_t m = p0 + q - nt;
      nxv = xs[m]; nyv = ys[m]; ndg = dgs[m]; nth = ths[m];
      if (SUMS || has_even) { npx = pxs[m]; npy = pys[m]; }
    }
    const float thr = theta_red(th);
    // e^{i H theta}: the bunching sums' phases, and (conjugated, times the
    // per-launch e^{-i H Phi/2}) the deposit's
    float2 eb[HM];
    harmonic_phases<HM>(eb, hh, H, thr);
    if (SUMS) beam_sums<HM>(acc7, bre, bim, eb, H, x, y, px, py, g);
    const float gx = (x - minX) * idx_, gy = (y - minY) * idy_;
    const int ii = (int)gx, jj = (int)gy;
    if (ii >= 0 && ii < nx && jj >= 0 && jj < ny && cells > 0) {
      const float wx1 = gx - ii, wy1 = gy - jj;
      float xi2 = 0.f;
      float2 eP = make_float2(1.f, 0.f);
      if (has_even) pol_phase(D.K0, D.ue, D.K0a, D.Phi_half, px, py, &xi2, &eP);
      int cidx[4], widx[4];
      float wv[4];
      if constexpr (SH) {
        // the whole box in shared memory: a corner outside it (an edge cell of
        // the grid; the particle may sit in the last column or row, beyond
        // bi1 / bj1) gets weight 0, and a zero term adds nothing
        const int base = (jj - bj0) * bw + (ii - bi0);
        const bool vx0 = ii >= bi0 && ii <= bi1, vx1 = ii + 1 >= bi0 && ii + 1 <= bi1;
        const bool vy0 = jj >= bj0 && jj <= bj1, vy1 = jj + 1 >= bj0 && jj + 1 <= bj1;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
          const bool in = ((cb & 1) ? vx1 : vx0) && ((cb >> 1) ? vy1 : vy0);
          cidx[cb] = in ? base + (cb & 1) + (cb >> 1) * bw : 0;
          widx[cb] = -1;
          wv[cb] = in ? ((cb & 1) ? wx1 : 1.f - wx1) * ((cb >> 1) ? wy1 : 1.f - wy1) : 0.f;
        }
      } else {
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
          const int ti = ii + (cb & 1), tj = jj + (cb >> 1);
          const bool in = ti >= bi0 && ti <= bi1 && tj >= bj0 && tj <= bj1;
          cidx[cb] = in ? (tj - bj0) * bw + (ti - bi0) : -1;
          const bool inw = ti >= wi0 && ti <= wi1 && tj >= wj0 && tj <= wj1;
          widx[cb] = inw ? (tj - wj0) * ww + (ti - wi0) : -1;
          wv[cb] = ((cb & 1) ? wx1 : 1.f - wx1) * ((cb >> 1) ? wy1 : 1.f - wy1);
        }
      }
      const float ig = 1.f / g;
#pragma unroll
      for (int h = 0; h < HM; ++h) {
        if (h >= H) break;
        const int Hh = hh[h];
        const float2 e = cm(make_float2(eb[h].x, -eb[h].y), ePhi[h]);  // e^{-i H (theta + Phi/2)}
        const float2 mc = cs(e, (float)Hh * weight * D.coef_U * ig);
        const int base = sp[h] * cells * 2, wbase = sp[h] * wcells * 2;
        if (Hh & 1) {
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) {
            if (!SH && cidx[cb] < 0) continue;
            const int wk = widx[cb] < 0 ? -1 : wbase + 2 * widx[cb];
            acc_to<SH>(gacc, sacc, base + 2 * cidx[cb], wk, fix(mc.x * wv[cb], iq2));
            acc_to<SH>(gacc, sacc, base + 2 * cidx[cb] + 1, wk < 0 ? -1 : wk + 1, fix(mc.y * wv[cb], iq2));
          }
        } else {
          float2 fx, fy;
          ffac_t(B, Hh, D.xi, xi2, D.K0a, eP, true, &fx, &fy);
          const float2 ax = cm(cm(D.etaX, fx), mc), ay = cm(cm(D.etaY, fy), mc);
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) {
            if (!SH && cidx[cb] < 0) continue;
            const int wk = widx[cb] < 0 ? -1 : wbase + 2 * widx[cb];
            const int wky = widx[cb] < 0 ? -1 : wbase + 2 * (wcells + widx[cb]);
            acc_to<SH>(gacc, sacc, base + 2 * cidx[cb], wk, fix(-ax.x * wv[cb], iq2));
            acc_to<SH>(gacc, sacc, base + 2 * cidx[cb] + 1, wk < 0 ? -1 : wk + 1, fix(-ax.y * wv[cb], iq2));
            acc_to<SH>(gacc, sacc, base + 2 * (cells + cidx[cb]), wky, fix(-ay.x * wv[cb], iq2));
            acc_to<SH>(gacc, sacc, base + 2 * (cells + cidx[cb]) + 1, wky < 0 ? -1 : wky + 1, fix(-ay.y * wv[cb], iq2));
          }
        }
      }
    }
    // radial source: every particle (solveField.cpp:331-357)
    const float r = sqrtf(x * x + y * y);
    const int ir = (int)(r / dr + 0.5f);
    if (ir >= 0 && ir < nr - 1) {
      const float phi = (F > 1) ? ((x == 0.f) ? 0.f : atan2f(y, x)) : 0.f;
      const float wr1 = ir > 0 ? (r * r * idr2 - (float)(ir * ir)) / (2.f * ir) : 0.f;
      const float w0 = ir > 0 ? 1.f - wr1 : 1.f;
      const bool two = ir > 0 && ir + 1 < nr - 1;
      const float mag0 = D.coef_Ez * weight / (ir > 0 ? (float)ir : 1.f);
      for (int l = 0; l < L; ++l)
        for (int f = 0; f < F; ++f) {
          if (ir == 0 && f > 0) continue;
          // e^{-i ((l + 1) theta + f phi)}: the conjugate of the first harmonic's
          // phase for the lowest mode when the first harmonic is the fundamental
          const float2 e = (l == 0 && f == 0 && hh[0] == 1) ? make_float2(eb[0].x, -eb[0].y)
                                                            : expif(-((float)(l + 1) * thr + (float)f * phi));
          const float mag = mag0 * (l + 1.f);
          const float2 cc = make_float2(-e.y * mag, e.x * mag);  // i * coef * e^{-i..}
          const unsigned b0 = sR + 8u * (unsigned)((l * F + f) * nr + ir);
          red_s(b0, fix(cc.x * w0, iqr));
          red_s(b0 + 4u, fix(cc.y * w0, iqr));
          if (two) {
            red_s(b0 + 8u, fix(cc.x * wr1, iqr));
            red_s(b0 + 12u, fix(cc.y * wr1, iqr));
          }
        }
    }
  }
}

// One register budget per (harmonic class, Ez-mode class) instance, the same
// for every launch shape: 128 threads per CTA and as many CTAs per SM as a
// 1024-slice step needs to run in one wave on 148 SMs where the registers
// allow it (seven for one harmonic: 72 registers).
template <int HM>
struct PushBlocks {
  static constexpr int value = HM == 1 ? 7 : (HM == 2 ? 5 : 4);
};

template <int HM, int LM>
__global__ void __launch_bounds__(kPushThreads, PushBlocks<HM>::value) k_batch_push(BatchLaunch a) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ __align__(16) float smap[48];  // transverse map: D0, M1, M2 (row-major 4x4 each)
  __shared__ __align__(8) unsigned long long fbar;  // bulk staging of the field box
  const int4 wi = a.work[blockIdx.x];
  const BInst& I = a.inst[wi.x];
  const BStep& T = a.step[wi.x];
  const int s = wi.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  // instance and step constants in registers; the particle arrays are
  // restrict-qualified, so the stores below cannot alias them
  const int S = I.S, nx = I.nx, ny = I.ny, N = I.N, H = I.H, nr = I.nr, L = I.L, F = I.F, LF = L * F;
  float* __restrict__ xs = I.x;
  float* __restrict__ ys = I.y;
  float* __restrict__ pxs = I.px;
  float* __restrict__ pys = I.py;
  float* __restrict__ dgs = I.dg;
  double* __restrict__ ths = I.th;
  const int64_t p0 = I.soff[s], p1 = I.soff[s + 1];
  const int P = (int)(p1 - p0);
  const float weight = I.weight[s];
  const double gR = I.gamR;
  const float gRf = (float)gR, igR = (float)(1.0 / gR);
  const float minX = (float)I.minX, minY = (float)I.minY, idx_ = (float)(1.0 / I.dx), idy_ = (float)(1.0 / I.dy);
  const float dr = (float)I.dr, idr2 = (float)(1.0 / (I.dr * I.dr));
  const BesselTab B{I.bessel, I.bn, I.bcols, (float)(1.0 / I.dBessel)};
  const int plane = (s + T.ring_base) % S;
  int hh[HM], sp[HM];
  bool has_even = false;
  int Hmax = 1;
#pragma unroll
  for (int h = 0; h < HM; ++h) {
    hh[h] = h < H ? I.harmony[h] : 1;
    sp[h] = h < H ? I.src_plane[h] : 0;
    if (h < H) { has_even |= (hh[h] % 2 == 0); Hmax = max(Hmax, hh[h]); }
  }
  const bool push = a.mode == BATCH_PUSH;
  const bool dep = T.deposit != 0 && P > 0;
  DepConst D;
  D.K0 = T.dep.K0; D.ue = T.dep.ue; D.K0a = T.dep.K0a; D.Phi_half = T.dep.Phi_half; D.coef_U = T.dep.coef_U;
  D.xi = T.dep.xi; D.coef_Ez = T.dep.coef_Ez; D.etaX = T.dep.etaX; D.etaY = T.dep.etaY;
  // shared memory: Ez of the slice | radial accumulators | 2D accumulators
  float2* sEz = reinterpret_cast<float2*>(sm);
  const size_t o1 = ((size_t)LF * nr * sizeof(float2) + 15) & ~(size_t)15;
  const size_t o2 = o1 + (((size_t)LF * nr * 2 * sizeof(acc_t) + 15) & ~(size_t)15);
  acc_t* sR = reinterpret_cast<acc_t*>(sm + o1);
  unsigned char* area = sm + o2;
  const size_t area_bytes = (size_t)a.smem_bytes - o2;
  // deposit statistics of the (pushed) beam: cell box and fixed-point bounds.
  // The bounds are conservative and free of per-particle divisions: the 2-D
  // term |w mc| / weight <= max(fb) / min|g| per thread (w <= 1); the radial term
  // (1 + |wr1|) / max(ir, 1) <= 1.625 (|wr1| <= 5/8 for ir >= 1), counted when
  // a particle may lie inside the radial grid.
  int ci0 = 1 << 30, ci1 = -(1 << 30), cj0 = 1 << 30, cj1 = -(1 << 30);
  float wfmax = 0.f, gmin = 3.0e38f;
  int rin = 0;
  const float rlim2 = ((float)nr + 0.5f) * dr * ((float)nr + 0.5f) * dr;
  auto stats = [&](auto even_c, int ii, int jj, float x, float y, float px, float py, float g) {
    if (ii >= 0 && ii < nx && jj >= 0 && jj < ny) {
      ci0 = min(ci0, ii); ci1 = max(ci1, ii); cj0 = min(cj0, jj); cj1 = max(cj1, jj);
      float fb = 1.f;  // odd harmonics accumulate w mc (|f| applied later); bilinear w <= 1
      if constexpr (decltype(even_c)::value) {
        float xi2;
        float2 eP;
        pol_phase(D.K0, D.ue, D.K0a, D.Phi_half, px, py, &xi2, &eP);
        fb = fmaxf(fb, 2.f * xi2 * Hmax);
      }
      wfmax = fmaxf(wfmax, fb);
      gmin = fminf(gmin, fabsf(g));
    }
    rin |= (x * x + y * y < rlim2) ? 1 : 0;
  };
  // ================= pass 1: push (particlePush.cpp) =================
  if (push) {
    for (int k = tid; k < 48; k += nt) smap[k] = k < 16 ? T.tD0[k] : (k < 32 ? T.tM1[k - 16] : T.tM2[k - 32]);
    // The push's step constants and the odd harmonics' linearised Bessel
    // factors in shared memory, read (volatile) where the loop uses them:
    // held in registers across the loop they would spill at the 72-register
    // budget, and as reloads from the step structure they would be global
    // loads (the particle stores may alias it).  Same values, same results.
    __shared__ float pcst[16 + 4 * HM];
    if (tid == 0) {
      pcst[0] = T.R0; pcst[1] = T.A0; pcst[2] = T.AQ0; pcst[3] = T.c1 * T.c2; pcst[4] = T.K0; pcst[5] = T.ue;
      pcst[6] = T.K0a; pcst[7] = T.Phi_half; pcst[8] = T.K0 * T.sq; pcst[9] = T.ksK0 * T.sq; pcst[10] = T.e_mc2;
      pcst[11] = T.dPhi; pcst[12] = T.etaX.x; pcst[13] = T.etaX.y; pcst[14] = T.etaY.x; pcst[15] = T.etaY.y;
    }
    const volatile float* vc = pcst;
    for (int k = tid; k < LF * nr; k += nt) {
      const int l = k / (F * nr), rest = k % (F * nr);
      sEz[k] = I.Ez[((size_t)l * S + s) * F * nr + rest];
    }
    const int shift = T.shift;
    const double wakeE = I.wakeOn ? I.wakeE[s + I.minI] / (K_MC2 * 1.0e6) : 0.0;
    const double dz = I.dz;
    const float dwake = (float)(dz * wakeE);
    const double dTh = I.numSlice * 2 * M_PI, idTh = 1.0 / dTh;
    const double thshift = T.theta_shift;
    const float dzf = (float)dz;
    const float2* __restrict__ Ubase = I.U + (size_t)plane * N;
    const size_t hpstride = (size_t)S * N;
    // the slice's field around the beam, staged in the area the deposit
    // uses afterwards: the cell box of the last deposit (where the particles
    // were after the last push) with a margin of 3 cells; a particle outside
    // it reads global memory.  Same values, so the same results.
    int fi0 = 0, fi1 = -1, fj0 = 0, fj1 = -1, fbw = 1, fcells = 0;
    const float2* sF = reinterpret_cast<const float2*>(area);
    {
      const int4 b = I.sbox[s];
      // On an even-width grid every row of every plane starts on a 16-byte
      // boundary (the planes hold an even number of cells): the box, widened
      // to an even first and an odd last column, is staged by the bulk-copy
      // engine, one copy per row.  Otherwise by 8-byte cp.async per cell.
      const bool bulk = (nx & 1) == 0 && ((reinterpret_cast<uintptr_t>(Ubase) & 15) == 0);
      bool bulk_used = false;
      if (b.y >= b.x && b.w >= b.z) {
        int i0 = max(0, b.x - 3), i1 = min(nx - 1, b.y + 3), j0 = max(0, b.z - 3), j1 = min(ny - 1, b.w + 3);
        // a box too large for the area: its central window (the beam's core)
        const int cap = (int)(area_bytes / ((size_t)2 * H * sizeof(float2)));
        if (bulk) {
          i0 &= ~1; i1 |= 1;
          if ((i1 - i0 + 1) * (j1 - j0 + 1) > cap) {
            // re-widening the window adds at most one column either side
            shrink_window(i0, i1, j0, j1, cap - 2 * (j1 - j0 + 1));
            if (i1 >= i0) { i0 &= ~1; i1 |= 1; }
          }
        } else {
          shrink_window(i0, i1, j0, j1, cap);
        }
        const int w = i1 - i0 + 1, rows = j1 - j0 + 1, cells = w * rows;
        if (i1 >= i0 && j1 >= j0) {
          fi0 = i0; fi1 = i1; fj0 = j0; fj1 = j1; fbw = w; fcells = cells;
          float2* dst = reinterpret_cast<float2*>(area);
          if (bulk) {
            bulk_used = true;
            if (tid == 0) bar_init_tx(smem_u32(&fbar), (unsigned)(2 * H * cells * sizeof(float2)));
            __syncthreads();
            for (int k = tid; k < 2 * H * rows; k += nt) {
              const int hp = k / rows, r = k - hp * rows;
              bulk_g2s(dst + (size_t)hp * cells + (size_t)r * w, Ubase + hp * hpstride + (size_t)(j0 + r) * nx + i0,
                       (unsigned)(w * sizeof(float2)), smem_u32(&fbar));
            }
          } else {
            for (int hp = 0; hp < 2 * H; ++hp)
              for (int k = tid; k < cells; k += nt)
                cp_async8(dst + (size_t)hp * cells + k,
                          Ubase + hp * hpstride + (size_t)(j0 + k / w) * nx + i0 + k % w);
          }
        }
      }
      cp_async_wait_all();
      if (bulk_used && !bar_wait0(smem_u32(&fbar), kBulkWaitTries)) {
        atomicOr(I.err + ERR_TIMEOUT, 1);
        bar_wait0(smem_u32(&fbar), kBulkWaitTries);  // once more for the copies in flight
      }
    }
    __syncthreads();
    const float4* m4 = reinterpret_cast<const float4*>(smap);
    // error flags of this thread's particles, one bit each
    constexpr int kBadOver = 1, kBadRange = 2, kBadNan = 4, kBadRadial = 8;
    int bad = 0;
    // The push loop, specialised on the drift / undulator mode and on even
    // harmonics (uniform per CTA), so that each copy holds only the constants
    // its mode reads.
    auto push_loop = [&](auto drift_c, auto even_c) {
      constexpr bool DRIFT = decltype(drift_c)::value, EVEN = decltype(even_c)::value;
      // odd harmonics: the Bessel factors as a linear function of xi (odd_factors)
      float fx0[HM], fy0[HM], dfx[HM], dfy[HM];
      float xi0 = 0.f;
      if constexpr (!DRIFT) {
        xi0 = T.cxi * igR * igR;
#pragma unroll
        for (int h = 0; h < HM; ++h) {
          fx0[h] = fy0[h] = dfx[h] = dfy[h] = 0.f;
          if (h < H && (hh[h] & 1)) odd_factors(B, hh[h], xi0, T.K0a, &fx0[h], &fy0[h], &dfx[h], &dfy[h]);
        }
        if (tid == 0)
          for (int h = 0; h < HM; ++h) {
            pcst[16 + 4 * h] = fx0[h]; pcst[17 + 4 * h] = fy0[h]; pcst[18 + 4 * h] = dfx[h]; pcst[19 + 4 * h] = dfy[h];
          }
        __syncthreads();
      }
      // the next particle's state is loaded one iteration ahead
      float nxv = 0.f, nyv = 0.f, npx = 0.f, npy = 0.f, ndg = 0.f;
      double nth = 0.0;
      if (tid < P) {
        const int64_t n = p0 + tid;
        nxv = xs[n]; nyv = ys[n]; npx = pxs[n]; npy = pys[n]; ndg = dgs[n]; nth = ths[n];
      }
      for (int q = tid; q < P; q += nt) {
        const int64_t n = p0 + q;
        float x = nxv, y = nyv, px = npx, py = npy, dg = ndg;
        double th = nth;
        if (q + nt < P) {
          const int64_t m = n + nt;
          nxv = xs[m]; nyv = ys[m]; npx = pxs[m]; npy = pys[m]; ndg = dgs[m]; nth = ths[m];
        }
        const float g = gRf + dg;
        {  // both transverse half-pushes as one linear map (see BStep)
          const float da = -dg * igR / g;
          float o[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const float4 Dr = m4[r], Ar = m4[4 + r], Br = m4[8 + r];
            const float m2 = Br.x * x + Br.y * y + Br.z * px + Br.w * py;
            const float m1 = Ar.x * x + Ar.y * y + Ar.z * px + Ar.w * py + da * m2;
            o[r] = Dr.x * x + Dr.y * y + Dr.z * px + Dr.w * py + da * m1;
          }
          x += o[0]; y += o[1]; px += o[2]; py += o[3];
        }
        const float gx = (x - minX) * idx_, gy = (y - minY) * idy_;
        const int ii = (int)gx, jj = (int)gy;
        if (ii >= 0 && ii < nx - 1 && jj >= 0 && jj < ny - 1) {
          const float wx1 = gx - ii, wy1 = gy - jj, wx0 = 1.f - wx1, wy0 = 1.f - wy1;
          float2 Ux[HM], Uy[HM];
          float sumU2 = 0.f;
          // the bilinear gather of both polarisations of every harmonic: from
          // the staged box or from the plane in global memory, as two
          // explicit paths, so that the staged one reads shared memory
          // directly instead of through generic addresses
          const bool staged = ii >= fi0 && ii < fi1 && jj >= fj0 && jj < fj1;
          auto gather = [&](const float2* __restrict__ fb, auto fps, int frs) {
#pragma unroll
            for (int h = 0; h < HM; ++h) {
              if (h >= H) break;
              const float2* Px = fb + (2 * h) * fps;
              const float2* Py = Px + fps;
              Ux[h] = cad(cad(cs(Px[0], wx0 * wy0), cs(Px[frs], wx0 * wy1)), cad(cs(Px[1], wx1 * wy0), cs(Px[frs + 1], wx1 * wy1)));
              Uy[h] = cad(cad(cs(Py[0], wx0 * wy0), cs(Py[frs], wx0 * wy1)), cad(cs(Py[1], wx1 * wy0), cs(Py[frs + 1], wx1 * wy1)));
            }
          };
          if (staged) gather(sF + (jj - fj0) * fbw + (ii - fi0), fcells, fbw);
          else gather(Ubase + jj * nx + ii, hpstride, nx);
#pragma unroll
          for (int h = 0; h < HM; ++h) {
            if (h >= H) break;
            const float Hh = (float)hh[h];
            sumU2 += (Ux[h].x * Ux[h].x + Ux[h].y * Ux[h].y + Uy[h].x * Uy[h].x + Uy[h].y * Uy[h].y) / (2.f * Hh * Hh);
          }
          if constexpr (!DRIFT) {
            const float R0 = vc[0], A0 = vc[1], AQ0 = vc[2], c12 = vc[3], K0 = vc[4], ue = vc[5], K0a = vc[6];
            const float Phi_half = vc[7], K0sq = vc[8], ksK0sq = vc[9];
            const float e_mc2 = vc[10], dPhi = vc[11];
            const float2 etaX = make_float2(vc[12], vc[13]), etaY = make_float2(vc[14], vc[15]);
            const float r2 = x * x + y * y;
            const float k2 = px * px + py * py + c12 * r2;  // K2 - Q0
            const float i10 = 1.f / (1.f + dg * igR), i20 = i10 * i10;
            const float dxi = xi0 * (i20 - 1.f);  // xi - xi0, xi = cxi / gamma^2
            float xi2 = 0.f;
            float2 eP = make_float2(1.f, 0.f);
            if constexpr (EVEN) pol_phase(K0, ue, K0a, Phi_half, px, py, &xi2, &eP);
#pragma unroll
            for (int h = 0; h < HM; ++h) {  // fold the polarisation factors into the field
              if (h >= H) break;
              float2 fx, fy;
              if (hh[h] & 1) {
                fx = make_float2(vc[16 + 4 * h] + vc[18 + 4 * h] * dxi, 0.f);
                fy = make_float2(vc[17 + 4 * h] + vc[19 + 4 * h] * dxi, 0.f);
              } else {
                ffac_t(B, hh[h], xi0 * i20, xi2, K0a, eP, false, &fx, &fy);
              }
              Ux[h] = cm(cm(etaX, fx), Ux[h]);
              Uy[h] = cm(cm(etaY, fy), Uy[h]);
            }
            const float r = sqrtf(r2);
            const int ir = (int)(r / dr + 0.5f);
            float2 Em[LM];
#pragma unroll
            for (int l = 0; l < LM; ++l) Em[l] = make_float2(0.f, 0.f);
            if (ir >= 0 && ir < nr) {
              const float wr1 = ir > 0 ? (r2 * idr2 - (float)(ir * ir)) / (2.f * ir) : 1.f;
              const float wr0 = ir > 0 ? 1.f - wr1 : 1.f;
#pragma unroll
              for (int l = 0; l < LM; ++l) {
                if (l >= L) break;
                for (int f = 0; f < F; ++f) {
                  const float2 a0 = sEz[(l * F + f) * nr + ir];
                  const float2 a1 = (ir + 1 < nr) ? sEz[(l * F + f) * nr + ir + 1] : make_float2(0.f, 0.f);
                  Em[l] = cad(Em[l], cad(cs(a0, wr0), cs(a1, wr1)));
                }
              }
            } else {
              // beyond the radial Ez grid: the reference reuses the previous
              // particle's Em there (particlePush.cpp:286-304); flagged
              bad |= kBadRadial;
            }
            // RK4 in z of (theta, gamma); the theta slope in FP32 relative to
            // the resonance (BStep), theta itself accumulated in FP64
            const float thr = theta_red(th);
            float kth_prev = 0.f, kth_sum = 0.f, kg_prev = 0.f, kg_sum = 0.f;
#pragma unroll
            for (int m = 1; m < 5; ++m) {
              const float clm = (m == 1) ? 0.f : (m == 4 ? 1.f : 0.5f);
              const float tm = thr + dzf * kth_prev * clm;
              const float dgm = dg + dzf * kg_prev * clm;
              const float d = dgm * igR;
              const float inv1 = 1.f / (1.f + d), inv2 = inv1 * inv1;
              float sumEz = 0.f, sumTh = 0.f, sumG = 0.f;
#pragma unroll
              for (int l = 0; l < LM; ++l) {
                if (l >= L) break;
                const float2 e = expif((l + 1.f) * tm);
                sumEz += 2.f * (Em[l].x * e.x - Em[l].y * e.y);
              }
#pragma unroll
              for (int h = 0; h < HM; ++h) {
                if (h >= H) break;
                const float Hh = (float)hh[h];
                const float2 e = expif(Hh * (tm + Phi_half));
                const float2 tc = cm(e, csb(Ux[h], Uy[h]));
                sumTh += -tc.y / Hh;
                sumG += tc.x;
              }
              sumG *= 0.5f * igR * inv1;  // 1 / (gR + dg) = (1 / gR) / (1 + d)
              kth_prev = R0 + AQ0 * (d * (2.f + d) * inv2) - A0 * inv2 * (k2 + sumU2 + K0sq * sumTh);
              kg_prev = ksK0sq * sumG + e_mc2 * sumEz;
              const float wgt = (m == 1 || m == 4) ? 1.f : 2.f;
              kth_sum += wgt * kth_prev;
              kg_sum += wgt * kg_prev;
            }
            const float dth = dzf / 6.f * kth_sum;
            if (dth > dPhi || dth < -dPhi) bad |= kBadOver;
            th += (double)dth;
            dg += dzf / 6.f * kg_sum - dwake;
          } else {
            const double K2 = 1.0 + (double)px * px + (double)py * py;
            const double tmp = T.ku - T.A0d * (K2 + sumU2);
            th += tmp * dz;
            th -= dz * wakeE;
          }
        }
        th += thshift;  // [Phase_shifter] (0 when no shifter sits in this step)
        // theta wrap (rearrangeParticles.cpp:301-320) into [0, dTh); a theta
        // that needs no wrap is in range, so the range and NaN checks of theta
        // run only after a wrap (a NaN theta takes the wrap branch too)
        if (!(th >= 0.0 && th < dTh)) {
          th -= dTh * floor(th * idTh);
          if (th >= dTh) th -= dTh;
          else if (th < 0) th += dTh;
          if (!(th >= 0.0 && th <= dTh)) bad |= (th - th == 0.0) ? kBadRange : kBadNan;
        }
        if (!(dg - dg == 0.f) || !(x - x == 0.f)) bad |= kBadNan;
        xs[n] = x; ys[n] = y; pxs[n] = px; pys[n] = py; dgs[n] = dg; ths[n] = th;
        if (dep) stats(even_c, ii, jj, x, y, px, py, gRf + dg);
      }
    };
    if (T.drift) {
      if (has_even) push_loop(std::true_type{}, std::true_type{});
      else push_loop(std::true_type{}, std::false_type{});
    } else {
      if (has_even) push_loop(std::false_type{}, std::true_type{});
      else push_loop(std::false_type{}, std::false_type{});
    }
    if (bad & kBadOver) atomicOr(I.err + ERR_THETA_OVERFLOW, 1);
    if (bad & kBadRange) atomicOr(I.err + ERR_OUT_OF_RANGE, 1);
    if (bad & kBadNan) atomicOr(I.err + ERR_NAN, 1);
    if (bad & kBadRadial) atomicOr(I.err + ERR_RADIAL, 1);
    // slippage shift: the plane of the last slice becomes the new first slice
    if (shift && s == S - 1) {
      __syncthreads();
      for (int hp = 0; hp < 2 * H; ++hp) {
        float2* Up = I.U + ((size_t)hp * S + plane) * N;
        for (int k = tid; k < N; k += nt) Up[k] = make_float2(0.f, 0.f);
      }
    }
  } else if (dep) {
    for (int q = tid; q < P; q += nt) {
      const int64_t n = p0 + q;
      const float x = xs[n], y = ys[n], gx = (x - minX) * idx_, gy = (y - minY) * idy_;
      const float px = has_even ? pxs[n] : 0.f, py = has_even ? pys[n] : 0.f;
      if (has_even) stats(std::true_type{}, (int)gx, (int)gy, x, y, px, py, gRf + dgs[n]);
      else stats(std::false_type{}, (int)gx, (int)gy, x, y, px, py, gRf + dgs[n]);
    }
  }
  // twiss / bunching partial sums of the pushed beam: FP32 over a thread's
  // particles (64 per thread on the 8192-particle slices), FP64 across
  // threads; taken in the deposit pass below when there is one, else here
  float acc7[7] = {0, 0, 0, 0, 0, 0, 0};
  float bre[HM], bim[HM];
#pragma unroll
  for (int h = 0; h < HM; ++h) { bre[h] = 0.f; bim[h] = 0.f; }
  // the 7 + 2 H + 1 block sums of the beam, each as block_sum_d forms it (warp
  // tree, then the warps in order), under one barrier
  __shared__ double rsum[kPushThreads / 32][7 + 2 * HM + 1];
  auto write_sums = [&]() {
    const int stride = 7 + 2 * H + 1;
    double* out = I.part_b + (size_t)s * stride;
    const double wsum = (double)weight * (double)max(0, (P - tid + nt - 1) / nt);
    double v[7 + 2 * HM + 1];
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = (double)acc7[k];
#pragma unroll
    for (int h = 0; h < HM; ++h) { v[7 + 2 * h] = (double)bre[h]; v[8 + 2 * h] = (double)bim[h]; }
    v[7 + 2 * HM] = wsum;
    const int w = tid >> 5, ln = tid & 31;
#pragma unroll
    for (int k = 0; k < 7 + 2 * HM + 1; ++k) {
      if (k >= 7 + 2 * H && k < 7 + 2 * HM) continue;  // harmonics beyond H
      double x = v[k];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (ln == 0) rsum[w][k] = x;
    }
    __syncthreads();
    if (tid == 0) {
      auto total = [&](int k) {
        double t = 0.0;
        for (int q = 0; q < (nt + 31) / 32; ++q) t += rsum[q][k];
        return t;
      };
      for (int k = 0; k < 7; ++k) out[k] = total(k);
      for (int h = 0; h < H; ++h) { out[7 + 2 * h] = total(7 + 2 * h) * weight; out[8 + 2 * h] = total(8 + 2 * h) * weight; }
      out[7 + 2 * H] = total(7 + 2 * HM);
    }
  };
  if (push && !dep) {
    for (int q = tid; q < P; q += nt) {
      const int64_t n = p0 + q;
      float2 eb[HM];
      harmonic_phases<HM>(eb, hh, H, theta_red(ths[n]));
      beam_sums<HM>(acc7, bre, bim, eb, H, xs[n], ys[n], pxs[n], pys[n], gRf + dgs[n]);
    }
    write_sums();
  }
  if (!dep) return;
  // ================= pass 2: deposit of the next solveField =================
  // bounds: |w mc| <= wm H weight coef_U / g for odd harmonics, times |f| <=
  // 2 xi2 H for even ones (|eta| <= 1, |e| = 1); radial |w c| <= coef_Ez L
  // weight (1 + |wr1|) / max(ir, 1)
  const float bmax = wfmax > 0.f ? wfmax / gmin : 0.f, rmax = rin ? 1.625f : 0.f;
  // the cell box and both bounds over the CTA: warp trees, then the warps,
  // one barrier for the six values
  int mi0, mi1, mj0, mj1;
  float bmx, rmx;
  {
    __shared__ int rbox[kPushThreads / 32][4];
    __shared__ float rbnd2[kPushThreads / 32][2];
    int iv[4] = {ci0, -ci1, cj0, -cj1};
    float fv[2] = {bmax, rmax};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      for (int o = 16; o > 0; o >>= 1) iv[k] = min(iv[k], __shfl_down_sync(0xffffffffu, iv[k], o));
#pragma unroll
    for (int k = 0; k < 2; ++k)
      for (int o = 16; o > 0; o >>= 1) fv[k] = fmaxf(fv[k], __shfl_down_sync(0xffffffffu, fv[k], o));
    if ((tid & 31) == 0) {
      for (int k = 0; k < 4; ++k) rbox[tid >> 5][k] = iv[k];
      for (int k = 0; k < 2; ++k) rbnd2[tid >> 5][k] = fv[k];
    }
    __syncthreads();
    int t[4] = {1 << 30, 1 << 30, 1 << 30, 1 << 30};
    float u[2] = {0.f, 0.f};
    for (int q = 0; q < (nt + 31) / 32; ++q) {
      for (int k = 0; k < 4; ++k) t[k] = min(t[k], rbox[q][k]);
      for (int k = 0; k < 2; ++k) u[k] = fmaxf(u[k], rbnd2[q][k]);
    }
    mi0 = t[0]; mi1 = -t[1]; mj0 = t[2]; mj1 = -t[3];
    bmx = u[0]; rmx = u[1];
  }
  const float tb = bmx * 1.0625f * Hmax * weight * fabsf(D.coef_U), bnd = tb * (float)P;
  const float rtb = rmx * 1.0625f * L * weight * fabsf(D.coef_Ez), rbnd = rtb * (float)P;
  // interior targets a particle can reach
  const int bi0 = max(1, mi0), bi1 = min(nx - 2, mi1 + 1), bj0 = max(1, mj0), bj1 = min(ny - 2, mj1 + 1);
  const int bw = bi1 - bi0 + 1, bh = bj1 - bj0 + 1;
  const int cells = (bw > 0 && bh > 0) ? bw * bh : 0;
  const float q2 = quantum(bnd, tb), qr = quantum(rbnd, rtb);
  const float iq2 = 1.f / q2, iqr = 1.f / qr;
  // accumulators: one interleaved (re, im) pair per cell of each source plane
  const int nsrc = I.nsrc;
  const size_t nacc = (size_t)nsrc * cells * 2;
  float2* gsrc = I.src + (size_t)s * nsrc * N;
  const bool in_smem = nacc * sizeof(acc_t) <= area_bytes;
  acc_t* acc = in_smem ? reinterpret_cast<acc_t*>(area) : reinterpret_cast<acc_t*>(gsrc);
  // a box too large for the area accumulates in the source buffer, its
  // central window (the beam's core, where most particles add) in the area;
  // integer sums, so the split does not change the result
  int wi0 = bi0, wi1 = bi1, wj0 = bj0, wj1 = bj1;
  if (!in_smem) shrink_window(wi0, wi1, wj0, wj1, (int)(area_bytes / ((size_t)nsrc * 2 * sizeof(acc_t))));
  const int wcells = (!in_smem && cells > 0 && wi1 >= wi0 && wj1 >= wj0) ? (wi1 - wi0 + 1) * (wj1 - wj0 + 1) : 0;
  if (!wcells) { wi0 = 1; wi1 = 0; wj0 = 1; wj1 = 0; }
  for (size_t k = tid; k < nacc; k += nt) acc[k] = 0;
  for (int k = tid; k < nsrc * wcells * 2; k += nt) reinterpret_cast<acc_t*>(area)[k] = 0;
  for (int k = tid; k < LF * nr * 2; k += nt) sR[k] = 0;
  __syncthreads();
  const unsigned sacc = (unsigned)__cvta_generic_to_shared(area);
  const unsigned sRa = (unsigned)__cvta_generic_to_shared(sR);
  auto dep_pass = [&](auto sh_c, auto sums_c) {
    constexpr bool SHc = decltype(sh_c)::value, SUMSc = decltype(sums_c)::value;
    if constexpr (SHc)
      deposit_pass<HM, SHc, SUMSc>(xs, ys, pxs, pys, dgs, ths, p0, P, hh, sp, H, has_even, D, B, weight, gRf, minX,
                                   minY, idx_, idy_, nx, ny, bi0, bi1, bj0, bj1, bw, cells, 1, 0, 1, 0, 0, iq2, iqr,
                                   nullptr, sacc, sRa, dr, idr2, nr, L, F, acc7, bre, bim);
    else
      deposit_pass<HM, SHc, SUMSc>(xs, ys, pxs, pys, dgs, ths, p0, P, hh, sp, H, has_even, D, B, weight, gRf, minX,
                                   minY, idx_, idy_, nx, ny, bi0, bi1, bj0, bj1, bw, cells, wi0, wi1, wj0, wj1, wcells,
                                   iq2, iqr, acc, sacc, sRa, dr, idr2, nr, L, F, acc7, bre, bim);
  };
  if (in_smem) {
    if (push) dep_pass(std::true_type{}, std::true_type{});
    else dep_pass(std::true_type{}, std::false_type{});
  } else {
    if (push) dep_pass(std::false_type{}, std::true_type{});
    else dep_pass(std::false_type{}, std::false_type{});
  }
  if (push) write_sums();
  __syncthreads();
  if (wcells > 0) {
    // the window's sums into the box's
    const int ww = wi1 - wi0 + 1;
    const int2* wa = reinterpret_cast<const int2*>(area);
    int2* ga = reinterpret_cast<int2*>(acc);
    for (int k = tid; k < nsrc * wcells; k += nt) {
      const int pl = k / wcells, w = k - pl * wcells;
      const size_t gi = (size_t)pl * cells + (size_t)(wj0 + w / ww - bj0) * bw + (wi0 + w % ww - bi0);
      const int2 a = wa[k];
      int2 g = ga[gi];
      g.x += a.x;
      g.y += a.y;
      ga[gi] = g;
    }
    __syncthreads();
  }
  // source box of the next ADI (float2 per cell, in place when the
  // accumulators live in the source buffer itself)
  for (size_t k = tid; k < nacc / 2; k += nt) {
    const int2 v = reinterpret_cast<const int2*>(acc)[k];
    gsrc[k] = make_float2((float)v.x * q2, (float)v.y * q2);
  }
  if (tid == 0) I.sbox[s] = make_int4(bi0, cells > 0 ? bi1 : bi0 - 1, bj0, bj1);
  __syncthreads();
  // radial Thomas solve in FP64 (solveField.cpp:361-397): the multipliers and
  // pivots come from the host's table (they do not depend on the particles).
  // The whole CTA lays out, per (l, f) and point j, the right-hand side
  // (d re, d im), the pivot b_j and the multiplier w_j in shared memory; one
  // thread per (l, f) then runs the recurrence d_j -= w_j d_{j-1}, which
  // waits on no global load; the divisions of every point by the whole CTA.
  for (int k = tid; k < LF * nr; k += nt) {
    const int lf = k / nr, j = k - lf * nr, f = lf % F;
    const double* rt = a.rad + T.rad_off + (size_t)lf * nr * 2;  // (w_j, b_j)
    double* db = reinterpret_cast<double*>(area) + (size_t)k * 4;
    const bool zero = j == nr - 1 || (j == 0 && f != 0);
    db[0] = zero ? 0.0 : (double)sR[k * 2] * qr;
    db[1] = zero ? 0.0 : (double)sR[k * 2 + 1] * qr;
    db[2] = rt[2 * j + 1];
    db[3] = rt[2 * j];
  }
  __syncthreads();
  if (tid < LF) {
    double* dbuf = reinterpret_cast<double*>(area) + (size_t)tid * nr * 4;  // d re, d im, b, w
    double dre = dbuf[0], dim = dbuf[1];
    for (int j = 1; j < nr; ++j) {
      const double ww = dbuf[j * 4 + 3];
      double djr = dbuf[j * 4], dji = dbuf[j * 4 + 1];
      djr -= ww * dre;
      dji -= ww * dim;
      dbuf[j * 4] = djr; dbuf[j * 4 + 1] = dji;
      dre = djr; dim = dji;
    }
  }
  __syncthreads();
  // the solution d_j / b_j, j < nr - 1: independent divisions, spread over the CTA
  for (int k = tid; k < LF * (nr - 1); k += nt) {
    const int lf = k / (nr - 1), j = k - lf * (nr - 1), l = lf / F, f = lf - l * F;
    const double* dbuf = reinterpret_cast<const double*>(area) + (size_t)lf * nr * 4;
    const float2 v = make_float2((float)(dbuf[j * 4] / dbuf[j * 4 + 2]), (float)(dbuf[j * 4 + 1] / dbuf[j * 4 + 2]));
    I.Ez[((size_t)l * S + s) * F * nr + (size_t)f * nr + j] = v;
  }
}

// Diagnostics of the current state without stepping (the row of the first
// iteration of a run): plane energies and beam partial sums per slice.
__global__ void __launch_bounds__(256) k_batch_measure(const BInst* inst, const BStep* step, const int4* work,
                                                       int nwork) {
  __shared__ double red[8];
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int4 wi = work[w];
    const BInst& I = inst[wi.x];
    const BStep& T = step[wi.x];
    const int s = wi.y, S = I.S, N = I.N, H = I.H;
    for (int hp = 0; hp < 2 * H; ++hp) {
      const float2* U = I.U + ((size_t)hp * S + ((s + T.ring_base) % S)) * N;
      double e = 0.0;
      for (int k = threadIdx.x; k < N; k += blockDim.x) e += (double)U[k].x * U[k].x + (double)U[k].y * U[k].y;
      const double t = block_sum_d(e, red);
      if (threadIdx.x == 0) I.part_e[(size_t)s * 2 * H + hp] = t;
    }
    const int stride = 7 + 2 * H + 1;
    const float weight = I.weight[s];
    double acc[7 + 2 * FELIS_MAX_HARMONY + 1];
    for (int k = 0; k < stride; ++k) acc[k] = 0.0;
    for (int64_t n = I.soff[s] + threadIdx.x; n < I.soff[s + 1]; n += blockDim.x) {
      const double x = I.x[n], y = I.y[n], ig = 1.0 / (I.gamR + (double)I.dg[n]), xp = I.px[n] * ig, yp = I.py[n] * ig;
      acc[0] += x * x; acc[1] += y * y; acc[2] += xp * xp; acc[3] += yp * yp; acc[4] += x * xp; acc[5] += y * yp;
      acc[6] += 1.0;
      const float thr = theta_red(I.th[n]);
      for (int h = 0; h < H; ++h) {
        const float2 e = expif((float)I.harmony[h] * thr);
        acc[7 + 2 * h] += (double)e.x * weight;
        acc[8 + 2 * h] += (double)e.y * weight;
      }
      acc[7 + 2 * H] += weight;
    }
    for (int k = 0; k < stride; ++k) {
      const double t = block_sum_d(acc[k], red);
      if (threadIdx.x == 0) I.part_b[(size_t)s * stride + k] = t;
    }
  }
}

// One block per instance: the power of the new state (slices of the shifted
// ring) and the twiss / bFactor of the pushed beam, summed in slice order.
__global__ void __launch_bounds__(256) k_batch_reduce(const BInst* inst, const BStep* step, double* hist_e,
                                                      double* hist_t, double* hist_b, int se, int st_, int sb) {
  // every component (2 H plane energies, then the beam sums) reduced in the
  // same order as block_sum_d (warp trees, then the warps in order), with one
  // barrier for all of them
  constexpr int kMaxV = 2 * FELIS_MAX_HARMONY + 7 + 2 * FELIS_MAX_HARMONY + 1;
  __shared__ double part[8][kMaxV];
  __shared__ double tot[kMaxV];
  const BInst& I = inst[blockIdx.x];
  const BStep& T = step[blockIdx.x];
  const int H = I.H, S = I.S, stride = 7 + 2 * H + 1, ne = 2 * H, nv = ne + stride;
  double* he = hist_e + (size_t)blockIdx.x * se;
  double* ht = hist_t + (size_t)blockIdx.x * st_;
  double* hb = hist_b + (size_t)blockIdx.x * sb;
  const int last = T.shift ? S - 1 : S;
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31, nw = (int)((blockDim.x + 31) >> 5);
  for (int k = 0; k < nv; ++k) {
    double v = 0.0;
    if (k < ne) {
      for (int s = threadIdx.x; s < last; s += blockDim.x) v += I.part_e[(size_t)s * 2 * H + k];
    } else {
      for (int s = threadIdx.x; s < S; s += blockDim.x) v += I.part_b[(size_t)s * stride + (k - ne)];
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (ln == 0) part[w][k] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < nv) {
    double t = 0.0;
    for (int k = 0; k < nw; ++k) t += part[k][threadIdx.x];
    tot[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int hp = 0; hp < ne; ++hp) he[hp] = tot[hp];
    const double* acc = tot + ne;
    for (int k = 0; k < 6; ++k) ht[k] = 0.0;
    const double cnt = acc[6];
    if (cnt > 0) {
      const double ax = acc[0] / cnt, ay = acc[1] / cnt, axp = acc[2] / cnt, ayp = acc[3] / cnt;
      const double cx = acc[4] / cnt, cy = acc[5] / cnt;
      const double ex = sqrt(ax * axp - cx * cx), ey = sqrt(ay * ayp - cy * cy);
      ht[0] = ex; ht[1] = ax / ex; ht[2] = -cx / ex; ht[3] = ey; ht[4] = ay / ey; ht[5] = -cy / ey;
    }
    for (int k = 0; k < 2 * H; ++k) hb[k] = acc[7 + k] / acc[7 + 2 * H];
  }
}

// First-lag moments of the field over the slices, per instance (one CTA
// each): R0 = sum |U_s|^2 and R1 = sum conj(U_s) U_{s+1} over the slices in
// bunch order (the ring read from ring[i]), every cell and both
// polarisations of harmonic index hidx, FP64 sums in a fixed order.
__global__ void __launch_bounds__(256) k_batch_spectrum(const BInst* inst, const int* ring, int hidx, double* out) {
  __shared__ double red[8];
  const BInst& I = inst[blockIdx.x];
  double r0 = 0.0, r1re = 0.0, r1im = 0.0;
  if (hidx < I.H) {
    const int S = I.S, N = I.N, rb = ring[blockIdx.x];
    const int64_t tot = (int64_t)S * N;
    for (int pol = 0; pol < 2; ++pol) {
      const float2* U = I.U + (size_t)(hidx * 2 + pol) * S * N;
      for (int64_t k = threadIdx.x; k < tot; k += blockDim.x) {
        const int s = (int)(k / N), c = (int)(k - (int64_t)s * N);
        const float2 a = U[(size_t)((s + rb) % S) * N + c];
        r0 += (double)a.x * a.x + (double)a.y * a.y;
        if (s + 1 < S) {
          const float2 b = U[(size_t)((s + 1 + rb) % S) * N + c];
          r1re += (double)a.x * b.x + (double)a.y * b.y;
          r1im += (double)a.x * b.y - (double)a.y * b.x;
        }
      }
    }
  }
  const double t0 = block_sum_d(r0, red), t1 = block_sum_d(r1re, red), t2 = block_sum_d(r1im, red);
  if (threadIdx.x == 0) {
    out[3 * blockIdx.x] = t0;
    out[3 * blockIdx.x + 1] = t1;
    out[3 * blockIdx.x + 2] = t2;
  }
}

// Instances by the largest harmonic count and the largest number of
// longitudinal Ez modes (sizes of the register arrays).
typedef void (*PushKernel)(BatchLaunch);
template <int LM>
PushKernel push_kernel_l(int H) {
  if (H <= 1) return k_batch_push<1, LM>;
  if (H <= 2) return k_batch_push<2, LM>;
  if (H <= 4) return k_batch_push<4, LM>;
  return k_batch_push<FELIS_MAX_HARMONY, LM>;
}
PushKernel push_kernel(int H, int L) { return L <= 1 ? push_kernel_l<1>(H) : push_kernel_l<4>(H); }

}  // namespace

size_t batch_adi_smem(int nx_max, int ny_max, int src_cells) {
  const int M = nx_max > ny_max ? nx_max : ny_max;
  const size_t NL = (size_t)M - 2;  // lines per chunk (the kernel's NL)
  return ((size_t)(ny_max - 2) * ((nx_max - 2) | 1) + 16 * (size_t)M + 9 * NL + (size_t)src_cells) * sizeof(float2);
}

int batch_adi_threads(int nx, int ny) {
  const int m = (nx > ny ? nx : ny) - 2;
  return ((4 * m + 31) / 32) * 32;  // four chunks of m lines, whole warps
}

size_t batch_push_smem(int nsrc_max, int LF_max, int nr_max, int box_cells) {
  const size_t head = (((size_t)LF_max * nr_max * sizeof(float2) + 15) & ~(size_t)15) +
                      (((size_t)LF_max * nr_max * 2 * sizeof(acc_t) + 15) & ~(size_t)15);
  size_t area = (size_t)nsrc_max * box_cells * 2 * sizeof(acc_t);  // a (re, im) pair per cell and plane
  const size_t thomas = (size_t)LF_max * nr_max * 4 * sizeof(double);  // d re, d im, b, w per point
  if (thomas > area) area = thomas;
  return head + area;
}

cudaError_t batch_set_smem(int H, int L, int adi_bytes, int push_bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_batch_adi, cudaFuncAttributeMaxDynamicSharedMemorySize, adi_bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(push_kernel(H, L), cudaFuncAttributeMaxDynamicSharedMemorySize, push_bytes);
  return e;
}

int batch_resident_adi(int threads, int smem_bytes) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_adi, threads, smem_bytes) != cudaSuccess) return 0;
  return n;
}

namespace {
__global__ void k_f64_to_f32(const double* __restrict__ src, float* __restrict__ dst, int64_t n, double off) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)(src[i] - off);
}
__global__ void k_f32_to_f64(const float* __restrict__ src, double* __restrict__ dst, int64_t n, double off) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = off + (double)src[i];
}
// slices [s0, s0 + ns) of one (harmonic, pol) field from the reference
// layout (complex FP64, plane s at src + (s - s0) N) into the ring
__global__ void k_field_to_f32(const double2* __restrict__ src, float2* __restrict__ U, int s0, int ns, int S, int N,
                               int ring_base) {
  const int64_t tot = (int64_t)ns * N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int s = s0 + (int)(i / N), k = (int)(i % N);
    const double2 v = src[i];
    U[(size_t)((s + ring_base) % S) * N + k] = make_float2((float)v.x, (float)v.y);
  }
}
}  // namespace

cudaError_t launch_f64_to_f32(const double* src, float* dst, int64_t n, double off, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + 255) / 256;
  k_f64_to_f32<<<(int)(blocks < 4736 ? blocks : 4736), 256, 0, st>>>(src, dst, n, off);
  return cudaGetLastError();
}

cudaError_t launch_f32_to_f64(const float* src, double* dst, int64_t n, double off, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int64_t blocks = (n + 255) / 256;
  k_f32_to_f64<<<(int)(blocks < 4736 ? blocks : 4736), 256, 0, st>>>(src, dst, n, off);
  return cudaGetLastError();
}

cudaError_t launch_field_to_f32(const double* src, float2* U, int s0, int ns, int S, int N, int ring_base,
                                cudaStream_t st) {
  const int64_t tot = (int64_t)ns * N;
  if (tot <= 0) return cudaSuccess;
  const int64_t blocks = (tot + 255) / 256;
  k_field_to_f32<<<(int)(blocks < 4736 ? blocks : 4736), 256, 0, st>>>(reinterpret_cast<const double2*>(src), U, s0,
                                                                        ns, S, N, ring_base);
  return cudaGetLastError();
}

void launch_batch_adi(const BatchLaunch& a, int threads, cudaStream_t st) {
  if (a.nwork > 0) k_batch_adi<<<a.nwork, threads, a.smem_bytes, st>>>(a);
}

void launch_batch_push(const BatchLaunch& a, int H, int L, cudaStream_t st) {
  if (a.nwork > 0) push_kernel(H, L)<<<a.nwork, kPushThreads, a.smem_bytes, st>>>(a);
}

void launch_batch_measure(const BInst* inst, const BStep* step, const int4* work, int nwork, cudaStream_t st) {
  if (nwork > 0) k_batch_measure<<<nwork < 1184 ? nwork : 1184, 256, 0, st>>>(inst, step, work, nwork);
}

void launch_batch_reduce(const BInst* inst, int ninst, const BStep* step, double* hist_e, double* hist_t,
                         double* hist_b, int se, int st_, int sb, cudaStream_t st) {
  k_batch_reduce<<<ninst, 256, 0, st>>>(inst, step, hist_e, hist_t, hist_b, se, st_, sb);
}

void launch_batch_spectrum(const BInst* inst, int ninst, const int* ring, int hidx, double* out, cudaStream_t st) {
  if (ninst > 0) k_batch_spectrum<<<ninst, 256, 0, st>>>(inst, ring, hidx, out);
}

}  // namespace felis
