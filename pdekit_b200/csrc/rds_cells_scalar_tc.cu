// Mixed-precision cell residual kernel for the scalar 2D physics with the basis contractions on
// the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// The FP32 cell kernel (rds_cells_scalar.cu) spends about 40 % of its arithmetic on three dense
// contractions per cell that share their right operand across all cells of an element type:
//   states at the p+1 flux nodes and at the quadrature points   S = dU [Vsf | V]^T
//   reference derivatives of the flux at the quadrature points  D = dF dVf^T  (block form)
// (src/interpolation/FluxSpaceMetric.hpp:545-746, SolutionSpaceMetric.hpp:288-327). Here a CTA
// of 128 threads takes 128 cells, one cell per TMEM lane, and issues both products as
// tcgen05.mma kind::tf32 (M = 128 cells, N = table columns, K = 8 per instruction) from shared
// memory. Each operand is split into a TF32 high part and a TF32 remainder and three products
// are accumulated in FP32 (hi*hi + hi*lo + lo*hi), which keeps the contraction at FP32 accuracy.
// The dofs enter in the deviation form of the FP32 path (u_n - u_0 in FP64, then FP32), so the
// products are small differences; everything after the contraction (fluxes, upwind coefficients,
// the FP64 inverse, the FP64 LDA / N accumulation, blending, wave speed) is the FP32 path's.
//
// Operand layout: K-major without swizzle, the canonical layout of 8-row x 16-byte core
// matrices: element (r, k) at byte (r / 8) * SBO + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4
// with LBO = 128 (next 16-byte column chunk) and SBO = K / 4 * 128 (next 8-row group).
//
// The CTAs are persistent over 128-cell tiles (the batch form walks the active tiles of the
// problems still iterating). TMEM is allocated once per CTA and released before the CTA exits on
// every path; the wait for the tensor-core commit is bounded and reports a status bit.
//
// Measured on B200 (configuration 2, Burgers P2 B, 524,288 cells): 64 us per launch against
// 42 us for the CUDA-core FP32 kernel -- the contractions are only 6-10 wide in K, and the two
// synchronised tensor-core round trips per tile cost more than the ~380 FMAs per cell they
// replace. The path is therefore opt-in (option "tensor_cores").

#include <cstdint>
#include <cstring>
#include <vector>

#include "rds_internal.h"
#include "rds_tables.cuh"

namespace rds
{

namespace
{

constexpr int kTcCells = 128; // cells per tile = TMEM lanes = threads per CTA

__host__ __device__ constexpr int round_up(int x, int m)
{
  return (x + m - 1) / m * m;
}

// Sizes of the two products for an element type.
template <int NDOF, int NQ, int NFL>
struct TcDims
{
  static constexpr int K1   = round_up(NDOF, 8);      // dofs
  static constexpr int N1   = round_up(NFL + NQ, 16); // flux nodes, then points
  static constexpr int K2   = round_up(2 * NFL, 8);   // F0 at flux nodes, then F1
  static constexpr int N2   = round_up(4 * NQ, 16);   // (q, [dxi F0, deta F0, dxi F1, deta F1])
  static constexpr int COLS = (N1 + N2) <= 32 ? 32 : (N1 + N2) <= 64 ? 64 : 128;
  // shared memory: A operand (hi, lo) sized for the larger K, B1 and B2 (hi, lo)
  static constexpr int KA     = K1 > K2 ? K1 : K2;
  static constexpr int TABLES = 2 * N1 * K1 + 2 * N2 * K2; // floats of the group's device table
  static constexpr int SMEM   = (2 * kTcCells * KA + TABLES) * 4; // bytes
};

__host__ __device__ inline int kmajor_off(int r, int k, int K)
{
  return (r >> 3) * (K / 4 * 128) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

// ---- tcgen05 / mbarrier primitives (inline PTX) ------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46; // descriptor version of sm_100; base offset 0; no swizzle
  return d;
}

// kind::tf32 instruction descriptor: D F32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
  const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0; // no output lanes disabled
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
               :
               : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0),
                 "r"(m1), "r"(m2), "r"(m3));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, int limit = 1 << 22)
{
  // bounded: every try_wait suspends for a limited time; give up after `limit` tries
  for (int i = 0; i < limit; ++i)
  {
    uint32_t done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}\n"
                 : "=r"(done)
                 : "r"(mbar), "r"(phase)
                 : "memory");
    if (done)
      return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4])
{
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 4; ++i)
    v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld()
{
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float to_tf32(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// ---- the kernel --------------------------------------------------------------------------------

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, bool BATCH>
__global__ void __launch_bounds__(kTcCells)
    cells_scalar2d_tc(const __grid_constant__ CellArgs a,
                      const __grid_constant__ Tables<float, 2, NDOF, NQ, NFL, 3> tb,
                      const float *__restrict__ btab, int ntiles)
{
  using TD = TcDims<NDOF, NQ, NFL>;
  using T  = float;
  extern __shared__ __align__(128) unsigned char smem[];
  float *sAh  = reinterpret_cast<float *>(smem);
  float *sAl  = sAh + kTcCells * TD::KA;
  float *sB1h = sAl + kTcCells * TD::KA;
  float *sB1l = sB1h + TD::N1 * TD::K1;
  float *sB2h = sB1l + TD::N1 * TD::K1;
  float *sB2l = sB2h + TD::N2 * TD::K2;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t mbar_idle; // nothing arrives on it (the timeout test)
  __shared__ uint32_t tmem_base;

  const int tid  = threadIdx.x;
  const int warp = tid >> 5;
  if (*a.stop)
    return; // uniform over the grid: before any TMEM allocation

  // tables (pre-split, already in the operand layout) into shared memory
  for (int i = tid; i < TD::TABLES; i += kTcCells)
    sB1h[i] = __ldg(btab + i);
  if (tid == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar_idle)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_addr(&tmem_base)), "r"(TD::COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem  = tmem_base;
  const uint32_t tlane = tmem + (uint32_t(warp * 32) << 16); // this warp's 32 TMEM lanes
  const uint32_t mb    = smem_addr(&mbar);
  uint32_t phase       = 0;
  bool timed_out       = false;
  // test of the bounded-wait path: a limited wait on a barrier that nothing completes runs out,
  // and the kernel goes on as after a timed-out commit (status bit, TMEM released)
  if (a.tc_test_wait > 0 && !mbar_wait(smem_addr(&mbar_idle), 0u, a.tc_test_wait))
    timed_out = true;

  const uint32_t aAh = smem_addr(sAh), aAl = smem_addr(sAl);
  const uint32_t aB1h = smem_addr(sB1h), aB1l = smem_addr(sB1l);
  const uint32_t aB2h = smem_addr(sB2h), aB2l = smem_addr(sB2l);

  if (BATCH)
    ntiles = a.bt.prefix[a.bt.nprob]; // active tiles, rebuilt on the device
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
  {
    // ---- this thread's cell
    int c = -1;
    if (BATCH)
    {
      const int32_t *prefix = a.bt.prefix;
      int lo = 0, hi = a.bt.nprob;
      while (hi - lo > 1)
      {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= t)
          lo = mid;
        else
          hi = mid;
      }
      const int cc = a.bt.cbeg[lo] + (t - prefix[lo]) * kTcCells + tid;
      c            = cc < a.bt.cend[lo] ? cc : -1;
    }
    else
    {
      const int cc = t * kTcCells + tid;
      c            = cc < a.ncells ? cc : -1;
    }
    const bool live = c >= 0;

    // ---- states (deviation form) and geometry
    double ud[NDOF];
    T dn[NDOF];
    T X0[3], X1[3];
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      ud[n] = live ? __ldg(a.u + __ldg(a.sol_conn + (size_t)n * a.ncells + c)) : 0.0;
      dn[n] = T(ud[n] - ud[0]);
    }
    {
      double xg0 = 0.0, yg0 = 0.0;
#pragma unroll
      for (int g = 0; g < 3; ++g)
      {
        const int v     = live ? __ldg(a.geo_conn + (size_t)g * a.ncells + c) : 0;
        const double xg = live ? __ldg(a.X + v) : double(g == 1);
        const double yg = live ? __ldg(a.X + a.ngeo_nodes + v) : double(g == 2);
        if (g == 0)
        {
          xg0 = xg;
          yg0 = yg;
        }
        X0[g] = T(xg - xg0);
        X1[g] = T(yg - yg0);
      }
    }
    const T u0 = T(ud[0]);

    // ---- product 1: [flux-node states | point states] (deviations) = dn [Vsf | V]^T
#pragma unroll
    for (int k = 0; k < TD::K1; ++k)
    {
      const T x                           = k < NDOF ? dn[k < NDOF ? k : 0] : T(0);
      const T xh                          = to_tf32(x);
      sAh[kmajor_off(tid, k, TD::K1) / 4] = xh;
      sAl[kmajor_off(tid, k, TD::K1) / 4] = to_tf32(x - xh);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0)
    {
      tc_fence_after();
      const uint32_t id = idesc_tf32(kTcCells, TD::N1);
      const uint32_t sa = TD::K1 / 4 * 128, sb = TD::K1 / 4 * 128;
#pragma unroll
      for (int s = 0; s < TD::K1 / 8; ++s)
      {
        const uint32_t off = s * 256;
        mma_tf32(tmem, smem_desc(aAh + off, 128, sa), smem_desc(aB1h + off, 128, sb), id, s > 0);
        mma_tf32(tmem, smem_desc(aAh + off, 128, sa), smem_desc(aB1l + off, 128, sb), id, 1);
        mma_tf32(tmem, smem_desc(aAl + off, 128, sa), smem_desc(aB1h + off, 128, sb), id, 1);
      }
      mma_commit(mb);
    }
    if (!mbar_wait(mb, phase))
      timed_out = true;
    phase ^= 1u;
    tc_fence_after();

    T sf[NFL], uqd[NQ];
    // columns 0 .. NFL-1: flux-node states, NFL .. NFL+NQ-1: point states
#pragma unroll
    for (int j = 0; j < TD::N1; j += 4)
    {
      float v[4];
      tmem_ld4(tlane + j, v);
      tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 4; ++i)
      {
        const int col = j + i;
        if (col < NFL)
          sf[col < NFL ? col : 0] = v[i];
        else if (col < NFL + NQ)
          uqd[(col >= NFL && col - NFL < NQ) ? col - NFL : 0] = v[i];
      }
    }

    // ---- product 2: flux derivatives at the points from the flux deviations at the nodes
#pragma unroll
    for (int k = 0; k < TD::K2; ++k)
    {
      T x = T(0);
      if (k < NFL)
      {
        const T s = sf[k < NFL ? k : 0];
        x         = (PHYS == RDS_BURGERS2D) ? s * (u0 + T(0.5) * s) : T(a.adv0) * s;
      }
      else if (k < 2 * NFL)
      {
        const T s = sf[(k >= NFL && k - NFL < NFL) ? k - NFL : 0];
        x         = (PHYS == RDS_BURGERS2D) ? s : T(a.adv1) * s;
      }
      const T xh                          = to_tf32(x);
      sAh[kmajor_off(tid, k, TD::K2) / 4] = xh;
      sAl[kmajor_off(tid, k, TD::K2) / 4] = to_tf32(x - xh);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0)
    {
      tc_fence_after();
      const uint32_t id = idesc_tf32(kTcCells, TD::N2);
      const uint32_t sa = TD::K2 / 4 * 128, sb = TD::K2 / 4 * 128;
      const uint32_t d  = tmem + TD::N1;
#pragma unroll
      for (int s = 0; s < TD::K2 / 8; ++s)
      {
        const uint32_t off = s * 256;
        mma_tf32(d, smem_desc(aAh + off, 128, sa), smem_desc(aB2h + off, 128, sb), id, s > 0);
        mma_tf32(d, smem_desc(aAh + off, 128, sa), smem_desc(aB2l + off, 128, sb), id, 1);
        mma_tf32(d, smem_desc(aAl + off, 128, sa), smem_desc(aB2h + off, 128, sb), id, 1);
      }
      mma_commit(mb);
    }
    if (!mbar_wait(mb, phase))
      timed_out = true;
    phase ^= 1u;
    tc_fence_after();

    // ---- the rest of the cell residual (the FP32 path of rds_cells_scalar.cu)
    T ij00, ij01, ij10, ij11, detj;
    {
      T J00 = tb.dVgeo[0][0][0] * X0[0], J01 = tb.dVgeo[0][0][0] * X1[0];
      T J10 = tb.dVgeo[1][0][0] * X0[0], J11 = tb.dVgeo[1][0][0] * X1[0];
#pragma unroll
      for (int g = 1; g < 3; ++g)
      {
        J00 = J00 + tb.dVgeo[0][0][g] * X0[g];
        J01 = J01 + tb.dVgeo[0][0][g] * X1[g];
        J10 = J10 + tb.dVgeo[1][0][g] * X0[g];
        J11 = J11 + tb.dVgeo[1][0][g] * X1[g];
      }
      detj            = J00 * J11 - J01 * J10;
      const T inv_det = T(1) / detj;
      ij00            = inv_det * J11;
      ij11            = inv_det * J00;
      ij01            = -inv_det * J01;
      ij10            = -inv_det * J10;
    }
    double lda[NDOF], diss[NDOF];
#pragma unroll
    for (int n = 0; n < NDOF; ++n)
    {
      lda[n]  = 0.0;
      diss[n] = 0.0;
    }
    double phi = 0.0, vol = 0.0;
    T wsmax    = T(0);
#pragma unroll
    for (int q = 0; q < NQ; ++q)
    {
      float dq[4];
      tmem_ld4(tlane + TD::N1 + 4 * q, dq);
      tmem_wait_ld();
      const T wjT     = tb.w[q] * detj;
      const double wj = double(wjT);
      vol += wj;
      const T rT      = (ij00 * dq[0] + ij01 * dq[1]) + (ij10 * dq[2] + ij11 * dq[3]);
      const double rq = double(rT);
      T ax, ay;
      if (PHYS == RDS_BURGERS2D)
      {
        ax = u0 + uqd[q];
        ay = T(1);
      }
      else
      {
        ax = T(a.adv0);
        ay = T(a.adv1);
      }
      T kp[NDOF];
      T sumkp = T(0);
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
      {
        const T gx = ij00 * tb.dV[0][q][n] + ij01 * tb.dV[1][q][n];
        const T gy = ij10 * tb.dV[0][q][n] + ij11 * tb.dV[1][q][n];
        const T k  = ax * gx + ay * gy;
        kp[n]      = k > T(0) ? k : T(0);
        wsmax      = fmax(wsmax, fmax(T(1.e-6), fabs(k)));
        sumkp      = sumkp + kp[n];
      }
      const double inv = 1.0 / double(sumkp);
      phi += wj * rq;
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
        lda[n] += wj * ((double(kp[n]) * inv) * rq);
      if (SCHEME != RDS_PGLDA)
      {
        double tku = 0.0;
#pragma unroll
        for (int m = 0; m < NDOF; ++m)
          tku += double(kp[m]) * ud[m];
        const double sk = double(sumkp);
#pragma unroll
        for (int n = 0; n < NDOF; ++n)
          diss[n] += wj * ((double(kp[n]) * inv) * (ud[n] * sk - tku));
      }
    }
    double theta = 1.0;
    if (SCHEME == RDS_PGB)
    {
      double abs_phiN = 0.0;
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
        abs_phiN += fabs(lda[n] + diss[n]);
      theta = fabs(phi) / (abs_phiN + 1.e-6);
    }
    if (live)
    {
      double *out = a.contrib + a.slot_base + c;
#pragma unroll
      for (int n = 0; n < NDOF; ++n)
        out[(size_t)n * a.ncells] = (SCHEME == RDS_PGLDA) ? lda[n] : lda[n] + theta * diss[n];
      a.wsc[a.ws_base + c] = vol * double(wsmax);
    }
    // TMEM is rewritten by the next tile's products: every lane's loads are complete here
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }

  if (timed_out)
    atomicOr(a.status, kFlagTimeout);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TD::COLS));
}

// ---- host side ------------------------------------------------------------------------------

// FP32 value rounded to TF32 (10-bit mantissa, round to nearest, ties away from zero).
float host_tf32(float x)
{
  uint32_t b;
  std::memcpy(&b, &x, 4);
  b = (b + 0x1000u) & ~0x1FFFu;
  float y;
  std::memcpy(&y, &b, 4);
  return y;
}

template <int NDOF, int NQ, int NFL>
void build_tables(const HostCellGroup &g, std::vector<float> &out)
{
  using TD = TcDims<NDOF, NQ, NFL>;
  out.assign(TD::TABLES, 0.0f);
  float *B1h = out.data(), *B1l = B1h + TD::N1 * TD::K1;
  float *B2h = B1l + TD::N1 * TD::K1, *B2l = B2h + TD::N2 * TD::K2;
  auto put = [](float *hi, float *lo, int r, int k, int K, double v) {
    const float f = float(v), h = host_tf32(f);
    hi[kmajor_off(r, k, K) / 4] = h;
    lo[kmajor_off(r, k, K) / 4] = host_tf32(f - h);
  };
  // B1 rows: flux nodes (Vsf) then points (V); columns: dofs
  for (int f = 0; f < NFL; ++f)
    for (int n = 0; n < NDOF; ++n)
      put(B1h, B1l, f, n, TD::K1, g.Vsf[f * NDOF + n]);
  for (int q = 0; q < NQ; ++q)
    for (int n = 0; n < NDOF; ++n)
      put(B1h, B1l, NFL + q, n, TD::K1, g.V[q * NDOF + n]);
  // B2 rows (q, j): j = 0 dxi F0, 1 deta F0, 2 dxi F1, 3 deta F1; columns: F0 nodes, F1 nodes
  for (int q = 0; q < NQ; ++q)
    for (int f = 0; f < NFL; ++f)
    {
      const double dx = g.dVf[(0 * NQ + q) * NFL + f], dy = g.dVf[(1 * NQ + q) * NFL + f];
      put(B2h, B2l, 4 * q + 0, f, TD::K2, dx);
      put(B2h, B2l, 4 * q + 1, f, TD::K2, dy);
      put(B2h, B2l, 4 * q + 2, NFL + f, TD::K2, dx);
      put(B2h, B2l, 4 * q + 3, NFL + f, TD::K2, dy);
    }
}

template <int PHYS, int SCHEME, int NDOF, int NQ, int NFL, bool BATCH>
cudaError_t launch_tc_one(const HostCellGroup &g, const CellArgs &a, int grid, int ntiles,
                          cudaStream_t s)
{
  using TD = TcDims<NDOF, NQ, NFL>;
  Tables<float, 2, NDOF, NQ, NFL, 3> tb;
  fill_tables(tb, g.w, g.V, g.dV, g.dVgeo, g.dVf, g.Vsf);
  auto k               = cells_scalar2d_tc<PHYS, SCHEME, NDOF, NQ, NFL, BATCH>;
  static bool attr_set = false;
  if (!attr_set)
  {
    const cudaError_t e =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, TD::SMEM);
    if (e != cudaSuccess)
      return e;
    attr_set = true;
  }
  k<<<grid, kTcCells, TD::SMEM, s>>>(a, tb, g.d_tc, ntiles);
  return cudaGetLastError();
}

template <int PHYS, int SCHEME, bool BATCH>
cudaError_t dispatch_tc(const HostCellGroup &g, const CellArgs &a, int grid, int ntiles,
                        cudaStream_t s, bool *ok)
{
  const rds_cell_group &d = g.desc;
  *ok                     = g.d_tc != nullptr;
  if (!*ok)
    return cudaSuccess;
  if (d.ndof == 3 && d.nq == 6 && d.nfl == 6)
    return launch_tc_one<PHYS, SCHEME, 3, 6, 6, BATCH>(g, a, grid, ntiles, s);
  if (d.ndof == 6 && d.nq == 7 && d.nfl == 10)
    return launch_tc_one<PHYS, SCHEME, 6, 7, 10, BATCH>(g, a, grid, ntiles, s);
  if (d.ndof == 10 && d.nq == 16 && d.nfl == 15)
    return launch_tc_one<PHYS, SCHEME, 10, 16, 15, BATCH>(g, a, grid, ntiles, s);
  *ok = false;
  return cudaSuccess;
}

} // namespace

bool tc_supported(const HostCellGroup &g)
{
  const rds_cell_group &d = g.desc;
  if (!(g.affine && d.shape == RDS_TRIAG && d.ngeo == 3))
    return false;
  if (g.physics != RDS_ADVECTION_CONST && g.physics != RDS_BURGERS2D)
    return false;
  return (d.ndof == 3 && d.nq == 6 && d.nfl == 6) || (d.ndof == 6 && d.nq == 7 && d.nfl == 10) ||
         (d.ndof == 10 && d.nq == 16 && d.nfl == 15);
}

void tc_tables(const HostCellGroup &g, std::vector<float> &out)
{
  const rds_cell_group &d = g.desc;
  out.clear();
  if (!tc_supported(g))
    return;
  if (d.ndof == 3)
    build_tables<3, 6, 6>(g, out);
  else if (d.ndof == 6)
    build_tables<6, 7, 10>(g, out);
  else
    build_tables<10, 16, 15>(g, out);
}

cudaError_t launch_cells_scalar_tc(const HostCellGroup &g, const CellArgs &a, bool batch, int grid,
                                   int ntiles, cudaStream_t s, const char **name, bool *ok)
{
  static const char *names[2][3] = {{"cells_adv_lda_tc", "cells_adv_n_tc", "cells_adv_b_tc"},
                                    {"cells_burgers_lda_tc", "cells_burgers_n_tc",
                                     "cells_burgers_b_tc"}};
  const int physics = g.physics, scheme = g.scheme;
  *ok               = false;
  if (!tc_supported(g) || scheme < 0 || scheme > 2 || grid <= 0)
    return cudaSuccess;
  *name = names[physics == RDS_BURGERS2D][scheme];
#define RDS_TC_CASE(PH, SC)                                                                        \
  if (physics == PH && scheme == SC)                                                               \
    return batch ? dispatch_tc<PH, SC, true>(g, a, grid, ntiles, s, ok)                            \
                 : dispatch_tc<PH, SC, false>(g, a, grid, ntiles, s, ok);
  RDS_TC_CASE(RDS_ADVECTION_CONST, RDS_PGLDA)
  RDS_TC_CASE(RDS_ADVECTION_CONST, RDS_PGN)
  RDS_TC_CASE(RDS_ADVECTION_CONST, RDS_PGB)
  RDS_TC_CASE(RDS_BURGERS2D, RDS_PGLDA)
  RDS_TC_CASE(RDS_BURGERS2D, RDS_PGN)
  RDS_TC_CASE(RDS_BURGERS2D, RDS_PGB)
#undef RDS_TC_CASE
  return cudaSuccess;
}

} // namespace rds
