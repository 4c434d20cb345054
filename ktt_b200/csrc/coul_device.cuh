// coul_device.cuh -- device-side building blocks of the direct Coulomb summation kernels (sm_100a).
//
// The path computes V(r_i) = sum_j q_j / |r_i - r_j| on a regular grid, the sum that KTT's
// directCoulombSum kernels evaluate (Examples/CoulombSum3d/CoulombSum3d.cu:1-47,
// Examples/CoulombSum2d/CoulombSum2dSimple.cl:29-79).  The B200 design:
//   * atoms stream through shared memory in tiles of kTileAtoms float4 (x, y, z, q), fetched by
//     one elected thread with TMA bulk copies (cp.async.bulk, local GPU memory, no multicast)
//     into a kStages-deep ring guarded by mbarriers; every thread reads each atom as a
//     shared-memory broadcast;
//   * each thread owns XP grid points along x (stored as one float/float2/float4 vector) and ZI
//     points along z (KTT's Z_ITERATIONS), so one atom read feeds XP*ZI pair evaluations and the
//     per-atom differences dx, dy, dz are amortised over the block;
//   * per pair: r2 = fma(dz, dz, dx^2 + dy^2) (one FP32 op), rsqrt on the MUFU unit or, for a
//     static share of the pairs, Newton iterations on the FMA pipe, then acc = fma(q, 1/r, acc);
//   * accumulation forms: plain FP32, FP32 sub-tile partials merged by two-sum, or merged into
//     FP64 (precision modes of coulktt.h);
//   * every wait on an mbarrier is bounded (iteration cap + globaltimer deadline); on expiry the
//     kernel records a status word, drains, and returns instead of hanging or trapping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace coul {

constexpr int kTileAtoms = 256;       // atoms per shared-memory stage
constexpr int kStages = 2;            // depth of the TMA ring
constexpr int kSubTile = 32;          // a ragged last stage is evaluated in whole sub-tiles of this many
constexpr int kMergeAtoms = 64;       // atoms per FP32 partial in the compensated / FP64-merge forms
constexpr int kMaxThreads = 256;      // launch bound of the forward kernels
constexpr int kConstAtoms = 4096;     // atoms per __constant__ chunk (64 KiB)
constexpr uint64_t kWaitBudgetNs = 1000000000ull;  // 1 s: a tile copy from L2 takes microseconds
constexpr float kPadCoord = 1.0e18f;  // padding atoms sit far away with zero charge

enum : int { kStatusOk = 0, kStatusTimeout = 1 };

enum : int { kModeGrid3d = 0, kModeSlice2d = 1 };

struct FwdParams {
    const float4* atoms;  // AoS: (x, y, z, q), or (x, y, dz2, q) for 2D slices
    const float* sx;      // SoA arrays (layout 1)
    const float* sy;
    const float* sz;
    const float* sq;
    int64_t n_atoms;
    int nx, ny, nz;
    int z_base;  // 3D: global z index of the output's first slice (0 for a whole map; slabs of a
                 // sharded map start later); points z in [z_base, nz) are evaluated
    float h, ox, oy, oz;
    float* out;
    int accumulate;
    int* status;
};

// ------------------------------------------------------------------------------------------
// PTX helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Device-scope atomic add with acquire-release semantics; returns the old value.
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Orders this thread's generic-proxy shared-memory accesses before later async-proxy (TMA) ones.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// TMA bulk copy global -> shared (this CTA), completion signalled on bar as transaction bytes.
// Requires 16-byte aligned src/dst and a byte count that is a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase with the given parity: true when it completed, false on expiry
// (after budget_ns of globaltimer time or 2^24 polls, whichever comes first).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint64_t budget_ns = kWaitBudgetNs)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 1; it < (1u << 24); ++it) {
        if (mbar_try_wait(bar, parity))
            return true;
        if ((it & 63u) == 0 && globaltimer_ns() - t0 > budget_ns)
            return false;
    }
    return false;
}

__device__ __forceinline__ void report_status(int* status, int code)
{
    if (status != nullptr)
        atomicCAS(status, kStatusOk, code);
}

// Thread-block clusters: this CTA's rank and the cluster's size, the cluster-wide barrier (a
// hardware barrier: every thread of every CTA of the cluster arrives, release/acquire ordering of
// shared-memory writes), and loads from a peer CTA's shared memory (distributed shared memory).
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ uint32_t cluster_size()
{
    uint32_t n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return n;
}

__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Address of `p` (this CTA's shared memory) in the shared-memory window of cluster CTA `rank`.
__device__ __forceinline__ uint32_t cluster_map(const void* p, uint32_t rank)
{
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}

__device__ __forceinline__ float ld_cluster_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}

// MUFU reciprocal square root (approximate, flush-to-zero), the instruction KTT's kernels reach
// through rsqrt()/half_rsqrt() under fast-math.
__device__ __forceinline__ float rsqrt_mufu(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ------------------------------------------------------------------------------------------
// FMA-pipe reciprocal square root.
//
// Initial estimate by the integer "magic constant" method (Blinn 1997; Lomont, "Fast Inverse
// Square-Root", 2003): reinterpret x as an integer, halve it and subtract it from a constant, which
// approximates -log2(x)/2 piecewise linearly.  Two steps of the Newton-Raphson form
//     y <- y * (a_k - x * y^2),   written  y <- y * fma(x, y * y, -a_k)
// follow; the textbook iteration is y (3/2 - (x/2) y^2) with Lomont's constant (error in
// [-4.7e-6, 0]).  Writing the steps with -a_k keeps x itself as the argument -- the r^2 the MUFU
// path forms anyway -- and the two sign flips cancel.  The constant and a_1 are chosen jointly to
// minimise the spread of the first step's relative error (+-6.5e-4), the analytic-constant
// approach of Moroz, Walczyk et al., "Fast calculation of inverse square root with the use of magic
// constant -- analytical approach" (2018); a_2 = 3 lambda^2 re-centres the second step on the first
// step's scale lambda, so the result is 1/sqrt(x) times a constant, whose reciprocal (with the
// centring of the residual one-signed error) the kernels fold into the charge: q * kSoftRsqrtScale,
// no cost per pair.  2 integer + 6 FP32 instructions; relative error in [-3.9e-7, +4.6e-7] over all
// normal inputs.  Derivation and exhaustive FP32 check: ktt_b200/soft_rsqrt.py.
// ------------------------------------------------------------------------------------------
constexpr uint32_t kSoftRsqrtMagic = 0x5f1ed000u;
constexpr float kSoftRsqrtA1 = 2.3597500324f;
constexpr float kSoftRsqrtA2 = 5.8324427605f;
constexpr float kSoftRsqrtScale = 0.1844490021f;

// Returns 1 / (kSoftRsqrtScale * sqrt(x)) (the caller multiplies by kSoftRsqrtScale).
__device__ __forceinline__ float rsqrt_fma(float x)
{
    float y = __uint_as_float(kSoftRsqrtMagic - (__float_as_uint(x) >> 1));
    float t = y * y;
    t = fmaf(x, t, -kSoftRsqrtA1);
    y = y * t;
    t = y * y;
    t = fmaf(x, t, -kSoftRsqrtA2);
    return y * t;
}

__device__ __forceinline__ float2 splat(float v) { return make_float2(v, v); }

// Two lanes at once with sm_100's packed FP32 instructions; lane-wise identical to rsqrt_fma.
__device__ __forceinline__ float2 rsqrt_fma_x2(float2 x)
{
    float2 y = make_float2(__uint_as_float(kSoftRsqrtMagic - (__float_as_uint(x.x) >> 1)),
                           __uint_as_float(kSoftRsqrtMagic - (__float_as_uint(x.y) >> 1)));
    float2 t = __fmul2_rn(y, y);
    t = __ffma2_rn(x, t, splat(-kSoftRsqrtA1));
    y = __fmul2_rn(y, t);
    t = __fmul2_rn(y, y);
    t = __ffma2_rn(x, t, splat(-kSoftRsqrtA2));
    return __fmul2_rn(y, t);
}

// ------------------------------------------------------------------------------------------
// Pair blocks: one atom against a thread's register block of grid points.
//
// Points along the blocked axis (z in 3D, y in 2D) are held in pairs, so the per-pair FP32 work
// -- r^2 = fma(d, d, w) and acc = fma(q, 1/r, acc) -- is issued as packed FFMA2 instructions, one
// issue slot for two pairs.  The reciprocal square roots go to the MUFU unit one lane at a time,
// or, for a static share of the lane pairs, to the FMA pipe (rsqrt_fma_x2).
// ------------------------------------------------------------------------------------------
// Static split between the MUFU unit and the FMA pipe.  A thread evaluates NP = x_points *
// ceil(z_iterations / 2) lane pairs per atom.  Within one stage of the atom stream (kTileAtoms atoms)
// every lane pair keeps one form for all atoms, so the form's bias scales that point's partial sum
// and cannot correlate with a pattern in the charges.  Stages (in the atom-split form also the
// warps of a CTA) take turns in a pattern of soft_group(NP) = max(1, 8 / NP) phases, which together
// hold 8 (or, for NP >= 8, NP) pair slots;
// slot s = (stage phase) * NP + p for NP < 8, s = p % 8 otherwise, and a slot takes the FMA pipe
// when s < SOFT.  The share is SOFT / 8 at every tile size.  From kSoftAlternate on
// (SOFT = kSoftAlternate + k) two such patterns alternate between k and k + 1 soft slots, a share
// of (2k + 1) / 16.  soft_phases is the number of stage phases of one whole pattern.
constexpr int kSoftAlternate = 10;
constexpr int soft_group(int np) { return np >= 8 ? 1 : 8 / np; }
constexpr int soft_phases(int soft, int np)
{
    return soft == 0 ? 1 : (soft >= kSoftAlternate ? 2 : 1) * soft_group(np);
}

// Calls f(std::integral_constant<int, phase>) for a run-time phase in [0, P): the stage loop is
// instantiated once per phase so that the soft/MUFU choice stays a compile-time one per pair.
template <int P, int G = 0, class F>
__device__ __forceinline__ void with_phase(const int phase, F&& f)
{
    if constexpr (G + 1 < P) {
        if (phase == G)
            f(std::integral_constant<int, G>{});
        else
            with_phase<P, G + 1>(phase, f);
    } else {
        f(std::integral_constant<int, G>{});
    }
}

template <int SOFT, int NP, int PHASE>
__device__ __forceinline__ constexpr bool pair_is_soft(int p)
{
    constexpr int G = soft_group(NP);
    constexpr int base = SOFT >= kSoftAlternate ? SOFT - kSoftAlternate + PHASE / G : SOFT;
    return (NP >= 8 ? (p & 7) : (PHASE % G) * NP + p) < base;
}

__device__ __forceinline__ float2 rsqrt_mufu_x2(float2 r2)
{
    return make_float2(rsqrt_mufu(r2.x), rsqrt_mufu(r2.y));
}

// One lane pair: acc += q / sqrt(r2) lane-wise, the rsqrt on the FMA pipe when SOFT_PAIR (the charge
// then comes pre-scaled by kSoftRsqrtScale in qs2).  HALF_PAIR: only the .x lane holds a point (an
// odd number of points along the blocked axis); it is evaluated alone, so no rsqrt is spent on a
// point that is never stored.
template <bool SOFT_PAIR, bool HALF_PAIR>
__device__ __forceinline__ void pair_update(float2 r2, float2 q2, float2 qs2, float2& acc)
{
    if constexpr (HALF_PAIR) {
        if constexpr (SOFT_PAIR)
            acc.x = fmaf(qs2.x, rsqrt_fma(r2.x), acc.x);
        else
            acc.x = fmaf(q2.x, rsqrt_mufu(r2.x), acc.x);
    } else {
        if constexpr (SOFT_PAIR)
            acc = __ffma2_rn(qs2, rsqrt_fma_x2(r2), acc);
        else
            acc = __ffma2_rn(q2, rsqrt_mufu_x2(r2), acc);
    }
}

// Unrolled k (x point), i (lane pair of the blocked axis) loops with the soft/MUFU choice and the
// half pair resolved at compile time.  r2 per pair from the per-k term pk and the per-i term pi:
//   SQUARE_I (3D):  r2 = pi^2 + pk   (pi = dz of the two points, pk = dx^2 + dy^2)
//   else (2D):      r2 = pk^2 + pi   (pk = dx, pi = dy^2 + dz^2 of the two rows)
// Only the first ZA <= ZH lane pairs are evaluated (the rest of a tile that overhangs the grid);
// HALF marks pair ZA - 1 as holding one point.
template <bool SQUARE_I, int XP, int ZH, int ZA, int SOFT, int PHASE, bool HALF, int K = 0, int I = 0>
__device__ __forceinline__ void pair_rows(const float (&pk)[XP], const float2 (&pi)[ZH], float2 q2, float2 qs2,
                                          float2 (&acc)[XP][ZH])
{
    static_assert(ZA >= 1 && ZA <= ZH, "active pairs within the tile");
    if constexpr (K < XP) {
        if constexpr (I < ZA) {
            constexpr bool soft = SOFT != 0 && pair_is_soft<SOFT, XP * ZH, PHASE>(K * ZH + I);
            constexpr bool half = HALF && I == ZA - 1;
            if constexpr (half) {
                const float r2 = SQUARE_I ? fmaf(pi[I].x, pi[I].x, pk[K]) : fmaf(pk[K], pk[K], pi[I].x);
                pair_update<soft, true>(make_float2(r2, 0.0f), q2, qs2, acc[K][I]);
            } else {
                const float2 r2 = SQUARE_I ? __ffma2_rn(pi[I], pi[I], splat(pk[K]))
                                           : __ffma2_rn(splat(pk[K]), splat(pk[K]), pi[I]);
                pair_update<soft, false>(r2, q2, qs2, acc[K][I]);
            }
            pair_rows<SQUARE_I, XP, ZH, ZA, SOFT, PHASE, HALF, K, I + 1>(pk, pi, q2, qs2, acc);
        } else {
            pair_rows<SQUARE_I, XP, ZH, ZA, SOFT, PHASE, HALF, K + 1, 0>(pk, pi, q2, qs2, acc);
        }
    }
}

// 3D: thread owns points (gx[k], gy, gz[i].x / gz[i].y); acc[k][i] += q / |r - a| lane-wise.
template <int XP, int ZH, int ZA, int SOFT, int PHASE, bool HALF>
__device__ __forceinline__ void pair_block_3d(const float (&gx)[XP], float gy, const float2 (&gz)[ZH], float4 a,
                                              float2 (&acc)[XP][ZH])
{
    const float dy = gy - a.y;
    const float dy2 = dy * dy;
    float dxy[XP];
#pragma unroll
    for (int k = 0; k < XP; ++k) {
        const float dx = gx[k] - a.x;
        dxy[k] = fmaf(dx, dx, dy2);
    }
    float2 dz[ZH];
    const float2 naz = splat(-a.z);
#pragma unroll
    for (int i = 0; i < ZA; ++i)
        dz[i] = __fadd2_rn(gz[i], naz);
    pair_rows<true, XP, ZH, ZA, SOFT, PHASE, HALF>(dxy, dz, splat(a.w), splat(a.w * kSoftRsqrtScale), acc);
}

// 2D slice (KTT's 2D convention): thread owns points (gx[k], gy[i].x / gy[i].y) of one slice, the
// atom's .z holds the squared z distance c; acc[k][i] += q / sqrt(dx^2 + dy^2 + c) lane-wise.
template <int XP, int YH, int ZA, int SOFT, int PHASE, bool HALF>
__device__ __forceinline__ void pair_block_2d(const float (&gx)[XP], const float2 (&gy)[YH], float4 a,
                                              float2 (&acc)[XP][YH])
{
    float2 dyc[YH];
    const float2 nay = splat(-a.y);
    const float2 c2 = splat(a.z);
#pragma unroll
    for (int i = 0; i < ZA; ++i) {
        const float2 dy = __fadd2_rn(gy[i], nay);
        dyc[i] = __ffma2_rn(dy, dy, c2);
    }
    float dx[XP];
#pragma unroll
    for (int k = 0; k < XP; ++k)
        dx[k] = gx[k] - a.x;
    pair_rows<false, XP, YH, ZA, SOFT, PHASE, HALF>(dx, dyc, splat(a.w), splat(a.w * kSoftRsqrtScale), acc);
}

// ------------------------------------------------------------------------------------------
// FP64 pairs (COUL_PREC_FP64_PAIRS): the atom's FP32 coordinates and charge widened to double, every
// difference exact in FP64, r^2 by FP64 fma, the reciprocal square root from the MUFU approximation
// rsqrt.approx.ftz.f64 (relative error below 2^-20) refined by one Newton step in FP64
// (y <- y + y (1 - r^2 y^2) / 2, relative error about 1.5 * 2^-40), accumulated in FP64.  Six FP64
// operations and one MUFU instruction per pair; the FP64 pipe bounds it.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ double rsqrt_mufu_f64(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

template <int XP, int ZI>
__device__ __forceinline__ void pair_block_3d_f64(const double (&gx)[XP], double gy, const double (&gz)[ZI], float4 a,
                                                  double (&acc)[XP][ZI])
{
    const double dy = gy - static_cast<double>(a.y);
    const double dy2 = dy * dy;
    const double q = static_cast<double>(a.w);
    double dxy[XP];
#pragma unroll
    for (int k = 0; k < XP; ++k) {
        const double dx = gx[k] - static_cast<double>(a.x);
        dxy[k] = fma(dx, dx, dy2);
    }
    double dz[ZI];
#pragma unroll
    for (int m = 0; m < ZI; ++m)
        dz[m] = gz[m] - static_cast<double>(a.z);
#pragma unroll
    for (int k = 0; k < XP; ++k) {
#pragma unroll
        for (int m = 0; m < ZI; ++m) {
            const double r2 = fma(dz[m], dz[m], dxy[k]);
            double y = rsqrt_mufu_f64(r2);
            const double e = fma(-r2, y * y, 1.0);
            y = fma(y * e, 0.5, y);
            acc[k][m] = fma(q, y, acc[k][m]);
        }
    }
}

// Knuth's two-sum: s + e == a + b exactly (round-to-nearest, no contraction of additions).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

}  // namespace coul
