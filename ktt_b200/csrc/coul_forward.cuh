// coul_forward.cuh -- the forward (potential map) kernel template and its launchers.
//
// One template covers KTT's 3D kernel (Examples/CoulombSum3d/CoulombSum3d.cu:1-47) and its 2D
// slice kernel (Examples/CoulombSum2d/CoulombSum2dSimple.cl:29-79).  Template parameters:
//   ZI    grid points per thread along z (3D, KTT Z_ITERATIONS) or along y (2D)
//   XP    grid points per thread along x, contiguous, stored as one vector (KTT VECTOR_SIZE /
//         OUTER_UNROLL_FACTOR)
//   UNR   unroll of the atom loop (KTT INNER_UNROLL_FACTOR)
//   SRC   atoms from TMA-staged shared memory or from __constant__ chunks (KTT USE_CONSTANT_MEMORY)
//   SOA   atoms as one float4 array or as four float arrays (KTT USE_SOA)
//   PREC  accumulation form (coulktt.h COUL_PREC_*)
//   SOFT  of every 8 rsqrts, how many run on the FMA pipe
//   MODE  3D grid or 2D slice (KTT's 2D argument convention)
// Block shape (KTT WORK_GROUP_SIZE_X/Y) is a launch-time choice, up to kMaxThreads threads.
#pragma once

#include <vector>

#include "coul_device.cuh"

namespace coul {

enum : int { kSrcShared = 0, kSrcConstant = 1 };
enum : int { kPrecFp32 = 0, kPrecCompensated = 1, kPrecFp64Merge = 2, kPrecFp64Pairs = 3, kPrecFp64MergeShared = 4 };

// The FP64 sums of kPrecFp64MergeShared: after the TMA ring and its barriers in dynamic shared
// memory, one double per point of every thread, point-major (thread t's point i at i * threads + t:
// consecutive threads, consecutive words).
__device__ __forceinline__ double* shared_sums(unsigned char* tiles)
{
    return reinterpret_cast<double*>(tiles + kStages * kTileAtoms * 16 + kStages * 8);
}
inline size_t shared_sums_bytes(int threads, int points) { return static_cast<size_t>(threads) * points * sizeof(double); }

// Cluster sizes of the atom-split form: 2..8 are portable; 9..16 use the B200's non-portable
// cluster sizes (opted into per kernel; refused with a device-limits error where the block does not fit).
constexpr int kMaxPortableSplit = 8;
constexpr int kMaxSplit = 16;
constexpr int kMaxQueueSplit = 256;  // chunks per tile of the queue form

// Per translation unit: the constant-memory atom chunk.  Only the TU that instantiates the
// constant-memory variants uses it; it has internal linkage so no relocatable device code is needed.
static __constant__ float4 c_atoms[kConstAtoms];

// Device-memory state of the queue form of the atom split (kept in the context, grown on demand).
struct SplitQueue {
    float* partial;               // one partial block per (tile, chunk) item
    unsigned* tile_done;          // items finished per tile, zero at launch
    unsigned long long* counter;  // the item queue's head, zero at launch
    int chunks;                   // atom chunks per tile
    int ctas;                     // persistent CTAs of the launch
};

struct FwdLaunch {
    FwdParams p;
    dim3 grid;  // one entry per point tile (the cluster form multiplies grid.x by `split`)
    dim3 block;
    size_t smem;
    int vec_store;  // 1 if x-vector stores are aligned for this launch
    int split;      // atom split: chunks of the atoms per point tile (0 / 1 = none)
    SplitQueue queue;  // the queue form's device memory (unused by the other forms)
};

template <int MODE, int XP, int ZH, int SOFT, int PHASE, bool HALF, int ZA = ZH>
__device__ __forceinline__ void eval_atom(const float (&gx)[XP], float gy, const float2 (&gb)[ZH], float4 a,
                                          float2 (&dst)[XP][ZH])
{
    if constexpr (MODE == kModeGrid3d)
        pair_block_3d<XP, ZH, ZA, SOFT, PHASE, HALF>(gx, gy, gb, a, dst);
    else
        pair_block_2d<XP, ZH, ZA, SOFT, PHASE, HALF>(gx, gb, a, dst);
}

// A thread's blocked-axis points in lane pairs: (z0 + 2i, z0 + 2i + 1) in 3D (gy = the row's y),
// rows (yrow + 2i, yrow + 2i + 1) in 2D (gy unused).
template <int ZH, int MODE>
__device__ __forceinline__ void blocked_coords(const FwdParams& p, const int yrow, const int z0, float& gy,
                                               float2 (&gb)[ZH])
{
    if constexpr (MODE == kModeGrid3d) {
        gy = fmaf(static_cast<float>(yrow), p.h, p.oy);
#pragma unroll
        for (int i = 0; i < ZH; ++i)
            gb[i] = make_float2(fmaf(static_cast<float>(z0 + 2 * i), p.h, p.oz),
                                fmaf(static_cast<float>(z0 + 2 * i + 1), p.h, p.oz));
    } else {
        gy = 0.0f;
#pragma unroll
        for (int i = 0; i < ZH; ++i)
            gb[i] = make_float2(fmaf(static_cast<float>(yrow + 2 * i), p.h, p.oy),
                                fmaf(static_cast<float>(yrow + 2 * i + 1), p.h, p.oy));
    }
}

__device__ __forceinline__ float lane(const float2& v, int l) { return l == 0 ? v.x : v.y; }

// Store XP contiguous values at row[x0 .. x0+XP), vectorised when aligned, guarded at the edge.
template <int XP>
__device__ __forceinline__ void store_points(float* __restrict__ row, int x0, int nx, const float (&v)[XP],
                                             int accumulate, int vec_ok)
{
    if constexpr (XP == 1) {
        if (x0 < nx)
            row[x0] = accumulate ? row[x0] + v[0] : v[0];
    } else {
        if (vec_ok && x0 + XP <= nx) {
            if constexpr (XP == 2) {
                float2* q = reinterpret_cast<float2*>(row + x0);
                float2 w = make_float2(v[0], v[1]);
                if (accumulate) {
                    const float2 o = *q;
                    w.x += o.x;
                    w.y += o.y;
                }
                *q = w;
            } else {
#pragma unroll
                for (int c = 0; c < XP; c += 4) {
                    float4* q = reinterpret_cast<float4*>(row + x0 + c);
                    float4 w = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                    if (accumulate) {
                        const float4 o = *q;
                        w.x += o.x;
                        w.y += o.y;
                        w.z += o.z;
                        w.w += o.w;
                    }
                    *q = w;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < XP; ++k)
                if (x0 + k < nx)
                    row[x0 + k] = accumulate ? row[x0 + k] + v[k] : v[k];
        }
    }
}

// Shared-memory ring of the TMA-staged atom stream: kStages stages of kTileAtoms float4 (or four
// float arrays), followed by one mbarrier per stage.
__device__ __forceinline__ void ring_init(uint64_t* full, const int tid)
{
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < kStages; ++s)
            mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// One thread's work for one tile: accumulate the potential of its register block of points
// (x0.., yrow, z0.. in 3D; x0.., rows yrow.. in 2D) over all atoms of p into val[x][z].  With
// SRC == kSrcShared the atoms come through the CTA's TMA ring (tiles / full); gstage counts the
// ring's stages across calls, so a persistent kernel can run many tiles through one ring.  Every
// thread of the CTA must call this together (it synchronises per stage).  Returns false (on every
// thread) when a bounded wait on the ring expired; the status word is then set and val is invalid.
// ZTRIM (3D only): a tile that overhangs the grid in z evaluates only its points inside the grid;
// the number of z points in the grid (block-uniform) selects one of ZI instantiations of the stage
// loop.  Used where many small grids make such tiles common (the batched kernel).
template <int ZI, int XP, int UNR, int SRC, int SOA, int PREC, int SOFT, int MODE, bool ZTRIM = false>
__device__ __forceinline__ bool tile_accumulate(const FwdParams& p, const int x0, const int yrow, const int z0,
                                                unsigned char* tiles, uint64_t* full, uint32_t& gstage,
                                                float (&val)[XP][ZI], const uint32_t phase_base = 0)
{
    static_assert(!ZTRIM || (MODE == kModeGrid3d && SRC == kSrcShared && PREC != kPrecFp64Pairs),
                  "z trimming: 3D maps, shared-memory atoms, FP32 pairs");
    static_assert(XP == 1 || XP == 2 || XP == 4 || XP == 8, "XP must be 1, 2, 4 or 8");
    // atoms per FP32 partial of the compensated / FP64-merge forms, and the ragged stage's granularity
    constexpr int SUB =
        (PREC == kPrecCompensated || PREC == kPrecFp64Merge || PREC == kPrecFp64MergeShared) ? kMergeAtoms : kSubTile;
    static_assert(PREC != kPrecFp64MergeShared || SRC == kSrcShared, "shared-memory FP64 sums: TMA-staged atoms");
    static_assert(kTileAtoms % SUB == 0, "sub-tiles must divide the stage");

    float gx[XP];
#pragma unroll
    for (int k = 0; k < XP; ++k)
        gx[k] = fmaf(static_cast<float>(x0 + k), p.h, p.ox);
    // Blocked-axis points in lane pairs (blocked_coords).  With an odd ZI the last pair holds one
    // point (HALF), evaluated on its own.
    constexpr int ZH = (ZI + 1) / 2;
    constexpr bool HALF = (ZI & 1) != 0;
    constexpr int P = soft_phases(SOFT, XP * ZH);  // stage phases of the FMA-pipe share's pattern
    float2 gb[ZH];
    float gy;
    blocked_coords<ZH, MODE>(p, yrow, z0, gy, gb);

    float2 acc[XP][ZH];
    float2 part[XP][ZH];
    float2 cmp[XP][ZH];
    double acc64[XP][2 * ZH];
    // FP64 pairs: the point coordinates widened once (3D only)
    static_assert(PREC != kPrecFp64Pairs || (MODE == kModeGrid3d && SOFT == 0 && SRC == kSrcShared),
                  "FP64 pairs: 3D maps, MUFU estimate, shared-memory atoms");
    double gxd[XP], gzd[ZI], accd[XP][ZI];
    const double gyd = static_cast<double>(gy);
#pragma unroll
    for (int k = 0; k < XP; ++k)
        gxd[k] = static_cast<double>(gx[k]);
#pragma unroll
    for (int m = 0; m < ZI; ++m) {
        gzd[m] = static_cast<double>(lane(gb[m / 2], m & 1));
#pragma unroll
        for (int k = 0; k < XP; ++k)
            accd[k][m] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < XP; ++k)
#pragma unroll
        for (int i = 0; i < ZH; ++i) {
            acc[k][i] = make_float2(0.0f, 0.0f);
            if constexpr (PREC == kPrecCompensated)
                cmp[k][i] = make_float2(0.0f, 0.0f);
            if constexpr (PREC == kPrecFp64Merge) {
                acc64[k][2 * i] = 0.0;
                acc64[k][2 * i + 1] = 0.0;
            }
        }
    // kPrecFp64MergeShared: this thread's FP64 sums in shared memory (thread-private slots, so no
    // barrier); the same arithmetic as kPrecFp64Merge, with the registers of the sums freed
    double* sums = nullptr;
    int sum_tid = 0, sum_stride = 0;
    if constexpr (PREC == kPrecFp64MergeShared) {
        sums = shared_sums(tiles);
        sum_tid = threadIdx.y * blockDim.x + threadIdx.x;
        sum_stride = blockDim.x * blockDim.y;
#pragma unroll
        for (int q = 0; q < XP * ZI; ++q)
            sums[q * sum_stride + sum_tid] = 0.0;
    }

    // Fold a sub-tile partial into the accumulator of the chosen form.
    auto merge = [&]() {
#pragma unroll
        for (int k = 0; k < XP; ++k)
#pragma unroll
            for (int i = 0; i < ZH; ++i) {
                if constexpr (PREC == kPrecCompensated) {
                    float s0, e0, s1, e1;
                    two_sum(acc[k][i].x, part[k][i].x, s0, e0);
                    two_sum(acc[k][i].y, part[k][i].y, s1, e1);
                    acc[k][i] = make_float2(s0, s1);
                    cmp[k][i] = __fadd2_rn(cmp[k][i], make_float2(e0, e1));
                } else if constexpr (PREC == kPrecFp64Merge) {
                    acc64[k][2 * i] += static_cast<double>(part[k][i].x);
                    acc64[k][2 * i + 1] += static_cast<double>(part[k][i].y);
                } else if constexpr (PREC == kPrecFp64MergeShared) {
                    double* s0 = sums + (k * ZI + 2 * i) * sum_stride + sum_tid;
                    *s0 += static_cast<double>(part[k][i].x);
                    if (2 * i + 1 < ZI)
                        s0[sum_stride] += static_cast<double>(part[k][i].y);
                }
            }
    };
    auto clear_part = [&]() {
#pragma unroll
        for (int k = 0; k < XP; ++k)
#pragma unroll
            for (int i = 0; i < ZH; ++i)
                part[k][i] = make_float2(0.0f, 0.0f);
    };

    if constexpr (SRC == kSrcConstant) {
        static_assert(PREC == kPrecFp32 && SOA == 0, "constant-memory variants are plain FP32 AoS");
        (void)tiles;
        (void)full;
        (void)gstage;
        const int n = static_cast<int>(p.n_atoms);
        // the chunk in blocks of kTileAtoms atoms, each block one phase of the FMA-pipe share
        for (int j0 = 0; j0 < n; j0 += kTileAtoms) {
            const int j1 = j0 + kTileAtoms < n ? j0 + kTileAtoms : n;
            with_phase<P>((j0 / kTileAtoms) % P, [&](auto phase) {
                constexpr int G = decltype(phase)::value;
#pragma unroll UNR
                for (int j = j0; j < j1; ++j)
                    eval_atom<MODE, XP, ZH, SOFT, G, HALF>(gx, gy, gb, c_atoms[j], acc);
            });
        }
    } else {
        const int nthreads = blockDim.x * blockDim.y;
        const int tid = threadIdx.y * blockDim.x + threadIdx.x;
        const int64_t n = p.n_atoms;
        const int64_t nst = (n + kTileAtoms - 1) / kTileAtoms;

        auto stage_count = [&](int64_t s) -> int {
            const int64_t rem = n - s * kTileAtoms;
            return static_cast<int>(rem < kTileAtoms ? rem : kTileAtoms);
        };
        // Producer: one thread arms the stage's barrier with the byte count and starts the copies.
        auto issue = [&](int64_t s) {
            const int buf = static_cast<int>((gstage + static_cast<uint32_t>(s)) % kStages);
            const int64_t base = s * kTileAtoms;
            const int cnt = stage_count(s);
            unsigned char* dst = tiles + buf * kTileAtoms * 16;
            if constexpr (SOA == 0) {
                const uint32_t bytes = static_cast<uint32_t>(cnt) * 16u;
                mbar_arrive_expect_tx(&full[buf], bytes);
                bulk_copy_g2s(dst, p.atoms + base, bytes, &full[buf]);
            } else {
                const int cnt4 = cnt & ~3;  // bulk copies move multiples of 16 bytes
                const uint32_t bytes = static_cast<uint32_t>(cnt4) * 4u;
                mbar_arrive_expect_tx(&full[buf], 4u * bytes);
                if (bytes > 0) {
                    bulk_copy_g2s(dst + 0 * kTileAtoms * 4, p.sx + base, bytes, &full[buf]);
                    bulk_copy_g2s(dst + 1 * kTileAtoms * 4, p.sy + base, bytes, &full[buf]);
                    bulk_copy_g2s(dst + 2 * kTileAtoms * 4, p.sz + base, bytes, &full[buf]);
                    bulk_copy_g2s(dst + 3 * kTileAtoms * 4, p.sq + base, bytes, &full[buf]);
                }
            }
        };

        if (tid == 0) {
            for (int64_t s = 0; s < nst && s < kStages; ++s)
                issue(s);
        }

        for (int64_t s = 0; s < nst; ++s) {
            const uint32_t g = gstage + static_cast<uint32_t>(s);
            const int buf = static_cast<int>(g % kStages);
            const uint32_t parity = static_cast<uint32_t>((g / kStages) & 1);
            const bool ok = mbar_wait_bounded(&full[buf], parity);
            const int cnt = stage_count(s);
            // atoms the stage evaluates: a ragged last stage rounds up to whole sub-tiles only
            const int ntr = cnt < kTileAtoms ? (cnt + SUB - 1) / SUB * SUB : kTileAtoms;
            __builtin_assume(ntr > 0 && ntr <= kTileAtoms && ntr % SUB == 0);
            unsigned char* tile = tiles + buf * kTileAtoms * 16;
            if (ok && cnt < kTileAtoms) {
                // Ragged last stage: the SoA remainder (< 4 atoms) by plain loads, then padding atoms
                // far away with zero charge up to the next whole sub-tile, so the unrolled sub-tile
                // loops below need no bound.
                if constexpr (SOA == 1) {
                    const int cnt4 = cnt & ~3;
                    for (int j = cnt4 + tid; j < cnt; j += nthreads) {
                        const int64_t g = s * kTileAtoms + j;
                        reinterpret_cast<float*>(tile)[0 * kTileAtoms + j] = p.sx[g];
                        reinterpret_cast<float*>(tile)[1 * kTileAtoms + j] = p.sy[g];
                        reinterpret_cast<float*>(tile)[2 * kTileAtoms + j] = p.sz[g];
                        reinterpret_cast<float*>(tile)[3 * kTileAtoms + j] = p.sq[g];
                    }
                }
                for (int j = cnt + tid; j < ntr; j += nthreads) {
                    if constexpr (SOA == 0) {
                        reinterpret_cast<float4*>(tile)[j] = make_float4(kPadCoord, kPadCoord, kPadCoord, 0.0f);
                    } else {
                        reinterpret_cast<float*>(tile)[0 * kTileAtoms + j] = kPadCoord;
                        reinterpret_cast<float*>(tile)[1 * kTileAtoms + j] = kPadCoord;
                        reinterpret_cast<float*>(tile)[2 * kTileAtoms + j] = kPadCoord;
                        reinterpret_cast<float*>(tile)[3 * kTileAtoms + j] = 0.0f;
                    }
                }
            }
            if (__syncthreads_or(ok ? 0 : 1)) {
                // A copy never completed: record it, drain what may still be in flight (bounded),
                // and leave without storing.
                if (tid == 0) {
                    report_status(p.status, kStatusTimeout);
                    for (int64_t r = s; r < nst && r < s + kStages; ++r) {
                        const uint32_t gr = gstage + static_cast<uint32_t>(r);
                        (void)mbar_wait_bounded(&full[gr % kStages], static_cast<uint32_t>((gr / kStages) & 1));
                    }
                }
                return false;
            }

            auto atom_at = [&](int j) -> float4 {
                if constexpr (SOA == 0) {
                    return reinterpret_cast<const float4*>(tile)[j];
                } else {
                    const float* f = reinterpret_cast<const float*>(tile);
                    return make_float4(f[j], f[kTileAtoms + j], f[2 * kTileAtoms + j], f[3 * kTileAtoms + j]);
                }
            };
            // the stage runs in whole sub-tiles of SUB atoms (ntr atoms: all kTileAtoms, or the ragged
            // last stage rounded up); the whole stage is one phase of the FMA-pipe share's pattern
            if constexpr (PREC == kPrecFp64Pairs) {
#pragma unroll UNR
                for (int j = 0; j < ntr; ++j)
                    pair_block_3d_f64<XP, ZI>(gxd, gyd, gzd, atom_at(j), accd);
            } else {
                // G: the stage's phase of the FMA-pipe share; LA: the z points the tile evaluates
                auto stage = [&](auto phase, auto lanes) {
                    constexpr int G = decltype(phase)::value;
                    constexpr int LA = decltype(lanes)::value;
                    constexpr int ZA = (LA + 1) / 2;
                    constexpr bool HA = (LA & 1) != 0;
                    if constexpr (PREC == kPrecFp32) {
#pragma unroll UNR
                        for (int j = 0; j < ntr; ++j)
                            eval_atom<MODE, XP, ZH, SOFT, G, HA, ZA>(gx, gy, gb, atom_at(j), acc);
                    } else {
                        for (int j0 = 0; j0 < ntr; j0 += SUB) {
                            clear_part();
#pragma unroll UNR
                            for (int j = 0; j < SUB; ++j)
                                eval_atom<MODE, XP, ZH, SOFT, G, HA, ZA>(gx, gy, gb, atom_at(j0 + j), part);
                            merge();
                        }
                    }
                };
                with_phase<P>(static_cast<int>((phase_base + static_cast<uint32_t>(s)) % P), [&](auto phase) {
                    if constexpr (ZTRIM) {
                        const int lanes = p.nz - z0 < ZI ? p.nz - z0 : ZI;  // >= 1: the tile starts inside
                        with_phase<ZI>(lanes - 1, [&](auto l) {
                            stage(phase, std::integral_constant<int, decltype(l)::value + 1>{});
                        });
                    } else {
                        stage(phase, std::integral_constant<int, ZI>{});
                    }
                });
            }
            // Everyone is done with this buffer; order the generic-proxy accesses before the next
            // TMA write into it, then refill.
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0 && s + kStages < nst)
                issue(s + kStages);
        }
        gstage += static_cast<uint32_t>(nst);
    }

#pragma unroll
    for (int k = 0; k < XP; ++k)
#pragma unroll
        for (int m = 0; m < ZI; ++m) {
            if constexpr (PREC == kPrecFp32)
                val[k][m] = lane(acc[k][m / 2], m & 1);
            else if constexpr (PREC == kPrecFp64Pairs)
                val[k][m] = static_cast<float>(accd[k][m]);
            else if constexpr (PREC == kPrecCompensated)
                val[k][m] = lane(acc[k][m / 2], m & 1) + lane(cmp[k][m / 2], m & 1);
            else if constexpr (PREC == kPrecFp64MergeShared)
                val[k][m] = static_cast<float>(sums[(k * ZI + m) * sum_stride + sum_tid]);
            else
                val[k][m] = static_cast<float>(acc64[k][m]);
        }
    (void)part;
    (void)cmp;
    (void)acc64;
    (void)accd;
    (void)sums;
    (void)sum_tid;
    (void)sum_stride;
    return true;
}

// Store one thread's register block (edge-guarded; vectorised along x when vec_ok).
template <int ZI, int XP, int MODE>
__device__ __forceinline__ void store_tile(const FwdParams& p, const int x0, const int yrow, const int z0,
                                           const int vec_ok, const float (&val)[XP][ZI])
{
#pragma unroll
    for (int m = 0; m < ZI; ++m) {
        float v[XP];
#pragma unroll
        for (int k = 0; k < XP; ++k)
            v[k] = val[k][m];
        if constexpr (MODE == kModeGrid3d) {
            const int z = z0 + m;
            if (z < p.nz && yrow < p.ny)
                store_points<XP>(p.out + (static_cast<int64_t>(z - p.z_base) * p.ny + yrow) * p.nx, x0, p.nx, v,
                                 p.accumulate, vec_ok);
        } else {
            const int yy = yrow + m;
            if (yy < p.ny)
                store_points<XP>(p.out + static_cast<int64_t>(yy) * p.nx, x0, p.nx, v, p.accumulate, vec_ok);
        }
    }
}

// tile_accumulate then store_tile.  Returns false when a bounded wait expired (nothing stored).
template <int ZI, int XP, int UNR, int SRC, int SOA, int PREC, int SOFT, int MODE, bool ZTRIM = false>
__device__ __forceinline__ bool tile_pass(const FwdParams& p, const int x0, const int yrow, const int z0, const int vec_ok,
                                          unsigned char* tiles, uint64_t* full, uint32_t& gstage)
{
    float val[XP][ZI];
    if (!tile_accumulate<ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE, ZTRIM>(p, x0, yrow, z0, tiles, full, gstage, val))
        return false;
    store_tile<ZI, XP, MODE>(p, x0, yrow, z0, vec_ok, val);
    return true;
}

// Resident 256-thread blocks the register budget of fwd_kernel is sized for: with its FP64 sums in
// shared memory a thread of up to 16 points fits in 51 registers (five such blocks per SM); otherwise
// the compiler's choice.
constexpr int fwd_min_blocks(const int prec, const int points)
{
    return prec == kPrecFp64MergeShared && points <= 16 ? 5 : 1;
}

// One tile per CTA: the block's position in the launch grid selects the tile.
template <int ZI, int XP, int UNR, int SRC, int SOA, int PREC, int SOFT, int MODE>
__global__ void __launch_bounds__(kMaxThreads, fwd_min_blocks(PREC, XP * ZI)) fwd_kernel(const FwdParams p, const int vec_ok)
{
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * XP;
    int yrow, z0;
    if constexpr (MODE == kModeGrid3d) {
        yrow = blockIdx.y * blockDim.y + threadIdx.y;
        z0 = p.z_base + static_cast<int>(blockIdx.z) * ZI;
    } else {
        yrow = (blockIdx.y * blockDim.y + threadIdx.y) * ZI;
        z0 = 0;
    }
    uint32_t gstage = 0;
    if constexpr (SRC == kSrcShared) {
        extern __shared__ __align__(128) unsigned char smem_raw[];
        uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kTileAtoms * 16);
        ring_init(full, threadIdx.y * blockDim.x + threadIdx.x);
        (void)tile_pass<ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE>(p, x0, yrow, z0, vec_ok, smem_raw, full, gstage);
    } else {
        (void)tile_pass<ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE>(p, x0, yrow, z0, vec_ok, nullptr, nullptr, gstage);
    }
}

// Stores value i = (k * ZI + m) * nthreads + t of a tile's register blocks -- thread t's k-th x point,
// m-th blocked point -- at its grid point (edge-guarded, accumulate semantics of p).  The tile is
// (tile_x, tile_y) of the launch's block geometry, z0 its first z point (3D).
template <int ZI, int XP, int MODE>
__device__ __forceinline__ void store_value(const FwdParams& p, const int tile_x, const int tile_y, const int z0,
                                            const int i, const float v)
{
    const int nthreads = static_cast<int>(blockDim.x * blockDim.y);
    const int t = i % nthreads;
    const int km = i / nthreads;
    const int k = km / ZI;
    const int m = km % ZI;
    const int x = (tile_x * static_cast<int>(blockDim.x) + t % static_cast<int>(blockDim.x)) * XP + k;
    const int ty = tile_y * static_cast<int>(blockDim.y) + t / static_cast<int>(blockDim.x);
    float* dst = nullptr;
    if constexpr (MODE == kModeGrid3d) {
        const int z = z0 + m;
        if (x < p.nx && ty < p.ny && z < p.nz)
            dst = p.out + (static_cast<int64_t>(z - p.z_base) * p.ny + ty) * p.nx + x;
    } else {
        const int yy = ty * ZI + m;
        if (x < p.nx && yy < p.ny)
            dst = p.out + static_cast<int64_t>(yy) * p.nx + x;
    }
    if (dst != nullptr)
        *dst = p.accumulate ? *dst + v : v;
}

// Atom-split form for maps with too few points to fill the GPU one tile per CTA (a 2D slice, a
// small 3D map): a thread-block cluster of S CTAs shares one point tile, CTA rank r takes the r-th
// of S contiguous atom ranges through its own TMA ring, and the ranks reduce-scatter the S partial
// blocks over distributed shared memory (rank r sums the r-th slice of the points, every rank's
// value added in rank order: deterministic) and store them.  The cluster size is a
// launch-time choice (2..8 portable, up to 16 with the B200's non-portable cluster sizes); plain FP32
// accumulation, AoS atoms.
template <int ZI, int XP, int UNR, int SOFT, int MODE>
__global__ void __launch_bounds__(kMaxThreads) split_kernel(const FwdParams p, const int vec_ok)
{
    const uint32_t S = cluster_size();
    const uint32_t r = cluster_rank();
    const int tile_x = static_cast<int>(blockIdx.x / S);
    const int x0 = (tile_x * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x)) * XP;
    int yrow, z0;
    if constexpr (MODE == kModeGrid3d) {
        yrow = blockIdx.y * blockDim.y + threadIdx.y;
        z0 = p.z_base + static_cast<int>(blockIdx.z) * ZI;
    } else {
        yrow = (blockIdx.y * blockDim.y + threadIdx.y) * ZI;
        z0 = 0;
    }
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;

    FwdParams q = p;
    const int64_t chunk = (p.n_atoms + S - 1) / S;
    const int64_t begin = chunk * r < p.n_atoms ? chunk * r : p.n_atoms;
    q.atoms = p.atoms + begin;
    q.n_atoms = (p.n_atoms - begin) < chunk ? (p.n_atoms - begin) : chunk;

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kTileAtoms * 16);
    float* red = reinterpret_cast<float*>(smem_raw + kStages * kTileAtoms * 16 + kStages * 8);
    ring_init(full, tid);
    uint32_t gstage = 0;
    float val[XP][ZI];
    // the phase of the FMA-pipe share advances with the rank and with the warp, so every CTA of at
    // least soft_phases warps splits its rsqrts SOFT/8 between the pipes even when it streams a
    // single stage (the cluster waits for its slowest CTA; the atom loop between two stage barriers
    // is warp-uniform code)
    (void)tile_accumulate<ZI, XP, UNR, kSrcShared, 0, kPrecFp32, SOFT, MODE>(q, x0, yrow, z0, smem_raw, full, gstage,
                                                                            val, r + static_cast<uint32_t>(tid) / 32u);
    // A CTA whose ring wait expired has set the status word; the cluster still meets at both
    // barriers so no CTA waits on one that left.
#pragma unroll
    for (int k = 0; k < XP; ++k)
#pragma unroll
        for (int m = 0; m < ZI; ++m)
            red[(k * ZI + m) * nthreads + tid] = val[k][m];
    cluster_sync();
    // Reduce-scatter over the cluster: rank r sums the r-th of S slices of the tile's partial blocks,
    // every rank's value of a point added in rank order (deterministic), and stores those points.
    const int tile_y = static_cast<int>(blockIdx.y);
    const int values = nthreads * XP * ZI;
    const int per = (values + static_cast<int>(S) - 1) / static_cast<int>(S);
    const int end = (static_cast<int>(r) + 1) * per < values ? (static_cast<int>(r) + 1) * per : values;
    for (int i = static_cast<int>(r) * per + tid; i < end; i += nthreads) {
        float part[kMaxSplit];
#pragma unroll
        for (int rank = 0; rank < kMaxSplit; ++rank)  // independent loads, issued together
            if (rank < static_cast<int>(S))
                part[rank] = ld_cluster_f32(cluster_map(red + i, static_cast<uint32_t>(rank)));
        float sum = part[0];
#pragma unroll
        for (int rank = 1; rank < kMaxSplit; ++rank)
            if (rank < static_cast<int>(S))
                sum += part[rank];
        store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, i, sum);
    }
    (void)vec_ok;
    cluster_sync();  // every rank's partial block stays valid until all ranks have read their slices
}

// The queue form of the atom split, for the same small maps without thread-block clusters: a
// persistent grid (as many CTAs as fit, so every SM gets the same share) claims (tile, chunk) items
// from a device counter -- the chunks of one tile are consecutive items -- evaluates the chunk's
// atoms on the tile through its TMA ring and writes the tile's partial block to device memory.  The
// CTA that finishes a tile's last chunk (a counter per tile; each writer fences its partial before
// counting) sums the tile's C partial blocks in chunk order, deterministic whichever CTAs ran them,
// and stores the tile.  No CTA waits on another.
template <int ZI, int XP, int UNR, int SOFT, int MODE>
__global__ void __launch_bounds__(kMaxThreads) queue_split_kernel(const FwdParams p, const SplitQueue sq,
                                                                  const int tiles_x, const int tiles_y,
                                                                  const int64_t items)
{
    static_assert((XP * ZI) % 4 == 0, "the reduction reads a thread's values four at a time");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kTileAtoms * 16);
    __shared__ long long s_item;
    __shared__ int s_last;
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int values = nthreads * XP * ZI;
    const int C = sq.chunks;
    const int64_t chunk = (p.n_atoms + C - 1) / C;
    ring_init(full, tid);
    uint32_t gstage = 0;

    for (;;) {
        if (tid == 0)
            s_item = static_cast<long long>(atomicAdd(sq.counter, 1ull));
        __syncthreads();
        const long long item = s_item;
        __syncthreads();
        if (item >= items)
            return;
        const int t = static_cast<int>(item / C);
        const int c = static_cast<int>(item % C);
        const int tile_x = t % tiles_x;
        const int tile_y = (t / tiles_x) % tiles_y;
        const int tile_z = t / (tiles_x * tiles_y);
        const int x0 = (tile_x * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x)) * XP;
        int yrow, z0;
        if constexpr (MODE == kModeGrid3d) {
            yrow = tile_y * static_cast<int>(blockDim.y) + static_cast<int>(threadIdx.y);
            z0 = p.z_base + tile_z * ZI;
        } else {
            yrow = (tile_y * static_cast<int>(blockDim.y) + static_cast<int>(threadIdx.y)) * ZI;
            z0 = 0;
        }
        FwdParams q = p;
        const int64_t begin = chunk * c < p.n_atoms ? chunk * c : p.n_atoms;
        q.atoms = p.atoms + begin;
        q.n_atoms = (p.n_atoms - begin) < chunk ? (p.n_atoms - begin) : chunk;
        float val[XP][ZI];
        // the FMA-pipe share's phase advances with the chunk and the warp (as in the cluster form)
        if (!tile_accumulate<ZI, XP, UNR, kSrcShared, 0, kPrecFp32, SOFT, MODE>(
                q, x0, yrow, z0, smem_raw, full, gstage, val, static_cast<uint32_t>(c) + static_cast<uint32_t>(tid) / 32u))
            return;  // a bounded wait expired: the status word says so, the tile stays unfinished
        float* part = sq.partial + item * values;
#pragma unroll
        for (int k = 0; k < XP; ++k)
#pragma unroll
            for (int m = 0; m < ZI; ++m)
                part[(k * ZI + m) * nthreads + tid] = val[k][m];
        __threadfence();  // the partial block is visible device-wide before this chunk is counted
        __syncthreads();
        if (tid == 0)
            s_last = atomicAdd(&sq.tile_done[t], 1u) == static_cast<unsigned>(C - 1) ? 1 : 0;
        __syncthreads();
        if (s_last) {
            __threadfence();
            // four consecutive values per thread (values is a multiple of 4: the partial blocks are
            // 16-byte aligned), the chunks' partials loaded kBatch at a time as independent 16-byte
            // loads of the L2 copies (other SMs wrote them), added in chunk order
            const float4* tile_parts = reinterpret_cast<const float4*>(sq.partial + static_cast<int64_t>(t) * C * values);
            const int quads = values / 4;
            constexpr int kBatch = 8;
            for (int i = tid; i < quads; i += nthreads) {
                float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                for (int c0 = 0; c0 < C; c0 += kBatch) {
                    float4 part[kBatch];
#pragma unroll
                    for (int j = 0; j < kBatch; ++j)
                        part[j] = c0 + j < C ? __ldcg(tile_parts + static_cast<int64_t>(c0 + j) * quads + i)
                                             : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                    for (int j = 0; j < kBatch; ++j)
                        if (c0 + j < C) {
                            if (c0 + j == 0) {
                                sum = part[j];
                            } else {
                                sum.x += part[j].x;
                                sum.y += part[j].y;
                                sum.z += part[j].z;
                                sum.w += part[j].w;
                            }
                        }
                }
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, 4 * i + 0, sum.x);
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, 4 * i + 1, sum.y);
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, 4 * i + 2, sum.z);
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, 4 * i + 3, sum.w);
            }
        }
    }
}

// Balanced form of the atom split: the work of a small map is the space of (point tile, atom)
// units, T tiles x N atoms, and CTA b of a resident grid of B takes the b-th of B contiguous,
// equal ranges of it (to one unit), so every SM does the same number of pairs.  A CTA's range
// crosses tile boundaries: it is a sequence of pieces (one tile, a contiguous atom range), streamed
// through the CTA's TMA ring in stages of kBalStageAtoms atoms; the ring runs on from one piece to
// the next.  Inside the CTA, blockDim.z groups of the tile's thread layout share the piece's
// points and split every stage's atoms between them; at the end of a piece the groups' partial
// blocks are added in group order in shared memory.  A piece that covers its tile's atoms is stored;
// the pieces of a tile split between CTAs go to device memory, each CTA counts its split pieces when
// it ends (a counter per split tile), and the CTA that counts a tile's last piece adds the tile's
// pieces in CTA order, stores it and zeroes the counter for the next launch: deterministic for a
// given grid, and no CTA waits on another.
// A CTA of up to kBalThreads threads fills an SM by itself (64 registers a thread): its warps meet at
// the barriers of refilled stages and piece ends, so they progress together -- where two CTAs share an
// SM, the warp schedulers let one run ahead and the other finishes alone at half the occupancy.
constexpr int kBalStageAtoms = 4096;  // atoms per stage of the balanced form's ring (at most)
constexpr int kBalFirstAtoms = 1024;  // atoms in a CTA's first stage: the SM starts work sooner
constexpr int kBalThreads = 1024;     // launch bound of the balanced form (tile threads x groups)
constexpr int kBalMaxGroups = 32;     // atom groups per CTA
constexpr int kBalAtomStep = 8;       // a group's atoms are evaluated in steps of this many

// The balanced form's split of the T x N unit space over B CTAs: q = U / B units per CTA, the first
// r = U % B CTAs one more.  start(b) = b q + min(b, r); cta_of(u) inverts it.
struct BalanceSplit {
    int64_t q, r;
    __host__ __device__ int64_t start(int64_t b) const { return b * q + (b < r ? b : r); }
    __host__ __device__ int64_t cta_of(int64_t u) const
    {
        const int64_t big = r * (q + 1);
        return u < big ? u / (q + 1) : r + (u - big) / q;
    }
};

template <int ZI, int XP, int UNR, int SOFT, int MODE>
__global__ void __launch_bounds__(kBalThreads, 1) balanced_split_kernel(const FwdParams p, const SplitQueue sq,
                                                                     const int tiles_x, const int tiles_y,
                                                                     const int tiles)
{
    constexpr int ZH = (ZI + 1) / 2;
    constexpr bool HALF = (ZI & 1) != 0;
    constexpr int P = soft_phases(SOFT, XP * ZH);
    static_assert(kBalStageAtoms % kBalAtomStep == 0, "steps must divide the stage");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const float4* ring = reinterpret_cast<const float4*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * kBalStageAtoms * 16);
    float* red = reinterpret_cast<float*>(smem_raw + kStages * kBalStageAtoms * 16 + kStages * 8);
    __shared__ int s_last;
    __shared__ int s_issue_t, s_issue_a;  // the producer's cursor: the next stage's tile and first atom
    __shared__ unsigned s_issued;         // stages issued so far

    const int tile_threads = static_cast<int>(blockDim.x * blockDim.y);
    const int groups = static_cast<int>(blockDim.z);
    const int grp = static_cast<int>(threadIdx.z);
    const int ttid = static_cast<int>(threadIdx.y * blockDim.x + threadIdx.x);
    const int tid = grp * tile_threads + ttid;
    const int nthreads = tile_threads * groups;
    const int values = tile_threads * XP * ZI;
    const int N = static_cast<int>(p.n_atoms);  // the host keeps tiles x atoms below 2^62 and atoms below 2^31

    // tile t's origin for this thread
    auto locate = [&](int t, int& tile_x, int& tile_y, int& x0, int& yrow, int& z0) {
        tile_x = t % tiles_x;
        tile_y = (t / tiles_x) % tiles_y;
        const int tile_z = t / (tiles_x * tiles_y);
        x0 = (tile_x * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x)) * XP;
        if constexpr (MODE == kModeGrid3d) {
            yrow = tile_y * static_cast<int>(blockDim.y) + static_cast<int>(threadIdx.y);
            z0 = p.z_base + tile_z * ZI;
        } else {
            yrow = (tile_y * static_cast<int>(blockDim.y) + static_cast<int>(threadIdx.y)) * ZI;
            z0 = 0;
        }
    };

    if (N == 0) {  // no units: the tiles' potentials are zero
        for (int t = static_cast<int>(blockIdx.x); t < tiles; t += static_cast<int>(gridDim.x)) {
            int tile_x, tile_y, x0, yrow, z0;
            locate(t, tile_x, tile_y, x0, yrow, z0);
            for (int v = tid; v < values; v += nthreads)
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, v, 0.0f);
        }
        return;
    }

    // This CTA's units [u_begin, u_end): from atom a_begin of tile t_begin to atom a_stop - 1 of tile
    // t_end.  Its pieces: tile t_begin from a_begin, the tiles between whole, tile t_end up to a_stop.
    const int64_t b = blockIdx.x;
    const BalanceSplit split{static_cast<int64_t>(tiles) * N / gridDim.x, static_cast<int64_t>(tiles) * N % gridDim.x};
    const int64_t u_begin = split.start(b);
    const int64_t u_last = split.start(b + 1) - 1;
    const int t_begin = static_cast<int>(u_begin / N);
    const int a_begin = static_cast<int>(u_begin - static_cast<int64_t>(t_begin) * N);
    const int t_end = static_cast<int>(u_last / N);
    const int a_stop = static_cast<int>(u_last - static_cast<int64_t>(t_end) * N) + 1;
    // the stage at (tile t, atom a): its atom count (a stage never leaves its piece)
    auto stage_count = [&](int t, int a) -> int {
        const int pe = t == t_end ? a_stop : N;
        const int cap = t == t_begin && a == a_begin ? kBalFirstAtoms : kBalStageAtoms;
        return pe - a < cap ? pe - a : cap;
    };

    // the producer (thread 0) keeps its cursor in shared memory, off the other threads' registers
    auto issue = [&]() {
        const int t = s_issue_t;
        const int a = s_issue_a;
        const int cnt = stage_count(t, a);
        const int buf = static_cast<int>(s_issued % kStages);
        const uint32_t bytes = static_cast<uint32_t>(cnt) * 16u;
        mbar_arrive_expect_tx(&full[buf], bytes);
        bulk_copy_g2s(smem_raw + buf * kBalStageAtoms * 16, p.atoms + a, bytes, &full[buf]);
        const bool piece_end = a + cnt == (t == t_end ? a_stop : N);
        s_issue_t = piece_end ? t + 1 : t;
        s_issue_a = piece_end ? 0 : a + cnt;
        s_issued += 1u;
    };
    // thread 0 initialises the ring and starts its first copies before the CTA's barrier, so the
    // first atoms are in flight while the CTA's later warps are still being launched
    if (tid == 0) {
        s_issue_t = t_begin;
        s_issue_a = a_begin;
        s_issued = 0u;
#pragma unroll
        for (int st = 0; st < kStages; ++st)
            mbar_init(&full[st], 1);
        fence_mbar_init();
        while (s_issued < static_cast<uint32_t>(kStages) && s_issue_t <= t_end)
            issue();
    }
    __syncthreads();

    // The CTA's stages (the same count in every thread): the first piece's first stage holds at most
    // kBalFirstAtoms atoms, every other at most kBalStageAtoms.  Only a stage whose buffer is refilled
    // ends with a barrier.
    auto stages_of = [](int atoms) { return (atoms + kBalStageAtoms - 1) / kBalStageAtoms; };
    const int first_len = (t_begin == t_end ? a_stop : N) - a_begin;
    const uint32_t n_stages = static_cast<uint32_t>(
        1 + stages_of(first_len > kBalFirstAtoms ? first_len - kBalFirstAtoms : 0) +
        (t_end > t_begin ? (t_end - t_begin - 1) * stages_of(N) + stages_of(a_stop) : 0));

    float gx[XP];
    float gy = 0.0f;
    float2 gb[ZH];
    float2 acc[XP][ZH];
    int tile_x = 0, tile_y = 0, x0 = 0, yrow = 0, z0 = 0;
    uint32_t k = 0;
    bool failed = false;  // this thread gave up on a stage's copy
    // A copy that never completed: the CTA learns of it at its next barrier; thread 0 then records it,
    // drains what may still be in flight (bounded) and the CTA leaves.  Only the last kStages issued
    // stages can be in flight: no stage is issued after a barrier that saw a failure.
    auto give_up = [&]() {
        if (tid == 0) {
            report_status(p.status, kStatusTimeout);
            const uint32_t issued = s_issued;
            for (uint32_t r = issued > kStages ? issued - kStages : 0u; r < issued; ++r)
                (void)mbar_wait_bounded(&full[r % kStages], (r / kStages) & 1u);
        }
    };
    for (int t = t_begin, a = a_begin; t <= t_end; ++k) {
        const int cnt = stage_count(t, a);
        const int piece_first = t == t_begin ? a_begin : 0;
        if (a == piece_first) {  // a new piece: this thread's points of tile t, zero partials
            locate(t, tile_x, tile_y, x0, yrow, z0);
#pragma unroll
            for (int i = 0; i < XP; ++i)
                gx[i] = fmaf(static_cast<float>(x0 + i), p.h, p.ox);
            blocked_coords<ZH, MODE>(p, yrow, z0, gy, gb);
#pragma unroll
            for (int i = 0; i < XP; ++i)
#pragma unroll
                for (int j = 0; j < ZH; ++j)
                    acc[i][j] = make_float2(0.0f, 0.0f);
        }
        const int buf = static_cast<int>(k % kStages);
        // once this thread has given up, it no longer waits (its values are void anyway)
        if (!failed && !mbar_wait_bounded(&full[buf], (k / kStages) & 1u))
            failed = true;
        // group grp's share of the stage: `per` atoms (a whole number of steps) from grp * per, the
        // last step of a ragged share atom by atom
        const int per = ((cnt + groups - 1) / groups + kBalAtomStep - 1) / kBalAtomStep * kBalAtomStep;
        const int j_begin = grp * per;
        const int j_count = cnt - j_begin < per ? cnt - j_begin : per;
        if (j_count > 0) {
            const int j_full = j_begin + j_count / kBalAtomStep * kBalAtomStep;
            const int j_stop = j_begin + j_count;
            const float4* tile = ring + buf * kBalStageAtoms;
            // the stage and the group select the phase of the FMA-pipe share (as in the other forms,
            // one form per lane pair for a contiguous run of atoms)
            with_phase<P>(static_cast<int>((k + static_cast<uint32_t>(grp)) % P), [&](auto phase) {
                constexpr int G = decltype(phase)::value;
                for (int j0 = j_begin; j0 < j_full; j0 += kBalAtomStep) {
#pragma unroll UNR
                    for (int j = 0; j < kBalAtomStep; ++j)
                        eval_atom<MODE, XP, ZH, SOFT, G, HALF>(gx, gy, gb, tile[j0 + j], acc);
                }
#pragma unroll 1
                for (int j = j_full; j < j_stop; ++j)
                    eval_atom<MODE, XP, ZH, SOFT, G, HALF>(gx, gy, gb, tile[j], acc);
            });
        }
        if (k + kStages < n_stages) {
            // the buffer is refilled: everyone is done with it (generic-proxy reads ordered before
            // the TMA's write)
            fence_proxy_async_smem();
            if (__syncthreads_or(failed ? 1 : 0)) {
                give_up();
                return;
            }
            if (tid == 0)
                issue();
        }
        a += cnt;
        const int piece_stop = t == t_end ? a_stop : N;
        if (a == piece_stop) {
            // the piece ends: add the groups' partial blocks in group order
#pragma unroll
            for (int i = 0; i < XP; ++i)
#pragma unroll
                for (int m = 0; m < ZI; ++m)
                    red[(grp * XP * ZI + i * ZI + m) * tile_threads + ttid] = lane(acc[i][m / 2], m & 1);
            if (__syncthreads_or(failed ? 1 : 0)) {
                give_up();
                return;
            }
            // A split tile's pieces: CTA c's first piece when c starts inside the tile, else its last
            // one; two partial-block slots per CTA.  Only a CTA's first and last pieces can be split;
            // they are counted when the CTA ends.
            const bool whole = piece_first == 0 && piece_stop == N;
            float* slot = sq.partial + (2 * b + (t == t_begin ? 0 : 1)) * values;
            for (int v = tid; v < values; v += nthreads) {
                float sum = red[v];
#pragma unroll 8
                for (int g2 = 1; g2 < groups; ++g2)
                    sum += red[g2 * values + v];
                if (whole)
                    store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, v, sum);
                else
                    slot[v] = sum;
            }
            __syncthreads();  // red is free for the next piece
            ++t;
            a = 0;
        }
    }

    // Count this CTA's split pieces (after all its partial blocks are written) and finish the tiles
    // whose last piece it added; the barriers order the CTA's threads against the counting threads.
    const bool first_split = a_begin > 0 || (t_begin == t_end && a_stop < N);
    const bool last_split = t_end != t_begin && a_stop < N;
    if (first_split || last_split) {
        if (tid == 0)
            s_last = 0;
        __syncthreads();
        // lane 0 of warp i counts the CTA's first (i = 0) or last (i = 1) split piece, with one
        // acquire-release atomic (release: the CTA's partial blocks, ordered before it by the barrier;
        // acquire: the other CTAs' partial blocks of a tile whose last piece this is)
        const int i = tid / 32;
        if (tid % 32 == 0 && i < 2 && (i == 0 ? first_split : last_split)) {
            const int64_t t = i == 0 ? t_begin : t_end;
            const int64_t first = split.cta_of(t * N);
            const int64_t last = split.cta_of((t + 1) * N - 1);
            if (atom_add_acq_rel_gpu(&sq.tile_done[first], 1u) == static_cast<unsigned>(last - first))
                atomicOr(&s_last, 1 << i);
        }
        __syncthreads();
        const int mask = s_last;
        for (int i = 0; i < 2; ++i) {
            if (!(mask & (1 << i)))
                continue;
            const int t = i == 0 ? t_begin : t_end;
            const int64_t t0 = static_cast<int64_t>(t) * N;
            const int64_t first = split.cta_of(t0);
            const int64_t last = split.cta_of(t0 + N - 1);
            locate(t, tile_x, tile_y, x0, yrow, z0);
            for (int v = tid; v < values; v += nthreads) {
                float sum = 0.0f;
                for (int64_t c = first; c <= last; ++c) {
                    const float part = __ldcg(sq.partial + (2 * c + (split.start(c) >= t0 ? 0 : 1)) * values + v);
                    sum = c == first ? part : sum + part;
                }
                store_value<ZI, XP, MODE>(p, tile_x, tile_y, z0, v, sum);
            }
            if (tid == 0)
                sq.tile_done[first] = 0u;  // every piece is counted: zero for the next launch
        }
    }
}

// ------------------------------------------------------------------------------------------
// Launchers and the variant registry
// ------------------------------------------------------------------------------------------
struct VariantKey {
    int zi, xp, unroll, src, soa, prec, soft, mode;
    int split;  // 1 for the atom-split cluster form, 2 for its queue form, 3 for its balanced form
    bool operator==(const VariantKey& o) const
    {
        return zi == o.zi && xp == o.xp && unroll == o.unroll && src == o.src && soa == o.soa && prec == o.prec &&
               soft == o.soft && mode == o.mode && split == o.split;
    }
};


// Dynamic shared memory of the atom-split form: the TMA ring, its barriers, the partial block.
inline size_t split_smem_bytes(int threads, int values_per_thread)
{
    return static_cast<size_t>(kStages) * kTileAtoms * 16 + kStages * 8 +
           static_cast<size_t>(threads) * values_per_thread * sizeof(float);
}

using FwdLaunchFn = cudaError_t (*)(const FwdLaunch&, cudaStream_t);

struct VariantEntry {
    VariantKey key;
    FwdLaunchFn launch;
    int regs;                        // filled lazily from cudaFuncGetAttributes (0 = unknown)
    const void* occupancy_kernel;    // the kernel a persistent form sizes its grid by (else null)
};

template <int ZI, int XP, int UNR, int SRC, int SOA, int PREC, int SOFT, int MODE>
cudaError_t launch_fwd(const FwdLaunch& L, cudaStream_t stream)
{
    auto kernel = fwd_kernel<ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE>;
    if constexpr (SRC == kSrcConstant) {
        // Chunks of kConstAtoms atoms go through this TU's __constant__ bank one launch at a time;
        // later chunks accumulate onto the earlier ones.  Stream order serialises copy and launch.
        FwdParams q = L.p;
        const int64_t n = L.p.n_atoms;
        int64_t off = 0;
        do {
            const int64_t cnt = (n - off) < kConstAtoms ? (n - off) : kConstAtoms;
            if (cnt > 0) {
                cudaError_t e = cudaMemcpyToSymbolAsync(c_atoms, L.p.atoms + off, static_cast<size_t>(cnt) * 16, 0,
                                                        cudaMemcpyDeviceToDevice, stream);
                if (e != cudaSuccess)
                    return e;
            }
            q.n_atoms = cnt;
            q.accumulate = (off > 0) ? 1 : L.p.accumulate;
            kernel<<<L.grid, L.block, 0, stream>>>(q, L.vec_store);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess)
                return e;
            off += cnt;
        } while (off < n);
        return cudaSuccess;
    } else {
        if (L.smem > 48u * 1024u) {
            const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(L.smem));
            if (e != cudaSuccess)
                return e;
        }
        kernel<<<L.grid, L.block, L.smem, stream>>>(L.p, L.vec_store);
        return cudaGetLastError();
    }
}

template <int ZI, int XP, int UNR, int SRC, int SOA, int PREC, int SOFT, int MODE>
void add_variant(std::vector<VariantEntry>& v)
{
    v.push_back(VariantEntry{VariantKey{ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE, 0},
                             &launch_fwd<ZI, XP, UNR, SRC, SOA, PREC, SOFT, MODE>, 0, nullptr});
}

// Cluster launch of the atom-split form: grid.x tiles x `split` CTAs, clusters of `split` along x.
template <int ZI, int XP, int UNR, int SOFT, int MODE>
cudaError_t launch_split(const FwdLaunch& L, cudaStream_t stream)
{
    auto kernel = split_kernel<ZI, XP, UNR, SOFT, MODE>;
    const unsigned S = static_cast<unsigned>(L.split);
    if (S < 2 || S > static_cast<unsigned>(kMaxSplit))
        return cudaErrorInvalidValue;
    if (L.smem > 48u * 1024u) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(L.smem));
        if (e != cudaSuccess)
            return e;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(L.grid.x * S, L.grid.y, L.grid.z);
    cfg.blockDim = L.block;
    cfg.dynamicSmemBytes = L.smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = S;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (S > static_cast<unsigned>(kMaxPortableSplit)) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess)
            return e;
        int clusters = 0;
        e = cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg);
        if (e != cudaSuccess)
            return e;
        if (clusters < 1)
            return cudaErrorLaunchOutOfResources;  // no SM group can hold such a cluster of these blocks
    }
    return cudaLaunchKernelEx(&cfg, kernel, L.p, L.vec_store);
}

// Persistent launch of the queue form: L.queue holds the zeroed counters and the partial blocks,
// L.grid the point tiles.
template <int ZI, int XP, int UNR, int SOFT, int MODE>
cudaError_t launch_queue_split(const FwdLaunch& L, cudaStream_t stream)
{
    auto kernel = queue_split_kernel<ZI, XP, UNR, SOFT, MODE>;
    const int64_t tiles = static_cast<int64_t>(L.grid.x) * L.grid.y * L.grid.z;
    const int64_t items = tiles * L.queue.chunks;
    kernel<<<dim3(static_cast<unsigned>(L.queue.ctas)), L.block, L.smem, stream>>>(
        L.p, L.queue, static_cast<int>(L.grid.x), static_cast<int>(L.grid.y), items);
    return cudaGetLastError();
}

template <int ZI, int XP, int UNR, int SOFT, int MODE>
void add_queue_split_variant(std::vector<VariantEntry>& v)
{
    v.push_back(VariantEntry{VariantKey{ZI, XP, UNR, kSrcShared, 0, kPrecFp32, SOFT, MODE, 2},
                             &launch_queue_split<ZI, XP, UNR, SOFT, MODE>, 0,
                             reinterpret_cast<const void*>(&queue_split_kernel<ZI, XP, UNR, SOFT, MODE>)});
}

// Persistent launch of the balanced form: L.queue holds the counters (zero) and the pieces' partial
// blocks, L.grid the point tiles, L.block.z the atom groups, L.queue.ctas the resident grid.
template <int ZI, int XP, int UNR, int SOFT, int MODE>
cudaError_t launch_balanced_split(const FwdLaunch& L, cudaStream_t stream)
{
    auto kernel = balanced_split_kernel<ZI, XP, UNR, SOFT, MODE>;
    const int tiles = static_cast<int>(L.grid.x * L.grid.y * L.grid.z);  // checked below 2^31 by the setup
    kernel<<<dim3(static_cast<unsigned>(L.queue.ctas)), L.block, L.smem, stream>>>(
        L.p, L.queue, static_cast<int>(L.grid.x), static_cast<int>(L.grid.y), tiles);
    return cudaGetLastError();
}

template <int ZI, int XP, int UNR, int SOFT, int MODE>
void add_balanced_split_variant(std::vector<VariantEntry>& v)
{
    v.push_back(VariantEntry{VariantKey{ZI, XP, UNR, kSrcShared, 0, kPrecFp32, SOFT, MODE, 3},
                             &launch_balanced_split<ZI, XP, UNR, SOFT, MODE>, 0,
                             reinterpret_cast<const void*>(&balanced_split_kernel<ZI, XP, UNR, SOFT, MODE>)});
}

template <int ZI, int XP, int UNR, int SOFT, int MODE>
void add_split_variant(std::vector<VariantEntry>& v)
{
    v.push_back(VariantEntry{VariantKey{ZI, XP, UNR, kSrcShared, 0, kPrecFp32, SOFT, MODE, 1},
                             &launch_split<ZI, XP, UNR, SOFT, MODE>, 0, nullptr});
}

// Register the four atom-loop unrolls {1, 2, 4, 8} of one variant family.
template <int ZI, int XP, int SRC, int SOA, int PREC, int SOFT, int MODE>
void add_unrolls(std::vector<VariantEntry>& v)
{
    add_variant<ZI, XP, 1, SRC, SOA, PREC, SOFT, MODE>(v);
    add_variant<ZI, XP, 2, SRC, SOA, PREC, SOFT, MODE>(v);
    add_variant<ZI, XP, 4, SRC, SOA, PREC, SOFT, MODE>(v);
    add_variant<ZI, XP, 8, SRC, SOA, PREC, SOFT, MODE>(v);
}

// Registration functions, one per translation unit (see coul_fwd_*.cu).
void register_fwd_3d_aos(std::vector<VariantEntry>& v);
void register_fwd_3d_aos_z32(std::vector<VariantEntry>& v);
void register_fwd_3d_soa(std::vector<VariantEntry>& v);
void register_fwd_3d_const(std::vector<VariantEntry>& v);
void register_fwd_3d_precise(std::vector<VariantEntry>& v);
void register_fwd_3d_soft(std::vector<VariantEntry>& v);
void register_fwd_3d_soft_precise(std::vector<VariantEntry>& v);
void register_fwd_3d_soft_fp64m(std::vector<VariantEntry>& v);
void register_fwd_3d_soft_fp64s(std::vector<VariantEntry>& v);
void register_fwd_3d_fp64(std::vector<VariantEntry>& v);
void register_fwd_2d(std::vector<VariantEntry>& v);
void register_fwd_split(std::vector<VariantEntry>& v);
void register_fwd_queue_split(std::vector<VariantEntry>& v);
void register_fwd_balanced_split(std::vector<VariantEntry>& v);

}  // namespace coul
