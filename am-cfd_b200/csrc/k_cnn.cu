// Learned warm start: a 4-layer 3x3x3 convolutional network on the solver grid
// (no counterpart in the reference; it only supplies an initial guess, the
// reference's own outer loop still decides convergence).
//
//   features (16 ch, 11 used) -> conv 16->32, ReLU -> conv 32->32, ReLU
//                            -> conv 32->32, ReLU -> conv 32->16 (2 used)
//
// Activations are BF16, channels-last [cell][C] over the full node grid
// (cell = (k*nj + j)*ni + i); boundary nodes are held at zero after every
// layer, which makes each convolution a zero-padded convolution over the
// interior.  Weights are FP32 masters [tap][cout][cin] (tap = 9(dk+1) +
// 3(dj+1) + (di+1)) packed to BF16 for the tensor cores.
//
// Convolutions are implicit GEMMs on the 5th-generation tensor cores: an
// output tile is 128 consecutive cells (M = 128), N = output channels, and the
// reduction runs over 27 taps x input channels in K = 16 slices
// (tcgen05.mma kind::f16, BF16 operands, FP32 accumulators in tensor memory).
// A CTA stages the nine (dk, dj) row groups of 136 cells that its tile needs
// once in shared memory; the three di taps of a group are the same rows
// shifted by one, i.e. operand descriptors 16 bytes apart.  The whole weight
// set of the layer stays in shared memory.  Tiles are double-buffered: the
// gather of tile q+1 and the epilogue of tile q overlap the MMAs.  The same
// kernel computes input gradients (transposed, tap-reversed weights) with the
// ReLU derivative applied in the epilogue.  Weight gradients are a third
// tensor-core contraction, over cells (wgrad_tc_kernel).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "amcfd.h"
#include "async.cuh"

namespace amcfd {
namespace cnn {

constexpr int kConvThreads = 160;  // convolution kernel: four epilogue warps + one TMA/MMA warp
constexpr int kM = 128;  // cells per tile
constexpr int kR = 136;  // rows per (dk, dj) group: 128 + 2 halo, rounded up to 8
constexpr int kLayers = 4;
constexpr int kCin[kLayers] = {16, 32, 32, 32};
constexpr int kCout[kLayers] = {32, 32, 32, 16};
constexpr int kFeat = 11;  // real input channels
constexpr int kOut = 2;   // real output channels

constexpr int kStages = 6;  // shared-memory ring of A units

template <int CIN, int COUT> struct ConvSmem {
    static constexpr int ROW = CIN * 2;                             // bytes per cell (one swizzled row)
    static constexpr int SLAB = (kR * ROW + 1023) / 1024 * 1024;    // one row group, 1 KiB aligned
    static constexpr int U_BYTES = 3 * SLAB;                        // one unit: three row groups
    static constexpr int B_BYTES = 27 * CIN * COUT * 2;
    // ring + weights + (2 kStages + 4) barriers + TMEM slot + alignment slack
    static constexpr size_t BYTES = (size_t)kStages * U_BYTES + B_BYTES + 8 * (2 * kStages + 4) + 16 + 1024;
};

struct ConvArgs {
    CUtensorMap xmap;         // x as [cell][CIN], box CIN x kR, rows swizzled (32 or 64 B)
    const __nv_bfloat16 *x;   // [ncell][CIN]
    const __nv_bfloat16 *w;   // packed [27][CIN/8][COUT][8]
    const float *bias;        // [COUT] or null
    const __nv_bfloat16 *gate;  // [ncell][COUT]: multiply by (gate > 0), or null
    __nv_bfloat16 *y;         // [ncell][COUT]
    float *y32;               // [ncell][n32] FP32 copy of the first n32 channels, or null
    int n32;
    int relu;
    int ni, nj, nk;
    long long ncell;
    int *err;
};

// ---- tensor-core plumbing (PTX) ------------------------------------------------
// Shared-memory matrix descriptor, K-major.  No swizzle (the weights): core
// matrices of 8 rows x 16 bytes stored as 128 contiguous bytes; lbo = byte
// distance between the two K-adjacent core matrices of one K=16 slice, sbo =
// between 8-row groups.  Swizzled (the activations): rows of CIN*2 bytes in the
// TMA's 32/64-byte swizzle, sbo = 8 rows.  The swizzle is a function of the
// shared-memory address, so an operand may start any whole row or 32 bytes
// into a 1 KiB-aligned slab.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout = 0)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;         // descriptor version of sm_100
    d |= (uint64_t)layout << 61;    // 0 no swizzle, 6 = 32-byte, 4 = 64-byte swizzle
    return d;                       // base offset 0
}
// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, M = 128.
template <int N> __host__ __device__ constexpr uint32_t idesc_bf16()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

template <int N> __device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[N]);
template <> __device__ __forceinline__ void tmem_ld<16>(uint32_t t, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                   "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(t));
}
template <> __device__ __forceinline__ void tmem_ld<32>(uint32_t t, uint32_t (&r)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                   "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
                   "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
                   "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
                   "=r"(r[31])
                 : "r"(t));
}

__device__ __forceinline__ bool interior_cell(long long c, int ni, int nj, int nk)
{
    const long long plane = (long long)ni * nj;
    const int k = (int)(c / plane);
    const long long r = c - (long long)k * plane;
    const int j = (int)(r / ni), i = (int)(r - (long long)j * ni);
    return i >= 1 && i <= ni - 2 && j >= 1 && j <= nj - 2 && k >= 1 && k <= nk - 2;
}

// Operand A of a tile, by thirds: unit (tile, dk) holds the three (dj) row
// groups of kR consecutive cells, starting one cell before the tile, of plane
// offset dk: slab j (1 KiB aligned) holds rows of CIN channels (CIN*2 bytes)
// as the TMA's swizzled box of the activation [cell][CIN] (rows outside the
// grid read zeros).
template <int CIN, int COUT>
__device__ __forceinline__ void tma_unit(const CUtensorMap *xmap, long long c0, int dk, int plane, int ni,
                                         unsigned char *A, uint64_t *bar)
{
    using S = ConvSmem<CIN, COUT>;
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)(3 * kR * S::ROW));
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int row0 = (int)(c0 - 1 + (long long)dk * plane + (long long)(j - 1) * ni);
        tma_load_3d(A + (size_t)j * S::SLAB, xmap, 0, row0, 0, bar);
    }
}

// The MMAs of one unit: taps (dk, dj, di) for its dk, 3 x 3 taps x CIN/16
// slices; tap di starts di rows into its slab, slice s 32 bytes into the row.
template <int CIN, int COUT>
__device__ __forceinline__ void issue_unit(uint32_t a_base, uint32_t b_base, int dk, uint32_t tmem_d,
                                           bool first)
{
    using S = ConvSmem<CIN, COUT>;
    constexpr uint32_t idesc = idesc_bf16<COUT>();
    constexpr uint32_t layout = CIN == 32 ? 4u : 6u;  // 64- / 32-byte swizzle
    const uint64_t a0 = smem_desc(a_base, 16, 8 * S::ROW, layout), b0 = smem_desc(b_base, COUT * 16, 128);
    uint32_t acc = first ? 0u : 1u;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int di = 0; di < 3; ++di) {
            const int t = (dk + 1) * 9 + j * 3 + di;
#pragma unroll
            for (int s = 0; s < CIN / 16; ++s) {
                const uint64_t a = a0 + (uint64_t)((j * S::SLAB + di * S::ROW + s * 32) >> 4);
                const uint64_t b = b0 + (uint64_t)((t * CIN * COUT * 2 + 2 * s * COUT * 16) >> 4);
                mma_bf16(tmem_d, a, b, idesc, acc);
                acc = 1u;
            }
        }
}

// Epilogue of one tile by four warps: accumulator row m = TMEM lane m = cell
// c0 + m; bias, ReLU, input-gradient gate, boundary nodes to zero; BF16 store
// (and FP32 copy of the first n32 channels).
template <int COUT>
__device__ __forceinline__ void epilogue(const ConvArgs &args, long long c0, uint32_t taddr)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t r[COUT];
    tmem_ld<COUT>(taddr + ((uint32_t)(32 * warp) << 16), r);
    tmem_wait_ld();
    const long long cell = c0 + 32 * warp + lane;
    if (cell >= args.ncell) return;
    const bool in = interior_cell(cell, args.ni, args.nj, args.nk);
    float v[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) {
        float x = __uint_as_float(r[c]);
        if (args.bias) x += args.bias[c];
        if (args.relu) x = fmaxf(x, 0.f);
        v[c] = in ? x : 0.f;
    }
    if (args.gate) {
        const uint4 *gp = reinterpret_cast<const uint4 *>(args.gate + cell * COUT);
#pragma unroll
        for (int c = 0; c < COUT; c += 8) {
            uint4 gv = gp[c / 8];
            const __nv_bfloat16 *gh = reinterpret_cast<const __nv_bfloat16 *>(&gv);
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (!(__bfloat162float(gh[e]) > 0.f)) v[c + e] = 0.f;
        }
    }
    __nv_bfloat16 *yp = args.y + cell * COUT;
#pragma unroll
    for (int c = 0; c < COUT; c += 8) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(v[c + 2 * e], v[c + 2 * e + 1]);
        *reinterpret_cast<uint4 *>(yp + c) = *reinterpret_cast<uint4 *>(h);
    }
    if (args.y32)
#pragma unroll
        for (int c = 0; c < COUT; ++c)
            if (c < args.n32) args.y32[cell * args.n32 + c] = v[c];
}

// One CTA per SM walks tiles it = 0, 1, ... (cells (blockIdx.x + it*gridDim.x)*128 ...).
// Warp 4 (one thread) streams units (tile, dk) through a ring of kStages
// shared-memory stages with TMA and issues their MMAs; warps 0-3 run the
// epilogues.  mbarriers: loaded[s] (TMA bytes), freed[s] (the MMAs reading
// stage s are done), full[b] (accumulator b holds a finished tile), drained[b]
// (the 128 epilogue threads have read accumulator b).  Every wait is bounded.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads, 1) conv_tc_kernel(const __grid_constant__ ConvArgs args)
{
    using S = ConvSmem<CIN, COUT>;
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char *base = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    unsigned char *Bs = base + (size_t)kStages * S::U_BYTES;
    uint64_t *loaded = reinterpret_cast<uint64_t *>(Bs + S::B_BYTES);
    uint64_t *freed = loaded + kStages, *full = freed + kStages, *drained = full + 2;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(drained + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr uint32_t kCols = COUT * 2 < 32 ? 32 : COUT * 2;  // two accumulators
    const long long ntiles = (args.ncell + kM - 1) / kM;
    const long long nmy = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int plane = args.ni * args.nj;
    auto tile_c0 = [&](long long it) { return (blockIdx.x + it * (long long)gridDim.x) * kM; };

    if (tid == 0) {
        for (int q = 0; q < kStages; ++q) {
            mbar_init(&loaded[q]);
            mbar_init(&freed[q]);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&full[q]);
            mbar_init_n(&drained[q], 128);
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tslot)), "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int q = tid; q < S::B_BYTES / 16; q += blockDim.x)
        reinterpret_cast<uint4 *>(Bs)[q] = reinterpret_cast<const uint4 *>(args.w)[q];
    fence_proxy_async();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tbase = *tslot;
    bool ok = true;

    if (warp == 4) {
        if (lane == 0) {
            const long long nunits = nmy * 3;
            const uint32_t b_addr = smem_u32(Bs);
            auto load = [&](long long v) {
                const int s = (int)(v % kStages);
                tma_unit<CIN, COUT>(&args.xmap, tile_c0(v / 3), (int)(v % 3) - 1, plane, args.ni,
                                    base + (size_t)s * S::U_BYTES, &loaded[s]);
            };
            long long ul = 0, u = 0;  // units loaded, units whose MMAs are issued
            for (; ul < nunits && ul < kStages; ++ul) load(ul);
            for (; u < nunits; ++u) {
                const int s = (int)(u % kStages);
                const long long it = u / 3;
                const int dk = (int)(u % 3) - 1, b = (int)(it & 1);
                ok = mbar_try(&loaded[s], (uint32_t)((u / kStages) & 1), kSpinLimit);
                if (ok && dk == -1 && it >= 2)  // accumulator b: epilogue of tile it - 2 done
                    ok = mbar_try(&drained[b], (uint32_t)(((it - 2) >> 1) & 1), kSpinLimit);
                if (!ok) break;
                tc_after_sync();
                issue_unit<CIN, COUT>(smem_u32(base + (size_t)s * S::U_BYTES), b_addr, dk,
                                      tbase + (uint32_t)(b * COUT), dk == -1);
                mma_commit(&freed[s]);
                if (dk == 1) mma_commit(&full[b]);
                // refill the stage of unit u - 1 (its MMAs run ahead of unit u's)
                if (u >= 1 && ul < nunits) {
                    const int sp = (int)((u - 1) % kStages);
                    ok = mbar_try(&freed[sp], (uint32_t)(((u - 1) / kStages) & 1), kSpinLimit);
                    if (!ok) { ++u; break; }
                    load(ul++);
                }
            }
            if (!ok) {
                atomicExch(args.err, AMCFD_E_TIMEOUT);
                for (long long v = u; v < ul; ++v)  // loads issued, not consumed
                    mbar_try(&loaded[v % kStages], (uint32_t)((v / kStages) & 1), kSpinLimit);
            }
            // the last MMA batch of each stage completes before the CTA releases its memory
            for (long long v = (u > kStages ? u - kStages : 0); v < u; ++v)
                mbar_try(&freed[v % kStages], (uint32_t)((v / kStages) & 1), kSpinLimit);
        }
        __syncwarp();
    } else {
        for (long long it = 0; it < nmy; ++it) {
            const int b = (int)(it & 1);
            if (!mbar_try(&full[b], (uint32_t)((it >> 1) & 1), kSpinLimit)) {
                if (tid == 0) atomicExch(args.err, AMCFD_E_TIMEOUT);
                break;
            }
            tc_after_sync();
            epilogue<COUT>(args, tile_c0(it), tbase + (uint32_t)(b * COUT));
            tc_before_sync();
            mbar_arrive(&drained[b]);
        }
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kCols) : "memory");
}

// ---- weight packing, gradients, loss, optimiser (CUDA cores) -----------------------
// forward operand B[t][n = cout][k = cin]: packed [t][cin/8][cout][8]
__global__ void pack_fwd_kernel(const float *w, __nv_bfloat16 *wp, int cin, int cout)
{
    const int n = 27 * cin * cout;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int e = q % 8, r = q / 8, nn = r % cout, r2 = r / cout, kc = r2 % (cin / 8), t = r2 / (cin / 8);
        wp[q] = __float2bfloat16_rn(w[((size_t)t * cout + nn) * cin + kc * 8 + e]);
    }
}
// input-gradient operand B'[t'][n = cin][k = cout] = W[26 - t'][cout][cin]: packed [t'][cout/8][cin][8]
__global__ void pack_bwd_kernel(const float *w, __nv_bfloat16 *wp, int cin, int cout)
{
    const int n = 27 * cin * cout;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int e = q % 8, r = q / 8, nn = r % cin, r2 = r / cin, kc = r2 % (cout / 8), t = r2 / (cout / 8);
        wp[q] = __float2bfloat16_rn(w[((size_t)(26 - t) * cout + kc * 8 + e) * cin + nn]);
    }
}

// ---- weight gradients on the tensor cores ----------------------------------------
// Per layer dW[t][co][ci] = sum over cells c of dz[c][co] x[c + off(t)][ci] (dz is
// zero on boundary nodes), with off(t) = (dk-1) plane + (dj-1) ni + (di-1) for
// t = 9 dk + 3 dj + di.  As D[m][n] = sum_k A[m][k] B[n][k] over K = cells: the CTAs
// of group dk (blockIdx.y) take rows m = (di, co), A[(di, co)][k] = dz[c - di + 1][co],
// and columns n = (dj, ci), B[(dj, ci)][k] = x[c + (dk-1) plane + (dj-1) ni][ci], for
// the cells c of their chunks; then D[(di, co)][(dj, ci)] = dW[9 dk + 3 dj + di][co][ci]
// (the three di taps share the x rows and differ by the shift of dz).  Chunks of 64
// cells cover c = -1 .. ncell, so every shifted pair is counted once.  M = 128 (rows
// past 3 COUT are zero), N = 3 CIN, FP32 accumulators in tensor memory across all
// chunks of the CTA, operands transposed into the K-major no-swizzle layout by the
// CUDA cores (element (r, k) at (k/8) LBO + (r/8) 128 + (r%8) 16 + (k%8) 2 bytes,
// LBO = rows x 16), two buffers so that staging chunk q+1 overlaps the MMAs of q.
constexpr int kWgThreads = 128;
constexpr int kWgK = 64;  // cells per chunk

template <int CIN, int COUT> struct WgSmem {
    static constexpr int NB = 3 * CIN;                 // rows of B
    static constexpr int A_BYTES = (kWgK / 8) * 128 * 16;
    static constexpr int B_BYTES = (kWgK / 8) * NB * 16;
    static constexpr size_t BYTES = 2 * (size_t)(A_BYTES + B_BYTES) + 8 * 2 + 16 + 1024;
    static constexpr uint32_t COLS = NB <= 32 ? 32 : NB <= 64 ? 64 : 128;  // TMEM columns
};

__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int lbo)
{
    return (uint32_t)((k >> 3) * lbo + ((r >> 3) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kWgThreads, 3) wgrad_tc_kernel(const __nv_bfloat16 *x, const __nv_bfloat16 *dz,
                                                               long long ncell, int ni, int nj, float *part,
                                                               int *err)
{
    using S = WgSmem<CIN, COUT>;
    constexpr int NW = 27 * COUT * CIN;
    constexpr int NB = S::NB;
    constexpr int LBO_A = 128 * 16, LBO_B = NB * 16;
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char *base = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    unsigned char *Abuf[2] = {base, base + S::A_BYTES};
    unsigned char *Bbuf[2] = {base + 2 * S::A_BYTES, base + 2 * S::A_BYTES + S::B_BYTES};
    uint64_t *done = reinterpret_cast<uint64_t *>(base + 2 * (S::A_BYTES + S::B_BYTES));
    uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int dk = blockIdx.y;
    const long long plane = (long long)ni * nj;
    const long long xoff = (long long)(dk - 1) * plane;
    const long long nch = (ncell + 2 + kWgK - 1) / kWgK;  // chunks over c = -1 .. ncell
    const long long nmy = blockIdx.x < nch ? (nch - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (tid == 0) {
        mbar_init(&done[0]);
        mbar_init(&done[1]);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tslot)), "r"(S::COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // rows 3 COUT .. 127 of A stay zero
    for (int q = tid; q < 2 * S::A_BYTES / 16; q += kWgThreads)
        reinterpret_cast<uint4 *>(base)[q] = make_uint4(0u, 0u, 0u, 0u);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tbase = *tslot;
    constexpr uint32_t idesc = idesc_bf16<NB>();
    bool ok = true;
    for (long long it = 0; it < nmy; ++it) {
        const int b = (int)(it & 1);
        if (it >= 2 && !mbar_try(&done[b], (uint32_t)(((it - 2) >> 1) & 1), kSpinLimit)) {
            ok = false;  // (the loop ends below for every thread: the flag is made uniform)
        }
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        const long long c0 = (it * gridDim.x + blockIdx.x) * kWgK - 1;
        unsigned char *A = Abuf[b], *Bm = Bbuf[b];
        // A: dz rows c0-1 .. c0+64, each row to the three di rows it feeds
        constexpr int GA = COUT / 8, NA = (kWgK + 2) * GA;
        for (int q = tid; q < NA; q += kWgThreads) {
            const int r = q / GA, g = q - r * GA;
            const long long c = c0 - 1 + r;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c >= 0 && c < ncell) v = *reinterpret_cast<const uint4 *>(dz + c * COUT + 8 * g);
            const unsigned short *h = reinterpret_cast<const unsigned short *>(&v);
#pragma unroll
            for (int di = 0; di < 3; ++di) {
                const int k = r - 2 + di;
                if (k < 0 || k >= kWgK) continue;
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    *reinterpret_cast<unsigned short *>(A + kmajor_off(di * COUT + 8 * g + e, k, LBO_A)) = h[e];
            }
        }
        // B: x rows of the three (dk, dj) row groups
        constexpr int GB = CIN / 8, NBI = 3 * kWgK * GB;
        for (int q = tid; q < NBI; q += kWgThreads) {
            const int g = q % GB, r = q / GB, k = r % kWgK, dj = r / kWgK;
            const long long c = c0 + k + xoff + (long long)(dj - 1) * ni;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (c >= 0 && c < ncell) v = *reinterpret_cast<const uint4 *>(x + c * CIN + 8 * g);
            const unsigned short *h = reinterpret_cast<const unsigned short *>(&v);
#pragma unroll
            for (int e = 0; e < 8; ++e)
                *reinterpret_cast<unsigned short *>(Bm + kmajor_off(dj * CIN + 8 * g + e, k, LBO_B)) = h[e];
        }
        fence_proxy_async();  // the generic-proxy stores, seen by the tensor cores
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_after_sync();
#pragma unroll
            for (int s = 0; s < kWgK / 16; ++s) {
                const uint64_t a = smem_desc(smem_u32(A) + 2 * s * LBO_A, LBO_A, 128);
                const uint64_t bd = smem_desc(smem_u32(Bm) + 2 * s * LBO_B, LBO_B, 128);
                mma_bf16(tbase, a, bd, idesc, (it == 0 && s == 0) ? 0u : 1u);
            }
            mma_commit(&done[b]);
        }
    }
    // the last commit covers every MMA of the CTA
    if (nmy > 0 && !mbar_try(&done[(int)((nmy - 1) & 1)], (uint32_t)(((nmy - 1) >> 1) & 1), kSpinLimit))
        ok = false;
    if (!ok && tid == 0) atomicExch(err, AMCFD_E_TIMEOUT);
    tc_after_sync();
    float *pp = part + (size_t)blockIdx.x * (NW + COUT);
    const int m = 32 * warp + lane;  // accumulator row = TMEM lane
#pragma unroll
    for (int n0 = 0; n0 < NB; n0 += 16) {
        uint32_t r[16];
        tmem_ld<16>(tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)n0, r);
        tmem_wait_ld();
        if (m < 3 * COUT) {
            const int di = m / COUT, co = m - di * COUT;
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int n = n0 + e, dj = n / CIN, ci = n - dj * CIN;
                const int t = 9 * dk + 3 * dj + di;
                pp[((size_t)t * COUT + co) * CIN + ci] = nmy > 0 ? __uint_as_float(r[e]) : 0.f;
            }
        }
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(S::COLS) : "memory");
}

// db[co] = sum over cells of dz[c][co]: CTA x sums its contiguous range of cells,
// in a fixed order, into the bias slots of its partial row.
template <int COUT>
__global__ void __launch_bounds__(256) bgrad_kernel(const __nv_bfloat16 *dz, long long ncell, float *part, int nw)
{
    __shared__ float sh[256];
    const long long a = ncell * blockIdx.x / gridDim.x, e = ncell * (blockIdx.x + 1) / gridDim.x;
    const int co = threadIdx.x % COUT, lanes = 256 / COUT;
    float acc = 0.f;
    for (long long c = a + threadIdx.x / COUT; c < e; c += lanes) acc += __bfloat162float(dz[c * COUT + co]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < COUT) {
        float s = 0.f;
        for (int q = 0; q < lanes; ++q) s += sh[q * COUT + threadIdx.x];
        part[(size_t)blockIdx.x * (nw + COUT) + nw + threadIdx.x] = s;
    }
}

__global__ void reduce_parts_kernel(const float *part, int nparts, int n, float *out)
{
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n; o += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nparts; ++b) s += part[(size_t)b * n + o];
        out[o] = s;
    }
}

// Features [cell][11] FP32 -> BF16 [cell][16], zero on boundary nodes and padding.
__global__ void features_kernel(const float *f, __nv_bfloat16 *x0, long long ncell, int ni, int nj, int nk)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const bool in = interior_cell(c, ni, nj, nk);
        __nv_bfloat16 v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = __float2bfloat16_rn((in && q < kFeat) ? f[c * kFeat + q] : 0.f);
        reinterpret_cast<uint4 *>(x0 + c * 16)[0] = reinterpret_cast<uint4 *>(v)[0];
        reinterpret_cast<uint4 *>(x0 + c * 16)[1] = reinterpret_cast<uint4 *>(v)[1];
    }
}

// Mean squared error over interior cells and the kOut outputs; dy = dL/dy as
// BF16 [cell][16] (zero elsewhere); per-CTA FP64 partial losses.
__global__ void mse_kernel(const float *y, const float *t, __nv_bfloat16 *dy, long long ncell, int ni, int nj,
                           int nk, double inv_n, double *part)
{
    double s = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const bool in = interior_cell(c, ni, nj, nk);
        __nv_bfloat16 v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = __float2bfloat16_rn(0.f);
        if (in) {
#pragma unroll
            for (int q = 0; q < kOut; ++q) {
                const double d = (double)y[c * kOut + q] - (double)t[c * kOut + q];
                s += d * d;
                v[q] = __float2bfloat16_rn((float)(2.0 * d * inv_n));
            }
        }
        reinterpret_cast<uint4 *>(dy + c * 16)[0] = reinterpret_cast<uint4 *>(v)[0];
        reinterpret_cast<uint4 *>(dy + c * 16)[1] = reinterpret_cast<uint4 *>(v)[1];
    }
    s = warp_sum(s);
    __shared__ double sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
        part[blockIdx.x] = r * inv_n;
    }
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, const unsigned char *live, int n,
                            float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        if (!live[q]) continue;
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq, vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    }
}

// ---- host side ------------------------------------------------------------------------
template <int CIN, int COUT> void set_conv_smem()
{
    cudaFuncSetAttribute(conv_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)ConvSmem<CIN, COUT>::BYTES);
}

template <int CIN, int COUT> void launch_conv(const ConvArgs &a, int grid, cudaStream_t s)
{
    conv_tc_kernel<CIN, COUT><<<grid, kConvThreads, ConvSmem<CIN, COUT>::BYTES, s>>>(a);
}

static int conv(int cin, int cout, ConvArgs a, int grid, cudaStream_t s)
{
    const uint64_t dims[3] = {(uint64_t)cin, (uint64_t)a.ncell, 1};
    const uint64_t strides[2] = {(uint64_t)cin * 2, (uint64_t)cin * 2 * (uint64_t)a.ncell};
    const uint32_t box[3] = {(uint32_t)cin, (uint32_t)kR, 1};
    if (encode_tiled_3d(&a.xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, a.x, dims, strides, box, cin * 2)) return -1;
    if (cin == 16 && cout == 32) launch_conv<16, 32>(a, grid, s);
    else if (cin == 32 && cout == 32) launch_conv<32, 32>(a, grid, s);
    else if (cin == 32 && cout == 16) launch_conv<32, 16>(a, grid, s);
    else if (cin == 16 && cout == 16) launch_conv<16, 16>(a, grid, s);
    return 0;
}

template <int CIN, int COUT> void set_wgrad_smem()
{
    cudaFuncSetAttribute(wgrad_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)WgSmem<CIN, COUT>::BYTES);
}

template <int CIN, int COUT>
static void launch_wgrad(const __nv_bfloat16 *x, const __nv_bfloat16 *dz, long long ncell, int ni, int nj,
                         float *part, int grid, int *err, cudaStream_t s)
{
    wgrad_tc_kernel<CIN, COUT><<<dim3(grid, 3), kWgThreads, WgSmem<CIN, COUT>::BYTES, s>>>(x, dz, ncell, ni, nj,
                                                                                          part, err);
    bgrad_kernel<COUT><<<grid, 256, 0, s>>>(dz, ncell, part, 27 * CIN * COUT);
}

// Per-CTA partial weight and bias gradients of one layer (grid rows of part).
static void wgrad(int cin, int cout, const __nv_bfloat16 *x, const __nv_bfloat16 *dz, long long ncell, int ni,
                  int nj, float *part, int grid, int *err, cudaStream_t s)
{
    if (cin == 16 && cout == 32) launch_wgrad<16, 32>(x, dz, ncell, ni, nj, part, grid, err, s);
    else if (cin == 32 && cout == 32) launch_wgrad<32, 32>(x, dz, ncell, ni, nj, part, grid, err, s);
    else if (cin == 32 && cout == 16) launch_wgrad<32, 16>(x, dz, ncell, ni, nj, part, grid, err, s);
}

}  // namespace cnn
}  // namespace amcfd

using namespace amcfd;
using namespace amcfd::cnn;

// Parameter vector layout: for each layer, W [27][cout][cin] then b [cout].
static size_t layer_off(int l)
{
    size_t o = 0;
    for (int q = 0; q < l; ++q) o += (size_t)27 * kCin[q] * kCout[q] + kCout[q];
    return o;
}
static size_t nparams() { return layer_off(kLayers); }

struct amcfd_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int sm = 148;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // FP32 parameters, grads, moments
    unsigned char *live = nullptr;                                  // 1 where a parameter is not padding
    __nv_bfloat16 *wf[kLayers] = {}, *wb[kLayers] = {};             // packed operands
    __nv_bfloat16 *act[kLayers + 1] = {};                           // act[0] features, act[l+1] layer l out
    __nv_bfloat16 *grad[2] = {};                                    // dZ ping-pong [cell][32]
    float *y = nullptr, *part = nullptr;
    double *lpart = nullptr;
    int *errd = nullptr;
    long long ncap = 0, ncell = 0;
    int ni = 0, nj = 0, nk = 0;
    long long step = 0;
    cudaEvent_t ev[4] = {};        // forward and backward bracketing events
    float fwd_ms = 0.f, bwd_ms = 0.f;
};

#define NCK(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            net->err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return AMCFD_E_CUDA;                                                          \
        }                                                                                 \
    } while (0)

static int net_pack(amcfd_net *net)
{
    for (int l = 0; l < kLayers; ++l) {
        const float *w = net->p + layer_off(l);
        pack_fwd_kernel<<<64, 256, 0, net->stream>>>(w, net->wf[l], kCin[l], kCout[l]);
        pack_bwd_kernel<<<64, 256, 0, net->stream>>>(w, net->wb[l], kCin[l], kCout[l]);
    }
    NCK(cudaGetLastError());
    return 0;
}

static int net_reserve(amcfd_net *net, int ni, int nj, int nk)
{
    const long long n = (long long)ni * nj * nk;
    net->ni = ni; net->nj = nj; net->nk = nk; net->ncell = n;
    if (n <= net->ncap) return 0;
    for (auto &a : net->act) if (a) cudaFree(a), a = nullptr;
    for (auto &a : net->grad) if (a) cudaFree(a), a = nullptr;
    if (net->y) cudaFree(net->y), net->y = nullptr;
    NCK(cudaMalloc(&net->act[0], n * 16 * sizeof(__nv_bfloat16)));
    for (int l = 0; l < kLayers; ++l) NCK(cudaMalloc(&net->act[l + 1], n * kCout[l] * sizeof(__nv_bfloat16)));
    for (auto &a : net->grad) NCK(cudaMalloc(&a, n * 32 * sizeof(__nv_bfloat16)));
    NCK(cudaMalloc(&net->y, n * kOut * sizeof(float)));
    net->ncap = n;
    return 0;
}

extern "C" {

size_t amcfd_net_param_count(void) { return nparams(); }

int amcfd_net_create(int device, unsigned long long seed, amcfd_net **out)
{
    if (!out) return AMCFD_E_ARG;
    amcfd_net *net = new amcfd_net();
    *out = net;
    net->device = device;
    NCK(cudaSetDevice(device));
    NCK(cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking));
    cudaDeviceGetAttribute(&net->sm, cudaDevAttrMultiProcessorCount, device);
    const size_t np = nparams();
    NCK(cudaMalloc(&net->p, np * sizeof(float)));
    NCK(cudaMalloc(&net->g, np * sizeof(float)));
    NCK(cudaMalloc(&net->m, np * sizeof(float)));
    NCK(cudaMalloc(&net->v, np * sizeof(float)));
    NCK(cudaMalloc(&net->live, np));
    NCK(cudaMalloc(&net->errd, sizeof(int)));
    NCK(cudaMemset(net->errd, 0, sizeof(int)));
    NCK(cudaMemset(net->g, 0, np * sizeof(float)));
    NCK(cudaMemset(net->m, 0, np * sizeof(float)));
    NCK(cudaMemset(net->v, 0, np * sizeof(float)));
    for (int l = 0; l < kLayers; ++l) {
        NCK(cudaMalloc(&net->wf[l], (size_t)27 * kCin[l] * kCout[l] * sizeof(__nv_bfloat16)));
        NCK(cudaMalloc(&net->wb[l], (size_t)27 * kCin[l] * kCout[l] * sizeof(__nv_bfloat16)));
    }
    NCK(cudaMalloc(&net->part, (size_t)net->sm * (27 * 32 * 32 + 32) * sizeof(float)));
    for (auto &e : net->ev) NCK(cudaEventCreate(&e));
    NCK(cudaMalloc(&net->lpart, (size_t)net->sm * 4 * sizeof(double)));
    set_conv_smem<16, 32>();
    set_conv_smem<32, 32>();
    set_conv_smem<32, 16>();
    set_conv_smem<16, 16>();
    set_wgrad_smem<16, 32>();
    set_wgrad_smem<32, 32>();
    set_wgrad_smem<32, 16>();
    // initialisation: uniform(-a, a), a = sqrt(6 / fan_in) (ReLU layers), the last
    // layer scaled by 0.1 so that the first predictions are near zero; padding 0
    std::vector<float> h(np, 0.f);
    std::vector<unsigned char> live(np, 0);
    unsigned long long x = seed ? seed : 0x9e3779b97f4a7c15ull;
    auto rnd = [&]() {
        x += 0x9e3779b97f4a7c15ull;
        unsigned long long z = x;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < kLayers; ++l) {
        const int cin_real = l == 0 ? kFeat : kCin[l], cout_real = l == kLayers - 1 ? kOut : kCout[l];
        const double a = std::sqrt(6.0 / (27.0 * cin_real)) * (l == kLayers - 1 ? 0.1 : 1.0);
        const size_t o = layer_off(l);
        for (int t = 0; t < 27; ++t)
            for (int co = 0; co < kCout[l]; ++co)
                for (int ci = 0; ci < kCin[l]; ++ci) {
                    const size_t q = o + ((size_t)t * kCout[l] + co) * kCin[l] + ci;
                    if (ci < cin_real && co < cout_real) {
                        h[q] = (float)((2.0 * rnd() - 1.0) * a);
                        live[q] = 1;
                    }
                }
        for (int co = 0; co < cout_real; ++co) live[o + (size_t)27 * kCin[l] * kCout[l] + co] = 1;
    }
    NCK(cudaMemcpy(net->p, h.data(), np * sizeof(float), cudaMemcpyHostToDevice));
    NCK(cudaMemcpy(net->live, live.data(), np, cudaMemcpyHostToDevice));
    return net_pack(net);
}

void amcfd_net_destroy(amcfd_net *net)
{
    if (!net) return;
    if (net->stream) cudaStreamSynchronize(net->stream);
    void *ptrs[] = {net->p, net->g, net->m, net->v, net->live, net->y, net->part, net->lpart, net->errd};
    for (void *q : ptrs) if (q) cudaFree(q);
    for (int l = 0; l < kLayers; ++l) {
        if (net->wf[l]) cudaFree(net->wf[l]);
        if (net->wb[l]) cudaFree(net->wb[l]);
    }
    for (auto a : net->act) if (a) cudaFree(a);
    for (auto a : net->grad) if (a) cudaFree(a);
    for (auto e : net->ev) if (e) cudaEventDestroy(e);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
}

const char *amcfd_net_last_error(const amcfd_net *net) { return net ? net->err.c_str() : "null network"; }

int amcfd_net_get_params(amcfd_net *net, float *host, size_t n)
{
    if (!net || !host || n != nparams()) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaMemcpy(host, net->p, n * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

int amcfd_net_set_params(amcfd_net *net, const float *host, size_t n)
{
    if (!net || !host || n != nparams()) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaMemcpy(net->p, host, n * sizeof(float), cudaMemcpyHostToDevice));
    return net_pack(net);
}

int amcfd_net_get_grads(amcfd_net *net, float *host, size_t n)
{
    if (!net || !host || n != nparams()) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaMemcpy(host, net->g, n * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
}

// Replaces the gradient buffer (what amcfd_net_adam applies next), e.g. with the
// average over the ranks of a data-parallel training run.
int amcfd_net_set_grads(amcfd_net *net, const float *host, size_t n)
{
    if (!net || !host || n != nparams()) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaMemcpy(net->g, host, n * sizeof(float), cudaMemcpyHostToDevice));
    return 0;
}

// Forward pass on device features [ncell][11] (FP32) over an ni x nj x nk node
// grid; y_dev (may be null) receives the two outputs [ncell][2] (FP32).
int amcfd_net_forward(amcfd_net *net, const float *feat_dev, int ni, int nj, int nk, float *y_dev)
{
    if (!net || !feat_dev || ni < 3 || nj < 3 || nk < 3) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    int rc = net_reserve(net, ni, nj, nk);
    if (rc) return rc;
    const long long n = net->ncell;
    NCK(cudaEventRecord(net->ev[0], net->stream));
    features_kernel<<<net->sm * 4, 256, 0, net->stream>>>(feat_dev, net->act[0], n, ni, nj, nk);
    const long long ntiles = (n + kM - 1) / kM;
    const int grid = (int)std::min<long long>(ntiles, net->sm);
    for (int l = 0; l < kLayers; ++l) {
        ConvArgs a{};
        a.x = net->act[l];
        a.w = net->wf[l];
        a.bias = net->p + layer_off(l) + (size_t)27 * kCin[l] * kCout[l];
        a.y = net->act[l + 1];
        a.relu = l < kLayers - 1;
        a.y32 = l == kLayers - 1 ? net->y : nullptr;
        a.n32 = kOut;
        a.ni = ni; a.nj = nj; a.nk = nk; a.ncell = n;
        a.err = net->errd;
        if (conv(kCin[l], kCout[l], a, grid, net->stream)) {
            net->err = "tensor-map encoding failed";
            return AMCFD_E_CUDA;
        }
    }
    NCK(cudaEventRecord(net->ev[1], net->stream));
    NCK(cudaGetLastError());
    if (y_dev) NCK(cudaMemcpyAsync(y_dev, net->y, n * kOut * sizeof(float), cudaMemcpyDeviceToDevice, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaEventElapsedTime(&net->fwd_ms, net->ev[0], net->ev[1]));
    int e = 0;
    NCK(cudaMemcpy(&e, net->errd, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { net->err = "tensor-core pipeline wait gave up"; return e; }
    return 0;
}

// Loss and gradients of the last forward pass against targets [ncell][2]
// (FP32, device): MSE over interior cells; grads of every parameter into the
// gradient buffer (amcfd_net_get_grads).  *loss receives the loss.
int amcfd_net_backward(amcfd_net *net, const float *target_dev, double *loss)
{
    if (!net || !target_dev || net->ncell == 0) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    const long long n = net->ncell;
    const int ni = net->ni, nj = net->nj, nk = net->nk;
    const double nint = (double)(ni - 2) * (nj - 2) * (nk - 2) * kOut;
    const int lg = net->sm;
    NCK(cudaEventRecord(net->ev[2], net->stream));
    mse_kernel<<<lg, 256, 0, net->stream>>>(net->y, target_dev, net->grad[0], n, ni, nj, nk, 1.0 / nint,
                                            net->lpart);
    const long long ntiles = (n + kM - 1) / kM;
    const int grid = (int)std::min<long long>(ntiles, net->sm);
    // grad[cur] holds dZ of layer l ([cell][kCout[l]], gradient w.r.t. its pre-activation)
    int cur = 0;
    for (int l = kLayers - 1; l >= 0; --l) {
        const size_t nw = (size_t)27 * kCin[l] * kCout[l];
        wgrad(kCin[l], kCout[l], net->act[l], net->grad[cur], n, ni, nj, net->part, net->sm, net->errd,
              net->stream);
        reduce_parts_kernel<<<64, 256, 0, net->stream>>>(net->part, net->sm, (int)(nw + kCout[l]),
                                                          net->g + layer_off(l));
        if (l > 0) {
            ConvArgs a{};
            a.x = net->grad[cur];
            a.w = net->wb[l];
            a.gate = net->act[l];  // ReLU derivative of the previous layer's output
            a.y = net->grad[cur ^ 1];
            a.ni = ni; a.nj = nj; a.nk = nk; a.ncell = n;
            a.err = net->errd;
            if (conv(kCout[l], kCin[l], a, grid, net->stream)) {
                net->err = "tensor-map encoding failed";
                return AMCFD_E_CUDA;
            }
            cur ^= 1;
        }
    }
    NCK(cudaEventRecord(net->ev[3], net->stream));
    NCK(cudaGetLastError());
    std::vector<double> lp(lg);
    NCK(cudaMemcpyAsync(lp.data(), net->lpart, lg * sizeof(double), cudaMemcpyDeviceToHost, net->stream));
    NCK(cudaStreamSynchronize(net->stream));
    NCK(cudaEventElapsedTime(&net->bwd_ms, net->ev[2], net->ev[3]));
    if (loss) {
        double s = 0.0;
        for (double q : lp) s += q;
        *loss = s;
    }
    int e = 0;
    NCK(cudaMemcpy(&e, net->errd, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) { net->err = "tensor-core pipeline wait gave up"; return e; }
    return 0;
}

// Device times (CUDA events on the network's stream) of the last forward and
// backward passes, ms.
int amcfd_net_last_ms(const amcfd_net *net, float *fwd_ms, float *bwd_ms)
{
    if (!net) return AMCFD_E_ARG;
    if (fwd_ms) *fwd_ms = net->fwd_ms;
    if (bwd_ms) *bwd_ms = net->bwd_ms;
    return 0;
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with the current gradients.
int amcfd_net_adam(amcfd_net *net, float lr)
{
    if (!net) return AMCFD_E_ARG;
    NCK(cudaSetDevice(net->device));
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
    adam_kernel<<<64, 256, 0, net->stream>>>(net->p, net->g, net->m, net->v, net->live, (int)nparams(), lr, b1,
                                             b2, 1e-8f, c1, c2);
    NCK(cudaGetLastError());
    int rc = net_pack(net);
    if (rc) return rc;
    NCK(cudaStreamSynchronize(net->stream));
    return 0;
}

}  // extern "C"
