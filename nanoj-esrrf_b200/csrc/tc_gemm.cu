// tc_gemm.cu -- the two dense passes of the Fourier interpolation on the 5th-generation tensor
// cores (tcgen05, kind::tf32) with a three-term TF32 split for FP32-level accuracy:
//     A B ~= Ah Bh + Ah Bl + Al Bh,   Ah = tf32_rn(A), Al = tf32_rn(A - Ah)  (same for B),
// accumulated in FP32 in tensor memory (TMEM).
//
//   pass 1:  rowsT[f] (WM x N)  = (X_f - c_f) Dx^T, written split into pass 2's operand panels
//   pass 2:  I'[f]    (HM x WM) = Dy rowsT[f]^T + rank-one terms + c_f s N^2
//
// Operands live in HBM already split and laid out as "panels": for a tile of R rows (128 for A,
// 256 for B) and a K block of 16, the hi part then the lo part, each in the canonical K-major
// no-swizzle core-matrix layout (core matrix = 8 rows x 16 bytes; the 16-byte chunk k4 of row r
// at ((k4 (R/8) + r/8) 128 + (r%8) 16) bytes).  Dx and Dy panels are built once per plan, the
// padded frame's panels by x_split_kernel, and pass 1's epilogue writes pass 2's B panels.  So a
// pipeline stage is filled by two plain bulk copies (cp.async.bulk, no tensor map, no multicast).
//
// CTA: 10 warps.  Warp 8 (one lane) streams the panels into a ring of 4 shared-memory stages of
// 48 KB; warp 9 (one lane) issues tcgen05.mma 128x256x8 (6 per K block) and commits; warps 0-7
// drain the accumulators.  The tensor core's FP32 accumulation behaves like round-toward-zero, so
// a run of K = 32 accumulates in one of two TMEM accumulators (columns 0-255 and 256-511) and is
// then drained by warps 0-7 into FP32 registers with round-to-nearest adds while the next run
// fills the other accumulator.  Every mbarrier wait is bounded: a role that gives up records the
// failure in `err`, waits (bounded) for the copies or MMAs it has in flight and leaves; the CTA
// then skips its stores and releases its TMEM.
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/esrrf.h"
#include "esrrf_internal.h"

namespace esrrf {

namespace {

constexpr int TC_M = 128, TC_N = 256, TC_BK = 16;
constexpr uint32_t TC_A_PANEL = TC_M * TC_BK * 4;   // 8 KB per part
constexpr uint32_t TC_B_PANEL = TC_N * TC_BK * 4;   // 16 KB per part
constexpr uint32_t TC_A_BYTES = 2 * TC_A_PANEL;     // hi + lo
constexpr uint32_t TC_B_BYTES = 2 * TC_B_PANEL;
constexpr uint32_t TC_STAGE = TC_A_BYTES + TC_B_BYTES;  // 48 KB
constexpr int TC_STAGES = 4;
constexpr uint32_t TC_SMEM_BYTES = TC_STAGES * TC_STAGE;
constexpr int TC_RUN = 2;                 // K blocks per accumulator run (K = 32)
constexpr uint32_t TC_TMEM_COLS = 512;    // two 128 x 256 FP32 accumulators
constexpr int TC_THREADS = 320;
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // ~2 s of SM clock before a wait gives up

// Instruction descriptor: D f32 (bits 4-5 = 1), A tf32 (7-9 = 2), B tf32 (10-12 = 2), both
// K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__host__ __device__ constexpr uint32_t panel_off(int R, int r, int k4) {
    return ((uint32_t)(k4 * (R / 8) + (r >> 3)) << 7) + ((uint32_t)(r & 7) << 4);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension (K direction) and
// stride-dimension (8-row group) byte offsets >> 4, version 1 at bit 46.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    return __uint_as_float(h);
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the completion of the mbarrier phase with the given parity: false once
// `limit` SM cycles have passed without it.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, long long limit = TC_WAIT_CYCLES) {
    if (mbar_try(addr, parity)) return true;
    const long long t0 = clock64();
    while (clock64() - t0 < limit)
        if (mbar_try(addr, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes)
                 : "memory");
}

// Plain (non-tensor, non-multicast) bulk copy global -> this CTA's shared memory, completing
// `bytes` of the mbarrier's transaction count.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u),
          "r"(0u)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcArgs {
    int Mr, Nc, nkb;                 // C (Mr x Nc) over nkb K blocks of 16
    const unsigned char* Ap;         // A panels [mt][kb], TC_A_BYTES each
    long a_frame;                    // bytes between frames' A panels (0: shared)
    const unsigned char* Bp;         // B panels [nt][kb], TC_B_BYTES each
    long b_frame;
    // pass 1: C written as pass 2's B panels [f][nt][kb2] (K of pass 2 = the rows here)
    unsigned char* Cp;
    long c_frame;
    // pass 2: C row-major [f][Mr][Nc] plus the rank-one terms
    float* C;
    const float* vec;
    const float* cx;
    const float* ux;
    const float* cy;
    const float* uy;
    int HM, WM;
    float cscale;
    int v8;                          // pass 2: rows 32-byte aligned (256-bit stores)
    int* err;
};

template <int PASS>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm_kernel(TcArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_full[TC_STAGES], bar_empty[TC_STAGES], bar_accf[2], bar_acce[2];
    __shared__ uint32_t tmem_slot;
    __shared__ __align__(16) float4 colterm[TC_N];  // pass 2: (cx, ux, q, r) of the tile's columns
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int f = blockIdx.z, mt = blockIdx.y, nt = blockIdx.x;
    const int m0 = mt * TC_M, n0 = nt * TC_N;
    const int nkb = g.nkb, nruns = (nkb + TC_RUN - 1) / TC_RUN;

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&bar_accf[a]), 1);
            mbar_init(smem_u32(&bar_acce[a]), 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 9) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (PASS == 2 && tid < TC_N) {
        const float* vec = g.vec + (long)f * (2L * g.HM + 2L * g.WM + 1);
        const int n = n0 + tid;
        colterm[tid] = n < g.Nc ? make_float4(g.cx[n], g.ux[n], vec[2 * g.HM + n], vec[2 * g.HM + g.WM + n])
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    bool ok = true;
    float racc[128];  // warps 0-7: rows 32 (w % 4) + lane, columns (w / 4) * 128 .. +127

    if (warp == 8) {
        // ---------------- producer: panels -> shared-memory ring ----------------
        if (lane == 0) {
            const unsigned char* Ab = g.Ap + (long)f * g.a_frame + (long)mt * nkb * TC_A_BYTES;
            const unsigned char* Bb = g.Bp + (long)f * g.b_frame + (long)nt * nkb * TC_B_BYTES;
            int issued = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb & (TC_STAGES - 1), u = kb / TC_STAGES;
                if (u > 0 && !mbar_wait(smem_u32(&bar_empty[s]), (uint32_t)((u - 1) & 1))) {
                    ok = false;
                    break;
                }
                const uint32_t full = smem_u32(&bar_full[s]);
                const uint32_t dst = smem_u32(smem + s * TC_STAGE);
                mbar_expect_tx(full, TC_STAGE);
                bulk_g2s(dst, Ab + (long)kb * TC_A_BYTES, TC_A_BYTES, full);
                bulk_g2s(dst + TC_A_BYTES, Bb + (long)kb * TC_B_BYTES, TC_B_BYTES, full);
                issued = kb + 1;
            }
            if (!ok) {
                // let the copies in flight land before the CTA can leave
                for (int kb = issued - TC_STAGES > 0 ? issued - TC_STAGES : 0; kb < issued; ++kb)
                    mbar_wait(smem_u32(&bar_full[kb & (TC_STAGES - 1)]), (uint32_t)((kb / TC_STAGES) & 1));
            }
        }
    } else if (warp == 9) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < nkb; ++kb) {
                const int s = kb & (TC_STAGES - 1), u = kb / TC_STAGES;
                const int r = kb / TC_RUN, a = r & 1;
                const bool first = kb % TC_RUN == 0;
                // the accumulator of run r was last used by run r - 2: wait for its drain
                if (first && r >= 2 && !mbar_wait(smem_u32(&bar_acce[a]), (uint32_t)(((r >> 1) - 1) & 1))) {
                    ok = false;
                    break;
                }
                if (!mbar_wait(smem_u32(&bar_full[s]), (uint32_t)(u & 1))) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t base = smem_u32(smem + s * TC_STAGE);
                const uint32_t ahi = base, alo = base + TC_A_PANEL;
                const uint32_t bhi = base + TC_A_BYTES, blo = base + TC_A_BYTES + TC_B_PANEL;
                const uint32_t d = tmem + (uint32_t)(a * TC_N);
#pragma unroll
                for (int ks = 0; ks < TC_BK / 8; ++ks) {
                    // one MMA consumes k chunks 2ks and 2ks+1 of every row: LBO steps between the
                    // two chunks (R/8 core matrices apart), SBO between 8-row groups
                    const uint32_t ao = (uint32_t)(2 * ks * (TC_M / 8)) << 7;
                    const uint32_t bo = (uint32_t)(2 * ks * (TC_N / 8)) << 7;
                    const uint64_t dah = umma_desc(ahi + ao, (TC_M / 8) << 7, 128);
                    const uint64_t dal = umma_desc(alo + ao, (TC_M / 8) << 7, 128);
                    const uint64_t dbh = umma_desc(bhi + bo, (TC_N / 8) << 7, 128);
                    const uint64_t dbl = umma_desc(blo + bo, (TC_N / 8) << 7, 128);
                    tc_mma(d, dah, dbh, (first && ks == 0) ? 0u : 1u);
                    tc_mma(d, dah, dbl, 1u);
                    tc_mma(d, dal, dbh, 1u);
                }
                tc_commit(smem_u32(&bar_empty[s]));  // the stage can be refilled
                if (kb % TC_RUN == TC_RUN - 1 || kb == nkb - 1) tc_commit(smem_u32(&bar_accf[a]));
                issued = kb + 1;
            }
            if (!ok && issued > 0) {
                // the MMAs in flight must finish before the TMEM is released
                const int kb = issued - 1;
                mbar_wait(smem_u32(&bar_empty[kb & (TC_STAGES - 1)]), (uint32_t)((kb / TC_STAGES) & 1));
            }
        }
    } else {
        // ---------------- drain warps ----------------
#pragma unroll
        for (int i = 0; i < 128; ++i) racc[i] = 0.f;
        const uint32_t tq = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 128);
        for (int r = 0; r < nruns; ++r) {
            const int a = r & 1;
            const bool got = __all_sync(0xffffffffu, mbar_wait(smem_u32(&bar_accf[a]), (uint32_t)((r >> 1) & 1)));
            if (!got) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // 16 columns at a time: with 10 warps a scheduler holds 3, which caps a thread at 168
            // registers, 128 of them the accumulator
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                float v[16];
                tmem_ld16(tq + (uint32_t)(a * TC_N + 16 * c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) racc[16 * c + j] += v[j];
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_acce[a]));
        }
    }

    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!all_ok) {
        if (tid == 0 && g.err) atomicExch(g.err, 1);
    } else if (warp < 8) {
        const int row = m0 + 32 * (warp & 3) + lane;
        const int cb = (warp >> 2) * 128;  // column offset within the tile
        if (PASS == 1) {
            // C^T (columns n = output columns of pass 2, rows = K of pass 2) into pass 2's B
            // panels, split: panel (nt, kb2 = row / 16), panel row n - n0, k = row % 16
            if (row < g.Mr) {
                unsigned char* P = g.Cp + (long)f * g.c_frame +
                                   ((long)nt * (g.Mr / TC_BK) + row / TC_BK) * TC_B_BYTES;
                const int k = row % TC_BK;
#pragma unroll
                for (int j = 0; j < 128; ++j) {
                    const int rr = cb + j;
                    if (n0 + rr >= g.Nc) break;
                    const uint32_t off = panel_off(TC_N, rr, k >> 2) + ((k & 3) << 2);
                    const float hi = tf32_rna(racc[j]);
                    *reinterpret_cast<float*>(P + off) = hi;
                    *reinterpret_cast<float*>(P + TC_B_PANEL + off) = tf32_rna(racc[j] - hi);
                }
            }
        } else {
            if (row < g.Mr) {
                const float* vec = g.vec + (long)f * (2L * g.HM + 2L * g.WM + 1);
                const float pm = vec[row], tm = vec[g.HM + row];
                const float cym = g.cy[row], uym = g.uy[row];
                const float cback = vec[2 * g.HM + 2 * g.WM] * g.cscale;
                float* out = g.C + (long)f * g.Mr * g.Nc + (long)row * g.Nc + n0 + cb;
                const bool full = g.v8 && n0 + cb + 128 <= g.Nc;
                // eight columns at a time: rank-one terms, then one 256-bit store (or scalars)
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    float o[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float4 ct = colterm[cb + 8 * q + i];  // broadcast
                        o[i] = racc[8 * q + i] + pm * ct.x + cym * ct.z - uym * ct.w - tm * ct.y + cback;
                    }
                    if (full) {
                        asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(out + 8 * q),
                                     "f"(o[0]), "f"(o[1]), "f"(o[2]), "f"(o[3]), "f"(o[4]), "f"(o[5]), "f"(o[6]),
                                     "f"(o[7])
                                     : "memory");
                    } else {
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            if (n0 + cb + 8 * q + i < g.Nc) out[8 * q + i] = o[i];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 9) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
    }
}

// Persistent form of tc_gemm_kernel: one CTA per SM walks the tiles t = blockIdx.x + i gridDim.x
// (column tile fastest, then row tile, then frame).  The producer keeps streaming the next tile's
// panels and the MMA warp keeps issuing into the two TMEM accumulators while the drain warps write
// the previous tile's epilogue, so a tile's epilogue overlaps the next tile's first two runs and
// the ring never drains between tiles.  Stage, run and parity counters run across tiles.  The
// drain warps reload pass 2's per-column terms into shared memory per tile between two named
// barriers of their own (bar 1, 256 threads).
template <int PASS>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm_pkernel(TcArgs g, int ntx, int nty, int nframes) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_full[TC_STAGES], bar_empty[TC_STAGES], bar_accf[2], bar_acce[2];
    __shared__ uint32_t tmem_slot;
    __shared__ __align__(16) float4 colterm[TC_N];  // pass 2: (cx, ux, q, r) of the tile's columns
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nkb = g.nkb, nruns = (nkb + TC_RUN - 1) / TC_RUN;
    const int T = ntx * nty * nframes;
    const int my_tiles = (int)blockIdx.x < T ? (T - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(smem_u32(&bar_full[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&bar_accf[a]), 1);
            mbar_init(smem_u32(&bar_acce[a]), 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 9) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    bool ok = true;

    if (warp == 8) {
        // ---------------- producer: panels of every tile of this CTA -> shared-memory ring ----------------
        if (lane == 0) {
            long q = 0;  // K blocks issued by this CTA
            for (int i = 0; i < my_tiles && ok; ++i) {
                const int t = (int)blockIdx.x + i * (int)gridDim.x;
                const int nt = t % ntx, mt = (t / ntx) % nty, f = t / (ntx * nty);
                const unsigned char* Ab = g.Ap + (long)f * g.a_frame + (long)mt * nkb * TC_A_BYTES;
                const unsigned char* Bb = g.Bp + (long)f * g.b_frame + (long)nt * nkb * TC_B_BYTES;
                for (int kb = 0; kb < nkb; ++kb, ++q) {
                    const int s = (int)(q & (TC_STAGES - 1));
                    const long u = q / TC_STAGES;
                    if (u > 0 && !mbar_wait(smem_u32(&bar_empty[s]), (uint32_t)((u - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    const uint32_t full = smem_u32(&bar_full[s]);
                    const uint32_t dst = smem_u32(smem + s * TC_STAGE);
                    mbar_expect_tx(full, TC_STAGE);
                    bulk_g2s(dst, Ab + (long)kb * TC_A_BYTES, TC_A_BYTES, full);
                    bulk_g2s(dst + TC_A_BYTES, Bb + (long)kb * TC_B_BYTES, TC_B_BYTES, full);
                }
            }
            if (!ok) {
                // let the copies in flight land before the CTA can leave
                for (long k = q - TC_STAGES > 0 ? q - TC_STAGES : 0; k < q; ++k)
                    mbar_wait(smem_u32(&bar_full[k & (TC_STAGES - 1)]), (uint32_t)((k / TC_STAGES) & 1));
            }
        }
    } else if (warp == 9) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            long q = 0, issued = 0, rbase = 0;
            for (int i = 0; i < my_tiles && ok; ++i, rbase += nruns) {
                for (int kb = 0; kb < nkb; ++kb, ++q) {
                    const int s = (int)(q & (TC_STAGES - 1));
                    const long u = q / TC_STAGES;
                    const long r = rbase + kb / TC_RUN;
                    const int a = (int)(r & 1);
                    const bool first = kb % TC_RUN == 0;
                    // the accumulator of run r was last used by run r - 2: wait for its drain
                    if (first && r >= 2 && !mbar_wait(smem_u32(&bar_acce[a]), (uint32_t)(((r >> 1) - 1) & 1))) {
                        ok = false;
                        break;
                    }
                    if (!mbar_wait(smem_u32(&bar_full[s]), (uint32_t)(u & 1))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(smem + s * TC_STAGE);
                    const uint32_t ahi = base, alo = base + TC_A_PANEL;
                    const uint32_t bhi = base + TC_A_BYTES, blo = base + TC_A_BYTES + TC_B_PANEL;
                    const uint32_t d = tmem + (uint32_t)(a * TC_N);
#pragma unroll
                    for (int ks = 0; ks < TC_BK / 8; ++ks) {
                        const uint32_t ao = (uint32_t)(2 * ks * (TC_M / 8)) << 7;
                        const uint32_t bo = (uint32_t)(2 * ks * (TC_N / 8)) << 7;
                        const uint64_t dah = umma_desc(ahi + ao, (TC_M / 8) << 7, 128);
                        const uint64_t dal = umma_desc(alo + ao, (TC_M / 8) << 7, 128);
                        const uint64_t dbh = umma_desc(bhi + bo, (TC_N / 8) << 7, 128);
                        const uint64_t dbl = umma_desc(blo + bo, (TC_N / 8) << 7, 128);
                        tc_mma(d, dah, dbh, (first && ks == 0) ? 0u : 1u);
                        tc_mma(d, dah, dbl, 1u);
                        tc_mma(d, dal, dbh, 1u);
                    }
                    tc_commit(smem_u32(&bar_empty[s]));  // the stage can be refilled
                    if (kb % TC_RUN == TC_RUN - 1 || kb == nkb - 1) tc_commit(smem_u32(&bar_accf[a]));
                    issued = q + 1;
                }
            }
            if (!ok && issued > 0) {
                // the MMAs in flight must finish before the TMEM is released
                const long k = issued - 1;
                mbar_wait(smem_u32(&bar_empty[k & (TC_STAGES - 1)]), (uint32_t)((k / TC_STAGES) & 1));
            }
        }
    } else {
        // ---------------- drain warps: runs into FP32 registers, then the tile's epilogue ----------------
        // Every drain thread runs the same number of iterations and reaches both named barriers of
        // every tile, also after a wait gave up (it then skips the waits and stores), so the
        // barriers cannot wait for a thread that left.
        float racc[128];  // rows 32 (w % 4) + lane, columns (w / 4) * 128 .. +127
        const uint32_t tq = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 128);
        long R = 0;
        for (int i = 0; i < my_tiles; ++i) {
            const int t = (int)blockIdx.x + i * (int)gridDim.x;
            const int nt = t % ntx, mt = (t / ntx) % nty, f = t / (ntx * nty);
            const int m0 = mt * TC_M, n0 = nt * TC_N;
#pragma unroll
            for (int j = 0; j < 128; ++j) racc[j] = 0.f;
            for (int rk = 0; rk < nruns; ++rk, ++R) {
                if (!ok) continue;
                const int a = (int)(R & 1);
                const bool got =
                    __all_sync(0xffffffffu, mbar_wait(smem_u32(&bar_accf[a]), (uint32_t)((R >> 1) & 1)));
                if (!got) {
                    ok = false;
                    continue;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    float v[16];
                    tmem_ld16(tq + (uint32_t)(a * TC_N + 16 * c), v);
#pragma unroll
                    for (int j = 0; j < 16; ++j) racc[16 * c + j] += v[j];
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&bar_acce[a]));
            }
            if (PASS == 2) {
                // the tile's per-column terms, once every drain thread is done with the last tile's
                asm volatile("bar.sync 1, 256;" ::: "memory");
                const float* vec = g.vec + (long)f * (2L * g.HM + 2L * g.WM + 1);
                const int n = n0 + tid;
                colterm[tid] = n < g.Nc ? make_float4(g.cx[n], g.ux[n], vec[2 * g.HM + n], vec[2 * g.HM + g.WM + n])
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
                asm volatile("bar.sync 1, 256;" ::: "memory");
            }
            if (!ok) continue;
            const int row = m0 + 32 * (warp & 3) + lane;
            const int cb = (warp >> 2) * 128;
            if (PASS == 1) {
                if (row < g.Mr) {
                    unsigned char* P = g.Cp + (long)f * g.c_frame +
                                       ((long)nt * (g.Mr / TC_BK) + row / TC_BK) * TC_B_BYTES;
                    const int k = row % TC_BK;
#pragma unroll
                    for (int j = 0; j < 128; ++j) {
                        const int rr = cb + j;
                        if (n0 + rr >= g.Nc) break;
                        const uint32_t off = panel_off(TC_N, rr, k >> 2) + ((k & 3) << 2);
                        const float hi = tf32_rna(racc[j]);
                        *reinterpret_cast<float*>(P + off) = hi;
                        *reinterpret_cast<float*>(P + TC_B_PANEL + off) = tf32_rna(racc[j] - hi);
                    }
                }
            } else if (row < g.Mr) {
                const float* vec = g.vec + (long)f * (2L * g.HM + 2L * g.WM + 1);
                const float pm = vec[row], tm = vec[g.HM + row];
                const float cym = g.cy[row], uym = g.uy[row];
                const float cback = vec[2 * g.HM + 2 * g.WM] * g.cscale;
                float* out = g.C + (long)f * g.Mr * g.Nc + (long)row * g.Nc + n0 + cb;
                const bool full = g.v8 && n0 + cb + 128 <= g.Nc;
#pragma unroll
                for (int qq = 0; qq < 16; ++qq) {
                    float o[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const float4 ct = colterm[cb + 8 * qq + k];  // broadcast
                        o[k] = racc[8 * qq + k] + pm * ct.x + cym * ct.z - uym * ct.w - tm * ct.y + cback;
                    }
                    if (full) {
                        asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(out + 8 * qq),
                                     "f"(o[0]), "f"(o[1]), "f"(o[2]), "f"(o[3]), "f"(o[4]), "f"(o[5]), "f"(o[6]),
                                     "f"(o[7])
                                     : "memory");
                    } else {
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            if (n0 + cb + 8 * qq + k < g.Nc) out[8 * qq + k] = o[k];
                    }
                }
            }
        }
    }
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!all_ok && tid == 0 && g.err) atomicExch(g.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 9) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
    }
}

// Padded frame minus its mean, split into pass 1's A panels [f][mt][kb].  One thread per 16-byte
// chunk; consecutive threads take consecutive rows of one chunk column (coalesced panel writes).
__global__ void __launch_bounds__(256) x_split_kernel(const void* __restrict__ raw, int is_u16, int w, int h,
                                                      int N, const int* __restrict__ srcx,
                                                      const int* __restrict__ srcy,
                                                      const float* __restrict__ vec, long vstride,
                                                      long cmean_off, unsigned char* __restrict__ xp) {
    const int f = blockIdx.y;
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;  // chunk index in the frame
    const long per_panel = TC_M * (TC_BK / 4);
    const long nchunks = (long)N * N / 4;
    if (q >= nchunks) return;
    const long p = q / per_panel;
    const int within = (int)(q - p * per_panel);
    const int k4 = within / TC_M, r = within % TC_M;
    const int nkb = N / TC_BK;
    const int mt = (int)(p / nkb), kb = (int)(p % nkb);
    const int m = mt * TC_M + r, x = kb * TC_BK + 4 * k4;
    const float c = vec[(long)f * vstride + cmean_off];
    const long row = (long)srcy[m] * w + (long)f * w * h;
    const int4 sx = *reinterpret_cast<const int4*>(srcx + x);
    float v[4];
    if (is_u16) {
        const unsigned short* s = (const unsigned short*)raw + row;
        v[0] = (float)s[sx.x]; v[1] = (float)s[sx.y]; v[2] = (float)s[sx.z]; v[3] = (float)s[sx.w];
    } else {
        const float* s = (const float*)raw + row;
        v[0] = s[sx.x]; v[1] = s[sx.y]; v[2] = s[sx.z]; v[3] = s[sx.w];
    }
    float4 hi, lo;
    float* hp = &hi.x;
    float* lp = &lo.x;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float d = v[i] - c;
        hp[i] = tf32_rna(d);
        lp[i] = tf32_rna(d - hp[i]);
    }
    unsigned char* P = xp + ((long)f * (N / TC_M) * nkb + p) * TC_A_BYTES;
    const uint32_t off = panel_off(TC_M, r, k4);
    *reinterpret_cast<float4*>(P + off) = hi;
    *reinterpret_cast<float4*>(P + TC_A_PANEL + off) = lo;
}

template <int PASS>
cudaError_t set_tc_smem() {
    static unsigned long long done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0;
    if (bit && (done & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(tc_gemm_kernel<PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TC_SMEM_BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_gemm_pkernel<PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TC_SMEM_BYTES);
    if (e == cudaSuccess) done |= bit;
    return e;
}

// ESRRF_TC_GEMM=tile selects one CTA per tile (the form before the persistent one; kept for A/B).
bool tc_persistent() {
    const char* s = std::getenv("ESRRF_TC_GEMM");
    return !(s && std::strcmp(s, "tile") == 0);
}

// Host form of cvt.rna.tf32.f32 for finite values: round to nearest, ties away from zero, at the
// 13th mantissa bit.
float host_tf32_rna(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    b = (b + 0x1000u) & 0xFFFFE000u;
    float y;
    std::memcpy(&y, &b, 4);
    return y;
}

// Panels of a row-major matrix Z (rows x K): [tile][kb] with R rows per tile, rows >= rows zero.
std::vector<float> make_panels(const std::vector<float>& Z, int rows, int K, int R) {
    const int tiles = (rows + R - 1) / R, nkb = K / TC_BK;
    const size_t part = (size_t)R * TC_BK;  // floats per part
    std::vector<float> P((size_t)tiles * nkb * 2 * part, 0.f);
    for (int t = 0; t < tiles; ++t)
        for (int kb = 0; kb < nkb; ++kb) {
            float* base = P.data() + ((size_t)t * nkb + kb) * 2 * part;
            for (int r = 0; r < R; ++r) {
                const int row = t * R + r;
                if (row >= rows) continue;
                for (int k = 0; k < TC_BK; ++k) {
                    const float v = Z[(size_t)row * K + kb * TC_BK + k];
                    const float hi = host_tf32_rna(v);
                    const size_t o = panel_off(R, r, k >> 2) / 4 + (k & 3);
                    base[o] = hi;
                    base[part + o] = host_tf32_rna(v - hi);
                }
            }
        }
    return P;
}

}  // namespace

bool tc_interp_supported(const InterpPlan& p) { return p.N >= 128 && p.N % TC_M == 0; }

size_t interp_rowT_floats(const InterpPlan& p) {
    const size_t simt = (size_t)p.N * p.WM;
    if (!p.tc) return simt;
    const size_t tc = (size_t)((p.WM + TC_N - 1) / TC_N) * TC_N * p.N * 2;
    return tc > simt ? tc : simt;
}

size_t interp_xs_floats(const InterpPlan& p) { return p.tc ? (size_t)p.N * p.N * 2 : 0; }

cudaError_t tc_plan_tables(InterpPlan& p, const std::vector<float>& dxT, const std::vector<float>& dy) {
    const int N = p.N;
    std::vector<float> dx((size_t)p.WM * N);
    for (int n = 0; n < p.WM; ++n)
        for (int m = 0; m < N; ++m) dx[(size_t)n * N + m] = dxT[(size_t)m * p.WM + n];
    const std::vector<float> dxp = make_panels(dx, p.WM, N, TC_N);
    const std::vector<float> dyp = make_panels(dy, p.HM, N, TC_M);
    cudaError_t e;
    if ((e = cudaMalloc((void**)&p.dxp, sizeof(float) * dxp.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpy(p.dxp, dxp.data(), sizeof(float) * dxp.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    if ((e = cudaMalloc((void**)&p.dyp, sizeof(float) * dyp.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpy(p.dyp, dyp.data(), sizeof(float) * dyp.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return e;
    if ((e = cudaMalloc((void**)&p.tc_err, sizeof(int))) != cudaSuccess) return e;
    return cudaMemset(p.tc_err, 0, sizeof(int));
}

cudaError_t interp_tc_check(const InterpPlan& p, cudaStream_t stream, bool* failed) {
    *failed = false;
    if (!p.tc_err) return cudaSuccess;
    int flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, p.tc_err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && flag) {
        *failed = true;
        e = cudaMemsetAsync(p.tc_err, 0, sizeof(int), stream);
    }
    return e;
}

cudaError_t tc_interp_passes(const InterpPlan& p, InterpScratch& sc, const void* raw, bool is_u16,
                             int F, float* out, cudaStream_t stream) {
    cudaError_t e;
    if ((e = set_tc_smem<1>()) != cudaSuccess) return e;
    if ((e = set_tc_smem<2>()) != cudaSuccess) return e;
    const int N = p.N, nkb = N / TC_BK;
    const int ntiles = (p.WM + TC_N - 1) / TC_N;
    const long vstride = 2L * p.HM + 2L * p.WM + 1;
    {
        const long chunks = (long)N * N / 4;
        x_split_kernel<<<dim3((unsigned)((chunks + 255) / 256), F), 256, 0, stream>>>(
            raw, is_u16 ? 1 : 0, p.w, p.h, N, p.srcx, p.srcy, sc.vec, vstride, 2L * p.HM + 2L * p.WM,
            reinterpret_cast<unsigned char*>(sc.xs));
    }
    TcArgs g{};
    g.vec = sc.vec;
    g.cx = p.cx;
    g.ux = p.ux;
    g.cy = p.cy;
    g.uy = p.uy;
    g.HM = p.HM;
    g.WM = p.WM;
    g.cscale = (float)(p.s * (double)N * (double)N);
    g.err = p.tc_err;
    const long rowT_frame = (long)ntiles * nkb * TC_B_BYTES;
    // pass 1: rows of (X - c) times Dx^T, written as pass 2's B panels
    g.Mr = N;
    g.Nc = p.WM;
    g.nkb = nkb;
    g.Ap = reinterpret_cast<const unsigned char*>(sc.xs);
    g.a_frame = (long)(N / TC_M) * nkb * TC_A_BYTES;
    g.Bp = reinterpret_cast<const unsigned char*>(p.dxp);
    g.b_frame = 0;
    g.Cp = reinterpret_cast<unsigned char*>(sc.rowT);
    g.c_frame = rowT_frame;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    const bool pers = tc_persistent();
    const int sms = sm_count(dev);
    auto pgrid = [&](int tiles) { return (unsigned)std::max(1, std::min(tiles, sms)); };
    if (pers)
        tc_gemm_pkernel<1><<<pgrid(ntiles * (N / TC_M) * F), TC_THREADS, TC_SMEM_BYTES, stream>>>(
            g, ntiles, N / TC_M, F);
    else
        tc_gemm_kernel<1><<<dim3(ntiles, N / TC_M, F), TC_THREADS, TC_SMEM_BYTES, stream>>>(g);
    // pass 2: Dy times the first-pass rows, plus the rank-one terms
    g.Mr = p.HM;
    g.Nc = p.WM;
    g.nkb = nkb;
    g.Ap = reinterpret_cast<const unsigned char*>(p.dyp);
    g.a_frame = 0;
    g.Bp = reinterpret_cast<const unsigned char*>(sc.rowT);
    g.b_frame = rowT_frame;
    g.C = out;
    g.v8 = (p.WM % 8 == 0 && reinterpret_cast<uintptr_t>(out) % 32 == 0) ? 1 : 0;
    const int mtiles = (p.HM + TC_M - 1) / TC_M;
    if (pers)
        tc_gemm_pkernel<2><<<pgrid(ntiles * mtiles * F), TC_THREADS, TC_SMEM_BYTES, stream>>>(g, ntiles, mtiles, F);
    else
        tc_gemm_kernel<2><<<dim3(ntiles, mtiles, F), TC_THREADS, TC_SMEM_BYTES, stream>>>(g);
    return cudaGetLastError();
}

namespace {

// The GEMM roles' bounded wait and failure record on a barrier of one expected arrival: with
// arrive = 1 the phase completes and the wait returns at once; with arrive = 0 nothing arrives, so
// the wait gives up after `limit` cycles and records it in the flag, as a GEMM role does.
__global__ void wait_check_kernel(long long limit, int arrive, int* __restrict__ err) {
    __shared__ __align__(8) unsigned long long bar;
    const uint32_t a = smem_u32(&bar);
    mbar_init(a, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (arrive) mbar_arrive(a);
    if (!mbar_wait(a, 0, limit)) atomicExch(err, 1);
}

}  // namespace

}  // namespace esrrf

extern "C" esrrf_status esrrf_check_bounded_wait(int device, int arrive, long long cycles) {
    using namespace esrrf;
    if (cycles < 1 || cycles > 1000000000LL) return ESRRF_ERR_INVALID;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return ESRRF_ERR_NODEVICE;
    }
    if (device < 0 || device >= n) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return ESRRF_ERR_CUDA;
    int* d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return ESRRF_ERR_NOMEM;
    }
    int flag = 0;
    cudaError_t e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) {
        wait_check_kernel<<<1, 1>>>(cycles, arrive ? 1 : 0, d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&flag, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ESRRF_ERR_CUDA;
    }
    return flag ? ESRRF_ERR_TIMEOUT : ESRRF_OK;
}
