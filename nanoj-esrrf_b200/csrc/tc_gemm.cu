// tc_gemm.cu -- the two dense passes of the Fourier interpolation on the 5th-generation tensor
// cores (tcgen05, kind::tf32) with a three-term TF32 split for FP32-level accuracy:
//     A B ~= Ah Bh + Ah Bl + Al Bh,   Ah = tf32_rn(A), Al = tf32_rn(A - Ah)  (same for B),
// accumulated in FP32 in tensor memory (TMEM).
//
//   pass 1:  rowsT[f] (WM x N)  = (X_f - c_f) Dx^T, stored transposed (K-major for pass 2)
//   pass 2:  I'[f]    (HM x WM) = Dy rowsT[f]^T + rank-one terms + c_f s N^2
//
// The large product Ah Bh and the two small correction products accumulate in separate TMEM
// accumulators (512 columns in all), summed in the epilogue, so the corrections add no rounding to
// the main sum.  CTA tile 128 (M) x 256 (N), K blocks of 32, two shared-memory stages of
// (A hi, A lo, B hi, B lo) in the canonical K-major no-swizzle core-matrix layout (8 rows x 16 bytes per core
// matrix).  All 256 threads stage a K block (global loads, TF32 split, shared stores), then one
// thread issues the 12 MMAs of the block and commits them to the stage's mbarrier; a stage is
// refilled only after that barrier completes.  Every mbarrier wait is bounded: on timeout the
// kernel records the failure in `err`, stops issuing work, releases its TMEM and returns.
#include <stdint.h>

#include "esrrf_internal.h"

namespace esrrf {

namespace {

constexpr int TC_M = 128, TC_N = 256, TC_BK = 32;
constexpr uint32_t TC_A_BYTES = TC_M * TC_BK * 4;  // 16 KB
constexpr uint32_t TC_B_BYTES = TC_N * TC_BK * 4;  // 32 KB
constexpr uint32_t TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;
constexpr uint32_t TC_SMEM_BYTES = 2 * TC_STAGE_BYTES + 128;
constexpr uint32_t TC_TMEM_COLS = 512;  // main accumulator in columns 0-255, corrections 256-511
constexpr int TC_DRAIN = 4;             // K blocks per main-accumulator run (K = 128)
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // ~2 s of SM clock before a wait gives up

// Instruction descriptor: D f32 (bits 4-5 = 1), A tf32 (7-9 = 2), B tf32 (10-12 = 2), both
// K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension (K direction) and
// stride-dimension (8-row group) byte offsets >> 4, version 1 at bit 46.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Byte offset of the 16-byte chunk (row r, k-chunk k4) in a K-major tile of R rows x 32 k.
template <int R>
__device__ __forceinline__ uint32_t kmaj(int r, int k4) {
    return ((uint32_t)(k4 * (R / 8) + (r >> 3)) << 7) + ((uint32_t)(r & 7) << 4);
}

// hi = x rounded to TF32; lo = the remainder (exact in FP32) rounded to TF32 as well, so the
// tensor core does not truncate it
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
    lo = __uint_as_float(l);
}

__device__ __forceinline__ void st_split(unsigned char* hi, unsigned char* lo, uint32_t off, float4 v) {
    float4 h, l;
    split_tf32(v.x, h.x, l.x);
    split_tf32(v.y, h.y, l.y);
    split_tf32(v.z, h.z, l.z);
    split_tf32(v.w, h.w, l.w);
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = l;
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

// Bounded wait for the completion of the mbarrier phase with the given parity.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    if (mbar_try(addr, parity)) return true;
    const long long t0 = clock64();
    while (clock64() - t0 < TC_WAIT_CYCLES)
        if (mbar_try(addr, parity)) return true;
    return false;
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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Adds a warp's 32 x 128 quarter of the main accumulator into the register accumulator.
__device__ __forceinline__ void drain_main(uint32_t taddr, float (&racc)[128]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float v[32];
        tmem_ld32(taddr + 32 * c, v);
#pragma unroll
        for (int j = 0; j < 32; ++j) racc[32 * c + j] += v[j];
    }
}

struct TcArgs {
    int Mr, Nc, K;             // C[f] (Mr x Nc) = A (Mr x K) . B^T, B stored K-major (Nc x K)
    // pass 1 A: padded frame gathered from raw, minus the frame mean
    const void* raw;
    int is_u16, w, h;
    const int* srcx;
    const int* srcy;
    // pass 2 A: shared row-major matrix
    const float* A;
    // B: K-major (rows of length K); per frame (stride Nc*K) when b_per_frame
    const float* B;
    int b_per_frame;
    float* C;
    // rank-one epilogue (pass 2) and frame means
    const float* vec;
    const float* cx;
    const float* ux;
    const float* cy;
    const float* uy;
    int HM, WM;
    float cscale;
    int* err;
};

// Staging map of the 16-byte chunk q of a K block: eight consecutive lanes take the eight rows of
// one core matrix, four lanes along K, so a warp stores four whole core matrices (512 contiguous
// bytes, no bank conflict) and loads eight rows x 64 contiguous bytes from global memory.
__device__ __forceinline__ void chunk_of(int q, int& r, int& k4) {
    r = ((q >> 6) << 3) | (q & 7);
    k4 = (((q >> 5) & 1) << 2) | ((q >> 3) & 3);
}

// PASS 1: A gathered from the raw frame (minus its mean), C stored transposed.
// PASS 2: A shared, rank-one epilogue, C row-major (written through a shared-memory transpose).
template <int PASS>
__global__ void __launch_bounds__(256, 1) tc_gemm_kernel(TcArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int f = blockIdx.z;
    const int m0 = blockIdx.y * TC_M, n0 = blockIdx.x * TC_N;
    const int nkb = g.K / TC_BK;

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    const void* rawf = nullptr;
    float cmean = 0.f;
    if (PASS == 1) {
        rawf = g.is_u16 ? (const void*)((const unsigned short*)g.raw + (long)f * g.w * g.h)
                        : (const void*)((const float*)g.raw + (long)f * g.w * g.h);
        cmean = g.vec[(long)f * (2L * g.HM + 2L * g.WM + 1) + 2 * g.HM + 2 * g.WM];
    }
    const float* Bf = g.b_per_frame ? g.B + (long)f * g.Nc * g.K : g.B;
    int issued = 0;  // K blocks whose MMAs have been issued and committed
    // This warp's TMEM quarter: lanes 32 (warp % 4) .. +31 (tile rows), columns (warp / 4) * 128.
    const uint32_t tq = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 128);
    // The tensor core's FP32 accumulation of the main product is drained into registers every
    // TC_DRAIN K blocks (round-to-nearest adds), which bounds the rounding bias a long TMEM
    // accumulation builds up.
    float racc[128];
#pragma unroll
    for (int i = 0; i < 128; ++i) racc[i] = 0.f;

    for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb & 1;
        unsigned char* st = smem + s * TC_STAGE_BYTES;
        unsigned char* Ahi = st;
        unsigned char* Alo = st + TC_A_BYTES;
        unsigned char* Bhi = st + 2 * TC_A_BYTES;
        unsigned char* Blo = st + 2 * TC_A_BYTES + TC_B_BYTES;
        // the stage is free once the MMAs of block kb - 2 (its previous use) have completed
        bool freed = true;
        if (kb >= 2) freed = mbar_wait(smem_u32(&mbar[s]), (uint32_t)(((kb >> 1) - 1) & 1));
        const int k0 = kb * TC_BK;
#pragma unroll
        for (int i = 0; i < 4; ++i) {  // A: 128 rows x 8 chunks
            int r, k4;
            chunk_of(tid + i * 256, r, k4);
            const int m = m0 + r, k = k0 + 4 * k4;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (m < g.Mr) {
                if (PASS == 1) {
                    const long row = (long)__ldg(g.srcy + m) * g.w;
                    const int4 sx = __ldg(reinterpret_cast<const int4*>(g.srcx + k));
                    if (g.is_u16) {
                        const unsigned short* src = (const unsigned short*)rawf + row;
                        v = make_float4((float)__ldg(src + sx.x) - cmean, (float)__ldg(src + sx.y) - cmean,
                                        (float)__ldg(src + sx.z) - cmean, (float)__ldg(src + sx.w) - cmean);
                    } else {
                        const float* src = (const float*)rawf + row;
                        v = make_float4(__ldg(src + sx.x) - cmean, __ldg(src + sx.y) - cmean,
                                        __ldg(src + sx.z) - cmean, __ldg(src + sx.w) - cmean);
                    }
                } else {
                    v = __ldg(reinterpret_cast<const float4*>(g.A + (long)m * g.K + k));
                }
            }
            st_split(Ahi, Alo, kmaj<TC_M>(r, k4), v);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {  // B: 256 rows x 8 chunks
            int r, k4;
            chunk_of(tid + i * 256, r, k4);
            const int n = n0 + r, k = k0 + 4 * k4;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n < g.Nc) v = __ldg(reinterpret_cast<const float4*>(Bf + (long)n * g.K + k));
            st_split(Bhi, Blo, kmaj<TC_N>(r, k4), v);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        // one barrier both publishes the stage and makes the give-up decision block-uniform
        if (!__syncthreads_and(freed ? 1 : 0)) break;
        if (kb > 0 && kb % TC_DRAIN == 0) {
            // block kb-1 closed a run: drain it before the MMAs of block kb restart the accumulator
            const bool ok = __all_sync(0xffffffffu,
                                       mbar_wait(smem_u32(&mbar[(kb - 1) & 1]), (uint32_t)(((kb - 1) >> 1) & 1)));
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (ok) drain_main(tq, racc);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            if (!__syncthreads_and(ok ? 1 : 0)) break;
        }
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ahi = smem_u32(Ahi), alo = smem_u32(Alo);
            const uint32_t bhi = smem_u32(Bhi), blo = smem_u32(Blo);
#pragma unroll
            for (int ks = 0; ks < TC_BK / 8; ++ks) {
                // one MMA consumes k chunks 2ks and 2ks+1 of every row: LBO steps between the two
                // chunks (R/8 core matrices apart), SBO between 8-row groups (one core matrix)
                const uint32_t ao = (uint32_t)(2 * ks * (TC_M / 8)) << 7;
                const uint32_t bo = (uint32_t)(2 * ks * (TC_N / 8)) << 7;
                const uint64_t dah = umma_desc(ahi + ao, (TC_M / 8) << 7, 128);
                const uint64_t dal = umma_desc(alo + ao, (TC_M / 8) << 7, 128);
                const uint64_t dbh = umma_desc(bhi + bo, (TC_N / 8) << 7, 128);
                const uint64_t dbl = umma_desc(blo + bo, (TC_N / 8) << 7, 128);
                tc_mma(tmem, dah, dbh, (kb % TC_DRAIN != 0 || ks > 0) ? 1u : 0u);
                tc_mma(tmem + TC_N, dah, dbl, (kb > 0 || ks > 0) ? 1u : 0u);
                tc_mma(tmem + TC_N, dal, dbh, 1u);
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&mbar[s]))
                : "memory");
        }
        issued = kb + 1;
    }
    // the accumulator is final once the commit of the last issued block has arrived (a commit
    // tracks every earlier MMA of the issuing thread); after a failed wait this still waits,
    // bounded, for the MMAs in flight before the tensor memory is released
    bool done = issued == nkb;
    if (issued > 0 &&
        !mbar_wait(smem_u32(&mbar[(issued - 1) & 1]), (uint32_t)(((issued - 1) >> 1) & 1)))
        done = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!__syncthreads_and(done ? 1 : 0)) {
        if (tid == 0 && g.err) atomicExch(g.err, 1);
    } else {
        // epilogue: the last run and the corrections join the register accumulator
        drain_main(tq, racc);
        drain_main(tq + TC_N, racc);
        const int rbase = m0 + 32 * (warp & 3);
        const int row = rbase + lane;
        const int cbase = n0 + (warp >> 2) * 128;
        float* Cf = g.C + (long)f * g.Mr * g.Nc;
        if (PASS == 1) {
            if (row < g.Mr) {
#pragma unroll
                for (int j = 0; j < 128; ++j) {
                    const int n = cbase + j;
                    if (n < g.Nc) Cf[(long)n * g.Mr + row] = racc[j];  // lanes write consecutive rows
                }
            }
        } else {
            // rank-one terms: row factors held by the lane of that row, column factors by the
            // lane of that column after the transpose
            const float* vec = g.vec + (long)f * (2L * g.HM + 2L * g.WM + 1);
            float pm = 0.f, tm = 0.f, cym = 0.f, uym = 0.f;
            if (row < g.Mr) {
                pm = vec[row];
                tm = vec[g.HM + row];
                cym = g.cy[row];
                uym = g.uy[row];
            }
            const float cback = vec[2 * g.HM + 2 * g.WM] * g.cscale;
            float* buf = reinterpret_cast<float*>(smem) + warp * (32 * 33);  // stages are idle now
#pragma unroll
            for (int c = 0; c < 4; ++c) {
#pragma unroll
                for (int j = 0; j < 32; ++j) buf[lane * 33 + j] = racc[32 * c + j];
                __syncwarp();
                const int n = cbase + 32 * c + lane;
                float cxn = 0.f, uxn = 0.f, qn = 0.f, rn = 0.f;
                if (n < g.Nc) {
                    cxn = g.cx[n];
                    uxn = g.ux[n];
                    qn = vec[2 * g.HM + n];
                    rn = vec[2 * g.HM + g.WM + n];
                }
#pragma unroll 4
                for (int r = 0; r < 32; ++r) {
                    const float pr = __shfl_sync(0xffffffffu, pm, r);
                    const float tr = __shfl_sync(0xffffffffu, tm, r);
                    const float cr = __shfl_sync(0xffffffffu, cym, r);
                    const float ur = __shfl_sync(0xffffffffu, uym, r);
                    if (rbase + r < g.Mr && n < g.Nc)
                        Cf[(long)(rbase + r) * g.Nc + n] =
                            buf[r * 33 + lane] + pr * cxn + cr * qn - ur * rn - tr * uxn + cback;
                }
                __syncwarp();
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
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
    if (e == cudaSuccess) done |= bit;
    return e;
}

}  // namespace

bool tc_interp_supported(const InterpPlan& p) { return p.N >= 32 && p.N % 32 == 0; }

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
    const int N = p.N;
    TcArgs g{};
    g.raw = raw;
    g.is_u16 = is_u16 ? 1 : 0;
    g.w = p.w;
    g.h = p.h;
    g.srcx = p.srcx;
    g.srcy = p.srcy;
    g.vec = sc.vec;
    g.cx = p.cx;
    g.ux = p.ux;
    g.cy = p.cy;
    g.uy = p.uy;
    g.HM = p.HM;
    g.WM = p.WM;
    g.cscale = (float)(p.s * (double)N * (double)N);
    g.err = p.tc_err;
    // pass 1: rowsT[f] (WM x N) = (X_f - c) . Dx^T, with B = Dx (WM x N, K-major)
    g.Mr = N;
    g.Nc = p.WM;
    g.K = N;
    g.B = p.dx;
    g.b_per_frame = 0;
    g.C = sc.rowT;
    tc_gemm_kernel<1><<<dim3((g.Nc + TC_N - 1) / TC_N, (g.Mr + TC_M - 1) / TC_M, F), 256, TC_SMEM_BYTES,
                        stream>>>(g);
    // pass 2: I'[f] (HM x WM) = Dy . rowsT[f]^T + epilogue, with B = rowsT[f] (WM x N, K-major)
    g.Mr = p.HM;
    g.Nc = p.WM;
    g.K = N;
    g.A = p.dy;
    g.B = sc.rowT;
    g.b_per_frame = 1;
    g.C = out;
    tc_gemm_kernel<2><<<dim3((g.Nc + TC_N - 1) / TC_N, (g.Mr + TC_M - 1) / TC_M, F), 256, TC_SMEM_BYTES,
                        stream>>>(g);
    return cudaGetLastError();
}

}  // namespace esrrf
