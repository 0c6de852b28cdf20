// sweep.cu -- batched parameter sweep and rolling analysis over uneven frame blocks, on one or
// several devices.
//
// The reference's ParametersSweep_ (gui/ParametersSweep_.java:328-519) re-initialises the
// engine -- context, program build, buffers, per-frame upload -- for every (radius, sensitivity)
// combination, and its rolling analysis (gui/LiveSRRF_optimised_.java:276-389) recomputes every
// frame once per block that contains it.  Here one captured CUDA graph per device does the work:
//   per magnification: Fourier-interpolate every frame once (interp.cu);
//   per radius: one fused-RGC launch over all frames that writes CGLH / sum-of-weights per frame
//     (the tap loop is shared by every sensitivity and every block);
//   per (sensitivity group, block group): one memory-bound launch that raises CGLH to the
//     sensitivity, weights it by the intensity and reduces AVG/VAR/TAC2/INT over each block, FP64
//     accumulators in registers.
// With drift (the sweep's vibration correction: one shift per frame of the stack,
// gui/ParametersSweep_.java:282-290, loaded into every combination's engine at :452-454) the RGC
// launch takes per-frame tap tables (rgc_fht_drift.cu) and the intensity is each frame's
// getInterpolatedValue at its shifted position, sampled once per magnification.
// The bicubic sweep (the reference sweep with "Use FHT interpolation" off) computes the 2-point
// gradients, their 2x resampling and the unit-gradient field of every frame once (none depends on
// the magnification or radius); per (magnification, radius) the tabulated bicubic RGC writes
// CGLH / sum of weights and the bicubic intensity of every frame; the cumulant launches apply the
// path's double (n - 1) division of TAC2, and every output gets the MP correction.
//
// Several devices: the (magnification, radius) pairs, or the blocks, are split across the devices
// (plan_shards below: longest-processing-time assignment of pairs by tap-count cost, or contiguous
// runs of blocks of balanced frame span, whichever finishes first); each device holds its own copy
// of the frames its part needs and runs its own graph; nothing crosses between devices and the
// results are gathered into the host output.
// Output: for each magnification, radius, sensitivity and block, the four [HM][WM] slices of
// readSRRFbuffer (AVG, VAR, TAC2, INT; NaN -> 0).
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/esrrf.h"
#include "device_common.cuh"
#include "esrrf_internal.h"

using namespace esrrf;

namespace {

constexpr int kSG = 2;  // sensitivities per cumulant launch
constexpr int kBG = 4;  // blocks per cumulant launch

struct CumArgs {
    const float* cg;   // [T][P]
    const float* v;    // [T][P]
    long P;
    int start[kBG], len[kBG], nb;
    float sens[kSG];
    int ns;
    int int_weighting;
    int tac_div2;      // bicubic path: TAC2 divided by (n - 1) twice (liveSRRF.cl:374,377)
    float* out;        // base of this (magnification, radius): [nS][nB][4][P]
    int s0, b0, nB;    // global indices of the first sensitivity and block of the launch
};

__global__ void __launch_bounds__(256) sweep_cumulants_kernel(CumArgs a) {
    const long pix = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= a.P) return;
    // block bounds in registers; unused block slots get an empty range, unused sensitivity slots
    // are skipped by guards (no early exits, so every index below is a compile-time constant)
    int bs[kBG], be[kBG];
#pragma unroll
    for (int b = 0; b < kBG; ++b) {
        bs[b] = b < a.nb ? a.start[b] : 0;
        be[b] = b < a.nb ? a.start[b] + a.len[b] : 0;
    }
    double acc[kSG][kBG][4];
    float prev[kSG];
#pragma unroll
    for (int s = 0; s < kSG; ++s) {
        prev[s] = 0.f;
#pragma unroll
        for (int b = 0; b < kBG; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[s][b][c] = 0.0;
    }
    int t_lo = bs[0], t_hi = be[0];
#pragma unroll
    for (int b = 1; b < kBG; ++b)
        if (b < a.nb) {
            t_lo = min(t_lo, bs[b]);
            t_hi = max(t_hi, be[b]);
        }
    // one frame's CGLH and intensity into the sums of every (sensitivity, block) slot
    auto frame = [&](int t, float c, float v) {
        const double vd = (double)v;
#pragma unroll
        for (int s = 0; s < kSG; ++s) {
            if (s < a.ns) {
                const float cg = dev::cglh_power(c, a.sens[s]);
                const float x = a.int_weighting ? v * cg : cg;
                const double xd = (double)x;
#pragma unroll
                for (int b = 0; b < kBG; ++b) {
                    if (t >= bs[b] && t < be[b]) {
                        acc[s][b][0] += xd;
                        acc[s][b][1] = fma(xd, xd, acc[s][b][1]);
                        if (t > bs[b]) acc[s][b][2] = fma(xd, (double)prev[s], acc[s][b][2]);
                        acc[s][b][3] += vd;
                    }
                }
                prev[s] = x;
            }
        }
    };
    // the planes are read once, straight from HBM: the loads of kU frames are issued before their
    // arithmetic, so that enough of them are in flight (frames still summed in order)
    constexpr int kU = 8;
    int t = t_lo;
    for (; t + kU <= t_hi; t += kU) {
        float cu[kU], vu[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            cu[u] = __ldg(a.cg + (long)(t + u) * a.P + pix);
            vu[u] = __ldg(a.v + (long)(t + u) * a.P + pix);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) frame(t + u, cu[u], vu[u]);
    }
    for (; t < t_hi; ++t) frame(t, __ldg(a.cg + (long)t * a.P + pix), __ldg(a.v + (long)t * a.P + pix));
#pragma unroll
    for (int s = 0; s < kSG; ++s) {
        if (s >= a.ns) continue;
#pragma unroll
        for (int b = 0; b < kBG; ++b) {
            if (b >= a.nb) continue;
            const int n = a.len[b];
            const double avg = acc[s][b][0] / n, av2 = avg * avg;
            double tac = n > 1 ? acc[s][b][2] / (n - 1) : 0.0;
            if (a.tac_div2 && n > 1) tac /= (n - 1);
            float o[4] = {(float)avg, (float)(acc[s][b][1] / n - av2), (float)(tac - av2),
                          (float)(acc[s][b][3] / n)};
            float* dst = a.out + (((long)(a.s0 + s) * a.nB + (a.b0 + b)) * 4) * a.P + pix;
#pragma unroll
            for (int k = 0; k < 4; ++k) dst[(long)k * a.P] = isnan(o[k]) ? 0.f : o[k];
        }
    }
}

// One magnification of a shard and the radii it handles at that magnification.
struct MagPlan {
    int M = 0, mi = 0;                  // magnification and its index in the sweep
    std::vector<int> ri;                // radius indices (into the sweep's radii)
    InterpPlan plan;
    std::vector<FhtGeometry> geo;       // per entry of ri
    std::vector<FhtFusedTables> tables; // per entry of ri
    std::vector<BicGeometry> bgeo;      // bicubic sweep: per entry of ri
    std::vector<BicTables> btab;        // bicubic sweep: per entry of ri (common field padding)
    float* d_shift = nullptr;           // drift x M, [2][T] (FHT sweep with drift)
};

std::string cuda_msg(cudaError_t e, const char* what) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}

// One device's part of a sweep: a set of (magnification, radius) pairs over the frames
// [f0, f0 + T) of the stack, which hold its blocks.
struct Shard {
    int device = -1;
    cudaStream_t stream = nullptr;
    int w = 0, h = 0, T = 0, f0 = 0;
    int int_weighting = 1;
    std::vector<int> sens, bstart, blen, bglob;  // blocks: local start, length, global index
    std::vector<MagPlan> mp;
    bool drift = false;
    std::vector<float> dx, dy;                  // [T] raw pixels (drift)
    FhtDriftTables dtab;                        // per-frame tap tables + shifted intensities
    InterpScratch scratch;
    float* d_interp = nullptr;  // [T][HM][WM] for the largest magnification
    float* d_cg = nullptr;
    void* d_in = nullptr;       // host-input staging on the device
    float* d_outbuf = nullptr;  // host-output staging on the device
    // bicubic sweep: frames as float, 2-point gradients, 2x gradients, unit-gradient field
    bool bic = false;
    float* d_fraw = nullptr;
    float* d_gx = nullptr;
    float* d_gy = nullptr;
    float* d_gxi = nullptr;
    float* d_gyi = nullptr;
    float2* d_u2 = nullptr;
    float* d_mpmap = nullptr;
    std::vector<size_t> offsets;  // local layout: per (mp entry, radius entry) in order
    size_t total = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* g_in = nullptr;
    float* g_out = nullptr;
    float* g_hout = nullptr;
    int g_u16 = -1;
    // host-output runs into pinned memory: each pair's outputs are copied out on copy_stream as
    // soon as its cumulants are written, while the next pairs compute
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> pair_ev;  // per (mp entry, radius entry)
    cudaEvent_t copy_done = nullptr;
    int launches_per_run = 0;
    std::string err;

    esrrf_status fail(esrrf_status s, const std::string& m) {
        err = m;
        return s;
    }
    esrrf_status fail_cuda(cudaError_t e, const char* what) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? ESRRF_ERR_NOMEM : ESRRF_ERR_CUDA, cuda_msg(e, what));
    }
    esrrf_status create(const std::vector<float>& radii, int interp);
    esrrf_status create_bic(const std::vector<float>& radii);
    esrrf_status enqueue(const void* frames, int is_u16, float* out, float* hout);
    esrrf_status enqueue_bic(const void* frames, int is_u16, float* out, float* hout);
    esrrf_status copy_pair(size_t oi, const float* out, float* hout);
    esrrf_status copy_join(float* hout);
    esrrf_status tc_check();
    esrrf_status run_device(const void* d_frames, int is_u16, float* d_out, float* h_out = nullptr);
    void release();
};

#define SK(call, what)                                         \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return s->fail_cuda(_e, what);  \
    } while (0)
#define SKS(call, what)                                         \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return sh->fail_cuda(_e, what);  \
    } while (0)

// Pair oi's outputs (its sensitivities and blocks, contiguous in the shard's layout) to the
// same place of the pinned host buffer, on copy_stream once the compute stream has written them.
esrrf_status Shard::copy_pair(size_t oi, const float* out, float* hout) {
    Shard* s = this;
    if (!hout) return ESRRF_OK;
    const size_t n = (oi + 1 < offsets.size() ? offsets[oi + 1] : total) - offsets[oi];
    SK(cudaEventRecord(pair_ev[oi], stream), "pair event");
    SK(cudaStreamWaitEvent(copy_stream, pair_ev[oi], 0), "copy wait");
    SK(cudaMemcpyAsync(hout + offsets[oi], out + offsets[oi], sizeof(float) * n, cudaMemcpyDeviceToHost,
                       copy_stream),
       "output copy");
    return ESRRF_OK;
}

// The compute stream waits for the last copy (joins copy_stream back, also inside a capture).
esrrf_status Shard::copy_join(float* hout) {
    Shard* s = this;
    if (!hout) return ESRRF_OK;
    SK(cudaEventRecord(copy_done, copy_stream), "copy event");
    SK(cudaStreamWaitEvent(stream, copy_done, 0), "copy join");
    return ESRRF_OK;
}

esrrf_status Shard::enqueue(const void* frames, int is_u16, float* out, float* hout) {
    Shard* s = this;
    const size_t fb = (is_u16 ? sizeof(uint16_t) : sizeof(float)) * (size_t)w * h;
    int launches = 0;
    if (bic) return enqueue_bic(frames, is_u16, out, hout);
    size_t oi = 0;
    for (size_t mi = 0; mi < mp.size(); ++mi) {
        const MagPlan& m = mp[mi];
        const long P = (long)m.plan.WM * m.plan.HM;
        for (int t = 0; t < T; t += scratch.capacity) {
            const int Fn = std::min(scratch.capacity, T - t);
            SK(interp_run(m.plan, scratch, (const unsigned char*)frames + fb * t, is_u16 != 0, Fn,
                          d_interp + (size_t)t * P, stream, &launches),
               "interpolation");
        }
        const float* vsrc = d_interp;
        if (drift) {  // every frame's intensity at its shifted position, shared by the radii
            SK(fht_shift_sample(d_interp, m.plan.WM, m.plan.HM, T, m.d_shift, m.d_shift + T, dtab.v, stream),
               "shifted intensities");
            ++launches;
            vsrc = dtab.v;
        }
        for (size_t e = 0; e < m.ri.size(); ++e, ++oi) {
            FhtRgcArgs a{};
            a.interp = d_interp;
            a.W = m.plan.WM;
            a.H = m.plan.HM;
            a.F = T;
            a.t0 = 0;
            a.int_weighting = int_weighting;
            a.cg_out = d_cg;
            if (drift) {
                SK(fht_drift_tables_build(m.geo[e], m.d_shift, m.d_shift + T, T, dtab, stream), "drift tables");
                SK(fht_rgc_fused_drift(m.geo[e], dtab, a, stream), "RGC");
                launches += 2;
            } else {
                SK(fht_rgc_fused(m.geo[e], m.tables[e], a, stream), "RGC");
                ++launches;
            }
            float* base = out + offsets[oi];
            for (int s0 = 0; s0 < (int)sens.size(); s0 += kSG)
                for (int b0 = 0; b0 < (int)bstart.size(); b0 += kBG) {
                    CumArgs c{};
                    c.cg = d_cg;
                    c.v = vsrc;
                    c.P = P;
                    c.nb = std::min(kBG, (int)bstart.size() - b0);
                    for (int b = 0; b < c.nb; ++b) {
                        c.start[b] = bstart[b0 + b];
                        c.len[b] = blen[b0 + b];
                    }
                    c.ns = std::min(kSG, (int)sens.size() - s0);
                    for (int q = 0; q < c.ns; ++q) c.sens[q] = (float)sens[s0 + q];
                    c.int_weighting = int_weighting;
                    c.out = base;
                    c.s0 = s0;
                    c.b0 = b0;
                    c.nB = (int)bstart.size();
                    sweep_cumulants_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(c);
                    SK(cudaGetLastError(), "cumulants");
                    ++launches;
                }
            esrrf_status r = copy_pair(oi, out, hout);
            if (r != ESRRF_OK) return r;
        }
    }
    launches_per_run = launches;
    return copy_join(hout);
}

esrrf_status Shard::enqueue_bic(const void* frames, int is_u16, float* out, float* hout) {
    Shard* s = this;
    int launches = 0;
    SK(bic_prepare(frames, is_u16, w, h, T, d_fraw, d_gx, d_gy, d_gxi, d_gyi, stream), "gradients");
    launches += 3;
    SK(unit_grad2d(d_gxi, d_gyi, w, h, T, mp[0].btab[0], d_u2, stream), "unit gradient");
    ++launches;
    size_t oi = 0;
    for (size_t mi = 0; mi < mp.size(); ++mi) {
        const MagPlan& m = mp[mi];
        const long P = (long)w * m.M * h * m.M;
        for (size_t e = 0; e < m.ri.size(); ++e, ++oi) {
            BicTabArgs a{};
            a.U = d_u2;
            a.fraw = d_fraw;
            a.w = w;
            a.h = h;
            a.M = m.M;
            a.F = T;
            a.t0 = 0;
            a.sens = 1.f;
            a.int_weighting = int_weighting;
            a.tab = m.btab[e];
            a.cg_out = d_cg;
            a.v_out = d_interp;
            SK(bic_rgc_tab(a, stream), "RGC");
            ++launches;
            float* base = out + offsets[oi];
            for (int s0 = 0; s0 < (int)sens.size(); s0 += kSG)
                for (int b0 = 0; b0 < (int)bstart.size(); b0 += kBG) {
                    CumArgs c{};
                    c.cg = d_cg;
                    c.v = d_interp;
                    c.P = P;
                    c.nb = std::min(kBG, (int)bstart.size() - b0);
                    for (int b = 0; b < c.nb; ++b) {
                        c.start[b] = bstart[b0 + b];
                        c.len[b] = blen[b0 + b];
                    }
                    c.ns = std::min(kSG, (int)sens.size() - s0);
                    for (int q = 0; q < c.ns; ++q) c.sens[q] = (float)sens[s0 + q];
                    c.int_weighting = int_weighting;
                    c.tac_div2 = 1;
                    c.out = base;
                    c.s0 = s0;
                    c.b0 = b0;
                    c.nB = (int)bstart.size();
                    sweep_cumulants_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(c);
                    SK(cudaGetLastError(), "cumulants");
                    ++launches;
                }
            // MP correction of AVG, VAR and TAC2 of every (sensitivity, block) output
            for (size_t q = 0; q < sens.size() * bstart.size(); ++q) {
                SK(mp_correct(base + q * 4 * P, w, h, 1, m.M, 0, d_mpmap, stream), "MP correction");
                launches += 2;
            }
            esrrf_status r = copy_pair(oi, out, hout);
            if (r != ESRRF_OK) return r;
        }
    }
    launches_per_run = launches;
    return copy_join(hout);
}

void Shard::release() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    for (auto& m : mp) {
        interp_plan_destroy(m.plan);
        for (auto& t : m.tables) fht_fused_tables_free(t);
        for (auto& t : m.btab) bic_tables_free(t);
        cudaFree(m.d_shift);
    }
    fht_drift_tables_free(dtab);
    for (float* b : {d_fraw, d_gx, d_gy, d_gxi, d_gyi, d_mpmap}) cudaFree(b);
    cudaFree(d_u2);
    d_fraw = d_gx = d_gy = d_gxi = d_gyi = d_mpmap = nullptr;
    d_u2 = nullptr;
    mp.clear();
    cudaFree(scratch.rowT);
    cudaFree(scratch.xs);
    cudaFree(scratch.alt);
    cudaFree(scratch.vec);
    scratch = InterpScratch();
    cudaFree(d_interp);
    cudaFree(d_cg);
    cudaFree(d_in);
    cudaFree(d_outbuf);
    d_interp = d_cg = d_outbuf = nullptr;
    d_in = nullptr;
    for (cudaEvent_t e : pair_ev) cudaEventDestroy(e);
    pair_ev.clear();
    if (copy_done) cudaEventDestroy(copy_done);
    copy_done = nullptr;
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

// Bicubic sweep set-up: per (magnification, radius) tap tables, all on one unit-gradient field
// whose zero halo is the widest any table needs; per-frame buffers for the shard's frames.
esrrf_status Shard::create_bic(const std::vector<float>& radii) {
    Shard* s = this;
    cudaError_t e;
    long maxP = 0;
    int padx = 0, pady = 0;
    total = 0;
    for (auto& m : mp) {
        const long P = (long)w * m.M * h * m.M;
        maxP = std::max(maxP, P);
        for (int r : m.ri) {
            const BicGeometry g = bic_geometry(radii[r], 1);
            BicTables t;
            bool built = false;
            if ((e = bic_tables_build(g, m.M, w, h, t, built, stream)) != cudaSuccess) {
                bic_tables_free(t);
                return fail_cuda(e, "RGC tables");
            }
            if (!built) {
                bic_tables_free(t);
                return fail(ESRRF_ERR_INVALID, "radius " + std::to_string(radii[r]) + " at magnification " +
                                                   std::to_string(m.M) + " reaches too far for the tabulated "
                                                   "bicubic kernel (shared memory or slab row width)");
            }
            padx = std::max(padx, t.padx);
            pady = std::max(pady, t.pady);
            m.bgeo.push_back(g);
            m.btab.push_back(t);
            offsets.push_back(total);
            total += (size_t)sens.size() * bstart.size() * 4 * P;
        }
    }
    for (auto& m : mp)
        for (auto& t : m.btab) {
            t.padx = padx;  // even: every table's padx is
            t.pady = pady;
            t.W2p = 2 * w + 2 * padx;
            t.H2p = 2 * h + 2 * pady;
        }
    const size_t plane = (size_t)w * h;
    const size_t field = bic_field_float2s(mp[0].btab[0], T);
    int maxM = 1;
    for (auto& m : mp) maxM = std::max(maxM, m.M);
    if ((e = cudaMalloc(&d_fraw, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&d_gx, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&d_gy, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&d_gxi, sizeof(float) * T * 4 * plane)) != cudaSuccess ||
        (e = cudaMalloc(&d_gyi, sizeof(float) * T * 4 * plane)) != cudaSuccess ||
        (e = cudaMalloc(&d_u2, sizeof(float2) * field)) != cudaSuccess ||
        (e = cudaMalloc(&d_mpmap, sizeof(float) * 3 * maxM * maxM)) != cudaSuccess ||
        (e = cudaMalloc(&d_interp, sizeof(float) * (size_t)T * maxP)) != cudaSuccess ||
        (e = cudaMalloc(&d_cg, sizeof(float) * (size_t)T * maxP)) != cudaSuccess)
        return fail_cuda(e, "sweep buffers");
    if ((e = cudaMemsetAsync(d_u2, 0, sizeof(float2) * field, stream)) != cudaSuccess)  // zero halo
        return fail_cuda(e, "sweep buffers");
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "sync");
    return ESRRF_OK;
}

esrrf_status Shard::create(const std::vector<float>& radii, int interp) {
    Shard* s = this;
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail_cuda(e, "stream");
    if (interp == ESRRF_INTERP_BIC) {
        bic = true;
        return create_bic(radii);
    }
    long maxP = 0;
    int maxN = 0, maxWM = 0, maxS = 4;
    total = 0;
    for (auto& m : mp) {
        if ((e = interp_plan_create(m.plan, w, h, m.M, 0)) != cudaSuccess) return fail_cuda(e, "interpolation plan");
        const long P = (long)m.plan.WM * m.plan.HM;
        maxP = std::max(maxP, P);
        maxN = std::max(maxN, m.plan.N);
        maxWM = std::max(maxWM, m.plan.WM);
        for (int r : m.ri) {
            FhtGeometry g = fht_geometry(m.M, radii[r], 1);
            if (!fht_fused_supported(g))
                return fail(ESRRF_ERR_INVALID, "radius " + std::to_string(radii[r]) + " at magnification " +
                                                   std::to_string(m.M) + " needs a tap box wider than 32 pixels");
            maxS = std::max(maxS, g.S);
            FhtFusedTables t;
            if (!drift && (e = fht_fused_tables(g, m.plan.WM, m.plan.HM, t, stream)) != cudaSuccess)
                return fail_cuda(e, "RGC tables");
            m.geo.push_back(std::move(g));
            m.tables.push_back(t);
            offsets.push_back(total);
            total += (size_t)sens.size() * bstart.size() * 4 * P;
        }
        if (drift) {  // the shifts x M (loadDriftXYGPUbuffer, LiveSRRF_CL.java:586-589)
            std::vector<float> sh(2 * (size_t)T);
            for (int t = 0; t < T; ++t) {
                sh[t] = m.M * dx[t];
                sh[T + t] = m.M * dy[t];
            }
            if ((e = cudaMalloc(&m.d_shift, sizeof(float) * 2 * T)) != cudaSuccess ||
                (e = cudaMemcpy(m.d_shift, sh.data(), sizeof(float) * 2 * T, cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail_cuda(e, "drift");
        }
    }
    scratch.capacity = std::min(16, T);
    const int Fi = scratch.capacity;
    size_t maxHM = 0, maxRowT = 0, maxXs = 0;
    for (auto& m : mp) {
        maxHM = std::max(maxHM, (size_t)m.plan.HM);
        maxRowT = std::max(maxRowT, interp_rowT_floats(m.plan));
        maxXs = std::max(maxXs, interp_xs_floats(m.plan));
    }
    if (maxXs && (e = cudaMalloc(&scratch.xs, sizeof(float) * Fi * maxXs)) != cudaSuccess)
        return fail_cuda(e, "sweep buffers");
    if ((e = cudaMalloc(&scratch.rowT, sizeof(float) * Fi * maxRowT)) != cudaSuccess ||
        (e = cudaMalloc(&scratch.alt, sizeof(float) * Fi * interp_alt_floats(maxN))) != cudaSuccess ||
        (e = cudaMalloc(&scratch.vec, sizeof(float) * Fi * interp_vec_floats((int)maxHM, maxWM))) != cudaSuccess ||
        (e = cudaMalloc(&d_interp, sizeof(float) * (size_t)T * maxP)) != cudaSuccess ||
        (e = cudaMalloc(&d_cg, sizeof(float) * (size_t)T * maxP)) != cudaSuccess)
        return fail_cuda(e, "sweep buffers");
    if (drift && (e = fht_drift_tables_alloc(maxS, T, maxP, dtab)) != cudaSuccess) return fail_cuda(e, "drift tables");
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return fail_cuda(e, "sync");
    return ESRRF_OK;
}

// Reads every plan's tensor-core failure flag after the stream has drained.
esrrf_status Shard::tc_check() {
    Shard* s = this;
    if (bic) return ESRRF_OK;
    for (auto& m : mp) {
        bool failed = false;
        SK(interp_tc_check(m.plan, stream, &failed), "interpolation status");
        if (failed) return fail(ESRRF_ERR_TIMEOUT, "interpolation tensor-core pass: a bounded wait gave up");
    }
    return ESRRF_OK;
}

// h_out: a pinned host buffer in the shard's layout that the run also fills (each pair's outputs
// copied while the next pairs compute), or null.
esrrf_status Shard::run_device(const void* d_frames, int is_u16, float* d_out, float* h_out) {
    Shard* s = this;
    if (cudaSetDevice(device) != cudaSuccess) return fail(ESRRF_ERR_CUDA, "cudaSetDevice failed");
    if (h_out && !copy_stream) {
        SK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "copy stream");
        SK(cudaEventCreateWithFlags(&copy_done, cudaEventDisableTiming), "copy event");
        pair_ev.assign(offsets.size(), nullptr);
        for (auto& e : pair_ev) SK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "pair event");
    }
    // The graph bakes in the input and output pointers: (re)capture when they change.
    if (!exec || g_in != d_frames || g_out != d_out || g_hout != h_out || g_u16 != is_u16) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        // one uncaptured pass sets the kernels' shared-memory attributes and checks the launches
        esrrf_status r = enqueue(d_frames, is_u16, d_out, h_out);
        if (r != ESRRF_OK) return r;
        SK(cudaStreamSynchronize(stream), "sweep warm-up");
        SK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        r = enqueue(d_frames, is_u16, d_out, h_out);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(stream, &g);
        if (r != ESRRF_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        SK(ce, "end capture");
        graph = g;
        SK(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
        g_in = d_frames;
        g_out = d_out;
        g_hout = h_out;
        g_u16 = is_u16;
        SK(cudaStreamSynchronize(stream), "sweep");
        return tc_check();
    }
    SK(cudaGraphLaunch(exec, stream), "graph launch");
    SK(cudaStreamSynchronize(stream), "sweep");
    return tc_check();
}

// ---------------------------------------------------------------------------------------------
// Partition of a sweep across devices.
// ---------------------------------------------------------------------------------------------

// Relative cost of one output pixel-frame of a (magnification, radius) pair: the taps of its disc
// plus a fixed share for the interpolation, the gradient and the cumulants.
double pair_cost_per_px(int M, float radius, int interp) {
    if (interp == ESRRF_INTERP_BIC) {
        const BicGeometry g = bic_geometry(radius, 1);
        const double r2 = 2.0 * g.tSO;  // taps on the 2x gradient grid
        return 3.14159265358979 * r2 * r2 + 30.0;
    }
    const FhtGeometry g = fht_geometry(M, radius, 1);
    long taps = 0;
    for (int ii = 0; ii < g.S; ++ii)
        if (g.jlo[ii] <= g.jhi[ii]) taps += g.jhi[ii] - g.jlo[ii] + 1;
    return (double)taps + 30.0;
}

struct ShardPlan {
    int device = 0;
    int slot = 0;             // index in the caller's device list (a device may be listed twice)
    std::vector<int> pairs;   // mi * n_radius + ri
    std::vector<int> blocks;  // global block indices
    double cost = 0;
};

// Mode A: the pairs in longest-processing-time order onto the least-loaded device, every device
// taking every block.  Mode B: every pair on every device, the blocks (by start) cut into contiguous
// runs whose frame spans are balanced (binary search on the largest span).  The mode with the
// smaller largest per-device cost wins; devices without work get no shard.
std::vector<ShardPlan> plan_shards(const esrrf_sweep_params& p, const std::vector<int>& devices) {
    const int nD = (int)devices.size(), nR = p.n_radius, nP = p.n_mag * p.n_radius, nB = p.n_blocks;
    std::vector<double> pc(nP);
    double pc_sum = 0;
    for (int mi = 0; mi < p.n_mag; ++mi)
        for (int ri = 0; ri < nR; ++ri) {
            const int M = p.magnifications[mi];
            pc[mi * nR + ri] = pair_cost_per_px(M, p.radii[ri], p.interp) * (double)p.width * M * p.height * M;
            pc_sum += pc[mi * nR + ri];
        }
    int lo = p.n_frames, hi = 0;
    for (int b = 0; b < nB; ++b) {
        lo = std::min(lo, p.block_start[b]);
        hi = std::max(hi, p.block_start[b] + p.block_length[b]);
    }
    const double span_all = hi - lo;
    std::vector<int> all_blocks(nB), all_pairs(nP);
    for (int b = 0; b < nB; ++b) all_blocks[b] = b;
    for (int q = 0; q < nP; ++q) all_pairs[q] = q;
    if (nD <= 1) {
        ShardPlan s;
        s.device = nD ? devices[0] : 0;
        s.slot = 0;
        s.pairs = all_pairs;
        s.blocks = all_blocks;
        s.cost = pc_sum * span_all;
        return {s};
    }
    // mode A
    std::vector<ShardPlan> a(nD);
    for (int d = 0; d < nD; ++d) {
        a[d].device = devices[d];
        a[d].slot = d;
    }
    std::vector<int> order(nP);
    for (int q = 0; q < nP; ++q) order[q] = q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return pc[x] > pc[y]; });
    for (int q : order) {
        int best = 0;
        for (int d = 1; d < nD; ++d)
            if (a[d].cost < a[best].cost) best = d;
        a[best].pairs.push_back(q);
        a[best].cost += pc[q] * span_all;
    }
    double make_a = 0;
    for (auto& s : a) {
        std::sort(s.pairs.begin(), s.pairs.end());
        s.blocks = all_blocks;
        make_a = std::max(make_a, s.cost);
    }
    // mode B
    std::vector<int> bo(nB);
    for (int b = 0; b < nB; ++b) bo[b] = b;
    std::stable_sort(bo.begin(), bo.end(), [&](int x, int y) { return p.block_start[x] < p.block_start[y]; });
    auto cut = [&](int L, std::vector<std::vector<int>>* groups) {
        int n = 0, g0 = 0, gend = 0;
        for (int k = 0; k < nB; ++k) {
            const int b = bo[k], s = p.block_start[b], e = s + p.block_length[b];
            if (k == 0 || std::max(gend, e) - g0 > L) {
                ++n;
                g0 = s;
                gend = e;
                if (groups) groups->emplace_back();
            } else {
                gend = std::max(gend, e);
            }
            if (groups) groups->back().push_back(b);
        }
        return n;
    };
    int Lmin = 1, Lmax = (int)span_all;
    for (int b = 0; b < nB; ++b) Lmin = std::max(Lmin, p.block_length[b]);
    while (Lmin < Lmax) {
        const int mid = Lmin + (Lmax - Lmin) / 2;
        if (cut(mid, nullptr) <= nD) Lmax = mid;
        else Lmin = mid + 1;
    }
    std::vector<std::vector<int>> groups;
    cut(Lmin, &groups);
    std::vector<ShardPlan> bplan;
    double make_b = 0;
    for (size_t g = 0; g < groups.size(); ++g) {
        ShardPlan s;
        s.device = devices[g];
        s.slot = (int)g;
        s.pairs = all_pairs;
        s.blocks = groups[g];
        std::sort(s.blocks.begin(), s.blocks.end());
        int glo = p.n_frames, ghi = 0;
        for (int b : s.blocks) {
            glo = std::min(glo, p.block_start[b]);
            ghi = std::max(ghi, p.block_start[b] + p.block_length[b]);
        }
        s.cost = pc_sum * (ghi - glo);
        make_b = std::max(make_b, s.cost);
        bplan.push_back(std::move(s));
    }
    std::vector<ShardPlan> out;
    for (auto& s : (make_b < make_a ? bplan : a))
        if (!s.pairs.empty() && !s.blocks.empty()) out.push_back(std::move(s));
    return out;
}

std::mutex g_sweep_mu;
std::string g_sweep_create_error;

esrrf_status reject(const std::string& m) {
    std::lock_guard<std::mutex> lk(g_sweep_mu);
    g_sweep_create_error = m;
    return ESRRF_ERR_INVALID;
}

// Host-side validation shared by esrrf_sweep_create and esrrf_sweep_plan (no device work).
esrrf_status validate(const esrrf_sweep_params* sp) {
    if (sp->width < 4 || sp->height < 4 || sp->n_frames < 1) return reject("bad stack size");
    if (sp->n_mag < 1 || !sp->magnifications || sp->n_radius < 1 || !sp->radii || sp->n_sens < 1 ||
        !sp->sensitivities || sp->n_blocks < 1 || !sp->block_start || !sp->block_length)
        return reject("magnifications, radii, sensitivities and blocks must be non-empty");
    for (int b = 0; b < sp->n_blocks; ++b)
        if (sp->block_start[b] < 0 || sp->block_length[b] < 1 ||
            sp->block_start[b] + sp->block_length[b] > sp->n_frames)
            return reject("block " + std::to_string(b) + " lies outside the stack");
    for (int i = 0; i < sp->n_mag; ++i) {
        if (sp->magnifications[i] < 1 || sp->magnifications[i] > 16) return reject("magnification out of range");
        const long long M = sp->magnifications[i];
        if ((long long)sp->width * M * ((long long)sp->height * M) > 2147483647LL)
            return reject("output too large: width x height x magnification^2 must stay below 2^31 pixels");
    }
    for (int i = 0; i < sp->n_radius; ++i)
        if (!(sp->radii[i] > 0.f) || sp->radii[i] > 20.f) return reject("radius out of range");
    for (int i = 0; i < sp->n_sens; ++i)
        if (sp->sensitivities[i] < 0 || sp->sensitivities[i] > 64) return reject("sensitivity out of range");
    if (sp->interp != ESRRF_INTERP_FHT && sp->interp != ESRRF_INTERP_BIC) return reject("unknown interpolation");
    if ((sp->drift_x == nullptr) != (sp->drift_y == nullptr))
        return reject("drift_x and drift_y must both be given or both be NULL");
    if (sp->drift_x)
        for (int t = 0; t < sp->n_frames; ++t)
            if (!(std::fabs(sp->drift_x[t]) <= 1e6f) || !(std::fabs(sp->drift_y[t]) <= 1e6f))
                return reject("drift shifts must be finite and at most 1e6 pixels");
    if (sp->drift_x && sp->interp == ESRRF_INTERP_BIC)
        return reject("drift correction is available in the FHT sweep only (run the bicubic engine per block)");
    if (sp->n_devices < 0 || (sp->n_devices > 0 && !sp->devices)) return reject("bad device list");
    return ESRRF_OK;
}

std::vector<int> device_list(const esrrf_sweep_params* sp) {
    if (sp->n_devices > 0) return std::vector<int>(sp->devices, sp->devices + sp->n_devices);
    return {sp->device >= 0 ? sp->device : 0};
}

}  // namespace

struct esrrf_sweep {
    esrrf_sweep_params p{};
    std::vector<int> mags, sens, bstart, blen, devices;
    std::vector<float> radii, dx, dy;
    std::vector<Shard*> shards;
    std::vector<size_t> offsets;  // global layout per (magnification, radius)
    size_t total = 0;
    std::string err;

    // the single shard holds every pair and block in order: its layout is the global one
    bool direct() const { return shards.size() == 1 && shards[0]->total == total && shards[0]->f0 == 0; }
    esrrf_status fail(esrrf_status s, const std::string& m) {
        err = m;
        return s;
    }
    void release() {
        for (Shard* s : shards) {
            s->release();
            delete s;
        }
        shards.clear();
    }
};

extern "C" {

esrrf_status esrrf_sweep_plan(const esrrf_sweep_params* sp, int* pair_device, int* block_device,
                              double* device_cost) {
    if (!sp) return ESRRF_ERR_INVALID;
    esrrf_status r = validate(sp);
    if (r != ESRRF_OK) return r;
    const std::vector<int> devs = device_list(sp);
    const std::vector<ShardPlan> plan = plan_shards(*sp, devs);
    const int nP = sp->n_mag * sp->n_radius;
    for (int q = 0; q < nP && pair_device; ++q) pair_device[q] = -2;  // not assigned
    for (int b = 0; b < sp->n_blocks && block_device; ++b) block_device[b] = -2;
    for (size_t d = 0; d < devs.size() && device_cost; ++d) device_cost[d] = 0;
    for (const ShardPlan& s : plan) {
        const int di = s.slot;
        const bool all_pairs = (int)s.pairs.size() == nP, all_blocks = (int)s.blocks.size() == sp->n_blocks;
        if (pair_device)
            for (int q : s.pairs) pair_device[q] = all_pairs && plan.size() > 1 ? -1 : s.device;
        if (block_device)
            for (int b : s.blocks) block_device[b] = all_blocks && plan.size() > 1 ? -1 : s.device;
        if (device_cost) device_cost[di] = s.cost;
    }
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_create(const esrrf_sweep_params* sp, esrrf_sweep** out) {
    if (!sp || !out) return ESRRF_ERR_INVALID;
    *out = nullptr;
    esrrf_status vr = validate(sp);
    if (vr != ESRRF_OK) return vr;

    esrrf_sweep* s = new esrrf_sweep();
    s->p = *sp;
    s->mags.assign(sp->magnifications, sp->magnifications + sp->n_mag);
    s->radii.assign(sp->radii, sp->radii + sp->n_radius);
    s->sens.assign(sp->sensitivities, sp->sensitivities + sp->n_sens);
    s->bstart.assign(sp->block_start, sp->block_start + sp->n_blocks);
    s->blen.assign(sp->block_length, sp->block_length + sp->n_blocks);
    s->devices = device_list(sp);
    bool any_drift = false;
    if (sp->drift_x) {
        s->dx.assign(sp->drift_x, sp->drift_x + sp->n_frames);
        s->dy.assign(sp->drift_y, sp->drift_y + sp->n_frames);
        for (int t = 0; t < sp->n_frames; ++t) any_drift |= s->dx[t] != 0.f || s->dy[t] != 0.f;
    }
    s->p.magnifications = nullptr;
    s->p.radii = nullptr;
    s->p.sensitivities = nullptr;
    s->p.block_start = s->p.block_length = nullptr;
    s->p.drift_x = s->p.drift_y = nullptr;
    s->p.devices = nullptr;
    auto bail = [&](esrrf_status st, const std::string& m) {
        {
            std::lock_guard<std::mutex> lk(g_sweep_mu);
            g_sweep_create_error = m;
        }
        s->release();
        delete s;
        return st;
    };
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return bail(ESRRF_ERR_NODEVICE, "no CUDA device");
    }
    for (int d : s->devices)
        if (d < 0 || d >= ndev) return bail(ESRRF_ERR_INVALID, "device " + std::to_string(d) + " does not exist");
    // global output layout
    const int nR = (int)s->radii.size();
    s->total = 0;
    for (int mi = 0; mi < sp->n_mag; ++mi)
        for (int ri = 0; ri < nR; ++ri) {
            s->offsets.push_back(s->total);
            s->total += s->sens.size() * s->bstart.size() * 4 * (size_t)sp->width * s->mags[mi] * sp->height * s->mags[mi];
        }
    // one shard per device of the plan, created in parallel
    const std::vector<ShardPlan> plan = plan_shards(*sp, s->devices);
    for (const ShardPlan& sp_ : plan) {
        Shard* sh = new Shard();
        sh->device = sp_.device;
        sh->w = sp->width;
        sh->h = sp->height;
        sh->int_weighting = sp->int_weighting;
        sh->sens = s->sens;
        int lo = sp->n_frames, hi = 0;
        for (int b : sp_.blocks) {
            lo = std::min(lo, s->bstart[b]);
            hi = std::max(hi, s->bstart[b] + s->blen[b]);
        }
        // a single-device sweep keeps the whole stack (its layout and frame indices are the caller's)
        if (plan.size() == 1) {
            lo = 0;
            hi = sp->n_frames;
        }
        sh->f0 = lo;
        sh->T = hi - lo;
        for (int b : sp_.blocks) {
            sh->bstart.push_back(s->bstart[b] - lo);
            sh->blen.push_back(s->blen[b]);
            sh->bglob.push_back(b);
        }
        for (int q : sp_.pairs) {
            const int mi = q / nR, ri = q % nR;
            if (sh->mp.empty() || sh->mp.back().mi != mi) {
                sh->mp.emplace_back();
                sh->mp.back().mi = mi;
                sh->mp.back().M = s->mags[mi];
            }
            sh->mp.back().ri.push_back(ri);
        }
        if (any_drift) {
            sh->drift = true;
            sh->dx.assign(s->dx.begin() + lo, s->dx.begin() + hi);
            sh->dy.assign(s->dy.begin() + lo, s->dy.begin() + hi);
        }
        s->shards.push_back(sh);
    }
    std::vector<esrrf_status> rs(s->shards.size(), ESRRF_OK);
    std::vector<std::thread> th;
    for (size_t i = 0; i < s->shards.size(); ++i)
        th.emplace_back([&, i] { rs[i] = s->shards[i]->create(s->radii, sp->interp); });
    for (auto& t : th) t.join();
    for (size_t i = 0; i < s->shards.size(); ++i)
        if (rs[i] != ESRRF_OK) return bail(rs[i], s->shards[i]->err);
    *out = s;
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_output_layout(const esrrf_sweep* s, size_t* total_floats, size_t* offsets) {
    if (!s) return ESRRF_ERR_INVALID;
    if (total_floats) *total_floats = s->total;
    if (offsets)
        for (size_t i = 0; i < s->offsets.size(); ++i) offsets[i] = s->offsets[i];
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_run_device(esrrf_sweep* s, const void* d_frames, int is_u16, float* d_out) {
    if (!s || !d_frames || !d_out) return ESRRF_ERR_INVALID;
    if (!s->direct())
        return s->fail(ESRRF_ERR_INVALID, "a sweep split across devices takes host frames (esrrf_sweep_run)");
    esrrf_status r = s->shards[0]->run_device(d_frames, is_u16, d_out);
    if (r != ESRRF_OK) s->err = s->shards[0]->err;
    return r;
}

esrrf_status esrrf_sweep_run(esrrf_sweep* s, const void* frames, int is_u16, float* out) {
    if (!s || !frames || !out) return ESRRF_ERR_INVALID;
    const size_t fbytes = (is_u16 ? sizeof(uint16_t) : sizeof(float)) * (size_t)s->p.width * s->p.height;
    const bool direct = s->direct();
    // a pinned output buffer of a one-shard sweep is filled pair by pair during the run
    bool overlap = false;
    if (direct && s->total > 0) {
        cudaPointerAttributes a0{}, a1{};
        overlap = cudaPointerGetAttributes(&a0, out) == cudaSuccess && a0.type == cudaMemoryTypeHost &&
                  cudaPointerGetAttributes(&a1, out + s->total - 1) == cudaSuccess && a1.type == cudaMemoryTypeHost;
        cudaGetLastError();
    }
    std::vector<esrrf_status> rs(s->shards.size(), ESRRF_OK);
    auto work = [&](size_t i) -> esrrf_status {
        Shard* sh = s->shards[i];
        if (cudaSetDevice(sh->device) != cudaSuccess) return sh->fail(ESRRF_ERR_CUDA, "cudaSetDevice failed");
        if (!sh->d_in) SKS(cudaMalloc(&sh->d_in, sizeof(float) * (size_t)s->p.width * s->p.height * sh->T), "input buffer");
        if (!sh->d_outbuf) SKS(cudaMalloc(&sh->d_outbuf, sizeof(float) * sh->total), "output buffer");
        SKS(cudaMemcpyAsync(sh->d_in, (const unsigned char*)frames + fbytes * sh->f0, fbytes * sh->T,
                            cudaMemcpyHostToDevice, sh->stream), "input copy");
        if (overlap) return sh->run_device(sh->d_in, is_u16, sh->d_outbuf, out);
        esrrf_status r = sh->run_device(sh->d_in, is_u16, sh->d_outbuf);
        if (r != ESRRF_OK) return r;
        if (direct) {
            SKS(cudaMemcpyAsync(out, sh->d_outbuf, sizeof(float) * s->total, cudaMemcpyDeviceToHost, sh->stream),
                "output copy");
        } else {  // gather: each (pair, sensitivity, local block) to its place in the global layout
            const int nR = (int)s->radii.size(), nB = (int)s->bstart.size();
            const int nS = (int)s->sens.size(), nBl = (int)sh->bstart.size();
            size_t oi = 0;
            for (const MagPlan& m : sh->mp) {
                const size_t P = (size_t)s->p.width * m.M * s->p.height * m.M;
                for (int ri : m.ri) {
                    const float* src = sh->d_outbuf + sh->offsets[oi++];
                    float* dst = out + s->offsets[m.mi * nR + ri];
                    for (int si = 0; si < nS; ++si)
                        for (int bl = 0; bl < nBl; ++bl)
                            SKS(cudaMemcpyAsync(dst + ((size_t)si * nB + sh->bglob[bl]) * 4 * P,
                                                src + ((size_t)si * nBl + bl) * 4 * P, sizeof(float) * 4 * P,
                                                cudaMemcpyDeviceToHost, sh->stream),
                                "output copy");
                }
            }
        }
        SKS(cudaStreamSynchronize(sh->stream), "sweep");
        return ESRRF_OK;
    };
    if (s->shards.size() == 1) {
        rs[0] = work(0);
    } else {
        std::vector<std::thread> th;
        for (size_t i = 0; i < s->shards.size(); ++i) th.emplace_back([&, i] { rs[i] = work(i); });
        for (auto& t : th) t.join();
    }
    for (size_t i = 0; i < s->shards.size(); ++i)
        if (rs[i] != ESRRF_OK) {
            s->err = "device " + std::to_string(s->shards[i]->device) + ": " + s->shards[i]->err;
            return rs[i];
        }
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_launch_count(const esrrf_sweep* s, int* launches) {
    if (!s || !launches) return ESRRF_ERR_INVALID;
    int n = 0;
    for (const Shard* sh : s->shards) n += sh->launches_per_run;
    *launches = n;
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_shard_count(const esrrf_sweep* s, int* shards) {
    if (!s || !shards) return ESRRF_ERR_INVALID;
    *shards = (int)s->shards.size();
    return ESRRF_OK;
}

const char* esrrf_sweep_last_error(const esrrf_sweep* s) {
    if (!s) {
        std::lock_guard<std::mutex> lk(g_sweep_mu);
        return g_sweep_create_error.c_str();
    }
    return s->err.c_str();
}

esrrf_status esrrf_sweep_destroy(esrrf_sweep* s) {
    if (!s) return ESRRF_ERR_INVALID;
    s->release();
    delete s;
    return ESRRF_OK;
}

}  // extern "C"
