// sweep.cu -- batched parameter sweep and rolling analysis over uneven frame blocks.
//
// The reference's ParametersSweep_ (gui/ParametersSweep_.java:328-519) re-initialises the
// engine -- context, program build, buffers, per-frame upload -- for every (radius, sensitivity)
// combination, and its rolling analysis (gui/LiveSRRF_optimised_.java:276-389) recomputes every
// frame once per block that contains it.  Here one captured CUDA graph does the whole sweep:
//   per magnification: Fourier-interpolate every frame once (interp.cu);
//   per radius: one fused-RGC launch over all frames that writes CGLH / sum-of-weights per frame
//     (the tap loop is shared by every sensitivity and every block);
//   per (sensitivity group, block group): one memory-bound launch that raises CGLH to the
//     sensitivity, weights it by the interpolated intensity and reduces AVG/VAR/TAC2/INT over each
//     block, FP64 accumulators in registers.
// The bicubic sweep (the reference sweep with "Use FHT interpolation" off) computes the 2-point
// gradients, their 2x resampling and the unit-gradient field of every frame once (none depends on
// the magnification or radius); per (magnification, radius) the tabulated bicubic RGC writes
// CGLH / sum of weights and the bicubic intensity of every frame; the cumulant launches apply the
// path's double (n - 1) division of TAC2, and every output gets the MP correction.
// Output: for each magnification, radius, sensitivity and block, the four [HM][WM] slices of
// readSRRFbuffer (AVG, VAR, TAC2, INT; NaN -> 0).
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
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
    for (int t = t_lo; t < t_hi; ++t) {
        const float c = __ldg(a.cg + (long)t * a.P + pix);
        const float v = __ldg(a.v + (long)t * a.P + pix);
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
    }
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

struct MagPlan {
    int M = 0;
    InterpPlan plan;
    std::vector<FhtGeometry> geo;       // per radius
    std::vector<FhtFusedTables> tables; // per radius
    std::vector<BicGeometry> bgeo;      // bicubic sweep: per radius
    std::vector<BicTables> btab;        // bicubic sweep: per radius (common field padding)
};

}  // namespace

struct esrrf_sweep {
    esrrf_sweep_params p{};
    std::vector<int> mags, sens, bstart, blen;
    std::vector<float> radii;
    int device = -1;
    cudaStream_t stream = nullptr;
    std::vector<MagPlan> mp;
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
    std::vector<size_t> offsets;
    size_t total = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* g_in = nullptr;
    float* g_out = nullptr;
    int g_u16 = -1;
    int launches_per_run = 0;
    std::string err;

    esrrf_status fail(esrrf_status s, const std::string& m) {
        err = m;
        return s;
    }
    esrrf_status fail_cuda(cudaError_t e, const char* what) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? ESRRF_ERR_NOMEM : ESRRF_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    }
    esrrf_status enqueue(const void* frames, int is_u16, float* out);
    esrrf_status enqueue_bic(const void* frames, int is_u16, float* out);
    void release();
};

#define SK(call, what)                                         \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return s->fail_cuda(_e, what);  \
    } while (0)

esrrf_status esrrf_sweep::enqueue(const void* frames, int is_u16, float* out) {
    esrrf_sweep* s = this;
    const int T = p.n_frames;
    const size_t fb = (is_u16 ? sizeof(uint16_t) : sizeof(float)) * (size_t)p.width * p.height;
    int launches = 0;
    if (bic) return enqueue_bic(frames, is_u16, out);
    for (size_t mi = 0; mi < mp.size(); ++mi) {
        const MagPlan& m = mp[mi];
        const long P = (long)m.plan.WM * m.plan.HM;
        for (int t = 0; t < T; t += scratch.capacity) {
            const int Fn = std::min(scratch.capacity, T - t);
            SK(interp_run(m.plan, scratch, (const unsigned char*)frames + fb * t, is_u16 != 0, Fn,
                          d_interp + (size_t)t * P, stream, &launches),
               "interpolation");
        }
        for (size_t ri = 0; ri < radii.size(); ++ri) {
            FhtRgcArgs a{};
            a.interp = d_interp;
            a.W = m.plan.WM;
            a.H = m.plan.HM;
            a.F = T;
            a.t0 = 0;
            a.int_weighting = p.int_weighting;
            a.cg_out = d_cg;
            SK(fht_rgc_fused(m.geo[ri], m.tables[ri], a, stream), "RGC");
            ++launches;
            float* base = out + offsets[mi * radii.size() + ri];
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
                    c.int_weighting = p.int_weighting;
                    c.out = base;
                    c.s0 = s0;
                    c.b0 = b0;
                    c.nB = (int)bstart.size();
                    sweep_cumulants_kernel<<<(unsigned)((P + 255) / 256), 256, 0, stream>>>(c);
                    SK(cudaGetLastError(), "cumulants");
                    ++launches;
                }
        }
    }
    launches_per_run = launches;
    return ESRRF_OK;
}

esrrf_status esrrf_sweep::enqueue_bic(const void* frames, int is_u16, float* out) {
    esrrf_sweep* s = this;
    const int T = p.n_frames, w = p.width, h = p.height;
    int launches = 0;
    SK(bic_prepare(frames, is_u16, w, h, T, d_fraw, d_gx, d_gy, d_gxi, d_gyi, stream), "gradients");
    launches += 3;
    SK(unit_grad2d(d_gxi, d_gyi, w, h, T, mp[0].btab[0], d_u2, stream), "unit gradient");
    ++launches;
    for (size_t mi = 0; mi < mp.size(); ++mi) {
        const MagPlan& m = mp[mi];
        const long P = (long)w * m.M * h * m.M;
        for (size_t ri = 0; ri < radii.size(); ++ri) {
            BicTabArgs a{};
            a.U = d_u2;
            a.fraw = d_fraw;
            a.w = w;
            a.h = h;
            a.M = m.M;
            a.F = T;
            a.t0 = 0;
            a.sens = 1.f;
            a.int_weighting = p.int_weighting;
            a.tab = m.btab[ri];
            a.cg_out = d_cg;
            a.v_out = d_interp;
            SK(bic_rgc_tab(a, stream), "RGC");
            ++launches;
            float* base = out + offsets[mi * radii.size() + ri];
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
                    c.int_weighting = p.int_weighting;
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
        }
    }
    launches_per_run = launches;
    return ESRRF_OK;
}

void esrrf_sweep::release() {
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    for (auto& m : mp) {
        interp_plan_destroy(m.plan);
        for (auto& t : m.tables) fht_fused_tables_free(t);
        for (auto& t : m.btab) bic_tables_free(t);
    }
    for (float* b : {d_fraw, d_gx, d_gy, d_gxi, d_gyi, d_mpmap}) cudaFree(b);
    cudaFree(d_u2);
    d_fraw = d_gx = d_gy = d_gxi = d_gyi = d_mpmap = nullptr;
    d_u2 = nullptr;
    mp.clear();
    cudaFree(scratch.rowT);
    cudaFree(scratch.xs);
    cudaFree(scratch.alt);
    cudaFree(scratch.vec);
    cudaFree(d_interp);
    cudaFree(d_cg);
    cudaFree(d_in);
    cudaFree(d_outbuf);
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

namespace {
std::mutex g_sweep_mu;
std::string g_sweep_create_error;
}  // namespace

// Bicubic sweep set-up: per (magnification, radius) tap tables, all on one unit-gradient field
// whose zero halo is the widest any table needs; per-frame buffers for the whole stack.
static esrrf_status sweep_create_bic(esrrf_sweep* s) {
    const int w = s->p.width, h = s->p.height, T = s->p.n_frames;
    cudaError_t e;
    long maxP = 0;
    int padx = 0, pady = 0;
    s->total = 0;
    for (int M : s->mags) {
        s->mp.emplace_back();
        MagPlan& m = s->mp.back();
        m.M = M;
        const long P = (long)w * M * h * M;
        maxP = std::max(maxP, P);
        for (float r : s->radii) {
            const BicGeometry g = bic_geometry(r, 1);
            BicTables t;
            bool built = false;
            if ((e = bic_tables_build(g, M, w, h, t, built, s->stream)) != cudaSuccess) {
                bic_tables_free(t);
                return s->fail_cuda(e, "RGC tables");
            }
            if (!built) {
                bic_tables_free(t);
                return s->fail(ESRRF_ERR_INVALID, "radius " + std::to_string(r) + " at magnification " +
                                                      std::to_string(M) + " reaches too far for the tabulated "
                                                      "bicubic kernel (shared memory or slab row width)");
            }
            padx = std::max(padx, t.padx);
            pady = std::max(pady, t.pady);
            m.bgeo.push_back(g);
            m.btab.push_back(t);
            s->offsets.push_back(s->total);
            s->total += (size_t)s->sens.size() * s->bstart.size() * 4 * P;
        }
    }
    for (auto& m : s->mp)
        for (auto& t : m.btab) {
            t.padx = padx;  // even: every table's padx is
            t.pady = pady;
            t.W2p = 2 * w + 2 * padx;
            t.H2p = 2 * h + 2 * pady;
        }
    const size_t plane = (size_t)w * h;
    const size_t field = bic_field_float2s(s->mp[0].btab[0], T);
    int maxM = 1;
    for (int M : s->mags) maxM = std::max(maxM, M);
    if ((e = cudaMalloc(&s->d_fraw, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_gx, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_gy, sizeof(float) * T * plane)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_gxi, sizeof(float) * T * 4 * plane)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_gyi, sizeof(float) * T * 4 * plane)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_u2, sizeof(float2) * field)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_mpmap, sizeof(float) * 3 * maxM * maxM)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_interp, sizeof(float) * (size_t)T * maxP)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_cg, sizeof(float) * (size_t)T * maxP)) != cudaSuccess)
        return s->fail_cuda(e, "sweep buffers");
    if ((e = cudaMemsetAsync(s->d_u2, 0, sizeof(float2) * field, s->stream)) != cudaSuccess)  // zero halo
        return s->fail_cuda(e, "sweep buffers");
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return s->fail_cuda(e, "sync");
    return ESRRF_OK;
}

extern "C" {

esrrf_status esrrf_sweep_create(const esrrf_sweep_params* sp, esrrf_sweep** out) {
    if (!sp || !out) return ESRRF_ERR_INVALID;
    *out = nullptr;
    auto reject = [](const std::string& m) {
        std::lock_guard<std::mutex> lk(g_sweep_mu);
        g_sweep_create_error = m;
        return ESRRF_ERR_INVALID;
    };
    if (sp->width < 4 || sp->height < 4 || sp->n_frames < 1) return reject("bad stack size");
    if (sp->n_mag < 1 || !sp->magnifications || sp->n_radius < 1 || !sp->radii || sp->n_sens < 1 ||
        !sp->sensitivities || sp->n_blocks < 1 || !sp->block_start || !sp->block_length)
        return reject("magnifications, radii, sensitivities and blocks must be non-empty");
    for (int b = 0; b < sp->n_blocks; ++b)
        if (sp->block_start[b] < 0 || sp->block_length[b] < 1 ||
            sp->block_start[b] + sp->block_length[b] > sp->n_frames)
            return reject("block " + std::to_string(b) + " lies outside the stack");
    for (int i = 0; i < sp->n_mag; ++i)
        if (sp->magnifications[i] < 1 || sp->magnifications[i] > 16) return reject("magnification out of range");
    for (int i = 0; i < sp->n_radius; ++i)
        if (!(sp->radii[i] > 0.f) || sp->radii[i] > 20.f) return reject("radius out of range");
    for (int i = 0; i < sp->n_sens; ++i)
        if (sp->sensitivities[i] < 0 || sp->sensitivities[i] > 64) return reject("sensitivity out of range");
    if (sp->interp != ESRRF_INTERP_FHT && sp->interp != ESRRF_INTERP_BIC) return reject("unknown interpolation");

    esrrf_sweep* s = new esrrf_sweep();
    s->p = *sp;
    s->mags.assign(sp->magnifications, sp->magnifications + sp->n_mag);
    s->radii.assign(sp->radii, sp->radii + sp->n_radius);
    s->sens.assign(sp->sensitivities, sp->sensitivities + sp->n_sens);
    s->bstart.assign(sp->block_start, sp->block_start + sp->n_blocks);
    s->blen.assign(sp->block_length, sp->block_length + sp->n_blocks);
    s->p.magnifications = nullptr;
    s->p.radii = nullptr;
    s->p.sensitivities = nullptr;
    s->p.block_start = s->p.block_length = nullptr;
    auto bail = [&](esrrf_status st) {
        {
            std::lock_guard<std::mutex> lk(g_sweep_mu);
            g_sweep_create_error = s->err;
        }
        s->release();
        delete s;
        return st;
    };
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        s->err = "no CUDA device";
        return bail(ESRRF_ERR_NODEVICE);
    }
    s->device = sp->device >= 0 ? sp->device : 0;
    cudaError_t e;
    if ((e = cudaSetDevice(s->device)) != cudaSuccess) return bail(s->fail_cuda(e, "cudaSetDevice"));
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(s->fail_cuda(e, "stream"));
    if (sp->interp == ESRRF_INTERP_BIC) {
        s->bic = true;
        esrrf_status r = sweep_create_bic(s);
        if (r != ESRRF_OK) return bail(r);
        *out = s;
        return ESRRF_OK;
    }
    long maxP = 0;
    int maxN = 0, maxWM = 0;
    s->total = 0;
    for (int M : s->mags) {
        s->mp.emplace_back();
        MagPlan& m = s->mp.back();
        m.M = M;
        if ((e = interp_plan_create(m.plan, sp->width, sp->height, M, 0)) != cudaSuccess)
            return bail(s->fail_cuda(e, "interpolation plan"));
        const long P = (long)m.plan.WM * m.plan.HM;
        maxP = std::max(maxP, P);
        maxN = std::max(maxN, m.plan.N);
        maxWM = std::max(maxWM, m.plan.WM);
        for (float r : s->radii) {
            FhtGeometry g = fht_geometry(M, r, 1);
            if (!fht_fused_supported(g)) {
                s->err = "radius " + std::to_string(r) + " at magnification " + std::to_string(M) +
                         " needs a tap box wider than 32 pixels";
                return bail(ESRRF_ERR_INVALID);
            }
            FhtFusedTables t;
            if ((e = fht_fused_tables(g, m.plan.WM, m.plan.HM, t, s->stream)) != cudaSuccess)
                return bail(s->fail_cuda(e, "RGC tables"));
            m.geo.push_back(std::move(g));
            m.tables.push_back(t);
            s->offsets.push_back(s->total);
            s->total += (size_t)s->sens.size() * s->bstart.size() * 4 * P;
        }
    }
    const int T = sp->n_frames;
    s->scratch.capacity = std::min(16, T);
    const int Fi = s->scratch.capacity;
    size_t maxHM = 0, maxRowT = 0, maxXs = 0;
    for (auto& m : s->mp) {
        maxHM = std::max(maxHM, (size_t)m.plan.HM);
        maxRowT = std::max(maxRowT, interp_rowT_floats(m.plan));
        maxXs = std::max(maxXs, interp_xs_floats(m.plan));
    }
    if (maxXs && (e = cudaMalloc(&s->scratch.xs, sizeof(float) * Fi * maxXs)) != cudaSuccess)
        return bail(s->fail_cuda(e, "sweep buffers"));
    if ((e = cudaMalloc(&s->scratch.rowT, sizeof(float) * Fi * maxRowT)) != cudaSuccess ||
        (e = cudaMalloc(&s->scratch.alt, sizeof(float) * Fi * interp_alt_floats(maxN))) != cudaSuccess ||
        (e = cudaMalloc(&s->scratch.vec, sizeof(float) * Fi * interp_vec_floats((int)maxHM, maxWM))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_interp, sizeof(float) * (size_t)T * maxP)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_cg, sizeof(float) * (size_t)T * maxP)) != cudaSuccess)
        return bail(s->fail_cuda(e, "sweep buffers"));
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return bail(s->fail_cuda(e, "sync"));
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

// Reads every plan's tensor-core failure flag after the stream has drained.
static esrrf_status sweep_tc_check(esrrf_sweep* s) {
    if (s->bic) return ESRRF_OK;
    for (auto& m : s->mp) {
        bool failed = false;
        SK(interp_tc_check(m.plan, s->stream, &failed), "interpolation status");
        if (failed) return s->fail(ESRRF_ERR_TIMEOUT, "interpolation tensor-core pass: a bounded wait gave up");
    }
    return ESRRF_OK;
}

static esrrf_status sweep_run_device(esrrf_sweep* s, const void* d_frames, int is_u16, float* d_out) {
    if (cudaSetDevice(s->device) != cudaSuccess) return s->fail(ESRRF_ERR_CUDA, "cudaSetDevice failed");
    // The graph bakes in the input and output pointers: (re)capture when they change.
    if (!s->exec || s->g_in != d_frames || s->g_out != d_out || s->g_u16 != is_u16) {
        if (s->exec) cudaGraphExecDestroy(s->exec);
        if (s->graph) cudaGraphDestroy(s->graph);
        s->exec = nullptr;
        s->graph = nullptr;
        // one uncaptured pass sets the kernels' shared-memory attributes and checks the launches
        esrrf_status r = s->enqueue(d_frames, is_u16, d_out);
        if (r != ESRRF_OK) return r;
        SK(cudaStreamSynchronize(s->stream), "sweep warm-up");
        SK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        r = s->enqueue(d_frames, is_u16, d_out);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
        if (r != ESRRF_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        SK(ce, "end capture");
        s->graph = g;
        SK(cudaGraphInstantiate(&s->exec, s->graph, 0), "graph instantiate");
        s->g_in = d_frames;
        s->g_out = d_out;
        s->g_u16 = is_u16;
        SK(cudaStreamSynchronize(s->stream), "sweep");
        return sweep_tc_check(s);
    }
    SK(cudaGraphLaunch(s->exec, s->stream), "graph launch");
    SK(cudaStreamSynchronize(s->stream), "sweep");
    return sweep_tc_check(s);
}

esrrf_status esrrf_sweep_run_device(esrrf_sweep* s, const void* d_frames, int is_u16, float* d_out) {
    if (!s || !d_frames || !d_out) return ESRRF_ERR_INVALID;
    return sweep_run_device(s, d_frames, is_u16, d_out);
}

esrrf_status esrrf_sweep_run(esrrf_sweep* s, const void* frames, int is_u16, float* out) {
    if (!s || !frames || !out) return ESRRF_ERR_INVALID;
    if (cudaSetDevice(s->device) != cudaSuccess) return s->fail(ESRRF_ERR_CUDA, "cudaSetDevice failed");
    const size_t in_bytes = (is_u16 ? sizeof(uint16_t) : sizeof(float)) * (size_t)s->p.width *
                            s->p.height * s->p.n_frames;
    if (!s->d_in) SK(cudaMalloc(&s->d_in, sizeof(float) * (size_t)s->p.width * s->p.height * s->p.n_frames),
                     "input buffer");
    if (!s->d_outbuf) SK(cudaMalloc(&s->d_outbuf, sizeof(float) * s->total), "output buffer");
    SK(cudaMemcpyAsync(s->d_in, frames, in_bytes, cudaMemcpyHostToDevice, s->stream), "input copy");
    esrrf_status r = sweep_run_device(s, s->d_in, is_u16, s->d_outbuf);
    if (r != ESRRF_OK) return r;
    SK(cudaMemcpyAsync(out, s->d_outbuf, sizeof(float) * s->total, cudaMemcpyDeviceToHost, s->stream),
       "output copy");
    SK(cudaStreamSynchronize(s->stream), "sweep");
    return ESRRF_OK;
}

esrrf_status esrrf_sweep_launch_count(const esrrf_sweep* s, int* launches) {
    if (!s || !launches) return ESRRF_ERR_INVALID;
    *launches = s->launches_per_run;
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
