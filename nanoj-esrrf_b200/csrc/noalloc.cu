// noalloc.cu -- an allocation-free entry point for one FHT-path SR block.
//
// Some callers of this library cannot allocate device memory at the moment they need a
// reconstruction: a live-acquisition callback (for example a camera frame handler in a
// microscope-control host) must not call cudaMalloc/cudaFree, because those calls can
// synchronise the whole device and stall the acquisition stream, and hosts that manage every
// device byte through their own pool or budget forbid allocations behind their back.  For them,
// esrrf_fht_block_noalloc() runs the same interpolation + fused RGC + FP64 finalisation as an
// esrrf_create() handle, but takes every temporary buffer from one file-scope device array.
//
// The array is kNoAllocScratchBytes (64 MiB) and every GPU that loads the library holds it
// until the process exits.  On the first call on a device the entry point looks up the array's
// device address with cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  All calls share the array and it keeps the previous
// call's contents, so the block accumulators are cleared at the start of every call; two calls
// whose work overlaps on the GPU (different streams, or different host threads without ordering)
// race on the array.
//
// The interpolation and tap tables sit at the front of the array and are kept between calls: a
// call with the same (frame size, magnification, radius, sensitivity) as the previous call on its
// device only enqueues kernels.  A call that changes them first builds the tables on the host and
// uploads them (pageable copies, which wait for the stream's earlier work); callers on a strict
// time budget make one such call at set-up.  The interpolation's two dense passes run on the FP32
// SIMT kernels here (the handle path uses the tensor-core passes on large frames); the two agree
// to ~1e-6 of each slice's range, far inside the 1e-4 parity bar.
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/esrrf.h"
#include "esrrf_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Tables placed in a device's array by the last call, and what they were built for.
struct TableCache {
    bool valid = false;
    int width = 0, height = 0, M = 0, sensitivity = 0;
    float fwhm = 0.f;
    esrrf::InterpPlan plan;
    esrrf::FhtGeometry geo;
    esrrf::FhtFusedTables tables;
    size_t fixed = 0;  // bytes of the tables at the front of the array
};
TableCache g_cache[kMaxDevices];

struct ErrSink {
    char* buf;
    size_t len;
    esrrf_status fail(esrrf_status s, const std::string& msg) const {
        if (buf && len) {
            strncpy(buf, msg.c_str(), len - 1);
            buf[len - 1] = 0;
        }
        return s;
    }
    esrrf_status fail_cuda(cudaError_t e, const char* what) const {
        cudaGetLastError();
        return fail(ESRRF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                                        cudaGetErrorString(e) + ")");
    }
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bytes of the per-frame buffers and block state for F frames per launch.
size_t chunk_bytes(const esrrf::InterpPlan& p, int F) {
    const size_t whM = (size_t)p.WM * p.HM;
    return align256(sizeof(float) * (size_t)F * p.N * p.WM)        // first-pass rows
           + align256(sizeof(float) * (size_t)F * esrrf::interp_alt_floats(p.N))   // alternating sums
           + align256(sizeof(float) * (size_t)F * esrrf::interp_vec_floats(p.HM, p.WM))  // rank-one vectors
           + align256(sizeof(float) * (size_t)F * whM)             // interpolated frames
           + align256(sizeof(double) * 4 * whM)                    // block accumulators
           + align256(sizeof(float) * whM)                         // previous X
           + align256(sizeof(float) * whM);                        // previous X of a grouped launch
}

}  // namespace

extern "C" {

esrrf_status esrrf_fht_block_noalloc(const void* d_frames, int is_u16, int n_frames, int width,
                                     int height, int magnification, float fwhm, int sensitivity,
                                     int int_weighting, float* d_out, void* stream_ptr,
                                     char* err, size_t err_len) {
    using namespace esrrf;
    const ErrSink es{err, err_len};
    if (err && err_len) err[0] = 0;
    if (!d_frames || !d_out) return es.fail(ESRRF_ERR_INVALID, "frames and output must be device pointers");
    if (n_frames < 1 || width < 4 || height < 4 || magnification < 1 || magnification > 16 ||
        !(fwhm > 0.f) || fwhm > 20.f || sensitivity < 0 || sensitivity > 64)
        return es.fail(ESRRF_ERR_INVALID, "invalid size or eSRRF parameter");
    // bound the magnified size before any int arithmetic on it (the scratch check below rejects
    // anything near this anyway)
    if ((long long)width * magnification > (1 << 20) || (long long)height * magnification > (1 << 20))
        return es.fail(ESRRF_ERR_INVALID, "frame size x magnification beyond 1048576 pixels per side");
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return es.fail_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return es.fail(ESRRF_ERR_INVALID, "device ordinal out of range");
    // one host thread at a time sets up and enqueues (the table cache is host state); the GPU work
    // of calls on different streams may still overlap, and then races on the array
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return es.fail_cuda(e, "cudaGetSymbolAddress(scratch)");
        g_scratch_addr[dev] = (unsigned char*)ptr;
    }
    unsigned char* base = g_scratch_addr[dev];

    // Layout: interpolation tables, RGC tables (kept between calls with the same key), then the
    // per-launch buffers and block state.
    TableCache& tc = g_cache[dev];
    const bool hit = tc.valid && tc.width == width && tc.height == height && tc.M == magnification &&
                     tc.fwhm == fwhm && tc.sensitivity == sensitivity;
    InterpPlan plan;
    FhtGeometry geo;
    FhtFusedTables tables;
    size_t fixed = 0;
    if (hit) {
        plan = tc.plan;
        geo = tc.geo;
        tables = tc.tables;
        fixed = tc.fixed;
    } else {
        size_t plan_bytes = 0;
        interp_plan_place(plan, width, height, magnification, 0, nullptr, &plan_bytes, stream);
        geo = fht_geometry(magnification, fwhm, sensitivity);
        if (!fht_fused_supported(geo))
            return es.fail(ESRRF_ERR_INVALID, "radius too large for the allocation-free entry point "
                                              "(tap box wider than 32 magnified pixels)");
        size_t table_bytes = 0;
        fht_fused_tables_place(geo, plan.WM, plan.HM, tables, nullptr, &table_bytes, stream);
        fixed = align256(plan_bytes) + align256(table_bytes);
    }
    int F = 8;
    while (F > 1 && fixed + chunk_bytes(plan, F) > kNoAllocScratchBytes) --F;
    const size_t need = fixed + chunk_bytes(plan, F);
    if (need > kNoAllocScratchBytes)
        return es.fail(ESRRF_ERR_INVALID,
                    "frame size needs " + std::to_string(need >> 20) + " MiB of scratch, more than the " +
                        std::to_string(kNoAllocScratchBytes >> 20) + " MiB the allocation-free entry point has");
    if (F > n_frames) F = n_frames;

    if (!hit) {
        tc.valid = false;  // the front of the array is rewritten below
        size_t plan_bytes = 0, table_bytes = 0;
        if ((e = interp_plan_place(plan, width, height, magnification, 0, base, &plan_bytes, stream)) != cudaSuccess)
            return es.fail_cuda(e, "interpolation tables");
        if ((e = fht_fused_tables_place(geo, plan.WM, plan.HM, tables, base + align256(plan_bytes), &table_bytes,
                                        stream)) != cudaSuccess)
            return es.fail_cuda(e, "RGC tables");
        tc.width = width;
        tc.height = height;
        tc.M = magnification;
        tc.fwhm = fwhm;
        tc.sensitivity = sensitivity;
        tc.plan = plan;
        tc.geo = geo;
        tc.tables = tables;
        tc.fixed = fixed;
        tc.valid = true;
    }
    size_t off = fixed;
    const size_t whM = (size_t)plan.WM * plan.HM;
    InterpScratch sc;
    sc.capacity = F;
    sc.rowT = (float*)(base + off);
    off += align256(sizeof(float) * (size_t)F * plan.N * plan.WM);
    sc.alt = (float*)(base + off);
    off += align256(sizeof(float) * (size_t)F * interp_alt_floats(plan.N));
    sc.vec = (float*)(base + off);
    off += align256(sizeof(float) * (size_t)F * interp_vec_floats(plan.HM, plan.WM));
    float* interp = (float*)(base + off);
    off += align256(sizeof(float) * (size_t)F * whM);
    BlockState st;
    st.pixels = (long)whM;
    st.acc = (double*)(base + off);
    off += align256(sizeof(double) * 4 * whM);
    st.prev = (float*)(base + off);
    off += align256(sizeof(float) * whM);
    float* prev_out = (float*)(base + off);  // lets small frames split a launch into frame groups
    off += align256(sizeof(float) * whM);

    // The array keeps the previous call's contents: the accumulators must start at zero.
    if ((e = zero_block(st, stream)) != cudaSuccess) return es.fail_cuda(e, "clear accumulators");
    const size_t fbytes = (is_u16 ? sizeof(uint16_t) : sizeof(float)) * (size_t)width * height;
    for (int s = 0; s < n_frames; s += F) {
        const int F_now = n_frames - s < F ? n_frames - s : F;
        const void* src = (const unsigned char*)d_frames + fbytes * s;
        if ((e = interp_run(plan, sc, src, is_u16 != 0, F_now, interp, stream, nullptr)) != cudaSuccess)
            return es.fail_cuda(e, "interpolation");
        FhtRgcArgs a{};
        a.interp = interp;
        a.W = plan.WM;
        a.H = plan.HM;
        a.F = F_now;
        a.t0 = s;
        a.int_weighting = int_weighting;
        a.st = st;
        a.prev_out = prev_out;
        if ((e = fht_rgc_fused(geo, tables, a, stream)) != cudaSuccess) return es.fail_cuda(e, "RGC");
    }
    if ((e = finalize_block(st, n_frames, 0, d_out, stream)) != cudaSuccess)
        return es.fail_cuda(e, "finalize");
    return ESRRF_OK;
}

}  // extern "C"
